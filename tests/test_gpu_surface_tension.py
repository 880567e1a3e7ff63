"""GPU parity of the WCSPH step with surface tension (wcsph.rs:261-278,
surface_tension.rs:112-220): the Akinci (2013) cohesion + curvature model and
the colour-field model, 3-D and 2-D. Bar: x, v, a, rho, p and the boundary
reactions equal the oracle's bit for bit.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import assert_bits_equal, dam_break_params_pe, oracle_dam_break, product_dam_break

pytestmark = pytest.mark.gpu

SMALL = dict(nx=12, ny=8, nz=8, box=(0.3, 0.15, 0.2))


def _pair(model, sigma, gamma=None):
    ps = product_dam_break(SMALL["nx"], SMALL["ny"], SMALL["nz"], box=SMALL["box"])
    os_ = oracle_dam_break(SMALL["nx"], SMALL["ny"], SMALL["nz"], box=SMALL["box"])
    p = dam_break_params_pe()
    p.surface_tension_model, p.surface_tension_sigma = model, sigma
    p.surface_tension_colour_gamma = sigma if gamma is None else gamma
    q = O.dam_break_params(materialize=False)
    q.st_model, q.st_sigma, q.st_colour_gamma = model, sigma, p.surface_tension_colour_gamma
    return pe.WcsphWorld(ps, p), O.World(os_, q)


def _compare(w, o, what):
    assert_bits_equal(w.positions(), o.x(), f"{what} x")
    assert_bits_equal(w.velocities(), o.v(), f"{what} v")
    assert_bits_equal(w.accelerations(), o.a(), f"{what} a")
    assert_bits_equal(w.densities(), o.rho(), f"{what} rho")
    assert_bits_equal(w.pressures(), o.p(), f"{what} p")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), f"{what} boundary force")


@pytest.mark.parametrize("model,sigma", [(pe.SURFACE_TENSION_AKINCI, 0.0728),
                                         (pe.SURFACE_TENSION_COLOUR_FIELD, 0.0728),
                                         (pe.SURFACE_TENSION_NONE, 0.0728)])
def test_surface_tension_3d_bit_exact(model, sigma):
    w, o = _pair(model, sigma)
    for s in range(6):
        w.step(1e-4)
        o.step(1e-4)
        if s in (0, 5):
            _compare(w, o, f"model {model} step {s}")
    w.close()


def test_surface_tension_2d_droplet_bit_exact():
    """A 2-D square block without walls or gravity (surface_tension.rs droplet
    setting): the Akinci model pulls it round."""
    dx, h, rho0 = 0.01, 0.024, 1000.0
    mass = pe.mass_from_spacing(rho0, dx, 2)
    ps = pe.Particles(2, rho0, mass, h)
    ps.fill_box((0.0, 0.0, 0.0), 14, 14, 1, dx)
    os_ = O.Scene(2, rho0, mass, h)
    os_.fill_box((0.0, 0.0, 0.0), 14, 14, 1, dx)
    p = pe.WcsphParams.water(rho0, 10.0, (0.0, 0.0, 0.0))
    p.adapt_sound_speed = False
    p.surface_tension_model, p.surface_tension_sigma = pe.SURFACE_TENSION_AKINCI, 5.0
    q = O.water_params(rho0, 10.0, (0.0, 0.0, 0.0), materialize=False)
    q.adapt_sound_speed = 0
    q.st_model, q.st_sigma, q.st_colour_gamma = 1, 5.0, 5.0
    w = pe.WcsphWorld(ps, p)
    o = O.World(os_, q)
    w.run(2e-4, 25)
    o.run(2e-4, 25)
    _compare(w, o, "2-D droplet")
    w.close()


def test_surface_tension_unsupported_in_f32():
    ps = product_dam_break(4, 4, 4, box=(0.1, 0.1, 0.1))
    p = dam_break_params_pe()
    p.surface_tension_model, p.surface_tension_sigma = pe.SURFACE_TENSION_AKINCI, 0.07
    with pytest.raises(pe.PeError) as e:
        pe.WcsphWorld(ps, p, pe.WcsphConfig(precision=pe.PRECISION_F32))
    assert e.value.code == pe.PE_ERR_UNSUPPORTED
