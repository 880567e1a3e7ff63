"""Diagnostics reduced on the device (diagnostics.rs:19-102, wcsph.rs:350-369)
against the oracle's restatement, field by field.

Bar: bit-exact. The device adds the fluid particles' terms in original index
order as the reference does (momentum, kinetic and potential energy, the
density error sum), reduces the maxima in parallel (order-free), and computes
the FNV-1a state hash in parallel by its low-byte state machine and affine
maps — each must give the oracle's bits.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import dam_break_params_pe, oracle_dam_break, product_dam_break

pytestmark = pytest.mark.gpu


def _fields_equal(d, o, g, what):
    want = {
        "total_mass": o.total_mass(),
        "kinetic_energy": o.kinetic_energy(),
        "gravitational_potential": o.gravitational_potential(g),
        "mean_density_error": o.mean_density_error(),
        "max_density_error": o.max_density_error(),
        "v_max": o.v_max(),
        "a_max": o.a_max(),
    }
    for k, v in want.items():
        assert np.float64(d[k]).view(np.uint64) == np.float64(v).view(np.uint64), (what, k, d[k], v)
    mom = np.asarray(d["linear_momentum"], np.float64)
    np.testing.assert_array_equal(mom.view(np.uint64), o.linear_momentum().view(np.uint64), err_msg=what)
    assert d["hash64"] == o.hash64(), what


def test_diagnostics_c1_after_ten_steps_bit_exact():
    """The 32^3 dam break (32,768 fluid + 24,802 boundary) after 10 steps."""
    ps = product_dam_break(32, 32, 32)
    w = pe.WcsphWorld(ps, dam_break_params_pe())
    o = O.World(oracle_dam_break(32, 32, 32), O.dam_break_params(materialize=False))
    _fields_equal(w.diagnostics(), o, 9.81, "C1 at rest")
    w.run(1e-4, 10)
    o.run(1e-4, 10)
    d = w.diagnostics()
    assert d["kinetic_energy"] > 0.0 and d["a_max"] > 0.0
    _fields_equal(d, o, 9.81, "C1 after 10 steps")
    w.close()


def test_diagnostics_two_dimensional_bit_exact():
    dx, h, rho0 = 0.05, 2.4 * 0.05, 1000.0
    mass = pe.mass_from_spacing(rho0, dx, 2)
    ps = pe.Particles(2, rho0, mass, h)
    ps.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    ps.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    os_ = O.Scene(2, rho0, mass, h)
    os_.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    os_.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    prm = pe.WcsphParams.water(rho0, 40.0, (0.0, -9.80665, 0.0))
    prm.adapt_sound_speed = False
    op = O.water_params(rho0, 40.0, (0.0, -9.80665, 0.0), materialize=False)
    op.adapt_sound_speed = 0
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    w.run(0.0002, 12)
    o.run(0.0002, 12)
    # gravity along -y: the world's potential uses -gravity.z = 0
    _fields_equal(w.diagnostics(), o, 0.0, "2-D")
    w.close()


def test_diagnostics_interleaved_kinds_and_chunk_edges():
    """Boundary samples before, between and after the fluid in index order,
    and more than one 512-particle hash chunk and 1024-particle sum chunk with
    ragged ends: compaction and chunk joins must keep index order."""
    dx = 0.01
    mass = pe.mass_from_spacing(1000.0, dx, 3)
    ps = pe.Particles(3, 1000.0, mass, 2 * dx)
    os_ = O.Scene(3, 1000.0, mass, 2 * dx)
    for s in (ps, os_):
        s.fill_box_boundary((0.0, 0.0, 0.0), (0.2, 0.1, 0.12), dx, 1)
        s.fill_box((dx, dx, dx), 9, 5, 4, dx)
        s.jitter_fluid(7, 1e-4)
    for k in range(37):
        ps.push_boundary((0.05 + 0.001 * k, 0.05, 0.115), 1e-6)
        os_.push_boundary((0.05 + 0.001 * k, 0.05, 0.115), 1e-6)
    for s in (ps, os_):
        s.fill_box((2 * dx, 2 * dx, 6 * dx), 7, 3, 3, dx)
    w = pe.WcsphWorld(ps, dam_break_params_pe())
    o = O.World(os_, O.dam_break_params(materialize=False))
    w.run(1e-4, 3)
    o.run(1e-4, 3)
    _fields_equal(w.diagnostics(), o, 9.81, "interleaved")
    w.close()
