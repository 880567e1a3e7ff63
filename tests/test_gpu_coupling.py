"""GPU parity of the fluid side of the WCSPH-rigid coupling.

Each coupled step is `CoupledWcsphWorld::step` (coupling.rs:853-866) with the
rigid integration replaced by prescribed motion: `sync_from_rigid`
(coupling.rs:289-306), the fluid step, `reduce_with_state`
(coupling.rs:308-330). Bar: the product's particle state after every sync and
step, and the per-body force and torque, equal the oracle's bit for bit.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from coupling_scene import cube_samples, interleave, rigid_state, ring_samples_2d
from helpers import assert_bits_equal, dam_break_params_pe, oracle_dam_break, product_dam_break

pytestmark = pytest.mark.gpu

DT = 1e-4


def _add_samples(ps, os_, X0, body, local, normal, psi):
    base = len(ps)
    for k in range(len(body)):
        x = X0[body[k]] + local[k]
        ps.push_boundary_oriented(x, psi, normal[k])
        os_.push_boundary(x, psi, normal[k])
    return base


def _run_coupled(w, o, cw, co, motion, steps, dim=3):
    x0, v, axis, om = motion
    for s in range(steps):
        X, Q, V, W = rigid_state(x0, v, axis, om, s * DT)
        cw.sync_from_rigid(X, Q, V, W)
        co.sync_from_rigid(X, Q, V, W)
        if s == 0:
            assert_bits_equal(w.positions(), o.x(), "x after sync")
            assert_bits_equal(w.velocities(), o.v(), "v after sync")
        w.step(DT)
        o.step(DT)
        fw, tw = cw.reduce_with_state(X)
        fo, to = co.reduce_with_state(X)
        assert_bits_equal(fw, fo, f"force step {s}")
        assert_bits_equal(tw, to, f"torque step {s}")
    assert_bits_equal(w.positions(), o.x(), "x")
    assert_bits_equal(w.velocities(), o.v(), "v")
    assert_bits_equal(w.densities(), o.rho(), "rho")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), "boundary force")
    return fw, tw


def test_two_bodies_3d_bit_exact():
    """A cube half in the fluid surface, sinking and spinning, and a smaller
    cube beside it translating; samples interleaved and mapped to shuffled
    particle indices."""
    box = (0.3, 0.15, 0.2)
    ps = product_dam_break(12, 8, 8, box=box)
    os_ = oracle_dam_break(12, 8, 8, box=box)
    l0, n0 = cube_samples(0.02, 4)
    l1, n1 = cube_samples(0.012, 3)
    body, local, normal = interleave([(l0, n0), (l1, n1)])
    X0 = np.array([[0.07, 0.05, 0.09], [0.2, 0.07, 0.05]])
    base = _add_samples(ps, os_, X0, body, local, normal, 2e-6)
    particle = base + np.arange(len(body), dtype=np.int64)
    # the coupler's sample order need not follow particle order
    perm = np.random.default_rng(7).permutation(len(body))
    body, local, normal, particle = body[perm], local[perm], normal[perm], particle[perm]
    w = pe.WcsphWorld(ps, dam_break_params_pe())
    o = O.World(os_, O.dam_break_params(materialize=False))
    cw = pe.FluidRigidCoupler(w, 2, body, local, normal, particle)
    co = O.Coupler(o, 2, body, local, normal, particle)
    motion = (X0, [(0.0, 0.0, -0.05), (0.1, 0.0, 0.0)], [(0.3, 1.0, 0.2), (0.0, 0.0, 1.0)], [4.0, -2.0])
    f, t = _run_coupled(w, o, cw, co, motion, 25)
    assert np.abs(f[0]).max() > 0.0  # the fluid pushes on the first cube
    cw.close()
    w.close()


def test_body_2d_bit_exact():
    """2-D: a ring of samples in a small tank; the z components are zeroed
    (coupling.rs:300-304) even when the prescribed spin axis is tilted."""
    dx, h, rho0 = 0.05, 2.4 * 0.05, 1000.0
    mass = pe.mass_from_spacing(rho0, dx, 2)
    ps = pe.Particles(2, rho0, mass, h)
    ps.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    ps.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    os_ = O.Scene(2, rho0, mass, h)
    os_.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    os_.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    local, normal = ring_samples_2d(0.06, 12)
    body = np.zeros(len(local), np.int64)
    X0 = np.array([[0.3, 0.3, 0.0]])
    base = _add_samples(ps, os_, X0, body, local, normal, 1e-3)
    particle = base + np.arange(len(body), dtype=np.int64)
    prm = pe.WcsphParams.water(rho0, 40.0, (0.0, -9.80665, 0.0))
    prm.adapt_sound_speed = False
    op = O.water_params(rho0, 40.0, (0.0, -9.80665, 0.0), materialize=False)
    op.adapt_sound_speed = 0
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    cw = pe.FluidRigidCoupler(w, 1, body, local, normal, particle)
    co = O.Coupler(o, 1, body, local, normal, particle)
    motion = (X0, [(-0.2, -0.1, 0.0)], [(0.1, 0.0, 1.0)], [3.0])
    _run_coupled(w, o, cw, co, motion, 30, dim=2)
    assert np.all(w.positions()[:, 2] == 0.0)
    cw.close()
    w.close()


def test_coupler_rejects_bad_tables():
    ps = product_dam_break(4, 4, 4, box=(0.1, 0.1, 0.1))
    n = len(ps)
    w = pe.WcsphWorld(ps, dam_break_params_pe())
    one = np.zeros((1, 3))
    with pytest.raises(pe.PeError):
        pe.FluidRigidCoupler(w, 1, [1], one, one, [0])  # body out of range
    with pytest.raises(pe.PeError):
        pe.FluidRigidCoupler(w, 1, [0], one, one, [n])  # particle out of range
    with pytest.raises(pe.PeError):
        pe.FluidRigidCoupler(w, 1, [0], np.full((1, 3), np.nan), one, [0])
    c = pe.FluidRigidCoupler(w, 1, [0], one, one, [0])
    with pytest.raises(pe.PeError):
        c.sync_from_rigid(np.full((1, 3), np.inf), [[1.0, 0, 0, 0]], one, one)
    c.close()
    w.close()
