"""GPU parity of the divergence-free SPH step (dfsph.rs:718-784).

Bar: bit-exact. The canonical tank reproduces the reference's locked hash
(scenarios.rs:119-125, `f1f2825b5eeaab0d`); on other scenes x, v, rho, p,
the boundary reactions, alpha and the solvers' iteration counts equal the
oracle's restatement (pinned by the same hash) bit for bit: oriented
boundary samples, free-slip planes with a velocity cap and no warm start, a
2-D tank and the adaptive step.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import assert_bits_equal

pytestmark = pytest.mark.gpu

DFSPH_TANK_HASH = 0xF1F2825B5EEAAB0D
DT = 1.0 / 240.0


def test_canonical_dfsph_hash_matches_reference():
    assert pe.canonical_dfsph_hash() == DFSPH_TANK_HASH


def _scenes(dim, nx, ny, nz, dx, box, jitter_seed=None, plates=False):
    rho0 = 1000.0
    h = 2.0 * dx
    mass = pe.mass_calibrated_to_rest(rho0, dx, h, dim)
    ps = pe.Particles(dim, rho0, mass, h)
    os_ = O.Scene(dim, rho0, mass, h)
    for s in (ps, os_):
        s.fill_box((0.1, 0.1, 0.1 if dim == 3 else 0.0), nx, ny, nz, dx)
        if jitter_seed is not None:
            s.jitter_fluid(jitter_seed, 0.05 * dx)
        s.fill_box_boundary((0.0, 0.0, 0.0), box, dx, 1)
    ps.recomputed_akinci_psi()
    os_.recompute_psi()
    if plates:
        # a plate inside the tank facing +x (toward the fluid) and one facing away
        for j in range(5):
            for k in range(5):
                y, z = 0.1 + dx * j, 0.1 + dx * k
                for x, nx_ in ((0.05, 1.0), (0.04, -1.0)):
                    ps.push_boundary_oriented((x, y, z), 1e-4, (nx_, 0.0, 0.0))
                    os_.push_boundary((x, y, z), 1e-4, (nx_, 0.0, 0.0))
    return ps, os_


def _params_pair(**kw):
    p = pe.DfsphParams(**kw)
    q = O.dfsph_default_params()
    q.kernel = p.kernel
    q.max_density_iters, q.max_divergence_iters = p.max_density_iters, p.max_divergence_iters
    q.density_error_tol, q.divergence_error_tol = p.density_error_tol, p.divergence_error_tol
    q.gravity[:] = p.gravity
    q.xsph_epsilon, q.particle_diameter, q.cfl_lambda = p.xsph_epsilon, p.particle_diameter, p.cfl_lambda
    q.adaptive_dt, q.warm_start = int(p.adaptive_dt), int(p.warm_start)
    for a, k in enumerate(pe.DfsphParams._SLIPS):
        v = getattr(p, k)
        q.has_slip[a] = 0 if v is None else 1
        q.slip[a] = 0.0 if v is None else v
    q.solver_omega, q.max_velocity_correction = p.solver_omega, p.max_velocity_correction
    return p, q


def _compare(w, o, what):
    assert_bits_equal(w.positions(), o.x(), f"{what} x")
    assert_bits_equal(w.velocities(), o.v(), f"{what} v")
    assert_bits_equal(w.densities(), o.rho(), f"{what} rho")
    assert_bits_equal(w.pressures(), o.p(), f"{what} p")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), f"{what} boundary force")
    assert_bits_equal(w.alphas(), o.alpha(), f"{what} alpha")
    assert w.last_iterations() == o.iterations(), what
    assert w.t == o.t


CASES = {
    "default": (dict(), False, 8),
    "oriented_plates": (dict(max_density_iters=6, max_divergence_iters=6, density_error_tol=0.005), True, 8),
    "free_slip_capped_cold": (dict(warm_start=False, max_velocity_correction=0.5, free_slip_xmin=0.06,
                                   free_slip_ymax=0.45, xsph_epsilon=0.0), False, 8),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_dfsph_3d_bit_exact(case):
    kw, plates, steps = CASES[case]
    ps, os_ = _scenes(3, 8, 6, 7, 0.05, (0.6, 0.5, 0.6), jitter_seed=5, plates=plates)
    p, q = _params_pair(adaptive_dt=False, particle_diameter=0.05, **kw)
    w = pe.DfsphWorld(ps, p)
    o = O.DfsphWorld(os_, q)
    assert_bits_equal(w.alphas(), o.alpha(), f"{case} alpha at creation")
    for s in range(steps):
        w.step(DT)
        o.step(DT)
        if s in (0, steps - 1):
            _compare(w, o, f"{case} step {s}")
    assert w.status() & ~pe.STATUS_SLOW_UNION == 0
    w.close()


def test_dfsph_2d_bit_exact():
    ps, os_ = _scenes(2, 10, 8, 1, 0.05, (0.8, 0.7, 0.0))
    p, q = _params_pair(gravity=(0.0, -pe.STANDARD_GRAVITY, 0.0), adaptive_dt=False, particle_diameter=0.05,
                        max_density_iters=4, max_divergence_iters=4, density_error_tol=0.01,
                        divergence_error_tol=0.01)
    w = pe.DfsphWorld(ps, p)
    o = O.DfsphWorld(os_, q)
    w.run(DT, 20)
    o.run(DT, 20)
    _compare(w, o, "2-D")
    w.close()


def test_dfsph_adaptive_step_bit_exact():
    ps, os_ = _scenes(3, 6, 6, 6, 0.05, (0.5, 0.5, 0.6))
    p, q = _params_pair(particle_diameter=0.05, max_density_iters=5, max_divergence_iters=5)
    w = pe.DfsphWorld(ps, p)
    o = O.DfsphWorld(os_, q)
    for _ in range(6):
        dw = w.step_adaptive()
        do = o.step_adaptive()
        assert dw == do
    _compare(w, o, "adaptive")
    w.close()


def test_dfsph_tank_demo_runs():
    x, rho, err = pe.fluid_dfsph_tank_demo(n_side=4, steps=10)
    assert x.shape == (64, 3) and rho.shape == (64,)
    assert np.isfinite(err)
