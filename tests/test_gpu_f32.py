"""The single-precision form of the step, against the f64 step on the same tank.

The f32 form is not bit-exact by design (cell-local f32 coordinates, Kahan
sums, f32 pair arithmetic); its error against the f64 step is bounded here with
explicit tolerances. Grid keys and sort order stay integer/f64, so after the
same steps both forms agree on the particle set and stay close in state.
"""
import numpy as np
import pytest

import physics_engine_rs as pe
from helpers import dam_break_params_pe, product_dam_break

pytestmark = pytest.mark.gpu

# tolerances of the f32 form after STEPS steps of the 20x12x12 dam break
STEPS = 40
DT = 1e-4
DENSITY_REL_MAX = 2e-4     # per fluid particle, |rho32 - rho64| / rho64
POSITION_ABS_MAX = 2e-6    # metres (dx = 0.01)
ENERGY_REL = 1e-5          # kinetic + gravitational potential energy


def _worlds(oriented=False):
    p = product_dam_break(20, 12, 12, box=(0.5, 0.2, 0.3))
    if oriented:
        # a plate beside the fluid block facing it, and one facing away: the
        # one-sided filter (particles.rs:126) keeps only the first
        for j in range(6):
            for k in range(6):
                y, z = 0.03 + 0.01 * j, 0.03 + 0.01 * k
                p.push_boundary_oriented((0.215, y, z), 1e-6, (-1.0, 0.0, 0.0))
                p.push_boundary_oriented((0.225, y, z), 1e-6, (1.0, 0.0, 0.0))
    prm = dam_break_params_pe()
    w64 = pe.WcsphWorld(p, prm, pe.WcsphConfig())
    w32 = pe.WcsphWorld(p, prm, pe.WcsphConfig(precision=pe.PRECISION_F32))
    fluid = p.arrays()["kind"] == 0
    return w64, w32, fluid


def _energy(w, fluid):
    x, v = w.positions()[fluid], w.velocities()[fluid]
    return float((0.5 * w.mass * (v * v).sum(1)).sum() + (w.mass * 9.81 * x[:, 2]).sum())


def test_f32_initial_density_close_to_f64():
    w64, w32, fluid = _worlds(oriented=True)
    for w in (w64, w32):
        w.rebuild_grid()
        w.compute_density()
    r64, r32 = w64.densities(), w32.densities()
    rel = np.abs(r32 - r64)[fluid] / r64[fluid]
    assert rel.max() < 2e-6, rel.max()
    w64.close()
    w32.close()


def test_f32_steps_track_f64():
    w64, w32, fluid = _worlds()
    e0 = _energy(w64, fluid)
    w64.run(DT, STEPS)
    w32.run(DT, STEPS)
    # informational bits (a slow neighbour-union path) are allowed; errors are not
    assert w32.status() & ~pe.STATUS_SLOW_UNION == 0
    assert w32.t == w64.t
    r64, r32 = w64.densities()[fluid], w32.densities()[fluid]
    rel = np.abs(r32 - r64) / r64
    assert rel.max() < DENSITY_REL_MAX, rel.max()
    dx = np.abs(w32.positions() - w64.positions()).max()
    assert dx < POSITION_ABS_MAX, dx
    e64, e32 = _energy(w64, fluid), _energy(w32, fluid)
    assert abs(e32 - e64) < ENERGY_REL * abs(e0), (e32, e64)
    # boundary reactions exist and are finite in both forms
    bf32 = w32.boundary_forces()
    assert np.isfinite(bf32).all()
    w64.close()
    w32.close()


def test_f32_is_deterministic():
    """Two f32 worlds on the same scene give identical bits (no atomics decide
    the fluid state; boundary reactions use float atomics and are excluded)."""
    p = product_dam_break(20, 12, 12, box=(0.5, 0.2, 0.3))
    prm = dam_break_params_pe()
    cfg = pe.WcsphConfig(precision=pe.PRECISION_F32)
    a = pe.WcsphWorld(p, prm, cfg)
    b = pe.WcsphWorld(p, prm, cfg)
    a.run(DT, 3)
    b.run(DT, 3)
    assert np.array_equal(a.densities(), b.densities())
    assert np.array_equal(a.positions(), b.positions())
    assert np.array_equal(a.velocities(), b.velocities())
    a.close()
    b.close()


@pytest.mark.parametrize("weights", [True, False])
def test_f32_with_and_without_pair_weights_track_f64(weights):
    """The density pass keeps each neighbour's W for XSPH (the default) or
    XSPH recomputes it: both stay within the f32 form's bounds, and the two
    differ by no more than rounding (well inside the same bounds)."""
    w64, w32, fluid = _worlds()
    w32.set_pair_weights(weights)
    assert w32.pair_weights() == weights
    ref = pe.WcsphWorld(product_dam_break(20, 12, 12, box=(0.5, 0.2, 0.3)), dam_break_params_pe(),
                        pe.WcsphConfig(precision=pe.PRECISION_F32))
    ref.set_pair_weights(not weights)
    for w in (w64, w32, ref):
        w.run(DT, STEPS)
    r64 = w64.densities()[fluid]
    for w in (w32, ref):
        rel = np.abs(w.densities()[fluid] - r64) / r64
        assert rel.max() < DENSITY_REL_MAX, rel.max()
        assert np.abs(w.positions() - w64.positions()).max() < POSITION_ABS_MAX
    assert np.abs(w32.velocities() - ref.velocities()).max() < 1e-6
    for w in (w64, w32, ref):
        w.close()
