"""GPU parity: the CUDA WCSPH path, called through the C ABI, against the CPU
oracle (an order-exact restatement of crates/pe-fluid/src/wcsph.rs).

Bar: bit-exact for integer work (cell keys, sort order, occupied cells and
ranges, neighbour counts) and for the f64 state (x, v, a, rho, p, boundary
force, sound speed) — the GPU reproduces the reference's operation order
and compiles without FMA contraction, so equality is exact, not a tolerance.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import (assert_bits_equal, dam_break_params_pe, oracle_dam_break,
                     product_dam_break)

pytestmark = pytest.mark.gpu

SMALL = dict(nx=12, ny=8, nz=8, box=(0.3, 0.15, 0.2))


def _pair(nx, ny, nz, box, jitter=1e-4, materialize=False, adapt=False):
    ps = product_dam_break(nx, ny, nz, box=box, jitter=jitter)
    os_ = oracle_dam_break(nx, ny, nz, box=box, jitter=jitter)
    w = pe.WcsphWorld(ps, dam_break_params_pe(adapt))
    o = O.World(os_, O.dam_break_params(materialize=materialize, adapt_sound_speed=adapt))
    return w, o


def _compare_grid(w, o):
    gg, go = w.grid(), o.grid()
    np.testing.assert_array_equal(gg["keys"], go["keys"])
    np.testing.assert_array_equal(gg["order"].astype(np.int64), go["order"])
    np.testing.assert_array_equal(gg["occupied"], go["occupied"])
    np.testing.assert_array_equal(gg["ranges"].astype(np.int64), go["ranges"])


def _compare_state(w, o, what):
    assert_bits_equal(w.positions(), o.x(), f"{what} x")
    assert_bits_equal(w.velocities(), o.v(), f"{what} v")
    assert_bits_equal(w.densities(), o.rho(), f"{what} rho")
    assert_bits_equal(w.pressures(), o.p(), f"{what} p")
    assert_bits_equal(w.accelerations(), o.a(), f"{what} a")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), f"{what} boundary force")
    assert w.sound_speed == o.sound_speed
    assert w.t == o.t


def test_scene_builders_identical():
    ps = product_dam_break(**SMALL)
    os_ = oracle_dam_break(**SMALL)
    a, b = ps.arrays(), os_.arrays()
    for k in ("x", "v", "kind", "psi", "n_out"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_grid_and_neighbour_counts_bit_exact():
    w, o = _pair(**SMALL)
    w.rebuild_grid()
    o.rebuild_grid()
    _compare_grid(w, o)
    cg, sg = w.neighbour_counts()
    co, so = o.neighbour_counts()
    np.testing.assert_array_equal(cg.astype(np.int64), co)
    np.testing.assert_array_equal(sg.astype(np.int64), so)


def test_phase_methods_bit_exact():
    w, o = _pair(**SMALL)
    for name in ("rebuild_grid", "compute_density", "compute_pressure", "compute_forces"):
        getattr(w, name)()
        getattr(o, name)()
    _compare_state(w, o, "phases")
    w.apply_xsph()
    o.apply_xsph()
    assert_bits_equal(w.velocities(), o.v(), "xsph v")


def test_steps_bit_exact_small():
    w, o = _pair(**SMALL)
    dt = 1e-4
    for k in range(25):
        w.step(dt)
        o.step(dt)
        if k % 5 == 4:
            _compare_state(w, o, f"step {k + 1}")
            _compare_grid(w, o)
    assert w.status() == 0


def test_pair_weights_on_and_off_bit_exact():
    """The density pass keeps each neighbour entry's W for the XSPH pass of
    the same lists (the default); with the buffer off, XSPH recomputes W from
    the neighbour's position. Both follow the oracle bit for bit, switched
    mid-run in both directions (run() replays captured graphs of six steps,
    which a switch must recapture), and an XSPH pass with no density pass
    since the grid was rebuilt takes the recomputing kernel."""
    _, o = _pair(**SMALL)
    w = pe.WcsphWorld(product_dam_break(SMALL["nx"], SMALL["ny"], SMALL["nz"], box=SMALL["box"], jitter=1e-4),
                      dam_break_params_pe(False), pe.WcsphConfig(use_graph=True))
    assert w.pair_weights()
    dt = 1e-4
    for on, steps in ((True, 7), (False, 7), (True, 13)):
        w.set_pair_weights(on)
        assert w.pair_weights() == on
        w.run(dt, steps)
        o.run(dt, steps)
        _compare_state(w, o, f"pair weights {on}")
    w.rebuild_grid()
    o.rebuild_grid()
    w.apply_xsph()
    o.apply_xsph()
    assert_bits_equal(w.velocities(), o.v(), "xsph after a grid rebuild")
    assert w.status() == 0


def test_autotune_between_density_and_xsph_bit_exact():
    """The autotuner rebuilds the lists in the shape it picks, which moves
    them in the pool: the pair weights the density pass kept no longer match,
    and the XSPH pass after it must recompute W."""
    w, o = _pair(**SMALL)
    for name in ("rebuild_grid", "compute_density"):
        getattr(w, name)()
        getattr(o, name)()
    w.autotune()
    w.apply_xsph()
    o.apply_xsph()
    assert_bits_equal(w.velocities(), o.v(), "xsph after autotune")
    w.step(1e-4)
    o.step(1e-4)
    _compare_state(w, o, "step after autotune")


def test_pair_weights_outgrown_by_the_lists_bit_exact():
    """A lattice spaced 1.25 dx with the mass of dx collapses: its lists grow
    by ~75% in 40 steps, past the pair-weight buffer (1.25x the lists the pool
    was sized for; a small first guess of the pool makes the first build size
    it to twice the need). A density pass that meets lists beyond the buffer
    keeps no weights and XSPH recomputes W; the status poll of each step()
    then extends the buffer. The state follows the oracle bit for bit
    throughout."""
    dx = 0.01
    rho0, mass = 1000.0, pe.mass_from_spacing(1000.0, dx, 3)
    ps = pe.Particles(3, rho0, mass, 2 * dx)
    os_ = O.Scene(3, rho0, mass, 2 * dx)
    for s in (ps, os_):
        s.fill_box((dx, dx, dx), 12, 8, 8, 1.25 * dx)
        s.fill_box_boundary((0.0, 0.0, 0.0), (0.3, 0.15, 0.2), dx, 1)
    w = pe.WcsphWorld(ps, dam_break_params_pe(False), pe.WcsphConfig(max_neighbours=16))
    o = O.World(os_, O.dam_break_params(materialize=False))
    w.step(1e-4)
    o.step(1e-4)
    info0 = w.pair_weight_info()
    assert info0["in_use"] and not info0["short"]
    short_steps, grew = 0, False
    for k in range(1, 45):
        w.step(1e-4)
        o.step(1e-4)
        info = w.pair_weight_info()
        short_steps += info["short"]
        grew = grew or info["entries"] > info0["entries"]
        if k in (20, 44):
            _compare_state(w, o, f"collapse step {k + 1}")
    assert short_steps > 0 and grew
    assert w.pair_weights()
    assert w.status() & ~pe.STATUS_SLOW_UNION == 0


def test_adaptive_sound_speed_bit_exact():
    """compute_pressure's c = max(c, 10 v_max), persisted (wcsph.rs:158-169).
    With the rule on, the free-surface start accelerates quickly (c grows each
    step); the first five steps stay in the grid domain and are compared."""
    w, o = _pair(**SMALL, adapt=True)
    cs = []
    for k in range(5):
        w.step(1e-4)
        o.step(1e-4)
        _compare_state(w, o, f"adaptive step {k + 1}")
        cs.append(w.sound_speed)
    assert cs[-1] > 20.0 and cs == sorted(cs)


def test_reference_bench_scene_bit_exact():
    """crates/pe-fluid/benches/fluid.rs:65-96 geometry: 8x8x4 lattice, dx 0.05,
    h 2.2 dx, c 25, dt 5e-4, 20 steps, standard gravity — with a fixed sound
    speed: under the water() default (adaptive c) this workload runs away
    (c reaches ~1.8e8 m/s in 20 steps and particles leave the tank)."""
    dx, h, rho0 = 0.05, 2.2 * 0.05, 1000.0
    mass = pe.mass_from_spacing(rho0, dx, 3)
    ps = pe.Particles(3, rho0, mass, h)
    ps.fill_box((0.1, 0.1, 0.1), 8, 8, 4, dx)
    ps.fill_box_boundary((0, 0, 0), (0.6, 0.6, 0.4), dx, 1)
    os_ = O.Scene(3, rho0, mass, h)
    os_.fill_box((0.1, 0.1, 0.1), 8, 8, 4, dx)
    os_.fill_box_boundary((0, 0, 0), (0.6, 0.6, 0.4), dx, 1)
    g = (0.0, 0.0, -9.80665)
    prm = pe.WcsphParams.water(rho0, 25.0, g)
    prm.adapt_sound_speed = False
    op = O.water_params(rho0, 25.0, g, materialize=False)
    op.adapt_sound_speed = 0
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    w.run(0.0005, 20)
    o.run(0.0005, 20)
    _compare_state(w, o, "bench scene")
    assert w.hash64() == o.hash64()


def test_two_dimensional_bit_exact():
    """fluid_analytic.rs:104 scene (2-D, h = 2.4 dx, c 40, alpha 0.05, adapt off)."""
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
    prm.visc_alpha = 0.05
    op = O.water_params(rho0, 40.0, (0.0, -9.80665, 0.0), materialize=False)
    op.adapt_sound_speed = 0
    op.visc_alpha = 0.05
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    for _ in range(30):
        w.step(0.0002)
        o.step(0.0002)
    _compare_state(w, o, "2-D")


def test_c1_scene_two_steps_bit_exact():
    """The 32^3 dam break (32,768 fluid + 24,802 boundary) for two steps."""
    w, o = _pair(32, 32, 32, (1.0, 0.4, 0.6))
    w.run(1e-4, 2)
    o.run(1e-4, 2)
    _compare_state(w, o, "C1")
    _compare_grid(w, o)
    cg, sg = w.neighbour_counts()
    co, so = o.neighbour_counts()
    np.testing.assert_array_equal(cg.astype(np.int64), co)
    np.testing.assert_array_equal(sg.astype(np.int64), so)


def test_state_write_back_bit_exact():
    """Writing positions back unchanged keeps the grid, lists and densities
    (they would be rebuilt to the same bits); writing changed positions
    rebuilds them. Both continue bit for bit with the oracle."""
    w, o = _pair(**SMALL)
    w.run(1e-4, 3)
    o.run(1e-4, 3)
    w.set_positions(w.positions())
    w.set_velocities(w.velocities())
    w.step(1e-4)
    o.step(1e-4)
    _compare_state(w, o, "unchanged write-back")
    x = w.positions()
    x[5] += 1e-4
    w.set_positions(x)
    o.set_x(x)
    w.run(1e-4, 2)
    o.run(1e-4, 2)
    _compare_state(w, o, "changed write-back")
    w.close()


def test_non_finite_state_rejected_untouched():
    """Non-finite positions or velocities are refused (PE_ERR_ARG, the pe-ffi
    rule) and leave the world's state as it was."""
    w, _ = _pair(**SMALL)
    w.run(1e-4, 2)
    x0, v0 = w.positions(), w.velocities()
    for setter, arr in ((w.set_positions, x0), (w.set_velocities, v0)):
        bad = arr.copy()
        bad[len(bad) // 2, 1] = np.nan
        with pytest.raises(pe.PeError) as e:
            setter(bad)
        assert e.value.code == pe.PE_ERR_ARG
    assert_bits_equal(w.positions(), x0, "x kept")
    assert_bits_equal(w.velocities(), v0, "v kept")
    w.close()


@pytest.mark.parametrize("kind", [pe.WENDLAND_C2, pe.POLY6, pe.SPIKY])
def test_other_kernel_kinds_bit_exact(kind):
    """WcsphParams.density_kernel (wcsph.rs:26) other than the cubic spline:
    Wendland C2 (support 2h) and poly6 / spiky (support h, grid cell h)."""
    ps = product_dam_break(SMALL["nx"], SMALL["ny"], SMALL["nz"], box=SMALL["box"])
    os_ = oracle_dam_break(SMALL["nx"], SMALL["ny"], SMALL["nz"], box=SMALL["box"])
    p = dam_break_params_pe()
    p.density_kernel = kind
    q = O.dam_break_params(materialize=False)
    q.kernel = kind
    w = pe.WcsphWorld(ps, p)
    o = O.World(os_, q)
    for s in range(4):
        w.step(1e-4)
        o.step(1e-4)
    _compare_state(w, o, f"kernel {kind}")
    _compare_grid(w, o)
    w.close()
