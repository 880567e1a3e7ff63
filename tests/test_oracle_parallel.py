"""The parallel oracle (std::threads over particles, forces as a gather)
gives the sequential oracle's bits.

The parallel mode times the CPU baseline on large tanks and runs the long
sensitivity studies; it may only be used because it reproduces the
sequential restatement of WcsphWorld::step (crates/pe-fluid/src/wcsph.rs:326)
exactly. The force gather rests on the same argument as the GPU's: the
reference's scatter gives a[k] the lower-index fluid terms in ascending index,
then its own visiting-order terms, and each pair force is antisymmetric bit
for bit.
"""
import numpy as np

import oracle as O
from helpers import assert_bits_equal, oracle_dam_break

FIELDS = ("x", "v", "a", "rho", "p", "boundary_force")


def _compare(a, b, what):
    for f in FIELDS:
        assert_bits_equal(getattr(a, f)(), getattr(b, f)(), f"{what} {f}")
    assert a.hash64() == b.hash64()
    assert a.sound_speed == b.sound_speed


def test_parallel_dam_break_steps_bit_exact():
    kw = dict(box=(0.3, 0.15, 0.2))
    a = O.World(oracle_dam_break(12, 8, 8, **kw), O.dam_break_params(materialize=True))
    b = O.World(oracle_dam_break(12, 8, 8, **kw), O.dam_break_params(materialize=True))
    b.set_threads(4)
    for k in range(8):
        a.step(1e-4)
        b.step(1e-4)
    _compare(a, b, "dam break")
    ga, gb = a.grid(), b.grid()
    for k in ga:
        np.testing.assert_array_equal(ga[k], gb[k])


def test_parallel_adaptive_sound_speed_and_oriented_boundary_bit_exact():
    def scene():
        s = oracle_dam_break(10, 6, 6, box=(0.2, 0.1, 0.12))
        for j in range(5):
            for k in range(5):
                s.push_boundary((0.06, 0.02 + 0.01 * j, 0.02 + 0.01 * k), 1e-6, (1.0, 0.0, 0.0))
        return s

    a = O.World(scene(), O.dam_break_params(materialize=False, adapt_sound_speed=True))
    b = O.World(scene(), O.dam_break_params(materialize=False, adapt_sound_speed=True))
    b.set_threads(3)
    for _ in range(4):
        a.step(1e-4)
        b.step(1e-4)
    _compare(a, b, "adaptive c, oriented samples")


def test_parallel_two_dimensional_bit_exact():
    dx, h, rho0 = 0.05, 2.4 * 0.05, 1000.0
    mass = O.mass_from_spacing(rho0, dx, 2)

    def world(threads):
        s = O.Scene(2, rho0, mass, h)
        s.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
        s.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
        p = O.water_params(rho0, 40.0, (0.0, -9.80665, 0.0), materialize=False)
        p.adapt_sound_speed = 0
        p.visc_alpha = 0.05
        w = O.World(s, p)
        w.set_threads(threads)
        return w

    a, b = world(1), world(5)
    for _ in range(20):
        a.step(0.0002)
        b.step(0.0002)
    _compare(a, b, "2-D")


def test_parallel_grid_sort_large_bit_exact():
    """More particles than the parallel sort's sequential cut-off (65,536),
    so the chunked sort and merges run."""
    a = O.World(oracle_dam_break(48, 40, 40, box=(0.6, 0.5, 0.5)), O.dam_break_params(materialize=False))
    b = O.World(oracle_dam_break(48, 40, 40, box=(0.6, 0.5, 0.5)), O.dam_break_params(materialize=False))
    b.set_threads(6)
    a.rebuild_grid()
    b.rebuild_grid()
    ga, gb = a.grid(), b.grid()
    for k in ga:
        np.testing.assert_array_equal(ga[k], gb[k])
