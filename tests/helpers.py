"""Shared scene builders for the tests (product side and oracle side)."""
import numpy as np

import oracle as O
import physics_engine_rs as pe


def product_dam_break(nx, ny, nz, dx=0.01, box=(1.0, 0.4, 0.6), jitter=1e-4, seed=0x5EED5EED):
    """The synthetic 3-D dam break built through the product API."""
    h = 2.0 * dx
    mass = pe.mass_from_spacing(1000.0, dx, 3)
    p = pe.Particles(3, 1000.0, mass, h)
    p.fill_box((dx, dx, dx), nx, ny, nz, dx)
    if jitter:
        p.jitter_fluid(seed, jitter)
    p.fill_box_boundary((0.0, 0.0, 0.0), box, dx, 1)
    return p


def oracle_dam_break(nx, ny, nz, dx=0.01, box=(1.0, 0.4, 0.6), jitter=1e-4, seed=0x5EED5EED):
    return O.dam_break_scene(None, dx=dx, box=box, jitter=jitter, seed=seed, nxyz=(nx, ny, nz))


def dam_break_params_pe(adapt_sound_speed=False):
    """Dam-break physics: `WcsphParams::water(1000, 20, g)` with a fixed sound
    speed (the adaptive rule c >= 10 v_max runs away on this free-surface start)."""
    p = pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81))
    p.adapt_sound_speed = adapt_sound_speed
    return p


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def assert_bits_equal(a, b, what=""):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    ba, bb = bits(a), bits(b)
    if not np.array_equal(ba, bb):
        bad = np.nonzero(ba.reshape(-1) != bb.reshape(-1))[0]
        i = bad[0]
        raise AssertionError(
            f"{what}: {bad.size} of {ba.size} values differ; first at flat index {i}: "
            f"{a.reshape(-1)[i]!r} vs {b.reshape(-1)[i]!r}")
