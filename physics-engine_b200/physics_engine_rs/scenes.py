"""Seeded synthetic dam-break scenes built with the particle builders.

A dam break is a lattice block of fluid filled from (dx, dx, dx) in the
reference's fill order (`fill_box`, particles.rs:220), jittered by the seeded
Xoshiro256** generator (`jitter_fluid`), inside a one-layer Akinci shell of the
tank (`fill_box_boundary`, particles.rs:286), with h = 2 dx and the mass of
`mass_from_spacing` (particles.rs:166).

The batched scene draws, per tank, a particle budget N uniformly from
[n_min, n_max] and tank extents uniformly from [l_min, l_max] per axis, from one
seeded generator in the order (N, Lx, Ly, Lz) tank after tank. The lattice
block is the largest nx * ny * nz <= N whose points dx * (1 + i) keep a gap of
at least dx to the far walls (n_axis <= floor(L / dx) - 1) and whose longest
side is at most twice its shortest (a compact column, not a one-particle
sheet); among equal products the smallest nx, then ny, is taken. If no block
meets the aspect bound the bound is dropped. Tank t's jitter seed is
seed + 1 + t.
"""
from __future__ import annotations

import numpy as np

from . import Particles, load_library, mass_from_spacing, _ok, _ptr

DX = 0.01
JITTER = 1e-4


def rng_uniform(seed: int, lo: float, hi: float, count: int) -> np.ndarray:
    """`count` sequential draws lo + (hi - lo) * u from Xoshiro256**(seed)."""
    out = np.zeros(int(count))
    _ok(load_library().pe_fluid_rng_uniform(int(seed) & 0xFFFFFFFFFFFFFFFF, float(lo), float(hi),
                                            int(count), _ptr(out) if count else None), "rng_uniform")
    return out


def dam_break_tank(nxyz, box, dx: float = DX, seed: int = 0x5EED5EED, jitter: float = JITTER) -> Particles:
    """One 3-D dam-break tank: fluid lattice nxyz from (dx, dx, dx) and the shell of [0, box]."""
    nx, ny, nz = (int(v) for v in nxyz)
    mass = mass_from_spacing(1000.0, dx, 3)
    p = Particles(3, 1000.0, mass, 2.0 * dx)
    p.fill_box((dx, dx, dx), nx, ny, nz, dx)
    if jitter:
        p.jitter_fluid(seed, jitter)
    p.fill_box_boundary((0.0, 0.0, 0.0), tuple(float(b) for b in box), dx, 1)
    return p


def lattice_block(n_budget: int, box, dx: float = DX):
    """Largest compact nx * ny * nz <= n_budget fitting the tank with a dx gap (see module doc)."""
    nmax = [max(1, int(np.floor(float(L) / dx + 1e-9)) - 1) for L in box]
    nx = np.arange(1, nmax[0] + 1, dtype=np.int64)[:, None, None]
    ny = np.arange(1, nmax[1] + 1, dtype=np.int64)[None, :, None]
    nz = np.arange(1, nmax[2] + 1, dtype=np.int64)[None, None, :]
    prod = nx * ny * nz
    lo = np.minimum(np.minimum(nx, ny), nz)
    hi = np.maximum(np.maximum(nx, ny), nz)
    fits = prod <= n_budget
    for ok in (fits & (hi <= 2 * lo), fits):
        score = np.where(ok, prod, 0)
        if score.max() > 0:
            i, j, k = np.unravel_index(int(np.argmax(score)), score.shape)  # first: smallest nx, ny
            return int(nx[i, 0, 0]), int(ny[0, j, 0]), int(nz[0, 0, k])
    return 1, 1, 1


def batch_spec(n_tanks: int = 512, seed: int = 0x5EED5EED, n_min: int = 2048, n_max: int = 65536,
               l_min: float = 0.3, l_max: float = 1.2, dx: float = DX):
    """Per-tank (budget, box, lattice block) of the seeded batch."""
    u = rng_uniform(seed, 0.0, 1.0, 4 * n_tanks).reshape(n_tanks, 4)
    spec = []
    for t in range(n_tanks):
        budget = n_min + min(int(u[t, 0] * (n_max - n_min + 1)), n_max - n_min)
        box = tuple(float(l_min + (l_max - l_min) * u[t, 1 + a]) for a in range(3))
        spec.append(dict(budget=budget, box=box, block=lattice_block(budget, box, dx)))
    return spec


def batch_dam_break(n_tanks: int = 512, seed: int = 0x5EED5EED, n_min: int = 2048, n_max: int = 65536,
                    l_min: float = 0.3, l_max: float = 1.2, dx: float = DX):
    """The tanks of the seeded batch as `Particles`, and their spec."""
    spec = batch_spec(n_tanks, seed, n_min, n_max, l_min, l_max, dx)
    tanks = [dam_break_tank(s["block"], s["box"], dx, seed + 1 + t) for t, s in enumerate(spec)]
    return tanks, spec
