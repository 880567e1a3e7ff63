"""The oracle against the reference's locked determinism hashes.

The reference locks two FNV-1a particle hashes in its CI and its
determinism record (scenarios.rs:27-125; the values are the locked ones of
the canonical fluid-tank and DFSPH-tank tables): the PBF tank after 40 steps
of 1/120 s and the DFSPH tank after 40 steps of 1/120 s. The oracle's PBF and
DFSPH restatements reproduce both bit for bit, which pins everything the
three solvers share with the WCSPH path: the particle builders
(`fill_box`, `fill_box_boundary`, `mass_from_spacing`,
`mass_calibrated_to_rest`, `recomputed_akinci_psi`), the sorted uniform grid
and its neighbour visiting order, the cubic-spline / poly6 / spiky kernels and
their `pow` normalisations, the oriented-boundary filter and the FNV-1a hash.
"""
import numpy as np

import oracle as O

PBF_TANK_HASH = 0x9D9E0DA856FD43D4
DFSPH_TANK_HASH = 0xF1F2825B5EEAAB0D
HASH_DT = 1.0 / 120.0
HASH_STEPS = 40


def test_pbf_tank_hash_matches_reference():
    w = O.pbf_hash_world()
    w.run(HASH_DT, HASH_STEPS)
    assert w.hash64() == PBF_TANK_HASH, hex(w.hash64())


def test_dfsph_tank_hash_matches_reference():
    w = O.dfsph_hash_world()
    w.run(HASH_DT, HASH_STEPS)
    assert w.hash64() == DFSPH_TANK_HASH, hex(w.hash64())


def test_pbf_hash_is_sensitive():
    """One ulp less gravity changes the hash: the pin is not vacuous."""
    dx, rho0 = 0.05, 1000.0
    s = O.Scene(3, rho0, O.mass_from_spacing(rho0, dx, 3), 2.0 * dx)
    s.fill_box((0.1, 0.1, 0.1), 4, 4, 4, dx)
    s.fill_box_boundary((0.0, 0.0, 0.0), (0.4, 0.4, 0.45), dx, 1)
    p = O.pbf_default_params()
    p.iterations, p.art_pressure_k, p.vorticity_eps = 4, 0.0, 0.0
    p.gravity[2] = float(np.nextafter(-9.80665, 0.0))
    w = O.PbfWorld(s, p)
    w.run(HASH_DT, HASH_STEPS)
    assert w.hash64() != PBF_TANK_HASH
