"""CPU tests of the C ABI library and the Python surface (no GPU needed):
the library loads, exports every entry point the header declares, its host-side
builders and helpers agree with the oracle bit for bit, and the reference's
Python function names are present."""
import ctypes as C
import math
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import oracle_dam_break, product_dam_break

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def _declared_functions():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if fn.endswith(".h"):
            text = open(os.path.join(HEADER_DIR, fn)).read()
            names |= set(re.findall(r"\b(pe_(?:fluid|surrogate|mlp)_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib_path = pe.library_path()
    assert os.path.exists(lib_path)
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = _declared_functions()
    assert len(declared) > 50
    missing = sorted(declared - exported)
    assert not missing, missing
    lib = C.CDLL(lib_path)
    for name in declared:
        getattr(lib, name)  # resolvable through the dynamic loader


def test_python_surface_keeps_reference_names():
    names = ["canonical_fluid_hash", "canonical_dfsph_hash", "canonical_coupling_hash",
             "fluid_ritter_front", "fluid_ritter_height", "fluid_hydrostatic_pressure",
             "fluid_archimedes_box_draft", "fluid_heave_period_analytic",
             "fluid_barge_heave_added_mass_2d", "fluid_heave_period_with_added_mass",
             "fluid_sphere_freefall_accel_added_mass", "fluid_pbf_tank_demo",
             "fluid_dfsph_tank_demo", "fluid_poly6_w0", "fluid_canonical_mass",
             "fluid_canonical_ke_after_hash_steps"]
    for n in names:
        assert callable(getattr(pe, n)), n
    assert pe.load_library().pe_fluid_version().startswith(b"physics-engine-b200")


def test_analytic_functions():
    """oracles.rs:37-84 and coupling.rs:413-441 formulas."""
    g, h0, t = 9.81, 1.0, 0.5
    assert pe.fluid_ritter_front(g, h0, t) == 2.0 * math.sqrt(g * h0) * t
    assert abs(pe.fluid_ritter_height(g, h0, 0.0, t) - 4.0 / 9.0 * h0) < 1e-9
    assert pe.fluid_ritter_height(g, h0, -5.0, t) == h0
    assert pe.fluid_hydrostatic_pressure(1000.0, 9.80665, 2.0) == 1000.0 * 9.80665 * 2.0
    assert pe.fluid_archimedes_box_draft(500.0, 1000.0, 2.0) == 1.0
    assert pe.fluid_barge_heave_added_mass_2d(1000.0, 2.0) == 1000.0 * math.pi * 4.0 / 8.0
    T0 = pe.fluid_heave_period_analytic(100.0, 1000.0, 1.0, 9.81)
    T1 = pe.fluid_heave_period_with_added_mass(100.0, 50.0, 1000.0, 1.0, 9.81)
    assert T1 > T0 > 0
    assert pe.fluid_sphere_freefall_accel_added_mass(2000.0, 1000.0, 9.81) == 9.81 * 1000.0 / 2500.0
    assert pe.fluid_canonical_mass() == pe.mass_from_spacing(1000.0, 0.05, 3) * 64
    assert pe.fluid_poly6_w0(0.1) > 0
    with pytest.raises(NotImplementedError):
        pe.canonical_coupling_hash()


def test_scene_builders_match_oracle():
    for nxyz, box in (((32, 32, 32), (1.0, 0.4, 0.6)), ((7, 5, 3), (0.2, 0.15, 0.1))):
        a = product_dam_break(*nxyz, box=box).arrays()
        b = oracle_dam_break(*nxyz, box=box).arrays()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    # 2-D builders
    p = pe.Particles(2, 1000.0, 2.5, 0.12)
    p.fill_box((0.1, 0.1, 0.0), 6, 6, 1, 0.05)
    p.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), 0.05, 2)
    s = O.Scene(2, 1000.0, 2.5, 0.12)
    s.fill_box((0.1, 0.1, 0.0), 6, 6, 1, 0.05)
    s.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), 0.05, 2)
    a, b = p.arrays(), s.arrays()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_recomputed_akinci_psi_matches_quadratic_reference_loop():
    """particles.rs:252 sums over all other boundary samples in index order; the
    grid-accelerated version must give the same bits."""
    p = pe.Particles(3, 1000.0, 1.0, 0.1)
    p.fill_box_boundary((0, 0, 0), (0.4, 0.4, 0.45), 0.05, 1)
    p.recomputed_akinci_psi()
    s = O.Scene(3, 1000.0, 1.0, 0.1)
    s.fill_box_boundary((0, 0, 0), (0.4, 0.4, 0.45), 0.05, 1)
    s.recompute_psi()
    assert np.array_equal(p.arrays()["psi"], s.arrays()["psi"])


def test_mass_helpers_match_oracle():
    assert pe.mass_from_spacing(1000.0, 0.01, 3) == O.mass_from_spacing(1000.0, 0.01, 3)
    for dim in (2, 3):
        assert pe.mass_calibrated_to_rest(1000.0, 0.05, 0.1, dim) == \
            O.mass_calibrated_to_rest(1000.0, 0.05, 0.1, dim)


def test_kernel_and_pair_helpers_match_oracle_bitwise():
    rng = np.random.default_rng(3)
    h = 0.02
    for _ in range(2000):
        rij = rng.uniform(-0.05, 0.05, 3)
        r = float(np.linalg.norm(rij))
        assert pe.kernel_w(0, r, h, 3) == O.kernel_w(0, r, h, 3)
        assert np.array_equal(pe.grad_w(0, rij, h, 3), O.grad_w(0, rij, h, 3))
        xi, xj = rng.uniform(0, 0.05, 3), rng.uniform(0, 0.05, 3)
        vi, vj = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)
        ri, rj = rng.uniform(900, 1100, 2)
        assert pe.pi_ij(0.01, 0.0, 0.01, h, 20.0, xi, xj, vi, vj, ri, rj) == \
            O.pi_ij(0.01, 0.0, 0.01, h, 20.0, xi, xj, vi, vj, ri, rj)
        rho = float(rng.uniform(300, 1300))
        assert pe.tait_pressure(1000.0, 20.0, 7.0, rho) == O.tait_pressure(1000.0, 20.0, 7.0, rho)
    for args in ((0.1, 20.0, 1.0, 10.0), (0.02, 20.0, 3.0, 0.0)):
        assert pe.suggested_dt(*args) == O.suggested_dt(*args)


def test_all_kernel_kinds_match_oracle_bitwise():
    """kernels.rs:40-215: cubic spline, Wendland C2, poly6 and spiky, W and
    grad W in 2-D and 3-D, inside, across and beyond the support."""
    rng = np.random.default_rng(11)
    for kind in (pe.CUBIC_SPLINE, pe.WENDLAND_C2, pe.POLY6, pe.SPIKY):
        for dim in (2, 3):
            for _ in range(500):
                h = float(rng.uniform(0.01, 0.2))
                rij = rng.uniform(-2.5 * h, 2.5 * h, 3)
                if dim == 2:
                    rij[2] = 0.0
                r = float(np.linalg.norm(rij))
                assert pe.kernel_w(kind, r, h, dim) == O.kernel_w(kind, r, h, dim)
                assert np.array_equal(pe.grad_w(kind, rij, h, dim), O.grad_w(kind, rij, h, dim))
            assert pe.kernel_w(kind, 0.0, 0.1, dim) == O.kernel_w(kind, 0.0, 0.1, dim)
            assert pe.kernel_w(kind, 0.05, -1.0, dim) == 0.0


def test_params_water_defaults():
    """wcsph.rs:43-53, viscosity.rs:39-45,82-86, eos.rs:25."""
    p = pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81))
    assert (p.eos_gamma, p.visc_alpha, p.visc_beta, p.visc_eps, p.xsph_epsilon) == \
        (7.0, 0.01, 0.0, 0.01, 0.25)
    assert p.adapt_sound_speed is True and p.surface_tension_sigma == 0.0


def test_invalid_particle_input_rejected():
    p = pe.Particles(3, 1000.0, 1.0, 0.02)
    with pytest.raises(pe.PeError) as e:
        p.push_fluid((float("nan"), 0.0, 0.0))
    assert e.value.code == pe.PE_ERR_ARG
    with pytest.raises(ValueError):
        pe.Particles(4, 1000.0, 1.0, 0.02)


def test_world_creation_fails_loudly_without_a_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except Exception:
        pass
    p = product_dam_break(4, 4, 4, box=(0.1, 0.1, 0.1))
    with pytest.raises(pe.PeError) as e:
        pe.WcsphWorld(p, pe.WcsphParams.water(1000.0, 20.0, (0, 0, -9.81)))
    assert e.value.code == pe.PE_ERR_DEVICE


def test_batch_scene_rules():
    """The seeded batch spec: budgets and extents in range, compact blocks within budget."""
    from physics_engine_rs import scenes

    spec = scenes.batch_spec(16, seed=3)
    assert spec == scenes.batch_spec(16, seed=3)
    for s in spec:
        assert 2048 <= s["budget"] <= 65536
        assert all(0.3 <= L <= 1.2 for L in s["box"])
        nx, ny, nz = s["block"]
        assert nx * ny * nz <= s["budget"]
        assert max(s["block"]) <= 2 * min(s["block"])
        for n, L in zip(s["block"], s["box"]):
            assert 0.01 * n <= L - 0.01 + 1e-12  # last lattice point keeps a dx gap


def test_rng_uniform_is_the_jitter_generator():
    """Draws come from the same Xoshiro256** stream the jitter uses (seeded alike)."""
    from physics_engine_rs import scenes

    u = scenes.rng_uniform(0x5EED5EED, -1e-4, 1e-4, 3)
    p = pe.Particles(3, 1000.0, 1e-3, 0.02)
    p.push_fluid((0.0, 0.0, 0.0))
    p.jitter_fluid(0x5EED5EED, 1e-4)
    assert np.array_equal(p.arrays()["x"][0], u)


def test_handle_entry_points_reject_null_handles():
    """pe-ffi convention: a NULL handle is PE_ERR_NULL, checked before any
    device work (so it holds on a machine without a GPU)."""
    lib = C.CDLL(pe.library_path())
    out = (C.c_uint64 * 8)()
    i32 = C.c_int32(0)
    u32 = C.c_uint32(0)
    calls = [
        (lib.pe_fluid_wcsph_set_pair_weights, (None, C.c_int32(1))),
        (lib.pe_fluid_wcsph_pair_weights, (None, C.byref(i32))),
        (lib.pe_fluid_wcsph_pair_weight_info, (None, out)),
        (lib.pe_fluid_wcsph_list_chunk, (None, C.byref(u32))),
        (lib.pe_fluid_wcsph_step, (None, C.c_double(1e-4))),
        (lib.pe_fluid_wcsph_run, (None, C.c_double(1e-4), C.c_uint64(1))),
        (lib.pe_fluid_wcsph_shapes, (None, out)),
    ]
    for fn, args in calls:
        fn.restype = C.c_int
        assert fn(*args) == pe.PE_ERR_NULL, fn.__name__
