"""The allocation-free density entry point, called through the C ABI.

`pe_fluid_density_noalloc` serves callers that cannot allocate device memory
(a fixed device budget, an application-owned allocator, or a real-time loop
that must avoid cudaMalloc's device-wide synchronisation). It keeps all its
working memory in one fixed array inside the library, so two calls in a row
reuse the same memory; each must reproduce, bit for bit, the densities that
the allocating world API computes for the same particles. This file is named
to be collected last, so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import physics_engine_rs as pe
from helpers import product_dam_break

pytestmark = pytest.mark.gpu


def _scene():
    p = product_dam_break(20, 14, 12, box=(0.5, 0.2, 0.3))
    # a few oriented samples (a thin plate facing +x) to exercise the
    # one-sided boundary filter (particles.rs:126)
    for j in range(6):
        for k in range(6):
            p.push_boundary_oriented((0.25, 0.03 + 0.01 * j, 0.03 + 0.01 * k), 1e-6, (1.0, 0.0, 0.0))
    return p


def _entry():
    lib = pe.load_library()
    f = lib.pe_fluid_density_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def test_noalloc_density_matches_world_density_on_two_calls():
    import torch

    parts = _scene()
    arr = parts.arrays()
    n = len(parts)
    world = pe.WcsphWorld(parts, pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81)))
    world.rebuild_grid()
    world.compute_density()
    want = world.densities()
    world.close()

    dev = torch.device("cuda:0")
    x = torch.from_numpy(arr["x"]).to(dev)
    kind = torch.from_numpy(arr["kind"]).to(dev)
    psi = torch.from_numpy(arr["psi"]).to(dev)
    nout = torch.from_numpy(arr["n_out"]).to(dev)
    f = _entry()
    for call in range(2):
        rho = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = f(3, parts.rest_density, parts.mass, parts.h, n, x.data_ptr(), kind.data_ptr(),
               psi.data_ptr(), nout.data_ptr(), rho.data_ptr(), None)
        assert rc == pe.PE_OK, rc
        torch.cuda.synchronize()
        got = rho.cpu().numpy()
        # tolerance: bit-exact, as every GPU parity test of this package
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_limit():
    f = _entry()
    too_many = 131072 + 1
    rc = f(3, 1000.0, 1e-3, 0.02, too_many, None, None, None, None, None, None)
    assert rc == pe.PE_ERR_BOUNDS
