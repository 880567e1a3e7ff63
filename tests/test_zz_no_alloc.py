"""The allocation-free density entry point, called through the C ABI.

`pe_fluid_density_noalloc` serves callers that cannot allocate device memory
(a fixed device budget, an application-owned allocator, or a real-time loop
that must avoid cudaMalloc's device-wide synchronisation). It keeps all its
working memory in one fixed array inside the library, so two calls in a row
reuse the same memory; each must reproduce, bit for bit, the densities of the
oracle and of the allocating world API for the same particles. This file is
named to be collected last, so a failure here comes after every other test has
run.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import assert_bits_equal, oracle_dam_break, product_dam_break

pytestmark = pytest.mark.gpu

SENTINEL = -12345.0


def _scene():
    p = product_dam_break(20, 14, 12, box=(0.5, 0.2, 0.3))
    # a few oriented samples (a thin plate facing +x) to exercise the
    # one-sided boundary filter (particles.rs:126)
    for j in range(6):
        for k in range(6):
            p.push_boundary_oriented((0.25, 0.03 + 0.01 * j, 0.03 + 0.01 * k), 1e-6, (1.0, 0.0, 0.0))
    return p


def _oracle_scene():
    o = oracle_dam_break(20, 14, 12, box=(0.5, 0.2, 0.3))
    for j in range(6):
        for k in range(6):
            o.push_boundary((0.25, 0.03 + 0.01 * j, 0.03 + 0.01 * k), 1e-6, (1.0, 0.0, 0.0))
    return o


def _oracle_density(scene):
    w = O.World(scene, O.dam_break_params(materialize=False))
    w.rebuild_grid()
    w.compute_density()
    return w.rho()


def _entry():
    lib = pe.load_library()
    f = lib.pe_fluid_density_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _call(dim, meta, arr, use_psi=True, use_nout=True):
    """One call on device copies of the arrays; returns (rc, rho on the host)."""
    import torch

    dev = torch.device("cuda:0")
    n = arr["x"].shape[0]
    x = torch.from_numpy(np.ascontiguousarray(arr["x"])).to(dev)
    kind = torch.from_numpy(np.ascontiguousarray(arr["kind"])).to(dev)
    psi = torch.from_numpy(np.ascontiguousarray(arr["psi"])).to(dev)
    nout = torch.from_numpy(np.ascontiguousarray(arr["n_out"])).to(dev)
    rho = torch.full((n,), SENTINEL, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rest, mass, h = meta
    rc = _entry()(dim, rest, mass, h, n, x.data_ptr(), kind.data_ptr(),
                  psi.data_ptr() if use_psi else None, nout.data_ptr() if use_nout else None,
                  rho.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, rho.cpu().numpy()


def test_noalloc_density_matches_oracle_and_world_on_two_calls():
    parts = _scene()
    arr = parts.arrays()
    world = pe.WcsphWorld(parts, pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81)))
    world.rebuild_grid()
    world.compute_density()
    want_world = world.densities()
    world.close()
    want = _oracle_density(_oracle_scene())
    # tolerance: bit-exact, as every GPU parity test of this package
    assert_bits_equal(want_world, want, "world API vs oracle")
    meta = (parts.rest_density, parts.mass, parts.h)
    for call in range(2):
        rc, got = _call(3, meta, arr)
        assert rc == pe.PE_OK, rc
        assert_bits_equal(got, want, f"call {call}")


def test_noalloc_two_dimensional_matches_oracle():
    """fluid_analytic.rs:104 scene (2-D, h = 2.4 dx): the DIM = 2 path."""
    dx, h, rho0 = 0.05, 2.4 * 0.05, 1000.0
    mass = pe.mass_from_spacing(rho0, dx, 2)
    ps = pe.Particles(2, rho0, mass, h)
    ps.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    ps.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    os_ = O.Scene(2, rho0, mass, h)
    os_.fill_box((0.1, 0.1, 0.0), 6, 6, 1, dx)
    os_.fill_box_boundary((0, 0, 0), (0.5, 0.5, 0.0), dx, 1)
    want = _oracle_density(os_)
    for call in range(2):
        rc, got = _call(2, (rho0, mass, h), ps.arrays())
        assert rc == pe.PE_OK, rc
        assert_bits_equal(got, want, f"2-D call {call}")


def test_noalloc_null_psi_and_normals_match_oracle():
    """psi = NULL gives every boundary sample psi 0 and n_out = NULL orients
    none: the oracle's scene with those values gives the same bits."""
    parts = _scene()
    arr = parts.arrays()
    o = O.Scene(3, parts.rest_density, parts.mass, parts.h)
    for xi, vi, ki in zip(arr["x"], arr["v"], arr["kind"]):
        if ki:
            o.push_boundary(xi, 0.0, None)
        else:
            o.push_fluid(xi, vi)
    want = _oracle_density(o)
    meta = (parts.rest_density, parts.mass, parts.h)
    rc, got = _call(3, meta, arr, use_psi=False, use_nout=False)
    assert rc == pe.PE_OK, rc
    assert_bits_equal(got, want, "psi and n_out NULL")


def test_noalloc_rejects_sizes_beyond_its_limit():
    f = _entry()
    too_many = 131072 + 1
    rc = f(3, 1000.0, 1e-3, 0.02, too_many, None, None, None, None, None, None)
    assert rc == pe.PE_ERR_BOUNDS


def test_noalloc_rejects_a_cell_box_beyond_its_limit_untouched():
    """Two particles 3 m apart on each axis with 0.04 m cells span 76^3 cells,
    more than PE_FLUID_NOALLOC_MAX_CELLS (262,144)."""
    arr = dict(x=np.array([[0.0, 0.0, 0.0], [3.0, 3.0, 3.0]]), kind=np.zeros(2, np.uint8),
               psi=np.zeros(2), n_out=np.zeros((2, 3)))
    rc, got = _call(3, (1000.0, 1e-3, 0.02), arr)
    assert rc == pe.PE_ERR_BOUNDS
    assert np.all(got == SENTINEL)


def test_noalloc_rejects_non_finite_input_untouched():
    parts = _scene()
    arr = parts.arrays()
    arr["x"][7, 2] = np.nan
    rc, got = _call(3, (parts.rest_density, parts.mass, parts.h), arr)
    assert rc == pe.PE_ERR_ARG
    assert np.all(got == SENTINEL)
