"""`physics_engine_rs` — Python surface of the B200 WCSPH fluid step.

Keeps the fluid function names and signatures of the reference's PyO3 module
(`python/src/fluid.rs:288-305`) and adds `WcsphWorld` / `Particles` bindings
for the WCSPH path. All work goes through the C ABI of
`libpe_fluid_b200.so` (declared in `include/pe_fluid_wcsph.h`) via ctypes;
ctypes releases the GIL for the duration of each call, as the reference's
bindings do around stepping (`python/src/fluid.rs:164,242`).

There is no CPU fallback: if the CUDA library is missing, importing the
world classes raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

__all__ = [
    "Particles", "WcsphParams", "WcsphConfig", "WcsphWorld", "PeError",
    "mass_from_spacing", "mass_calibrated_to_rest", "fill_box", "fill_box_boundary",
    "recomputed_akinci_psi", "kernel_w", "grad_w", "tait_pressure", "pi_ij", "suggested_dt",
    "library_path", "load_library",
    # names kept from python/src/fluid.rs:288-305
    "canonical_fluid_hash", "canonical_dfsph_hash", "canonical_coupling_hash",
    "fluid_ritter_front", "fluid_ritter_height", "fluid_hydrostatic_pressure",
    "fluid_archimedes_box_draft", "fluid_heave_period_analytic",
    "fluid_barge_heave_added_mass_2d", "fluid_heave_period_with_added_mass",
    "fluid_sphere_freefall_accel_added_mass", "fluid_pbf_tank_demo", "fluid_dfsph_tank_demo",
    "fluid_poly6_w0", "fluid_canonical_mass", "fluid_canonical_ke_after_hash_steps",
]

PE_OK, PE_ERR_NULL, PE_ERR_BOUNDS, PE_ERR_ARG, PE_ERR_PANIC, PE_ERR_SCENE = 0, 1, 2, 3, 4, 5
PE_ERR_UNSUPPORTED, PE_ERR_DEVICE = 6, 7
STATUS_DOMAIN, STATUS_NEIGHBOUR_OVERFLOW, STATUS_NONFINITE, STATUS_SLOW_UNION = 1, 2, 4, 8
FLUID, BOUNDARY = 0, 1
CUBIC_SPLINE, WENDLAND_C2, POLY6, SPIKY = 0, 1, 2, 3
DIM_2, DIM_3 = 2, 3
SURFACE_TENSION_NONE, SURFACE_TENSION_AKINCI, SURFACE_TENSION_COLOUR_FIELD = 0, 1, 2
STANDARD_GRAVITY = 9.80665  # pe-math units.rs:7

_ERRNAMES = {1: "PE_ERR_NULL", 2: "PE_ERR_BOUNDS", 3: "PE_ERR_ARG", 4: "PE_ERR_PANIC",
             5: "PE_ERR_SCENE", 6: "PE_ERR_UNSUPPORTED", 7: "PE_ERR_DEVICE"}


class PeError(RuntimeError):
    """Non-zero return code of the C ABI."""

    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {_ERRNAMES.get(code, code)}")
        self.code = code


_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def library_path() -> str:
    return os.environ.get("PE_FLUID_LIB", os.path.join(_PKG_DIR, "libpe_fluid_b200.so"))


class _Params(C.Structure):
    _fields_ = [
        ("density_kernel", C.c_int32),
        ("eos_rest_density", C.c_double),
        ("eos_sound_speed", C.c_double),
        ("eos_gamma", C.c_double),
        ("visc_alpha", C.c_double),
        ("visc_beta", C.c_double),
        ("visc_eps", C.c_double),
        ("xsph_epsilon", C.c_double),
        ("gravity", C.c_double * 3),
        ("adapt_sound_speed", C.c_int32),
        ("surface_tension_sigma", C.c_double),
        ("surface_tension_model", C.c_int32),
        ("surface_tension_colour_gamma", C.c_double),
    ]


class _Config(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_neighbours", C.c_uint32),
        ("max_lower", C.c_uint32),
        ("domain_margin", C.c_double),
        ("domain_margin_cells", C.c_uint32),
        ("precision", C.c_int32),
        ("use_graph", C.c_int32),
    ]


PRECISION_F64, PRECISION_F32 = 0, 1


class _DfsphParams(C.Structure):
    _fields_ = [
        ("kernel", C.c_int32),
        ("max_density_iters", C.c_uint64),
        ("max_divergence_iters", C.c_uint64),
        ("density_error_tol", C.c_double),
        ("divergence_error_tol", C.c_double),
        ("gravity", C.c_double * 3),
        ("xsph_epsilon", C.c_double),
        ("particle_diameter", C.c_double),
        ("cfl_lambda", C.c_double),
        ("adaptive_dt", C.c_int32),
        ("warm_start", C.c_int32),
        ("free_slip_set", C.c_int32 * 4),
        ("free_slip", C.c_double * 4),
        ("solver_omega", C.c_double),
        ("max_velocity_correction", C.c_double),
    ]


class _PbfParams(C.Structure):
    _fields_ = [
        ("density_kernel", C.c_int32),
        ("grad_kernel", C.c_int32),
        ("iterations", C.c_uint64),
        ("epsilon_lambda", C.c_double),
        ("art_pressure_k", C.c_double),
        ("art_pressure_n", C.c_double),
        ("art_pressure_dq_over_h", C.c_double),
        ("viscosity_eps", C.c_double),
        ("vorticity_eps", C.c_double),
        ("gravity", C.c_double * 3),
        ("reuse_neighbours", C.c_int32),
    ]


class _Profile(C.Structure):
    _fields_ = [("ms", C.c_double * 7), ("count", C.c_uint64 * 7)]


PROFILE_PHASES = ("grid", "lists", "density", "pressure", "forces", "boundary_force", "xsph")


class _Diag(C.Structure):
    _fields_ = [
        ("total_mass", C.c_double),
        ("linear_momentum", C.c_double * 3),
        ("kinetic_energy", C.c_double),
        ("gravitational_potential", C.c_double),
        ("mean_density_error", C.c_double),
        ("max_density_error", C.c_double),
        ("v_max", C.c_double),
        ("a_max", C.c_double),
        ("hash64", C.c_uint64),
    ]


_lib = None


def load_library():
    """Load the CUDA library (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise OSError(f"libpe_fluid_b200.so not found at {path}; build it with "
                      "`make -C physics-engine_b200` (there is no CPU fallback)")
    L = C.CDLL(path)
    vp, d, i32, u32, u64 = C.c_void_p, C.c_double, C.c_int32, C.c_uint32, C.c_uint64
    D3 = C.POINTER(C.c_double)
    P = C.POINTER(_Params)
    sig = {
        "pe_fluid_particles_new": (vp, [i32, d, d, d]),
        "pe_fluid_particles_free": (None, [vp]),
        "pe_fluid_particles_len": (C.c_int, [vp, C.POINTER(u64)]),
        "pe_fluid_particles_push_fluid": (C.c_int, [vp, D3, D3]),
        "pe_fluid_particles_push_boundary": (C.c_int, [vp, D3, d]),
        "pe_fluid_particles_push_boundary_oriented": (C.c_int, [vp, D3, d, D3]),
        "pe_fluid_fill_box": (C.c_int, [vp, D3, u64, u64, u64, d, D3]),
        "pe_fluid_fill_box_boundary": (C.c_int, [vp, D3, D3, d, u64]),
        "pe_fluid_recomputed_akinci_psi": (C.c_int, [vp, i32]),
        "pe_fluid_particles_jitter_fluid": (C.c_int, [vp, u64, d]),
        "pe_fluid_particles_export": (C.c_int, [vp, vp, vp, vp, vp, vp, u64]),
        "pe_fluid_mass_from_spacing": (d, [d, d, i32]),
        "pe_fluid_mass_calibrated_to_rest": (d, [d, d, d, i32, i32]),
        "pe_fluid_wcsph_params_water": (C.c_int, [d, d, D3, P]),
        "pe_fluid_wcsph_create": (C.c_int, [vp, P, C.POINTER(_Config), C.POINTER(vp)]),
        "pe_fluid_wcsph_create_from_arrays": (C.c_int, [P, i32, d, d, d, u64, vp, vp, vp, vp, vp,
                                                        C.POINTER(_Config), C.POINTER(vp)]),
        "pe_fluid_wcsph_create_batch": (C.c_int, [P, i32, d, d, d, u64, vp, vp, vp, vp, vp, u32, vp,
                                                  C.POINTER(_Config), C.POINTER(vp)]),
        "pe_fluid_wcsph_tanks": (C.c_int, [vp, C.POINTER(u32)]),
        "pe_fluid_wcsph_get_sound_speeds": (C.c_int, [vp, vp, u32]),
        "pe_fluid_wcsph_autotune": (C.c_int, [vp, vp]),
        "pe_fluid_wcsph_shapes": (C.c_int, [vp, vp]),
        "pe_fluid_rng_uniform": (C.c_int, [u64, d, d, u64, vp]),
        "pe_fluid_wcsph_destroy": (None, [vp]),
        "pe_fluid_wcsph_step": (C.c_int, [vp, d]),
        "pe_fluid_wcsph_run": (C.c_int, [vp, d, u64]),
        "pe_fluid_wcsph_rebuild_grid": (C.c_int, [vp]),
        "pe_fluid_wcsph_compute_density": (C.c_int, [vp]),
        "pe_fluid_wcsph_compute_pressure": (C.c_int, [vp]),
        "pe_fluid_wcsph_compute_forces": (C.c_int, [vp]),
        "pe_fluid_wcsph_apply_xsph": (C.c_int, [vp]),
        "pe_fluid_wcsph_len": (C.c_int, [vp, C.POINTER(u64)]),
        "pe_fluid_wcsph_get_time": (C.c_int, [vp, D3]),
        "pe_fluid_wcsph_set_time": (C.c_int, [vp, d]),
        "pe_fluid_wcsph_get_sound_speed": (C.c_int, [vp, D3]),
        "pe_fluid_wcsph_get_params": (C.c_int, [vp, P]),
        "pe_fluid_wcsph_set_params": (C.c_int, [vp, P]),
        "pe_fluid_wcsph_get_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_accelerations": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_boundary_forces": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_densities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_pressures": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_kinds": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_set_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_set_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_set_densities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_set_pressures": (C.c_int, [vp, vp, u64]),
        "pe_fluid_wcsph_get_grid": (C.c_int, [vp, vp, vp, u64, vp, vp, u64, C.POINTER(u64)]),
        "pe_fluid_wcsph_get_neighbour_counts": (C.c_int, [vp, vp, vp, u64]),
        "pe_fluid_wcsph_status": (C.c_int, [vp, C.POINTER(u32)]),
        "pe_fluid_wcsph_clear_status": (C.c_int, [vp]),
        "pe_fluid_wcsph_capacity_info": (C.c_int, [vp, vp]),
        "pe_fluid_wcsph_diagnostics": (C.c_int, [vp, C.POINTER(_Diag)]),
        "pe_fluid_wcsph_fluid_center_of_mass": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "pe_fluid_wcsph_list_chunk": (C.c_int, [vp, C.POINTER(C.c_uint32)]),
        "pe_fluid_wcsph_set_pair_weights": (C.c_int, [vp, C.c_int32]),
        "pe_fluid_wcsph_pair_weights": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "pe_fluid_wcsph_pair_weight_info": (C.c_int, [vp, vp]),
        "pe_fluid_wcsph_kernel_launches": (C.c_int, [vp, C.POINTER(u64), i32]),
        "pe_fluid_wcsph_profile": (C.c_int, [vp, i32]),
        "pe_fluid_wcsph_profile_read": (C.c_int, [vp, C.POINTER(_Profile), i32]),
        "pe_fluid_wcsph_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "pe_fluid_pbf_params_default": (C.c_int, [C.POINTER(_PbfParams)]),
        "pe_fluid_pbf_create": (C.c_int, [vp, C.POINTER(_PbfParams), C.POINTER(_Config), C.POINTER(vp)]),
        "pe_fluid_pbf_destroy": (None, [vp]),
        "pe_fluid_pbf_step": (C.c_int, [vp, d]),
        "pe_fluid_pbf_run": (C.c_int, [vp, d, u64]),
        "pe_fluid_pbf_len": (C.c_int, [vp, C.POINTER(u64)]),
        "pe_fluid_pbf_get_time": (C.c_int, [vp, D3]),
        "pe_fluid_pbf_get_params": (C.c_int, [vp, C.POINTER(_PbfParams)]),
        "pe_fluid_pbf_set_params": (C.c_int, [vp, C.POINTER(_PbfParams)]),
        "pe_fluid_pbf_get_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_get_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_get_densities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_get_lambdas": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_set_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_set_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_pbf_mean_density_error": (C.c_int, [vp, D3]),
        "pe_fluid_pbf_v_max": (C.c_int, [vp, D3]),
        "pe_fluid_pbf_status": (C.c_int, [vp, C.POINTER(u32)]),
        "pe_fluid_pbf_kernel_launches": (C.c_int, [vp, C.POINTER(u64), i32]),
        "pe_fluid_pbf_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "pe_fluid_dfsph_params_default": (C.c_int, [C.POINTER(_DfsphParams)]),
        "pe_fluid_dfsph_create": (C.c_int, [vp, C.POINTER(_DfsphParams), C.POINTER(_Config), C.POINTER(vp)]),
        "pe_fluid_dfsph_destroy": (None, [vp]),
        "pe_fluid_dfsph_step": (C.c_int, [vp, d]),
        "pe_fluid_dfsph_run": (C.c_int, [vp, d, u64]),
        "pe_fluid_dfsph_step_adaptive": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_suggest_dt": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_rebuild_neighbours": (C.c_int, [vp]),
        "pe_fluid_dfsph_compute_density": (C.c_int, [vp]),
        "pe_fluid_dfsph_compute_alpha": (C.c_int, [vp]),
        "pe_fluid_dfsph_len": (C.c_int, [vp, C.POINTER(u64)]),
        "pe_fluid_dfsph_get_time": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_get_last_dt": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_get_params": (C.c_int, [vp, C.POINTER(_DfsphParams)]),
        "pe_fluid_dfsph_set_params": (C.c_int, [vp, C.POINTER(_DfsphParams)]),
        "pe_fluid_dfsph_get_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_get_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_get_densities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_get_pressures": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_get_boundary_forces": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_get_alphas": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_set_positions": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_set_velocities": (C.c_int, [vp, vp, u64]),
        "pe_fluid_dfsph_last_iterations": (C.c_int, [vp, vp]),
        "pe_fluid_dfsph_mean_density_error": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_v_max": (C.c_int, [vp, D3]),
        "pe_fluid_dfsph_status": (C.c_int, [vp, C.POINTER(u32)]),
        "pe_fluid_dfsph_kernel_launches": (C.c_int, [vp, C.POINTER(u64), i32]),
        "pe_fluid_dfsph_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "pe_fluid_coupler_create": (C.c_int, [vp, u32, u64, vp, vp, vp, vp, C.POINTER(vp)]),
        "pe_fluid_coupler_destroy": (None, [vp]),
        "pe_fluid_coupler_sync": (C.c_int, [vp, vp, vp, vp, vp]),
        "pe_fluid_coupler_reduce": (C.c_int, [vp, vp, vp, vp]),
        "pe_fluid_kernel_w": (d, [i32, d, d, i32]),
        "pe_fluid_grad_w": (C.c_int, [i32, D3, d, i32, D3]),
        "pe_fluid_tait_pressure": (d, [d, d, d, d]),
        "pe_fluid_pi_ij": (d, [d, d, d, d, d, D3, D3, D3, D3, d, d]),
        "pe_fluid_suggested_dt": (d, [d, d, d, d, d, d]),
        "pe_fluid_version": (C.c_char_p, []),
        "pe_fluid_probe_fp64_rate": (C.c_int, [i32, D3]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _v3(v):
    return (C.c_double * 3)(*[float(t) for t in v])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _ok(rc: int, what: str):
    if rc != PE_OK:
        raise PeError(rc, what)


def _arr(a, dtype, shape):
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.shape != shape:
        a = a.reshape(shape)
    return a


# --------------------------------------------------------------------------
# Particles (crates/pe-fluid/src/particles.rs)
# --------------------------------------------------------------------------
class Particles:
    """Structure-of-arrays particle builder (`Particles`, particles.rs:20)."""

    def __init__(self, dim: int, rest_density: float, mass: float, h: float):
        L = load_library()
        self.dim, self.rest_density, self.mass, self.h = int(dim), float(rest_density), float(mass), float(h)
        self._p = L.pe_fluid_particles_new(self.dim, self.rest_density, self.mass, self.h)
        if not self._p:
            raise ValueError("invalid particle parameters (dim must be 2 or 3, values finite)")

    def __del__(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.pe_fluid_particles_free(self._p)
            self._p = None

    def __len__(self):
        n = C.c_uint64()
        _ok(_lib.pe_fluid_particles_len(self._p, C.byref(n)), "len")
        return n.value

    def push_fluid(self, x, v=(0.0, 0.0, 0.0)):
        _ok(_lib.pe_fluid_particles_push_fluid(self._p, _v3(x), _v3(v)), "push_fluid")

    def push_boundary(self, x, psi):
        _ok(_lib.pe_fluid_particles_push_boundary(self._p, _v3(x), float(psi)), "push_boundary")

    def push_boundary_oriented(self, x, psi, n_out):
        _ok(_lib.pe_fluid_particles_push_boundary_oriented(self._p, _v3(x), float(psi), _v3(n_out)),
            "push_boundary_oriented")

    def fill_box(self, origin, nx, ny, nz, dx, v0=(0.0, 0.0, 0.0)):
        _ok(_lib.pe_fluid_fill_box(self._p, _v3(origin), int(nx), int(ny), int(nz), float(dx), _v3(v0)),
            "fill_box")

    def fill_box_boundary(self, mn, mx, dx, layers=1):
        _ok(_lib.pe_fluid_fill_box_boundary(self._p, _v3(mn), _v3(mx), float(dx), int(layers)),
            "fill_box_boundary")

    def recomputed_akinci_psi(self, kernel=CUBIC_SPLINE):
        _ok(_lib.pe_fluid_recomputed_akinci_psi(self._p, kernel), "recomputed_akinci_psi")

    def jitter_fluid(self, seed: int, amplitude: float):
        _ok(_lib.pe_fluid_particles_jitter_fluid(self._p, int(seed), float(amplitude)), "jitter_fluid")

    def arrays(self):
        n = len(self)
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); kind = np.zeros(n, np.uint8)
        psi = np.zeros(n); nout = np.zeros((n, 3))
        _ok(_lib.pe_fluid_particles_export(self._p, _ptr(x), _ptr(v), _ptr(kind), _ptr(psi),
                                           _ptr(nout), n), "export")
        return dict(x=x, v=v, kind=kind, psi=psi, n_out=nout)

    def pack_positions(self):
        """`Particles::pack_positions` (particles.rs:137): flat [x0, y0, z0, ...]."""
        return self.arrays()["x"].reshape(-1)

    def pack_velocities(self):
        return self.arrays()["v"].reshape(-1)

    def fluid_count(self):
        return int(np.count_nonzero(self.arrays()["kind"] == FLUID))


def mass_from_spacing(rest_density, dx, dim):
    return load_library().pe_fluid_mass_from_spacing(float(rest_density), float(dx), int(dim))


def mass_calibrated_to_rest(rest_density, dx, h, dim, kernel=CUBIC_SPLINE):
    return load_library().pe_fluid_mass_calibrated_to_rest(float(rest_density), float(dx), float(h),
                                                           int(dim), kernel)


def fill_box(parts: Particles, origin, nx, ny, nz, dx, v0=(0.0, 0.0, 0.0)):
    parts.fill_box(origin, nx, ny, nz, dx, v0)


def fill_box_boundary(parts: Particles, mn, mx, dx, layers=1):
    parts.fill_box_boundary(mn, mx, dx, layers)


def recomputed_akinci_psi(parts: Particles, kernel=CUBIC_SPLINE):
    parts.recomputed_akinci_psi(kernel)


# --------------------------------------------------------------------------
# WCSPH (crates/pe-fluid/src/wcsph.rs)
# --------------------------------------------------------------------------
class WcsphParams:
    """`WcsphParams` (wcsph.rs:24) flattened; `water()` gives wcsph.rs:43 defaults."""

    _FIELDS = ("density_kernel", "eos_rest_density", "eos_sound_speed", "eos_gamma", "visc_alpha",
               "visc_beta", "visc_eps", "xsph_epsilon", "gravity", "adapt_sound_speed",
               "surface_tension_sigma", "surface_tension_model", "surface_tension_colour_gamma")

    def __init__(self, **kw):
        self.density_kernel = CUBIC_SPLINE
        self.eos_rest_density = 1000.0
        self.eos_sound_speed = 20.0
        self.eos_gamma = 7.0
        self.visc_alpha, self.visc_beta, self.visc_eps = 0.01, 0.0, 0.01
        self.xsph_epsilon = 0.25
        self.gravity = (0.0, 0.0, -STANDARD_GRAVITY)
        self.adapt_sound_speed = True
        self.surface_tension_sigma = 0.0
        self.surface_tension_model = SURFACE_TENSION_NONE
        self.surface_tension_colour_gamma = 0.0
        for k, v in kw.items():
            if k not in self._FIELDS:
                raise TypeError(f"unknown WcsphParams field {k!r}")
            setattr(self, k, v)

    @classmethod
    def water(cls, rest_density, sound_speed, gravity):
        c = _Params()
        _ok(load_library().pe_fluid_wcsph_params_water(float(rest_density), float(sound_speed),
                                                       _v3(gravity), C.byref(c)), "params_water")
        return cls._from_c(c)

    def _to_c(self) -> _Params:
        c = _Params()
        c.density_kernel = int(self.density_kernel)
        c.eos_rest_density = float(self.eos_rest_density)
        c.eos_sound_speed = float(self.eos_sound_speed)
        c.eos_gamma = float(self.eos_gamma)
        c.visc_alpha, c.visc_beta, c.visc_eps = float(self.visc_alpha), float(self.visc_beta), float(self.visc_eps)
        c.xsph_epsilon = float(self.xsph_epsilon)
        c.gravity[:] = [float(g) for g in self.gravity]
        c.adapt_sound_speed = 1 if self.adapt_sound_speed else 0
        c.surface_tension_sigma = float(self.surface_tension_sigma)
        c.surface_tension_model = int(self.surface_tension_model)
        c.surface_tension_colour_gamma = float(self.surface_tension_colour_gamma)
        return c

    @classmethod
    def _from_c(cls, c: _Params):
        return cls(density_kernel=c.density_kernel, eos_rest_density=c.eos_rest_density,
                   eos_sound_speed=c.eos_sound_speed, eos_gamma=c.eos_gamma, visc_alpha=c.visc_alpha,
                   visc_beta=c.visc_beta, visc_eps=c.visc_eps, xsph_epsilon=c.xsph_epsilon,
                   gravity=tuple(c.gravity), adapt_sound_speed=bool(c.adapt_sound_speed),
                   surface_tension_sigma=c.surface_tension_sigma, surface_tension_model=c.surface_tension_model,
                   surface_tension_colour_gamma=c.surface_tension_colour_gamma)

    def __repr__(self):
        return "WcsphParams(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._FIELDS) + ")"


class WcsphConfig:
    """GPU placement and capacities (no reference counterpart)."""

    def __init__(self, device=-1, max_neighbours=0, max_lower=0, domain_margin=-1.0,
                 domain_margin_cells=0, precision=PRECISION_F64, use_graph=False):
        self.device, self.max_neighbours, self.max_lower = device, max_neighbours, max_lower
        self.domain_margin, self.domain_margin_cells = domain_margin, domain_margin_cells
        self.precision = precision
        self.use_graph = use_graph

    def _to_c(self):
        c = _Config()
        c.device = int(self.device)
        c.max_neighbours = int(self.max_neighbours)
        c.max_lower = int(self.max_lower)
        c.domain_margin = float(self.domain_margin)
        c.domain_margin_cells = int(self.domain_margin_cells)
        c.precision = int(self.precision)
        c.use_graph = 1 if self.use_graph else 0
        return c


class WcsphWorld:
    """`WcsphWorld` (wcsph.rs:58) on one B200. State arrays are in original order."""

    def __init__(self, particles: Particles, params: WcsphParams, config: WcsphConfig | None = None):
        L = load_library()
        self._w = None
        h = C.c_void_p()
        cfg = config._to_c() if config is not None else None
        _ok(L.pe_fluid_wcsph_create(particles._p, C.byref(params._to_c()),
                                    C.byref(cfg) if cfg is not None else None, C.byref(h)), "create")
        self._w = h
        n = C.c_uint64()
        _ok(L.pe_fluid_wcsph_len(self._w, C.byref(n)), "len")
        self.n = n.value
        self.dim, self.mass, self.h, self.rest_density = particles.dim, particles.mass, particles.h, particles.rest_density

    @classmethod
    def from_arrays(cls, params: WcsphParams, dim, rest_density, mass, h, x, v=None, kind=None,
                    psi=None, n_out=None, config: WcsphConfig | None = None):
        L = load_library()
        x = _arr(x, np.float64, (-1, 3)) if np.ndim(x) == 2 else np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        n = x.shape[0]
        v = None if v is None else np.ascontiguousarray(v, np.float64).reshape(n, 3)
        kind = np.zeros(n, np.uint8) if kind is None else np.ascontiguousarray(kind, np.uint8)
        psi = None if psi is None else np.ascontiguousarray(psi, np.float64)
        n_out = None if n_out is None else np.ascontiguousarray(n_out, np.float64).reshape(n, 3)
        self = cls.__new__(cls)
        self._w = None
        hnd = C.c_void_p()
        cfg = config._to_c() if config is not None else None
        _ok(L.pe_fluid_wcsph_create_from_arrays(
            C.byref(params._to_c()), int(dim), float(rest_density), float(mass), float(h), n, _ptr(x),
            _ptr(v) if v is not None else None, _ptr(kind), _ptr(psi) if psi is not None else None,
            _ptr(n_out) if n_out is not None else None, C.byref(cfg) if cfg is not None else None,
            C.byref(hnd)), "create_from_arrays")
        self._w = hnd
        self.n, self.dim, self.mass, self.h, self.rest_density = n, int(dim), float(mass), float(h), float(rest_density)
        return self

    @classmethod
    def from_tanks(cls, params: WcsphParams, tanks, config: WcsphConfig | None = None):
        """Batched form: independent tanks (a list of `Particles` with the same
        dim, rest density, mass and h) stepped together by one world. State
        arrays are the tanks' arrays concatenated in order; `tank_offsets`
        gives each tank's range."""
        L = load_library()
        tanks = list(tanks)
        if not tanks:
            raise ValueError("no tanks")
        p0 = tanks[0]
        for t in tanks:
            if (t.dim, t.rest_density, t.mass, t.h) != (p0.dim, p0.rest_density, p0.mass, p0.h):
                raise ValueError("tanks must share dim, rest density, mass and h")
        arrs = [t.arrays() for t in tanks]
        counts = np.array([a["x"].shape[0] for a in arrs], np.uint64)
        offsets = np.zeros(len(tanks) + 1, np.uint64)
        offsets[1:] = np.cumsum(counts)
        cat = {k: np.ascontiguousarray(np.concatenate([a[k] for a in arrs])) for k in arrs[0]}
        n = int(offsets[-1])
        self = cls.__new__(cls)
        self._w = None
        hnd = C.c_void_p()
        cfg = config._to_c() if config is not None else None
        _ok(L.pe_fluid_wcsph_create_batch(
            C.byref(params._to_c()), int(p0.dim), float(p0.rest_density), float(p0.mass), float(p0.h), n,
            _ptr(cat["x"]), _ptr(cat["v"]), _ptr(cat["kind"]), _ptr(cat["psi"]), _ptr(cat["n_out"]),
            len(tanks), _ptr(offsets), C.byref(cfg) if cfg is not None else None, C.byref(hnd)),
            "create_batch")
        self._w = hnd
        self.n, self.dim, self.mass, self.h, self.rest_density = n, p0.dim, p0.mass, p0.h, p0.rest_density
        self.tank_offsets = offsets
        return self

    def tanks(self) -> int:
        t = C.c_uint32()
        _ok(_lib.pe_fluid_wcsph_tanks(self._w, C.byref(t)), "tanks")
        return t.value

    def sound_speeds(self):
        out = np.zeros(self.tanks())
        _ok(_lib.pe_fluid_wcsph_get_sound_speeds(self._w, _ptr(out), out.size), "get_sound_speeds")
        return out

    def autotune(self) -> dict:
        """Pick the passes' block sizes and the list build's tile and CTAs per
        SM by timing them on the current state (the simulation does not
        advance)."""
        out = np.zeros(4, np.uint32)
        _ok(_lib.pe_fluid_wcsph_autotune(self._w, _ptr(out)), "autotune")
        return self.shapes()

    def shapes(self) -> dict:
        out = np.zeros(4, np.uint32)
        _ok(_lib.pe_fluid_wcsph_shapes(self._w, _ptr(out)), "shapes")
        r = dict(zip(("density", "forces", "xsph", "list_ctas_per_sm"), (int(v) for v in out)))
        c = C.c_uint32(0)
        _ok(_lib.pe_fluid_wcsph_list_chunk(self._w, C.byref(c)), "list_chunk")
        r["list_chunk"] = int(c.value)
        return r

    def set_pair_weights(self, on: bool = True):
        """Let the density pass keep each neighbour entry's W for the XSPH pass
        (on by default, while the device has room for the buffer); off, XSPH
        recomputes W. The f64 step's results are identical either way."""
        _ok(_lib.pe_fluid_wcsph_set_pair_weights(self._w, 1 if on else 0), "set_pair_weights")

    def pair_weights(self) -> bool:
        """Whether the pair-weight buffer is in use."""
        c = C.c_int32(0)
        _ok(_lib.pe_fluid_wcsph_pair_weights(self._w, C.byref(c)), "pair_weights")
        return bool(c.value)

    def pair_weight_info(self) -> dict:
        """{in_use, entries (list entries the buffer covers), short (the last
        density pass met a list beyond them, so XSPH recomputed W)}."""
        out = np.zeros(3, np.uint64)
        _ok(_lib.pe_fluid_wcsph_pair_weight_info(self._w, _ptr(out)), "pair_weight_info")
        return {"in_use": bool(out[0]), "entries": int(out[1]), "short": bool(out[2])}

    def close(self):
        if getattr(self, "_w", None) and _lib is not None:
            _lib.pe_fluid_wcsph_destroy(self._w)
        self._w = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- stepping (wcsph.rs:102-347) --
    def step(self, dt: float):
        _ok(_lib.pe_fluid_wcsph_step(self._w, float(dt)), "step")

    def run(self, dt: float, steps: int):
        _ok(_lib.pe_fluid_wcsph_run(self._w, float(dt), int(steps)), "run")

    def rebuild_grid(self):
        _ok(_lib.pe_fluid_wcsph_rebuild_grid(self._w), "rebuild_grid")

    def compute_density(self):
        _ok(_lib.pe_fluid_wcsph_compute_density(self._w), "compute_density")

    def compute_pressure(self):
        _ok(_lib.pe_fluid_wcsph_compute_pressure(self._w), "compute_pressure")

    def compute_forces(self):
        _ok(_lib.pe_fluid_wcsph_compute_forces(self._w), "compute_forces")

    def apply_xsph(self):
        _ok(_lib.pe_fluid_wcsph_apply_xsph(self._w), "apply_xsph")

    # -- scalars --
    @property
    def t(self) -> float:
        t = C.c_double()
        _ok(_lib.pe_fluid_wcsph_get_time(self._w, C.byref(t)), "get_time")
        return t.value

    @t.setter
    def t(self, value):
        _ok(_lib.pe_fluid_wcsph_set_time(self._w, float(value)), "set_time")

    @property
    def sound_speed(self) -> float:
        c = C.c_double()
        _ok(_lib.pe_fluid_wcsph_get_sound_speed(self._w, C.byref(c)), "get_sound_speed")
        return c.value

    @property
    def params(self) -> WcsphParams:
        c = _Params()
        _ok(_lib.pe_fluid_wcsph_get_params(self._w, C.byref(c)), "get_params")
        return WcsphParams._from_c(c)

    @params.setter
    def params(self, p: WcsphParams):
        _ok(_lib.pe_fluid_wcsph_set_params(self._w, C.byref(p._to_c())), "set_params")

    # -- state in original order --
    def _get3(self, fn, what, out=None):
        if out is None:
            out = np.empty((self.n, 3))
        elif out.shape != (self.n, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"{what}: out must be a C-contiguous float64 array of shape ({self.n}, 3)")
        _ok(fn(self._w, _ptr(out), self.n), what)
        return out

    def _get1(self, fn, what):
        out = np.empty(self.n)
        _ok(fn(self._w, _ptr(out), self.n), what)
        return out

    def positions(self, out=None):
        """Positions in original order; `out` (n x 3 float64, e.g. pinned) is filled in place."""
        return self._get3(_lib.pe_fluid_wcsph_get_positions, "get_positions", out)

    def velocities(self, out=None):
        return self._get3(_lib.pe_fluid_wcsph_get_velocities, "get_velocities", out)

    def accelerations(self):
        return self._get3(_lib.pe_fluid_wcsph_get_accelerations, "get_accelerations")

    def boundary_forces(self):
        return self._get3(_lib.pe_fluid_wcsph_get_boundary_forces, "get_boundary_forces")

    def densities(self):
        return self._get1(_lib.pe_fluid_wcsph_get_densities, "get_densities")

    def pressures(self):
        return self._get1(_lib.pe_fluid_wcsph_get_pressures, "get_pressures")

    def kinds(self):
        out = np.empty(self.n, np.uint8)
        _ok(_lib.pe_fluid_wcsph_get_kinds(self._w, _ptr(out), self.n), "get_kinds")
        return out

    def set_positions(self, x):
        x = _arr(x, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_wcsph_set_positions(self._w, _ptr(x), self.n), "set_positions")

    def set_velocities(self, v):
        v = _arr(v, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_wcsph_set_velocities(self._w, _ptr(v), self.n), "set_velocities")

    def set_densities(self, r):
        r = _arr(r, np.float64, (self.n,))
        _ok(_lib.pe_fluid_wcsph_set_densities(self._w, _ptr(r), self.n), "set_densities")

    def set_pressures(self, p):
        p = _arr(p, np.float64, (self.n,))
        _ok(_lib.pe_fluid_wcsph_set_pressures(self._w, _ptr(p), self.n), "set_pressures")

    # -- grid / diagnostics --
    def grid(self):
        """`UniformGrid` fields (grid.rs:32-45): keys, order, occupied, ranges."""
        m = C.c_uint64()
        _ok(_lib.pe_fluid_wcsph_get_grid(self._w, None, None, self.n, None, None, 0, C.byref(m)), "grid")
        keys = np.empty((self.n, 3), np.int32)
        order = np.empty(self.n, np.uint64)
        occ = np.empty((max(m.value, 1), 3), np.int32)
        rng = np.empty((max(m.value, 1), 2), np.uint64)
        _ok(_lib.pe_fluid_wcsph_get_grid(self._w, _ptr(keys), _ptr(order), self.n, _ptr(occ), _ptr(rng),
                                         max(m.value, 1), C.byref(m)), "grid")
        return dict(keys=keys, order=order, occupied=occ[: m.value], ranges=rng[: m.value])

    def neighbour_counts(self):
        cand = np.empty(self.n, np.uint32)
        sup = np.empty(self.n, np.uint32)
        _ok(_lib.pe_fluid_wcsph_get_neighbour_counts(self._w, _ptr(cand), _ptr(sup), self.n), "counts")
        return cand, sup

    def status(self) -> int:
        s = C.c_uint32()
        _ok(_lib.pe_fluid_wcsph_status(self._w, C.byref(s)), "status")
        return s.value

    def capacity_info(self) -> dict:
        out = np.zeros(8, np.uint64)
        _ok(_lib.pe_fluid_wcsph_capacity_info(self._w, _ptr(out)), "capacity_info")
        keys = ("status", "max_union", "list_groups_used", "union_capacity", "list_groups_capacity",
                "occupied_cells", "dense_cells", "list_ctas")
        return {k: int(v) for k, v in zip(keys, out)}

    def clear_status(self):
        _ok(_lib.pe_fluid_wcsph_clear_status(self._w), "clear_status")

    def diagnostics(self) -> dict:
        d = _Diag()
        _ok(_lib.pe_fluid_wcsph_diagnostics(self._w, C.byref(d)), "diagnostics")
        return dict(total_mass=d.total_mass, linear_momentum=np.array(d.linear_momentum[:]),
                    kinetic_energy=d.kinetic_energy, gravitational_potential=d.gravitational_potential,
                    mean_density_error=d.mean_density_error, max_density_error=d.max_density_error,
                    v_max=d.v_max, a_max=d.a_max, hash64=d.hash64)

    def fluid_center_of_mass(self) -> np.ndarray:
        """Fluid positions summed in index order on the device / fluid count."""
        out = (C.c_double * 3)()
        _ok(_lib.pe_fluid_wcsph_fluid_center_of_mass(self._w, out), "fluid_center_of_mass")
        return np.array(out[:])

    def v_max(self):
        return self.diagnostics()["v_max"]

    def a_max(self):
        return self.diagnostics()["a_max"]

    def hash64(self):
        return self.diagnostics()["hash64"]

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) all of this world's kernels run on."""
        out = C.c_void_p()
        _ok(_lib.pe_fluid_wcsph_stream(self._w, C.byref(out)), "stream")
        return out.value or 0

    def set_profiling(self, on: bool):
        _ok(_lib.pe_fluid_wcsph_profile(self._w, 1 if on else 0), "profile")

    def profile(self, reset=False) -> dict:
        """Per-phase device milliseconds and launch counts (CUDA events)."""
        pr = _Profile()
        _ok(_lib.pe_fluid_wcsph_profile_read(self._w, C.byref(pr), 1 if reset else 0), "profile_read")
        return {name: (pr.ms[i], pr.count[i]) for i, name in enumerate(PROFILE_PHASES)}

    def kernel_launches(self, reset=False):
        out = C.c_uint64()
        _ok(_lib.pe_fluid_wcsph_kernel_launches(self._w, C.byref(out), 1 if reset else 0), "launches")
        return out.value


# --------------------------------------------------------------------------
# stateless helpers
# --------------------------------------------------------------------------
# --------------------------------------------------------------------------
# Position Based Fluids (crates/pe-fluid/src/pbf.rs)
# --------------------------------------------------------------------------
class PbfParams:
    """`PbfParams` (pbf.rs:26-53); the defaults are `PbfParams::default` (pbf.rs:55-74)."""

    _FIELDS = ("density_kernel", "grad_kernel", "iterations", "epsilon_lambda", "art_pressure_k",
               "art_pressure_n", "art_pressure_dq_over_h", "viscosity_eps", "vorticity_eps", "gravity",
               "reuse_neighbours")

    def __init__(self, **kw):
        c = _PbfParams()
        _ok(load_library().pe_fluid_pbf_params_default(C.byref(c)), "pbf_params_default")
        for k in self._FIELDS:
            v = getattr(c, k)
            setattr(self, k, tuple(v) if k == "gravity" else v)
        self.reuse_neighbours = bool(self.reuse_neighbours)
        for k, v in kw.items():
            if k not in self._FIELDS:
                raise TypeError(f"unknown PbfParams field {k!r}")
            setattr(self, k, v)

    def _to_c(self) -> _PbfParams:
        c = _PbfParams()
        c.density_kernel, c.grad_kernel = int(self.density_kernel), int(self.grad_kernel)
        c.iterations = int(self.iterations)
        c.epsilon_lambda, c.art_pressure_k = float(self.epsilon_lambda), float(self.art_pressure_k)
        c.art_pressure_n, c.art_pressure_dq_over_h = float(self.art_pressure_n), float(self.art_pressure_dq_over_h)
        c.viscosity_eps, c.vorticity_eps = float(self.viscosity_eps), float(self.vorticity_eps)
        c.gravity[:] = [float(g) for g in self.gravity]
        c.reuse_neighbours = 1 if self.reuse_neighbours else 0
        return c

    def __repr__(self):
        return "PbfParams(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._FIELDS) + ")"


class PbfWorld:
    """`PbfWorld` (pbf.rs:77-459) on one B200, bit-identical to the reference's
    step. State arrays are in original order."""

    def __init__(self, particles: Particles, params: PbfParams | None = None,
                 config: WcsphConfig | None = None):
        L = load_library()
        self._w = None
        params = params if params is not None else PbfParams()
        h = C.c_void_p()
        cfg = config._to_c() if config is not None else None
        _ok(L.pe_fluid_pbf_create(particles._p, C.byref(params._to_c()),
                                  C.byref(cfg) if cfg is not None else None, C.byref(h)), "pbf_create")
        self._w = h
        self.n = len(particles)
        self._kinds = particles.arrays()["kind"].copy()
        self.dim, self.mass, self.h, self.rest_density = particles.dim, particles.mass, particles.h, particles.rest_density

    def close(self):
        if getattr(self, "_w", None) and _lib is not None:
            _lib.pe_fluid_pbf_destroy(self._w)
        self._w = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, dt: float):
        _ok(_lib.pe_fluid_pbf_step(self._w, float(dt)), "pbf_step")

    def run(self, dt: float, steps: int):
        _ok(_lib.pe_fluid_pbf_run(self._w, float(dt), int(steps)), "pbf_run")

    @property
    def t(self) -> float:
        t = C.c_double()
        _ok(_lib.pe_fluid_pbf_get_time(self._w, C.byref(t)), "pbf_time")
        return t.value

    @property
    def params(self) -> PbfParams:
        c = _PbfParams()
        _ok(_lib.pe_fluid_pbf_get_params(self._w, C.byref(c)), "pbf_params")
        p = PbfParams()
        for k in PbfParams._FIELDS:
            v = getattr(c, k)
            setattr(p, k, tuple(v) if k == "gravity" else v)
        p.reuse_neighbours = bool(p.reuse_neighbours)
        return p

    @params.setter
    def params(self, p: PbfParams):
        _ok(_lib.pe_fluid_pbf_set_params(self._w, C.byref(p._to_c())), "pbf_set_params")

    def _get(self, fn, shape, what):
        out = np.empty(shape)
        _ok(fn(self._w, _ptr(out), self.n), what)
        return out

    def positions(self):
        return self._get(_lib.pe_fluid_pbf_get_positions, (self.n, 3), "pbf_positions")

    def velocities(self):
        return self._get(_lib.pe_fluid_pbf_get_velocities, (self.n, 3), "pbf_velocities")

    def densities(self):
        return self._get(_lib.pe_fluid_pbf_get_densities, (self.n,), "pbf_densities")

    def lambdas(self):
        return self._get(_lib.pe_fluid_pbf_get_lambdas, (self.n,), "pbf_lambdas")

    def set_positions(self, x):
        x = _arr(x, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_pbf_set_positions(self._w, _ptr(x), self.n), "pbf_set_positions")

    def set_velocities(self, v):
        v = _arr(v, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_pbf_set_velocities(self._w, _ptr(v), self.n), "pbf_set_velocities")

    def mean_density_error(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_pbf_mean_density_error(self._w, C.byref(d)), "pbf_mean_density_error")
        return d.value

    def v_max(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_pbf_v_max(self._w, C.byref(d)), "pbf_v_max")
        return d.value

    def status(self) -> int:
        s = C.c_uint32()
        _ok(_lib.pe_fluid_pbf_status(self._w, C.byref(s)), "pbf_status")
        return s.value

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) all of this world's kernels run on."""
        h = C.c_void_p()
        _ok(_lib.pe_fluid_pbf_stream(self._w, C.byref(h)), "stream")
        return h.value or 0

    def kernel_launches(self, reset=False) -> int:
        c = C.c_uint64()
        _ok(_lib.pe_fluid_pbf_kernel_launches(self._w, C.byref(c), 1 if reset else 0), "pbf_launches")
        return c.value

    def kinds(self):
        """Particle kinds in original order (fixed at creation)."""
        return self._kinds

    def hash64(self) -> int:
        """`particles_hash64` (diagnostics.rs:10-33) of the current state."""
        return particles_hash64(self.positions(), self.velocities(), self._kinds)


def particles_hash64(x, v, kind) -> int:
    """FNV-1a 64 over the IEEE bits of fluid (x, v), little-endian, in index
    order (diagnostics.rs:10-33)."""
    fluid = np.asarray(kind) == FLUID
    data = np.concatenate([np.asarray(x, np.float64)[fluid], np.asarray(v, np.float64)[fluid]], axis=1)
    h = 0xCBF29CE484222325
    for b in np.ascontiguousarray(data).astype("<f8").tobytes():
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


# --------------------------------------------------------------------------
# Divergence-free SPH (crates/pe-fluid/src/dfsph.rs)
# --------------------------------------------------------------------------
class DfsphParams:
    """`DfsphParams` (dfsph.rs:33-80) without surface tension; the defaults are
    `DfsphParams::default` (dfsph.rs:82-104). The free-slip planes are
    `free_slip_xmin`, `free_slip_ymin`, `free_slip_xmax`, `free_slip_ymax`
    (None = off)."""

    _FIELDS = ("kernel", "max_density_iters", "max_divergence_iters", "density_error_tol",
               "divergence_error_tol", "gravity", "xsph_epsilon", "particle_diameter", "cfl_lambda",
               "adaptive_dt", "warm_start", "free_slip_xmin", "free_slip_ymin", "free_slip_xmax",
               "free_slip_ymax", "solver_omega", "max_velocity_correction")
    _SLIPS = ("free_slip_xmin", "free_slip_ymin", "free_slip_xmax", "free_slip_ymax")

    def __init__(self, **kw):
        c = _DfsphParams()
        _ok(load_library().pe_fluid_dfsph_params_default(C.byref(c)), "dfsph_params_default")
        self._load(c)
        for k, v in kw.items():
            if k not in self._FIELDS:
                raise TypeError(f"unknown DfsphParams field {k!r}")
            setattr(self, k, v)

    def _load(self, c):
        for k in self._FIELDS:
            if k in self._SLIPS:
                a = self._SLIPS.index(k)
                setattr(self, k, float(c.free_slip[a]) if c.free_slip_set[a] else None)
            elif k == "gravity":
                self.gravity = tuple(c.gravity)
            else:
                setattr(self, k, getattr(c, k))
        self.adaptive_dt, self.warm_start = bool(self.adaptive_dt), bool(self.warm_start)

    def _to_c(self) -> _DfsphParams:
        c = _DfsphParams()
        c.kernel = int(self.kernel)
        c.max_density_iters, c.max_divergence_iters = int(self.max_density_iters), int(self.max_divergence_iters)
        c.density_error_tol, c.divergence_error_tol = float(self.density_error_tol), float(self.divergence_error_tol)
        c.gravity[:] = [float(g) for g in self.gravity]
        c.xsph_epsilon, c.particle_diameter = float(self.xsph_epsilon), float(self.particle_diameter)
        c.cfl_lambda = float(self.cfl_lambda)
        c.adaptive_dt, c.warm_start = 1 if self.adaptive_dt else 0, 1 if self.warm_start else 0
        for a, k in enumerate(self._SLIPS):
            v = getattr(self, k)
            c.free_slip_set[a] = 0 if v is None else 1
            c.free_slip[a] = 0.0 if v is None else float(v)
        c.solver_omega, c.max_velocity_correction = float(self.solver_omega), float(self.max_velocity_correction)
        return c

    def __repr__(self):
        return "DfsphParams(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._FIELDS) + ")"


class DfsphWorld:
    """`DfsphWorld` (dfsph.rs:107-800) on one B200, bit-identical to the
    reference's step. State arrays are in original order."""

    def __init__(self, particles: Particles, params: DfsphParams | None = None,
                 config: WcsphConfig | None = None):
        L = load_library()
        self._w = None
        params = params if params is not None else DfsphParams()
        h = C.c_void_p()
        cfg = config._to_c() if config is not None else None
        _ok(L.pe_fluid_dfsph_create(particles._p, C.byref(params._to_c()),
                                    C.byref(cfg) if cfg is not None else None, C.byref(h)), "dfsph_create")
        self._w = h
        self.n = len(particles)
        self._kinds = particles.arrays()["kind"].copy()
        self.dim, self.mass, self.h, self.rest_density = particles.dim, particles.mass, particles.h, particles.rest_density

    def close(self):
        if getattr(self, "_w", None) and _lib is not None:
            _lib.pe_fluid_dfsph_destroy(self._w)
        self._w = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, dt: float):
        _ok(_lib.pe_fluid_dfsph_step(self._w, float(dt)), "dfsph_step")

    def run(self, dt: float, steps: int):
        _ok(_lib.pe_fluid_dfsph_run(self._w, float(dt), int(steps)), "dfsph_run")

    def step_adaptive(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_dfsph_step_adaptive(self._w, C.byref(d)), "dfsph_step_adaptive")
        return d.value

    def suggest_dt(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_dfsph_suggest_dt(self._w, C.byref(d)), "dfsph_suggest_dt")
        return d.value

    def rebuild_neighbours(self):
        _ok(_lib.pe_fluid_dfsph_rebuild_neighbours(self._w), "dfsph_rebuild_neighbours")

    def compute_density(self):
        _ok(_lib.pe_fluid_dfsph_compute_density(self._w), "dfsph_compute_density")

    def compute_alpha(self):
        _ok(_lib.pe_fluid_dfsph_compute_alpha(self._w), "dfsph_compute_alpha")

    @property
    def t(self) -> float:
        t = C.c_double()
        _ok(_lib.pe_fluid_dfsph_get_time(self._w, C.byref(t)), "dfsph_time")
        return t.value

    @property
    def last_dt(self) -> float:
        t = C.c_double()
        _ok(_lib.pe_fluid_dfsph_get_last_dt(self._w, C.byref(t)), "dfsph_last_dt")
        return t.value

    @property
    def params(self) -> DfsphParams:
        c = _DfsphParams()
        _ok(_lib.pe_fluid_dfsph_get_params(self._w, C.byref(c)), "dfsph_params")
        p = DfsphParams()
        p._load(c)
        return p

    @params.setter
    def params(self, p: DfsphParams):
        _ok(_lib.pe_fluid_dfsph_set_params(self._w, C.byref(p._to_c())), "dfsph_set_params")

    def _get(self, fn, shape, what):
        out = np.empty(shape)
        _ok(fn(self._w, _ptr(out), self.n), what)
        return out

    def positions(self):
        return self._get(_lib.pe_fluid_dfsph_get_positions, (self.n, 3), "dfsph_positions")

    def velocities(self):
        return self._get(_lib.pe_fluid_dfsph_get_velocities, (self.n, 3), "dfsph_velocities")

    def densities(self):
        return self._get(_lib.pe_fluid_dfsph_get_densities, (self.n,), "dfsph_densities")

    def pressures(self):
        return self._get(_lib.pe_fluid_dfsph_get_pressures, (self.n,), "dfsph_pressures")

    def boundary_forces(self):
        return self._get(_lib.pe_fluid_dfsph_get_boundary_forces, (self.n, 3), "dfsph_boundary_forces")

    def alphas(self):
        return self._get(_lib.pe_fluid_dfsph_get_alphas, (self.n,), "dfsph_alphas")

    def set_positions(self, x):
        x = _arr(x, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_dfsph_set_positions(self._w, _ptr(x), self.n), "dfsph_set_positions")

    def set_velocities(self, v):
        v = _arr(v, np.float64, (self.n, 3))
        _ok(_lib.pe_fluid_dfsph_set_velocities(self._w, _ptr(v), self.n), "dfsph_set_velocities")

    def last_iterations(self):
        out = np.zeros(2, np.uint64)
        _ok(_lib.pe_fluid_dfsph_last_iterations(self._w, _ptr(out)), "dfsph_iterations")
        return int(out[0]), int(out[1])

    def mean_density_error(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_dfsph_mean_density_error(self._w, C.byref(d)), "dfsph_mean_density_error")
        return d.value

    def v_max(self) -> float:
        d = C.c_double()
        _ok(_lib.pe_fluid_dfsph_v_max(self._w, C.byref(d)), "dfsph_v_max")
        return d.value

    def status(self) -> int:
        s = C.c_uint32()
        _ok(_lib.pe_fluid_dfsph_status(self._w, C.byref(s)), "dfsph_status")
        return s.value

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) all of this world's kernels run on."""
        h = C.c_void_p()
        _ok(_lib.pe_fluid_dfsph_stream(self._w, C.byref(h)), "stream")
        return h.value or 0

    def kernel_launches(self, reset=False) -> int:
        c = C.c_uint64()
        _ok(_lib.pe_fluid_dfsph_kernel_launches(self._w, C.byref(c), 1 if reset else 0), "dfsph_launches")
        return c.value

    def kinds(self):
        return self._kinds

    def hash64(self) -> int:
        return particles_hash64(self.positions(), self.velocities(), self._kinds)


# --------------------------------------------------------------------------
# Fluid side of the WCSPH-rigid coupling (crates/pe-fluid/src/coupling.rs)
# --------------------------------------------------------------------------
class FluidRigidCoupler:
    """The rigid samples of a world (`FluidRigidCoupler`, coupling.rs:42-51).

    Sample k is world particle `particle[k]`, an oriented boundary sample on
    body `body[k]` at body-frame offset `local[k]` with body-frame normal
    `local_n[k]`. The rigid bodies stay with the caller: each coupled step
    (`CoupledWcsphWorld::step`, coupling.rs:853-866) is `sync_from_rigid`,
    `world.step(dt)`, `reduce_with_state`, then the caller's rigid step.
    """

    def __init__(self, world: "WcsphWorld", n_bodies: int, body, local, local_n, particle):
        L = load_library()
        body = _arr(body, np.int64, (-1,))
        ns = body.shape[0]
        self._keep = (_arr(local, np.float64, (ns, 3)), _arr(local_n, np.float64, (ns, 3)),
                      _arr(particle, np.int64, (ns,)))
        self.n_bodies, self.n_samples, self.world = int(n_bodies), ns, world
        self.body = body
        h = C.c_void_p()
        _ok(L.pe_fluid_coupler_create(world._w, self.n_bodies, ns, _ptr(body), _ptr(self._keep[0]),
                                      _ptr(self._keep[1]), _ptr(self._keep[2]), C.byref(h)), "coupler_create")
        self._c = h

    def close(self):
        if getattr(self, "_c", None) and _lib is not None:
            _lib.pe_fluid_coupler_destroy(self._c)
        self._c = None

    def __del__(self):
        self.close()

    def sync_from_rigid(self, x, q, v, omega):
        """Sample positions, velocities and normals from per-body centre of mass
        `x`, orientation `q` (w, x, y, z), velocity `v` and world-frame angular
        velocity `omega` (`sync_from_rigid`, coupling.rs:289-306)."""
        nb = self.n_bodies
        a = [_arr(x, np.float64, (nb, 3)), _arr(q, np.float64, (nb, 4)), _arr(v, np.float64, (nb, 3)),
             _arr(omega, np.float64, (nb, 3))]
        _ok(_lib.pe_fluid_coupler_sync(self._c, *[_ptr(t) for t in a]), "coupler_sync")

    def reduce_with_state(self, x):
        """Per-body (force, torque) of the samples' boundary reactions about the
        centres of mass `x` (`reduce_with_state`, coupling.rs:308-330)."""
        nb = self.n_bodies
        xb = _arr(x, np.float64, (nb, 3))
        f = np.empty((nb, 3))
        t = np.empty((nb, 3))
        _ok(_lib.pe_fluid_coupler_reduce(self._c, _ptr(xb), _ptr(f), _ptr(t)), "coupler_reduce")
        return f, t


def kernel_w(kernel, r, h, dim):
    return load_library().pe_fluid_kernel_w(int(kernel), float(r), float(h), int(dim))


def grad_w(kernel, rij, h, dim):
    out = (C.c_double * 3)()
    _ok(load_library().pe_fluid_grad_w(int(kernel), _v3(rij), float(h), int(dim), out), "grad_w")
    return np.array(out[:])


def tait_pressure(rest_density, sound_speed, gamma, density):
    return load_library().pe_fluid_tait_pressure(float(rest_density), float(sound_speed), float(gamma),
                                                 float(density))


def pi_ij(alpha, beta, eps, h, sound_speed, xi, xj, vi, vj, rho_i, rho_j):
    return load_library().pe_fluid_pi_ij(float(alpha), float(beta), float(eps), float(h),
                                         float(sound_speed), _v3(xi), _v3(xj), _v3(vi), _v3(vj),
                                         float(rho_i), float(rho_j))


def suggested_dt(h, sound_speed, v_max, a_max, lambda_v=0.25, lambda_f=0.25):
    return load_library().pe_fluid_suggested_dt(float(h), float(sound_speed), float(v_max),
                                                float(a_max), float(lambda_v), float(lambda_f))


# --------------------------------------------------------------------------
# Functions kept from the reference module (python/src/fluid.rs:288-305).
# The analytic ones restate crates/pe-fluid/src/oracles.rs and coupling.rs;
# the canonical PBF and DFSPH tanks step on the GPU solvers of this package.
# The coupled-tank hash needs the rigid-body world (pe-rigid), which this
# package does not contain, so it raises NotImplementedError with that reason.
# --------------------------------------------------------------------------
_NOT_ON_PATH = ("this package provides the fluid side only; the {} is not included")


FLUID_HASH_STEPS, FLUID_HASH_DT = 40, 1.0 / 120.0


def fluid_hash_world(config: WcsphConfig | None = None) -> PbfWorld:
    """The canonical PBF tank (scenarios.rs:28-61): a 4x4x4 block (dx 0.05,
    h 2 dx) in a 0.4 x 0.4 x 0.45 shell; 4 iterations, no tensile correction,
    no vorticity."""
    dx, rho0 = 0.05, 1000.0
    parts = Particles(DIM_3, rho0, mass_from_spacing(rho0, dx, DIM_3), 2.0 * dx)
    parts.fill_box((0.1, 0.1, 0.1), 4, 4, 4, dx)
    parts.fill_box_boundary((0.0, 0.0, 0.0), (0.4, 0.4, 0.45), dx, 1)
    params = PbfParams(gravity=(0.0, 0.0, -STANDARD_GRAVITY), iterations=4, art_pressure_k=0.0,
                       vorticity_eps=0.0)
    return PbfWorld(parts, params, config)


def canonical_fluid_hash() -> int:
    """`fluid_tank_hash` (scenarios.rs:64-71): the canonical PBF tank after 40
    steps of 1/120 s, hashed; stepped on the GPU."""
    w = fluid_hash_world()
    w.run(FLUID_HASH_DT, FLUID_HASH_STEPS)
    h = w.hash64()
    w.close()
    return h


DFSPH_HASH_STEPS, DFSPH_HASH_DT = 40, 1.0 / 120.0


def dfsph_hash_world(config: WcsphConfig | None = None) -> DfsphWorld:
    """The canonical DFSPH tank (scenarios.rs:74-116): the PBF tank's geometry
    with the calibrated mass and recomputed Akinci volumes; 8 + 8 solver
    iterations at 1% tolerance, XSPH 0.05, warm start, fixed dt."""
    dx, rho0 = 0.05, 1000.0
    h = 2.0 * dx
    parts = Particles(DIM_3, rho0, mass_calibrated_to_rest(rho0, dx, h, DIM_3, CUBIC_SPLINE), h)
    parts.fill_box((0.1, 0.1, 0.1), 4, 4, 4, dx)
    parts.fill_box_boundary((0.0, 0.0, 0.0), (0.4, 0.4, 0.45), dx, 1)
    parts.recomputed_akinci_psi(CUBIC_SPLINE)
    params = DfsphParams(gravity=(0.0, 0.0, -STANDARD_GRAVITY), particle_diameter=dx, density_error_tol=0.01,
                         divergence_error_tol=0.01, max_density_iters=8, max_divergence_iters=8,
                         xsph_epsilon=0.05, adaptive_dt=False, warm_start=True)
    return DfsphWorld(parts, params, config)


def canonical_dfsph_hash() -> int:
    """`dfsph_tank_hash` (scenarios.rs:119-125): the canonical DFSPH tank after
    40 steps of 1/120 s, hashed; stepped on the GPU."""
    w = dfsph_hash_world()
    w.run(DFSPH_HASH_DT, DFSPH_HASH_STEPS)
    h = w.hash64()
    w.close()
    return h


def canonical_coupling_hash() -> int:
    raise NotImplementedError(_NOT_ON_PATH.format("rigid-body world of the coupled tank"))


def fluid_ritter_front(g: float, h0: float, t: float) -> float:
    """oracles.rs:43 `x_f = 2 sqrt(g h0) t`."""
    return 2.0 * math.sqrt(g * h0) * t


def fluid_ritter_height(g: float, h0: float, x: float, t: float) -> float:
    """oracles.rs:48 Ritter height."""
    if t <= 0.0:
        return h0 if x < 0.0 else 0.0
    c0 = math.sqrt(g * h0)
    x_l = -c0 * t
    x_f = 2.0 * c0 * t
    if x <= x_l:
        return h0
    if x >= x_f:
        return 0.0
    c = (2.0 * c0 - x / t) / 3.0
    return (c * c) / g


def fluid_hydrostatic_pressure(rho: float, g: float, depth: float) -> float:
    """oracles.rs:82 `p = rho g h`."""
    return rho * g * depth


def fluid_archimedes_box_draft(rho_body: float, rho_fluid: float, height: float) -> float:
    """coupling.rs:413."""
    return (rho_body / max(rho_fluid, 1e-12)) * height


def fluid_heave_period_analytic(mass: float, rho_fluid: float, a_wp: float, g: float) -> float:
    """coupling.rs:419."""
    return 2.0 * math.pi * math.sqrt(mass / max(rho_fluid * g * a_wp, 1e-12))


def fluid_barge_heave_added_mass_2d(rho_fluid: float, beam: float) -> float:
    """coupling.rs:426."""
    return rho_fluid * math.pi * beam * beam / 8.0


def fluid_heave_period_with_added_mass(mass: float, m_a: float, rho_fluid: float, a_wp: float,
                                       g: float) -> float:
    """coupling.rs:432."""
    return 2.0 * math.pi * math.sqrt((mass + m_a) / max(rho_fluid * g * a_wp, 1e-12))


def fluid_sphere_freefall_accel_added_mass(rho_s: float, rho_f: float, g: float) -> float:
    """coupling.rs:439."""
    return g * (rho_s - rho_f) / max(rho_s + 0.5 * rho_f, 1e-12)


def _parse_dim(dim) -> int:
    d = str(dim).lower().replace("d", "")
    if d not in ("2", "3"):
        raise ValueError(f"dim must be '2' or '3', got {dim!r}")
    return int(d)


def _mean_density_error_diag(rho, kind, rest_density) -> float:
    """diagnostics.rs:74-88, summed in index order."""
    s, n = 0.0, 0
    for r, k in zip(np.asarray(rho).tolist(), np.asarray(kind).tolist()):
        if k == FLUID:
            s += abs(r - rest_density) / rest_density
            n += 1
    return 0.0 if n == 0 else s / n


def _tank_parts(dim, n_side, dx, h, mass, rho0):
    parts = Particles(dim, rho0, mass, h)
    nz = 1 if dim == DIM_2 else n_side
    parts.fill_box((0.1, 0.1, 0.1), n_side, n_side, nz, dx)
    zmax = 0.0 if dim == DIM_2 else 0.1 + n_side * dx + 0.05
    ext = 0.1 + n_side * dx + 0.1
    parts.fill_box_boundary((0.0, 0.0, 0.0), (ext, ext, max(zmax, 0.45)), dx, 1)
    return parts


def fluid_pbf_tank_demo(n_side=4, steps=40, dt=1.0 / 120.0, dim="3"):
    """Small PBF tank (python/src/fluid.rs:188-243): returns (fluid positions
    [N, 3], fluid densities [N], mean density error)."""
    d = _parse_dim(dim)
    dx, rho0 = 0.05, 1000.0
    h = 2.2 * dx
    parts = _tank_parts(d, int(n_side), dx, h, mass_from_spacing(rho0, dx, d), rho0)
    g = (0.0, -STANDARD_GRAVITY, 0.0) if d == DIM_2 else (0.0, 0.0, -STANDARD_GRAVITY)
    w = PbfWorld(parts, PbfParams(gravity=g, iterations=2, art_pressure_k=0.0))
    w.run(float(dt), int(steps))
    fluid = w.kinds() == FLUID
    x, rho = w.positions(), w.densities()
    err = _mean_density_error_diag(rho, w.kinds(), rho0)
    w.close()
    return x[fluid], rho[fluid], err


def fluid_dfsph_tank_demo(n_side=4, steps=40, dt=1.0 / 120.0, dim="3"):
    """Small DFSPH tank (python/src/fluid.rs:100-184): returns (fluid positions
    [N, 3], fluid densities [N], mean density error)."""
    d = _parse_dim(dim)
    dx, rho0 = 0.05, 1000.0
    h = 2.0 * dx
    parts = _tank_parts(d, int(n_side), dx, h, mass_calibrated_to_rest(rho0, dx, h, d, CUBIC_SPLINE), rho0)
    parts.recomputed_akinci_psi(CUBIC_SPLINE)
    g = (0.0, -STANDARD_GRAVITY, 0.0) if d == DIM_2 else (0.0, 0.0, -STANDARD_GRAVITY)
    w = DfsphWorld(parts, DfsphParams(gravity=g, particle_diameter=dx, adaptive_dt=False, max_density_iters=4,
                                      max_divergence_iters=4, density_error_tol=0.01, divergence_error_tol=0.01))
    w.run(float(dt), int(steps))
    fluid = w.kinds() == FLUID
    x, rho = w.positions(), w.densities()
    err = _mean_density_error_diag(rho, w.kinds(), rho0)
    w.close()
    return x[fluid], rho[fluid], err


def fluid_poly6_w0(h: float) -> float:
    """kernels.rs:161-175: poly6 W(0, h) in 3-D = 315 / (64 pi h^9) * (h^2)^3."""
    a = 315.0 / (64.0 * math.pi * math.pow(h, 9.0))
    t = h * h - 0.0 * 0.0
    return a * t * t * t


def fluid_canonical_mass() -> float:
    """Total fluid mass of the canonical hash tank (scenarios.rs:28-61): 4x4x4
    fluid at dx = 0.05, mass_from_spacing(1000, 0.05, D3) each."""
    return mass_from_spacing(1000.0, 0.05, 3) * 64.0


def _kinetic_energy_diag(v, kind, mass) -> float:
    """diagnostics.rs:52-60: sum of 0.5 m |v|^2 over fluid particles in index
    order (|v|^2 = x*x + y*y + z*z, pe-math vec3.rs)."""
    ke = 0.0
    for (vx, vy, vz), k in zip(np.asarray(v).tolist(), np.asarray(kind).tolist()):
        if k == FLUID:
            ke += 0.5 * mass * (vx * vx + vy * vy + vz * vz)
    return ke


def fluid_canonical_ke_after_hash_steps() -> float:
    """python/src/fluid.rs:277-285: kinetic energy of the canonical PBF tank
    after FLUID_HASH_STEPS steps of FLUID_HASH_DT, stepped on the GPU."""
    w = fluid_hash_world()
    w.run(FLUID_HASH_DT, FLUID_HASH_STEPS)
    ke = _kinetic_energy_diag(w.velocities(), w.kinds(), w.mass)
    w.close()
    return ke
