"""TEST INFRASTRUCTURE — ctypes wrapper around the CPU oracle (`liboracle_wcsph.so`).

The oracle is an order-exact C++ restatement of eranyid/physics-engine's
`pe-fluid` WCSPH path (`crates/pe-fluid/src/wcsph.rs:83-347`, `grid.rs:62-157`,
`kernels.rs:32-116`, `eos.rs:59-80`, `viscosity.rs:30-100`,
`particles.rs:90-347`). Only `tests/`, `__graft_entry__.smoke()` and the CPU
baseline of `bench.py` use it, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_wcsph.so")
_lib = None

FLUID, BOUNDARY = 0, 1
CUBIC, WENDLAND, POLY6, SPIKY = 0, 1, 2, 3


class OParams(C.Structure):
    """Mirror of `WParams` in wcsph_oracle.cpp (fields of `WcsphParams`, wcsph.rs:24)."""

    _fields_ = [
        ("kernel", C.c_int32),
        ("eos_rest_density", C.c_double),
        ("eos_sound_speed", C.c_double),
        ("eos_gamma", C.c_double),
        ("visc_alpha", C.c_double),
        ("visc_beta", C.c_double),
        ("visc_eps", C.c_double),
        ("xsph_epsilon", C.c_double),
        ("gravity", C.c_double * 3),
        ("adapt_sound_speed", C.c_int32),
        ("materialize_neigh_lists", C.c_int32),
        ("st_model", C.c_int32),
        ("st_sigma", C.c_double),
        ("st_colour_gamma", C.c_double),
    ]



class PParams(C.Structure):
    """Mirror of `PParams` in wcsph_oracle.cpp (fields of `PbfParams`, pbf.rs:26-53)."""

    _fields_ = [
        ("density_kernel", C.c_int32),
        ("grad_kernel", C.c_int32),
        ("iterations", C.c_int64),
        ("epsilon_lambda", C.c_double),
        ("art_pressure_k", C.c_double),
        ("art_pressure_n", C.c_double),
        ("art_pressure_dq_over_h", C.c_double),
        ("viscosity_eps", C.c_double),
        ("vorticity_eps", C.c_double),
        ("gravity", C.c_double * 3),
        ("reuse_neighbours", C.c_int32),
    ]


def pbf_default_params() -> PParams:
    """`PbfParams::default` (pbf.rs:55-74)."""
    p = PParams()
    p.density_kernel, p.grad_kernel, p.iterations = POLY6, SPIKY, 5
    p.epsilon_lambda, p.art_pressure_k, p.art_pressure_n, p.art_pressure_dq_over_h = 0.01, 0.01, 4.0, 0.25
    p.viscosity_eps, p.vorticity_eps = 0.01, 0.0
    p.gravity[:] = (0.0, 0.0, -9.80665)
    p.reuse_neighbours = 1
    return p


class DParams(C.Structure):
    """Mirror of `DParams` in wcsph_oracle.cpp (fields of `DfsphParams`,
    dfsph.rs:33-80; the four free-slip planes as flag + value)."""

    _fields_ = [
        ("kernel", C.c_int32),
        ("max_density_iters", C.c_int64),
        ("max_divergence_iters", C.c_int64),
        ("density_error_tol", C.c_double),
        ("divergence_error_tol", C.c_double),
        ("gravity", C.c_double * 3),
        ("xsph_epsilon", C.c_double),
        ("particle_diameter", C.c_double),
        ("cfl_lambda", C.c_double),
        ("adaptive_dt", C.c_int32),
        ("warm_start", C.c_int32),
        ("has_slip", C.c_int32 * 4),
        ("slip", C.c_double * 4),
        ("solver_omega", C.c_double),
        ("max_velocity_correction", C.c_double),
    ]


def dfsph_default_params() -> DParams:
    """`DfsphParams::default` (dfsph.rs:82-104)."""
    p = DParams()
    p.kernel, p.max_density_iters, p.max_divergence_iters = CUBIC, 50, 50
    p.density_error_tol, p.divergence_error_tol = 0.001, 0.001
    p.gravity[:] = (0.0, 0.0, -9.80665)
    p.xsph_epsilon, p.particle_diameter, p.cfl_lambda = 0.05, 0.0, 0.4
    p.adaptive_dt, p.warm_start = 1, 1
    p.solver_omega, p.max_velocity_correction = 1.0, 0.0
    return p

def water_params(rest_density, sound_speed, gravity, materialize=True) -> OParams:
    """`WcsphParams::water` defaults (wcsph.rs:43-53, viscosity.rs:39,82)."""
    p = OParams()
    p.kernel = CUBIC
    p.eos_rest_density = rest_density
    p.eos_sound_speed = sound_speed
    p.eos_gamma = 7.0
    p.visc_alpha, p.visc_beta, p.visc_eps = 0.01, 0.0, 0.01
    p.xsph_epsilon = 0.25
    p.gravity[:] = list(gravity)
    p.adapt_sound_speed = 1
    p.materialize_neigh_lists = 1 if materialize else 0
    return p


def build() -> str:
    """Compile the oracle library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, d, i32, i64, u64 = C.c_void_p, C.c_double, C.c_int32, C.c_long, C.c_uint64
        dp = C.POINTER(C.c_double)
        sig = {
            "oscene_new": (vp, [C.c_int, d, d, d]),
            "oscene_free": (None, [vp]),
            "oscene_len": (i64, [vp]),
            "oscene_push_fluid": (None, [vp, dp, dp]),
            "oscene_push_boundary": (None, [vp, dp, d, dp]),
            "oscene_fill_box": (None, [vp, dp, i64, i64, i64, d, dp]),
            "oscene_fill_box_boundary": (None, [vp, dp, dp, d, i64]),
            "oscene_recompute_psi": (None, [vp, C.c_int]),
            "oscene_jitter_fluid": (None, [vp, u64, d]),
            "oscene_export": (None, [vp, vp, vp, vp, vp, vp]),
            "o_mass_from_spacing": (d, [d, d, C.c_int]),
            "o_mass_calibrated_to_rest": (d, [d, d, d, C.c_int, C.c_int]),
            "o_kernel_w": (d, [C.c_int, d, d, C.c_int]),
            "o_grad_w": (None, [C.c_int, dp, d, C.c_int, dp]),
            "o_pow": (d, [d, d]),
            "o_pi_ij": (d, [d, d, d, d, d, dp, dp, dp, dp, d, d]),
            "o_tait_pressure": (d, [d, d, d, d]),
            "o_floor_i32": (i32, [d]),
            "o_xoshiro_first": (u64, [u64, i64, vp]),
            "ow_create": (vp, [vp, C.POINTER(OParams)]),
            "ow_free": (None, [vp]),
            "ow_len": (i64, [vp]),
            "ow_step": (None, [vp, d]),
            "ow_run": (None, [vp, d, i64]),
            "ow_rebuild_grid": (None, [vp]),
            "ow_compute_density": (None, [vp]),
            "ow_compute_pressure": (None, [vp]),
            "ow_compute_forces": (None, [vp]),
            "ow_apply_xsph": (None, [vp]),
            "ow_time": (d, [vp]),
            "ow_sound_speed": (d, [vp]),
            "ow_a_max": (d, [vp]),
            "ow_v_max": (d, [vp]),
            "ow_hash": (u64, [vp]),
            "ow_set_threads": (None, [vp, C.c_int]),
            "ow_set_pow_perturbation": (None, [vp, d, u64]),
            "ow_get_x": (None, [vp, vp]),
            "ow_get_v": (None, [vp, vp]),
            "ow_get_a": (None, [vp, vp]),
            "ow_get_boundary_force": (None, [vp, vp]),
            "ow_get_rho": (None, [vp, vp]),
            "ow_get_p": (None, [vp, vp]),
            "ow_set_x": (None, [vp, vp]),
            "ow_set_v": (None, [vp, vp]),
            "ow_set_rho": (None, [vp, vp]),
            "ow_set_p": (None, [vp, vp]),
            "ow_grid_occupied_count": (i64, [vp]),
            "ow_get_grid": (None, [vp, vp, vp, vp, vp]),
            "ow_neighbour_counts": (None, [vp, vp, vp]),
            "o_total_mass": (d, [vp]),
            "o_linear_momentum": (None, [vp, dp]),
            "o_kinetic_energy": (d, [vp]),
            "o_gravitational_potential": (d, [vp, d]),
            "o_mean_density_error": (d, [vp]),
            "o_max_density_error": (d, [vp]),
            "o_suggested_dt": (d, [d, d, d, d, d, d]),
            "opbf_create": (vp, [vp, C.POINTER(PParams)]),
            "opbf_free": (None, [vp]),
            "opbf_run": (None, [vp, d, i64]),
            "opbf_hash": (u64, [vp]),
            "opbf_time": (d, [vp]),
            "opbf_get_x": (None, [vp, vp]),
            "opbf_get_v": (None, [vp, vp]),
            "opbf_get_rho": (None, [vp, vp]),
            "opbf_get_lambda": (None, [vp, vp]),
            "odfsph_create": (vp, [vp, C.POINTER(DParams)]),
            "odfsph_free": (None, [vp]),
            "odfsph_run": (None, [vp, d, i64]),
            "odfsph_step_adaptive": (d, [vp]),
            "odfsph_hash": (u64, [vp]),
            "odfsph_time": (d, [vp]),
            "odfsph_iters": (None, [vp, vp]),
            "odfsph_get_x": (None, [vp, vp]),
            "odfsph_get_v": (None, [vp, vp]),
            "odfsph_get_boundary_force": (None, [vp, vp]),
            "odfsph_get_rho": (None, [vp, vp]),
            "odfsph_get_p": (None, [vp, vp]),
            "odfsph_get_alpha": (None, [vp, vp]),
            "o_coupler_sync": (None, [vp, u64, vp, vp, vp, vp, vp, vp, vp, vp]),
            "o_coupler_reduce": (None, [vp, u64, vp, vp, u64, vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d3(v):
    return (C.c_double * 3)(*[float(t) for t in v])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Scene:
    """Particle builder (`Particles` + scene builders, particles.rs:20-347)."""

    def __init__(self, dim: int, rest_density: float, mass: float, h: float):
        self.dim, self.rest_density, self.mass, self.h = dim, rest_density, mass, h
        self._s = lib().oscene_new(dim, rest_density, mass, h)

    def __del__(self):
        if getattr(self, "_s", None):
            lib().oscene_free(self._s)
            self._s = None

    def __len__(self):
        return lib().oscene_len(self._s)

    def push_fluid(self, x, v=(0, 0, 0)):
        lib().oscene_push_fluid(self._s, _d3(x), _d3(v))

    def push_boundary(self, x, psi, n_out=None):
        lib().oscene_push_boundary(self._s, _d3(x), psi, _d3(n_out) if n_out is not None else None)

    def fill_box(self, origin, nx, ny, nz, dx, v0=(0, 0, 0)):
        lib().oscene_fill_box(self._s, _d3(origin), nx, ny, nz, dx, _d3(v0))

    def fill_box_boundary(self, mn, mx, dx, layers=1):
        lib().oscene_fill_box_boundary(self._s, _d3(mn), _d3(mx), dx, layers)

    def recompute_psi(self, kernel=CUBIC):
        lib().oscene_recompute_psi(self._s, kernel)

    def jitter_fluid(self, seed: int, amp: float):
        lib().oscene_jitter_fluid(self._s, seed, amp)

    def arrays(self):
        n = len(self)
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); k = np.zeros(n, np.uint8)
        psi = np.zeros(n); nout = np.zeros((n, 3))
        lib().oscene_export(self._s, _ptr(x), _ptr(v), _ptr(k), _ptr(psi), _ptr(nout))
        return dict(x=x, v=v, kind=k, psi=psi, n_out=nout)


class World:
    """`WcsphWorld` restated (wcsph.rs:58-370)."""

    def __init__(self, scene: Scene, params: OParams):
        self.scene_meta = (scene.dim, scene.rest_density, scene.mass, scene.h)
        self.params = params
        self._w = lib().ow_create(scene._s, C.byref(params))
        self.n = lib().ow_len(self._w)

    def __del__(self):
        if getattr(self, "_w", None):
            lib().ow_free(self._w)
            self._w = None

    def step(self, dt):
        lib().ow_step(self._w, dt)

    def run(self, dt, steps):
        lib().ow_run(self._w, dt, steps)

    def rebuild_grid(self):
        lib().ow_rebuild_grid(self._w)

    def compute_density(self):
        lib().ow_compute_density(self._w)

    def compute_pressure(self):
        lib().ow_compute_pressure(self._w)

    def compute_forces(self):
        lib().ow_compute_forces(self._w)

    def apply_xsph(self):
        lib().ow_apply_xsph(self._w)

    @property
    def t(self):
        return lib().ow_time(self._w)

    @property
    def sound_speed(self):
        return lib().ow_sound_speed(self._w)

    def _vec(self, fn):
        out = np.zeros((self.n, 3))
        fn(self._w, _ptr(out))
        return out

    def _scal(self, fn):
        out = np.zeros(self.n)
        fn(self._w, _ptr(out))
        return out

    def x(self):
        return self._vec(lib().ow_get_x)

    def v(self):
        return self._vec(lib().ow_get_v)

    def a(self):
        return self._vec(lib().ow_get_a)

    def boundary_force(self):
        return self._vec(lib().ow_get_boundary_force)

    def rho(self):
        return self._scal(lib().ow_get_rho)

    def p(self):
        return self._scal(lib().ow_get_p)

    def set_x(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().ow_set_x(self._w, _ptr(x))

    def set_v(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().ow_set_v(self._w, _ptr(v))

    def set_rho(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        lib().ow_set_rho(self._w, _ptr(r))

    def set_p(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        lib().ow_set_p(self._w, _ptr(p))

    def grid(self):
        m = lib().ow_grid_occupied_count(self._w)
        keys = np.zeros((self.n, 3), np.int32)
        order = np.zeros(self.n, np.int64)
        occ = np.zeros((m, 3), np.int32)
        rng = np.zeros((m, 2), np.int64)
        lib().ow_get_grid(self._w, _ptr(keys), _ptr(order), _ptr(occ), _ptr(rng))
        return dict(keys=keys, order=order, occupied=occ, ranges=rng)

    def neighbour_counts(self):
        cand = np.zeros(self.n, np.int32)
        sup = np.zeros(self.n, np.int32)
        lib().ow_neighbour_counts(self._w, _ptr(cand), _ptr(sup))
        return cand, sup

    def hash64(self):
        return lib().ow_hash(self._w)

    def set_threads(self, threads: int):
        """Parallel oracle: OpenMP over particles, forces as the bit-identical
        gather (same results as one thread)."""
        lib().ow_set_threads(self._w, int(threads))

    def set_pow_perturbation(self, rate: float, seed: int):
        """Sensitivity hook: each fluid particle's Tait power moves one ulp
        with probability `rate` per pressure pass (seeded)."""
        lib().ow_set_pow_perturbation(self._w, float(rate), int(seed))

    def v_max(self):
        return lib().ow_v_max(self._w)

    def a_max(self):
        return lib().ow_a_max(self._w)

    def total_mass(self):
        return lib().o_total_mass(self._w)

    def linear_momentum(self):
        out = (C.c_double * 3)()
        lib().o_linear_momentum(self._w, out)
        return np.array(out[:])

    def kinetic_energy(self):
        return lib().o_kinetic_energy(self._w)

    def gravitational_potential(self, g):
        return lib().o_gravitational_potential(self._w, g)

    def mean_density_error(self):
        return lib().o_mean_density_error(self._w)

    def max_density_error(self):
        return lib().o_max_density_error(self._w)




class PbfWorld:
    """`PbfWorld` restated (pbf.rs:77-459)."""

    def __init__(self, scene: Scene, params: PParams):
        self.params = params
        self._w = lib().opbf_create(scene._s, C.byref(params))
        self.n = len(scene)

    def __del__(self):
        if getattr(self, "_w", None):
            lib().opbf_free(self._w)
            self._w = None

    def run(self, dt, steps):
        lib().opbf_run(self._w, dt, steps)

    def step(self, dt):
        self.run(dt, 1)

    @property
    def t(self):
        return lib().opbf_time(self._w)

    def hash64(self):
        return lib().opbf_hash(self._w)

    def _get(self, fn, shape):
        out = np.empty(shape)
        fn(self._w, _ptr(out))
        return out

    def x(self):
        return self._get(lib().opbf_get_x, (self.n, 3))

    def v(self):
        return self._get(lib().opbf_get_v, (self.n, 3))

    def rho(self):
        return self._get(lib().opbf_get_rho, (self.n,))

    def lam(self):
        return self._get(lib().opbf_get_lambda, (self.n,))


def pbf_hash_world():
    """The reference's canonical PBF tank (scenarios.rs:28-61): a 4x4x4 block,
    dx 0.05, h 2 dx, in a 0.4 x 0.4 x 0.45 shell; 4 iterations, no tensile
    correction, no vorticity."""
    dx, rho0 = 0.05, 1000.0
    s = Scene(3, rho0, mass_from_spacing(rho0, dx, 3), 2.0 * dx)
    s.fill_box((0.1, 0.1, 0.1), 4, 4, 4, dx)
    s.fill_box_boundary((0.0, 0.0, 0.0), (0.4, 0.4, 0.45), dx, 1)
    p = pbf_default_params()
    p.gravity[:] = (0.0, 0.0, -9.80665)
    p.iterations, p.art_pressure_k, p.vorticity_eps = 4, 0.0, 0.0
    return PbfWorld(s, p)


class DfsphWorld:
    """`DfsphWorld` restated (dfsph.rs:107-800)."""

    def __init__(self, scene: Scene, params: DParams):
        self.params = params
        self._w = lib().odfsph_create(scene._s, C.byref(params))
        self.n = len(scene)

    def __del__(self):
        if getattr(self, "_w", None):
            lib().odfsph_free(self._w)
            self._w = None

    def run(self, dt, steps):
        lib().odfsph_run(self._w, dt, steps)

    def step(self, dt):
        self.run(dt, 1)

    def step_adaptive(self):
        return lib().odfsph_step_adaptive(self._w)

    @property
    def t(self):
        return lib().odfsph_time(self._w)

    def hash64(self):
        return lib().odfsph_hash(self._w)

    def iterations(self):
        out = np.zeros(2, np.int64)
        lib().odfsph_iters(self._w, _ptr(out))
        return int(out[0]), int(out[1])

    def _get(self, fn, shape):
        out = np.empty(shape)
        fn(self._w, _ptr(out))
        return out

    def x(self):
        return self._get(lib().odfsph_get_x, (self.n, 3))

    def v(self):
        return self._get(lib().odfsph_get_v, (self.n, 3))

    def boundary_force(self):
        return self._get(lib().odfsph_get_boundary_force, (self.n, 3))

    def rho(self):
        return self._get(lib().odfsph_get_rho, (self.n,))

    def p(self):
        return self._get(lib().odfsph_get_p, (self.n,))

    def alpha(self):
        return self._get(lib().odfsph_get_alpha, (self.n,))


def dfsph_hash_world():
    """The reference's canonical DFSPH tank (scenarios.rs:76-116): the PBF
    tank's geometry with the calibrated mass and recomputed Akinci volumes."""
    dx, rho0 = 0.05, 1000.0
    h = 2.0 * dx
    s = Scene(3, rho0, mass_calibrated_to_rest(rho0, dx, h, 3, CUBIC), h)
    s.fill_box((0.1, 0.1, 0.1), 4, 4, 4, dx)
    s.fill_box_boundary((0.0, 0.0, 0.0), (0.4, 0.4, 0.45), dx, 1)
    s.recompute_psi(CUBIC)
    p = dfsph_default_params()
    p.particle_diameter = dx
    p.density_error_tol, p.divergence_error_tol = 0.01, 0.01
    p.max_density_iters, p.max_divergence_iters = 8, 8
    p.xsph_epsilon, p.adaptive_dt, p.warm_start = 0.05, 0, 1
    return DfsphWorld(s, p)

class Coupler:
    """`FluidRigidCoupler` restated (coupling.rs:42-51, 289-330): sample k is
    particle `particle[k]` on body `body[k]` with body-frame offset `local[k]`
    and normal `local_n[k]`."""

    def __init__(self, world: World, n_bodies, body, local, local_n, particle):
        self.w, self.nb = world, int(n_bodies)
        self.body = np.ascontiguousarray(body, np.int64).reshape(-1)
        ns = self.body.shape[0]
        self.local = np.ascontiguousarray(local, np.float64).reshape(ns, 3)
        self.local_n = np.ascontiguousarray(local_n, np.float64).reshape(ns, 3)
        self.particle = np.ascontiguousarray(particle, np.int64).reshape(ns)

    def sync_from_rigid(self, x, q, v, omega):
        a = [np.ascontiguousarray(t, np.float64) for t in (x, q, v, omega)]
        lib().o_coupler_sync(self.w._w, self.body.shape[0], _ptr(self.body), _ptr(self.local),
                             _ptr(self.local_n), _ptr(self.particle), *[_ptr(t) for t in a])

    def reduce_with_state(self, x):
        xb = np.ascontiguousarray(x, np.float64)
        f = np.zeros((self.nb, 3))
        t = np.zeros((self.nb, 3))
        lib().o_coupler_reduce(self.w._w, self.body.shape[0], _ptr(self.body), _ptr(self.particle), self.nb,
                               _ptr(xb), _ptr(f), _ptr(t))
        return f, t

def kernel_w(kernel, r, h, dim):
    return lib().o_kernel_w(kernel, r, h, dim)


def grad_w(kernel, rij, h, dim):
    out = (C.c_double * 3)()
    lib().o_grad_w(kernel, _d3(rij), h, dim, out)
    return np.array(out[:])


def opow(x, y):
    return lib().o_pow(x, y)


def pi_ij(alpha, beta, eps, h, c, xi, xj, vi, vj, rho_i, rho_j):
    return lib().o_pi_ij(alpha, beta, eps, h, c, _d3(xi), _d3(xj), _d3(vi), _d3(vj), rho_i, rho_j)


def tait_pressure(rest_density, sound_speed, gamma, density):
    return lib().o_tait_pressure(rest_density, sound_speed, gamma, density)


def floor_i32(x):
    return lib().o_floor_i32(x)


def mass_from_spacing(rho0, dx, dim):
    return lib().o_mass_from_spacing(rho0, dx, dim)


def mass_calibrated_to_rest(rho0, dx, h, dim, kernel=CUBIC):
    return lib().o_mass_calibrated_to_rest(rho0, dx, h, dim, kernel)


def suggested_dt(h, c, vmax, amax, lambda_v=0.25, lambda_f=0.25):
    return lib().o_suggested_dt(h, c, vmax, amax, lambda_v, lambda_f)


def xoshiro_first(seed, n):
    out = np.zeros(n, np.uint64)
    lib().o_xoshiro_first(seed, n, _ptr(out))
    return out


def dam_break_scene(n_side, dx=0.01, box=(1.0, 0.4, 0.6), jitter=1e-4, seed=0x5EED5EED,
                    nxyz=None):
    """Synthetic 3-D dam break: `fill_box(origin=(dx,dx,dx), n, n, n, dx)` with seeded
    xoshiro jitter, then a 1-layer Akinci shell `fill_box_boundary(0, box, dx, 1)`;
    h = 2 dx, rho0 = 1000, mass = `mass_from_spacing` (particles.rs:166)."""
    nx, ny, nz = nxyz if nxyz is not None else (n_side, n_side, n_side)
    h = 2.0 * dx
    mass = mass_from_spacing(1000.0, dx, 3)
    s = Scene(3, 1000.0, mass, h)
    s.fill_box((dx, dx, dx), nx, ny, nz, dx)
    if jitter:
        s.jitter_fluid(seed, jitter)
    s.fill_box_boundary((0.0, 0.0, 0.0), box, dx, 1)
    return s


def dam_break_params(materialize=True, adapt_sound_speed=False):
    """Physics of the synthetic dam break: water defaults with a fixed c0 = 20 m/s
    (adapt_sound_speed off, as the reference's own WCSPH validation runs,
    validation.rs:425) and g = (0, 0, -9.81)."""
    p = water_params(1000.0, 20.0, (0.0, 0.0, -9.81), materialize)
    p.adapt_sound_speed = 1 if adapt_sound_speed else 0
    return p
