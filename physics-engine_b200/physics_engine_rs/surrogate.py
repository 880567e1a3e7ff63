"""The learned surrogate (include/pe_fluid_surrogate.h) through ctypes."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import PeError, _ok, _ptr, load_library

_SIGS = {
    "pe_surrogate_create": (C.c_int, [C.c_uint64, C.c_double, C.POINTER(C.c_void_p)]),
    "pe_surrogate_destroy": (None, [C.c_void_p]),
    "pe_surrogate_num_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "pe_surrogate_param_info": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "pe_surrogate_get_param": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "pe_surrogate_set_param": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "pe_surrogate_get_grad": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "pe_surrogate_set_graph": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "pe_surrogate_set_targets": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pe_surrogate_forward": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pe_surrogate_set_fused_edges": (C.c_int, [C.c_void_p, C.c_int32]),
    "pe_surrogate_train_step": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_float)]),
    "pe_surrogate_get_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pe_surrogate_set_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pe_surrogate_graph_from_world": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "pe_surrogate_targets_from_world": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int32]),
    "pe_fluid_wcsph_tank_range": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_uint32)]),
    "pe_fluid_wcsph_step_learned": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "pe_fluid_wcsph_judge_density": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "pe_fluid_wcsph_run_learned": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_uint64, C.c_uint32,
                                             C.c_double, C.c_void_p]),
}


def _lib():
    L = load_library()
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    return L


class Surrogate:
    """Two-hop message-passing network on the tensor cores (see the header)."""

    def __init__(self, seed: int = 1, r_msg_over_h: float = 1.0):
        self._L = _lib()
        self._s = None
        h = C.c_void_p()
        _ok(self._L.pe_surrogate_create(int(seed), float(r_msg_over_h), C.byref(h)), "surrogate_create")
        self._s = h

    def close(self):
        if self._s:
            self._L.pe_surrogate_destroy(self._s)
        self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params_info(self):
        n = C.c_int32()
        _ok(self._L.pe_surrogate_num_params(self._s, C.byref(n)), "num_params")
        out = []
        for i in range(n.value):
            name = C.create_string_buffer(64)
            K, N, hb = C.c_int32(), C.c_int32(), C.c_int32()
            _ok(self._L.pe_surrogate_param_info(self._s, i, name, 64, C.byref(K), C.byref(N), C.byref(hb)),
                "param_info")
            out.append((name.value.decode(), K.value, N.value, bool(hb.value)))
        return out

    def _io(self, fn, i, K, N, W=None, b=None):
        W = np.zeros((K, N), np.float32) if W is None else np.ascontiguousarray(W, np.float32)
        b = np.zeros(N, np.float32) if b is None else np.ascontiguousarray(b, np.float32)
        _ok(fn(self._s, i, _ptr(W), _ptr(b)), "param")
        return W, b

    def get_params(self, grads: bool = False) -> dict:
        out = {}
        fn = self._L.pe_surrogate_get_grad if grads else self._L.pe_surrogate_get_param
        for i, (name, K, N, hb) in enumerate(self.params_info()):
            W, b = self._io(fn, i, K, N)
            out[name + ".W"] = W
            if hb:
                out[name + ".b"] = b
        return out

    def set_params(self, p: dict):
        for i, (name, K, N, hb) in enumerate(self.params_info()):
            self._io(self._L.pe_surrogate_set_param, i, K, N, p[name + ".W"], p.get(name + ".b"))

    def set_graph(self, f, xe, row, src, fluid):
        f = np.ascontiguousarray(f, np.float32)
        xe = np.ascontiguousarray(xe, np.float32).reshape(-1, 16)
        row = np.ascontiguousarray(row, np.int32)
        src = np.ascontiguousarray(src, np.int32)
        fluid = np.ascontiguousarray(fluid, np.uint8)
        self.n = f.shape[0]
        _ok(self._L.pe_surrogate_set_graph(self._s, self.n, src.shape[0], _ptr(row), _ptr(src), _ptr(f),
                                           _ptr(xe) if xe.size else None, _ptr(fluid)), "set_graph")

    def set_targets(self, t):
        t = np.ascontiguousarray(t, np.float32)
        _ok(self._L.pe_surrogate_set_targets(self._s, _ptr(t)), "set_targets")

    def forward(self):
        y = np.zeros((self.n, 4), np.float32)
        _ok(self._L.pe_surrogate_forward(self._s, _ptr(y)), "forward")
        return y

    def set_fused_edges(self, on: bool):
        """Inference's edge MLP as one fused kernel (True, the default) or as
        the GEMMs and segment sum that training uses (False)."""
        _ok(self._L.pe_surrogate_set_fused_edges(self._s, 1 if on else 0), "set_fused_edges")

    def train_step(self, lr: float = 0.0) -> float:
        loss = C.c_float()
        _ok(self._L.pe_surrogate_train_step(self._s, float(lr), C.byref(loss)), "train_step")
        return loss.value

    # ---- normalisation, persistence ----
    def stats(self):
        m, sd = np.zeros(4, np.float32), np.zeros(4, np.float32)
        _ok(self._L.pe_surrogate_get_stats(self._s, _ptr(m), _ptr(sd)), "get_stats")
        return m, sd

    def set_stats(self, mean, std):
        m, sd = np.ascontiguousarray(mean, np.float32), np.ascontiguousarray(std, np.float32)
        _ok(self._L.pe_surrogate_set_stats(self._s, _ptr(m), _ptr(sd)), "set_stats")

    def save(self, path):
        m, sd = self.stats()
        np.savez(path, __mean=m, __std=sd, **self.get_params())

    def load(self, path):
        d = np.load(path)
        self.set_params({k: d[k] for k in d.files if not k.startswith("__")})
        self.set_stats(d["__mean"], d["__std"])

    # ---- training on a world's plain steps ----
    def graph_from_world(self, world, slot_begin: int, slot_end: int):
        _ok(self._L.pe_surrogate_graph_from_world(self._s, world._w, int(slot_begin), int(slot_end)),
            "graph_from_world")
        self.n = int(slot_end) - int(slot_begin)

    def targets_from_world(self, world, dt: float, update_stats: bool = False):
        _ok(self._L.pe_surrogate_targets_from_world(self._s, world._w, float(dt), 1 if update_stats else 0),
            "targets_from_world")


def tank_range(world, tank: int):
    L = _lib()
    a, b = C.c_uint32(), C.c_uint32()
    _ok(L.pe_fluid_wcsph_tank_range(world._w, int(tank), C.byref(a), C.byref(b)), "tank_range")
    return a.value, b.value


def step_learned(world, surrogate: Surrogate, dt: float):
    _ok(_lib().pe_fluid_wcsph_step_learned(world._w, surrogate._s, float(dt)), "step_learned")


def judge_density(world) -> float:
    e = C.c_double()
    _ok(_lib().pe_fluid_wcsph_judge_density(world._w, C.byref(e)), "judge_density")
    return e.value


def run_learned(world, surrogate: Surrogate, dt: float, steps: int, judge_every: int = 10,
                bound: float = 0.01) -> dict:
    """Learned steps judged every `judge_every` steps by the plain density; a
    window whose relative density error exceeds `bound` is rerun with the
    plain step from its start."""
    out = np.zeros(6)
    _ok(_lib().pe_fluid_wcsph_run_learned(world._w, surrogate._s, float(dt), int(steps), int(judge_every),
                                          float(bound), _ptr(out)), "run_learned")
    return dict(windows=int(out[0]), fallbacks=int(out[1]), learned_steps=int(out[2]),
                plain_steps=int(out[3]), max_error=float(out[4]), last_error=float(out[5]))


def heldout_comparison(surrogate: Surrogate, world, dt: float, steps_before: int = 150, tank: int = 0) -> dict:
    """One-step prediction loss on a world never trained on (the mean of the
    normalised squared error over tank `tank`'s fluid particles, the training
    loss), after `steps_before` plain steps, for three predictors of the next
    plain step's (a, drho/dt): the trained network; the mean prediction (the
    network's output zeroed); and persistence (the previous plain step's
    (dv/dt, drho/dt) reused, which needs no network)."""
    a, b = tank_range(world, tank)
    world.run(dt, max(steps_before - 1, 0))
    # tanks are stored tank-major: original indices [a, b) are the tank's
    v0, r0 = world.velocities()[a:b], world.densities()[a:b]
    world.step(dt)
    v1, r1 = world.velocities()[a:b], world.densities()[a:b]
    surrogate.graph_from_world(world, a, b)
    world.step(dt)
    v2, r2 = world.velocities()[a:b], world.densities()[a:b]
    surrogate.targets_from_world(world, dt, update_stats=False)
    trained = surrogate.train_step(0.0)
    fluid = world.kinds()[a:b] == 0
    mean, std = (np.asarray(t, np.float64) for t in surrogate.stats())
    t_prev = np.concatenate([(v1 - v0) / dt, ((r1 - r0) / dt)[:, None]], axis=1)[fluid]
    t_now = np.concatenate([(v2 - v1) / dt, ((r2 - r1) / dt)[:, None]], axis=1)[fluid]
    persist = float((((t_prev - t_now) / std) ** 2).sum(axis=1).mean())
    mean_pred = float((((t_now - mean) / std) ** 2).sum(axis=1).mean())
    return {"trained": float(trained), "mean_prediction": mean_pred, "persistence": persist,
            "after_steps": steps_before, "fluid_particles": int(fluid.sum())}


def train_on_rollouts(surrogate: Surrogate, world, dt: float, steps: int, iters_per_step: int = 2,
                      lr: float = 1e-3, stat_steps: int = 20, log=None):
    """Online training on a (batched) world's plain rollout. The first
    `stat_steps` plain steps only fit the target normalisation (every tank in
    turn); then, before each plain step the graph of one tank (in turn) is
    taken, after it the targets, then `iters_per_step` Adam steps. Returns the
    losses."""
    tanks = world.tanks()
    losses = []
    for k in range(stat_steps + steps):
        a, b = tank_range(world, k % tanks)
        surrogate.graph_from_world(world, a, b)
        world.step(dt)
        fitting = k < stat_steps
        surrogate.targets_from_world(world, dt, update_stats=fitting)
        if fitting:
            continue
        for _ in range(iters_per_step):
            losses.append(surrogate.train_step(lr))
        if log and (k - stat_steps) % 50 == 0:
            log(k - stat_steps, losses[-1])
    return losses
