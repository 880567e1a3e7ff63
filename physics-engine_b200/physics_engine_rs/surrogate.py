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
    "pe_surrogate_train_step": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_float)]),
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

    def train_step(self, lr: float = 0.0) -> float:
        loss = C.c_float()
        _ok(self._L.pe_surrogate_train_step(self._s, float(lr), C.byref(loss)), "train_step")
        return loss.value
