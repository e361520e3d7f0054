"""ctypes wrapper of the CPU oracle (oracle/sph_oracle.cpp). TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker or the CPU baseline; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from nonnewton_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsph_oracle.so")

FIELDS = {
    "x": (0, 3), "x_0": (1, 3), "v": (2, 3), "acceleration": (3, 3), "volume": (4, 1), "m": (5, 1),
    "density": (6, 1), "pressure": (7, 1), "dfsph_factor": (8, 1), "density_adv": (9, 1),
    "material": (10, 1), "is_dynamic": (11, 1), "phase_id": (12, 1), "strain_rate_norm": (13, 1),
    "nonnewton_viscosity": (14, 1), "stress": (15, 6), "rotations": (16, 9), "rest_volume": (17, 1),
}

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.c_int, C.POINTER(_abi.nn_scene_params), C.c_int, C.c_int, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_destroy.argtypes = [C.c_void_p]
        for f in ("or_initialize",):
            getattr(L, f).argtypes = [C.c_void_p]
        L.or_step.argtypes = [C.c_void_p, C.c_int]
        L.or_run_pass.argtypes = [C.c_void_p, C.c_int]
        L.or_set_animation.argtypes = [C.c_void_p, C.c_void_p]
        L.or_get_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.or_set_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.or_get_neighbors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.or_neighbor_total.argtypes = [C.c_void_p]
        L.or_neighbor_total.restype = C.c_int64
        L.or_get_stats.argtypes = [C.c_void_p, C.POINTER(_abi.nn_stats)]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        L.or_polar_rotation.argtypes = [C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleSim:
    """One scene simulated by the CPU restatement (float32 or float64)."""

    def __init__(self, particles, param, precision: str = "f32", velocities=None):
        L = lib()
        self.n = particles.n
        self.params = param.to_c() if hasattr(param, "to_c") else param
        x = np.ascontiguousarray(particles.x, dtype=np.float64)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64)
        self._keep = [x, v,
                      np.ascontiguousarray(particles.material, dtype=np.int32),
                      np.ascontiguousarray(particles.is_dynamic, dtype=np.int32),
                      np.ascontiguousarray(particles.phase_id, dtype=np.int32),
                      np.ascontiguousarray(particles.mass, dtype=np.float64)]
        self.h = L.or_create(1 if precision == "f64" else 0, C.byref(self.params), self.n, int(particles.n_fluid),
                             *[_ptr(a) for a in self._keep])
        if not self.h:
            raise RuntimeError("or_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def _rc(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {_abi.ERROR_NAMES.get(rc, '?')}")

    def initialize(self):
        self._rc(lib().or_initialize(self.h))

    def step(self, n=1):
        self._rc(lib().or_step(self.h, int(n)))

    def run_pass(self, p):
        self._rc(lib().or_run_pass(self.h, int(p)))

    def set_animation(self, d):
        """Displacement added to every particle by the next step (animate_particles)."""
        a = np.ascontiguousarray(np.asarray(d, dtype=np.float64).reshape(3))
        self._rc(lib().or_set_animation(self.h, _ptr(a)))

    def get(self, name):
        fid, w = FIELDS[name]
        out = np.zeros(self.n * w, dtype=np.float64)
        self._rc(lib().or_get_field(self.h, fid, _ptr(out)))
        return out.reshape(self.n, w) if w > 1 else out

    def set(self, name, arr):
        fid, w = FIELDS[name]
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64).reshape(-1))
        assert a.size == self.n * w
        self._rc(lib().or_set_field(self.h, fid, _ptr(a)))

    def neighbors(self, width=60):
        counts = np.zeros(self.n, np.int32)
        lists = np.zeros((self.n, width), np.int32)
        rc = lib().or_get_neighbors(self.h, _ptr(counts), _ptr(lists), int(width))
        if rc not in (0, _abi.NN_ERR_NEIGHBOR_OVERFLOW):
            self._rc(rc)
        return counts, lists

    def neighbor_total(self):
        return int(lib().or_neighbor_total(self.h))

    def stats(self):
        s = _abi.nn_stats()
        self._rc(lib().or_get_stats(self.h, C.byref(s)))
        return s.as_dict()


def set_threads(t: int):
    lib().or_set_threads(int(t))


def get_threads() -> int:
    return int(lib().or_get_threads())


def polar_rotation(A: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(A, dtype=np.float64).reshape(9)
    r = np.zeros(9, np.float64)
    lib().or_polar_rotation(_ptr(a), _ptr(r))
    return r.reshape(3, 3)
