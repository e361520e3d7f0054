"""ctypes wrapper of the CPU oracle of the surface reconstruction
(oracle/surf_oracle.cpp). TEST INFRASTRUCTURE: only tests/ and bench.py's
CPU-baseline leg use it, as the checker or the CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from nonnewton_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsurf_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P, vp, i32 = C.POINTER(_abi.nn_sr_params), C.c_void_p, C.c_int32
        L.sro_dual_contouring.argtypes = [P, vp, i32] + [vp] * 6 + [vp, i32, vp, i32, vp, vp, vp]
        L.sro_prepass.argtypes = [P, vp, i32, vp, vp]
        L.sro_splat.argtypes = [P, vp, i32, vp, vp, vp, vp]
        L.sro_smooth.argtypes = [P, vp, vp, vp]
        L.sro_contour.argtypes = [P, vp, vp, vp, i32, vp, i32, vp, vp, vp]
        for f in ("sro_dual_contouring", "sro_prepass", "sro_splat", "sro_smooth", "sro_contour"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"surface oracle failed: {rc}")


def _shape(params):
    dims = list(params.dims)
    nb = [-(-d // _abi.NN_SR_BLOCK) for d in dims]
    return dims, dims[0] * dims[1] * dims[2], nb[0] * nb[1] * nb[2]


def dual_contouring(params: _abi.nn_sr_params, pos: np.ndarray, max_vertices: int = 1 << 20,
                    max_indices: int = 1 << 23) -> dict:
    """The whole pipeline on the CPU; returns every stage output as numpy arrays."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = pos.shape[0]
    dims, cells, blocks = _shape(params)
    out = {
        "field_splat": np.zeros(cells, np.float64), "field": np.zeros(cells, np.float64),
        "active": np.zeros(blocks, np.uint8), "G": np.zeros((n, 9), np.float32), "xbar": np.zeros((n, 3), np.float32),
        "vertices": np.zeros((max_vertices, 3), np.float64), "indices": np.zeros(max_indices, np.int32),
        "normals": np.zeros((max_vertices, 3), np.float64),
    }
    sd = C.c_double()
    nv, ni = C.c_int32(), C.c_int32()
    _check(lib().sro_dual_contouring(C.byref(params), _p(pos), n, _p(out["field_splat"]), _p(out["field"]),
                                     _p(out["active"]), _p(out["G"]), _p(out["xbar"]), C.byref(sd),
                                     _p(out["vertices"]), max_vertices, _p(out["indices"]), max_indices,
                                     _p(out["normals"]), C.byref(nv), C.byref(ni)))
    out["sd"] = sd.value
    out["vertices"] = out["vertices"][: nv.value]
    out["normals"] = out["normals"][: nv.value]
    out["indices"] = out["indices"][: ni.value]
    out["field_splat"] = out["field_splat"].reshape(dims[2], dims[1], dims[0])
    out["field"] = out["field"].reshape(dims[2], dims[1], dims[0])
    return out


def prepass(params, pos):
    pos = np.ascontiguousarray(pos, np.float32)
    n = pos.shape[0]
    G, xb = np.zeros((n, 9), np.float32), np.zeros((n, 3), np.float32)
    _check(lib().sro_prepass(C.byref(params), _p(pos), n, _p(G), _p(xb)))
    return G, xb


def splat(params, pos, G=None, xbar=None):
    pos = np.ascontiguousarray(pos, np.float32)
    dims, cells, blocks = _shape(params)
    f, a = np.zeros(cells, np.float64), np.zeros(blocks, np.uint8)
    G = None if G is None else np.ascontiguousarray(G, np.float32)
    xbar = None if xbar is None else np.ascontiguousarray(xbar, np.float32)
    _check(lib().sro_splat(C.byref(params), _p(pos), pos.shape[0], _p(G), _p(xbar), _p(f), _p(a)))
    return f.reshape(dims[2], dims[1], dims[0]), a


def smooth(params, field, active):
    dims, cells, _ = _shape(params)
    f = np.ascontiguousarray(field, np.float64).reshape(-1).copy()
    a = np.ascontiguousarray(active, np.uint8)
    sd = C.c_double()
    _check(lib().sro_smooth(C.byref(params), _p(f), _p(a), C.byref(sd)))
    return f.reshape(dims[2], dims[1], dims[0]), sd.value


def contour(params: _abi.nn_sr_params, field: np.ndarray, active: np.ndarray, max_vertices: int = 1 << 20,
            max_indices: int = 1 << 23) -> dict:
    """Only the contouring stages, on a given field [z, y, x] and active-block flags."""
    f = np.ascontiguousarray(field, np.float64).reshape(-1)
    a = np.ascontiguousarray(active, np.uint8)
    v = np.zeros((max_vertices, 3), np.float64)
    idx = np.zeros(max_indices, np.int32)
    nrm = np.zeros((max_vertices, 3), np.float64)
    nv, ni = C.c_int32(), C.c_int32()
    _check(lib().sro_contour(C.byref(params), _p(f), _p(a), _p(v), max_vertices, _p(idx), max_indices, _p(nrm),
                             C.byref(nv), C.byref(ni)))
    return {"vertices": v[: nv.value], "indices": idx[: ni.value], "normals": nrm[: nv.value]}


def vel_field(params, pos, vel):
    pos = np.ascontiguousarray(pos, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    dims, cells, _ = _shape(params)
    f = np.zeros(3 * cells, np.float64)
    L = lib()
    L.sro_vel_field.argtypes = [C.POINTER(_abi.nn_sr_params), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    L.sro_vel_field.restype = C.c_int
    _check(L.sro_vel_field(C.byref(params), _p(pos), _p(vel), pos.shape[0], _p(f)))
    return f


def mesh_velocity(params, vfield, vertices):
    v = np.ascontiguousarray(vertices, np.float64)
    out = np.zeros_like(v)
    L = lib()
    L.sro_mesh_velocity.argtypes = [C.POINTER(_abi.nn_sr_params), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    L.sro_mesh_velocity.restype = C.c_int
    _check(L.sro_mesh_velocity(C.byref(params), _p(np.ascontiguousarray(vfield, np.float64)), _p(v), len(v),
                               _p(out)))
    return out


def marching_cubes(params: _abi.nn_sr_params, field: np.ndarray, active: np.ndarray, max_vertices: int = 1 << 21,
                   max_indices: int = 1 << 23) -> dict:
    """Marching cubes on a given field [z, y, x] and active-block flags."""
    f = np.ascontiguousarray(field, np.float64).reshape(-1)
    a = np.ascontiguousarray(active, np.uint8)
    v = np.zeros((max_vertices, 3), np.float64)
    idx = np.zeros(max_indices, np.int32)
    nrm = np.zeros((max_vertices, 3), np.float64)
    nv, ni = C.c_int32(), C.c_int32()
    L = lib()
    L.sro_marching_cubes.argtypes = [C.POINTER(_abi.nn_sr_params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                     C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sro_marching_cubes.restype = C.c_int
    _check(L.sro_marching_cubes(C.byref(params), _p(f), _p(a), _p(v), max_vertices, _p(idx), max_indices, _p(nrm),
                                C.byref(nv), C.byref(ni)))
    return {"vertices": v[: nv.value], "indices": idx[: ni.value], "normals": nrm[: nv.value]}


def mc_table():
    """(triangle count [256], edge ids [256, 12, 3], -1 past the count) of the oracle's
    marching-cubes triangulation."""
    nt = np.zeros(256, np.int32)
    tris = np.zeros((256, 12, 3), np.int32)
    L = lib()
    L.sro_mc_table.argtypes = [C.c_void_p, C.c_void_p]
    L.sro_mc_table.restype = C.c_int
    _check(L.sro_mc_table(_p(nt), _p(tris)))
    return nt, tris
