"""ctypes binding of libnnsph.so (include/nnsph.h) and a thin engine object.

The CUDA library is the only compute path: if `libnnsph.so` is missing or no CUDA
device is present, constructing an Engine raises. There is no CPU fallback.
`precision="f64"` binds libnnsph64.so instead, the same kernels built with double
arithmetic (the FP64 run the FP32 path's error is measured against).
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnnsph.so")
LIB_PATHS = {"f32": LIB_PATH, "f64": os.path.join(HERE, "libnnsph64.so")}
REAL_BYTES = {"f32": 4, "f64": 8}
X_SPLIT_DEFAULT = 2  # x cells per cell edge of a new context (the library's NN_DEFAULT_XSPLIT)

_libs = {}


class NNError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_abi.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib(precision: str = "f32"):
    if precision not in _libs:
        path = LIB_PATHS[precision]
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python __graft_entry__.py build` "
                              "(or nonnewton_b200.build.build())")
        L = C.CDLL(path)
        vp, i32, i64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
        L.nn_abi_version.restype = C.c_int
        L.nn_last_error.restype = C.c_char_p
        L.nn_last_error.argtypes = [vp]
        L.nn_ctx_create.argtypes = [i32, i32, i32, i64, C.POINTER(vp)]
        L.nn_ctx_destroy.argtypes = [vp]
        L.nn_ctx_set_stream.argtypes = [vp, vp]
        L.nn_bind_state.argtypes = [vp, C.POINTER(_abi.nn_state)]
        L.nn_set_scenes.argtypes = [vp, i32, C.POINTER(_abi.nn_scene_desc)]
        L.nn_initialize.argtypes = [vp]
        L.nn_step.argtypes = [vp, i32, u32]
        L.nn_run_pass.argtypes = [vp, i32]
        L.nn_set_animation.argtypes = [vp, i32, C.POINTER(C.c_float)]
        L.nn_set_animation.restype = C.c_int
        L.nn_get_neighbors.argtypes = [vp, vp, vp, i32]
        L.nn_get_stats.argtypes = [vp, i32, C.POINTER(_abi.nn_stats)]
        L.nn_launch_count.argtypes = [vp]
        L.nn_launch_count.restype = i64
        L.nn_set_block_size.argtypes = [vp, i32]
        L.nn_time_kernel.argtypes = [vp, i32, i32, C.POINTER(C.c_float)]
        L.nn_get_stats_range.argtypes = [vp, i32, i32, C.POINTER(_abi.nn_stats)]
        L.nn_get_stats_range.restype = C.c_int
        L.nn_time_kernel.restype = C.c_int
        for name in ("nn_ctx_create", "nn_ctx_destroy", "nn_ctx_set_stream", "nn_bind_state", "nn_set_scenes",
                     "nn_initialize", "nn_step", "nn_run_pass", "nn_get_neighbors", "nn_get_stats",
                     "nn_set_block_size"):
            getattr(L, name).restype = C.c_int
        if L.nn_abi_version() != 1:
            raise ImportError(f"{os.path.basename(path)}: ABI version mismatch")
        L.nn_real_bytes.restype = C.c_int
        if L.nn_real_bytes() != REAL_BYTES[precision]:
            raise ImportError(f"{os.path.basename(path)} computes in {L.nn_real_bytes()}-byte reals, not {precision}")
        _libs[precision] = L
    return _libs[precision]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Engine:
    """One nn_ctx: capacities fixed at creation, state bound from torch tensors."""

    def __init__(self, max_particles: int, max_scenes: int = 1, max_neighbors: int = 64, max_cells: int = 0,
                 device=None, precision: str = "f32"):
        if not torch.cuda.is_available():
            raise RuntimeError("nonnewton_b200 needs a CUDA device (the SPH step runs only as sm_100a kernels)")
        dev = torch.device(device if device is not None else "cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        torch.cuda.set_device(self.device)
        self.precision = precision
        self.L = lib(precision)
        h = C.c_void_p()
        self._rc(self.L.nn_ctx_create(int(max_particles), int(max_scenes), int(max_neighbors), int(max_cells),
                                      C.byref(h)), None)
        self.h = h
        self.max_neighbors = max_neighbors
        self.x_split = X_SPLIT_DEFAULT
        self.set_x_split(X_SPLIT_DEFAULT)
        self._state = None
        self._scenes = None
        self._keep = []

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.nn_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _rc(self, rc, h="ctx"):
        if rc != 0:
            msg = self.L.nn_last_error(self.h if h == "ctx" else None)
            raise NNError(rc, msg.decode() if msg else "")

    def set_stream(self, stream: torch.cuda.Stream | None):
        self._rc(self.L.nn_ctx_set_stream(self.h, C.c_void_p(stream.cuda_stream if stream is not None else 0)))

    def set_block_size(self, threads: int):
        self._rc(self.L.nn_set_block_size(self.h, int(threads)))

    def set_tuning(self, block: int = 0, unroll: int = 0, cell_factor: int = 0):
        """Launch shape of the neighbour passes; a new cell factor needs set_scenes again."""
        f = self.L.nn_set_tuning
        f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
        f.restype = C.c_int
        self._rc(f(self.h, int(block), int(unroll), int(cell_factor)))

    def set_x_split(self, x_split: int = 0):
        """x cells per cell edge of the search grid (see nn_set_x_split); set_scenes again after."""
        f = self.L.nn_set_x_split
        f.argtypes = [C.c_void_p, C.c_int32]
        f.restype = C.c_int
        self._rc(f(self.h, int(x_split)))
        self.x_split = int(x_split) if x_split else X_SPLIT_DEFAULT

    def bind(self, pd, n: int | None = None) -> None:
        """Bind the fields of `pd`; `n` active particles (default: all rows)."""
        st = _abi.nn_state()
        st.size = C.sizeof(_abi.nn_state)
        st.n = int(pd.x.shape[0] if n is None else n)
        for name in ("x", "x_0", "v", "acceleration", "volume", "m", "density", "pressure", "dfsph_factor",
                     "density_adv", "material", "is_dynamic", "phase_id", "strain_rate_norm",
                     "nonnewton_viscosity", "stress", "rotations"):
            t = getattr(pd, name, None)
            if t is not None:
                assert t.is_cuda and t.is_contiguous(), name
                setattr(st, name, t.data_ptr())
        self._state = st
        self._rc(self.L.nn_bind_state(self.h, C.byref(st)))

    def set_scenes(self, scenes):
        """scenes: list of (start, n, n_fluid, nn_scene_params)."""
        arr = (_abi.nn_scene_desc * len(scenes))()
        for k, (start, n, nf, p) in enumerate(scenes):
            arr[k].size = C.sizeof(_abi.nn_scene_desc)
            arr[k].start, arr[k].n, arr[k].n_fluid = int(start), int(n), int(nf)
            arr[k].params = p
        self._scenes = arr
        self._rc(self.L.nn_set_scenes(self.h, len(scenes), arr))

    def initialize(self):
        self._rc(self.L.nn_initialize(self.h))

    def step(self, nsteps: int = 1, sync: bool = True, host_loop: bool = False, resume: bool = False):
        """nsteps steps; `sync` writes the state back to the bound fields at the end,
        `resume` continues from the state the previous step left on the device."""
        flags = ((_abi.NN_STEP_SYNC_STATE if sync else 0) | (_abi.NN_STEP_HOST_LOOP if host_loop else 0)
                 | (_abi.NN_STEP_RESUME if resume else 0))
        self._rc(self.L.nn_step(self.h, int(nsteps), flags))

    def set_animation(self, scene: int, displacement):
        """The next step moves every particle of `scene` by `displacement` (3 floats)."""
        d = (C.c_float * 3)(*[float(v) for v in displacement])
        self._rc(self.L.nn_set_animation(self.h, int(scene), d))

    def run_pass(self, p: int):
        self._rc(self.L.nn_run_pass(self.h, int(p)))

    def neighbors(self, n: int, width: int = 60):
        num = torch.zeros(n, dtype=torch.int32, device=self.device)
        lists = torch.full((n, width), -1, dtype=torch.int32, device=self.device)
        self._rc(self.L.nn_get_neighbors(self.h, _ptr(num), _ptr(lists), int(width)))
        return num, lists

    def set_neighbor_cap(self, max_neighbors: int):
        """Re-size the neighbour lists (see nn_set_neighbor_cap); clears overflow statuses."""
        f = self.L.nn_set_neighbor_cap
        f.argtypes = [C.c_void_p, C.c_int32]
        f.restype = C.c_int
        self._rc(f(self.h, int(max_neighbors)))
        self.max_neighbors = int(max_neighbors)

    def status_async(self, out: torch.Tensor, scene: int = 0):
        """Enqueue the copy of (status, max_neighbors_seen) of `scene` into `out`, two
        int32 in pinned host memory (see nn_status_async); status_wait() waits for it."""
        f = self.L.nn_status_async
        f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        f.restype = C.c_int
        self._rc(f(self.h, int(scene), C.c_void_p(out.data_ptr())))

    def status_wait(self):
        f = self.L.nn_status_wait
        f.argtypes = [C.c_void_p]
        f.restype = C.c_int
        self._rc(f(self.h))

    def stats(self, scene: int = 0) -> dict:
        s = _abi.nn_stats()
        self._rc(self.L.nn_get_stats(self.h, int(scene), C.byref(s)))
        return s.as_dict()

    def stats_range(self, first: int, count: int) -> list[dict]:
        arr = (_abi.nn_stats * max(count, 1))()
        self._rc(self.L.nn_get_stats_range(self.h, int(first), int(count), arr))
        return [arr[k].as_dict() for k in range(count)]

    def time_kernel(self, kernel: int, reps: int = 20) -> float:
        ms = C.c_float()
        self._rc(self.L.nn_time_kernel(self.h, int(kernel), int(reps), C.byref(ms)))
        return float(ms.value)

    def launch_count(self) -> int:
        return int(self.L.nn_launch_count(self.h))
