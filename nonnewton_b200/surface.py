"""Surface reconstruction of a particle set: the reference's SRTool
(SPH/surf_recon/srtool.py:869-1838) on the GPU through libnnsph's nn_sr_* entry points.

Same constructor arguments, `dual_contouring(...)` call and mesh attributes
(`mesh_vertex`, `mesh_index`, `num_vertices[None]`, `num_indices[None]`,
`mesh_normal`, `mesh_velocity`) as the reference, so `SPH/surf_recon/example.py` works unchanged apart
from the import:

    sr = SRTool([[0, 0, 0], [1, 1, 1]], voxel_size=0.01, particle_radius=0.02,
                max_num_vertices=20000, max_num_indices=600000)
    sr.dual_contouring(isolevel=0, smooth_radius=0.06, num_particles=n, pos=positions)
    sr.export_mesh("out.ply")

`pos` (and `velocity`, with `record_velocity=True`) is a [n, 3] array (torch on the
GPU, numpy, or a field with `to_numpy()` such as the reference example's Taichi field). The mesh stays on the GPU as torch tensors. `marching_cubes(...)`
takes the same arguments and ends the same pipeline with marching cubes
(srtool.py:1765-1800) instead of dual contouring.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _abi
from .engine import NNError, lib


class _Scalar:
    """Stands in for the reference's 0-d Taichi fields (`sr.num_vertices[None]`)."""

    def __init__(self, v: int = 0):
        self.value = int(v)

    def __getitem__(self, key):
        return self.value

    def __int__(self):
        return self.value


def _sr_lib():
    L = lib()
    if not getattr(L, "_sr_bound", False):
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        L.nn_sr_create.argtypes = [i32, i64, i32, i32, i32, C.POINTER(vp)]
        L.nn_sr_destroy.argtypes = [vp]
        L.nn_sr_last_error.argtypes = [vp]
        L.nn_sr_last_error.restype = C.c_char_p
        L.nn_sr_dual_contouring.argtypes = [vp, C.POINTER(_abi.nn_sr_params), vp, vp, i32, vp]
        L.nn_sr_marching_cubes.argtypes = [vp, C.POINTER(_abi.nn_sr_params), vp, vp, i32, vp]
        L.nn_sr_get_mesh.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), vp, vp, vp, vp, vp]
        L.nn_sr_get_stage.argtypes = [vp, i32, vp, vp, vp, vp, C.POINTER(C.c_double), vp]
        for f in ("nn_sr_create", "nn_sr_destroy", "nn_sr_dual_contouring", "nn_sr_marching_cubes", "nn_sr_get_mesh",
                  "nn_sr_get_stage"):
            getattr(L, f).restype = C.c_int
        L._sr_bound = True
    return L


class SRTool:
    def __init__(self, bounding_box_extent, voxel_size=0.01, particle_radius=0.01, record_normals=False,
                 record_velocity=False, max_num_vertices=8000000, max_num_indices=100000000,
                 max_num_particles=9000000, hash_level_dimensions=None, device="cuda"):
        self.bounding_box_extent = [[float(v) for v in bounding_box_extent[0]],
                                    [float(v) for v in bounding_box_extent[1]]]
        self.voxel_size = float(voxel_size)
        self.radius = float(particle_radius)
        self.record_normals = bool(record_normals)
        self.record_velocity = bool(record_velocity)
        self.max_num_vertices = int(max_num_vertices)
        self.max_num_indices = int(max_num_indices)
        self.max_num_particles = int(max_num_particles)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("SRTool runs on the GPU (libnnsph); there is no CPU path")
        self.num_vertices = _Scalar(0)
        self.num_indices = _Scalar(0)
        self.mesh_vertex = torch.zeros((0, 3), dtype=torch.float32, device=self.device)
        self.mesh_index = torch.zeros(0, dtype=torch.int32, device=self.device)
        self.mesh_normal = torch.zeros((0, 3), dtype=torch.float32, device=self.device)
        self.mesh_velocity = torch.zeros((0, 3), dtype=torch.float32, device=self.device)
        self._h = None
        self._cells = 0
        self.last_params = None

    # -- grid ------------------------------------------------------------------------------
    def grid_dims(self, smooth_radius: float, use_smooth_fluid_field: bool = True) -> list[int]:
        """Vertices per axis: the box, the splat reach beyond it, and the ring the
        smoothing and contouring read."""
        vs = self.voxel_size
        rng = int(math.ceil(4 * smooth_radius / vs)) + 1
        reach = (rng - rng // 2 + 1) if use_smooth_fluid_field else 2
        return [int(math.ceil((self.bounding_box_extent[1][k] - self.bounding_box_extent[0][k]) / vs)) + reach + 3
                for k in range(3)]

    def _ensure(self, cells: int):
        if self._h is not None and cells <= self._cells:
            return
        self.close()
        h = C.c_void_p()
        rc = _sr_lib().nn_sr_create(self.max_num_particles, int(cells), self.max_num_vertices, self.max_num_indices,
                                    _abi.NN_SR_VELOCITY if self.record_velocity else 0, C.byref(h))
        if rc != 0:
            raise NNError(rc, "nn_sr_create failed")
        self._h, self._cells = h, int(cells)

    def close(self):
        if self._h is not None:
            _sr_lib().nn_sr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _rc(self, rc):
        if rc != 0:
            raise NNError(rc, _sr_lib().nn_sr_last_error(self._h).decode())

    # -- the reference's API -----------------------------------------------------------------
    def reset(self):
        self.num_vertices = _Scalar(0)
        self.num_indices = _Scalar(0)

    def dual_contouring(self, isolevel, smooth_radius, num_particles, pos, velocity=None,
                        use_smooth_fluid_field=True, record_normals=True):
        """SRTool.dual_contouring (srtool.py:1264-1304). `record_normals` is accepted
        and, as in the reference, ignored: the constructor's flags decide; `velocity`
        is used when the tool records velocities."""
        return self._run(_sr_lib().nn_sr_dual_contouring, isolevel, smooth_radius, num_particles, pos, velocity,
                         use_smooth_fluid_field)

    def marching_cubes(self, isolevel, smooth_radius, num_particles, pos, velocity=None,
                       use_smooth_fluid_field=True, record_normals=True):
        """The dual_contouring pipeline with marching cubes as the last stage
        (marching_cube_impl, srtool.py:1765-1800, which the reference defines but never
        calls). One vertex per crossing edge of each cube, as the reference emits them;
        the triangles come from the library's own case table (nn_sr_marching_cubes)."""
        return self._run(_sr_lib().nn_sr_marching_cubes, isolevel, smooth_radius, num_particles, pos, velocity,
                         use_smooth_fluid_field)

    def _run(self, entry, isolevel, smooth_radius, num_particles, pos, velocity, use_smooth_fluid_field):
        n = int(num_particles)

        def dev(a):
            if hasattr(a, "to_numpy"):  # a Taichi field, as the reference's callers pass
                a = a.to_numpy()
            if torch.is_tensor(a):
                return a[:n].to(device=self.device, dtype=torch.float32).contiguous()
            return torch.as_tensor(np.asarray(a)[:n], dtype=torch.float32, device=self.device).contiguous()
        p = dev(pos)
        vel = None
        if self.record_velocity:
            if velocity is None:
                raise ValueError("SRTool(record_velocity=True) needs the particle velocities")
            vel = dev(velocity)
        dims = self.grid_dims(smooth_radius, use_smooth_fluid_field)
        self._ensure(dims[0] * dims[1] * dims[2])
        prm = _abi.make_sr_params(dims, self.bounding_box_extent[0], self.voxel_size, self.radius, smooth_radius,
                                  isolevel, use_smooth_field=use_smooth_fluid_field,
                                  record_normals=self.record_normals)
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        self._rc(entry(self._h, C.byref(prm), C.c_void_p(p.data_ptr()),
                       C.c_void_p(vel.data_ptr()) if vel is not None else None, n, stream))
        nv, ni = C.c_int32(), C.c_int32()
        self._rc(_sr_lib().nn_sr_get_mesh(self._h, C.byref(nv), C.byref(ni), None, None, None, None, stream))
        self.mesh_vertex = torch.empty((nv.value, 3), dtype=torch.float32, device=self.device)
        self.mesh_index = torch.empty(ni.value, dtype=torch.int32, device=self.device)
        self.mesh_normal = torch.empty((nv.value if self.record_normals else 0, 3), dtype=torch.float32,
                                       device=self.device)
        self.mesh_velocity = torch.empty((nv.value if self.record_velocity else 0, 3), dtype=torch.float32,
                                         device=self.device)

        def ptr(t):
            return C.c_void_p(t.data_ptr()) if t.numel() else None
        self._rc(_sr_lib().nn_sr_get_mesh(self._h, None, None, ptr(self.mesh_vertex), ptr(self.mesh_index),
                                          ptr(self.mesh_normal) if self.record_normals else None,
                                          ptr(self.mesh_velocity) if self.record_velocity else None, stream))
        self.num_vertices = _Scalar(nv.value)
        self.num_indices = _Scalar(ni.value)
        self.last_params = prm
        return self

    def stage(self, which: int, n: int) -> dict:
        """Stage outputs of the last call (for parity checks): field [z, y, x] after the
        splats (0) or after smoothing (1), active-block flags, G [n, 9], x_bar [n, 3], sd."""
        prm = self.last_params
        dims = list(prm.dims)
        nb = [-(-d // _abi.NN_SR_BLOCK) for d in dims]
        field = torch.empty(dims[2] * dims[1] * dims[0], dtype=torch.float32, device=self.device)
        act = torch.empty(nb[0] * nb[1] * nb[2], dtype=torch.uint8, device=self.device)
        G = torch.empty((max(n, 1), 9), dtype=torch.float32, device=self.device)
        xb = torch.empty((max(n, 1), 3), dtype=torch.float32, device=self.device)
        sd = C.c_double()
        cs = torch.cuda.current_stream(self.device)
        self._rc(_sr_lib().nn_sr_get_stage(self._h, int(which), C.c_void_p(field.data_ptr()),
                                           C.c_void_p(act.data_ptr()), C.c_void_p(G.data_ptr()),
                                           C.c_void_p(xb.data_ptr()), C.byref(sd), C.c_void_p(cs.cuda_stream)))
        cs.synchronize()
        return {"field": field.reshape(dims[2], dims[1], dims[0]), "active": act, "G": G[:n], "xbar": xb[:n],
                "sd": sd.value}

    def export_mesh(self, file_path: str, output_normal=False, output_velocity=False):
        """Binary little-endian PLY with the vertices, triangles and optionally the
        normals and the velocities (export_mesh, srtool.py:1802-1838)."""
        if not file_path.endswith("ply"):
            raise ValueError("Output file must be in ply format!")
        if output_velocity and len(self.mesh_velocity) != len(self.mesh_vertex):
            raise RuntimeError("velocities were not recorded: SRTool(record_velocity=True)")
        v = self.mesh_vertex.cpu().numpy().astype("<f4")
        f = self.mesh_index.cpu().numpy().astype("<i4").reshape(-1, 3)
        if output_normal and len(self.mesh_normal) != len(v):
            raise RuntimeError("normals were not recorded: SRTool(record_normals=True)")
        head = ["ply", "format binary_little_endian 1.0", f"element vertex {len(v)}",
                "property float x", "property float y", "property float z"]
        if output_normal:
            head += ["property float nx", "property float ny", "property float nz"]
        if output_velocity:
            head += ["property float vx", "property float vy", "property float vz"]
        head += [f"element face {len(f)}", "property list uchar int vertex_indices", "end_header"]
        cols = [v]
        if output_normal:
            cols.append(self.mesh_normal.cpu().numpy().astype("<f4"))
        if output_velocity:
            cols.append(self.mesh_velocity.cpu().numpy().astype("<f4"))
        vert = np.concatenate(cols, axis=1)
        face = np.zeros(len(f), dtype=[("n", "u1"), ("i", "<i4", (3,))])
        face["n"] = 3
        face["i"] = f
        with open(file_path, "wb") as fh:
            fh.write(("\n".join(head) + "\n").encode())
            fh.write(np.ascontiguousarray(vert, dtype="<f4").tobytes())
            fh.write(face.tobytes())
