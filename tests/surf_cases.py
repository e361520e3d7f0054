"""Particle sets and mesh checks shared by the surface-reconstruction tests."""
from __future__ import annotations

import math

import numpy as np

from nonnewton_b200 import _abi


def ball(seed=0, radius=0.15, spacing=0.02, center=0.5, jitter=1e-3):
    """A lattice ball of particles, jittered uniformly per coordinate."""
    rng = np.random.default_rng(seed)
    g = np.arange(-radius, radius + 1e-9, spacing)
    p = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    p = p[np.linalg.norm(p, axis=1) <= radius]
    return (p + center + rng.uniform(-jitter, jitter, size=p.shape)).astype(np.float32)


def block(seed=0, n=(12, 10, 8), spacing=0.02, corner=(0.3, 0.25, 0.35), jitter=1e-3):
    """A dam-break-like box of fluid particles."""
    rng = np.random.default_rng(seed)
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), -1).reshape(-1, 3)
    p = np.asarray(corner) + idx * spacing
    return (p + rng.uniform(-jitter, jitter, size=p.shape)).astype(np.float32)


def torus(R=0.12, r=0.045, spacing=0.02, center=0.5):
    """A solid lattice torus around the y axis, like the reference example's model
    (SPH/surf_recon/example.py reads a 604-point voxelised torus): 640 particles."""
    g = np.arange(center - 0.2, center + 0.2 + 1e-9, spacing)
    p = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rho = np.hypot(p[:, 0] - center, p[:, 2] - center)
    return p[(rho - R) ** 2 + (p[:, 1] - center) ** 2 <= r * r].astype(np.float32)


def default_params(dims=None, voxel_size=0.01, particle_radius=0.02, smooth_radius=0.06, isolevel=0.0,
                   use_smooth_field=True, record_normals=True, box=1.0):
    """The reference example's settings (SPH/surf_recon/example.py): voxel 0.01,
    particle radius 0.02, smoothing radius 0.06, level 0, in a unit box; the grid is
    the one SRTool.grid_dims gives for that box."""
    if dims is None:
        rng = int(math.ceil(4 * smooth_radius / voxel_size)) + 1
        dims = [int(math.ceil(box / voxel_size)) + (rng - rng // 2 + 1) + 3] * 3
    return _abi.make_sr_params(dims, [0, 0, 0], voxel_size, particle_radius, smooth_radius, isolevel,
                               use_smooth_field=use_smooth_field, record_normals=record_normals)


def closed_oriented(faces: np.ndarray, nv: int) -> bool:
    """Every directed edge occurs once and its reverse once: a closed 2-manifold with
    consistent winding (and every vertex used)."""
    f = np.asarray(faces, np.int64)
    if len(f) == 0:
        return False
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    key = e[:, 0] * nv + e[:, 1]
    rev = e[:, 1] * nv + e[:, 0]
    u, cnt = np.unique(key, return_counts=True)
    if np.any(cnt != 1):
        return False
    return bool(np.all(np.isin(rev, u))) and len(np.unique(f)) == nv


def weld(vertices: np.ndarray, faces: np.ndarray, tol: float = 1e-6):
    """Merge vertices closer than `tol` (marching cubes emits each crossing edge once per
    cube, and the two copies of an edge's crossing may differ in the last f32 bit);
    returns (vertices, faces) of the welded mesh."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree

    v = np.asarray(vertices, np.float64)
    pairs = cKDTree(v).query_pairs(tol, output_type="ndarray")
    g = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])), shape=(len(v), len(v)))
    _, label = connected_components(g, directed=False)
    first = np.full(label.max() + 1, -1, np.int64)
    first[label[::-1]] = np.arange(len(v))[::-1]
    return v[first], label[np.asarray(faces, np.int64).reshape(-1)].reshape(-1, 3)


def signed_volume(vertices: np.ndarray, faces: np.ndarray) -> float:
    v = np.asarray(vertices, np.float64)
    f = np.asarray(faces, np.int64).reshape(-1, 3)
    return float(np.einsum("ij,ij->i", v[f[:, 0]], np.cross(v[f[:, 1]], v[f[:, 2]])).sum() / 6.0)


# corners of each cube edge and corner offsets (srtool.py:775-783, 931-942)
CUBE_OFF = np.array([[0, 1, 0], [1, 1, 0], [1, 0, 0], [0, 0, 0], [0, 1, 1], [1, 1, 1], [1, 0, 1], [0, 0, 1]])
CUBE_EDGE = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6], [6, 7], [7, 4], [0, 4], [1, 5], [2, 6], [3, 7]])
