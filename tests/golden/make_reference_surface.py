"""Runs the reference's own surface reconstruction (SPH/surf_recon/srtool.py, SRTool)
on a small particle ball and stores its stage outputs as a golden fixture
(tests/golden/ref_surface.npz). TEST INFRASTRUCTURE: it needs the reference checkout,
so it runs only where that checkout is (the fixture it writes is committed).

srtool.py is executed in plain Python against the Taichi stand-in
(tests/golden/refrun/ti_stub.py) with the source rewrites of make_reference_run.py.
Its sparse fields (pointer levels over 32^3 dense leaf blocks, dynamic per-voxel
particle lists) are stored per leaf block. The stages of SRTool.dual_contouring
(srtool.py:1264-1304) are called one by one so that each output is recorded: the
anisotropic kernels G and x_bar, the field after the splats, the smoothing's standard
deviation and the smoothed field, and the active leaf blocks. The smoothing radius is
two voxels (a 9^3 range) so that the plain-Python splats finish in minutes.

Usage: python tests/golden/make_reference_surface.py [/path/to/reference]
"""
from __future__ import annotations

import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_reference_run as M  # noqa: E402

BOX = [[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]
VOXEL, RADIUS, SMOOTH, ISO = 0.01, 0.01, 0.02, 0.0


def ball(seed=5, radius=0.05, spacing=0.015, center=0.5, jitter=1e-3):
    rng = np.random.default_rng(seed)
    g = np.arange(-radius, radius + 1e-9, spacing)
    p = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    p = p[np.linalg.norm(p, axis=1) <= radius]
    return (p + center + rng.uniform(-jitter, jitter, size=p.shape)).astype(np.float32)


def dense(f, dims):
    """A sparse field of the run as a dense [z, y, x] array over `dims` vertices; every
    active block must lie inside."""
    out = np.zeros((dims[2], dims[1], dims[0]), np.float64)
    for bk, blk in f.blocks.items():
        lo = [b * e for b, e in zip(bk, f.block)]
        assert all(0 <= lo[a] and lo[a] + f.block[a] <= dims[a] + f.block[a] for a in range(3))
        for x in range(f.block[0]):
            for y in range(f.block[1]):
                for z in range(f.block[2]):
                    v = blk[x, y, z]
                    if v != 0:
                        gx, gy, gz = lo[0] + x, lo[1] + y, lo[2] + z
                        assert gx < dims[0] and gy < dims[1] and gz < dims[2]
                        out[gz, gy, gx] = v
    return out


def main(ref_root: str):
    sr_mod = M.load_reference(ref_root, "SPH/surf_recon/srtool.py", "srtool_reference")
    ti = sys.modules["taichi"]
    pos = ball()
    n = len(pos)
    field = ti.Vector.field(3, dtype=ti.f32, shape=n)
    field.from_numpy(pos)
    with contextlib.redirect_stdout(io.StringIO()):
        sr = sr_mod.SRTool(BOX, voxel_size=VOXEL, particle_radius=RADIUS, max_num_vertices=20000,
                           max_num_indices=120000, max_num_particles=n)
        sr.reset()
        sr.update_particles(n, field)
        sr.generate_fluid_field(SMOOTH, n, field)
        sr.generate_smooth_fluid_field(SMOOTH, n, field)
    rng_ = int(np.ceil(4 * SMOOTH / VOXEL)) + 1
    dims = [int(np.ceil((BOX[1][k] - BOX[0][k]) / VOXEL)) + (rng_ - rng_ // 2 + 1) + 3 for k in range(3)]
    f_splat = dense(sr.voxel.voxel_vertex_value, dims)
    blocks = np.array(sorted(sr.voxel.voxel_vertex_value.blocks), np.int32)
    with contextlib.redirect_stdout(io.StringIO()):
        sd = float(sr.density_field_stats())
        sr.smooth_sdf(iteration=1, radius=1)
    f_smooth = dense(sr.voxel.voxel_vertex_value, dims)
    out = dict(pos=pos, dims=np.array(dims, np.int32), G=sr.G.to_numpy()[:n].reshape(n, 9),
               xbar=sr.x_bar.to_numpy()[:n], field_splat=f_splat, field_smooth=f_smooth, sd=np.float64(sd),
               blocks=blocks, params=np.array([VOXEL, RADIUS, SMOOTH, ISO], np.float64))
    path = os.path.join(HERE, "ref_surface.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {n} particles, grid {dims}, {len(blocks)} active blocks, sd {sd:.6g}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
    main(sys.argv[1])
