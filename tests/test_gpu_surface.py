"""CUDA surface reconstruction (nn_sr_*, nonnewton_b200.surface.SRTool) against the CPU
oracle, stage by stage, on the same inputs:

  - anisotropic kernels G, x_bar: 1e-4 / 1e-6 of each array's scale;
  - splat field from the CUDA G, x_bar: 1e-5 of the field's scale, identical active blocks;
  - smoothing of the CUDA splat field: 1e-5 of the field's scale (sd 1e-6 relative);
  - contouring of the CUDA smoothed field: the same triangles, index for index, and
    vertices within 1e-6 m;
and end to end: a closed, consistently wound mesh of the same size."""
import numpy as np
import pytest
import torch

from .surf_cases import ball, block, closed_oriented, default_params, torus

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def surf():
    from oracle import surf as S

    S.build()
    return S


def _tool(**kw):
    from nonnewton_b200.surface import SRTool

    kw.setdefault("record_normals", True)
    kw.setdefault("max_num_vertices", 200000)
    return SRTool([[0, 0, 0], [1, 1, 1]], voxel_size=0.01, particle_radius=0.02, max_num_indices=2000000,
                  max_num_particles=100000, **kw)


def _scale_err(g, r):
    g, r = np.asarray(g, np.float64), np.asarray(r, np.float64)
    return float(np.abs(g - r).max() / max(np.abs(r).max(), 1e-30))


@pytest.mark.parametrize("case", ["ball", "block"])
def test_surface_stages_match_oracle(cuda_lib, surf, case):
    pos = ball(seed=10) if case == "ball" else block(seed=11)
    n = len(pos)
    sr = _tool()
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=n, pos=torch.from_numpy(pos).cuda())
    prm = sr.last_params
    s0, s1 = sr.stage(0, n), sr.stage(1, n)
    # anisotropic kernels
    G, xb = surf.prepass(prm, pos)
    assert _scale_err(s0["G"].cpu().numpy(), G) < 1e-4
    assert _scale_err(s0["xbar"].cpu().numpy(), xb) < 1e-6
    # splats from the CUDA kernels
    f_or, act_or = surf.splat(prm, pos, s0["G"].cpu().numpy(), s0["xbar"].cpu().numpy())
    assert np.array_equal(s0["active"].cpu().numpy(), act_or)
    assert _scale_err(s0["field"].cpu().numpy(), f_or) < 1e-5
    # smoothing of the CUDA splat field
    f_sm, sd = surf.smooth(prm, s0["field"].cpu().numpy(), act_or)
    assert abs(s1["sd"] - sd) <= 1e-6 * abs(sd)
    assert _scale_err(s1["field"].cpu().numpy(), f_sm) < 1e-5
    # contouring of the CUDA smoothed field
    o = surf.contour(prm, s1["field"].cpu().numpy(), act_or)
    assert sr.num_vertices[None] == len(o["vertices"]) > 0
    assert sr.num_indices[None] == len(o["indices"])
    assert np.array_equal(sr.mesh_index.cpu().numpy(), o["indices"])
    assert np.abs(sr.mesh_vertex.cpu().numpy() - o["vertices"]).max() < 1e-6
    assert np.abs(sr.mesh_normal.cpu().numpy() - o["normals"]).max() < 1e-4


def test_surface_end_to_end_closed_mesh(cuda_lib, surf):
    pos = ball(seed=12)
    sr = _tool()
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=torch.from_numpy(pos).cuda())
    f = sr.mesh_index.cpu().numpy().reshape(-1, 3)
    nv = sr.num_vertices[None]
    assert closed_oriented(f, nv) and len(f) == 2 * nv - 4
    o = surf.dual_contouring(default_params(), pos)
    assert abs(nv - len(o["vertices"])) <= max(2, nv // 1000)
    # the same bits on a second run (fixed-point splats)
    v1 = sr.mesh_vertex.clone()
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=torch.from_numpy(pos).cuda())
    assert torch.equal(v1, sr.mesh_vertex)


def test_surface_export_ply(cuda_lib, tmp_path):
    pos = block(seed=13)
    sr = _tool()
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=pos)
    path = str(tmp_path / "mesh.ply")
    sr.export_mesh(path, output_normal=True)
    raw = open(path, "rb").read()
    head, body = raw.split(b"end_header\n", 1)
    nv, nf = sr.num_vertices[None], sr.num_indices[None] // 3
    assert f"element vertex {nv}".encode() in head and f"element face {nf}".encode() in head
    assert len(body) == nv * 24 + nf * 13
    v = np.frombuffer(body[: nv * 24], "<f4").reshape(nv, 6)
    assert np.array_equal(v[:, :3], sr.mesh_vertex.cpu().numpy())


def test_surface_errors(cuda_lib):
    from nonnewton_b200 import _abi
    from nonnewton_b200.engine import NNError
    from nonnewton_b200.surface import SRTool

    pos = ball(seed=14)
    bad = pos.copy()
    bad[3] = [-0.5, 0.5, 0.5]
    sr = _tool()
    with pytest.raises(NNError) as e:
        sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(bad), pos=bad)
    assert e.value.code == _abi.NN_ERR_INVALID_ARG
    small = SRTool([[0, 0, 0], [1, 1, 1]], voxel_size=0.01, particle_radius=0.02, max_num_vertices=100,
                   max_num_indices=600, max_num_particles=10000)
    with pytest.raises(NNError) as e:
        small.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=pos)
    assert e.value.code == _abi.NN_ERR_CAPACITY
    # the context stays usable after an error
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=pos)
    assert sr.num_vertices[None] > 0


def test_surface_velocity_matches_oracle(cuda_lib, surf, tmp_path):
    """SRTool(record_velocity=True): the vertex velocity splat and the mesh velocities
    (process_velocity) against the oracle at the CUDA mesh's vertices, 1e-5 of the
    velocities' scale; the mesh itself is the one a run without velocities makes."""
    pos = ball(seed=15)
    rng = np.random.default_rng(16)
    vel = (rng.normal(size=pos.shape) + np.array([0.0, -1.0, 0.5])).astype(np.float32)
    sr = _tool(record_velocity=True)
    sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=torch.from_numpy(pos).cuda(),
                       velocity=torch.from_numpy(vel).cuda())
    plain = _tool()
    plain.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=torch.from_numpy(pos).cuda())
    assert torch.equal(sr.mesh_vertex, plain.mesh_vertex) and torch.equal(sr.mesh_index, plain.mesh_index)
    nv = sr.num_vertices[None]
    assert nv > 0 and sr.mesh_velocity.shape == (nv, 3)
    vf = surf.vel_field(sr.last_params, pos, vel)
    ref = surf.mesh_velocity(sr.last_params, vf, sr.mesh_vertex.cpu().numpy())
    assert _scale_err(sr.mesh_velocity.cpu().numpy(), ref) < 1e-5
    # PLY with normals and velocities
    path = str(tmp_path / "vel.ply")
    sr.export_mesh(path, output_normal=True, output_velocity=True)
    head, body = open(path, "rb").read().split(b"end_header\n", 1)
    assert b"property float vx" in head
    v = np.frombuffer(body[: nv * 36], "<f4").reshape(nv, 9)
    assert np.array_equal(v[:, 6:], sr.mesh_velocity.cpu().numpy())
    # a tool without velocity recording refuses to export them; one with it needs them
    with pytest.raises(RuntimeError):
        plain.export_mesh(str(tmp_path / "x.ply"), output_velocity=True)
    with pytest.raises(ValueError):
        sr.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=pos)


@pytest.mark.parametrize("case", ["ball", "block"])
def test_marching_cubes_matches_oracle(cuda_lib, surf, case):
    """SRTool.marching_cubes: on the CUDA path's smoothed field, the oracle's marching
    cubes gives the same triangles index for index, vertices within 1e-6 m and normals
    within 1e-4; the mesh closes once the per-cube vertices are welded, with dual
    contouring's orientation; mesh velocities match the oracle's (1e-5 of scale)."""
    from .surf_cases import signed_volume, weld

    pos = ball(seed=17) if case == "ball" else block(seed=18)
    n = len(pos)
    vel = np.random.default_rng(19).normal(size=pos.shape).astype(np.float32)
    sr = _tool(record_velocity=True, max_num_vertices=400000)
    sr.marching_cubes(isolevel=0.0, smooth_radius=0.06, num_particles=n, pos=torch.from_numpy(pos).cuda(),
                      velocity=torch.from_numpy(vel).cuda())
    prm = sr.last_params
    s1 = sr.stage(1, n)
    o = surf.marching_cubes(prm, s1["field"].cpu().numpy(), s1["active"].cpu().numpy())
    nv = sr.num_vertices[None]
    assert nv == len(o["vertices"]) > 0 and sr.num_indices[None] == len(o["indices"])
    assert np.array_equal(sr.mesh_index.cpu().numpy(), o["indices"])
    vg = sr.mesh_vertex.cpu().numpy()
    assert np.abs(vg - o["vertices"]).max() < 1e-6
    assert np.abs(sr.mesh_normal.cpu().numpy() - o["normals"]).max() < 1e-4
    v, f = weld(vg, sr.mesh_index.cpu().numpy())
    assert closed_oriented(f, len(v))
    dc = _tool()
    dc.dual_contouring(isolevel=0.0, smooth_radius=0.06, num_particles=n, pos=torch.from_numpy(pos).cuda())
    vd = signed_volume(dc.mesh_vertex.cpu().numpy(), dc.mesh_index.cpu().numpy())
    assert vd > 0 and abs(signed_volume(vg, sr.mesh_index.cpu().numpy()) - vd) < 0.03 * vd
    ref = surf.mesh_velocity(prm, surf.vel_field(prm, pos, vel), vg)
    assert _scale_err(sr.mesh_velocity.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("method", ["dual_contouring", "marching_cubes"])
def test_surface_empty_and_single_particle(cuda_lib, surf, method):
    """No particles: an empty mesh. One particle: the pre-pass skips particle 0
    (srtool.py:1013), so only the isotropic splat runs, the field has no negative
    value and no surface results, as in the oracle. The tool stays usable after both."""
    sr = _tool()
    run = getattr(sr, method)
    run(isolevel=0.0, smooth_radius=0.06, num_particles=0, pos=np.zeros((0, 3), np.float32))
    assert sr.num_vertices[None] == 0 and sr.num_indices[None] == 0 and sr.mesh_vertex.shape == (0, 3)
    one = np.array([[0.5, 0.5, 0.5]], np.float32)
    run(isolevel=0.0, smooth_radius=0.06, num_particles=1, pos=one)
    o = surf.dual_contouring(sr.last_params, one)
    assert sr.num_vertices[None] == len(o["vertices"]) == 0 and sr.num_indices[None] == 0
    pos = ball(seed=20)
    run(isolevel=0.0, smooth_radius=0.06, num_particles=len(pos), pos=pos)
    assert sr.num_vertices[None] > 0


def test_surface_torus_from_a_field_object(cuda_lib, surf):
    """The reference example hands SRTool a Taichi vector field; anything with
    to_numpy() is taken. The torus closes with genus one under both methods, and dual
    contouring matches the oracle's vertex and triangle counts."""
    from .surf_cases import weld

    class Field:  # the part of ti.Vector.field that SRTool reads
        def __init__(self, a):
            self._a = a

        def to_numpy(self):
            return self._a.copy()

    pos = torus()
    sr = _tool()
    sr.dual_contouring(isolevel=0, smooth_radius=0.06, num_particles=len(pos), pos=Field(pos))
    nv, f = sr.num_vertices[None], sr.mesh_index.cpu().numpy().reshape(-1, 3)
    o = surf.dual_contouring(default_params(), pos)
    assert abs(nv - len(o["vertices"])) <= 2 and closed_oriented(f, nv) and len(f) == 2 * nv
    sr.marching_cubes(isolevel=0, smooth_radius=0.06, num_particles=len(pos), pos=Field(pos))
    v, f = weld(sr.mesh_vertex.cpu().numpy(), sr.mesh_index.cpu().numpy())
    assert closed_oriented(f, len(v)) and len(f) == 2 * len(v)


def test_surface_matches_the_reference_run(cuda_lib):
    """The CUDA surface stages against the reference's own SRTool run
    (tests/golden/ref_surface.npz, srtool.py through the Taichi stand-in): G and x_bar
    within 1e-4 of scale, the same active blocks, the splat field within 3e-4 and the
    smoothed field within 2e-4 of scale (the reference sums its splats in f32), sd 1e-4."""
    import os

    from nonnewton_b200.surface import SRTool

    R = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_surface.npz"))
    vs, r, srad, iso = (float(v) for v in R["params"])
    pos = R["pos"]
    sr = SRTool([[0, 0, 0], [1, 1, 1]], voxel_size=vs, particle_radius=r, max_num_vertices=20000,
                max_num_indices=200000, max_num_particles=len(pos))
    assert sr.grid_dims(srad) == [int(d) for d in R["dims"]]
    sr.dual_contouring(isolevel=iso, smooth_radius=srad, num_particles=len(pos), pos=pos)
    s0, s1 = sr.stage(0, len(pos)), sr.stage(1, len(pos))
    assert _scale_err(s0["G"].cpu().numpy(), R["G"]) < 1e-4 and _scale_err(s0["xbar"].cpu().numpy(), R["xbar"]) < 1e-4
    dims = [int(d) for d in R["dims"]]
    nb = [-(-d // 32) for d in dims]
    act = s0["active"].cpu().numpy().reshape(nb[2], nb[1], nb[0])
    assert np.array_equal(np.argwhere(act)[:, ::-1], R["blocks"])
    assert _scale_err(s0["field"].cpu().numpy(), R["field_splat"]) < 3e-4
    assert abs(s1["sd"] - float(R["sd"])) < 1e-4 * float(R["sd"])
    assert _scale_err(s1["field"].cpu().numpy(), R["field_smooth"]) < 2e-4
