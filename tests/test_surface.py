"""The CPU oracle of the surface reconstruction (SRTool, SPH/surf_recon/srtool.py)
on known shapes: closed, consistently oriented meshes around particle balls and an
analytic sphere, the reference's quirks (particle 0 skipped, no surface without
negative field values). No GPU."""
import numpy as np
import pytest

from .surf_cases import ball, block, closed_oriented, default_params, torus


@pytest.fixture(scope="module")
def surf():
    from oracle import surf as S

    S.build()
    return S


def test_oracle_ball_is_a_closed_sphere(surf):
    pos = ball(seed=0)
    o = surf.dual_contouring(default_params(), pos)
    v, f = o["vertices"], o["indices"].reshape(-1, 3)
    assert len(v) > 1000
    assert closed_oriented(f, len(v))
    assert len(f) == 2 * len(v) - 4  # Euler characteristic 2
    r = np.linalg.norm(v - 0.5, axis=1)
    assert 0.10 < r.min() and r.max() < 0.16
    assert np.isfinite(o["sd"]) and o["sd"] > 0


def test_oracle_block_is_closed(surf):
    o = surf.dual_contouring(default_params(), block(seed=1))
    f = o["indices"].reshape(-1, 3)
    assert len(f) > 0 and closed_oriented(f, len(o["vertices"]))


def test_oracle_contour_of_an_analytic_sphere(surf):
    """Dual contouring of a signed distance field (negative inside): every vertex lies
    within a voxel of the sphere and the mesh is closed with consistent winding."""
    prm = default_params(dims=(48, 48, 48))
    vs = prm.voxel_size
    idx = np.stack(np.meshgrid(*[np.arange(48)] * 3, indexing="ij"), -1)  # x, y, z
    c, R = np.array([0.24, 0.23, 0.25]), 0.13
    sdf = np.linalg.norm(idx * vs - c, axis=-1) - R
    o = surf.contour(prm, np.transpose(sdf, (2, 1, 0)), np.ones(8, np.uint8))
    v, f = o["vertices"], o["indices"].reshape(-1, 3)
    assert closed_oriented(f, len(v))
    assert np.abs(np.linalg.norm(v - c, axis=1) - R).max() < vs


def test_oracle_particle_zero_is_skipped(surf):
    """pre_process_data starts at particle 1 (srtool.py:1013): G and x_bar of particle 0
    stay 0, every other particle gets a symmetric positive definite G."""
    G, xb = surf.prepass(default_params(), ball(seed=2))
    assert np.all(G[0] == 0) and np.all(xb[0] == 0)
    M = G[1:].reshape(-1, 3, 3).astype(np.float64)
    assert np.allclose(M, np.transpose(M, (0, 2, 1)), rtol=1e-5, atol=1e-3)
    assert np.all(np.linalg.eigvalsh(M) > 0)


def test_oracle_isotropic_field_alone_gives_no_surface(surf):
    """Without the anisotropic splat the field has no negative value, the smoothing's
    standard deviation is 0/0 and the field turns NaN, so no cube crosses the level,
    which is what the reference computes (density_field_stats, srtool.py:1436-1456)."""
    o = surf.dual_contouring(default_params(use_smooth_field=False), ball(seed=3))
    assert np.isnan(o["sd"])
    assert len(o["vertices"]) == 0 and len(o["indices"]) == 0


def test_oracle_rejects_particles_outside_the_grid(surf):
    pos = ball(seed=4)
    pos[5] = [-1.0, 0.5, 0.5]
    with pytest.raises(RuntimeError):
        surf.dual_contouring(default_params(), pos)


def test_oracle_velocity_field_of_a_uniform_flow(surf):
    """A uniform particle velocity u gives vertex velocities u * W, W the poly6
    weight sum (srtool.py:1159-1190), and mesh velocities that are trilinear blends
    of those (process_velocity, srtool.py:1351-1381): exact at grid vertices."""
    pos = block(seed=21, n=(5, 4, 3))
    prm = default_params()
    u = np.array([0.5, -2.0, 0.25], np.float32)
    vf = surf.vel_field(prm, pos, np.tile(u, (len(pos), 1))).reshape(3, -1)
    w = vf[0] / u[0]
    assert w.max() > 0
    assert np.allclose(vf[1], u[1] * w, rtol=1e-12, atol=0) and np.allclose(vf[2], u[2] * w, rtol=1e-12, atol=0)
    # linear in the velocities
    rng = np.random.default_rng(3)
    a, b = rng.normal(size=(2, len(pos), 3)).astype(np.float32)
    lin = surf.vel_field(prm, pos, a) + surf.vel_field(prm, pos, b) - surf.vel_field(prm, pos, (a + b))
    assert np.abs(lin).max() < 1e-6 * np.abs(surf.vel_field(prm, pos, a)).max()
    # at a grid vertex the blend is that vertex's velocity; half-way, the mean of two
    dims = list(prm.dims)
    k = int(np.argmax(w))
    z, y, x = np.unravel_index(k, (dims[2], dims[1], dims[0]))
    vs = prm.voxel_size
    pts = np.array([[x * vs, y * vs, z * vs], [(x + 0.5) * vs, y * vs, z * vs]], np.float64)
    mv = surf.mesh_velocity(prm, vf.reshape(-1), pts)
    assert np.allclose(mv[0], vf[:, k], rtol=1e-6)
    assert np.allclose(mv[1], 0.5 * (vf[:, k] + vf[:, k + 1]), rtol=1e-6)


def test_oracle_mc_table_is_a_set_of_disks_on_the_crossing_edges(surf):
    """The marching-cubes case table: every case's triangles use exactly its crossing
    edges; they form disks whose boundary runs along the cube's faces, as segments
    between two crossing edges of one face, once each; the count is #edges - 2 #loops."""
    from .surf_cases import CUBE_EDGE, CUBE_OFF

    nt, tris = surf.mc_table()
    assert nt[0] == 0 and nt[255] == 0 and nt.max() <= 5
    for ci in range(256):
        inside = [(ci >> c) & 1 for c in range(8)]
        cross = {w for w in range(12) if inside[CUBE_EDGE[w][0]] != inside[CUBE_EDGE[w][1]]}
        t = tris[ci, : nt[ci]]
        assert np.all(tris[ci, nt[ci]:] == -1)
        assert set(t.reshape(-1).tolist()) == cross
        directed = [(a, b) for tr in t for a, b in ((tr[0], tr[1]), (tr[1], tr[2]), (tr[2], tr[0]))]
        assert len(set(directed)) == len(directed)
        boundary = [(a, b) for a, b in directed if (b, a) not in directed]
        # each crossing edge starts one boundary segment and ends one
        assert sorted(a for a, _ in boundary) == sorted(cross) == sorted(b for _, b in boundary)
        for a, b in boundary:  # a segment lies on a face: the two edges share a face
            ca, cb = CUBE_OFF[CUBE_EDGE[a]], CUBE_OFF[CUBE_EDGE[b]]
            assert any(np.all(ca[:, k] == ca[0, k]) and np.all(cb[:, k] == ca[0, k]) for k in range(3))
        nxt = dict(boundary)
        loops, seen = 0, set()
        for e in cross:
            if e in seen:
                continue
            loops += 1
            while e not in seen:
                seen.add(e)
                e = nxt[e]
        assert nt[ci] == len(cross) - 2 * loops


def test_oracle_marching_cubes_closes_around_the_ball(surf):
    """Marching cubes on the ball's field: closed and consistently wound once the per-cube
    vertices are welded, genus 0, and the same orientation and volume as dual contouring."""
    from .surf_cases import signed_volume, weld

    prm = default_params()
    o = surf.dual_contouring(prm, ball(seed=0))
    mc = surf.marching_cubes(prm, o["field"], o["active"])
    v, f = weld(mc["vertices"], mc["indices"])
    assert len(f) > 1000 and closed_oriented(f, len(v)) and len(f) == 2 * len(v) - 4
    vd = signed_volume(o["vertices"], o["indices"])
    vm = signed_volume(mc["vertices"], mc["indices"])
    assert vd > 0 and abs(vm - vd) < 0.02 * vd


def test_oracle_marching_cubes_of_an_analytic_sphere(surf):
    """Every marching-cubes vertex of a sphere's signed distance field lies on an edge
    crossing, within a small fraction of a voxel of the sphere."""
    from .surf_cases import weld

    prm = default_params(dims=(48, 48, 48))
    vs = prm.voxel_size
    idx = np.stack(np.meshgrid(*[np.arange(48)] * 3, indexing="ij"), -1)
    c, R = np.array([0.24, 0.23, 0.25]), 0.13
    sdf = np.linalg.norm(idx * vs - c, axis=-1) - R
    o = surf.marching_cubes(prm, np.transpose(sdf, (2, 1, 0)), np.ones(8, np.uint8))
    assert np.abs(np.linalg.norm(o["vertices"] - c, axis=1) - R).max() < 0.05 * vs
    # a sphere through grid vertices puts several edges' crossings on one point; move it
    # off the vertices before welding
    c, R = np.array([0.2413, 0.2327, 0.2491]), 0.1307
    sdf = np.linalg.norm(idx * vs - c, axis=-1) - R
    o = surf.marching_cubes(prm, np.transpose(sdf, (2, 1, 0)), np.ones(8, np.uint8))
    v, f = weld(o["vertices"], o["indices"])
    assert closed_oriented(f, len(v)) and len(f) == 2 * len(v) - 4


def test_oracle_torus_has_genus_one(surf):
    """The reference example's shape: a solid torus of lattice particles gives a closed
    mesh whose Euler characteristic is 0 (F = 2V), the hole kept open."""
    o = surf.dual_contouring(default_params(), torus())
    f, nv = o["indices"].reshape(-1, 3), len(o["vertices"])
    assert nv > 1000 and closed_oriented(f, nv) and len(f) == 2 * nv
