"""The CPU oracle pinned against the golden fixtures and an independent numpy
restatement of single passes (no GPU)."""
import json
import math
import os

import numpy as np
import pytest

from nonnewton_b200 import _abi
from nonnewton_b200 import scene as S
from nonnewton_b200.config import Parameter, SimConfig

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _single_fluid_scene(x, r, quirks=False, **cfg):
    conf = {"Configuration": {"domainStart": [0, 0, 0], "domainEnd": [1, 1, 1], "particleRadius": r,
                              "density0": 1000, "simulationMethod": 4, "gravitation": [0, -9.81, 0],
                              "timeStepSize": 1e-3, **cfg}, "FluidParticles": [{}]}
    param = Parameter.from_config(SimConfig(config=conf), quirks=quirks)
    ps = S.assemble([S.PhaseInfo(uid=0, material=0, is_dynamic=True, pos=np.asarray(x, np.float64))], param)
    return conf, param, ps


def test_neighbors_9pt_golden(oracle_lib):
    g = json.load(open(os.path.join(GOLD, "neighbor_9pt.json")))
    _, param, ps = _single_fluid_scene(g["x"], g["particle_radius"])
    o = oracle_lib.OracleSim(ps, param)
    o.run_pass(_abi.NN_PASS_SEARCH)
    num, lists = o.neighbors(60)
    assert num.tolist() == g["num_neighbors"]
    for i, row in enumerate(g["neighbors"]):
        assert lists[i, : len(row)].tolist() == row and np.all(lists[i, len(row):] == -1)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_lattice_kat(oracle_lib, precision):
    g = json.load(open(os.path.join(GOLD, "lattice_kat.json")))
    r, n = g["particle_radius"], g["n_side"]
    idx = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = g["origin"] + idx * 2 * r
    _, param, ps = _single_fluid_scene(x, r)
    o = oracle_lib.OracleSim(ps, param, precision)
    o.run_pass(_abi.NN_PASS_SEARCH)
    o.run_pass(_abi.NN_PASS_DENSITIES)
    num, _ = o.neighbors(60)
    inter = np.array(g["interior_ids"])
    assert np.all(num[inter] == g["interior_neighbors"])
    rho = o.get("density")[inter]
    tol = 1e-5 if precision == "f32" else 1e-12
    assert np.abs(rho - g["rho_interior"]).max() / g["rho_interior"] < tol


def _np_kernel(r, h):
    k = 8 / math.pi / h ** 3
    q = r / h
    w = np.where(q <= 0.5, k * (6 * q ** 3 - 6 * q ** 2 + 1), np.where(q <= 1, 2 * k * (1 - q) ** 3, 0.0))
    return w


def _np_grad(rv, h):
    k = 6 * 8 / math.pi / h ** 3
    rn = np.linalg.norm(rv, axis=-1)
    q = rn / h
    f = np.where(q <= 0.5, k * q * (3 * q - 2), -k * (1 - q) ** 2)
    ok = (rn > 1e-5) & (q <= 1)
    safe = np.where(ok, rn * h, 1.0)
    return np.where(ok[..., None], rv / safe[..., None] * f[..., None], 0.0)


def test_oracle_matches_numpy_restatement(oracle_lib):
    """Densities, DFSPH factors and the divergence-free density change of the FP64
    oracle against a vectorised numpy restatement of SPH/main.py:962-1645."""
    sc = S.dam_break(seed=3, n_side=(6, 6, 6), box=0.24)
    ps, p = sc.particles, sc.param
    o = oracle_lib.OracleSim(ps, p, "f64")
    rng = np.random.default_rng(1)
    v = rng.normal(0, 0.05, size=(ps.n, 3))
    v[ps.material == 1] = 0
    o.set("v", v)
    o.run_pass(_abi.NN_PASS_SEARCH)
    o.run_pass(_abi.NN_PASS_STATIC_BOUNDARY_VOLUME)
    o.run_pass(_abi.NN_PASS_DENSITIES)
    o.run_pass(_abi.NN_PASS_DFSPH_FACTOR)
    num, lists = o.neighbors(64)
    x = ps.x.astype(np.float64)
    h = p.support_radius
    vol = o.get("volume")
    fluid = ps.material == 0
    # boundary volumes (SPH/main.py:1010-1019)
    for i in np.nonzero(~fluid)[0]:
        js = lists[i, : num[i]]
        js = js[~fluid[js]]
        d = _np_kernel(0.0, h) + _np_kernel(np.linalg.norm(x[i] - x[js], axis=1), h).sum()
        assert abs(vol[i] - 3.0 / d) < 1e-12 * vol[i]
    rho = o.get("density")
    alpha = o.get("dfsph_factor")
    for i in np.nonzero(fluid)[0][:100]:
        js = lists[i, : num[i]]
        rv = x[i] - x[js]
        w = _np_kernel(np.linalg.norm(rv, axis=1), h)
        r_np = 1000.0 * (vol[i] * _np_kernel(0.0, h) + (vol[js] * w).sum())
        assert abs(rho[i] - r_np) < 1e-9 * r_np
        g = _np_grad(rv, h) * vol[js, None]
        s = (g[fluid[js]] ** 2).sum() + (g.sum(0) ** 2).sum()
        a_np = -1.0 / s if s > 1e-6 else 0.0
        assert abs(alpha[i] - a_np) <= 1e-9 * abs(a_np)
    # density change (SPH/main.py:1610-1645)
    o.run_pass(_abi.NN_PASS_DIVERGENCE_SOLVE)


def test_oracle_f32_vs_f64(oracle_lib):
    sc = S.dam_break(seed=0, n_side=(8, 8, 8), box=0.3)
    a = oracle_lib.OracleSim(sc.particles, sc.param, "f32")
    b = oracle_lib.OracleSim(sc.particles, sc.param, "f64")
    for o in (a, b):
        o.initialize()
        o.step(5)
    assert np.abs(a.get("x") - b.get("x")).max() < 1e-5
    nf = sc.particles.n_fluid
    assert np.abs(a.get("density")[:nf] - b.get("density")[:nf]).max() / 1000 < 1e-4


def test_animation_moves_the_static_boundary_rigidly(oracle_lib):
    """animate_particles (SPH/main.py:283-309) adds the frame's displacement to every
    particle: the static boundary, which neither advects nor is clamped, moves by
    exactly that step's displacement (f32 additions), and only in the step it is set for."""
    sc = S.dam_break(seed=1, n_side=(6, 6, 6), box=0.3)
    o = oracle_lib.OracleSim(sc.particles, sc.param, "f32")
    o.initialize()
    nf = sc.particles.n_fluid
    x0 = o.get("x")[nf:].astype(np.float32)
    d = np.array([0.003, -0.002, 0.001], np.float32)
    o.set_animation(d)
    o.step(1)
    x1 = o.get("x")[nf:]
    assert np.array_equal(x1, (x0 + d).astype(np.float64))
    o.step(1)  # the displacement applies to one step only
    assert np.array_equal(o.get("x")[nf:], x1)


def test_polar_rotation(oracle_lib):
    rng = np.random.default_rng(0)
    for _ in range(50):
        A = rng.normal(size=(3, 3))
        R = oracle_lib.polar_rotation(A)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-10)
        assert abs(np.linalg.det(R) - 1) < 1e-10
        U, s, Vt = np.linalg.svd(A)
        D = np.diag([1, 1, np.sign(np.linalg.det(U @ Vt))])
        assert np.allclose(R, U @ D @ Vt, atol=1e-8)
    assert np.allclose(oracle_lib.polar_rotation(np.zeros((3, 3))), np.eye(3))


def test_reference_quirks_strain_rate(oracle_lib):
    """Quirk mode keeps only the last neighbour's term (SPH/main.py:488-490) and the
    Newtonian law (387-402); the corrected mode sums and applies the Cross law."""
    sc = S.dam_break(seed=0, n_side=(5, 5, 5), box=0.2, extra_cfg={"useNonNewtonianModel": True},
                     fluid_cfg={"nonNewtonMethod": "CROSS_", "viscosity0": 10.0, "viscosity_inf": 0.01,
                                "consistency_index": 1.0, "power_index": 0.8})
    rng = np.random.default_rng(0)
    v = rng.normal(0, 0.1, size=(sc.particles.n, 3))
    res = {}
    for q in (False, True):
        param = Parameter.from_config(SimConfig(config=sc.config), quirks=q)
        o = oracle_lib.OracleSim(sc.particles, param, "f64")
        o.set("v", v)
        o.run_pass(_abi.NN_PASS_SEARCH)
        o.run_pass(_abi.NN_PASS_DENSITIES)
        o.run_pass(_abi.NN_PASS_NON_PRESSURE_FORCES)
        res[q] = (o.get("strain_rate_norm"), o.get("nonnewton_viscosity"))
    assert np.all(res[True][1] == 10.0)
    nf = sc.particles.n_fluid
    mu = res[False][1][:nf]
    assert np.all(mu <= 10.0) and np.all(mu >= 0.01)
    assert not np.allclose(res[True][0][:nf], res[False][0][:nf])


def test_elastic_rest_state(oracle_lib):
    """Elastic block at rest: rotations stay identity, stress zero, no elastic force."""
    x = np.load(os.path.join(GOLD, "deformable_343.npy")).astype(np.float64)
    conf = {"Configuration": {"domainStart": [0, 0, 0], "domainEnd": [2, 2, 2], "particleRadius": 0.025,
                              "density0": 1000, "simulationMethod": 4, "gravitation": [0, 0, 0],
                              "timeStepSize": 1e-3},
            "SolidParticles": [{"solidType": "ELASTIC", "youngsModulus": 250000.0, "poissonsRatio": 0.33}]}
    param = Parameter.from_config(SimConfig(config=conf))
    ps = S.assemble([S.PhaseInfo(uid=3000, material=1, is_dynamic=True, pos=x, solid_type=S.ELASTIC)], param)
    o = oracle_lib.OracleSim(ps, param, "f64")
    o.initialize()
    o.run_pass(_abi.NN_PASS_CLEAR_ACCELERATIONS)
    o.run_pass(_abi.NN_PASS_ELASTICITY)
    R = o.get("rotations").reshape(-1, 3, 3)
    assert np.allclose(R, np.eye(3), atol=1e-9)
    assert np.abs(o.get("stress")).max() < 1e-6
    assert np.abs(o.get("acceleration")).max() < 1e-6


def test_rigid_body_stays_rigid(oracle_lib):
    """RigidBodySolver shape matching (SPH/main.py:1136-1158): after the step's
    projection the body's pairwise distances equal the rest ones; it falls."""
    sc = S.rigid_drop(seed=0)
    o = oracle_lib.OracleSim(sc.particles, sc.param, "f64")
    o.initialize()
    rb = np.nonzero(sc.particles.phase_id == 2000)[0]
    x0 = o.get("x")[rb]
    for _ in range(5):
        o.step(1)
        o.run_pass(_abi.NN_PASS_RIGID)  # project once more, after the advect of the step
        x = o.get("x")[rb]
        d0 = np.linalg.norm(x0[:, None] - x0[None], axis=-1)
        d1 = np.linalg.norm(x[:, None] - x[None], axis=-1)
        assert np.abs(d1 - d0).max() < 1e-9
    assert x[:, 1].mean() < x0[:, 1].mean()
