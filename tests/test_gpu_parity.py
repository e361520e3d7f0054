"""CUDA path vs the CPU oracle, through the reference-facing object API and the C ABI.

Tolerances: neighbour lists bit-exact as sorted id sets (pairs within 4 ulp of h are
excluded); FP32 fields within 1e-4 relative to the field's scale; iteration counts
equal.
"""
import json
import os

import numpy as np
import pytest

from nonnewton_b200 import _abi
from nonnewton_b200 import scene as S
from nonnewton_b200.config import Parameter, SimConfig

from .helpers import field_err, gpu_sim, near_cutoff_pairs, oracle_sim, pd_field, rel_err

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4


def _scene_9pt():
    g = json.load(open(os.path.join(GOLD, "neighbor_9pt.json")))
    conf = {"Configuration": {"domainStart": [0, 0, 0], "domainEnd": [0.1, 0.1, 0.1], "particleRadius": 0.01,
                              "density0": 1000, "simulationMethod": 4, "gravitation": [0, -9.81, 0],
                              "timeStepSize": 0.004}, "FluidParticles": [{}]}
    param = Parameter.from_config(SimConfig(config=conf))
    ps = S.assemble([S.PhaseInfo(uid=0, material=0, is_dynamic=True, pos=np.array(g["x"]))], param)
    return S.Scene("9pt", conf, param, ps, 1), g


def test_neighbors_9pt_golden(cuda_lib):
    sc, g = _scene_9pt()
    m, solver = gpu_sim(sc)
    m.ns.run_search()
    num = m.ns.num_neighbors.cpu().numpy()
    lists = m.ns.neighbors.cpu().numpy()
    assert num.tolist() == g["num_neighbors"]
    for i, row in enumerate(g["neighbors"]):
        assert lists[i, : len(row)].tolist() == row and np.all(lists[i, len(row):] == -1)


def test_lattice_kat(cuda_lib):
    g = json.load(open(os.path.join(GOLD, "lattice_kat.json")))
    r, n = g["particle_radius"], g["n_side"]
    idx = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = g["origin"] + idx * 2 * r
    conf = {"Configuration": {"domainStart": [0, 0, 0], "domainEnd": [1, 1, 1], "particleRadius": r,
                              "density0": 1000, "simulationMethod": 4, "timeStepSize": 1e-3},
            "FluidParticles": [{}]}
    param = Parameter.from_config(SimConfig(config=conf))
    ps = S.assemble([S.PhaseInfo(uid=0, material=0, is_dynamic=True, pos=x)], param)
    m, solver = gpu_sim(S.Scene("lat", conf, param, ps, 1))
    m.ns.run_search()
    solver.compute_densities()
    inter = np.array(g["interior_ids"])
    assert np.all(m.ns.num_neighbors.cpu().numpy()[inter] == 26)
    rho = pd_field(m, "density")[inter]
    assert np.abs(rho - g["rho_interior"]).max() / g["rho_interior"] < 1e-5


@pytest.mark.parametrize("seed", [0, 1])
def test_neighbor_lists_bit_exact(cuda_lib, seed):
    sc = S.dam_break(seed=seed, n_side=(12, 12, 12), box=0.4)
    m, solver = gpu_sim(sc)
    m.ns.run_search()
    o = oracle_sim(sc)
    o.run_pass(_abi.NN_PASS_SEARCH)
    on, ol = o.neighbors(60)
    gn = m.ns.num_neighbors.cpu().numpy()
    gl = m.ns.neighbors.cpu().numpy()
    ties = near_cutoff_pairs(sc.particles.x, sc.param.support_radius)
    bad = np.nonzero((gn != on) | np.any(gl != ol, axis=1))[0]
    tie_ids = {a for a, b in ties} | {b for a, b in ties}
    assert set(bad.tolist()) <= tie_ids, f"{len(bad)} rows differ outside cut-off ties"


def test_neighbor_lists_exact_at_the_cutoff(cuda_lib):
    """No tie exceptions: a fluid lattice at spacing h / 2, so that the pairs two steps
    apart along an axis sit at the cut-off, with every fluid coordinate moved by -3..3
    ulp at random, puts thousands of pairs within a few ulp of h. Both sides evaluate the
    reference's f32 expression with separately rounded operations (SPH/main.py:845; the
    list build two candidates at a time with packed f32x2 arithmetic), so the lists equal
    the oracle's exactly."""
    sc = S.dam_break(seed=0, n_side=(16, 16, 16), box=0.6, jitter=0.0)
    nf = sc.particles.n_fluid
    x = np.asarray(sc.particles.x, np.float32).copy()
    bits = x[:nf].view(np.int32)  # positive coordinates: +k on the bits is +k ulp
    bits += np.random.default_rng(5).integers(-3, 4, size=bits.shape, dtype=np.int32)
    sc.particles.x = x
    ties = near_cutoff_pairs(x, sc.param.support_radius)
    assert len(ties) > 1000, len(ties)
    m, solver = gpu_sim(sc)
    m.ns.run_search()
    o = oracle_sim(sc)
    o.run_pass(_abi.NN_PASS_SEARCH)
    on, ol = o.neighbors(60)
    gn = m.ns.num_neighbors.cpu().numpy()
    gl = m.ns.neighbors.cpu().numpy()
    bad = np.nonzero((gn != on) | np.any(gl != ol, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} rows differ ({len(ties)} pairs within 4 ulp of h)"


def test_nonpressure_terms_folded_or_not(cuda_lib):
    """The fluid's non-pressure terms (surface tension, strain rate and Cross law, the
    implicit viscosity's coefficients) come from the divergence loop's density change in
    the body predicted to be the last (as many bodies as in the step before), or from the
    force pass when the prediction misses. This dam break runs 1, 2, 1, 1, ... divergence
    loop bodies, so the first steps take both paths (hit, miss, miss, hit); every step
    matches the oracle's iteration counts and fields in lockstep."""
    sc = S.dam_break(seed=3, n_side=(12, 12, 12), box=0.4,
                     extra_cfg={"useNonNewtonianModel": True, "useSurfaceTensionModel": True},
                     fluid_cfg={"nonNewtonMethod": "CROSS_", "viscosity0": 1.0, "viscosity_inf": 0.001,
                                "consistency_index": 0.25, "power_index": 0.6, "viscosityMethod": 13,
                                "viscoMaxError": 1e-4})
    nf = sc.particles.n_fluid
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    folded = []
    for k in range(12):
        o.set("x", pd_field(m, "x"))
        o.set("v", pd_field(m, "v"))
        solver.step()
        o.step(1)
        gs, os_ = m.engine.stats(0), o.stats()
        assert gs["status"] == 0, (k, gs)
        assert (gs["iterations_v"], gs["iterations"]) == (os_["iterations_v"], os_["iterations"]), (k, gs, os_)
        assert abs(gs["cg_iterations"] - os_["cg_iterations"]) <= 1, (k, gs, os_)
        folded.append(gs["nonpressure_folded"])
        for name in ("x", "v", "acceleration", "density", "strain_rate_norm", "nonnewton_viscosity"):
            g, r = pd_field(m, name), o.get(name)
            if name in ("density", "strain_rate_norm", "nonnewton_viscosity"):
                g, r = g[:nf], r[:nf]
            e = rel_err(g, r)
            assert e < TOL, f"step {k} {name}: {e:.2e} (folded {folded[-1]})"
    print("non-pressure terms folded per step:", folded)
    assert 0 < sum(folded) < len(folded), folded


def _init_both(sc, **kw):
    m, solver = gpu_sim(sc, **kw)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    return m, solver, o


def _compare(m, o, names, nf=None, tol=TOL):
    for name in names:
        g = pd_field(m, name)
        r = o.get(name)
        if nf is not None and name in ("density", "dfsph_factor", "density_adv"):
            g, r = g[:nf], r[:nf]
        e = field_err(name, g, r)
        assert e < tol, f"{name}: rel err {e:.2e}"


def test_passes_one_by_one(cuda_lib):
    sc = S.dam_break(seed=0, n_side=(10, 10, 10), box=0.4)
    m, solver, o = _init_both(sc)
    nf = sc.particles.n_fluid
    _compare(m, o, ["volume"])
    rng = np.random.default_rng(0)
    v = rng.normal(0, 0.2, size=(sc.particles.n, 3)).astype(np.float32)
    v[nf:] = 0
    import torch
    m.pd.v.copy_(torch.from_numpy(v))
    o.set("v", v)
    for p, names in [(_abi.NN_PASS_CLEAR_ACCELERATIONS, ["acceleration"]),
                     (_abi.NN_PASS_DENSITIES, ["density"]),
                     (_abi.NN_PASS_DFSPH_FACTOR, ["dfsph_factor"]),
                     (_abi.NN_PASS_DIVERGENCE_SOLVE, ["v", "dfsph_factor", "density_adv"]),
                     (_abi.NN_PASS_CLEAR_ACCELERATIONS, ["acceleration"]),
                     (_abi.NN_PASS_NON_PRESSURE_FORCES, ["acceleration"]),
                     (_abi.NN_PASS_NON_PRESSURE_ADVECT, ["v"]),
                     (_abi.NN_PASS_PRESSURE_SOLVE, ["v", "dfsph_factor", "density_adv"]),
                     (_abi.NN_PASS_ADVECT, ["x", "v"]),
                     (_abi.NN_PASS_ENFORCE_BOUNDARY, ["x", "v"])]:
        m.engine.run_pass(p)
        o.run_pass(p)
        _compare(m, o, names, nf)
    gs, os_ = m.engine.stats(0), o.stats()
    assert gs["iterations_v"] == os_["iterations_v"] and gs["iterations"] == os_["iterations"]


@pytest.mark.parametrize("quirks", [False, True])
def test_step_parity(cuda_lib, quirks):
    """Each step starts from identical input states (the oracle takes the GPU's x, v)."""
    sc = S.dam_break(seed=0, n_side=(10, 10, 10), box=0.4, quirks=quirks)
    m, solver, o = _init_both(sc)
    nf = sc.particles.n_fluid
    for k in range(12):
        o.set("x", pd_field(m, "x"))
        o.set("v", pd_field(m, "v"))
        solver.step()
        o.step(1)
        gs, os_ = m.engine.stats(0), o.stats()
        assert (gs["iterations_v"], gs["iterations"]) == (os_["iterations_v"], os_["iterations"]), k
        _compare(m, o, ["x", "v", "acceleration", "density", "dfsph_factor", "density_adv"], nf)
        assert abs(gs["avg_density_err"] - os_["avg_density_err"]) <= 1e-4 * sc.param.density0


def test_trajectory_parity(cuda_lib):
    """Free-running 30 steps: summation-order differences compound, so the tolerance is
    1e-3 of the field scale; the final density error stays within the 0.1 % target."""
    sc = S.dam_break(seed=1, n_side=(10, 10, 10), box=0.4)
    m, solver, o = _init_both(sc)
    nf = sc.particles.n_fluid
    for _ in range(30):
        solver.step()
    o.step(30)
    _compare(m, o, ["x", "v", "density"], nf, tol=1e-3)
    assert m.engine.stats(0)["avg_density_err"] <= 0.1 * 0.01 * sc.param.density0 + 1e-9


def test_graph_equals_host_loop(cuda_lib):
    sc = S.dam_break(seed=2, n_side=(10, 10, 10), box=0.4)
    outs = []
    for host in (False, True):
        m, solver = gpu_sim(sc)
        solver.host_loop = host
        solver.initialize()
        for _ in range(5):
            solver.step()
        outs.append((pd_field(m, "x"), pd_field(m, "v")))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_resident_run_equals_steps(cuda_lib):
    sc = S.dam_break(seed=4, n_side=(10, 10, 10), box=0.4)
    m1, s1 = gpu_sim(sc)
    s1.initialize()
    for _ in range(6):
        s1.step()
    x1 = pd_field(m1, "x")
    m2, s2 = gpu_sim(sc)
    s2.initialize()
    s2.run(6)
    assert np.array_equal(x1, pd_field(m2, "x"))


@pytest.mark.parametrize("tuning", [dict(block=128, unroll=1, cell_factor=2), dict(block=512, unroll=2, cell_factor=1),
                                    dict(block=64, unroll=4, cell_factor=2),
                                    dict(block=128, unroll=2, cell_factor=1, x_split=2),
                                    dict(block=128, unroll=2, cell_factor=1, x_split=4),
                                    dict(block=256, unroll=4, cell_factor=2, x_split=3)])
def test_tuning_invariance(cuda_lib, tuning):
    """Launch shape and cell layout (cell factor, x cells per cell edge) change neither
    the neighbour sets nor (beyond summation-order rounding) the trajectory."""
    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    sc = S.dam_break(seed=9, n_side=(10, 10, 10), box=0.4)
    out = []
    for tn in (None, tuning):
        m = sph.initialize(SimConfig(config=sc.config), particles=sc.particles, tuning=tn)
        solver = sph.build_solver()
        m.ns.run_search()
        num, lists = m.ns.num_neighbors.cpu().numpy(), m.ns.neighbors.cpu().numpy()
        solver.initialize()
        for _ in range(5):
            solver.step()
        out.append((num, lists, pd_field(m, "x"), pd_field(m, "v")))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert np.abs(out[0][2] - out[1][2]).max() < 1e-6
    assert rel_err(out[1][3], out[0][3]) < 1e-4


@pytest.mark.parametrize("n_side", [(1, 1, 1), (1, 1, 2)])
def test_lone_particles_step_parity(cuda_lib, n_side):
    """One fluid particle (the reference's onepar.ply case) and a pair, in the corner of a
    boundary box: a particle without fluid neighbours has only its own density and the
    walls' contributions, which push it out of the corner; ten steps agree with the oracle."""
    sc = S.dam_break(seed=3, n_side=n_side, box=0.2)
    m, solver, o = _init_both(sc)
    nf = sc.particles.n_fluid
    for _ in range(10):
        solver.step()
    o.step(10)
    _compare(m, o, ["x", "v", "density", "dfsph_factor"], nf)
    gs, os_ = m.engine.stats(0), o.stats()
    assert (gs["iterations_v"], gs["iterations"]) == (os_["iterations_v"], os_["iterations"])
    assert gs["status"] == 0
    x = pd_field(m, "x")[:nf]
    assert np.all(np.isfinite(x)) and np.abs(x - sc.particles.x[:nf]).max() > 1e-3  # it moved


def test_animation_moves_the_boundary_too(cuda_lib):
    """animate_particles (SPH/main.py:283-309) through SPHBase.run: the frames of the
    table (two rows on frame 2, none on 1 and 3) shift every particle, the static
    boundary box included, between advection and the clamp; eight steps agree with the
    oracle given the same per-frame displacements."""
    from .helpers import frame_displacement

    sc = S.dam_break(seed=4, n_side=(8, 8, 8), box=0.3)
    m, solver, o = _init_both(sc)
    nf = sc.particles.n_fluid
    anime = (np.array([0, 2, 2, 4, 5, 6, 7], np.int64),
             np.array([[0.004, 0, 0], [0, 0.003, 0], [0, 0, -0.002], [-0.005, 0, 0.001], [0, -0.004, 0],
                       [0.002, 0.002, 0.002], [0, 0, 0.003]], np.float32))
    m.anime = anime
    x0 = pd_field(m, "x")[nf:]
    solver.run(8)
    for s in range(8):
        d = frame_displacement(anime, s)
        if d is not None:
            o.set_animation(d)
        o.step(1)
    _compare(m, o, ["x", "v", "density", "dfsph_factor"], nf)
    # the box moved as a whole by the table's total
    assert np.abs(pd_field(m, "x")[nf:] - x0 - anime[1].sum(0)).max() < 1e-5
    assert m.engine.stats(0)["status"] == 0


@pytest.mark.parametrize("name", ["dam", "nonnewton", "elastic", "rigid", "deformable", "neighbor9", "anime"])
def test_gpu_matches_the_reference_run(cuda_lib, name):
    """The CUDA step in the reference-quirks mode against the reference's own step
    (tests/golden/ref_<scene>.npz, SPH/main.py run through a Taichi stand-in), free
    running from the same initial state: every recorded field within 1e-4 of its scale."""
    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    from .helpers import reference_animation, reference_errors, reference_run, reference_steps

    R, cfg, param, ps = reference_run(name)
    m = sph.initialize(SimConfig(config=cfg), particles=ps, quirks=True)
    m.anime = reference_animation(R)  # what initialize reads from an animeFile
    solver = sph.build_solver()
    solver.initialize()
    for s in range(reference_steps(R)):
        solver.step()
        err = reference_errors(R, s, lambda k: pd_field(m, k), ps.n_fluid)
        assert err and max(err.values()) < TOL, (s, err)
    assert m.engine.stats(0)["status"] == 0


def test_crowded_cells(cuda_lib):
    """A cluster of 150 fluid particles in a cube of side h/4 (inside one cell) beside a
    normal fluid block in its box: the in-cell sort takes its warp path for the
    crowded cell. The neighbour sets equal the oracle's search, and three steps are
    deterministic (graph-driven and host-driven loops bit for bit) with a clean status."""
    import copy

    base = S.dam_break(seed=21, n_side=(8, 8, 8), box=0.3)
    h = base.param.support_radius
    rng = np.random.default_rng(21)
    cluster = np.array([0.2, 0.08, 0.2]) + rng.uniform(0.0, h / 4, size=(150, 3))
    conf = copy.deepcopy(base.config)
    conf["FluidParticles"] = [{}, {}]
    param = Parameter.from_config(SimConfig(config=conf))
    fl = base.particles.x[: base.particles.n_fluid]
    bd = base.particles.x[base.particles.n_fluid:]
    ps = S.assemble([S.PhaseInfo(uid=0, material=0, is_dynamic=True, pos=fl),
                     S.PhaseInfo(uid=1, material=0, is_dynamic=True, pos=cluster),
                     S.PhaseInfo(uid=1000, material=1, is_dynamic=False, pos=bd, solid_type=S.STATIC)], param)
    sc = S.Scene("crowded", conf, param, ps, 3)
    m, solver = gpu_sim(sc, max_neighbors=256)
    m.ns.run_search()
    gn, gl = m.engine.neighbors(ps.n, 256)
    o = oracle_sim(sc)
    o.run_pass(_abi.NN_PASS_SEARCH)
    on, ol = o.neighbors(256)
    assert int(gn.max()) >= 149  # the cluster's particles see each other
    assert np.array_equal(gn.cpu().numpy(), on) and np.array_equal(gl.cpu().numpy(), ol)
    outs = []
    for host in (False, True):
        m, solver = gpu_sim(sc, max_neighbors=256)
        solver.host_loop = host
        solver.initialize()
        for _ in range(3):
            solver.step()
        assert m.engine.stats(0)["status"] == 0
        outs.append((pd_field(m, "x"), pd_field(m, "v")))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
