"""CUDA path vs the CPU oracle for the non-Newtonian, implicit viscosity, elasticity,
CFL and batching parts of the step (per step from identical input states, 1e-4 of
each field's scale unless stated)."""
import os

import numpy as np
import pytest

from nonnewton_b200 import _abi
from nonnewton_b200 import scene as S
from nonnewton_b200.config import Parameter, SimConfig

from .helpers import gpu_sim, oracle_sim, pd_field, rel_err

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4


def _lockstep(sc, steps, fields, tol=TOL, nf_fields=("density",), cg=False, extra=None):
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    nf = sc.particles.n_fluid
    for k in range(steps):
        o.set("x", pd_field(m, "x"))
        o.set("v", pd_field(m, "v"))
        solver.step()
        o.step(1)
        gs, os_ = m.engine.stats(0), o.stats()
        assert (gs["iterations_v"], gs["iterations"]) == (os_["iterations_v"], os_["iterations"]), (k, gs, os_)
        if cg:
            assert abs(gs["cg_iterations"] - os_["cg_iterations"]) <= 1, (k, gs, os_)
        for name in fields:
            g, r = pd_field(m, name), o.get(name)
            if name in nf_fields:
                g, r = g[:nf], r[:nf]
            e = rel_err(g, r)
            assert e < tol, f"step {k} {name}: {e:.2e}"
        if extra:
            extra(m, o, k)
    return m, o


def _small_drop(quirks=False, law="CROSS_", implicit=True, boundary=0.0):
    fcfg = {"nonNewtonMethod": law, "viscosity0": 10.0, "viscosity_inf": 0.01, "consistency_index": 1.0,
            "power_index": 0.8, "viscoMaxError": 1e-4, "viscoMaxIter": 200, "viscosityBoundary": boundary}
    if implicit:
        fcfg["viscosityMethod"] = 13
    return S.dam_break(seed=5, n_side=(9, 9, 9), box=0.4, quirks=quirks,
                       extra_cfg={"useNonNewtonianModel": True}, fluid_cfg=fcfg)


@pytest.mark.parametrize("quirks", [False, True])
def test_nonnewton_strain_rate_and_law(cuda_lib, quirks):
    sc = _small_drop(quirks=quirks, implicit=False)
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    rng = np.random.default_rng(3)
    v = rng.normal(0, 0.2, size=(sc.particles.n, 3)).astype(np.float32)
    v[sc.particles.n_fluid:] = 0
    import torch
    m.pd.v.copy_(torch.from_numpy(v))
    o.set("v", v)
    for p in (_abi.NN_PASS_DENSITIES, _abi.NN_PASS_CLEAR_ACCELERATIONS, _abi.NN_PASS_NON_PRESSURE_FORCES):
        m.engine.run_pass(p)
        o.run_pass(p)
    n = sc.particles.n if quirks else sc.particles.n_fluid
    for name in ("strain_rate_norm", "nonnewton_viscosity", "acceleration"):
        e = rel_err(pd_field(m, name)[:n], o.get(name)[:n])
        assert e < TOL, f"{name}: {e:.2e}"


@pytest.mark.parametrize("law", ["POWER_LAW_", "CROSS_", "CASSON_", "CARREAU_", "BINGHAM_", "HERSCHEL_BULKLEY_"])
def test_viscosity_laws(cuda_lib, law):
    sc = _small_drop(law=law, implicit=False)
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    rng = np.random.default_rng(4)
    v = rng.normal(0, 0.5, size=(sc.particles.n, 3)).astype(np.float32)
    v[sc.particles.n_fluid:] = 0
    import torch
    m.pd.v.copy_(torch.from_numpy(v))
    o.set("v", v)
    for p in (_abi.NN_PASS_DENSITIES, _abi.NN_PASS_NON_PRESSURE_FORCES):
        m.engine.run_pass(p)
        o.run_pass(p)
    nf = sc.particles.n_fluid
    g, r = pd_field(m, "nonnewton_viscosity")[:nf], o.get("nonnewton_viscosity")[:nf]
    ok = np.isfinite(r)
    assert np.all(np.isfinite(g[ok]))
    assert np.abs(g[ok] - r[ok]).max() <= 1e-4 * np.abs(r[ok]).max()


def test_implicit_viscosity_step(cuda_lib):
    sc = _small_drop(implicit=True)
    m, o = _lockstep(sc, 6, ["x", "v", "acceleration", "nonnewton_viscosity"], cg=True,
                     nf_fields=("density", "nonnewton_viscosity"))
    gs = m.engine.stats(0)
    assert gs["cg_iterations"] >= 1 and gs["cg_residual"] <= 1e-4


def test_implicit_viscosity_damps_shear(cuda_lib):
    """Physical check of the Weiler solve: with a shear flow (plus the pressure
    transient of the dam break's walls) the kinetic energy after 5 steps decreases
    with the viscosity, and the implicit step stays stable at dt * nu / h^2 = 62."""
    energies = []
    for mu0 in (1.0, 1000.0, 1e5):
        sc = S.dam_break(seed=6, n_side=(10, 10, 10), box=0.4, extra_cfg={"useSurfaceTensionModel": False,
                                                                          "gravitation": [0, 0, 0]},
                         fluid_cfg={"viscosityMethod": 13, "viscoMaxError": 1e-5, "viscoMaxIter": 500,
                                    "nonNewtonMethod": "NEWTONIAN_", "viscosity0": mu0})
        sc.config["Configuration"]["useNonNewtonianModel"] = True
        sc = S.Scene(sc.name, sc.config, Parameter.from_config(SimConfig(config=sc.config)), sc.particles, 1)
        m, solver = gpu_sim(sc)
        solver.initialize()
        import torch
        x = m.pd.x.clone()
        v = torch.zeros_like(x)
        nf = sc.particles.n_fluid
        v[:nf, 0] = 0.5 * (x[:nf, 1] - x[:nf, 1].mean()) / 0.2
        m.pd.v.copy_(v)
        e0 = float((v[:nf] ** 2).sum())
        for _ in range(5):
            solver.step()
        e1 = float((m.pd.v[:nf] ** 2).sum())
        assert np.isfinite(e1)
        energies.append(e1 / e0)
    assert energies[1] < energies[0]
    assert energies[2] < energies[0]  # stable (and still damped) far past the explicit limit


def _elastic_scene(quirks):
    x = np.load(os.path.join(GOLD, "deformable_343.npy")).astype(np.float64)
    conf = {"Configuration": {"domainStart": [0, 0, 0], "domainEnd": [2, 2, 2], "particleRadius": 0.025,
                              "density0": 1000, "simulationMethod": 4, "gravitation": [0, -9.81, 0],
                              "timeStepSize": 1e-3, "referenceQuirks": quirks},
            "SolidParticles": [{"solidType": "ELASTIC", "youngsModulus": 250000.0, "poissonsRatio": 0.33}]}
    param = Parameter.from_config(SimConfig(config=conf), quirks=quirks)
    ps = S.assemble([S.PhaseInfo(uid=3000, material=1, is_dynamic=True, pos=x, solid_type=S.ELASTIC)], param)
    return S.Scene("deformable", conf, param, ps, 10)


@pytest.mark.parametrize("quirks", [False, True])
def test_elastic_fixture(cuda_lib, quirks):
    """test_deformable.ply (the reference's elastic fixture) falling under gravity with
    a twist (no strain: corotational) plus a stretch along x (strain): rotations, stress
    and the elastic accelerations per step."""
    sc = _elastic_scene(quirks)
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc)
    o.initialize()
    import torch
    x = m.pd.x.clone()
    c = x.mean(0)
    w = torch.tensor([0.0, 2.0, 0.0], device=x.device)
    v = torch.cross(w.expand_as(x), x - c, dim=1)
    v[:, 0] += 2.0 * (x[:, 0] - c[0])
    m.pd.v.copy_(v)
    # step 0 computes the stress of the undeformed body (zero up to rounding), so each
    # field's scale has a floor: 1 Pa for the stress (E = 2.5e5 Pa), 1 for the rest
    floors = {"x": 1.0, "v": 1.0, "acceleration": 1.0, "stress": 1.0, "rotations": 1.0}
    for k in range(5):
        o.set("x", pd_field(m, "x"))
        o.set("v", pd_field(m, "v"))
        solver.step()
        o.step(1)
        for name, fl in floors.items():
            r = o.get(name)
            e = rel_err(pd_field(m, name), r, scale=max(np.abs(r).max(), fl))
            assert e < TOL, f"step {k} {name}: {e:.2e}"
    assert np.abs(o.get("stress")).max() > 100.0  # the stretch did strain the body


def test_fluid_elastic_coupling(cuda_lib):
    """Elastic block over a fluid pool with two-way pressure coupling (pushes gathered
    by the solid particles) and per-phase rest density."""
    sc = S.fluid_elastic(n_el=6)
    # shrink the tank for a test-sized scene
    ps = sc.particles
    keep = np.ones(ps.n, bool)
    fl = np.nonzero(ps.material == 0)[0]
    keep[fl[(ps.x[fl, 1] > 0.3)]] = False
    sub = S.ParticleSet(x=ps.x[keep], material=ps.material[keep], is_dynamic=ps.is_dynamic[keep],
                        phase_id=ps.phase_id[keep], mass=ps.mass[keep], n_fluid=int((ps.material[keep] == 0).sum()))
    sc = S.Scene(sc.name, sc.config, sc.param, sub, 5)
    m, o = _lockstep(sc, 4, ["x", "v", "acceleration"], cg=True)
    el = np.nonzero(sub.phase_id >= 3000)[0]
    assert np.abs(pd_field(m, "acceleration")[el]).max() > 0


def test_cfl_time_step(cuda_lib):
    sc = S.dam_break(seed=7, n_side=(8, 8, 8), box=0.3,
                     extra_cfg={"cflMethod": 1, "cflFactor": 1.0, "cflMaxTimeStepSize": 2e-3,
                                "cflMinTimeStepSize": 1e-5})
    m, o = _lockstep(sc, 8, ["x", "v"])
    assert abs(m.engine.stats(0)["dt"] - o.stats()["dt"]) <= 1e-7 * o.stats()["dt"] + 1e-12


def test_batch_equals_alone(cuda_lib):
    """Scenes packed in one segmented array give the same result as each alone."""
    from nonnewton_b200.batch import Batch

    scenes = [S.dam_break(seed=21, n_side=(8, 9, 10), box=0.36),
              _small_drop(implicit=True),
              S.dam_break(seed=22, n_side=(6, 6, 6), box=0.3, quirks=True)]
    alone = []
    for sc in scenes:
        b = Batch(sc.particles.n, 1)
        b.set([sc])
        b.step(5)
        alone.append(b.scene_view(0, "x").cpu().numpy())
    b = Batch(sum(sc.particles.n for sc in scenes), 4)
    b.set(scenes)
    b.step(5)
    for k, sc in enumerate(scenes):
        x = b.scene_view(k, "x").cpu().numpy()
        assert np.abs(x - alone[k]).max() <= 1e-6, k


@pytest.mark.parametrize("coupling", [1, 2])
def test_rigid_body_coupling(cuda_lib, coupling):
    """Rigid cube dropped into fluid: shape matching and two-way pressure coupling
    per step from identical inputs."""
    sc = S.rigid_drop(seed=3, coupling=coupling)
    m, o = _lockstep(sc, 8, ["x", "v", "acceleration"])
    rb = np.nonzero(sc.particles.phase_id == 2000)[0]
    assert np.abs(pd_field(m, "acceleration")[rb]).max() > 0
