"""Per-field error of the FP32 GPU step against FP64 runs, from identical initial
states, free-running:

  - against the FP64 build of the same CUDA kernels (libnnsph64.so: the same source
    with double arithmetic; the caller's float32 state is read once at the start and
    the run stays resident in double) on the benchmark scenes at their own sizes;
  - against the FP64 run of the same algorithm on the CPU (the oracle in double
    precision) on small scenes.

The bounds are the stated accuracy of the FP32 path; the measured values are printed
(pytest -s) and recorded in the design notes."""
import os

import numpy as np
import pytest

from nonnewton_b200 import scene as S

from .helpers import gpu_sim, oracle_sim, pd_field

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _err(g, r, nf=None):
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    return float(np.abs(g - r).max() / max(np.abs(r).max(), 1e-30))


@pytest.mark.parametrize("name,steps,bounds", [
    ("dam_break", 20, {"x": 1e-5, "v": 2e-3, "density": 1e-4}),
    ("drop_implicit", 10, {"x": 1e-5, "v": 2e-3, "density": 1e-4}),
    ("elastic", 10, {"x": 1e-5, "v": 2e-3, "stress": 1e-2}),
])
def test_fp32_vs_fp64_per_field(cuda_lib, name, steps, bounds):
    if name == "dam_break":
        sc = S.dam_break(seed=11, n_side=(10, 10, 10), box=0.4)
    elif name == "drop_implicit":
        sc = S.dam_break(seed=12, n_side=(9, 9, 9), box=0.4, extra_cfg={"useNonNewtonianModel": True},
                         fluid_cfg={"nonNewtonMethod": "CARREAU_", "viscosity0": 1.0, "viscosity_inf": 0.001,
                                    "consistency_index": 0.25, "power_index": 0.6, "viscosityMethod": 13,
                                    "viscoMaxError": 1e-4})
    else:  # the reference's elastic fixture, stretched so that it carries stress
        from .test_gpu_physics import _elastic_scene

        sc = _elastic_scene(False)
    m, solver = gpu_sim(sc)
    solver.initialize()
    o = oracle_sim(sc, "f64")
    o.initialize()
    if name == "elastic":
        x = pd_field(m, "x")
        v = np.zeros_like(x)
        v[:, 0] = 2.0 * (x[:, 0] - x[:, 0].mean())
        import torch
        m.pd.v.copy_(torch.from_numpy(v.astype(np.float32)))
        o.set("v", v.astype(np.float32))
    for _ in range(steps):
        solver.step()
    o.step(steps)
    nf = sc.particles.n_fluid
    errs = {}
    for f in bounds:
        g, r = pd_field(m, f), o.get(f)
        if f == "density":
            g, r = g[:nf], r[:nf]
        errs[f] = _err(g, r)
    print(f"\nFP32 GPU vs FP64 oracle, {name}, {steps} steps: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for f, b in bounds.items():
        assert errs[f] < b, (f, errs[f])


def _run_build(sc, precision, steps):
    """Fields after `steps` resident steps of the CUDA build of `precision`."""
    import torch

    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    m = sph.initialize(SimConfig(config=sc.config), particles=sc.particles, quirks=sc.param.quirks,
                       precision=precision)
    assert m.engine.precision == precision
    solver = sph.build_solver()
    solver.initialize()
    solver.run(steps)
    st = m.engine.stats(0)
    out = {k: pd_field(m, k) for k in ("x", "v", "density", "stress")}
    out["stats"] = st
    m.engine.close()
    torch.cuda.empty_cache()
    return out


@pytest.mark.parametrize("name,steps,bounds", [
    ("roofline_2m", 50, {"x": 1e-5, "v": 1e-2, "density": 1e-3}),
    ("shear_thinning_drop", 200, {"x": 1e-3, "v": 5e-2, "density": 2e-2}),
    ("fluid_elastic", 200, {"x": 1e-3, "v": 5e-2, "density": 2e-2, "stress": 5e-2}),
])
def test_fp32_vs_fp64_build_at_bench_sizes(cuda_lib, name, steps, bounds):
    """The FP32 product path against the FP64 build of the same kernels, free-running
    from the same float32 initial state over the scene's own step count: the error of
    each field (max |FP32 - FP64| over the field's scale, and the RMS of the same)."""
    sc = {"roofline_2m": S.roofline_scene, "shear_thinning_drop": S.shear_thinning_drop,
          "fluid_elastic": S.fluid_elastic}[name](seed=0)
    a = _run_build(sc, "f32", steps)
    b = _run_build(sc, "f64", steps)
    nf = sc.particles.n_fluid
    el = np.nonzero(np.asarray(sc.particles.phase_id) >= 3000)[0]
    errs, rms = {}, {}
    for f in bounds:
        g, r = a[f], b[f]
        if f == "density":
            g, r = g[:nf], r[:nf]
        elif f == "stress":
            g, r = g[el], r[el]
        scale = max(np.abs(r).max(), 1e-30)
        errs[f] = float(np.abs(g - r).max() / scale)
        rms[f] = float(np.sqrt(np.mean((g - r) ** 2)) / scale)
    sa, sb = a["stats"], b["stats"]
    print(f"\nFP32 vs FP64 build, {name} ({sc.particles.n} particles), {steps} steps: "
          + ", ".join(f"{k} max {errs[k]:.2e} rms {rms[k]:.2e}" for k in errs)
          + f"; last step iterations (div, pressure, cg) f32 {sa['iterations_v'], sa['iterations'], sa['cg_iterations']}"
          + f" f64 {sb['iterations_v'], sb['iterations'], sb['cg_iterations']}")
    assert sa["status"] == 0 and sb["status"] == 0
    for f, bd in bounds.items():
        assert errs[f] < bd, (f, errs[f])
