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


def _engine(sc, precision, nudge=False):
    """ParticleData + Engine of one scene for the CUDA build of `precision` (the pieces
    sph.initialize assembles, without its global `meta`, so that two builds can hold
    the same scene at once). `nudge` moves every fluid position up by one float32 ulp."""
    import torch

    from nonnewton_b200.engine import Engine
    from nonnewton_b200.sph import ParticleData, initialize_particles

    ps = sc.particles
    pd = ParticleData(ps.n)
    initialize_particles(pd, ps, sc.param)
    if nudge:
        x = pd.x[: ps.n_fluid]
        x.copy_(torch.nextafter(x, torch.full_like(x, float("inf"))))
    eng = Engine(ps.n, 1, 64, precision=precision)
    eng.bind(pd)
    eng.set_scenes([(0, ps.n, ps.n_fluid, sc.param.to_c())])
    eng.initialize()
    return pd, eng


def _fields(pd, names, nf, el):
    """Fields of `pd` as float64 arrays: density of the fluid, stress of the elastic."""
    out = {}
    for f in names:
        a = getattr(pd, f).detach().cpu().numpy().astype(np.float64)
        out[f] = a[:nf] if f == "density" else a[el] if f == "stress" else a
    return out


def _errors(a, b, floors=None):
    """(max |a - b| / scale, RMS(a - b) / scale) per field, scale = max |b|, at least
    the field's floor (stress: 1e-4 of Young's modulus, below which an unstrained
    block's stress is float32 noise)."""
    out = {}
    for f in a:
        scale = max(np.abs(b[f]).max(), (floors or {}).get(f, 1e-30))
        out[f] = (float(np.abs(a[f] - b[f]).max() / scale), float(np.sqrt(np.mean((a[f] - b[f]) ** 2)) / scale))
    return out


def test_fp64_build_matches_the_fp64_oracle(cuda_lib):
    """The FP64 build is the same algorithm as the oracle in double: ten free-running
    steps of a small dam break with the Carreau law and the implicit viscosity agree
    to double-precision rounding (summation order differs)."""
    sc = S.dam_break(seed=12, n_side=(9, 9, 9), box=0.4, extra_cfg={"useNonNewtonianModel": True},
                     fluid_cfg={"nonNewtonMethod": "CARREAU_", "viscosity0": 1.0, "viscosity_inf": 0.001,
                                "consistency_index": 0.25, "power_index": 0.6, "viscosityMethod": 13,
                                "viscoMaxError": 1e-4})
    pd, eng = _engine(sc, "f64")
    o = oracle_sim(sc, "f64")
    o.initialize()
    eng.step(10, sync=True)
    o.step(10)
    nf = sc.particles.n_fluid
    for f in ("x", "v", "density"):
        g = getattr(pd, f).detach().cpu().numpy().astype(np.float64)
        r = o.get(f)
        if f == "density":
            g, r = g[:nf], r[:nf]
        # the FP64 run's state is written to the float32 fields: compare at f32 resolution
        assert _err(g, r) < 1e-6, (f, _err(g, r))
    st, ost = eng.stats(0), o.stats()
    assert (st["iterations_v"], st["iterations"]) == (ost["iterations_v"], ost["iterations"])
    eng.close()


# per-step bounds (max, RMS) over the field's scale
@pytest.mark.parametrize("name,steps,lockstep,bounds", [
    ("roofline_2m", 50, 10, {"x": (1e-5, 1e-7), "v": (3e-2, 2e-5), "density": (3e-6, 5e-7)}),
    ("shear_thinning_drop", 200, 20, {"x": (3e-5, 1e-7), "v": (3e-2, 5e-5), "density": (3e-6, 5e-7)}),
    ("fluid_elastic", 200, 20, {"x": (1e-6, 1e-7), "v": (3e-4, 2e-6), "density": (3e-6, 5e-7),
                                "stress": (1e-1, 1e-2)}),
])
def test_fp32_vs_fp64_build_at_bench_sizes(cuda_lib, name, steps, lockstep, bounds):
    """The FP32 product path against the FP64 build of the same kernels at the
    benchmark scenes' sizes, two ways:

      - per step: along the FP64 run, every `steps // lockstep`-th step starts both
        builds from the same float32 state; the error of that one step is the cost of
        FP32 arithmetic (bounded below);
      - free-running over the scene's step count, each build resident in its own
        precision: the divergence that cost grows into (printed, max and RMS over the
        field's scale; splashing flows amplify it, and so do the rule's discontinuities:
        the neighbour cut-off, the 20-neighbour rule of the divergence solve, the
        boundary clamp)."""
    import torch

    sc = {"roofline_2m": S.roofline_scene, "shear_thinning_drop": S.shear_thinning_drop,
          "fluid_elastic": S.fluid_elastic}[name](seed=0)
    nf = sc.particles.n_fluid
    el = np.nonzero(np.asarray(sc.particles.phase_id) >= 3000)[0]
    names = list(bounds)
    floors = {"stress": 1e-4 * sc.param.youngs_modulus}
    pd32, e32 = _engine(sc, "f32")
    pd64, e64 = _engine(sc, "f64")
    every = max(steps // lockstep, 1)
    worst = {f: (0.0, 0.0) for f in names}
    for k in range(steps):
        if k % every == 0:  # one step of each build from the FP64 run's current state
            pd32.x.copy_(pd64.x)
            pd32.v.copy_(pd64.v)
            e32.step(1, sync=True)
            e64.step(1, sync=True)
            err = _errors(_fields(pd32, names, nf, el), _fields(pd64, names, nf, el), floors)
            worst = {f: (max(worst[f][0], err[f][0]), max(worst[f][1], err[f][1])) for f in names}
        else:
            e64.step(1, sync=True)
    torch.cuda.synchronize()
    print(f"\nFP32 vs FP64 build, {name} ({sc.particles.n} particles), one step from the same state, worst of "
          f"{lockstep}: " + ", ".join(f"{f} max {worst[f][0]:.2e} rms {worst[f][1]:.2e}" for f in names))
    for f, (bmax, brms) in bounds.items():
        assert worst[f][0] < bmax and worst[f][1] < brms, (f, worst[f])
    e32.close()
    e64.close()
    del pd32, pd64
    torch.cuda.empty_cache()
    # free-running: each build resident in its precision from the same initial state
    out = {}
    for prec in ("f32", "f64"):
        pd, eng = _engine(sc, prec)
        eng.step(steps, sync=True)
        st = eng.stats(0)
        assert st["status"] == 0, (prec, st)
        out[prec] = _fields(pd, names, nf, el)
        eng.close()
        del pd
        torch.cuda.empty_cache()
    # the flow's own sensitivity: the FP64 build against itself, the fluid's initial
    # positions moved by one float32 ulp
    pd, eng = _engine(sc, "f64", nudge=True)
    eng.step(steps, sync=True)
    nudged = _fields(pd, names, nf, el)
    eng.close()
    del pd
    torch.cuda.empty_cache()
    err = _errors(out["f32"], out["f64"], floors)
    sens = _errors(nudged, out["f64"], floors)
    print(f"FP32 vs FP64 build, {name}, free-running {steps} steps: "
          + ", ".join(f"{f} max {err[f][0]:.2e} rms {err[f][1]:.2e}" for f in names))
    print(f"FP64 vs FP64 with the fluid moved by one float32 ulp, {name}, {steps} steps: "
          + ", ".join(f"{f} max {sens[f][0]:.2e} rms {sens[f][1]:.2e}" for f in names))
    for f in names:
        assert err[f][1] < 0.05, (f, err[f])  # a sanity bound on the RMS divergence
