"""Per-field error of the FP32 GPU step against the FP64 run of the same algorithm
(the oracle in double precision), from identical initial states, free-running.

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
