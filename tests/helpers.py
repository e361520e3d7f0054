"""Shared helpers of the parity tests: run a scene on the GPU and on the oracle."""
from __future__ import annotations

import numpy as np

FIELDS_V3 = ("x", "v", "acceleration")
FIELDS_S = ("volume", "density", "dfsph_factor", "density_adv")


def gpu_sim(sc, max_neighbors=64, block=None):
    """Set up a scene through the reference-facing object API; returns (meta, solver)."""
    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    m = sph.initialize(SimConfig(config=sc.config), particles=sc.particles, quirks=sc.param.quirks,
                       max_neighbors=max_neighbors)
    if block:
        m.engine.set_block_size(block)
    return m, sph.build_solver()


def oracle_sim(sc, precision="f32"):
    from oracle import oracle as O

    return O.OracleSim(sc.particles, sc.param, precision)


def pd_field(m, name):
    import torch

    torch.cuda.synchronize()
    return getattr(m.pd, name).detach().cpu().numpy().astype(np.float64)


def rel_err(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = scale if scale is not None else max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / s)


def factor_denominator(f):
    """-1 / dfsph_factor where the factor is set, else 0: the gradient sum the reference
    divides by (SPH/main.py:1586-1593), up to the solver's time-step scaling."""
    f = np.asarray(f, np.float64)
    out = np.zeros_like(f)
    nz = f != 0
    out[nz] = -1.0 / f[nz]
    return out


def field_err(name, a, b):
    """rel_err of one field. The DFSPH factor is compared through its denominator: a
    particle whose few neighbours all sit near the edge of the kernel support has a
    gradient sum of a few kernel gradients near r = h, where the f32 rounding of 1 - r/h
    moves each term by about 1e-4 of itself; its factor, the reciprocal of that small sum,
    is then both the field's largest value and its least accurate one. The denominators
    carry the same information, scaled by the well-conditioned interior."""
    if name == "dfsph_factor":
        return rel_err(factor_denominator(a), factor_denominator(b))
    return rel_err(a, b)


def sorted_sets_equal(n1, l1, n2, l2):
    """Per-particle neighbour id sets equal (rows are already sorted by id)."""
    n1 = np.asarray(n1); n2 = np.asarray(n2)
    if not np.array_equal(n1, n2):
        return False
    w = min(l1.shape[1], l2.shape[1])
    return bool(np.array_equal(np.asarray(l1)[:, :w], np.asarray(l2)[:, :w]))


def near_cutoff_pairs(x, h, tol_ulps=4):
    """Pairs whose f32 distance lies within a few ulp of h (may flip under rounding)."""
    from scipy.spatial import cKDTree

    t = cKDTree(x.astype(np.float64))
    pairs = t.query_pairs(h * (1 + 1e-5), output_type="ndarray")
    if len(pairs) == 0:
        return set()
    d = np.linalg.norm(x[pairs[:, 0]].astype(np.float64) - x[pairs[:, 1]].astype(np.float64), axis=1)
    ulp = np.spacing(np.float32(h))
    sel = np.abs(d - h) < tol_ulps * ulp
    return {(int(a), int(b)) for a, b in pairs[sel]}


# ---- the reference's own step, run once through a Taichi stand-in
# (tests/golden/make_reference_run.py), stored as tests/golden/ref_<scene>.npz
REF_SCENES = ("dam", "nonnewton", "elastic", "rigid", "deformable", "neighbor9", "anime")
REF_FIELDS = ("x", "v", "acceleration", "density", "dfsph_factor", "density_adv", "volume", "strain_rate_norm",
              "nonnewton_viscosity", "stress", "rotations")
FLUID_ONLY = ("density", "dfsph_factor", "density_adv", "strain_rate_norm", "nonnewton_viscosity")


def reference_run(name):
    """(fixture, config dict, Parameter in quirks mode, ParticleSet) of a reference run:
    the phases rebuilt from the run's own initial positions and phase ids."""
    import json
    import os

    from nonnewton_b200 import scene as S
    from nonnewton_b200.config import Parameter, SimConfig

    R = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"ref_{name}.npz")))
    cfg = json.loads(R["config"].tobytes().decode())
    cfg["Configuration"].pop("animeFile", None)  # its table is in the fixture (reference_animation)
    param = Parameter.from_config(SimConfig(config=cfg), quirks=True)
    phases = []
    for uid in dict.fromkeys(R["phase_id"].tolist()):
        m = R["phase_id"] == uid
        st = S.RIGID if 2000 <= uid < 3000 else S.ELASTIC if uid >= 3000 else S.STATIC
        phases.append(S.PhaseInfo(uid=uid, material=int(R["material"][m][0]), is_dynamic=bool(R["is_dynamic"][m][0]),
                                  pos=R["init_x"][m], solid_type=st))
    return R, cfg, param, S.assemble(phases, param)


def reference_animation(R):
    """(frames, displacements) of the run's animeFile, or None."""
    return (R["anime_frames"], R["anime_disp"]) if "anime_frames" in R else None


def frame_displacement(anime, frame):
    """The displacement animate_particles (SPH/main.py:283-309) adds at `frame`: the sum
    of the table's rows for that frame, or None."""
    if anime is None or not (anime[0] == frame).any():
        return None
    return anime[1][anime[0] == frame].astype(np.float32).sum(axis=0)


def reference_steps(R):
    return sum(1 for k in R if k.startswith("step") and k.endswith("_x"))


def reference_errors(R, step, get, nf):
    """{field: max |ours - reference| / scale} for the fields the run recorded at `step`;
    the stress scale is at least 10 Pa: below that it is f32 noise (Young's modulus
    2.5e5 Pa times a few f32 ulps of the deformation gradient), as in a barely strained
    elastic cube."""
    floor = {"stress": 10.0}
    out = {}
    for k in REF_FIELDS:
        key = f"step{step}_{k}"
        if key not in R:
            continue
        b = R[key].astype(np.float64)
        a = np.asarray(get(k), np.float64).reshape(b.shape)
        if k in FLUID_ONLY:
            if nf == 0:
                continue
            a, b = a[:nf], b[:nf]
        out[k] = float(np.abs(a - b).max() / max(np.abs(b).max(), floor.get(k, 1e-30)))
    return out
