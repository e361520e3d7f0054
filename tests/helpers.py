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
