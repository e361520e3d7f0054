"""Generate the golden fixtures of the parity tests.

Run in the build container (where the reference checkout is readable):
    python tests/golden/make_golden.py [reference_root]

Fixtures (all derived from the reference's own data files and formulas, computed
here with independent pure-Python / numpy code, not with the oracle):
- neighbor_9pt.json: SPH/data/models/test_neighbor.ply (the fixture of the
  reference's test_neighborhoodSearchSparse, SPH/test.py:73-87) with the neighbour
  lists the reference's rule gives: p_i != p_j and |x_i - x_j| < h in f32
  (SPH/main.py:845), h = 4 r with r = 0.01 from SPH/data/scenes/test_neighbor.json.
- lattice_kat.json: a lattice with exactly representable coordinates (r = 2^-7,
  spacing 2r, h = 4r): interior particles have 26 neighbours (pairs at exactly h are
  excluded by the strict <) and the rest density rho0 V0 (W(0) + sum W) from the
  cubic spline of SPH/main.py:859-880 in float64 (about 800, since V0 = 0.8 (2r)^3).
- deformable_343.npy: positions of SPH/data/models/test_deformable.ply (the elastic
  fixture of SPH/data/scenes/test_deformable.json).
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from nonnewton_b200.scene import read_ply_particles  # noqa: E402


def brute_neighbors(x32: np.ndarray, h: float):
    n = x32.shape[0]
    hf = np.float32(h)
    lists = []
    for i in range(n):
        row = []
        for j in range(n):
            if i == j:
                continue
            d = x32[i] - x32[j]
            s = np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1]))
            s = np.float32(s + np.float32(d[2] * d[2]))
            if np.float32(np.sqrt(s)) < hf:
                row.append(j)
        lists.append(row)
    return lists


def cubic_w(r, h):
    k = 8.0 / math.pi / h ** 3
    q = r / h
    if q <= 0.5:
        return k * (6 * q ** 3 - 6 * q ** 2 + 1)
    if q <= 1.0:
        return k * 2 * (1 - q) ** 3
    return 0.0


def main(ref_root: str):
    # 9-point neighbour fixture
    ply = os.path.join(ref_root, "SPH/data/models/test_neighbor.ply")
    grid = np.array([[0.03 * i, 0.03 * j, 0.0] for j in range(3) for i in range(3)], dtype=np.float32)
    if os.path.exists(ply):
        pts = read_ply_particles(ply)
        assert np.allclose(pts, grid), "test_neighbor.ply is the 3x3 grid at 0.03 m"
    pts = grid
    r = 0.01
    h = 4 * r
    lists = brute_neighbors(pts, h)
    json.dump({"source": "SPH/data/models/test_neighbor.ply", "particle_radius": r, "support_radius": h,
               "x": pts.tolist(), "num_neighbors": [len(L) for L in lists], "neighbors": lists},
              open(os.path.join(HERE, "neighbor_9pt.json"), "w"), indent=1)
    # power-of-two lattice
    r = 2.0 ** -7
    sp = 2 * r
    h = 4 * r
    n_side = 8
    org = 0.25
    idx = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = (org + idx * sp).astype(np.float32)
    assert np.all(x.astype(np.float64) == org + idx * sp), "coordinates exactly representable"
    V0 = 0.8 * (2 * r) ** 3
    s = cubic_w(0.0, h) + 6 * cubic_w(sp, h) + 12 * cubic_w(math.sqrt(2) * sp, h) + 8 * cubic_w(math.sqrt(3) * sp, h)
    rho_interior = 1000.0 * V0 * s
    interior = np.all((idx > 0) & (idx < n_side - 1), axis=1)
    json.dump({"particle_radius": r, "support_radius": h, "origin": org, "n_side": n_side,
               "interior_neighbors": 26, "rho_interior": rho_interior,
               "interior_ids": np.nonzero(interior)[0].tolist()},
              open(os.path.join(HERE, "lattice_kat.json"), "w"), indent=1)
    # elastic fixture
    ply = os.path.join(ref_root, "SPH/data/models/test_deformable.ply")
    if os.path.exists(ply):
        np.save(os.path.join(HERE, "deformable_343.npy"), read_ply_particles(ply))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
    main(sys.argv[1])
