"""The allocation-free neighbour search (nn_neighbors_noalloc) against the regular
path (nn_run_pass(NN_PASS_SEARCH) + nn_get_neighbors), called through the C ABI.

The entry point serves callers that cannot allocate device memory themselves; its
scratch is a device array inside the library. The tests make calls in a row on
different inputs (the array keeps the previous call's contents, so each later call
also checks that everything that must start cleared is cleared) and require the
rows to be identical to the regular path's: neighbour lists are integer data.
"""
import ctypes as C

import numpy as np
import pytest

from nonnewton_b200 import scene as S
from nonnewton_b200.config import Parameter, SimConfig

from .helpers import gpu_sim

pytestmark = pytest.mark.gpu
NB_MAX = 64  # NN_NOALLOC_MAX_NEIGHBORS


def _fn():
    from nonnewton_b200.engine import lib

    L = lib()
    f = L.nn_neighbors_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_int32,
                  C.c_void_p, C.c_void_p, C.c_void_p]
    return L, f


def _noalloc(x, sc, width):
    import torch

    L, f = _fn()
    n = x.shape[0]
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    num = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    lists = torch.full((n, width), -7, dtype=torch.int32, device="cuda")
    lo = (C.c_double * 3)(*sc.param.domain_start)
    hi = (C.c_double * 3)(*sc.param.domain_end)
    stream = torch.cuda.current_stream().cuda_stream
    rc = f(xd.data_ptr(), n, lo, hi, sc.param.support_radius, width, num.data_ptr(), lists.data_ptr(), stream)
    assert rc == 0, L.nn_last_error(None)
    torch.cuda.synchronize()
    return num.cpu().numpy(), lists.cpu().numpy()


def _regular(sc, width, max_neighbors=NB_MAX):
    m, _ = gpu_sim(sc, max_neighbors=max_neighbors)
    m.ns.run_search()
    num, lists = m.engine.neighbors(sc.particles.n, width)
    return num.cpu().numpy(), lists.cpu().numpy()


def _fluid_scene(x, domain, r=0.01):
    """A fluid-only scene of the given positions (for the search, only positions,
    the domain and the support radius 4r matter)."""
    conf = {"Configuration": {"domainStart": list(domain[0]), "domainEnd": list(domain[1]), "particleRadius": r,
                              "density0": 1000, "simulationMethod": 4, "timeStepSize": 1e-3},
            "FluidParticles": [{}]}
    param = Parameter.from_config(SimConfig(config=conf))
    ps = S.assemble([S.PhaseInfo(uid=0, material=0, is_dynamic=True, pos=x)], param)
    return S.Scene("noalloc", conf, param, ps, 1)


def test_noalloc_matches_regular_search_twice(cuda_lib):
    scenes = [S.dam_break(seed=11, n_side=(12, 12, 12), box=0.4),
              S.dam_break(seed=12, n_side=(9, 10, 11), box=0.36)]
    for sc in scenes:  # two calls in a row, different sizes and positions
        a_num, a_lists = _noalloc(sc.particles.x, sc, 60)
        b_num, b_lists = _regular(sc, 60)
        assert np.array_equal(a_num, b_num)
        assert np.array_equal(a_lists, b_lists)
        assert a_num.max() > 20


def test_noalloc_at_the_particle_limit(cuda_lib):
    """Exactly NN_NOALLOC_MAX_PARTICLES = 16,384 particles (a jittered 16 x 32 x 32
    block), then a smaller scene on the same array."""
    rng = np.random.default_rng(3)
    x = S.block((0.1, 0.1, 0.1), (16, 32, 32), 0.02, jitter=2e-3, rng=rng)
    assert x.shape[0] == 16384
    sc = _fluid_scene(x, ((0.0, 0.0, 0.0), (0.8, 0.8, 0.8)))
    a_num, a_lists = _noalloc(x, sc, 64)
    b_num, b_lists = _regular(sc, 64)
    assert np.array_equal(a_num, b_num) and np.array_equal(a_lists, b_lists)
    assert a_num.max() <= NB_MAX and a_num.min() >= 5
    small = S.dam_break(seed=13, n_side=(8, 8, 8), box=0.3)
    a_num, a_lists = _noalloc(small.particles.x, small, 60)
    b_num, b_lists = _regular(small, 60)
    assert np.array_equal(a_num, b_num) and np.array_equal(a_lists, b_lists)


def test_noalloc_reports_neighbor_overflow(cuda_lib):
    """A lattice at spacing h/3 gives interior particles at least 92 neighbours (more
    where a pair at exactly h rounds inside), above the
    64-entry rows of the scratch array. num_neighbors carries the full count (the
    overflow signal), equal to a regular context with room for 128; the rows equal a
    regular context capped at 64, whose count saturates there."""
    r = 0.01
    h = 4 * r
    idx = np.stack(np.meshgrid(*[np.arange(12)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = 0.1 + idx * (h / 3.0)
    sc = _fluid_scene(x, ((0.0, 0.0, 0.0), (0.4, 0.4, 0.4)), r=r)
    a_num, a_lists = _noalloc(x, sc, 128)
    full_num, full_lists = _regular(sc, 128, max_neighbors=128)
    cap_num, cap_lists = _regular(sc, 128, max_neighbors=NB_MAX)
    assert a_num.max() >= 92 and (a_num > NB_MAX).sum() > 100
    assert np.array_equal(a_num, full_num)
    assert np.array_equal(a_lists, cap_lists)
    assert np.array_equal(cap_num, np.minimum(full_num, NB_MAX))
    over = np.nonzero(a_num > NB_MAX)[0]
    for i in over[:50]:  # an overflowed row holds 64 true neighbours
        row = a_lists[i][a_lists[i] >= 0]
        assert len(row) == NB_MAX and set(row.tolist()) <= set(full_lists[i][: full_num[i]].tolist())
    ok = a_num <= NB_MAX
    assert np.array_equal(a_lists[ok], full_lists[ok])


def test_noalloc_positions_outside_the_domain(cuda_lib):
    """Particles outside the domain are clamped into the border cells, as in the
    regular search; the rows agree, the ones across the border included."""
    sc = S.dam_break(seed=14, n_side=(8, 8, 8), box=0.3)
    x = sc.particles.x.copy()
    rng = np.random.default_rng(14)
    out = rng.choice(len(x), size=40, replace=False)
    lo = np.asarray(sc.param.domain_start)
    hi = np.asarray(sc.param.domain_end)
    x[out[:20]] = lo - rng.uniform(0.0, 0.03, size=(20, 3))
    x[out[20:]] = hi + rng.uniform(0.0, 0.03, size=(20, 3))
    sc.particles.x = x
    a_num, a_lists = _noalloc(x, sc, 60)
    b_num, b_lists = _regular(sc, 60)
    assert np.array_equal(a_num, b_num) and np.array_equal(a_lists, b_lists)
    assert a_num[out].max() > 0  # the clustered outside particles see each other


def test_noalloc_rejects_oversize(cuda_lib):
    """Beyond the limits the call fails with NN_ERR_CAPACITY (-8) and launches nothing:
    more particles than NN_NOALLOC_MAX_PARTICLES, or a domain needing more than
    NN_NOALLOC_MAX_CELLS cells of edge h."""
    import torch

    L, f = _fn()
    sc = S.dam_break(seed=0, n_side=(4, 4, 4), box=0.2)
    x = np.zeros((16385, 3), np.float32)
    xd = torch.from_numpy(x).cuda()
    out = torch.zeros(16385 * 8, dtype=torch.int32, device="cuda")
    lo = (C.c_double * 3)(*sc.param.domain_start)
    hi = (C.c_double * 3)(*sc.param.domain_end)
    rc = f(xd.data_ptr(), 16385, lo, hi, 0.04, 4, out.data_ptr(), out.data_ptr(), None)
    assert rc == -8 and b"exceed" in L.nn_last_error(None)
    big_lo = (C.c_double * 3)(0.0, 0.0, 0.0)
    big_hi = (C.c_double * 3)(3.0, 3.0, 3.0)  # 3 m / 0.04 m: about 80^3 cells
    rc = f(xd.data_ptr(), 100, big_lo, big_hi, 0.04, 4, out.data_ptr(), out.data_ptr(), None)
    assert rc == -8 and b"cells" in L.nn_last_error(None)
