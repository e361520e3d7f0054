"""The allocation-free neighbour search (nn_neighbors_noalloc) against the regular
path (nn_run_pass(NN_PASS_SEARCH) + nn_get_neighbors), called through the C ABI.

The entry point serves callers that cannot allocate device memory themselves; its
scratch is a device array inside the library. The test makes two calls in a row on
different inputs (the array keeps the previous call's contents, so the second call
also checks that everything that must start cleared is cleared) and requires the
rows to be identical to the regular path's: neighbour lists are integer data.
"""
import ctypes as C

import numpy as np
import pytest

from nonnewton_b200 import scene as S

from .helpers import gpu_sim

pytestmark = pytest.mark.gpu


def _noalloc(x, sc, width):
    import torch

    from nonnewton_b200.engine import lib

    L = lib()
    f = L.nn_neighbors_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_int32,
                  C.c_void_p, C.c_void_p, C.c_void_p]
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


def _regular(sc, width):
    m, _ = gpu_sim(sc)
    m.ns.run_search()
    num, lists = m.engine.neighbors(sc.particles.n, width)
    return num.cpu().numpy(), lists.cpu().numpy()


def test_noalloc_matches_regular_search_twice(cuda_lib):
    scenes = [S.dam_break(seed=11, n_side=(12, 12, 12), box=0.4),
              S.dam_break(seed=12, n_side=(9, 10, 11), box=0.36)]
    for sc in scenes:  # two calls in a row, different sizes and positions
        a_num, a_lists = _noalloc(sc.particles.x, sc, 60)
        b_num, b_lists = _regular(sc, 60)
        assert np.array_equal(a_num, b_num)
        assert np.array_equal(a_lists, b_lists)
        assert a_num.max() > 20


def test_noalloc_rejects_oversize(cuda_lib):
    from nonnewton_b200.engine import lib

    L = lib()
    sc = S.dam_break(seed=0, n_side=(4, 4, 4), box=0.2)
    x = np.zeros((16385, 3), np.float32)
    import torch

    xd = torch.from_numpy(x).cuda()
    out = torch.zeros(16385 * 8, dtype=torch.int32, device="cuda")
    lo = (C.c_double * 3)(*sc.param.domain_start)
    hi = (C.c_double * 3)(*sc.param.domain_end)
    rc = L.nn_neighbors_noalloc(C.c_void_p(xd.data_ptr()), C.c_int32(16385), lo, hi, C.c_double(0.04),
                                C.c_int32(4), C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == -8 and b"exceed" in L.nn_last_error(None)
