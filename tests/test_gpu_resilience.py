"""Checkpoint/resume and failure detection on the GPU, without faulting it: bad
inputs are made on the host (a non-finite particle, a too-small neighbour capacity)
and must come back as status codes while the context stays usable."""
import numpy as np
import pytest

from nonnewton_b200 import _abi
from nonnewton_b200 import scene as S

from .helpers import gpu_sim, pd_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["fluid", "elastic"])
def test_checkpoint_resume_bit_identical(cuda_lib, tmp_path, kind):
    from nonnewton_b200 import sph

    if kind == "fluid":
        sc = S.dam_break(seed=8, n_side=(9, 9, 9), box=0.36, extra_cfg={"useNonNewtonianModel": True},
                         fluid_cfg={"nonNewtonMethod": "CROSS_", "viscosity0": 5.0, "viscosity_inf": 0.01,
                                    "consistency_index": 1.0, "power_index": 0.7, "viscosityMethod": 13})
    else:
        sc = S.fluid_elastic(n_el=5)
    m, solver = gpu_sim(sc)
    solver.initialize()
    for _ in range(10):
        solver.step()
    x_ref, v_ref = pd_field(m, "x"), pd_field(m, "v")
    m, solver = gpu_sim(sc)
    solver.initialize()
    for _ in range(5):
        solver.step()
    path = str(tmp_path / "ck.pt")
    sph.save_checkpoint(path)
    m2, solver2 = sph.load_checkpoint(path)
    assert m2.step_num == 5
    for _ in range(5):
        solver2.step()
    assert np.array_equal(pd_field(m2, "x"), x_ref) and np.array_equal(pd_field(m2, "v"), v_ref)


def test_checkpoint_keeps_the_animation(cuda_lib, tmp_path):
    """A checkpoint carries the animeFile table and the frame count: a resumed run moves
    by the frames it had not reached, bit-identical to the uninterrupted one."""
    from nonnewton_b200 import sph

    sc = S.dam_break(seed=2, n_side=(6, 6, 6), box=0.25)
    anime = (np.array([1, 3, 6, 8], np.int64),
             np.array([[0.003, 0, 0], [0, 0.002, 0], [0, 0, 0.004], [-0.002, 0, 0]], np.float32))
    m, solver = gpu_sim(sc)
    m.anime = anime
    solver.initialize()
    for _ in range(10):
        solver.step()
    x_ref = pd_field(m, "x")
    m, solver = gpu_sim(sc)
    m.anime = anime
    solver.initialize()
    for _ in range(5):
        solver.step()
    path = str(tmp_path / "ck.pt")
    sph.save_checkpoint(path)
    m2, solver2 = sph.load_checkpoint(path)
    assert m2.step_num == 5 and np.array_equal(m2.anime[0], anime[0])
    for _ in range(5):
        solver2.step()
    assert np.array_equal(pd_field(m2, "x"), x_ref)


def test_nonfinite_state_sets_status(cuda_lib):
    import torch

    sc = S.dam_break(seed=1, n_side=(8, 8, 8), box=0.3)
    m, solver = gpu_sim(sc)
    solver.initialize()
    m.pd.v[3, 0] = float("nan")
    solver.step()
    st = m.engine.stats(0)
    assert st["status"] == _abi.NN_ERR_NAN
    # the context is still usable: a fresh scene on a new context steps normally
    m2, s2 = gpu_sim(sc)
    s2.initialize()
    s2.step()
    assert m2.engine.stats(0)["status"] == 0 and torch.isfinite(m2.pd.x).all()


def test_neighbor_overflow_sets_status(cuda_lib):
    sc = S.dam_break(seed=1, n_side=(8, 8, 8), box=0.3)
    m, solver = gpu_sim(sc, max_neighbors=16)
    solver.initialize()
    solver.step()
    st = m.engine.stats(0)
    assert st["status"] == _abi.NN_ERR_NEIGHBOR_OVERFLOW and st["max_neighbors_seen"] > 16


def test_served_failed_request_is_evicted(cuda_lib):
    from nonnewton_b200.serve import Request, Server, run_plain

    reqs = []
    for k in range(6):
        sc = S.dam_break(seed=30 + k, n_side=(6, 6, 7), box=0.28)
        if k == 2:  # poison one particle of one request
            sc.particles.x[5] = np.nan
        reqs.append(Request(k, sc, 10, 0.0))
    srv = Server(capacity=sum(r.scene.particles.n for r in reqs[:3]), max_scenes=3, chunk=5)
    res = srv.run(reqs, realtime=False)
    assert res["requests"] == 6 and res["failed"] == [2]
    alone = [Request(r.rid, r.scene, r.steps, 0.0) for r in reqs if r.rid != 2]
    run_plain(alone)
    fin = {r.rid: r for r in res["finished"]}
    for a in alone:
        assert np.array_equal(fin[a.rid].result_x, a.result_x)
