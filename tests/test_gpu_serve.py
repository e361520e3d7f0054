"""Served form: continuous batching completes every request, and each result equals
the same request run alone (the plain per-scene path), within 1e-6 m."""
import numpy as np
import pytest

from nonnewton_b200 import scene as S

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone(cuda_lib):
    from nonnewton_b200.serve import Request, Server, run_plain

    work = S.mixed_workload(n_requests=10, seed=5, rate=1e6, steps=12)
    # shrink the requests to test size: keep the generator's parameters, smaller blocks
    reqs = []
    for k, (t, sc) in enumerate(work):
        small = S.dam_break(seed=k, n_side=(6 + k % 4, 7, 6 + k % 3), box=0.3 + 0.02 * (k % 3),
                            extra_cfg={"useNonNewtonianModel": True}, fluid_cfg=sc.config["FluidParticles"][0])
        reqs.append(Request(k, small, 12 + 4 * (k % 3), t))
    cap = sum(r.scene.particles.n for r in reqs[:4])  # forces several admission rounds
    srv = Server(capacity=cap, max_scenes=4, chunk=4)
    res = srv.run(reqs, realtime=False)
    assert res["requests"] == len(reqs) and res["repacks"] >= 3
    alone = [Request(r.rid, r.scene, r.steps, 0.0) for r in reqs]
    run_plain(alone)
    fin = {r.rid: r for r in res["finished"]}
    for a in alone:
        assert np.abs(fin[a.rid].result_x - a.result_x).max() <= 1e-6, a.rid
        assert fin[a.rid].stats["avg_density_err"] <= 0.1 * 0.01 * 1000.0 + 1e-9


def test_a_failing_request_is_evicted_and_the_others_go_on(cuda_lib):
    """Failure detection in the served loop: a request with a non-finite particle sets
    its scene's status word in its first chunk and retires with that status; the
    requests batched with it, before and after, still equal their runs alone."""
    import copy

    from nonnewton_b200 import _abi
    from nonnewton_b200.serve import Request, Server, run_plain

    reqs = []
    for k in range(6):
        sc = S.dam_break(seed=20 + k, n_side=(6, 6 + k % 2, 6), box=0.3)
        if k == 2:
            sc = copy.deepcopy(sc)
            sc.particles.x[5] = np.nan
        reqs.append(Request(k, sc, 12, 0.0))
    srv = Server(capacity=sum(r.scene.particles.n for r in reqs[:3]), max_scenes=3, chunk=4)
    res = srv.run(reqs, realtime=False)
    assert res["requests"] == len(reqs) and res["failed"] == [2]
    fin = {r.rid: r for r in res["finished"]}
    assert fin[2].failed == _abi.NN_ERR_NAN and fin[2].done_steps == fin[2].steps
    good = [Request(r.rid, r.scene, r.steps, 0.0) for r in reqs if r.rid != 2]
    run_plain(good)
    for a in good:
        assert fin[a.rid].failed == 0
        assert np.abs(fin[a.rid].result_x - a.result_x).max() <= 1e-6, a.rid
