"""Multi-rank host logic on CPU with the gloo backend (world size 2): every rank
derives the same disjoint, balanced shard of the request list, and metrics combine
with one sum / max reduction after the run (no collective on the data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from nonnewton_b200 import scene as S
    from nonnewton_b200.serve import Request
    from nonnewton_b200.shard import combine_metrics, request_cost, shard_requests

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        work = S.mixed_workload(n_requests=40, seed=3, steps=10)
        reqs = [Request(k, sc, 10, t) for k, (t, sc) in enumerate(work)]
        shards = shard_requests(reqs, world)
        mine = shards[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        loads = [sum(request_cost(reqs[k]) for k in s) for s in shards]
        local = {"particle_steps": float(sum(request_cost(reqs[k]) for k in mine)), "requests": len(mine),
                 "wall_s": 1.0 + rank, "device_s": 0.5 * (rank + 1)}
        tot = combine_metrics(local, world)
        q.put((rank, gathered, loads, tot, len(reqs), sum(request_cost(r) for r in reqs)))
    finally:
        dist.destroy_process_group()


def test_shards_are_consistent_disjoint_and_balanced():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, g0, loads, tot0, nreq, cost), (_, g1, _, tot1, _, _) = res
    assert g0 == g1  # every rank computed the same assignment
    ids = [k for s in g0 for k in s]
    assert sorted(ids) == list(range(nreq))
    assert max(loads) - min(loads) <= max(loads) * 0.15
    for tot in (tot0, tot1):
        assert tot["particle_steps"] == pytest.approx(cost)
        assert tot["requests"] == nreq and tot["wall_s"] == 2.0 and tot["device_s"] == 1.0


def _serve_worker(rank, world, port, q):
    """One rank of a served run over the stand-in batch of the host tests."""
    import torch
    import torch.distributed as dist

    from nonnewton_b200 import scene as S
    from nonnewton_b200 import serve as SV
    from nonnewton_b200.shard import serve_sharded
    from tests import test_serve_host as H

    torch.cuda.Event = H._Event
    torch.cuda.current_stream = lambda *a, **k: None
    empty = torch.empty
    torch.empty = lambda *a, pin_memory=False, **k: empty(*a, **k)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = [SV.Request(k, S.dam_break(seed=k, n_side=(3 + k % 2, 3, 3), box=0.2), 3 + k % 4, 0.002 * k)
                for k in range(14)]
        cap = sum(r.scene.particles.n for r in reqs[:3])
        res = serve_sharded(H._server(H._Batch(cap, max_scenes=3), chunk=2), reqs, world, rank, realtime=True)
        done = {r.rid: (int(r.result_x[0, 0]), r.steps) for r in res["finished"]}
        q.put((rank, res["mine"], done, res["combined"], sum(r.scene.particles.n * r.steps for r in reqs)))
    finally:
        dist.destroy_process_group()


def test_served_requests_finish_once_on_one_rank():
    """Two servers (gloo ranks, stand-in batches) share one arrival stream: every
    request finishes exactly once, on the rank its shard names, with all its steps;
    the combined particle-steps are the stream's total."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_serve_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seen = []
    for rank, mine, done, comb, total in res:
        assert sorted(done) == sorted(mine)  # finished here exactly what the shard gave this rank
        assert all(x == steps for x, steps in done.values())
        assert comb["particle_steps"] == total and comb["requests"] == 14
        seen += list(done)
    assert sorted(seen) == list(range(14))  # each request once, on one rank
