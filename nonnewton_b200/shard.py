"""Multi-GPU form of the batched/served step: whole scenes are sharded across ranks
(one process per GPU); scenes never interact, so there is no collective on the data
path. Ranks only combine their metrics (particle-steps summed, times max-reduced)
once, after the run.

A single scene is not split across GPUs (replicas only): a spatial split would need
a halo exchange before every neighbour pass.
"""
from __future__ import annotations

import heapq


def request_cost(req) -> float:
    """Work of a request: particles x steps."""
    return float(req.scene.particles.n) * float(req.steps)


def shard_requests(requests, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of requests to `world` ranks by
    particle-steps (deterministic: ties broken by request id). Returns, per rank, the
    indices into `requests`, in arrival order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(requests)), key=lambda k: (-request_cost(requests[k]), requests[k].rid))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + request_cost(requests[k]), r))
    for r in range(world):
        out[r].sort(key=lambda k: (requests[k].arrival, requests[k].rid))
    return out


def combine_metrics(local: dict, world: int) -> dict:
    """Sum particle-steps and requests, max-reduce wall and device times over ranks
    (torch.distributed, any backend)."""
    if world <= 1:
        return dict(local)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    s = torch.tensor([local["particle_steps"], local["requests"]], dtype=torch.float64, device=dev)
    m = torch.tensor([local["wall_s"], local.get("device_s", 0.0)], dtype=torch.float64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    out = dict(local)
    out.update(particle_steps=float(s[0]), requests=int(s[1]), wall_s=float(m[0]), device_s=float(m[1]))
    out["throughput"] = out["particle_steps"] / out["wall_s"] if out["wall_s"] > 0 else 0.0
    return out


def serve_sharded(server, requests, world: int, rank: int, realtime: bool = True) -> dict:
    """Serve this rank's shard of one arrival stream (every rank passes the same
    `requests`; shard_requests picks the same disjoint shards on each). Each request
    keeps its arrival time, so a rank sees a thinned copy of the stream. Returns the
    server's local result with "mine" (the request ids served here) and "combined":
    particle-steps and requests summed, wall and device time max-reduced, and the
    step-latency percentiles over the steps of all ranks."""
    import numpy as np

    idx = shard_requests(requests, world)[rank]
    res = server.run([requests[k] for k in idx], realtime=realtime)
    local = {"particle_steps": float(res["particle_steps"]), "requests": res["requests"], "wall_s": res["wall_s"],
             "device_s": server.device_ms / 1e3}
    comb = combine_metrics(local, world)
    lat = np.asarray(res["step_ms"], np.float64)
    if world > 1:
        import torch.distributed as dist

        parts = [None] * world
        dist.all_gather_object(parts, lat.tolist())
        lat = np.concatenate([np.asarray(p, np.float64) for p in parts])
    comb["step_ms_p50"] = float(np.percentile(lat, 50))
    comb["step_ms_p99"] = float(np.percentile(lat, 99))
    comb["device_throughput"] = comb["particle_steps"] / comb["device_s"] if comb["device_s"] > 0 else 0.0
    res["mine"] = [requests[k].rid for k in idx]
    res["combined"] = comb
    return res
