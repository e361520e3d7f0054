"""Served form: continuous batching of scene-solve requests on one GPU.

Requests (a scene and a step count) arrive over time. The server keeps the state of
every admitted scene resident in one segmented particle array (`Batch`), admits
waiting requests as slots and memory free up (admission by HBM footprint: the
particle capacity of the batch, and a scene-slot limit), and advances all resident
scenes together with the captured step graph, in chunks of a few steps. Between
chunks, finished requests retire (their final state is copied out) and newly
arrived ones are packed in. Because scenes never interact, a request's result does
not depend on what it was batched with.

Reported: throughput (particle-steps/s over the whole run), per-request latency, and
p50/p99 of the batch step latency seen by the requests.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import Batch, scene_grid_cells
from .scene import Scene


@dataclass
class Request:
    rid: int
    scene: Scene
    steps: int
    arrival: float
    admitted: float | None = None
    finished: float | None = None
    done_steps: int = 0
    step_ms: list = field(default_factory=list)
    result_x: np.ndarray | None = None
    stats: dict | None = None
    failed: int = 0          # NN_ERR_* status that evicted the request, 0 if it completed


def footprint_bytes(n_particles: int, max_neighbors: int = 64) -> int:
    """Device bytes per resident particle of a context (working sets, lists, solver
    vectors), used for admission by HBM footprint."""
    return int(n_particles) * (560 + 4 * max_neighbors)


class Server:
    def __init__(self, capacity: int, max_scenes: int = 256, chunk: int = 10, max_neighbors: int = 64,
                 max_cells: int | None = None, device="cuda", block: int | None = None):
        self.capacity = int(capacity)
        self.max_scenes = int(max_scenes)
        self.chunk = int(chunk)
        self.max_cells = int(max_cells or 32 * 1024 * 1024)
        self.batch = Batch(capacity, max_scenes, max_neighbors, self.max_cells, device=device, block=block)
        self.resident: list[Request] = []
        self.stream = torch.cuda.current_stream()
        self.chunks = 0
        self.repacks = 0
        self.device_ms = 0.0

    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        """Serve `requests` (sorted by arrival). With `realtime`, arrival times are
        seconds of wall clock from the start of the run; otherwise all are queued.

        The host work of a chunk boundary overlaps the chunk in flight: which requests
        retire after it is known from the step counts, so the admissions are planned
        while the GPU runs. Then the loop waits for the chunk, reads the status words
        (a failed scene retires at once), and enqueues back to back the copy of the
        finished results into pinned memory, the repack and the next chunk. Results
        reach their requests when their copy has landed."""
        queue = sorted(requests, key=lambda r: r.arrival)
        qi = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        finished = []
        total_ps = 0
        cells: dict[int, int] = {}  # grid cells of each request's scene (admission by footprint)

        def cells_of(r):
            c = cells.get(id(r))
            if c is None:
                c = cells[id(r)] = scene_grid_cells(r.scene)
            return c

        pending = None  # the chunk in flight: (start event, end event, steps)
        outbox = []     # retired requests whose results are on their way to the host

        def deliver(block: bool):
            nonlocal outbox
            left = []
            for reqs, stats, host, ev in outbox:
                if not block and not ev.query():
                    left.append((reqs, stats, host, ev))
                    continue
                ev.synchronize()
                tf = now()
                xs = host.numpy()
                off = 0
                for r, y in zip(reqs, stats):
                    m = r.scene.particles.n
                    r.result_x = xs[off:off + m].copy()
                    off += m
                    r.stats = y
                    r.finished = tf
                    finished.append(r)
            outbox = left

        while qi < len(queue) or self.resident or pending is not None:
            # plan while the chunk in flight runs: who retires after it, who is admitted
            keep_idx = [k for k, r in enumerate(self.resident) if r.done_steps < r.steps]
            t = now()
            if not self.resident and qi < len(queue) and realtime and queue[qi].arrival > t:
                time.sleep(max(0.0, queue[qi].arrival - t))
                t = now()
            new = []
            n_res = sum(self.resident[k].scene.particles.n for k in keep_idx)
            c_res = sum(cells_of(self.resident[k]) for k in keep_idx)
            while qi < len(queue) and (not realtime or queue[qi].arrival <= t):
                r = queue[qi]
                if r.scene.particles.n > self.capacity:
                    raise ValueError(f"request {r.rid} exceeds the batch capacity")
                c = cells_of(r)
                if (n_res + r.scene.particles.n > self.capacity or c_res + c > self.max_cells
                        or len(keep_idx) + len(new) >= self.max_scenes):
                    break
                r.admitted = t
                new.append(r)
                n_res += r.scene.particles.n
                c_res += c
                qi += 1
            staged = self.batch.stage([r.scene for r in new])  # pinned host copies, made while the GPU runs
            # the chunk's end: its timing, and failure detection (a scene whose device
            # status word is set, from a non-finite state or a neighbour overflow, is
            # evicted at once; the others go on)
            st = None
            if pending is not None:
                e0, e1, k = pending
                e1.synchronize()
                ms = e0.elapsed_time(e1) / k
                self.device_ms += ms * k
                for r in self.resident:
                    r.step_ms.extend([ms] * k)
                st = self.batch.engine.stats_range(0, len(self.resident))
                for r, y in zip(self.resident, st):
                    if y["status"] != 0:
                        r.failed = y["status"]
                        r.done_steps = r.steps
                pending = None
            done_idx = [k for k, r in enumerate(self.resident) if r.done_steps >= r.steps]
            keep_idx = [k for k, r in enumerate(self.resident) if r.done_steps < r.steps]
            if done_idx:  # one device-to-host copy of all finished results, into pinned memory
                xs = torch.cat([self.batch.scene_view(k, "x") for k in done_idx])
                host = torch.empty(xs.shape, dtype=xs.dtype, pin_memory=True)
                host.copy_(xs, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.stream)
                if st is None:
                    st = self.batch.engine.stats_range(0, len(self.resident))
                outbox.append(([self.resident[k] for k in done_idx], [st[k] for k in done_idx], host, ev))
            if done_idx or new:
                done = bool(done_idx)
                self.resident = [self.resident[k] for k in keep_idx] + new
                if self.resident:
                    if self.batch.scenes and (keep_idx or not done):
                        self.batch.repack(keep_idx, [r.scene for r in new], staged=staged)
                    else:  # nothing kept: the resident scenes are the new ones
                        self.batch.set([r.scene for r in self.resident], staged=staged)
                    self.repacks += 1
            if self.resident:  # advance all resident scenes by one chunk
                k = min(self.chunk, min(r.steps - r.done_steps for r in self.resident))
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(self.stream)
                self.batch.step(k, sync=True)
                e1.record(self.stream)
                pending = (e0, e1, k)
                self.chunks += 1
                for r in self.resident:
                    r.done_steps += k
                    total_ps += r.scene.particles.n * k
            deliver(block=False)
        deliver(block=True)
        wall = now()
        lat = np.concatenate([np.asarray(r.step_ms) for r in finished]) if finished else np.zeros(1)
        return {
            "requests": len(finished),
            "wall_s": wall,
            "particle_steps": total_ps,
            "throughput": total_ps / wall if wall > 0 else 0.0,
            "step_ms_p50": float(np.percentile(lat, 50)),
            "step_ms_p99": float(np.percentile(lat, 99)),
            "request_s_p50": float(np.percentile([r.finished - r.arrival for r in finished], 50)),
            "request_s_p99": float(np.percentile([r.finished - r.arrival for r in finished], 99)),
            "max_density_err": max(((r.stats or {}).get("avg_density_err", 0.0) for r in finished if not r.failed),
                                   default=0.0),
            "failed": [r.rid for r in finished if r.failed],
            "device_throughput": total_ps / (self.device_ms / 1e3) if self.device_ms > 0 else 0.0,
            "repacks": self.repacks,
            "chunks": self.chunks,
            "finished": finished,
        }


def run_plain(requests: list[Request], max_neighbors: int = 64) -> dict:
    """The plain per-scene loop: each request alone, one after another."""
    total_ps = 0
    cap = max(r.scene.particles.n for r in requests)
    cells = max(scene_grid_cells(r.scene) for r in requests)
    b = Batch(cap, 1, max_neighbors, cells)  # one context, reused: its step graph is captured once
    t0 = time.perf_counter()
    for r in requests:
        b.set([r.scene])
        b.step(r.steps, sync=True)
        r.result_x = b.scene_view(0, "x").cpu().numpy()
        r.stats = b.stats(0)
        total_ps += r.scene.particles.n * r.steps
    wall = time.perf_counter() - t0
    b.engine.close()
    return {"requests": len(requests), "wall_s": wall, "particle_steps": total_ps,
            "throughput": total_ps / wall}
