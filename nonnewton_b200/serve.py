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
        seconds of wall clock from the start of the run; otherwise all are queued."""
        queue = sorted(requests, key=lambda r: r.arrival)
        qi = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        finished = []
        total_ps = 0
        while qi < len(queue) or self.resident:
            # retire finished requests
            done = [r for r in self.resident if r.done_steps >= r.steps]
            keep_idx = [k for k, r in enumerate(self.resident) if r.done_steps < r.steps]
            if done:  # one device-to-host copy of all finished results and stats
                ks = [k for k, r in enumerate(self.resident) if r.done_steps >= r.steps]
                xs = torch.cat([self.batch.scene_view(k, "x") for k in ks]).cpu().numpy()
                st = self.batch.engine.stats_range(0, len(self.resident))
                off = 0
                tf = now()
                for k in ks:
                    r = self.resident[k]
                    m = r.scene.particles.n
                    r.result_x = xs[off:off + m]
                    off += m
                    r.stats = st[k]
                    r.finished = tf
                    finished.append(r)
            # admit arrived requests that fit
            t = now()
            if not self.resident and qi < len(queue) and realtime and queue[qi].arrival > t:
                time.sleep(max(0.0, queue[qi].arrival - t))
                t = now()
            new = []
            n_res = sum(self.resident[k].scene.particles.n for k in keep_idx)
            c_res = sum(scene_grid_cells(self.resident[k].scene) for k in keep_idx)
            while qi < len(queue) and (not realtime or queue[qi].arrival <= t):
                r = queue[qi]
                if r.scene.particles.n > self.capacity:
                    raise ValueError(f"request {r.rid} exceeds the batch capacity")
                cells = scene_grid_cells(r.scene)
                if (n_res + r.scene.particles.n > self.capacity or c_res + cells > self.max_cells
                        or len(keep_idx) + len(new) >= self.max_scenes):
                    break
                r.admitted = t
                new.append(r)
                n_res += r.scene.particles.n
                c_res += cells
                qi += 1
            if done or new:
                self.resident = [self.resident[k] for k in keep_idx] + new
                if self.resident:
                    if self.batch.scenes and (keep_idx or not done):
                        self.batch.repack(keep_idx, [r.scene for r in new])
                    else:
                        self.batch.set([r.scene for r in self.resident])
                    self.repacks += 1
            if not self.resident:
                continue
            # advance all resident scenes by one chunk
            k = min(self.chunk, min(r.steps - r.done_steps for r in self.resident))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            self.batch.step(k, sync=True)
            e1.record(self.stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / k
            self.device_ms += ms * k
            self.chunks += 1
            for r in self.resident:
                r.done_steps += k
                r.step_ms.extend([ms] * k)
                total_ps += r.scene.particles.n * k
            # failure detection: a scene whose device status word is set (non-finite
            # state, neighbour overflow) is evicted at once; the others go on
            st = self.batch.engine.stats_range(0, len(self.resident))
            for r, y in zip(self.resident, st):
                if y["status"] != 0:
                    r.failed = y["status"]
                    r.done_steps = r.steps
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
