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
    max_err: float = 0.0     # largest average density error at the end of any of its steps


# Device bytes of a resident particle, from what a server allocates per particle of
# its capacity: the context's two sorted working sets (position+volume 16, velocity+mass
# 16, mass 4, density 4, flags 4, id 4: 2 x 48), its per-slot scratch (scene of id 4,
# acceleration 16, alpha / rho_adv / kappa / strain rate / viscosity 20, slot of id 4,
# sort key / rank / source 12), the neighbour counts 4 and 4 B per list entry, the CG
# vectors (x, r, z, p, Ap and the matvec's positions: 6 x 16, coefficients 8,
# preconditioner 24) and the elastic index 4; plus
# the batch's ParticleData fields (168: x, x_0, v, a 48; six scalars 24; four int32 16;
# color 12; strain rate and viscosity 8; stress 24; rotations 36). A grid cell costs
# CELL_BYTES (its count / start).
CTX_BYTES_PER_PARTICLE = 96 + 56 + 4 + 128 + 4
PD_BYTES_PER_PARTICLE = 168
CELL_BYTES = 4
DEFAULT_RESERVE_BYTES = 4 << 30  # left free for torch, graphs and the repack's temporaries


def footprint_bytes(n_particles: int, max_neighbors: int = 64, cells: int = 0) -> int:
    """Device bytes that `n_particles` resident particles (and `cells` grid cells) take
    in a server's batch; admission and the batch's size both follow this model."""
    per = CTX_BYTES_PER_PARTICLE + PD_BYTES_PER_PARTICLE + 4 * int(max_neighbors)
    return int(n_particles) * per + CELL_BYTES * int(cells)


def hbm_budget(free_bytes: int | None = None, reserve_bytes: int | None = None, device=None) -> int:
    """Device bytes a server may take: the free memory (torch.cuda.mem_get_info, or
    `free_bytes`) minus a reserve (DEFAULT_RESERVE_BYTES unless given)."""
    if free_bytes is None:
        free_bytes, _ = torch.cuda.mem_get_info(device)
    reserve = DEFAULT_RESERVE_BYTES if reserve_bytes is None else int(reserve_bytes)
    return max(0, int(free_bytes) - reserve)


def plan_pools(budget: int, max_neighbors: int = 64, cells_per_particle: float = 4.0) -> tuple[int, int]:
    """The largest (particles, grid cells) pools, cells at `cells_per_particle` per
    particle, whose footprint fits `budget` bytes."""
    per = footprint_bytes(1, max_neighbors) + CELL_BYTES * cells_per_particle
    capacity = int(budget // per)
    return capacity, int(capacity * cells_per_particle)


class Server:
    """Continuous batching on one GPU. The batch's particle and grid-cell pools are
    sized from the device memory budget (hbm_budget: free memory minus a reserve,
    through footprint_bytes), or from the caller's `capacity` / `max_cells` where those
    are smaller (a cap on resident work bounds the step latency); a request is
    admitted when its particles and cells fit what the pools have left.

    With `autotune`, the launch shape is tuned (autotune.py) on the first packing that
    fills at least `tune_fill` of the particle pool while every resident scene is still
    at its initial state, and kept for the server's lifetime."""

    def __init__(self, capacity: int | None = None, max_scenes: int = 256, chunk: int = 10, max_neighbors: int = 64,
                 max_cells: int | None = None, device="cuda", block: int | None = None,
                 hbm_free: int | None = None, hbm_reserve: int | None = None, cells_per_particle: float = 4.0,
                 autotune: bool = False, tune_fill: float = 0.5, tune_candidates=None, batch=None):
        self.budget = hbm_budget(hbm_free, hbm_reserve, device if batch is None else None)
        cap_hbm, cells_hbm = plan_pools(self.budget, max_neighbors, cells_per_particle)
        self.capacity = min(int(capacity), cap_hbm) if capacity else cap_hbm
        self.max_cells = int(max_cells) if max_cells else int(self.capacity * cells_per_particle)
        self.max_neighbors = int(max_neighbors)
        if self.capacity <= 0 or footprint_bytes(self.capacity, max_neighbors, self.max_cells) > self.budget:
            raise ValueError(f"a batch of {self.capacity} particles and {self.max_cells} cells "
                             f"({footprint_bytes(self.capacity, max_neighbors, self.max_cells)} B) does not fit the "
                             f"device budget of {self.budget} B")
        self.max_scenes = int(max_scenes)
        self.chunk = int(chunk)
        self.batch = batch if batch is not None else Batch(self.capacity, max_scenes, max_neighbors, self.max_cells,
                                                           device=device, block=block)
        self.resident: list[Request] = []
        self.stream = torch.cuda.current_stream()
        self.chunks = 0
        self.repacks = 0
        self.device_ms = 0.0
        self.autotune = autotune
        self.tune_fill = float(tune_fill)
        self.tune_candidates = tune_candidates
        self.tuning = None  # the autotuner's result, once it ran

    def particle_bytes(self, n: int) -> int:
        return footprint_bytes(n, self.max_neighbors)

    def fits(self, used_particles: int, used_cells: int, n: int, cells: int) -> bool:
        """Admission by footprint: the request's particles and cells within what the
        particle pool and the cell pool have left."""
        return (self.particle_bytes(used_particles + n) <= self.particle_bytes(self.capacity)
                and CELL_BYTES * (used_cells + cells) <= CELL_BYTES * self.max_cells)

    def tune(self) -> dict:
        """Autotune the launch shape on the resident batch, which must be at its
        scenes' initial states (the tuner restarts it from them for each candidate)."""
        from .autotune import autotune

        self.tuning = autotune(self.batch, candidates=self.tune_candidates)
        return self.tuning

    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        """Serve `requests` (sorted by arrival). With `realtime`, arrival times are
        seconds of wall clock from the start of the run; otherwise all are queued.

        The host work of a chunk boundary overlaps the chunk in flight: which requests
        retire after it is known from the step counts, so the admissions are planned
        while the GPU runs. Then the loop waits for the chunk, reads the status words
        (a failed scene retires at once), and enqueues back to back the copy of the
        finished results into pinned memory, the repack and the next chunk. Results
        reach their requests when their copy has landed.

        Every step of a chunk is its own launch with an event after it (the steps
        after the first continue from the resident state, NN_STEP_RESUME), so each
        request records the latency of each of its steps; the chunk's first event is
        recorded before the repack, so the first step after one includes it, as the
        requests see it. The density error of every step comes from the scenes' running
        maximum (nn_stats.max_avg_density_err), read at each chunk's end."""
        queue = sorted(requests, key=lambda r: r.arrival)
        qi = 0
        self.chunks = self.repacks = self.batch_steps = 0  # counters of this run
        self.device_ms = 0.0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        finished = []
        total_ps = 0
        cells: dict[int, int] = {}  # grid cells of each request's scene (admission by footprint)

        layout = (getattr(self.batch, "cell_factor", 1), getattr(getattr(self.batch, "engine", None), "x_split", 1))

        def cells_of(r):
            c = cells.get(id(r))
            if c is None:
                c = cells[id(r)] = scene_grid_cells(r.scene, *layout)
            return c

        pending = None  # the chunk in flight: (events, steps)
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
                c = cells_of(r)
                if not self.fits(0, 0, r.scene.particles.n, c):
                    raise ValueError(f"request {r.rid} ({r.scene.particles.n} particles, {c} cells) exceeds the "
                                     f"batch's pools ({self.capacity} particles, {self.max_cells} cells)")
                if not self.fits(n_res, c_res, r.scene.particles.n, c) or len(keep_idx) + len(new) >= self.max_scenes:
                    break
                r.admitted = t
                new.append(r)
                n_res += r.scene.particles.n
                c_res += c
                qi += 1
            staged = self.batch.stage([r.scene for r in new])  # pinned host copies, made while the GPU runs
            # the chunk's end: the latency of each of its steps, and failure detection (a
            # scene whose device status word is set, from a non-finite state or a
            # neighbour overflow, is evicted at once; the others go on)
            st = None
            if pending is not None:
                evs, k = pending
                evs[-1].synchronize()
                ms = [evs[j].elapsed_time(evs[j + 1]) for j in range(k)]
                self.device_ms += sum(ms)
                st = self.batch.engine.stats_range(0, len(self.resident))
                for r, y in zip(self.resident, st):
                    r.step_ms.extend(ms)
                    r.max_err = max(r.max_err, y.get("max_avg_density_err", y.get("avg_density_err", 0.0)))
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
            evs = [torch.cuda.Event(enable_timing=True)]
            evs[0].record(self.stream)  # before the repack: the chunk's first step includes it
            if done_idx or new:
                done = bool(done_idx)
                self.resident = [self.resident[k] for k in keep_idx] + new
                if self.resident:
                    if self.batch.scenes and (keep_idx or not done):
                        self.batch.repack(keep_idx, [r.scene for r in new], staged=staged)
                    else:  # nothing kept: the resident scenes are the new ones
                        self.batch.set([r.scene for r in self.resident], staged=staged)
                    self.repacks += 1
                    if (self.autotune and self.tuning is None and all(r.done_steps == 0 for r in self.resident)
                            and n_res >= self.tune_fill * self.capacity):
                        self.tune()
                        evs[0].record(self.stream)  # the tuner's steps are not the requests'
            if self.resident:  # advance all resident scenes by one chunk, one launch per step
                k = min(self.chunk, min(r.steps - r.done_steps for r in self.resident))
                for j in range(k):
                    self.batch.step(1, sync=(j == k - 1), resume=(j > 0))
                    evs.append(torch.cuda.Event(enable_timing=True))
                    evs[-1].record(self.stream)
                pending = (evs, k)
                self.chunks += 1
                self.batch_steps += k
                for r in self.resident:
                    r.done_steps += k
                    total_ps += r.scene.particles.n * k
            deliver(block=False)
        deliver(block=True)
        wall = now()
        lat = np.concatenate([np.asarray(r.step_ms) for r in finished]) if finished else np.zeros(1)
        ok = [r for r in finished if not r.failed]
        return {
            "requests": len(finished),
            "wall_s": wall,
            "particle_steps": total_ps,
            "throughput": total_ps / wall if wall > 0 else 0.0,
            "step_ms_p50": float(np.percentile(lat, 50)),
            "step_ms_p99": float(np.percentile(lat, 99)),
            "step_ms_max": float(lat.max()),
            "step_ms": lat,
            "request_s_p50": float(np.percentile([r.finished - r.arrival for r in finished], 50)),
            "request_s_p99": float(np.percentile([r.finished - r.arrival for r in finished], 99)),
            # largest average density error of any step of any completed request, in
            # kg/m^3 and in % of the request's rest density (the reference's maxError unit)
            "max_density_err": max((r.max_err for r in ok), default=0.0),
            "max_density_err_pct": max((100.0 * r.max_err / r.scene.param.density0 for r in ok), default=0.0),
            "failed": [r.rid for r in finished if r.failed],
            "device_throughput": total_ps / (self.device_ms / 1e3) if self.device_ms > 0 else 0.0,
            "repacks": self.repacks,
            "chunks": self.chunks,
            "batch_steps": self.batch_steps,
            "tuning": self.tuning,
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
