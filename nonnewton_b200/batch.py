"""Batched form: many scenes of uneven sizes packed into one segmented particle
array and advanced together by the same captured step graph.

Each scene keeps its own parameters, grid, solver loop state (per-scene convergence
masks inside the graph's while-loops) and statistics; scenes never interact (cell keys
are offset per scene, reductions are per scene, solids gather instead of receiving
atomics), so a scene's result does not depend on what it is batched with.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Engine
from .scene import Scene
from .sph import ParticleData


def scene_grid_cells(sc: Scene, cell_factor: int = 1, x_split: int = 1) -> int:
    """Cells of the scene's grid (edge h / cell_factor in y and z, that divided by
    x_split in x; Morton-ordered rows), as libnnsph lays it out."""
    p = sc.param
    h = p.support_radius
    g = []
    for k in range(3):
        ext = (p.domain_end[k] - p.domain_start[k]) + 4 * h
        edge = h / cell_factor * (1.0 + 1e-3) / (x_split if k == 0 else 1)  # the library's 0.1 % margin
        g.append(int(min(65535, max(1, np.ceil(ext / edge) + 1))))
    mb = 0
    while (1 << mb) < max(g[1], g[2]):
        mb += 1
    return g[0] * (1 << (2 * mb))


class Batch:
    """Scenes packed one after another in a ParticleData of `capacity` rows."""

    def __init__(self, capacity: int, max_scenes: int, max_neighbors: int = 64, max_cells: int = 0,
                 device="cuda", block: int | None = None):
        self.capacity = int(capacity)
        self.pd = ParticleData(self.capacity, device=device)
        self.engine = Engine(self.capacity, max_scenes, max_neighbors, max_cells, device=device)
        if block:
            self.engine.set_block_size(block)
        self.scenes: list[Scene] = []
        self.starts: list[int] = []
        self.n = 0
        self.cell_factor = 1
        self._cparams: dict = {}
        self._pin = None      # pinned staging buffers (see stage)
        self._pin_ev = None   # recorded after the last copies out of them

    # -- packing -----------------------------------------------------------------
    _STAGED = (("x", 3, torch.float32), ("m", 1, torch.float32), ("material", 1, torch.int32),
               ("is_dynamic", 1, torch.int32), ("phase_id", 1, torch.int32), ("volume", 1, torch.float32),
               ("density", 1, torch.float32))

    def stage(self, scenes: list[Scene]) -> dict | None:
        """The initial states of `scenes`, written field by field into pinned host
        buffers of the batch's capacity (allocated once), so that packing them is one
        asynchronous copy per field. Host work only: a server stages arriving scenes
        while the GPU runs the batch."""
        if not scenes:
            return None
        n = sum(sc.particles.n for sc in scenes)
        if n > self.capacity:
            raise ValueError(f"{n} particles exceed the batch capacity {self.capacity}")
        if self._pin is None:
            self._pin = {name: torch.empty((self.capacity, w) if w > 1 else (self.capacity,), dtype=dt,
                                           pin_memory=True) for name, w, dt in self._STAGED}
        if self._pin_ev is not None:
            self._pin_ev.synchronize()  # the previous staging's copies have left the buffers
        buf = {name: t.numpy() for name, t in self._pin.items()}
        off = 0
        for sc in scenes:
            p = sc.particles
            sl = slice(off, off + p.n)
            buf["x"][sl] = p.x.reshape(-1, 3)
            buf["m"][sl] = p.mass
            buf["material"][sl] = p.material
            buf["is_dynamic"][sl] = p.is_dynamic
            buf["phase_id"][sl] = p.phase_id
            buf["volume"][sl] = sc.param.volume0
            buf["density"][sl] = sc.param.density0
            off += p.n
        return {"n": n, **{name: t[:n] for name, t in self._pin.items()}}

    def _write_staged(self, st: dict, start: int):
        """Rows [start, start + n) from a staging of `stage`: the initial state of each
        scene (x_0 = x, zero velocity and acceleration, volume0, density0)."""
        pd = self.pd
        sl = slice(start, start + st["n"])
        for name, _, _ in self._STAGED:
            getattr(pd, name)[sl].copy_(st[name], non_blocking=True)
        pd.x_0[sl].copy_(pd.x[sl])
        for name in ("v", "acceleration", "dfsph_factor", "density_adv"):
            getattr(pd, name)[sl].zero_()
        self._pin_ev = torch.cuda.Event()
        self._pin_ev.record()

    def set(self, scenes: list[Scene], initialize: bool = True, staged: dict | None = None):
        """Pack `scenes` from their initial states and initialise them. `staged` is
        `stage(scenes)` when the caller made it beforehand."""
        total = sum(sc.particles.n for sc in scenes)
        if total > self.capacity:
            raise ValueError(f"{total} particles exceed the batch capacity {self.capacity}")
        self.scenes, self.starts = list(scenes), []
        start = 0
        for sc in scenes:
            self.starts.append(start)
            start += sc.particles.n
        if scenes:
            self._write_staged(staged if staged is not None else self.stage(scenes), 0)
        self.n = total
        self._bind_and_describe()
        if initialize:
            self.engine.initialize()

    def _bind_and_describe(self):
        """Bind the state and describe the scenes. A scene's parameter struct is made
        when it is packed and reused while it stays resident."""
        cache = {}
        for sc in self.scenes:
            ent = self._cparams.get(id(sc))
            cache[id(sc)] = ent if ent is not None and ent[0] is sc else (sc, sc.param.to_c())
        self._cparams = cache
        self.engine.bind(self.pd, self.n)
        self.engine.set_scenes([(s, sc.particles.n, sc.particles.n_fluid, cache[id(sc)][1])
                                for s, sc in zip(self.starts, self.scenes)])

    def repack(self, keep: list[int], new: list[Scene], staged: dict | None = None):
        """Continuous batching: keep the resident scenes `keep` (indices into the
        current list) with their current states, drop the others, append `new` ones
        from their initial states (`staged` = `stage(new)` when made beforehand). Only
        the new scenes need initialising, but the static-boundary volumes of all scenes
        are recomputed (same values)."""
        pd = self.pd
        dev = pd.x.device
        # source row of every kept particle: its new row plus its scene's shift
        lens = [self.scenes[k].particles.n for k in keep]
        m = sum(lens)
        shift, at = [], 0
        for k, ln in zip(keep, lens):
            shift.append(self.starts[k] - at)
            at += ln
        idx = torch.arange(m, device=dev)
        if m:
            idx += torch.repeat_interleave(torch.tensor(shift, dtype=torch.long, device=dev),
                                           torch.tensor(lens, dtype=torch.long, device=dev), output_size=m)
        for name in ("x", "x_0", "v", "acceleration", "volume", "m", "density", "pressure", "dfsph_factor",
                     "density_adv", "material", "is_dynamic", "phase_id", "strain_rate_norm",
                     "nonnewton_viscosity", "stress", "rotations"):
            t = getattr(pd, name)
            t[:m] = t.index_select(0, idx)
        scenes = [self.scenes[k] for k in keep]
        starts, start = [], 0
        for sc in scenes:
            starts.append(start)
            start += sc.particles.n
        total = start + sum(sc.particles.n for sc in new)
        if total > self.capacity:
            raise ValueError("repack exceeds capacity")
        if new:
            self._write_staged(staged if staged is not None else self.stage(new), start)
        for sc in new:
            starts.append(start)
            scenes.append(sc)
            start += sc.particles.n
        self.scenes, self.starts, self.n = scenes, starts, total
        self._bind_and_describe()
        self.engine.initialize()

    # -- stepping ----------------------------------------------------------------
    def step(self, nsteps: int = 1, sync: bool = True, resume: bool = False):
        self.engine.step(nsteps, sync=sync, resume=resume)

    def scene_view(self, k: int, name: str) -> torch.Tensor:
        s = self.starts[k]
        return getattr(self.pd, name)[s:s + self.scenes[k].particles.n]

    def stats(self, k: int) -> dict:
        return self.engine.stats(k)
