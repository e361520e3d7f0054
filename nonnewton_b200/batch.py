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


def scene_grid_cells(sc: Scene, cell_factor: int = 1) -> int:
    """Cells of the scene's grid (edge h / cell_factor, Morton-ordered rows), as
    libnnsph lays it out."""
    p = sc.param
    h = p.support_radius
    g = []
    for k in range(3):
        ext = (p.domain_end[k] - p.domain_start[k]) + 4 * h
        g.append(int(min(65535, max(1, np.ceil(ext / (h / cell_factor)) + 1))))
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

    # -- packing -----------------------------------------------------------------
    def _write_scene(self, sc: Scene, start: int):
        ps = sc.particles
        dev = self.pd.x.device
        sl = slice(start, start + ps.n)
        x = torch.from_numpy(np.ascontiguousarray(ps.x, np.float32)).to(dev)
        pd = self.pd
        pd.x[sl] = x
        pd.x_0[sl] = x
        pd.v[sl] = 0
        pd.acceleration[sl] = 0
        pd.volume[sl] = sc.param.volume0
        pd.m[sl] = torch.from_numpy(ps.mass).to(dev)
        pd.density[sl] = sc.param.density0
        pd.dfsph_factor[sl] = 0
        pd.density_adv[sl] = 0
        pd.material[sl] = torch.from_numpy(ps.material).to(dev)
        pd.is_dynamic[sl] = torch.from_numpy(ps.is_dynamic).to(dev)
        pd.phase_id[sl] = torch.from_numpy(ps.phase_id).to(dev)

    def set(self, scenes: list[Scene], initialize: bool = True):
        """Pack `scenes` from their initial states and initialise them."""
        total = sum(sc.particles.n for sc in scenes)
        if total > self.capacity:
            raise ValueError(f"{total} particles exceed the batch capacity {self.capacity}")
        self.scenes, self.starts = list(scenes), []
        start = 0
        for sc in scenes:
            self._write_scene(sc, start)
            self.starts.append(start)
            start += sc.particles.n
        self.n = total
        self._bind_and_describe()
        if initialize:
            self.engine.initialize()

    def _bind_and_describe(self):
        self.engine.bind(self.pd, self.n)
        self.engine.set_scenes([(s, sc.particles.n, sc.particles.n_fluid, sc.param.to_c())
                                for s, sc in zip(self.starts, self.scenes)])

    def repack(self, keep: list[int], new: list[Scene]):
        """Continuous batching: keep the resident scenes `keep` (indices into the
        current list) with their current states, drop the others, append `new` ones
        from their initial states. Only the new scenes need initialising, but the
        static-boundary volumes of all scenes are recomputed (same values)."""
        pd = self.pd
        rows = [torch.arange(self.starts[k], self.starts[k] + self.scenes[k].particles.n, device=pd.x.device)
                for k in keep]
        idx = torch.cat(rows) if rows else torch.zeros(0, dtype=torch.long, device=pd.x.device)
        m = int(idx.numel())
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
        for sc in new:
            self._write_scene(sc, start)
            starts.append(start)
            scenes.append(sc)
            start += sc.particles.n
        self.scenes, self.starts, self.n = scenes, starts, total
        self._bind_and_describe()
        self.engine.initialize()

    # -- stepping ----------------------------------------------------------------
    def step(self, nsteps: int = 1, sync: bool = True):
        self.engine.step(nsteps, sync=sync)

    def scene_view(self, k: int, name: str) -> torch.Tensor:
        s = self.starts[k]
        return getattr(self.pd, name)[s:s + self.scenes[k].particles.n]

    def stats(self, k: int) -> dict:
        return self.engine.stats(k)
