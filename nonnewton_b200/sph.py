"""The reference's object API for the SPH step, backed by libnnsph.so.

Mirrors SPH/main.py: the global `meta` (19-23), `ParticleData` (697-723),
`NeighborhoodSearchSparse` (764-853), `SPHBase` / `DFSPHSolver` (908-1848),
`initialize()` (1870-1895), `build_solver()` (196-203) and the headless main loop
(1909-1921). Field names, shapes and dtypes are the reference's; the fields are
torch CUDA tensors instead of Taichi fields. Every method runs sm_100a kernels
through the C ABI.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from . import _abi
from .config import Parameter, SimConfig
from .engine import Engine
from .scene import ParticleSet, export_ply_particles, geometry_path, load_particles, read_animation

FLUID, SOLID = _abi.NN_FLUID, _abi.NN_SOLID


class Meta:
    """Global simulation state (`meta`, SPH/main.py:19-23)."""


meta = Meta()


class ParticleData:
    """`ParticleData` (SPH/main.py:697-723): SoA particle fields on the GPU."""

    def __init__(self, particle_max_num: int, device="cuda"):
        n = int(particle_max_num)
        self.particle_max_num = n
        self.dim = 3
        f = dict(dtype=torch.float32, device=device)
        i = dict(dtype=torch.int32, device=device)
        self.phase_id = torch.zeros(n, **i)
        self.x = torch.zeros(n, 3, **f)
        self.x_0 = torch.zeros(n, 3, **f)
        self.v = torch.zeros(n, 3, **f)
        self.acceleration = torch.zeros(n, 3, **f)
        self.volume = torch.zeros(n, **f)
        self.m = torch.zeros(n, **f)
        self.density = torch.zeros(n, **f)
        self.pressure = torch.zeros(n, **f)
        self.material = torch.zeros(n, **i)
        self.color = torch.zeros(n, 3, **f)
        self.is_dynamic = torch.zeros(n, **i)
        self.particle_id = torch.arange(n, **i)
        self.dfsph_factor = torch.zeros(n, **f)
        self.density_adv = torch.zeros(n, **f)
        # NonNewton / Elasticity outputs (SPH/main.py:340-342, 1201-1203)
        self.strain_rate_norm = torch.zeros(n, **f)
        self.nonnewton_viscosity = torch.zeros(n, **f)
        self.stress = torch.zeros(n, 6, **f)
        self.rotations = torch.zeros(n, 9, **f)


def initialize_particles(pd: ParticleData, ps: ParticleSet, param: Parameter) -> None:
    """`initialize_particles` (SPH/main.py:735-758)."""
    dev = pd.x.device
    x = torch.from_numpy(np.ascontiguousarray(ps.x, dtype=np.float32)).to(dev)
    pd.x.copy_(x)
    pd.x_0.copy_(x)
    pd.v.zero_()
    pd.volume.fill_(param.volume0)
    pd.m.copy_(torch.from_numpy(ps.mass).to(dev))
    pd.density.fill_(param.density0)
    pd.pressure.zero_()
    pd.material.copy_(torch.from_numpy(ps.material).to(dev))
    pd.is_dynamic.copy_(torch.from_numpy(ps.is_dynamic).to(dev))
    pd.phase_id.copy_(torch.from_numpy(ps.phase_id).to(dev))
    pd.color.fill_(1.0)
    pd.rotations.zero_()
    pd.rotations[:, [0, 4, 8]] = 1.0


class NeighborhoodSearchSparse:
    """`NeighborhoodSearchSparse` (SPH/main.py:764-853) over the engine's cell-sorted
    lists. `neighbors` / `num_neighbors` are materialised in particle-id order, each
    row sorted by id and padded with -1, after every `run_search()`."""

    max_num_neighbors = 60

    def __init__(self, positions, num_particle, support_radius, domain_size, use_sparse_grid=False, engine=None):
        self.positions = positions
        self.num_particle = int(num_particle)
        self.support_radius = support_radius
        self.domain_size = np.asarray(domain_size)
        self.grid_size = support_radius
        self.grid_num = np.ceil(self.domain_size / self.grid_size).astype(int)
        self.engine = engine
        self._lists = None

    def run_search(self):
        solver = getattr(meta, "solver", None)
        if solver is not None:
            solver._settle()  # a pending step check may still change the positions
        self.engine.run_pass(_abi.NN_PASS_SEARCH)
        self._lists = None

    def _materialise(self):
        if self._lists is None:
            self._lists = self.engine.neighbors(self.num_particle, self.max_num_neighbors)
        return self._lists

    @property
    def num_neighbors(self):
        return self._materialise()[0]

    @property
    def neighbors(self):
        return self._materialise()[1]

    def get_num_neighbors(self, i):
        return int(self.num_neighbors[i])

    def get_neighbor(self, i, j):
        return int(self.neighbors[i, j])


class SPHBase:
    """`SPHBase` (SPH/main.py:908-1093): every method is one or more CUDA passes."""

    def __init__(self):
        self.gravity = meta.parm.gravity
        self.density_0 = meta.parm.density0
        self.dt = meta.parm.dt
        self.engine: Engine = meta.engine
        self.host_loop = False
        # re-run a step whose neighbour lists overflowed, with a larger cap
        self.grow_neighbors = True
        self._snap = None
        self._status = None
        self._pending = None       # the last call's unchecked status copy
        self._last_max = None      # largest neighbour count last seen

    def step(self):
        """SPHBase.step (SPH/main.py:915-940) as one CUDA-graph replay. With an animeFile,
        the frame's displacement (animate_particles, SPH/main.py:283-309) goes in first:
        the frame is the number of steps taken, the counter the reference's GUI loop
        keeps (its noGUI loop has none and fails on such a scene)."""
        anime = getattr(meta, "anime", None)
        d = None
        if anime is not None:
            frames, disp = anime
            rows = disp[frames == getattr(meta, "step_num", 0)]
            if len(rows):
                d = np.zeros(3, np.float32)
                for r in rows:  # the reference adds each matching row in turn
                    d = d + r
        self._advance(1, d)
        meta.ns._lists = None
        meta.step_num = getattr(meta, "step_num", 0) + 1
        if meta.config.get_cfg("exportPly"):
            torch.cuda.synchronize()
            export_ply_particles(meta.pd.x.cpu().numpy(), f"results/{meta.step_num - 1}.ply")

    def run(self, nsteps: int):
        """`nsteps` steps with the particle state kept resident in cell order between
        steps; meta.pd is written back once at the end (step by step with an animeFile)."""
        if getattr(meta, "anime", None) is not None:
            for _ in range(int(nsteps)):
                self.step()
            return
        self._advance(int(nsteps))
        meta.ns._lists = None
        meta.step_num = getattr(meta, "step_num", 0) + int(nsteps)

    def _advance(self, nsteps: int, displacement=None):
        """`nsteps` steps through the engine. The reference's neighbour list has 60
        slots (SPH/main.py:777-781) and store_neighbors writes past them unchecked
        (845-847); here the lists have a checked capacity, and with `grow_neighbors`
        work whose lists overflowed it runs again from the state before it (x and v,
        kept on the device) with the capacity raised past the largest count seen.

        A call whose last known neighbour count is within a quarter of the capacity
        reads the scene's status right after its steps (one host synchronisation).
        Otherwise the status is copied to pinned memory without waiting and checked
        when the next call (or stats()) begins; in the rare case that it overflowed,
        the state it started from is restored and its steps run again, checked, before
        the new work. Until then meta.pd holds that call's unverified result."""
        eng = self.engine
        if not self.grow_neighbors:
            if displacement is not None:
                eng.set_animation(0, displacement)
            eng.step(nsteps, sync=True, host_loop=self.host_loop)
            return
        self._settle()
        pd = meta.pd
        if self._snap is None or self._snap[0].shape != pd.x.shape:
            self._snap = (torch.empty_like(pd.x), torch.empty_like(pd.v))
            self._status = torch.zeros(2, dtype=torch.int32, pin_memory=torch.cuda.is_available())
        self._snap[0].copy_(pd.x)
        self._snap[1].copy_(pd.v)
        near = self._last_max is None or 4 * self._last_max >= 3 * eng.max_neighbors
        if displacement is not None:
            eng.set_animation(0, displacement)
        eng.step(nsteps, sync=True, host_loop=self.host_loop)
        if near:
            self._check(nsteps, displacement)
        else:
            eng.status_async(self._status)
            self._pending = (nsteps, displacement)

    def _check(self, nsteps, displacement):
        """Status after the steps just enqueued: on overflow, grow and run them again."""
        eng = self.engine
        while True:
            st = eng.stats(0)
            self._last_max = st["max_neighbors_seen"]
            if st["status"] != _abi.NN_ERR_NEIGHBOR_OVERFLOW or eng.max_neighbors >= 1024:
                return
            self._rerun(nsteps, displacement, st["max_neighbors_seen"])

    def _rerun(self, nsteps, displacement, seen):
        eng = self.engine
        cap = max(seen, eng.max_neighbors) * 5 // 4
        eng.set_neighbor_cap(min(1024, (cap + 7) // 8 * 8))
        meta.pd.x.copy_(self._snap[0])
        meta.pd.v.copy_(self._snap[1])
        if getattr(meta, "num_elastic_bodies", 0):
            eng.initialize()  # re-sized rest lists, rebuilt from x_0 (the same rest state)
        if displacement is not None:
            eng.set_animation(0, displacement)
        eng.step(nsteps, sync=True, host_loop=self.host_loop)

    def _settle(self):
        """Check the previous call's status copy (see _advance)."""
        if self._pending is None:
            return
        nsteps, displacement = self._pending
        self._pending = None
        self.engine.status_wait()
        status, seen = (int(v) for v in self._status)
        self._last_max = seen
        if status == _abi.NN_ERR_NEIGHBOR_OVERFLOW:
            self._rerun(nsteps, displacement, seen)
            self._check(nsteps, displacement)

    def _grow_cap(self, st):
        cap = max(st["max_neighbors_seen"], self.engine.max_neighbors) * 5 // 4
        self.engine.set_neighbor_cap(min(1024, (cap + 7) // 8 * 8))

    def initialize(self):
        """SPHBase.initialize (SPH/main.py:957-960) and the elastic rest state; with
        `grow_neighbors`, again with larger lists while they overflow."""
        self._settle()
        self.engine.initialize()
        while self.grow_neighbors and self.engine.max_neighbors < 1024:
            st = self.engine.stats(0)
            if st["status"] != _abi.NN_ERR_NEIGHBOR_OVERFLOW:
                break
            self._grow_cap(st)
            self.engine.initialize()
        meta.ns._lists = None

    def _pass(self, p):
        self._settle()
        self.engine.run_pass(p)

    def clear_accelerations(self):
        self._pass(_abi.NN_PASS_CLEAR_ACCELERATIONS)

    def compute_densities(self):
        self._pass(_abi.NN_PASS_DENSITIES)

    def compute_static_boundary_volume(self):
        self._pass(_abi.NN_PASS_STATIC_BOUNDARY_VOLUME)

    def compute_moving_boundary_volume(self):
        self._pass(_abi.NN_PASS_MOVING_BOUNDARY_VOLUME)

    def enforce_boundary_3D(self, positions=None, vel=None, particle_type=None):
        """Both materials in one pass (the reference calls it for FLUID then SOLID)."""
        self._pass(_abi.NN_PASS_ENFORCE_BOUNDARY)

    def advect(self):
        self._pass(_abi.NN_PASS_ADVECT)

    def stats(self) -> dict:
        self._settle()
        return self.engine.stats(0)


class DFSPHSolver(SPHBase):
    """`DFSPHSolver` (SPH/main.py:1519-1848)."""

    def __init__(self):
        super().__init__()
        p = meta.parm
        self.enable_divergence_solver = p.enable_divergence_solver
        self.m_max_iterations_v = p.max_iterations_v
        self.m_max_iterations = p.max_iterations
        self.m_eps = p.m_eps
        self.max_error_V = p.max_error_v
        self.max_error = p.max_error
        self.num_particles = meta.particle_max_num
        self.use_surfaceTensionModel = p.use_surface_tension
        self.use_nonNewtonianModel = p.use_nonnewtonian
        self.use_viscosityModel = p.use_viscosity

    def substep(self):
        self._pass(_abi.NN_PASS_SUBSTEP)

    def compute_DFSPH_factor(self):
        self._pass(_abi.NN_PASS_DFSPH_FACTOR)

    def divergence_solve(self):
        self._pass(_abi.NN_PASS_DIVERGENCE_SOLVE)

    def compute_non_pressure_forces(self):
        self._pass(_abi.NN_PASS_NON_PRESSURE_FORCES)

    def non_pressure_advect(self):
        self._pass(_abi.NN_PASS_NON_PRESSURE_ADVECT)

    def pressure_solve(self):
        self._pass(_abi.NN_PASS_PRESSURE_SOLVE)

    def elasticity_substep(self):
        self._pass(_abi.NN_PASS_ELASTICITY)


def build_solver():
    """`build_solver` (SPH/main.py:196-203)."""
    solver_type = meta.config.get_cfg("simulationMethod")
    if solver_type == 4:
        meta.solver = DFSPHSolver()
        return meta.solver
    raise NotImplementedError(f"Solver type {solver_type} has not been implemented.")


def initialize(config: SimConfig | str | dict | None = None, particles: ParticleSet | None = None,
               quirks: bool = False, max_neighbors: int = 64, device="cuda", tuning: dict | None = None,
               precision: str = "f32"):
    """`initialize()` (SPH/main.py:1870-1895): parameters, particles, fields, the
    neighbour search object and the CUDA engine (which also sets up elastic bodies)."""
    if isinstance(config, str):
        config = SimConfig(config)
    elif isinstance(config, dict):
        config = SimConfig(config=config)
    if config is not None:
        meta.config = config
    meta.parm = Parameter.from_config(meta.config, quirks=quirks)
    meta.solver = None
    ps = particles if particles is not None else load_particles(meta.config, meta.parm)
    meta.phase_info = ps.phase_info
    meta.particle_max_num = ps.n
    meta.fluid_particle_num = ps.n_fluid
    meta.pd = ParticleData(ps.n, device=device)
    initialize_particles(meta.pd, ps, meta.parm)
    meta.engine = Engine(max(ps.n, 1), 1, max_neighbors, device=device, precision=precision)
    if tuning:
        meta.engine.set_tuning(tuning.get("block", 0), tuning.get("unroll", 0), tuning.get("cell_factor", 0))
        meta.engine.set_x_split(tuning.get("x_split", 0))
    meta.engine.bind(meta.pd)
    meta.engine.set_scenes([(0, ps.n, ps.n_fluid, meta.parm.to_c())])
    meta.ns = NeighborhoodSearchSparse(meta.pd.x, ps.n, meta.parm.support_radius, meta.parm.domain_size,
                                       use_sparse_grid=True, engine=meta.engine)
    meta.num_elastic_bodies = len([p for p in ps.phase_info.values() if getattr(p, "solid_type", 0) == 2])
    meta.step_num = 0
    anime = meta.config.get_cfg("animeFile", None)
    meta.anime = read_animation(geometry_path(anime, meta.config.scene_path)) if anime else None
    return meta


def main(scene_path: str):
    """Headless `main()` (the reference's noGUI branch, SPH/main.py:1909-1921)."""
    initialize(scene_path)
    solver = build_solver()
    solver.initialize()
    meta.step_num = 0
    for _ in range(int(meta.config.get_cfg("maxStep", 1))):
        solver.step()
    return meta


# ---------------------------------------------------------------- checkpoint / resume
CHECKPOINT_FIELDS = ("x", "x_0", "v", "acceleration", "volume", "m", "density", "pressure", "dfsph_factor",
                     "density_adv", "material", "is_dynamic", "phase_id", "strain_rate_norm",
                     "nonnewton_viscosity", "stress", "rotations")


def save_checkpoint(path: str) -> None:
    """Full particle state, step counter and scene configuration (the reference only
    exports positions to PLY, SPH/main.py:939-940). Resuming runs the same kernels in
    the same order, so the continuation is bit-identical."""
    torch.cuda.synchronize()
    torch.save({"fields": {k: getattr(meta.pd, k).detach().cpu() for k in CHECKPOINT_FIELDS},
                "step_num": getattr(meta, "step_num", 0), "config": meta.config.config,
                "quirks": bool(meta.parm.quirks), "n_fluid": int(meta.fluid_particle_num),
                "anime": getattr(meta, "anime", None)}, path)


def load_checkpoint(path: str, max_neighbors: int = 64, device="cuda", tuning: dict | None = None):
    """Rebuild `meta` from a checkpoint and re-initialise the solver state that is not
    part of the fields (neighbour lists, boundary volumes, elastic rest neighbourhoods
    from x_0). Returns (meta, solver)."""
    from .scene import ParticleSet

    ck = torch.load(path, weights_only=False)
    f = ck["fields"]
    ps = ParticleSet(x=f["x"].numpy(), material=f["material"].numpy(), is_dynamic=f["is_dynamic"].numpy(),
                     phase_id=f["phase_id"].numpy(), mass=f["m"].numpy(), n_fluid=ck["n_fluid"])
    cfg = {**ck["config"], "Configuration": dict(ck["config"].get("Configuration", {}))}
    cfg["Configuration"].pop("animeFile", None)  # the table travels in the checkpoint
    initialize(SimConfig(config=cfg), particles=ps, quirks=ck["quirks"], max_neighbors=max_neighbors,
               device=device, tuning=tuning)
    for k in CHECKPOINT_FIELDS:
        getattr(meta.pd, k).copy_(f[k].to(meta.pd.x.device))
    solver = build_solver()
    solver.initialize()
    # initialize recomputes the static boundary volumes from the current positions; the
    # run computed them at the initial ones (an animeFile moves the boundary since)
    meta.pd.volume.copy_(f["volume"].to(meta.pd.x.device))
    meta.step_num = ck["step_num"]
    meta.anime = ck.get("anime")
    meta.config = SimConfig(config=ck["config"])
    return meta, solver
