"""Scene I/O and synthetic scenes.

- PLY read/write of `x, y, z` float vertices (the reference's `read_ply_particles`
  and `export_ply_particles`, SPH/main.py:121-124, 184-190), without plyfile.
- `transform` (SPH/main.py:133-144) and `fill_tank` (SPH/main.py:147-181) without
  trimesh, restating what the trimesh calls compute (trimesh is not installed here and
  the reference pins no version): the rotation is about the origin (trimesh's
  center_mass of the face-less mesh the reference builds from a point cloud), then the
  translation; the tank is the filled voxelisation of a box, a lattice at integer
  multiples of the pitch 2r.
- `load_particles` (SPH/main.py:628-691): phases ordered fluid -> static solid ->
  rigid solid -> elastic solid, with the reference's phase_id bases 0 / 1000 / 2000 /
  3000.
- Generators for the benchmark scenes (dam break, shear-thinning drop, fluid +
  elastic, the 2.4M-particle roofline scene, the mixed served workload), all seeded.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .config import Parameter, SimConfig

FLUID, SOLID = _abi.NN_FLUID, _abi.NN_SOLID
STATIC, RIGID, ELASTIC = 0, 1, 2


# --------------------------------------------------------------------------- PLY
_PLY_TYPES = {"float": "<f4", "float32": "<f4", "double": "<f8", "float64": "<f8", "int": "<i4", "int32": "<i4",
              "uchar": "u1", "uint8": "u1", "char": "i1", "int8": "i1", "short": "<i2", "int16": "<i2",
              "ushort": "<u2", "uint16": "<u2", "uint": "<u4", "uint32": "<u4"}


def read_ply_vertex_data(path: str) -> dict:
    """The vertex properties of an ASCII or binary little-endian PLY by name, each with its
    declared type (what plyfile's PlyData.read(path)["vertex"] gives the reference)."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.find(b"end_header")
    if end < 0:
        raise ValueError(f"{path}: not a PLY file")
    header = data[:end].decode("ascii", "replace").splitlines()
    body_start = data.find(b"\n", end) + 1
    fmt = None
    nvert = 0
    props = []
    in_vertex = False
    for line in header:
        t = line.split()
        if not t:
            continue
        if t[0] == "format":
            fmt = t[1]
        elif t[0] == "element":
            in_vertex = t[1] == "vertex"
            if in_vertex:
                nvert = int(t[2])
        elif t[0] == "property" and in_vertex:
            props.append((t[-1], t[1]))
    if fmt == "ascii":
        rows = data[body_start:].decode("ascii").split("\n")
        vals = [r.split() for r in rows if r.strip()][:nvert]
        cols = list(zip(*[r[: len(props)] for r in vals])) if vals else [[] for _ in props]
        return {n: np.array([float(v) for v in c], dtype=np.float64).astype(_PLY_TYPES[t])
                for (n, t), c in zip(props, cols)}
    if fmt == "binary_little_endian":
        dt = np.dtype([(n, _PLY_TYPES[t]) for n, t in props])
        rec = np.frombuffer(data, dtype=dt, count=nvert, offset=body_start)
        return {n: rec[n].copy() for n, _ in props}
    raise ValueError(f"{path}: unsupported PLY format {fmt}")


def read_ply_particles(path: str) -> np.ndarray:
    """Vertex positions [n,3] float32 from an ASCII or binary little-endian PLY."""
    v = read_ply_vertex_data(path)
    return np.stack([v["x"], v["y"], v["z"]], axis=1).astype(np.float32)


def read_animation(path: str):
    """An animeFile (SPH/main.py:283-309): frames [k] and displacements [k,3] float32."""
    v = read_ply_vertex_data(path)
    return v["frame"].astype(np.int64), np.stack([v["dx"], v["dy"], v["dz"]], axis=1).astype(np.float32)


def export_ply_particles(particles: np.ndarray, filename: str) -> None:
    """Binary little-endian PLY of float32 x, y, z (SPH/main.py:184-190)."""
    p = np.ascontiguousarray(np.asarray(particles, dtype=np.float32).reshape(-1, 3))
    header = ("ply\nformat binary_little_endian 1.0\n"
              f"element vertex {p.shape[0]}\nproperty float x\nproperty float y\n"
              "property float z\nend_header\n").encode("ascii")
    os.makedirs(os.path.dirname(os.path.abspath(filename)), exist_ok=True)
    with open(filename, "wb") as f:
        f.write(header)
        f.write(p.tobytes())


def transform(points: np.ndarray, cfg: dict) -> np.ndarray:
    """`transform` (SPH/main.py:133-144): rotation by rotationAngle degrees about
    rotationAxis through `trimesh.Trimesh(vertices=points).center_mass`, then the
    translation, in float64.

    The reference's mesh has vertices and no faces. trimesh's mass properties integrate
    over the triangles (the divergence-theorem integrals of its `triangles.mass_properties`),
    so the volume is 0, and for a volume below its zero tolerance trimesh returns a center
    of mass of (0, 0, 0). The rotation is therefore about the axis through the origin,
    not through the point cloud's centroid (in the reference's test_transform.json this
    swings cube.ply, [0.26, 0.74]^3, partly below y = 0)."""
    pts = np.asarray(points, dtype=np.float64)
    ang = cfg.get("rotationAngle")
    axis = cfg.get("rotationAxis")
    if ang is not None and axis is not None:
        k = np.asarray(axis, dtype=np.float64)
        k = k / np.linalg.norm(k)
        th = np.deg2rad(ang)
        K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
        R = math.cos(th) * np.eye(3) + math.sin(th) * K + (1 - math.cos(th)) * np.outer(k, k)
        pts = pts @ R.T
    t = cfg.get("translation")
    if t is not None:
        pts = pts + np.asarray(t, dtype=np.float64)
    return pts


def fill_tank(param: Parameter, height: float) -> np.ndarray:
    """`fill_tank` (SPH/main.py:147-181): `mesh.voxelized(pitch=2r).fill().points` of the
    box [domain_start + padding, (domain_end - padding) with y = height].

    trimesh's subdivide voxelisation (its default) splits the surface until every edge
    is shorter than half the pitch, rounds each vertex / pitch to the nearest integer
    (numpy's round, half to even) and keeps the hit cells; their grid starts at the
    smallest hit index i0, placed at i0 * pitch. The face coordinates stay exact under
    the splits, so a box covers the indices round(lo / pitch) .. round(hi / pitch) on
    each axis. fill() closes the interior (binary hole filling), and the points are the
    cell centres (i - i0) * pitch + i0 * pitch in C order of the grid (x slowest)."""
    p = param.particle_radius * 2
    lo = np.asarray(param.domain_start, np.float64) + param.padding
    hi = np.asarray(param.domain_end, np.float64) - param.padding
    hi = np.array([hi[0], height, hi[2]], np.float64)
    i0 = np.round(lo / p).astype(np.int64)
    i1 = np.round(hi / p).astype(np.int64)
    if np.any(i1 < i0):
        return np.zeros((0, 3), np.float64)
    axes = [np.arange(i1[d] - i0[d] + 1, dtype=np.float64) * p + float(i0[d]) * p for d in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([a.ravel() for a in g], axis=1)


# ---------------------------------------------------------------- particle sets
@dataclass
class PhaseInfo:
    """`PhaseInfo` (SPH/main.py:99-109)."""
    uid: int = 0
    parnum: int = 0
    startnum: int = 0
    material: int = FLUID
    is_dynamic: bool = False
    cfg: dict | None = None
    pos: np.ndarray | None = None
    solid_type: int = STATIC
    density0: float | None = None


@dataclass
class ParticleSet:
    """Concatenated phases in reference order, host numpy arrays."""
    x: np.ndarray
    material: np.ndarray
    is_dynamic: np.ndarray
    phase_id: np.ndarray
    mass: np.ndarray
    n_fluid: int
    phase_info: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])


def assemble(phases: list[PhaseInfo], param: Parameter, mass_density_default: float = 1000.0) -> ParticleSet:
    """`initialize_particles` (SPH/main.py:735-758). Mass is volume0 * 1000
    (SPH/main.py:743) unless the phase sets its own density0 (extension)."""
    order = sorted(phases, key=lambda ph: (0 if ph.material == FLUID else
                                           (1 if ph.solid_type == STATIC else (2 if ph.solid_type == RIGID else 3))))
    start = 0
    xs, mats, dyns, pids, masses = [], [], [], [], []
    info = {}
    n_fluid = 0
    for ph in order:
        ph.startnum = start
        ph.parnum = ph.pos.shape[0]
        start += ph.parnum
        xs.append(np.asarray(ph.pos, dtype=np.float32))
        mats.append(np.full(ph.parnum, ph.material, np.int32))
        dyns.append(np.full(ph.parnum, int(ph.is_dynamic), np.int32))
        pids.append(np.full(ph.parnum, ph.uid, np.int32))
        rho = ph.density0 if (ph.density0 is not None and not param.quirks) else mass_density_default
        masses.append(np.full(ph.parnum, param.volume0 * rho, np.float32))
        if ph.material == FLUID:
            n_fluid += ph.parnum
        info[ph.uid] = ph
    cat = lambda a, dt: np.concatenate(a).astype(dt) if a else np.zeros(0, dt)
    x = np.concatenate(xs).astype(np.float32) if xs else np.zeros((0, 3), np.float32)
    return ParticleSet(x=x, material=cat(mats, np.int32), is_dynamic=cat(dyns, np.int32),
                       phase_id=cat(pids, np.int32), mass=cat(masses, np.float32),
                       n_fluid=n_fluid, phase_info=info)


def geometry_path(geometry_file: str, scene_path: str = "", root: str | None = None) -> str:
    """Where a scene's `geometryFile` lies. The reference reads
    `sph_root_path + geometryFile` (SPH/main.py:673), the directory of main.py joined
    without a separator to paths such as "./data/models/cube.ply", which names a
    directory "SPH." that does not exist. Here the path is taken relative to `root` when
    given, else to the first of: the directory holding the scene's data/ folder (the
    reference's layout, <root>/data/scenes/x.json), the scene's parent and own
    directories, and the working directory."""
    if os.path.isabs(geometry_file):
        return geometry_file
    if root is not None:
        return os.path.join(root, geometry_file)
    cands = []
    if scene_path:
        d = os.path.dirname(os.path.abspath(scene_path))
        cands += [os.path.dirname(os.path.dirname(d)), os.path.dirname(d), d]
    cands.append(os.getcwd())
    for c in cands:
        if os.path.exists(os.path.join(c, geometry_file)):
            return os.path.join(c, geometry_file)
    raise FileNotFoundError(f"geometryFile {geometry_file!r} not found relative to any of {cands}")


def load_particles(cfg: SimConfig, param: Parameter, root: str | None = None) -> ParticleSet:
    """`load_particles` / `parse_cfg` (SPH/main.py:628-691) for PLY-backed scenes."""
    phases = []

    def _pos(c, pos=None):
        if pos is None:
            pos = read_ply_particles(geometry_path(c["geometryFile"], cfg.scene_path, root))
        return transform(pos, c)

    for cnt, c in enumerate(cfg.get_fluid_cfg()):
        phases.append(PhaseInfo(uid=c.get("id", cnt), material=FLUID, is_dynamic=True, cfg=c, pos=_pos(c),
                                density0=c.get("density0")))
    base = len(phases)
    for k, c in enumerate(cfg.get_cfg_list("FluidTanks", [])):
        phases.append(PhaseInfo(uid=c.get("id", base + k), material=FLUID, is_dynamic=True, cfg=c,
                                pos=_pos(c, fill_tank(param, c["height"]))))
    cnt_s = cnt_e = cnt_r = 0
    for c in cfg.get_solid_cfg():
        st = c.get("solidType", "STATIC")
        if st == "RIGID":
            phases.append(PhaseInfo(uid=c.get("id", cnt_r) + 2000, material=SOLID, is_dynamic=True, cfg=c,
                                    pos=_pos(c), solid_type=RIGID))
            cnt_r += 1
        elif st == "ELASTIC":
            phases.append(PhaseInfo(uid=c.get("id", cnt_e) + 3000, material=SOLID, is_dynamic=True, cfg=c,
                                    pos=_pos(c), solid_type=ELASTIC, density0=c.get("density0")))
            cnt_e += 1
        else:
            phases.append(PhaseInfo(uid=c.get("id", cnt_s) + 1000, material=SOLID, is_dynamic=False, cfg=c,
                                    pos=_pos(c), solid_type=STATIC))
            cnt_s += 1
    return assemble(phases, param)


# --------------------------------------------------------------- synthetic scenes
def box_shell(lo, hi, spacing) -> np.ndarray:
    """One layer of particles on the faces of the box [lo, hi] at the given spacing."""
    n = [int(round((hi[d] - lo[d]) / spacing)) + 1 for d in range(3)]
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), axis=-1).reshape(-1, 3)
    on = np.zeros(idx.shape[0], bool)
    for d in range(3):
        on |= (idx[:, d] == 0) | (idx[:, d] == n[d] - 1)
    idx = idx[on]
    return np.asarray(lo, np.float64) + idx * spacing


def open_tank(lo, hi, spacing) -> np.ndarray:
    """Floor and four side walls (no lid) of the box [lo, hi]."""
    n = [int(round((hi[d] - lo[d]) / spacing)) + 1 for d in range(3)]
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), axis=-1).reshape(-1, 3)
    on = (idx[:, 1] == 0) | (idx[:, 0] == 0) | (idx[:, 0] == n[0] - 1) | (idx[:, 2] == 0) | (idx[:, 2] == n[2] - 1)
    return np.asarray(lo, np.float64) + idx[on] * spacing


def block(origin, counts, spacing, jitter=0.0, rng=None) -> np.ndarray:
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in counts], indexing="ij"), axis=-1).reshape(-1, 3)
    p = np.asarray(origin, np.float64) + idx * spacing
    if jitter > 0:
        p = p + rng.uniform(-jitter, jitter, size=p.shape)
    return p


@dataclass
class Scene:
    name: str
    config: dict
    param: Parameter
    particles: ParticleSet
    steps: int


def _base_config(r, domain_start, domain_end, dt, **extra):
    c = {
        "domainStart": list(map(float, domain_start)), "domainEnd": list(map(float, domain_end)),
        "particleRadius": r, "density0": 1000.0, "simulationMethod": 4,
        "gravitation": [0.0, -9.81, 0.0], "timeStepSize": dt, "maxError": 0.1, "maxErrorV": 1.0,
        "maxIterations": 100, "maxIterationsV": 100, "viscosity": 0.01, "noGUI": True,
    }
    c.update(extra)
    return c


def _make(name, conf, phases_fn, steps, quirks=False) -> Scene:
    cfg = SimConfig(config=conf)
    param = Parameter.from_config(cfg, quirks=quirks)
    phases = phases_fn(param)
    return Scene(name=name, config=conf, param=param, particles=assemble(phases, param), steps=steps)


def dam_break(seed=0, n_side=(20, 20, 20), box=1.0, r=0.01, jitter=1e-4, quirks=False, extra_cfg=None,
              fluid_cfg=None, steps=100) -> Scene:
    """Fluid lattice at spacing 2r in the corner of a one-layer boundary box of side
    `box` placed at [h, box+h]^3 with domain [0, box+2h]^3, so that the domain clamp
    (SPH/main.py:1046-1051) coincides with the walls (the reference's pos_to_index
    ignores domainStart, SPH/main.py:805-807, so the domain starts at 0)."""
    h = 4 * r
    sp = 2 * r
    rng = np.random.default_rng(seed)
    conf = {"Configuration": _base_config(r, [0, 0, 0], [box + 2 * h] * 3, 1e-3, **(extra_cfg or {})),
            "FluidParticles": [dict(fluid_cfg or {})],
            "SolidParticles": [{"solidType": "STATIC"}]}

    def phases(param):
        fl = block([h + sp] * 3, n_side, sp, jitter, rng)
        bd = box_shell([h] * 3, [box + h] * 3, sp)
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=fl),
                PhaseInfo(uid=1000, material=SOLID, is_dynamic=False, pos=bd, solid_type=STATIC)]

    return _make("dam_break", conf, phases, steps, quirks)


def shear_thinning_drop(seed=0, n_side=50, r=0.01, quirks=False, steps=200) -> Scene:
    """50^3 fluid cube (spacing 0.02 m) with its bottom at y = 0.5 m over a 101x101
    boundary floor (2 x 2 m); Cross viscosity mu0=10, mu_inf=0.01, K=1, n=0.8 through
    the implicit viscosity CG (tolerance 1e-3); CFL capped at 2e-3 s."""
    h = 4 * r
    sp = 2 * r
    rng = np.random.default_rng(seed)
    L = 2.0
    conf = {"Configuration": _base_config(r, [0, 0, 0], [L + 2 * h, 2.0, L + 2 * h], 1e-3,
                                          useNonNewtonianModel=True, useSurfaceTensionModel=True,
                                          cflMethod=1, cflFactor=1.0, cflMaxTimeStepSize=2e-3,
                                          cflMinTimeStepSize=1e-4),
            "FluidParticles": [{"nonNewtonMethod": "CROSS_", "viscosity0": 10.0, "viscosity_inf": 0.01,
                                "consistency_index": 1.0, "power_index": 0.8, "viscosityMethod": 13,
                                "viscoMaxError": 1e-3, "viscoMaxIter": 100, "viscosityBoundary": 0.0}],
            "SolidParticles": [{"solidType": "STATIC"}]}

    def phases(param):
        side = (n_side - 1) * sp
        org = [h + L / 2 - side / 2, 0.5, h + L / 2 - side / 2]
        fl = block(org, [n_side] * 3, sp, 1e-4, rng)
        nf = int(round(L / sp)) + 1
        floor = block([h, h, h], [nf, 1, nf], sp)
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=fl),
                PhaseInfo(uid=1000, material=SOLID, is_dynamic=False, pos=floor, solid_type=STATIC)]

    return _make("shear_thinning_drop", conf, phases, steps, quirks)


def fluid_elastic(seed=0, n_el=40, r=0.01, quirks=False, steps=200) -> Scene:
    """Elastic block 40^3 (spacing 0.02 m, E=1e5, nu=0.3, rho0 1200) above a fluid pool
    filling a 1.2 x 0.6 x 1.2 m open tank of boundary particles; the fluid uses the
    Cross law of the drop scene through the implicit viscosity CG."""
    h = 4 * r
    sp = 2 * r
    rng = np.random.default_rng(seed)
    T = np.array([1.2, 0.6, 1.2])
    conf = {"Configuration": _base_config(r, [0, 0, 0], [T[0] + 2 * h, 2.2, T[2] + 2 * h], 1e-3,
                                          useNonNewtonianModel=True),
            "FluidParticles": [{"nonNewtonMethod": "CROSS_", "viscosity0": 10.0, "viscosity_inf": 0.01,
                                "consistency_index": 1.0, "power_index": 0.8, "viscosityMethod": 13,
                                "viscoMaxError": 1e-3, "viscoMaxIter": 100}],
            "SolidParticles": [{"solidType": "STATIC"},
                               {"solidType": "ELASTIC", "youngsModulus": 1e5, "poissonsRatio": 0.3,
                                "density0": 1200.0}]}

    def phases(param):
        tank = open_tank([h] * 3, [h + T[0], h + T[1], h + T[2]], sp)
        nx = int(round(T[0] / sp)) - 1
        ny = int(round(T[1] / sp)) - 1
        nz = int(round(T[2] / sp)) - 1
        fl = block([h + sp, h + sp, h + sp], [nx, ny, nz], sp, 1e-4, rng)
        side = (n_el - 1) * sp
        el = block([h + T[0] / 2 - side / 2, h + T[1] + 3 * sp, h + T[2] / 2 - side / 2], [n_el] * 3, sp)
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=fl),
                PhaseInfo(uid=1000, material=SOLID, is_dynamic=False, pos=tank, solid_type=STATIC),
                PhaseInfo(uid=3000, material=SOLID, is_dynamic=True, pos=el, solid_type=ELASTIC,
                          density0=1200.0)]

    return _make("fluid_elastic", conf, phases, steps, quirks)


def roofline_scene(seed=0, counts=(200, 100, 100), r=0.005, quirks=False, steps=50, implicit=True) -> Scene:
    """2M fluid particles (200 x 100 x 100 at 0.01 m, the long side along x) in the
    corner of a 4 x 2 x 2 m one-layer boundary box (401*201*201 - 399*199*199 =
    400,002 particles); Carreau mu0=1, mu_inf=0.001, lambda=0.5 (K = lambda^2 in the
    reference form), n=0.6; h = 0.02 m, dt = 0.5 ms. The lattice at 2r sits near
    800 kg/m^3 (volume0 = 0.8 (2r)^3), so the fluid first settles under gravity: the
    pressure solve acts after about 400 steps and then runs several bodies per step."""
    h = 4 * r
    sp = 2 * r
    rng = np.random.default_rng(seed)
    B = np.array([4.0, 2.0, 2.0])
    fcfg = {"nonNewtonMethod": "CARREAU_", "viscosity0": 1.0, "viscosity_inf": 0.001,
            "consistency_index": 0.25, "power_index": 0.6, "viscoMaxError": 1e-3, "viscoMaxIter": 100}
    if implicit:
        fcfg["viscosityMethod"] = 13
    conf = {"Configuration": _base_config(r, [0, 0, 0], list(B + 2 * h), 5e-4, useNonNewtonianModel=True),
            "FluidParticles": [fcfg], "SolidParticles": [{"solidType": "STATIC"}]}

    def phases(param):
        fl = block([h + sp] * 3, counts, sp, 1e-4 * 0.5, rng)
        bd = box_shell([h] * 3, list(h + B), sp)
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=fl),
                PhaseInfo(uid=1000, material=SOLID, is_dynamic=False, pos=bd, solid_type=STATIC)]

    return _make("roofline_2m", conf, phases, steps, quirks)


def served_request(rng: np.random.Generator, r=0.01, steps=100) -> Scene:
    """One request of the mixed workload: a dam break with fluid count log-uniform in
    [2k, 128k] in a box scaled to 50 % fill; Cross mu0 ~ U[0.1, 20], n ~ U[0.5, 1],
    mu_inf 0.01, K 1, through the implicit viscosity CG."""
    sp = 2 * r
    h = 4 * r
    nf = float(np.exp(rng.uniform(np.log(2000), np.log(128000))))
    a = max(int(round(nf ** (1 / 3))), 2)
    counts = [a, a, max(int(round(nf / (a * a))), 1)]
    fluid_vol = np.prod(counts) * sp ** 3
    side = (2.0 * fluid_vol) ** (1 / 3)
    side = max(side, (max(counts) + 2) * sp)
    side = math.ceil(side / sp) * sp
    mu0 = float(rng.uniform(0.1, 20.0))
    n_pow = float(rng.uniform(0.5, 1.0))
    seed = int(rng.integers(0, 2 ** 31 - 1))
    return dam_break(seed=seed, n_side=tuple(counts), box=side, r=r, steps=steps,
                     extra_cfg={"useNonNewtonianModel": True},
                     fluid_cfg={"nonNewtonMethod": "CROSS_", "viscosity0": mu0, "viscosity_inf": 0.01,
                                "consistency_index": 1.0, "power_index": n_pow, "viscosityMethod": 13,
                                "viscoMaxError": 1e-3, "viscoMaxIter": 100})


def mixed_workload(n_requests=512, seed=0, rate=None, steps=100):
    """Requests with Poisson arrival times (seeded). Returns [(arrival_s, Scene)]."""
    rng = np.random.default_rng(seed)
    rate = rate if rate is not None else 200.0
    t = 0.0
    out = []
    for _ in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        out.append((t, served_request(rng, steps=steps)))
    return out


def lattice_block(n_side=10, r=0.01, quirks=False) -> Scene:
    """A perfect fluid lattice at spacing 2r (26 neighbours inside, rest density ~800)."""
    h = 4 * r
    sp = 2 * r
    conf = {"Configuration": _base_config(r, [0, 0, 0], [1.0, 1.0, 1.0], 1e-3),
            "FluidParticles": [{}]}

    def phases(param):
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=block([0.3] * 3, [n_side] * 3, sp))]

    return _make("lattice", conf, phases, 1, quirks)


SCENES = {
    "dam_break": dam_break,
    "shear_thinning_drop": shear_thinning_drop,
    "fluid_elastic": fluid_elastic,
    "roofline_2m": roofline_scene,
}


def rigid_drop(seed=0, n_fluid=(10, 5, 10), n_body=(4, 4, 4), box=0.4, r=0.01, coupling=1, quirks=False,
               steps=100) -> Scene:
    """A rigid cube (RIGID phase, shape matching with two-way pressure coupling,
    SPH/main.py:1099-1158) dropped into a shallow fluid layer in a boundary box."""
    h = 4 * r
    sp = 2 * r
    rng = np.random.default_rng(seed)
    conf = {"Configuration": _base_config(r, [0, 0, 0], [box + 2 * h] * 3, 1e-3, couplingInterval=coupling),
            "FluidParticles": [{}],
            "SolidParticles": [{"solidType": "STATIC"}, {"solidType": "RIGID"}]}

    def phases(param):
        fl = block([h + sp] * 3, n_fluid, sp, 1e-4, rng)
        bd = box_shell([h] * 3, [box + h] * 3, sp)
        side = (n_body[0] - 1) * sp
        top = h + sp + n_fluid[1] * sp + 3 * sp
        rb = block([h + box / 2 - side / 2, top, h + box / 2 - side / 2], n_body, sp)
        return [PhaseInfo(uid=0, material=FLUID, is_dynamic=True, pos=fl),
                PhaseInfo(uid=1000, material=SOLID, is_dynamic=False, pos=bd, solid_type=STATIC),
                PhaseInfo(uid=2000, material=SOLID, is_dynamic=True, pos=rb, solid_type=RIGID)]

    return _make("rigid_drop", conf, phases, steps, quirks)
