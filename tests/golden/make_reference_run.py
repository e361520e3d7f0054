"""Runs the reference's own SPH step (SPH/main.py, unmodified on disk) on small scenes
and stores its particle state after every step as golden fixtures
(tests/golden/ref_<scene>.npz). TEST INFRASTRUCTURE: it needs the reference checkout,
so it runs only where that checkout is (the fixtures it writes are committed).

Taichi is not installed here, so the reference's source is executed in plain Python
against tests/golden/refrun/ti_stub.py. A Taichi ti.func is inlined into its caller,
so an argument annotated ti.template() is passed by reference; plain Python passes
values, so the source is rewritten (ast) where the reference relies on that:
  - `ns.for_all_neighbors(p_i, task, ret)` becomes the loop it stands for, with
    `ret = task(p_i, p_j, ret)`, and every such task returns its accumulator;
  - writes through a field element (`x[i][1] = v`, `a[i].fill(0)`) and
    `ti.atomic_add(f[i], v)` go through helpers that store into the field;
  - `a = b` copies vectors (Taichi vectors are values); `all` / `any` reduce arrays.
The geometry files of the scenes are replaced by the arrays below (read_ply_particles
is swapped), and meta.config by the scene dicts. An animeFile's table is read with
this build's PLY reader and served to the reference's animate_particles. The run sets
meta.frame to the step index before each step, as the reference's GUI loop counts it.
The fixture carries the table, so its tests need no reference files.

Usage: python tests/golden/make_reference_run.py [/path/to/reference]
"""
from __future__ import annotations

import ast
import contextlib
import io
import json
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Rewrite(ast.NodeTransformer):
    def __init__(self, tasks):
        self.tasks = tasks
        self.n = 0
        self.cur_task_ret = None

    def visit_FunctionDef(self, node):
        saved = self.cur_task_ret
        self.cur_task_ret = node.args.args[-1].arg if node.name in self.tasks else None
        self.generic_visit(node)
        if self.cur_task_ret:
            node.body.append(ast.Return(value=ast.Name(self.cur_task_ret, ast.Load())))
        self.cur_task_ret = saved
        return node

    def visit_Return(self, node):
        self.generic_visit(node)
        if self.cur_task_ret and node.value is None:
            node.value = ast.Name(self.cur_task_ret, ast.Load())
        return node

    @staticmethod
    def _ti(name):
        return ast.Attribute(ast.Name("ti", ast.Load()), name, ast.Load())

    def visit_Expr(self, node):
        c = node.value
        if isinstance(c, ast.Call) and isinstance(c.func, ast.Attribute):
            if c.func.attr == "for_all_neighbors" and len(c.args) == 3 and isinstance(c.args[2], ast.Name):
                self.n += 1
                k, pj = f"_nb_k{self.n}", f"_nb_j{self.n}"
                recv, pi, task, ret = c.func.value, c.args[0], c.args[1], c.args[2]
                loop = ast.For(
                    target=ast.Name(k, ast.Store()),
                    iter=ast.Call(ast.Name("range", ast.Load()),
                                  [ast.Subscript(ast.Attribute(recv, "num_neighbors", ast.Load()), pi, ast.Load())], []),
                    body=[ast.Assign([ast.Name(pj, ast.Store())],
                                     ast.Subscript(ast.Attribute(recv, "neighbors", ast.Load()),
                                                   ast.Tuple([pi, ast.Name(k, ast.Load())], ast.Load()), ast.Load())),
                          ast.Assign([ast.Name(ret.id, ast.Store())],
                                     ast.Call(task, [pi, ast.Name(pj, ast.Load()), ast.Name(ret.id, ast.Load())], []))],
                    orelse=[])
                return self.visit(loop)
            if c.func.attr == "fill" and isinstance(c.func.value, ast.Subscript) and len(c.args) == 1:
                s = c.func.value
                return ast.Expr(ast.Call(self._ti("_fill_elem"), [self.visit(s.value), self.visit(s.slice),
                                                                  self.visit(c.args[0])], []))
        self.generic_visit(node)
        return node

    def visit_Assign(self, node):
        self.generic_visit(node)
        t = node.targets[0]
        if len(node.targets) == 1 and isinstance(t, ast.Subscript) and isinstance(t.value, ast.Subscript):
            return ast.Expr(ast.Call(self._ti("_setcomp"), [t.value.value, t.value.slice, t.slice, node.value], []))
        if isinstance(node.value, ast.Name):
            node.value = ast.Call(self._ti("_copy"), [node.value], [])
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        t = node.target
        if isinstance(t, ast.Subscript) and isinstance(t.value, ast.Subscript):
            load = ast.Subscript(ast.Subscript(t.value.value, t.value.slice, ast.Load()), t.slice, ast.Load())
            return ast.Expr(ast.Call(self._ti("_setcomp"),
                                     [t.value.value, t.value.slice, t.slice, ast.BinOp(load, node.op, node.value)], []))
        return node

    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if (isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name) and f.value.id == "ti"
                and f.attr in ("atomic_add", "atomic_max", "atomic_min") and isinstance(node.args[0], ast.Subscript)):
            s = node.args[0]
            return ast.Call(self._ti("_atomic"), [s.value, s.slice, node.args[1],
                                                  ast.Constant(f.attr.split("_")[1])], [])
        if isinstance(f, ast.Name) and f.id in ("all", "any") and len(node.args) == 1:
            return ast.Call(self._ti("_" + f.id), node.args, [])
        return node


def load_reference(ref_root: str, rel_path: str = "SPH/main.py", module: str = "sph_reference"):
    """A reference source file (SPH/main.py by default), rewritten and executed against
    the stand-in."""
    sys.path.insert(0, os.path.join(HERE, "refrun"))
    import ti_stub

    import trimesh_stub

    sys.modules["taichi"] = ti_stub
    sys.modules["trimesh"] = trimesh_stub
    for name in ("meshio", "plyfile"):  # read_ply_particles is swapped for the scenes' arrays
        sys.modules.setdefault(name, types.ModuleType(name))
    path = os.path.join(ref_root, rel_path)
    src = open(path).read()
    tree = ast.parse(src)
    tasks = set()
    for n in ast.walk(tree):
        if (isinstance(n, ast.Call) and isinstance(n.func, ast.Attribute) and n.func.attr == "for_all_neighbors"
                and len(n.args) == 3 and isinstance(n.args[1], ast.Attribute)):
            tasks.add(n.args[1].attr)
    tree = ast.fix_missing_locations(_Rewrite(tasks).visit(tree))
    mod = types.ModuleType(module)
    mod.__file__ = path
    sys.modules[module] = mod  # dataclasses look the module up
    with contextlib.redirect_stdout(io.StringIO()):
        exec(compile(tree, path, "exec"), mod.__dict__)
    return mod


FIELDS = ("x", "v", "acceleration", "density", "dfsph_factor", "density_adv", "volume")


def run_scene(ref, config: dict, geometry: dict, steps: int, anime=None) -> dict:
    """initialize(), build_solver(), solver.initialize() and `steps` solver.step() calls
    of the reference, with the state after the initialisation and after each step."""
    with tempfile.NamedTemporaryFile("w", suffix=".json", delete=False) as f:
        json.dump(config, f)
        scene = f.name
    meta = ref.meta
    for a in list(vars(meta)):
        if a != "sph_root_path":
            delattr(meta, a)
    # The reference's lists hold each particle's neighbours in the order of its cell
    # walk and, within a cell, of Taichi's atomics, which no run fixes. The non-Newtonian
    # strain rate keeps only the last neighbour's term (SPH/main.py:488-490), so it
    # depends on that order; the lists are sorted by id here, the order the oracle's
    # quirk mode reproduces (every other sum only changes by rounding).
    if not getattr(ref.NeighborhoodSearchSparse, "_sorted", False):
        search = ref.NeighborhoodSearchSparse.run_search

        def run_search(self):
            search(self)
            num, nb = self.num_neighbors.data, self.neighbors.data
            for i in range(len(num)):
                nb[i, :num[i]] = np.sort(nb[i, :num[i]])

        ref.NeighborhoodSearchSparse.run_search = run_search
        ref.NeighborhoodSearchSparse._sorted = True
    with contextlib.redirect_stdout(io.StringIO()):
        meta.config = ref.SimConfig(scene)
        ref.read_ply_particles = lambda p: geometry[os.path.basename(p)]
        if anime is not None:  # the animeFile's columns, as plyfile gives them
            ref.read_ply_particles_with_user_data = lambda p: {
                "frame": anime[0], "dx": anime[1][:, 0], "dy": anime[1][:, 1], "dz": anime[1][:, 2]}
        ref.initialize()
        solver = ref.build_solver()
        solver.initialize()
        meta.step_num = 0
        out = {f"init_{k}": getattr(meta.pd, k).to_numpy() for k in FIELDS}
        for s in range(steps):
            meta.frame = s  # the GUI loop's frame counter, which animate_particles reads
            solver.step()
            meta.step_num += 1
            for k in FIELDS:
                out[f"step{s}_{k}"] = getattr(meta.pd, k).to_numpy()
            out[f"step{s}_num_neighbors"] = meta.ns.num_neighbors.to_numpy()
            if meta.elastic_bodies:  # every body runs over all particles (quirk); the last one's state
                out[f"step{s}_stress"] = meta.elastic_bodies[-1].m_stress.to_numpy()
                out[f"step{s}_rotations"] = meta.elastic_bodies[-1].m_rotations.to_numpy().reshape(-1, 9)
            nn = getattr(solver, "nonNewtonianModel", None)
            if nn is not None:  # a 3-vector field holding the norm in every component
                out[f"step{s}_strain_rate_norm"] = nn.strainRateNorm.to_numpy()[:, 0]
                out[f"step{s}_nonnewton_viscosity"] = nn.nonNewtonViscosity.to_numpy()
    os.unlink(scene)
    out["material"] = meta.pd.material.to_numpy()
    out["is_dynamic"] = meta.pd.is_dynamic.to_numpy()
    out["phase_id"] = meta.pd.phase_id.to_numpy()
    out["config"] = np.frombuffer(json.dumps(config).encode(), np.uint8)
    if anime is not None:
        out["anime_frames"], out["anime_disp"] = anime
    return out


def _lattice(n, spacing, corner):
    g = [np.arange(k) * spacing for k in n]
    p = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3) + np.asarray(corner)
    return p.astype(np.float32)


def _shell(lo, hi, spacing):
    n = np.round((np.asarray(hi) - np.asarray(lo)) / spacing).astype(int) + 1
    p = _lattice(n, spacing, lo)
    on = np.zeros(len(p), bool)
    for a in range(3):
        on |= np.isclose(p[:, a], lo[a]) | np.isclose(p[:, a], hi[a])
    return p[on]


def scenes():
    """Small scenes of the reference's own kinds: a fluid block in a one-layer boundary
    box (surface tension and the explicit viscosity on, as the reference defaults them),
    with the non-Newtonian model on in the second."""
    r, h = 0.01, 0.04
    fluid = _lattice((6, 7, 6), 2 * r, (h + 2 * r, h + 2 * r, h + 2 * r))
    box = _shell((h, h, h), (h + 0.24, h + 0.24, h + 0.24), 2 * r)
    base = {"domainStart": [0.0, 0.0, 0.0], "domainEnd": [0.24 + 2 * h] * 3, "particleRadius": r,
            "density0": 1000, "simulationMethod": 4, "gravitation": [0.0, -9.81, 0.0],
            "timeStepSize": 0.002, "maxError": 0.1, "maxErrorV": 0.1, "viscosity": 0.01}
    geo = {"fluid.ply": fluid, "box.ply": box}
    dam = {"Configuration": dict(base),
           "FluidParticles": [{"geometryFile": "./fluid.ply"}],
           "SolidParticles": [{"geometryFile": "./box.ply", "solidType": "STATIC"}]}
    nn = {"Configuration": dict(base, useNonNewtonianModel=True),
          "FluidParticles": [{"geometryFile": "./fluid.ply", "nonNewtonMethod": 2}],
          "SolidParticles": [{"geometryFile": "./box.ply", "solidType": "STATIC"}]}
    small = _lattice((4, 4, 4), 2 * r, (h + 0.16, h + 2 * r, h + 0.16))
    geo2 = dict(geo, **{"small.ply": small})
    el = {"Configuration": dict(base),
          "FluidParticles": [{"geometryFile": "./fluid.ply"}],
          "SolidParticles": [{"geometryFile": "./box.ply", "solidType": "STATIC"},
                             {"geometryFile": "./small.ply", "solidType": "ELASTIC"}]}
    rb = {"Configuration": dict(base),
          "FluidParticles": [{"geometryFile": "./fluid.ply"}],
          "SolidParticles": [{"geometryFile": "./box.ply", "solidType": "STATIC"},
                             {"geometryFile": "./small.ply", "solidType": "RIGID"}]}
    return {"dam": (dam, geo, 6), "nonnewton": (nn, geo, 4), "elastic": (el, geo2, 3), "rigid": (rb, geo2, 4)}


def reference_scene_files(ref_root: str):
    """Scenes of the reference's own data/scenes folder, with their models read from its
    data/models folder: the elastic fixture test_deformable.json (343 particles), the
    neighbour-search fixture test_neighbor.json (9 particles) and test_anime.json (one
    particle moved by the animeFile test_anime.ply)."""
    sys.path.insert(0, os.path.dirname(HERE))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from nonnewton_b200.scene import read_animation, read_ply_particles

    out = {}
    for name, scene, steps in (("deformable", "test_deformable.json", 5), ("neighbor9", "test_neighbor.json", 5),
                               ("anime", "test_anime.json", 8)):
        cfg = json.load(open(os.path.join(ref_root, "SPH", "data", "scenes", scene)))
        geo = {}
        for c in cfg.get("FluidParticles", []) + cfg.get("SolidParticles", []):
            f = os.path.basename(c["geometryFile"])
            geo[f] = read_ply_particles(os.path.join(ref_root, "SPH", "data", "models", f))
        af = cfg["Configuration"].get("animeFile")
        anime = read_animation(os.path.join(ref_root, "SPH", "data", "models", os.path.basename(af))) if af else None
        out[name] = (cfg, geo, steps, anime)
    return out


def main(ref_root: str):
    ref = load_reference(ref_root)
    runs = {k: v + (None,) for k, v in scenes().items()}
    runs.update(reference_scene_files(ref_root))
    for name, (cfg, geo, steps, anime) in runs.items():
        out = run_scene(ref, cfg, geo, steps, anime)
        path = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: {len(out['material'])} particles, {steps} steps")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
    main(sys.argv[1])
