"""The C ABI without a GPU: libnnsph.so loads, exports every function the header
declares, and the ctypes mirror of the structs matches the C layout."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from nonnewton_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nnsph.h")


@pytest.fixture(scope="module")
def lib():
    from nonnewton_b200 import build as B

    B.build()
    return C.CDLL(B.OUT)


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(nn_\w+)\s*\(", src, flags=re.M)))


def test_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(lib):
    lib.nn_abi_version.restype = C.c_int
    assert lib.nn_abi_version() == 1


def test_struct_layout_matches_header():
    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "nnsph.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(nn_scene_params), sizeof(nn_scene_desc), sizeof(nn_state), sizeof(nn_stats));
  printf("%zu %zu %zu %zu\n", offsetof(nn_scene_params, max_iterations_v), offsetof(nn_scene_params, cfl_max_dt),
         offsetof(nn_state, rotations), offsetof(nn_stats, steps));
  printf("%zu %zu %zu\n", sizeof(nn_sr_params), offsetof(nn_sr_params, isolevel),
         offsetof(nn_sr_params, record_normals));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        open(src, "w").write(code)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = list(map(int, out[:4]))
    offs = list(map(int, out[4:8]))
    assert list(map(int, out[8:])) == [C.sizeof(_abi.nn_sr_params), _abi.nn_sr_params.isolevel.offset,
                                       _abi.nn_sr_params.record_normals.offset]
    assert sizes == [C.sizeof(_abi.nn_scene_params), C.sizeof(_abi.nn_scene_desc), C.sizeof(_abi.nn_state),
                     C.sizeof(_abi.nn_stats)]
    assert offs == [_abi.nn_scene_params.max_iterations_v.offset, _abi.nn_scene_params.cfl_max_dt.offset,
                    _abi.nn_state.rotations.offset, _abi.nn_stats.steps.offset]


def test_invalid_arguments_are_rejected_without_a_context(lib):
    """Argument checks happen before any device call."""
    lib.nn_ctx_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_void_p)]
    lib.nn_ctx_create.restype = C.c_int
    h = C.c_void_p()
    assert lib.nn_ctx_create(0, 1, 64, 0, C.byref(h)) == _abi.NN_ERR_INVALID_ARG
    assert lib.nn_ctx_create(100, 1, 5000, 0, C.byref(h)) == _abi.NN_ERR_INVALID_ARG
    lib.nn_last_error.restype = C.c_char_p
    lib.nn_last_error.argtypes = [C.c_void_p]
    assert b"invalid" in lib.nn_last_error(None)
    lib.nn_neighbors_noalloc.restype = C.c_int
    lo = (C.c_double * 3)(0, 0, 0)
    hi = (C.c_double * 3)(1, 1, 1)
    assert lib.nn_neighbors_noalloc(None, C.c_int32(10), lo, hi, C.c_double(0.04), C.c_int32(8), None, None,
                                    None) == _abi.NN_ERR_INVALID_ARG
    lib.nn_set_animation.restype = C.c_int
    d = (C.c_float * 3)(0.01, 0, 0)
    assert lib.nn_set_animation(None, C.c_int32(0), d) == _abi.NN_ERR_INVALID_ARG
    lib.nn_sr_create.argtypes = [C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    lib.nn_sr_create.restype = C.c_int
    assert lib.nn_sr_create(0, 1000, 10, 10, 0, C.byref(h)) == _abi.NN_ERR_INVALID_ARG
    assert lib.nn_sr_create(10, 0, 10, 10, 0, C.byref(h)) == _abi.NN_ERR_INVALID_ARG
    assert lib.nn_sr_create(10, 1000, 10, 10, 4, C.byref(h)) == _abi.NN_ERR_INVALID_ARG


def test_config_parses_reference_scenes():
    """The reference's scene JSON schema and defaults (SPH/main.py:594-621)."""
    from nonnewton_b200.config import Parameter, SimConfig

    cfg = SimConfig(config={"Configuration": {"particleRadius": 0.01, "simulationMethod": 4,
                                              "timeStepSize": 0.004},
                            "FluidParticles": [{"nonNewtonMethod": 2, "viscosityMethod": 13,
                                                "viscoMaxError": 0.001, "viscosityBoundary": 0.1}]})
    p = Parameter.from_config(cfg)
    assert abs(p.support_radius - 0.04) < 1e-15 and abs(p.volume0 - 0.8 * 0.02 ** 3) < 1e-18
    assert p.density0 == 1000.0 and list(p.gravity) == [0.0, -9.8, 0.0] and p.max_error == 0.05
    assert p.use_surface_tension and p.use_viscosity and not p.use_nonnewtonian
    assert p.implicit_viscosity and p.visco_max_error == 0.001 and p.visco_boundary == 0.1
    assert p.flags() & _abi.NN_F_IMPLICIT_VISCOSITY and not p.flags() & _abi.NN_F_ELASTICITY
    with pytest.raises(NotImplementedError):
        Parameter.from_config(SimConfig(config={"Configuration": {"simulationMethod": 0}}))
    with pytest.raises(NotImplementedError):  # the reference's drag hook has no model behind it
        Parameter.from_config(SimConfig(config={"Configuration": {"simulationMethod": 4, "useDragForceModel": True}}))


def test_ply_roundtrip(tmp_path):
    import numpy as np

    from nonnewton_b200.scene import export_ply_particles, read_ply_particles

    x = np.random.default_rng(0).normal(size=(100, 3)).astype(np.float32)
    f = tmp_path / "p.ply"
    export_ply_particles(x, str(f))
    assert np.array_equal(read_ply_particles(str(f)), x)


def test_scene_geometry_resolves_like_the_reference_layout(tmp_path, monkeypatch):
    """A reference scene (<root>/data/scenes/x.json) names its models as
    "./data/models/m.ply", relative to <root>, the directory of SPH/main.py; the loader
    finds them there from any working directory and loads the phases."""
    import json

    import numpy as np

    from nonnewton_b200.config import Parameter, SimConfig
    from nonnewton_b200.scene import export_ply_particles, geometry_path, load_particles

    (tmp_path / "data" / "scenes").mkdir(parents=True)
    (tmp_path / "data" / "models").mkdir(parents=True)
    g = np.arange(5) * 0.02
    cube = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    export_ply_particles(cube, str(tmp_path / "data" / "models" / "cube.ply"))
    scene = {"Configuration": {"particleRadius": 0.01, "simulationMethod": 4},
             "FluidBlocks": [],
             "FluidParticles": [{"geometryFile": "./data/models/cube.ply", "translation": [0.5, 0.5, 0.5]}],
             "SolidParticles": [{"geometryFile": "./data/models/cube.ply", "solidType": "STATIC",
                                 "translation": [0.2, 0.1, 0.2]}]}
    path = tmp_path / "data" / "scenes" / "s.json"
    path.write_text(json.dumps(scene))
    monkeypatch.chdir("/")
    import os

    assert os.path.normpath(geometry_path("./data/models/cube.ply", str(path))) == \
        str(tmp_path / "data" / "models" / "cube.ply")
    cfg = SimConfig(str(path))
    ps = load_particles(cfg, Parameter.from_config(cfg))
    assert ps.x.shape == (250, 3) and ps.n_fluid == 125
    assert np.allclose(ps.x[:125], cube + 0.5, atol=1e-6)
    with pytest.raises(FileNotFoundError):
        geometry_path("./data/models/missing.ply", str(path))


def test_transform_rotates_about_the_origin_like_trimesh():
    """transform (SPH/main.py:133-144) rotates about trimesh's center_mass of a mesh
    without faces, which is the origin, then translates."""
    import numpy as np

    from nonnewton_b200.scene import transform

    pts = np.array([[1.0, 0.0, 0.0], [0.5, 0.5, 0.2], [2.0, 1.0, -1.0]])
    out = transform(pts, {"rotationAxis": [0, 0, 2], "rotationAngle": 90, "translation": [0.1, 0.0, 0.0]})
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    assert np.allclose(out, pts @ R.T + [0.1, 0.0, 0.0], atol=1e-15)
    # the reference's test_transform.json: cube.ply's [0.26, 0.74]^3 turned 45 degrees
    # about x through the origin reaches below y = 0
    cube = np.array([[x, y, z] for x in (0.26, 0.74) for y in (0.26, 0.74) for z in (0.26, 0.74)])
    turned = transform(cube, {"rotationAxis": [1, 0, 0], "rotationAngle": 45})
    assert turned[:, 1].min() < -0.3 and np.allclose(turned[:, 0], cube[:, 0])
    assert np.array_equal(transform(cube, {}), cube)


def test_fill_tank_is_the_filled_voxelisation_of_the_box():
    """fill_tank (SPH/main.py:147-181) as trimesh's voxelized(2r).fill().points: cell
    centres at integer multiples of the pitch, from round(lo / pitch) to round(hi / pitch)
    on each axis, x slowest."""
    import numpy as np

    from nonnewton_b200.config import Parameter, SimConfig
    from nonnewton_b200.scene import fill_tank

    def param(start, end):
        conf = {"Configuration": {"domainStart": start, "domainEnd": end, "particleRadius": 0.01,
                                  "density0": 1000, "simulationMethod": 4, "timeStepSize": 0.004},
                "FluidParticles": [{}]}
        return Parameter.from_config(SimConfig(config=conf))

    p = 0.02
    pts = fill_tank(param([0, 0, 0], [1, 1, 1]), 0.3)  # padding = support radius 0.04
    i = np.rint(pts / p).astype(int)
    assert np.allclose(pts, i * p, atol=1e-12)
    assert [i[:, d].min() for d in range(3)] == [2, 2, 2] and [i[:, d].max() for d in range(3)] == [48, 15, 48]
    assert len(pts) == 47 * 14 * 47
    assert np.array_equal(i[:3], [[2, 2, 2], [2, 2, 3], [2, 2, 4]])  # z fastest
    # a domain start off the pitch: the lattice stays on multiples of the pitch
    pts = fill_tank(param([0.013, 0.0, 0.0], [1, 1, 1]), 0.3)
    assert np.isclose(pts[:, 0].min(), 0.06) and np.isclose(pts[:, 0].max(), 0.96)
    assert len(fill_tank(param([0, 0, 0], [1, 1, 1]), 0.0)) == 0


def test_animation_file_reads_as_plyfile_gives_it(tmp_path):
    """An animeFile (SPH/main.py:283-309) is a PLY whose vertices carry frame, dx, dy and
    dz; ASCII and binary files give the same table, each column with its declared type."""
    import numpy as np

    from nonnewton_b200.scene import read_animation, read_ply_vertex_data

    frames = np.array([0, 3, 3, 7], np.int32)
    disp = np.array([[0.5, 0, 0], [0, -0.25, 0], [0, 0, 0.125], [1, 2, 3]], np.float32)
    head = "ply\nformat {}\nelement vertex 4\nproperty int frame\nproperty float dx\nproperty float dy\n" \
           "property float dz\nend_header\n"
    a = tmp_path / "a.ply"
    a.write_text(head.format("ascii 1.0") + "".join(f"{f} {x} {y} {z}\n" for f, (x, y, z) in zip(frames, disp)))
    b = tmp_path / "b.ply"
    rec = np.zeros(4, np.dtype([("frame", "<i4"), ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4")]))
    rec["frame"], rec["dx"], rec["dy"], rec["dz"] = frames, disp[:, 0], disp[:, 1], disp[:, 2]
    b.write_bytes(head.format("binary_little_endian 1.0").encode() + rec.tobytes())
    for f in (a, b):
        v = read_ply_vertex_data(str(f))
        assert v["frame"].dtype == np.int32 and v["dx"].dtype == np.float32
        fr, d = read_animation(str(f))
        assert np.array_equal(fr, frames) and np.array_equal(d, disp)


def test_animation_frames_reach_the_engine(monkeypatch):
    """SPHBase.step passes each frame's displacement (the sum of the animeFile rows for
    that frame, the frame being the number of steps taken) before the step, and only on
    frames the table names; run(n) then takes its steps one by one."""
    import types

    import numpy as np

    from nonnewton_b200 import sph

    calls = []

    import torch

    class Eng:
        max_neighbors = 64

        def set_animation(self, scene, d):
            calls.append(("anim", scene, np.asarray(d, np.float32).copy()))

        def step(self, n, sync=True, host_loop=False):
            calls.append(("step", n))

        def stats(self, scene=0):
            return {"status": 0, "max_neighbors_seen": 30}

        def status_async(self, out, scene=0):
            out[0], out[1] = 0, 30

        def status_wait(self):
            pass

    cfg = types.SimpleNamespace(get_cfg=lambda k, d=None: None)
    pd = types.SimpleNamespace(x=torch.zeros(4, 3), v=torch.zeros(4, 3))
    m = types.SimpleNamespace(engine=Eng(), parm=types.SimpleNamespace(gravity=0, density0=1000, dt=1e-3),
                              ns=types.SimpleNamespace(_lists=None), config=cfg, step_num=0, pd=pd,
                              anime=(np.array([0, 2, 2, 5], np.int64),
                                     np.array([[1, 0, 0], [0, 2, 0], [0, 0.5, 3], [4, 4, 4]], np.float32)))
    monkeypatch.setattr(sph, "meta", m)
    s = sph.SPHBase()
    s.run(6)
    assert [c[0] for c in calls] == ["anim", "step", "step", "anim", "step", "step", "step", "anim", "step"]
    anims = [c for c in calls if c[0] == "anim"]
    assert np.array_equal(anims[0][2], [1, 0, 0]) and np.array_equal(anims[1][2], [0, 2.5, 3])
    assert np.array_equal(anims[2][2], [4, 4, 4]) and m.step_num == 6


def test_overflowed_step_runs_again_with_larger_lists(monkeypatch):
    """SPHBase's growth of the neighbour lists (host logic, fake engine): a step that
    reports NN_ERR_NEIGHBOR_OVERFLOW is run again after the capacity grows past the
    largest count seen (by a quarter, rounded to 8), from the x and v it started from,
    with the frame's displacement set again; a clean step is run once."""
    import types

    import numpy as np
    import torch

    from nonnewton_b200 import _abi, sph

    calls = []

    class Eng:
        max_neighbors = 64
        overflow_once = True

        def set_animation(self, scene, d):
            calls.append(("anim",))

        def step(self, n, sync=True, host_loop=False):
            calls.append(("step", n, float(pd.x[0, 0])))
            pd.x += 1.0  # the step moves the particles

        def stats(self, scene=0):
            if self.overflow_once:
                self.overflow_once = False
                return {"status": _abi.NN_ERR_NEIGHBOR_OVERFLOW, "max_neighbors_seen": 77}
            return {"status": 0, "max_neighbors_seen": 77}

        def set_neighbor_cap(self, cap):
            calls.append(("cap", cap))
            self.max_neighbors = cap

    cfg = types.SimpleNamespace(get_cfg=lambda k, d=None: None)
    pd = types.SimpleNamespace(x=torch.zeros(4, 3), v=torch.zeros(4, 3))
    m = types.SimpleNamespace(engine=Eng(), parm=types.SimpleNamespace(gravity=0, density0=1000, dt=1e-3),
                              ns=types.SimpleNamespace(_lists=None), config=cfg, step_num=0, pd=pd,
                              anime=(np.array([0], np.int64), np.array([[1, 0, 0]], np.float32)))
    monkeypatch.setattr(sph, "meta", m)
    s = sph.SPHBase()
    s.step()
    # 77 * 5 / 4 = 96.25 -> 96; the re-run starts from the same x (0.0) and re-sets the frame
    assert calls == [("anim",), ("step", 1, 0.0), ("cap", 96), ("anim",), ("step", 1, 0.0)]
    assert float(pd.x[0, 0]) == 1.0 and m.step_num == 1
    calls.clear()
    s.step()
    assert calls == [("step", 1, 1.0)]


def test_unchecked_step_is_checked_by_the_next_call(monkeypatch):
    """Far from the capacity, a step's status is copied without waiting and read when
    the next call begins: an overflow found there restores the x, v that step started
    from and runs it again (checked) before the new step (host logic, fake engine)."""
    import types

    import torch

    from nonnewton_b200 import _abi, sph

    calls = []
    reports = iter([(0, 20), (_abi.NN_ERR_NEIGHBOR_OVERFLOW, 70), (0, 20)])  # async copies of steps 2, 3, 4

    class Eng:
        max_neighbors = 64

        def set_animation(self, scene, d):
            pass

        def step(self, n, sync=True, host_loop=False):
            calls.append(("step", float(pd.x[0, 0])))
            pd.x += 1.0

        def stats(self, scene=0):
            calls.append(("stats",))
            return {"status": 0, "max_neighbors_seen": 20}

        def status_async(self, out, scene=0):
            calls.append(("async",))
            out[0], out[1] = next(reports)

        def status_wait(self):
            pass

        def set_neighbor_cap(self, cap):
            calls.append(("cap", cap))
            self.max_neighbors = cap

    cfg = types.SimpleNamespace(get_cfg=lambda k, d=None: None)
    pd = types.SimpleNamespace(x=torch.zeros(4, 3), v=torch.zeros(4, 3))
    m = types.SimpleNamespace(engine=Eng(), parm=types.SimpleNamespace(gravity=0, density0=1000, dt=1e-3),
                              ns=types.SimpleNamespace(_lists=None), config=cfg, step_num=0, pd=pd, anime=None)
    monkeypatch.setattr(sph, "meta", m)
    s = sph.SPHBase()
    s.step()  # no count known yet: checked at once
    s.step()  # 20 of 64: status copied without waiting
    s.step()  # the copy says clean; this step's copy goes out unchecked
    assert calls == [("step", 0.0), ("stats",), ("step", 1.0), ("async",), ("step", 2.0), ("async",)]
    calls.clear()
    s.step()  # the third step overflowed (70 seen): restored to x = 2 and run again first
    assert calls == [("cap", 88), ("step", 2.0), ("stats",), ("step", 3.0), ("async",)]
    assert float(pd.x[0, 0]) == 4.0 and m.step_num == 4


def test_kernel_ids_match_the_header_enum():
    """_abi's NN_K_* (the ids nn_time_kernel takes) are the header's enum nn_kernel_id,
    in order from 0."""
    import os
    import re

    from nonnewton_b200 import _abi

    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "nnsph.h")).read()
    body = re.search(r"enum nn_kernel_id \{(.*?)\};", hdr, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = [t.split("=")[0].strip() for t in body.split(",") if t.strip()]
    assert names[-1] == "NN_K_COUNT"
    assert {n: getattr(_abi, n) for n in names} == {n: k for k, n in enumerate(names)}


def test_constants_match_the_header():
    """Every NN_* constant that _abi restates (status codes, materials, phase bases, scene
    flags, viscosity laws, step flags, pass ids, allocation-free limits) has the header's
    value."""
    import os
    import re

    from nonnewton_b200 import _abi

    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "nnsph.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    vals = {}
    for name, expr in re.findall(r"^#define (NN_\w+)\s+(.+)$", hdr, re.M):
        expr = re.sub(r"(\d+)u\b", r"\1", expr.strip())
        if re.fullmatch(r"[\d\s()<+-]+", expr):
            vals[name] = eval(expr)  # integer literals and shifts only
    for body in re.findall(r"enum \w+ \{(.*?)\};", hdr, re.S):
        k = 0
        for item in (t.strip() for t in body.split(",") if t.strip()):
            name, _, v = (p.strip() for p in item.partition("="))
            k = int(v) if v else k
            vals[name] = k
            k += 1
    checked = {n: v for n, v in vals.items() if hasattr(_abi, n)}
    assert len(checked) >= 40, sorted(checked)
    assert {n: getattr(_abi, n) for n in checked} == checked
