"""The served loop's host logic on CPU: `Server.run` drives a stand-in batch that
records what it is asked to do (no GPU). Every request is stepped exactly its own
number of steps while resident, the batch never holds more particles or scenes than
its limits, requests are admitted in arrival order, and a scene whose status word is
set is evicted at the end of the chunk that set it, with the others unaffected."""
import numpy as np
import pytest
import torch

from nonnewton_b200 import scene as S
from nonnewton_b200 import serve as SV


class _Event:
    def __init__(self, enable_timing=False):
        self.t = None

    def record(self, stream=None):
        self.t = _Batch.clock

    def synchronize(self):
        pass

    def query(self):
        return True

    def elapsed_time(self, other):
        return float(other.t - self.t)


class _Engine:
    def __init__(self, batch):
        self.b = batch

    def stats_range(self, first, count):
        return [{"status": self.b.status.get(id(sc), 0), "avg_density_err": 0.0, "steps": self.b.done[id(sc)]}
                for sc in self.b.scenes[first:first + count]]


class _Batch:
    """Stands in for Batch: scenes in packing order; a scene's "x" rows hold the
    number of steps it has taken."""
    clock = 0

    def __init__(self, capacity, max_scenes, fail=None):
        self.capacity, self.max_scenes = capacity, max_scenes
        self.scenes, self.done, self.status = [], {}, {}
        self.resumable = False
        self.fail = fail or {}  # id(scene) -> step count at which its status word is set
        self.engine = _Engine(self)
        self.log = []

    def _check(self):
        assert sum(sc.particles.n for sc in self.scenes) <= self.capacity
        assert len(self.scenes) <= self.max_scenes

    def stage(self, scenes):
        return {"n": sum(sc.particles.n for sc in scenes), "ids": [id(sc) for sc in scenes]} if scenes else None

    def set(self, scenes, initialize=True, staged=None):
        assert staged is None or staged["ids"] == [id(sc) for sc in scenes]
        self.scenes = list(scenes)
        self.resumable = False
        for sc in scenes:
            self.done[id(sc)] = 0
        self.log.append(("set", [id(sc) for sc in scenes]))
        self._check()

    def repack(self, keep, new, staged=None):
        assert staged is None or staged["ids"] == [id(sc) for sc in new]
        assert keep == sorted(keep)
        self.scenes = [self.scenes[k] for k in keep] + list(new)
        self.resumable = False
        for sc in new:
            self.done[id(sc)] = 0
        self.log.append(("repack", [id(sc) for sc in self.scenes]))
        self._check()

    def step(self, k, sync=True, resume=False):
        assert not resume or self.resumable  # resume only what the last step left resident
        self.resumable = True
        _Batch.clock += k
        for sc in self.scenes:
            self.done[id(sc)] += k
            at = self.fail.get(id(sc))
            if at is not None and self.done[id(sc)] >= at:
                self.status[id(sc)] = -6

    def scene_view(self, k, name):
        sc = self.scenes[k]
        return torch.full((sc.particles.n, 3), float(self.done[id(sc)]))


@pytest.fixture
def fake_cuda(monkeypatch):
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    empty = torch.empty
    monkeypatch.setattr(torch, "empty", lambda *a, pin_memory=False, **k: empty(*a, **k))
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: None)


def _server(batch, chunk, **kw):
    kw.setdefault("max_cells", 1 << 40)
    return SV.Server(capacity=batch.capacity, max_scenes=batch.max_scenes, chunk=chunk, batch=batch,
                     hbm_free=1 << 62, hbm_reserve=0, **kw)


@pytest.mark.parametrize("chunk", [1, 3, 10])
def test_every_request_gets_exactly_its_steps(fake_cuda, chunk):
    rng = np.random.default_rng(chunk)
    reqs = []
    for k in range(14):
        sc = S.dam_break(seed=k, n_side=(3 + k % 3, 3, 3), box=0.2)
        reqs.append(SV.Request(k, sc, int(rng.integers(1, 12)), float(k)))
    cap = sum(r.scene.particles.n for r in reqs[:4])
    b = _Batch(cap, max_scenes=3)
    res = _server(b, chunk).run(reqs, realtime=False)
    assert res["requests"] == len(reqs) and res["failed"] == []
    fin = {r.rid: r for r in res["finished"]}
    for r in reqs:
        assert fin[r.rid].result_x.shape == (r.scene.particles.n, 3)
        assert np.all(fin[r.rid].result_x == r.steps), (r.rid, r.steps)  # stepped exactly its steps
        assert len(fin[r.rid].step_ms) == r.steps
    # admitted in arrival order: each scene's first appearance in the packing log
    first = []
    for _, ids in b.log:
        first += [i for i in ids if i not in first]
    assert first == [id(r.scene) for r in reqs]
    assert res["particle_steps"] == sum(r.scene.particles.n * r.steps for r in reqs)


def test_a_failing_scene_is_evicted_after_its_chunk(fake_cuda):
    reqs = [SV.Request(k, S.dam_break(seed=k, n_side=(3, 3, 3), box=0.2), 9, 0.0) for k in range(5)]
    b = _Batch(10 ** 9, max_scenes=5, fail={id(reqs[1].scene): 2})
    res = _server(b, chunk=3).run(reqs, realtime=False)
    fin = {r.rid: r for r in res["finished"]}
    assert res["failed"] == [1] and fin[1].failed == -6
    assert np.all(fin[1].result_x == 3)  # retired at the end of the chunk that set its status
    for k in (0, 2, 3, 4):
        assert fin[k].failed == 0 and np.all(fin[k].result_x == 9)


def test_realtime_arrivals_wait_and_all_finish(fake_cuda):
    """With realtime arrivals the loop sleeps while nothing is resident and admits
    requests only once they have arrived; every request still gets its steps."""
    reqs = [SV.Request(k, S.dam_break(seed=k, n_side=(3, 3, 3), box=0.2), 4 + k % 3, 0.004 * k) for k in range(8)]
    b = _Batch(10 ** 9, max_scenes=8)
    res = _server(b, chunk=2).run(reqs, realtime=True)
    fin = {r.rid: r for r in res["finished"]}
    assert res["requests"] == len(reqs) and res["failed"] == []
    for r in reqs:
        assert fin[r.rid].admitted >= r.arrival
        assert np.all(fin[r.rid].result_x == r.steps)


def test_staging_concatenates_the_initial_states(monkeypatch):
    """Batch.stage writes the scenes' initial states field by field, one after another,
    into buffers of the batch's capacity, and refuses more particles than that."""
    from nonnewton_b200.batch import Batch

    empty = torch.empty
    monkeypatch.setattr(torch, "empty", lambda *a, pin_memory=False, **k: empty(*a, **k))
    b = Batch.__new__(Batch)
    b.capacity, b._pin, b._pin_ev = 5000, None, None
    scs = [S.dam_break(seed=k, n_side=(3 + k, 4, 3), box=0.2 + 0.05 * k) for k in range(3)]
    st = b.stage(scs)
    ps = [sc.particles for sc in scs]
    assert st["n"] == sum(p.n for p in ps)
    assert np.array_equal(st["x"].numpy(), np.concatenate([p.x for p in ps]))
    for f, a in (("m", "mass"), ("material", "material"), ("is_dynamic", "is_dynamic"), ("phase_id", "phase_id")):
        assert np.array_equal(st[f].numpy(), np.concatenate([getattr(p, a) for p in ps])), f
    assert np.array_equal(st["volume"].numpy(), np.concatenate([np.full(p.n, sc.param.volume0, np.float32)
                                                                for sc, p in zip(scs, ps)]))
    assert np.array_equal(st["density"].numpy(), np.concatenate([np.full(p.n, sc.param.density0, np.float32)
                                                                 for sc, p in zip(scs, ps)]))
    assert b.stage([]) is None
    with pytest.raises(ValueError):
        b.stage([S.dam_break(seed=9, n_side=(20, 20, 20), box=1.0)])


def test_pools_are_sized_from_the_device_budget(fake_cuda):
    """Without a cap, the batch's particle and cell pools are the largest whose
    footprint fits the free memory minus the reserve; a cap smaller than that wins;
    a batch that does not fit the budget is refused."""
    gib = 1 << 30
    b = _Batch(10 ** 12, max_scenes=4)
    srv = SV.Server(max_scenes=4, batch=b, hbm_free=10 * gib, hbm_reserve=2 * gib)
    per = SV.footprint_bytes(1, 64) + 4 * SV.CELL_BYTES  # 4 cells per particle
    assert srv.budget == 8 * gib and srv.capacity == 8 * gib // per and srv.max_cells == 4 * srv.capacity
    assert SV.footprint_bytes(srv.capacity, 64, srv.max_cells) <= srv.budget
    assert SV.footprint_bytes(srv.capacity + 1, 64, srv.max_cells + 4) > srv.budget
    capped = SV.Server(capacity=1000, max_scenes=4, batch=b, hbm_free=10 * gib, hbm_reserve=2 * gib)
    assert capped.capacity == 1000 and capped.max_cells == 4000
    with pytest.raises(ValueError):
        SV.Server(capacity=1000, max_cells=10 ** 10, max_scenes=4, batch=b, hbm_free=10 * gib, hbm_reserve=2 * gib)
    with pytest.raises(ValueError):
        SV.Server(max_scenes=4, batch=b, hbm_free=gib, hbm_reserve=2 * gib)


def test_admission_follows_the_footprint_model(fake_cuda):
    """A budget that holds the particles of two requests and the grid cells of one
    (a small cell pool) admits them one at a time: the cell pool binds."""
    reqs = [SV.Request(k, S.dam_break(seed=k, n_side=(3, 3, 3), box=0.2), 3, 0.0) for k in range(3)]
    n = reqs[0].scene.particles.n
    cells = SV.scene_grid_cells(reqs[0].scene)
    budget = SV.footprint_bytes(2 * n, 64, cells)
    b = _Batch(2 * n, max_scenes=4)
    srv = SV.Server(capacity=2 * n, max_cells=cells, max_scenes=4, chunk=3, batch=b, hbm_free=budget,
                    hbm_reserve=0)
    res = srv.run(reqs, realtime=False)
    assert res["requests"] == 3 and all(len(ids) == 1 for _, ids in b.log)
    assert srv.fits(0, 0, n, cells) and not srv.fits(0, 1, n, cells) and not srv.fits(2 * n, 0, 1, 0)


def test_autotune_records_failures_and_needs_one_success(monkeypatch):
    """The tuner keeps every candidate's error, picks the fastest that ran, and raises
    when none ran."""
    from nonnewton_b200 import autotune as AT

    class Eng:
        def __init__(self):
            self.cfg = None

        def set_tuning(self, b, u, f):
            if b == 512:
                raise RuntimeError("candidate does not fit")
            self.cfg = (b, u, f)

        def set_x_split(self, x):
            pass

    class B:
        n, scenes, cell_factor = 100, [], 1

        def __init__(self):
            self.engine = Eng()

        def set(self, scenes):
            pass

    monkeypatch.setattr(AT, "_key", lambda batch: f"key{id(batch)}")
    monkeypatch.setattr(AT, "_sync", lambda: None)
    monkeypatch.setattr(AT, "time_steps", lambda batch, steps, warmup: {128: 3.0, 256: 2.0}[batch.engine.cfg[0]])
    cands = [dict(block=b, unroll=2, cell_factor=1) for b in (128, 256, 512)]
    b = B()
    out = AT.autotune(b, candidates=cands)
    assert out["best"]["block"] == 256 and b.engine.cfg == (256, 2, 1)
    assert len(out["errors"]) == 1 and "does not fit" in next(iter(out["errors"].values()))
    with pytest.raises(RuntimeError):
        AT.autotune(B(), candidates=[dict(block=512, unroll=2, cell_factor=1)])
