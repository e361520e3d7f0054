"""Autotuner of the step's launch shape.

Knobs (see nn_set_tuning, nn_set_x_split): threads per block of the neighbour
passes, neighbour chains each thread keeps in flight ("unroll": how many neighbours of
a particle a thread gathers at once; 0 gives each pass its own measured depth), the cell factor f (cells of edge h / f with a
(2f+1)-cell stencil) and the x split (x cells per cell edge). The tuner times each candidate on the actual batch, from the
batch's initial state after a few untimed steps, and keeps the fastest; results are
cached per device, scene mix and particle count (rounded to a power of two).
"""
from __future__ import annotations

import itertools
import json
import os

import torch

DEFAULT_CANDIDATES = ([dict(block=b, unroll=u, cell_factor=1, x_split=x)
                       for b, u, x in itertools.product((128, 256, 512), (0, 1, 2), (1, 2))]
                      + [dict(block=b, unroll=u, cell_factor=2, x_split=1)
                         for b, u in itertools.product((128, 256, 512), (0, 1, 2))])

# a shorter list for tuning inside a served run (block x chains, cell factor 1)
QUICK_CANDIDATES = [dict(block=b, unroll=u, cell_factor=1) for b, u in itertools.product((128, 256), (0, 2))]

_cache: dict = {}


def _key(batch) -> str:
    n = max(batch.n, 1)
    bucket = 1 << (n - 1).bit_length()
    feats = sorted({(sc.param.flags(), round(sc.param.particle_radius, 6)) for sc in batch.scenes})
    return f"{torch.cuda.get_device_name()}|{bucket}|{len(batch.scenes) > 1}|{feats}"


def time_steps(batch, steps: int, warmup: int) -> float:
    """ms per step of `steps` graph replays after `warmup` (state resident)."""
    batch.step(warmup, sync=False)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    s = torch.cuda.current_stream()
    e0.record(s)
    batch.step(steps, sync=False)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def apply(batch, cfg: dict) -> None:
    batch.engine.set_tuning(cfg["block"], cfg["unroll"], cfg["cell_factor"])
    batch.engine.set_x_split(cfg.get("x_split", 0))
    batch.cell_factor = cfg["cell_factor"]


def _sync():
    torch.cuda.synchronize()


def autotune(batch, candidates=None, steps: int = 3, warmup: int = 5, cache_path: str | None = None) -> dict:
    """Try `candidates` on `batch` (re-initialised from its scenes' initial states for
    each), leave the best applied and the batch re-initialised; returns
    {"best": cfg, "ms": {cfg: ms}, "errors": {cfg: message}}. A candidate that fails
    (a launch shape that does not fit, for example) is recorded with its error; an
    error that persists on the device stops the tuning; RuntimeError when no
    candidate ran."""
    key = _key(batch)
    if cache_path and os.path.exists(cache_path) and not _cache:
        try:
            _cache.update(json.load(open(cache_path)))
        except Exception:
            pass
    if key in _cache:
        best = _cache[key]["best"]
        apply(batch, best)
        batch.set(batch.scenes)
        return _cache[key]
    scenes = list(batch.scenes)
    results, errors = {}, {}
    for cfg in candidates or DEFAULT_CANDIDATES:
        key_c = json.dumps(cfg, sort_keys=True)
        try:
            apply(batch, cfg)
            batch.set(scenes)
            results[key_c] = time_steps(batch, steps, warmup)
        except Exception as e:
            errors[key_c] = f"{type(e).__name__}: {e}"
            _sync()  # raises if the failure left the device in an error state
    if not results:
        raise RuntimeError(f"autotune: no candidate ran: {errors}")
    best = json.loads(min(results, key=results.get))
    apply(batch, best)
    batch.set(scenes)
    out = {"best": best, "ms": results, "errors": errors}
    _cache[key] = out
    if cache_path:
        try:
            json.dump(_cache, open(cache_path, "w"))
        except Exception:
            pass
    return out
