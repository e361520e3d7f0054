"""Benchmark of the B200 SPH step (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One "step" is one SPHBase.step of the workload's scene(s) (neighbour search, DFSPH
divergence and density solves, non-Newtonian implicit viscosity, elasticity,
advection). `value` times K steps with the state resident in HBM (CUDA events,
barrier + synchronize on both sides, max over ranks); `e2e` times the same steps
through the public object API with the state copied from pinned host memory before
each step and the positions read back after it (the copies run on copy streams and
overlap the neighbouring steps' compute). Inputs are synthetic (seeded numpy
generators with the shapes of the benchmark scenes). `--impl reference` times the
CPU restatement of the reference step (the reference itself is Python + Taichi, which
is not installed) on all host cores over a bounded sample of the same workload.

`--workload surface` times the surface reconstruction instead (SRTool.dual_contouring
on a 125,000-particle fluid block; one step is one reconstruction, in particles/s).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

# Algorithmic bytes per particle of the passes (each field read or written once per
# pass; neighbour gathers assumed served on chip; float4 position+volume and velocity):
ALG_BYTES = {
    "pressure_update": 16 + 16 + 4 + 4 + 16,      # pos4, vel4, kappa, flags -> vel4
    "density_adv": 16 + 16 + 4 + 4 + 4 + 4 + 4,   # pos4, vel4, dens, alpha, flags -> rho_adv, kappa
    "divergence_update": 16 + 16 + 4 + 4 + 16,
    "density_change": 16 + 16 + 4 + 4 + 4 + 4,
    # the instance the step runs with the divergence solve's first density change:
    # pos4, vel4, flags -> dens, alpha, rho_adv, kappa
    "density_factor": 16 + 16 + 4 + 4 + 4 + 4 + 4,
    "cg_matvec": 16 + 16 + 8 + 4 + 4 + 16,        # pos4, p, aux2, mass, flags -> Ap
    "nonpressure": 4 + 16 + 16 + 4 + 4 + 16 + 4 + 4 + 8,  # flags, pos4, vel4, mass, dens -> acc4, srn, mu, aux2
    "build_lists": 16 + 4 + 4,                    # pos4, flags -> count; + 4 B per list entry (added live)
    # flags, pos4, vel4, aux2, mass, dens -> x, r, z, p, matvec positions (float4 each), preconditioner 24
    "cg_setup": 4 + 16 + 16 + 8 + 4 + 4 + 5 * 16 + 24,
}
# the density change that also computes the non-pressure terms (run in the divergence
# loop's predicted last body) reads mass and density besides and writes acc4, srn, mu, aux2
ALG_BYTES["density_change_np"] = ALG_BYTES["density_change"] + 4 + 4 + 16 + 4 + 4 + 8
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch on the
# 2.4M-particle dam break, from `ncu --set full` captures of the current kernels.
# list entries of the captured k_build_lists launch (step 5 of the 2.4M scene); the line
# scales that launch's traffic to the timed launch's entries, which the bytes follow
NCU_ENTRIES_2M = 62_580_972
NCU_TRAFFIC_2M = {"build_lists": 477530368, "density_adv": 372967680,
                  "nonpressure": 431172096, "density_factor": 365270272,
                  "density_change": 366368512, "divergence_update": 376274432,
                  "pressure_update": 383854080, "cg_matvec": 433442816, "density_change_np": 430826240,
                  "cg_setup": 567003648}
# what bounds each kernel instead of DRAM, from its ncu capture on the 2.4M scene:
# the HBM fraction above is low because none is DRAM-bound
LIMITER_2M = {
    "build_lists": "instruction issue: 72 % issue active, ~160 exact f32 distance tests per particle, two per packed f32x2 instruction; DRAM 13 %",
    "density_adv": "L1 data pipe: LSU wavefronts at 78 % of peak (neighbour gathers); DRAM 19 %",
    "nonpressure": "L1 data pipe and gather latency: LSU wavefronts 62 %, 46 % warps active; DRAM 13 %",
    "density_factor": "gather latency: LSU wavefronts 64 %, issue 64 %, 53 % warps active; DRAM 15 %",
    "density_change": "L1 data pipe: LSU wavefronts 85 % of peak; DRAM 18 %",
    "divergence_update": "L1 data pipe: LSU wavefronts 65 % of peak, 64 % issue active; DRAM 20 %",
    "pressure_update": "L1 data pipe: LSU wavefronts 72 % of peak; DRAM 24 %",
    "cg_matvec": "gather latency: LSU wavefronts 66 %, issue 63 %, 46 % warps active at 64 registers; DRAM 20 %",
    "cg_setup": "L1 data pipe and gather latency: LSU wavefronts 72 %, issue 64 %, 46 % warps active; DRAM 21 %",
    "density_change_np": "gather latency with the folded force terms: LSU wavefronts 55 %, issue 68 %, "
                         "46 % warps active at 64 registers; DRAM 13 %",
}
KERNEL_IDS = {"pressure_update": 0, "density_adv": 1, "divergence_update": 2, "density_change": 3,
              "density_factor": 4, "build_lists": 5, "cg_matvec": 6, "nonpressure": 7, "density_change_np": 8,
              "cg_setup": 9}


def step_bytes(iters_v, iters_p, iters_cg, f_el, implicit):
    """Algorithmic bytes per particle-step of the whole step (frozen constants):
    324 + 88 I_div + 88 I_p + [40 + 120 I_cg] + 600 f_el."""
    b = 324 + 88 * iters_v + 88 * iters_p + 600 * f_el
    if implicit:
        b += 40 + 120 * iters_cg
    return b


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def workload_config(sc, world=1):
    """The `config` object of a bench line, the same in both arms: which workload, its
    sizes, how it is spread over the ranks and whether its inputs exceed the L2 (so
    that no flush is needed between timed steps). The working set counts 48 B of state
    and about 26 four-byte neighbour-list entries per particle."""
    n = sc.particles.n
    return {"workload": sc.name, "particles": n, "fluid": sc.particles.n_fluid,
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2" if n * (48 + 4 * 26) > 126e6 else "inputs smaller than L2; not flushed"}


def make_workload(name, seed=0):
    from nonnewton_b200 import scene as S

    if name == "roofline_2m":
        return [S.roofline_scene(seed=seed)]
    if name == "dam_break":
        return [S.dam_break(seed=seed)]
    if name == "shear_thinning_drop":
        return [S.shear_thinning_drop(seed=seed)]
    if name == "fluid_elastic":
        return [S.fluid_elastic(seed=seed)]
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            # this rank's GPU: LOCAL_RANK, through CUDA_VISIBLE_DEVICES when that is set
            local = int(os.environ.get("LOCAL_RANK", "0"))
            vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
            dev = vis[local] if local < len(vis) else str(local)
            self.p = subprocess.Popen(["nvidia-smi", "-i", dev, f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_baseline(scenes, budget_s=20.0, threads=None):
    """The oracle (FP32 restatement of the reference step) on all host cores over a
    bounded number of steps of the same scene."""
    from oracle import oracle as O

    O.build()
    threads = threads or os.cpu_count()
    O.set_threads(threads)
    sc = scenes[0]
    o = O.OracleSim(sc.particles, sc.param, "f32")
    o.initialize()
    t0 = time.perf_counter()
    steps = 0
    while True:
        o.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or steps >= 50:
            break
    n = sc.particles.n
    return {"value": n * steps / el, "unit": "particle-steps/s", "cores": O.get_threads(), "kind": "port",
            "sample": f"{steps} steps of {sc.name} ({n} particles), FP32 oracle, OpenMP {O.get_threads()} threads"}


def run_reference(args):
    """The reference arm: the oracle (FP32 restatement of the reference step, the
    reference's own Taichi code being unavailable) on all host cores, on the same
    workload. Each timed step is one full SPH step of the scene; the run stops after K
    steps or when --cpu-budget seconds of timed steps are used up, whichever comes
    first (the line states how many ran), so that it ends within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "surface":
        run_reference_surface(args)
        return
    from oracle import oracle as O

    if args.workload == "served":
        # the reference has no batching: its form of the served workload is the plain
        # per-request loop, over the requests in arrival order
        from nonnewton_b200 import scene as S

        work = S.mixed_workload(n_requests=args.requests, seed=1000, rate=args.rate, steps=args.request_steps)
        scenes, name = [sc for _, sc in work], "served_mixed"
    else:
        scenes = make_workload(args.workload)
        name = scenes[0].name
    O.build()
    O.set_threads(os.cpu_count())
    times, psteps, warm = [], 0, 0
    t_all = time.perf_counter()

    def out_of_budget():
        return len(times) >= args.steps or time.perf_counter() - t_all >= args.ref_budget

    for sc in scenes:
        o = O.OracleSim(sc.particles, sc.param, "f32")
        o.initialize()
        if warm < args.warmup:  # as many untimed steps as the GPU arm warms up
            k = args.warmup - warm if args.workload != "served" else min(args.warmup - warm, args.request_steps)
            o.step(k)
            warm += k
        for _ in range(args.request_steps if args.workload == "served" else args.steps):
            if out_of_budget():
                break
            t0 = time.perf_counter()
            o.step(1)
            times.append(time.perf_counter() - t0)
            psteps += sc.particles.n
        if out_of_budget():
            break
    v = psteps / sum(times)
    cb = {"value": v, "unit": "particle-steps/s", "cores": O.get_threads(), "kind": "port",
          "sample": f"{len(times)} timed steps ({args.steps} requested, {args.ref_budget:.0f} s budget) of {name} "
                    f"({psteps} particle-steps) after {warm} untimed; one full SPH step each, FP32 oracle, "
                    f"OpenMP {O.get_threads()} threads"}
    if args.workload == "served":
        config = {"workload": "served_mixed", "requests": args.requests, "steps_per_request": args.request_steps,
                  "arrival_rate_per_s": args.rate}
    else:
        config = workload_config(scenes[0], args.gpus)
    # `steps` is the number of steps actually timed (the budget may stop the run early)
    print(json.dumps({"impl": "reference", "metric": "particle-steps/s", "value": v, "unit": "particle-steps/s",
                      "n_gpus": args.gpus, "steps": len(times), "steps_requested": args.steps,
                      "warmup": warm, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None,
                      "dtype": "f32", "data": "synthetic (seeded numpy scene generator)",
                      "config": config, "cpu_baseline": cb,
                      "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))


def iterating_measure(args, world, rank, steps=10, presteps=600):
    """The 2.4M-particle scene at a state whose solver loops iterate: after `presteps`
    untimed steps (0.3 s of simulated time), the fluid, which starts as a lattice below
    the rest density, has settled to it under gravity and the pressure solve runs
    several bodies per step. Then `steps` steps with the state resident, timed with CUDA
    events (max over ranks), and each solver loop's cost per body from its kernels' own
    times on the same slots."""
    import torch

    from nonnewton_b200 import scene as S
    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    sc = S.roofline_scene(seed=0)
    n = sc.particles.n
    m = sph.initialize(SimConfig(config=sc.config), particles=sc.particles, quirks=sc.param.quirks)
    solver = sph.build_solver()
    solver.initialize()
    solver.run(presteps)
    solver.stats()  # the run's last status check
    eng = m.engine
    eng.step(max(args.warmup, 1), sync=False, resume=True)
    torch.cuda.synchronize()
    barrier(world)
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.step(steps, sync=False, resume=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    st = eng.stats(0)
    folded = bool(st["nonpressure_folded"])
    kms = {k: eng.time_kernel(KERNEL_IDS[k], reps=10)
           for k in ("pressure_update", "density_adv", "divergence_update", "density_change", "density_change_np",
                     "cg_matvec")}
    eng.close()
    sph.meta.pd = sph.meta.engine = sph.meta.ns = sph.meta.solver = None
    del m, solver
    torch.cuda.empty_cache()
    bodies = {"divergence": st["iterations_v"] + 1, "pressure": st["iterations"] + 1, "cg": st["cg_iterations"]}
    return {
        "workload": f"roofline_2m after {presteps} steps (settled to the rest density)",
        "particles": n, "steps": steps, "ms_per_step": ms / steps,
        "value": float(n) * steps * world / (ms / 1e3), "unit": "particle-steps/s",
        "loop_bodies_per_step": bodies, "max_neighbors_seen": st["max_neighbors_seen"],
        "avg_density_err_pct": 100.0 * st["avg_density_err"] / sc.param.density0,
        "nonpressure": "in the divergence loop's last density change" if folded else "force pass",
        "kernel_ms": kms,
        # one body of each loop: its neighbour passes (the loop checks add a few us)
        "ms_per_loop_body": {"pressure": kms["pressure_update"] + kms["density_adv"],
                             "divergence": kms["divergence_update"] + kms["density_change"],
                             "divergence_last (non-pressure terms folded in)":
                                 kms["divergence_update"] + kms["density_change_np"],
                             "cg_matvec": kms["cg_matvec"]},
    }


def served_measure(args, world, rank):
    """The mixed served workload: one seeded stream of Poisson-arriving dam-break
    requests (fluid count log-uniform in [2k, 128k], box at 50 % fill, Cross law with
    mu0 ~ U[0.1, 20], n ~ U[0.5, 1], implicit viscosity), K steps each, continuously
    batched; with N ranks, each serves its shard of the stream (serve_sharded). The
    server's pools come from the device memory budget, capped at --capacity resident
    particles; its launch shape is autotuned on the first full packing of its shard
    (untimed). The plain per-scene loop runs a seeded sample of the same requests one
    after another. Returns every figure of the served block (on every rank)."""
    import torch

    from nonnewton_b200 import scene as S
    from nonnewton_b200.autotune import QUICK_CANDIDATES
    from nonnewton_b200.serve import Request, Server, run_plain, scene_grid_cells
    from nonnewton_b200.shard import serve_sharded, shard_requests

    work = S.mixed_workload(n_requests=args.requests, seed=1000, rate=args.rate, steps=args.request_steps)
    reqs = [Request(k, sc, args.request_steps, t) for k, (t, sc) in enumerate(work)]
    mine = [reqs[k] for k in shard_requests(reqs, world)[rank]]
    srv = Server(capacity=args.capacity, max_scenes=args.max_scenes, chunk=args.chunk,
                 tune_candidates=QUICK_CANDIDATES)
    # the first full packing of this rank's stream: what the autotuner and the roofline use
    pack, n, c = [], 0, 0
    for r in mine:
        cr = scene_grid_cells(r.scene)
        if not srv.fits(n, c, r.scene.particles.n, cr) or len(pack) >= args.max_scenes:
            break
        pack.append(r.scene)
        n += r.scene.particles.n
        c += cr
    tuning = None
    if not args.no_served_autotune:
        srv.batch.set(pack)
        tuning = srv.tune()
    # warm-up: a small served run (captures the step graphs of the server context)
    warm = [Request(-1 - k, sc, max(args.warmup, 1), 0.0) for k, sc in enumerate(pack[:4])]
    srv.run(warm, realtime=False)
    torch.cuda.synchronize()
    barrier(world)
    eng = srv.batch.engine
    l0 = eng.launch_count()
    clocks_path = os.path.join(args.clocks_dir, f"clocks_served_rank{rank}.csv")
    with ClockSampler(clocks_path) as cs:
        torch.cuda.nvtx.range_push("timed_served")
        res = serve_sharded(srv, reqs, world, rank, realtime=True)
        torch.cuda.nvtx.range_pop()
    launches = eng.launch_count() - l0
    comb = res["combined"]
    # plain per-scene loop on a sample of this rank's requests, and alone-vs-mix agreement
    rng = np.random.default_rng(7 + rank)
    k_plain = min(args.plain_sample, len(mine))
    sample = [mine[k] for k in sorted(rng.choice(len(mine), size=k_plain, replace=False))]
    plain_reqs = [Request(r.rid, r.scene, r.steps, 0.0) for r in sample]
    plain = run_plain(plain_reqs)
    fin = {r.rid: r for r in res["finished"]}
    mix_err = max(float(np.abs(fin[p.rid].result_x - p.result_x).max()) for p in plain_reqs)
    plain_tp = sum_over_ranks(plain["throughput"], world)  # N independent per-scene loops
    mix_err = max_over_ranks(mix_err, world)
    max_err_pct = max_over_ranks(res["max_density_err_pct"], world)
    failed = sum_over_ranks(float(len(res["failed"])), world)
    # bytes copied per batch step on this rank: each request's initial state in (x, mass
    # and three int32 class fields), its final positions out
    h2d = sum(r.scene.particles.n * (12 + 4 + 4 * 3) for r in res["finished"])
    d2h = sum(r.scene.particles.n * 12 for r in res["finished"])
    bsteps = max(res["batch_steps"], 1)
    return {
        "srv": srv, "pack": pack, "reqs": reqs, "clocks": cs.summary(), "launches": launches,
        "block": {
            "workload": "served_mixed", "requests": args.requests, "steps_per_request": args.request_steps,
            "arrival_rate_per_s": args.rate, "ranks": world,
            "throughput_wall": comb["particle_steps"] / comb["wall_s"], "wall_s": comb["wall_s"],
            "device_throughput": comb["device_throughput"],
            "plain_throughput": plain_tp, "plain_requests": k_plain * world,
            "ratio_served_over_plain": (comb["particle_steps"] / comb["wall_s"]) / plain_tp,
            "step_ms_p50": comb["step_ms_p50"], "step_ms_p99": comb["step_ms_p99"],
            "step_latency": "CUDA-event pair around each step's graph launch, every step of every request; the "
                            "first step after a repack includes the repack",
            "request_s_p50": res["request_s_p50"], "request_s_p99": res["request_s_p99"],
            "max_avg_density_err_pct": max_err_pct, "max_error_pct": 0.1,
            "density_err_basis": "largest DFSPH average density error at the end of any step of any request",
            "failed_requests": int(failed), "alone_vs_mix_max_abs_dx": mix_err,
            "capacity_particles": srv.capacity, "hbm_budget_bytes": srv.budget,
            "chunk_steps": args.chunk, "repacks": res["repacks"], "chunks": res["chunks"],
            "tuning": tuning["best"] if tuning else None,
        },
        "h2d_bytes_per_step": int(h2d / bsteps), "d2h_bytes_per_step": int(d2h / bsteps),
        "particle_steps": comb["particle_steps"], "wall_s": comb["wall_s"], "device_s": comb["device_s"],
    }


def run_served(args, world, rank):
    """`--workload served`: the served workload's own bench line."""
    import torch

    m = served_measure(args, world, rank)
    srv, pack, blk = m["srv"], m["pack"], m["block"]
    # roofline of the dominant kernel on the first full packing
    n = sum(sc.particles.n for sc in pack)
    srv.batch.set(pack)
    srv.batch.step(2, sync=False)
    eng = srv.batch.engine
    kms = {k: eng.time_kernel(KERNEL_IDS[k], reps=10) for k in ("pressure_update", "density_adv", "build_lists",
                                                                "density_factor", "cg_matvec")}
    torch.cuda.synchronize()
    peaks, peak_kind = load_peaks()
    if rank != 0:
        return
    dom = "density_adv"
    achieved = ALG_BYTES[dom] * n / (kms[dom] / 1e3) / 1e9
    hbm = peaks["hbm_gbs"]
    line = {
        "metric": "particle-steps/s (served, continuous batching)", "value": m["particle_steps"] / m["device_s"],
        "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": blk["step_ms_p50"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded numpy scene generator, Poisson arrivals)",
        "config": {"workload": "served_mixed", "requests": args.requests, "steps_per_request": args.request_steps,
                   "arrival_rate_per_s": args.rate},
        "served": blk,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": f"{peak_kind} hbm_gbs", "alg_bytes_per_launch":
                     ALG_BYTES[dom] * n, "traffic": None, "kernel_ms": kms, "particles": n},
        "gpu_launches": m["launches"],
        "e2e": {"value": blk["throughput_wall"], "unit": "particle-steps/s",
                "h2d_bytes_per_step": m["h2d_bytes_per_step"], "d2h_bytes_per_step": m["d2h_bytes_per_step"]},
        "clocks": m["clocks"],
    }
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline is an N=1 measurement
        line["cpu_baseline"] = cpu_baseline([m["reqs"][0].scene], budget_s=args.cpu_budget)
    print(json.dumps(line))


def surface_setup(seed=0):
    """The surface workload: the fluid of the shear-thinning drop (125,000 particles at
    0.02 m) with the reference example's settings (SPH/surf_recon/example.py: voxel
    0.01 m, particle radius 0.02 m, smoothing radius 0.06 m, level 0)."""
    from nonnewton_b200 import scene as S

    sc = S.shear_thinning_drop(seed=seed)
    nf = sc.particles.n_fluid
    pos = np.ascontiguousarray(sc.particles.x[:nf], np.float32)
    p = sc.param
    return pos, [list(p.domain_start), list(p.domain_end)]


def surface_sample(pos):
    """A bounded CPU sample of the surface workload: a 12 x 12 x 12 corner of the block."""
    lo = pos.min(0)
    return pos[np.all(pos < lo + 12 * 0.02 - 1e-3, axis=1)]


def surface_params(bbox, record_normals=False):
    from nonnewton_b200 import _abi

    vs, sr_ = 0.01, 0.06
    rng = int(math.ceil(4 * sr_ / vs)) + 1
    dims = [int(math.ceil((bbox[1][k] - bbox[0][k]) / vs)) + (rng - rng // 2 + 1) + 3 for k in range(3)]
    return _abi.make_sr_params(dims, bbox[0], vs, 0.02, sr_, 0.0, record_normals=record_normals)


def run_reference_surface(args):
    """The reference arm of the surface workload: the C++ oracle of SRTool on a bounded
    sample of the same block, one reconstruction per step, within --cpu-budget seconds."""
    from oracle import surf as OS

    pos, bbox = surface_setup()
    sub = surface_sample(pos)
    prm = surface_params(bbox)
    times = []
    t_all = time.perf_counter()
    while len(times) < args.steps and time.perf_counter() - t_all < args.cpu_budget:
        t0 = time.perf_counter()
        OS.dual_contouring(prm, sub)
        times.append(time.perf_counter() - t0)
    v = len(sub) * len(times) / sum(times)
    cb = {"value": v, "unit": "particles/s", "cores": 1, "kind": "port",
          "sample": f"{len(times)} of {args.steps} requested reconstructions of {len(sub)} particles (a corner of "
                    f"the surface_drop block), single-threaded C++ oracle"}
    print(json.dumps({"impl": "reference", "metric": "particles/s (surface reconstruction)", "value": v,
                      "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "samples": len(times), "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None,
                      "dtype": "f32", "data": "synthetic (seeded numpy scene generator)",
                      "config": {"workload": "surface_drop", "particles": int(len(sub))}, "cpu_baseline": cb,
                      "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# Algorithmic bytes per grid vertex of one reconstruction: each dense per-vertex array
# written once and read once (fixed-point field 8 + 8, splat copy 4, field 4 + 4,
# smoothing output 4 + 4, crossing flags 4 + 4, index counts 4 + 4, voxel counts 4 + 4)
SR_BYTES_PER_CELL = 60
SR_LAUNCHES = 26  # kernels one SRTool.dual_contouring call launches (three 3-kernel scans included)


def run_surface(args, world, rank):
    """SRTool.dual_contouring on the surface workload; one step is one reconstruction.
    `value` = particles / s with the positions resident; `e2e` copies the positions in
    from pinned host memory and the mesh out, each step. `marching_cubes` times the same
    pipeline ending in marching cubes (outside the step count)."""
    import torch

    from nonnewton_b200.surface import SRTool

    pos, bbox = surface_setup(seed=rank)
    nf = len(pos)
    kw = dict(isolevel=0.0, smooth_radius=0.06, num_particles=nf)
    sr = SRTool(bbox, voxel_size=0.01, particle_radius=0.02, max_num_vertices=4_000_000, max_num_indices=24_000_000,
                max_num_particles=nf)
    d_pos = torch.from_numpy(pos).cuda()
    stream = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 1)):
        sr.dual_contouring(pos=d_pos, **kw)
    torch.cuda.synchronize()
    barrier(world)
    times = []
    clocks_path = os.path.join(args.clocks_dir, f"clocks_rank{rank}.csv")
    with ClockSampler(clocks_path) as cs:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sr.dual_contouring(pos=d_pos, **kw)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(sum(times), world)
    value = sum_over_ranks(float(nf) * args.steps, world) / (ms / 1e3)
    nv, ni = sr.num_vertices[None], sr.num_indices[None]
    # end to end: host positions in, mesh out
    h_pos = torch.from_numpy(pos).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        d_pos.copy_(h_pos, non_blocking=True)
        sr.dual_contouring(pos=d_pos, **kw)
        hv = sr.mesh_vertex.to("cpu", non_blocking=True)
        hi = sr.mesh_index.to("cpu", non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    del hv, hi
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    # the same pipeline ending in marching cubes (SRTool.marching_cubes), timed beside it
    for _ in range(max(args.warmup, 1)):
        sr.marching_cubes(pos=d_pos, **kw)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mc_steps = min(args.steps, 10)
    e0.record(stream)
    for _ in range(mc_steps):
        sr.marching_cubes(pos=d_pos, **kw)
    e1.record(stream)
    e1.synchronize()
    mc_ms = max_over_ranks(e0.elapsed_time(e1), world) / mc_steps
    mc_mesh = {"vertices": sr.num_vertices[None], "triangles": sr.num_indices[None] // 3}
    if rank != 0:
        return
    dims = list(sr.last_params.dims)
    cells = dims[0] * dims[1] * dims[2]
    peaks, peak_kind = load_peaks()
    ab = cells * SR_BYTES_PER_CELL + nf * (12 + 36 + 12)
    achieved = ab / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": "particles/s (surface reconstruction)", "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy scene generator)",
        "config": {"workload": "surface_drop", "particles": nf, "grid": dims, "voxel_size": 0.01,
                   "smooth_radius": 0.06, "particle_radius": 0.02, "l2": "grid larger than L2",
                   "mesh": {"vertices": nv, "triangles": ni // 3}},
        "roofline": {"bound": "hbm", "kernel": "whole call", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": ab, "traffic": None,
                     "limiter": "the anisotropic splat's instruction issue (80 % issue active, 60 % of the "
                                "call in the ncu launch list), not memory"},
        "gpu_launches": SR_LAUNCHES * args.steps,
        "marching_cubes": {"ms_per_call": mc_ms, "particles_per_s": nf / (mc_ms / 1e3), "calls": mc_steps,
                           "mesh": mc_mesh},
        "e2e": {"value": nf * args.steps / (e2e_ms / 1e3), "unit": "particles/s", "h2d_bytes_per_step": nf * 12,
                "d2h_bytes_per_step": nv * 12 + ni * 4},
        "clocks": cs.summary(),
    }
    if not args.no_cpu_baseline and world == 1:  # an N=1 measurement
        from oracle import surf as OS

        sub = surface_sample(pos)
        t0 = time.perf_counter()
        OS.dual_contouring(surface_params(bbox), sub)
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(sub) / el, "unit": "particles/s", "cores": 1, "kind": "port",
                                "sample": f"{len(sub)} particles (a corner of the same block), one reconstruction, "
                                          f"single-threaded C++ oracle"}
    print(json.dumps(line))


def run_ours(args):
    import torch

    from nonnewton_b200 import sph
    from nonnewton_b200.config import SimConfig

    world, rank, local = dist_setup(args)
    if args.workload == "surface":
        run_surface(args, world, rank)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "served":
        run_served(args, world, rank)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    scenes = make_workload(args.workload, seed=rank)
    sc = scenes[0]
    tuning, tune_ms = None, None
    if args.tuning:
        t_ = [int(t) for t in args.tuning.split(",")]
        tuning = {"block": t_[0], "unroll": t_[1], "cell_factor": t_[2], "x_split": t_[3] if len(t_) > 3 else 0}
    if args.autotune:
        from nonnewton_b200.autotune import autotune
        from nonnewton_b200.batch import Batch

        b = Batch(sc.particles.n, 1)
        b.set([sc])
        r = autotune(b, steps=3, warmup=2)
        tuning, tune_ms = r["best"], {k: round(v, 4) for k, v in r["ms"].items()}
        b.engine.close()
        del b
    m = sph.initialize(SimConfig(config=sc.config), particles=sc.particles, quirks=sc.param.quirks, tuning=tuning)
    solver = sph.build_solver()
    solver.initialize()
    n = sc.particles.n
    eng = m.engine
    stream = torch.cuda.current_stream()
    if args.presteps:
        # advance the scene first (untimed, resident, through the step graph); the
        # object API's run() grows the neighbour lists if the scene outgrows them
        solver.run(args.presteps)
    # warm-up (also captures the step graphs)
    eng_step = lambda k, sync: eng.step(k, sync=sync, host_loop=args.host_loop)
    eng_step(max(args.warmup, 1), True)
    torch.cuda.synchronize()
    barrier(world)
    l0 = eng.launch_count()
    clocks_path = os.path.join(args.clocks_dir, f"clocks_rank{rank}.csv")
    # ---- device-resident timing: K steps, state in HBM, one graph replay per step
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    it_v = it_p = it_cg = 0
    with ClockSampler(clocks_path) as cs:
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.nvtx.range_push("timed")
        e0.record(stream)
        eng_step(args.steps, False)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = eng.launch_count() - l0
    st = eng.stats(0)
    barrier(world)
    ms_max = max_over_ranks(ms, world)
    total_ps = sum_over_ranks(float(n) * args.steps, world)
    value = total_ps / (ms_max / 1e3)
    # ---- roofline of the dominant kernel: timed live on the current slots
    implicit = bool(sc.param.implicit_viscosity)
    # when the last step took its non-pressure terms from the divergence loop's last
    # density change, the force pass skipped the scene and that body ran the NP instance
    folded = bool(st["nonpressure_folded"])
    kms = {}
    for k in ("pressure_update", "density_adv", "build_lists", "density_factor", "divergence_update",
              "density_change") + (("density_change_np",) if folded else ("nonpressure",)) + \
             (("cg_setup", "cg_matvec") if implicit else ()):
        kms[k] = eng.time_kernel(KERNEL_IDS[k], reps=10)
    # launches per step of each timed kernel at the iteration counts of the last step;
    # the dominant kernel is the one with the largest time per step
    it_v, it_p = st["iterations_v"] + 1, st["iterations"] + 1
    per_step = {"build_lists": 1, "density_factor": 1, "nonpressure": 0 if folded else 1,
                "density_adv": it_p + 1, "pressure_update": it_p, "divergence_update": it_v,
                "density_change": it_v - (1 if folded else 0), "density_change_np": 1 if folded else 0,
                "cg_matvec": st["cg_iterations"], "cg_setup": 1}
    dom = max(kms, key=lambda k: kms[k] * per_step[k])
    num_nb, _ = eng.neighbors(n, 1)
    entries = int(num_nb.sum().item())
    del num_nb
    # ---- end to end through the public API: every step uploads its inputs (x, v) from
    # pinned host memory and reads its result (x) back to pinned host memory. The
    # copies run on two copy streams (host-to-device, device-to-host) through device
    # staging buffers, so step k+1's upload and step k's readback overlap the compute
    # of the steps around them; every step still moves all of its bytes over the bus.
    pd = m.pd
    h_x = torch.empty_like(pd.x, device="cpu").pin_memory()
    h_v = torch.empty_like(pd.v, device="cpu").pin_memory()
    h_out = [torch.empty_like(pd.x, device="cpu").pin_memory() for _ in range(2)]
    h_x.copy_(pd.x)
    h_v.copy_(pd.v)
    cs_in, cs_out = torch.cuda.Stream(), torch.cuda.Stream()
    st_x = [torch.empty_like(pd.x) for _ in range(2)]
    st_v = [torch.empty_like(pd.v) for _ in range(2)]
    st_o = [torch.empty_like(pd.x) for _ in range(2)]
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("up", "used", "done", "read")}
    torch.cuda.synchronize()
    barrier(world)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    cs_in.wait_stream(stream)
    cs_out.wait_stream(stream)

    def upload(k):
        b = k % 2
        with torch.cuda.stream(cs_in):
            if k >= 2:
                cs_in.wait_event(ev["used"][b])  # step k-2 has consumed this staging pair
            st_x[b].copy_(h_x, non_blocking=True)
            st_v[b].copy_(h_v, non_blocking=True)
            ev["up"][b].record(cs_in)

    upload(0)
    for k in range(args.steps):
        b = k % 2
        if k + 1 < args.steps:
            upload(k + 1)
        stream.wait_event(ev["up"][b])
        pd.x.copy_(st_x[b])
        pd.v.copy_(st_v[b])
        ev["used"][b].record(stream)
        solver.step()
        if k >= 2:
            stream.wait_event(ev["read"][b])  # the readback of step k-2 has left st_o[b]
        st_o[b].copy_(pd.x)
        ev["done"][b].record(stream)
        with torch.cuda.stream(cs_out):
            cs_out.wait_event(ev["done"][b])
            h_out[b].copy_(st_o[b], non_blocking=True)
            ev["read"][b].record(cs_out)
    stream.wait_stream(cs_out)
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1), world)
    e2e_val = total_ps / (e2e_ms / 1e3)
    peaks, peak_kind = load_peaks()
    served = iterating = None
    if args.workload == "roofline_2m" and not (args.no_served and args.no_iterating):
        del st_x, st_v, st_o, h_x, h_v, h_out
        eng.close()
        sph.meta.pd = sph.meta.engine = sph.meta.ns = sph.meta.solver = None
        del m, pd, solver
        torch.cuda.empty_cache()
        if not args.no_iterating:
            # the same scene at a state whose solver loops iterate several times per step
            iterating = iterating_measure(args, world, rank)
        if not args.no_served:
            # the headline comparison of the served form with the plain loop, on the mixed
            # workload, in the same run (every rank takes part: it has collectives)
            served = served_measure(args, world, rank)["block"]
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    ab = ALG_BYTES[dom] * n + (4 * entries if dom == "build_lists" else 0)
    achieved = ab / (kms[dom] / 1e3) / 1e9
    traffic = NCU_TRAFFIC_2M.get(dom) if sc.name == "roofline_2m" else None
    traffic_src = "ncu dram bytes of one launch, same kernel and workload" if traffic else None
    if traffic and dom == "build_lists":
        ab_capture = ALG_BYTES["build_lists"] * n + 4 * NCU_ENTRIES_2M
        traffic = traffic * ab / ab_capture
        traffic_src = (f"ncu dram bytes of one launch of the same kernel and workload at "
                       f"{NCU_ENTRIES_2M} list entries, scaled to this launch's {entries} by the algorithmic bytes")
    hbm = peaks["hbm_gbs"]
    bytes_step = step_bytes(st["iterations_v"] + 1, st["iterations"] + 1, st["cg_iterations"], 0.0, implicit)
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        # the same rate counting only dynamic particles (fluid and moving solids)
        "value_dynamic": value * float(np.count_nonzero(sc.particles.is_dynamic)) / n,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy scene generator)",
        "config": workload_config(sc, world),
        "launch": {"step_graph": "host-driven loops" if args.host_loop else "CUDA graph with while-node solver loops",
                   "tuning": tuning or {"block": 128, "unroll": 0, "cell_factor": 1, "x_split": 2},
                   "nonpressure": "in the divergence loop's last density change" if folded else "force pass"},
        "autotune_ms_per_step": tune_ms,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": ab, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "kernel_ms": kms, "launches_per_step": per_step, "list_entries": entries,
                     "limiter": LIMITER_2M.get(dom) if sc.name == "roofline_2m" else None},
        "step_alg_bytes_per_particle": bytes_step,
        "step_roofline_frac": bytes_step * total_ps / (ms_max / 1e3) / 1e9 / hbm,
        "solver": dict({k: st[k] for k in ("iterations_v", "iterations", "cg_iterations", "avg_density_err",
                                           "max_neighbors_seen", "dt", "status")},
                       # the reference's loop test: avg |rho_adv - rho0| <= maxError % of rho0 (SPH/main.py:1776-1782)
                       avg_density_err_pct=100.0 * st["avg_density_err"] / sc.param.density0,
                       max_error_pct=sc.param.max_error),
        "gpu_launches": launches,
        "e2e": {"value": e2e_val, "unit": "particle-steps/s", "h2d_bytes_per_step": int(24 * n),
                "d2h_bytes_per_step": int(12 * n),
                "copies": "pinned host <-> device staging on two copy streams, overlapped with the steps"},
        "clocks": cs.summary(),
    }
    if iterating is not None:
        line["iterating"] = iterating
    if served is not None:
        line["served"] = served
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline is an N=1 measurement
        line["cpu_baseline"] = cpu_baseline(scenes, budget_s=args.cpu_budget)
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200, help="timed steps (200 keep nvidia-smi sampling the clocks during the timed region)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="roofline_2m")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of the CPU-baseline sample")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of timed steps of the reference arm at most (it reports how many ran)")
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--request-steps", type=int, default=100, help="steps of each served request")
    ap.add_argument("--rate", type=float, default=200.0, help="Poisson arrival rate of the served workload (1/s)")
    ap.add_argument("--capacity", type=int, default=4_000_000, help="resident particles of the server")
    ap.add_argument("--max-scenes", type=int, default=256)
    ap.add_argument("--chunk", type=int, default=10, help="steps between admissions")
    ap.add_argument("--plain-sample", type=int, default=48)
    ap.add_argument("--no-served", action="store_true", help="leave the served block out of the default line")
    ap.add_argument("--no-iterating", action="store_true",
                    help="leave the iterating-state block (the scene after 600 steps) out of the default line")
    ap.add_argument("--presteps", type=int, default=0,
                    help="untimed steps before the warm-up (to reach a later state of the scene)")
    ap.add_argument("--no-served-autotune", action="store_true",
                    help="serve with the default launch shape instead of tuning it on the first packing")
    ap.add_argument("--autotune", action="store_true", help="pick block size, unroll and cell factor first")
    ap.add_argument("--tuning", default=None, help="block,unroll,cell_factor[,x_split] (e.g. 128,0,1,2; unroll 0: each pass its own depth)")
    ap.add_argument("--clocks-dir", default=tempfile.gettempdir(),
                    help="where the nvidia-smi clock samples of the timed region go (clocks_rank<r>.csv)")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the solver loops from the host instead of CUDA-graph while-nodes "
                         "(for ncu launch lists: ncu does not profile kernel nodes inside conditional nodes)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
