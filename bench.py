#!/usr/bin/env python
"""Benchmark of the octree finite-volume step: leaf cell-updates/s on the 3D air-water shock-drop.

Workload: the five-equation model (multi<3>) on an 8 x 4 x 4 mm box, 64 x 32 x 32 base cells and
4 refinement levels, local time stepping on, Mach 1.5 shock into air hitting a water drop of radius
0.5 mm (synthetic initial condition). A step is one global step of the LTS scheme
(Integrator::integrate), i.e. every ACTI level substep it contains; leaf cell-updates are the
cluster sizes of the executed substeps. `value` is the plain FP64 form (the reference's arithmetic);
the mixed form (FP32 reconstruction and flux, FP64 update and EOS recovery) is reported beside it as
`chosen_over_plain`, with its error against the FP64 form per conserved component and the number of
cells whose refinement differs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

N > 1 runs one independent replica of the shock-drop step per GPU (weak scaling; the step has no
exchange in this build), and splits the batched section's independent trees among the GPUs (strong
scaling of the batch, no exchange). `--impl reference` times the reference's own CPU solver (built from its sources by
oracle/Makefile) on this box's host cores, in bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "leaf cell-updates/s at fixed L1 err vs FP64: mixed+batched+learned vs plain GPU"
UNIT = "cell-updates/s"
BYTES_PER_UPDATE = {2: 148, 3: 148}  # multi<3>: 16 E + 8 D + 12 with E = 7, D = 3
NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e datasheet figure, for context beside the measured copy bandwidth
REF_RUNNER = os.path.join(HERE, "oracle", "_ref", "dacti_ref_runner_fast")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    ap.add_argument("--base-level", type=int, default=6)
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-level", type=int, default=-1,
                    help="with --profile-substep -3: the largest substep of this ACTI level instead")
    ap.add_argument("--batch-trees", type=int, default=256, help="trees of the batched 2D Riemann workload")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--learned", action="store_true",
                    help="also run the learned-forecaster section at config 4's size (about 15 minutes)")
    ap.add_argument("--no-learned", action="store_true", help="kept for older command lines; the section is opt-in")
    ap.add_argument("--scale", action="store_true",
                    help="also run the scale workload: the shock-drop at 128 x 64 x 64 base, +5 levels (~28M leaves)")
    ap.add_argument("--scale-steps", type=int, default=1)
    ap.add_argument("--scale-only", action="store_true", help="run only the scale workload and print its section")
    ap.add_argument("--learned-only", action="store_true", help="run only the learned sections and print them")
    ap.add_argument("--batched-only", action="store_true", help="run only the batched section and print it")
    ap.add_argument("--no-pregrow", action="store_true", help="batched section: grow pools only at the capacity check")
    ap.add_argument("--batch-groups", type=int, default=0,
                    help="batched section: also time this many lockstep groups stepped concurrently (0: not)")
    ap.add_argument("--learned-shock", action="store_true",
                    help="also run the forecast-driven regrid on the shock-drop of the bench workload")
    ap.add_argument("--forms", default="fp64,mixed",
                    help="numerical forms to time; `value` is fp64 when it is among them, else the first one")
    ap.add_argument("--profile-substep", type=int, default=-1,
                    help="bracket only this substep of the first timed step of the last form with "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off); -2 brackets the whole timed "
                         "region of the last form, -3 the substep that ran the largest cluster in the last "
                         "warm-up step")
    return ap.parse_args()


def workload_config(args) -> dict:
    nb = 1 << args.base_level
    return {
        "workload": f"shock_drop_3d multi<3> {nb}x{nb // 2}x{nb // 2} base +{args.levels} levels, LTS, max_cfl 0.25, "
                    f"Mach 1.5 shock on a 0.5 mm water drop, plain FP64 form",
        "model": "multi<3> (five-equation, stiffened gas)",
        "base_grid": [nb, nb // 2, nb // 2],
        "levels": args.levels,
        "step": "one global LTS step (all ACTI level substeps)",
        "l2": "state resident in HBM and larger than L2 (no flush needed)",
        "parallelism": f"replicas x{args.gpus}",
    }


def make_case(args):
    from dacti_b200 import cases
    return cases.shock_drop(base_level=args.base_level, levels=args.levels)


def measured_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        self.out.flush()
        self.out.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_samples(case_path: str, samples: int, substeps: int, threads: int) -> dict:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([REF_RUNNER, case_path, os.path.join(tempfile.gettempdir(), "dg_ref"), "0",
                        "--sample-substeps", str(substeps), "--samples", str(samples)],
                       capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"reference runner failed: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


REF_CHUNK_SUBSTEPS = 40


def run_reference_chunks(case_path: str, chunk: int, threads: int) -> dict:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([REF_RUNNER, case_path, os.path.join(tempfile.gettempdir(), "dg_ref"), "0",
                        "--chunk-substeps", str(chunk)], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"reference runner failed: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ------------------------------------------------------------------------------------------------
def bench_reference(args, rank: int, world: int) -> None:
    """The reference's own CPU solver (oracle/_ref/dacti_ref_runner_fast, built from the reference
    sources) on all host threads, over one complete global LTS step of the workload: the step's
    substeps are timed in consecutive chunks; the first `warmup` chunks are warm-up and every later
    chunk is timed (at least `steps` of them), so the timed region covers the rest of the step with its
    real mix of fine and coarse ACTI levels."""
    if rank != 0:
        return
    from dacti_b200.casefile import write_case
    case = make_case(args)
    threads = host_threads()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "case.bin")
        write_case(case, path)
        res = run_reference_chunks(path, REF_CHUNK_SUBSTEPS, threads)
    chunks = res["chunks"]
    timed = chunks[min(args.warmup, max(len(chunks) - 1, 0)):]
    upd = sum(c["updates"] for c in timed)
    sec = sum(c["seconds"] for c in timed)
    value = upd / sec if sec > 0 else 0.0
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sec / max(len(timed), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"the first global step, {res['substeps']} LTS substeps in {len(chunks)} chunks of "
                                   f"{REF_CHUNK_SUBSTEPS}; the first {len(chunks) - len(timed)} chunks warm-up, the other "
                                   f"{len(timed)} timed ({upd:.0f} updates, {sec:.1f} s); reference Integrator "
                                   f"(oracle/_ref/dacti_ref_runner_fast, -O3 -fopenmp) on {threads} threads of "
                                   f"{cpu_model()}; ms_per_step is per chunk"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profiler_range(on: bool) -> None:
    """cudaProfilerStart/Stop, so that `ncu --profile-from-start off` captures only the chosen range."""
    import ctypes
    rt = ctypes.CDLL("libcudart.so.12")
    (rt.cudaProfilerStart if on else rt.cudaProfilerStop)()


def timed_run(case, form: str, args, stream, local_rank: int, world: int, profile: int = -1) -> dict:
    """W warm-up global steps, then K timed ones with CUDA events on the solver's stream."""
    import torch
    import torch.distributed as dist
    from dacti_b200.solver import KERNEL_KINDS, Solver

    solver = Solver(case, device=local_rank)
    solver.set_stream(stream.cuda_stream)
    solver.set_form(form)
    sizes = []
    for k in range(args.warmup):
        if k == args.warmup - 1:
            solver.integrate(lambda _s, level, at, n, dt, size: sizes.append((size, level)))
        else:
            solver.integrate()
    if profile == -3 and sizes:
        cand = [j for j in range(len(sizes)) if args.profile_level < 0 or sizes[j][1] == args.profile_level]
        profile = max(cand, key=lambda j: sizes[j][0])
        print(f"profiled substep {profile}: level {sizes[profile][1]}, {sizes[profile][0]} cells in the warm-up "
              f"step", file=sys.stderr)
    st0 = solver.stats()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    seen = [0]

    def hook(_s, level, at, n, dt, size):
        # substep k of the first timed step: start after substep k - 1, stop after substep k
        if seen[0] == profile - 1:
            profiler_range(True)
        if seen[0] == profile:
            profiler_range(False)
        seen[0] += 1

    with ClockSampler(local_rank) as clk:
        if profile == -2:
            profiler_range(True)
        if profile == 0:
            profiler_range(True)
        ev0.record(stream)
        for k in range(args.steps):
            solver.integrate(hook if (profile >= 0 and k == 0) else None)
        ev1.record(stream)
        torch.cuda.synchronize()
        if profile == -2:
            profiler_range(False)
    if world > 1:
        dist.barrier()
    st1 = solver.stats()
    # per-kernel-kind device times from CUDA events around every launch, over one more global step
    # outside the timed region (the events add host work per launch)
    solver.set_profiling(True)
    solver.integrate()
    st2 = solver.stats()
    solver.set_profiling(False)
    out = {
        "ms": ev0.elapsed_time(ev1),
        "updates": float(st1.cell_updates - st0.cell_updates),
        "launches": int(st1.n_launches - st0.n_launches),
        "kms": {k: st2.kernel_ms[i] - st1.kernel_ms[i] for i, k in enumerate(KERNEL_KINDS)},
        "kl": {k: st2.kernel_launches[i] - st1.kernel_launches[i] for i, k in enumerate(KERNEL_KINDS)},
        "kc": {k: st2.kernel_cells[i] - st1.kernel_cells[i] for i, k in enumerate(KERNEL_KINDS)},
        "clocks": clk.summary(),
        "snap": solver.active_cells(),
        "substeps": int(st1.n_substeps - st0.n_substeps),
    }
    solver.close()
    return out


def learned_run(args, local_rank: int) -> dict:
    """Regrid forecaster on 2D Navier-Stokes flow past a cylinder (cases.cylinder_ns: domain 40 x 20,
    128 x 64 base (the power-of-two grid nearest the stated 80 x 40), +5 levels, Re 200): sixteen
    training runs with inflow Mach from U(0.2, 0.4) (seeds 11-26), one held-out run (seed 41), 20 global
    steps each, horizon 8 steps. Reports the network's and persistence's scores on the held-out run, the
    training time, the prediction rate, and a 16-step forecast-driven run (forecast every 8 steps, the
    held cells never coarsened, coarsening at every step otherwise) against the plain regrid."""
    import time as _t

    from dacti_b200 import cases
    from dacti_b200.accuracy import density_rel_l1
    from dacti_b200.forecast import collect, run_with_forecast, scores, train_forecaster
    from dacti_b200.solver import Solver

    def run(seed):
        mach = float(np.random.default_rng(seed).uniform(0.2, 0.4))
        return collect(lambda: cases.cylinder_ns(mach=mach, base_level=BASE, levels=LEVELS), 20, 8)

    BASE, LEVELS = 7, 5
    train = [run(s) for s in range(11, 27)]
    test = run(41)
    t0 = _t.perf_counter()
    net, cut, loss = train_forecaster(train, n_in=15, epochs=30)
    train_s = _t.perf_counter() - t0
    net.predict(test.x[:1024])
    t0 = _t.perf_counter()
    prob = net.predict(test.x)
    pred_s = _t.perf_counter() - t0
    truth = test.y.astype(bool)
    mlp, base = scores(prob >= cut, truth), scores(test.persistence, truth)

    def cyl():
        return cases.cylinder_ns(mach=0.3, base_level=BASE, levels=LEVELS)

    plain, fc = Solver(cyl(), device=local_rank), Solver(cyl(), device=local_rank)
    t0 = _t.perf_counter()
    for _ in range(16):
        plain.integrate()
    plain_s = _t.perf_counter() - t0
    t0 = _t.perf_counter()
    res = run_with_forecast(fc, net, cut, steps=16, interval=8, coarsen_every=1)
    fc_s = _t.perf_counter() - t0
    sp = plain.stats()
    err = density_rel_l1(plain.active_cells(), fc.active_cells(), 40.0, (40.0, 20.0), 8, 1)
    plain.close(), fc.close(), net.close()
    keep = ("precision", "recall", "f1")
    return {
        "workload": "2D Navier-Stokes cylinder, 40 x 20, base 128 x 64 +5 levels, Re 200; 16 training runs, 1 held-out",
        "network": "15 -> 64 -> 64 -> 1, BF16 inference weights, FP32 master + Adam",
        "held_out": {"samples": int(truth.size), "positive_rate": float(truth.mean()), "cut": cut,
                     "forecaster": {k: mlp[k] for k in keep}, "persistence": {k: base[k] for k in keep}},
        "train_seconds": train_s, "train_samples": int(sum(r.y.size for r in train)), "last_epoch_loss": loss,
        "predict_samples_per_s": truth.size / pred_s,
        "regrid": {"steps": 16, "interval": 8, "coarsen_every": 1,
                   "plain": {"splits": sp.n_splits, "unsplits": sp.n_unsplits, "cell_updates": sp.cell_updates,
                             "seconds": plain_s},
                   "forecast": {"splits": res["splits"], "unsplits": res["unsplits"], "held": res["held"],
                                "cell_updates": res["cell_updates"], "seconds": fc_s},
                   "density_rel_l1_vs_plain": err},
    }


def learned_shock_run(args, local_rank: int) -> dict:
    """The forecast-driven regrid on the bench's shock-drop (64 x 32 x 32 base, +4 levels): a network
    trained on four smaller shock-drops (32 x 16 x 16 base, +3 levels, Mach from U(1.3, 1.7), seeds 31-34,
    12 global steps each, horizon 4) holds the cells it expects the indicator to flag within 4 steps;
    coarsening runs at every step otherwise. Against the plain regrid over 8 global steps: splits,
    unsplits, cell updates, device time, active cells at the end, density rel-L1 and the device memory
    high-water mark."""
    import torch
    from dacti_b200 import cases
    from dacti_b200.accuracy import density_rel_l1
    from dacti_b200.forecast import collect, run_with_forecast, train_forecaster
    from dacti_b200.solver import Solver

    def run(seed):
        mach = float(np.random.default_rng(seed).uniform(1.3, 1.7))
        return collect(lambda: cases.shock_drop(mach=mach, base_level=5, levels=3), 12, 4)

    train = [run(s) for s in (31, 32, 33, 34)]
    net, cut, _ = train_forecaster(train, n_in=train[0].x.shape[1], epochs=20)
    case = make_case(args)
    out = {}
    for name in ("plain", "forecast"):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        s = Solver(case, device=local_rank)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        if name == "plain":
            for _ in range(8):
                s.integrate()
            st = s.stats()
            res = {"splits": st.n_splits, "unsplits": st.n_unsplits, "cell_updates": st.cell_updates}
        else:
            res = run_with_forecast(s, net, cut, steps=8, interval=4, coarsen_every=1)
        b.record()
        torch.cuda.synchronize()
        res["device_ms"] = a.elapsed_time(b)
        res["active_cells"] = s.n_active_cells()
        res["device_gb_used_after"] = (free0 - torch.cuda.mem_get_info()[0]) / 1e9
        res["snap"] = s.active_cells()
        s.close()
        out[name] = res
    err = density_rel_l1(out["forecast"]["snap"], out["plain"]["snap"], case.params.side_length,
                         case.params.active_size, args.base_level, int(case.shape.model))
    for k in out:
        out[k].pop("snap")
    net.close()
    return {"workload": "shock_drop_3d 64x32x32 +4, 8 global steps; network trained on four 32x16x16 +3 runs",
            "plain": out["plain"], "forecast": out["forecast"], "density_rel_l1_vs_plain": err,
            "interval": 4, "coarsen_every": 1}


def batched_run(args, rank: int, local_rank: int, world: int) -> dict:
    """Batched 2D Euler quadtree Riemann problems (seeded, see cases.riemann_batch), mixed form. The
    lockstep batch (dg_batch: merged ACTI schedules, one launch per stage for all trees of a level, the
    global step planned on the host and issued with no synchronisation, device guards stopping a run
    where the live counts leave the plan) is timed around its steps, beside dg_step_many (host threads,
    one stream per tree, one synchronisation per tree and substep) and the same trees stepped one after
    another. One more step with per-stage CUDA-event timing gives the device time per stage kind. With N
    ranks the trees are split among them (dacti_b200.batch, no exchange): the batch's total work is fixed
    (strong scaling)."""
    import torch
    import torch.distributed as dist
    from dacti_b200 import cases
    from dacti_b200.batch import my_trees, tree_work
    from dacti_b200.solver import Batch, Solver, step_many

    batch = cases.riemann_batch(args.batch_trees, seed=3)
    mine = my_trees([tree_work(c) for c in batch], rank, world)

    def make():
        out = [Solver(batch[i], device=local_rank) for i in mine]
        for s in out:
            s.set_form("mixed")
        return out

    def updates(solvers):
        return float(sum(s.stats().cell_updates for s in solvers))

    # lockstep batch: W warm-up steps, K timed steps between events on the batch's stream
    solvers = make()
    b = Batch(solvers)
    b.set_pregrow(not args.no_pregrow)
    for _ in range(args.warmup):
        b.step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    u0, t0 = updates(solvers), time.perf_counter()
    breaks = 0
    for _ in range(args.steps):
        breaks += sum(b.step())
    torch.cuda.synchronize()
    l_sec, l_upd = time.perf_counter() - t0, updates(solvers) - u0
    runs = b.run_stats()
    l_tree = [s.stats().cell_updates for s in solvers]
    l_broke = [s.stats().n_global_steps < args.warmup + args.steps for s in solvers]
    # one more step with per-stage device timing: how much of the step the stage kernels fill
    b.set_profiling(True)
    b.stage_times()
    t1 = time.perf_counter()
    b.step()
    torch.cuda.synchronize()
    prof_ms = (time.perf_counter() - t1) * 1e3
    stages = {k: round(v[0], 3) for k, v in b.stage_times().items()}
    b.close()
    cells = sum(s.n_active_cells() for s in solvers)
    for s in solvers:
        s.close()

    # the trees in work-balanced groups, one lockstep batch and host thread each: merged launches within a
    # group, concurrent streams across groups
    from dacti_b200.batch import partition
    from dacti_b200.solver import step_batches
    groups = args.batch_groups
    g_sec, g_upd = 0.0, 0.0
    if groups > 1:
        solvers = make()
        parts = partition([tree_work(batch[i]) for i in mine], groups)
        gb = [Batch([solvers[k] for k in part]) for part in parts if part]
        for x in gb:
            x.set_pregrow(not args.no_pregrow)
        for _ in range(args.warmup):
            step_batches(gb)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        u0, t0 = updates(solvers), time.perf_counter()
        for _ in range(args.steps):
            step_batches(gb)
        torch.cuda.synchronize()
        g_sec, g_upd = time.perf_counter() - t0, updates(solvers) - u0
        for x in gb:
            x.close()
        for s in solvers:
            s.close()

    # host-threaded dg_step_many over fresh copies of the same trees
    threads = min(32, max(8, 2 * host_threads()))
    solvers = make()
    for _ in range(args.warmup):
        step_many(solvers, threads=threads)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    u0, t0 = updates(solvers), time.perf_counter()
    for _ in range(args.steps):
        step_many(solvers, threads=threads)
    torch.cuda.synchronize()
    m_sec, m_upd = time.perf_counter() - t0, updates(solvers) - u0
    m_tree = [s.stats().cell_updates for s in solvers]
    m_broke = [s.stats().n_global_steps < args.warmup + args.steps for s in solvers]
    # trees that never reached a NaN in either arm: their work is defined, and equal between the arms
    clean = [k for k in range(len(solvers)) if not l_broke[k] and not m_broke[k]]
    clean_mismatch = sum(1 for k in clean if l_tree[k] != m_tree[k])
    u0, t0 = updates(solvers), time.perf_counter()
    for s in solvers:
        s.integrate()
    torch.cuda.synchronize()
    s_sec, s_upd = time.perf_counter() - t0, updates(solvers) - u0
    for s in solvers:
        s.close()
    _, cells = reduce_ranks(0.0, float(cells), world)
    l_ms, l_u = reduce_ranks(l_sec * 1e3, l_upd, world)
    m_ms, m_u = reduce_ranks(m_sec * 1e3, m_upd, world)
    g_ms, g_u = reduce_ranks(g_sec * 1e3, g_upd, world)
    s_ms, s_u = reduce_ranks(s_sec * 1e3, s_upd, world)
    split = (f"; trees split across {world} ranks by estimated work (longest first to the least-loaded "
             f"rank), no exchange" if world > 1 else "")
    return {
        "workload": f"{args.batch_trees} independent 2D Euler quadtree Riemann problems, base 2^k, k ~ U{{5..8}}, "
                    f"+2..4 levels, seeded quadrant states (seed 3), LTS, mixed form{split}",
        "scaling": "strong", "trees_rank0": len(mine), "unit": UNIT, "steps": args.steps,
        "value": l_u / (l_ms * 1e-3), "ms_per_step": l_ms / args.steps,
        "timing": "host wall clock around K lockstep batch steps (dg_batch_step), synchronised before and after",
        "planned_runs": runs,
        "pregrow": not args.no_pregrow,
        "force_breaks": int(breaks),
        "profiled_step": {"wall_ms": prof_ms, "stage_ms": stages, "stage_sum_ms": round(sum(stages.values()), 3)},
        "grouped": {"value": g_u / (g_ms * 1e-3), "groups": groups, "ms_per_step": g_ms / args.steps,
                    "speedup_vs_step_many": (g_u / g_ms) / (m_u / m_ms) if m_u > 0 else None,
                    "timing": "host wall clock around K steps of every group (dacti_b200.solver.step_batches)"}
        if groups > 1 else None,
        "step_many": {"value": m_u / (m_ms * 1e-3), "threads": threads, "ms_per_step": m_ms / args.steps},
        "one_tree_at_a_time": {"value": s_u / (s_ms * 1e-3), "steps": 1},
        "speedup_vs_step_many": (l_u / l_ms) / (m_u / m_ms) if m_u > 0 else None,
        "step_time_ratio_step_many_over_lockstep": m_ms / l_ms if l_ms > 0 else None,
        "trees_that_broke": {"lockstep": int(sum(l_broke)), "step_many": int(sum(m_broke))},
        "clean_trees": {"count": len(clean), "cell_update_mismatches": int(clean_mismatch),
                        "note": "trees with no force_break in either arm; the cell updates of a tree after a NaN "
                                "are not defined, so arm totals differ by them"},
        "speedup_vs_one_at_a_time": (l_u / l_ms) / (s_u / s_ms) if s_u > 0 else None,
        "active_cells": int(cells),
    }


def host_memory_available_gb():
    """Host memory this process may still use: the smaller of MemAvailable and the cgroup limit's room,
    in GB (None when neither can be read)."""
    vals = []
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    vals.append(int(line.split()[1]) * 1024 / 1e9)
    except OSError:
        pass
    for lim, cur in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            with open(lim) as f:
                raw = f.read().strip()
            with open(cur) as f:
                used = int(f.read().strip())
            if raw != "max" and int(raw) < (1 << 60):
                vals.append((int(raw) - used) / 1e9)
            break
        except (OSError, ValueError):
            continue
    return min(vals) if vals else None


def scale_run(args, local_rank: int) -> dict:
    """The scale workload: the five-equation shock-drop of the bench at twice the base resolution per axis
    (128 x 64 x 64) and one more level (+5; finest cells 2 um), built on the device
    (scene_build.cu), uploaded without the subtrees that hold no active leaf (casefile.prune_inactive;
    results unchanged), then one warm-up and `scale_steps` timed global steps of the FP64 form with CUDA
    events. Reports cells, node slots, the device memory in use after construction and its high-water
    mark over the steps (free memory sampled after every step)."""
    import torch
    from dacti_b200 import cases
    from dacti_b200.casefile import Case, prune_inactive
    from dacti_b200.scene_gpu import build_tree_device
    from dacti_b200.solver import Solver

    # the host holds the built tree (about 150 B per node, ~100 M nodes) and its pruned copy at once;
    # run only with room for that on the host, so a short box fails this section instead of its host
    need_gb = 48.0
    avail_gb = host_memory_available_gb()
    if avail_gb is not None and avail_gb < need_gb:
        return {"workload": "shock_drop_3d multi<3> 128x64x64 base +5 levels (the scale configuration)",
                "skipped": f"host memory available {avail_gb:.0f} GB < {need_gb:.0f} GB for the host-side build"}
    torch.cuda.synchronize()
    free0, total = torch.cuda.mem_get_info()
    t0 = time.perf_counter()
    spec, prm = cases.shock_drop_spec(base_level=7, levels=5)
    tree = build_tree_device(spec)
    n_full = tree.n_nodes
    case = prune_inactive(Case(tree, prm))
    del tree
    n_kept = case.tree.n_nodes
    leaves = int(case.tree.leaf_mask().sum())
    # a pool of 3.3 x the uploaded nodes (the first steps refine the shock and the interface): growing a
    # pool holds the old and the new one at once, which at this size leaves little room to grow
    case.params = dataclasses.replace(case.params, pool_capacity=int(n_kept * 3.3) + 1024)
    t1 = time.perf_counter()
    s = Solver(case, device=local_rank)
    del case
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    free1, _ = torch.cuda.mem_get_info()
    low = free1
    error = None
    ms, u0, done = 0.0, 0, 0
    try:
        s.integrate()
        torch.cuda.synchronize()
        low = min(low, torch.cuda.mem_get_info()[0])
        u0 = s.stats().cell_updates
        for _ in range(args.scale_steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            s.integrate()
            b.record()
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
            done += 1
            low = min(low, torch.cuda.mem_get_info()[0])
    except Exception as e:  # a device allocation that did not fit: report what was reached
        error = f"{type(e).__name__}: {e}"
    st = s.stats()
    cells = s.n_active_cells() if error is None else None
    s.close()
    upd = float(st.cell_updates - u0)
    if error is not None:
        return {"workload": "shock_drop_3d multi<3> 128x64x64 base +5 levels, LTS, FP64 (the scale configuration)",
                "error": error, "nodes_built": int(n_full), "nodes_uploaded": int(n_kept),
                "initial_active_leaves": leaves, "tree_size_reached": int(st.tree_size),
                "substeps_reached": int(st.n_substeps), "device_gb_after_construction": (free0 - free1) / 1e9,
                "device_gb_total": total / 1e9}
    return {
        "workload": "shock_drop_3d multi<3> 128x64x64 base +5 levels, LTS, FP64 (the scale configuration)",
        "nodes_built": int(n_full), "nodes_uploaded": int(n_kept), "initial_active_leaves": leaves,
        "active_cells": int(cells), "tree_size": int(st.tree_size), "steps": done,
        "value": upd / (ms * 1e-3) if ms > 0 else None, "unit": UNIT, "ms_per_step": ms / max(args.scale_steps, 1),
        "build_s": t1 - t0, "construct_s": t2 - t1,
        "device_gb_after_construction": (free0 - free1) / 1e9, "device_gb_high_water": (free0 - low) / 1e9,
        "device_gb_total": total / 1e9,
        "bytes_per_active_leaf_high_water": (free0 - low) / max(cells, 1),
    }


END_TIME = 2e-6  # the shock-drop configuration runs to 2 us


def end_time_accuracy(case, form: str, level: int, t_end: float, device: int) -> dict:
    """The form's error against the FP64 form at the configuration's end time: both run from the initial
    state over the same global steps until the time reaches t_end (the reference driver's last step is
    the first at or past t_end, driver/default_driver.hpp:197-213)."""
    from dacti_b200.solver import Solver
    out = {}
    for f in ("fp64", form):
        s = Solver(case, device=device)
        s.set_form(f)
        t, n = 0.0, 0
        while t < t_end:
            gdt, fb = s.integrate()
            t += gdt
            n += 1
            if fb:
                break
        out[f] = (s.active_cells(), t, n)
        s.close()
    acc = form_accuracy(out[form][0], out["fp64"][0], case, level)
    acc["horizon"] = f"t = {out['fp64'][1]:.3e} s after {out['fp64'][2]} global steps (end time {t_end:g} s)"
    return acc


def form_accuracy(snap, ref, case, level: int) -> dict:
    """Error of one form's solution against the FP64 form's after the same steps: mixture-density and
    per-component relative L1 on the uniform grid of `level` (conservative projection), and the cells
    whose refinement differs (present in one solution only)."""
    from dacti_b200.accuracy import density_rel_l1, project_uniform
    from dacti_b200.parity import compare
    prm = case.params
    a = project_uniform(snap, prm.side_length, prm.active_size, level)
    b = project_uniform(ref, prm.side_length, prm.active_size, level)
    comp = np.abs(a - b).sum(axis=0) / np.maximum(np.abs(b).sum(axis=0), 1e-300)
    err = density_rel_l1(snap, ref, prm.side_length, prm.active_size, level, int(case.shape.model))
    rep = compare(ref, snap, prm.side_length)
    return {"density_rel_l1_vs_plain_fp64": err, "bound": 1e-4, "ok": bool(err <= 1e-4),
            "component_rel_l1": [float(x) for x in comp], "cells_only_in_plain": rep.only_ref,
            "cells_only_in_form": rep.only_gpu, "acti_level_mismatch": rep.acti_mismatch,
            "grid": f"uniform base level {level}"}


def reduce_ranks(ms: float, updates: float, world: int):
    """Max of the timed region and sum of the cell updates over all ranks."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    u = torch.tensor([updates], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def bench_gpu(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    from dacti_b200.casefile import write_case
    from dacti_b200.solver import Solver

    torch.cuda.set_device(local_rank)
    if args.scale_only:
        if rank == 0:
            print(json.dumps({"scale": scale_run(args, local_rank)}), flush=True)
        return
    if args.batched_only:
        out = batched_run(args, rank, local_rank, world)
        if rank == 0:
            print(json.dumps({"batched": out}), flush=True)
        return
    if args.learned_only:
        if rank == 0:
            out = {"learned": learned_run(args, local_rank)}
            if args.learned_shock:
                out["learned_shock"] = learned_shock_run(args, local_rank)
            print(json.dumps(out), flush=True)
        return
    stream = torch.cuda.Stream()
    case = make_case(args)
    D = case.shape.dims

    forms = args.forms.split(",")
    primary = "fp64" if "fp64" in forms else forms[0]
    runs = {}
    for k, f in enumerate(forms):
        runs[f] = timed_run(case, f, args, stream, local_rank, world,
                            profile=args.profile_substep if k == len(forms) - 1 else -1)
    plain = runs[primary]

    ms_max, total_updates = reduce_ranks(plain["ms"], plain["updates"], world)
    value = total_updates / (ms_max * 1e-3)

    # Roofline of the cell-update kernel (k_update: the conservative update from the face-flux sums and
    # received fluxes, source, EOS recovery and floors): algorithmic bytes per leaf cell-update (16 E +
    # 8 D + 12: U read and written in FP64, 2D neighbour ids, level and time) times the cells of its
    # launches, over its CUDA-event time on the solver's stream. `traffic` is the DRAM bytes per launch
    # from the committed ncu summary of the same kernel, scaled to this run's cells per launch.
    peak, peak_kind = measured_peak()
    kms, kl, kc = plain["kms"], plain["kl"], plain["kc"]
    dom = max(kms, key=lambda k: kms[k])
    b_per = BYTES_PER_UPDATE[D]
    upd_ms = kms["update"]
    launches = max(kl["update"], 1)
    achieved = (b_per * kc["update"] / launches) / (upd_ms * 1e-3 / launches) / 1e9 if upd_ms > 0 else 0.0
    traffic = None
    tpath = os.path.join(HERE, "profiles", "stage_kernels_shock_drop_3d_small.md")
    if os.path.exists(tpath):
        with open(tpath) as f:
            for line in f:
                if line.startswith("k_update_dram_bytes_per_cell"):
                    traffic = float(line.split("=")[1]) * (kc["update"] / launches)
    step_achieved = b_per * plain["updates"] / (plain["ms"] * 1e-3) / 1e9
    roofline = {
        "bound": "hbm", "kernel": "k_update (conservative cell update)", "achieved": achieved,
        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
        "bytes_per_cell_update": b_per, "launches": kl["update"], "avg_launch_us": 1e3 * upd_ms / launches,
        "frac_of_nominal": achieved / NOMINAL_HBM_GBS, "nominal_gbs": NOMINAL_HBM_GBS,
        "whole_step": {"achieved": step_achieved, "frac": step_achieved / peak},
        "kernel_share": {k: round(v / max(sum(kms.values()), 1e-9), 4) for k, v in kms.items() if v > 0},
        "dominant_kernel_kind_by_time": dom,
    }

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if primary == "fp64" else "f64 update / f32 flux", "data": "synthetic",
        "config": workload_config(args),
        "form": "plain: FP64 throughout, the reference's arithmetic" if primary == "fp64" else primary,
        "gpu_launches": plain["launches"], "roofline": roofline, "clocks": plain["clocks"],
        "cells": plain["snap"].n, "substeps_timed": plain["substeps"],
    }
    for f in forms:
        if f == primary:
            continue
        other = runs[f]
        o_ms, o_upd = reduce_ranks(other["ms"], other["updates"], world)
        acc = form_accuracy(other["snap"], plain["snap"], case, args.base_level)
        acc["horizon"] = f"after {args.warmup + args.steps + 1} global steps from the initial state (the timed run's end)"
        result["chosen_over_plain"] = {
            "form": "mixed: FP32 reconstruction + HLLC flux, FP64 update, totals and EOS recovery" if f == "mixed" else f,
            "value": o_upd / (o_ms * 1e-3), "ms_per_step": o_ms / args.steps, "gpu_launches": other["launches"],
            "ratio_to_plain": (o_upd / o_ms) / (total_updates / ms_max), "clocks": other["clocks"],
            "accuracy_at_end_time": end_time_accuracy(case, f, args.base_level, END_TIME, local_rank),
            "accuracy": acc,
        }

    # end to end through the public API: host tree -> device, K steps with the per-step scalars read
    # back, then every active cell read back to the host
    if not args.no_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = Solver(case, device=local_rank)
        s2.set_stream(stream.cuda_stream)
        s2.set_form(primary)
        e_upd0 = s2.stats().cell_updates
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(args.steps):
            s2.integrate()
            s2.stats()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        snap = s2.active_cells()
        torch.cuda.synchronize()
        e_sec = time.perf_counter() - t0
        e_split = {"construct_s": t1 - t0, "steps_s": t2 - t1, "readback_s": e_sec - (t2 - t0)}
        e_upd = float(s2.stats().cell_updates - e_upd0)
        e_ms, e_u = reduce_ranks(e_sec * 1e3, e_upd, world)
        tree = case.tree
        h2d = (tree.parent.nbytes + tree.children.nbytes + tree.level.nbytes + tree.flags.nbytes + tree.bc.nbytes +
               tree.center.nbytes + tree.p.nbytes)
        d2h = snap.n * (8 * (D + 1 + 2 * case.shape.E + 3 + case.shape.P) + 8)
        result["e2e"] = {"value": e_u / (e_ms * 1e-3), "unit": UNIT,
                         "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                         "includes": "solver construction from the host tree, K steps, read-back of all cells",
                         "breakdown": e_split}
        s2.close()

    if not args.no_batched:
        try:
            result["batched"] = batched_run(args, rank, local_rank, world)
        except Exception as e:  # reported in the line, the headline and the other sections stand
            result["batched"] = {"error": str(e)[:300]}
    if args.learned and not args.no_learned and world == 1:
        result["learned"] = learned_run(args, local_rank)
    if args.learned_shock and world == 1:
        result["learned_shock"] = learned_shock_run(args, local_rank)
    if args.scale and world == 1:
        try:
            result["scale"] = scale_run(args, local_rank)
        except Exception as e:  # reported in the line, the other sections stand
            result["scale"] = {"error": str(e)[:300]}

    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_RUNNER):
        try:
            result["cpu_baseline"] = cpu_baseline(case, write_case)
        except Exception as e:  # reported in the line, the headline and the other sections stand
            result["cpu_baseline"] = {"error": str(e)[:300]}
    if rank == 0:
        print(json.dumps(result), flush=True)


def cpu_baseline(case, write_case) -> dict:
    """The reference solver built from its sources on the host cores: the first 60 substeps of the first
    global step with every host thread, and the first 20 with one."""
    threads = host_threads()
    sub = 60
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "case.bin")
        write_case(case, path)
        res = run_reference_samples(path, 1, sub, threads)
        one = run_reference_samples(path, 1, 20, 1)["samples"][0]
    s = res["samples"][0]
    return {
        "value": s["updates"] / s["seconds"], "unit": UNIT, "cores": threads, "kind": "reference",
        "sample": f"first {sub} LTS substeps of the first global step ({s['updates']:.0f} updates), reference "
                  f"Integrator built from its sources (-O3 -fopenmp), {threads} threads of {cpu_model()}",
        "single_thread": {"value": one["updates"] / one["seconds"], "cores": 1,
                          "sample": f"first 20 LTS substeps ({one['updates']:.0f} updates), OMP_NUM_THREADS=1"},
    }


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        bench_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        bench_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
