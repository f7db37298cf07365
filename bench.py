#!/usr/bin/env python
"""Benchmark: adaptive Dormand-Prince steps of the 512x512x8 multilayer
(exchange + interfacial DMI + uniaxial anisotropy + Zeeman + PBC demag) on
B200, reported as cell-updates/s (cells x accepted steps / s).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank advances its own replica of the workload on
its own GPU (independent solves: no collective on the data path); the timed
region is bracketed by barriers and the reported time is the max over ranks.
`--impl reference` times the CPU FP64 restatement of the reference algorithm
(oracle/, all host cores) on bounded samples of the same workload; under
torchrun only rank 0 runs it.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

GAMMA_EVALS_REFERENCE_DP = 7  # the reference's Dormand-Prince evaluates the torque 7 times per step (no FSAL)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["multilayer", "film", "precision", "batched", "serving"],
                    default="multilayer")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=8)
    # batched / served forms
    ap.add_argument("--duration", type=float, default=0.2e-9,
                    help="batched: simulated seconds per relaxation (the full problem runs 2 ns)")
    ap.add_argument("--plain-every", type=int, default=8,
                    help="batched: the plain form runs every k-th instance")
    ap.add_argument("--rate", type=float, default=1.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--seconds", type=float, default=30.0, help="serving: length of the arrival window (s)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: device-memory budget")
    return ap.parse_args()


def workload(name):
    import mumaxplus_b200.workloads as W

    return {"multilayer": W.multilayer, "film": W.film, "precision": W.precision}[name]()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(wname):
    """dram bytes per k_yz launch from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"k_yz_{wname}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(w, n_evals=1):
    """FP64 oracle on the host cores: one effective-field evaluation of the
    full workload (a bounded sample), scaled to a reference Dormand-Prince step."""
    import oracle as O
    from mumaxplus_b200 import workloads as Wl

    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w.get("world_bias", (0, 0, 0)))
    q = ow.add_magnet(Wl.desc(w, keep))
    ow.set_m(q, w["m0"]())
    t0 = time.time()
    ow.eval(q, O.abi.Q_DEMAG_FIELD)  # builds the FP64 kernel spectrum (setup, untimed below)
    t_setup = time.time() - t0
    times = []
    for _ in range(n_evals):
        t0 = time.time()
        ow.eval(q, O.abi.Q_EFFECTIVE_FIELD)
        times.append(time.time() - t0)
    t_eval = statistics.median(times)
    N = Wl.ncells(w)
    return {
        "value": N / (GAMMA_EVALS_REFERENCE_DP * t_eval),
        "unit": "cell-updates/s",
        "cores": os.cpu_count(),
        "kind": "port",
        "sample": (f"{n_evals} FP64 effective-field evaluation(s) of the full {w['name']} grid "
                   f"({t_eval:.2f} s each, kernel build {t_setup:.1f} s untimed), scaled by the "
                   f"{GAMMA_EVALS_REFERENCE_DP} evaluations of one reference Dormand-Prince step"),
    }


def run_reference_many(args):
    """CPU FP64 oracle on a bounded sample of the batched / served solves: one
    effective-field evaluation per sampled solve, scaled by the 7 evaluations of
    one reference Dormand-Prince step."""
    import oracle as O
    from mumaxplus_b200 import batch as B
    from mumaxplus_b200 import workloads as Wl

    if args.workload == "batched":
        ws = Wl.batch_instances(256)[::32]
    else:
        ws = Wl.serving_requests(rate=2.0, seconds=4.0)[:6]
    t_tot, cells = 0.0, 0
    for k in range(args.warmup + args.steps):
        w = ws[k % len(ws)]
        keep = []
        ow = O.OracleWorld()
        q = ow.add_magnet(B.solve_desc(w, keep))
        ow.set_m(q, w["m0"]())
        ow.eval(q, O.abi.Q_DEMAG_FIELD)  # kernel construction, untimed
        t0 = time.time()
        ow.eval(q, O.abi.Q_EFFECTIVE_FIELD)
        if k >= args.warmup:
            t_tot += time.time() - t0
            cells += Wl.ncells(w)
    value = cells / (GAMMA_EVALS_REFERENCE_DP * t_tot)
    sample = (f"{args.steps} FP64 effective-field evaluations of {args.workload} solves ({cells} cells), "
              f"scaled by {GAMMA_EVALS_REFERENCE_DP} evaluations per reference Dormand-Prince step")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * GAMMA_EVALS_REFERENCE_DP * t_tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "method": "DormandPrince", "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload in ("batched", "serving"):
        return run_reference_many(args)
    w = workload(args.workload)
    from mumaxplus_b200 import workloads as Wl
    import oracle as O

    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w.get("world_bias", (0, 0, 0)))
    q = ow.add_magnet(Wl.desc(w, keep))
    ow.set_m(q, w["m0"]())
    ow.eval(q, O.abi.Q_DEMAG_FIELD)  # kernel build, untimed
    for _ in range(args.warmup):
        ow.eval(q, O.abi.Q_EFFECTIVE_FIELD)
    t0 = time.time()
    for _ in range(args.steps):
        ow.eval(q, O.abi.Q_EFFECTIVE_FIELD)
    t = (time.time() - t0) / args.steps
    N = Wl.ncells(w)
    value = N / (GAMMA_EVALS_REFERENCE_DP * t)
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": GAMMA_EVALS_REFERENCE_DP * t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "method": "DormandPrince", "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"each step = one FP64 effective-field evaluation of the full grid, scaled by "
                                   f"{GAMMA_EVALS_REFERENCE_DP} evaluations per reference Dormand-Prince step"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    import mumaxplus_b200 as mpx
    from mumaxplus_b200 import workloads as Wl

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    w = workload(args.workload)
    N = Wl.ncells(w)
    world, magnet = Wl.build(mpx, w, device=local)
    stream = torch.cuda.Stream(device=dev)
    world._engine.set_stream(stream.cuda_stream)
    ts = world.timesolver
    ts.set_method("DormandPrince")
    eng = world._engine

    # warm-up (also builds the CUDA graph of one attempt)
    ts.steps(max(args.warmup, 1))
    eng.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    info0 = eng.group_info(world._group)
    l0 = eng.launch_count()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ts.steps(args.steps)
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1)
    launches = eng.launch_count() - l0
    info1 = eng.group_info(world._group)
    clocks = sampler.stop()
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world_size * N * args.steps / (ms_max / 1e3)

    # end to end through the public API: host m in (pinned), one step, host m out
    host_in = torch.empty((3, *magnet.grid.shape), dtype=torch.float32).pin_memory().numpy()
    host_in[...] = magnet.magnetization.get()
    host_out = torch.empty_like(torch.from_numpy(host_in)).pin_memory().numpy()
    k_e2e = max(1, min(args.e2e_steps, args.steps))
    barrier()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        eng.set_m(magnet._id, host_in)
        ts.step()
        eng.get_m(magnet._id, host_in.shape, out=host_out)  # pinned: direct DMA
        host_in, host_out = host_out, host_in
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_value = world_size * N * k_e2e / e2e_s
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = world_size * N * k_e2e / float(t.item())

    # TimeSolver.solve of the film configuration (<m> every 10 ps over 1 ns): the
    # device-sampled table against the host loop (run() + one average per point),
    # both from the same state
    solve_info = None
    if args.workload == "film" and rank == 0:
        tps = [ts.time + 10e-12 * (k + 1) for k in range(100)]
        m_save, t_save, dt_save = magnet.magnetization.get(), ts.time, ts.timestep

        def timed_solve(qd):
            magnet.magnetization = m_save
            ts.time, ts.timestep = t_save, dt_save
            eng.synchronize()
            t0 = time.perf_counter()
            out = ts.solve(tps, qd)
            eng.synchronize()
            return time.perf_counter() - t0, out

        info_s0 = eng.group_info(world._group)
        t_dev, o_dev = timed_solve({"m": magnet.magnetization.average})
        info_s1 = eng.group_info(world._group)
        t_host, o_host = timed_solve({"m": lambda: magnet.magnetization.average()})
        solve_info = {"timepoints": len(tps), "interval_s": 10e-12, "accepted_steps": int(info_s1.steps - info_s0.steps),
                      "device_sampled_s": t_dev, "host_loop_s": t_host,
                      "same_table": o_dev["m"] == o_host["m"] and o_dev["time"] == o_host["time"]}

    # dominant kernel, timed live with CUDA events on the engine's stream
    kms = eng.profile_eval(magnet._id, reps=10)
    names = ["k_xfwd", "k_yz", "k_xinv", "k_local"]
    dom = int(np.argmax(kms))
    d = magnet._engine  # noqa: F841
    nx, ny, nz = w["size"]
    P = [1 if n == 1 else 1 << int(np.ceil(np.log2(2 * n - 1))) for n in (nx, ny, nz)]
    Fh = P[0] // 2 + 1
    spec_bytes = Fh * 3 * ny * nz * 8
    kspec_bytes = Fh * (P[1] // 2 + 1) * (P[2] // 2 + 1) * (6 if P[2] > 1 else 4) * 4
    alg_bytes = {
        "k_xfwd": 12 * N + spec_bytes,              # read m, write the x spectrum
        "k_yz": 2 * spec_bytes + kspec_bytes,       # read + write the spectrum, read the kernel spectrum
        "k_xinv": spec_bytes + 12 * N + 12 * N,     # read spectrum and m, write the result
        "k_local": 24 * N,
    }[names[dom]]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kms[dom] / 1e3) / 1e9
    traffic = profile_traffic(w["name"]) if names[dom] == "k_yz" else None

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(w)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {exc}"}

    if rank == 0:
        steps = info1.steps - info0.steps
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": w["name"], "method": "DormandPrince (adaptive, max_error 1e-5)",
                       "cells_per_gpu": N, "accepted_steps": int(steps),
                       "rejected_attempts": int(info1.rejected - info0.rejected),
                       "l2": "inputs larger than L2 (state + spectra + kernel ~ 340 MB per replica)",
                       "parallelism": f"replicas x{world_size}" if world_size > 1 else "single GPU",
                       "fft_padding": f"{P[0]}x{P[1]}x{P[2]}"},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel_ms": {n: round(t, 4) for n, t in zip(names, kms)}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": 12 * N,
                    "d2h_bytes_per_step": 12 * N, "steps": k_e2e},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if solve_info is not None:
            line["solve"] = solve_info
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _dist_setup():
    import torch

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    torch.cuda.set_device(local)
    if world_size > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world_size, rank, local, dist


def _max_over_ranks(dist, value, device):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_batched(args):
    """Relaxation batch: 256 solves of side 32-256 (nz 1 or 2) advanced together
    vs the same solves one at a time (the plain form, on every k-th instance).
    Under torchrun a pool of 256 solves per rank is spread over the ranks by a
    cell-balanced bin packing (independent solves, no collective on the data
    path)."""
    import torch

    from mumaxplus_b200 import batch as B
    from mumaxplus_b200 import workloads as Wl

    world_size, rank, local, dist = _dist_setup()
    dev = torch.device("cuda", local)
    # 256 solves per GPU: a pool of 256 x N spread over the ranks by cells
    pool = Wl.batch_instances(256 * world_size)
    insts = [pool[i] for i in B.shard(pool, rank, world_size)]
    wb = B.Batch(device=local)  # warm-up: first graph captures, pool growth
    B.relax_batch(wb, insts[: max(1, args.warmup)], duration=2e-12, torque_stop=1e-4)
    del wb
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    b = B.Batch(device=local)
    l0 = b.engine.launch_count()
    t0 = time.perf_counter()
    solves, t_run, t_setup = B.relax_batch(b, insts, duration=args.duration, torque_stop=1e-4)
    t_e2e = time.perf_counter() - t0
    launches = b.engine.launch_count() - l0
    clocks = sampler.stop()
    upd = sum(s.cells * s.steps for s in solves)
    t_run_max = _max_over_ranks(dist, t_run, dev)
    t_e2e_max = _max_over_ranks(dist, t_e2e, dev)
    # the plain form: the same solves one at a time (one solve resident)
    k = max(1, args.plain_every)
    sub = insts[::k]
    psol, p_run, p_setup = B.run_plain(B.Batch(device=local), sub, duration=args.duration, torque_stop=1e-4)
    p_upd = sum(s.cells * s.steps for s in psol)
    same = {s.key: s for s in solves}
    worst = max(float(np.max(np.abs(same[k * i].m - p.m))) for i, p in enumerate(psol))
    # per-kernel time of one attempt stage over the whole started batch
    kb = B.Batch(device=local)
    started = [kb.add(w, key=i) for i, w in enumerate(insts)]
    for s in started:
        kb.start(s, 1e-9, 0.0)
    kb.advance(2)
    kb.poll()
    kms = kb.engine.profile_attempt("DormandPrince", reps=5)
    del kb, started
    if rank == 0:
        value = world_size * upd / t_run_max
        plain = p_upd / p_run
        steps = [s.steps for s in solves]
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world_size,
            "steps": int(sum(steps)), "warmup": args.warmup, "ms_per_step": 1e3 * t_run_max / max(1, max(steps)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch_256_relax", "instances": len(insts),
                       "cells": int(sum(s.cells for s in solves)), "duration_s": args.duration,
                       "torque_stop_T": 1e-4, "method": "DormandPrince 1e-5",
                       "parallelism": f"solves sharded over {world_size} ranks" if world_size > 1 else "single GPU",
                       "l2": "state + spectra of the batch ~ 2 GB, larger than L2"},
            "batched": {"cell_updates": upd, "seconds": t_run, "setup_seconds": t_setup,
                        "solves_per_s": len(solves) / t_run,
                        "steps_min_median_max": [int(min(steps)), float(np.median(steps)), int(max(steps))],
                        "stopped_on_torque": int(sum(1 for s in solves if s.sim_time < 0.999 * args.duration)),
                        "failed": int(sum(s.failed for s in solves)),
                        "autotuned_shape_divisors": {"x": b.tuned[0], "y_z": b.tuned[1]}},
            "plain": {"instances": len(sub), "cell_updates": p_upd, "seconds": p_run, "setup_seconds": p_setup,
                      "value": plain, "unit": "cell-updates/s"},
            "batched_over_plain": value / world_size / plain,
            "stage_kernel_ms": {"combine+x_forward": kms[0], "stray_pairs": kms[1], "y_z": kms[2],
                                "x_inverse+epilogue": kms[3], "note": "one stage (of 6 per accepted step) over all "
                                                                      "256 started solves"},
            "max_abs_dm_batched_vs_plain": worst,
            "e2e": {"value": world_size * upd / t_e2e_max, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": int(sum(12 * s.cells for s in solves)),
                    "d2h_bytes_per_step": int(sum(12 * s.cells for s in solves)),
                    "note": "one step = the whole batch: host m0 in, kernel construction, integration, host m out"},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_serving(args):
    """Open-loop Poisson request stream served by continuous batching, vs the
    same requests served one at a time (the plain form: one solve resident)."""
    import torch

    from mumaxplus_b200 import batch as B
    from mumaxplus_b200 import workloads as Wl

    world_size, rank, local, dist = _dist_setup()
    dev = torch.device("cuda", local)
    reqs = Wl.serving_requests(rate=args.rate, seconds=args.seconds, seed=5 + rank)
    budget = args.budget_gb * 1e9
    wb = B.Batch(device=local)  # warm-up
    B.relax_batch(wb, [dict(r) for r in reqs[: max(1, args.warmup)]], duration=2e-12, torque_stop=0.0)
    del wb
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    b = B.Batch(device=local)
    l0 = b.engine.launch_count()
    t0 = time.perf_counter()
    served = B.Server(b, budget).run(reqs)
    span = time.perf_counter() - t0
    launches = b.engine.launch_count() - l0
    clocks = sampler.stop()
    span_max = _max_over_ranks(dist, span, dev)
    t0 = time.perf_counter()
    plain = B.Server(B.Batch(device=local), budget, max_active=1).run(reqs)
    p_span = time.perf_counter() - t0
    p50, p99 = B.latency_stats(served)
    q50, q99 = B.latency_stats(plain)
    upd = sum(s.cells * s.steps for s in served)
    p_upd = sum(s.cells * s.steps for s in plain)
    by = {s.key: s for s in plain}
    worst = max((float(np.max(np.abs(s.m - by[s.key].m))) for s in served if s.key in by), default=0.0)
    if rank == 0:
        per_req = int(sum(12 * s.cells for s in served) / max(1, len(served)))
        line = {
            "metric": "solves/s", "value": world_size * len(served) / span_max, "unit": "solves/s",
            "n_gpus": world_size, "steps": int(sum(s.steps for s in served)), "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "serving_poisson", "rate_per_s": args.rate, "window_s": args.seconds,
                       "requests": len(reqs), "budget_gb": args.budget_gb, "method": "DormandPrince 1e-5"},
            "served": {"p50_s": p50, "p99_s": p99, "makespan_s": span, "cell_updates_per_s": upd / span},
            "plain": {"p50_s": q50, "p99_s": q99, "makespan_s": p_span, "solves_per_s": len(plain) / p_span,
                      "cell_updates_per_s": p_upd / p_span},
            "max_abs_dm_served_vs_plain": worst,
            "e2e": {"value": world_size * len(served) / span_max, "unit": "solves/s",
                    "h2d_bytes_per_step": per_req, "d2h_bytes_per_step": per_req,
                    "note": "per request: host m0 in, host m out; latency from arrival to result on the host"},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_precision(args):
    """Precision form: demag-only field of 1024x1024x4 random unit vectors
    (padded FFT 2048x2048x8) against the FP64 oracle, per cell
    |dB| / |B_ref| over cells with |B_ref| > 1e-6 max|B_ref|, and the
    evaluation rate of the field on the GPU."""
    import torch

    import mumaxplus_b200 as mpx
    import oracle as O
    from mumaxplus_b200 import workloads as Wl

    world_size, rank, local, dist = _dist_setup()
    w = Wl.precision()
    N = Wl.ncells(w)
    world, magnet = Wl.build(mpx, w, device=local)
    eng = magnet._engine
    q = mpx._abi.Q_DEMAG_FIELD
    shape = (3, *magnet.grid.shape)
    got = eng.eval(magnet._id, q, shape).astype(np.float64)
    stream = torch.cuda.Stream(device=local)
    eng.set_stream(stream.cuda_stream)
    for _ in range(max(3, args.warmup)):
        eng.eval_only(magnet._id, q)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        eng.eval_only(magnet._id, q)
    e1.record(stream)
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1) / args.steps
    ms = _max_over_ranks(dist, ms, torch.device("cuda", local))
    kms = eng.profile_eval(magnet._id, reps=5)
    if rank == 0:
        keep = []
        ow = O.OracleWorld()
        oq = ow.add_magnet(Wl.desc(w, keep))
        ow.set_m(oq, w["m0"]())
        t0 = time.time()
        want = ow.eval(oq, O.abi.Q_DEMAG_FIELD)
        t_oracle = time.time() - t0
        nref = np.linalg.norm(want, axis=0)
        mask = nref > 1e-6 * nref.max()
        rel = np.linalg.norm(got - want, axis=0)[mask] / nref[mask]
        # the same FP64 convolution with the GPU's own kernel values: separates the
        # FP32 FFT arithmetic from the FP64 rounding noise of the two kernel
        # constructions, which dominates far from the source (newell.cu's
        # 27-point differences of O(r^3) terms cancel to O(r^-3) values)
        K = eng.demag_kernel(magnet._id)
        nx, ny, nz = w["size"]
        o = [K.shape[3] - nx, K.shape[2] - ny, K.shape[1] - nz]
        oct = K[:, o[2]:, o[1]:, o[0]:].astype(np.float64)
        del K
        ow2 = O.OracleWorld()
        oq2 = ow2.add_magnet(Wl.desc(w, keep))
        ow2.set_m(oq2, w["m0"]())
        ow2.set_kernel_octant(oq2, oct)
        want2 = ow2.eval(oq2, O.abi.Q_DEMAG_FIELD)
        nref2 = np.linalg.norm(want2, axis=0)
        mask2 = nref2 > 1e-6 * nref2.max()
        rel2 = np.linalg.norm(got - want2, axis=0)[mask2] / nref2[mask2]
        line = {
            "metric": "B_demag max relative error vs FP64", "value": float(rel.max()), "unit": "relative",
            "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["name"], "fft_padding": "2048x2048x8", "dft": "FP32 shared-memory Stockham",
                       "cells_compared": int(mask.sum())},
            "rms_relative_error": float(np.sqrt(np.mean(rel * rel))),
            "max_abs_error_over_max_field": float(np.abs(got - want).max() / np.abs(want).max()),
            "same_kernel": {"max_relative_error": float(rel2.max()),
                            "rms_relative_error": float(np.sqrt(np.mean(rel2 * rel2))),
                            "max_abs_error_over_max_field": float(np.abs(got - want2).max() / np.abs(want2).max()),
                            "note": "FP64 oracle convolution with the GPU's FP64 kernel values (rounded to FP32)"},
            "evals_per_s": world_size * 1e3 / ms, "cell_evals_per_s": world_size * N * 1e3 / ms,
            "kernel_ms": {"k_xfwd": kms[0], "k_yz": kms[1], "k_xinv": kms[2]},
            "oracle_seconds": t_oracle,
            "e2e": {"value": float(rel.max()), "unit": "relative", "h2d_bytes_per_step": 12 * N,
                    "d2h_bytes_per_step": 12 * N},
            "gpu_launches": 3 * args.steps,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "precision":
        run_precision(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
