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
    ap.add_argument("--no-batched", action="store_true",
                    help="default workload: leave out the batched-form sub-record (configuration 4)")
    ap.add_argument("--batched-duration", type=float, default=2e-9,
                    help="default workload: simulated seconds per relaxation of the batched sub-record")
    # batched / served forms
    ap.add_argument("--duration", type=float, default=0.2e-9,
                    help="batched: simulated seconds per relaxation (the full problem runs 2 ns)")
    ap.add_argument("--plain-every", type=int, default=8,
                    help="batched: the plain form runs every k-th instance")
    ap.add_argument("--rate", type=float, default=1.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--seconds", type=float, default=30.0, help="serving: length of the arrival window (s)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: device-memory budget")
    ap.add_argument("--time-limit", type=float, default=None,
                    help="serving: wall-clock limit of each served run (s); unfinished requests are reported")
    ap.add_argument("--max-cells", type=float, default=None,
                    help="serving: also run the served form with admission capped at this many resident cells")
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


# CUDA sources each profiled kernel is compiled from (the hash in its
# committed ncu summary covers these files)
PROFILE_SOURCES = {
    "k_yz": ("kernels.cuh", "fft.cuh", "physics.cuh"),
    "k_xinv": ("kernels.cuh", "fft.cuh", "physics.cuh"),
    "k_xfwd": ("kernels.cuh", "fft.cuh", "physics.cuh"),
}


_CODE_TOKENS = None


def code_only(text):
    """C++ / CUDA source text without its comments and blank lines (string
    literals kept), so that a change of comments leaves the hash of the code."""
    import re

    global _CODE_TOKENS
    if _CODE_TOKENS is None:
        _CODE_TOKENS = re.compile(r'//[^\n]*|/\*.*?\*/|"(?:\\.|[^"\\\n])*"|\'(?:\\.|[^\'\\\n])*\'', re.S)
    text = _CODE_TOKENS.sub(lambda m: m.group(0) if m.group(0)[0] in "\"'" else "", text)
    return "\n".join(line.rstrip() for line in text.splitlines() if line.strip())


def kernel_sources_sha(files):
    """Hash of the code (comments left out) of the given CUDA sources of the
    product library (csrc/)."""
    import hashlib

    d = os.path.join(ROOT, "mumax-plus_b200", "csrc")
    h = hashlib.sha256()
    for name in sorted(files):
        with open(os.path.join(d, name), encoding="utf-8") as f:
            h.update(name.encode() + b"\0" + code_only(f.read()).encode())
    return h.hexdigest()[:16]


def profile_traffic(kernel, wname):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    profiles/<kernel>_<workload>.md, with the hash of the CUDA sources it was
    captured from.  The bytes are reported only while that hash equals the
    hash of the sources this run was built from (else the capture is stale
    and traffic is null)."""
    rel = os.path.join("profiles", f"{kernel}_{wname}.md")
    files = PROFILE_SOURCES.get(kernel, ())
    src = {"file": rel, "sources": list(files), "sources_sha": None,
           "build_sources_sha": kernel_sources_sha(files) if files else None, "matches_build": False}
    val = None
    try:
        for line in open(os.path.join(ROOT, rel)):
            if line.startswith("traffic_bytes_per_launch:"):
                val = float(line.split(":")[1])
            elif line.startswith("sources_sha:"):
                src["sources_sha"] = line.split(":")[1].strip()
    except OSError:
        return None, src
    src["matches_build"] = src["sources_sha"] is not None and src["sources_sha"] == src["build_sources_sha"]
    return (val if src["matches_build"] else None), src


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


def _oracle_world(w):
    """FP64 oracle world of workload `w` with its initial state, the kernel
    spectrum already built (setup, outside every timed region), Dormand-Prince
    from the sensible time step."""
    import oracle as O
    from mumaxplus_b200 import workloads as Wl

    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w.get("world_bias", (0, 0, 0)))
    q = ow.add_magnet(Wl.desc(w, keep))
    ow.set_m(q, w["m0"]())
    t0 = time.time()
    ow.eval(q, O.abi.Q_DEMAG_FIELD)  # builds the FP64 kernel spectrum
    t_setup = time.time() - t0
    ow.set_method("DormandPrince")
    ow.timestep = ow.sensible_timestep()
    return ow, q, keep, t_setup


def _oracle_steps(ow, n):
    """n Dormand-Prince step attempts of the oracle (the reference's
    TimeSolver::step: 7 torque evaluations each, rejected attempts retried on
    the next call); returns (seconds, accepted steps, attempts)."""
    c0 = ow.counters()
    t0 = time.time()
    ow.steps(n)
    t = time.time() - t0
    c1 = ow.counters()
    return t, c1["steps"] - c0["steps"], n


def cpu_baseline(w, n_steps=2):
    """FP64 oracle on the host cores: a bounded sample of real Dormand-Prince
    steps of the full workload (stage combinations, normalisation, torque,
    error norm and controller included)."""
    from mumaxplus_b200 import workloads as Wl

    ow, q, keep, t_setup = _oracle_world(w)
    t, acc, att = _oracle_steps(ow, n_steps)
    N = Wl.ncells(w)
    return {
        "value": N * acc / t,
        "unit": "cell-updates/s",
        "cores": os.cpu_count(),
        "kind": "port",
        "sample": (f"{att} FP64 Dormand-Prince step attempts ({acc} accepted, 7 torque evaluations each) of the "
                   f"full {w['name']} grid from its initial state, {t:.1f} s; FP64 kernel build {t_setup:.1f} s "
                   f"untimed"),
    }


def run_reference_many(args):
    """CPU FP64 oracle on a bounded sample of the batched / served solves: per
    sampled solve, real Dormand-Prince steps from its initial state."""
    from mumaxplus_b200 import batch as B
    from mumaxplus_b200 import workloads as Wl

    if args.workload == "batched":
        ws = Wl.batch_instances(256)[::32]
    else:
        ws = Wl.serving_requests(rate=2.0, seconds=4.0)[:6]
    t_tot, upd, att_tot = 0.0, 0, 0
    for k in range(args.warmup + args.steps):
        w = dict(ws[k % len(ws)])
        w.setdefault("name", f"solve_{k}")
        import oracle as O

        keep = []
        ow = O.OracleWorld()  # the applied field is the solve's own bias field (solve_desc)
        q = ow.add_magnet(B.solve_desc(w, keep))
        ow.set_m(q, w["m0"]())
        ow.eval(q, O.abi.Q_DEMAG_FIELD)  # kernel construction, untimed
        ow.set_method("DormandPrince")
        ow.timestep = ow.sensible_timestep()
        t, acc, att = _oracle_steps(ow, 4)
        if k >= args.warmup:
            t_tot += t
            upd += Wl.ncells(w) * acc
            att_tot += att
    value = upd / t_tot
    sample = (f"{args.steps} {args.workload} solves (every 32nd of the pool), 4 FP64 Dormand-Prince step "
              f"attempts each ({att_tot} in all) from the initial state")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "method": "DormandPrince", "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    """The reference arm: the CPU FP64 restatement of the reference's path
    (oracle/, all host cores) taking real Dormand-Prince steps of the same
    workload; each timed step is one step attempt of the full grid."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload in ("batched", "serving"):
        return run_reference_many(args)
    w = workload(args.workload)
    from mumaxplus_b200 import workloads as Wl

    ow, q, keep, t_setup = _oracle_world(w)
    _oracle_steps(ow, args.warmup)
    t, acc, att = _oracle_steps(ow, args.steps)
    N = Wl.ncells(w)
    value = N * acc / t
    sample = (f"{att} FP64 Dormand-Prince step attempts of the full grid ({acc} accepted, 7 torque evaluations "
              f"each) after {args.warmup} warm-up attempts; FP64 kernel build {t_setup:.1f} s untimed")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "method": "DormandPrince (adaptive, max_error 1e-5)",
                   "accepted_steps": int(acc), "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
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

    # dominant kernel of the timed region, whose launches are Runge-Kutta stage
    # evaluations: stage 1 of an attempt of the same magnet started alone (the
    # tile shapes of the single solve), each kernel timed live with CUDA events
    # on the engine's stream.  The kernels of one evaluation of the effective
    # field quantity (another epilogue, not in the timed region) are reported
    # beside them.
    eval_kms = eng.profile_eval(magnet._id, reps=10)
    kms = stage_kernel_ms(w, local)
    names = ["k_xfwd", "k_yz", "k_xinv"]
    dom = int(np.argmax(kms))
    nx, ny, nz = w["size"]
    P = [1 if n == 1 else 1 << int(np.ceil(np.log2(2 * n - 1))) for n in (nx, ny, nz)]
    Fh = P[0] // 2 + 1
    spec_bytes = Fh * 3 * ny * nz * 8
    kspec_bytes = Fh * (P[1] // 2 + 1) * (P[2] // 2 + 1) * (6 if P[2] > 1 else 4) * 4
    alg_bytes = {
        "k_xfwd": 36 * N + spec_bytes,              # read x0 and k0, write the stage state and the x spectrum
        "k_yz": 2 * spec_bytes + kspec_bytes,       # read + write the spectrum, read the kernel spectrum
        "k_xinv": spec_bytes + 12 * N + 12 * N,     # read spectrum and stage state, write the stage torque
    }[names[dom]]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kms[dom] / 1e3) / 1e9
    traffic, traffic_src = profile_traffic(names[dom], w["name"])

    # configuration 4 as a sub-record of the default line (one GPU): the 256
    # relaxations batched vs the plain one-at-a-time form
    batched = None
    if world_size == 1 and args.workload == "multilayer" and not args.no_batched:
        insts = Wl.batch_instances(256)
        r = _batched_measure(insts, args.batched_duration, args.plain_every, 1, local)
        batched = {"workload": "batch_256_relax", **r}

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
                         "traffic": traffic, "traffic_source": traffic_src,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel_ms": {n: round(t, 4) for n, t in zip(names, kms)},
                         "kernel_form": "Runge-Kutta stage 1 (combination + x forward, y/z, x inverse + torque)",
                         "field_eval_kernel_ms": {n: round(t, 4) for n, t in
                                                  zip(["k_xfwd", "k_yz", "k_xinv", "k_local"], eval_kms)}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": 12 * N,
                    "d2h_bytes_per_step": 12 * N, "steps": k_e2e},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if solve_info is not None:
            line["solve"] = solve_info
        if batched is not None:
            line["batched_form"] = batched
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


def stage_kernel_ms(w, local, reps=10):
    """Mean ms per launch of [stage combination + x forward, y/z pass, x inverse +
    torque] over stage 1 of a Dormand-Prince attempt of workload `w` started
    alone (mpx_profile_attempt: CUDA events on the engine's stream)."""
    from mumaxplus_b200 import batch as B

    kb = B.Batch(device=local)
    s = kb.add(w, key=0)
    kb.start(s, 1e-9, 0.0)
    kb.advance(2)
    kb.poll()
    kms = kb.engine.profile_attempt("DormandPrince", reps=reps)
    del kb, s
    return [kms[0], kms[2], kms[3]]


def _batched_measure(insts, duration, plain_every, warmup, local):
    """Configuration 4 on this GPU: `insts` relaxed together in one batch
    (torque stop 1e-4 T or `duration`), then every `plain_every`-th of them
    one at a time (the plain form); per-kernel times of one stage over the
    started batch.  Returns a dict of the measurements."""
    from mumaxplus_b200 import batch as B

    wb = B.Batch(device=local)  # warm-up: first graph captures, pool growth
    B.relax_batch(wb, insts[: max(1, warmup)], duration=2e-12, torque_stop=1e-4)
    del wb
    b = B.Batch(device=local)
    l0 = b.engine.launch_count()
    t0 = time.perf_counter()
    solves, t_run, t_setup = B.relax_batch(b, insts, duration=duration, torque_stop=1e-4)
    t_e2e = time.perf_counter() - t0
    launches = b.engine.launch_count() - l0
    tuned = b.tuned
    del b
    upd = sum(s.cells * s.steps for s in solves)
    k = max(1, plain_every)
    sub = insts[::k]
    psol, p_run, p_setup = B.run_plain(B.Batch(device=local), sub, duration=duration, torque_stop=1e-4)
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
    steps = [s.steps for s in solves]
    sub_set = set(range(0, len(insts), k))
    b_sub_upd = sum(s.cells * s.steps for s in solves if s.key in sub_set)
    return {
        "instances": len(insts), "cells": int(sum(s.cells for s in solves)), "duration_s": duration,
        "torque_stop_T": 1e-4,
        "batched": {"cell_updates": int(upd), "seconds": t_run, "setup_seconds": t_setup,
                    "value": upd / t_run, "unit": "cell-updates/s", "solves_per_s": len(solves) / t_run,
                    "steps_min_median_max": [int(min(steps)), float(np.median(steps)), int(max(steps))],
                    "stopped_on_torque": int(sum(1 for s in solves if s.sim_time < 0.999 * duration)),
                    "failed": int(sum(s.failed for s in solves)),
                    "autotuned_shape_divisors": {"x": tuned[0], "y_z": tuned[1]}},
        "plain": {"instances": len(sub), "every": k, "cell_updates": int(p_upd), "seconds": p_run,
                  "setup_seconds": p_setup, "value": p_upd / p_run, "unit": "cell-updates/s",
                  "solves_per_s": len(sub) / p_run,
                  "same_solves_cell_updates_in_batch": int(b_sub_upd)},
        "batched_over_plain": (upd / t_run) / (p_upd / p_run),
        "stage_kernel_ms": {"combine+x_forward": kms[0], "stray_pairs": kms[1], "y_z": kms[2],
                            "x_inverse+epilogue": kms[3],
                            "note": "one stage (of 6 per accepted step) over all started solves"},
        "max_abs_dm_batched_vs_plain": worst,
        "e2e_seconds": t_e2e, "e2e_bytes_each_way": int(sum(12 * s.cells for s in solves)),
        "gpu_launches": int(launches),
    }


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
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    r = _batched_measure(insts, args.duration, args.plain_every, args.warmup, local)
    clocks = sampler.stop()
    t_run_max = _max_over_ranks(dist, r["batched"]["seconds"], dev)
    t_e2e_max = _max_over_ranks(dist, r["e2e_seconds"], dev)
    if rank == 0:
        upd = r["batched"]["cell_updates"]
        value = world_size * upd / t_run_max
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world_size,
            "steps": None, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch_256_relax", "instances": r["instances"], "cells": r["cells"],
                       "duration_s": args.duration, "torque_stop_T": 1e-4, "method": "DormandPrince 1e-5",
                       "parallelism": f"solves sharded over {world_size} ranks" if world_size > 1 else "single GPU",
                       "l2": "state + spectra of the batch ~ 2 GB, larger than L2"},
            "batched": r["batched"], "plain": r["plain"], "batched_over_plain": r["batched_over_plain"],
            "stage_kernel_ms": r["stage_kernel_ms"],
            "max_abs_dm_batched_vs_plain": r["max_abs_dm_batched_vs_plain"],
            "e2e": {"value": world_size * upd / t_e2e_max, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": r["e2e_bytes_each_way"], "d2h_bytes_per_step": r["e2e_bytes_each_way"],
                    "note": "one step = the whole batch: host m0 in, kernel construction, integration, host m out"},
            "gpu_launches": r["gpu_launches"],
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
    st_served, st_plain = {}, {}
    served = B.Server(b, budget).run(reqs, time_limit=args.time_limit, stats=st_served)
    span = time.perf_counter() - t0
    launches = b.engine.launch_count() - l0
    clocks = sampler.stop()
    del b
    span_max = _max_over_ranks(dist, span, dev)
    capped = None
    if args.max_cells:
        st_cap = {}
        t0 = time.perf_counter()
        served_cap = B.Server(B.Batch(device=local), budget, max_cells=args.max_cells).run(
            reqs, time_limit=args.time_limit, stats=st_cap)
        c_span = time.perf_counter() - t0
        c50, c99 = B.latency_stats(served_cap)
        c_upd = sum(s.cells * s.steps for s in served_cap)
        capped = {"max_cells": args.max_cells, "p50_s": c50, "p99_s": c99, "makespan_s": c_span,
                  "solves_per_s": len(served_cap) / c_span, "cell_updates_per_s": c_upd / c_span,
                  **_serving_summary(st_cap)}
    t0 = time.perf_counter()
    plain = B.Server(B.Batch(device=local), budget, max_active=1).run(reqs, time_limit=args.time_limit,
                                                                      stats=st_plain)
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
                       "requests": len(reqs), "budget_gb": args.budget_gb, "method": "DormandPrince 1e-5",
                       "time_limit_s": args.time_limit},
            "served": {"p50_s": p50, "p99_s": p99, "makespan_s": span, "cell_updates_per_s": upd / span,
                       **_serving_summary(st_served)},
            "plain": {"p50_s": q50, "p99_s": q99, "makespan_s": p_span, "solves_per_s": len(plain) / p_span,
                      "cell_updates_per_s": p_upd / p_span, **_serving_summary(st_plain)},
            "served_cell_capped": capped,
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


def _serving_summary(st):
    """Counts and queue history of one served run (Server.run stats)."""
    smp = st.get("samples", [])
    step = max(1, len(smp) // 40)
    return {"arrived": st.get("arrived"), "admitted": st.get("admitted"), "finished": st.get("finished"),
            "still_queued": st.get("still_queued"), "still_running": st.get("still_running"),
            "max_queued": max((q for _, q, _ in smp), default=0),
            "max_running": max((r for _, _, r in smp), default=0),
            "host_admit_s": st.get("host_admit_s"), "host_advance_s": st.get("host_advance_s"),
            "queue_samples_t_queued_running": smp[::step]}


def run_precision(args):
    """Precision form: demag-only field of 1024x1024x4 random unit vectors
    (padded FFT 2048x2048x8) against the FP64 oracle, for both arithmetics of
    the y transforms: the FP32 shared-memory FFT and the TF32 tensor-core DFT
    GEMMs with 3xTF32 split products.  Per cell |dB| / |B_ref| over cells
    with |B_ref| > 1e-6 max|B_ref| (max and RMS), and max|dB| / max|B_ref|,
    against (i) the oracle's own FP64 kernel and (ii) the oracle convolving
    the GPU's kernel values in FP64 (which isolates the transform arithmetic
    from the FP64 rounding noise of the two Newell constructions); and the
    evaluation rate of each form."""
    import torch

    import mumaxplus_b200 as mpx
    import oracle as O
    from mumaxplus_b200 import workloads as Wl

    world_size, rank, local, dist = _dist_setup()
    w = Wl.precision()
    N = Wl.ncells(w)
    q = mpx._abi.Q_DEMAG_FIELD
    forms = {}
    kernel_oct = None
    for dft in ("fp32", "tf32x3"):
        world, magnet = Wl.build(mpx, w, device=local, demag_dft=dft)
        eng = magnet._engine
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
        ms = _max_over_ranks(dist, e0.elapsed_time(e1) / args.steps, torch.device("cuda", local))
        kms = eng.profile_eval(magnet._id, reps=5)
        if kernel_oct is None and rank == 0:
            K = eng.demag_kernel(magnet._id)
            nx, ny, nz = w["size"]
            o = [K.shape[3] - nx, K.shape[2] - ny, K.shape[1] - nz]
            kernel_oct = K[:, o[2]:, o[1]:, o[0]:].astype(np.float64)
            del K
        forms[dft] = {"field": got, "ms": ms, "kernel_ms": {"x_forward": kms[0], "y_z": kms[1], "x_inverse": kms[2]},
                      "timeouts": mpx._engine.Engine.tc_timeouts()}
        eng.synchronize()
        del world, magnet, eng
    if rank == 0:
        keep = []
        ow = O.OracleWorld()
        oq = ow.add_magnet(Wl.desc(w, keep))
        ow.set_m(oq, w["m0"]())
        t0 = time.time()
        want = ow.eval(oq, O.abi.Q_DEMAG_FIELD)
        t_oracle = time.time() - t0
        del ow
        ow2 = O.OracleWorld()
        oq2 = ow2.add_magnet(Wl.desc(w, keep))
        ow2.set_m(oq2, w["m0"]())
        ow2.set_kernel_octant(oq2, kernel_oct)
        want2 = ow2.eval(oq2, O.abi.Q_DEMAG_FIELD)
        del ow2, kernel_oct

        def errs(got, ref):
            nref = np.linalg.norm(ref, axis=0)
            mask = nref > 1e-6 * nref.max()
            rel = np.linalg.norm(got - ref, axis=0)[mask] / nref[mask]
            return {"max_relative_error": float(rel.max()), "rms_relative_error": float(np.sqrt(np.mean(rel * rel))),
                    "max_abs_error_over_max_field": float(np.abs(got - ref).max() / np.abs(ref).max()),
                    "cells_compared": int(mask.sum())}

        report = {}
        for dft, f in forms.items():
            report[dft] = {"vs_fp64_own_kernel": errs(f["field"], want),
                           "vs_fp64_same_kernel": errs(f["field"], want2),
                           "ms_per_eval": f["ms"], "evals_per_s": world_size * 1e3 / f["ms"],
                           "cell_evals_per_s": world_size * N * 1e3 / f["ms"], "kernel_ms": f["kernel_ms"],
                           "tensor_core_wait_timeouts": f["timeouts"]}
        report["tf32x3_vs_fp32_gpu"] = errs(forms["tf32x3"]["field"], forms["fp32"]["field"])
        tc = report["tf32x3"]
        line = {
            "metric": "B_demag max relative error vs FP64", "value": tc["vs_fp64_same_kernel"]["max_relative_error"],
            "unit": "relative", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tc["ms_per_eval"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "tf32x3 (y DFT) / f32", "data": "synthetic",
            "config": {"workload": w["name"], "fft_padding": "2048x2048x8",
                       "dft": "y stages: TF32 tensor-core GEMMs with 3xTF32 split (tcgen05); x stages FP32 FFT",
                       "value_is": "TF32x3 form vs the FP64 oracle convolving the same kernel values"},
            "forms": report,
            "oracle_seconds": t_oracle,
            "e2e": {"value": tc["vs_fp64_same_kernel"]["max_relative_error"], "unit": "relative",
                    "h2d_bytes_per_step": 12 * N, "d2h_bytes_per_step": 12 * N},
            "gpu_launches": 5 * args.steps,
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
