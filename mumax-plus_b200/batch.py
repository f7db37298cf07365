"""Batched and served forms: many independent Landau-Lifshitz-Gilbert solves
advanced together on one engine.

Every solve is its own group (own time, time step and Dormand-Prince
controller, the device-side restatement of core/timesolver.cpp:60-111)
holding one magnet.  `Engine.advance(k)` replays k attempts of one CUDA graph
whose kernels cover the tiles of every started magnet at once, so a few
hundred small solves cost the launches of one; a solve whose duration is
reached, or whose max|torque|/gamma_LL drops below its stop value, leaves the
launch tables at the next poll.  The per-solve applied field is the magnet's
own bias field (physics/zeeman.cu:53-91 adds it to the world field).

  Batch        the mechanism: add / start / advance / poll / finish
  relax_batch  the relaxation batch: every solve started at once, run to the end
  run_plain    the same solves one at a time (one solve resident), the plain form
  Server       continuous batching of an arriving request stream, admitted
               against a device-memory budget, with per-request latency

A solve's trajectory does not depend on what else is resident: each block of
every kernel works on one magnet, and the error / torque maxima are taken per
group, so a solve gives bit-identical results alone and in any mix.
"""
import collections
import concurrent.futures
import time

import numpy as np

from . import _abi, workloads
from ._engine import Engine, magnet_bytes

GS_FAILED = 3


class Solve:
    """One solve of a batch: its workload, device ids and outcome."""

    __slots__ = ("key", "w", "group", "magnet", "shape", "cells", "resident", "transient", "duration", "t_start",
                 "torque_stop", "arrival", "t_admit", "t_done", "steps", "rejected", "sim_time", "failed", "m")

    def __init__(self, key, w):
        self.key = key
        self.w = w
        nx, ny, nz = w["size"]
        self.shape = (3, nz, ny, nx)
        self.cells = nx * ny * nz
        self.group = self.magnet = None
        self.duration = self.torque_stop = self.t_start = 0.0
        self.arrival = self.t_admit = self.t_done = None
        self.steps = self.rejected = 0
        self.sim_time = 0.0
        self.failed = False
        self.m = None


def solve_desc(w, keep):
    """mpx_magnet_desc of a solve: the workload's parameters, its applied field
    as the magnet's bias field."""
    d = workloads.desc(w, keep)
    for c, v in enumerate(w.get("world_bias", (0.0, 0.0, 0.0))):
        d.bias_magnetic_field.uniform[c] = float(v)
    return d


def solve_bytes(w):
    """(resident, transient) device bytes of one solve."""
    return magnet_bytes(solve_desc(w, []))


class Batch:
    """Independent solves on one engine (one CUDA stream on one device)."""

    def __init__(self, device=None, method="DormandPrince", max_error=1e-5, engine=None):
        self.engine = engine if engine is not None else Engine(device)
        self.method = _abi.RK_METHODS[method]
        self.max_error = float(max_error)
        self.solves = {}  # group id -> Solve
        self.resident = 0
        self.tuned = (1, 1)  # tile-shape divisors chosen by the last autotune

    def add(self, w, key=None, m0=None):
        """Create the solve for workload `w` (magnet + group), set its initial
        magnetization and the sensible initial time step for it."""
        eng = self.engine
        s = Solve(key if key is not None else w.get("name"), w)
        g = eng.group_create()
        try:
            p = eng.solver_params(g)
            p.method = self.method
            p.adaptive = 1
            p.max_error = self.max_error
            eng.set_solver_params(g, p)
            keep = []
            d = solve_desc(w, keep)
            s.resident, s.transient = magnet_bytes(d)
            # the magnet with its initial state: the group's time step is then
            # the sensible one for that state
            s.magnet = eng.magnet_add_state(g, d, w["m0"]() if m0 is None else m0)
        except Exception:
            eng.group_destroy(g)
            raise
        s.group = g
        self.solves[g] = s
        self.resident += s.resident
        return s

    def start(self, s, duration, torque_stop=0.0):
        """Arm `s` for `duration` seconds of simulated time, or until
        max|torque|/gamma_LL < torque_stop tesla."""
        s.duration = float(duration)
        s.torque_stop = float(torque_stop)
        s.t_start = float(self.engine.group_info(s.group).time)
        self.engine.group_start(s.group, s.duration, s.torque_stop)

    def advance(self, attempts):
        self.engine.advance(attempts)

    def poll(self):
        """Waits for the queued attempts; returns (finished solves, number running)."""
        done, running = self.engine.poll()
        return [self.solves[g] for g in done], running

    def finish(self, s, fetch=True):
        """Read the outcome (and the final magnetization) of `s`, then free it."""
        info = self.engine.group_info(s.group)
        s.steps = int(info.steps)
        s.rejected = int(info.rejected)
        s.sim_time = float(info.time)
        s.failed = info.status == GS_FAILED
        if fetch:
            s.m = self.engine.get_m(s.magnet, s.shape)
        self.engine.group_destroy(s.group)
        del self.solves[s.group]
        self.resident -= s.resident
        return s


class Checkpoint:
    """A solve taken off the device mid-run: its workload, its group state
    (Engine.group_save) and the simulated time left."""

    __slots__ = ("key", "w", "state", "t_stop", "torque_stop")

    def __init__(self, key, w, state, t_stop, torque_stop):
        self.key, self.w, self.state, self.t_stop, self.torque_stop = key, w, state, t_stop, torque_stop


def checkpoint(batch, s):
    """Save running solve `s` to host memory and free it (preemption).  The
    queued attempts must have been polled."""
    info = batch.engine.group_info(s.group)
    ck = Checkpoint(s.key, s.w, batch.engine.group_save(s.group), s.t_start + s.duration, s.torque_stop)
    s.sim_time = float(info.time)
    batch.engine.group_destroy(s.group)
    del batch.solves[s.group]
    batch.resident -= s.resident
    return ck


def resume(batch, ck):
    """Re-admit a checkpointed solve: a new group with the same magnet, the
    saved state loaded, started for the simulated time it had left.  It then
    continues bit for bit as it would have without the interruption."""
    s = batch.add(ck.w, key=ck.key)
    batch.engine.group_load(s.group, ck.state)
    t = float(batch.engine.group_info(s.group).time)
    s.duration = ck.t_stop - t
    s.t_start = t
    s.torque_stop = ck.torque_stop
    batch.engine.group_start(s.group, s.duration, s.torque_stop)
    return s


class _Pacer:
    """Attempts per poll: enough that the host round trip stays small next to
    the device work, few enough that finished solves leave the tables soon."""

    def __init__(self, target_s=0.004, cap=64):
        self.target = target_s
        self.cap = cap
        self.n = 1

    def update(self, attempts, seconds):
        if attempts > 0 and seconds > 0:
            per = seconds / attempts
            self.n = int(max(1, min(self.cap, self.target / per)))
        return self.n


def relax_batch(batch, instances, duration=2e-9, torque_stop=1e-4, fetch=True, trace=None, autotune=True):
    """Add every instance, start them all, advance until all have finished.
    Returns (solves, seconds of the integration loop, seconds of set-up).
    `trace`, a list, receives (seconds, attempts, solves running, cells
    running) at every poll.  With `autotune` the tile shapes of the started
    batch are chosen by timing after the first attempt (mpx_autotune); they
    hold while the running solves keep more than half of the cells."""
    t0 = time.perf_counter()
    solves = [batch.add(w, key=i) for i, w in enumerate(instances)]
    batch.engine.synchronize()
    t_setup = time.perf_counter() - t0
    for s in solves:
        batch.start(s, duration, torque_stop)
    pacer = _Pacer()
    t0 = time.perf_counter()
    running = len(solves)
    cells = sum(s.cells for s in solves)
    attempts = 0
    if autotune and running > 1:  # one attempt (k0 of every solve), then the tile shapes
        batch.advance(1)
        done, running = batch.poll()
        attempts = 1
        for s in done:
            batch.finish(s, fetch=fetch)
            s.t_done = time.perf_counter() - t0
            cells -= s.cells
        if running:
            batch.tuned = batch.engine.autotune(_abi.RK_NAMES[batch.method])
    while running:
        n = pacer.n
        ta = time.perf_counter()
        batch.advance(n)
        done, running = batch.poll()
        pacer.update(n, time.perf_counter() - ta)
        attempts += n
        for s in done:
            batch.finish(s, fetch=fetch)
            s.t_done = time.perf_counter() - t0
            cells -= s.cells
        if trace is not None:
            trace.append((time.perf_counter() - t0, attempts, running, cells))
    return solves, time.perf_counter() - t0, t_setup


def run_plain(batch, instances, duration=2e-9, torque_stop=1e-4, fetch=True):
    """The same solves one at a time: each is added, run to its end and
    freed before the next is added.  Returns (solves, seconds integrating,
    seconds of set-up)."""
    solves = []
    t_run = t_setup = 0.0
    for i, w in enumerate(instances):
        t0 = time.perf_counter()
        s = batch.add(w, key=i)
        batch.engine.synchronize()
        t1 = time.perf_counter()
        batch.start(s, duration, torque_stop)
        pacer = _Pacer()
        running = 1
        while running:
            n = pacer.n
            ta = time.perf_counter()
            batch.advance(n)
            done, running = batch.poll()
            pacer.update(n, time.perf_counter() - ta)
        batch.finish(s, fetch=fetch)
        t2 = time.perf_counter()
        t_setup += t1 - t0
        t_run += t2 - t1
        solves.append(s)
    return solves, t_run, t_setup


class Server:
    """Continuous batching of an open-loop request stream.

    Requests (workload dicts with `arrival` seconds and `duration`) enter a
    FIFO queue when their arrival time has passed; the head of the queue is
    admitted whenever the resident bytes of the admitted solves plus its own
    resident and transient bytes fit the budget.  Admitted solves keep their
    state on the device and advance together; finished ones return their final
    magnetization to the host and free their memory.  Initial magnetizations
    are generated ahead of arrival on host threads (client-side data)."""

    def __init__(self, batch, budget_bytes, max_active=None, prefetch=32, workers=4, max_cells=None):
        """`max_cells` (optional): admit only while the resident solves hold
        at most this many cells, i.e. bound the device work of one attempt,
        so that under overload the admitted solves keep finishing instead of
        all sharing the device (the memory budget alone admits everything
        that fits)."""
        self.batch = batch
        self.budget = int(budget_bytes)
        self.max_active = max_active
        self.max_cells = max_cells
        self.prefetch = prefetch
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=workers)

    def run(self, requests, torque_stop=0.0, fetch=True, time_limit=None, stats=None):
        """Serve `requests` (sorted by arrival) and return the finished solves,
        each with arrival, t_admit and t_done (seconds since the stream start).
        With `time_limit` (seconds) the loop stops there, requests still queued
        or running unfinished.  `stats`, a dict, receives the counts of
        arrived, admitted and finished requests, the host seconds spent
        admitting (add + start) and advancing (advance + poll), and samples
        (seconds, queued, running) about every 0.5 s."""
        reqs = sorted(enumerate(requests), key=lambda kv: kv[1]["arrival"])
        m0 = {}
        nxt_gen = 0

        def pregen(upto):
            nonlocal nxt_gen
            while nxt_gen < min(upto, len(reqs)):
                k, w = reqs[nxt_gen]
                m0[k] = self.pool.submit(w["m0"])
                nxt_gen += 1

        pregen(self.prefetch)
        queue = collections.deque()
        finished = []
        nxt = 0
        pacer = _Pacer()
        b = self.batch
        admitted = 0
        t_admit = t_adv = 0.0
        samples = []
        t_sample = 0.0
        t0 = time.perf_counter()
        while nxt < len(reqs) or queue or b.solves:
            now = time.perf_counter() - t0
            if now >= t_sample:
                samples.append((round(now, 3), len(queue), len(b.solves)))
                t_sample = now + 0.5
            if time_limit is not None and now > time_limit:
                break
            while nxt < len(reqs) and reqs[nxt][1]["arrival"] <= now:
                queue.append(reqs[nxt])
                nxt += 1
            pregen(nxt + self.prefetch)
            # admission against the memory budget, in arrival order
            while queue:
                k, w = queue[0]
                res, tr = solve_bytes(w)
                if b.resident + res + tr > self.budget and b.solves:
                    break
                if self.max_active is not None and len(b.solves) >= self.max_active:
                    break
                if (self.max_cells is not None and b.solves
                        and sum(x.cells for x in b.solves.values()) + workloads.ncells(w) > self.max_cells):
                    break
                queue.popleft()
                m0k = m0.pop(k).result()
                ta = time.perf_counter()
                s = b.add(w, key=k, m0=m0k)
                s.arrival = w["arrival"]
                s.t_admit = time.perf_counter() - t0
                b.start(s, w["duration"], torque_stop)
                t_admit += time.perf_counter() - ta
                admitted += 1
            if not b.solves:
                if nxt < len(reqs):  # idle until the next arrival
                    time.sleep(max(0.0, reqs[nxt][1]["arrival"] - (time.perf_counter() - t0)))
                continue
            n = pacer.n
            ta = time.perf_counter()
            b.advance(n)
            done, _ = b.poll()
            pacer.update(n, time.perf_counter() - ta)
            t_adv += time.perf_counter() - ta
            for s in done:
                b.finish(s, fetch=fetch)
                s.t_done = time.perf_counter() - t0
                finished.append(s)
        if stats is not None:
            stats.update(arrived=nxt, admitted=admitted, finished=len(finished), still_queued=len(queue),
                         still_running=len(b.solves), host_admit_s=t_admit, host_advance_s=t_adv,
                         wall_s=time.perf_counter() - t0, samples=samples)
        return finished


def shard(instances, rank, world_size):
    """Instances of this rank when independent solves are spread over
    `world_size` GPUs: greedy longest-processing-time bin packing on the cells
    of each solve (the device work of a step is about proportional to them),
    deterministic on every rank.  Returns the instance indices, in order."""
    order = sorted(range(len(instances)), key=lambda i: (-workloads.ncells(instances[i]), i))
    load = [0] * world_size
    owner = [0] * len(instances)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += workloads.ncells(instances[i])
    return [i for i in range(len(instances)) if owner[i] == rank]


def latency_stats(solves):
    """p50 / p99 latency (seconds from arrival to result) of finished solves."""
    lat = np.array([s.t_done - s.arrival for s in solves if s.t_done is not None and s.arrival is not None])
    if lat.size == 0:
        return None, None
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
