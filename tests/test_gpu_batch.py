"""Batched and served forms on the GPU: a solve gives the same result alone, in
a batch, and admitted mid-run into a served stream; the relaxation stop and
the memory estimate behave; a batch solve follows the FP64 oracle.

Tolerance: final m of a solve in a mix vs alone <= 1e-6 absolute (the
batched form's parity bound is 1e-5; the arithmetic is the same per magnet,
so the results are expected to agree bit for bit).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
GAMMALL = 1.7595e11

MIX_TOL = 1e-6


def _solve(k, size, cell, msat, aex, alpha, bias, dmi=0.0, duration=20e-12, arrival=0.0):
    from mumaxplus_b200 import workloads as W

    nx, ny, nz = size
    return dict(name=f"s{k}", size=size, cellsize=(cell, cell, cell), msat=msat, aex=aex, alpha=alpha,
                world_bias=bias, dmi={"xxz": dmi, "yyz": dmi} if dmi else {}, duration=duration,
                arrival=arrival, m0=(lambda s=(nz, ny, nx), seed=100 + k: W.smoothed_random_m(s, seed)))


def _mix():
    return [
        _solve(0, (48, 40, 1), 3e-9, 8e5, 1.3e-11, 0.1, (0.02, 0.0, 0.05)),
        _solve(1, (64, 64, 2), 2.5e-9, 6e5, 1.0e-11, 0.3, (0.0, 0.03, 0.0), dmi=2e-3),
        _solve(2, (32, 24, 1), 4e-9, 1e6, 2.0e-11, 0.02, (0.0, 0.0, -0.08)),
        _solve(3, (100, 36, 2), 2e-9, 5e5, 8e-12, 0.5, (0.05, 0.05, 0.0)),
    ]


def test_batch_results_match_plain(mpx):
    from mumaxplus_b200 import batch as B

    sols = _mix()
    plain, _, _ = B.run_plain(B.Batch(), sols, duration=20e-12, torque_stop=0.0)
    mixed, _, _ = B.relax_batch(B.Batch(), sols, duration=20e-12, torque_stop=0.0)
    for p, q in zip(plain, mixed):
        assert p.steps == q.steps and p.steps > 0
        assert not p.failed and not q.failed
        assert q.sim_time == pytest.approx(20e-12, rel=1e-12)
        diff = float(np.max(np.abs(p.m - q.m)))
        assert diff <= MIX_TOL, f"solve {p.key}: |dm| {diff:.3e}"


def test_batch_with_2048_point_rows_matches_plain(mpx):
    """A batch holding a solve with 2048-point x rows launches the x passes in
    their warp-pair forms for every solve; each solve still gives the result it
    gives alone (where only that one takes those forms)."""
    from mumaxplus_b200 import batch as B

    sols = _mix() + [_solve(4, (600, 16, 1), 2e-9, 8e5, 1.3e-11, 0.1, (0.0, 0.02, 0.05))]
    plain, _, _ = B.run_plain(B.Batch(), sols, duration=10e-12, torque_stop=0.0)
    mixed, _, _ = B.relax_batch(B.Batch(), sols, duration=10e-12, torque_stop=0.0)
    for p, q in zip(plain, mixed):
        assert p.steps == q.steps and p.steps > 0
        assert not p.failed and not q.failed
        diff = float(np.max(np.abs(p.m - q.m)))
        assert diff <= MIX_TOL, f"solve {p.key}: |dm| {diff:.3e}"


def test_relaxation_stops_on_torque(mpx):
    from mumaxplus_b200 import batch as B

    w = _solve(0, (32, 32, 1), 3e-9, 8e5, 1.3e-11, 0.5, (0.0, 0.0, 0.1))
    (s,), _, _ = B.relax_batch(B.Batch(), [w], duration=2e-9, torque_stop=2e-2)
    assert 0 < s.sim_time < 2e-9
    # the stop criterion holds for the returned state (FP64 torque of the FP32 state)
    keep = []
    ow = O.OracleWorld()
    q = ow.add_magnet(B.solve_desc(w, keep))
    ow.set_m(q, s.m)
    tau = ow.eval(q, O.abi.Q_TORQUE)
    assert np.max(np.linalg.norm(tau, axis=0)) / GAMMALL < 2e-2 * 1.001


def test_served_stream_matches_plain(mpx):
    """Requests arriving while others run are admitted as memory frees up; each
    result equals the same request run alone."""
    from mumaxplus_b200 import batch as B

    reqs = [dict(r, arrival=0.01 * i, duration=(8 + 4 * i) * 1e-12) for i, r in enumerate(_mix() * 2)]
    for i, r in enumerate(reqs):
        r["name"] = f"r{i}"
    res = [B.solve_bytes(r) for r in reqs]
    budget = int(2.2 * max(a + b for a, b in res))  # about two solves resident at a time
    served = B.Server(B.Batch(), budget).run(reqs)
    assert sorted(s.key for s in served) == list(range(len(reqs)))
    assert all(s.t_done >= s.t_admit >= s.arrival - 1e-9 for s in served)
    p50, p99 = B.latency_stats(served)
    assert 0 < p50 <= p99
    by_key = {s.key: s for s in served}
    for i, r in enumerate(reqs):
        (p,), _, _ = B.run_plain(B.Batch(), [r], duration=r["duration"], torque_stop=0.0)
        s = by_key[i]
        assert s.steps == p.steps
        assert float(np.max(np.abs(s.m - p.m))) <= MIX_TOL


def test_magnet_bytes_matches_engine_accounting(mpx):
    from mumaxplus_b200 import batch as B

    b = B.Batch()
    w = _mix()[1]
    before = b.engine.memory()
    s = b.add(w)
    grown = b.engine.memory() - before
    # the estimate also counts the small work tables, which the engine tallies apart
    assert grown <= s.resident <= grown + 64 * 1024
    b.finish(s, fetch=False)
    assert b.engine.memory() == before


def test_batch_solve_follows_oracle(mpx):
    """One solve of a batch against the FP64 oracle's Dormand-Prince run."""
    from mumaxplus_b200 import batch as B

    sols = _mix()[:3]
    mixed, _, _ = B.relax_batch(B.Batch(), sols, duration=10e-12, torque_stop=0.0)
    for w, got in zip(sols, mixed):
        keep = []
        ow = O.OracleWorld()
        q = ow.add_magnet(B.solve_desc(w, keep))
        ow.set_m(q, w["m0"]())
        ow.set_method("DormandPrince")
        ow.timestep = ow.sensible_timestep()
        ow.run(10e-12)
        want = ow.get_m(q)
        assert float(np.max(np.abs(got.m - want))) < 1e-4, w["name"]


def test_same_result_with_small_and_large_tiles(mpx):
    """Alone, a small solve runs with small tiles (the shape planner spreads it
    over the GPU); in a large batch with the default large tiles.  Tiles start
    on even rows, so the arithmetic and the result are the same."""
    from mumaxplus_b200 import batch as B

    w = _solve(7, (64, 30, 1), 3e-9, 8e5, 1.3e-11, 0.1, (0.02, 0.0, 0.05))
    fill = [_solve(10 + k, (128, 96, 2), 3e-9, 7e5, 1.2e-11, 0.2, (0.0, 0.01, 0.02)) for k in range(30)]
    (alone,), _, _ = B.run_plain(B.Batch(), [w], duration=15e-12, torque_stop=0.0)
    mixed, _, _ = B.relax_batch(B.Batch(), [w] + fill, duration=15e-12, torque_stop=0.0)
    assert alone.steps == mixed[0].steps
    assert np.array_equal(alone.m, mixed[0].m)


def test_membership_changes_update_the_attempt_graph(mpx):
    """A solve that starts or finishes while others run changes only the launch
    sizes and tables of the attempt: the captured graphs are updated in place
    (no new instantiation), and the solves give the same results as without
    the change."""
    from mumaxplus_b200 import batch as B

    sols = [_solve(10 + k, (40, 32, 1), 3e-9, 8e5, 1.3e-11, 0.1, (0.02, 0.0, 0.05), duration=1e-6) for k in range(3)]
    ref = B.Batch()
    rs = [ref.add(w, key=i) for i, w in enumerate(sols)]
    for s in rs:
        ref.start(s, 1e-6)
    ref.advance(20)
    ref.poll()
    want = ref.engine.get_m(rs[0].magnet, rs[0].shape)

    b = B.Batch()
    ss = [b.add(w, key=i) for i, w in enumerate(sols)]
    b.start(ss[0], 1e-6)
    b.start(ss[1], 1e-6)
    b.advance(8)
    b.poll()
    inst0, upd0 = b.engine.graph_stats()
    b.start(ss[2], 1e-6)  # a new solve of the same shape class joins
    b.advance(12)
    b.poll()
    inst1, upd1 = b.engine.graph_stats()
    assert inst1 == inst0 and upd1 > upd0, (inst0, upd0, inst1, upd1)
    np.testing.assert_array_equal(b.engine.get_m(ss[0].magnet, ss[0].shape), want)


def test_launch_tables_keep_places_through_churn(mpx):
    """Many short solves finishing while others arrive: the launch tables
    leave holes for the finished ones, append the newcomers and compact when
    the holes outnumber the live entries; every solve still ends as it does
    alone (bit for bit)."""
    from mumaxplus_b200 import batch as B

    sols = [_solve(20 + k, (48 + 16 * (k % 3), 32, 1 + (k % 2)), 3e-9, 8e5, 1.3e-11, 0.2, (0.01, 0.02, 0.03),
                   duration=(2 + (k % 5)) * 1e-12) for k in range(24)]
    alone = {}
    for k in (0, 7, 13, 23):
        b1 = B.Batch()
        s = b1.add(sols[k], key=k)
        b1.start(s, sols[k]["duration"])
        while True:
            b1.advance(4)
            done, running = b1.poll()
            if running == 0:
                break
        alone[k] = b1.engine.get_m(s.magnet, s.shape)
    b = B.Batch()
    live, got = {}, {}
    nxt = 0
    while nxt < len(sols) or live:
        while nxt < len(sols) and len(live) < 6:  # a few resident at a time: arrivals and completions interleave
            s = b.add(sols[nxt], key=nxt)
            b.start(s, sols[nxt]["duration"])
            live[s.group] = s
            nxt += 1
        b.advance(3)
        done, _ = b.poll()
        for s in done:
            if s.key in alone:
                got[s.key] = b.engine.get_m(s.magnet, s.shape)
            b.finish(s, fetch=False)
            live.pop(s.group)
    for k, want in alone.items():
        np.testing.assert_array_equal(got[k], want)
