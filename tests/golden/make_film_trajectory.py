#!/usr/bin/env python
"""Writes tests/golden/film_256x64_dp_1ns.json: the FP64 oracle's <m>(t) of
the 256x64x1 film (3 nm cells, Ms 8.6e5 A/m, A 1.3e-11 J/m, alpha 0.02, open
boundaries, B_ext = (-30, 5, 0) mT, exchange + demag + Zeeman; m0 seeded
Gaussian vectors smoothed by 3 Jacobi passes and normalised), Dormand-Prince
with max error 1e-5 from the sensible time step, sampled every 10 ps over
1 ns.  The trajectory takes minutes on the CPU, so the GPU test compares
against this file instead of rerunning the oracle.

The film's dynamics (alpha 0.02, a random smoothed start) is chaotic: the
file also holds the oracle's trajectory from the same m0 with every value
changed by one float32 ulp (seeded signs).  Its distance to the unperturbed
one is the sensitivity of the problem itself, which any FP32 computation
(this library's, the reference's SINGLE build) meets at least.

    python tests/golden/make_film_trajectory.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from mumaxplus_b200 import workloads as W  # noqa: E402

OUT = os.path.join(HERE, "film_256x64_dp_1ns.json")


def trajectory(w, m0, dt0=None):
    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w["world_bias"])
    q = ow.add_magnet(W.desc(w, keep))
    ow.set_m(q, m0)
    ow.set_method("DormandPrince")
    ow.timestep = ow.sensible_timestep() if dt0 is None else dt0
    dt0 = ow.timestep
    times, avgs = [0.0], [[float(v) for v in ow.average(q, O.abi.Q_MAGNETIZATION)]]
    for k in range(1, 101):
        tp = k * 10e-12
        ow.run(tp - ow.time)
        times.append(ow.time)
        avgs.append([float(v) for v in ow.average(q, O.abi.Q_MAGNETIZATION)])
    return times, avgs, dt0, ow.counters()


def main():
    w = W.film()
    m0 = w["m0"]()
    t0 = time.time()
    times, avgs, dt0, counters = trajectory(w, m0)
    rng = np.random.default_rng(99)
    m1 = (m0 * (1 + 2.0 ** -23 * rng.choice([-1, 1], size=m0.shape))).astype(np.float32)
    _, avgs1, _, _ = trajectory(w, m1, dt0)
    out = {
        "_about": "FP64 oracle <m>(t) of the 256x64x1 film workload (mumaxplus_b200.workloads.film), "
                  "Dormand-Prince, max error 1e-5, every 10 ps over 1 ns; made by make_film_trajectory.py",
        "workload": w["name"],
        "method": "DormandPrince",
        "max_error": 1e-5,
        "initial_timestep": dt0,
        "m0_sha": __import__("hashlib").sha256(m0.tobytes()).hexdigest()[:16],
        "counters": {k: int(v) for k, v in counters.items()},
        "seconds": time.time() - t0,
        "time": times,
        "m": avgs,
        "m_ulp_perturbed": avgs1,
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT}: {len(times)} points, {out['seconds']:.0f} s, counters {out['counters']}")


if __name__ == "__main__":
    main()
