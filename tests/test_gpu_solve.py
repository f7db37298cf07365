"""TimeSolver.solve with the device-sampled output table (the loop of
mumaxplus/timesolver.py:114-152 for average magnetizations) against the same
loop on the host (quantities given as lambdas take the host path: run() to each
time point, then an average per point).

Both paths run the same attempts and the same reduction, so the tables must be
identical: times and averages compared exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _film(mpx, origin2=None, seed=3):
    world = mpx.World(cellsize=(3e-9, 3e-9, 3e-9))
    mags = []
    shapes = [((48, 24, 1), (0, 0, 0))]
    if origin2 is not None:
        shapes.append(((32, 16, 1), origin2))
    rng = np.random.default_rng(seed)
    for k, (size, origin) in enumerate(shapes):
        mag = mpx.Ferromagnet(world, mpx.Grid(size, origin), name=f"m{k}")
        mag.msat, mag.aex, mag.alpha = 8e5, 1.3e-11, 0.05
        m0 = rng.standard_normal((3, size[2], size[1], size[0])).astype(np.float32)
        m0[2] += 2.0
        mag.magnetization = m0
        mags.append(mag)
    world.bias_magnetic_field = (0.0, 0.02, 0.01)
    world.timesolver.set_method("DormandPrince")
    return world, mags


def _both(mpx, times, origin2=None):
    w1, m1 = _film(mpx, origin2)
    dev = w1.timesolver.solve(times, {f"m{k}": m.magnetization.average for k, m in enumerate(m1)})
    assert w1.timesolver._magnetization_columns({"m": m1[0].magnetization.average}) is not None
    w2, m2 = _film(mpx, origin2)
    host = w2.timesolver.solve(times, {f"m{k}": (lambda m=m: m.magnetization.average()) for k, m in enumerate(m2)})
    assert w2.timesolver._magnetization_columns({"m": lambda: 0}) is None
    return dev, host, (w1, m1), (w2, m2)


def test_sampled_solve_matches_host_loop(mpx):
    times = np.linspace(0.0, 60e-12, 13)
    dev, host, (w1, m1), (w2, m2) = _both(mpx, times)
    assert dev["time"] == host["time"]
    assert dev["m0"] == host["m0"]
    assert abs(dev["time"][-1] - 60e-12) < 1e-24
    assert w1.timesolver.time == w2.timesolver.time
    np.testing.assert_array_equal(m1[0].magnetization.get(), m2[0].magnetization.get())
    # the state moved: the samples are not all the same
    assert np.ptp(np.array(dev["m0"])[:, 0]) > 1e-4


def test_sampled_solve_two_magnets_repeated_points(mpx):
    times = [0.0, 0.0, 5e-12, 5e-12, 17e-12, 40e-12]
    dev, host, _, _ = _both(mpx, times, origin2=(60, 4, 0))
    assert dev["time"] == host["time"]
    assert dev["m0"] == host["m0"]
    assert dev["m1"] == host["m1"]
    assert dev["m0"][0] == dev["m0"][1] and dev["m0"][2] == dev["m0"][3]


def test_sampled_solve_continues_like_run(mpx):
    """After a sampled solve the solver state (time, time step, FSAL k0) is the
    one the host loop leaves: further steps agree exactly."""
    times = np.linspace(1e-12, 20e-12, 5)
    _, _, (w1, m1), (w2, m2) = _both(mpx, times)
    assert w1.timesolver.timestep == w2.timesolver.timestep
    w1.timesolver.steps(5)
    w2.timesolver.steps(5)
    np.testing.assert_array_equal(m1[0].magnetization.get(), m2[0].magnetization.get())


def test_run_sampled_rejects_decreasing_points(mpx):
    w, m = _film(mpx)
    with pytest.raises(ValueError):
        w._engine.run_sampled(w._group, [2e-12, 1e-12], 1)
