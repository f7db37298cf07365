"""Checkpoint / resume of the time integration (mpx_group_save / mpx_group_load):
a run continued from a saved state, in the same world, in a fresh world, with
thermal noise, and a batch solve taken off the device and re-admitted, all
continue bit for bit as the uninterrupted run (compared exactly)."""
import numpy as np
import pytest

from test_gpu_batch import _mix

pytestmark = pytest.mark.gpu


def _film(mpx, temperature=0.0):
    world = mpx.World(cellsize=(3e-9, 3e-9, 3e-9))
    magnet = mpx.Ferromagnet(world, mpx.Grid((64, 32, 1)))
    magnet.msat, magnet.aex, magnet.alpha = 8e5, 1.3e-11, 0.05
    if temperature:
        magnet.temperature = temperature
        magnet.thermal_seed = 1234
    rng = np.random.default_rng(9)
    m0 = rng.standard_normal((3, 1, 32, 64)).astype(np.float32)
    m0[2] += 1.5
    magnet.magnetization = m0
    world.bias_magnetic_field = (0.0, 0.01, 0.02)
    world.timesolver.set_method("DormandPrince")
    return world, magnet


@pytest.mark.parametrize("temperature", [0.0, 50.0])
def test_save_load_continues_exactly(mpx, temperature):
    world, magnet = _film(mpx, temperature)
    world.timesolver.steps(5)
    state = world.save_state()
    world.timesolver.steps(7)
    want = magnet.magnetization.get()
    t_want, dt_want = world.timesolver.time, world.timesolver.timestep

    world.load_state(state)  # the same world, rewound
    world.timesolver.steps(7)
    np.testing.assert_array_equal(magnet.magnetization.get(), want)
    assert world.timesolver.time == t_want and world.timesolver.timestep == dt_want

    world2, magnet2 = _film(mpx, temperature)  # a fresh world with a magnet of the same size
    world2.load_state(state)
    world2.timesolver.steps(7)
    np.testing.assert_array_equal(magnet2.magnetization.get(), want)
    assert world2.timesolver.time == t_want


def test_load_rejects_a_state_of_other_magnets(mpx):
    world, _ = _film(mpx)
    state = world.save_state()
    other = mpx.World(cellsize=(3e-9, 3e-9, 3e-9))
    mpx.Ferromagnet(other, mpx.Grid((32, 32, 1)))
    with pytest.raises(ValueError):
        other.load_state(state)
    with pytest.raises(ValueError):
        world.load_state(state[:16])


def test_batch_solve_preempted_and_resumed(mpx):
    from mumaxplus_b200 import batch as B

    sols = _mix()[:2]
    duration = 1e-6  # not reached: both runs stop after the same number of attempts

    ref = B.Batch()
    rs = [ref.add(w, key=i) for i, w in enumerate(sols)]
    for s in rs:
        ref.start(s, duration)
    ref.advance(30)
    ref.poll()
    want = ref.engine.get_m(rs[0].magnet, rs[0].shape)

    b = B.Batch()
    ss = [b.add(w, key=i) for i, w in enumerate(sols)]
    for s in ss:
        b.start(s, duration)
    b.advance(12)
    b.poll()
    ck = B.checkpoint(b, ss[0])  # off the device; the other solve keeps running
    b.advance(9)
    b.poll()
    s0 = B.resume(b, ck)
    b.advance(18)
    b.poll()
    np.testing.assert_array_equal(b.engine.get_m(s0.magnet, s0.shape), want)
    assert b.engine.group_info(s0.group).time == ref.engine.group_info(rs[0].group).time


def test_load_refused_while_running_and_clean_after_a_run(mpx):
    """A group in the middle of a started run refuses a state (its controller
    state belongs to that run); after run() has finished, a loaded state
    continues exactly like the uninterrupted run (the final-step phase of the
    earlier run does not carry over)."""
    from mumaxplus_b200 import batch as B

    sols = _mix()[:1]
    b = B.Batch()
    s = b.add(sols[0], key=0)
    state0 = b.engine.group_save(s.group)
    b.start(s, 1e-6)
    b.advance(3)
    b.poll()
    with pytest.raises(ValueError):
        b.engine.group_load(s.group, state0)

    world, magnet = _film(mpx)
    world.timesolver.steps(4)
    state = world.save_state()
    world.timesolver.steps(6)
    want = magnet.magnetization.get()
    t_want = world.timesolver.time
    world.load_state(state)
    world.timesolver.run(3.7e-12)  # ends with a shortened final step
    world.load_state(state)
    world.timesolver.steps(6)
    np.testing.assert_array_equal(magnet.magnetization.get(), want)
    assert world.timesolver.time == t_want
