"""Thermal noise on the GPU (physics/thermalnoise.cu, core/rungekutta.cpp:94-106):
Boltzmann statistics of independent macrospins, the same noise realisation as
the oracle's restatement of the generator (fixed-step Heun), and reproducibility
from the seed.

Tolerances: <m_z> within 0.02 of the Langevin function (statistical); final m
of a 20-step noisy run vs the oracle <= 1e-4 per cell."""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, random_m
from test_oracle_golden import thermal_macrospins

pytestmark = pytest.mark.gpu
abi = O.abi


def test_thermal_noise_langevin(mpx):
    st = {}

    def run_steps(spec, n):
        if "ts" not in st:
            m0 = np.zeros((3, *spec.shape), np.float32)
            m0[2] = 1.0
            world, magnet = spec.product(mpx, m0)
            ts = world.timesolver
            ts.set_method("Heun")
            ts.adaptive_timestep = False
            ts.timestep = 2e-13
            st.update(ts=ts, magnet=magnet)
        st["ts"].steps(n)

    got, want = thermal_macrospins(run_steps, lambda: st["magnet"].magnetization.average()[2])
    assert abs(got - want) < 0.02, (got, want)


def _noisy_film(seed=77):
    return MagnetSpec(size=(24, 12, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.1,
                      temperature=300.0, thermal_seed=seed, world_bias=(0.0, 0.0, 0.05))


def test_thermal_noise_matches_oracle_realisation(mpx):
    s = _noisy_film()
    m0 = random_m(s.shape, seed=8, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_solver(method=abi.RK_METHODS["Heun"], adaptive=0)
    ow.timestep = 5e-14
    world, magnet = s.product(mpx, m0)
    ts = world.timesolver
    ts.set_method("Heun")
    ts.adaptive_timestep = False
    ts.timestep = 5e-14
    ow.steps(20)
    ts.steps(20)
    got = magnet.magnetization.get()
    want = ow.get_m(q)
    assert float(np.max(np.abs(got - want))) < 1e-4


def test_thermal_noise_seeded_dormand_prince(mpx):
    """Adaptive Dormand-Prince with noise (k0 is not reused): the same seed gives
    the same run, another seed another one."""
    finals = []
    for seed in (5, 5, 6):
        s = _noisy_film(seed)
        world, magnet = s.product(mpx, random_m(s.shape, seed=8, smooth=3))
        ts = world.timesolver
        ts.set_method("DormandPrince")
        ts.run(20e-12)
        finals.append(magnet.magnetization.get())
    assert np.array_equal(finals[0], finals[1])
    assert not np.array_equal(finals[0], finals[2])
