"""Stray fields between the magnets of one world on the GPU
(physics/zeeman.cu:70-88) against the FP64 oracle: fields of each magnet,
the source / destination switches, and a two-magnet trajectory.

Tolerances: fields |dB|max / |B|max <= 1e-5; <m>(t) <= 1e-4."""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, max_rel, random_m

pytestmark = pytest.mark.gpu
abi = O.abi
CS = (2e-9, 3e-9, 2.5e-9)


def _specs(dst_on=True, src_on=True):
    A = MagnetSpec(size=(24, 10, 2), cellsize=CS, msat=8e5, aex=1.1e-11, alpha=0.2, stray_source=src_on)
    B = MagnetSpec(size=(16, 12, 2), origin=(28, 3, 0), cellsize=CS, msat=6e5, aex=1.3e-11, alpha=0.1,
                   stray_destination=dst_on)
    return A, B


def _oracle(specs, ms, bias=(0.0, 0.0, 0.0)):
    ow = O.OracleWorld()
    ow.set_world_bias(bias)
    keep = []
    qs = [ow.add_magnet(s.desc(keep)) for s in specs]
    for q, m in zip(qs, ms):
        ow.set_m(q, m)
    return ow, qs


def _product(mpx, specs, ms, bias=(0.0, 0.0, 0.0)):
    world = mpx.World(CS)
    mags = []
    for s, m in zip(specs, ms):
        mag = mpx.Ferromagnet(world, mpx.Grid(s.size, s.origin))
        mag._suspend = True
        mag.msat, mag.aex, mag.alpha = s.msat, s.aex, s.alpha
        mag.enable_as_stray_field_source = s.stray_source
        mag.enable_as_stray_field_destination = s.stray_destination
        mag._suspend = False
        mag._update()
        mag.magnetization = m
        mags.append(mag)
    if any(bias):
        world.bias_magnetic_field = bias
    return world, mags


@pytest.mark.parametrize("switches", [(True, True), (False, True), (True, False)])
def test_two_magnet_fields(mpx, switches):
    specs = _specs(*switches)
    ms = [random_m(s.shape, seed=20 + k, smooth=2) for k, s in enumerate(specs)]
    ow, qs = _oracle(specs, ms)
    world, mags = _product(mpx, specs, ms)
    for q, mag, s in zip(qs, mags, specs):
        for quantity in (abi.Q_EXTERNAL_FIELD, abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE):
            want = ow.eval(q, quantity)
            got = mag._engine.eval(mag._id, quantity, (3, *s.shape))
            if np.max(np.abs(want)) == 0:
                assert np.max(np.abs(got)) == 0
                continue
            assert max_rel(got, want) < 1e-5, (quantity, max_rel(got, want))


def test_two_magnet_trajectory(mpx):
    specs = _specs()
    ms = [random_m(s.shape, seed=30 + k, smooth=3) for k, s in enumerate(specs)]
    bias = (0.0, 0.02, 0.01)
    ow, qs = _oracle(specs, ms, bias)
    ow.set_method("DormandPrince")
    world, mags = _product(mpx, specs, ms, bias)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = 0.0
    for k in range(1, 5):
        tp = k * 5e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        for q, mag in zip(qs, mags):
            a = np.array(mag.magnetization.average())
            b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
            worst = max(worst, float(np.max(np.abs(a - b))))
    assert worst < 1e-4, worst


def _large_specs(dz=0):
    A = MagnetSpec(size=(48, 24, 2), cellsize=CS, msat=8e5, aex=1.1e-11, alpha=0.2)
    B = MagnetSpec(size=(48, 20, 2), origin=(52, 6, dz), cellsize=CS, msat=6e5, aex=1.3e-11, alpha=0.1)
    return A, B


@pytest.mark.parametrize("dz", [0, 3])
def test_large_pair_fft_form(mpx, dz):
    """Pairs of at least 2^22 cell interactions take the FFT form (a helper magnet spanning both, its demag field
    at the destination cells): fields of both magnets against the oracle's direct sum."""
    specs = _large_specs(dz)
    assert specs[0].shape[0] * specs[0].shape[1] * specs[0].shape[2] * \
        specs[1].shape[0] * specs[1].shape[1] * specs[1].shape[2] >= 1 << 22
    ms = [random_m(s.shape, seed=40 + k, smooth=2) for k, s in enumerate(specs)]
    ow, qs = _oracle(specs, ms)
    world, mags = _product(mpx, specs, ms)
    for q, mag, s in zip(qs, mags, specs):
        for quantity in (abi.Q_EXTERNAL_FIELD, abi.Q_EFFECTIVE_FIELD):
            want = ow.eval(q, quantity)
            got = mag._engine.eval(mag._id, quantity, (3, *s.shape))
            assert max_rel(got, want) < 1e-5, (quantity, max_rel(got, want))


def test_large_pair_fft_form_trajectory(mpx):
    specs = _large_specs(1)
    ms = [random_m(s.shape, seed=50 + k, smooth=3) for k, s in enumerate(specs)]
    ow, qs = _oracle(specs, ms)
    ow.set_method("DormandPrince")
    world, mags = _product(mpx, specs, ms)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = 0.0
    for k in range(1, 3):
        tp = k * 1.5e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        for q, mag in zip(qs, mags):
            worst = max(worst, float(np.max(np.abs(np.array(mag.magnetization.average())
                                                    - np.array(ow.average(q, abi.Q_MAGNETIZATION))))))
    assert worst < 1e-5, worst
