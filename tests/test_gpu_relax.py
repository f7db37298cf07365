"""minimize() and relax() on the GPU: the reference's standard problem 2
coercivity known answer through the mumaxplus-style API, and the final states
against the FP64 oracle's restatement of physics/minimizer.cu and
physics/relaxer.cpp.

Tolerances: coercive field 1e-5 (the reference test's); final magnetization of
a single-domain minimum <= 1e-4 per cell (FP32 vs FP64 descent paths to the same
minimum, both stopped at changes of 1e-6 per step or at a relaxed torque)."""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec
from test_oracle_golden import check_nanowire, nanowire_canting, sp2_coercivity

pytestmark = pytest.mark.gpu
abi = O.abi


def test_minimize_sp2_coercivity(mpx):
    st = {}

    def make(cs, msat, aex):
        world = mpx.World(cellsize=cs)
        magnet = mpx.Ferromagnet(world, mpx.Grid((1, 1, 1)))
        magnet.msat = msat
        magnet.aex = aex
        magnet.magnetization = (1, 1, 1)
        st.update(world=world, magnet=magnet)

    def set_field(b):
        st["world"].bias_magnetic_field = tuple(float(v) for v in b)

    rhc = sp2_coercivity(make, lambda: st["magnet"].minimize(), set_field,
                         lambda: float(np.sum(st["magnet"].magnetization.average())))
    assert abs(0.057069478 - rhc) < 1e-5, rhc


def test_minimize_nanowire_canting_golden(mpx):
    """test/test_boundaries.py through the mumaxplus-style API: Neumann canting vs the mumax3 value, open
    boundaries vs the analytic and the mumax3 value (tests/golden/known_answers.json, 2e-4)."""
    cs, D = 0.05, 0.9 * 4 / np.pi
    st = {}

    def make(openbc, m0):
        world = mpx.World(cellsize=(cs, cs, cs))
        magnet = mpx.Ferromagnet(world, mpx.Grid((1024, 1, 1)))
        magnet.dmi_tensor.set_interfacial_dmi(D)
        magnet.enable_demag = False
        magnet.enable_openbc = openbc
        magnet.anisU = (0, 0, 1)
        magnet.aex = 1.0
        magnet.ku1 = 1.0
        magnet.msat = 1.0
        magnet.magnetization = m0
        st.update(magnet=magnet, world=world)
        return lambda: magnet.magnetization.eval()

    check_nanowire(*nanowire_canting(lambda: st["magnet"].minimize(1e-7), None, make))


def _film():
    s = MagnetSpec(size=(24, 16, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.1, ku1=2e5,
                   anisU=(1.0, 0.2, 0.0), world_bias=(0.01, 0.02, 0.0))
    rng = np.random.default_rng(7)
    m0 = np.zeros((3, 1, 16, 24), np.float32)
    m0[0], m0[1], m0[2] = 0.5, 0.7, 0.5
    m0 += 0.05 * rng.standard_normal(m0.shape).astype(np.float32)
    return s, m0


def test_minimize_matches_oracle(mpx):
    s, m0 = _film()
    ow, q = s.oracle_world(m0)
    ow.minimize(1e-6, 10)
    world, magnet = s.product(mpx, m0)
    magnet.minimize(1e-6, 10)
    got = magnet.magnetization.get()
    want = ow.get_m(q)
    assert float(np.max(np.abs(got - want))) < 1e-4


def test_relax_matches_oracle_and_restores_solver(mpx):
    s, m0 = _film()
    ow, q = s.oracle_world(m0)
    ow.relax(1e-9)
    world, magnet = s.product(mpx, m0)
    ts = world.timesolver
    ts.set_method("DormandPrince")
    ts.time = 2e-12
    dt_before = ts.timestep
    magnet.relax(1e-9)
    got = magnet.magnetization.get()
    want = ow.get_m(q)
    assert float(np.max(np.abs(got - want))) < 1e-4
    assert ts.time == 2e-12
    assert ts.method == "DormandPrince"
    assert ts.timestep > 0 and dt_before > 0


def test_relax_with_torque_threshold(mpx):
    s, m0 = _film()
    world, magnet = s.product(mpx, m0)
    magnet.RelaxTorqueThreshold = 1e7
    magnet.relax(1e-6)
    tau = magnet._engine.max_norm(magnet._id, abi.Q_DAMPING_TORQUE)
    assert tau <= 1e7
    with pytest.raises(AssertionError):
        magnet.RelaxTorqueThreshold = 0
