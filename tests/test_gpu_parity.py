"""GPU parity: the sm_100a engine (through the mumaxplus-style Python API and the
C ABI) against the CPU FP64 oracle on identical seeded float32 inputs.

Tolerances: fields |dB|max / |B|max <= 1e-5 (the FP32 bound stated for B_eff);
<m>(t) trajectories <= 1e-4 absolute; the analytic macrospin test keeps the
reference's own 1e-4 (test/test_timesolver.py:120-122).
"""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, max_rel, random_m

abi = O.abi
pytestmark = pytest.mark.gpu
GAMMALL = 1.7595e11

FIELD_TOL = 1e-5

LOCAL_QUANTITIES = [abi.Q_EXCHANGE_FIELD, abi.Q_DMI_FIELD, abi.Q_ANISOTROPY_FIELD, abi.Q_EXTERNAL_FIELD]


def compare(spec, mpx, quantities, seed=1, smooth=2, tol=FIELD_TOL):
    m0 = random_m(spec.shape, seed=seed, smooth=smooth)
    ow, q = spec.oracle_world(m0)
    world, magnet = spec.product(mpx, m0)
    eng = magnet._engine
    worst = {}
    for quantity in quantities:
        nc = 1 if abi.Q_EXCHANGE_ENERGY_DENSITY <= quantity <= abi.Q_TOTAL_ENERGY_DENSITY else 3
        got = eng.eval(magnet._id, quantity, (nc, *spec.shape))
        want = ow.eval(q, quantity)
        if np.max(np.abs(want)) == 0:
            assert np.max(np.abs(got)) == 0, f"quantity {quantity} should be zero"
            continue
        err = max_rel(got, want)
        worst[quantity] = err
        assert err < tol, f"quantity {quantity}: rel err {err:.3e}"
    return worst


def test_library_loads_and_sees_device(mpx):
    lib = mpx._abi.load()
    assert lib.mpx_device_count() >= 1


def test_exchange_neumann(mpx):
    compare(MagnetSpec(size=(16, 16, 4), cellsize=(1e-9, 2e-9, 3e-9), aex=1.3e-11, msat=8e5, enable_demag=False),
            mpx, [abi.Q_EXCHANGE_FIELD])


def test_exchange_openbc_and_pbc_wrap(mpx):
    s = MagnetSpec(size=(24, 12, 3), cellsize=(2e-9, 2e-9, 1e-9), aex=1.5e-11, msat=5.8e5,
                   mastergrid_size=(24, 12, 0), pbc=(1, 1, 0), enable_demag=False)
    compare(s, mpx, [abi.Q_EXCHANGE_FIELD])
    s.enable_openbc = True
    compare(s, mpx, [abi.Q_EXCHANGE_FIELD])


def test_exchange_mastergrid_larger_than_grid(mpx):
    # wrapped neighbours that land outside the magnet take the Neumann ghost
    s = MagnetSpec(size=(10, 8, 2), origin=(3, 2, 0), cellsize=(1e-9, 1e-9, 1e-9), aex=1e-11, msat=6e5,
                   mastergrid_size=(14, 8, 0), mastergrid_origin=(1, 2, 0), pbc=(1, 1, 0),
                   dmi={"xxz": 2e-3, "yyz": 2e-3}, enable_demag=False)
    compare(s, mpx, [abi.Q_EXCHANGE_FIELD, abi.Q_DMI_FIELD])


@pytest.mark.parametrize("openbc", [False, True])
def test_interfacial_dmi(mpx, openbc):
    s = MagnetSpec(size=(20, 12, 3), cellsize=(1.1e-9, 2e-9, 3.2e-9), msat=6e5, aex=1e-11,
                   dmi={"xxz": 3e-3, "yyz": 3e-3}, enable_openbc=openbc, enable_demag=False)
    compare(s, mpx, [abi.Q_DMI_FIELD, abi.Q_EXCHANGE_FIELD])


def test_general_dmi_tensor_per_cell(mpx):
    shape = (3, 9, 13)
    rng = np.random.default_rng(4)
    dmi = {k: (rng.uniform(0.5e-3, 3e-3, shape).astype(np.float32) if i % 2 == 0 else float(rng.uniform(-2e-3, 2e-3)))
           for i, k in enumerate(abi.DMI_ORDER)}
    s = MagnetSpec(size=(13, 9, 3), cellsize=(1e-9, 1.5e-9, 2e-9), msat=7e5, aex=1.2e-11, dmi=dmi,
                   enable_demag=False)
    compare(s, mpx, [abi.Q_DMI_FIELD, abi.Q_EXCHANGE_FIELD])


def test_anisotropy_zeeman_per_cell(mpx):
    shape = (2, 6, 10)
    rng = np.random.default_rng(5)
    u = rng.standard_normal((3, *shape)).astype(np.float32)
    bias = (rng.standard_normal((3, *shape)) * 0.05).astype(np.float32)
    s = MagnetSpec(size=(10, 6, 2), msat=rng.uniform(3e5, 9e5, shape).astype(np.float32),
                   ku1=rng.uniform(1e5, 8e5, shape).astype(np.float32), ku2=2e4, anisU=u, bias=bias,
                   world_bias=(0.01, -0.02, 0.03), enable_demag=False)
    compare(s, mpx, [abi.Q_ANISOTROPY_FIELD, abi.Q_EXTERNAL_FIELD, abi.Q_ANISOTROPY_ENERGY_DENSITY,
                     abi.Q_ZEEMAN_ENERGY_DENSITY])


def test_geometry_regions_lut_frozen(mpx):
    shape = (2, 10, 12)
    geom = np.ones(shape, dtype=bool)
    geom[:, 4:7, 5:9] = False
    geom[1, 0, :] = False
    regions = np.zeros(shape, dtype=np.uint32)
    regions[:, :, 6:] = 1
    regions[1] = 2
    frozen = np.zeros(shape, np.float32)
    frozen[0, 2, 3] = 1
    msat = np.full(shape, 8e5, np.float32)
    msat[0, 8, 8] = 0.0
    s = MagnetSpec(size=(12, 10, 2), cellsize=(2e-9, 2e-9, 1e-9), geometry=geom, regions=regions, msat=msat,
                   aex=1.3e-11, alpha=0.1, dmi={"xxz": 1e-3, "yyz": 1e-3}, frozen=frozen,
                   inter_pairs={(1, 0): 5e-12}, scale_pairs={(2, 1): 0.5}, world_bias=(0, 0, 0.1))
    compare(s, mpx, [abi.Q_EXCHANGE_FIELD, abi.Q_DMI_FIELD, abi.Q_EXTERNAL_FIELD, abi.Q_DEMAG_FIELD,
                     abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE])


@pytest.mark.parametrize("size", [(16, 4, 3), (17, 4, 1), (8, 10, 2), (33, 20, 5), (1, 1, 1), (64, 1, 1),
                                  (5, 3, 8), (40, 7, 4)])
def test_demag_shapes(mpx, size):
    compare(MagnetSpec(size=size, cellsize=(1e-9, 2e-9, 3.1e-9), msat=8e5), mpx, [abi.Q_DEMAG_FIELD])


@pytest.mark.parametrize("pbc", [(1, 2, 0), (2, 2, 0), (1, 0, 1)])
def test_demag_pbc(mpx, pbc):
    size = (16, 12, 2)
    s = MagnetSpec(size=size, cellsize=(2e-9, 2e-9, 1e-9), msat=5.8e5,
                   mastergrid_size=tuple(size[a] if pbc[a] else 0 for a in range(3)), pbc=pbc)
    compare(s, mpx, [abi.Q_DEMAG_FIELD])


def test_demag_kernel_reference_layout(mpx):
    s = MagnetSpec(size=(16, 4, 3), cellsize=(1e-9, 1e-9, 1e-9))
    ow, q = s.oracle_world()
    world, magnet = s.product(mpx)
    got = magnet._engine.demag_kernel(magnet._id)
    want = ow.demag_kernel(q)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))


def test_small_film_effective_field_torque_energies(mpx):
    # 256x64x1-like film (exchange + demag + Zeeman), scaled down
    s = MagnetSpec(size=(64, 16, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8.6e5, aex=1.3e-11, alpha=0.02,
                   world_bias=(-0.030, 0.005, 0.0))
    compare(s, mpx, [abi.Q_EFFECTIVE_FIELD, abi.Q_DEMAG_FIELD, abi.Q_TORQUE, abi.Q_DAMPING_TORQUE,
                     abi.Q_EXCHANGE_ENERGY_DENSITY, abi.Q_DEMAG_ENERGY_DENSITY, abi.Q_ZEEMAN_ENERGY_DENSITY,
                     abi.Q_TOTAL_ENERGY_DENSITY], seed=1, smooth=3)


def test_multilayer_effective_field(mpx):
    # 512x512x8 multilayer parameters, scaled down: PBC in x,y, iDMI, Ku1 along z
    s = MagnetSpec(size=(32, 32, 8), cellsize=(2e-9, 2e-9, 1e-9), msat=5.8e5, aex=1.5e-11,
                   dmi={"xxz": 3e-3, "yyz": 3e-3}, ku1=8e5, anisU=(0, 0, 1), alpha=0.1,
                   world_bias=(0, 0, 0.2), mastergrid_size=(32, 32, 0), pbc=(2, 2, 0))
    compare(s, mpx, [abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE, abi.Q_DEMAG_FIELD], seed=2, smooth=2)


def test_energies_and_averages(mpx):
    s = MagnetSpec(size=(20, 12, 2), cellsize=(2e-9, 2e-9, 2e-9), msat=8e5, aex=1e-11, ku1=3e5,
                   anisU=(1, 1, 0), dmi={"xxz": 1e-3, "yyz": 1e-3}, world_bias=(0.01, 0, 0.02))
    m0 = random_m(s.shape, seed=9, smooth=2)
    ow, q = s.oracle_world(m0)
    world, magnet = s.product(mpx, m0)
    for quantity, prop in [(abi.Q_EXCHANGE_ENERGY_DENSITY, "exchange_energy"),
                           (abi.Q_DMI_ENERGY_DENSITY, "dmi_energy"),
                           (abi.Q_ANISOTROPY_ENERGY_DENSITY, "anisotropy_energy"),
                           (abi.Q_ZEEMAN_ENERGY_DENSITY, "zeeman_energy"),
                           (abi.Q_DEMAG_ENERGY_DENSITY, "demag_energy"),
                           (abi.Q_TOTAL_ENERGY_DENSITY, "total_energy")]:
        got = getattr(magnet, prop).eval()
        want = ow.energy(q, quantity)
        assert got == pytest.approx(want, rel=1e-5, abs=1e-30), prop
    np.testing.assert_allclose(magnet.magnetization.average(), ow.average(q, abi.Q_MAGNETIZATION), atol=1e-6)
    np.testing.assert_allclose(magnet.effective_field.average(), ow.average(q, abi.Q_EFFECTIVE_FIELD),
                               atol=1e-5 * np.max(np.abs(ow.eval(q, abi.Q_EFFECTIVE_FIELD))))


def _macrospin_exact(t, m0, hz, damping):
    mx, my, mz = m0
    theta0 = np.arccos(mz / np.sqrt(mx**2 + my**2 + mz**2))
    phi0 = np.arctan(my / mx)
    freq = GAMMALL * hz / (1 + damping**2)
    phi = phi0 + freq * t
    theta = np.pi - 2 * np.arctan(np.exp(damping * freq * t) * np.tan(np.pi / 2 - theta0 / 2))
    return {"mx": np.sin(theta) * np.cos(phi), "my": np.sin(theta) * np.sin(phi), "mz": np.cos(theta)}


@pytest.mark.parametrize("method", ["Heun", "BogackiShampine", "CashKarp", "Fehlberg", "DormandPrince"])
def test_solve_single_system(mpx, method):
    # test/test_timesolver.py:90-122, through the mumaxplus-style API
    world = mpx.World(cellsize=(1, 1, 1))
    magnet = mpx.Ferromagnet(world, grid=mpx.Grid((1, 1, 1)))
    magnet.enable_demag = False
    magnet.magnetization = (1, 0, 0)
    magnet.alpha = 0.2
    world.bias_magnetic_field = (0, 0, 0.11)
    world.timesolver.set_method(method)
    tps = np.linspace(0, 5e-10, 20)
    out = world.timesolver.solve(tps, {
        "mx": lambda: magnet.magnetization.average()[0],
        "my": lambda: magnet.magnetization.average()[1],
        "mz": lambda: magnet.magnetization.average()[2],
    })
    exact = _macrospin_exact(tps, (1, 0, 0), 0.11, 0.2)
    for mc in ("mx", "my", "mz"):
        assert np.max(np.abs(np.array(out[mc]) - exact[mc])) < 1e-4


def test_fixed_timestep_and_setters(mpx):
    world = mpx.World(cellsize=(1, 1, 1))
    ts = world.timesolver
    assert ts.time == 0.0
    ts.time = 1e-9
    assert ts.time == pytest.approx(1e-9)
    ts.time = 0.0
    assert ts.adaptive_timestep is True
    ts.adaptive_timestep = False
    ts.timestep = 2.3e-9
    ts.steps(103)
    assert ts.time == pytest.approx(103 * 2.3e-9, rel=1e-5)
    for bad in ("", "asdf"):
        with pytest.raises(ValueError):
            ts.set_method(bad)
    with pytest.raises(TypeError):
        ts.set_method(2)


@pytest.mark.parametrize("method", ["DormandPrince", "Fehlberg"])
def test_film_trajectory_vs_oracle(mpx, method):
    # <m>(t) of a small film with exchange + demag + Zeeman vs the FP64 oracle
    s = MagnetSpec(size=(32, 16, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8.6e5, aex=1.3e-11, alpha=0.02,
                   world_bias=(-0.030, 0.005, 0.0))
    m0 = random_m(s.shape, seed=1, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_method(method)
    world, magnet = s.product(mpx, m0)
    world.timesolver.set_method(method)
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = 0.0
    for k in range(1, 9):
        tp = k * 25e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        a = np.array(magnet.magnetization.average())
        b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
        worst = max(worst, float(np.max(np.abs(a - b))))
    assert worst < 1e-4, worst
    assert world.timesolver.time == pytest.approx(ow.time, rel=1e-12)


def test_two_groups_one_engine_match_alone(mpx):
    """A group advanced beside another group gives the same result as alone."""
    from mumaxplus_b200._engine import Engine

    def build(eng, size, seed, bias):
        s = MagnetSpec(size=size, cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.1,
                       world_bias=(0, 0, 0))
        s.bias = bias
        g = eng.group_create()
        keep = []
        mid = eng.magnet_add(g, s.desc(keep))
        eng.set_m(mid, random_m(s.shape, seed=seed, smooth=2))
        p = eng.solver_params(g)
        p.method = abi.RK_METHODS["DormandPrince"]
        eng.set_solver_params(g, p)
        eng.set_timestep(g, 1e-13)
        return g, mid, s.shape

    alone = Engine()
    ga, ma, shape_a = build(alone, (24, 20, 1), 3, (0.02, 0, 0.05))
    alone.group_start(ga, 30e-12)
    while True:
        alone.advance(8)
        done, running = alone.poll()
        if running == 0:
            break
    ref = alone.get_m(ma, (3, *shape_a))

    mixed = Engine()
    g1, m1, _ = build(mixed, (24, 20, 1), 3, (0.02, 0, 0.05))
    g2, m2, shape2 = build(mixed, (40, 8, 2), 4, (0, 0.03, 0))
    mixed.group_start(g1, 30e-12)
    mixed.group_start(g2, 45e-12)
    while True:
        mixed.advance(8)
        done, running = mixed.poll()
        if running == 0:
            break
    got = mixed.get_m(m1, (3, *shape_a))
    assert np.array_equal(got, ref)
    assert mixed.get_time(g1) == pytest.approx(30e-12, rel=1e-12)
    assert mixed.get_time(g2) == pytest.approx(45e-12, rel=1e-12)


def test_nan_state_fails_cleanly(mpx):
    world = mpx.World(cellsize=(1e-9, 1e-9, 1e-9))
    magnet = mpx.Ferromagnet(world, mpx.Grid((4, 4, 1)))
    magnet.enable_demag = False
    magnet.aex = 1e-11
    magnet.alpha = 0.1
    magnet.msat = float("nan")
    world.timesolver.timestep = 1e-13
    with pytest.raises(RuntimeError):
        world.timesolver.run(1e-12)
    # the engine stays usable afterwards
    magnet.msat = 8e5
    magnet.magnetization = (1, 0.1, 0)
    world.timesolver.timestep = 1e-13
    world.timesolver.run(1e-12)
    assert world.timesolver.time == pytest.approx(1e-12, rel=1e-9)


@pytest.mark.parametrize("per_cell", [False, True])
def test_cubic_anisotropy(mpx, per_cell):
    """Cubic anisotropy field, energy density and torque (uniform parameters take
    the specialised epilogue, per-cell ones the general one)."""
    rng = np.random.default_rng(5)
    shape = (2, 12, 20)
    if per_cell:
        c1 = rng.standard_normal((3, *shape)).astype(np.float32)
        c2 = np.cross(c1, rng.standard_normal((3, *shape)), axis=0).astype(np.float32)
        kc1 = rng.uniform(1e5, 5e6, shape).astype(np.float32)
    else:
        c1 = (1.0, 2.0, 0.5)
        c2 = tuple(np.cross(c1, [0.3, -1.0, 2.0]))
        kc1 = 4.1e6
    s = MagnetSpec(size=(20, 12, 2), cellsize=(2e-9, 2e-9, 2e-9), msat=8e5, aex=1e-11, alpha=0.1, kc1=kc1,
                   kc2=-2e5, kc3=3e4, anisC1=c1, anisC2=c2)
    compare(s, mpx, [abi.Q_ANISOTROPY_FIELD, abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE, abi.Q_ANISOTROPY_ENERGY_DENSITY,
                     abi.Q_TOTAL_ENERGY_DENSITY])


@pytest.mark.parametrize("kind", ["zhangli", "zhangli_pbc", "slonczewski", "slonczewski_below"])
def test_spin_transfer_torque(mpx, kind):
    common = dict(size=(24, 12, 3), cellsize=(2e-9, 3e-9, 1e-9), msat=7e5, aex=1.1e-11, alpha=0.05)
    if kind.startswith("zhangli"):
        extra = dict(pbc=(1, 0, 0), mastergrid_size=(24, 0, 0)) if kind == "zhangli_pbc" else {}
        s = MagnetSpec(**common, **extra, pol=0.6, xi=0.1, jcur=(2e11, -1e11, 5e10))
    else:
        s = MagnetSpec(**common, pol=0.5, Lambda=1.3, epsilon_prime=0.02, jcur=(0, 0, 3e11),
                       fixed_layer=(1.0, 0.0, 1.0), fixed_layer_on_top=(kind == "slonczewski"))
    compare(s, mpx, [abi.Q_SPIN_TRANSFER_TORQUE, abi.Q_LLG_TORQUE, abi.Q_TORQUE])


def test_zhang_li_trajectory_vs_oracle(mpx):
    s = MagnetSpec(size=(32, 8, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.05, pol=0.7,
                   xi=0.05, jcur=(5e11, 0.0, 0.0))
    m0 = random_m(s.shape, seed=6, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_method("DormandPrince")
    world, magnet = s.product(mpx, m0)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = 0.0
    for k in range(1, 5):
        tp = k * 10e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        a = np.array(magnet.magnetization.average())
        b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
        worst = max(worst, float(np.max(np.abs(a - b))))
    assert worst < 1e-4, worst


@pytest.mark.parametrize("size", [(16, 8, 16), (12, 6, 9), (8, 4, 33), (40, 7, 20), (24, 20, 12)])
def test_demag_thick_magnets_split_path(mpx, size):
    """nz > 8 takes the three-pass y/z path (k_ycols, k_zmul, k_ycols)."""
    compare(MagnetSpec(size=size, cellsize=(1e-9, 2e-9, 1.5e-9), msat=8e5), mpx, [abi.Q_DEMAG_FIELD])


def test_thick_magnet_pbc_and_trajectory(mpx):
    s = MagnetSpec(size=(16, 12, 10), cellsize=(2e-9, 2e-9, 2e-9), msat=8e5, aex=1.3e-11, alpha=0.2,
                   pbc=(1, 0, 1), mastergrid_size=(16, 0, 10), world_bias=(0.0, 0.01, 0.02))
    compare(s, mpx, [abi.Q_DEMAG_FIELD, abi.Q_EFFECTIVE_FIELD])
    m0 = random_m(s.shape, seed=9, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_method("DormandPrince")
    world, magnet = s.product(mpx, m0)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    ow.run(10e-12)
    world.timesolver._e.run(world._group, 10e-12)
    a = np.array(magnet.magnetization.average())
    b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
    assert float(np.max(np.abs(a - b))) < 1e-4


@pytest.mark.parametrize("size", [(6, 40, 3), (5, 70, 1), (4, 200, 2), (3, 300, 6), (3, 400, 2), (200, 6, 2),
                                  (300, 5, 1), (130, 70, 4), (4, 200, 7), (3, 500, 8), (5, 100, 5)])
def test_demag_warp_transform_lengths(mpx, size):
    """y lengths 128 .. 1024 (k_yzw, k_yzw32: four-step Q x 32 with 32/Q columns per warp) at z lengths 1 .. 16
    (z length 16, nz 5 .. 8, in one lane per ky), and x rows of 512 and 1024 points (warp rows)."""
    compare(MagnetSpec(size=size, cellsize=(1e-9, 2e-9, 1.5e-9), msat=8e5), mpx, [abi.Q_DEMAG_FIELD])


@pytest.mark.parametrize("size", [(3, 600, 1), (2, 700, 2), (3, 1000, 3), (2, 513, 4), (1, 1024, 2), (600, 3, 2),
                                  (1000, 2, 1), (700, 4, 3), (520, 520, 1)])
def test_demag_warp_pair_length_2048(mpx, size):
    """Length 2048 in warp pairs (four-step 64 x 32, the inverse folding the upper half in): y transforms
    (k_yzw64) at z lengths 1, 4, 8 and 8, several kx per block for thin magnets, ny from 513 to 1024; x rows
    (pair_rows in both x passes) for nx from 520 to 1000."""
    compare(MagnetSpec(size=size, cellsize=(1e-9, 2e-9, 1.5e-9), msat=8e5), mpx, [abi.Q_DEMAG_FIELD])


@pytest.mark.parametrize("size", [(12, 600, 2), (600, 12, 2)])
def test_warp_pair_trajectory_vs_oracle(mpx, size):
    """Dormand-Prince stages through the warp-pair transforms of length 2048 (y transforms at Pz = 4, then the
    x passes with the stage combination and the lean epilogue): <m>(t) against the FP64 oracle."""
    s = MagnetSpec(size=size, cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.1,
                   world_bias=(0.0, 0.01, 0.0))
    m0 = random_m(s.shape, seed=9, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_method("DormandPrince")
    world, magnet = s.product(mpx, m0)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = 0.0
    for k in range(1, 4):
        tp = k * 3e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        a = np.array(magnet.magnetization.average())
        b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
        worst = max(worst, float(np.max(np.abs(a - b))))
    assert worst < 1e-4, worst


def test_warp_transform_trajectory_vs_oracle(mpx):
    """Dormand-Prince stages through the warp transforms of both axes (Px = 512, Py = 128) and the lean stage
    epilogue (uniform parameters): <m>(t) and the field m(t) against the FP64 oracle."""
    s = MagnetSpec(size=(132, 40, 2), cellsize=(3e-9, 3e-9, 3e-9), msat=8e5, aex=1.3e-11, alpha=0.1,
                   dmi={"xxz": 1e-3, "yyz": 1e-3}, ku1=1e5, anisU=(0.0, 0.0, 1.0), world_bias=(0.0, 0.01, 0.0))
    m0 = random_m(s.shape, seed=8, smooth=3)
    ow, q = s.oracle_world(m0)
    ow.set_method("DormandPrince")
    world, magnet = s.product(mpx, m0)
    world.timesolver.set_method("DormandPrince")
    dt0 = ow.sensible_timestep()
    ow.timestep = dt0
    world.timesolver.timestep = dt0
    worst = worst_cell = 0.0
    for k in range(1, 4):
        tp = k * 4e-12
        ow.run(tp - ow.time)
        world.timesolver._e.run(world._group, tp - world.timesolver.time)
        a = np.array(magnet.magnetization.average())
        b = np.array(ow.average(q, abi.Q_MAGNETIZATION))
        worst = max(worst, float(np.max(np.abs(a - b))))
        worst_cell = max(worst_cell, float(np.max(np.abs(magnet.magnetization.get() - ow.get_m(q)))))
    assert worst < 1e-5, worst
    assert worst_cell < 1e-3, worst_cell


def test_warp_transforms_with_geometry_regions_frozen(mpx):
    """A magnet with geometry, regions, per-cell parameters and frozen cells (the generic epilogue) at sizes that
    take the warp transforms (Px = 512, Py = 256)."""
    shape = (2, 70, 132)
    zz, yy, xx = np.meshgrid(np.arange(2), np.arange(70), np.arange(132), indexing="ij")
    geom = ((xx - 66) ** 2 / 66.0 ** 2 + (yy - 35) ** 2 / 35.0 ** 2) <= 1.0
    regions = (xx >= 66).astype(np.uint32)
    msat = np.where(yy < 20, 6e5, 8e5).astype(np.float32)
    frozen = np.zeros(shape, np.float32)
    frozen[1, 35, 60:70] = 1
    s = MagnetSpec(size=(132, 70, 2), cellsize=(2e-9, 2e-9, 1.5e-9), geometry=geom, regions=regions, msat=msat,
                   aex=1.3e-11, alpha=0.1, dmi={"xxz": 1e-3, "yyz": 1e-3}, frozen=frozen,
                   inter_pairs={(1, 0): 5e-12}, world_bias=(0, 0, 0.05))
    compare(s, mpx, [abi.Q_DEMAG_FIELD, abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE])
