"""Pins the CPU FP64 oracle against the known answers the reference's own tests
hold for this path (CPU only, no GPU).

  exchange     test/test_exchange.py:6-46     numpy Laplacian, Neumann edges
               test/test_exchange.py:48-85    spiral energy vs A k^2 up to 20 degrees
  DMI          test/test_interfacialdmi.py     numpy, open boundaries
  anisotropy   test/test_anisotropy.py:15-57   numpy uniaxial field / energy
  demag        test/test_demag.py:6-45         numpy FFT of the real-space kernel
  stray field  test/test_strayfield.py:57-84   FFT vs direct sum, with PBC
  time solver  test/test_timesolver.py:19-169  analytic macrospin precession, all 5 methods
  PBC          test/test_PBC.py:14-91          <m> after 1 ns vs the mumax3 value
  minimize     test/test_standardproblem2_coercivity.py, test/test_boundaries.py (coercivity, wire canting)
  frozen spins test/test_frozenspins.py:28-56   <m> after minimize and a 1 ns reversal, half the film frozen
  STT          test/test_free_layer_thickness.py  Slonczewski torque unchanged by empty layers

The known answers themselves are in tests/golden/known_answers.json.
"""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, known, max_rel, random_m

abi = O.abi
GAMMALL = 1.7595e11


def test_newell_cube_self_demag():
    # a cube's self-demag tensor is 1/3 on the diagonal, 0 off the diagonal
    for c in range(3):
        assert O.newell(c, 0, 0, 0, (1e-9, 1e-9, 1e-9)) == pytest.approx(1 / 3, rel=1e-12)
    for c in range(3, 6):
        assert O.newell(c, 0, 0, 0, (1e-9, 1e-9, 1e-9)) == 0.0
    # trace of the self term is 1 for any cell shape
    cs = (1e-9, 2e-9, 3.1e-9)
    tr = sum(O.newell(c, 0, 0, 0, cs) for c in range(3))
    assert tr == pytest.approx(1.0, rel=1e-10)


def test_newell_far_field_dipole():
    # far away the tensor tends to the point dipole V/(4 pi r^3) (3 r r / r^2 - 1)
    cs = (1e-9, 1e-9, 1e-9)
    x = 12
    nxx = O.newell(0, x, 0, 0, cs)
    assert nxx == pytest.approx(-2.0 / (4 * np.pi * x**3), rel=2e-2)


def _exchange_numpy(m, cellsize, aex, msat):
    # test/test_exchange.py:6-31 (Neumann: the missing neighbour adds nothing)
    h = np.zeros(m.shape)
    for ax, c in ((1, cellsize[2]), (2, cellsize[1]), (3, cellsize[0])):
        for shift in (1, -1):
            m_ = np.roll(m, shift, axis=ax)
            sl = [slice(None)] * 4
            sl[ax] = slice(1, None) if shift == 1 else slice(0, -1)
            h[tuple(sl)] += (m_ - m)[tuple(sl)] / c**2
    return 2 * aex * h / msat


def test_exchange_neumann_vs_numpy():
    s = MagnetSpec(size=(16, 16, 4), cellsize=(1e3, 2e3, 3e3), aex=3.2e7, msat=5.4, enable_demag=False)
    m0 = random_m(s.shape, seed=11)
    w, q = s.oracle_world(m0)
    m = w.get_m(q)
    wanted = _exchange_numpy(m, s.cellsize, s.aex, s.msat)
    got = w.eval(q, abi.Q_EXCHANGE_FIELD)
    assert np.max(np.abs(got - wanted) / np.abs(wanted)) < 1e-9


def test_exchange_energy_of_spirals_vs_analytic():
    """test/test_exchange.py:48-85 (figure 5 of the MuMax3 verification paper): the exchange energy of the
    spiral m = (cos kx, sin kx, 0) on a 100 um x 1 nm x 1 nm wire, in units of Km V (Km = mu0 Msat^2 / 2),
    against the continuum value A k^2 / Km, for k = 1e7, 2e7, ... 1/m until the angle between neighbouring
    cells reaches 20 degrees; relative error < 1e-2 (the discrete energy is 2A(1 - cos k dx)/dx^2 per volume,
    plus the two free ends)."""
    msat, aex, dx = 800e3, 5e-12, 1e-9
    nx = 100_000
    mu0 = 4 * np.pi * 1e-7
    km = 0.5 * mu0 * msat**2
    volume = nx * dx * dx * dx
    s = MagnetSpec(size=(nx, 1, 1), cellsize=(dx, dx, dx), aex=aex, msat=msat, enable_demag=False)
    X = np.arange(nx, dtype=np.float64) * dx
    w, q = s.oracle_world(np.stack([np.ones(nx), np.zeros(nx), np.zeros(nx)]).reshape(3, 1, 1, nx))
    assert w.energy(q, abi.Q_EXCHANGE_ENERGY_DENSITY) == pytest.approx(0.0, abs=1e-30)
    errors = []
    k = 1e7
    while k * dx < 20 * np.pi / 180:
        m = np.stack([np.cos(k * X), np.sin(k * X), np.zeros(nx)]).reshape(3, 1, 1, nx)
        w.set_m(q, m)
        e_num = w.energy(q, abi.Q_EXCHANGE_ENERGY_DENSITY) / (km * volume)
        e_ana = aex * k**2 / km
        errors.append(abs(e_ana - e_num) / e_ana)
        k += 1e7
    assert len(errors) >= 30
    assert max(errors) < 1e-2


def _idmi_numpy(m, cs, Dxxz, Dyyz, msat):
    # test/test_interfacialdmi.py:8-43 (open boundaries)
    X, Y, Z = 0, 1, 2
    h = np.zeros(m.shape)
    m_ = np.roll(m, 1, axis=3)
    h[X][:, :, 1:] -= Dxxz * m_[Z][:, :, 1:] / cs[0]
    h[Z][:, :, 1:] += Dxxz * m_[X][:, :, 1:] / cs[0]
    m_ = np.roll(m, -1, axis=3)
    h[X][:, :, 0:-1] += Dxxz * m_[Z][:, :, 0:-1] / cs[0]
    h[Z][:, :, 0:-1] -= Dxxz * m_[X][:, :, 0:-1] / cs[0]
    m_ = np.roll(m, 1, axis=2)
    h[Y][:, 1:, :] -= Dyyz * m_[Z][:, 1:, :] / cs[1]
    h[Z][:, 1:, :] += Dyyz * m_[Y][:, 1:, :] / cs[1]
    m_ = np.roll(m, -1, axis=2)
    h[Y][:, 0:-1, :] += Dyyz * m_[Z][:, 0:-1, :] / cs[1]
    h[Z][:, 0:-1, :] -= Dyyz * m_[Y][:, 0:-1, :] / cs[1]
    return h / msat


def test_interfacial_dmi_openbc_vs_numpy():
    s = MagnetSpec(size=(4, 5, 3), cellsize=(1.1, 2.0, 3.2), msat=3.1, dmi={"xxz": 7.1, "yyz": -7.1},
                   enable_openbc=True, enable_demag=False)
    w, q = s.oracle_world(random_m(s.shape, seed=3))
    m = w.get_m(q)
    wanted = _idmi_numpy(m, s.cellsize, 7.1, -7.1, 3.1)
    got = w.eval(q, abi.Q_DMI_FIELD)
    assert np.max(np.abs(got - wanted) / np.abs(wanted)) < 1e-9


def test_uniaxial_anisotropy_vs_numpy():
    s = MagnetSpec(size=(16, 32, 4), cellsize=(1e-9, 2e-9, 4e-9), msat=800e3, ku1=4.1e6, ku2=2.1e6,
                   anisU=(0.3, 0.4, 1.0), enable_demag=False)
    w, q = s.oracle_world(random_m(s.shape, seed=5))
    m = w.get_m(q)
    u = np.array([0.3, 0.4, 1.0]) / np.linalg.norm([0.3, 0.4, 1.0])
    mu = np.einsum("c...,c->...", m, u)
    wanted = (2 * 4.1e6 * mu + 4 * 2.1e6 * mu**3)[None] * u[:, None, None, None] / 800e3
    assert max_rel(w.eval(q, abi.Q_ANISOTROPY_FIELD), wanted) < 1e-12
    e_wanted = -4.1e6 * mu**2 - 2.1e6 * mu**4
    assert np.max(np.abs(w.eval(q, abi.Q_ANISOTROPY_ENERGY_DENSITY)[0] - e_wanted)) < 1e-6 * np.max(np.abs(e_wanted))
    E = w.energy(q, abi.Q_ANISOTROPY_ENERGY_DENSITY)
    assert E == pytest.approx(np.sum(e_wanted) * 1e-9 * 2e-9 * 4e-9, rel=1e-10)


def _demag_numpy(kernel, mag):
    # test/test_demag.py:6-36: numpy FFT convolution on the reference kernel grid,
    # cropping the LAST n cells of the padded result
    pad = [(0, kernel.shape[i + 1] - mag.shape[i + 1]) for i in range(3)]
    m = np.pad(mag, ((0, 0), *pad), "constant")
    m = np.fft.fftn(m, axes=(1, 2, 3))
    kxx, kyy, kzz, kxy, kxz, kyz = np.fft.fftn(kernel, axes=(1, 2, 3))
    hx = np.fft.ifftn(m[0] * kxx + m[1] * kxy + m[2] * kxz)
    hy = np.fft.ifftn(m[0] * kxy + m[1] * kyy + m[2] * kyz)
    hz = np.fft.ifftn(m[0] * kxz + m[1] * kyz + m[2] * kzz)
    h = -1.25663706212e-6 * np.array([hx, hy, hz]).real
    return h[:, (h.shape[1] - mag.shape[1]):, (h.shape[2] - mag.shape[2]):, (h.shape[3] - mag.shape[3]):]


def test_demag_vs_numpy_fft_of_reference_kernel_layout():
    s = MagnetSpec(size=(16, 4, 3), cellsize=(1e-9, 1e-9, 1e-9), msat=1.0)
    w, q = s.oracle_world(random_m(s.shape, seed=7))
    kernel = w.demag_kernel(q)
    assert kernel.shape == (6, 5, 8, 32)  # 2n-1, padded to even when above 5
    wanted = _demag_numpy(kernel, 1.0 * w.get_m(q))
    got = w.eval(q, abi.Q_DEMAG_FIELD)
    assert max_rel(got, wanted) < 1e-12


@pytest.mark.parametrize("pbc", [None, (1, 2, 0)])
@pytest.mark.parametrize("size", [(17, 4, 1), (8, 10, 2), (6, 7, 5)])
def test_demag_fft_vs_direct_sum(size, pbc):
    # test/test_strayfield.py:57-84 (same source and destination grid)
    kw = dict(size=size, cellsize=(1e-9, 2e-9, 3.1e-9), msat=800e3)
    if pbc is not None:
        kw.update(mastergrid_size=tuple(size[a] if pbc[a] else 0 for a in range(3)), pbc=pbc)
    s = MagnetSpec(**kw)
    w, q = s.oracle_world(random_m(s.shape, seed=17))
    assert max_rel(w.eval(q, abi.Q_DEMAG_FIELD), w.demag_brute(q)) < 1e-10


def test_demag_with_geometry_and_regions_vs_direct_sum():
    geom = np.ones((2, 9, 11), dtype=bool)
    geom[:, 3:6, 4:8] = False
    s = MagnetSpec(size=(11, 9, 2), cellsize=(2e-9, 2e-9, 1e-9), msat=np.linspace(3e5, 9e5, 198).reshape(2, 9, 11),
                   geometry=geom)
    w, q = s.oracle_world(random_m(s.shape, seed=19))
    got, wanted = w.eval(q, abi.Q_DEMAG_FIELD), w.demag_brute(q)
    assert max_rel(got, wanted) < 1e-12
    assert np.all(got[:, ~geom] == 0)


def _macrospin_exact(t, m0, hz, damping):
    # test/test_timesolver.py:19-29 analytic LLG precession about z
    mx, my, mz = m0
    theta0 = np.arccos(mz / np.sqrt(mx**2 + my**2 + mz**2))
    phi0 = np.arctan(my / mx)
    freq = GAMMALL * hz / (1 + damping**2)
    phi = phi0 + freq * t
    theta = np.pi - 2 * np.arctan(np.exp(damping * freq * t) * np.tan(np.pi / 2 - theta0 / 2))
    return np.array([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)])


@pytest.mark.parametrize("method", list(abi.RK_METHODS))
def test_macrospin_vs_analytic(method):
    s = MagnetSpec(size=(1, 1, 1), cellsize=(1, 1, 1), alpha=0.2, enable_demag=False, world_bias=(0, 0, 0.11))
    w, q = s.oracle_world(np.array([1, 0, 0], np.float32).reshape(3, 1, 1, 1))
    w.set_method(method)
    w.timestep = w.sensible_timestep()
    tps = np.linspace(0, 5e-10, 20)
    got = []
    for tp in tps:
        w.run(tp - w.time)
        got.append(w.get_m(q)[:, 0, 0, 0])
    exact = _macrospin_exact(tps, (1, 0, 0), 0.11, 0.2)
    assert np.max(np.abs(np.array(got).T - exact)) < 1e-4


def test_fixed_timestep_time_accumulation():
    # test/test_timesolver.py:80-86
    s = MagnetSpec(size=(1, 1, 1), cellsize=(1, 1, 1), enable_demag=False)
    w, q = s.oracle_world()
    w.set_solver(adaptive=0)
    w.timestep = 2.3e-9
    w.steps(103)
    assert w.time == pytest.approx(103 * 2.3e-9, rel=1e-5)


def _pbc_rectangle_geometry(nx, ny, corners=False):
    # test/test_PBC.py:34-51: Rectangle(nx/2 c, ny/2 c) centred in the box,
    # repeated; cells at positions i*c.  Inside: nx/4 <= i < 3nx/4 (and y alike).
    ix = np.arange(nx)
    iy = np.arange(ny)
    if corners:
        ix = (ix - nx // 2) % nx
        iy = (iy - ny // 2) % ny
    inx = (ix >= nx // 4) & (ix < 3 * nx // 4)
    iny = (iy >= ny // 4) & (iy < 3 * ny // 4)
    return (iny[:, None] & inx[None, :])[None]


@pytest.mark.slow
def test_pbc_run_center_matches_mumax3_golden():
    # test/test_PBC.py:77-82: <m> after 1 ns, mumax3 value, relative error < 1e-3
    nx, ny, c = 128, 64, 5e-9
    s = MagnetSpec(size=(nx, ny, 1), cellsize=(c, c, c), mastergrid_size=(nx, ny, 0), pbc=(2, 2, 0),
                   geometry=_pbc_rectangle_geometry(nx, ny), msat=1000e3, aex=10e-12, alpha=1.0)
    m0 = np.zeros((3, 1, ny, nx), np.float32)
    m0[0], m0[1], m0[2] = 1.0, 0.1, 0.01
    w, q = s.oracle_world(m0)
    w.timestep = w.sensible_timestep()
    w.run(1e-9)
    avg = w.average(q, abi.Q_MAGNETIZATION)
    k = known("pbc_center_m_1ns")
    wanted = np.array(k["value"])
    assert np.linalg.norm(np.array(avg) - wanted) / np.linalg.norm(wanted) < k["rel_tol"]


def test_oracle_external_kernel_octant_reproduces_own(oracle):
    """The external-kernel hook (used to compare convolution arithmetic apart
    from kernel construction): feeding back the oracle's own real-space kernel
    octant reproduces its demag field (to the FP64 rounding by which the
    direct 27-point evaluation of the exported kernel differs from the shared
    lattice evaluation of the octant)."""
    s = MagnetSpec(size=(20, 12, 3), cellsize=(2e-9, 3e-9, 1.5e-9), msat=7e5)
    m0 = random_m(s.shape, seed=9, smooth=1)
    ow, q = s.oracle_world(m0)
    want = ow.eval(q, oracle.abi.Q_DEMAG_FIELD)
    K = ow.demag_kernel(q)  # reference layout, origin -(n-1)-pad per axis
    nx, ny, nz = s.size
    o = [K.shape[3] - nx, K.shape[2] - ny, K.shape[1] - nz]  # index of displacement 0
    oct = K[:, o[2]:, o[1]:, o[0]:]
    ow2, q2 = s.oracle_world(m0)
    ow2.set_kernel_octant(q2, oct)
    got = ow2.eval(q2, oracle.abi.Q_DEMAG_FIELD)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))


def sp2_coercivity(make, minimize, set_field, m_sum):
    """Standard problem 2 in the small-particle limit, the protocol of the
    reference's test/test_standardproblem2_coercivity.py:14-66: one cell of
    L x d x t = 0.5 x 0.1 x 0.01 exchange lengths, minimize from (1,1,1), then
    raise a field along -(1,1,1) in steps of 5e-5 Msat until m flips; returns
    the interpolated relative coercive field."""
    d = 0.1
    t, L = 0.1 * d, 5.0 * d
    msat, aex, mu0 = 800e3, 13e-12, 1.25663706212e-6
    lex = np.sqrt(2 * aex / (mu0 * msat ** 2))
    make((L * lex, d * lex, t * lex), msat, aex)
    minimize()
    hdir = -np.ones(3) / np.sqrt(3)
    h1 = 0.05
    set_field(mu0 * h1 * msat * hdir)
    minimize()
    m1 = m_sum()
    h0, m0 = 0.0, None
    while m1 > 0:
        h0, m0 = h1, m1
        h1 += 0.00005
        set_field(mu0 * h1 * msat * hdir)
        minimize()
        m1 = m_sum()
    return (m0 * h1 - m1 * h0) / (m0 - m1)


def nanowire_canting(minimize, x_of_m, make):
    """test/test_boundaries.py: canting of the first cell of a 1024-cell wire with interfacial DMI after
    minimize(1e-7), Neumann boundaries first, then open boundaries from that state (the reference's order).
    make(openbc, m0) builds the magnet; returns (Neumann, open) cantings."""
    m0 = np.zeros((3, 1, 1, 1024), np.float32)
    m0[2] = 1.0
    out = []
    for openbc in (False, True):
        get_m = make(openbc, m0)
        minimize()
        m = get_m()
        out.append(float(np.arctan2(m[0, 0, 0, 0], m[2, 0, 0, 0])))
        m0 = m.astype(np.float32)
    return out


NANOWIRE = dict(cs=0.05, D=0.9 * 4 / np.pi)


def nanowire_spec(openbc):
    cs, D = NANOWIRE["cs"], NANOWIRE["D"]
    return MagnetSpec(size=(1024, 1, 1), cellsize=(cs, cs, cs), msat=1.0, aex=1.0, ku1=1.0, anisU=(0.0, 0.0, 1.0),
                      dmi={"xxz": D, "yyz": D}, enable_demag=False, enable_openbc=openbc)


def check_nanowire(neumann, open_):
    cs, D = NANOWIRE["cs"], NANOWIRE["D"]
    k = known("nanowire_canting_neumann")
    assert abs(neumann - k["value"]) / k["value"] < k["rel_tol"], neumann
    analytic = 2 * np.arctan(np.exp(-cs / 2) * np.tan(np.arcsin(D / 2) / 2))
    k = known("nanowire_canting_open")
    assert abs(open_ - analytic) / analytic < k["rel_tol"], open_
    k = known("nanowire_canting_open_mumax3")
    assert abs(open_ - k["value"]) / k["value"] < k["rel_tol"], open_


def test_oracle_nanowire_canting_golden(oracle):
    st = {}

    def make(openbc, m0):
        ow, q = nanowire_spec(openbc).oracle_world(m0)
        st.update(ow=ow)
        return lambda: ow.get_m(q)

    check_nanowire(*nanowire_canting(lambda: st["ow"].minimize(1e-7, 10), None, make))


def test_oracle_frozen_half_film_golden(oracle):
    """test/test_frozenspins.py:28-56: a standard-problem-4 film (128 x 32 x 2) with the cells right of the centre
    frozen (the centre is the midpoint of the first and last cell positions, so cells x >= 64), minimized from
    (1, 0.1, 0), then run for 1 ns with the bias field (-24.6, 4.3, 0) mT on, Fehlberg (the reference's default
    method) from the sensible time step; <m> after each against the reference's vectors (1e-4 per component).
    The bias is applied as the world bias, which enters the Zeeman term like the magnet's own."""
    nx, ny, nz = 128, 32, 2
    frozen = np.zeros((nz, ny, nx), np.float32)
    frozen[:, :, 64:] = 1
    s = MagnetSpec(size=(nx, ny, nz), cellsize=(500e-9 / 128, 125e-9 / 32, 3e-9 / 2), msat=800e3, aex=13e-12,
                   alpha=0.02, frozen=frozen)
    m0 = np.zeros((3, nz, ny, nx))
    m0[0], m0[1] = 1.0, 0.1
    w, q = s.oracle_world(m0)
    w.set_method("Fehlberg")
    w.minimize()
    k = known("frozen_half_minimized_m")
    assert np.max(np.abs(np.array(w.average(q, abi.Q_MAGNETIZATION)) - k["value"])) < k["abs_tol"]
    frozen_m = w.get_m(q)[:, :, :, 64:].copy()
    w.set_world_bias((-24.6e-3, 4.3e-3, 0.0))
    w.timestep = w.sensible_timestep()
    w.run(1e-9)
    k = known("frozen_half_reversal_m_1ns")
    assert np.max(np.abs(np.array(w.average(q, abi.Q_MAGNETIZATION)) - k["value"])) < k["abs_tol"]
    assert np.array_equal(w.get_m(q)[:, :, :, 64:], frozen_m)  # frozen cells never move


def test_oracle_minimize_sp2_coercivity_golden(oracle):
    """Known answer of the reference test: H_c / Msat (tests/golden/known_answers.json)."""
    st = {}

    def make(cs, msat, aex):
        s = MagnetSpec(size=(1, 1, 1), cellsize=cs, msat=msat, aex=aex)
        ow, q = s.oracle_world(np.ones((3, 1, 1, 1), np.float32))
        st.update(ow=ow, q=q)

    rhc = sp2_coercivity(make, lambda: st["ow"].minimize(1e-6, 10),
                         lambda b: st["ow"].set_world_bias(tuple(b)),
                         lambda: float(np.sum(st["ow"].average(st["q"], oracle.abi.Q_MAGNETIZATION))))
    k = known("sp2_coercivity")
    assert abs(k["value"] - rhc) < k["abs_tol"], rhc


def test_oracle_relax_reaches_the_minimum_of_a_uniaxial_film(oracle):
    """relax from a tilted state of a film with a strong uniaxial axis and a
    field along it ends aligned with the axis, with the solver's time, time step
    and settings restored."""
    s = MagnetSpec(size=(8, 6, 1), cellsize=(2e-9, 2e-9, 2e-9), msat=8e5, aex=1e-11, alpha=0.1, ku1=5e5,
                   anisU=(0.0, 0.0, 1.0), world_bias=(0.0, 0.0, 0.05), enable_demag=False)
    m0 = np.zeros((3, 1, 6, 8), np.float32)
    m0[0], m0[2] = 0.6, 0.8
    ow, q = s.oracle_world(m0)
    ow.set_method("DormandPrince")
    ow.timestep = 1e-13
    ow.time = 3e-12
    ow.relax(1e-9)
    m = np.array(ow.average(q, oracle.abi.Q_MAGNETIZATION))
    assert m[2] > 1 - 1e-6
    assert ow.time == 3e-12
    assert oracle.abi.RK_NAMES[ow.solver.method] == "DormandPrince"


def _cubic_numpy(m, msat, kc, c1, c2):
    """numpy restatement of the reference's cubic anisotropy field and energy
    density (test/test_anisotropy.py:73-112, physics/anisotropy.cu:57-106)."""
    c1 = c1 / np.linalg.norm(c1, axis=0)
    c2 = c2 / np.linalg.norm(c2, axis=0)
    c3 = np.cross(c1, c2, axis=0)
    a, b, c = (np.sum(v * m, axis=0) for v in (c1, c2, c3))
    k1, k2, k3 = kc
    h = -2 / msat * (k1 * ((b**2 + c**2) * a * c1 + (a**2 + c**2) * b * c2 + (a**2 + b**2) * c * c3)
                     + k2 * (b**2 * c**2 * a * c1 + a**2 * c**2 * b * c2 + a**2 * b**2 * c * c3)
                     + 2 * k3 * ((b**4 + c**4) * a**3 * c1 + (a**4 + c**4) * b**3 * c2 + (a**4 + b**4) * c**3 * c3))
    e = (k1 * (a**2 * b**2 + a**2 * c**2 + b**2 * c**2) + k2 * a**2 * b**2 * c**2
         + k3 * (a**4 * b**4 + a**4 * c**4 + b**4 * c**4))
    return h, e


@pytest.mark.parametrize("per_cell", [False, True])
def test_oracle_cubic_anisotropy_vs_numpy(oracle, per_cell):
    rng = np.random.default_rng(21)
    shape = (2, 5, 6)
    m = random_m(shape, seed=3, smooth=0).astype(np.float64)
    if per_cell:
        c1 = rng.standard_normal((3, *shape)).astype(np.float32)
        c2 = np.cross(c1, rng.standard_normal((3, *shape)), axis=0).astype(np.float32)
        kc1 = rng.uniform(1e5, 5e6, shape).astype(np.float32)
        c1v, c2v, kc1v = c1, c2, kc1
    else:
        c1 = np.array([1.0, 2.0, 0.5], np.float32)
        c2 = np.cross(c1, [0.3, -1.0, 2.0]).astype(np.float32)
        c1v = np.broadcast_to(c1[:, None, None, None], (3, *shape)).astype(np.float64)
        c2v = np.broadcast_to(c2[:, None, None, None], (3, *shape)).astype(np.float64)
        kc1 = kc1v = 4.1e6
        c1, c2 = tuple(c1), tuple(c2)
    s = MagnetSpec(size=(6, 5, 2), msat=8e5, kc1=kc1, kc2=-2e5, kc3=3e4, anisC1=c1, anisC2=c2, enable_demag=False)
    ow, q = s.oracle_world(m.astype(np.float32))
    mm = ow.get_m(q)
    h, e = _cubic_numpy(mm, 8e5, (np.asarray(kc1v, np.float64), -2e5, 3e4), np.asarray(c1v, np.float64),
                        np.asarray(c2v, np.float64))
    np.testing.assert_allclose(ow.eval(q, oracle.abi.Q_ANISOTROPY_FIELD), h, rtol=1e-9, atol=1e-12 * np.abs(h).max())
    np.testing.assert_allclose(ow.eval(q, oracle.abi.Q_ANISOTROPY_ENERGY_DENSITY)[0], e, rtol=1e-9,
                               atol=1e-9 * np.abs(e).max())


def test_oracle_stray_field_between_magnets_equals_union_demag(oracle):
    """Two magnets of one world: self demag (FFT) + stray field of the other
    (direct sum over the tabulated tensor) equals the demag field of a single
    magnet covering both, with the gap masked out (independent code paths of
    the oracle, physics/zeeman.cu:70-88 vs strayfieldfft.cu)."""
    cs = (2e-9, 3e-9, 2.5e-9)
    A = MagnetSpec(size=(10, 6, 2), cellsize=cs, msat=8e5)
    B = MagnetSpec(size=(7, 6, 2), origin=(13, 2, 0), cellsize=cs, msat=6e5)
    mA = random_m(A.shape, seed=11, smooth=1)
    mB = random_m(B.shape, seed=12, smooth=1)
    ow = O.OracleWorld()
    keep = []
    qa = ow.add_magnet(A.desc(keep))
    qb = ow.add_magnet(B.desc(keep))
    ow.set_m(qa, mA)
    ow.set_m(qb, mB)
    got_b = ow.eval(qb, oracle.abi.Q_EFFECTIVE_FIELD)
    got_a = ow.eval(qa, oracle.abi.Q_EFFECTIVE_FIELD)
    # union grid 20 x 8 x 2 at the origin
    nz, ny, nx = 2, 8, 20
    geom = np.zeros((nz, ny, nx), np.uint8)
    msat = np.zeros((nz, ny, nx), np.float32)
    m = np.zeros((3, nz, ny, nx), np.float32)
    m[0] = 1.0
    geom[:, 0:6, 0:10] = 1
    geom[:, 2:8, 13:20] = 1
    msat[:, 0:6, 0:10] = 8e5
    msat[:, 2:8, 13:20] = 6e5
    m[:, :, 0:6, 0:10] = mA
    m[:, :, 2:8, 13:20] = mB
    U = MagnetSpec(size=(nx, ny, nz), cellsize=cs, msat=msat, geometry=geom)
    ou, qu = U.oracle_world(m)
    want = ou.eval(qu, oracle.abi.Q_EFFECTIVE_FIELD)
    scale = np.abs(want).max()
    assert np.abs(got_a - want[:, :, 0:6, 0:10]).max() < 1e-9 * scale
    assert np.abs(got_b - want[:, :, 2:8, 13:20]).max() < 1e-9 * scale
    # switches: B no longer receives, A no longer sends
    B2 = MagnetSpec(size=(7, 6, 2), origin=(13, 2, 0), cellsize=cs, msat=6e5, stray_destination=False)
    ow2 = O.OracleWorld()
    qa2 = ow2.add_magnet(A.desc(keep))
    qb2 = ow2.add_magnet(B2.desc(keep))
    ow2.set_m(qa2, mA)
    ow2.set_m(qb2, mB)
    alone = O.OracleWorld()
    ql = alone.add_magnet(B.desc(keep))
    alone.set_m(ql, mB)
    np.testing.assert_array_equal(ow2.eval(qb2, oracle.abi.Q_EFFECTIVE_FIELD), alone.eval(ql, oracle.abi.Q_EFFECTIVE_FIELD))


def _stt_numpy(m, spec):
    """numpy restatement of physics/stt.cu (k_ZhangLi with open edges, no
    mastergrid; k_Slonczewski) for uniform parameters."""
    QE, MUB, HBAR, G = 1.60217646e-19, 9.2740091523e-24, 1.054571817e-34, 1.7595e11
    ms, alpha = spec.msat, spec.alpha
    j = np.array(spec.jcur, float)
    if spec.epsilon_prime or (spec.Lambda and spec.pol):  # Slonczewski
        p = np.array(spec.fixed_layer, float)[:, None, None, None]
        d = spec.size[2] * spec.cellsize[2] if spec.free_layer_thickness is None else spec.free_layer_thickness
        d = d if spec.fixed_layer_on_top else -d
        B = (HBAR / QE) * j[2] / (ms * d)
        l2 = spec.Lambda ** 2
        eps = spec.pol * l2 / ((l2 + 1) + (l2 - 1) * np.sum(m * p, axis=0))
        pxm = np.cross(p, m, axis=0)
        mxpxm = np.cross(m, pxm, axis=0)
        return ((eps + spec.epsilon_prime * alpha) * mxpxm + (spec.epsilon_prime - eps * alpha) * pxm) \
            * B / (1 + alpha ** 2) * G
    xi = spec.xi
    u = MUB * spec.pol / (QE * ms * (1 + xi ** 2)) * j
    hs = np.zeros_like(m)
    for ax, arr_ax in ((0, 3), (1, 2), (2, 1)):
        n = m.shape[arr_ax]
        for sg in (-1, 1):
            shifted = np.zeros_like(m)
            src = [slice(None)] * 4
            dst = [slice(None)] * 4
            if sg == 1:
                src[arr_ax], dst[arr_ax] = slice(1, n), slice(0, n - 1)
            else:
                src[arr_ax], dst[arr_ax] = slice(0, n - 1), slice(1, n)
            shifted[tuple(dst)] = m[tuple(src)]
            hs += sg * u[ax] * shifted / (2 * spec.cellsize[ax])
    mxh = np.cross(m, hs, axis=0)
    mxmxh = np.cross(m, mxh, axis=0)
    return -1 / (1 + alpha ** 2) * ((1 + xi * alpha) * mxmxh + (xi - alpha) * mxh)


@pytest.mark.parametrize("kind", ["zhangli", "slonczewski", "slonczewski_below"])
def test_oracle_spin_transfer_torque_vs_numpy(oracle, kind):
    common = dict(size=(9, 7, 3), cellsize=(2e-9, 3e-9, 1e-9), msat=7e5, alpha=0.05, enable_demag=False)
    if kind == "zhangli":
        s = MagnetSpec(**common, pol=0.6, xi=0.1, jcur=(2e11, -1e11, 5e10))
    else:
        s = MagnetSpec(**common, pol=0.5, Lambda=1.3, epsilon_prime=0.02, jcur=(0, 0, 3e11),
                       fixed_layer=(1.0, 0.0, 1.0), fixed_layer_on_top=(kind == "slonczewski"))
    ow, q = s.oracle_world(random_m(s.shape, seed=4, smooth=1))
    m = ow.get_m(q)
    want = _stt_numpy(m, s)
    got = ow.eval(q, oracle.abi.Q_SPIN_TRANSFER_TORQUE)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
    llg = ow.eval(q, oracle.abi.Q_LLG_TORQUE)
    np.testing.assert_allclose(ow.eval(q, oracle.abi.Q_TORQUE), llg + got, rtol=1e-12, atol=1e-9)


def _langevin(x):
    return 1 / np.tanh(x) - 1 / x


def thermal_macrospins(run_steps, mean_mz):
    """Independent macrospins (no exchange, no demag) in B = 0.1 T along z at
    20 K: after equilibration <m_z> follows the Langevin function of
    x = Ms V B / (kB T) (Boltzmann statistics of a classical moment), which pins
    the amplitude of the thermal field (physics/thermalnoise.cu:60-66)."""
    ms, cs, b, temp = 8e5, 2e-9, 0.1, 20.0
    x = ms * cs ** 3 * b / (1.38064852e-23 * temp)
    spec = MagnetSpec(size=(32, 32, 2), cellsize=(cs, cs, cs), msat=ms, alpha=0.5, temperature=temp,
                      world_bias=(0.0, 0.0, b), enable_demag=False)
    run_steps(spec, 2000)  # equilibrate
    samples = []
    for _ in range(40):
        run_steps(spec, 50)
        samples.append(mean_mz())
    return float(np.mean(samples)), _langevin(x)


def test_oracle_thermal_noise_langevin(oracle):
    st = {}

    def run_steps(spec, n):
        if "ow" not in st:
            m0 = np.zeros((3, *spec.shape), np.float32)
            m0[2] = 1.0
            ow, q = spec.oracle_world(m0)
            ow.set_solver(method=oracle.abi.RK_METHODS["Heun"], adaptive=0)
            ow.timestep = 2e-13
            st.update(ow=ow, q=q)
        st["ow"].steps(n)

    got, want = thermal_macrospins(run_steps, lambda: st["ow"].average(st["q"], oracle.abi.Q_MAGNETIZATION)[2])
    assert abs(got - want) < 0.02, (got, want)


def test_oracle_slonczewski_torque_unchanged_by_empty_layers(oracle):
    """test/test_free_layer_thickness.py:27-61: with the free-layer thickness given explicitly, the Slonczewski
    torque of a 1 x 1 x 2 stack equals that of the same two cells in a 1 x 1 x 4 stack whose top two cells are
    outside the geometry (the empty layers change nothing), within 1e-5 per cell.  The reference test leaves
    Lambda at its default 0, which with epsilon' = 0 makes the Slonczewski term assuredly zero
    (src/physics/stt.cu:18-26, src/physics/ferromagnet.cpp:36), so it compares rounding noise of the Zhang-Li
    term; Lambda = 1 here makes the Slonczewski torque the one compared."""
    rng = np.random.default_rng(21)
    mdir = rng.uniform(size=3)
    mdir /= np.linalg.norm(mdir)
    common = dict(cellsize=(1e-9, 1e-9, 1e-9), msat=4.3, jcur=(0.0, 0.0, 5.4), pol=0.6, fixed_layer=(1.0, 0.0, 1.0),
                  free_layer_thickness=1e-9, Lambda=1.0, enable_demag=False)
    wanted_spec = MagnetSpec(size=(1, 1, 2), **common)
    w1, q1 = wanted_spec.oracle_world(np.broadcast_to(mdir[:, None, None, None], (3, 2, 1, 1)).copy())
    wanted = w1.eval(q1, abi.Q_SPIN_TRANSFER_TORQUE)[:, :, 0, 0]
    geom = np.array([1, 1, 0, 0], dtype=np.uint8).reshape(4, 1, 1)
    result_spec = MagnetSpec(size=(1, 1, 4), geometry=geom, **common)
    w2, q2 = result_spec.oracle_world(np.broadcast_to(mdir[:, None, None, None], (3, 4, 1, 1)).copy())
    got = w2.eval(q2, abi.Q_SPIN_TRANSFER_TORQUE)[:, :, 0, 0]
    assert np.all(np.linalg.norm(wanted, axis=0) > 1e-3)  # a real torque, not rounding noise
    err = np.linalg.norm(got[:, :2] - wanted, axis=0) / np.linalg.norm(wanted, axis=0)
    assert np.max(err) < 1e-5
    assert np.all(got[:, 2:] == 0)  # outside the geometry
