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
    """Pairs of at least 2^22 cell interactions take the FFT form on the pair's kernel grid (n_A + n_B - 1 per
    axis): fields of both magnets against the oracle's direct sum."""
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


def test_large_pair_fft_form_periodic(mpx):
    """The FFT form in a world with periodic images (mastergrid 128 x 64, one repetition along x and y): the
    tabulated tensor carries the images, so the pair keeps the FFT form; fields of both magnets against the
    oracle's direct sum with the same images."""
    mg, pbc = (128, 64, 0), (1, 1, 0)
    specs = _large_specs(0)
    for s in specs:
        s.mastergrid_size, s.pbc = mg, pbc
    ms = [random_m(s.shape, seed=60 + k, smooth=2) for k, s in enumerate(specs)]
    ow, qs = _oracle(specs, ms)
    world = mpx.World(CS, pbc_repetitions=pbc, mastergrid=mpx.Grid(mg))
    mags = []
    for s, m in zip(specs, ms):
        mag = mpx.Ferromagnet(world, mpx.Grid(s.size, s.origin))
        mag._suspend = True
        mag.msat, mag.aex, mag.alpha = s.msat, s.aex, s.alpha
        mag._suspend = False
        mag._update()
        mag.magnetization = m
        mags.append(mag)
    for q, mag, s in zip(qs, mags, specs):
        for quantity in (abi.Q_EXTERNAL_FIELD, abi.Q_EFFECTIVE_FIELD):
            want = ow.eval(q, quantity)
            got = mag._engine.eval(mag._id, quantity, (3, *s.shape))
            assert max_rel(got, want) < 1e-5, (quantity, max_rel(got, want))


# Grids far apart: the pair's kernel grid depends on the two sizes only (a
# single-layer source and a single-layer destination 40 layers above convolve
# in 2-D; a destination 600 cells along x needs no longer x transforms than an
# adjacent one).  z lengths 1 .. 8 take the fused y / z pass, 16 the three
# separate passes.
FAR_CASES = [
    ((64, 48, 1), (0, 0, 0), (64, 48, 1), (0, 0, 40)),
    ((64, 48, 1), (0, 0, 0), (40, 30, 2), (600, 10, 3)),
    ((30, 20, 3), (0, 0, 0), (50, 70, 1), (-20, -90, -12)),
    ((20, 16, 8), (0, 0, 0), (16, 12, 8), (30, 0, 4)),  # z length 16: the y / z passes unfused
]


@pytest.mark.parametrize("pbc", [None, (1, 1, 0)])
@pytest.mark.parametrize("case", FAR_CASES)
def test_stray_field_far_grids_fft_against_brute(mpx, case, pbc):
    msize, morig, hsize, horig = case
    world = mpx.World(STRAY_CS)
    magnet = mpx.Ferromagnet(world, mpx.Grid(msize, morig))
    magnet.msat = 800e3
    magnet.magnetization = random_m((msize[2], msize[1], msize[0]), seed=7, smooth=1)
    if pbc is not None:
        world.set_pbc(pbc)
    sf = mpx.StrayField(magnet, mpx.Grid(hsize, horig))
    result = sf.eval()
    sf.set_method("brute")
    wanted = sf.eval()
    assert max_rel(result, wanted) < 1e-5, max_rel(result, wanted)


def test_stray_field_repeated_evaluations(mpx):
    """The FFT form keeps the kernel spectra of recent evaluations by geometry:
    a second evaluation gives the same field, a new magnetization the new field
    (against the direct sum), and switching between three grids (more than the
    cache holds) and back gives the same fields again."""
    world = mpx.World(STRAY_CS)
    magnet = mpx.Ferromagnet(world, mpx.Grid((24, 20, 2), (0, 0, 0)))
    magnet.msat = 800e3
    magnet.magnetization = random_m((2, 20, 24), seed=8, smooth=1)
    grids = [mpx.Grid((30, 10, 1), (5, 25, 3)), mpx.Grid((16, 16, 2), (-20, 0, 0)), mpx.Grid((8, 40, 1), (0, 0, 9))]
    first = []
    for g in grids:
        sf = mpx.StrayField(magnet, g)
        a = sf.eval()
        np.testing.assert_array_equal(sf.eval(), a)
        sf.set_method("brute")
        assert max_rel(a, sf.eval()) < 1e-5
        first.append(a)
    for g, a in zip(grids, first):
        np.testing.assert_array_equal(mpx.StrayField(magnet, g).eval(), a)
    magnet.magnetization = random_m((2, 20, 24), seed=9, smooth=1)
    sf = mpx.StrayField(magnet, grids[0])
    new = sf.eval()
    assert max_rel(new, first[0]) > 1e-2
    sf.set_method("brute")
    assert max_rel(new, sf.eval()) < 1e-5


# ------------------------------------------------ StrayField on other grids
# test/test_strayfield.py:29-136: a magnet on mgrid, its field on hgrid, by the
# FFT method against the brute-force method (with and without periodic
# images), and against the demag field of one magnet spanning both grids whose
# msat is zero outside mgrid; here also against the FP64 oracle's demag of
# that union magnet.
STRAY_CASES = [
    ((17, 4, 1), (3, 6, 0), (17, 4, 1), (3, 6, 0)),
    ((8, 10, 1), (2, 15, 0), (6, 7, 2), (-5, 0, 2)),
    ((8, 10, 1), (2, 15, 0), (32, 32, 1), (-5, 0, 0)),
    ((8, 10, 1), (2, 15, -1), (32, 32, 1), (-5, 0, 0)),
    ((8, 10, 2), (2, 15, -1), (32, 32, 1), (-5, 0, 1)),
    ((8, 10, 2), (2, 15, 2), (32, 32, 5), (0, 0, 1)),
]
STRAY_CS = (1e-9, 2e-9, 3.1e-9)


def _rel_err_cellwise(result, wanted):
    """test/test_strayfield.py:7-10: max over cells of |dH| / |H_wanted|."""
    err = np.linalg.norm(np.asarray(result, np.float64) - np.asarray(wanted, np.float64), axis=0)
    return float(np.max(err / np.linalg.norm(np.asarray(wanted, np.float64), axis=0)))


def _extended(g1, g2):
    lo = [min(g1[1][c], g2[1][c]) for c in range(3)]
    hi = [max(g1[1][c] + g1[0][c], g2[1][c] + g2[0][c]) for c in range(3)]
    return tuple(hi[c] - lo[c] for c in range(3)), tuple(lo)


@pytest.mark.parametrize("pbc", [None, (1, 2, 0)])
@pytest.mark.parametrize("case", STRAY_CASES)
def test_stray_field_fft_against_brute(mpx, case, pbc):
    msize, morig, hsize, horig = case
    world = mpx.World(STRAY_CS)
    magnet = mpx.Ferromagnet(world, mpx.Grid(msize, morig))
    magnet.msat = 800e3
    magnet.magnetization = (1, 0, 0)
    if pbc is not None:
        world.set_pbc(pbc)
    sf = mpx.StrayField(magnet, mpx.Grid(hsize, horig))
    sf.set_method("fft")
    result = sf.eval()
    sf.set_method("brute")
    wanted = sf.eval()
    assert result.shape == (3, hsize[2], hsize[1], hsize[0])
    assert _rel_err_cellwise(result, wanted) < 1e-4


@pytest.mark.parametrize("pbc", [None, (1, 2, 1)])
@pytest.mark.parametrize("case", STRAY_CASES)
def test_stray_field_equals_union_demag(mpx, case, pbc):
    msize, morig, hsize, horig = case
    bsize, borig = _extended((msize, morig), (hsize, horig))
    box = mpx.Grid(bsize, borig)
    world = mpx.World(STRAY_CS, (0, 0, 0) if pbc is None else pbc, mpx.Grid((0, 0, 0)) if pbc is None else box)
    magnet = mpx.Ferromagnet(world, mpx.Grid(msize, morig))
    magnet.msat = 800e3
    magnet.magnetization = (1, -1, 2)
    hfield = mpx.StrayField(magnet, mpx.Grid(hsize, horig)).eval()
    hbrute = mpx.StrayField(magnet, mpx.Grid(hsize, horig))
    hbrute.set_method("brute")
    hbrute = hbrute.eval()

    world2 = mpx.World(STRAY_CS, (0, 0, 0) if pbc is None else pbc, mpx.Grid((0, 0, 0)) if pbc is None else box)
    magnet2 = mpx.Ferromagnet(world2, box)
    mi = [morig[c] - borig[c] for c in range(3)]
    mf = [mi[c] + msize[c] for c in range(3)]
    hi = [horig[c] - borig[c] for c in range(3)]
    hf = [hi[c] + hsize[c] for c in range(3)]
    ms = np.zeros((bsize[2], bsize[1], bsize[0]), np.float32)
    ms[mi[2]:mf[2], mi[1]:mf[1], mi[0]:mf[0]] = 800e3
    magnet2.msat = ms
    m = np.ones((3, bsize[2], bsize[1], bsize[0]), np.float32)
    m[:, mi[2]:mf[2], mi[1]:mf[1], mi[0]:mf[0]] = magnet.magnetization.eval()
    magnet2.magnetization = m
    wanted = magnet2.demag_field.eval()[:, hi[2]:hf[2], hi[1]:hf[1], hi[0]:hf[0]]
    assert _rel_err_cellwise(hfield, wanted) < 1e-4
    assert _rel_err_cellwise(hbrute, wanted) < 1e-4

    # the FP64 oracle's demag field of the same union magnet
    s = MagnetSpec(size=bsize, origin=borig, cellsize=STRAY_CS, msat=ms,
                   mastergrid_size=(0, 0, 0) if pbc is None else bsize,
                   mastergrid_origin=(0, 0, 0) if pbc is None else borig,
                   pbc=(0, 0, 0) if pbc is None else pbc)
    ow, q = s.oracle_world(magnet2.magnetization.eval())
    want64 = ow.eval(q, abi.Q_DEMAG_FIELD)[:, hi[2]:hf[2], hi[1]:hf[1], hi[0]:hf[0]]
    assert max_rel(hfield, want64) < 1e-5
    assert max_rel(hbrute, want64) < 1e-5


def test_stray_field_from_magnet(mpx):
    """Magnet.stray_field_from_magnet(source) (mumaxplus/magnet.py:532-552):
    the source's field on this magnet's grid, zero outside its geometry, the
    same as the StrayField of the source on that grid; both methods; the
    magnet's own stray field is its demag field; a magnet of another world
    has none."""
    A, B = _specs()
    geomB = np.ones(B.shape, bool)
    geomB[:, 4:8, 2:9] = False
    B.geometry = geomB
    ms = [random_m(A.shape, seed=3, smooth=1), random_m(B.shape, seed=4, smooth=1)]
    world = mpx.World(CS)
    ma = mpx.Ferromagnet(world, mpx.Grid(A.size, A.origin))
    mb = mpx.Ferromagnet(world, mpx.Grid(B.size, B.origin), geometry=geomB)
    for mag, s, m in ((ma, A, ms[0]), (mb, B, ms[1])):
        mag.msat, mag.aex, mag.alpha = s.msat, s.aex, s.alpha
        mag.magnetization = m
    sf = mb.stray_field_from_magnet(ma)
    got = sf.eval()
    plain = mpx.StrayField(ma, mb.grid).eval()
    np.testing.assert_array_equal(got[:, ~geomB], 0.0)
    assert max_rel(got[:, geomB], plain[:, geomB]) < 1e-6
    sf.set_method("brute")
    assert max_rel(sf.eval(), got) < 1e-5
    own = ma.stray_field_from_magnet(ma).eval()
    np.testing.assert_array_equal(own, ma.demag_field.eval())
    other = mpx.World(CS)
    mc = mpx.Ferromagnet(other, mpx.Grid((4, 4, 1)))
    with pytest.raises(RuntimeError):
        mc.stray_field_from_magnet(ma)


def test_stray_field_argument_errors(mpx):
    """bindings/wrap_strayfield.cpp:16-24: an unknown method is a ValueError;
    a destination grid of no cells is refused by the C ABI."""
    import ctypes as C

    world = mpx.World(STRAY_CS)
    magnet = mpx.Ferromagnet(world, mpx.Grid((8, 4, 1)))
    magnet.msat = 8e5
    sf = mpx.StrayField(magnet, mpx.Grid((4, 4, 1), (10, 0, 0)))
    with pytest.raises(ValueError):
        sf.set_method("direct")
    lib = mpx._abi.load()
    out = np.zeros(12, np.float32)
    st = lib.mpx_stray_field(magnet._engine.handle, magnet._id, -1, (C.c_int * 3)(0, 4, 1), (C.c_int * 3)(0, 0, 0),
                             mpx._abi.MPX_STRAY_FFT, out.ctypes.data, 0)
    assert st == mpx._abi.MPX_ERR_INVALID
    st = lib.mpx_stray_field(magnet._engine.handle, magnet._id, -1, (C.c_int * 3)(4, 4, 1), (C.c_int * 3)(0, 0, 0), 7,
                             out.ctypes.data, 0)
    assert st == mpx._abi.MPX_ERR_INVALID
    # a source with msat 0 gives no field
    magnet.msat = 0.0
    np.testing.assert_array_equal(sf.eval(), 0.0)
