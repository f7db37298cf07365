"""The tensor-core y transforms of the demag convolution (World(...,
demag_dft="tf32x3"): tcgen05 TF32 GEMMs with 3xTF32 split products) against
the FP64 oracle convolving the GPU's own kernel values (so that only the
transform arithmetic is compared), at <= 1e-5 of max|B| like the FP32 path
(measured: 2e-6 of max|B| on the 1024x1024x4 precision case, FP32 2.8e-7),
for y lengths 1024 and 2048 with and without z padding, periodic images and
geometry; a Dormand-Prince trajectory through the gated stage launches; and
no tensor-core wait that gave up."""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, max_rel, random_m

abi = O.abi
pytestmark = pytest.mark.gpu
FIELD_TOL = 1e-5


def _product(spec, mpx, m0, dft):
    world = mpx.World(spec.cellsize, pbc_repetitions=tuple(spec.pbc), mastergrid=mpx.Grid(spec.mastergrid_size),
                      demag_dft=dft)
    magnet = mpx.Ferromagnet(world, mpx.Grid(spec.size), geometry=spec.geometry)
    magnet._suspend = True
    magnet.msat = spec.msat
    magnet.aex = spec.aex
    magnet.alpha = spec.alpha
    magnet._suspend = False
    magnet._update()
    magnet.magnetization = m0
    return world, magnet


def _same_kernel_oracle(spec, eng, magnet, m0):
    K = eng.demag_kernel(magnet._id)
    nx, ny, nz = spec.size
    o = (K.shape[1] - nz, K.shape[2] - ny, K.shape[3] - nx)
    octant = K[:, o[0]:, o[1]:, o[2]:].astype(np.float64)
    ow, q = spec.oracle_world(m0)
    ow.set_kernel_octant(q, octant)
    return ow, q


CASES = [
    ("py1024_nz2", dict(size=(16, 512, 2), cellsize=(2e-9, 2e-9, 1e-9))),
    ("py1024_ny300", dict(size=(20, 300, 1), cellsize=(3e-9, 2e-9, 2e-9))),
    ("py2048_nz1", dict(size=(8, 1000, 1), cellsize=(2e-9, 2e-9, 1e-9))),
    ("py2048_nz3_pbc", dict(size=(12, 700, 3), cellsize=(2e-9, 1e-9, 1e-9), mastergrid_size=(12, 0, 0),
                            pbc=(2, 0, 0))),
    ("py2048_geometry", dict(size=(10, 1024, 2), cellsize=(2e-9, 2e-9, 2e-9))),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_tc_demag_vs_oracle_same_kernel(mpx, name, kw):
    s = MagnetSpec(msat=8e5, aex=1.3e-11, **kw)
    if name == "py2048_geometry":
        g = np.ones(s.shape, bool)
        g[:, 100:300, 3:7] = False
        s.geometry = g
    m0 = random_m(s.shape, seed=11, smooth=1)
    world, magnet = _product(s, mpx, m0, "tf32x3")
    eng = magnet._engine
    got = eng.eval(magnet._id, abi.Q_DEMAG_FIELD, (3, *s.shape))
    ow, q = _same_kernel_oracle(s, eng, magnet, m0)
    want = ow.eval(q, abi.Q_DEMAG_FIELD)
    err = max_rel(got, want)
    assert err < FIELD_TOL, err
    # and against the FP32 shared-memory FFT of the same magnet
    w2, m2 = _product(s, mpx, m0, "fp32")
    ref32 = m2._engine.eval(m2._id, abi.Q_DEMAG_FIELD, (3, *s.shape))
    assert max_rel(got, ref32) < 2 * FIELD_TOL
    assert mpx._engine.Engine.tc_timeouts() == 0


def test_tc_mode_is_fixed_before_magnets(mpx):
    world = mpx.World((1e-9, 1e-9, 1e-9), demag_dft="tf32x3")
    assert world.demag_dft == "tf32x3"
    mpx.Ferromagnet(world, mpx.Grid((8, 8, 1)))
    with pytest.raises(ValueError):
        world._engine.set_dft(mpx._abi.MPX_DFT_FP32)
    with pytest.raises(ValueError):
        mpx.World((1e-9, 1e-9, 1e-9), demag_dft="fp16")


def test_tc_trajectory_vs_fp32_path(mpx):
    """Dormand-Prince steps of a 16x512x2 film (stage launches with the group
    gate) in both DFT modes: <m> and the state agree to the FP32 level."""
    s = MagnetSpec(size=(16, 512, 2), cellsize=(2e-9, 2e-9, 2e-9), msat=8e5, aex=1.3e-11, alpha=0.1)
    m0 = random_m(s.shape, seed=5, smooth=2)
    out = {}
    for dft in ("fp32", "tf32x3"):
        world, magnet = _product(s, mpx, m0, dft)
        world.bias_magnetic_field = (0.01, 0.0, 0.02)
        ts = world.timesolver
        ts.set_method("DormandPrince")
        ts.timestep = 1e-13
        ts.steps(40)
        out[dft] = (np.array(magnet.magnetization.average()), magnet.magnetization.get(), ts.time)
    assert np.max(np.abs(out["fp32"][0] - out["tf32x3"][0])) < 1e-5
    # per cell the two roundings (field differences ~2e-6 of max|B|) grow over
    # 40 steps to ~1e-4
    assert np.max(np.abs(out["fp32"][1] - out["tf32x3"][1])) < 5e-4
    assert mpx._engine.Engine.tc_timeouts() == 0


def test_tc_multilayer_full_size(mpx):
    """The 512x512x8 multilayer (y length 1024, PBC) with the tensor-core y
    transforms: demag and effective field against the oracle with the GPU's
    kernel values, <= 1e-5."""
    from mumaxplus_b200 import workloads as W

    w = W.multilayer()
    nx, ny, nz = w["size"]
    m0 = random_m((nz, ny, nx), seed=7, smooth=3)
    world, magnet = W.build(mpx, w, demag_dft="tf32x3")
    magnet.magnetization = m0
    eng = magnet._engine
    K = eng.demag_kernel(magnet._id)
    o = (K.shape[1] - nz, K.shape[2] - ny, K.shape[3] - nx)
    octant = K[:, o[0]:, o[1]:, o[2]:].astype(np.float64)
    del K
    keep = []
    ow = O.OracleWorld()
    ow.set_world_bias(w["world_bias"])
    q = ow.add_magnet(W.desc(w, keep))
    ow.set_m(q, m0)
    ow.set_kernel_octant(q, octant)
    del octant
    errs = {qq: max_rel(eng.eval(magnet._id, qq, (3, nz, ny, nx)), ow.eval(q, qq))
            for qq in (abi.Q_DEMAG_FIELD, abi.Q_EFFECTIVE_FIELD)}
    # B_eff at the FP32 bound; the demag field alone of this disordered state
    # sits at the FP32 rounding of its x-pass FFTs (1.9e-5 of its maximum, as
    # with the FP32 y transforms)
    assert errs[abi.Q_EFFECTIVE_FIELD] < FIELD_TOL, errs
    assert errs[abi.Q_DEMAG_FIELD] < 5 * FIELD_TOL, errs
    assert mpx._engine.Engine.tc_timeouts() == 0


def test_tc_mode_leaves_other_lengths_on_the_fp32_path(mpx):
    """In the tensor-core mode a magnet whose padded y length is neither 1024
    nor 2048 keeps the FP32 y transforms: the same field, bit for bit."""
    s = MagnetSpec(size=(24, 100, 2), cellsize=(2e-9, 2e-9, 1e-9), msat=8e5, aex=1.3e-11)  # Py = 256
    m0 = random_m(s.shape, seed=3, smooth=1)
    _, a = _product(s, mpx, m0, "tf32x3")
    _, b = _product(s, mpx, m0, "fp32")
    fa = a._engine.eval(a._id, abi.Q_DEMAG_FIELD, (3, *s.shape))
    fb = b._engine.eval(b._id, abi.Q_DEMAG_FIELD, (3, *s.shape))
    np.testing.assert_array_equal(fa, fb)


def test_tc_wait_timeout_path_leaves_the_device_usable(mpx):
    """Failure detection without a fault: a block of the tensor-core kind waits
    on an mbarrier that nothing arrives at; its bounded wait runs out, the
    timeout is counted and its tensor memory released, and the next
    tensor-core evaluation runs normally (no timeout, same field)."""
    import ctypes as C

    lib = mpx._abi.load()
    n = C.c_uint(0)
    assert lib.mpx_tc_timeout_selftest(C.byref(n)) == 0
    assert n.value == 1
    s = MagnetSpec(size=(16, 512, 2), cellsize=(2e-9, 2e-9, 1e-9), msat=8e5, aex=1.3e-11)
    m0 = random_m(s.shape, seed=2, smooth=1)
    world, magnet = _product(s, mpx, m0, "tf32x3")
    eng = magnet._engine
    got = eng.eval(magnet._id, abi.Q_DEMAG_FIELD, (3, *s.shape))
    ow, q = _same_kernel_oracle(s, eng, magnet, m0)
    assert max_rel(got, ow.eval(q, abi.Q_DEMAG_FIELD)) < FIELD_TOL
    assert mpx._engine.Engine.tc_timeouts() == 0
