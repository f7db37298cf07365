"""mpx_reduce_noalloc: the reduction for callers that may not allocate device
memory (e.g. a monitoring hook inside another application's loop with a fixed
device-memory budget).  Through the C ABI it must give the same sums and max
norms as the engine's own mpx_average / mpx_max_norm (which use engine-owned
scratch), on two calls in a row, and reject out-of-range sizes.

The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _magnet(mpx):
    world = mpx.World((2e-9, 2e-9, 1e-9))
    magnet = mpx.Ferromagnet(world, mpx.Grid((48, 20, 3)))
    magnet.msat = 8e5
    magnet.aex = 1.3e-11
    magnet.enable_demag = False
    rng = np.random.default_rng(12)
    magnet.magnetization = rng.standard_normal((3, 3, 20, 48)).astype(np.float32)
    return world, magnet


def test_reduce_noalloc_matches_engine_reductions(mpx):
    import torch

    world, magnet = _magnet(mpx)
    eng = magnet._engine
    lib = mpx._abi.load()
    N = magnet.grid.ncells
    Q = mpx._abi.Q_MAGNETIZATION
    buf = torch.empty(3 * N, dtype=torch.float32, device="cuda")
    eng.eval_device(magnet._id, Q, buf.data_ptr())
    eng.synchronize()
    torch.cuda.synchronize()
    avg = eng.average(magnet._id, Q)
    mx = eng.max_norm(magnet._id, Q)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out = (C.c_double * 3)()
        assert lib.mpx_reduce_noalloc(buf.data_ptr(), N, 3, None, 0, None, out) == 0
        np.testing.assert_allclose(np.array(out[:]) / N, avg, rtol=1e-12, atol=1e-15)
        out = (C.c_double * 3)()
        assert lib.mpx_reduce_noalloc(buf.data_ptr(), N, 3, None, 1, None, out) == 0
        assert out[0] == pytest.approx(mx, rel=1e-12)


def test_reduce_noalloc_rejects_out_of_range_sizes(mpx):
    import torch

    lib = mpx._abi.load()
    buf = torch.zeros(12, dtype=torch.float32, device="cuda")
    out = (C.c_double * 3)()
    assert lib.mpx_reduce_noalloc(buf.data_ptr(), 0, 3, None, 0, None, out) == mpx._abi.MPX_ERR_INVALID
    assert lib.mpx_reduce_noalloc(buf.data_ptr(), 4, 4, None, 0, None, out) == mpx._abi.MPX_ERR_INVALID
    assert lib.mpx_reduce_noalloc(buf.data_ptr(), 800_000_000, 3, None, 0, None, out) == mpx._abi.MPX_ERR_INVALID
    assert b"ncells" in lib.mpx_last_error()


@pytest.mark.parametrize("ncomp", [1, 2, 3])
def test_reduce_noalloc_masked_on_a_side_stream_vs_numpy(mpx, ncomp):
    """A geometry mask, 1-3 components and a caller's stream, against numpy
    FP64 sums and max norms of the same buffer; the components past ncomp
    (and out[1:] of the max norm) come back zero."""
    import torch

    lib = mpx._abi.load()
    rng = np.random.default_rng(40 + ncomp)
    N = 7919  # not a multiple of the block size
    host = rng.standard_normal((ncomp, N)).astype(np.float32)
    mask = (rng.uniform(size=N) < 0.6).astype(np.uint8)
    want_sum = np.zeros(3)
    want_sum[:ncomp] = host.astype(np.float64)[:, mask.astype(bool)].sum(axis=1)
    want_max = float(np.max(np.linalg.norm(host.astype(np.float64)[:, mask.astype(bool)], axis=0)))
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        buf = torch.from_numpy(host.reshape(-1)).to("cuda", non_blocking=False)
        geom = torch.from_numpy(mask).to("cuda", non_blocking=False)
    side.synchronize()
    for _ in range(2):
        out = (C.c_double * 3)(7.0, 7.0, 7.0)
        assert lib.mpx_reduce_noalloc(buf.data_ptr(), N, ncomp, C.c_void_p(geom.data_ptr()), 0,
                                      C.c_void_p(side.cuda_stream), out) == 0
        np.testing.assert_allclose(np.array(out[:]), want_sum, rtol=1e-12, atol=1e-9)
        assert all(out[c] == 0.0 for c in range(ncomp, 3))
        out = (C.c_double * 3)(7.0, 7.0, 7.0)
        assert lib.mpx_reduce_noalloc(buf.data_ptr(), N, ncomp, C.c_void_p(geom.data_ptr()), 1,
                                      C.c_void_p(side.cuda_stream), out) == 0
        assert out[0] == pytest.approx(want_max, rel=1e-12)
        assert out[1] == 0.0 and out[2] == 0.0
