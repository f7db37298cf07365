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
