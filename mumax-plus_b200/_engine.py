"""Thin Python handle over the libmpx.so engine (include/mpx.h).

Errors come back as status codes and are raised here the way the reference's
pybind11 layer maps its C++ exceptions: invalid argument -> ValueError, out of
range -> IndexError, runtime error -> RuntimeError.
"""
import ctypes as C
import os

import numpy as np

from . import _abi

_EXC = {
    _abi.MPX_ERR_INVALID: ValueError,
    _abi.MPX_ERR_RANGE: IndexError,
    _abi.MPX_ERR_RUNTIME: RuntimeError,
    _abi.MPX_ERR_NOMEM: MemoryError,
    _abi.MPX_ERR_CUDA: RuntimeError,
    _abi.MPX_ERR_UNSUPPORTED: NotImplementedError,
    _abi.MPX_ERR_TIMEOUT: TimeoutError,
    _abi.MPX_ERR_NODEVICE: RuntimeError,
}


def lib():
    """The loaded libmpx.so; fails loudly when the CUDA library was not built."""
    if not os.path.exists(_abi.LIB_PATH):
        raise RuntimeError(
            f"libmpx.so not found at {_abi.LIB_PATH}; build it with "
            "`python mumax-plus_b200/build.py` (nvcc, sm_100a)")
    return _abi.load()


def check(status):
    if status != _abi.MPX_OK:
        msg = lib().mpx_last_error().decode(errors="replace")
        raise _EXC.get(status, RuntimeError)(msg)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Engine:
    """One mpx_engine: a CUDA stream on one device holding magnets and groups."""

    def __init__(self, device=None):
        L = lib()
        if L.mpx_device_count() <= 0:
            raise RuntimeError("no CUDA device available: the mumax-plus B200 engine has no CPU path")
        if device is None:
            device = int(os.environ.get("MPX_DEVICE", "0"))
        h = C.c_void_p()
        check(L.mpx_engine_create(int(device), C.byref(h)))
        self._h = h
        self.device = device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _abi.load().mpx_engine_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- engine level
    def set_stream(self, stream_ptr):
        check(lib().mpx_engine_set_stream(self._h, C.c_void_p(stream_ptr)))

    def synchronize(self):
        check(lib().mpx_engine_synchronize(self._h))

    def set_dft(self, mode):
        """_abi.MPX_DFT_FP32 or _abi.MPX_DFT_TF32X3 (before the first magnet)."""
        check(lib().mpx_engine_set_dft(self._h, int(mode)))

    @staticmethod
    def tc_timeouts():
        """Tensor-core waits that gave up since the last call (device synchronised, count cleared)."""
        n = C.c_uint(0)
        check(lib().mpx_tc_status(C.byref(n)))
        return n.value

    def set_world_bias(self, b):
        arr = (C.c_double * 3)(*[float(v) for v in b])
        check(lib().mpx_engine_set_world_bias(self._h, arr))

    def memory(self):
        v = C.c_int64()
        check(lib().mpx_engine_memory(self._h, C.byref(v)))
        return v.value

    def graph_stats(self):
        """(instantiations, in-place updates) of the attempt graphs."""
        a, b = C.c_int64(), C.c_int64()
        check(lib().mpx_engine_graph_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def launch_count(self):
        v = C.c_int64()
        check(lib().mpx_engine_launch_count(self._h, C.byref(v)))
        return v.value

    # -- groups
    def group_create(self):
        g = C.c_int()
        check(lib().mpx_group_create(self._h, C.byref(g)))
        return g.value

    def group_destroy(self, g):
        check(lib().mpx_group_destroy(self._h, int(g)))

    def group_info(self, g):
        info = _abi.GroupInfo()
        check(lib().mpx_group_info_get(self._h, int(g), C.byref(info)))
        return info

    def group_save(self, g):
        """Snapshot of group g (time, time step, step count, m and FSAL k0 of its
        magnets) as a uint8 array."""
        n = C.c_int64()
        check(lib().mpx_group_state_bytes(self._h, int(g), C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        check(lib().mpx_group_save(self._h, int(g), buf.ctypes.data, int(n.value)))
        return buf

    def group_load(self, g, state):
        buf = np.ascontiguousarray(state, dtype=np.uint8)
        check(lib().mpx_group_load(self._h, int(g), buf.ctypes.data, int(buf.size)))

    # -- magnets
    def magnet_add(self, group, desc):
        m = C.c_int()
        check(lib().mpx_magnet_add(self._h, int(group), C.byref(desc), C.byref(m)))
        return m.value

    def magnet_add_state(self, group, desc, m0):
        """Add a magnet with its initial magnetization (float32 (3, nz, ny, nx))."""
        a = np.ascontiguousarray(m0, dtype=np.float32)
        m = C.c_int()
        check(lib().mpx_magnet_add_state(self._h, int(group), C.byref(desc), a.ctypes.data, 0, C.byref(m)))
        return m.value

    def magnet_update(self, magnet, desc):
        check(lib().mpx_magnet_update(self._h, int(magnet), C.byref(desc)))

    def magnet_remove(self, magnet):
        check(lib().mpx_magnet_remove(self._h, int(magnet)))

    def set_m(self, magnet, m):
        a = np.ascontiguousarray(m, dtype=np.float32)
        check(lib().mpx_magnet_set_m(self._h, int(magnet), a.ctypes.data, 0))

    def set_m_device(self, magnet, dev_ptr):
        check(lib().mpx_magnet_set_m(self._h, int(magnet), C.c_void_p(dev_ptr), 1))

    def get_m(self, magnet, shape, out=None):
        """Magnetization as (3, nz, ny, nx) float32; into `out` (e.g. a pinned
        host buffer, for a direct DMA copy) when given."""
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.shape == tuple(shape)
        check(lib().mpx_magnet_get_m(self._h, int(magnet), out.ctypes.data, 0))
        return out

    def get_m_device(self, magnet, dev_ptr):
        check(lib().mpx_magnet_get_m(self._h, int(magnet), C.c_void_p(dev_ptr), 1))

    def eval(self, magnet, quantity, shape):
        out = np.empty(shape, dtype=np.float32)
        check(lib().mpx_eval(self._h, int(magnet), int(quantity), out.ctypes.data, 0))
        return out

    def eval_only(self, magnet, quantity):
        """Evaluate into the engine's scratch buffer, no copy (timing)."""
        check(lib().mpx_eval(self._h, int(magnet), int(quantity), None, 2))

    def eval_device(self, magnet, quantity, dev_ptr):
        check(lib().mpx_eval(self._h, int(magnet), int(quantity), C.c_void_p(dev_ptr), 1))

    def average(self, magnet, quantity):
        out = (C.c_double * 3)()
        check(lib().mpx_average(self._h, int(magnet), int(quantity), out))
        return [out[0], out[1], out[2]]

    def max_norm(self, magnet, quantity):
        out = C.c_double()
        check(lib().mpx_max_norm(self._h, int(magnet), int(quantity), C.byref(out)))
        return out.value

    def energy(self, magnet, quantity):
        out = C.c_double()
        check(lib().mpx_energy(self._h, int(magnet), int(quantity), C.byref(out)))
        return out.value

    def profile_eval(self, magnet, reps=10):
        """Mean ms per launch of [x-forward, y/z, x-inverse, local-only] kernels."""
        out = (C.c_double * 4)()
        check(lib().mpx_profile_eval(self._h, int(magnet), int(reps), out))
        return [out[i] for i in range(4)]

    def profile_attempt(self, method="DormandPrince", reps=5):
        """Mean ms of [combination + x-forward, stray pairs, y/z passes, x-inverse +
        epilogue] of stage 1 over every started group."""
        out = (C.c_double * 4)()
        check(lib().mpx_profile_attempt(self._h, _abi.RK_METHODS[method], int(reps), out))
        return [out[i] for i in range(4)]

    def autotune(self, method="DormandPrince"):
        """Pick the tile-shape divisors of the started groups by timing (returns (div_x, div_yz))."""
        dx, dy = C.c_int(), C.c_int()
        check(lib().mpx_autotune(self._h, _abi.RK_METHODS[method], C.byref(dx), C.byref(dy)))
        return dx.value, dy.value

    def demag_kernel(self, magnet):
        dims = (C.c_int * 3)()
        check(lib().mpx_demag_kernel(self._h, int(magnet), None, dims))
        kx, ky, kz = dims[0], dims[1], dims[2]
        out = np.empty((6, kz, ky, kx), dtype=np.float32)
        check(lib().mpx_demag_kernel(self._h, int(magnet), out.ctypes.data, dims))
        return out

    # -- solver
    def solver_params(self, g):
        p = _abi.SolverParams()
        check(lib().mpx_solver_get_params(self._h, int(g), C.byref(p)))
        return p

    def set_solver_params(self, g, p):
        check(lib().mpx_solver_set_params(self._h, int(g), C.byref(p)))

    def get_time(self, g):
        v = C.c_double()
        check(lib().mpx_solver_get_time(self._h, int(g), C.byref(v)))
        return v.value

    def set_time(self, g, t):
        check(lib().mpx_solver_set_time(self._h, int(g), float(t)))

    def get_timestep(self, g):
        v = C.c_double()
        check(lib().mpx_solver_get_timestep(self._h, int(g), C.byref(v)))
        return v.value

    def set_timestep(self, g, dt):
        check(lib().mpx_solver_set_timestep(self._h, int(g), float(dt)))

    def sensible_timestep(self, g):
        v = C.c_double()
        check(lib().mpx_solver_sensible_timestep(self._h, int(g), C.byref(v)))
        return v.value

    def step(self, g):
        check(lib().mpx_solver_step(self._h, int(g)))

    def steps(self, g, n):
        check(lib().mpx_solver_steps(self._h, int(g), int(n)))

    def run(self, g, duration):
        check(lib().mpx_solver_run(self._h, int(g), float(duration)))

    def run_sampled(self, g, times, nmag):
        """Run through the time points and return the table recorded on the
        device: one row [t, <m> of each of the group's nmag magnets] per point."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        out = np.zeros((t.size, 1 + 3 * int(nmag)), dtype=np.float64)
        dp = C.POINTER(C.c_double)
        check(lib().mpx_solver_run_sampled(self._h, int(g), t.ctypes.data_as(dp), int(t.size), out.ctypes.data_as(dp)))
        return out

    def minimize(self, g, tol=1e-6, nsamples=10):
        check(lib().mpx_minimize(self._h, int(g), float(tol), int(nsamples)))

    def relax(self, g, tol=1e-9, threshold=-1.0):
        check(lib().mpx_relax(self._h, int(g), float(tol), float(threshold)))

    # -- batched
    def group_start(self, g, duration, torque_stop=0.0):
        check(lib().mpx_group_start(self._h, int(g), float(duration), float(torque_stop)))

    def advance(self, attempts):
        check(lib().mpx_advance(self._h, int(attempts)))

    def poll(self, cap=4096):
        done = (C.c_int * cap)()
        nd, nr = C.c_int(), C.c_int()
        check(lib().mpx_poll(self._h, done, cap, C.byref(nd), C.byref(nr)))
        return [done[i] for i in range(nd.value)], nr.value


def magnet_bytes(desc):
    """(resident, transient) device bytes that adding `desc` takes (no GPU needed)."""
    res, tr = C.c_int64(), C.c_int64()
    check(_abi.load().mpx_magnet_bytes(C.byref(desc), C.byref(res), C.byref(tr)))
    return res.value, tr.value
