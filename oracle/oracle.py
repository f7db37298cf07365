"""ctypes wrapper of the CPU FP64 oracle (oracle/mpx_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product library never
loads it.  The magnet description is the same mpx_magnet_desc struct the C ABI
of the product takes (include/mpx.h), so both sides get identical inputs.
"""
import ctypes as C
import importlib.util
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_build", "libmpx_oracle.so")


def _load_abi():
    """The product's ctypes ABI description (pure ctypes, no GPU needed)."""
    path = os.path.join(ROOT, "mumax-plus_b200", "_abi.py")
    spec = importlib.util.spec_from_file_location("_mpx_abi_for_oracle", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


abi = _load_abi()


def build(force=False):
    """Compile the oracle with the Makefile beside this file."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "mpx_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        V = C.c_void_p
        P_D = C.POINTER(C.c_double)
        L.ox_create.restype = V
        L.ox_destroy.argtypes = [V]
        L.ox_last_error.restype = C.c_char_p
        # descriptions by address: any struct with the mpx_magnet_desc layout
        L.ox_add_magnet.argtypes = [V, C.c_void_p]
        L.ox_update_magnet.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_set_world_bias.argtypes = [V, P_D]
        L.ox_set_m.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_set_m_raw.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_get_m.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_eval.argtypes = [V, C.c_int, C.c_int, C.c_void_p]
        L.ox_demag_brute.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_demag_kernel.argtypes = [V, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.ox_set_kernel_octant.argtypes = [V, C.c_int, C.c_void_p]
        L.ox_minimize.argtypes = [V, C.c_double, C.c_int]
        L.ox_relax.argtypes = [V, C.c_double, C.c_double]
        L.ox_newell.restype = C.c_double
        L.ox_newell.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.ox_average.argtypes = [V, C.c_int, C.c_int, P_D]
        L.ox_energy.argtypes = [V, C.c_int, C.c_int, P_D]
        L.ox_set_solver.argtypes = [V, C.POINTER(abi.SolverParams)]
        L.ox_get_solver.argtypes = [V, C.POINTER(abi.SolverParams)]
        L.ox_set_time.argtypes = [V, C.c_double]
        L.ox_get_time.restype = C.c_double
        L.ox_get_time.argtypes = [V]
        L.ox_set_timestep.argtypes = [V, C.c_double]
        L.ox_get_timestep.restype = C.c_double
        L.ox_get_timestep.argtypes = [V]
        L.ox_sensible_timestep.restype = C.c_double
        L.ox_sensible_timestep.argtypes = [V]
        L.ox_counters.argtypes = [V, C.POINTER(C.c_int64)]
        L.ox_step.argtypes = [V]
        L.ox_steps.argtypes = [V, C.c_int]
        L.ox_run.argtypes = [V, C.c_double]
        _lib = L
    return _lib


def newell(comp, x, y, z, cs):
    """One component (xx, yy, zz, xy, xz, yz) of the Newell tensor at (x, y, z) cells."""
    return lib().ox_newell(int(comp), int(x), int(y), int(z), float(cs[0]), float(cs[1]), float(cs[2]))


class OracleWorld:
    """A world of the FP64 oracle: magnets, world bias and one time solver."""

    def __init__(self):
        self._h = C.c_void_p(lib().ox_create())
        self._shapes = []

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().ox_destroy(self._h)
            self._h = None

    def _check(self, st):
        if st != 0:
            raise RuntimeError(lib().ox_last_error().decode())

    def add_magnet(self, desc):
        q = lib().ox_add_magnet(self._h, C.byref(desc))
        if q < 0:
            raise RuntimeError(lib().ox_last_error().decode())
        self._shapes.append((desc.size[2], desc.size[1], desc.size[0]))
        return q

    def update_magnet(self, q, desc):
        self._check(lib().ox_update_magnet(self._h, q, C.byref(desc)))

    def set_world_bias(self, b):
        lib().ox_set_world_bias(self._h, (C.c_double * 3)(*[float(v) for v in b]))

    def set_m(self, q, m):
        a = np.ascontiguousarray(m, dtype=np.float32)
        self._check(lib().ox_set_m(self._h, q, a.ctypes.data))

    def set_m_raw(self, q, m):
        a = np.ascontiguousarray(m, dtype=np.float64)
        self._check(lib().ox_set_m_raw(self._h, q, a.ctypes.data))

    def get_m(self, q):
        out = np.empty((3, *self._shapes[q]), dtype=np.float64)
        self._check(lib().ox_get_m(self._h, q, out.ctypes.data))
        return out

    def eval(self, q, quantity):
        nc = 1 if abi.Q_EXCHANGE_ENERGY_DENSITY <= quantity <= abi.Q_TOTAL_ENERGY_DENSITY else 3
        out = np.empty((nc, *self._shapes[q]), dtype=np.float64)
        self._check(lib().ox_eval(self._h, q, int(quantity), out.ctypes.data))
        return out

    def demag_brute(self, q):
        out = np.empty((3, *self._shapes[q]), dtype=np.float64)
        self._check(lib().ox_demag_brute(self._h, q, out.ctypes.data))
        return out

    def demag_kernel(self, q):
        dims = (C.c_int * 3)()
        self._check(lib().ox_demag_kernel(self._h, q, None, dims))
        out = np.empty((6, dims[2], dims[1], dims[0]), dtype=np.float64)
        self._check(lib().ox_demag_kernel(self._h, q, out.ctypes.data, dims))
        return out

    def set_kernel_octant(self, q, oct):
        """Use a given kernel octant (6, nz, ny, nx) of displacements r >= 0."""
        a = np.ascontiguousarray(oct, dtype=np.float64)
        self._check(lib().ox_set_kernel_octant(self._h, q, a.ctypes.data))

    def average(self, q, quantity):
        out = (C.c_double * 3)()
        self._check(lib().ox_average(self._h, q, int(quantity), out))
        return [out[0], out[1], out[2]]

    def energy(self, q, quantity):
        out = C.c_double()
        self._check(lib().ox_energy(self._h, q, int(quantity), C.byref(out)))
        return out.value

    @property
    def solver(self):
        p = abi.SolverParams()
        lib().ox_get_solver(self._h, C.byref(p))
        return p

    def set_solver(self, **kw):
        p = self.solver
        for k, v in kw.items():
            setattr(p, k, v)
        lib().ox_set_solver(self._h, C.byref(p))

    def set_method(self, name):
        self.set_solver(method=abi.RK_METHODS[name])

    @property
    def time(self):
        return lib().ox_get_time(self._h)

    @time.setter
    def time(self, t):
        lib().ox_set_time(self._h, float(t))

    @property
    def timestep(self):
        return lib().ox_get_timestep(self._h)

    @timestep.setter
    def timestep(self, dt):
        lib().ox_set_timestep(self._h, float(dt))

    def sensible_timestep(self):
        return lib().ox_sensible_timestep(self._h)

    def counters(self):
        out = (C.c_int64 * 3)()
        lib().ox_counters(self._h, out)
        return {"steps": out[0], "rejected": out[1], "evaluations": out[2]}

    def step(self):
        self._check(lib().ox_step(self._h))

    def steps(self, n):
        self._check(lib().ox_steps(self._h, int(n)))

    def minimize(self, tol=1e-6, nsamples=10):
        self._check(lib().ox_minimize(self._h, float(tol), int(nsamples)))

    def relax(self, tol=1e-9, threshold=-1.0):
        self._check(lib().ox_relax(self._h, float(tol), float(threshold)))

    def run(self, duration):
        self._check(lib().ox_run(self._h, float(duration)))
