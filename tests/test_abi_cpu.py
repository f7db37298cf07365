"""CPU checks of the C ABI and the host-side logic (no GPU, no compute calls)."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mumax-plus_b200", "libmpx.so")


@pytest.fixture(scope="module")
def built_lib():
    import importlib.util

    spec = importlib.util.spec_from_file_location("_mpx_build", os.path.join(ROOT, "mumax-plus_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def test_library_exports_every_header_symbol(built_lib):
    import mumaxplus_b200 as mpx

    names = mpx._abi.header_symbols()
    assert len(names) >= 30
    lib = C.CDLL(built_lib)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes signature table covers the whole header
    assert sorted(mpx._abi.SIGNATURES) == names
    # the checked build (-DMPX_BOUNDS_CHECK) exports the same ABI
    checked = C.CDLL(os.path.join(ROOT, "mumax-plus_b200", "libmpx_checked.so"))
    missing = [n for n in names if not hasattr(checked, n)]
    assert not missing, missing


def test_device_count_without_gpu_is_safe(built_lib):
    lib = C.CDLL(built_lib)
    n = lib.mpx_device_count()
    assert n >= 0
    lib.mpx_version.restype = C.c_char_p
    assert b"sm_100a" in lib.mpx_version()


def test_engine_create_fails_loudly_without_device(built_lib):
    lib = C.CDLL(built_lib)
    if lib.mpx_device_count() > 0:
        pytest.skip("a device is present")
    h = C.c_void_p()
    st = lib.mpx_engine_create(0, C.byref(h))
    assert st == 8  # MPX_ERR_NODEVICE
    import mumaxplus_b200 as mpx

    with pytest.raises(RuntimeError, match="no CUDA device"):
        mpx.World((1e-9, 1e-9, 1e-9))


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "mpx.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("mpx_magnet_desc %zu\n", sizeof(mpx_magnet_desc));
  printf("mpx_solver_params %zu\n", sizeof(mpx_solver_params));
  printf("mpx_group_info %zu\n", sizeof(mpx_group_info));
  P(mpx_magnet_desc, geometry) P(mpx_magnet_desc, regions) P(mpx_magnet_desc, msat)
  P(mpx_magnet_desc, anis_u) P(mpx_magnet_desc, bias_magnetic_field) P(mpx_magnet_desc, dmi)
  P(mpx_magnet_desc, lut_regions) P(mpx_magnet_desc, scale_exchange_lut) P(mpx_magnet_desc, enable_openbc)
  P(mpx_magnet_desc, kc1) P(mpx_magnet_desc, anis_c2) P(mpx_magnet_desc, stray_destination_off)
  P(mpx_magnet_desc, pol) P(mpx_magnet_desc, jcur) P(mpx_magnet_desc, fixed_layer_below)
  P(mpx_magnet_desc, slonczewski_off)
  P(mpx_solver_params, max_error) P(mpx_solver_params, sensible_timestep_default)
  P(mpx_group_info, status) P(mpx_group_info, max_torque)
  return 0;
}
"""


def test_ctypes_struct_layout_matches_header():
    import mumaxplus_b200 as mpx

    abi = mpx._abi
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write(LAYOUT_C)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    got = {k: int(v) for k, v in got.items()}
    assert got["mpx_magnet_desc"] == C.sizeof(abi.MagnetDesc)
    assert got["mpx_solver_params"] == C.sizeof(abi.SolverParams)
    assert got["mpx_group_info"] == C.sizeof(abi.GroupInfo)
    types = {"mpx_magnet_desc": abi.MagnetDesc, "mpx_solver_params": abi.SolverParams,
             "mpx_group_info": abi.GroupInfo}
    for key, off in got.items():
        if "." in key:
            t, f = key.split(".")
            assert getattr(types[t], f).offset == off, key


class _FakeMagnet:
    """Stand-in owner for host-side Parameter tests."""

    def __init__(self, size=(4, 3, 2)):
        import mumaxplus_b200 as mpx

        self.grid = mpx.Grid(size)
        self.name = "fake"
        self._regions = None
        self.changes = 0
        nx, ny, nz = size
        idx = np.flip(np.mgrid[0:nz, 0:ny, 0:nx], axis=0)
        self.meshgrid = np.array([idx[c] * 1e-9 for c in range(3)])

    def _geometry_mask(self):
        return None

    def touch(self):
        self.changes += 1


def test_parameter_set_semantics():
    import mumaxplus_b200 as mpx

    fm = _FakeMagnet()
    p = mpx.Parameter(fm, "msat", "A/m", 1, 1.0, fm.touch)
    assert p.is_uniform and p.uniform_value == 1.0
    p.set(8e5)
    assert p.eval().shape == (1, 2, 3, 4) and np.all(p.eval() == 8e5)
    arr = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    p.set(arr)
    assert not p.is_uniform and np.array_equal(p.eval()[0], arr)
    p.set(lambda x, y, z: x * 1e9)  # function of position
    assert p.eval()[0, 0, 0, 3] == pytest.approx(3.0)
    with pytest.raises(NotImplementedError):
        p.set(lambda t: 1.0)  # time-dependent term
    with pytest.raises(ValueError):
        p.set(np.zeros((3, 3, 3), np.float32))
    v = mpx.Parameter(fm, "anisU", "", 3, (0, 0, 0), fm.touch)
    v.set((0, 0, 1))
    assert v.eval()[2].min() == 1.0
    assert fm.changes == 4


def test_interparameter_lut_index():
    import mumaxplus_b200 as mpx

    fm = _FakeMagnet()
    fm._regions = np.array([0, 1, 2, 3], dtype=np.uint32)
    ip = mpx.InterParameter(fm, "inter_exchange", "J/m", 0.0, fm.touch)
    ip.set_between(3, 1, 7.0)
    ip.set_between(0, 2, 5.0)
    lut = ip._lut()
    # core/inter_parameter.hpp getLutIndex: i(i-1)/2 + j for i > j
    assert lut[3 * 2 // 2 + 1] == 7.0
    assert lut[2 * 1 // 2 + 0] == 5.0
    assert ip.get_between(1, 3) == 7.0 and ip.get_between(1, 2) == 0.0


def test_dmi_tensor_helpers():
    import mumaxplus_b200 as mpx

    fm = _FakeMagnet()
    t = mpx.DmiTensor(fm, fm.touch)
    t.set_interfacial_dmi(3e-3)
    assert t.xxz.uniform_value == 3e-3 and t.yyz.uniform_value == 3e-3 and t.xyz.uniform_value == 0
    t.set_bulk_dmi(2e-3)
    assert t.xyz.uniform_value == 2e-3 and t.yxz.uniform_value == -2e-3 and t.zxy.uniform_value == 2e-3
    assert t.xxz.uniform_value == 0


def test_grid_semantics():
    import mumaxplus_b200 as mpx

    g = mpx.Grid((4, 5, 6), (1, 2, 3))
    assert g.shape == (6, 5, 4) and g.ncells == 120
    assert g == mpx.Grid((4, 5, 6), (1, 2, 3)) and g != mpx.Grid((4, 5, 6))
    assert g.overlaps(mpx.Grid((2, 2, 2), (4, 6, 8)))
    assert not g.overlaps(mpx.Grid((2, 2, 2), (5, 2, 3)))
    with pytest.raises(ValueError):
        mpx.Grid((1, 2))


def test_solve_takes_device_sampling_only_for_magnetization_averages():
    """TimeSolver.solve uses the device-sampled table (mpx_solver_run_sampled) when every quantity is the bound
    average of the magnetization of a magnet of this world; any other callable keeps the host loop."""
    import mumaxplus_b200 as mpx
    from mumaxplus_b200 import _abi
    from mumaxplus_b200.fieldquantity import FieldQuantity
    from mumaxplus_b200.parameter import Variable
    from mumaxplus_b200.timesolver import TimeSolver

    class _World:
        pass

    w = _World()
    a, b, stranger = _FakeMagnet(), _FakeMagnet(), _FakeMagnet()
    w._magnets = {"a": a, "b": b}
    ts = TimeSolver(w)
    cols = ts._magnetization_columns({"ma": Variable(a).average, "mb": Variable(b).average,
                                      "fa": FieldQuantity(a, _abi.Q_MAGNETIZATION, "m", "").average})
    assert cols == {"ma": 1, "mb": 4, "fa": 1}
    assert ts._magnetization_columns({}) == {}
    assert ts._magnetization_columns({"m": lambda: Variable(a).average()}) is None
    assert ts._magnetization_columns({"m": Variable(stranger).average}) is None
    assert ts._magnetization_columns({"h": FieldQuantity(a, _abi.Q_DEMAG_FIELD, "h", "T").average}) is None
    assert ts._magnetization_columns({"m": Variable(a).average, "e": Variable(a).get}) is None
    assert mpx.TimeSolver is TimeSolver


def test_checked_build_command_defines_the_check():
    import importlib.util

    spec = importlib.util.spec_from_file_location("_mpx_build", os.path.join(ROOT, "mumax-plus_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    plain, checked = mod._command(mod.OUT, ()), mod._command(mod.OUT_CHECKED, ())
    assert "-DMPX_BOUNDS_CHECK" in checked and "-DMPX_BOUNDS_CHECK" not in plain
    for cmd in (plain, checked):
        assert "arch=compute_100a,code=sm_100a" in cmd
    assert [a for a in plain if a != mod.OUT] == [a for a in checked if a not in (mod.OUT_CHECKED, "-DMPX_BOUNDS_CHECK")]


def test_grid_argument_validation():
    """test/test_grid.py:7-56: integer sizes >= 0 and integer origins of three components; anything else is a
    ValueError or TypeError."""
    import mumaxplus_b200 as mpx

    for size in [(1, 1, 1), [12, 5, 1], (3, 1, 64), (0, 0, 0)]:
        for origin in [(-2, 7, 0), (0, 0, 0)]:
            g = mpx.Grid(size, origin)
            assert g.size == tuple(size) and g.origin == tuple(origin)
        assert mpx.Grid(size).origin == (0, 0, 0)
    assert mpx.Grid(tuple(np.array([4, 2, 1]))).size == (4, 2, 1)  # numpy integers are integers
    for size in [(2, -1, 1), [-3, 4, 4], (2.5, 3.0, 1.0), (4, 4), 7, (1, 2, 3, 4), "xy"]:
        with pytest.raises((ValueError, TypeError)):
            mpx.Grid(size)
        with pytest.raises((ValueError, TypeError)):
            mpx.Grid(size, (1, 1, 1))
    for origin in [(0, 1.5, 0), (3, 3), 1]:
        with pytest.raises((ValueError, TypeError)):
            mpx.Grid((2, 2, 2), origin)


def test_geometry_and_region_masks():
    """test/test_geometry.py:8-56 on the host-side mask conversion of Ferromagnet (no device): an array of the
    grid shape or a function of (x, y, z) at the cell positions origin + index * cellsize; a wrong shape is a
    ValueError, a function of the wrong arity a TypeError, negative region indices a ValueError."""
    import mumaxplus_b200 as mpx
    from mumaxplus_b200.ferromagnet import Ferromagnet

    class _World:
        cellsize = (3e-9, 4e-9, 5e-9)

    fm = Ferromagnet.__new__(Ferromagnet)
    fm._world, fm._grid = _World(), mpx.Grid((32, 16, 3), (2, -1, 0))
    nx, ny, nz = fm._grid.size
    geom = np.random.default_rng(4).uniform(size=(nz, ny, nx)) > 0.3
    assert np.array_equal(fm._mask(geom, "geometry").astype(bool), geom)
    f = lambda x, y, z: x**2 + y**2 < (40e-9) ** 2  # noqa: E731
    X, Y, Z = fm.meshgrid
    assert X[0, 0, 1] == pytest.approx(3 * 3e-9) and Y[0, 0, 0] == pytest.approx(-4e-9)
    assert np.array_equal(fm._mask(f, "geometry").astype(bool), X**2 + Y**2 < (40e-9) ** 2)
    with pytest.raises(ValueError):
        fm._mask(np.ones((nz, ny, nx + 1), bool), "geometry")
    with pytest.raises(TypeError):
        fm._mask(lambda x, y: True, "geometry")
    regions = np.arange(nx * ny * nz).reshape(nz, ny, nx) % 5
    assert np.array_equal(fm._mask(regions, "regions"), regions)
    with pytest.raises(ValueError):
        fm._mask(-regions - 1, "regions")
