"""Parameter, InterParameter, DmiTensor and Variable (mirrors of
mumaxplus/parameter.py, interparameter.py, dmitensor.py and variable.py).

Parameter values live on the host until they change; every change re-sends the
magnet's description to the engine (mpx_magnet_update), which uploads uniform
values as constants and per-cell values as device arrays
(core/parameter.hpp:16-240 keeps the same uniform-or-per-cell split).
"""
import ctypes as C

import numpy as _np

from . import _abi


class Parameter:
    """A material parameter of a magnet: uniform, or one value per cell."""

    def __init__(self, magnet, name, unit, ncomp=1, default=0.0, on_change=None):
        self._magnet = magnet
        self._name = name
        self._unit = unit
        self._ncomp = ncomp
        self._default = default
        self._uniform = tuple(float(v) for v in default) if ncomp == 3 else float(default)
        self._cells = None
        self._on_change = on_change

    def __repr__(self):
        return (f"Parameter(grid={self.grid}, name='{self.name}', "
                f"ncomp={self.ncomp}, unit={self.unit})")

    # -- FieldQuantity-like surface
    @property
    def name(self):
        return f"{self._magnet.name}:{self._name}"

    @property
    def unit(self):
        return self._unit

    @property
    def ncomp(self):
        return self._ncomp

    @property
    def grid(self):
        return self._magnet.grid

    @property
    def shape(self):
        return (self._ncomp, *self.grid.shape)

    @property
    def meshgrid(self):
        return self._magnet.meshgrid

    @property
    def is_uniform(self):
        return self._cells is None

    @property
    def is_dynamic(self):
        return False

    @property
    def uniform_value(self):
        return self._uniform

    @uniform_value.setter
    def uniform_value(self, value):
        self.set(value)

    def eval(self):
        """Values in every cell: array (ncomp, nz, ny, nx), float32."""
        if self._cells is not None:
            return self._cells.copy()
        out = _np.empty(self.shape, dtype=_np.float32)
        if self._ncomp == 1:
            out[0] = self._uniform
        else:
            for c in range(3):
                out[c] = self._uniform[c]
        return out

    def __call__(self):
        return self.eval()

    def average(self):
        vals = self.eval().astype(_np.float64)
        geo = self._magnet._geometry_mask()
        if geo is None:
            return [float(v.mean()) for v in vals]
        n = max(int(geo.sum()), 1)
        return [float(v[geo].sum() / n) for v in vals]

    def _assured_zero(self):
        if self._cells is not None:
            return False
        return all(v == 0 for v in (self._uniform if self._ncomp == 3 else (self._uniform,)))

    # -- setting
    def set(self, value):
        """Uniform value (float, or 3-tuple for vectors), a numpy array of the
        grid shape, or a function of the cell position (x, y, z)."""
        if callable(value):
            try:
                value(0)
                is_time = True
            except TypeError:
                is_time = False
            if is_time:
                raise NotImplementedError(
                    "time-dependent parameter terms are not part of the accelerated path")
            X, Y, Z = self.meshgrid
            vals = _np.vectorize(value, otypes=[float] * self._ncomp)(X, Y, Z)
            self._set_array(_np.array(vals if self._ncomp == 3 else [vals]))
        elif isinstance(value, tuple) and len(value) > 0 and callable(value[0]):
            raise NotImplementedError("time-dependent parameter terms are not part of the accelerated path")
        elif isinstance(value, _np.ndarray) and value.ndim >= 3:
            self._set_array(value)
        elif self._ncomp == 1:
            self._cells = None
            self._uniform = float(value)
        else:
            v = tuple(float(x) for x in value)
            if len(v) != 3:
                raise ValueError("a vector parameter needs three values")
            self._cells = None
            self._uniform = v
        self._changed()

    def _set_array(self, arr):
        arr = _np.asarray(arr, dtype=_np.float32)
        want = self.shape
        if arr.shape == want[1:] and self._ncomp == 1:
            arr = arr[None]
        if arr.shape != want:
            raise ValueError(f"The shape of the data {arr.shape} does not match the shape {want}")
        self._cells = _np.ascontiguousarray(arr)

    def set_in_region(self, region_idx, value):
        """Set a uniform value in the cells of one region."""
        regions = self._magnet._regions
        if regions is None:
            regions = _np.zeros(self.grid.shape, dtype=_np.uint32)
        cells = self.eval()
        sel = regions == int(region_idx)
        if self._ncomp == 1:
            cells[0][sel] = float(value)
        else:
            for c in range(3):
                cells[c][sel] = float(value[c])
        self._cells = _np.ascontiguousarray(cells)
        self._changed()

    def add_time_term(self, term, mask=None):
        raise NotImplementedError("time-dependent parameter terms are not part of the accelerated path")

    def remove_time_terms(self):
        pass

    def _changed(self):
        if self._on_change is not None:
            self._on_change()

    # -- C description
    def _scalar(self, keep):
        s = _abi.Scalar()
        s.uniform = float(self._uniform) if self._ncomp == 1 else 0.0
        if self._cells is not None:
            a = _np.ascontiguousarray(self._cells.reshape(-1), dtype=_np.float32)
            keep.append(a)
            s.cells = a.ctypes.data_as(C.POINTER(C.c_float))
        return s

    def _vector(self, keep):
        v = _abi.Vector()
        for c in range(3):
            v.uniform[c] = float(self._uniform[c])
        if self._cells is not None:
            a = _np.ascontiguousarray(self._cells.reshape(-1), dtype=_np.float32)
            keep.append(a)
            v.cells = a.ctypes.data_as(C.POINTER(C.c_float))
        return v


class InterParameter:
    """Inter-region parameter (inter_exchange, scale_exchange):
    core/inter_parameter.hpp:14-91, LUT index i(i-1)/2 + j."""

    def __init__(self, magnet, name, unit, default, on_change=None):
        self._magnet = magnet
        self._name = name
        self._unit = unit
        self._uniform = float(default)
        self._pairs = {}
        self._on_change = on_change

    def __repr__(self):
        return f"InterParameter(name='{self.name}', unit={self.unit})"

    @property
    def name(self):
        return f"{self._magnet.name}:{self._name}"

    @property
    def unit(self):
        return self._unit

    @property
    def ncomp(self):
        return 1

    @property
    def region_indices(self):
        r = self._magnet._regions
        return sorted(set(_np.unique(r).tolist())) if r is not None else [0]

    @property
    def number_of_regions(self):
        return len(self.region_indices)

    @property
    def is_uniform(self):
        return not self._pairs

    @property
    def uniform_value(self):
        return self._uniform

    @uniform_value.setter
    def uniform_value(self, value):
        self.set(value)

    def set(self, value):
        assert isinstance(value, (float, int)), "The value should be uniform and static."
        self._uniform = float(value)
        self._pairs = {}
        if self._on_change:
            self._on_change()

    def set_between(self, i, j, value):
        if i == j:
            raise ValueError("Can not set the value between a region and itself.")
        self._pairs[(max(i, j), min(i, j))] = float(value)
        if self._on_change:
            self._on_change()

    def get_between(self, i, j):
        return self._pairs.get((max(i, j), min(i, j)), self._uniform)

    def eval(self):
        return self._lut()

    def _lut(self):
        if not self._pairs:
            return None
        n = max(max(self.region_indices), max(max(p) for p in self._pairs)) + 1
        lut = _np.full(n * (n - 1) // 2, self._uniform, dtype=_np.float32)
        for (i, j), v in self._pairs.items():
            lut[i * (i - 1) // 2 + j] = v
        return lut


class DmiTensor:
    """The 9 independent DMI parameters D_ijk (physics/dmitensor.hpp)."""

    def __init__(self, magnet, on_change=None):
        self._magnet = magnet
        self._params = {k: Parameter(magnet, "dmi_" + k, "J/m2", 1, 0.0, on_change) for k in _abi.DMI_ORDER}

    def make_zero(self):
        for k in _abi.DMI_ORDER:
            self._params[k]._cells = None
            self._params[k]._uniform = 0.0
        self._params["xxy"]._changed()

    def set_interfacial_dmi(self, value):
        """xxz = yyz = value, everything else zero (mumaxplus/dmitensor.py:106-124)."""
        self.make_zero()
        self.xxz.set(value)
        self.yyz.set(value)

    def set_bulk_dmi(self, value):
        """xyz = value, yxz = -value, zxy = value."""
        self.make_zero()
        self.xyz.set(value)
        if callable(value) or isinstance(value, _np.ndarray):
            self.yxz.set(-_np.asarray(self.xyz.eval()[0]))
        else:
            self.yxz.set(-value)
        self.zxy.set(value)

    @property
    def assured_zero(self):
        return all(p._assured_zero() for p in self._params.values())

    def _list(self):
        return [self._params[k] for k in _abi.DMI_ORDER]


def _dmi_property(key):
    def getter(self):
        return self._params[key]

    def setter(self, value):
        self._params[key].set(value)

    return property(getter, setter)


for _k in _abi.DMI_ORDER:
    setattr(DmiTensor, _k, _dmi_property(_k))


class Variable:
    """The magnetization m of a magnet (a normalised 3-vector field)."""

    def __init__(self, magnet):
        self._magnet = magnet

    def __repr__(self):
        return f"Variable(grid={self.grid}, name='{self.name}', ncomp=3, unit=)"

    @property
    def name(self):
        return f"{self._magnet.name}:magnetization"

    @property
    def unit(self):
        return ""

    @property
    def ncomp(self):
        return 3

    @property
    def grid(self):
        return self._magnet.grid

    @property
    def shape(self):
        return (3, *self.grid.shape)

    @property
    def meshgrid(self):
        return self._magnet.meshgrid

    def set(self, value):
        """A 3-tuple (uniform), an array (3, nz, ny, nx), or a function of (x, y, z).
        The engine normalises every cell (core/variable.cpp:76-87)."""
        if callable(value):
            X, Y, Z = self.meshgrid
            arr = _np.array(_np.vectorize(value, otypes=[float] * 3)(X, Y, Z), dtype=_np.float32)
        elif isinstance(value, _np.ndarray) and value.ndim == 4:
            arr = value
        else:
            v = [float(x) for x in value]
            if len(v) != 3:
                raise ValueError("The magnetization needs three components")
            arr = _np.empty(self.shape, dtype=_np.float32)
            for c in range(3):
                arr[c] = v[c]
        arr = _np.asarray(arr, dtype=_np.float32)
        if arr.shape != self.shape:
            raise ValueError(f"The shape of the data {arr.shape} does not match {self.shape}")
        self._magnet._engine.set_m(self._magnet._id, arr)

    def get(self):
        m = self._magnet
        return m._engine.get_m(m._id, self.shape)

    def eval(self):
        return self.get()

    def __call__(self):
        return self.get()

    def average(self):
        m = self._magnet
        return m._engine.average(m._id, _abi.Q_MAGNETIZATION)
