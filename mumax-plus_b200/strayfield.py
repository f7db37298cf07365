"""StrayField (mirror of mumaxplus/strayfield.py, bindings/wrap_strayfield.cpp).

The field (T) of a magnet's current magnetisation on a grid: the magnet's own
grid (its demag field, Magnet.demag_field), any other grid of the world
(StrayField(magnet, grid)), or another magnet's grid with that magnet's
geometry (Magnet.stray_field_from_magnet).  Two methods, as in the reference:
"fft" (default, FFT convolution) and "brute" (direct sum over the source
cells); both include the world's periodic images.
"""
import ctypes as _C

import numpy as _np

from . import _abi
from ._engine import check as _check
from ._engine import lib as _lib
from .fieldquantity import FieldQuantity
from .grid import Grid


class StrayField(FieldQuantity):
    """Stray field of `magnet` evaluated on `grid` (physics/strayfield.cpp:45-82)."""

    def __init__(self, magnet, grid):
        if not isinstance(grid, Grid):
            raise TypeError("grid should be a Grid")
        super().__init__(magnet, _abi.Q_DEMAG_FIELD, "stray_field", "T", 3)
        self._grid = Grid(grid.size, grid.origin)
        self._method = "fft"
        self._dst_magnet = None  # set by Magnet.stray_field_from_magnet

    @classmethod
    def _between(cls, source, destination):
        sf = cls(source, destination.grid)
        sf._dst_magnet = destination
        return sf

    def __repr__(self):
        return f"StrayField(source={self._magnet.name}, grid={self._grid}, method='{self._method}')"

    @property
    def name(self):
        return f"{self._magnet.name}:stray_field"

    @property
    def grid(self):
        return self._grid

    @property
    def source(self):
        return self._magnet

    def set_method(self, method):
        """'fft' (default) or 'brute' (bindings/wrap_strayfield.cpp:16-24)."""
        if method not in ("fft", "brute"):
            raise ValueError('Method should be "fft" or "brute"')
        self._method = method

    def eval(self):
        """The field on the grid: numpy array (3, nz, ny, nx), float32."""
        m = self._magnet
        own = self._dst_magnet is None and self._grid == m.grid and self._method == "fft"
        if own:  # the magnet's demag field: the fused FFT passes of its own evaluation
            return super().eval()
        out = _np.empty((3, *self._grid.shape), dtype=_np.float32)
        size = (_C.c_int * 3)(*self._grid.size)
        origin = (_C.c_int * 3)(*self._grid.origin)
        dst = -1 if self._dst_magnet is None else self._dst_magnet._id
        method = _abi.MPX_STRAY_FFT if self._method == "fft" else _abi.MPX_STRAY_BRUTE
        _check(_lib().mpx_stray_field(m._engine.handle, m._id, int(dst), size, origin, method, out.ctypes.data, 0))
        return out

    def average(self):
        g = self.eval().astype(_np.float64)
        return tuple(float(v) for v in g.reshape(3, -1).mean(axis=1))
