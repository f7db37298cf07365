"""FieldQuantity / ScalarQuantity (mirror of mumaxplus/fieldquantity.py and
mumaxplus/scalarquantity.py).  Each quantity is evaluated by the CUDA engine
through mpx_eval / mpx_average / mpx_energy (core/fieldquantity.hpp:29-30)."""
import time as _time

import numpy as _np


class FieldQuantity:
    """A field quantity of a magnet, evaluated on the GPU."""

    def __init__(self, magnet, quantity, name, unit, ncomp=3):
        self._magnet = magnet
        self._q = quantity
        self._name = name
        self._unit = unit
        self._ncomp = ncomp

    def __repr__(self):
        return (f"FieldQuantity(grid={self.grid}, name='{self.name}', "
                f"ncomp={self.ncomp}, unit={self.unit})")

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
        return (self.ncomp, *self.grid.shape)

    def eval(self):
        """Evaluate the quantity: numpy array (ncomp, nz, ny, nx), float32."""
        m = self._magnet
        return m._engine.eval(m._id, self._q, self.shape)

    def __call__(self):
        return self.eval()

    def average(self):
        """Per-component mean over the cells in the geometry (FP64 accumulation)."""
        m = self._magnet
        return m._engine.average(m._id, self._q)[: self.ncomp]

    @property
    def meshgrid(self):
        """x, y, z coordinate of every cell: array (3, nz, ny, nx)."""
        return self._magnet.meshgrid

    def _bench(self, ntimes=100):
        """Mean wall time of one evaluation (mumaxplus/fieldquantity.py:111-118)."""
        m = self._magnet
        start = _time.time()
        for _ in range(ntimes):
            m._engine.eval_only(m._id, self._q)
        stop = _time.time()
        return (stop - start) / ntimes


class ScalarQuantity:
    """A scalar quantity of a magnet (energies, max torque)."""

    def __init__(self, func, name, unit):
        self._func = func
        self._name = name
        self._unit = unit

    def __repr__(self):
        return f"ScalarQuantity(name='{self._name}', unit={self._unit})"

    @property
    def name(self):
        return self._name

    @property
    def unit(self):
        return self._unit

    def eval(self):
        return self._func()

    def __call__(self):
        return self.eval()
