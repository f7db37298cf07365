"""Ferromagnet (mirror of mumaxplus/ferromagnet.py and mumaxplus/magnet.py).

The parameter bag follows physics/ferromagnet.cpp:18-60 (defaults msat = 1,
everything else 0, scale_exchange = 1, demag on, open boundaries off).  Every
quantity is evaluated by the CUDA engine; parameters of terms outside the
accelerated path (spin-transfer torque, temperature, magnetoelastics, ...)
raise NotImplementedError when set to non-zero values.
"""
import ctypes as C
import os as _os
import warnings

import numpy as _np

from . import _abi
from .fieldquantity import FieldQuantity, ScalarQuantity
from .grid import Grid
from .parameter import DmiTensor, InterParameter, Parameter, Variable

GAMMALL = 1.7595e11


class _Unsupported(Parameter):
    """A reference parameter whose physics is outside the accelerated path."""

    def set(self, value):
        if isinstance(value, (int, float)) and value == 0:
            return
        if isinstance(value, tuple) and all(isinstance(v, (int, float)) and v == 0 for v in value):
            return
        raise NotImplementedError(f"'{self._name}' is outside the accelerated effective-field path")


class Ferromagnet:
    """A ferromagnet on `grid` in `world` (physics/mumaxworld.cpp:57-80).

    geometry / regions: None, an array of the grid shape, or a function of the
    cell position (x, y, z) (mumaxplus/magnet.py:46-77).
    """

    def __init__(self, world, grid, name="", geometry=None, regions=None):
        self._world = world
        self._grid = Grid(grid.size, grid.origin)
        world._check_addibility(self._grid, name)
        if not name:
            name = world._next_name()
        self._name = name
        self._geometry = self._mask(geometry, "geometry")
        self._regions = self._mask(regions, "regions")
        self._engine = world._engine
        self._group = world._group
        self._relax_threshold = -1.0
        self._stray_source = True
        self._stray_destination = True
        self._suspend = True
        ch = self._update
        self._msat = Parameter(self, "msat", "A/m", 1, 1.0, ch)
        self._aex = Parameter(self, "aex", "J/m", 1, 0.0, ch)
        self._alpha = Parameter(self, "alpha", "", 1, 0.0, ch)
        self._ku1 = Parameter(self, "ku1", "J/m3", 1, 0.0, ch)
        self._ku2 = Parameter(self, "ku2", "J/m3", 1, 0.0, ch)
        self._anisU = Parameter(self, "anisU", "", 3, (0.0, 0.0, 0.0), ch)
        self._bias = Parameter(self, "bias_magnetic_field", "T", 3, (0.0, 0.0, 0.0), ch)
        self._frozen = Parameter(self, "frozen_spins", "", 1, 0.0, ch)
        self._kc1 = Parameter(self, "kc1", "J/m3", 1, 0.0, ch)
        self._kc2 = Parameter(self, "kc2", "J/m3", 1, 0.0, ch)
        self._kc3 = Parameter(self, "kc3", "J/m3", 1, 0.0, ch)
        self._anisC1 = Parameter(self, "anisC1", "", 3, (0.0, 0.0, 0.0), ch)
        self._anisC2 = Parameter(self, "anisC2", "", 3, (0.0, 0.0, 0.0), ch)
        # spin-transfer torque (physics/ferromagnet.cpp:34-52 defaults)
        self._pol = Parameter(self, "pol", "", 1, 0.0, ch)
        self._xi = Parameter(self, "xi", "", 1, 0.0, ch)
        self._Lambda = Parameter(self, "Lambda", "", 1, 0.0, ch)
        self._epsilon_prime = Parameter(self, "epsilon_prime", "", 1, 0.0, ch)
        self._jcur = Parameter(self, "jcur", "A/m2", 3, (0.0, 0.0, 0.0), ch)
        self._fixed_layer = Parameter(self, "fixed_layer", "", 3, (0.0, 0.0, 0.0), ch)
        self._free_layer_thickness = Parameter(self, "free_layer_thickness", "m", 1,
                                               float(self._grid.size[2] * world.cellsize[2]), ch)
        self._temperature = Parameter(self, "temperature", "K", 1, 0.0, ch)
        # the reference seeds its generator from the clock (ferromagnet.cpp:79-81)
        self._thermal_seed = int.from_bytes(_os.urandom(8), "little")
        self._fixed_layer_on_top = True
        self._enable_zhang_li = True
        self._enable_slonczewski = True
        self._dmi = DmiTensor(self, ch)
        self._inter_exchange = InterParameter(self, "inter_exchange", "J/m", 0.0, ch)
        self._scale_exchange = InterParameter(self, "scale_exchange", "", 1.0, ch)
        self._enable_demag = True
        self._enable_openbc = False
        self._unsupported = {}
        for n, nc in (("B1", 1), ("B2", 1), ("conductivity", 1), ("amr_ratio", 1)):
            self._unsupported[n] = _Unsupported(self, n, "", nc, (0.0, 0.0, 0.0) if nc == 3 else 0.0)
        self._suspend = False
        self._id = self._engine.magnet_add(self._group, self._desc())
        world._register(self)

    def __repr__(self):
        return f"Ferromagnet(grid={self.grid}, name='{self.name}')"

    # ------------------------------------------------------------- helpers
    def _mask(self, value, kind):
        if value is None:
            return None
        T = bool if kind == "geometry" else int
        if callable(value):
            X, Y, Z = self.meshgrid
            arr = _np.vectorize(value, otypes=[T])(X, Y, Z)
        else:
            arr = _np.array(value, dtype=T)
        if arr.shape != self._grid.shape:
            raise ValueError(f"The dimensions of the {kind} do not match the dimensions of the grid.")
        if kind == "geometry":
            return _np.ascontiguousarray(arr.astype(_np.uint8))
        if (arr < 0).any():
            raise ValueError("region indices must be non-negative")
        return _np.ascontiguousarray(arr.astype(_np.uint32))

    def _geometry_mask(self):
        return None if self._geometry is None else self._geometry.astype(bool)

    def _desc(self):
        keep = []
        d = _abi.MagnetDesc()
        w = self._world
        for a in range(3):
            d.size[a] = self._grid.size[a]
            d.origin[a] = self._grid.origin[a]
            d.cellsize[a] = float(w.cellsize[a])
            d.mastergrid_size[a] = w.mastergrid.size[a]
            d.mastergrid_origin[a] = w.mastergrid.origin[a]
            d.pbc_repetitions[a] = w.pbc_repetitions[a]
        if self._geometry is not None:
            keep.append(self._geometry)
            d.geometry = self._geometry.ctypes.data_as(C.POINTER(C.c_ubyte))
        if self._regions is not None:
            keep.append(self._regions)
            d.regions = self._regions.ctypes.data_as(C.POINTER(C.c_uint))
        d.msat = self._msat._scalar(keep)
        d.aex = self._aex._scalar(keep)
        d.alpha = self._alpha._scalar(keep)
        d.ku1 = self._ku1._scalar(keep)
        d.ku2 = self._ku2._scalar(keep)
        d.frozen_spins = self._frozen._scalar(keep)
        d.anis_u = self._anisU._vector(keep)
        d.bias_magnetic_field = self._bias._vector(keep)
        d.kc1 = self._kc1._scalar(keep)
        d.kc2 = self._kc2._scalar(keep)
        d.kc3 = self._kc3._scalar(keep)
        d.anis_c1 = self._anisC1._vector(keep)
        d.anis_c2 = self._anisC2._vector(keep)
        d.pol = self._pol._scalar(keep)
        d.xi = self._xi._scalar(keep)
        d.lambda_ = self._Lambda._scalar(keep)
        d.epsilon_prime = self._epsilon_prime._scalar(keep)
        d.free_layer_thickness = self._free_layer_thickness._scalar(keep)
        d.jcur = self._jcur._vector(keep)
        d.fixed_layer = self._fixed_layer._vector(keep)
        d.fixed_layer_below = 0 if self._fixed_layer_on_top else 1
        d.zhang_li_off = 0 if self._enable_zhang_li else 1
        d.temperature = self._temperature._scalar(keep)
        d.thermal_seed = self._thermal_seed
        d.slonczewski_off = 0 if self._enable_slonczewski else 1
        d.stray_source_off = 0 if self._stray_source else 1
        d.stray_destination_off = 0 if self._stray_destination else 1
        for i, p in enumerate(self._dmi._list()):
            d.dmi[i] = p._scalar(keep)
        li, ls = self._inter_exchange._lut(), self._scale_exchange._lut()
        nreg = 0
        for lut in (li, ls):
            if lut is not None:
                n = int(round((1 + (1 + 8 * len(lut)) ** 0.5) / 2))
                nreg = max(nreg, n)
        if nreg:
            li = li if li is None or len(li) == nreg * (nreg - 1) // 2 else _pad_lut(li, nreg, self._inter_exchange._uniform)
            ls = ls if ls is None or len(ls) == nreg * (nreg - 1) // 2 else _pad_lut(ls, nreg, self._scale_exchange._uniform)
        d.lut_regions = nreg
        d.inter_exchange = self._inter_exchange._uniform
        d.scale_exchange = self._scale_exchange._uniform
        if li is not None:
            keep.append(li)
            d.inter_exchange_lut = li.ctypes.data_as(C.POINTER(C.c_float))
        if ls is not None:
            keep.append(ls)
            d.scale_exchange_lut = ls.ctypes.data_as(C.POINTER(C.c_float))
        d.enable_demag = 1 if self._enable_demag else 0
        d.enable_openbc = 1 if self._enable_openbc else 0
        d._keep = keep  # keep the arrays alive while the struct is in use
        return d

    def _update(self):
        if self._suspend:
            return
        self._engine.magnet_update(self._id, self._desc())

    def _q(self, quantity, name, unit, ncomp=3):
        return FieldQuantity(self, quantity, name, unit, ncomp)

    # ------------------------------------------------------------- identity
    @property
    def name(self):
        return self._name

    @property
    def grid(self):
        return self._grid

    @property
    def cellsize(self):
        return self._world.cellsize

    @property
    def world(self):
        return self._world

    @property
    def geometry(self):
        if self._geometry is None:
            return _np.ones(self._grid.shape, dtype=bool)
        return self._geometry.astype(bool)

    @property
    def regions(self):
        if self._regions is None:
            return _np.zeros(self._grid.shape, dtype=_np.uint32)
        return self._regions.copy()

    @property
    def origin(self):
        """Position of the first cell (core/system.cpp:48-56)."""
        return tuple(self._grid.origin[a] * self.cellsize[a] for a in range(3))

    @property
    def center(self):
        o, s, c = self._grid.origin, self._grid.size, self.cellsize
        return tuple(((o[a] + s[a] - 1) * c[a] + o[a] * c[a]) / 2 for a in range(3))

    @property
    def meshgrid(self):
        nx, ny, nz = self._grid.size
        cs = self.cellsize
        idx = _np.flip(_np.mgrid[0:nz, 0:ny, 0:nx], axis=0)
        return _np.array([(self._grid.origin[c] + idx[c]) * cs[c] for c in range(3)])

    @property
    def is_sublattice(self):
        return False

    # ------------------------------------------------------------- state
    @property
    def magnetization(self):
        return Variable(self)

    @magnetization.setter
    def magnetization(self, value):
        Variable(self).set(value)

    @property
    def enable_demag(self):
        return self._enable_demag

    @enable_demag.setter
    def enable_demag(self, value):
        self._enable_demag = bool(value)
        self._update()

    @property
    def enable_openbc(self):
        return self._enable_openbc

    @enable_openbc.setter
    def enable_openbc(self, value):
        self._enable_openbc = bool(value)
        self._update()

    # ------------------------------------------------------------- parameters
    def _param_prop(attr):
        def getter(self):
            return getattr(self, attr)

        def setter(self, value):
            getattr(self, attr).set(value)

        return property(getter, setter)

    msat = _param_prop("_msat")
    aex = _param_prop("_aex")
    alpha = _param_prop("_alpha")
    ku1 = _param_prop("_ku1")
    ku2 = _param_prop("_ku2")
    anisU = _param_prop("_anisU")
    kc1 = _param_prop("_kc1")
    pol = _param_prop("_pol")
    temperature = _param_prop("_temperature")
    xi = _param_prop("_xi")
    Lambda = _param_prop("_Lambda")
    epsilon_prime = _param_prop("_epsilon_prime")
    jcur = _param_prop("_jcur")
    fixed_layer = _param_prop("_fixed_layer")
    free_layer_thickness = _param_prop("_free_layer_thickness")
    kc2 = _param_prop("_kc2")
    kc3 = _param_prop("_kc3")
    anisC1 = _param_prop("_anisC1")
    anisC2 = _param_prop("_anisC2")
    bias_magnetic_field = _param_prop("_bias")
    frozen_spins = _param_prop("_frozen")

    @property
    def dmi_tensor(self):
        return self._dmi

    @property
    def inter_exchange(self):
        return self._inter_exchange

    @inter_exchange.setter
    def inter_exchange(self, value):
        self._inter_exchange.set(value)

    @property
    def scale_exchange(self):
        return self._scale_exchange

    @scale_exchange.setter
    def scale_exchange(self, value):
        self._scale_exchange.set(value)

    # ------------------------------------------------------------- quantities
    @property
    def effective_field(self):
        return self._q(_abi.Q_EFFECTIVE_FIELD, "effective_field", "T")

    @property
    def exchange_field(self):
        return self._q(_abi.Q_EXCHANGE_FIELD, "exchange_field", "T")

    @property
    def dmi_field(self):
        return self._q(_abi.Q_DMI_FIELD, "dmi_field", "T")

    @property
    def anisotropy_field(self):
        return self._q(_abi.Q_ANISOTROPY_FIELD, "anisotropy_field", "T")

    @property
    def external_field(self):
        return self._q(_abi.Q_EXTERNAL_FIELD, "external_field", "T")

    @property
    def demag_field(self):
        from .strayfield import StrayField
        return StrayField(self, self.grid)

    def stray_field_from_magnet(self, source_magnet):
        """The field created by `source_magnet`, felt by this magnet: a
        StrayField on this magnet's grid, zero outside its geometry
        (mumaxplus/magnet.py:532-552).  The source must be in the same world."""
        from .strayfield import StrayField
        if source_magnet is self:
            return StrayField(self, self.grid)
        if getattr(source_magnet, "_world", None) is not self._world:
            raise RuntimeError("Can not compute the magnetic field of the magnet")
        return StrayField._between(source_magnet, self)

    @property
    def torque(self):
        return self._q(_abi.Q_TORQUE, "torque", "rad/s")

    @property
    def llg_torque(self):
        return self._q(_abi.Q_LLG_TORQUE, "llg_torque", "rad/s")

    @property
    def damping_torque(self):
        return self._q(_abi.Q_DAMPING_TORQUE, "damping_torque", "rad/s")

    @property
    def max_torque(self):
        return ScalarQuantity(lambda: self._engine.max_norm(self._id, _abi.Q_TORQUE), "max_torque", "rad/s")

    def _edens(self, q, name):
        return self._q(q, name, "J/m3", 1)

    def _energy(self, q, name):
        return ScalarQuantity(lambda: self._engine.energy(self._id, q), name, "J")

    @property
    def exchange_energy_density(self):
        return self._edens(_abi.Q_EXCHANGE_ENERGY_DENSITY, "exchange_energy_density")

    @property
    def exchange_energy(self):
        return self._energy(_abi.Q_EXCHANGE_ENERGY_DENSITY, "exchange_energy")

    @property
    def dmi_energy_density(self):
        return self._edens(_abi.Q_DMI_ENERGY_DENSITY, "dmi_energy_density")

    @property
    def dmi_energy(self):
        return self._energy(_abi.Q_DMI_ENERGY_DENSITY, "dmi_energy")

    @property
    def anisotropy_energy_density(self):
        return self._edens(_abi.Q_ANISOTROPY_ENERGY_DENSITY, "anisotropy_energy_density")

    @property
    def anisotropy_energy(self):
        return self._energy(_abi.Q_ANISOTROPY_ENERGY_DENSITY, "anisotropy_energy")

    @property
    def zeeman_energy_density(self):
        return self._edens(_abi.Q_ZEEMAN_ENERGY_DENSITY, "zeeman_energy_density")

    @property
    def zeeman_energy(self):
        return self._energy(_abi.Q_ZEEMAN_ENERGY_DENSITY, "zeeman_energy")

    @property
    def demag_energy_density(self):
        return self._edens(_abi.Q_DEMAG_ENERGY_DENSITY, "demag_energy_density")

    @property
    def demag_energy(self):
        return self._energy(_abi.Q_DEMAG_ENERGY_DENSITY, "demag_energy")

    @property
    def total_energy_density(self):
        return self._edens(_abi.Q_TOTAL_ENERGY_DENSITY, "total_energy_density")

    @property
    def total_energy(self):
        return self._energy(_abi.Q_TOTAL_ENERGY_DENSITY, "total_energy")

    # ------------------------------------------------------------- energy minima
    def minimize(self, tol=1e-6, nsamples=10):
        """Minimize the total energy (mumaxplus/ferromagnet.py:144-164): steepest
        descent on the damping torque with Barzilai-Borwein steps until the last
        `nsamples` largest changes of m are all <= tol.  In a world with several
        magnets every magnet of the world takes part."""
        self._engine.minimize(self._group, tol, nsamples)

    def relax(self, tol=1e-9):
        """Relax to an energy minimum (mumaxplus/ferromagnet.py:166-192): time
        evolution without precession while the energy decreases, then while the
        torque decreases, lowering the solver's maximum error down to `tol`."""
        if tol >= 1e-5:
            warnings.warn("The set tolerance is greater than or equal to the default value"
                           + " used for the timesolver (1e-5). Using this value results"
                           + " in no torque minimization, only energy minimization.", UserWarning)
        self._engine.relax(self._group, tol, self._relax_threshold)

    def _flag(name, doc):
        def getter(self):
            return getattr(self, name)

        def setter(self, value):
            setattr(self, name, bool(value))
            self._update()

        return property(getter, setter, doc=doc)

    fixed_layer_on_top = _flag("_fixed_layer_on_top", "Slonczewski fixed layer above the free layer (default True).")
    enable_zhang_li_torque = _flag("_enable_zhang_li", "Zhang-Li spin-transfer torque on (default True).")
    enable_slonczewski_torque = _flag("_enable_slonczewski", "Slonczewski spin-transfer torque on (default True).")

    @property
    def thermal_seed(self):
        """Seed of the thermal-noise generator (random at creation; set it for
        reproducible runs).  The noise of a step is a function of the seed, the
        step count, the cell and the component."""
        return self._thermal_seed

    @thermal_seed.setter
    def thermal_seed(self, value):
        self._thermal_seed = int(value) & 0xFFFFFFFFFFFFFFFF
        self._update()

    @property
    def spin_transfer_torque(self):
        """Spin-transfer torque (1/s), physics/stt.cu:143-185."""
        return self._q(_abi.Q_SPIN_TRANSFER_TORQUE, "spintransfer_torque", "1/s")

    @property
    def enable_as_stray_field_source(self):
        """Whether this magnet's stray field acts on the other magnets of the
        world (mumaxplus/magnet.py:155-172; default True)."""
        return self._stray_source

    @enable_as_stray_field_source.setter
    def enable_as_stray_field_source(self, value):
        self._stray_source = bool(value)
        self._update()

    @property
    def enable_as_stray_field_destination(self):
        """Whether the stray fields of the other magnets of the world act on
        this magnet (default True)."""
        return self._stray_destination

    @enable_as_stray_field_destination.setter
    def enable_as_stray_field_destination(self, value):
        self._stray_destination = bool(value)
        self._update()

    @property
    def RelaxTorqueThreshold(self):
        """Threshold torque for relax (default -1: relax until the torque is
        steady or increasing; positive: until the max torque is <= it)."""
        return self._relax_threshold

    @RelaxTorqueThreshold.setter
    def RelaxTorqueThreshold(self, value):
        assert value != 0, "The relax threshold should not be zero."
        self._relax_threshold = float(value)


def _pad_lut(lut, n, uniform):
    out = _np.full(n * (n - 1) // 2, uniform, dtype=_np.float32)
    out[: len(lut)] = lut
    return out


def _unsupported_prop(name):
    def getter(self):
        return self._unsupported[name]

    def setter(self, value):
        self._unsupported[name].set(value)

    return property(getter, setter)


for _n in ("B1", "B2", "conductivity", "amr_ratio"):
    setattr(Ferromagnet, _n, _unsupported_prop(_n))
