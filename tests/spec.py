"""A magnet problem described once and built twice: as an oracle world (through
the mpx_magnet_desc struct) and as a product World/Ferromagnet (through the
Python API that mirrors mumaxplus).  Both get the same float32 inputs."""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

import oracle as O

abi = O.abi


@dataclass
class MagnetSpec:
    size: tuple
    cellsize: tuple = (1e-9, 1e-9, 1e-9)
    origin: tuple = (0, 0, 0)
    mastergrid_size: tuple = (0, 0, 0)
    mastergrid_origin: tuple = (0, 0, 0)
    pbc: tuple = (0, 0, 0)
    geometry: object = None
    regions: object = None
    msat: object = 1.0
    aex: object = 0.0
    alpha: object = 0.0
    ku1: object = 0.0
    ku2: object = 0.0
    anisU: object = (0.0, 0.0, 0.0)
    bias: object = (0.0, 0.0, 0.0)
    kc1: object = 0.0
    kc2: object = 0.0
    kc3: object = 0.0
    anisC1: object = (0.0, 0.0, 0.0)
    anisC2: object = (0.0, 0.0, 0.0)
    stray_source: bool = True
    stray_destination: bool = True
    pol: object = 0.0
    xi: object = 0.0
    Lambda: object = 0.0
    epsilon_prime: object = 0.0
    free_layer_thickness: object = None  # None: nz * cellsize z (the reference's default)
    jcur: object = (0.0, 0.0, 0.0)
    fixed_layer: object = (0.0, 0.0, 0.0)
    fixed_layer_on_top: bool = True
    zhang_li: bool = True
    slonczewski: bool = True
    temperature: object = 0.0
    thermal_seed: int = 12345
    frozen: object = 0.0
    dmi: dict = field(default_factory=dict)
    inter_exchange: float = 0.0
    scale_exchange: float = 1.0
    inter_pairs: dict = field(default_factory=dict)
    scale_pairs: dict = field(default_factory=dict)
    enable_demag: bool = True
    enable_openbc: bool = False
    world_bias: tuple = (0.0, 0.0, 0.0)

    @property
    def shape(self):
        return (self.size[2], self.size[1], self.size[0])

    # ---------------------------------------------------------------- oracle
    def _scalar(self, v, keep):
        s = abi.Scalar()
        if isinstance(v, np.ndarray):
            a = np.ascontiguousarray(v, dtype=np.float32).reshape(-1)
            keep.append(a)
            s.cells = a.ctypes.data_as(C.POINTER(C.c_float))
        else:
            s.uniform = float(v)
        return s

    def _vector(self, v, keep):
        s = abi.Vector()
        if isinstance(v, np.ndarray):
            a = np.ascontiguousarray(v, dtype=np.float32).reshape(-1)
            keep.append(a)
            s.cells = a.ctypes.data_as(C.POINTER(C.c_float))
        else:
            for c in range(3):
                s.uniform[c] = float(v[c])
        return s

    def _lut(self, pairs, uniform):
        if not pairs:
            return None, 0
        regs = [0] if self.regions is None else list(np.unique(self.regions))
        n = int(max(max(regs), max(max(p) for p in pairs))) + 1
        lut = np.full(n * (n - 1) // 2, uniform, dtype=np.float32)
        for (i, j), v in pairs.items():
            a, b = max(i, j), min(i, j)
            lut[a * (a - 1) // 2 + b] = v
        return lut, n

    def desc(self, keep):
        d = abi.MagnetDesc()
        for a in range(3):
            d.size[a] = self.size[a]
            d.origin[a] = self.origin[a]
            d.cellsize[a] = self.cellsize[a]
            d.mastergrid_size[a] = self.mastergrid_size[a]
            d.mastergrid_origin[a] = self.mastergrid_origin[a]
            d.pbc_repetitions[a] = self.pbc[a]
        if self.geometry is not None:
            g = np.ascontiguousarray(self.geometry, dtype=np.uint8).reshape(-1)
            keep.append(g)
            d.geometry = g.ctypes.data_as(C.POINTER(C.c_ubyte))
        if self.regions is not None:
            r = np.ascontiguousarray(self.regions, dtype=np.uint32).reshape(-1)
            keep.append(r)
            d.regions = r.ctypes.data_as(C.POINTER(C.c_uint))
        d.msat = self._scalar(self.msat, keep)
        d.aex = self._scalar(self.aex, keep)
        d.alpha = self._scalar(self.alpha, keep)
        d.ku1 = self._scalar(self.ku1, keep)
        d.ku2 = self._scalar(self.ku2, keep)
        d.frozen_spins = self._scalar(self.frozen, keep)
        d.anis_u = self._vector(self.anisU, keep)
        d.kc1 = self._scalar(self.kc1, keep)
        d.kc2 = self._scalar(self.kc2, keep)
        d.kc3 = self._scalar(self.kc3, keep)
        d.anis_c1 = self._vector(self.anisC1, keep)
        d.anis_c2 = self._vector(self.anisC2, keep)
        d.pol = self._scalar(self.pol, keep)
        d.xi = self._scalar(self.xi, keep)
        d.lambda_ = self._scalar(self.Lambda, keep)
        d.epsilon_prime = self._scalar(self.epsilon_prime, keep)
        flt = self.size[2] * self.cellsize[2] if self.free_layer_thickness is None else self.free_layer_thickness
        d.free_layer_thickness = self._scalar(flt, keep)
        d.jcur = self._vector(self.jcur, keep)
        d.fixed_layer = self._vector(self.fixed_layer, keep)
        d.fixed_layer_below = 0 if self.fixed_layer_on_top else 1
        d.zhang_li_off = 0 if self.zhang_li else 1
        d.slonczewski_off = 0 if self.slonczewski else 1
        d.temperature = self._scalar(self.temperature, keep)
        d.thermal_seed = self.thermal_seed
        d.stray_source_off = 0 if self.stray_source else 1
        d.stray_destination_off = 0 if self.stray_destination else 1
        d.bias_magnetic_field = self._vector(self.bias, keep)
        for i, k in enumerate(abi.DMI_ORDER):
            d.dmi[i] = self._scalar(self.dmi.get(k, 0.0), keep)
        li, ni = self._lut(self.inter_pairs, self.inter_exchange)
        ls, ns = self._lut(self.scale_pairs, self.scale_exchange)
        n = max(ni, ns)
        if li is not None and ni < n:
            li = np.concatenate([li, np.full(n * (n - 1) // 2 - len(li), self.inter_exchange, np.float32)])
        if ls is not None and ns < n:
            ls = np.concatenate([ls, np.full(n * (n - 1) // 2 - len(ls), self.scale_exchange, np.float32)])
        d.lut_regions = n
        d.inter_exchange = self.inter_exchange
        d.scale_exchange = self.scale_exchange
        if li is not None:
            keep.append(li)
            d.inter_exchange_lut = li.ctypes.data_as(C.POINTER(C.c_float))
        if ls is not None:
            keep.append(ls)
            d.scale_exchange_lut = ls.ctypes.data_as(C.POINTER(C.c_float))
        d.enable_demag = int(self.enable_demag)
        d.enable_openbc = int(self.enable_openbc)
        return d

    def oracle_world(self, m0=None):
        w = O.OracleWorld()
        w.set_world_bias(self.world_bias)
        keep = []
        q = w.add_magnet(self.desc(keep))
        if m0 is not None:
            w.set_m(q, m0)
        return w, q

    # ---------------------------------------------------------------- product
    def product(self, mpx, m0=None, device=None):
        mg = mpx.Grid(self.mastergrid_size, self.mastergrid_origin)
        world = mpx.World(self.cellsize, pbc_repetitions=tuple(int(p) for p in self.pbc), mastergrid=mg,
                          device=device)
        magnet = mpx.Ferromagnet(world, mpx.Grid(self.size, self.origin), geometry=self.geometry,
                                 regions=self.regions)
        magnet._suspend = True
        magnet.msat = self.msat
        magnet.aex = self.aex
        magnet.alpha = self.alpha
        magnet.ku1 = self.ku1
        magnet.ku2 = self.ku2
        magnet.anisU = self.anisU
        magnet.kc1 = self.kc1
        magnet.kc2 = self.kc2
        magnet.kc3 = self.kc3
        magnet.anisC1 = self.anisC1
        magnet.anisC2 = self.anisC2
        magnet.pol = self.pol
        magnet.xi = self.xi
        magnet.Lambda = self.Lambda
        magnet.epsilon_prime = self.epsilon_prime
        if self.free_layer_thickness is not None:
            magnet.free_layer_thickness = self.free_layer_thickness
        magnet.jcur = self.jcur
        magnet.fixed_layer = self.fixed_layer
        magnet._fixed_layer_on_top = self.fixed_layer_on_top
        magnet._enable_zhang_li = self.zhang_li
        magnet._enable_slonczewski = self.slonczewski
        magnet.temperature = self.temperature
        magnet._thermal_seed = self.thermal_seed
        magnet.bias_magnetic_field = self.bias
        magnet.frozen_spins = self.frozen
        for k, v in self.dmi.items():
            setattr(magnet.dmi_tensor, k, v)
        magnet.inter_exchange = self.inter_exchange
        magnet.scale_exchange = self.scale_exchange
        for (i, j), v in self.inter_pairs.items():
            magnet.inter_exchange.set_between(i, j, v)
        for (i, j), v in self.scale_pairs.items():
            magnet.scale_exchange.set_between(i, j, v)
        magnet._enable_demag = self.enable_demag
        magnet._enable_openbc = self.enable_openbc
        magnet._suspend = False
        magnet._update()
        if any(b != 0 for b in self.world_bias):
            world.bias_magnetic_field = self.world_bias
        if m0 is not None:
            magnet.magnetization = m0
        return world, magnet


def random_m(shape, seed, smooth=0):
    """Seeded Gaussian vectors, optionally smoothed by Jacobi passes, normalised."""
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((3, *shape))
    for _ in range(smooth):
        acc = m.copy()
        cnt = np.ones(shape)
        for ax in (1, 2, 3):
            n = m.shape[ax]
            if n < 2:
                continue
            sl_lo = [slice(None)] * 4
            sl_hi = [slice(None)] * 4
            sl_lo[ax] = slice(0, n - 1)
            sl_hi[ax] = slice(1, n)
            acc[tuple(sl_lo)] += m[tuple(sl_hi)]
            acc[tuple(sl_hi)] += m[tuple(sl_lo)]
            c_lo = [slice(None)] * 3
            c_hi = [slice(None)] * 3
            c_lo[ax - 1] = slice(0, n - 1)
            c_hi[ax - 1] = slice(1, n)
            cnt[tuple(c_lo)] += 1
            cnt[tuple(c_hi)] += 1
        m = acc / cnt
    m /= np.linalg.norm(m, axis=0)
    return m.astype(np.float32)


def max_rel(result, wanted):
    """max over cells of |result - wanted| / max |wanted| (vector norms)."""
    num = np.linalg.norm(np.asarray(result, dtype=np.float64) - np.asarray(wanted, dtype=np.float64), axis=0)
    den = np.max(np.linalg.norm(np.asarray(wanted, dtype=np.float64), axis=0))
    return float(np.max(num) / den) if den > 0 else float(np.max(num))


_KNOWN = None


def known(name):
    """Known answer `name` of the reference's tests (tests/golden/known_answers.json)."""
    global _KNOWN
    if _KNOWN is None:
        import json
        import os

        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")) as f:
            _KNOWN = json.load(f)
    return _KNOWN[name]
