"""Seeded synthetic workloads: the film, multilayer, precision, batched and
serving problems the benchmarks run (no datasets: every input is generated
from a seed with numpy).

A workload is a dict of magnet parameters; `desc()` turns one into the
mpx_magnet_desc of the C ABI (no GPU needed), `build()` creates it through the
World / Ferromagnet API.
"""
import ctypes as C

import numpy as np

from . import _abi


def smoothed_random_m(shape, seed, passes=3):
    """N(0,1) vectors, `passes` Jacobi passes (each cell <- mean of itself and
    its in-grid face neighbours), then normalised.  shape = (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((3, *shape))
    for _ in range(passes):
        acc = m.copy()
        cnt = np.ones(shape)
        for ax in (1, 2, 3):
            n = m.shape[ax]
            if n < 2:
                continue
            lo = [slice(None)] * 4
            hi = [slice(None)] * 4
            lo[ax], hi[ax] = slice(0, n - 1), slice(1, n)
            acc[tuple(lo)] += m[tuple(hi)]
            acc[tuple(hi)] += m[tuple(lo)]
            clo = [slice(None)] * 3
            chi = [slice(None)] * 3
            clo[ax - 1], chi[ax - 1] = slice(0, n - 1), slice(1, n)
            cnt[tuple(clo)] += 1
            cnt[tuple(chi)] += 1
        m = acc / cnt
    m /= np.linalg.norm(m, axis=0)
    return m.astype(np.float32)


def disc_domains_m(nx, ny, nz, seed=2, ndiscs=40, rmin=5, rmax=15):
    """+z with `ndiscs` reversed discs (centre uniform over the grid, radius
    uniform integer in [rmin, rmax] cells, through all layers, periodic in x, y)."""
    rng = np.random.default_rng(seed)
    m = np.zeros((3, nz, ny, nx), np.float32)
    m[2] = 1.0
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    for _ in range(ndiscs):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        r = rng.integers(rmin, rmax + 1)
        dx = np.abs(X - cx)
        dy = np.abs(Y - cy)
        dx = np.minimum(dx, nx - dx)
        dy = np.minimum(dy, ny - dy)
        m[2, :, (dx * dx + dy * dy) < r * r] = -1.0
    return m


def film(nx=256, ny=64):
    """Film: 256x64x1 cells of 3 nm, Ms 8.6e5, A 1.3e-11, alpha 0.02, open
    boundaries, B_ext = (-30, 5, 0) mT; exchange + demag + Zeeman; m0 seeded
    Gaussian smoothed by 3 Jacobi passes."""
    return dict(name=f"film_{nx}x{ny}x1", size=(nx, ny, 1), cellsize=(3e-9, 3e-9, 3e-9), msat=8.6e5,
                aex=1.3e-11, alpha=0.02, world_bias=(-0.030, 0.005, 0.0), m0=lambda: smoothed_random_m((1, ny, nx), 1))


def multilayer(nx=512, ny=512, nz=8, pbc=(2, 2, 0)):
    """Multilayer: 512x512x8 cells of 2x2x1 nm, PBC in x and y (mastergrid
    512x512x0, pbc_repetitions (2,2,0)), Ms 5.8e5, A 1.5e-11, interfacial
    D 3e-3 (xxz = yyz), Ku1 8e5 along z, alpha 0.1, B_ext (0, 0, 0.2) T;
    m0 = +z with 40 reversed discs of radius 5-15 cells (seed 2)."""
    return dict(name=f"multilayer_{nx}x{ny}x{nz}", size=(nx, ny, nz), cellsize=(2e-9, 2e-9, 1e-9),
                mastergrid=(nx if pbc[0] else 0, ny if pbc[1] else 0, nz if pbc[2] else 0), pbc=pbc,
                msat=5.8e5, aex=1.5e-11, dmi={"xxz": 3e-3, "yyz": 3e-3}, ku1=8e5, anisU=(0.0, 0.0, 1.0),
                alpha=0.1, world_bias=(0.0, 0.0, 0.2), m0=lambda: disc_domains_m(nx, ny, nz, seed=2))


def precision(nx=1024, ny=1024, nz=4):
    """Demag only: 1024x1024x4 cells of 2x2x1 nm (padded FFT 2048x2048x8),
    Ms 8e5, m seeded random unit vectors (seed 3)."""
    def m0():
        rng = np.random.default_rng(3)
        m = rng.standard_normal((3, nz, ny, nx))
        return (m / np.linalg.norm(m, axis=0)).astype(np.float32)
    return dict(name=f"precision_{nx}x{ny}x{nz}", size=(nx, ny, nz), cellsize=(2e-9, 2e-9, 1e-9), msat=8e5,
                m0=m0)


def batch_instances(count=256, seed=4):
    """Relaxation batch: square side floor(32 * 8**u), u ~ U(0,1); nz in {1, 2};
    cubic cells of c ~ U(2, 4) nm; Ms ~ U(4e5, 1e6); A ~ U(5e-12, 2e-11);
    alpha ~ U(0.01, 0.5); B_ext isotropic random direction x U(0, 100) mT;
    m0 random, smoothed by 3 Jacobi passes."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        side = int(np.floor(32 * 8 ** rng.uniform()))
        nz = int(rng.integers(1, 3))
        c = float(rng.uniform(2e-9, 4e-9))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        b = d * rng.uniform(0, 0.1)
        mseed = int(rng.integers(1 << 30))
        out.append(dict(name=f"batch_{k}", size=(side, side, nz), cellsize=(c, c, c),
                        msat=float(rng.uniform(4e5, 1e6)), aex=float(rng.uniform(5e-12, 2e-11)),
                        alpha=float(rng.uniform(0.01, 0.5)), world_bias=tuple(float(v) for v in b),
                        m0=(lambda s=(nz, side, side), ms=mseed: smoothed_random_m(s, ms))))
    return out


def serving_requests(rate=200.0, seconds=60.0, seed=5, dmi_probability=0.5):
    """Open-loop Poisson arrivals; each request: side floor(64 * 8**u), nz in
    {1, 2, 4}, duration U(0.1, 2) ns, batch parameter distributions, and iDMI
    D ~ U(0, 4e-3) with probability `dmi_probability`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        side = int(np.floor(64 * 8 ** rng.uniform()))
        nz = int(rng.choice([1, 2, 4]))
        c = float(rng.uniform(2e-9, 4e-9))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        b = d * rng.uniform(0, 0.1)
        D = float(rng.uniform(0, 4e-3)) if rng.uniform() < dmi_probability else 0.0
        mseed = int(rng.integers(1 << 30))
        reqs.append(dict(arrival=t, duration=float(rng.uniform(0.1e-9, 2e-9)),
                         name=f"req_{len(reqs)}", size=(side, side, nz), cellsize=(c, c, c),
                         msat=float(rng.uniform(4e5, 1e6)), aex=float(rng.uniform(5e-12, 2e-11)),
                         alpha=float(rng.uniform(0.01, 0.5)), world_bias=tuple(float(v) for v in b),
                         dmi={"xxz": D, "yyz": D} if D else {},
                         m0=(lambda s=(nz, side, side), ms=mseed: smoothed_random_m(s, ms))))
    return reqs


def desc(w, keep):
    """mpx_magnet_desc for workload dict `w` (uniform parameters)."""
    d = _abi.MagnetDesc()
    mg = w.get("mastergrid", (0, 0, 0))
    pbc = w.get("pbc", (0, 0, 0))
    for a in range(3):
        d.size[a] = w["size"][a]
        d.cellsize[a] = w["cellsize"][a]
        d.mastergrid_size[a] = mg[a]
        d.pbc_repetitions[a] = pbc[a]
    d.msat.uniform = w.get("msat", 1.0)
    d.aex.uniform = w.get("aex", 0.0)
    d.alpha.uniform = w.get("alpha", 0.0)
    d.ku1.uniform = w.get("ku1", 0.0)
    d.ku2.uniform = w.get("ku2", 0.0)
    for c, v in enumerate(w.get("anisU", (0.0, 0.0, 0.0))):
        d.anis_u.uniform[c] = v
    for i, k in enumerate(_abi.DMI_ORDER):
        d.dmi[i].uniform = w.get("dmi", {}).get(k, 0.0)
    d.scale_exchange = 1.0
    d.enable_demag = int(w.get("enable_demag", True))
    d.enable_openbc = int(w.get("enable_openbc", False))
    return d


def build(mpx, w, device=None, demag_dft="fp32"):
    """World + Ferromagnet for workload `w` through the mumaxplus-style API."""
    mg = w.get("mastergrid", (0, 0, 0))
    world = mpx.World(w["cellsize"], pbc_repetitions=tuple(w.get("pbc", (0, 0, 0))), mastergrid=mpx.Grid(mg),
                      device=device, demag_dft=demag_dft)
    magnet = mpx.Ferromagnet(world, mpx.Grid(w["size"]))
    magnet._suspend = True
    magnet.msat = w.get("msat", 1.0)
    magnet.aex = w.get("aex", 0.0)
    magnet.alpha = w.get("alpha", 0.0)
    magnet.ku1 = w.get("ku1", 0.0)
    magnet.anisU = w.get("anisU", (0.0, 0.0, 0.0))
    for k, v in w.get("dmi", {}).items():
        setattr(magnet.dmi_tensor, k, v)
    magnet._enable_demag = bool(w.get("enable_demag", True))
    magnet._suspend = False
    magnet._update()
    if any(v != 0 for v in w.get("world_bias", (0, 0, 0))):
        world.bias_magnetic_field = w["world_bias"]
    magnet.magnetization = w["m0"]()
    return world, magnet


def ncells(w):
    nx, ny, nz = w["size"]
    return nx * ny * nz
