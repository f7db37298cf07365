"""Seeded random magnets against the FP64 oracle: uneven sizes that reach every
FFT path (block-wide Stockham passes, warp columns of every length, warp rows,
the split y/z path for thick magnets), random periodic boundaries, random
geometry, DMI and anisotropy.  Fields |dB|max / |B|max <= 1e-5.

Each case is drawn from numpy.random.default_rng(1000 + case); the draw is
printed in the assertion message so that a failure names its configuration."""
import numpy as np
import pytest

import oracle as O
from spec import MagnetSpec, max_rel, random_m

pytestmark = pytest.mark.gpu
abi = O.abi
NCASES = 24


def draw(case):
    rng = np.random.default_rng(1000 + case)
    # lengths spread over the padded sizes 1 .. 1024 along x and y, 1 .. 32 along z
    nx = int(rng.choice([1, 3, 7, 17, 40, 70, 130, 200, 300]))
    ny = int(rng.choice([1, 2, 5, 12, 33, 64, 100, 260, 400]))
    nz = int(rng.choice([1, 1, 2, 3, 5, 8, 11]))
    while nx * ny * nz > 40000:  # keep the FP64 oracle quick
        ny = max(1, ny // 2)
    size = (nx, ny, nz)
    pbc = tuple(int(rng.integers(0, 2)) if size[a] > 1 and a < 2 else 0 for a in range(3))
    kw = dict(size=size, cellsize=tuple(float(c) for c in rng.uniform(1e-9, 4e-9, 3)),
              msat=float(rng.uniform(4e5, 1e6)), aex=float(rng.uniform(5e-12, 2e-11)), alpha=0.1)
    if any(pbc):
        kw.update(mastergrid_size=tuple(size[a] if pbc[a] else 0 for a in range(3)), pbc=pbc)
    if rng.random() < 0.5:
        d = float(rng.uniform(5e-4, 3e-3))
        kw["dmi"] = {"xxz": d, "yyz": d}
    if rng.random() < 0.5:
        u = rng.standard_normal(3)
        kw.update(ku1=float(rng.uniform(1e4, 5e5)), anisU=tuple(float(c) for c in u))
    if rng.random() < 0.4 and nx > 2 and ny > 2:
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        cx, cy = (nx - 1) / 2, (ny - 1) / 2
        kw["geometry"] = ((xx - cx) ** 2 / max(cx, 1) ** 2 + (yy - cy) ** 2 / max(cy, 1) ** 2) <= 1.0
    if rng.random() < 0.3:
        kw["world_bias"] = tuple(float(c) for c in rng.uniform(-0.05, 0.05, 3))
    return kw


@pytest.mark.parametrize("case", range(NCASES))
def test_random_magnet_fields(mpx, case):
    kw = draw(case)
    s = MagnetSpec(**kw)
    m0 = random_m(s.shape, seed=case, smooth=2)
    ow, q = s.oracle_world(m0)
    world, magnet = s.product(mpx, m0)
    for quantity in (abi.Q_DEMAG_FIELD, abi.Q_EFFECTIVE_FIELD, abi.Q_TORQUE):
        want = ow.eval(q, quantity)
        got = magnet._engine.eval(magnet._id, quantity, (3, *s.shape))
        if np.max(np.abs(want)) == 0:
            assert np.max(np.abs(got)) == 0, (case, quantity, kw["size"])
            continue
        err = max_rel(got, want)
        assert err < 1e-5, (case, quantity, err, {k: v for k, v in kw.items() if k != "geometry"})
