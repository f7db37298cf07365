"""numpy restatement of the one-lane z stage of the warp-column y/z passes
(zstage_full<PZ> in mumax-plus_b200/csrc/kernels.cuh), no GPU: for one (kx, ky)
the zero-padded PZ-point z transform of nz <= PZ/2 values per component, the
3x3 multiply by the Newell spectrum per kz, and the inverse transform's first nz
outputs, computed as the kernel does (even kz from the PZ/2-point transform of
x, odd kz from that of x[n] W_PZ^n, kernel entries of kz' = min(kz, PZ - kz) with
the xz and yz signs flipped above PZ/2, output = even inverse + twiddled odd
inverse) against the direct PZ-point computation."""
import numpy as np
import pytest

XX, YY, ZZ, XY, XZ, YZ = range(6)


def kernel_matrix(R, kz, pz):
    """3x3 Newell matrix at kz from the stored kz' = 0 .. PZ/2 entries R[kz'][6]."""
    p = min(kz, pz - kz)
    s = -1.0 if kz > pz // 2 else 1.0
    k = R[p]
    return np.array([[k[XX], k[XY], s * k[XZ]],
                     [k[XY], k[YY], s * k[YZ]],
                     [s * k[XZ], s * k[YZ], k[ZZ]]])


def direct(x, R, pz):
    nz = x.shape[1]
    xp = np.zeros((3, pz), complex)
    xp[:, :nz] = x
    X = np.fft.fft(xp, axis=1)  # exp(-2 pi i n kz / PZ)
    Y = np.stack([kernel_matrix(R, kz, pz) @ X[:, kz] for kz in range(pz)], axis=1)
    return (np.fft.ifft(Y, axis=1) * pz)[:, :nz]  # unnormalised inverse, exp(+)


def one_lane(x, R, pz):
    h = pz // 2
    nz = x.shape[1]
    xin = np.zeros((3, h), complex)
    xin[:, :nz] = x
    n = np.arange(h)
    e = np.fft.fft(xin, axis=1)                                  # kz = 2q
    o = np.fft.fft(xin * np.exp(-2j * np.pi * n / pz), axis=1)  # kz = 2q + 1
    for q in range(h):
        kz_e, kz_o = 2 * q, 2 * q + 1
        # the kernel's kz' and sign maps, spelled out as in zstage_full
        pe = kz_e if kz_e <= h else pz - kz_e
        po = kz_o if kz_o <= h else pz - kz_o
        se = -1.0 if kz_e > h else 1.0
        so = -1.0 if kz_o > h else 1.0
        Ke, Ko = R[pe].copy(), R[po].copy()
        Ke[[XZ, YZ]] *= se
        Ko[[XZ, YZ]] *= so
        for K, v in ((Ke, e), (Ko, o)):
            m = np.array([[K[XX], K[XY], K[XZ]], [K[XY], K[YY], K[YZ]], [K[XZ], K[YZ], K[ZZ]]])
            v[:, q] = m @ v[:, q]
    e = np.fft.ifft(e, axis=1) * h
    o = np.fft.ifft(o, axis=1) * h * np.exp(2j * np.pi * n / pz)
    return (e + o)[:, :nz]


@pytest.mark.parametrize("pz", [4, 8, 16])
def test_one_lane_z_stage_matches_the_direct_transform(pz):
    rng = np.random.default_rng(pz)
    for nz in range(1, pz // 2 + 1):
        x = rng.standard_normal((3, nz)) + 1j * rng.standard_normal((3, nz))
        R = rng.standard_normal((pz // 2 + 1, 6))
        R[0, [XZ, YZ]] = 0.0  # odd in z: zero at kz = 0 and kz = PZ/2
        R[pz // 2, [XZ, YZ]] = 0.0
        want = direct(x, R, pz)
        got = one_lane(x, R, pz)
        assert np.max(np.abs(got - want)) < 1e-12 * max(1.0, np.max(np.abs(want)))
