"""numpy restatements of transform plans of the CUDA kernels, no GPU.

- Two real rows per complex x transform (the x passes' pack and unpack).
- Warp columns for lengths 64 .. 1024 (32 x q four-step, one warp per column):
  against np.fft, the forward with the upper half zero, the inverse's first half.
- Warp pairs for length 2048 (fft.cuh `pair_inner` / `pair_outer`): a column is
  64 x 32; warp p of the pair forms the inner outputs s = 2s' + p of lane j as
  one 32-point DFT over r of x[j + 32r] W64^(rp) (the forward's inputs r >= 32
  are zero padding; the inverse first folds them in as x_r + (-1)^p x_(r+32)),
  then the twiddles W2048^(js) and, after the transpose, the outer 32-point DFT
  of index c = lane + 32p.  Against np.fft.
- The pair-grid stray-field convolution (pairfft.cuh): the Newell table of the
  displacements from grid A to grid B (K = nA + nB - 1 per axis) and Ms m of A
  zero-padded to P = 2^ceil(log2 K), the y / z transforms of the non-zero rows
  only, the 3x3 complex multiply, the inverse transforms of the output window
  (which starts at nA - 1) only, the Hermitian completion of the x half
  spectrum.  Against the direct sum over source cells.
"""
import numpy as np
import pytest


def _w(n, e, d):
    return np.exp(d * 2j * np.pi * e / n)


def _dft32(v, d):
    return np.fft.fft(v) if d < 0 else np.fft.ifft(v) * 32


def _pair_transform(xin, d, fold):
    L = 2048
    C = np.zeros(L, complex)
    for p in (0, 1):  # inner step: warp p, lanes j
        for j in range(32):
            if fold:
                v = np.array([xin[j + 32 * b] + (-1) ** p * xin[j + 32 * b + 1024] for b in range(32)])
            else:
                v = np.array([xin[j + 32 * r] for r in range(32)])
            if p:
                v = v * _w(2048, 32 * np.arange(32), d)  # W64^r
            v = _dft32(v, d)
            for q in range(32):
                s = 2 * q + p
                C[j + 32 * s] = v[q] * _w(2048, j * s, d)
    out = np.zeros(L, complex)
    for p in (0, 1):  # outer step: lane c of the pair
        for lane in range(32):
            c = lane + 32 * p
            v = _dft32(C[32 * c: 32 * c + 32], d)
            out[c + 64 * np.arange(32)] = v
    return out


@pytest.mark.parametrize("ny", [513, 777, 1024])
def test_warp_pair_2048_maps_match_numpy(ny):
    rng = np.random.default_rng(ny)
    x = np.zeros(2048, complex)
    x[:ny] = rng.standard_normal(ny) + 1j * rng.standard_normal(ny)
    X = _pair_transform(x, -1, False)
    ref = np.fft.fft(x)
    assert np.max(np.abs(X - ref)) < 1e-12 * np.max(np.abs(ref))
    Y = rng.standard_normal(2048) + 1j * rng.standard_normal(2048)
    y = _pair_transform(Y, +1, True)
    ref = np.fft.ifft(Y) * 2048
    assert np.max(np.abs(y[:1024] - ref[:1024])) < 1e-12 * np.max(np.abs(ref))


def _four_step(x, q, d):
    """Warp columns (fft.cuh `four_step_inner` / `four_step_outer`) of length
    L = 32 q: lane j takes x[j + 32 r] (r < q), a q-point DFT over r gives
    Y_j[s], times W_L^(j s); after the transpose lane (s) does the 32-point DFT
    over j and holds X[s + q t] in t."""
    L = 32 * q
    Y = np.zeros((32, q), complex)
    for j in range(32):
        u = np.array([x[j + 32 * r] for r in range(q)])
        u = np.fft.fft(u) if d < 0 else np.fft.ifft(u) * q
        Y[j] = u * _w(L, j * np.arange(q), d)
    X = np.zeros(L, complex)
    for s in range(q):
        X[s + q * np.arange(32)] = _dft32(Y[:, s], d)
    return X


@pytest.mark.parametrize("q", [2, 4, 8, 16, 32])
def test_warp_column_maps_match_numpy(q):
    L = 32 * q
    rng = np.random.default_rng(q)
    x = np.zeros(L, complex)  # forward: the upper half is zero padding (r >= q/2 not read)
    x[:L // 2] = rng.standard_normal(L // 2) + 1j * rng.standard_normal(L // 2)
    X = _four_step(x, q, -1)
    ref = np.fft.fft(x)
    assert np.max(np.abs(X - ref)) < 1e-12 * np.max(np.abs(ref))
    Y = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    y = _four_step(Y, q, +1)  # inverse: outputs t < 16 (y < L/2) kept
    ref = np.fft.ifft(Y) * L
    assert np.max(np.abs(y[:L // 2] - ref[:L // 2])) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("L,n", [(16, 9), (512, 300), (1024, 512)])
def test_two_real_rows_per_complex_transform(L, n):
    """The x passes (k_xfwd / k_xinv) transform two real rows a, b (zero-padded
    from n to L) as one complex row z = a + i b.  Forward unpack: A[k] = (Z[k] +
    conj Z[L-k]) / 2, B[k] = -i/2 (Z[k] - conj Z[L-k]) for k <= L/2.  Inverse
    gather: Z[k] = A[k] + i B[k] and Z[L-k] = conj A[k] + i conj B[k], with the
    imaginary parts of A, B dropped at k = 0 and L/2."""
    rng = np.random.default_rng(L + n)
    a = np.zeros(L)
    b = np.zeros(L)
    a[:n] = rng.standard_normal(n)
    b[:n] = rng.standard_normal(n)
    Z = np.fft.fft(a + 1j * b)
    k = np.arange(L // 2 + 1)
    zc = np.conj(Z[(L - k) % L])
    A = 0.5 * (Z[k] + zc)
    B = -0.5j * (Z[k] - zc)
    assert np.max(np.abs(A - np.fft.rfft(a))) < 1e-12 * L and np.max(np.abs(B - np.fft.rfft(b))) < 1e-12 * L
    # inverse from the half spectra (here those of two other real rows)
    c = rng.standard_normal(L)
    e = rng.standard_normal(L)
    Ac, Ae = np.fft.rfft(c), np.fft.rfft(e)
    Ac[[0, L // 2]] = Ac[[0, L // 2]].real
    Ae[[0, L // 2]] = Ae[[0, L // 2]].real
    Zi = np.zeros(L, complex)
    for kx in range(L // 2 + 1):
        Zi[kx] = Ac[kx] + 1j * Ae[kx]
        if 0 < kx < L - kx:
            Zi[L - kx] = np.conj(Ac[kx]) + 1j * np.conj(Ae[kx])
    z = np.fft.ifft(Zi) * L
    assert np.max(np.abs(z.real - L * c)) < 1e-9 * L and np.max(np.abs(z.imag - L * e)) < 1e-9 * L


def _p2(k):
    return 1 << int(np.ceil(np.log2(k))) if k > 1 else 1


def _pair_grid(nA, nB, tab, M):
    """Field on B (3, nzB, nyB, nxB) from Ms m of A (3, nzA, nyA, nxA) through the
    displacement table tab (6, Kz, Ky, Kx) of components xx, yy, zz, xy, xz, yz."""
    K = [nA[a] + nB[a] - 1 for a in range(3)]
    Px, Py, Pz = (_p2(k) for k in K)
    Hx = Px // 2 + 1

    def forward_xy(src, nin, ncomp):
        T = np.zeros((Hx, ncomp, Pz, Py), complex)
        for c in range(ncomp):
            for z in range(nin[2]):
                for y in range(nin[1]):
                    row = np.zeros(Px)
                    row[:nin[0]] = src[c, z, y]
                    T[:, c, z, y] = np.fft.fft(row)[:Hx]
        for kx in range(Hx):
            for c in range(ncomp):
                for z in range(nin[2]):  # rows y >= nin_y are zero padding
                    T[kx, c, z] = np.fft.fft(T[kx, c, z])
        return T

    KS = forward_xy(tab, K, 6)
    KS = np.fft.fft(KS, axis=2)  # z of the table: planes z >= K_z are zero
    T = forward_xy(M, nA, 3)
    win = [nA[a] - 1 for a in range(3)]
    for kx in range(Hx):
        for ky in range(Py):
            D = np.fft.fft(T[kx, :, :, ky], axis=1)
            k = KS[kx, :, :, ky]
            H = np.stack([k[0] * D[0] + k[3] * D[1] + k[4] * D[2],
                          k[3] * D[0] + k[1] * D[1] + k[5] * D[2],
                          k[4] * D[0] + k[5] * D[1] + k[2] * D[2]])
            H = np.fft.ifft(H, axis=1) * Pz
            T[kx, :, win[2]:win[2] + nB[2], ky] = H[:, win[2]:win[2] + nB[2]]
    for kx in range(Hx):
        for c in range(3):
            for z in range(win[2], win[2] + nB[2]):
                col = np.fft.ifft(T[kx, c, z]) * Py
                T[kx, c, z, win[1]:win[1] + nB[1]] = col[win[1]:win[1] + nB[1]]
    out = np.zeros((3, nB[2], nB[1], nB[0]))
    for c in range(3):
        for zz in range(nB[2]):
            for y in range(nB[1]):
                D = np.zeros(Px, complex)
                for kx in range(Hx):  # Hermitian completion of the half spectrum
                    v = T[kx, c, win[2] + zz, win[1] + y]
                    D[kx] = v
                    if 0 < kx < Px - kx:
                        D[Px - kx] = np.conj(v)
                out[c, zz, y] = (np.fft.ifft(D) * Px).real[win[0]:win[0] + nB[0]] / (Px * Py * Pz)
    return out


def _direct(nA, nB, tab, M):
    idx = [[0, 3, 4], [3, 1, 5], [4, 5, 2]]
    want = np.zeros((3, nB[2], nB[1], nB[0]))
    for z in range(nB[2]):
        for y in range(nB[1]):
            for x in range(nB[0]):
                for zp in range(nA[2]):
                    for yp in range(nA[1]):
                        for xp in range(nA[0]):
                            d = (z - zp + nA[2] - 1, y - yp + nA[1] - 1, x - xp + nA[0] - 1)
                            for a in range(3):
                                want[a, z, y, x] += sum(tab[idx[a][b], d[0], d[1], d[2]] * M[b, zp, yp, xp]
                                                        for b in range(3))
    return want


@pytest.mark.parametrize("nA,nB", [((3, 2, 1), (4, 3, 1)), ((5, 1, 2), (2, 3, 3)), ((1, 1, 1), (3, 2, 2)),
                                   ((4, 3, 2), (1, 1, 1)), ((2, 5, 3), (3, 2, 1))])
def test_pair_grid_convolution_matches_direct_sum(nA, nB):
    rng = np.random.default_rng(sum(nA) * 7 + sum(nB))
    K = [nA[a] + nB[a] - 1 for a in range(3)]
    tab = rng.standard_normal((6, K[2], K[1], K[0]))
    M = rng.standard_normal((3, nA[2], nA[1], nA[0]))
    got = _pair_grid(nA, nB, tab, M)
    want = _direct(nA, nB, tab, M)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
