// pairfft.cuh -- FFT form of the stray field of a source magnet A on a
// destination grid B, on the pair's own kernel grid (the layout of
// physics/strayfieldkernel.cu:80-99, the convolution of
// physics/strayfieldfft.cu:182-250).
//
// The Newell tensor is tabulated at the displacements O + j, j in [0, K) with
// K = n_A + n_B - 1 and O = o_B - o_A - (n_A - 1) per axis (periodic images
// included, k_newell_reflayout), and convolved with Ms m of A by FFTs of
// power-of-two lengths P >= K.  With A zero-padded to P the circular sum at
// n = i + n_A - 1 never wraps (n - i' runs over [i, i + n_A - 1], inside
// [0, K)), so destination cell i reads the output at the window w = n_A - 1.
// The grid depends on the sizes of A and B only, not on their distance: two
// single-layer magnets at any z distance convolve in 2-D.
//
// The table is not symmetric about zero displacement, so its spectrum is a
// general complex (Hermitian) one, six components.  Layouts, kx < Hx = Px/2 + 1:
//   work spectrum    T [kx][c][z][y]     c < 3, z < Pz, y < Py
//   kernel spectrum  KS[kx][q][kz][ky]   q < 6 (xx, yy, zz, xy, xz, yz)
// Passes of one evaluation:
//   k_pair_xfwd      rows (c, z < nA_z, y < nA_y): Ms m_c along x, zero-padded,
//                    forward FFT; kx < Hx into T
//   k_pair_yfft<-1>  columns (kx, c, z < nA_z): y FFT, rows y >= nA_y zero
//   k_pair_zmul      per kx and tile of ky: z FFT (planes z >= nA_z zero),
//                    3x3 multiply by KS, inverse z FFT; the window's planes
//   k_pair_yfft<+1>  columns (kx, c, z of the window): inverse y FFT, the
//                    window's rows
//   (k_pair_yz<PZ>   the three middle passes in one block per kx when its
//                    3 Pz columns fit in shared memory, Pz <= 8)
//   k_pair_xinv      rows (c, z, y of the window): Hermitian completion,
//                    inverse x FFT, x of the window times -mu0 / (Px Py Pz)
//                    into the destination (zero outside its geometry)
// KS is made once per pair by the first three passes over the table (six
// components, no multiply).  All transforms are the shared-memory Stockham
// FFTs of fft.cuh with radix-8 passes: 512 threads of 8 values (4096 points
// per group) and at most 64 registers, so that two blocks share an SM (the
// radix-16 form needed ~150 registers: one 8-warp block per SM).
#pragma once
#include "stray.cuh"

namespace mpx {

constexpr int PF_THREADS = 512;
constexpr int PF_LR = 3;                              // log2 of the largest radix
constexpr int PF_POINTS = (1 << PF_LR) * PF_THREADS;  // points of one transform group

struct PairFft {
  float2* t;         // work spectrum (or, while it is made, the kernel spectrum)
  const float2* ks;  // kernel spectrum
  int logP[3];
  int nin[3];   // rows of the input per axis (source grid, or the table K)
  int win[3];   // first row of the output window per axis (n_A - 1)
  int nout[3];  // rows of the output window per axis (n_B)
  float scale;  // -mu0 / (Px Py Pz)
};

// Forward x transforms.  TABLE: input the tabulated tensor [q][z][y][x] of
// `ncomp` = 6 components; else Ms m of the source magnet's state for `stage`
// (zero outside its geometry).  Block: rows y0 .. y0 + ry - 1 of (c, z).
template <bool TABLE>
__global__ void __launch_bounds__(PF_THREADS, 2) k_pair_xfwd(const MagnetDev* __restrict__ mags,
                                                          const GroupDev* __restrict__ groups, int src, int stage,
                                                          int gate, const float* __restrict__ tab, PairFft pf,
                                                          int ncomp, int ry, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev MA;
  __shared__ GroupDev G;
  const int logPx = pf.logP[0], Px = 1 << logPx, cs = plen(Px);
  const int nxi = pf.nin[0], nyi = pf.nin[1], nzi = pf.nin[2];
  const int nyt = (nyi + ry - 1) / ry;
  const int yt = blockIdx.x % nyt, z = (blockIdx.x / nyt) % nzi, c = blockIdx.x / (nyt * nzi);
  if (c >= ncomp) return;
  if (!TABLE && !load_descs(MA, G, mags, groups, src, gate, stage)) return;
  const int y0 = yt * ry, nr = min(ry, nyi - y0);
  float2* D = sm;
  float2* tws = sm + ry * cs;
  load_twiddles<PF_LR>(tws, tw, logPx);
  const float* m = TABLE ? nullptr : stage_m(MA, G, stage);
  for (int e = threadIdx.x; e < (nr << logPx); e += blockDim.x) {
    const int r = e >> logPx, x = e & (Px - 1);
    float v = 0.f;
    if (x < nxi) {
      if (TABLE) {
        const size_t ti = (((size_t)c * nzi + z) * nyi + y0 + r) * nxi + x;
        if (span_ok(ti, (size_t)ncomp * nzi * nyi * nxi)) v = __ldg(tab + ti);
      } else {
        const int j = x + nxi * (y0 + r + nyi * z);
        if (cell_ok(MA.N, j) && (!MA.geom || MA.geom[j])) v = MA.msat.at(j) * m[(size_t)c * MA.N + j];
      }
    }
    D[r * cs + pidx(x)] = make_float2(v, 0.f);
  }
  __syncthreads();
  fft_many<-1, PF_LR>(D, logPx, nr, cs, tws);
  __syncthreads();
  const int Hx = Px / 2 + 1, Py = 1 << pf.logP[1], Pz = 1 << pf.logP[2];
  const size_t tsize = (size_t)Hx * ncomp * Pz * Py;  // elements of the spectrum (checked build)
  for (int e = threadIdx.x; e < Hx * nr; e += blockDim.x) {  // consecutive threads: consecutive y
    const int r = e % nr, kx = e / nr;
    const size_t ti = (((size_t)kx * ncomp + c) * Pz + z) * Py + y0 + r;
    if (span_ok(ti, tsize)) pf.t[ti] = D[r * cs + pidx(kx)];
  }
}

// y transforms of the columns (kx, c, z): forward over z < nin_z (rows
// y >= nin_y zero, all Py rows out), or inverse over the window's planes (the
// window's rows out).  Block: zc consecutive columns of one (kx, c).  src >= 0:
// the source magnet decides the group gate.
template <int DIR>
__global__ void __launch_bounds__(PF_THREADS, 2) k_pair_yfft(const MagnetDev* __restrict__ mags,
                                                          const GroupDev* __restrict__ groups, int src, int stage,
                                                          int gate, PairFft pf, int ncomp, int zc,
                                                          const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev MA;
  __shared__ GroupDev G;
  if (src >= 0 && !load_descs(MA, G, mags, groups, src, gate, stage)) return;
  const int logPy = pf.logP[1], Py = 1 << logPy, Pz = 1 << pf.logP[2], cs = plen(Py);
  const int zlo = DIR < 0 ? 0 : pf.win[2], nzc = DIR < 0 ? pf.nin[2] : pf.nout[2];
  const int nzt = (nzc + zc - 1) / zc;
  const int zt = blockIdx.x % nzt, c = (blockIdx.x / nzt) % ncomp, kx = blockIdx.x / (nzt * ncomp);
  const int z0 = zlo + zt * zc, nc = min(zc, zlo + nzc - z0);
  float2* D = sm;
  float2* tws = sm + zc * cs;
  load_twiddles<PF_LR>(tws, tw, logPy);
  const size_t t0 = (((size_t)kx * ncomp + c) * Pz + z0) * Py;
  const size_t tleft = (size_t)((1 << pf.logP[0]) / 2 + 1) * ncomp * Pz * Py - t0;  // elements from T on (checked build)
  float2* __restrict__ T = pf.t + t0;
  const int nyin = DIR < 0 ? pf.nin[1] : Py;
  for (int e = threadIdx.x; e < (nc << logPy); e += blockDim.x) {
    const int col = e >> logPy, y = e & (Py - 1);
    D[col * cs + pidx(y)] =
        (y < nyin && span_ok((size_t)col * Py + y, tleft)) ? T[(size_t)col * Py + y] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_many<DIR, PF_LR>(D, logPy, nc, cs, tws);
  __syncthreads();
  if (DIR < 0) {
    for (int e = threadIdx.x; e < (nc << logPy); e += blockDim.x) {
      const int col = e >> logPy, y = e & (Py - 1);
      if (span_ok((size_t)col * Py + y, tleft)) T[(size_t)col * Py + y] = D[col * cs + pidx(y)];
    }
  } else {
    const int ylo = pf.win[1], ny = pf.nout[1];
    for (int e = threadIdx.x; e < nc * ny; e += blockDim.x) {
      const int col = e / ny, y = ylo + e % ny;
      if (span_ok((size_t)col * Py + y, tleft)) T[(size_t)col * Py + y] = D[col * cs + pidx(y)];
    }
  }
}

// z stage of one kx and a tile of nky consecutive ky: the columns (c, ky)
// along z gathered from T (planes z >= nin_z zero), forward z FFT; with MUL the
// 3x3 product with the kernel spectrum, the inverse z FFT and the window's
// planes back into T; without MUL (making the kernel spectrum) all Pz planes.
template <bool MUL>
__global__ void __launch_bounds__(PF_THREADS, 2) k_pair_zmul(const MagnetDev* __restrict__ mags,
                                                          const GroupDev* __restrict__ groups, int src, int stage,
                                                          int gate, PairFft pf, int ncomp, int tky,
                                                          const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev MA;
  __shared__ GroupDev G;
  if (src >= 0 && !load_descs(MA, G, mags, groups, src, gate, stage)) return;
  const int Py = 1 << pf.logP[1], logPz = pf.logP[2], Pz = 1 << logPz, cs = plen(Pz);
  const int nyt = (Py + tky - 1) / tky;
  const int kx = blockIdx.x / nyt, ky0 = (blockIdx.x % nyt) * tky, nky = min(tky, Py - ky0);
  const int ncol = ncomp * nky;
  float2* D = sm;
  float2* tws = sm + ncomp * tky * cs;
  load_twiddles<PF_LR>(tws, tw, logPz);
  const size_t tk0 = (size_t)kx * ncomp * Pz * Py + ky0;
  const int Hx = (1 << pf.logP[0]) / 2 + 1;
  const size_t tleft = (size_t)Hx * ncomp * Pz * Py - tk0;  // elements from Tk on (checked build)
  float2* __restrict__ Tk = pf.t + tk0;
  const int nzin = pf.nin[2];
  for (int e = threadIdx.x; e < (ncol << logPz); e += blockDim.x) {  // consecutive threads: consecutive ky
    const int kyl = e % nky, rest = e / nky, c = rest % ncomp, z = rest / ncomp;
    const size_t ti = ((size_t)c * Pz + z) * Py + kyl;
    D[(c * nky + kyl) * cs + pidx(z)] = (z < nzin && span_ok(ti, tleft)) ? Tk[ti] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_many<-1, PF_LR>(D, logPz, ncol, cs, tws);
  __syncthreads();
  if (MUL) {
    const size_t k0 = (size_t)kx * 6 * Pz * Py + ky0;
    const size_t kleft = (size_t)Hx * 6 * Pz * Py - k0;  // elements of the kernel spectrum from K on (checked build)
    const float2* __restrict__ K = pf.ks + k0;
    for (int t = threadIdx.x; t < (nky << logPz); t += blockDim.x) {
      const int kyl = t % nky, kz = t / nky;
      float2 k[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const size_t ki = ((size_t)q * Pz + kz) * Py + kyl;
        k[q] = span_ok(ki, kleft) ? __ldg(K + ki) : make_float2(0.f, 0.f);
      }
      float2* p0 = &D[kyl * cs + pidx(kz)];
      float2* p1 = &D[(nky + kyl) * cs + pidx(kz)];
      float2* p2 = &D[(2 * nky + kyl) * cs + pidx(kz)];
      const float2 m0 = *p0, m1 = *p1, m2 = *p2;
      *p0 = cadd(cadd(cmul(k[0], m0), cmul(k[3], m1)), cmul(k[4], m2));
      *p1 = cadd(cadd(cmul(k[3], m0), cmul(k[1], m1)), cmul(k[5], m2));
      *p2 = cadd(cadd(cmul(k[4], m0), cmul(k[5], m1)), cmul(k[2], m2));
    }
    __syncthreads();
    fft_many<1, PF_LR>(D, logPz, ncol, cs, tws);
    __syncthreads();
    const int zlo = pf.win[2], nz = pf.nout[2];
    for (int e = threadIdx.x; e < ncol * nz; e += blockDim.x) {
      const int kyl = e % nky, rest = e / nky, c = rest % ncomp, z = zlo + rest / ncomp;
      const size_t ti = ((size_t)c * Pz + z) * Py + kyl;
      if (span_ok(ti, tleft)) Tk[ti] = D[(c * nky + kyl) * cs + pidx(z)];
    }
  } else {
    for (int e = threadIdx.x; e < (ncol << logPz); e += blockDim.x) {
      const int kyl = e % nky, rest = e / nky, c = rest % ncomp, z = rest / ncomp;
      const size_t ti = ((size_t)c * Pz + z) * Py + kyl;
      if (span_ok(ti, tleft)) Tk[ti] = D[(c * nky + kyl) * cs + pidx(z)];
    }
  }
}

// The y / z stage of one kx in one block when its 3 PZ columns fit in shared
// memory (z length PZ <= 8): forward y FFT of the source planes (rows
// y >= nin_y zero), per ky (one thread each) the z FFT in registers, the 3x3
// product with the kernel spectrum and the inverse z FFT, then the inverse y
// FFT of the window's planes; the window's rows back into T.  It replaces
// k_pair_yfft<-1>, k_pair_zmul<true> and k_pair_yfft<+1> (same arithmetic
// order: y, z, multiply, z, y) without their two round trips through T.
template <int PZ>
__global__ void __launch_bounds__(PF_THREADS, 2) k_pair_yz(const MagnetDev* __restrict__ mags,
                                                        const GroupDev* __restrict__ groups, int src, int stage,
                                                        int gate, PairFft pf, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev MA;
  __shared__ GroupDev G;
  if (!load_descs(MA, G, mags, groups, src, gate, stage)) return;
  const int kx = blockIdx.x;
  const int logPy = pf.logP[1], Py = 1 << logPy, cs = plen(Py);
  float2* D = sm;  // column (z, c) at D + (3 z + c) cs
  float2* tws = sm + 3 * PZ * cs;
  load_twiddles<PF_LR>(tws, tw, logPy);
  float2* __restrict__ Tk = pf.t + (size_t)kx * 3 * PZ * Py;  // [c][z][y]
  const size_t tleft = (size_t)((1 << pf.logP[0]) / 2 + 1 - kx) * 3 * PZ * Py;  // elements from Tk on (checked build)
  const int nzi = pf.nin[2], nyi = pf.nin[1];
  for (int e = threadIdx.x; e < ((3 * nzi) << logPy); e += blockDim.x) {
    const int col = e >> logPy, y = e & (Py - 1);
    const int z = col / 3, c = col - 3 * z;
    const size_t ti = ((size_t)c * PZ + z) * Py + y;
    D[col * cs + pidx(y)] = (y < nyi && span_ok(ti, tleft)) ? Tk[ti] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_many<-1, PF_LR>(D, logPy, 3 * nzi, cs, tws);
  __syncthreads();
  const float2* __restrict__ K = pf.ks + (size_t)kx * 6 * PZ * Py;
  const size_t kleft = 2 * tleft;  // the kernel spectrum has 6 components where T has 3
  const int zlo = pf.win[2], nzo = pf.nout[2];
  for (int ky = threadIdx.x; ky < Py; ky += blockDim.x) {
    float2 v[3][PZ];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int z = 0; z < PZ; ++z) v[c][z] = z < nzi ? D[(3 * z + c) * cs + pidx(ky)] : make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 3; ++c) dft_reg<PZ, -1>(v[c]);
#pragma unroll
    for (int kz = 0; kz < PZ; ++kz) {
      float2 k[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const size_t ki = ((size_t)q * PZ + kz) * Py + ky;
        k[q] = span_ok(ki, kleft) ? __ldg(K + ki) : make_float2(0.f, 0.f);
      }
      const float2 m0 = v[0][kz], m1 = v[1][kz], m2 = v[2][kz];
      v[0][kz] = cadd(cadd(cmul(k[0], m0), cmul(k[3], m1)), cmul(k[4], m2));
      v[1][kz] = cadd(cadd(cmul(k[3], m0), cmul(k[1], m1)), cmul(k[5], m2));
      v[2][kz] = cadd(cadd(cmul(k[4], m0), cmul(k[5], m1)), cmul(k[2], m2));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) dft_reg<PZ, 1>(v[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int z = 0; z < PZ; ++z)
        if (z >= zlo && z < zlo + nzo) D[(3 * z + c) * cs + pidx(ky)] = v[c][z];
  }
  __syncthreads();
  fft_many<1, PF_LR>(D + 3 * zlo * cs, logPy, 3 * nzo, cs, tws);
  __syncthreads();
  const int ylo = pf.win[1], nyo = pf.nout[1];
  for (int e = threadIdx.x; e < 3 * nzo * nyo; e += blockDim.x) {
    const int col = e / nyo, y = ylo + (e - col * nyo);
    const int z = zlo + col / 3, c = col % 3;
    const size_t ti = ((size_t)c * PZ + z) * Py + y;
    if (span_ok(ti, tleft)) Tk[ti] = D[(3 * zlo + col) * cs + pidx(y)];
  }
}

// Inverse x transforms of the window's rows (c, z, y): kx < Hx from T, the
// rest by Hermitian symmetry, inverse FFT; x of the window, scaled, into
// `out` (3 x N_B, component-major; added with `add`), zero outside the
// destination's geometry.  Block: rows y0 .. y0 + ry - 1 of (c, z).
__global__ void __launch_bounds__(PF_THREADS, 2) k_pair_xinv(const MagnetDev* __restrict__ mags,
                                                          const GroupDev* __restrict__ groups, int dst, int stage,
                                                          int gate, PairFft pf, int ry, int add,
                                                          float* __restrict__ out, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev MB;
  __shared__ GroupDev G;
  if (!load_descs(MB, G, mags, groups, dst, gate, stage)) return;
  const int logPx = pf.logP[0], Px = 1 << logPx, Hx = Px / 2 + 1, cs = plen(Px);
  const int Py = 1 << pf.logP[1], Pz = 1 << pf.logP[2];
  const int nxo = pf.nout[0], nyo = pf.nout[1], nzo = pf.nout[2];
  const int nyt = (nyo + ry - 1) / ry;
  const int yt = blockIdx.x % nyt, zz = (blockIdx.x / nyt) % nzo, c = blockIdx.x / (nyt * nzo);
  if (c >= 3) return;
  const int y0 = yt * ry, nr = min(ry, nyo - y0);
  float2* D = sm;
  float2* tws = sm + ry * cs;
  load_twiddles<PF_LR>(tws, tw, logPx);
  const size_t t0 = ((size_t)c * Pz + pf.win[2] + zz) * Py + pf.win[1] + y0;
  const size_t tleft = (size_t)Hx * 3 * Pz * Py - t0;  // elements from T on (checked build)
  const float2* __restrict__ T = pf.t + t0;
  for (int e = threadIdx.x; e < Hx * nr; e += blockDim.x) {  // consecutive threads: consecutive y
    const int r = e % nr, kx = e / nr;
    const size_t ti = (size_t)kx * 3 * Pz * Py + r;
    const float2 v = span_ok(ti, tleft) ? T[ti] : make_float2(0.f, 0.f);
    D[r * cs + pidx(kx)] = v;
    if (kx > 0 && kx < Px - kx) D[r * cs + pidx(Px - kx)] = cconj(v);
  }
  __syncthreads();
  fft_many<1, PF_LR>(D, logPx, nr, cs, tws);
  __syncthreads();
  const int NB = MB.N;
  for (int e = threadIdx.x; e < nr * nxo; e += blockDim.x) {
    const int r = e / nxo, x = e - r * nxo;
    const int i = x + nxo * (y0 + r + nyo * zz);
    if (!cell_ok(NB, i)) continue;
    float v = pf.scale * D[r * cs + pidx(pf.win[0] + x)].x;
    if (MB.geom && !MB.geom[i]) v = 0.f;
    if (add) v += out[(size_t)c * NB + i];
    out[(size_t)c * NB + i] = v;
  }
}

}  // namespace mpx
