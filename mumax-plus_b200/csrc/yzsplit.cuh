// yzsplit.cuh -- the y/z part of the demag convolution in three passes, for
// magnets whose 3*nz columns of one kx do not fit one block (nz > 8, or long y
// transforms): the z transform then needs its own pass.
//
//   k_ycols<-1>  per group of consecutive spectrum columns (kx, c, z): load the
//                ny rows of S (zero padding above), forward FFT along y (pruned
//                first pass), store all Py rows into T[kx][c][z][ky]
//   k_zmul       per (kx, tile of ky): gather the 3 x nz values of every ky from
//                T into shared memory columns along z, forward FFT along z of
//                length Pz (pruned), 3x3 multiply by the Newell spectrum, inverse
//                FFT along z (only the nz outputs), store back into T
//   k_ycols<+1>  per group of columns: inverse FFT along y of T (only the ny
//                outputs), store into S
//
// Same arithmetic as k_yz (the same FFT passes, the same kernel spectrum
// lookup); the spectrum makes two extra round trips through global memory.
#pragma once
#include "kernels.cuh"

namespace mpx {

// Kernel spectrum entry at (kx, ky, kz) for a runtime z length Pz, from the
// symmetry-reduced storage [kx][kz'][kcomp][ky'] (as kernel_at).
__device__ __forceinline__ void kernel_at_rt(const float* __restrict__ Kx, int kc, int hy, int kyp, float sy, int kz,
                                             int Pz, float& kxx, float& kyy, float& kzz, float& kxy, float& kxz,
                                             float& kyz, size_t left) {
  const int kzp = min(kz, Pz - kz);
  const float sz = (kz > Pz / 2) ? -1.f : 1.f;
  if (!span_ok((size_t)kzp * kc * hy + kyp + (size_t)(kc - 1) * hy, left)) {
    kxx = kyy = kzz = kxy = kxz = kyz = 0.f;
    return;
  }
  const float* Kk = Kx + (size_t)kzp * kc * hy + kyp;
  kxx = __ldg(Kk);
  kyy = __ldg(Kk + hy);
  kzz = __ldg(Kk + 2 * hy);
  kxy = sy * __ldg(Kk + 3 * hy);
  if (kc == 6) {
    kxz = sz * __ldg(Kk + 4 * hy);
    kyz = sy * sz * __ldg(Kk + 5 * hy);
  } else {
    kxz = kyz = 0.f;
  }
}

// Work item: magnet, first column (kx*3 + c)*nz + z in z, number of columns in y0.
template <int DIR, int MAXLR>
__global__ void __launch_bounds__(384, MAXLR == 3 ? 2 : 1)
    k_ycols(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
            int stage, int gate, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  const int col0 = wk.z, ncol = wk.y0;
  const int ny = M.n[1];
  const int logPy = M.logP[1], Py = 1 << logPy, cs = plen(Py);
  float2* D = sm;
  float2* tws = sm + ncol * cs;
  load_twiddles<MAXLR>(tws, tw, logPy);
  float2* __restrict__ T = M.tspec + (size_t)col0 * Py;
  float2* __restrict__ S = M.spec + (size_t)col0 * ny;
  const size_t ncols_all = (size_t)M.Fh * 3 * M.n[2];  // columns of S and T (checked build)
  const size_t sleft = (ncols_all - col0) * ny, tleft = (ncols_all - col0) * Py;
  if (DIR < 0) {  // S (ny rows, zero above) -> lower half of each column
    const int logh = logPy > 0 ? logPy - 1 : 0;
    const int total = ncol << logh;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int col = e >> logh, y = e & ((1 << logh) - 1);
      D[col * cs + pidx(y)] =
          (y < ny && span_ok((size_t)col * ny + y, sleft)) ? __ldg(S + (size_t)col * ny + y) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_many<-1, MAXLR, 1>(D, logPy, ncol, cs, tws);
    for (int e = threadIdx.x; e < (ncol << logPy); e += blockDim.x) {
      const int col = e >> logPy, y = e & (Py - 1);
      if (span_ok((size_t)col * Py + y, tleft)) T[(size_t)col * Py + y] = D[col * cs + pidx(y)];
    }
  } else {  // T (Py rows) -> S (the ny rows that are not padding)
    for (int e = threadIdx.x; e < (ncol << logPy); e += blockDim.x) {
      const int col = e >> logPy, y = e & (Py - 1);
      D[col * cs + pidx(y)] = span_ok((size_t)col * Py + y, tleft) ? __ldg(T + (size_t)col * Py + y)
                                                                    : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_many<1, MAXLR, 2>(D, logPy, ncol, cs, tws);
    for (int e = threadIdx.x; e < ncol * ny; e += blockDim.x) {
      const int col = e / ny, y = e - col * ny;
      if (span_ok((size_t)col * ny + y, sleft)) S[(size_t)col * ny + y] = D[col * cs + pidx(y)];
    }
  }
}

// Work item: magnet, kx in z, first ky in y0, number of ky in ty.
template <int MAXLR>
__global__ void __launch_bounds__(384, MAXLR == 3 ? 2 : 1)
    k_zmul(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
           int stage, int gate, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  const int kx = wk.z, ky0 = wk.y0, nky = wk.ty;
  const int nz = M.n[2];
  const int logPy = M.logP[1], Py = 1 << logPy;
  const int logPz = M.logP[2], Pz = 1 << logPz, cs = plen(Pz);
  const int ncol = 3 * nky;  // column (c, kyl) along z
  float2* D = sm;
  float2* tws = sm + ncol * cs;
  load_twiddles<MAXLR>(tws, tw, logPz);
  const float2* __restrict__ Tk = M.tspec + (size_t)kx * 3 * nz * Py;
  const size_t tleft = (size_t)(M.Fh - kx) * 3 * nz * Py;  // elements of T from Tk on (checked build)
  // gather: consecutive threads take consecutive ky (coalesced rows of T)
  const int logh = logPz > 0 ? logPz - 1 : 0;
  for (int e = threadIdx.x; e < (ncol << logh); e += blockDim.x) {
    const int kyl = e % nky, rest = e / nky;
    const int c = rest % 3, z = rest / 3;
    D[(c * nky + kyl) * cs + pidx(z)] = (z < nz && span_ok(((size_t)c * nz + z) * Py + ky0 + kyl, tleft))
                                            ? __ldg(Tk + ((size_t)c * nz + z) * Py + ky0 + kyl)
                                            : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_many<-1, MAXLR, 1>(D, logPz, ncol, cs, tws);
  // 3x3 multiply by the real kernel spectrum at (kx, ky, kz)
  const int hy = Py / 2 + 1, kc = M.kcomp;
  const float* __restrict__ Kx = M.kspec + (size_t)kx * (Pz / 2 + 1) * kc * hy;
  for (int t = threadIdx.x; t < (nky << logPz); t += blockDim.x) {
    const int kyl = t % nky, kz = t / nky;
    const int ky = ky0 + kyl;
    const int kyp = min(ky, Py - ky);
    const float sy = (ky > Py / 2) ? -1.f : 1.f;
    float kxx, kyy, kzz, kxy, kxz, kyz;
    kernel_at_rt(Kx, kc, hy, kyp, sy, kz, Pz, kxx, kyy, kzz, kxy, kxz, kyz, (size_t)(M.Fh - kx) * (Pz / 2 + 1) * kc * hy);
    apply3(&D[(0 * nky + kyl) * cs + pidx(kz)], &D[(1 * nky + kyl) * cs + pidx(kz)],
           &D[(2 * nky + kyl) * cs + pidx(kz)], kxx, kyy, kzz, kxy, kxz, kyz);
  }
  __syncthreads();
  fft_many<1, MAXLR, 2>(D, logPz, ncol, cs, tws);
  float2* __restrict__ Tw = M.tspec + (size_t)kx * 3 * nz * Py;
  for (int e = threadIdx.x; e < ncol * nz; e += blockDim.x) {
    const int kyl = e % nky, rest = e / nky;
    const int c = rest % 3, z = rest / 3;
    if (span_ok(((size_t)c * nz + z) * Py + ky0 + kyl, tleft))
      Tw[((size_t)c * nz + z) * Py + ky0 + kyl] = D[(c * nky + kyl) * cs + pidx(z)];
  }
}

}  // namespace mpx
