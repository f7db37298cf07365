// stray.cuh -- stray fields between the magnets of one world.
//
// physics/zeeman.cu:70-88 adds to a magnet's external field the stray field
// of every other magnet of its world (source and destination switches on the
// magnets).  Here the field of source A in the cells of destination B is a
// direct sum over A's cells (the restatement of physics/strayfieldbrute.cu:15-57)
// with the FP64-built Newell tensor of their displacements tabulated in FP32:
//   B_B(r) = -mu0 sum_{r' in A} N(r - r') Ms_A(r') m_A(r'),
// r, r' world cell coordinates (grid origin + index).  The table covers the
// displacements O .. O + K - 1 per axis with K = n_A + n_B - 1 and
// O = o_B - o_A - (n_A - 1), components xx, yy, zz, xy, xz, yz.
#pragma once
#include "kernels.cuh"

namespace mpx {

constexpr float MU0_F = 1.25663706212e-6f;  // physics/constants.hpp

struct StrayTable {
  const float* __restrict__ k;  // [6][K2][K1][K0]
  int K[3], O[3];
};

// One thread per destination cell; the source cells are walked in tiles of
// blockDim.x staged in shared memory (Ms m and cell coordinates).  `add`
// accumulates into out (a later source of the same destination); cells of B
// outside its geometry get no stray field.  The source state is A's state for
// `stage` (x0 for stage 0, the stage state otherwise); `gate` skips groups that
// are not running, as the other stage kernels.
__global__ void __launch_bounds__(256) k_stray_pair(const MagnetDev* __restrict__ mags,
                                                    const GroupDev* __restrict__ groups, int src, int dst,
                                                    StrayTable tab, int stage, int gate, int add,
                                                    float* __restrict__ out) {
  __shared__ MagnetDev MB;
  __shared__ GroupDev G;
  __shared__ float sM[3][256];
  __shared__ int sC[3][256];
  if (!load_descs(MB, G, mags, groups, dst, gate, stage)) return;
  const MagnetDev& MA = mags[src];  // read through the cache (same group as B)
  const int NA = MA.N, NB = MB.N;
  const float* mA = stage_m(MA, G, stage);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int bx = 0, by = 0, bz = 0;
  if (i < NB) {
    bx = i % MB.n[0];
    by = (i / MB.n[0]) % MB.n[1];
    bz = i / (MB.n[0] * MB.n[1]);
  }
  const int K0 = tab.K[0], K1 = tab.K[1];
  const size_t KK = (size_t)tab.K[0] * tab.K[1] * tab.K[2];
  // displacement index base of this destination cell: (o_B + b) - (o_A + a) - O
  const int dx0 = MB.o[0] + bx - MA.o[0] - tab.O[0];
  const int dy0 = MB.o[1] + by - MA.o[1] - tab.O[1];
  const int dz0 = MB.o[2] + bz - MA.o[2] - tab.O[2];
  float hx = 0.f, hy = 0.f, hz = 0.f;
  for (int j0 = 0; j0 < NA; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    __syncthreads();
    if (j < NA) {
      const bool ing = !MA.geom || MA.geom[j];
      const float ms = ing ? MA.msat.at(j) : 0.f;
      const float3 m = load3(mA, NA, j);
      sM[0][threadIdx.x] = ms * m.x;
      sM[1][threadIdx.x] = ms * m.y;
      sM[2][threadIdx.x] = ms * m.z;
      sC[0][threadIdx.x] = j % MA.n[0];
      sC[1][threadIdx.x] = (j / MA.n[0]) % MA.n[1];
      sC[2][threadIdx.x] = j / (MA.n[0] * MA.n[1]);
    }
    __syncthreads();
    const int nt = min((int)blockDim.x, NA - j0);
    if (i < NB) {
      for (int t = 0; t < nt; ++t) {
        const size_t p = ((size_t)(dz0 - sC[2][t]) * K1 + (dy0 - sC[1][t])) * K0 + (dx0 - sC[0][t]);
        const float nxx = __ldg(tab.k + p), nyy = __ldg(tab.k + KK + p), nzz = __ldg(tab.k + 2 * KK + p);
        const float nxy = __ldg(tab.k + 3 * KK + p), nxz = __ldg(tab.k + 4 * KK + p), nyz = __ldg(tab.k + 5 * KK + p);
        const float Mx = sM[0][t], My = sM[1][t], Mz = sM[2][t];
        hx -= nxx * Mx + nxy * My + nxz * Mz;
        hy -= nxy * Mx + nyy * My + nyz * Mz;
        hz -= nxz * Mx + nyz * My + nzz * Mz;
      }
    }
  }
  if (i >= NB) return;
  float3 h = f3(MU0_F * hx, MU0_F * hy, MU0_F * hz);
  if (MB.geom && !MB.geom[i]) h = f3(0.f, 0.f, 0.f);
  if (add) h = h + load3(out, NB, i);
  store3(out, NB, i, h);
}

}  // namespace mpx
