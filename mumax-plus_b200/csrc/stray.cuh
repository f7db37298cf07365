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

// FFT form for large pairs (the reference's default executor, physics/strayfieldfft.cu):
// a helper magnet spanning the bounding box of A and B (msat 1, demag only)
// takes Ms_A m_A in A's cells and zero elsewhere; its demag field, evaluated by
// the x / y-z / x passes, is at B's cells the stray field of A (the Newell
// tensor depends on the displacement only).

// Ms_A m_A of the stage state into the helper's magnetisation buffer (buf[0]) at A's cells.
__global__ void __launch_bounds__(256) k_hull_scatter(const MagnetDev* __restrict__ mags,
                                                      const GroupDev* __restrict__ groups, int src, int hull, int stage,
                                                      int gate) {
  __shared__ MagnetDev MA;
  __shared__ GroupDev G;
  if (!load_descs(MA, G, mags, groups, src, gate, stage)) return;
  const MagnetDev& MH = mags[hull];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MA.N) return;
  const int x = i % MA.n[0], y = (i / MA.n[0]) % MA.n[1], z = i / (MA.n[0] * MA.n[1]);
  const int h = (MA.o[0] - MH.o[0] + x) + MH.n[0] * ((MA.o[1] - MH.o[1] + y) + MH.n[1] * (MA.o[2] - MH.o[2] + z));
  const bool ing = !MA.geom || MA.geom[i];
  const float ms = ing ? MA.msat.at(i) : 0.f;
  const float3 m = load3(stage_m(MA, G, stage), MA.N, i);
  store3(MH.buf[0], MH.N, h, ms * m);
}

// The helper's demag field (buf[1]) at B's cells into out (added with `add`),
// zero outside B's geometry, as k_stray_pair.
__global__ void __launch_bounds__(256) k_hull_gather(const MagnetDev* __restrict__ mags,
                                                     const GroupDev* __restrict__ groups, int hull, int dst, int stage,
                                                     int gate, int add, float* __restrict__ out) {
  __shared__ MagnetDev MB;
  __shared__ GroupDev G;
  if (!load_descs(MB, G, mags, groups, dst, gate, stage)) return;
  const MagnetDev& MH = mags[hull];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MB.N) return;
  const int x = i % MB.n[0], y = (i / MB.n[0]) % MB.n[1], z = i / (MB.n[0] * MB.n[1]);
  const int h = (MB.o[0] - MH.o[0] + x) + MH.n[0] * ((MB.o[1] - MH.o[1] + y) + MH.n[1] * (MB.o[2] - MH.o[2] + z));
  float3 v = load3(MH.buf[1], MH.N, h);
  if (MB.geom && !MB.geom[i]) v = f3(0.f, 0.f, 0.f);
  if (add) v = v + load3(out, MB.N, i);
  store3(out, MB.N, i, v);
}

}  // namespace mpx
