// kernels.cuh -- the demag / effective-field / Runge-Kutta kernels.
//
// Demag convolution (replaces physics/strayfieldfft.cu:191-246, whose k_pad,
// 3 cuFFT R2C, k_apply_kernel_3d/2d, 3 cuFFT C2R and k_unpad are 9 launches over
// the padded grid) as three passes over a spectrum that only holds the rows
// that are not zero padding:
//   k_xfwd   per tile of TY rows (fixed z): [RK stage combination] -> Ms*m ->
//            real-to-complex FFT along x (two real rows per complex FFT) ->
//            S[kx][c][z][y]
//   k_yz     per kx: FFT along y of the 3*nz columns, then per ky an in-register
//            FFT along z (in one lane in the warp-column kernels, split over
//            two lanes, even / odd kz, in the block-wide one), the 3x3 multiply
//            by the real Newell spectrum (its -mu0/P prefactor folded in) and
//            the inverse z FFT, then the inverse FFT along y; writes back S
//   k_xinv   per tile: complex-to-real FFT along x -> B_demag in shared memory ->
//            epilogue: local terms + LLG torque (-> k_s) or a requested quantity,
//            and for the last stage of an FSAL method the max-norm error and the
//            max torque of the step.
// The padded sizes are powers of two P >= 2n-1 and the kernel is stored
// circularly (r = 0 at index 0), so the result is the reference's linear
// convolution of the zero-padded magnetisation (strayfieldkernel.cu:80-99).
// Each block first copies its magnet and group descriptors to shared memory.
#pragma once
#include "fft.cuh"
#include "physics.cuh"

namespace mpx {

// Butcher tableau of the current method (core/butchertableau.cpp), in constant memory.
struct TableauDev {
  int S, order1, order2, fsal;
  double c[7];
  double a[7][7];
  double b1[7], b2[7];
};
__constant__ TableauDev c_tab;

// Block size bounds: the x passes hold 8 FFT values per thread, so a block of
// X_THREADS_MAX threads covers transforms of up to 8*X_THREADS_MAX points; the
// y/z pass holds 16 per thread.
constexpr int X_THREADS_MAX = 384;
constexpr int X_VPT = 8;
constexpr int YZ_VPT = 16;

// Work item of the row-tile kernels: magnet slot, z, first row y0, rows in tile (<= TY_MAX).
// Work item of k_yz: magnet slot, first kx (in z), number of consecutive kx (in y0).
constexpr int TY_MAX = 16;
struct Work {
  int mag, z, y0, ty;
};

enum { EPI_STAGE = 0, EPI_EVAL = 1 };

struct EpiArgs {
  int mode;      // EPI_STAGE: write k_s ; EPI_EVAL: write `quantity` into out
  int stage;
  int quantity;  // mpx_quantity
  int fsal_err;  // fuse error + max torque (last stage of an FSAL method)
  int gate;      // skip groups that are not running
  float* out;    // EPI_EVAL output (device, 3N or N floats)
  const float* msrc;  // EPI_EVAL: magnetisation source (NULL: group state x0)
};

template <typename T>
__device__ __forceinline__ void copy_to_smem(T* dst, const T* __restrict__ src) {
  static_assert(sizeof(T) % 4 == 0, "descriptor size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) d[i] = s[i];
}

// Loads the magnet and group descriptors of this block; returns false when the
// block has nothing to do (group not running, or k0 already valid for stage 0).
// A negative magnet slot marks a hole of a launch table (a solve that is no
// longer launched): the block has nothing to do.
__device__ __forceinline__ bool load_descs(MagnetDev& sM, GroupDev& sG, const MagnetDev* __restrict__ mags,
                                           const GroupDev* __restrict__ groups, int mag, int gate, int stage) {
  if (mag < 0) return false;
  copy_to_smem(&sM, mags + mag);
  __syncthreads();
  copy_to_smem(&sG, groups + sM.group);
  __syncthreads();
  if (!gate) return true;
  if (sG.status != GS_RUNNING) return false;
  if (stage == 0 && sG.k0_valid) return false;
  return true;
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// serialisation attribute may start while the previous kernel of the stream is
// still running (after every block of that kernel has passed pdl_trigger or
// exited): before pdl_wait it reads only data that no kernel of the current
// attempt writes (magnet and group descriptors, twiddle tables); pdl_wait
// returns once the previous kernel has completed and its writes are visible.
// Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Bulk L2 prefetch (cp.async.bulk.prefetch.L2) of the 16-byte-aligned interior
// of [p, p + bytes), in pieces of at most 64 KB: a hint with no completion to
// wait for, issued by one thread for data that the block reads later (the
// Newell spectrum slab of its kx), so that those loads find the lines in L2
// instead of DRAM.  The range never leaves the given buffer.  (The tile rows of
// the x passes are L2 hits already: prefetching them measured slower.)
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
  uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)p + bytes) & ~(uintptr_t)15;
  while (a < e) {
    const uint32_t n = (uint32_t)min((uintptr_t)65536, e - a);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
    a += n;
  }
}

// Current magnetisation used by stage `stage`: x0 for stage 0, the stage state otherwise.
__device__ __forceinline__ const float* stage_m(const MagnetDev& M, const GroupDev& G, int stage) {
  return stage == 0 ? M.buf[G.map[0]] : M.buf[G.map[1]];
}

// x^2 + y^2 + z^2 with its roundings spelled out, so that every form of the
// stage combination below rounds alike
__device__ __forceinline__ float norm2_rn(float x, float y, float z) {
  return __fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x)));
}

// Stage combination x_s = normalize(x0 + sum_j dt a_sj k_j) of one cell
// (core/rungekutta.cpp:108-134, core/fieldops.cu:232-258).
__device__ __forceinline__ float3 combine_cell(const MagnetDev& M, const GroupDev& G, int stage, int i,
                                               bool final_b1) {
  const int N = M.N;
  float3 v = ldg3(M.buf[G.map[0]], N, i);
  const int nj = final_b1 ? c_tab.S : stage;
  // unrolled over the 7 possible stages (predicated), so that the loads of all
  // k_j are in flight together; the sum keeps the order j = 0, 1, ...
  float3 k[7];
#pragma unroll
  for (int j = 0; j < 7; ++j)
    if (j < nj) k[j] = ldg3(M.buf[G.map[2 + j]], N, i);
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    if (j < nj) {
      const double co = final_b1 ? c_tab.b1[j] : c_tab.a[stage][j];
      const float cf = (float)(G.dt * co);
      v = f3(__fmaf_rn(cf, k[j].x, v.x), __fmaf_rn(cf, k[j].y, v.y), __fmaf_rn(cf, k[j].z, v.z));
    }
  }
  const float inv = rsqrtf(norm2_rn(v.x, v.y, v.z));
  return f3(__fmul_rn(v.x, inv), __fmul_rn(v.y, inv), __fmul_rn(v.z, inv));
}

// combine_cell for a stage (not the final b1 sum) with the coefficients
// (float)(dt a_sj) and the k_j pointers of the block taken from shared memory:
// the same sums, without an FP64 product and a double indirection per cell.
__device__ __forceinline__ float3 combine_cell_pre(const float* __restrict__ x0, int N, int stage, int i,
                                                   const float* cf, const float* const* kp) {
  float3 v = ldg3(x0, N, i);
  float3 k[7];
#pragma unroll
  for (int j = 0; j < 7; ++j)
    if (j < stage) k[j] = ldg3(kp[j], N, i);
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    if (j < stage) {
      const float c = cf[j];
      v = f3(__fmaf_rn(c, k[j].x, v.x), __fmaf_rn(c, k[j].y, v.y), __fmaf_rn(c, k[j].z, v.z));
    }
  }
  const float inv = rsqrtf(norm2_rn(v.x, v.y, v.z));
  return f3(__fmul_rn(v.x, inv), __fmul_rn(v.y, inv), __fmul_rn(v.z, inv));
}

__device__ __forceinline__ float f4c(const float4& a, int q) { return q == 0 ? a.x : q == 1 ? a.y : q == 2 ? a.z : a.w; }
__device__ __forceinline__ void f4set(float4& a, int q, float v) {
  if (q == 0) a.x = v; else if (q == 1) a.y = v; else if (q == 2) a.z = v; else a.w = v;
}

// combine_cell_pre for the four consecutive cells i .. i + 3 (i a multiple of
// 4, every buffer 16-byte aligned): 16-byte loads and stores, the same sums in
// the same order per cell. The stage state goes to xs; returns it in r.
__device__ __forceinline__ void combine_quad_pre(const float* __restrict__ x0, float* xs, int N, int stage, int i,
                                                 const float* cf, const float* const* kp, float4 r[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) r[c] = __ldg(reinterpret_cast<const float4*>(x0 + c * N + i));
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    if (j < stage) {
      const float cj = cf[j];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float4 k = __ldg(reinterpret_cast<const float4*>(kp[j] + c * N + i));
        r[c] = make_float4(__fmaf_rn(cj, k.x, r[c].x), __fmaf_rn(cj, k.y, r[c].y), __fmaf_rn(cj, k.z, r[c].z),
                           __fmaf_rn(cj, k.w, r[c].w));
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float vx = f4c(r[0], q), vy = f4c(r[1], q), vz = f4c(r[2], q);
    const float inv = rsqrtf(norm2_rn(vx, vy, vz));
    f4set(r[0], q, __fmul_rn(vx, inv));
    f4set(r[1], q, __fmul_rn(vy, inv));
    f4set(r[2], q, __fmul_rn(vz, inv));
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) *reinterpret_cast<float4*>(xs + c * N + i) = r[c];
}

// Row index e / n within a tile of at most TY_MAX rows of length n, without
// an integer division: a float estimate of (e + 1/2) / n (exact unless n is
// very large) corrected by one step either way.
__device__ __forceinline__ int tile_row(int e, int n, float rn) {
  int r = (int)(((float)e + 0.5f) * rn);
  r -= (r * n > e) ? 1 : 0;
  r += ((r + 1) * n <= e) ? 1 : 0;
  return r;
}

// log2 of the power of two >= ty (ty <= TY_MAX): row slots of a tile
__device__ __forceinline__ int tile_log(int ty) { return ty <= 1 ? 0 : 32 - __clz(ty - 1); }

// ------------------------------------------------------------------ k_xfwd
// smem: padded rows [ty] for (Mx + i My) of each row, then [(ty+1)/2] for
// (Mz(y) + i Mz(y+1)).
// PAIR: the 2048-point rows of the warp pairs are compiled in (the forms launched
// when a magnet with such rows is in the launch; without them the others keep
// the registers and code of the shorter lengths).
template <bool COMBINE, bool PAIR = false>
__global__ void __launch_bounds__(X_THREADS_MAX, 2) k_xfwd(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups,
                                              const Work* __restrict__ work, int stage, int gate,
                                              const float* __restrict__ msrc_override,
                                              const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();  // the y/z pass may start its prologue during this kernel's last wave
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  const int z = wk.z, y0 = wk.y0, ty = wk.ty;
  const int nx = M.n[0], ny = M.n[1], nz = M.n[2], N = M.N;
  const int logL = M.logP[0], L = 1 << logL, cs = xrow_stride(L, ty);
  if (!PAIR && logL == 11) return;  // 2048-point rows only in the PAIR form (the host never launches them here)
  const int nzrows = (ty + 1) >> 1;
  const float* src = msrc_override ? msrc_override : stage_m(M, G, stage);
  float* xs = M.buf[G.map[1]];
  const float* x0 = M.buf[G.map[0]];
  const int rowbase = nx * (y0 + ny * z);
  float2* tws = sm + (ty + nzrows) * cs;  // twiddles of length L
  const bool wrow = (PAIR && logL == 11) || logL == 10 || logL == 9;  // 2048- / 1024- / 512-point rows: warp (pair) rows
  const int sh = wrow ? 5 : 4;
  if (wrow) load_twq(tws, tw, logL);
  else load_twiddles<3>(tws, tw, logL);
  __shared__ float s_cf[8];
  __shared__ const float* s_kp[8];
  __shared__ int s_al;  // every buffer the block reads or writes is 16-byte aligned
  if (threadIdx.x == 0) {
    uintptr_t a = (uintptr_t)src | (uintptr_t)xs | (uintptr_t)x0;
    if (COMBINE)
      for (int j = 0; j < stage; ++j) a |= (uintptr_t)M.buf[G.map[2 + j]];
    s_al = (a & 15) == 0;
  }
  if (COMBINE) {  // the stage's coefficients and k_j buffers, once per block
    if (threadIdx.x < 7) {
      const int j = threadIdx.x;
      s_cf[j] = (j < stage) ? (float)(G.dt * c_tab.a[stage][j]) : 0.f;
      s_kp[j] = M.buf[G.map[2 + j]];
    }
  }
  __syncthreads();
  pdl_wait();  // the stage state and derivatives are written by the earlier passes

  // only the lower half of each row: the upper half (x >= L/2 >= nx) is zero
  // padding that the pruned first FFT pass does not read
  const int logLh = logL > 0 ? logL - 1 : 0;
  if ((nx & 3) == 0 && logLh >= 2 && !M.geom && !M.msat.p && s_al) {
    // four consecutive cells per thread with 16-byte loads and stores (no
    // geometry, uniform Ms; nx and so N a multiple of 4)
    const int lq = logLh - 2;
    const float ms = M.msat.u;
    for (int e = threadIdx.x; e < (ty << lq); e += blockDim.x) {
      const int yl = e >> lq, x = (e & ((1 << lq) - 1)) << 2;
      float4 r[3];
      const int i = rowbase + yl * nx + x;
      if (x < nx && cell_ok(N, i) && cell_ok(N, i + 3)) {
        if (COMBINE) {
          combine_quad_pre(x0, xs, N, stage, i, s_cf, s_kp, r);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) r[c] = __ldg(reinterpret_cast<const float4*>(src + c * N + i));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
          r[c] = make_float4(__fmul_rn(ms, r[c].x), __fmul_rn(ms, r[c].y), __fmul_rn(ms, r[c].z), __fmul_rn(ms, r[c].w));
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) r[c] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      float2* row = sm + yl * cs;
      float* zr = reinterpret_cast<float*>(sm + (ty + (yl >> 1)) * cs);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int xi = xidx(x + q, sh);
        row[xi] = make_float2(f4c(r[0], q), f4c(r[1], q));
        zr[2 * xi + (yl & 1)] = f4c(r[2], q);
        if ((ty & 1) && yl == ty - 1) zr[2 * xi + 1] = 0.0f;
      }
    }
  } else {
#pragma unroll 2
  for (int e = threadIdx.x; e < (ty << logLh); e += blockDim.x) {
    const int yl = e >> logLh, x = e & ((1 << logLh) - 1);
    float3 Mv = f3(0, 0, 0);
    if (x < nx) {
      const int i = rowbase + yl * nx + x;
      if (in_geom(M, i)) {
        float3 m;
        if (COMBINE) {
          m = combine_cell_pre(x0, N, stage, i, s_cf, s_kp);
          store3(xs, N, i, m);
        } else {
          m = ldg3(src, N, i);
        }
        Mv = M.msat.at(i) * m;
      } else if (COMBINE) {
        store3(xs, N, i, load3(x0, N, i));
      }
    }
    sm[yl * cs + xidx(x, sh)] = make_float2(Mv.x, Mv.y);
    float* zr = reinterpret_cast<float*>(sm + (ty + (yl >> 1)) * cs + xidx(x, sh));
    zr[yl & 1] = Mv.z;
    if ((ty & 1) && yl == ty - 1) zr[1] = 0.0f;
  }
  }
  __syncthreads();
  if (wrow) {
    if (PAIR && logL == 11) pair_rows<-1, true, false>(sm, ty + nzrows, cs, tws);
    else if (logL == 10) warp_rows<32, -1, true, false>(sm, ty + nzrows, cs, tws);
    else warp_rows<16, -1, true, false>(sm, ty + nzrows, cs, tws);
    __syncthreads();
  } else {
    fft_many<-1, 3, 1>(sm, logL, ty + nzrows, cs, tws);
  }

  // unpack the two real transforms of each complex row and store the half spectrum
  const int Fh = M.Fh;
  float2* S = M.spec;
  const int tyl = tile_log(ty);
  if ((ny & 1) == 0) {
    // even ny: rows 2p, 2p + 1 of one kx, all three components (one 16-byte
    // store each, every offset is even); the x and y values come from the two
    // complex rows, the z values of the pair from one packed row
    const int pl = tyl - 1;
    const size_t cstr = (size_t)nz * ny, stot = (size_t)Fh * 3 * cstr;
    for (int e = threadIdx.x; e < Fh << pl; e += blockDim.x) {
      const int yp = e & ((1 << pl) - 1);
      if (2 * yp >= ty) continue;
      const int kx = e >> pl;
      const int xk = xidx(kx, sh), xc = xidx((L - kx) & (L - 1), sh);
      const float2* Z0 = sm + (2 * yp) * cs;
      const float2* Z1 = Z0 + cs;
      const float2* Zz = sm + (ty + yp) * cs;
      const float2 zk0 = Z0[xk], zc0 = cconj(Z0[xc]), zk1 = Z1[xk], zc1 = cconj(Z1[xc]);
      const float2 zkz = Zz[xk], zcz = cconj(Zz[xc]);
      const size_t si = ((size_t)kx * 3 * nz + z) * ny + y0 + 2 * yp;
      if (span_ok(si + 2 * cstr + 1, stot)) {
        // x: (zk + zc) / 2 ; y: -i/2 (zk - zc), of each row
        *reinterpret_cast<float4*>(S + si) = make_float4(0.5f * (zk0.x + zc0.x), 0.5f * (zk0.y + zc0.y),
                                                         0.5f * (zk1.x + zc1.x), 0.5f * (zk1.y + zc1.y));
        *reinterpret_cast<float4*>(S + si + cstr) = make_float4(0.5f * (zk0.y - zc0.y), -0.5f * (zk0.x - zc0.x),
                                                                0.5f * (zk1.y - zc1.y), -0.5f * (zk1.x - zc1.x));
        *reinterpret_cast<float4*>(S + si + 2 * cstr) = make_float4(0.5f * (zkz.x + zcz.x), 0.5f * (zkz.y + zcz.y),
                                                                    0.5f * (zkz.y - zcz.y), -0.5f * (zkz.x - zcz.x));
      }
    }
    return;
  }
  // odd ny: row yl of one kx, all three components (x, y from its complex row,
  // z from the first or second half of the packed row of its pair)
  const size_t cstr = (size_t)nz * ny, stot = (size_t)Fh * 3 * cstr;
  for (int e = threadIdx.x; e < Fh << tyl; e += blockDim.x) {
    const int yl = e & ((1 << tyl) - 1);
    if (yl >= ty) continue;
    const int kx = e >> tyl;
    const int xk = xidx(kx, sh), xc = xidx((L - kx) & (L - 1), sh);
    const float2* Z = sm + yl * cs;
    const float2* Zz = sm + (ty + (yl >> 1)) * cs;
    const float2 zk = Z[xk], zc = cconj(Z[xc]), zkz = Zz[xk], zcz = cconj(Zz[xc]);
    const size_t si = ((size_t)kx * 3 * nz + z) * ny + y0 + yl;
    if (span_ok(si + 2 * cstr, stot)) {
      S[si] = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
      S[si + cstr] = make_float2(0.5f * (zk.y - zc.y), -0.5f * (zk.x - zc.x));  // -i/2 (zk - zc)
      S[si + 2 * cstr] = (yl & 1) ? make_float2(0.5f * (zkz.y - zcz.y), -0.5f * (zkz.x - zcz.x))
                                  : make_float2(0.5f * (zkz.x + zcz.x), 0.5f * (zkz.y + zcz.y));
    }
  }
}

// --------------------------------------------------------------------- k_yz
// Kernel spectrum entry (comp cc of the xx,yy,zz,xy,xz,yz order) at (kx, ky, kz)
// from the symmetry-reduced storage [kx][kz'][kcomp][ky'].
// `left`: elements of the kernel spectrum from Kx to its end (checked build).
template <int PZ>
__device__ __forceinline__ void kernel_at(const float* __restrict__ Kx, int kc, int hy, int kyp, float sy, int kz,
                                          float& kxx, float& kyy, float& kzz, float& kxy, float& kxz, float& kyz,
                                          size_t left) {
  const int kzp = min(kz, PZ - kz);
  const float sz = (kz > PZ / 2) ? -1.f : 1.f;
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

__device__ __forceinline__ void apply3(float2* v0, float2* v1, float2* v2, float kxx, float kyy, float kzz, float kxy,
                                       float kxz, float kyz) {
  const float2 mx = *v0, my = *v1, mz = *v2;
  *v0 = make_float2(kxx * mx.x + kxy * my.x + kxz * mz.x, kxx * mx.y + kxy * my.y + kxz * mz.y);
  *v1 = make_float2(kxy * mx.x + kyy * my.x + kyz * mz.x, kxy * mx.y + kyy * my.y + kyz * mz.y);
  *v2 = make_float2(kxz * mx.x + kyz * my.x + kzz * mz.x, kxz * mx.y + kyz * my.y + kzz * mz.y);
}

// z stage of one ky, half = 0 / 1 computing the even / odd kz of the PZ-point
// transform of nz <= PZ/2 inputs as a PZ/2-point transform (of x, or of
// x[n] W_PZ^n); the partner lane (lane ^ PARTNER) holds the other half and the
// two inverse halves are summed with one shuffle.  Q5: columns in the qidx
// layout of the warp transforms (else pidx).  PARTNER 16: the two halves of a
// warp take the even / odd kz of the same 16 ky, so that every store of a
// half-warp goes to one column at 16 consecutive ky (no bank conflicts).
template <int PZ, bool Q5 = false, int PARTNER = 1>
__device__ __forceinline__ void zstage_pair(float2* D, int cs, const MagnetDev& M, int kx, int ky, int half, int nz,
                                            int Py) {
  constexpr int H = PZ / 2;
  float2 v[3][H];
  const int pky = Q5 ? qidx(ky) : pidx(ky);
  // kernel spectrum of this lane's kz values, issued before the transforms
  const int hy = Py / 2 + 1;
  const int kyp = min(ky, Py - ky);
  const float sy = (ky > Py / 2) ? -1.f : 1.f;
  const int kc = M.kcomp;
  const float* __restrict__ Kx = M.kspec + (size_t)kx * (PZ / 2 + 1) * kc * hy;
  const size_t kleft = (size_t)(M.Fh - kx) * (PZ / 2 + 1) * kc * hy;
  float kk[H][6];
#pragma unroll
  for (int q = 0; q < H; ++q)
    kernel_at<PZ>(Kx, kc, hy, kyp, sy, 2 * q + half, kk[q][0], kk[q][1], kk[q][2], kk[q][3], kk[q][4], kk[q][5],
                  kleft);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int n = 0; n < H; ++n) v[c][n] = (n < nz) ? D[(c * nz + n) * cs + pky] : make_float2(0.f, 0.f);
  if (half) {
#pragma unroll
    for (int n = 1; n < H; ++n)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        switch ((16 / PZ) * n) {  // times exp(-2 pi i n / PZ)
          case 1: v[c][n] = rot16<-1, 1>(v[c][n]); break;
          case 2: v[c][n] = rot16<-1, 2>(v[c][n]); break;
          case 3: v[c][n] = rot16<-1, 3>(v[c][n]); break;
          case 4: v[c][n] = rot16<-1, 4>(v[c][n]); break;
          case 5: v[c][n] = rot16<-1, 5>(v[c][n]); break;
          case 6: v[c][n] = rot16<-1, 6>(v[c][n]); break;
          case 7: v[c][n] = rot16<-1, 7>(v[c][n]); break;
          default: break;
        }
      }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) dft_reg<H, -1>(v[c]);
#pragma unroll
  for (int q = 0; q < H; ++q)
    apply3(&v[0][q], &v[1][q], &v[2][q], kk[q][0], kk[q][1], kk[q][2], kk[q][3], kk[q][4], kk[q][5]);
#pragma unroll
  for (int c = 0; c < 3; ++c) dft_reg<H, 1>(v[c]);
  if (half) {
#pragma unroll
    for (int n = 1; n < H; ++n)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        switch ((16 / PZ) * n) {  // times exp(+2 pi i n / PZ)
          case 1: v[c][n] = rot16<1, 1>(v[c][n]); break;
          case 2: v[c][n] = rot16<1, 2>(v[c][n]); break;
          case 3: v[c][n] = rot16<1, 3>(v[c][n]); break;
          case 4: v[c][n] = rot16<1, 4>(v[c][n]); break;
          case 5: v[c][n] = rot16<1, 5>(v[c][n]); break;
          case 6: v[c][n] = rot16<1, 6>(v[c][n]); break;
          case 7: v[c][n] = rot16<1, 7>(v[c][n]); break;
          default: break;
        }
      }
  }
  // reduce-scatter over the lane pair: lane `half` keeps the outputs n with
  // n % 2 == half (own value + the partner's), so each lane sends only the half
  // its partner keeps
  const unsigned mask = __activemask();
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; 2 * k < H; ++k) {
      const float2 ev = v[c][2 * k];
      const float2 od = (2 * k + 1 < H) ? v[c][2 * k + 1] : make_float2(0.f, 0.f);
      const float2 send = half ? ev : od;
      const float2 mine = half ? od : ev;
      const float ox = __shfl_xor_sync(mask, send.x, PARTNER);
      const float oy = __shfl_xor_sync(mask, send.y, PARTNER);
      const int n = 2 * k + half;
      if (n < H && n < nz) D[(c * nz + n) * cs + pky] = make_float2(mine.x + ox, mine.y + oy);
    }
}

// exp(DIR 2 pi i m / 16) v for m = 0 .. 7 known at compile time after unrolling
template <int DIR>
__device__ __forceinline__ float2 rot16_m(float2 v, int m) {
  switch (m) {
    case 1: return rot16<DIR, 1>(v);
    case 2: return rot16<DIR, 2>(v);
    case 3: return rot16<DIR, 3>(v);
    case 4: return rot16<DIR, 4>(v);
    case 5: return rot16<DIR, 5>(v);
    case 6: return rot16<DIR, 6>(v);
    case 7: return rot16<DIR, 7>(v);
    default: return v;
  }
}

// z stage of one ky in one lane (PZ = 2 .. 16): both halves of zstage_pair<PZ>
// (the even kz = 2q from the PZ/2-point transform of x, the odd kz = 2q + 1
// from that of x[n] W_PZ^n), the 3x3 multiply per kz, and the output as the
// sum of the two PZ/2-point inverses: the same operations on the same values,
// without the lane exchange, the per-lane branch of the odd half's twiddles or
// the selects of the reduce-scatter.  kz and PZ - kz share their kernel entries
// up to the sign of the xz and yz components (odd in z), so each lane loads the
// PZ/2 + 1 kz' once.  The even half's inverse is parked in the lane's own input
// entries while the odd half runs, so that one set of 3 PZ/2 values is live.
template <int PZ, bool Q5>
__device__ __forceinline__ void zstage_full(float2* D, int cs, const MagnetDev& M, int kx, int ky, int nz, int Py) {
  constexpr int H = PZ / 2, R = 16 / PZ;  // kz per half; W_PZ = W16^R
  const int pky = Q5 ? qidx(ky) : pidx(ky);
  const int hy = Py / 2 + 1;
  const int kyp = min(ky, Py - ky);
  const float sy = (ky > Py / 2) ? -1.f : 1.f;
  const int kc = M.kcomp;
  const float* __restrict__ Kx = M.kspec + (size_t)kx * (H + 1) * kc * hy;
  const size_t kleft = (size_t)(M.Fh - kx) * (H + 1) * kc * hy;
  float kk[H + 1][6];  // kz' = 0 .. H: the even ones now, the odd ones before the odd kz
#pragma unroll
  for (int p = 0; p <= H; p += 2)
    kernel_at<PZ>(Kx, kc, hy, kyp, sy, p, kk[p][0], kk[p][1], kk[p][2], kk[p][3], kk[p][4], kk[p][5], kleft);
  float2 e[3][H];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int n = 0; n < H; ++n) e[c][n] = (n < nz) ? D[(c * nz + n) * cs + pky] : make_float2(0.f, 0.f);
    dft_reg<H, -1>(e[c]);
  }
#pragma unroll
  for (int q = 0; q < H; ++q) {  // kz = 2q, kz' = min(kz, PZ - kz), mirrored above PZ/2
    const int p = 2 * q <= H ? 2 * q : PZ - 2 * q;
    const float sg = 2 * q > H ? -1.f : 1.f;
    apply3(&e[0][q], &e[1][q], &e[2][q], kk[p][0], kk[p][1], kk[p][2], kk[p][3], sg * kk[p][4], sg * kk[p][5]);
  }
#pragma unroll
  for (int p = 1; p <= H; p += 2)
    kernel_at<PZ>(Kx, kc, hy, kyp, sy, p, kk[p][0], kk[p][1], kk[p][2], kk[p][3], kk[p][4], kk[p][5], kleft);
#pragma unroll
  for (int c = 0; c < 3; ++c) dft_reg<H, 1>(e[c]);
  float2 o[3][H];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int n = 0; n < H; ++n) o[c][n] = (n < nz) ? D[(c * nz + n) * cs + pky] : make_float2(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int n = 0; n < H; ++n)
      if (n < nz) D[(c * nz + n) * cs + pky] = e[c][n];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int n = 1; n < H; ++n) o[c][n] = rot16_m<-1>(o[c][n], R * n);
    dft_reg<H, -1>(o[c]);
  }
#pragma unroll
  for (int q = 0; q < H; ++q) {  // kz = 2q + 1
    const int p = 2 * q + 1 <= H ? 2 * q + 1 : PZ - 2 * q - 1;
    const float sg = 2 * q + 1 > H ? -1.f : 1.f;
    apply3(&o[0][q], &o[1][q], &o[2][q], kk[p][0], kk[p][1], kk[p][2], kk[p][3], sg * kk[p][4], sg * kk[p][5]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dft_reg<H, 1>(o[c]);
#pragma unroll
    for (int n = 1; n < H; ++n) o[c][n] = rot16_m<1>(o[c][n], R * n);
#pragma unroll
    for (int n = 0; n < H; ++n)
      if (n < nz) {
        const float2 ev = D[(c * nz + n) * cs + pky];
        D[(c * nz + n) * cs + pky] = make_float2(ev.x + o[c][n].x, ev.y + o[c][n].y);
      }
  }
}

template <bool Q5 = false>
__device__ __forceinline__ void zstage_single(float2* D, int cs, const MagnetDev& M, int kx, int ky, int Py) {
  const int pky = Q5 ? qidx(ky) : pidx(ky);
  float2 v0 = D[pky], v1 = D[cs + pky], v2 = D[2 * cs + pky];
  const int hy = Py / 2 + 1;
  const int kyp = min(ky, Py - ky);
  const float sy = (ky > Py / 2) ? -1.f : 1.f;
  const int kc = M.kcomp;
  const float* __restrict__ Kx = M.kspec + (size_t)kx * kc * hy;
  float kxx, kyy, kzz, kxy, kxz, kyz;
  kernel_at<1>(Kx, kc, hy, kyp, sy, 0, kxx, kyy, kzz, kxy, kxz, kyz, (size_t)(M.Fh - kx) * kc * hy);
  apply3(&v0, &v1, &v2, kxx, kyy, kzz, kxy, kxz, kyz);
  D[pky] = v0;
  D[cs + pky] = v1;
  D[2 * cs + pky] = v2;
}

// L2 prefetch (thread 0) of the Newell spectrum slabs [kx][kz'][kcomp][ky'] of
// kx0 .. kx0 + nkx - 1 that a y/z block reads in its z stage: constant data, so
// it is issued before pdl_wait and lands while the y transforms run.
__device__ __forceinline__ void prefetch_kslab(const MagnetDev& M, int kx0, int nkx, int Pz) {
  if (threadIdx.x != 0) return;
  const int n = min(nkx, M.Fh - kx0);
  if (n <= 0) return;
  const size_t slab = (size_t)(Pz / 2 + 1) * M.kcomp * ((1 << M.logP[1]) / 2 + 1);
  prefetch_l2(M.kspec + (size_t)kx0 * slab, (size_t)n * slab * sizeof(float));
}

// MAXLR = 4: radix-16 passes, 16 values per thread (y lengths up to 4096, one
// 384-thread block per SM by registers); MAXLR = 3: radix-8 passes, 8 values
// per thread, two blocks per SM (y lengths up to 2048, z length up to 8).  At
// z length 16 the radix-8 form measured slower (more passes, and the z stage
// needs 128 registers, so at most 512 threads).
template <int PZ, int MAXLR>
__global__ void __launch_bounds__(384, MAXLR == 3 ? 2 : 1)
    k_yz(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups,
                                            const Work* __restrict__ work, int stage, int gate,
                                            const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  const int kx0 = wk.z, nkx = wk.y0;
  const int ny = M.n[1], nz = M.n[2];
  const int logPy = M.logP[1], Py = 1 << logPy, cs = plen(Py);
  float2* S = M.spec + (size_t)kx0 * 3 * nz * ny;  // the nkx slabs are consecutive
  const size_t sleft = (size_t)(M.Fh - kx0) * 3 * nz * ny;  // elements of the spectrum from S on (checked build)
  float2* D = sm;  // [nkx][3*nz] padded columns of length Py
  const int ncol = nkx * 3 * nz;
  float2* tws = sm + ncol * cs;  // twiddles of length Py
  load_twiddles<MAXLR>(tws, tw, logPy);
  prefetch_kslab(M, kx0, nkx, PZ);
  pdl_wait();  // the spectrum is written by the x pass
  // slab load: 8 independent read-only loads in flight per thread; only the
  // lower half of each column (y < Py/2, of which y >= ny is zero padding),
  // which is all the pruned first FFT pass reads
  const int logPyh = logPy > 0 ? logPy - 1 : 0;
  const int total = ncol << logPyh;
  for (int e0 = threadIdx.x; e0 < total; e0 += 8 * blockDim.x) {
    float2 r[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * blockDim.x;
      const int col = e >> logPyh, y = e & ((1 << logPyh) - 1);
      r[u] = (e < total && y < ny && span_ok((size_t)col * ny + y, sleft)) ? __ldg(S + col * ny + y)
                                                                           : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < total) D[(e >> logPyh) * cs + pidx(e & ((1 << logPyh) - 1))] = r[u];
    }
  }
  __syncthreads();
  fft_many<-1, MAXLR, 1>(D, logPy, ncol, cs, tws);
  if constexpr (PZ == 1) {
    for (int t = threadIdx.x; t < nkx << logPy; t += blockDim.x) {
      const int j = t >> logPy;
      zstage_single(D + j * 3 * cs, cs, M, kx0 + j, t & (Py - 1), Py);
    }
  } else {
    // lanes 2u and 2u+1 share one (kx, ky): the even and odd kz halves
    for (int t = threadIdx.x; t < (2 * nkx) << logPy; t += blockDim.x) {
      const int u = t >> 1, j = u >> logPy;
      zstage_pair<PZ>(D + j * 3 * nz * cs, cs, M, kx0 + j, u & (Py - 1), t & 1, nz, Py);
    }
  }
  __syncthreads();
  fft_many<1, MAXLR, 2>(D, logPy, ncol, cs, tws);  // only y < ny <= Py/2 is written back
  for (int e = threadIdx.x; e < (ncol << logPy); e += blockDim.x) {
    const int col = e >> logPy, y = e & (Py - 1);
    if (y < ny && span_ok((size_t)col * ny + y, sleft)) S[col * ny + y] = D[col * cs + pidx(y)];
  }
}

// ---------------------------------------------------------------- k_yzw
// The y/z pass for y lengths 64 .. 1024 (Py = 32 Q): every warp transforms
// whole columns in registers (four-step Q x 32, 32 / Q columns at a time),
// reading its columns of S straight into the inner step and writing the y < ny
// outputs straight back; the block synchronises only around the z stage.
// Columns in the qidx layout, cs = qlen(Py).

// Forward y transforms of the ncol columns of S (ny rows each, zero padding
// above) into D.
template <int Q>
__device__ __forceinline__ void yzw_forward(const float2* __restrict__ S, int ny, float2* D, int ncol,
                                            const float2* twq, size_t sleft) {
  constexpr int W = 32 / Q, cs = qlen(32 * Q);
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int lc = lane / Q, ls = lane % Q;  // column and s of this lane in the outer step
  for (int col0 = (threadIdx.x >> 5) * W; col0 < ncol; col0 += nw * W) {
    const int nc = W == 1 ? 1 : min(W, ncol - col0);
    float2 v[32];
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
      for (int r = 0; r < Q; ++r) {  // y = lane + 32 r < Py/2; y >= ny is zero padding
        const int y = lane + 32 * r;
        v[c * Q + r] = (c < nc && r < Q / 2 && y < ny && span_ok((size_t)(col0 + c) * ny + y, sleft))
                           ? __ldg(S + (size_t)(col0 + c) * ny + y)
                           : make_float2(0.f, 0.f);
      }
    four_step_inner<Q, -1, true>(v, twq, lane);
    float2* C = D + col0 * cs;
    four_step_outer<Q, -1, false>(v, C, cs, nc, lane);
    if constexpr (W == 1) {
#pragma unroll
      for (int t = 0; t < 32; ++t) C[lane + 33 * t] = v[t];  // ky = lane + 32 t
    } else if (lc < nc) {
#pragma unroll
      for (int t = 0; t < 32; ++t) C[lc * cs + qidx(ls + Q * t)] = v[t];  // ky = s + Q t
    }
  }
}

// Inverse y transforms of the columns of D; the y < ny outputs go to S.
template <int Q>
__device__ __forceinline__ void yzw_inverse(float2* __restrict__ S, int ny, float2* D, int ncol, const float2* twq,
                                            size_t sleft) {
  constexpr int W = 32 / Q, cs = qlen(32 * Q);
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int lc = lane / Q, ls = lane % Q;
  for (int col0 = (threadIdx.x >> 5) * W; col0 < ncol; col0 += nw * W) {
    const int nc = W == 1 ? 1 : min(W, ncol - col0);
    float2* C = D + col0 * cs;
    float2 v[32];
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
      for (int r = 0; r < Q; ++r) v[c * Q + r] = (c < nc) ? C[c * cs + lane + 33 * r] : make_float2(0.f, 0.f);
    four_step_inner<Q, 1, false>(v, twq, lane);
    four_step_outer<Q, 1, true>(v, C, cs, nc, lane);
    const int cl = W == 1 ? 0 : lc, sl = W == 1 ? lane : ls;
    if (cl < nc) {
      float2* __restrict__ Sc = S + (size_t)(col0 + cl) * ny;
#pragma unroll
      for (int t = 0; t < 16; ++t) {  // y = s + Q t < Py/2: only y < ny is kept
        const int y = sl + Q * t;
        if (y < ny && span_ok((size_t)(col0 + cl) * ny + y, sleft)) Sc[y] = v[t];
      }
    }
  }
}

// Threads per block: 384 at z length 16 (the z stage needs ~128 registers:
// one block per SM), else 256 (128 registers, two blocks per SM).
template <int PZ>
constexpr int yzw_threads() { return PZ == 16 ? 384 : 256; }

// The whole y/z pass of one block for y length Py = 32 Q (every length and
// stride a compile-time constant).
template <int PZ, int Q>
__device__ __forceinline__ void yzw_body(const MagnetDev& M, int kx0, int nkx, float2* sm,
                                         const float2* __restrict__ tw) {
  constexpr int Py = 32 * Q, cs = qlen(Py);
  constexpr int LOGPY = Q == 2 ? 6 : Q == 4 ? 7 : Q == 8 ? 8 : Q == 16 ? 9 : 10;
  const int ny = M.n[1], nz = M.n[2];
  const int ncol = nkx * 3 * nz;
  float2* D = sm;
  float2* twq = sm + ncol * cs;
  load_twq(twq, tw, LOGPY);
  prefetch_kslab(M, kx0, nkx, PZ);
  __syncthreads();
  pdl_wait();  // the spectrum is written by the x pass
  float2* S = M.spec + (size_t)kx0 * 3 * nz * ny;
  const size_t sleft = (size_t)(M.Fh - kx0) * 3 * nz * ny;  // elements from S on (checked build)
  yzw_forward<Q>(S, ny, D, ncol, twq, sleft);
  __syncthreads();
  if constexpr (PZ == 1) {
    for (int t = threadIdx.x; t < nkx << LOGPY; t += blockDim.x) {
      const int j = t >> LOGPY;
      zstage_single<true>(D + j * 3 * cs, cs, M, kx0 + j, t & (Py - 1), Py);
    }
  } else if constexpr (PZ >= 4) {  // one lane per (kx, ky)
    for (int t = threadIdx.x; t < nkx << LOGPY; t += blockDim.x) {
      const int j = t >> LOGPY;
      zstage_full<PZ, true>(D + j * 3 * nz * cs, cs, M, kx0 + j, t & (Py - 1), nz, Py);
    }
  } else {
    // lanes l and l + 16 of a warp share one (kx, ky): the even and odd kz
    // halves (the item count is a multiple of 32 and so is the block)
    for (int t = threadIdx.x; t < (2 * nkx) << LOGPY; t += blockDim.x) {
      const int u = ((t >> 5) << 4) | (t & 15), j = u >> LOGPY;
      zstage_pair<PZ, true, 16>(D + j * 3 * nz * cs, cs, M, kx0 + j, u & (Py - 1), (t >> 4) & 1, nz, Py);
    }
  }
  __syncthreads();
  yzw_inverse<Q>(S, ny, D, ncol, twq, sleft);
}

// Work item: magnet, first kx in z, number of consecutive kx in y0.  y lengths 64 .. 512.
template <int PZ>
__global__ void __launch_bounds__(yzw_threads<PZ>(), PZ == 16 ? 1 : 2)
    k_yzw(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
          int stage, int gate, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();  // the x-inverse pass may start its prologue during the last wave
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  const int kx0 = wk.z, nkx = wk.y0;
  switch (M.logP[1]) {
    case 6: yzw_body<PZ, 2>(M, kx0, nkx, sm, tw); break;
    case 7: yzw_body<PZ, 4>(M, kx0, nkx, sm, tw); break;
    case 8: yzw_body<PZ, 8>(M, kx0, nkx, sm, tw); break;
    default: yzw_body<PZ, 16>(M, kx0, nkx, sm, tw); break;
  }
}

// y length 1024 in a kernel of its own: the body of one length keeps the hot
// code small (several fully unrolled bodies in one kernel stalled on
// instruction fetch).
template <int PZ>
__global__ void __launch_bounds__(yzw_threads<PZ>(), PZ == 16 ? 1 : 2)
    k_yzw32(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
            int stage, int gate, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();  // the x-inverse pass may start its prologue during the last wave
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  yzw_body<PZ, 32>(M, wk.z, wk.y0, sm, tw);
}

// y length 2048 in warp pairs (pair_inner / pair_outer of fft.cuh): every pair
// of warps transforms whole columns of length 2048, one at a time, with one
// shared-memory transpose per direction; nkx consecutive kx per block
// (3 nz nkx <= 12 columns, 6 pairs); the z stage as in k_yzw.  Columns in the
// qidx layout, cs = qlen(2048).
constexpr int YZP_THREADS = 384;
template <int PZ>
__global__ void __launch_bounds__(YZP_THREADS, 1)
    k_yzw64(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
            int stage, int gate, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();  // the x-inverse pass may start its prologue during the last wave
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) return;
  constexpr int Py = 2048, LOGPY = 11, cs = qlen(Py);
  const int kx0 = wk.z, nkx = wk.y0;
  const int ny = M.n[1], nz = M.n[2];
  const int ncol = nkx * 3 * nz;
  float2* D = sm;
  float2* twq = sm + ncol * cs;
  load_twq(twq, tw, LOGPY);
  prefetch_kslab(M, kx0, nkx, PZ);
  __syncthreads();
  pdl_wait();  // the spectrum is written by the x pass
  float2* S = M.spec + (size_t)kx0 * 3 * nz * ny;
  const size_t sleft = (size_t)(M.Fh - kx0) * 3 * nz * ny;  // elements from S on (checked build)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, pair = warp >> 1, p = warp & 1;
  const int npairs = blockDim.x >> 6, c = lane + 32 * p;
  for (int col = pair; col < ncol; col += npairs) {  // forward: y < ny in, zero above
    float2* C = D + col * cs;
    float2 v[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      const int y = lane + 32 * r;
      v[r] = (y < ny && span_ok((size_t)col * ny + y, sleft)) ? __ldg(S + (size_t)col * ny + y) : make_float2(0.f, 0.f);
    }
    pair_inner<-1>(v, twq, lane, p, C);
    pair_sync(pair);
    pair_outer<-1, false>(v, C, c);
    pair_sync(pair);  // both warps have read the column before it takes the outputs
#pragma unroll
    for (int t = 0; t < 32; ++t) C[qidx(c + 64 * t)] = v[t];  // ky = c + 64 t
  }
  __syncthreads();
  if constexpr (PZ == 1) {
    for (int t = threadIdx.x; t < nkx << LOGPY; t += blockDim.x) {
      const int j = t >> LOGPY;
      zstage_single<true>(D + j * 3 * cs, cs, M, kx0 + j, t & (Py - 1), Py);
    }
  } else if constexpr (PZ >= 4) {  // one lane per (kx, ky)
    for (int t = threadIdx.x; t < nkx << LOGPY; t += blockDim.x) {
      const int j = t >> LOGPY;
      zstage_full<PZ, true>(D + j * 3 * nz * cs, cs, M, kx0 + j, t & (Py - 1), nz, Py);
    }
  } else {
    // lanes l and l + 16 of a warp share one (kx, ky): the even and odd kz halves
    for (int t = threadIdx.x; t < (2 * nkx) << LOGPY; t += blockDim.x) {
      const int u = ((t >> 5) << 4) | (t & 15), j = u >> LOGPY;
      zstage_pair<PZ, true, 16>(D + j * 3 * nz * cs, cs, M, kx0 + j, u & (Py - 1), (t >> 4) & 1, nz, Py);
    }
  }
  __syncthreads();
  for (int col = pair; col < ncol; col += npairs) {  // inverse: the y < ny outputs go to S
    float2* C = D + col * cs;
    float2 v[32];
#pragma unroll
    for (int b = 0; b < 32; ++b) {  // fold k and k + 1024: x + (-1)^p x'
      const float2 lo = C[qidx(lane + 32 * b)], hi = C[qidx(lane + 32 * b + 1024)];
      v[b] = p ? csub(lo, hi) : cadd(lo, hi);
    }
    pair_sync(pair);  // both warps have read the column before the inner step overwrites it
    pair_inner<1>(v, twq, lane, p, C);
    pair_sync(pair);
    pair_outer<1, true>(v, C, c);
#pragma unroll
    for (int t = 0; t < 16; ++t) {  // y = c + 64 t < 1024
      const int y = c + 64 * t;
      if (y < ny && span_ok((size_t)col * ny + y, sleft)) S[(size_t)col * ny + y] = v[t];
    }
  }
}

// ------------------------------------------------------------- epilogue
__device__ __forceinline__ void block_max2(double a, double b, unsigned long long* pa, unsigned long long* pb) {
  // warp max then one atomic per warp (values are >= 0 or NaN; NaN bits order above +inf)
  unsigned long long ua = __double_as_longlong(a), ub = __double_as_longlong(b);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ua = max(ua, (unsigned long long)__shfl_xor_sync(0xffffffffu, (long long)ua, o));
    ub = max(ub, (unsigned long long)__shfl_xor_sync(0xffffffffu, (long long)ub, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (ua) atomicMax(pa, ua);
    if (ub) atomicMax(pb, ub);
  }
}

// Per-cell epilogue: effective field (+ B_demag) -> torque or requested quantity.
// err_n / tq_n receive the cell's error and torque norms for the FSAL error fusion.
__device__ __forceinline__ void epilogue_cell(const MagnetDev& M, const GroupDev& G, const EpiArgs& ea,
                                              const float* __restrict__ m, int x, int y, int z, int i, float3 bdemag,
                                              double& err_n, double& tq_n) {
  const int N = M.N;
  const bool ing = in_geom(M, i);
  const float3 mc = load3(m, N, i);
  if (ea.mode == EPI_STAGE) {
    float3 k = f3(0, 0, 0);
    if (ing && M.frozen.at(i) == 0.0f) {
      float3 h = f3(0, 0, 0);
      if (M.fast) {
        const LocalOut lo = local_terms_fast(M, m, x, y, z, mc);
        h = lo.exch;
        h = h + lo.anis;
        h = h + lo.ext;
        h = h + lo.dmi;
      } else if (M.msat.at(i) != 0.0f) {
        const LocalOut lo = local_terms(M, m, x, y, z, i, mc, TERM_EXCH | TERM_DMI | TERM_ANIS | TERM_EXT);
        h = lo.exch;
        h = h + lo.anis;
        h = h + lo.ext;
        h = h + lo.dmi;
      } else if (M.terms & TERM_EXT) {
        h = local_terms(M, m, x, y, z, i, mc, TERM_EXT).ext;
      }
      h = h + bdemag;
      k = G.torque_kind ? damping_torque(mc, h) : llg_torque(mc, h, M.alpha.at(i));
      if (!G.torque_kind && (M.terms & (FLAG_STT_ZL | FLAG_STT_SL))) k = k + stt_torque(M, m, x, y, z, i, mc);
      if (M.terms & FLAG_THERMAL) k = k + thermal_term(M, i, G.steps, G.dt);
    }
    store3(M.buf[G.map[2 + ea.stage]], N, i, k);
    if (ea.fsal_err && ing) {
      float3 e = f3(0, 0, 0);
      for (int j = 0; j < c_tab.S; ++j) {
        const float cf = (float)(G.dt * (c_tab.b1[j] - c_tab.b2[j]));
        const float3 kj = (j == ea.stage) ? k : load3(M.buf[G.map[2 + j]], N, i);
        e = f3(e.x + cf * kj.x, e.y + cf * kj.y, e.z + cf * kj.z);
      }
      err_n = sqrt((double)e.x * e.x + (double)e.y * e.y + (double)e.z * e.z);
      tq_n = sqrt((double)k.x * k.x + (double)k.y * k.y + (double)k.z * k.z);
    }
    return;
  }
  // ---- EPI_EVAL
  const int q = ea.quantity;
  float* out = ea.out;
  const bool scalar = MPX_Q_IS_SCALAR(q);
  if (!ing) {
    if (scalar) {
      out[i] = 0.f;
    } else if (q == 5 && (M.terms & TERM_EXT)) {  // external field outside the geometry: world bias
      store3(out, N, i, f3(M.wb[0], M.wb[1], M.wb[2]));
    } else if (q == 0) {
      store3(out, N, i, mc);
    } else {
      store3(out, N, i, f3(0, 0, 0));
    }
    return;
  }
  const float ms = M.msat.at(i);
  LocalOut lo;
  lo.exch = lo.anis = lo.ext = lo.dmi = f3(0, 0, 0);
  if (M.fast) {
    lo = local_terms_fast(M, m, x, y, z, mc);
  } else if (ms != 0.0f) {
    lo = local_terms(M, m, x, y, z, i, mc, TERM_EXCH | TERM_DMI | TERM_ANIS | TERM_EXT);
  } else if (M.terms & TERM_EXT) {
    lo.ext = local_terms(M, m, x, y, z, i, mc, TERM_EXT).ext;
  }
  float3 h = lo.exch;
  h = h + lo.anis;
  h = h + lo.ext;
  h = h + lo.dmi;
  h = h + bdemag;
  float3 r = f3(0, 0, 0);
  float s = 0.f;
  switch (q) {
    case 0: r = mc; break;
    case 1: r = h; break;
    case 2: r = lo.exch; break;
    case 3: r = lo.dmi; break;
    case 4: r = lo.anis; break;
    case 5: r = lo.ext; break;
    case 6: r = bdemag; break;
    case 7:  // total torque: LLG + spin transfer (physics/torque.cu:78-90)
    case 8:
      if (M.frozen.at(i) == 0.0f) {
        r = llg_torque(mc, h, M.alpha.at(i));
        if (q == 7 && (M.terms & (FLAG_STT_ZL | FLAG_STT_SL))) r = r + stt_torque(M, m, x, y, z, i, mc);
      }
      break;
    case 16:
      if (M.frozen.at(i) == 0.0f && (M.terms & (FLAG_STT_ZL | FLAG_STT_SL))) r = stt_torque(M, m, x, y, z, i, mc);
      break;
    case 9:
      if (M.frozen.at(i) == 0.0f) r = damping_torque(mc, h);
      break;
    case 10: s = (M.terms & TERM_EXCH) ? -0.5f * ms * dot3(mc, lo.exch) : 0.f; break;
    case 11: s = (M.terms & TERM_DMI) ? -0.5f * ms * dot3(mc, lo.dmi) : 0.f; break;
    case 12:
    case 15: {
      float ea_ = 0.f;
      if ((M.terms & TERM_ANIS) && (M.terms & FLAG_CUBIC) && ms != 0.0f) {  // physics/anisotropy.cu:185-215
        const float3 c1 = normalized3(M.anisC1.at(i, N)), c2 = normalized3(M.anisC2.at(i, N));
        ea_ = cubic_energy(mc, c1, c2, cross3(c1, c2), M.kc1.at(i), M.kc2.at(i), M.kc3.at(i));
      } else if ((M.terms & TERM_ANIS) && ms != 0.0f) {  // physics/anisotropy.cu:142-173
        float3 u = M.anisU.at(i, N);
        const float nu = sqrtf(dot3(u, u));
        u = ((nu == 0.0f) ? 0.0f : 1.0f / nu) * u;
        const float mu = dot3(mc, u);
        ea_ -= M.ku1.at(i) * mu * mu;
        ea_ -= M.ku2.at(i) * mu * mu * mu * mu;
      }
      if (q == 12) {
        s = ea_;
      } else {  // total energy density (physics/energy.cu:37-56)
        float t = 0.f;
        if (M.terms & TERM_EXCH) t += -0.5f * ms * dot3(mc, lo.exch);
        if (M.terms & TERM_ANIS) t += ea_;
        if (M.terms & TERM_EXT) t += -1.0f * ms * dot3(mc, lo.ext);
        if (M.terms & TERM_DMI) t += -0.5f * ms * dot3(mc, lo.dmi);
        if (M.terms & TERM_DEMAG) t += -0.5f * ms * dot3(mc, bdemag);
        s = t;
      }
      break;
    }
    case 13: s = (M.terms & TERM_EXT) ? -1.0f * ms * dot3(mc, lo.ext) : 0.f; break;
    case 14: s = (M.terms & TERM_DEMAG) ? -0.5f * ms * dot3(mc, bdemag) : 0.f; break;
    default: break;
  }
  if (scalar) out[i] = s;
  else store3(out, N, i, r);
}

// ------------------------------------------------------- lean stage epilogue
// Neighbour rows of a tile for the lean epilogue: for tile row yl the index of
// x = 0 in the rows y-1, y+1, z-1, z+1 (-1: no neighbour there), and the x
// neighbours of the first and the last cell of a row (nb_coord of each).
struct NbRows {
  int r[TY_MAX][4];
  int xl, xr;
};

__device__ __forceinline__ void nb_rows_fill(NbRows& T, const MagnetDev& M, int y0, int ty, int z) {
  for (int t = threadIdx.x; t < 4 * ty + 2; t += blockDim.x) {
    if (t < 4 * ty) {
      const int yl = t >> 2, q = t & 3, y = y0 + yl;
      int yy = y, zz = z, nc;
      if (q < 2) {
        nc = nb_coord(y, q ? 1 : -1, M.n[1], M.o[1], M.mg[1], M.mgo[1]);
        yy = nc;
      } else {
        nc = nb_coord(z, (q & 1) ? 1 : -1, M.n[2], M.o[2], M.mg[2], M.mgo[2]);
        zz = nc;
      }
      T.r[yl][q] = nc >= 0 ? M.n[0] * (yy + M.n[1] * zz) : -1;
    } else if (t == 4 * ty) {
      T.xl = nb_coord(0, -1, M.n[0], M.o[0], M.mg[0], M.mgo[0]);
    } else {
      T.xr = nb_coord(M.n[0] - 1, 1, M.n[0], M.o[0], M.mg[0], M.mgo[0]);
    }
  }
}

// The lean epilogue applies to magnets on the fast path (uniform parameters,
// no geometry) whose x range lies inside one mastergrid period, so that the
// x neighbours of inner cells are x - 1 and x + 1.
__device__ __forceinline__ bool lean_ok(const MagnetDev& M) {
  const int off = M.o[0] - M.mgo[0];
  return M.fast && !M.geom && (M.mg[0] == 0 || (off >= 0 && off + M.n[0] <= M.mg[0]));
}

// DMI tensor kinds of the lean path: DMI_IFACE when the only nonzero entries
// are D_x^{xz} and D_y^{yz} (interfacial DMI: the x and y neighbours each add
// two products, the z neighbours none), DMI_GENERAL otherwise.  Leaving out
// the products with zero coefficients changes no sum: each of them added an
// exact zero.
constexpr int DMI_IFACE = 1, DMI_GENERAL = 2;
__device__ __forceinline__ int dmi_kind(const MagnetDev& M) {
  const float* f = M.fd;
  return (f[0] == 0.f && f[2] == 0.f && f[3] == 0.f && f[4] == 0.f && f[6] == 0.f && f[7] == 0.f && f[8] == 0.f)
             ? DMI_IFACE
             : DMI_GENERAL;
}

// Contribution of neighbour r (0..5: x-, x+, y-, y+, z-, z+) of a cell with
// state mc to its exchange (he) and DMI (hd) sums on the lean path; `present`:
// the neighbour exists (its state mn), else the Neumann ghost or nothing.
// INNER: every neighbour is present (the ghost-cell code is left out).  DK:
// the DMI tensor kind.
template <bool INNER, int DK = DMI_GENERAL>
__device__ __forceinline__ void neighbour_term(const MagnetDev& M, int r, bool present, float3 mn, float3 mc,
                                               bool neumann, bool dmi_open, bool do_exch, bool do_dmi, float3& he,
                                               float3& hd) {
  const int axis = r >> 1;
  const int d = (r & 1) ? 1 : -1;
  const bool nin = INNER || present;
  float3 m_ = nin ? mn : mc;
  if (!INNER && !nin && neumann) {  // ghost cell m + Gamma/(2A) delta
    const float3 Gm = gamma_uniform(M.fd, axis, mc);
    m_ = mc + (d * M.cs[axis]) * (M.finv_2a * Gm);
  }
  if (do_exch && (nin || neumann)) {  // he += fe (m_ - mc), one rounding per operation as written
    const float fe = M.fe[axis];
    he = f3(__fmaf_rn(fe, __fsub_rn(m_.x, mc.x), he.x), __fmaf_rn(fe, __fsub_rn(m_.y, mc.y), he.y),
            __fmaf_rn(fe, __fsub_rn(m_.z, mc.z), he.z));
  }
  if (do_dmi && (nin || !dmi_open)) {
    const float inv_delta = d * M.inv_cs[axis];
    if constexpr (DK == DMI_IFACE) {  // hd += (D m_) / delta, roundings as written
      if (axis == 0) {
        const float Dxz = M.fd[1];
        hd.x = __fmaf_rn(__fmul_rn(Dxz, m_.z), inv_delta, hd.x);
        hd.z = __fmaf_rn(__fmul_rn(-Dxz, m_.x), inv_delta, hd.z);
      } else if (axis == 1) {
        const float Dyz = M.fd[5];
        hd.y = __fmaf_rn(__fmul_rn(Dyz, m_.z), inv_delta, hd.y);
        hd.z = __fmaf_rn(__fmul_rn(-Dyz, m_.y), inv_delta, hd.z);
      }
    } else {
      const float Dxy = M.fd[3 * axis], Dxz = M.fd[3 * axis + 1], Dyz = M.fd[3 * axis + 2];
      hd.x += (Dxy * m_.y + Dxz * m_.z) * inv_delta;
      hd.y += (-Dxy * m_.x + Dyz * m_.z) * inv_delta;
      hd.z += (-Dxz * m_.x - Dyz * m_.y) * inv_delta;
    }
  }
}

// Exchange and DMI sums over the six neighbours nb[] (-1: none) of the lean
// path, in the order of local_terms_fast.
template <bool INNER, int DK>
__device__ __forceinline__ void neighbour_sums(const MagnetDev& M, const float* __restrict__ m, int N, const int (&nb)[6],
                                               float3 mc, bool neumann, bool dmi_open, bool do_exch, bool do_dmi,
                                               float3& he, float3& hd) {
  float3 mn[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) mn[r] = (INNER || nb[r] >= 0) ? ldg3(m, N, nb[r]) : mc;
#pragma unroll
  for (int r = 0; r < 6; ++r)
    neighbour_term<INNER, DK>(M, r, nb[r] >= 0, mn[r], mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
}

// The rest of a lean-path cell once its exchange / DMI sums are known:
// anisotropy, applied field, demag, the sum in local_terms_fast's order and the
// torque of epilogue_cell.  `ext` is the applied field of the cell.
// LLG torque of the lean path with every rounding spelled out (the packed
// four-cell form below repeats the same operations per component).
__device__ __forceinline__ float llg_coef(float a) { return -GAMMA_LL / __fmaf_rn(a, a, 1.0f); }
__device__ __forceinline__ float3 cross_rn(float3 a, float3 b) {
  return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float3 llg_torque_rn(float3 m, float3 h, float a) {
  const float g = llg_coef(a);
  const float3 mxh = cross_rn(m, h), mxmxh = cross_rn(m, mxh);
  return f3(__fmul_rn(g, __fmaf_rn(a, mxmxh.x, mxh.x)), __fmul_rn(g, __fmaf_rn(a, mxmxh.y, mxh.y)),
            __fmul_rn(g, __fmaf_rn(a, mxmxh.z, mxh.z)));
}

__device__ __forceinline__ float3 finish_cell_lean(const MagnetDev& M, const GroupDev& G, float3 mc, float3 he,
                                                   float3 hd, float3 ext, float3 bdemag) {
  const unsigned terms = M.terms;
  const float s = M.finv_ms;
  float3 exch = f3(0, 0, 0), dmi = f3(0, 0, 0), anis = f3(0, 0, 0);
  if (terms & TERM_EXCH) exch = f3(__fmul_rn(s, he.x), __fmul_rn(s, he.y), __fmul_rn(s, he.z));
  if (terms & TERM_DMI) dmi = f3(__fmul_rn(s, hd.x), __fmul_rn(s, hd.y), __fmul_rn(s, hd.z));
  if ((terms & TERM_ANIS) && (terms & FLAG_CUBIC)) {
    anis = cubic_field(mc, f3(M.fc[0][0], M.fc[0][1], M.fc[0][2]), f3(M.fc[1][0], M.fc[1][1], M.fc[1][2]),
                       f3(M.fc[2][0], M.fc[2][1], M.fc[2][2]), M.fkc[0], M.fkc[1], M.fkc[2], M.finv_ms);
  } else if (terms & TERM_ANIS) {  // (2 K1 mu + 4 K2 mu^3) u / Ms, roundings as written
    const float3 u = f3(M.fu[0], M.fu[1], M.fu[2]);
    const float mu = __fmaf_rn(mc.z, u.z, __fmaf_rn(mc.y, u.y, __fmul_rn(mc.x, u.x)));
    const float c = __fadd_rn(__fmul_rn(2 * M.fk1, mu), __fmul_rn(__fmul_rn(__fmul_rn(4 * M.fk2, mu), mu), mu));
    anis = f3(__fmul_rn(s, __fmul_rn(c, u.x)), __fmul_rn(s, __fmul_rn(c, u.y)), __fmul_rn(s, __fmul_rn(c, u.z)));
  }
  // h = exch + anis + ext + dmi + bdemag, left to right
  const float3 h = f3(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(exch.x, anis.x), ext.x), dmi.x), bdemag.x),
                      __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(exch.y, anis.y), ext.y), dmi.y), bdemag.y),
                      __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(exch.z, anis.z), ext.z), dmi.z), bdemag.z));
  return G.torque_kind ? damping_torque(mc, h) : llg_torque_rn(mc, h, M.alpha.u);
}

// Right-hand side of one cell of a stage on the lean path: the arithmetic of
// local_terms_fast and of the torque in epilogue_cell, in the same order,
// with the neighbours taken from the block's row table.
__device__ __forceinline__ float3 stage_cell_lean(const MagnetDev& M, const GroupDev& G, const NbRows& T,
                                                  const float* __restrict__ m, int i, int x, int yl, int y, int z,
                                                  float3 bdemag) {
  const int N = M.N;
  if (M.frozen.u != 0.0f) return f3(0.f, 0.f, 0.f);
  const unsigned terms = M.terms;
  const float3 mc = ldg3(m, N, i);
  float3 he = f3(0, 0, 0), hd = f3(0, 0, 0);
  const bool openbc = (terms & FLAG_OPENBC) != 0;
  const bool do_exch = (terms & TERM_EXCH) != 0;
  const bool do_dmi = (terms & TERM_DMI) != 0;
  if (do_exch || do_dmi) {
    const float a = M.fa;
    const bool dmi_open = (a == 0.0f) || openbc;
    const bool neumann = !openbc && a != 0.0f;
    const int r0 = i - x;
    int nb[6];
    nb[0] = x > 0 ? i - 1 : (T.xl >= 0 ? r0 + T.xl : -1);
    nb[1] = x < M.n[0] - 1 ? i + 1 : (T.xr >= 0 ? r0 + T.xr : -1);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int b = T.r[yl][q];
      nb[2 + q] = b >= 0 ? b + x : -1;
    }
    const bool inner = nb[0] >= 0 && nb[1] >= 0 && nb[2] >= 0 && nb[3] >= 0 && nb[4] >= 0 && nb[5] >= 0;
    const bool ifc = do_dmi && dmi_kind(M) == DMI_IFACE;
    if (__all_sync(__activemask(), inner)) {  // every neighbour present: no ghost cells
      if (ifc) neighbour_sums<true, DMI_IFACE>(M, m, N, nb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
      else neighbour_sums<true, DMI_GENERAL>(M, m, N, nb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
    } else {
      if (ifc) neighbour_sums<false, DMI_IFACE>(M, m, N, nb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
      else neighbour_sums<false, DMI_GENERAL>(M, m, N, nb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
    }
  }
  float3 ext = f3(0, 0, 0);
  if (terms & TERM_EXT) {
    ext = f3(M.fb[0], M.fb[1], M.fb[2]);
    if (terms & FLAG_STRAY) {
      const float3 s = load3(M.hstray, N, i);
      ext = f3(ext.x + s.x, ext.y + s.y, ext.z + s.z);
    }
  }
  float3 k = finish_cell_lean(M, G, mc, he, hd, ext, bdemag);
  if (!G.torque_kind && (terms & (FLAG_STT_ZL | FLAG_STT_SL))) k = k + stt_torque(M, m, x, y, z, i, mc);
  if (terms & FLAG_THERMAL) k = k + thermal_term(M, i, G.steps, G.dt);
  return k;
}

// Four consecutive cells i0 .. i0 + 3 (i0 a multiple of 4, buffers 16-byte
// aligned) of a SoA field: three 16-byte loads.
__device__ __forceinline__ void ld4x3(const float* __restrict__ a, int N, int i0, float3 (&v)[4]) {
  if (!cell_ok(N, i0) || !cell_ok(N, i0 + 3)) {
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = f3(0.f, 0.f, 0.f);
    return;
  }
  const float4 x = *reinterpret_cast<const float4*>(a + i0);
  const float4 y = *reinterpret_cast<const float4*>(a + N + i0);
  const float4 z = *reinterpret_cast<const float4*>(a + 2 * N + i0);
  v[0] = f3(x.x, y.x, z.x);
  v[1] = f3(x.y, y.y, z.y);
  v[2] = f3(x.z, y.z, z.z);
  v[3] = f3(x.w, y.w, z.w);
}
__device__ __forceinline__ void ldg4x3(const float* __restrict__ a, int N, int i0, float3 (&v)[4]) {
  if (!cell_ok(N, i0) || !cell_ok(N, i0 + 3)) {
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = f3(0.f, 0.f, 0.f);
    return;
  }
  const float4 x = __ldg(reinterpret_cast<const float4*>(a + i0));
  const float4 y = __ldg(reinterpret_cast<const float4*>(a + N + i0));
  const float4 z = __ldg(reinterpret_cast<const float4*>(a + 2 * N + i0));
  v[0] = f3(x.x, y.x, z.x);
  v[1] = f3(x.y, y.y, z.y);
  v[2] = f3(x.z, y.z, z.z);
  v[3] = f3(x.w, y.w, z.w);
}
__device__ __forceinline__ void st4x3(float* a, int N, int i0, const float3 (&v)[4]) {
  if (!cell_ok(N, i0) || !cell_ok(N, i0 + 3)) return;
  *reinterpret_cast<float4*>(a + i0) = make_float4(v[0].x, v[1].x, v[2].x, v[3].x);
  *reinterpret_cast<float4*>(a + N + i0) = make_float4(v[0].y, v[1].y, v[2].y, v[3].y);
  *reinterpret_cast<float4*>(a + 2 * N + i0) = make_float4(v[0].z, v[1].z, v[2].z, v[3].z);
}

// The exchange / DMI sums of four consecutive cells x0 .. x0 + 3 of tile row
// yl: the y and z neighbour rows with 16-byte loads, the x neighbours inside
// the quad from its own values, per cell the terms in the order r = 0 .. 5
// of neighbour_sums (so each cell gets the same arithmetic as there).
template <bool INNER, int DK>
__device__ __forceinline__ void quad_sums(const MagnetDev& M, const float* __restrict__ m, int N, int i0, int x0,
                                          int il, int ir, const int (&rb)[4], const float3 (&mc)[4], bool neumann,
                                          bool dmi_open, bool do_exch, bool do_dmi, float3 (&he)[4],
                                          float3 (&hd)[4]) {
  {  // x-
    const float3 xl = (INNER || il >= 0) ? ldg3(m, N, il) : mc[0];
    neighbour_term<INNER, DK>(M, 0, il >= 0, xl, mc[0], neumann, dmi_open, do_exch, do_dmi, he[0], hd[0]);
#pragma unroll
    for (int q = 1; q < 4; ++q)
      neighbour_term<INNER, DK>(M, 0, true, mc[q - 1], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
  }
  {  // x+
#pragma unroll
    for (int q = 0; q < 3; ++q)
      neighbour_term<INNER, DK>(M, 1, true, mc[q + 1], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
    const float3 xr = (INNER || ir >= 0) ? ldg3(m, N, ir) : mc[3];
    neighbour_term<INNER, DK>(M, 1, ir >= 0, xr, mc[3], neumann, dmi_open, do_exch, do_dmi, he[3], hd[3]);
  }
#pragma unroll
  for (int r = 2; r < 6; ++r) {  // y-, y+, z-, z+: whole neighbour rows
    const int b = rb[r - 2];
    if (INNER || b >= 0) {
      float3 nn[4];
      ldg4x3(m, N, b + x0, nn);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        neighbour_term<INNER, DK>(M, r, true, nn[q], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        neighbour_term<INNER, DK>(M, r, false, mc[q], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
    }
  }
}

// ------------------------------------------------ packed pairs of cells
// The four cells of a quad as the pairs (0, 1) and (2, 3), every component a
// float2 for the packed FP32 pair instructions (pmul, pfma, padd, psub of
// fft.cuh, each rounded as its scalar counterpart).
struct P3 {
  float2 x, y, z;
};
__device__ __forceinline__ float2 bc(float v) { return make_float2(v, v); }
__device__ __forceinline__ P3 pcross(const P3& a, const P3& b) {  // cross_rn per component pair
  return P3{psub(pmul(a.y, b.z), pmul(a.z, b.y)), psub(pmul(a.z, b.x), pmul(a.x, b.z)),
            psub(pmul(a.x, b.y), pmul(a.y, b.x))};
}
__device__ __forceinline__ P3 pick(const float3 (&v)[4], int p) {
  return P3{make_float2(v[2 * p].x, v[2 * p + 1].x), make_float2(v[2 * p].y, v[2 * p + 1].y),
            make_float2(v[2 * p].z, v[2 * p + 1].z)};
}

// stage_quad_lean with interfacial DMI or none, uniaxial anisotropy or none and
// the LLG torque: the x neighbours per cell (as quad_sums, ghost cells
// included), then the y / z neighbour terms, the field and the torque on the two
// cell pairs with packed instructions.  Every operation is the one
// neighbour_term and finish_cell_lean perform, with the same rounding, so a cell
// gets the same bits whichever path its warp takes.  A y / z neighbour row may
// be missing (rb < 0) only where the caller has found that its ghost adds
// nothing (no DMI entries along that axis): it is left out.
template <int DK, typename BD>
__device__ __forceinline__ void stage_quad_packed(const MagnetDev& M, const float* __restrict__ m, int N, int i0,
                                                  int x0, int il, int ir, const int (&rb)[4], const float3 (&mc)[4],
                                                  bool neumann, bool dmi_open, bool do_exch, bool do_dmi, float3 ext,
                                                  BD bdemag, float4& kx, float4& ky, float4& kz) {
  float3 he[4], hd[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) he[q] = hd[q] = f3(0.f, 0.f, 0.f);
  {  // x-, x+ (the x neighbours inside the quad are its own cells)
    const float3 xl = il >= 0 ? ldg3(m, N, il) : mc[0];
    neighbour_term<false, DK>(M, 0, il >= 0, xl, mc[0], neumann, dmi_open, do_exch, do_dmi, he[0], hd[0]);
#pragma unroll
    for (int q = 1; q < 4; ++q)
      neighbour_term<false, DK>(M, 0, true, mc[q - 1], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      neighbour_term<false, DK>(M, 1, true, mc[q + 1], mc[q], neumann, dmi_open, do_exch, do_dmi, he[q], hd[q]);
    const float3 xr = ir >= 0 ? ldg3(m, N, ir) : mc[3];
    neighbour_term<false, DK>(M, 1, ir >= 0, xr, mc[3], neumann, dmi_open, do_exch, do_dmi, he[3], hd[3]);
  }
  P3 MC[2] = {pick(mc, 0), pick(mc, 1)}, HE[2] = {pick(he, 0), pick(he, 1)}, HD[2] = {pick(hd, 0), pick(hd, 1)};
#pragma unroll
  for (int r = 2; r < 6; ++r) {  // y-, y+, z-, z+: whole neighbour rows
    const int axis = r >> 1;
    if (rb[r - 2] < 0) continue;  // missing, and its ghost adds nothing (see the caller)
    float3 nn[4];
    ldg4x3(m, N, rb[r - 2] + x0, nn);
    const float2 fe = bc(M.fe[axis]);
    const float inv_delta = ((r & 1) ? 1.f : -1.f) * M.inv_cs[axis];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const P3 nb = pick(nn, p);
      if (do_exch) {
        HE[p].x = pfma(fe, psub(nb.x, MC[p].x), HE[p].x);
        HE[p].y = pfma(fe, psub(nb.y, MC[p].y), HE[p].y);
        HE[p].z = pfma(fe, psub(nb.z, MC[p].z), HE[p].z);
      }
      if (DK == DMI_IFACE && do_dmi && axis == 1) {
        const float Dyz = M.fd[5];
        HD[p].y = pfma(pmul(bc(Dyz), nb.z), bc(inv_delta), HD[p].y);
        HD[p].z = pfma(pmul(bc(-Dyz), nb.y), bc(inv_delta), HD[p].z);
      }
    }
  }
  const unsigned terms = M.terms;
  const float2 s = bc(M.finv_ms), zero = make_float2(0.f, 0.f);
  const float a = M.alpha.u;
  const float2 g = bc(llg_coef(a)), a2 = bc(a);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    P3 ex = {zero, zero, zero}, dm = ex, an = ex;
    if (terms & TERM_EXCH) ex = P3{pmul(s, HE[p].x), pmul(s, HE[p].y), pmul(s, HE[p].z)};
    if (terms & TERM_DMI) dm = P3{pmul(s, HD[p].x), pmul(s, HD[p].y), pmul(s, HD[p].z)};
    if (terms & TERM_ANIS) {
      const float2 ux = bc(M.fu[0]), uy = bc(M.fu[1]), uz = bc(M.fu[2]);
      const float2 mu = pfma(MC[p].z, uz, pfma(MC[p].y, uy, pmul(MC[p].x, ux)));
      const float2 c = padd(pmul(bc(2 * M.fk1), mu), pmul(pmul(pmul(bc(4 * M.fk2), mu), mu), mu));
      an = P3{pmul(s, pmul(c, ux)), pmul(s, pmul(c, uy)), pmul(s, pmul(c, uz))};
    }
    const float3 b0 = bdemag(2 * p), b1 = bdemag(2 * p + 1);
    const P3 h{padd(padd(padd(padd(ex.x, an.x), bc(ext.x)), dm.x), make_float2(b0.x, b1.x)),
               padd(padd(padd(padd(ex.y, an.y), bc(ext.y)), dm.y), make_float2(b0.y, b1.y)),
               padd(padd(padd(padd(ex.z, an.z), bc(ext.z)), dm.z), make_float2(b0.z, b1.z))};
    const P3 mxh = pcross(MC[p], h), mxmxh = pcross(MC[p], mxh);
    const float2 tx = pmul(g, pfma(a2, mxmxh.x, mxh.x));
    const float2 ty = pmul(g, pfma(a2, mxmxh.y, mxh.y));
    const float2 tz = pmul(g, pfma(a2, mxmxh.z, mxh.z));
    if (p == 0) {
      kx.x = tx.x; kx.y = tx.y; ky.x = ty.x; ky.y = ty.y; kz.x = tz.x; kz.y = tz.y;
    } else {
      kx.z = tx.x; kx.w = tx.y; ky.z = ty.x; ky.w = ty.y; kz.z = tz.x; kz.w = tz.y;
    }
  }
}

// stage_cell_lean for four consecutive cells (no stray field, spin-transfer
// torque or thermal noise on the magnet): the same arithmetic per cell.  The
// demag field of cell q comes from bdemag(q); the torques go to kx / ky / kz
// (component-wise, cell q in lane q of the float4).
template <typename BD>
__device__ __forceinline__ void stage_quad_lean(const MagnetDev& M, const GroupDev& G, const NbRows& T,
                                                const float* __restrict__ m, int i0, int x0, int yl, BD bdemag,
                                                float4& kx, float4& ky, float4& kz) {
  const int N = M.N;
  if (M.frozen.u != 0.0f) {
    kx = ky = kz = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  const unsigned terms = M.terms;
  float3 mc[4];
  ldg4x3(m, N, i0, mc);
  float3 he[4], hd[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) he[q] = hd[q] = f3(0.f, 0.f, 0.f);
  const bool openbc = (terms & FLAG_OPENBC) != 0;
  const bool do_exch = (terms & TERM_EXCH) != 0;
  const bool do_dmi = (terms & TERM_DMI) != 0;
  if (do_exch || do_dmi) {
    const float a = M.fa;
    const bool dmi_open = (a == 0.0f) || openbc;
    const bool neumann = !openbc && a != 0.0f;
    const int r0 = i0 - x0;
    const int il = x0 > 0 ? i0 - 1 : (T.xl >= 0 ? r0 + T.xl : -1);
    const int ir = x0 + 4 < M.n[0] ? i0 + 4 : (T.xr >= 0 ? r0 + T.xr : -1);
    int rb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) rb[q] = T.r[yl][q];
    const bool inner = il >= 0 && ir >= 0 && rb[0] >= 0 && rb[1] >= 0 && rb[2] >= 0 && rb[3] >= 0;
    const bool ifc = do_dmi && dmi_kind(M) == DMI_IFACE;
    if (!(terms & FLAG_CUBIC) && !G.torque_kind && (!do_dmi || ifc)) {
      // a missing y / z neighbour adds exactly nothing when the DMI tensor has no
      // entries along its axis: with open boundaries it is skipped, and the
      // Neumann ghost m + Gamma/(2A) delta is m itself (Gamma = 0)
      const float* f = M.fd;
      const bool y0 = f[3] == 0.f && f[4] == 0.f && f[5] == 0.f;
      const bool z0 = f[6] == 0.f && f[7] == 0.f && f[8] == 0.f;
      const bool qok = (y0 || (rb[0] >= 0 && rb[1] >= 0)) && (z0 || (rb[2] >= 0 && rb[3] >= 0));
      if (__all_sync(__activemask(), qok)) {
        const float3 ext = (terms & TERM_EXT) ? f3(M.fb[0], M.fb[1], M.fb[2]) : f3(0.f, 0.f, 0.f);
        stage_quad_packed<DMI_IFACE>(M, m, N, i0, x0, il, ir, rb, mc, neumann, dmi_open, do_exch, do_dmi, ext,
                                     bdemag, kx, ky, kz);
        return;
      }
    }
    if (__all_sync(__activemask(), inner)) {
      if (ifc) quad_sums<true, DMI_IFACE>(M, m, N, i0, x0, il, ir, rb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
      else quad_sums<true, DMI_GENERAL>(M, m, N, i0, x0, il, ir, rb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
    } else {
      if (ifc) quad_sums<false, DMI_IFACE>(M, m, N, i0, x0, il, ir, rb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
      else quad_sums<false, DMI_GENERAL>(M, m, N, i0, x0, il, ir, rb, mc, neumann, dmi_open, do_exch, do_dmi, he, hd);
    }
  }
  const float3 ext = (terms & TERM_EXT) ? f3(M.fb[0], M.fb[1], M.fb[2]) : f3(0.f, 0.f, 0.f);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float3 k = finish_cell_lean(M, G, mc[q], he[q], hd[q], ext, bdemag(q));
    f4set(kx, q, k.x);
    f4set(ky, q, k.y);
    f4set(kz, q, k.z);
  }
}

// ------------------------------------------------------------------ k_xinv
// PAIR as for k_xfwd.
template <bool PAIR = false>
__global__ void __launch_bounds__(X_THREADS_MAX, 2) k_xinv(const MagnetDev* __restrict__ mags, GroupDev* __restrict__ groups,
                                              const Work* __restrict__ work, EpiArgs ea,
                                              const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  pdl_trigger();  // the next stage's x pass may start its prologue during the last wave
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, ea.gate, ea.stage)) return;
  const int z = wk.z, y0 = wk.y0, ty = wk.ty;
  const int nx = M.n[0], ny = M.n[1], nz = M.n[2];
  const int logL = M.logP[0], L = 1 << logL, cs = xrow_stride(L, ty);
  if (!PAIR && logL == 11) return;  // 2048-point rows only in the PAIR form (the host never launches them here)
  const int nzrows = (ty + 1) >> 1;
  const int Fh = M.Fh;
  float2* rows_z = sm + ty * cs;
  float2* tws = sm + (ty + nzrows) * cs;  // twiddles of length L
  const bool wrow = (PAIR && logL == 11) || logL == 10 || logL == 9;  // 2048- / 1024- / 512-point rows: warp (pair) rows
  const int sh = wrow ? 5 : 4;
  if (wrow) load_twq(tws, tw, logL);
  else load_twiddles<3>(tws, tw, logL);
  __shared__ NbRows T;
  __shared__ float cf[8];  // FSAL error weights dt (b1 - b2) of the stages
  __shared__ int s_quad;   // lean epilogue four cells at a time (16-byte loads and stores)
  const bool lean = ea.mode == EPI_STAGE && lean_ok(M);
  if (lean) {
    nb_rows_fill(T, M, y0, ty, z);
    if (threadIdx.x < c_tab.S) cf[threadIdx.x] = (float)(G.dt * (c_tab.b1[threadIdx.x] - c_tab.b2[threadIdx.x]));
    if (threadIdx.x == 0) {
      // every buffer the epilogue touches 16-byte aligned (N, nx multiples of
      // 4); no per-cell stray field, spin-transfer torque or thermal noise
      uintptr_t a = (uintptr_t)stage_m(M, G, ea.stage) | (uintptr_t)M.buf[G.map[2 + ea.stage]];
      if (ea.fsal_err)
        for (int j = 0; j < c_tab.S; ++j) a |= (uintptr_t)M.buf[G.map[2 + j]];
      s_quad = (a & 15) == 0 && (nx & 3) == 0 && (M.N & 3) == 0 &&
               !(M.terms & (FLAG_STRAY | FLAG_STT_ZL | FLAG_STT_SL | FLAG_THERMAL));
    }
  }
  pdl_wait();  // the spectrum and the stage state are written by the earlier passes
  const float2* __restrict__ S = M.spec;
  const size_t cstride = (size_t)nz * ny;
  // rebuild full-length Hermitian rows: Z = A + iB.  Lanes e (kx = e >> tyl,
  // row yl = e & (2^tyl - 1), rows fastest) each load their x, y and z values;
  // the z value of the odd row comes from the next lane by a shuffle, so every
  // lane issues its three loads together and all lanes run the same trip count.
  const int tyl = tile_log(ty);
  if ((ny & 1) == 0) {
    // even ny: tiles have an even number of rows starting on even rows, and every
    // spectrum offset of a row pair is even, so each lane loads rows 2p, 2p + 1
    // of its kx with 16-byte loads (the same values, half the load instructions)
    const int pl = tyl - 1;
    const int totalp = Fh << pl;
#pragma unroll 2
    for (int e0 = 0; e0 < totalp; e0 += blockDim.x) {
      const int e = e0 + threadIdx.x;
      const int yp = e & ((1 << pl) - 1), kx = e >> pl;
      if (e >= totalp || 2 * yp >= ty) continue;
      const size_t base = (size_t)kx * 3 * cstride + (size_t)z * ny + y0 + 2 * yp;
      if (!span_ok(base + 2 * cstride + 1, (size_t)Fh * 3 * cstride)) continue;
      const float4 a2 = __ldg(reinterpret_cast<const float4*>(S + base));
      const float4 b2 = __ldg(reinterpret_cast<const float4*>(S + base + cstride));
      const float4 c2 = __ldg(reinterpret_cast<const float4*>(S + base + 2 * cstride));
      float2 A0 = make_float2(a2.x, a2.y), A1 = make_float2(a2.z, a2.w);
      float2 B0 = make_float2(b2.x, b2.y), B1 = make_float2(b2.z, b2.w);
      float2 C0 = make_float2(c2.x, c2.y), C1 = make_float2(c2.z, c2.w);
      const bool edge = (kx == 0) || (2 * kx == L);
      if (edge) {
        A0.y = A1.y = B0.y = B1.y = C0.y = C1.y = 0.f;
      }
      const bool mirror = kx > 0 && 2 * kx < L;
      const int y = 2 * yp;
      sm[y * cs + xidx(kx, sh)] = make_float2(A0.x - B0.y, A0.y + B0.x);
      sm[(y + 1) * cs + xidx(kx, sh)] = make_float2(A1.x - B1.y, A1.y + B1.x);
      rows_z[yp * cs + xidx(kx, sh)] = make_float2(C0.x - C1.y, C0.y + C1.x);
      if (mirror) {
        sm[y * cs + xidx(L - kx, sh)] = make_float2(A0.x + B0.y, -A0.y + B0.x);
        sm[(y + 1) * cs + xidx(L - kx, sh)] = make_float2(A1.x + B1.y, -A1.y + B1.x);
        rows_z[yp * cs + xidx(L - kx, sh)] = make_float2(C0.x + C1.y, -C0.y + C1.x);
      }
    }
  } else {
    const int total = Fh << tyl;
#pragma unroll 2
    for (int e0 = 0; e0 < total; e0 += blockDim.x) {
      const int e = e0 + threadIdx.x;
      const int yl = e & ((1 << tyl) - 1), kx = e >> tyl;
      const size_t base = (size_t)kx * 3 * cstride + (size_t)z * ny + y0 + yl;
      const bool act = e < total && yl < ty && span_ok(base + 2 * cstride, (size_t)Fh * 3 * cstride);
      float2 A = make_float2(0.f, 0.f), B = A, Cz = A;
      if (act) {
        A = __ldg(S + base);
        B = __ldg(S + base + cstride);
        Cz = __ldg(S + base + 2 * cstride);
      }
      const float dx = __shfl_down_sync(0xffffffffu, Cz.x, 1), dy = __shfl_down_sync(0xffffffffu, Cz.y, 1);
      if (!act) continue;
      const bool edge = (kx == 0) || (2 * kx == L);
      if (edge) {
        A.y = 0.f;
        B.y = 0.f;
        Cz.y = 0.f;
      }
      sm[yl * cs + xidx(kx, sh)] = make_float2(A.x - B.y, A.y + B.x);
      if (kx > 0 && 2 * kx < L) sm[yl * cs + xidx(L - kx, sh)] = make_float2(A.x + B.y, -A.y + B.x);
      if ((yl & 1) == 0) {
        float2 Dv = (yl + 1 < ty) ? make_float2(dx, dy) : make_float2(0.f, 0.f);
        if (edge) Dv.y = 0.f;
        rows_z[(yl >> 1) * cs + xidx(kx, sh)] = make_float2(Cz.x - Dv.y, Cz.y + Dv.x);
        if (kx > 0 && 2 * kx < L) rows_z[(yl >> 1) * cs + xidx(L - kx, sh)] = make_float2(Cz.x + Dv.y, -Cz.y + Dv.x);
      }
    }
  }
  __syncthreads();
  if (wrow) {  // only x < nx <= L/2 is used
    if (PAIR && logL == 11) pair_rows<1, false, true>(sm, ty + nzrows, cs, tws);
    else if (logL == 10) warp_rows<32, 1, false, true>(sm, ty + nzrows, cs, tws);
    else warp_rows<16, 1, false, true>(sm, ty + nzrows, cs, tws);
    __syncthreads();
  } else {
    fft_many<1, 3, 2>(sm, logL, ty + nzrows, cs, tws);
  }

  const float* m = ea.msrc ? ea.msrc : stage_m(M, G, ea.stage);
  double en = 0.0, tn = 0.0;
  const int rowbase = nx * (y0 + ny * z);
  const float rn = 1.0f / (float)nx;
  if (lean) {
    // squared error / torque norms: the maximum of the squares gives the same
    // maximum norm after one square root per thread
    const int N = M.N;
    float* __restrict__ kout = M.buf[G.map[2 + ea.stage]];
    if (s_quad) {
      const int nq = nx >> 2;
      const float rq = 1.0f / (float)nq;
      for (int e = threadIdx.x; e < ty * nq; e += blockDim.x) {
        const int yl = tile_row(e, nq, rq), x0 = (e - yl * nq) << 2;
        const int i0 = rowbase + yl * nx + x0;
        const float2* __restrict__ hrow = sm + yl * cs;
        const float2* __restrict__ zrow = rows_z + (yl >> 1) * cs;
        const bool odd = yl & 1;
        auto bdemag = [&](int q) {
          const float2 hxy = hrow[xidx(x0 + q, sh)];
          const float2 hz2 = zrow[xidx(x0 + q, sh)];
          return f3(hxy.x, hxy.y, odd ? hz2.y : hz2.x);
        };
        float4 kx, ky, kz;
        stage_quad_lean(M, G, T, m, i0, x0, yl, bdemag, kx, ky, kz);
        if (cell_ok(N, i0) && cell_ok(N, i0 + 3)) {
          *reinterpret_cast<float4*>(kout + i0) = kx;
          *reinterpret_cast<float4*>(kout + N + i0) = ky;
          *reinterpret_cast<float4*>(kout + 2 * N + i0) = kz;
        }
        if (ea.fsal_err) {
          float4 ex = make_float4(0.f, 0.f, 0.f, 0.f), ey = ex, ez = ex;
          for (int j = 0; j < c_tab.S; ++j) {
            const float c = cf[j];
            float4 jx = kx, jy = ky, jz = kz;
            if (j != ea.stage && cell_ok(N, i0) && cell_ok(N, i0 + 3)) {
              const float* __restrict__ kb = M.buf[G.map[2 + j]];
              jx = *reinterpret_cast<const float4*>(kb + i0);
              jy = *reinterpret_cast<const float4*>(kb + N + i0);
              jz = *reinterpret_cast<const float4*>(kb + 2 * N + i0);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              f4set(ex, q, f4c(ex, q) + c * f4c(jx, q));
              f4set(ey, q, f4c(ey, q) + c * f4c(jy, q));
              f4set(ez, q, f4c(ez, q) + c * f4c(jz, q));
            }
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double erx = f4c(ex, q), ery = f4c(ey, q), erz = f4c(ez, q);
            const double es = erx * erx + ery * ery + erz * erz;
            const double kxq = f4c(kx, q), kyq = f4c(ky, q), kzq = f4c(kz, q);
            const double ts = kxq * kxq + kyq * kyq + kzq * kzq;
            en = (es > en || es != es) ? es : en;
            tn = fmax(tn, ts);
          }
        }
      }
      if (ea.fsal_err) block_max2(sqrt(en), sqrt(tn), &groups[M.group].err_bits, &groups[M.group].tmax_bits);
      return;
    }
    for (int e = threadIdx.x; e < ty * nx; e += blockDim.x) {
      const int yl = tile_row(e, nx, rn), x = e - yl * nx;
      const int i = rowbase + e;
      const float2 hxy = sm[yl * cs + xidx(x, sh)];
      const float2 hz2 = rows_z[(yl >> 1) * cs + xidx(x, sh)];
      const float3 bd = f3(hxy.x, hxy.y, (yl & 1) ? hz2.y : hz2.x);
      const float3 k = stage_cell_lean(M, G, T, m, i, x, yl, y0 + yl, z, bd);
      store3(kout, N, i, k);
      if (ea.fsal_err) {
        float3 er = f3(0, 0, 0);
        for (int j = 0; j < c_tab.S; ++j) {
          const float c = cf[j];
          const float3 kj = (j == ea.stage) ? k : load3(M.buf[G.map[2 + j]], N, i);
          er = f3(er.x + c * kj.x, er.y + c * kj.y, er.z + c * kj.z);
        }
        const double es = (double)er.x * er.x + (double)er.y * er.y + (double)er.z * er.z;
        const double ts = (double)k.x * k.x + (double)k.y * k.y + (double)k.z * k.z;
        en = (es > en || es != es) ? es : en;
        tn = fmax(tn, ts);
      }
    }
    if (ea.fsal_err) block_max2(sqrt(en), sqrt(tn), &groups[M.group].err_bits, &groups[M.group].tmax_bits);
    return;
  }
  for (int e = threadIdx.x; e < ty * nx; e += blockDim.x) {
    const int yl = tile_row(e, nx, rn), x = e - yl * nx;
    const int i = rowbase + e;
    float3 bd = f3(0, 0, 0);
    if (in_geom(M, i)) {
      const float2 hxy = sm[yl * cs + xidx(x, sh)];
      const float2 hz2 = rows_z[(yl >> 1) * cs + xidx(x, sh)];
      bd = f3(hxy.x, hxy.y, (yl & 1) ? hz2.y : hz2.x);
    }
    double a = 0.0, b = 0.0;
    epilogue_cell(M, G, ea, m, x, y0 + yl, z, i, bd, a, b);
    en = (a > en || a != a) ? a : en;
    tn = fmax(tn, b);
  }
  if (ea.fsal_err) block_max2(en, tn, &groups[M.group].err_bits, &groups[M.group].tmax_bits);
}

// Local terms only (no demag): same tiles, no dynamic shared memory.
__global__ void __launch_bounds__(256) k_local(const MagnetDev* __restrict__ mags, GroupDev* __restrict__ groups,
                                               const Work* __restrict__ work, EpiArgs ea) {
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, ea.gate, ea.stage)) return;
  const int nx = M.n[0], ny = M.n[1];
  const float* m = ea.msrc ? ea.msrc : stage_m(M, G, ea.stage);
  double en = 0.0, tn = 0.0;
  const int rowbase = nx * (wk.y0 + ny * wk.z);
  const float rn = 1.0f / (float)nx;
  for (int e = threadIdx.x; e < wk.ty * nx; e += blockDim.x) {
    const int yl = tile_row(e, nx, rn), x = e - yl * nx;
    double a = 0.0, b = 0.0;
    epilogue_cell(M, G, ea, m, x, wk.y0 + yl, wk.z, rowbase + e, f3(0, 0, 0), a, b);
    en = (a > en || a != a) ? a : en;
    tn = fmax(tn, b);
  }
  if (ea.fsal_err) block_max2(en, tn, &groups[M.group].err_bits, &groups[M.group].tmax_bits);
}

// Stage combination without a demag pass (writes the stage state xs), or the
// final combination of a non-FSAL method with its error estimate
// (core/rungekutta.cpp:123-151).
__global__ void __launch_bounds__(256) k_combine(const MagnetDev* __restrict__ mags, GroupDev* __restrict__ groups,
                                                 const Work* __restrict__ work, int stage, int final_b1) {
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  const Work wk = work[blockIdx.x];
  if (!load_descs(M, G, mags, groups, wk.mag, 1, 1)) return;
  const int nx = M.n[0], ny = M.n[1], N = M.N;
  float* xs = M.buf[G.map[1]];
  const float* x0 = M.buf[G.map[0]];
  double en = 0.0;
  const int rowbase = nx * (wk.y0 + ny * wk.z);
  for (int e = threadIdx.x; e < wk.ty * nx; e += blockDim.x) {
    const int i = rowbase + e;
    if (!in_geom(M, i)) {
      store3(xs, N, i, load3(x0, N, i));
      continue;
    }
    store3(xs, N, i, combine_cell(M, G, stage, i, final_b1 != 0));
    if (final_b1 && G.adaptive) {
      float3 ev = f3(0, 0, 0);
      for (int j = 0; j < c_tab.S; ++j) {
        const float cf = (float)(G.dt * (c_tab.b1[j] - c_tab.b2[j]));
        const float3 kj = load3(M.buf[G.map[2 + j]], N, i);
        ev = f3(ev.x + cf * kj.x, ev.y + cf * kj.y, ev.z + cf * kj.z);
      }
      const double a = sqrt((double)ev.x * ev.x + (double)ev.y * ev.y + (double)ev.z * ev.z);
      en = (a > en || a != a) ? a : en;
    }
  }
  if (final_b1) block_max2(en, 0.0, &groups[M.group].err_bits, &groups[M.group].tmax_bits);
}

// --------------------------------------------------------------- controller
// core/rungekutta.cpp:60-82 and core/timesolver.cpp:60-111, one thread per group,
// in FP64.  Also runs the run()/steps() state machine on the device.
// Sampled run: time point samp_k has been reached.  Its row (and the rows of
// the next points that need no step, as run(t_k - t) with t_k <= t takes none)
// become due with the time; the next point that needs steps is armed as run()
// arms its end (core/timesolver.cpp:100-109).  Returns false when no point is
// left.
__device__ __forceinline__ bool sample_advance(GroupDev& G) {
  G.samp_lo = G.samp_k;
  do {
    G.samp_out[(size_t)G.samp_k * G.samp_row] = G.t;
    ++G.samp_k;
  } while (G.samp_k < G.samp_n && !(G.samp_t[G.samp_k] - G.t > 0.0));
  G.samp_hi = G.samp_k;
  if (G.samp_k >= G.samp_n) return false;
  G.phase = 0;
  G.t_stop = G.t + (G.samp_t[G.samp_k] - G.t);
  if (!(G.t < G.t_stop - G.dt)) {
    G.phase = 1;
    G.dt_saved = G.dt;
    G.dt = G.t_stop - G.t;
  }
  return true;
}

__global__ void k_controller(GroupDev* __restrict__ groups, int ngroups) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  GroupDev& G = groups[g];
  if (G.status != GS_RUNNING) return;
  G.samp_lo = G.samp_hi;  // the rows of the previous attempt have been written
  const double err = __longlong_as_double((long long)G.err_bits);
  const double tmax = __longlong_as_double((long long)G.tmax_bits);
  G.err_bits = 0ull;
  G.tmax_bits = 0ull;
  G.attempts++;
  const double dt = G.dt;
  bool success = true;
  if (G.adaptive) {
    success = err < G.max_error;
    double corr = success ? pow(G.max_error / err, 1.0 / (c_tab.order2 + 1))
                          : pow(G.max_error / err, 1.0 / (c_tab.order1 + 1));
    if (isnan(corr)) corr = 1.0;
    corr *= G.headroom;
    corr = corr > G.upper ? G.upper : corr;
    corr = corr < G.lower ? G.lower : corr;
    G.dt = dt * corr;
    if (isnan(err)) {  // the reference would retry forever; fail the solve instead
      G.status = GS_FAILED;
      G.finished_flag = 1;
      return;
    }
  }
  if (!success) {
    G.rejected++;
    G.k0_valid = G.thermal ? 0 : 1;  // with noise k0 depends on dt (noise / sqrt(dt))
    return;
  }
  // accept: t = t0 + dt; x0 <- x_new; FSAL: k0 <- k_{S-1}
  G.t += dt;
  G.steps++;
  const int t0 = G.map[0];
  G.map[0] = G.map[1];
  G.map[1] = t0;
  if (c_tab.fsal) {
    const int k0 = G.map[2];
    G.map[2] = G.map[2 + c_tab.S - 1];
    G.map[2 + c_tab.S - 1] = k0;
    G.k0_valid = G.thermal ? 0 : 1;  // a new step draws new noise
  } else {
    G.k0_valid = 0;
  }
  bool done = false;
  if (G.phase == 1) {
    done = true;
    if (!G.adaptive) G.dt = G.dt_saved;
    if (G.mode == 2) done = !sample_advance(G);
  } else if (G.mode == 1) {
    if (--G.steps_left <= 0) done = true;
  } else {
    if (G.torque_stop > 0.0 && c_tab.fsal && tmax / (double)GAMMA_LL < G.torque_stop) {
      done = true;
    } else if (!(G.t < G.t_stop - G.dt)) {
      G.phase = 1;
      G.dt_saved = G.dt;
      G.dt = G.t_stop - G.t;
    }
  }
  if (done) {
    G.status = GS_FINISHED;
    G.finished_flag = 1;
    G.phase = 0;
  }
}

// ---------------------------------------------------------------- reductions
// Deterministic two-level reductions over the geometry: block partials in a
// fixed order, then one block.  op 0: per-component sum, op 1: max |v|.
__global__ void k_reduce_partial(const float* __restrict__ a, int N, int ncomp,
                                 const unsigned char* __restrict__ geom, int op, double* partial) {
  __shared__ double sh[3][256];
  double acc[3] = {0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    if (geom && !geom[i]) continue;
    if (op == 0) {
      for (int c = 0; c < ncomp; ++c) acc[c] += (double)a[(size_t)c * N + i];
    } else if (op == 2) {  // sum of squared norms (dotSum(a, a), core/reduce.cu)
      for (int c = 0; c < ncomp; ++c) {
        const double v = a[(size_t)c * N + i];
        acc[0] += v * v;
      }
    } else {
      double s = 0;
      for (int c = 0; c < ncomp; ++c) {
        const double v = a[(size_t)c * N + i];
        s += v * v;
      }
      s = sqrt(s);
      acc[0] = (s > acc[0] || s != s) ? s : acc[0];
    }
  }
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int c = 0; c < 3; ++c) {
        if (op != 1) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
        else {
          const double o = sh[c][threadIdx.x + s];
          if (o > sh[c][threadIdx.x] || o != o) sh[c][threadIdx.x] = o;
        }
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partial[blockIdx.x * 3 + c] = sh[c][0];
}

__global__ void k_reduce_final(const double* __restrict__ partial, int nblocks, int op, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double r[3] = {0, 0, 0};
  for (int b = 0; b < nblocks; ++b)
    for (int c = 0; c < 3; ++c) {
      const double v = partial[b * 3 + c];
      if (op != 1) r[c] += v;
      else if (v > r[c] || v != v) r[c] = v;
    }
  for (int c = 0; c < 3; ++c) out[c] = r[c];
}

// Sampled run: <m> of one magnet into the due rows of its group's table, with
// the arithmetic of mpx_average (k_reduce_partial / k_reduce_final over the
// same 256 x 256 grid), so the values equal a host-side average of the state.
// Both kernels do nothing unless rows are due.
__global__ void __launch_bounds__(256) k_sample_partial(const MagnetDev* __restrict__ mags,
                                                        const GroupDev* __restrict__ groups, int slot,
                                                        double* partial) {
  __shared__ double sh[3][256];
  const MagnetDev& M = mags[slot];
  const GroupDev& G = groups[M.group];
  if (G.samp_hi <= G.samp_lo) return;
  const int N = M.N;
  const float* __restrict__ a = M.buf[G.map[0]];
  const unsigned char* __restrict__ geom = M.geom;
  double acc[3] = {0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    if (geom && !geom[i]) continue;
    for (int c = 0; c < 3; ++c) acc[c] += (double)a[(size_t)c * N + i];
  }
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partial[blockIdx.x * 3 + c] = sh[c][0];
}

__global__ void k_sample_final(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, int slot,
                               const double* __restrict__ partial, int nblocks, long long ngeo, int col) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const GroupDev& G = groups[mags[slot].group];
  if (G.samp_hi <= G.samp_lo) return;
  double r[3] = {0, 0, 0};
  for (int b = 0; b < nblocks; ++b)
    for (int c = 0; c < 3; ++c) r[c] += partial[b * 3 + c];
  for (int row = G.samp_lo; row < G.samp_hi; ++row)
    for (int c = 0; c < 3; ++c) G.samp_out[(size_t)row * G.samp_row + col + c] = ngeo > 0 ? r[c] / ngeo : 0.0;
}

// Set m: normalise per cell inside the geometry (core/variable.cpp:76-87).
__global__ void k_normalize_into(float* dst, const float* __restrict__ src, int N,
                                 const unsigned char* __restrict__ geom) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float x = src[i], y = src[N + i], z = src[2 * N + i];
  if (!geom || geom[i]) {
    const float inv = rsqrtf(x * x + y * y + z * z);
    x *= inv;
    y *= inv;
    z *= inv;
  }
  dst[i] = x;
  dst[N + i] = y;
  dst[2 * N + i] = z;
}

// n normal(0,1) numbers for the initial magnetisation of a new magnet: the
// splitmix64 finaliser of (seed, index) (Steele, Lea and Flood, OOPSLA 2014)
// gives two 24-bit uniforms, turned into one normal by Box-Muller.
__global__ void k_random_normal(float* __restrict__ out, int n, unsigned long long seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const float u1 = (float)((unsigned)(z >> 40) + 1u) * (1.0f / 16777216.0f);  // (0, 1]
    const float u2 = (float)(unsigned)(z & 0xFFFFFFull) * (1.0f / 16777216.0f);  // [0, 1)
    out[i] = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
  }
}

// ------------------------------------------------------------- minimizer
// One steepest-descent step of physics/minimizer.cu (k_step): from the state m0
// and its damping torque t0, m1 = ((4 - dt^2 t0^2) m0 + 4 dt t0) / (4 + dt^2 t0^2)
// over every cell of the grid; m0 and the unnormalised m1 are kept for the
// Barzilai-Borwein step size, the state becomes m1 normalised inside the
// geometry (the reference's magnetization()->set(m1)).
__global__ void k_min_step(float* __restrict__ state, float* __restrict__ m0_out, float* __restrict__ m1_out,
                           const float* __restrict__ t0, int N, float dt, const unsigned char* __restrict__ geom) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float3 m0 = load3(state, N, i), t = load3(t0, N, i);
    const float t2 = dt * dt * dot3(t, t);
    const float inv = 1.0f / (4.0f + t2);
    const float3 m1 = f3(((4.0f - t2) * m0.x + 4.0f * dt * t.x) * inv, ((4.0f - t2) * m0.y + 4.0f * dt * t.y) * inv,
                         ((4.0f - t2) * m0.z + 4.0f * dt * t.z) * inv);
    store3(m0_out, N, i, m0);
    store3(m1_out, N, i, m1);
    float3 n = m1;
    if (!geom || geom[i]) {
      const float r = rsqrtf(dot3(m1, m1));
      n = f3(m1.x * r, m1.y * r, m1.z * r);
    }
    store3(state, N, i, n);
  }
}

// Block partials (FP64) of dm.dm, dm.dt, dt.dt and max|dm| with dm = m1 - m0 and
// dt = t0 - t1 (physics/minimizer.cu: BarzilianBorweinStepSize, maxVecNorm(dm)).
__global__ void k_min_partial(const float* __restrict__ m0, const float* __restrict__ m1, const float* __restrict__ t0,
                              const float* __restrict__ t1, int N, double* __restrict__ partial) {
  __shared__ double sh[4][256];
  double a = 0, b = 0, c = 0, mx = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float3 p = load3(m0, N, i), q = load3(m1, N, i), u = load3(t0, N, i), v = load3(t1, N, i);
    const float3 dm = f3(q.x - p.x, q.y - p.y, q.z - p.z);
    const float3 dt = f3(u.x - v.x, u.y - v.y, u.z - v.z);
    const double mm = (double)dm.x * dm.x + (double)dm.y * dm.y + (double)dm.z * dm.z;
    a += mm;
    b += (double)dm.x * dt.x + (double)dm.y * dt.y + (double)dm.z * dt.z;
    c += (double)dt.x * dt.x + (double)dt.y * dt.y + (double)dt.z * dt.z;
    const double n = sqrt(mm);
    mx = (n > mx || n != n) ? n : mx;
  }
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b;
  sh[2][threadIdx.x] = c;
  sh[3][threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
      const double o = sh[3][threadIdx.x + s];
      if (o > sh[3][threadIdx.x] || o != o) sh[3][threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) partial[blockIdx.x * 4 + k] = sh[k][0];
}

__global__ void k_min_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double r[4] = {0, 0, 0, 0};
  for (int b = 0; b < nblocks; ++b) {
    for (int k = 0; k < 3; ++k) r[k] += partial[b * 4 + k];
    const double v = partial[b * 4 + 3];
    if (v > r[3] || v != v) r[3] = v;
  }
  for (int k = 0; k < 4; ++k) out[k] = r[k];
}

}  // namespace mpx
