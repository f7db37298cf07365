// dft_tc.cuh -- the y transforms of the demag convolution as TF32 tensor-core
// GEMMs (tcgen05, sm_100a) with 3xTF32 split products, accumulated in FP32.
//
// Replaces the cuFFT y stages of physics/strayfieldfft.cu:216-218 (forward)
// and :238-240 (inverse) for y lengths Py = 1024 R (R = 1 or 2), in the split
// y/z path (yzsplit.cuh): k_ydft_tc<-1> takes the ny rows of spectrum columns
// S[kx][c][z][y] to all Py rows of T[kx][c][z][ky]; k_zmul does the z
// transform and the Newell multiply; k_ydft_tc<+1> takes T back to the ny rows
// of S.  Unnormalised transforms (the -mu0/P factor is in the kernel spectrum).
//
// Arithmetic.  The 1024-point transform is four-step 32 x 32: with
// n = n1 + 32 n2 and k = k2 + 32 k1,
//   X[k2 + 32 k1] = sum_n1 W32^{n1 k1} [ W1024^{n1 k2} sum_n2 W32^{n2 k2} x[n1 + 32 n2] ].
// Each 32-point DFT is a real GEMM D = A B^T on the interleaved
// (re, im) representation: A rows are sequences (K = 2 x 32 inputs), B is
// the fixed 64 x 64 real form of the forward DFT32 matrix.  Every product is
// split: a = a_hi + a_lo with a_hi = tf32(a), a_lo = tf32(a - a_hi), and
// D = A_hi B_hi + A_lo B_hi + A_hi B_lo, so the result carries about 21
// significant bits like the FP32 FFT.  R = 2 adds one radix-2 step in FP32
// (decimation in time forward, in frequency inverse).  The inverse transform
// is conj(forward(conj(.))).  Pruning: the forward first stage reads only
// n2 < 16 (y < Py/2: the rest is zero padding), the inverse second stage
// writes only the outputs y < Py/2.
//
// Layout.  One tile = 128 sequences = 4 / R columns; one thread per sequence
// row (128 threads, warp w owns TMEM lanes 32w .. 32w + 31).  Operands in
// shared memory in the K-major no-swizzle canonical layout: 8-row x 16-byte
// core matrices, rows of a group 16 B apart, 8-row groups 128 B apart (SBO),
// 16-byte K chunks LBO apart (padded by 16 B so that the transposing stores
// of the first stage's epilogue spread over the banks).  Accumulators in TMEM
// (64 columns per stage).  One elected thread issues the MMAs and commits
// them to an mbarrier; every wait is bounded and reports a timeout in a
// device word instead of hanging.
#pragma once
#include "kernels.cuh"

namespace mpx {

__device__ unsigned int g_tc_timeouts = 0;  // mbarrier waits that gave up (read by mpx_tc_status)

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of sm_100 (no swizzle): start address,
// leading (K) byte offset, stride (8-row group) byte offset, version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32: D f32, A and B tf32, both K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void commit(void* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(void* mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(mbar)), "r"(1));
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Waits for the phase `parity` of the mbarrier to complete, at most `limit`
// polls (about 64 ns apart); false when it gave up.
__device__ __forceinline__ bool mbar_wait(void* mbar, uint32_t parity, int limit) {
  const uint32_t a = smem_u32(mbar);
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 16 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// a = hi + lo, both TF32 (round to nearest, ties away): hi carries the top
// 11 significant bits, lo the next 11
__device__ __forceinline__ void split_tf32(float a, float& hi, float& lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(a));
  hi = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(l) : "f"(a - hi));
  lo = __uint_as_float(l);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

}  // namespace tc

// Shared-memory plan of k_ydft_tc (bytes).  B: the 64 x 64 DFT32 real form,
// hi and lo (K-major, LBO 1024).  A: the operand of one stage, hi and lo, 128
// rows x 64 K (16 chunks, LBO padded to 2064).  Twiddles: W1024^{ab} as
// [b][a] (1024), and for R = 2 the factors of W2048^(c + 32 d) =
// W2048^c W64^d (32 + 32).  107,840 bytes: two blocks per SM.
constexpr int TC_ROWS = 128;
constexpr int TC_B_BYTES = 64 * 64 * 4;                 // one of hi / lo
constexpr int TC_B_LBO = 8 * 128;                       // 64 rows / 8 x 128 B
constexpr int TC_A_LBO = (TC_ROWS / 8) * 128 + 16;      // 2064
constexpr int TC_A_BYTES = 16 * TC_A_LBO;               // 64 K = 16 chunks (33,024 B)
constexpr int TC_SMEM = 2 * TC_B_BYTES + 2 * TC_A_BYTES + (1024 + 64) * 8 + 64;
constexpr int TC_TMEM_COLS = 128;
constexpr int TC_BLOCKS_PER_SM = 2;

// Byte offset of element (row, k) in a K-major no-swizzle tile with LBO `lbo`.
__host__ __device__ constexpr int tc_off(int row, int k, int lbo) {
  return (k >> 2) * lbo + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

// One stage: D (64 TMEM columns at d) = A (K = 2 kin) x B^T restricted to the
// first n_out rows of B (N = n_out) and its first 2 kin K columns, 3 products
// per 8-wide K step.  Issued by one thread.
__device__ __forceinline__ void tc_stage(uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo,
                                         int ksteps, int n_out) {
  const uint32_t id = tc::idesc_tf32(128, n_out);
  for (int s = 0; s < ksteps; ++s) {
    const uint64_t ah = tc::sdesc(a_hi + s * 2 * TC_A_LBO, TC_A_LBO, 128);
    const uint64_t al = tc::sdesc(a_lo + s * 2 * TC_A_LBO, TC_A_LBO, 128);
    const uint64_t bh = tc::sdesc(b_hi + s * 2 * TC_B_LBO, TC_B_LBO, 128);
    const uint64_t bl = tc::sdesc(b_lo + s * 2 * TC_B_LBO, TC_B_LBO, 128);
    tc::mma(d, ah, bh, id, s > 0);
    tc::mma(d, al, bh, id, 1);
    tc::mma(d, ah, bl, id, 1);
  }
}

// Work item: magnet, first column (kx*3 + c)*nz + z in z, number of columns
// (<= 4 / R) in y0.  DIR -1: S -> T (forward), +1: T -> S (inverse).
// dftB: the DFT32 real form, hi then lo, each 64 x 64 floats row-major [n][k].
// Grid: persistent, blocks loop over the work items.
template <int DIR>
__global__ void __launch_bounds__(128, TC_BLOCKS_PER_SM)
    k_ydft_tc(const MagnetDev* __restrict__ mags, const GroupDev* __restrict__ groups, const Work* __restrict__ work,
              int nwork, int stage, int gate, const float* __restrict__ dftB) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* sBh = tsm;
  unsigned char* sBl = sBh + TC_B_BYTES;
  unsigned char* sAh = sBl + TC_B_BYTES;
  unsigned char* sAl = sAh + TC_A_BYTES;
  float2* tw1 = reinterpret_cast<float2*>(sAl + TC_A_BYTES);  // W1024^{ab} at [b * 32 + a]
  float2* twc = tw1 + 1024;                                    // W2048^c, c < 32
  float2* twd = twc + 32;                                      // W64^d, d < 32
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(twd + 32);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(mbar + 1);
  __shared__ MagnetDev M;
  __shared__ GroupDev G;
  const int tid = threadIdx.x, warp = tid >> 5;

  // B (hi, lo) into the K-major core layout; twiddle tables
  for (int e = tid; e < 64 * 64; e += 128) {
    const int n = e >> 6, k = e & 63;
    *reinterpret_cast<float*>(sBh + tc_off(n, k, TC_B_LBO)) = __ldg(dftB + e);
    *reinterpret_cast<float*>(sBl + tc_off(n, k, TC_B_LBO)) = __ldg(dftB + 4096 + e);
  }
  for (int e = tid; e < 1024; e += 128) {
    const int b = e >> 5, a = e & 31;
    double sd, cd;
    sincospi(-2.0 * (double)(a * b) / 1024.0, &sd, &cd);
    tw1[e] = make_float2((float)cd, (float)sd);
  }
  if (tid < 64) {
    double sd, cd;
    sincospi(tid < 32 ? -2.0 * tid / 2048.0 : -2.0 * (tid - 32) / 64.0, &sd, &cd);
    twc[tid] = make_float2((float)cd, (float)sd);  // twd follows twc
  }
  if (tid == 0) tc::mbar_init(mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::smem_u32(tbase)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = *tbase;
  const uint32_t d1 = tm, d2 = tm + 64;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  const uint32_t aBh = tc::smem_u32(sBh), aBl = tc::smem_u32(sBl), aAh = tc::smem_u32(sAh), aAl = tc::smem_u32(sAl);
  uint32_t phase = 0;
  bool ok = true;

  for (int wi = blockIdx.x; wi < nwork && ok; wi += gridDim.x) {
    const Work wk = work[wi];
    __syncthreads();  // the previous item's descriptors are no longer read
    if (!load_descs(M, G, mags, groups, wk.mag, gate, stage)) continue;
    const int Py = M.P[1], ny = M.n[1];
    const int R = Py >> 10;            // 1 or 2
    const int spc = 32 * R;            // sequences per column
    const int ncol = wk.y0;
    const int row = tid;
    const int cl = row / spc;          // column of this row within the tile
    const int q = row - cl * spc;      // q = a * R + p
    const int a = q / R, p = q - a * R;
    const bool live = cl < ncol;
    const int col = wk.z + cl;
    float2* __restrict__ T = M.tspec + (size_t)col * Py;
    float2* __restrict__ S = M.spec + (size_t)col * ny;
    // elements of S and T from this column on (index checks of the checked build)
    const size_t ncols_all = (size_t)M.Fh * 3 * M.n[2];
    const size_t sleft = live ? (ncols_all - col) * ny : 0, tleft = live ? (ncols_all - col) * Py : 0;

    // ---- stage 1 operand: 32 (inverse) or 16 (forward, pruned) inputs per row
    if (DIR < 0) {
      // x_p[a + 32 b] = x[R (a + 32 b) + p], b < 16; zero beyond ny
#pragma unroll 4
      for (int j = 0; j < 8; ++j) {  // K chunk j: inputs b = 2j, 2j+1
        float v[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int y = R * (a + 32 * (2 * j + h)) + p;
          const float2 x = (live && y < ny && span_ok(y, sleft)) ? __ldg(S + y) : make_float2(0.f, 0.f);
          v[2 * h] = x.x;
          v[2 * h + 1] = x.y;
        }
        float4 hi, lo;
        tc::split_tf32(v[0], hi.x, lo.x);
        tc::split_tf32(v[1], hi.y, lo.y);
        tc::split_tf32(v[2], hi.z, lo.z);
        tc::split_tf32(v[3], hi.w, lo.w);
        *reinterpret_cast<float4*>(sAh + tc_off(row, 4 * j, TC_A_LBO)) = hi;
        *reinterpret_cast<float4*>(sAl + tc_off(row, 4 * j, TC_A_LBO)) = lo;
      }
    } else {
      // inverse: with Y = conj(T), z[k] = Y[k] + Y[k+1024] (p = 0) or
      // (Y[k] - Y[k+1024]) W2048^k (p = 1) for R = 2, Y[k] for R = 1, at
      // k = a + 32 b, b < 32
      const float2 wa = twc[a];  // W2048^(a + 32 b) = W2048^a W64^b
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        // the 32 loads of 16 inputs (both halves of the transform) issued together
        float2 t0[16], t1[16];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const int k = a + 32 * (16 * half + jj);
          const bool ok = live && span_ok(k + (size_t)(R - 1) * 1024, tleft);
          t0[jj] = ok ? __ldg(T + k) : make_float2(0.f, 0.f);
          t1[jj] = (ok && R == 2) ? __ldg(T + k + 1024) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j8 = 0; j8 < 8; ++j8) {
        const int j = 8 * half + j8;
        float v[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int jj = 2 * j8 + h;
          const float2 y0 = make_float2(t0[jj].x, -t0[jj].y);
          float2 z;
          if (R == 1) {
            z = y0;
          } else if (p == 0) {
            z = make_float2(y0.x + t1[jj].x, y0.y - t1[jj].y);
          } else {
            const float2 d = make_float2(y0.x - t1[jj].x, y0.y + t1[jj].y);
            z = tc::cmul(d, tc::cmul(wa, twd[2 * j + h]));
          }
          v[2 * h] = z.x;
          v[2 * h + 1] = z.y;
        }
        float4 hi, lo;
        tc::split_tf32(v[0], hi.x, lo.x);
        tc::split_tf32(v[1], hi.y, lo.y);
        tc::split_tf32(v[2], hi.z, lo.z);
        tc::split_tf32(v[3], hi.w, lo.w);
        *reinterpret_cast<float4*>(sAh + tc_off(row, 4 * j, TC_A_LBO)) = hi;
        *reinterpret_cast<float4*>(sAl + tc_off(row, 4 * j, TC_A_LBO)) = lo;
        }
      }
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    // ---- stage 1: D1 = A1 B^T (forward: K = 32 pruned inputs; inverse: 64)
    if (tid == 0) {
      tc::fence_after();
      tc_stage(d1, aAh, aAl, aBh, aBl, DIR < 0 ? 4 : 8, 64);
      tc::commit(mbar);
    }
    if (__syncthreads_or(!tc::mbar_wait(mbar, phase, 1 << 22))) {  // the same decision in every thread
      ok = false;
      break;
    }
    phase ^= 1;
    tc::fence_after();
    // ---- twiddle W1024^{a c}, stage 2 operand: row (cl, c, p), K = 2 a + ri
    {
      float v[64];
#pragma unroll
      for (int c16 = 0; c16 < 4; ++c16) tc::tmem_ld16(d1 + lane_base + 16 * c16, v + 16 * c16);
      tc::tmem_wait_ld();
      tc::fence_before();
      __syncthreads();  // every row of A1 was read by the MMA; A2 overwrites it
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const float2 w = tw1[c * 32 + a];
        const float xr = v[2 * c], xi = v[2 * c + 1];
        const float yr = xr * w.x - xi * w.y, yi = xr * w.y + xi * w.x;
        float hr, lr, hi_, li;
        tc::split_tf32(yr, hr, lr);
        tc::split_tf32(yi, hi_, li);
        const int r2 = cl * spc + c * R + p;
        *reinterpret_cast<float2*>(sAh + tc_off(r2, 2 * a, TC_A_LBO)) = make_float2(hr, hi_);
        *reinterpret_cast<float2*>(sAl + tc_off(r2, 2 * a, TC_A_LBO)) = make_float2(lr, li);
      }
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    // ---- stage 2: D2 = A2 B^T (K = 64; inverse: only the 16 outputs y < Py/2)
    if (tid == 0) {
      tc::fence_after();
      tc_stage(d2, aAh, aAl, aBh, aBl, 8, DIR < 0 ? 64 : 32);
      tc::commit(mbar);
    }
    if (__syncthreads_or(!tc::mbar_wait(mbar, phase, 1 << 22))) {
      ok = false;
      break;
    }
    phase ^= 1;
    tc::fence_after();
    // ---- epilogue: this thread holds row (cl, c, p) of D2 (c = a here)
    const int c = a;
    if (DIR < 0) {
      // X_p[c + 32 d], d < 32; R = 2: X[k] = E + W2048^k O, X[k + 1024] = E - W2048^k O
#pragma unroll
      for (int c16 = 0; c16 < 4; ++c16) {
        float v[16];
        tc::tmem_ld16(d2 + lane_base + 16 * c16, v);
        tc::tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int dd = 8 * c16 + h;
          const int k = c + 32 * dd;
          float2 x = make_float2(v[2 * h], v[2 * h + 1]);
          if (R == 2) {
            if (p == 1) x = tc::cmul(x, tc::cmul(twc[c], twd[dd]));  // W2048^(c + 32 dd)
            const float ox = __shfl_xor_sync(0xffffffffu, x.x, 1);
            const float oy = __shfl_xor_sync(0xffffffffu, x.y, 1);
            x = p == 0 ? make_float2(x.x + ox, x.y + oy) : make_float2(ox - x.x, oy - x.y);
          }
          if (live && span_ok(k + (size_t)1024 * p, tleft)) T[k + 1024 * p] = x;
        }
      }
    } else {
      // x[R (c + 32 d) + p] = conj(D2), d < 16, kept where y < ny
#pragma unroll
      for (int c16 = 0; c16 < 2; ++c16) {
        float v[16];
        tc::tmem_ld16(d2 + lane_base + 16 * c16, v);
        tc::tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int y = R * (c + 32 * (8 * c16 + h)) + p;
          if (live && y < ny && span_ok(y, sleft)) S[y] = make_float2(v[2 * h], -v[2 * h + 1]);
        }
      }
    }
    tc::fence_before();
  }
  if (!ok) {
    // a wait gave up: report it, and give the MMAs in flight a second bounded
    // wait before the tensor memory they write is released
    if (tid == 0) atomicAdd(&g_tc_timeouts, 1u);
    tc::mbar_wait(mbar, phase, 1 << 22);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tm), "r"(TC_TMEM_COLS));
}

// The timeout path of the tensor-core kernels, without a fault: one block
// takes tensor memory and an mbarrier as k_ydft_tc does, but nothing arrives
// on the barrier, so its bounded wait (`polls` polls) runs out.  The block then
// counts the timeout, waits once more (bounded), releases its tensor memory and
// returns; the context stays usable.
__global__ void __launch_bounds__(128, 1) k_tc_timeout_probe(int polls) {
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) tc::mbar_init(&mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::smem_u32(&tbase)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = tbase;
  const bool gave_up = __syncthreads_or(!tc::mbar_wait(&mbar, 0, polls));
  if (gave_up) {
    if (tid == 0) atomicAdd(&g_tc_timeouts, 1u);
    tc::mbar_wait(&mbar, 0, polls);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tm), "r"(TC_TMEM_COLS));
}

}  // namespace mpx
