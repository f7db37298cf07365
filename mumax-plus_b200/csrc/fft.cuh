// fft.cuh -- shared-memory FFTs for the demag convolution (sm_100a, FP32).
//
// Power-of-two complex FFTs run in place in shared memory as Stockham
// autosort passes of radix 2/4/8/16 (natural-order output, no bit reversal):
// pass with sub-transform size Ns and radix R takes butterfly j of a column,
// loads x[j + r*L/R], twiddles by W_{Ns R}^{r (j mod Ns)}, does an R-point DFT
// in registers and stores to ((j - j mod Ns) R + j mod Ns) + r Ns.
// Every thread holds 16 complex values per pass, so one call transforms at
// most 16*blockDim.x elements; callers loop over groups of columns.
//
// Shared-memory layout: element i of a column sits at pidx(i) = i + i/16 (one
// float2 of padding per 16), which makes the strided stores of the first
// passes (stride R) bank-conflict free.  All index arithmetic is shifts and
// masks (lengths are powers of two).
//
// Twiddles come from a 4096-entry table exp(-2 pi i k / 4096) computed in FP64
// on the host (accurate to FP32 rounding); each block copies the L entries of
// its transform length into shared memory once.
#pragma once
#include <cuda_runtime.h>

namespace mpx {

constexpr int TW_LOG = 12;  // twiddle table covers transforms up to 4096 points
constexpr int TW_N = 1 << TW_LOG;

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// Packed FP32 pair arithmetic (add/sub.rn.f32x2 of sm_100): one instruction for
// both components, each rounded like the scalar add/sub.  Used in the
// butterflies whose twiddle is 1 or a general rotation; a quarter turn swaps and
// negates components, which the scalar adds absorb for free.
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mul.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// a * b + c per component with one rounding (as __fmaf_rn)
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}
// Butterfly e +- t where t = o rotated by exp(DIR 2 pi i M / P) (M < P/2):
// packed unless the rotation is a quarter turn.
template <int M, int P>
__device__ __forceinline__ void bfly(float2 e, float2 t, float2& lo, float2& hi) {
  if constexpr (M != 0 && 4 * M == P) {
    lo = cadd(e, t);
    hi = csub(e, t);
  } else {
    lo = padd(e, t);
    hi = psub(e, t);
  }
}

// padded shared-memory index and padded column length
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int plen(int L) { return L + (L >> 4); }
// Row stride of the x passes: the padded length plus 4 complex values, so that
// consecutive rows start 8 banks apart (the row unpack and gather read the same
// x of several rows at once).
__host__ __device__ constexpr int xstride(int L) { return plen(L) + 4; }

// Twiddle of entry e of a per-pass shared-memory table (DIR = -1 forward, +1 inverse)
template <int DIR>
__device__ __forceinline__ float2 twiddle_raw(const float2* tw, int e) {
  const float2 w = tw[e];
  return DIR < 0 ? w : make_float2(w.x, -w.y);
}

// log2 radix of pass i (of ceil(logL/maxlr) passes) for a 2^logL transform
__host__ __device__ __forceinline__ int fft_npass(int logL, int maxlr) { return (logL + maxlr - 1) / maxlr; }
__host__ __device__ __forceinline__ int fft_pass_lr(int logL, int maxlr, int i) {
  const int p = fft_npass(logL, maxlr);
  const int base = logL / p, extra = logL - base * p;
  return base + (i < extra ? 1 : 0);
}

// Fill the shared-memory twiddle table of the Stockham plan of a 2^logL
// transform (radices up to 2^MAXLR) from the global 4096-entry table.  The
// pass with sub-transform size Ns and radix R keeps W_{Ns R}^{r k} at
// (Ns - 1) + k (R - 1) + (r - 1), so lanes with consecutive k read
// consecutive (R-1)-strided entries, free of bank conflicts.  L - 1 entries;
// the caller synchronises before use.
template <int MAXLR>
__device__ __forceinline__ void load_twiddles(float2* dst, const float2* __restrict__ tw4096, int logL) {
  const int p = fft_npass(logL, MAXLR);
  int logNs = 0;
  for (int i = 0; i < p; ++i) {
    const int lr = fft_pass_lr(logL, MAXLR, i);
    const int Rm1 = (1 << lr) - 1, Ns = 1 << logNs;
    const int shift = TW_LOG - logNs - lr;
    for (int t = threadIdx.x; t < Ns * Rm1; t += blockDim.x) {
      const int k = t / Rm1, r = t - k * Rm1 + 1;
      dst[Ns - 1 + t] = __ldg(&tw4096[(r * k) << shift]);
    }
    logNs += lr;
  }
}

// cos(2 pi m / 16), m = 0..4 (decimal expansions of the constants)
__host__ __device__ constexpr float c16(int m) {
  return m == 0 ? 1.0f : m == 1 ? 0.923879532511286756f : m == 2 ? 0.707106781186547524f
         : m == 3 ? 0.382683432365089772f : 0.0f;
}

// Multiply by exp(DIR * 2 pi i M / 16), M a compile-time constant in [0, 16).
template <int DIR, int M>
__device__ __forceinline__ float2 rot16(float2 v) {
  constexpr int q = M / 4, r = M % 4;  // quarter turns and remainder
  float2 a = v;
  if (q == 1) a = DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  if (q == 2) a = make_float2(-v.x, -v.y);
  if (q == 3) a = DIR < 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  if (r == 0) return a;
  constexpr float c = c16(r), s = DIR * c16(4 - r);
  return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// Recursive radix-2 DFT of N values held in registers (N = 1, 2, 4, 8, 16),
// unnormalised, natural order in and out.  The even / odd split and the
// twiddles exp(DIR 2 pi i k / N) are all compile-time, so the values stay in
// registers.
template <int DIR, int N, int K>
__device__ __forceinline__ float2 rotN(float2 v) {
  static_assert(16 % N == 0 || N == 1, "radix");
  return rot16<DIR, (K * (16 / N)) % 16>(v);
}

template <int N, int DIR>
struct Dft {
  template <int K>
  __device__ __forceinline__ static void combine(float2 (&v)[N], const float2 (&e)[N / 2], const float2 (&o)[N / 2]) {
    if constexpr (K < N / 2) {
      const float2 t = rotN<DIR, N, K>(o[K]);
      bfly<(K * (16 / N)) % 16, 16>(e[K], t, v[K], v[K + N / 2]);
      combine<K + 1>(v, e, o);
    }
  }
  template <int I>
  __device__ __forceinline__ static void split(const float2 (&v)[N], float2 (&e)[N / 2], float2 (&o)[N / 2]) {
    if constexpr (I < N / 2) {
      e[I] = v[2 * I];
      o[I] = v[2 * I + 1];
      split<I + 1>(v, e, o);
    }
  }
  __device__ __forceinline__ static void run(float2 (&v)[N]) {
    float2 e[N / 2], o[N / 2];
    split<0>(v, e, o);
    Dft<N / 2, DIR>::run(e);
    Dft<N / 2, DIR>::run(o);
    combine<0>(v, e, o);
  }
};
template <int DIR>
struct Dft<1, DIR> {
  __device__ __forceinline__ static void run(float2 (&)[1]) {}
};

// In-register R-point DFT (R = 1, 2, 4, 8, 16), unnormalised.
template <int R, int DIR>
__device__ __forceinline__ void dft_reg(float2 (&v)[R]) {
  Dft<R, DIR>::run(v);
}

// Compile-time Stockham plan of a 2^LOGL transform with radices up to 2^MAXLR:
// ceil(LOGL/MAXLR) passes, the larger radices first.
template <int LOGL, int MAXLR>
struct Plan {
  static constexpr int P = (LOGL + MAXLR - 1) / MAXLR;
  static constexpr int lr(int i) { return LOGL / P + (i < LOGL - (LOGL / P) * P ? 1 : 0); }
  static constexpr int logns(int i) { return i == 0 ? 0 : logns(i - 1) + lr(i - 1); }
};

// padded offset of element i + r*S relative to pidx(i) when S is a multiple of 16
template <int S>
__device__ __forceinline__ constexpr int pstride() { return S + (S >> 4); }

// One Stockham pass (radix 2^LR, sub-transform size 2^LOGNS) over `ncols`
// padded columns of length 2^LOGL (column c at buf + c*cs), VPT values per
// thread.  Requires ncols*L <= VPT*blockDim.x.  Strides that are multiples of
// 16 turn every padded address of a butterfly into a constant offset.
// ZIN (first pass only): the upper half of each column is zero padding, so the
// butterfly inputs r >= R/2 (indices >= L/2) are not loaded.  ZOUT (last pass
// only): the caller reads only the lower half, so the outputs r >= R/2 are
// neither stored nor, once dead, computed.
template <int LOGL, int LR, int LOGNS, int DIR, int VPT, bool ZIN, bool ZOUT>
__device__ __forceinline__ void stockham_pass(float2* buf, int ncols, int cs, const float2* tw) {
  constexpr int R = 1 << LR, BPT = VPT / R;
  constexpr int LOGNB = LOGL - LR, NB = 1 << LOGNB, NS = 1 << LOGNS;
  const int total = ncols << LOGNB;
  float2 v[BPT][R];
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < total) {
      const int j = b & (NB - 1);
      const int c0 = (b >> LOGNB) * cs;
      constexpr int RL = ZIN ? R / 2 : R;  // inputs that are loaded
      if constexpr (NB % 16 == 0) {
        const int o0 = c0 + pidx(j);
#pragma unroll
        for (int r = 0; r < RL; ++r) v[q][r] = buf[o0 + r * pstride<NB>()];
      } else {
#pragma unroll
        for (int r = 0; r < RL; ++r) v[q][r] = buf[c0 + pidx(j + r * NB)];
      }
#pragma unroll
      for (int r = RL; r < R; ++r) v[q][r] = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < total) {
      const int j = b & (NB - 1);
      const int c0 = (b >> LOGNB) * cs;
      const int k = j & (NS - 1);
      if constexpr (LOGNS > 0) {
        const int t0 = (NS - 1) + k * (R - 1) - 1;  // this pass's twiddles, [k][r-1]
#pragma unroll
        for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], twiddle_raw<DIR>(tw, t0 + r));
      }
      dft_reg<R, DIR>(v[q]);
      const int o = ((j - k) << LR) + k;
      constexpr int RS = ZOUT ? R / 2 : R;  // outputs that are stored
      if constexpr (NS % 16 == 0) {
        const int o0 = c0 + pidx(o);
#pragma unroll
        for (int r = 0; r < RS; ++r) buf[o0 + r * pstride<NS>()] = v[q][r];
      } else if constexpr (NS == 1 && R == 16) {  // o = 16 j: padded 17 j + r
        const int o0 = c0 + 17 * j;
#pragma unroll
        for (int r = 0; r < RS; ++r) buf[o0 + r] = v[q][r];
      } else {
#pragma unroll
        for (int r = 0; r < RS; ++r) buf[c0 + pidx(o + r * NS)] = v[q][r];
      }
    }
  }
  __syncthreads();
}

// PRUNE: bit 0 = the upper half of every input column is zero (not read),
// bit 1 = only the lower half of every output column is used (not written).
template <int LOGL, int MAXLR, int PASS, int DIR, int PRUNE>
__device__ __forceinline__ void fft_passes(float2* buf, int ncols, int cs, const float2* tw) {
  using PL = Plan<LOGL, MAXLR>;
  if constexpr (PASS < PL::P) {
    stockham_pass<LOGL, PL::lr(PASS), PL::logns(PASS), DIR, (1 << MAXLR), (PRUNE & 1) && PASS == 0,
                  (PRUNE & 2) && PASS == PL::P - 1>(buf, ncols, cs, tw);
    fft_passes<LOGL, MAXLR, PASS + 1, DIR, PRUNE>(buf, ncols, cs, tw);
  }
}

// FFT of many padded columns of length 2^LOGL, in groups that fit 2^MAXLR
// values per thread.  All threads of the block must call it.
template <int LOGL, int MAXLR, int DIR, int PRUNE>
__device__ __forceinline__ void fft_many_ct(float2* buf, int ncols, int cs, const float2* tw) {
  const int per = max(1, ((1 << MAXLR) * (int)blockDim.x) >> LOGL);
  for (int c0 = 0; c0 < ncols; c0 += per)
    fft_passes<LOGL, MAXLR, 0, DIR, PRUNE>(buf + c0 * cs, min(per, ncols - c0), cs, tw);
}

// Runtime length dispatch (2^logL <= 4096).
template <int DIR, int MAXLR, int PRUNE = 0>
__device__ __forceinline__ void fft_many(float2* buf, int logL, int ncols, int cs, const float2* tw) {
  switch (logL) {
    case 1: fft_many_ct<1, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 2: fft_many_ct<2, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 3: fft_many_ct<3, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 4: fft_many_ct<4, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 5: fft_many_ct<5, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 6: fft_many_ct<6, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 7: fft_many_ct<7, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 8: fft_many_ct<8, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 9: fft_many_ct<9, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 10: fft_many_ct<10, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 11: fft_many_ct<11, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    case 12: fft_many_ct<12, MAXLR, DIR, PRUNE>(buf, ncols, cs, tw); break;
    default: break;  // logL == 0: identity
  }
}

// ------------------------------------------------ warp columns (four-step)
// A transform of length L = 32 Q (Q = 2 .. 32) as Q x 32: with n = j + 32 r and
// k = s + Q t,  X[s + Q t] = sum_j W32^{j t} W_L^{j s} sum_r x[j + 32 r] W_Q^{r s}.
// A warp takes W = 32 / Q columns together, 32 values per lane: lane j does the
// inner Q-point DFTs over r of every column and the twiddles W_L^{j s}; one
// transpose through the columns in shared memory; lane c Q + s does the outer
// 32-point DFT over j of column c.  Only __syncwarp, no block barrier.
//
// Column layout: element i at qidx(i) = i + i/32.  Lane j reading or writing
// element j + 32 r, and lanes (c, s) reading element j + 32 s of column c, both
// touch 16 different 8-byte banks per half-warp.

__device__ __forceinline__ int qidx(int i) { return i + (i >> 5); }
__host__ __device__ constexpr int qlen(int L) { return L + (L >> 5); }

// cos(2 pi m / 32), m = 0..8 (decimal expansions; the even entries equal c16)
__host__ __device__ constexpr float c32(int m) {
  return m == 0 ? 1.0f : m == 1 ? 0.980785280403230449126f : m == 2 ? 0.923879532511286756128f
         : m == 3 ? 0.831469612302545237079f : m == 4 ? 0.707106781186547524401f
         : m == 5 ? 0.555570233019602224743f : m == 6 ? 0.382683432365089771728f
         : m == 7 ? 0.195090322016128267848f : 0.0f;
}

// Multiply by exp(DIR * 2 pi i M / 32), M a compile-time constant in [0, 32).
template <int DIR, int M>
__device__ __forceinline__ float2 rot32(float2 v) {
  constexpr int q = M / 8, r = M % 8;
  float2 a = v;
  if (q == 1) a = DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  if (q == 2) a = make_float2(-v.x, -v.y);
  if (q == 3) a = DIR < 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  if (r == 0) return a;
  constexpr float c = c32(r), s = DIR * c32(8 - r);
  return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// Radix-2 decimation-in-time DFT of N register values (N = 1 .. 32),
// unnormalised, natural order.  ZH: inputs N/2 .. N-1 are zero (never read;
// the zeros stay zeros down the even / odd splits).  LO: only outputs
// 0 .. N/2-1 are formed.
template <int N, int DIR, bool ZH, bool LO>
struct DftZ {
  template <int K>
  __device__ __forceinline__ static void combine(float2 (&v)[N], const float2 (&e)[N / 2], const float2 (&o)[N / 2]) {
    if constexpr (K < N / 2) {
      const float2 t = rot32<DIR, (K * (32 / N)) % 32>(o[K]);
      constexpr int M = (K * (32 / N)) % 32;
      if constexpr (LO) {
        v[K] = (M != 0 && 4 * M == 32) ? cadd(e[K], t) : padd(e[K], t);
      } else {
        bfly<M, 32>(e[K], t, v[K], v[K + N / 2]);
      }
      combine<K + 1>(v, e, o);
    }
  }
  __device__ __forceinline__ static void run(float2 (&v)[N]) {
    float2 e[N / 2], o[N / 2];
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    DftZ<N / 2, DIR, ZH, false>::run(e);
    DftZ<N / 2, DIR, ZH, false>::run(o);
    combine<0>(v, e, o);
  }
};
template <int DIR, bool ZH, bool LO>
struct DftZ<2, DIR, ZH, LO> {
  __device__ __forceinline__ static void run(float2 (&v)[2]) {
    if constexpr (ZH) {
      v[1] = v[0];
    } else {
      const float2 a = v[0], b = v[1];
      v[0] = padd(a, b);
      if constexpr (!LO) v[1] = psub(a, b);
    }
  }
};
template <int DIR, bool ZH, bool LO>
struct DftZ<1, DIR, ZH, LO> {
  __device__ __forceinline__ static void run(float2 (&)[1]) {}
};

// Twiddles W_L^{j s} of the four-step transform of length L = 32 Q at
// [j * (Q - 1) + s - 1] (j in [0, 32), s in [1, Q)): lanes j reading the same s
// hit 16 different banks (odd row stride).  32 (Q - 1) entries; the caller
// synchronises before use.
__device__ __forceinline__ void load_twq(float2* dst, const float2* __restrict__ tw4096, int logL) {
  const int qm1 = (1 << (logL - 5)) - 1;
  for (int t = threadIdx.x; t < 32 * qm1; t += blockDim.x) {
    const int j = t / qm1, s = t - j * qm1 + 1;
    dst[t] = __ldg(&tw4096[(j * s) << (TW_LOG - logL)]);
  }
}

// Inner step of lane j for W = 32 / Q columns of length L = 32 Q held together:
// v[c Q + r] = x_c[j + 32 r] (r < Q; with ZH the values r >= Q/2 are zero and
// unread).  On return v[c Q + s] holds W_L^{j s} sum_r x_c[j + 32 r] W_Q^{r s}.
template <int Q, int DIR, bool ZH>
__device__ __forceinline__ void four_step_inner(float2 (&v)[32], const float2* twq, int lane) {
  constexpr int W = 32 / Q;
#pragma unroll
  for (int c = 0; c < W; ++c) {
    float2 u[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) u[r] = v[c * Q + r];
    DftZ<Q, DIR, ZH, false>::run(u);
#pragma unroll
    for (int r = 0; r < Q; ++r) v[c * Q + r] = u[r];
  }
  if constexpr (Q > 1) {
    const float2* t = twq + lane * (Q - 1) - 1;
#pragma unroll
    for (int s = 1; s < Q; ++s) {
      const float2 w = twiddle_raw<DIR>(t, s);
#pragma unroll
      for (int c = 0; c < W; ++c) v[c * Q + s] = cmul(v[c * Q + s], w);
    }
  }
}

// Transpose the inner results of the warp through its columns (column c at
// base + c*cs, qidx layout; only the first nc of the W columns exist) and do the
// outer 32-point step: on return lane l = c Q + s holds X_c[s + Q t] in v[t]
// (t < 16 only with LO).  The columns are free again when this returns.
// With cs = qlen(L) = 33 Q (mod 16: Q) the reads of the outer step, lanes
// (c, s) at element j + 32 s of column c, hit 16 different banks per half-warp.
template <int Q, int DIR, bool LO>
__device__ __forceinline__ void four_step_outer(float2 (&v)[32], float2* base, int cs, int nc, int lane) {
  constexpr int W = 32 / Q;
  if constexpr (W == 1) {  // one column: no column index, no guard
#pragma unroll
    for (int s = 0; s < 32; ++s) base[lane + 33 * s] = v[s];  // element lane + 32 s
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = base[j + 33 * lane];  // element j + 32 lane
  } else {
#pragma unroll
    for (int c = 0; c < W; ++c)
      if (c < nc)
#pragma unroll
        for (int s = 0; s < Q; ++s) base[c * cs + lane + 33 * s] = v[c * Q + s];  // element lane + 32 s
    __syncwarp();
    const int c = lane / Q, s = lane % Q;
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = (c < nc) ? base[c * cs + j + 33 * s] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  DftZ<32, DIR, false, LO>::run(v);
}

// ------------------------------------------- warp pairs (four-step, L = 2048)
// A 2048-point column as 64 x 32 taken by a pair of warps p = 0, 1 (64 lanes):
// with n = j + 32 r and k = s + 64 t,
//   X[s + 64 t] = sum_j W32^{j t} W2048^{j s} Y_j[s],  Y_j[s] = sum_r x[j + 32 r] W64^{r s}.
// Warp p forms the inner outputs s = 2 s' + p of lane j's 32 values as a
// 32-point DFT over r (s' its index) of x[j + 32 r] W64^{r p}: inputs r < 32
// only, the rest being zero padding (forward) or folded in beforehand as
// x[j + 32 r] + (-1)^p x[j + 32 (r + 32)] (inverse, all 64 inputs).  The pair
// then transposes through the column in shared memory (qidx layout) and lane
// c = lane + 32 p does the outer 32-point DFT of index s = c.  Registers stay at
// 32 values per lane, as in the single-warp form of length 1024.

// 64-thread barrier of warp pair `pair` (named barriers 1 .. 8; 0 is the block's).
__device__ __forceinline__ void pair_sync(int pair) { asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory"); }

// Inner step of warp p for lane j: v[r] (r < 32) in, Y_j[2 s' + p] W2048^{j (2 s' + p)}
// stored at element j + 32 (2 s' + p) of column C.  twq: W2048^{j s} at
// [j * 63 + s - 1] (load_twq of length 2048).
template <int DIR>
__device__ __forceinline__ void pair_inner(float2 (&v)[32], const float2* twq, int lane, int p, float2* C) {
  if (p) {
#pragma unroll
    for (int r = 1; r < 32; ++r) v[r] = cmul(v[r], twiddle_raw<DIR>(twq + r * 63 - 1, 32));  // W64^r = W2048^{32 r}
  }
  DftZ<32, DIR, false, false>::run(v);
  const float2* t = twq + lane * 63 - 1;
#pragma unroll
  for (int q = 0; q < 32; ++q) {
    const int s = 2 * q + p;
    const float2 w = (s == 0) ? v[q] : cmul(v[q], twiddle_raw<DIR>(t, s));
    C[qidx(lane + 32 * s)] = w;
  }
}

// Outer step of lane c = lane + 32 p of the pair: v[t] = X[c + 64 t] (t < 16 only with LO).
template <int DIR, bool LO>
__device__ __forceinline__ void pair_outer(float2 (&v)[32], const float2* C, int c) {
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = C[qidx(j + 32 * c)];
  DftZ<32, DIR, false, LO>::run(v);
}

// Transforms of length 2048 of `nrows` rows in shared memory (row r at
// buf + r*cs, qidx layout) by warp pairs, one row per pair at a time, in
// place.  ZIN: the upper half of every input row is zero padding (not read);
// otherwise the inner step folds it in.  LO: only the lower half of every output
// row is written.  A trailing warp without a partner takes no row.  No block
// barrier: the caller synchronises before (rows and twiddles written) and after.
template <int DIR, bool ZIN, bool LO>
__device__ __forceinline__ void pair_rows(float2* buf, int nrows, int cs, const float2* twq) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, pair = warp >> 1, p = warp & 1;
  const int npairs = blockDim.x >> 6;
  if (pair >= npairs) return;
  const int c = lane + 32 * p;
  for (int r0 = pair; r0 < nrows; r0 += npairs) {
    float2* R = buf + r0 * cs;
    float2 v[32];
#pragma unroll
    for (int b = 0; b < 32; ++b) {
      const float2 lo = R[qidx(lane + 32 * b)];
      if constexpr (ZIN) {
        v[b] = lo;
      } else {  // x + (-1)^p x' of elements lane + 32 b and lane + 32 b + 1024
        const float2 hi = R[qidx(lane + 32 * b + 1024)];
        v[b] = p ? csub(lo, hi) : cadd(lo, hi);
      }
    }
    pair_sync(pair);  // both warps have read the row before the inner step overwrites it
    pair_inner<DIR>(v, twq, lane, p, R);
    pair_sync(pair);
    pair_outer<DIR, LO>(v, R, c);
    pair_sync(pair);  // both warps have read the row before it takes the outputs
#pragma unroll
    for (int t = 0; t < (LO ? 16 : 32); ++t) R[qidx(c + 64 * t)] = v[t];
  }
}

// Transforms of length 32 Q of `nrows` rows in shared memory (row r at
// buf + r*cs, qidx layout), W = 32 / Q rows per warp at a time, in place.  ZIN:
// the upper half of every input row is zero padding (not read).  LO: only the
// lower half of every output row is written.  No block barrier: the caller
// synchronises before (rows and twiddles written) and after.
template <int Q, int DIR, bool ZIN, bool LO>
__device__ __forceinline__ void warp_rows(float2* buf, int nrows, int cs, const float2* twq) {
  constexpr int W = 32 / Q;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r0 = (threadIdx.x >> 5) * W; r0 < nrows; r0 += nw * W) {
    float2* R = buf + r0 * cs;
    const int nc = W == 1 ? 1 : min(W, nrows - r0);
    float2 v[32];
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
      for (int r = 0; r < Q; ++r)
        v[c * Q + r] = (c < nc && (!ZIN || r < Q / 2)) ? R[c * cs + lane + 33 * r] : make_float2(0.f, 0.f);
    four_step_inner<Q, DIR, ZIN>(v, twq, lane);
    four_step_outer<Q, DIR, LO>(v, R, cs, nc, lane);
    if constexpr (W == 1) {
#pragma unroll
      for (int t = 0; t < (LO ? 16 : 32); ++t) R[lane + 33 * t] = v[t];
    } else {
      const int c = lane / Q, s = lane % Q;
      if (c < nc)
#pragma unroll
        for (int t = 0; t < (LO ? 16 : 32); ++t) R[c * cs + qidx(s + Q * t)] = v[t];
    }
  }
}

// Padded index of the x rows: i + i/32 for 1024-point rows (warp transforms),
// else pidx.
__device__ __forceinline__ int xidx(int i, int sh) { return i + (i >> sh); }

// Row stride of the x passes for tiles of ty rows.  512-, 1024- and 2048-point
// rows (warp rows and warp-pair rows, qidx layout): qlen plus 16 / (row slots of
// the tile, ty rounded up to a power of two) complex values, so that the gather
// and the unpack, whose half-warps touch the same few x of every row slot, hit
// 16 different 8-byte banks (the outer step of these lengths reads within one
// row per half-warp).
__host__ __device__ inline int xrow_stride(int L, int ty) {
  if (L != 1024 && L != 512 && L != 2048) return xstride(L);
  int slots = 1;
  while (slots < ty) slots <<= 1;
  return qlen(L) + (slots >= 16 ? 1 : 16 / slots);
}

}  // namespace mpx
