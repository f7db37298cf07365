// physics.cuh -- device-side magnet description and the local effective-field
// terms (exchange, DMI, uniaxial anisotropy, Zeeman) plus the LLG torque.
//
// Each term follows the reference kernel cell by cell (paths relative to the
// mumax-plus source tree):
//   exchange   physics/exchange.cu:20-104  (harmonic-mean A, inter-region LUT,
//              Neumann ghost m + Gamma/(2A) delta, open boundaries)
//   DMI        physics/dmi.cu:19-110, getGamma physics/dmi.hpp:53-69
//   anisotropy physics/anisotropy.cu:25-55 (uniaxial)
//   Zeeman     physics/zeeman.cu:53-91 (world bias + magnet bias)
//   torque     physics/torque.cu:21-45 (LLG), :58-77 (damping only)
// Grid indexing and wrapping: core/grid.hpp:55-89, core/system.hpp:91-119.
// The terms are evaluated from SoA float32 m with FP32 arithmetic, like the
// reference SINGLE build, and summed in the order of
// physics/effectivefield.cpp:15-28 (exchange, anisotropy, external, DMI, demag).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mpx {

constexpr float GAMMA_LL = 1.7595e11f;     // rad/(T s), physics/constants.hpp
constexpr double MU0_D = 1.25663706212e-6; // H/m

// Term bits of a magnet (a term whose parameters are assured zero is skipped,
// as the reference's *AssuredZero checks do).
enum : unsigned {
  TERM_EXCH = 1u, TERM_DMI = 2u, TERM_ANIS = 4u, TERM_EXT = 8u, TERM_DEMAG = 16u,
  FLAG_OPENBC = 256u, FLAG_MAGNET_BIAS = 512u,
  FLAG_CUBIC = 1024u,  // the anisotropy term is cubic (uniaxial otherwise)
  FLAG_STRAY = 2048u,  // stray fields of other magnets in `hstray`
  FLAG_STT_ZL = 4096u, FLAG_STT_SL = 8192u,  // spin-transfer torque: Zhang-Li or Slonczewski
  FLAG_THERMAL = 16384u  // thermal noise (temperature not zero)
};

struct DScalar {  // uniform value or per-cell array
  float u;
  const float* __restrict__ p;
  __device__ __forceinline__ float at(int i) const { return p ? __ldg(p + i) : u; }
};
struct DVector {  // uniform value or per-cell SoA array (3*N)
  float u[3];
  const float* __restrict__ p;
  __device__ __forceinline__ float3 at(int i, int N) const {
    if (!p) return make_float3(u[0], u[1], u[2]);
    return make_float3(__ldg(p + i), __ldg(p + N + i), __ldg(p + 2 * N + i));
  }
};

// Device description of one magnet (lives in a device array, indexed by slot).
struct MagnetDev {
  int n[3], N;
  int o[3];          // grid origin
  int mg[3], mgo[3]; // mastergrid size / origin (size 0: no wrap)
  float cs[3];       // cell size
  float w[3];        // 1/cellsize^2
  float inv_cs[3];   // 1/cellsize (divisions by the finite difference become products)
  const unsigned char* __restrict__ geom;  // NULL: all cells in geometry
  const unsigned* __restrict__ reg;        // NULL: region 0
  DScalar msat, aex, alpha, ku1, ku2, frozen;
  DVector anisU, bias;
  DScalar kc1, kc2, kc3;  // cubic anisotropy constants
  DVector anisC1, anisC2; // cubic anisotropy axes
  DScalar pol, xi, lambda_, epsp, flt;  // spin-transfer torque parameters
  DVector jcur, fixl;
  int fl_below;           // Slonczewski fixed layer below the free layer
  DScalar temp;           // temperature (K)
  unsigned long long seed;  // thermal noise generator seed
  float noise_pref;       // 2 kB gamma_LL / cell volume
  DScalar dmi[9];  // xxy, xxz, xyz, yxy, yxz, yyz, zxy, zxz, zyz
  float inter_u, scale_u;
  const float* __restrict__ inter_lut;
  const float* __restrict__ scale_lut;
  float wb[3];       // world bias field
  unsigned terms;    // TERM_* and FLAG_* bits
  int group;         // solve group slot
  // demag FFT plan: padded sizes P = 2^logP, Fh = Px/2+1
  int logP[3], P[3], Fh;
  int kcomp;         // 6 (3-D kernel) or 4 (Pz == 1)
  float2* spec;      // spectrum S[kx][c][z][y]
  float2* tspec;     // split y/z path: y-transformed spectrum T[kx][c][z][ky] (Py rows), else NULL
  const float* __restrict__ kspec;  // kernel spectrum [kx][kz'][kcomp][ky']
  float* buf[9];     // field buffers (3N floats each); roles given by the group map
  const float* hstray;  // stray field of the other magnets of the world (3N), or NULL
  // Fast path: every parameter uniform, no geometry, no regions.  Set on the
  // host together with the precomputed uniform values below.
  int fast;
  float fe[3];       // 2 A w[axis]: exchange coefficient per axis
  float fd[9];       // uniform DMI tensor, MPX_DMI_* order
  float fu[3];       // normalised uniaxial axis
  float fb[3];       // world bias + magnet bias
  float fa, finv_2a, finv_ms, fk1, fk2;
  float fc[3][3];    // cubic axes c1, c2 (normalised) and c3 = c1 x c2
  float fkc[3];      // cubic constants kc1, kc2, kc3
};

// Solve-group state (time integration); lives in a device array.
struct GroupDev {
  double t, dt, t_stop, dt_saved, max_error, headroom, lower, upper, torque_stop;
  unsigned long long err_bits;   // max error of the current attempt (double bits)
  unsigned long long tmax_bits;  // max |torque| of the accepted state (double bits)
  long long steps, rejected, attempts, steps_left;
  int status;     // 0 idle, 1 running, 2 finished, 3 failed
  int mode;       // 0 run(duration), 1 steps(n), 2 sampled run through samp_t
  int phase;      // 0 regular steps, 1 final step of run()
  int adaptive;
  int k0_valid;
  int finished_flag;  // set when the group finished, cleared by the host poll
  int map[9];     // buffer roles: [0] x0 (state), [1] xs (stage / new state), [2+s] k_s
  int torque_kind;  // right-hand side of the stages: 0 LLG torque, 1 damping torque only (relax)
  int thermal;      // some magnet of the group has thermal noise: k0 is never reused
  // sampled run (mode 2): increasing time points samp_t[0, samp_n), the next one
  // samp_k; rows [samp_lo, samp_hi) of the table samp_out (samp_row doubles
  // per row: t, then <m> of every magnet of the group) are due after this attempt
  const double* samp_t;
  double* samp_out;
  int samp_n, samp_k, samp_lo, samp_hi, samp_row;
};

enum { GS_IDLE = 0, GS_RUNNING = 1, GS_FINISHED = 2, GS_FAILED = 3 };

__device__ __forceinline__ float harmonic_mean(float a, float b) {  // core/datatypes.hpp
  if (a + b == 0.0f) return 0.0f;
  if (a == b) return a;
  return 2 * a * b / (a + b);
}

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ bool in_geom(const MagnetDev& M, int i) { return !M.geom || M.geom[i]; }

#ifdef MPX_BOUNDS_CHECK
// Checked build (libmpx_checked.so): every per-cell access of a SoA field
// buffer through load3 / ldg3 / store3 verifies 0 <= i < N.  The first bad
// access is recorded (bit 63 set, N in bits 32..62, i in the low word) and
// skipped -- a load gives 0 -- so the kernel runs to its end and the host reads
// the record with mpx_bounds_check.  Nothing traps.
__device__ unsigned long long g_bounds_first_bad;
__device__ __forceinline__ bool cell_ok(int N, int i) {
  if ((unsigned)i < (unsigned)N) return true;
  atomicCAS(&g_bounds_first_bad, 0ull, (1ull << 63) | ((unsigned long long)(unsigned)N << 32) | (unsigned)i);
  return false;
}
// the same for an element index i of an array of n elements (spectra, vector
// accesses); n above 2^31 - 1 is recorded as 2^31 - 1, i by its low 32 bits
__device__ __forceinline__ bool span_ok(size_t i, size_t n) {
  if (i < n) return true;
  const unsigned long long nn = n < 0x7fffffffull ? n : 0x7fffffffull;
  atomicCAS(&g_bounds_first_bad, 0ull, (1ull << 63) | (nn << 32) | (i & 0xffffffffull));
  return false;
}
#else
__device__ __forceinline__ bool cell_ok(int, int) { return true; }
__device__ __forceinline__ bool span_ok(size_t, size_t) { return true; }
#endif

__device__ __forceinline__ float3 load3(const float* __restrict__ a, int N, int i) {
  if (!cell_ok(N, i)) return f3(0.f, 0.f, 0.f);
  return f3(a[i], a[N + i], a[2 * N + i]);
}
// read-only path: for buffers a kernel never writes
__device__ __forceinline__ float3 ldg3(const float* __restrict__ a, int N, int i) {
  if (!cell_ok(N, i)) return f3(0.f, 0.f, 0.f);
  return f3(__ldg(a + i), __ldg(a + N + i), __ldg(a + 2 * N + i));
}
__device__ __forceinline__ void store3(float* a, int N, int i, float3 v) {
  if (!cell_ok(N, i)) return;
  a[i] = v.x;
  a[N + i] = v.y;
  a[2 * N + i] = v.z;
}

// Neighbour coordinate along one axis after the mastergrid wrap
// (core/grid.hpp:73-81); -1 when it leaves the grid.  The grid lies inside the
// mastergrid, so one conditional wrap suffices.
__device__ __forceinline__ int nb_coord(int c, int d, int n, int go, int mg, int mgo) {
  int g = c + d + go;
  if (mg > 0) {
    int r = g - mgo;
    r = r < 0 ? r + mg : (r >= mg ? r - mg : r);
    g = mgo + r;
  }
  const int l = g - go;
  return (l >= 0 && l < n) ? l : -1;
}

// physics/dmi.hpp:53-69 getGamma with normal (nx, ny, nz)
__device__ __forceinline__ float3 get_gamma(const MagnetDev& M, int i, int nx, int ny, int nz, float3 m) {
  const float Dxxy = M.dmi[0].at(i), Dxxz = M.dmi[1].at(i), Dxyz = M.dmi[2].at(i);
  const float Dyxy = M.dmi[3].at(i), Dyxz = M.dmi[4].at(i), Dyyz = M.dmi[5].at(i);
  const float Dzxy = M.dmi[6].at(i), Dzxz = M.dmi[7].at(i), Dzyz = M.dmi[8].at(i);
  return f3(-Dxxy * nx * m.y - Dxxz * nx * m.z - Dyxz * ny * m.z - Dzxy * nz * m.y - Dyxy * ny * m.y -
                Dzxz * nz * m.z,
            Dxxy * nx * m.x - Dzyz * nz * m.z + Dyxy * ny * m.x - Dxyz * nx * m.z + Dzxy * nz * m.x -
                Dyyz * ny * m.z,
            Dxxz * nx * m.x + Dyyz * ny * m.y + Dxyz * nx * m.y + Dyxz * ny * m.x + Dzxz * nz * m.x +
                Dzyz * nz * m.y);
}

__device__ __forceinline__ float lut_value(const float* __restrict__ lut, float u, unsigned i, unsigned j) {
  if (!lut) return u;
  const int k = (i > j) ? (int)(i * (i - 1) / 2 + j) : (int)(j * (j - 1) / 2 + i);
  return __ldg(lut + k);
}

// The local terms of the effective field of cell (x, y, z) = i, which is in the
// geometry with msat != 0.  `mask` selects terms (TERM_*).  Each term is
// computed on its own, then added in the reference's order.
// a / |a|, or 0 for a zero vector (core/datatypes.hpp normalized)
__device__ __forceinline__ float3 normalized3(float3 a) {
  const float n = sqrtf(dot3(a, a));
  const float s = (n == 0.0f) ? 0.0f : 1.0f / n;
  return f3(s * a.x, s * a.y, s * a.z);
}

// physics/anisotropy.cu:57-106 (k_cubicanisotropyField): cubic anisotropy field of
// axes c1, c2, c3 = c1 x c2 and constants kc1..kc3, times 1/Ms.
__device__ __forceinline__ float3 cubic_field(float3 m, float3 c1, float3 c2, float3 c3, float kc1, float kc2,
                                              float kc3, float inv_ms) {
  const float a = dot3(c1, m), b = dot3(c2, m), c = dot3(c3, m);
  const float a2 = a * a, b2 = b * b, c2_ = c * c;
  const float f1 = -2 * kc1 * (b2 + c2_) * a - 2 * kc2 * (b2 * c2_) * a - 4 * kc3 * (b2 * b2 + c2_ * c2_) * (a2 * a);
  const float f2 = -2 * kc1 * (a2 + c2_) * b - 2 * kc2 * (a2 * c2_) * b - 4 * kc3 * (a2 * a2 + c2_ * c2_) * (b2 * b);
  const float f3_ = -2 * kc1 * (a2 + b2) * c - 2 * kc2 * (a2 * b2) * c - 4 * kc3 * (a2 * a2 + b2 * b2) * (c2_ * c);
  return f3(inv_ms * (f1 * c1.x + f2 * c2.x + f3_ * c3.x), inv_ms * (f1 * c1.y + f2 * c2.y + f3_ * c3.y),
            inv_ms * (f1 * c1.z + f2 * c2.z + f3_ * c3.z));
}

// physics/anisotropy.cu:185-215 (k_cubanisotropyEnergyDensity)
__device__ __forceinline__ float cubic_energy(float3 m, float3 c1, float3 c2, float3 c3, float kc1, float kc2,
                                              float kc3) {
  const float a = dot3(c1, m), b = dot3(c2, m), c = dot3(c3, m);
  const float a2 = a * a, b2 = b * b, c2_ = c * c;
  float e = kc1 * (a2 * b2 + a2 * c2_ + b2 * c2_);
  e += kc2 * a2 * b2 * c2_;
  e += kc3 * (a2 * a2 * b2 * b2 + a2 * a2 * c2_ * c2_ + b2 * b2 * c2_ * c2_);
  return e;
}

struct LocalOut {
  float3 exch, anis, ext, dmi;
};

__device__ __forceinline__ LocalOut local_terms(const MagnetDev& M, const float* __restrict__ m, int x, int y,
                                                int z, int i, float3 mc, unsigned mask) {
  LocalOut o;
  o.exch = o.anis = o.ext = o.dmi = f3(0, 0, 0);
  const int N = M.N;
  const float ms = M.msat.at(i);
  const bool openbc = (M.terms & FLAG_OPENBC) != 0;
  const bool do_exch = (mask & TERM_EXCH) && (M.terms & TERM_EXCH);
  const bool do_dmi = (mask & TERM_DMI) && (M.terms & TERM_DMI);
  // Divisions by Ms, 2A and the finite difference are products with
  // reciprocals (one division per cell): IEEE division takes a slow path on
  // subnormal operands, which the in-plane components of a nearly uniform
  // state produce (results agree to 1 ulp per operation).
  const float inv_ms = 1.0f / ms;
  if (do_exch || do_dmi) {
    const float a = M.aex.at(i);
    const float inv_2a = (a == 0.0f) ? 0.0f : 0.5f / a;
    const bool dmi_open = (a == 0.0f) ? true : openbc;
    float3 he = f3(0, 0, 0), hd = f3(0, 0, 0);
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int axis = r >> 1;
      const int d = (r & 1) ? 1 : -1;
      int xx = x, yy = y, zz = z;
      int nc;
      if (axis == 0) { nc = nb_coord(x, d, M.n[0], M.o[0], M.mg[0], M.mgo[0]); xx = nc; }
      else if (axis == 1) { nc = nb_coord(y, d, M.n[1], M.o[1], M.mg[1], M.mgo[1]); yy = nc; }
      else { nc = nb_coord(z, d, M.n[2], M.o[2], M.mg[2], M.mgo[2]); zz = nc; }
      const int j = (nc >= 0) ? xx + M.n[0] * (yy + M.n[1] * zz) : -1;
      const bool nin = (nc >= 0) && in_geom(M, j);
      const float delta = d * M.cs[axis];
      const float inv_delta = d * M.inv_cs[axis];
      const int nx_ = axis == 0, ny_ = axis == 1, nz_ = axis == 2;
      // ---- exchange (physics/exchange.cu:58-102)
      if (do_exch) {
        bool skip = (!nin && openbc) || (openbc && M.msat.at(j) == 0.0f);
        if (!skip) {
          float inter = 0.0f, scale = 1.0f, a_;
          float3 m_;
          bool neumann_skip = false;
          if (nin) {
            m_ = ldg3(m, N, j);
            a_ = M.aex.at(j);
            const unsigned ri = M.reg ? M.reg[i] : 0u, rj = M.reg ? M.reg[j] : 0u;
            if (ri != rj) {
              scale = lut_value(M.scale_lut, M.scale_u, ri, rj);
              inter = lut_value(M.inter_lut, M.inter_u, ri, rj);
            }
          } else {
            if (a == 0.0f) {
              neumann_skip = true;
              m_ = mc;
              a_ = a;
            } else {
              const float3 G = get_gamma(M, i, nx_, ny_, nz_, mc);
              m_ = mc + delta * (inv_2a * G);
              a_ = a;
            }
          }
          if (!neumann_skip) {
            float A = (inter != 0.0f) ? inter : harmonic_mean(a, a_);
            A *= scale;
            he = he + (2 * A * M.w[axis]) * (m_ - mc);
          }
        }
      }
      // ---- DMI (physics/dmi.cu:46-106)
      if (do_dmi) {
        const int jj = nin ? j : i;
        const bool skip = dmi_open && (!nin || M.msat.at(jj) == 0.0f);
        if (!skip) {
          const int c0 = 3 * axis;  // x: xxy,xxz,xyz ; y: yxy,yxz,yyz ; z: zxy,zxz,zyz
          float Dxy, Dxz, Dyz;
          if (jj == i) {
            Dxy = M.dmi[c0].at(i); Dxz = M.dmi[c0 + 1].at(i); Dyz = M.dmi[c0 + 2].at(i);
          } else {
            Dxy = harmonic_mean(M.dmi[c0].at(i), M.dmi[c0].at(jj));
            Dxz = harmonic_mean(M.dmi[c0 + 1].at(i), M.dmi[c0 + 1].at(jj));
            Dyz = harmonic_mean(M.dmi[c0 + 2].at(i), M.dmi[c0 + 2].at(jj));
          }
          const float Dzx = -Dxz, Dyx = -Dxy, Dzy = -Dyz;
          float3 m_;
          if (!nin && !dmi_open) {
            const float3 G = get_gamma(M, i, nx_, ny_, nz_, mc);
            m_ = mc + delta * (inv_2a * G);
          } else {
            m_ = ldg3(m, N, jj);
          }
          hd.x += (Dxy * m_.y + Dxz * m_.z) * inv_delta;
          hd.y += (Dyx * m_.x + Dyz * m_.z) * inv_delta;
          hd.z += (Dzx * m_.x + Dzy * m_.y) * inv_delta;
        }
      }
    }
    if (do_exch) o.exch = inv_ms * he;
    if (do_dmi) o.dmi = inv_ms * hd;
  }
  if ((mask & TERM_ANIS) && (M.terms & TERM_ANIS) && (M.terms & FLAG_CUBIC)) {  // physics/anisotropy.cu:57-106
    const float3 c1 = normalized3(M.anisC1.at(i, N)), c2 = normalized3(M.anisC2.at(i, N));
    o.anis = cubic_field(mc, c1, c2, cross3(c1, c2), M.kc1.at(i), M.kc2.at(i), M.kc3.at(i), inv_ms);
  } else if ((mask & TERM_ANIS) && (M.terms & TERM_ANIS)) {  // physics/anisotropy.cu:45-54
    float3 u = M.anisU.at(i, N);
    const float nu = sqrtf(dot3(u, u));
    const float s = (nu == 0.0f) ? 0.0f : 1.0f / nu;
    u = s * u;
    const float k1 = M.ku1.at(i), k2 = M.ku2.at(i);
    const float mu = dot3(mc, u);
    o.anis = inv_ms * ((2 * k1 * mu + 4 * k2 * mu * mu * mu) * u);
  }
  if ((mask & TERM_EXT) && (M.terms & TERM_EXT)) {  // physics/zeeman.cu:64-68
    float3 b = f3(M.wb[0], M.wb[1], M.wb[2]);
    if (M.terms & FLAG_MAGNET_BIAS) b = b + M.bias.at(i, N);
    if (M.terms & FLAG_STRAY) b = b + load3(M.hstray, N, i);
    o.ext = b;
  }
  return o;
}

// The same local terms when every parameter is uniform and there is no
// geometry mask and no region map (MagnetDev::fast): the harmonic means reduce
// to the uniform values, all neighbours inside the grid are in the geometry,
// and the per-axis exchange coefficients, DMI tensor, normalised anisotropy
// axis and total bias field are precomputed.
__device__ __forceinline__ float3 gamma_uniform(const float* D, int axis, float3 m) {
  // physics/dmi.hpp:53-69 with normal e_axis and uniform tensor D
  if (axis == 0) return f3(-D[0] * m.y - D[1] * m.z, D[0] * m.x - D[2] * m.z, D[1] * m.x + D[2] * m.y);
  if (axis == 1) return f3(-D[4] * m.z - D[3] * m.y, D[3] * m.x - D[5] * m.z, D[5] * m.y + D[4] * m.x);
  return f3(-D[6] * m.y - D[7] * m.z, -D[8] * m.z + D[6] * m.x, D[7] * m.x + D[8] * m.y);
}

__device__ __forceinline__ LocalOut local_terms_fast(const MagnetDev& M, const float* __restrict__ m, int x, int y,
                                                     int z, float3 mc) {
  LocalOut o;
  o.exch = o.anis = o.ext = o.dmi = f3(0, 0, 0);
  const int N = M.N;
  const bool openbc = (M.terms & FLAG_OPENBC) != 0;
  const bool do_exch = (M.terms & TERM_EXCH) != 0;
  const bool do_dmi = (M.terms & TERM_DMI) != 0;
  if (do_exch || do_dmi) {
    const float a = M.fa;
    const bool dmi_open = (a == 0.0f) || openbc;
    const bool neumann = !openbc && a != 0.0f;
    float3 he = f3(0, 0, 0), hd = f3(0, 0, 0);
    // all six neighbour loads first (independent, in flight together), then the sums
    float3 mn[6];
    bool nin[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int axis = r >> 1;
      const int d = (r & 1) ? 1 : -1;
      int xx = x, yy = y, zz = z, nc;
      if (axis == 0) { nc = nb_coord(x, d, M.n[0], M.o[0], M.mg[0], M.mgo[0]); xx = nc; }
      else if (axis == 1) { nc = nb_coord(y, d, M.n[1], M.o[1], M.mg[1], M.mgo[1]); yy = nc; }
      else { nc = nb_coord(z, d, M.n[2], M.o[2], M.mg[2], M.mgo[2]); zz = nc; }
      nin[r] = nc >= 0;
      mn[r] = nin[r] ? ldg3(m, N, xx + M.n[0] * (yy + M.n[1] * zz)) : mc;
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int axis = r >> 1;
      const int d = (r & 1) ? 1 : -1;
      float3 m_ = mn[r];
      if (!nin[r] && neumann) {  // ghost cell m + Gamma/(2A) delta
        const float3 G = gamma_uniform(M.fd, axis, mc);
        m_ = mc + (d * M.cs[axis]) * (M.finv_2a * G);
      }
      if (do_exch && (nin[r] || neumann)) he = he + M.fe[axis] * (m_ - mc);
      if (do_dmi && (nin[r] || !dmi_open)) {
        const float Dxy = M.fd[3 * axis], Dxz = M.fd[3 * axis + 1], Dyz = M.fd[3 * axis + 2];
        const float inv_delta = d * M.inv_cs[axis];
        hd.x += (Dxy * m_.y + Dxz * m_.z) * inv_delta;
        hd.y += (-Dxy * m_.x + Dyz * m_.z) * inv_delta;
        hd.z += (-Dxz * m_.x - Dyz * m_.y) * inv_delta;
      }
    }
    if (do_exch) o.exch = M.finv_ms * he;
    if (do_dmi) o.dmi = M.finv_ms * hd;
  }
  if ((M.terms & TERM_ANIS) && (M.terms & FLAG_CUBIC)) {
    o.anis = cubic_field(mc, f3(M.fc[0][0], M.fc[0][1], M.fc[0][2]), f3(M.fc[1][0], M.fc[1][1], M.fc[1][2]),
                         f3(M.fc[2][0], M.fc[2][1], M.fc[2][2]), M.fkc[0], M.fkc[1], M.fkc[2], M.finv_ms);
  } else if (M.terms & TERM_ANIS) {
    const float3 u = f3(M.fu[0], M.fu[1], M.fu[2]);
    const float mu = dot3(mc, u);
    o.anis = M.finv_ms * ((2 * M.fk1 * mu + 4 * M.fk2 * mu * mu * mu) * u);
  }
  if (M.terms & TERM_EXT) {
    o.ext = f3(M.fb[0], M.fb[1], M.fb[2]);
    if (M.terms & FLAG_STRAY) {
      const float3 s = load3(M.hstray, N, x + M.n[0] * (y + M.n[1] * z));
      o.ext = f3(o.ext.x + s.x, o.ext.y + s.y, o.ext.z + s.z);
    }
  }
  return o;
}

// physics/torque.cu:36-42
__device__ __forceinline__ float3 llg_torque(float3 m, float3 h, float a) {
  const float3 mxh = cross3(m, h);
  const float3 mxmxh = cross3(m, mxh);
  return (-GAMMA_LL / (1 + a * a)) * (mxh + a * mxmxh);
}

// physics/stt.cu:26-185: spin-transfer torque (1/s) of the cell, Zhang-Li (central
// differences of m along the current, neighbours in the grid with msat != 0,
// mastergrid wrap) or Slonczewski (current along z through a free layer).
constexpr float MUB_F = 9.274009152e-24f, QE_F = 1.60217646e-19f, HBAR_F = 1.054571817e-34f;
__device__ __noinline__ float3 stt_torque(const MagnetDev& M, const float* __restrict__ m, int x, int y, int z, int i,
                                          float3 mc) {
  const int N = M.N;
  const float ms = M.msat.at(i), alpha = M.alpha.at(i);
  if (M.terms & FLAG_STT_SL) {
    const float jz = M.jcur.at(i, N).z;
    const float pol = M.pol.at(i), lambda = M.lambda_.at(i), eps_p = M.epsp.at(i);
    const float3 p = M.fixl.at(i, N);
    float d = M.flt.at(i);
    if (M.fl_below) d = -d;
    if (ms == 0.f || jz == 0.f || d == 0.f || (p.x == 0.f && p.y == 0.f && p.z == 0.f) ||
        (eps_p == 0.f && (lambda == 0.f || pol == 0.f)))
      return f3(0.f, 0.f, 0.f);
    const float B = (HBAR_F / QE_F) * jz / (ms * d);
    const float l2 = lambda * lambda;
    const float eps = pol * l2 / ((l2 + 1) + (l2 - 1) * dot3(mc, p));
    const float3 pxm = cross3(p, mc);
    const float3 mxpxm = cross3(mc, pxm);
    const float s = (B / (1 + alpha * alpha)) * GAMMA_LL;
    return f3(((eps + eps_p * alpha) * mxpxm.x + (eps_p - eps * alpha) * pxm.x) * s,
              ((eps + eps_p * alpha) * mxpxm.y + (eps_p - eps * alpha) * pxm.y) * s,
              ((eps + eps_p * alpha) * mxpxm.z + (eps_p - eps * alpha) * pxm.z) * s);
  }
  const float3 j = M.jcur.at(i, N);
  const float pol = M.pol.at(i), xi = M.xi.at(i);
  if (ms == 0.f || pol == 0.f || (j.x == 0.f && j.y == 0.f && j.z == 0.f)) return f3(0.f, 0.f, 0.f);
  const float cu = MUB_F * pol / (QE_F * ms * (1 + xi * xi));
  const float u[3] = {cu * j.x, cu * j.y, cu * j.z};
  float3 hs = f3(0.f, 0.f, 0.f);
  for (int axis = 0; axis < 3; ++axis)
    for (int d = -1; d <= 1; d += 2) {
      int xx = x, yy = y, zz = z, nc;
      if (axis == 0) { nc = nb_coord(x, d, M.n[0], M.o[0], M.mg[0], M.mgo[0]); xx = nc; }
      else if (axis == 1) { nc = nb_coord(y, d, M.n[1], M.o[1], M.mg[1], M.mgo[1]); yy = nc; }
      else { nc = nb_coord(z, d, M.n[2], M.o[2], M.mg[2], M.mgo[2]); zz = nc; }
      if (nc < 0) continue;
      const int jn = xx + M.n[0] * (yy + M.n[1] * zz);
      if (M.msat.at(jn) == 0.f) continue;
      const float3 mn = load3(m, N, jn);
      const float c = d * u[axis] / (2 * M.cs[axis]);
      hs = f3(hs.x + c * mn.x, hs.y + c * mn.y, hs.z + c * mn.z);
    }
  const float3 mxh = cross3(mc, hs);
  const float3 mxmxh = cross3(mc, mxh);
  const float s = -1 / (1 + alpha * alpha);
  return f3(s * ((1 + xi * alpha) * mxmxh.x + (xi - alpha) * mxh.x), s * ((1 + xi * alpha) * mxmxh.y + (xi - alpha) * mxh.y),
            s * ((1 + xi * alpha) * mxmxh.z + (xi - alpha) * mxh.z));
}

// Standard normal number of (seed, step, cell, component): splitmix64
// finaliser (Steele, Lea and Flood, OOPSLA 2014) of the combined counter, two
// 24-bit uniforms, Box-Muller.  The same step gives the same numbers in every
// stage and every retried attempt (the reference evaluates the noise once per
// step, core/rungekutta.cpp:94-98).
__device__ __forceinline__ float thermal_normal(unsigned long long seed, long long step, int i, int c) {
  unsigned long long z = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(step + 1));
  z += 0xD1B54A32D192ED03ull * (unsigned long long)(3 * (long long)i + c + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const float u1 = (float)((unsigned)(z >> 40) + 1u) * (1.0f / 16777216.0f);
  const float u2 = (float)(unsigned)(z & 0xFFFFFFull) * (1.0f / 16777216.0f);
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// physics/thermalnoise.cu:20-43: the thermal field of the step times 1/sqrt(dt)
// (added to every stage, core/rungekutta.cpp:100-106)
__device__ __noinline__ float3 thermal_term(const MagnetDev& M, int i, long long step, double dt) {
  const float ms = M.msat.at(i), T = M.temp.at(i), a = M.alpha.at(i);
  if (ms == 0.f || T == 0.f) return f3(0.f, 0.f, 0.f);
  const float s = sqrtf(M.noise_pref * a * T / ((1 + a * a) * ms)) * (float)(1.0 / sqrt(dt));
  return f3(s * thermal_normal(M.seed, step, i, 0), s * thermal_normal(M.seed, step, i, 1),
            s * thermal_normal(M.seed, step, i, 2));
}

// physics/torque.cu:58-76 (k_dampingtorque): the relax torque -gamma_LL m x (m x h)
__device__ __forceinline__ float3 damping_torque(float3 m, float3 h) {
  return (-GAMMA_LL) * cross3(m, cross3(m, h));
}

}  // namespace mpx
