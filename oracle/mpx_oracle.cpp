// mpx_oracle.cpp -- CPU FP64 oracle for the effective-field + Runge-Kutta path.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain, serial-per-cell (OpenMP over
// cells / FFT lines) restatement of the mumax+ algorithms in double precision.
// It is used by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg, and only as the checker -- never by the product library.
//
// Parity pins: tests/test_oracle_golden.py checks this oracle against the
// known-answer values held by the reference's own tests (analytic macrospin
// precession test/test_timesolver.py:19-29, PBC relaxation <m> from
// test/test_PBC.py:82-91, cube self-demag, numpy restatements of exchange /
// DMI / anisotropy / demag from test/test_exchange.py, test_interfacialdmi.py,
// test_anisotropy.py, test_demag.py) and FFT-vs-direct-sum demag
// (test/test_strayfield.py:57-84).
//
// Each function cites the reference file:line it restates (paths relative to
// the mumax-plus source tree).  The demag convolution uses its own radix-2 FFT
// on a power-of-two padded grid P >= 2n-1 with the kernel stored circularly
// (r = 0 at index 0); this is the same linear convolution as the reference's
// kernel-grid layout (physics/strayfieldkernel.cu:80-99, strayfieldfft.cu:75-100).

#include <cmath>
#include <deque>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../include/mpx.h"

namespace {

using cd = std::complex<double>;

constexpr double GAMMALL = 1.7595e11;       // physics/constants.hpp:24 (DOUBLE)
constexpr double MU0 = 1.25663706212e-6;    // physics/constants.hpp:26 (DOUBLE)
constexpr double QE = 1.60217646e-19;       // physics/constants.hpp:26-30 (DOUBLE)
constexpr double MUB = 9.2740091523e-24;
constexpr double HBAR = 1.054571817e-34;

thread_local std::string g_err;

struct V3 {
  double x = 0, y = 0, z = 0;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
// core/datatypes.hpp normalized(): zero vector stays zero
inline V3 normalized(V3 a) {
  double n = norm(a);
  double s = (n == 0.0) ? 0.0 : 1.0 / n;
  return s * a;
}

// core/datatypes.hpp harmonicMean
inline double harmonic_mean(double a, double b) {
  if (a + b == 0.0) return 0.0;
  if (a == b) return a;
  return 2 * a * b / (a + b);
}

// core/grid.hpp modulo
inline int modulo(int i, int d) {
  i %= d;
  return i >= 0 ? i : i + d;
}

struct Param {
  double u = 0;
  std::vector<double> cells;
  void load(const mpx_scalar& s, int n) {
    u = s.uniform;
    cells.clear();
    if (s.cells) cells.assign(s.cells, s.cells + n);
  }
  double at(int i) const { return cells.empty() ? u : cells[i]; }
  // core/parameter.cu assuredZero: uniform and zero
  bool zero() const { return cells.empty() && u == 0.0; }
};

struct VParam {
  double u[3] = {0, 0, 0};
  std::vector<double> cells;  // SoA
  int n = 0;
  void load(const mpx_vector& s, int ncells) {
    n = ncells;
    for (int c = 0; c < 3; ++c) u[c] = s.uniform[c];
    cells.clear();
    if (s.cells) cells.assign(s.cells, s.cells + 3 * (size_t)ncells);
  }
  V3 at(int i) const {
    if (cells.empty()) return {u[0], u[1], u[2]};
    return {cells[i], cells[(size_t)n + i], cells[2 * (size_t)n + i]};
  }
  bool zero() const { return cells.empty() && u[0] == 0 && u[1] == 0 && u[2] == 0; }
};

// ---------------------------------------------------------------- FFT (FP64)
// Twiddles exp(-2 pi i k / n), k < n/2, for one transform length.
const std::vector<cd>& twiddles(int n) {
  static thread_local std::vector<std::vector<cd>> cache(32);
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  std::vector<cd>& t = cache[lg];
  if ((int)t.size() != n / 2) {
    t.resize(n / 2);
    for (int k = 0; k < n / 2; ++k) t[k] = cd(std::cos(-2.0 * M_PI * k / n), std::sin(-2.0 * M_PI * k / n));
  }
  return t;
}

// Iterative radix-2 complex FFT, sign -1 forward, +1 inverse (unnormalised),
// on a contiguous copy of the (strided) line.
void fft1d(cd* a, int n, size_t stride, int sign) {
  if (n <= 1) return;
  static thread_local std::vector<cd> buf;
  buf.resize(n);
  for (int i = 0; i < n; ++i) buf[i] = a[(size_t)i * stride];
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(buf[i], buf[j]);
  }
  const std::vector<cd>& tw = twiddles(n);
  for (int len = 2; len <= n; len <<= 1) {
    const int step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < len / 2; ++k) {
        cd w = tw[(size_t)k * step];
        if (sign > 0) w = std::conj(w);
        cd u = buf[i + k];
        cd v = buf[i + k + len / 2] * w;
        buf[i + k] = u + v;
        buf[i + k + len / 2] = u - v;
      }
    }
  }
  for (int i = 0; i < n; ++i) a[(size_t)i * stride] = buf[i];
}

// 3-D FFT of a P[0] x P[1] x P[2] array (x fastest).  Lines that are known to
// be zero on input (forward: only y < n1, z < n2 rows and z < n2 planes hold
// data) or whose output is not needed (inverse: only y < n1, z < n2 is kept)
// are skipped; pass n = P to transform everything.
void fft3d(std::vector<cd>& a, const int P[3], int sign, const int n[3]) {
  const int px = P[0], py = P[1], pz = P[2];
  if (sign < 0) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n[2]; ++z)
      for (int y = 0; y < n[1]; ++y) fft1d(&a[((size_t)z * py + y) * px], px, 1, sign);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n[2]; ++z)
      for (int x = 0; x < px; ++x) fft1d(&a[(size_t)z * py * px + x], py, px, sign);
#pragma omp parallel for collapse(2) schedule(static)
    for (int y = 0; y < py; ++y)
      for (int x = 0; x < px; ++x) fft1d(&a[(size_t)y * px + x], pz, (size_t)px * py, sign);
  } else {
#pragma omp parallel for collapse(2) schedule(static)
    for (int y = 0; y < py; ++y)
      for (int x = 0; x < px; ++x) fft1d(&a[(size_t)y * px + x], pz, (size_t)px * py, sign);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n[2]; ++z)
      for (int x = 0; x < px; ++x) fft1d(&a[(size_t)z * py * px + x], py, px, sign);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n[2]; ++z)
      for (int y = 0; y < n[1]; ++y) fft1d(&a[((size_t)z * py + y) * px], px, 1, sign);
  }
}

int next_pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// ------------------------------------------------------------ Newell tensor
// physics/newell.cu:7-33 (Nxx indefinite integral, Newell et al. eq. 27)
double nxx_indef(int ix, int iy, int iz, double cx, double cy, double cz) {
  double x = ix * cx, y = iy * cy, z = iz * cz;
  double R = std::sqrt(x * x + y * y + z * z);
  double r = 0;
  if (ix != 0 || iz != 0) r += (y / 2) * (z * z - x * x) * std::asinh(y / std::sqrt(x * x + z * z));
  if (ix != 0 || iy != 0) r += (z / 2) * (y * y - x * x) * std::asinh(z / std::sqrt(x * x + y * y));
  if (ix != 0) r -= x * y * z * std::atan((y * z) / (x * R));
  r += (1. / 6.) * (2 * x * x - y * y - z * z) * R;
  return r;
}

// physics/newell.cu:35-63 (Nxy indefinite integral, eq. 32)
double nxy_indef(int ix, int iy, int iz, double cx, double cy, double cz) {
  if (iy == 0 || ix == 0) return 0.0;
  double x = ix * cx, y = iy * cy, z = iz * cz;
  double R = std::sqrt(x * x + y * y + z * z);
  double r = 0;
  r += (x * y * z) * std::asinh(z / std::sqrt(x * x + y * y));
  r += (y / 6) * (3 * z * z - y * y) * std::asinh(x / std::sqrt(y * y + z * z));
  r += (x / 6) * (3 * z * z - x * x) * std::asinh(y / std::sqrt(x * x + z * z));
  r -= (z * y * y / 2) * std::atan((x * z) / (y * R));
  r -= (z * x * x / 2) * std::atan((y * z) / (x * R));
  r -= x * y * R / 3;
  if (iz != 0) r -= (z * z * z / 6) * std::atan((x * y) / (z * R));
  return r;
}

// physics/newell.cu:65-82 weights of the 27-point combination
int newell_weight(int dx, int dy, int dz) {
  switch (dx * dx + dy * dy + dz * dz) {
    case 0: return 8;
    case 1: return -4;
    case 2: return 2;
    case 3: return -1;
    default: return 0;
  }
}

// physics/newell.cu:84-101
double newell_nxx(int ix, int iy, int iz, double cx, double cy, double cz) {
  double r = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz)
        r += newell_weight(dx, dy, dz) * nxx_indef(ix + dx, iy + dy, iz + dz, cx, cy, cz);
  return r / (4 * M_PI * cx * cy * cz);
}

// physics/newell.cu:103-120
double newell_nxy(int ix, int iy, int iz, double cx, double cy, double cz) {
  if (ix == 0 || iy == 0) return 0;
  double r = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz)
        r += newell_weight(dx, dy, dz) * nxy_indef(ix + dx, iy + dy, iz + dz, cx, cy, cz);
  return r / (4 * M_PI * cx * cy * cz);
}

// physics/newell.cu:122-138 component permutations; order xx,yy,zz,xy,xz,yz
void newell6(int x, int y, int z, double cx, double cy, double cz, double out[6]) {
  out[0] = newell_nxx(x, y, z, cx, cy, cz);
  out[1] = newell_nxx(y, z, x, cy, cz, cx);
  out[2] = newell_nxx(z, x, y, cz, cx, cy);
  out[3] = newell_nxy(x, y, z, cx, cy, cz);
  out[4] = newell_nxy(x, z, y, cx, cz, cy);
  out[5] = newell_nxy(y, z, x, cy, cz, cx);
}

// physics/strayfieldkernel.cu:25-56: sum over PBC images (FP64 here)
void kernel_at(int x, int y, int z, const int mg[3], const int pbc[3], const double cs[3],
               double out[6]) {
  for (int c = 0; c < 6; ++c) out[c] = 0;
  for (int i = -pbc[0]; i <= pbc[0]; ++i)
    for (int j = -pbc[1]; j <= pbc[1]; ++j)
      for (int k = -pbc[2]; k <= pbc[2]; ++k) {
        double v[6];
        newell6(x + i * mg[0], y + j * mg[1], z + k * mg[2], cs[0], cs[1], cs[2], v);
        for (int c = 0; c < 6; ++c) out[c] += v[c];
      }
}

// ------------------------------------------------------------------ magnet
struct Magnet {
  int n[3], o[3], mg[3], mgo[3], pbc[3];
  double cs[3];
  int N = 0;
  std::vector<uint8_t> geom;
  std::vector<uint32_t> reg;
  Param msat, aex, alpha, ku1, ku2, frozen;
  VParam anisU, bias;
  Param kc1, kc2, kc3;
  VParam anisC1, anisC2;
  Param pol, xi, lambda, epsp, flt;
  VParam jcur, fixl;
  bool fl_below = false, zl_off = false, sl_off = false;
  Param temp;
  uint64_t seed = 0;
  Param dmi[9];
  int lutn = 0;
  double inter_u = 0, scale_u = 1;
  std::vector<double> inter_lut, scale_lut;
  bool demag = true, openbc = false;
  std::vector<double> m;  // SoA 3N
  // demag spectrum on the power-of-two padded grid
  int P[3] = {1, 1, 1};
  std::vector<cd> khat[6];
  bool kready = false;
  std::vector<double> ext_oct;  // octant supplied by the caller (replaces kernel_octant when set)
  bool stray_src_off = false, stray_dst_off = false;  // Magnet::enableAsStrayFieldSource/Destination

  int idx(int x, int y, int z) const { return x + n[0] * (y + n[1] * z); }
  V3 mv(int i) const { return {m[i], m[(size_t)N + i], m[2 * (size_t)N + i]}; }
  bool in_grid_local(int x, int y, int z) const {
    return x >= 0 && x < n[0] && y >= 0 && y < n[1] && z >= 0 && z < n[2];
  }
  bool in_geom_local(int x, int y, int z) const {
    return in_grid_local(x, y, z) && (geom.empty() || geom[idx(x, y, z)]);
  }
  bool in_geom(int i) const { return geom.empty() || geom[i]; }
  // core/grid.hpp:73-81 Grid::wrap of the mastergrid, applied to global coords;
  // returns local coords
  void wrap_local(int& x, int& y, int& z) const {
    int g[3] = {x + o[0], y + o[1], z + o[2]};
    for (int a = 0; a < 3; ++a)
      if (mg[a] > 0) g[a] = mgo[a] + modulo(g[a] - mgo[a], mg[a]);
    x = g[0] - o[0];
    y = g[1] - o[1];
    z = g[2] - o[2];
  }
  unsigned region(int i) const { return reg.empty() ? 0u : reg[i]; }
  // core/inter_parameter.hpp:73-91 (LUT index i(i-1)/2+j)
  double lut_value(const std::vector<double>& lut, double u, unsigned i, unsigned j) const {
    if (lut.empty()) return u;
    int k = (i > j) ? (int)(i * (i - 1) / 2 + j) : (int)(j * (j - 1) / 2 + i);
    return lut[k];
  }
};

int load_magnet(Magnet& mg, const mpx_magnet_desc* d) {
  for (int a = 0; a < 3; ++a) {
    if (d->size[a] <= 0) { g_err = "grid size must be positive"; return MPX_ERR_INVALID; }
    mg.n[a] = d->size[a];
    mg.o[a] = d->origin[a];
    mg.stray_src_off = d->stray_source_off != 0;
    mg.stray_dst_off = d->stray_destination_off != 0;
    mg.mg[a] = d->mastergrid_size[a];
    mg.mgo[a] = d->mastergrid_origin[a];
    mg.pbc[a] = d->pbc_repetitions[a];
    mg.cs[a] = d->cellsize[a];
  }
  mg.N = mg.n[0] * mg.n[1] * mg.n[2];
  const int N = mg.N;
  mg.geom.clear();
  if (d->geometry) mg.geom.assign(d->geometry, d->geometry + N);
  mg.reg.clear();
  if (d->regions) mg.reg.assign(d->regions, d->regions + N);
  mg.msat.load(d->msat, N);
  mg.aex.load(d->aex, N);
  mg.alpha.load(d->alpha, N);
  mg.ku1.load(d->ku1, N);
  mg.ku2.load(d->ku2, N);
  mg.frozen.load(d->frozen_spins, N);
  mg.anisU.load(d->anis_u, N);
  mg.bias.load(d->bias_magnetic_field, N);
  mg.kc1.load(d->kc1, N);
  mg.kc2.load(d->kc2, N);
  mg.kc3.load(d->kc3, N);
  mg.anisC1.load(d->anis_c1, N);
  mg.anisC2.load(d->anis_c2, N);
  mg.pol.load(d->pol, N);
  mg.xi.load(d->xi, N);
  mg.lambda.load(d->lambda, N);
  mg.epsp.load(d->epsilon_prime, N);
  mg.flt.load(d->free_layer_thickness, N);
  mg.jcur.load(d->jcur, N);
  mg.fixl.load(d->fixed_layer, N);
  mg.fl_below = d->fixed_layer_below != 0;
  mg.zl_off = d->zhang_li_off != 0;
  mg.sl_off = d->slonczewski_off != 0;
  mg.temp.load(d->temperature, N);
  mg.seed = d->thermal_seed;
  for (int c = 0; c < 9; ++c) mg.dmi[c].load(d->dmi[c], N);
  mg.lutn = d->lut_regions;
  int L = mg.lutn * (mg.lutn - 1) / 2;
  mg.inter_u = d->inter_exchange;
  mg.scale_u = d->scale_exchange;
  mg.inter_lut.clear();
  mg.scale_lut.clear();
  if (d->inter_exchange_lut && L > 0) mg.inter_lut.assign(d->inter_exchange_lut, d->inter_exchange_lut + L);
  if (d->scale_exchange_lut && L > 0) mg.scale_lut.assign(d->scale_exchange_lut, d->scale_exchange_lut + L);
  mg.demag = d->enable_demag != 0;
  mg.openbc = d->enable_openbc != 0;
  if ((int)mg.m.size() != 3 * N) {
    mg.m.assign(3 * (size_t)N, 0.0);
    for (int i = 0; i < N; ++i) mg.m[i] = 1.0;
  }
  mg.kready = false;
  return MPX_OK;
}

// ---------------------------------------------------------------- physics
// physics/dmi.hpp:53-69 getGamma
V3 get_gamma(const Magnet& mg, int i, int nx, int ny, int nz, V3 m) {
  double Dxxz = mg.dmi[MPX_DMI_XXZ].at(i), Dxxy = mg.dmi[MPX_DMI_XXY].at(i);
  double Dxyz = mg.dmi[MPX_DMI_XYZ].at(i), Dyxz = mg.dmi[MPX_DMI_YXZ].at(i);
  double Dyxy = mg.dmi[MPX_DMI_YXY].at(i), Dyyz = mg.dmi[MPX_DMI_YYZ].at(i);
  double Dzxz = mg.dmi[MPX_DMI_ZXZ].at(i), Dzxy = mg.dmi[MPX_DMI_ZXY].at(i);
  double Dzyz = mg.dmi[MPX_DMI_ZYZ].at(i);
  return {-Dxxy * nx * m.y - Dxxz * nx * m.z - Dyxz * ny * m.z - Dzxy * nz * m.y - Dyxy * ny * m.y -
              Dzxz * nz * m.z,
          Dxxy * nx * m.x - Dzyz * nz * m.z + Dyxy * ny * m.x - Dxyz * nx * m.z + Dzxy * nz * m.x -
              Dyyz * ny * m.z,
          Dxxz * nx * m.x + Dyyz * ny * m.y + Dxyz * nx * m.y + Dyxz * ny * m.x + Dzxz * nz * m.x +
              Dzyz * nz * m.y};
}

const int REL[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

bool exchange_zero(const Magnet& mg) {  // physics/exchange.cu:14-18
  return (mg.aex.zero() && mg.inter_lut.empty() && mg.inter_u == 0) ||
         (mg.scale_lut.empty() && mg.scale_u == 0) || mg.msat.zero();
}
bool dmi_zero(const Magnet& mg) {  // physics/dmi.cu:12-17
  if (mg.msat.zero()) return true;
  for (int c = 0; c < 9; ++c)
    if (!mg.dmi[c].zero()) return false;
  return true;
}
bool uni_zero(const Magnet& mg) {  // physics/anisotropy.cu:9-12
  return (mg.ku1.zero() && mg.ku2.zero()) || mg.anisU.zero() || mg.msat.zero();
}
bool cubic_zero(const Magnet& mg) {  // physics/anisotropy.cu:14-18
  return (mg.kc1.zero() && mg.kc2.zero() && mg.kc3.zero()) || (mg.anisC1.zero() && mg.anisC2.zero()) ||
         mg.msat.zero();
}
bool anis_zero(const Magnet& mg) { return uni_zero(mg) && cubic_zero(mg); }  // :20-23
bool external_zero(const Magnet& mg, const double wb[3]) {  // physics/zeeman.cu:37-51
  return wb[0] == 0 && wb[1] == 0 && wb[2] == 0 && mg.bias.zero();
}
bool demag_zero(const Magnet& mg) { return !mg.demag || mg.msat.zero(); }  // demag.cpp:9-11

// physics/exchange.cu:20-104 (FM kernel)
void exchange_field(const Magnet& mg, std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (exchange_zero(mg)) return;
  const double w[3] = {1 / (mg.cs[0] * mg.cs[0]), 1 / (mg.cs[1] * mg.cs[1]), 1 / (mg.cs[2] * mg.cs[2])};
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i)) continue;
    if (mg.msat.at(i) == 0) continue;
    int x = i % mg.n[0], y = (i / mg.n[0]) % mg.n[1], z = i / (mg.n[0] * mg.n[1]);
    V3 m = mg.mv(i);
    double a = mg.aex.at(i);
    V3 hh;
    for (int r = 0; r < 6; ++r) {
      int xx = x + REL[r][0], yy = y + REL[r][1], zz = z + REL[r][2];
      mg.wrap_local(xx, yy, zz);
      bool nin = mg.in_geom_local(xx, yy, zz);
      if (!nin && mg.openbc) continue;
      int j = nin ? mg.idx(xx, yy, zz) : -1;
      if (!(!mg.openbc || mg.msat.at(j) != 0)) continue;
      int nrm[3] = {REL[r][0] * REL[r][0], REL[r][1] * REL[r][1], REL[r][2] * REL[r][2]};
      double inter = 0, scale = 1, a_;
      V3 m_;
      if (nin) {
        m_ = mg.mv(j);
        a_ = mg.aex.at(j);
        unsigned ri = mg.region(i), rj = mg.region(j);
        if (ri != rj) {
          scale = mg.lut_value(mg.scale_lut, mg.scale_u, ri, rj);
          inter = mg.lut_value(mg.inter_lut, mg.inter_u, ri, rj);
        }
      } else {  // Neumann BC
        if (a == 0) continue;
        V3 G = get_gamma(mg, i, nrm[0], nrm[1], nrm[2], m);
        double delta = REL[r][0] * mg.cs[0] + REL[r][1] * mg.cs[1] + REL[r][2] * mg.cs[2];
        m_ = m + (delta / (2 * a)) * G;
        a_ = a;
      }
      double A = (inter != 0) ? inter : harmonic_mean(a, a_);
      A *= scale;
      double wd = nrm[0] * w[0] + nrm[1] * w[1] + nrm[2] * w[2];
      hh = hh + (2 * A * wd) * (m_ - m);
    }
    hh = hh / mg.msat.at(i);
    h[i] = hh.x;
    h[(size_t)N + i] = hh.y;
    h[2 * (size_t)N + i] = hh.z;
  }
}

// physics/dmi.cu:19-110 (FM kernel)
void dmi_field(const Magnet& mg, std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (dmi_zero(mg)) return;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i) || mg.msat.at(i) == 0) continue;
    int x = i % mg.n[0], y = (i / mg.n[0]) % mg.n[1], z = i / (mg.n[0] * mg.n[1]);
    V3 m = mg.mv(i);
    V3 hh;
    double a = mg.aex.at(i);
    bool open = (a == 0) ? true : mg.openbc;
    for (int r = 0; r < 6; ++r) {
      int xx = x + REL[r][0], yy = y + REL[r][1], zz = z + REL[r][2];
      mg.wrap_local(xx, yy, zz);
      bool nin = mg.in_geom_local(xx, yy, zz);
      int j = nin ? mg.idx(xx, yy, zz) : i;
      if (open && (!nin || mg.msat.at(j) == 0)) continue;
      auto hm = [&](int c) {  // CuParameter::harmonicMean (core/parameter.hpp:107-110)
        return (i == j) ? mg.dmi[c].at(i) : harmonic_mean(mg.dmi[c].at(i), mg.dmi[c].at(j));
      };
      double Dxz, Dxy, Dyz;
      if (REL[r][0]) {
        Dxz = hm(MPX_DMI_XXZ); Dxy = hm(MPX_DMI_XXY); Dyz = hm(MPX_DMI_XYZ);
      } else if (REL[r][1]) {
        Dxz = hm(MPX_DMI_YXZ); Dxy = hm(MPX_DMI_YXY); Dyz = hm(MPX_DMI_YYZ);
      } else {
        Dxz = hm(MPX_DMI_ZXZ); Dxy = hm(MPX_DMI_ZXY); Dyz = hm(MPX_DMI_ZYZ);
      }
      double Dzx = -Dxz, Dyx = -Dxy, Dzy = -Dyz;
      double delta = REL[r][0] * mg.cs[0] + REL[r][1] * mg.cs[1] + REL[r][2] * mg.cs[2];
      V3 m_;
      if (!nin && !open) {
        V3 G = get_gamma(mg, i, REL[r][0] * REL[r][0], REL[r][1] * REL[r][1], REL[r][2] * REL[r][2], m);
        m_ = m + (delta / (2 * a)) * G;
      } else {
        m_ = mg.mv(j);
      }
      hh.x += (Dxy * m_.y + Dxz * m_.z) / delta;
      hh.y += (Dyx * m_.x + Dyz * m_.z) / delta;
      hh.z += (Dzx * m_.x + Dzy * m_.y) / delta;
    }
    hh = hh / mg.msat.at(i);
    h[i] = hh.x;
    h[(size_t)N + i] = hh.y;
    h[2 * (size_t)N + i] = hh.z;
  }
}

// physics/anisotropy.cu:25-55 (uniaxial)
void anisotropy_field(const Magnet& mg, std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (anis_zero(mg)) return;
  const bool cubic = uni_zero(mg);  // uniaxial takes precedence (physics/anisotropy.cu:121-138)
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i) || mg.msat.at(i) == 0) continue;
    if (cubic) {  // physics/anisotropy.cu:57-106
      V3 c1 = normalized(mg.anisC1.at(i)), c2 = normalized(mg.anisC2.at(i)), c3 = cross(c1, c2), m = mg.mv(i);
      double k1 = mg.kc1.at(i), k2 = mg.kc2.at(i), k3 = mg.kc3.at(i), Ms = mg.msat.at(i);
      double a = dot(c1, m), b = dot(c2, m), c = dot(c3, m);
      V3 hh = (-2 * k1 / Ms) * ((b * b + c * c) * a * c1 + (a * a + c * c) * b * c2 + (a * a + b * b) * c * c3) +
              (-2 * k2 / Ms) * ((b * b * c * c) * a * c1 + (a * a * c * c) * b * c2 + (a * a * b * b) * c * c3) +
              (-4 * k3 / Ms) * ((std::pow(b, 4) + std::pow(c, 4)) * std::pow(a, 3) * c1 +
                                (std::pow(a, 4) + std::pow(c, 4)) * std::pow(b, 3) * c2 +
                                (std::pow(a, 4) + std::pow(b, 4)) * std::pow(c, 3) * c3);
      h[i] = hh.x;
      h[(size_t)N + i] = hh.y;
      h[2 * (size_t)N + i] = hh.z;
      continue;
    }
    V3 u = normalized(mg.anisU.at(i));
    V3 m = mg.mv(i);
    double k1 = mg.ku1.at(i), k2 = mg.ku2.at(i), Ms = mg.msat.at(i);
    double mu = dot(m, u);
    V3 hh = ((2 * k1 * mu + 4 * k2 * mu * mu * mu) / Ms) * u;
    h[i] = hh.x;
    h[(size_t)N + i] = hh.y;
    h[2 * (size_t)N + i] = hh.z;
  }
}

// physics/zeeman.cu:53-91 (world bias everywhere, magnet bias inside the geometry)
void external_field(const Magnet& mg, const double wb[3], std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (external_zero(mg, wb)) return;
  for (int i = 0; i < N; ++i) {
    V3 b{wb[0], wb[1], wb[2]};
    if (mg.in_geom(i) && !mg.bias.zero()) b = b + mg.bias.at(i);
    h[i] = b.x;
    h[(size_t)N + i] = b.y;
    h[2 * (size_t)N + i] = b.z;
  }
}

// Demag kernel on the octant |r_a| < n_a, summed over the PBC images.  For each
// image and component the indefinite integral is evaluated once per lattice
// point of the (n+2)^3 box and shared by the 27-point combinations of all
// displacements (the same weighted sum as physics/newell.cu:84-120, each term
// computed once instead of up to 27 times).  Components follow the
// permutations of physics/newell.cu:122-138.
void kernel_octant(const int n[3], const int mgs[3], const int pbc[3], const double cs[3],
                   std::vector<double>& oct) {
  const size_t noct = (size_t)n[0] * n[1] * n[2];
  oct.assign(6 * noct, 0.0);
  const int L0 = n[0] + 2, L1 = n[1] + 2, L2 = n[2] + 2;
  std::vector<double> lat((size_t)L0 * L1 * L2);
  // permutation of (x, y, z) and type (0: xx-like, 1: xy-like) per component
  const int perm[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  const int type[6] = {0, 0, 0, 1, 1, 1};
  for (int ii = -pbc[0]; ii <= pbc[0]; ++ii)
    for (int jj = -pbc[1]; jj <= pbc[1]; ++jj)
      for (int kk = -pbc[2]; kk <= pbc[2]; ++kk) {
        const int s[3] = {ii * mgs[0], jj * mgs[1], kk * mgs[2]};
        for (int c = 0; c < 6; ++c) {
          const int* p = perm[c];
          const double pcs[3] = {cs[p[0]], cs[p[1]], cs[p[2]]};
#pragma omp parallel for collapse(2) schedule(static)
          for (int cz = 0; cz < L2; ++cz)
            for (int cy = 0; cy < L1; ++cy)
              for (int cx = 0; cx < L0; ++cx) {
                const int q[3] = {cx - 1 + s[0], cy - 1 + s[1], cz - 1 + s[2]};
                const double v = type[c] == 0 ? nxx_indef(q[p[0]], q[p[1]], q[p[2]], pcs[0], pcs[1], pcs[2])
                                              : nxy_indef(q[p[0]], q[p[1]], q[p[2]], pcs[0], pcs[1], pcs[2]);
                lat[((size_t)cz * L1 + cy) * L0 + cx] = v;
              }
          const double norm = 4 * M_PI * pcs[0] * pcs[1] * pcs[2];
#pragma omp parallel for collapse(2) schedule(static)
          for (int rz = 0; rz < n[2]; ++rz)
            for (int ry = 0; ry < n[1]; ++ry)
              for (int rx = 0; rx < n[0]; ++rx) {
                const int rr[3] = {rx + s[0], ry + s[1], rz + s[2]};
                if (type[c] == 1 && (rr[p[0]] == 0 || rr[p[1]] == 0)) continue;  // Nxy == 0 exactly
                double sum = 0;
                for (int dx = -1; dx <= 1; ++dx)
                  for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz)
                      sum += newell_weight(dx, dy, dz) *
                             lat[((size_t)(rz + dz + 1) * L1 + (ry + dy + 1)) * L0 + (rx + dx + 1)];
                oct[c * noct + ((size_t)rz * n[1] + ry) * n[0] + rx] += sum / norm;
              }
        }
      }
}

void build_demag_kernel(Magnet& mg) {
  for (int a = 0; a < 3; ++a) mg.P[a] = (mg.n[a] == 1) ? 1 : next_pow2_at_least(2 * mg.n[a] - 1);
  const int px = mg.P[0], py = mg.P[1], pz = mg.P[2];
  const size_t PP = (size_t)px * py * pz;
  std::vector<double> oct;
  if (!mg.ext_oct.empty())
    oct = mg.ext_oct;
  else
    kernel_octant(mg.n, mg.mg, mg.pbc, mg.cs, oct);
  const size_t noct = (size_t)mg.n[0] * mg.n[1] * mg.n[2];
  auto rel = [](int i, int P, int n) -> int {  // circular index -> displacement, or INT32_MIN if unused
    if (i <= n - 1) return i;
    if (i >= P - (n - 1)) return i - P;
    return INT32_MIN;
  };
  // parity: xy odd in x,y; xz odd in x,z; yz odd in y,z; diagonal even
  const int odd[6][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
  for (int c = 0; c < 6; ++c) {
    mg.khat[c].assign(PP, cd(0, 0));
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < pz; ++k)
      for (int j = 0; j < py; ++j)
        for (int i = 0; i < px; ++i) {
          const int r[3] = {rel(i, px, mg.n[0]), rel(j, py, mg.n[1]), rel(k, pz, mg.n[2])};
          if (r[0] == INT32_MIN || r[1] == INT32_MIN || r[2] == INT32_MIN) continue;
          double v = oct[c * noct + ((size_t)std::abs(r[2]) * mg.n[1] + std::abs(r[1])) * mg.n[0] + std::abs(r[0])];
          for (int a = 0; a < 3; ++a)
            if (odd[c][a] && r[a] < 0) v = -v;
          mg.khat[c][((size_t)k * py + j) * px + i] = v;
        }
    const int full[3] = {px, py, pz};
    fft3d(mg.khat[c], mg.P, -1, full);
  }
  mg.kready = true;
}

// physics/strayfieldfft.cu:191-246: B = -mu0 * N (*) (Ms m), zero outside geometry
void demag_field(Magnet& mg, std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (demag_zero(mg)) return;
  if (!mg.kready) build_demag_kernel(mg);
  const int px = mg.P[0], py = mg.P[1], pz = mg.P[2];
  const size_t PP = (size_t)px * py * pz;
  std::vector<cd> M[3];
  for (int c = 0; c < 3; ++c) {
    M[c].assign(PP, cd(0, 0));
    for (int z = 0; z < mg.n[2]; ++z)
      for (int y = 0; y < mg.n[1]; ++y)
        for (int x = 0; x < mg.n[0]; ++x) {
          int i = mg.idx(x, y, z);
          if (!mg.in_geom(i)) continue;
          M[c][((size_t)z * py + y) * px + x] = mg.msat.at(i) * mg.m[(size_t)c * N + i];
        }
    fft3d(M[c], mg.P, -1, mg.n);
  }
  // order xx,yy,zz,xy,xz,yz
#pragma omp parallel for schedule(static)
  for (long long q = 0; q < (long long)PP; ++q) {
    cd mx = M[0][q], my = M[1][q], mz = M[2][q];
    cd kxx = mg.khat[0][q], kyy = mg.khat[1][q], kzz = mg.khat[2][q];
    cd kxy = mg.khat[3][q], kxz = mg.khat[4][q], kyz = mg.khat[5][q];
    M[0][q] = kxx * mx + kxy * my + kxz * mz;
    M[1][q] = kxy * mx + kyy * my + kyz * mz;
    M[2][q] = kxz * mx + kyz * my + kzz * mz;
  }
  const double pref = -MU0 / (double)PP;
  for (int c = 0; c < 3; ++c) {
    fft3d(M[c], mg.P, +1, mg.n);
    for (int z = 0; z < mg.n[2]; ++z)
      for (int y = 0; y < mg.n[1]; ++y)
        for (int x = 0; x < mg.n[0]; ++x) {
          int i = mg.idx(x, y, z);
          if (!mg.in_geom(i)) continue;
          h[(size_t)c * N + i] = pref * M[c][((size_t)z * py + y) * px + x].real();
        }
  }
}

// physics/strayfieldbrute.cu:15-57: direct O(N^2) sum (cross-check only)
void demag_brute(const Magnet& mg, std::vector<double>& h) {
  const int N = mg.N;
  h.assign(3 * (size_t)N, 0.0);
  if (demag_zero(mg)) return;
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i)) continue;
    int x = i % mg.n[0], y = (i / mg.n[0]) % mg.n[1], z = i / (mg.n[0] * mg.n[1]);
    V3 hh;
    for (int s = 0; s < N; ++s) {
      if (!mg.in_geom(s)) continue;
      int sx = s % mg.n[0], sy = (s / mg.n[0]) % mg.n[1], sz = s / (mg.n[0] * mg.n[1]);
      double k[6];
      kernel_at(x - sx, y - sy, z - sz, mg.mg, mg.pbc, mg.cs, k);
      V3 M = mg.msat.at(s) * mg.mv(s);
      hh.x -= k[0] * M.x + k[3] * M.y + k[4] * M.z;
      hh.y -= k[3] * M.x + k[1] * M.y + k[5] * M.z;
      hh.z -= k[4] * M.x + k[5] * M.y + k[2] * M.z;
    }
    h[i] = MU0 * hh.x;
    h[(size_t)N + i] = MU0 * hh.y;
    h[2 * (size_t)N + i] = MU0 * hh.z;
  }
}

struct World {
  std::vector<Magnet> mags;
  double wb[3] = {0, 0, 0};
  mpx_solver_params sp{MPX_RK_FEHLBERG, 1, 1e-5, 0.8, 0.5, 2.0, 0.01, 1e-14};
  double t = 0, dt = 0;
  int64_t steps = 0, rejected = 0, evals = 0;
  bool relax_torque = false;  // the equations use the damping torque (physics/relaxer.cpp)
};

// physics/zeeman.cu:70-88: the destination receives the stray field of every
// other enabled source of its world
bool has_stray(const World& w, const Magnet& dst) {
  if (dst.stray_dst_off) return false;
  for (const Magnet& src : w.mags)
    if (&src != &dst && !src.stray_src_off && !src.msat.zero()) return true;
  return false;
}

// physics/strayfieldbrute.cu:15-57: B(r) = -mu0 sum_{r' in src} N(r - r') Ms m(r'),
// r, r' world cell coordinates, the tensor (with PBC images) tabulated over the
// displacements of the two grids; zero outside the destination's geometry.
void add_stray(const World& w, const Magnet& dst, std::vector<double>& h) {
  if (dst.stray_dst_off) return;
  const int NB = dst.N;
  for (const Magnet& src : w.mags) {
    if (&src == &dst || src.stray_src_off || src.msat.zero()) continue;
    int K[3], O[3];
    for (int a = 0; a < 3; ++a) {
      K[a] = src.n[a] + dst.n[a] - 1;
      O[a] = dst.o[a] - src.o[a] - (src.n[a] - 1);
    }
    const size_t KK = (size_t)K[0] * K[1] * K[2];
    std::vector<double> tab(6 * KK);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = 0; k < K[2]; ++k)
      for (int j = 0; j < K[1]; ++j)
        for (int i = 0; i < K[0]; ++i) {
          double v[6];
          kernel_at(O[0] + i, O[1] + j, O[2] + k, dst.mg, dst.pbc, dst.cs, v);
          const size_t p = ((size_t)k * K[1] + j) * K[0] + i;
          for (int c = 0; c < 6; ++c) tab[c * KK + p] = v[c];
        }
    const int NA = src.N;
#pragma omp parallel for schedule(static)
    for (int ib = 0; ib < NB; ++ib) {
      if (!dst.in_geom(ib)) continue;
      const int bx = ib % dst.n[0], by = (ib / dst.n[0]) % dst.n[1], bz = ib / (dst.n[0] * dst.n[1]);
      double hx = 0, hy = 0, hz = 0;
      for (int ia = 0; ia < NA; ++ia) {
        if (!src.in_geom(ia)) continue;
        const int ax = ia % src.n[0], ay = (ia / src.n[0]) % src.n[1], az = ia / (src.n[0] * src.n[1]);
        const size_t p = ((size_t)(dst.o[2] + bz - src.o[2] - az - O[2]) * K[1] +
                          (dst.o[1] + by - src.o[1] - ay - O[1])) * K[0] +
                         (dst.o[0] + bx - src.o[0] - ax - O[0]);
        const double ms = src.msat.at(ia);
        const V3 M = ms * src.mv(ia);
        const double nxx = tab[p], nyy = tab[KK + p], nzz = tab[2 * KK + p];
        const double nxy = tab[3 * KK + p], nxz = tab[4 * KK + p], nyz = tab[5 * KK + p];
        hx -= nxx * M.x + nxy * M.y + nxz * M.z;
        hy -= nxy * M.x + nyy * M.y + nyz * M.z;
        hz -= nxz * M.x + nyz * M.y + nzz * M.z;
      }
      h[ib] += MU0 * hx;
      h[(size_t)NB + ib] += MU0 * hy;
      h[2 * (size_t)NB + ib] += MU0 * hz;
    }
  }
}

bool ext_zero(const World& w, const Magnet& mg) { return external_zero(mg, w.wb) && !has_stray(w, mg); }
void ext_field(const World& w, const Magnet& mg, std::vector<double>& h) {
  external_field(mg, w.wb, h);
  add_stray(w, mg, h);
}

// physics/effectivefield.cpp:15-28 (terms added in this order)
void effective_field(World& w, Magnet& mg, std::vector<double>& h) {
  const size_t n3 = 3 * (size_t)mg.N;
  h.assign(n3, 0.0);
  std::vector<double> t;
  auto add = [&](const std::vector<double>& f) {
    for (int i = 0; i < mg.N; ++i) {
      if (!mg.in_geom(i)) continue;  // core/fieldops.cu:9-22 adds inside the geometry only
      for (int c = 0; c < 3; ++c) h[(size_t)c * mg.N + i] += f[(size_t)c * mg.N + i];
    }
  };
  if (!exchange_zero(mg)) { exchange_field(mg, t); add(t); }
  if (!anis_zero(mg)) { anisotropy_field(mg, t); add(t); }
  if (!ext_zero(w, mg)) { ext_field(w, mg, t); add(t); }
  if (!dmi_zero(mg)) { dmi_field(mg, t); add(t); }
  if (!demag_zero(mg)) { demag_field(mg, t); add(t); }
}

// physics/stt.cu:9-24
bool zl_zero(const Magnet& mg) { return mg.zl_off || mg.msat.zero() || mg.jcur.zero() || mg.pol.zero(); }
bool sl_zero(const Magnet& mg) {
  return mg.sl_off || mg.msat.zero() || mg.jcur.zero() || mg.flt.zero() || mg.fixl.zero() ||
         (mg.epsp.zero() && (mg.lambda.zero() || mg.pol.zero()));
}

// physics/stt.cu:26-185: spin-transfer torque, Slonczewski unless assured zero, else Zhang-Li
void stt_torque(const Magnet& mg, std::vector<double>& tq) {
  const int N = mg.N;
  tq.assign(3 * (size_t)N, 0.0);
  const bool sl = !sl_zero(mg), zl = !zl_zero(mg);
  if (!sl && !zl) return;
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i) || mg.frozen.at(i) != 0) continue;
    const V3 m = mg.mv(i);
    const double ms = mg.msat.at(i), alpha = mg.alpha.at(i);
    V3 t{0, 0, 0};
    if (sl) {
      const double jz = mg.jcur.at(i).z, pol = mg.pol.at(i), lambda = mg.lambda.at(i), eps_p = mg.epsp.at(i);
      const V3 p = mg.fixl.at(i);
      double d = mg.flt.at(i);
      if (mg.fl_below) d = -d;
      if (ms == 0 || jz == 0 || d == 0 || (p.x == 0 && p.y == 0 && p.z == 0) ||
          (eps_p == 0 && (lambda == 0 || pol == 0)))
        continue;
      const double B = (HBAR / QE) * jz / (ms * d);
      const double l2 = lambda * lambda;
      const double eps = pol * l2 / ((l2 + 1) + (l2 - 1) * dot(m, p));
      const V3 pxm = cross(p, m), mxpxm = cross(m, pxm);
      t = ((B / (1 + alpha * alpha)) * GAMMALL) * ((eps + eps_p * alpha) * mxpxm + (eps_p - eps * alpha) * pxm);
    } else {
      const V3 j = mg.jcur.at(i);
      const double pol = mg.pol.at(i), xi = mg.xi.at(i);
      if (ms == 0 || pol == 0 || (j.x == 0 && j.y == 0 && j.z == 0)) continue;
      const double cu = MUB * pol / (QE * ms * (1 + xi * xi));
      const double u[3] = {cu * j.x, cu * j.y, cu * j.z};
      const int x = i % mg.n[0], y = (i / mg.n[0]) % mg.n[1], z = i / (mg.n[0] * mg.n[1]);
      V3 hs{0, 0, 0};
      for (int axis = 0; axis < 3; ++axis)
        for (int sg = -1; sg <= 1; sg += 2) {
          int xx = x + (axis == 0 ? sg : 0), yy = y + (axis == 1 ? sg : 0), zz = z + (axis == 2 ? sg : 0);
          mg.wrap_local(xx, yy, zz);
          if (!mg.in_grid_local(xx, yy, zz)) continue;
          const int jn = mg.idx(xx, yy, zz);
          if (mg.msat.at(jn) == 0) continue;
          hs = hs + (sg * u[axis] / (2 * mg.cs[axis])) * mg.mv(jn);
        }
      const V3 mxh = cross(m, hs), mxmxh = cross(m, mxh);
      t = (-1 / (1 + alpha * alpha)) * ((1 + xi * alpha) * mxmxh + (xi - alpha) * mxh);
    }
    tq[i] = t.x;
    tq[(size_t)N + i] = t.y;
    tq[2 * (size_t)N + i] = t.z;
  }
}

// physics/torque.cu:21-45 (LLG) and :58-77 (damping only)
void torque(World& w, Magnet& mg, std::vector<double>& tq, bool damping_only = false, bool with_stt = true) {
  std::vector<double> h;
  effective_field(w, mg, h);
  const int N = mg.N;
  tq.assign(3 * (size_t)N, 0.0);
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i) || mg.frozen.at(i) != 0) continue;
    V3 m = mg.mv(i), b{h[i], h[(size_t)N + i], h[2 * (size_t)N + i]};
    V3 mxh = cross(m, b), mxmxh = cross(m, mxh);
    V3 t;
    if (damping_only) {
      t = (-GAMMALL) * mxmxh;
    } else {
      double a = mg.alpha.at(i);
      t = (-GAMMALL / (1 + a * a)) * (mxh + a * mxmxh);
    }
    tq[i] = t.x;
    tq[(size_t)N + i] = t.y;
    tq[2 * (size_t)N + i] = t.z;
  }
  if (!damping_only && with_stt && (!zl_zero(mg) || !sl_zero(mg))) {  // total torque = LLG + STT (torque.cu:78-90)
    std::vector<double> s;
    stt_torque(mg, s);
    for (size_t k = 0; k < tq.size(); ++k) tq[k] += s[k];
  }
  w.evals++;
}

void energy_density(World& w, Magnet& mg, int q, std::vector<double>& e) {
  const int N = mg.N;
  e.assign(N, 0.0);
  std::vector<double> h;
  auto from_field = [&](double pref) {  // physics/energy.cu:18-35
    for (int i = 0; i < N; ++i) {
      if (!mg.in_geom(i)) continue;
      V3 m = mg.mv(i), b{h[i], h[(size_t)N + i], h[2 * (size_t)N + i]};
      e[i] = -pref * mg.msat.at(i) * dot(m, b);
    }
  };
  switch (q) {
    case MPX_Q_EXCHANGE_ENERGY_DENSITY:
      if (exchange_zero(mg)) return;
      exchange_field(mg, h); from_field(0.5); return;
    case MPX_Q_DMI_ENERGY_DENSITY:
      if (dmi_zero(mg)) return;
      dmi_field(mg, h); from_field(0.5); return;
    case MPX_Q_ZEEMAN_ENERGY_DENSITY:
      if (ext_zero(w, mg)) return;
      ext_field(w, mg, h); from_field(1.0); return;
    case MPX_Q_DEMAG_ENERGY_DENSITY:
      if (demag_zero(mg)) return;
      demag_field(mg, h); from_field(0.5); return;
    case MPX_Q_ANISOTROPY_ENERGY_DENSITY:  // physics/anisotropy.cu:142-173
      if (anis_zero(mg)) return;
      for (int i = 0; i < N; ++i) {
        if (!mg.in_geom(i) || mg.msat.at(i) == 0) continue;
        if (uni_zero(mg)) {  // physics/anisotropy.cu:175-215 (cubic)
          V3 c1 = normalized(mg.anisC1.at(i)), c2 = normalized(mg.anisC2.at(i)), c3 = cross(c1, c2), m = mg.mv(i);
          double a2 = std::pow(dot(c1, m), 2), b2 = std::pow(dot(c2, m), 2), c2_ = std::pow(dot(c3, m), 2);
          e[i] = mg.kc1.at(i) * (a2 * b2 + a2 * c2_ + b2 * c2_) + mg.kc2.at(i) * a2 * b2 * c2_ +
                 mg.kc3.at(i) * (a2 * a2 * b2 * b2 + a2 * a2 * c2_ * c2_ + b2 * b2 * c2_ * c2_);
          continue;
        }
        V3 u = normalized(mg.anisU.at(i));
        double mu = dot(mg.mv(i), u), k1 = mg.ku1.at(i), k2 = mg.ku2.at(i);
        e[i] = -k1 * mu * mu - k2 * mu * mu * mu * mu;
      }
      return;
    case MPX_Q_TOTAL_ENERGY_DENSITY: {  // physics/energy.cu:37-56
      std::vector<double> t;
      for (int qq : {MPX_Q_EXCHANGE_ENERGY_DENSITY, MPX_Q_ANISOTROPY_ENERGY_DENSITY,
                     MPX_Q_ZEEMAN_ENERGY_DENSITY, MPX_Q_DMI_ENERGY_DENSITY, MPX_Q_DEMAG_ENERGY_DENSITY}) {
        energy_density(w, mg, qq, t);
        for (int i = 0; i < N; ++i)
          if (mg.in_geom(i)) e[i] += t[i];
      }
      return;
    }
  }
}

// ------------------------------------------------------- Butcher tableaus
// core/butchertableau.cpp (Heun, Bogacki-Shampine, Fehlberg, Cash-Karp, Dormand-Prince)
struct Tableau {
  int S, order1, order2;
  double c[7], a[7][7], b1[7], b2[7];
};

Tableau tableau(int method) {
  Tableau t{};
  switch (method) {
    case MPX_RK_HEUN:
      t.S = 2; t.order1 = 2; t.order2 = 1;
      t.c[1] = 1; t.a[1][0] = 1;
      t.b1[0] = 0.5; t.b1[1] = 0.5; t.b2[0] = 1; t.b2[1] = 0;
      break;
    case MPX_RK_BOGACKI_SHAMPINE:
      t.S = 4; t.order1 = 3; t.order2 = 2;
      t.c[1] = 0.5; t.c[2] = 0.75; t.c[3] = 1;
      t.a[1][0] = 0.5; t.a[2][1] = 0.75;
      t.a[3][0] = 2. / 9; t.a[3][1] = 1. / 3; t.a[3][2] = 4. / 9;
      t.b1[0] = 2. / 9; t.b1[1] = 1. / 3; t.b1[2] = 4. / 9; t.b1[3] = 0;
      t.b2[0] = 7. / 24; t.b2[1] = 1. / 4; t.b2[2] = 1. / 3; t.b2[3] = 1. / 8;
      break;
    case MPX_RK_FEHLBERG:
      t.S = 6; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 4; t.c[2] = 3. / 8; t.c[3] = 12. / 13; t.c[4] = 1; t.c[5] = 1. / 2;
      t.a[1][0] = 1. / 4;
      t.a[2][0] = 3. / 32; t.a[2][1] = 9. / 32;
      t.a[3][0] = 1932. / 2197; t.a[3][1] = -7200. / 2197; t.a[3][2] = 7296. / 2197;
      t.a[4][0] = 439. / 216; t.a[4][1] = -8; t.a[4][2] = 3680. / 513; t.a[4][3] = -845. / 4104;
      t.a[5][0] = -8. / 27; t.a[5][1] = 2; t.a[5][2] = -3544. / 2565; t.a[5][3] = 1859. / 4104;
      t.a[5][4] = -11. / 40;
      t.b1[0] = 16. / 135; t.b1[2] = 6656. / 12825; t.b1[3] = 28561. / 56430; t.b1[4] = -9. / 50;
      t.b1[5] = 2. / 55;
      t.b2[0] = 25. / 216; t.b2[2] = 1408. / 2565; t.b2[3] = 2197. / 4104; t.b2[4] = -1. / 5;
      break;
    case MPX_RK_CASH_KARP:
      t.S = 6; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 5; t.c[2] = 3. / 10; t.c[3] = 3. / 5; t.c[4] = 1; t.c[5] = 7. / 8;
      t.a[1][0] = 1. / 5;
      t.a[2][0] = 3. / 40; t.a[2][1] = 9. / 40;
      t.a[3][0] = 3. / 10; t.a[3][1] = -9. / 10; t.a[3][2] = 6. / 5;
      t.a[4][0] = -11. / 54; t.a[4][1] = 5. / 2; t.a[4][2] = -70. / 27; t.a[4][3] = 35. / 27;
      t.a[5][0] = 1631. / 55296; t.a[5][1] = 175. / 512; t.a[5][2] = 575. / 13824;
      t.a[5][3] = 44275. / 110592; t.a[5][4] = 253. / 4096;
      t.b1[0] = 37. / 378; t.b1[2] = 250. / 621; t.b1[3] = 125. / 594; t.b1[5] = 512. / 1771;
      t.b2[0] = 2825. / 27648; t.b2[2] = 18575. / 48384; t.b2[3] = 13525. / 55296;
      t.b2[4] = 277. / 14336; t.b2[5] = 1. / 4;
      break;
    default:  // MPX_RK_DORMAND_PRINCE
      t.S = 7; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 5; t.c[2] = 3. / 10; t.c[3] = 4. / 5; t.c[4] = 8. / 9; t.c[5] = 1; t.c[6] = 1;
      t.a[1][0] = 1. / 5;
      t.a[2][0] = 3. / 40; t.a[2][1] = 9. / 40;
      t.a[3][0] = 44. / 45; t.a[3][1] = -56. / 15; t.a[3][2] = 32. / 9;
      t.a[4][0] = 19372. / 6561; t.a[4][1] = -25360. / 2187; t.a[4][2] = 64448. / 6561;
      t.a[4][3] = -212. / 729;
      t.a[5][0] = 9017. / 3168; t.a[5][1] = -355. / 33; t.a[5][2] = 46732. / 5247;
      t.a[5][3] = 49. / 176; t.a[5][4] = -5103. / 18656;
      t.a[6][0] = 35. / 384; t.a[6][2] = 500. / 1113; t.a[6][3] = 125. / 192;
      t.a[6][4] = -2187. / 6784; t.a[6][5] = 11. / 84;
      t.b1[0] = 35. / 384; t.b1[2] = 500. / 1113; t.b1[3] = 125. / 192; t.b1[4] = -2187. / 6784;
      t.b1[5] = 11. / 84;
      t.b2[0] = 5179. / 57600; t.b2[2] = 7571. / 16695; t.b2[3] = 393. / 640;
      t.b2[4] = -92097. / 339200; t.b2[5] = 187. / 2100; t.b2[6] = 1. / 40;
      break;
  }
  return t;
}

// core/fieldops.cu:232-258 normalize (inside the geometry)
void set_normalized(Magnet& mg, const std::vector<double>& src) {
  for (int i = 0; i < mg.N; ++i) {
    if (!mg.in_geom(i)) continue;
    double x = src[i], y = src[(size_t)mg.N + i], z = src[2 * (size_t)mg.N + i];
    double inv = 1.0 / std::sqrt(x * x + y * y + z * z);
    mg.m[i] = x * inv;
    mg.m[(size_t)mg.N + i] = y * inv;
    mg.m[2 * (size_t)mg.N + i] = z * inv;
  }
}

double max_norm(const Magnet& mg, const std::vector<double>& v) {  // core/reduce.cu:53-99
  double r = 0;
  for (int i = 0; i < mg.N; ++i) {
    if (!mg.in_geom(i)) continue;
    double n = std::sqrt(v[i] * v[i] + v[(size_t)mg.N + i] * v[(size_t)mg.N + i] +
                         v[2 * (size_t)mg.N + i] * v[2 * (size_t)mg.N + i]);
    if (n > r) r = n;
  }
  return r;
}

// core/timesolver.cpp:37-47
double sensible_timestep(World& w) {
  if (w.mags.empty()) return 0.0;
  double gmax = 0;
  for (auto& mg : w.mags) {
    std::vector<double> tq;
    torque(w, mg, tq, w.relax_torque);
    gmax = std::max(gmax, max_norm(mg, tq));
  }
  if (gmax == 0) return w.sp.sensible_timestep_default;
  return w.sp.sensible_factor / gmax;
}

// core/timesolver.cpp:60-75
void adapt_timestep(World& w, double corr) {
  if (!w.sp.adaptive) return;
  if (std::isnan(corr)) corr = 1.;
  corr *= w.sp.headroom;
  corr = corr > w.sp.upper_bound ? w.sp.upper_bound : corr;
  corr = corr < w.sp.lower_bound ? w.sp.lower_bound : corr;
  w.dt *= corr;
}

// Standard normal number of (seed, step, cell, component), the generator of the
// device path restated in FP64: splitmix64 finaliser of the combined counter,
// two 24-bit uniforms, Box-Muller.
double thermal_normal(uint64_t seed, long long step, int i, int c) {
  uint64_t z = seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(step + 1));
  z += 0xD1B54A32D192ED03ull * (uint64_t)(3 * (long long)i + c + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u1 = (double)((uint32_t)(z >> 40) + 1u) / 16777216.0;
  const double u2 = (double)(uint32_t)(z & 0xFFFFFFull) / 16777216.0;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

// physics/thermalnoise.cu:20-66: thermal field of step `step` (zero where T or Ms is 0)
bool thermal_zero(const Magnet& mg) { return mg.temp.zero() || mg.msat.zero(); }
void thermal_noise(const Magnet& mg, long long step, std::vector<double>& out) {
  const int N = mg.N;
  out.assign(3 * (size_t)N, 0.0);
  const double pref = 2 * 1.38064852e-23 * GAMMALL / (mg.cs[0] * mg.cs[1] * mg.cs[2]);
  for (int i = 0; i < N; ++i) {
    if (!mg.in_geom(i)) continue;
    const double ms = mg.msat.at(i), T = mg.temp.at(i), a = mg.alpha.at(i);
    if (ms == 0 || T == 0) continue;
    const double s = std::sqrt(pref * a * T / ((1 + a * a) * ms));
    for (int c = 0; c < 3; ++c) out[(size_t)c * N + i] = s * thermal_normal(mg.seed, step, i, c);
  }
}

// core/rungekutta.cpp:25-151
void rk_step(World& w) {
  if (w.mags.empty()) {
    w.t += w.dt;
    return;
  }
  const Tableau T = tableau(w.sp.method);
  const double t0 = w.t;
  std::vector<std::vector<double>> x0(w.mags.size());
  for (size_t q = 0; q < w.mags.size(); ++q) x0[q] = w.mags[q].m;
  std::vector<std::vector<std::vector<double>>> k(w.mags.size(), std::vector<std::vector<double>>(T.S));
  // noise of this step, the same for every stage and retry (core/rungekutta.cpp:94-106)
  std::vector<std::vector<double>> noise(w.mags.size());
  for (size_t q = 0; q < w.mags.size(); ++q)
    if (!thermal_zero(w.mags[q])) thermal_noise(w.mags[q], w.steps, noise[q]);
  bool success = false;
  while (!success) {
    const double dt = w.dt;
    for (int s = 0; s < T.S; ++s) {
      w.t = t0 + dt * T.c[s];
      for (size_t q = 0; q < w.mags.size(); ++q) {  // setStageX
        if (s == 0) continue;
        Magnet& mg = w.mags[q];
        std::vector<double> xs = x0[q];
        for (int j = 0; j < s; ++j) {
          double cf = dt * T.a[s][j];
          for (int i = 0; i < mg.N; ++i) {
            if (!mg.in_geom(i)) continue;
            for (int c = 0; c < 3; ++c) xs[(size_t)c * mg.N + i] += cf * k[q][j][(size_t)c * mg.N + i];
          }
        }
        set_normalized(mg, xs);
      }
      for (size_t q = 0; q < w.mags.size(); ++q) {  // setStageK
        torque(w, w.mags[q], k[q][s], w.relax_torque);
        if (!noise[q].empty()) {
          const double f = 1 / std::sqrt(dt);
          for (size_t c = 0; c < noise[q].size(); ++c) k[q][s][c] += f * noise[q][c];
        }
      }
    }
    w.t = t0 + dt;
    for (size_t q = 0; q < w.mags.size(); ++q) {  // setFinalX
      Magnet& mg = w.mags[q];
      std::vector<double> xs = x0[q];
      for (int j = 0; j < T.S; ++j) {
        double cf = dt * T.b1[j];
        for (int i = 0; i < mg.N; ++i) {
          if (!mg.in_geom(i)) continue;
          for (int c = 0; c < 3; ++c) xs[(size_t)c * mg.N + i] += cf * k[q][j][(size_t)c * mg.N + i];
        }
      }
      set_normalized(mg, xs);
    }
    if (!w.sp.adaptive) break;
    double error = 0;
    for (size_t q = 0; q < w.mags.size(); ++q) {  // getError
      Magnet& mg = w.mags[q];
      std::vector<double> err(3 * (size_t)mg.N, 0.0);
      for (int j = 0; j < T.S; ++j) {
        double cf = dt * (T.b1[j] - T.b2[j]);
        for (int i = 0; i < mg.N; ++i) {
          if (!mg.in_geom(i)) continue;
          for (int c = 0; c < 3; ++c) err[(size_t)c * mg.N + i] += cf * k[q][j][(size_t)c * mg.N + i];
        }
      }
      error = std::max(error, max_norm(mg, err));
    }
    success = error < w.sp.max_error;
    double corr = success ? std::pow(w.sp.max_error / error, 1. / (T.order2 + 1))
                          : std::pow(w.sp.max_error / error, 1. / (T.order1 + 1));
    adapt_timestep(w, corr);
    if (!success) {
      for (size_t q = 0; q < w.mags.size(); ++q) w.mags[q].m = x0[q];
      w.t = t0;
      w.rejected++;
    }
  }
  w.steps++;
}

int solver_step(World& w) {  // core/timesolver.cpp:77-83
  if (w.dt <= 0) {
    g_err = "Timesolver can not make a step because the timestep is smaller than or equal to zero.";
    return MPX_ERR_RUNTIME;
  }
  rk_step(w);
  return MPX_OK;
}

}  // namespace

// =====================================================================
// C interface of the oracle (loaded with ctypes by the tests / bench)
// =====================================================================
extern "C" {

typedef struct ox_world ox_world;

const char* ox_last_error(void) { return g_err.c_str(); }

ox_world* ox_create(void) { return reinterpret_cast<ox_world*>(new World()); }
void ox_destroy(ox_world* w) { delete reinterpret_cast<World*>(w); }

int ox_add_magnet(ox_world* wp, const mpx_magnet_desc* d) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet mg;
  int st = load_magnet(mg, d);
  if (st) return -1;
  w.mags.push_back(std::move(mg));
  return (int)w.mags.size() - 1;
}

int ox_update_magnet(ox_world* wp, int q, const mpx_magnet_desc* d) {
  World& w = *reinterpret_cast<World*>(wp);
  return load_magnet(w.mags.at(q), d);
}

void ox_set_world_bias(ox_world* wp, const double b[3]) {
  World& w = *reinterpret_cast<World*>(wp);
  for (int c = 0; c < 3; ++c) w.wb[c] = b[c];
}

// Sets m (float SoA) and normalises it in FP64 (core/variable.cpp:76-79).
int ox_set_m(ox_world* wp, int q, const float* m) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  std::vector<double> src(m, m + 3 * (size_t)mg.N);
  mg.m.assign(3 * (size_t)mg.N, 0.0);
  for (int i = 0; i < mg.N; ++i)
    if (!mg.in_geom(i))
      for (int c = 0; c < 3; ++c) mg.m[(size_t)c * mg.N + i] = src[(size_t)c * mg.N + i];
  set_normalized(mg, src);
  return MPX_OK;
}

// Sets m (double SoA) verbatim, no normalisation (used to continue a state).
int ox_set_m_raw(ox_world* wp, int q, const double* m) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  mg.m.assign(m, m + 3 * (size_t)mg.N);
  return MPX_OK;
}

int ox_get_m(ox_world* wp, int q, double* out) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  std::memcpy(out, mg.m.data(), sizeof(double) * 3 * (size_t)mg.N);
  return MPX_OK;
}

int ox_eval(ox_world* wp, int q, int quantity, double* out) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  std::vector<double> h;
  switch (quantity) {
    case MPX_Q_MAGNETIZATION: h = mg.m; break;
    case MPX_Q_EFFECTIVE_FIELD: effective_field(w, mg, h); break;
    case MPX_Q_EXCHANGE_FIELD: exchange_field(mg, h); break;
    case MPX_Q_DMI_FIELD: dmi_field(mg, h); break;
    case MPX_Q_ANISOTROPY_FIELD: anisotropy_field(mg, h); break;
    case MPX_Q_EXTERNAL_FIELD: ext_field(w, mg, h); break;
    case MPX_Q_DEMAG_FIELD: demag_field(mg, h); break;
    case MPX_Q_TORQUE: torque(w, mg, h); break;
    case MPX_Q_LLG_TORQUE: torque(w, mg, h, false, false); break;
    case MPX_Q_DAMPING_TORQUE: torque(w, mg, h, true); break;
    case MPX_Q_SPIN_TRANSFER_TORQUE: stt_torque(mg, h); break;
    case MPX_Q_EXCHANGE_ENERGY_DENSITY:
    case MPX_Q_DMI_ENERGY_DENSITY:
    case MPX_Q_ANISOTROPY_ENERGY_DENSITY:
    case MPX_Q_ZEEMAN_ENERGY_DENSITY:
    case MPX_Q_DEMAG_ENERGY_DENSITY:
    case MPX_Q_TOTAL_ENERGY_DENSITY: energy_density(w, mg, quantity, h); break;
    default: g_err = "unknown quantity"; return MPX_ERR_INVALID;
  }
  std::memcpy(out, h.data(), sizeof(double) * h.size());
  return MPX_OK;
}

// Test hook: use the given real-space kernel octant (6 components x n cells,
// displacements r >= 0, layout [c][z][y][x]) instead of building one, so that
// the convolution arithmetic can be compared apart from kernel construction.
int ox_set_kernel_octant(ox_world* wp, int q, const double* oct) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  const size_t noct = (size_t)mg.n[0] * mg.n[1] * mg.n[2];
  mg.ext_oct.assign(oct, oct + 6 * noct);
  mg.kready = false;
  return MPX_OK;
}

int ox_demag_brute(ox_world* wp, int q, double* out) {
  World& w = *reinterpret_cast<World*>(wp);
  std::vector<double> h;
  demag_brute(w.mags.at(q), h);
  std::memcpy(out, h.data(), sizeof(double) * h.size());
  return MPX_OK;
}

// Real-space kernel on the reference's kernel grid (physics/strayfieldkernel.cu:80-99):
// size 2n-1 (+1 if > 5 and odd), origin -(n-1) - padding.  out: 6 x K values.
int ox_demag_kernel(ox_world* wp, int q, double* out, int dims[3]) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  int K[3], O[3];
  for (int a = 0; a < 3; ++a) {
    K[a] = 2 * mg.n[a] - 1;
    int pad = (K[a] > 5 && K[a] % 2 == 1) ? 1 : 0;
    K[a] += pad;
    O[a] = -(mg.n[a] - 1) - pad;
    dims[a] = K[a];
  }
  if (!out) return MPX_OK;
  const size_t KK = (size_t)K[0] * K[1] * K[2];
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int k = 0; k < K[2]; ++k)
    for (int j = 0; j < K[1]; ++j)
      for (int i = 0; i < K[0]; ++i) {
        double v[6];
        kernel_at(O[0] + i, O[1] + j, O[2] + k, mg.mg, mg.pbc, mg.cs, v);
        size_t p = ((size_t)k * K[1] + j) * K[0] + i;
        for (int c = 0; c < 6; ++c) out[c * KK + p] = v[c];
      }
  return MPX_OK;
}

double ox_newell(int comp, int x, int y, int z, double cx, double cy, double cz) {
  double v[6];
  newell6(x, y, z, cx, cy, cz, v);
  return v[comp];
}

int ox_average(ox_world* wp, int q, int quantity, double out[3]) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  int nc = MPX_Q_IS_SCALAR(quantity) ? 1 : 3;
  std::vector<double> h((size_t)nc * mg.N);
  int st = ox_eval(wp, q, quantity, h.data());
  if (st) return st;
  int ngeo = 0;
  for (int i = 0; i < mg.N; ++i) ngeo += mg.in_geom(i) ? 1 : 0;
  for (int c = 0; c < nc; ++c) {
    double s = 0;
    for (int i = 0; i < mg.N; ++i)
      if (mg.in_geom(i)) s += h[(size_t)c * mg.N + i];
    out[c] = s / ngeo;
  }
  return MPX_OK;
}

// energy = ncells * <e> * cell volume (physics/energy.cu:52-92)
int ox_energy(ox_world* wp, int q, int quantity, double* out) {
  World& w = *reinterpret_cast<World*>(wp);
  Magnet& mg = w.mags.at(q);
  double avg[3];
  int st = ox_average(wp, q, quantity, avg);
  if (st) return st;
  *out = mg.N * avg[0] * mg.cs[0] * mg.cs[1] * mg.cs[2];
  return MPX_OK;
}

void ox_set_solver(ox_world* wp, const mpx_solver_params* p) {
  World& w = *reinterpret_cast<World*>(wp);
  w.sp = *p;
}
void ox_get_solver(ox_world* wp, mpx_solver_params* p) { *p = reinterpret_cast<World*>(wp)->sp; }
void ox_set_time(ox_world* wp, double t) { reinterpret_cast<World*>(wp)->t = t; }
double ox_get_time(ox_world* wp) { return reinterpret_cast<World*>(wp)->t; }
void ox_set_timestep(ox_world* wp, double dt) { reinterpret_cast<World*>(wp)->dt = dt; }
double ox_get_timestep(ox_world* wp) { return reinterpret_cast<World*>(wp)->dt; }
double ox_sensible_timestep(ox_world* wp) { return sensible_timestep(*reinterpret_cast<World*>(wp)); }
void ox_counters(ox_world* wp, int64_t out[3]) {
  World& w = *reinterpret_cast<World*>(wp);
  out[0] = w.steps;
  out[1] = w.rejected;
  out[2] = w.evals;
}

int ox_step(ox_world* wp) { return solver_step(*reinterpret_cast<World*>(wp)); }

int ox_steps(ox_world* wp, int n) {
  for (int i = 0; i < n; ++i) {
    int st = ox_step(wp);
    if (st) return st;
  }
  return MPX_OK;
}

// core/timesolver.cpp:97-111
int ox_run(ox_world* wp, double duration) {
  World& w = *reinterpret_cast<World*>(wp);
  if (duration <= 0) return MPX_OK;
  double stop = w.t + duration;
  while (w.t < stop - w.dt) {
    int st = solver_step(w);
    if (st) return st;
  }
  double old = w.dt;
  w.dt = stop - w.t;
  int st = solver_step(w);
  if (!w.sp.adaptive) w.dt = old;
  return st;
}


// physics/minimizer.cu:73-160 (Minimizer::exec): steepest descent on the damping
// torque with Barzilai-Borwein step sizes, all magnets of the world.
int ox_minimize(ox_world* wp, double tol, int nsamples) {
  World& w = *reinterpret_cast<World*>(wp);
  const size_t nm = w.mags.size();
  if (nm == 0) return MPX_OK;
  const size_t nkeep = (size_t)nsamples * nm;
  std::vector<std::vector<double>> t0(nm), t1(nm);
  std::vector<double> step(nm, 1e-14);
  std::deque<double> diffs;
  for (size_t q = 0; q < nm; ++q) torque(w, w.mags[q], t0[q], true);
  for (long long n = 0;; ++n) {
    if (diffs.size() >= nkeep) {
      bool conv = true;
      for (double d : diffs) conv = conv && d <= tol;
      if (conv) break;
    }
    if (n >= 10000000) {
      g_err = "minimize did not converge";
      return MPX_ERR_RUNTIME;
    }
    std::vector<std::vector<double>> m0(nm), m1(nm);
    for (size_t q = 0; q < nm; ++q) {  // k_step
      Magnet& mg = w.mags[q];
      const int N = mg.N;
      m0[q] = mg.m;
      m1[q].assign(3 * (size_t)N, 0.0);
      const double dt = step[q];
      for (int i = 0; i < N; ++i) {
        V3 a = mg.mv(i), t{t0[q][i], t0[q][(size_t)N + i], t0[q][2 * (size_t)N + i]};
        const double t2 = dt * dt * dot(t, t);
        const V3 b = (1.0 / (4 + t2)) * ((4 - t2) * a + (4 * dt) * t);
        m1[q][i] = b.x;
        m1[q][(size_t)N + i] = b.y;
        m1[q][2 * (size_t)N + i] = b.z;
      }
      mg.m = m1[q];
      set_normalized(mg, m1[q]);
    }
    for (size_t q = 0; q < nm; ++q) torque(w, w.mags[q], t1[q], true);
    for (size_t q = 0; q < nm; ++q) {
      const int N = w.mags[q].N;
      double dmdm = 0, dmdt = 0, dtdt = 0, mx = 0;
      for (int i = 0; i < N; ++i) {
        double s = 0;
        for (int c = 0; c < 3; ++c) {
          const size_t k = (size_t)c * N + i;
          const double dm = m1[q][k] - m0[q][k], dtq = t0[q][k] - t1[q][k];
          dmdm += dm * dm;
          dmdt += dm * dtq;
          dtdt += dtq * dtq;
          s += dm * dm;
        }
        mx = std::max(mx, std::sqrt(s));
      }
      const double nom = (n % 2 == 0) ? dmdm : dmdt, div = (n % 2 == 0) ? dmdt : dtdt;
      step[q] = (div == 0.0) ? 1e-14 : nom / div;
      diffs.push_back(mx);
      if (diffs.size() > nkeep) diffs.pop_front();
    }
    std::swap(t0, t1);
  }
  return MPX_OK;
}

// physics/relaxer.cpp:88-174 (Relaxer::exec) for all magnets of the world.
int ox_relax(ox_world* wp, double tol, double threshold) {
  World& w = *reinterpret_cast<World*>(wp);
  if (threshold == 0.0) {
    g_err = "The relax threshold should not be zero.";
    return MPX_ERR_INVALID;
  }
  if (w.mags.empty()) return MPX_OK;
  const mpx_solver_params saved = w.sp;
  const double t_saved = w.t, dt_saved = w.dt;
  w.sp.adaptive = 1;
  w.sp.method = MPX_RK_FEHLBERG;
  w.relax_torque = true;
  w.dt = sensible_timestep(w);
  auto energy = [&]() {
    double E = 0;
    for (size_t q = 0; q < w.mags.size(); ++q) {
      double v;
      ox_energy(wp, (int)q, MPX_Q_TOTAL_ENERGY_DENSITY, &v);
      E += v;
    }
    return E;
  };
  auto torque_sq = [&]() {
    double s = 0;
    for (auto& mg : w.mags) {
      std::vector<double> t;
      torque(w, mg, t, true);
      for (int i = 0; i < mg.N; ++i)
        if (mg.in_geom(i))
          for (int c = 0; c < 3; ++c) s += t[(size_t)c * mg.N + i] * t[(size_t)c * mg.N + i];
    }
    return s;
  };
  int st = MPX_OK;
  long long nsteps = 0;
  auto steps3 = [&]() {
    nsteps += 3;
    if (nsteps > 10000000) {
      g_err = "relax did not converge";
      return (int)MPX_ERR_RUNTIME;
    }
    return ox_steps(wp, 3);
  };
  do {
    double E0 = energy();
    if ((st = steps3())) break;
    double E1 = energy();
    while (E1 < E0) {
      if ((st = steps3())) break;
      E0 = E1;
      E1 = energy();
    }
    if (st) break;
    double err = w.sp.max_error;
    if (threshold < 0) {
      double tq1 = torque_sq(), tq0;
      while (err > tol && !st) {
        err /= std::sqrt(2.0);
        w.sp.max_error = err;
        if ((st = steps3())) break;
        tq0 = tq1;
        tq1 = torque_sq();
        while (tq1 < tq0) {
          if ((st = steps3())) break;
          tq0 = tq1;
          tq1 = torque_sq();
        }
      }
    } else {
      while (err > tol && !st) {
        bool conv = true;
        for (auto& mg : w.mags) {
          std::vector<double> t;
          torque(w, mg, t, true);
          if (max_norm(mg, t) > threshold) {
            conv = false;
            break;
          }
        }
        if (conv) {
          err /= std::sqrt(2.0);
          w.sp.max_error = err;
        }
        st = steps3();
      }
    }
  } while (false);
  w.sp = saved;
  w.relax_torque = false;
  w.t = t_saved;
  w.dt = dt_saved;
  if (saved.adaptive) w.dt = sensible_timestep(w);
  return st;
}

}  // extern "C"
