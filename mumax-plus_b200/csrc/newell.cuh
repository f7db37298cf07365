// newell.cuh -- FP64 construction of the demag kernel and its spectrum.
//
// The Newell tensor (Newell, Williams & Dunlop 1993, eqs. 27 and 32) is the
// 27-point weighted combination of the indefinite integrals, evaluated in
// double precision exactly as physics/newell.cu:7-139 does, and summed over the
// PBC images (2r+1 per periodic axis) as physics/strayfieldkernel.cu:25-56 does
// -- here the image sum is also FP64.  It is evaluated once per octant point
// |r| (the tensor is even in every axis for xx/yy/zz and odd in the axes its
// off-diagonal indices name), expanded to the circular padded grid, transformed
// with an FP64 radix-2 FFT, and the real, symmetry-reduced spectrum
// (kx in [0,Px/2], ky in [0,Py/2], kz in [0,Pz/2]) is stored in FP32 with the
// convolution prefactor -mu0/(Px Py Pz) folded in.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mpx {

__device__ __forceinline__ double nxx_indef(int ix, int iy, int iz, double cx, double cy, double cz) {
  const double x = ix * cx, y = iy * cy, z = iz * cz;
  const double R = sqrt(x * x + y * y + z * z);
  double r = 0;
  if (ix != 0 || iz != 0) r += (y / 2) * (z * z - x * x) * asinh(y / sqrt(x * x + z * z));
  if (ix != 0 || iy != 0) r += (z / 2) * (y * y - x * x) * asinh(z / sqrt(x * x + y * y));
  if (ix != 0) r -= x * y * z * atan((y * z) / (x * R));
  r += (1. / 6.) * (2 * x * x - y * y - z * z) * R;
  return r;
}

__device__ __forceinline__ double nxy_indef(int ix, int iy, int iz, double cx, double cy, double cz) {
  if (iy == 0 || ix == 0) return 0.0;
  const double x = ix * cx, y = iy * cy, z = iz * cz;
  const double R = sqrt(x * x + y * y + z * z);
  double r = 0;
  r += (x * y * z) * asinh(z / sqrt(x * x + y * y));
  r += (y / 6) * (3 * z * z - y * y) * asinh(x / sqrt(y * y + z * z));
  r += (x / 6) * (3 * z * z - x * x) * asinh(y / sqrt(x * x + z * z));
  r -= (z * y * y / 2) * atan((x * z) / (y * R));
  r -= (z * x * x / 2) * atan((y * z) / (x * R));
  r -= x * y * R / 3;
  if (iz != 0) r -= (z * z * z / 6) * atan((x * y) / (z * R));
  return r;
}

__device__ __forceinline__ int newell_w(int dx, int dy, int dz) {
  const int s = dx * dx + dy * dy + dz * dz;
  return s == 0 ? 8 : s == 1 ? -4 : s == 2 ? 2 : -1;
}

__device__ double newell_nxx(int ix, int iy, int iz, double cx, double cy, double cz) {
  double r = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz)
        r += newell_w(dx, dy, dz) * nxx_indef(ix + dx, iy + dy, iz + dz, cx, cy, cz);
  return r / (4 * M_PI * cx * cy * cz);
}

__device__ double newell_nxy(int ix, int iy, int iz, double cx, double cy, double cz) {
  if (ix == 0 || iy == 0) return 0;
  double r = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz)
        r += newell_w(dx, dy, dz) * nxy_indef(ix + dx, iy + dy, iz + dz, cx, cy, cz);
  return r / (4 * M_PI * cx * cy * cz);
}

// component c (xx, yy, zz, xy, xz, yz) at displacement (x, y, z) cells
__device__ double newell_comp(int c, int x, int y, int z, double cx, double cy, double cz) {
  switch (c) {
    case 0: return newell_nxx(x, y, z, cx, cy, cz);
    case 1: return newell_nxx(y, z, x, cy, cz, cx);
    case 2: return newell_nxx(z, x, y, cz, cx, cy);
    case 3: return newell_nxy(x, y, z, cx, cy, cz);
    case 4: return newell_nxy(x, z, y, cx, cz, cy);
    default: return newell_nxy(y, z, x, cy, cz, cx);
  }
}

struct KernelGeom {
  int n[3];      // source/destination grid size
  int mg[3];     // mastergrid size (image period)
  int pbc[3];    // image repetitions
  double cs[3];  // cell size
};

// Octant values N_c(|rx|, |ry|, |rz|) for |r_a| < n_a, all 6 components, FP64.
// out layout: [c][rz][ry][rx]
__global__ void k_newell_octant(double* __restrict__ out, KernelGeom g) {
  const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int rx = (int)(t % g.n[0]);
    const int ry = (int)((t / g.n[0]) % g.n[1]);
    const int rz = (int)(t / ((long long)g.n[0] * g.n[1]));
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int i = -g.pbc[0]; i <= g.pbc[0]; ++i)
      for (int j = -g.pbc[1]; j <= g.pbc[1]; ++j)
        for (int k = -g.pbc[2]; k <= g.pbc[2]; ++k) {
          const int x = rx + i * g.mg[0], y = ry + j * g.mg[1], z = rz + k * g.mg[2];
#pragma unroll 1
          for (int c = 0; c < 6; ++c) v[c] += newell_comp(c, x, y, z, g.cs[0], g.cs[1], g.cs[2]);
        }
    for (int c = 0; c < 6; ++c) out[c * total + t] = v[c];
  }
}

// Reference-layout real-space kernel (physics/strayfieldkernel.cu:80-99):
// grid K with origin O (cells), 6 comps, cast to float.
__global__ void k_newell_reflayout(float* __restrict__ out, KernelGeom g, int K0, int K1, int K2, int O0, int O1,
                                   int O2) {
  const long long total = (long long)K0 * K1 * K2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int x0 = O0 + (int)(t % K0);
    const int y0 = O1 + (int)((t / K0) % K1);
    const int z0 = O2 + (int)(t / ((long long)K0 * K1));
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int i = -g.pbc[0]; i <= g.pbc[0]; ++i)
      for (int j = -g.pbc[1]; j <= g.pbc[1]; ++j)
        for (int k = -g.pbc[2]; k <= g.pbc[2]; ++k)
#pragma unroll 1
          for (int c = 0; c < 6; ++c)
            v[c] += newell_comp(c, x0 + i * g.mg[0], y0 + j * g.mg[1], z0 + k * g.mg[2], g.cs[0], g.cs[1], g.cs[2]);
    for (int c = 0; c < 6; ++c) out[c * total + t] = (float)v[c];
  }
}

// The same table from one over absolute displacements: entry j of the output
// is displacement O + j (K per axis); the input holds |d| = A + a (a < L per
// axis), same layout.  Diagonal components are even in every displacement
// component, xy odd in x and y, xz in x and z, yz in y and z, also after the sum
// over periodic images (their repetitions run over -p .. p), so each output is
// an input entry times the signs of its odd components.
__global__ void k_newell_expand_abs(float* __restrict__ out, const float* __restrict__ abs_tab, int K0, int K1,
                                    int K2, int O0, int O1, int O2, int A0, int A1, int A2, int L0, int L1, int L2) {
  const long long total = (long long)K0 * K1 * K2, ltot = (long long)L0 * L1 * L2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int x = O0 + (int)(t % K0);
    const int y = O1 + (int)((t / K0) % K1);
    const int z = O2 + (int)(t / ((long long)K0 * K1));
    const long long p = ((long long)(abs(z) - A2) * L1 + (abs(y) - A1)) * L0 + (abs(x) - A0);
    const float sx = x < 0 ? -1.f : 1.f, sy = y < 0 ? -1.f : 1.f, sz = z < 0 ? -1.f : 1.f;
    out[t] = abs_tab[p];
    out[total + t] = abs_tab[ltot + p];
    out[2 * total + t] = abs_tab[2 * ltot + p];
    out[3 * total + t] = (sx * sy) * abs_tab[3 * ltot + p];
    out[4 * total + t] = (sx * sz) * abs_tab[4 * ltot + p];
    out[5 * total + t] = (sy * sz) * abs_tab[5 * ltot + p];
  }
}

// Expand component c of the octant table to the circular P-grid (imag = 0).
// Parity: xy odd in x,y; xz odd in x,z; yz odd in y,z; diagonal even.
__global__ void k_kernel_expand(double2* __restrict__ full, const double* __restrict__ oct, int c, KernelGeom g,
                                int P0, int P1, int P2) {
  const long long total = (long long)P0 * P1 * P2;
  const long long noct = (long long)g.n[0] * g.n[1] * g.n[2];
  const int oddx = (c == 3 || c == 4), oddy = (c == 3 || c == 5), oddz = (c == 4 || c == 5);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % P0), j = (int)((t / P0) % P1), k = (int)(t / ((long long)P0 * P1));
    auto circ = [](int q, int P, int n) { return q <= n - 1 ? q : (q >= P - (n - 1) ? q - P : INT_MIN); };
    const int rx = circ(i, P0, g.n[0]), ry = circ(j, P1, g.n[1]), rz = circ(k, P2, g.n[2]);
    double v = 0.0;
    if (rx != INT_MIN && ry != INT_MIN && rz != INT_MIN) {
      const int ax = abs(rx), ay = abs(ry), az = abs(rz);
      v = oct[c * noct + ((long long)az * g.n[1] + ay) * g.n[0] + ax];
      if (oddx && rx < 0) v = -v;
      if (oddy && ry < 0) v = -v;
      if (oddz && rz < 0) v = -v;
    }
    full[t] = make_double2(v, 0.0);
  }
}

// One radix-2 Stockham pass (FP64) along `axis` of a P0 x P1 x P2 array.
// Consecutive threads take consecutive butterflies of a line along x and
// consecutive lines (adjacent x) along y and z, so that every load and store
// of a warp is contiguous.
__global__ void k_fft64_pass(const double2* __restrict__ in, double2* __restrict__ out, int P0, int P1, int P2,
                             int axis, int Ns) {
  const int L = axis == 0 ? P0 : axis == 1 ? P1 : P2;
  const long long stride = axis == 0 ? 1 : axis == 1 ? P0 : (long long)P0 * P1;
  const long long nlines = (long long)P0 * P1 * P2 / L;
  const long long total = nlines * (L / 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = axis == 0 ? (int)(t % (L / 2)) : (int)(t / nlines);
    const long long line = axis == 0 ? t / (L / 2) : t % nlines;
    long long base;
    if (axis == 0) base = line * P0;
    else if (axis == 1) base = (line / P0) * ((long long)P0 * P1) + (line % P0);
    else base = line;
    const int k = j & (Ns - 1);
    const double2 a = in[base + j * stride];
    double2 b = in[base + (j + L / 2) * stride];
    double s, c;
    sincospi(-(double)k / Ns, &s, &c);
    b = make_double2(b.x * c - b.y * s, b.x * s + b.y * c);
    const int o = (j - k) * 2 + k;
    out[base + o * stride] = make_double2(a.x + b.x, a.y + b.y);
    out[base + (o + Ns) * stride] = make_double2(a.x - b.x, a.y - b.y);
  }
}

// Store the real, symmetry-reduced spectrum of component c (slot kc of kcomp)
// in the layout read by k_yz: [kx][kz'][kcomp][ky'].
__global__ void k_kernel_extract(float* __restrict__ kspec, const double2* __restrict__ full, int kc, int kcomp,
                                 int P0, int P1, int P2, double pref) {
  const int Fh = P0 / 2 + 1, hy = P1 / 2 + 1, hz = P2 / 2 + 1;
  const long long total = (long long)Fh * hy * hz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int ky = (int)(t % hy), kz = (int)((t / hy) % hz), kx = (int)(t / ((long long)hy * hz));
    const double v = full[kx + (long long)P0 * (ky + (long long)P1 * kz)].x;
    kspec[(((long long)kx * hz + kz) * kcomp + kc) * hy + ky] = (float)(pref * v);
  }
}

}  // namespace mpx
