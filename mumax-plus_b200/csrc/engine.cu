// engine.cu -- host engine and C ABI (include/mpx.h) of libmpx.so.
//
// An engine owns one CUDA stream on one device, the ferromagnets added to it
// (their parameters, field buffers, demag spectra) and the solve groups that
// step them.  All per-step decisions (accept/reject, new time step, run/steps
// bookkeeping) are taken on the device by k_controller, so a run is a stream of
// kernel launches with a status read every few attempts; no per-kernel host
// synchronisation as in the reference (cudautil/cudalaunch.hpp:10-19).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/mpx.h"
#include "kernels.cuh"
#include "newell.cuh"
#include "stray.cuh"
#include "pairfft.cuh"
#include "yzsplit.cuh"
#include "dft_tc.cuh"

using namespace mpx;

namespace {

// NVTX range over a host entry point or phase (shown by Nsight tools, no cost
// without one attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

thread_local std::string g_last_error;

mpx_status fail(mpx_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

#define CUDA_TRY(expr)                                                                    \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) return fail(MPX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define MPX_TRY(expr)               \
  do {                              \
    mpx_status _s = (expr);         \
    if (_s != MPX_OK) return _s;    \
  } while (0)

int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

// padded FFT length: smallest power of two >= 2n-1 (1 when n == 1)
int padded(int n) { return n == 1 ? 1 : 1 << ilog2(2 * n - 1); }

constexpr int MAX_FFT = 4096;
constexpr int SMEM_MAX = 227 * 1024;
// dynamic shared memory left next to the static descriptor copies of a block
constexpr int SMEM_DYN_MAX = SMEM_MAX - 2048;
constexpr int YZ_CLASSES = 24;  // k_yz / k_yzw / k_yzw32 / k_yzw64 launch classes (yz_class)

// ------------------------------------------------------------ tableaus
// core/butchertableau.cpp: Heun, Bogacki-Shampine, Cash-Karp, Fehlberg, Dormand-Prince
TableauDev make_tableau(int method) {
  TableauDev t;
  std::memset(&t, 0, sizeof(t));
  switch (method) {
    case MPX_RK_HEUN:
      t.S = 2; t.order1 = 2; t.order2 = 1;
      t.c[1] = 1; t.a[1][0] = 1;
      t.b1[0] = 1. / 2.; t.b1[1] = 1. / 2.; t.b2[0] = 1.; t.b2[1] = 0.;
      break;
    case MPX_RK_BOGACKI_SHAMPINE:
      t.S = 4; t.order1 = 3; t.order2 = 2;
      t.c[1] = 1. / 2.; t.c[2] = 3. / 4.; t.c[3] = 1.;
      t.a[1][0] = 1. / 2.; t.a[2][0] = 0.; t.a[2][1] = 3. / 4.;
      t.a[3][0] = 2. / 9.; t.a[3][1] = 1. / 3.; t.a[3][2] = 4. / 9.;
      t.b1[0] = 2. / 9.; t.b1[1] = 1. / 3.; t.b1[2] = 4. / 9.; t.b1[3] = 0.;
      t.b2[0] = 7. / 24.; t.b2[1] = 1. / 4.; t.b2[2] = 1. / 3.; t.b2[3] = 1. / 8.;
      break;
    case MPX_RK_CASH_KARP:
      t.S = 6; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 5.; t.c[2] = 3. / 10.; t.c[3] = 3. / 5.; t.c[4] = 1.; t.c[5] = 7. / 8.;
      t.a[1][0] = 1. / 5.;
      t.a[2][0] = 3. / 40.; t.a[2][1] = 9. / 40.;
      t.a[3][0] = 3. / 10.; t.a[3][1] = -9. / 10.; t.a[3][2] = 6. / 5.;
      t.a[4][0] = -11. / 54.; t.a[4][1] = 5. / 2.; t.a[4][2] = -70. / 27.; t.a[4][3] = 35. / 27.;
      t.a[5][0] = 1631. / 55296.; t.a[5][1] = 175. / 512.; t.a[5][2] = 575. / 13824.;
      t.a[5][3] = 44275. / 110592.; t.a[5][4] = 253. / 4096.;
      t.b1[0] = 37. / 378.; t.b1[2] = 250. / 621.; t.b1[3] = 125. / 594.; t.b1[5] = 512. / 1771.;
      t.b2[0] = 2825. / 27648.; t.b2[2] = 18575. / 48384.; t.b2[3] = 13525. / 55296.;
      t.b2[4] = 277. / 14336.; t.b2[5] = 1. / 4.;
      break;
    case MPX_RK_FEHLBERG:
      t.S = 6; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 4.; t.c[2] = 3. / 8.; t.c[3] = 12. / 13.; t.c[4] = 1.; t.c[5] = 1. / 2.;
      t.a[1][0] = 1. / 4.;
      t.a[2][0] = 3. / 32.; t.a[2][1] = 9. / 32.;
      t.a[3][0] = 1932. / 2197.; t.a[3][1] = -7200. / 2197.; t.a[3][2] = 7296. / 2197.;
      t.a[4][0] = 439. / 216.; t.a[4][1] = -8.; t.a[4][2] = 3680. / 513.; t.a[4][3] = -845. / 4104.;
      t.a[5][0] = -8. / 27.; t.a[5][1] = 2.; t.a[5][2] = -3544. / 2565.; t.a[5][3] = 1859. / 4104.;
      t.a[5][4] = -11. / 40.;
      t.b1[0] = 16. / 135.; t.b1[2] = 6656. / 12825.; t.b1[3] = 28561. / 56430.; t.b1[4] = -9. / 50.;
      t.b1[5] = 2. / 55.;
      t.b2[0] = 25. / 216.; t.b2[2] = 1408. / 2565.; t.b2[3] = 2197. / 4104.; t.b2[4] = -1. / 5.;
      break;
    default:  // MPX_RK_DORMAND_PRINCE
      t.S = 7; t.order1 = 5; t.order2 = 4;
      t.c[1] = 1. / 5.; t.c[2] = 3. / 10.; t.c[3] = 4. / 5.; t.c[4] = 8. / 9.; t.c[5] = 1.; t.c[6] = 1.;
      t.a[1][0] = 1. / 5.;
      t.a[2][0] = 3. / 40.; t.a[2][1] = 9. / 40.;
      t.a[3][0] = 44. / 45.; t.a[3][1] = -56. / 15.; t.a[3][2] = 32. / 9.;
      t.a[4][0] = 19372. / 6561.; t.a[4][1] = -25360. / 2187.; t.a[4][2] = 64448. / 6561.;
      t.a[4][3] = -212. / 729.;
      t.a[5][0] = 9017. / 3168.; t.a[5][1] = -355. / 33.; t.a[5][2] = 46732. / 5247.;
      t.a[5][3] = 49. / 176.; t.a[5][4] = -5103. / 18656.;
      t.a[6][0] = 35. / 384.; t.a[6][2] = 500. / 1113.; t.a[6][3] = 125. / 192.;
      t.a[6][4] = -2187. / 6784.; t.a[6][5] = 11. / 84.;
      t.b1[0] = 35. / 384.; t.b1[2] = 500. / 1113.; t.b1[3] = 125. / 192.; t.b1[4] = -2187. / 6784.;
      t.b1[5] = 11. / 84.;
      t.b2[0] = 5179. / 57600.; t.b2[2] = 7571. / 16695.; t.b2[3] = 393. / 640.;
      t.b2[4] = -92097. / 339200.; t.b2[5] = 187. / 2100.; t.b2[6] = 1. / 40.;
      t.fsal = 1;  // last row of a equals b1: x_new is the last stage state, k_new0 = k_last
      break;
  }
  return t;
}

// ---------------------------------------------------------------- objects
struct Magnet {
  int slot = -1, group = -1;
  uint64_t uid = 0;  // unique per magnet object of the engine (slots are reused)
  uint64_t ver = 0;  // bumped whenever its work lists (tiles, y/z blocks) change
  MagnetDev dev;
  unsigned terms_base = 0;        // TERM_* / FLAG_* from the parameters, before stray fields
  bool msat_zero = false;
  bool stray_src = true, stray_dst = true;
  bool probe = false;  // probe grid of a stray-field evaluation: never stepped, in no group's tables
  int pbc_rep[3] = {0, 0, 0};
  double cs_d[3] = {1, 1, 1};
  float* hstray = nullptr;        // stray field of the other magnets (3N floats), when a destination
  std::vector<void*> allocs;  // per-magnet device allocations (params, masks, buffers...)
  int64_t bytes = 0;
  bool demag = false;
  int ty = 4;    // rows per x-pass tile
  int nkx = 1;   // consecutive kx per y/z block
  int ty_def = 4, nkx_def = 1;  // the shapes for a magnet launched with many others
  bool split = false;        // y/z in three passes (k_ycols, k_zmul, k_ycols)
  int ncy = 1, nkz = 1;      // columns per k_ycols block, ky per k_zmul block
  float2* tspec = nullptr;
  int64_t tspec_bytes = 0;
  std::vector<Work> ycw, zmw;            // k_ycols / k_zmul work items
  Work *d_ycw = nullptr, *d_zmw = nullptr;
  bool tc = false;                       // split path with the tensor-core y transforms (k_ydft_tc)
  std::vector<Work> tcw;                 // k_ydft_tc work items (tiles of 4 / R columns)
  Work* d_tcw = nullptr;
  int P[3] = {1, 1, 1};
  // kernel-defining geometry (rebuild the spectrum when it changes)
  int kkey_n[3], kkey_mg[3], kkey_pbc[3];
  double kkey_cs[3];
  bool kspec_ready = false;
  float* kspec = nullptr;
  float2* spec = nullptr;
  float* fields = nullptr;   // 9 buffers of 3N floats
  int64_t fields_bytes = 0, spec_bytes = 0, kspec_bytes = 0;
  unsigned char* geom = nullptr;
  int ngeo = 0;
  std::vector<Work> tiles;   // row tiles (mag, z, y0, ty)
  std::vector<Work> kxw;     // (mag, kx)
  Work* d_tiles = nullptr;   // eval tables of this magnet only
  Work* d_kxw = nullptr;
};

struct Group {
  int slot = -1;
  mpx_solver_params sp{MPX_RK_FEHLBERG, 1, 1e-5, 0.8, 0.5, 2.0, 0.01, 1e-14};
  std::vector<int> magnets;
  bool active = false;  // started and not yet seen finished: its magnets are in the attempt tables
  int torque_kind = 0;  // 0: LLG torque, 1: damping torque (during relax), mirrors GroupDev::torque_kind
  int thermal = 0;      // mirrors GroupDev::thermal
};

// A launch table whose entries keep their place while solves come and go.
// Each magnet occupies one contiguous range (its work items, in order); a
// magnet that is no longer launched leaves a hole (entries with mag = -1,
// which every kernel skips in load_descs).  New magnets are appended, and
// the table is compacted when the holes outnumber the live entries.  Only
// the changed range is uploaded: a solve that arrives or finishes costs a
// copy of its own items, not a rebuild of every table.
struct SlotTable {
  struct Place {
    int off, len;
    uint64_t ver;
  };
  std::vector<Work> items;                     // host copy of the used entries
  std::unordered_map<uint64_t, Place> place;   // by magnet uid
  Work* dev = nullptr;                         // device copy, capacity cap
  int cap = 0, live = 0;
  int dlo = 1 << 30, dhi = -1;                 // entries to upload
  void dirty(int lo, int hi) {
    dlo = std::min(dlo, lo);
    dhi = std::max(dhi, hi);
  }
  void remove(uint64_t uid) {
    auto it = place.find(uid);
    if (it == place.end()) return;
    const Place p = it->second;
    for (int i = p.off; i < p.off + p.len; ++i) items[i].mag = -1;
    dirty(p.off, p.off + p.len);
    live -= p.len;
    place.erase(it);
  }
  void add(uint64_t uid, uint64_t ver, const std::vector<Work>& w) {
    const int off = (int)items.size();
    items.insert(items.end(), w.begin(), w.end());
    dirty(off, off + (int)w.size());
    live += (int)w.size();
    place[uid] = Place{off, (int)w.size(), ver};
  }
  void clear() {
    items.clear();
    place.clear();
    live = 0;
    dlo = 0;
    dhi = 0;
  }
};

}  // namespace

// FFT form of a stray-field pair on its own kernel grid (pairfft.cuh): the
// lengths, buffers and launch shapes of its five passes.
struct PairPlan {
  PairFft pf{};
  float2* t = nullptr;   // work spectrum, 3 components
  float2* ks = nullptr;  // kernel spectrum, 6 components
  int ry_f = 1, zc_f = 1, tky = 1, zc_i = 1, ry_i = 1;  // rows / columns per block of each pass
  int g_xf = 0, g_yf = 0, g_z = 0, g_yi = 0, g_xi = 0;  // grids
  int s_xf = 0, s_yf = 0, s_z = 0, s_yi = 0, s_xi = 0;  // dynamic shared memory (bytes)
  int s_yz = 0;  // > 0: the fused y / z pass k_pair_yz (one block per kx) with this shared memory
  int launches() const { return s_yz > 0 ? 3 : 5; }
};

struct mpx_engine {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  // stream-ordered pool for everything a magnet owns (kept reserved when freed,
  // so adding and removing solves neither synchronises the device nor returns
  // memory to the driver)
  cudaMemPool_t pool = nullptr;
  std::vector<std::unique_ptr<Magnet>> mags;
  std::vector<std::unique_ptr<Group>> groups;
  MagnetDev* d_mags = nullptr;
  int d_mags_cap = 0;
  GroupDev* d_groups = nullptr;
  int d_groups_cap = 0;
  float2* d_tw = nullptr;
  double* d_red = nullptr;   // reduction partials
  double* d_redout = nullptr;
  float* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  // run tables over all magnets: x tiles (demag / local), y/z blocks per
  // class, split path (k_ycols, k_zmul, k_ydft_tc)
  enum { TT_DEMAG = 0, TT_LOCAL, TT_YCOLS, TT_ZMUL, TT_TC, TT_YZ0 };
  SlotTable tt[TT_YZ0 + YZ_CLASSES];
  uint64_t next_uid = 1;
  bool tables_dirty = true;
  bool tables_valid = false;     // the device tables below hold tables_sig
  std::vector<long long> tables_sig;
  Work *d_t_demag = nullptr, *d_t_local = nullptr;
  int n_t_demag = 0, n_t_local = 0;
  // k_yz work per class (yz_class: the z length and whether Py > 2048)
  Work* d_kx_demag[YZ_CLASSES] = {};
  int n_kx_demag[YZ_CLASSES] = {};
  int smem_yz[YZ_CLASSES] = {};
  // split y/z path over all split magnets
  Work *d_t_ycols = nullptr, *d_t_zmul = nullptr;
  int n_t_ycols = 0, n_t_zmul = 0, smem_ycols = 0, smem_zmul = 0, maxpy_split = 0, maxpz_split = 0;
  Work* d_t_tc = nullptr;  // k_ydft_tc items over all started tensor-core magnets
  int n_t_tc = 0;
  // y transforms of the demag convolution: MPX_DFT_FP32 (shared-memory FFT) or
  // MPX_DFT_TF32X3 (tcgen05 GEMMs, for y lengths 1024 and 2048); the DFT32
  // matrix (hi, lo) of the tensor-core form
  int dft_mode = MPX_DFT_FP32;
  float* d_dftB = nullptr;
  int n_sm = 148;  // multiprocessors of the engine's device
  int smem_x = 0, nt_x = 256;
  bool x_pair = false;  // a launched magnet has 2048-point x rows: the PAIR forms of the x passes
  bool any_nodemag = false;
  int64_t bytes = 0;
  int64_t launches = 0;
  double wb[3] = {0, 0, 0};
  int tab_method = -1;
  // stray-field pairs (source -> destination magnet of one group)
  struct Pair {
    int src, dst;
    float* k;         // direct-sum table (brute-force form), or NULL
    StrayTable tab;
    bool fft = false;  // FFT form on the pair's kernel grid (plan), else the direct sum (k, tab)
    PairPlan plan;
    int launches = 1;  // kernels per evaluation
  };
  std::vector<Pair> pairs;
  // FFT plans of recent stray-field evaluations on other grids (mpx_stray_field),
  // by geometry: source and destination grids, cell size, periodic images
  struct PairCacheEntry {
    int key[18];
    double cs[3];
    PairPlan plan;
    uint64_t used;
  };
  std::vector<PairCacheEntry> pair_cache;
  uint64_t pair_cache_tick = 0;
  bool pairs_dirty = true;
  bool any_thermal = false;  // some started group has thermal noise: stage 0 is evaluated every attempt
  int sampling_group = -1;   // group of the sampled run in progress (its magnets get sample kernels)
  int samp_magnets = 0;
  // autotuned shape divisors and the launched set they belong to (mpx_autotune)
  int tune_div_x = 1, tune_div_yz = 1;
  long long tune_cells = 0;
  // CUDA graphs of one attempt: every stage, and (FSAL methods) without
  // stage 0, whose torque k0 is the last stage of the previous step
  cudaGraphExec_t graph = nullptr, graph_nok0 = nullptr;
  int graph_method = -1;
  bool graph_dirty = true;
  int64_t graph_instantiations = 0, graph_updates = 0;  // attempt graphs built anew / updated in place
  bool need_stage0 = true;  // some started group may lack a valid k0
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Stream-ordered allocation from the engine's pool (usable by every later
// operation on the engine's stream).
mpx_status palloc(mpx_engine* e, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return MPX_OK;
  cudaError_t st = cudaMallocFromPoolAsync(p, bytes, e->pool, e->stream);
  if (st != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(MPX_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                   cudaGetErrorString(st));
  }
  return MPX_OK;
}
// Stream-ordered release: the memory returns to the pool once the work queued
// before it on the engine's stream has finished.
void pfree(mpx_engine* e, void* p) {
  if (p) cudaFreeAsync(p, e->stream);
}

mpx_status dalloc(mpx_engine* e, Magnet* m, void** p, size_t bytes) {
  MPX_TRY(palloc(e, p, bytes));
  if (!*p) return MPX_OK;
  if (m) {
    m->allocs.push_back(*p);
    m->bytes += (int64_t)bytes;
  }
  e->bytes += (int64_t)bytes;
  return MPX_OK;
}

void free_magnet(mpx_engine* e, Magnet* m) {
  for (void* p : m->allocs) pfree(e, p);
  e->bytes -= m->bytes;
  m->allocs.clear();
  m->bytes = 0;
}

// Frees every device allocation of a magnet.
void release_all(mpx_engine* e, Magnet* m) {
  free_magnet(e, m);
  pfree(e, m->hstray);
  m->hstray = nullptr;
  e->pairs_dirty = true;
  pfree(e, m->tspec);
  e->bytes -= m->tspec_bytes;
  m->tspec = nullptr;
  m->tspec_bytes = 0;
  pfree(e, m->d_ycw);
  pfree(e, m->d_zmw);
  pfree(e, m->d_tcw);
  m->d_ycw = m->d_zmw = nullptr;
  m->d_tcw = nullptr;
  pfree(e, m->fields);
  pfree(e, m->spec);
  pfree(e, m->kspec);
  e->bytes -= m->fields_bytes + m->spec_bytes + m->kspec_bytes;
  m->fields = nullptr;
  m->spec = nullptr;
  m->kspec = nullptr;
  m->fields_bytes = m->spec_bytes = m->kspec_bytes = 0;
  pfree(e, m->d_tiles);
  pfree(e, m->d_kxw);
  m->d_tiles = nullptr;
  m->d_kxw = nullptr;
}

Magnet* get_mag(mpx_engine* e, int id) {
  if (!e || id < 0 || id >= (int)e->mags.size()) return nullptr;
  return e->mags[id].get();
}
Group* get_group(mpx_engine* e, int id) {
  if (!e || id < 0 || id >= (int)e->groups.size()) return nullptr;
  return e->groups[id].get();
}

mpx_status read_group(mpx_engine* e, int g, GroupDev* out) {
  CUDA_TRY(cudaMemcpyAsync(out, e->d_groups + g, sizeof(GroupDev), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}
mpx_status write_group(mpx_engine* e, int g, const GroupDev* in) {
  if (!in->k0_valid) e->need_stage0 = true;  // the next attempt must evaluate k0
  CUDA_TRY(cudaMemcpyAsync(e->d_groups + g, in, sizeof(GroupDev), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status upload_magnet_desc(mpx_engine* e, Magnet* m) {
  if (m->slot >= e->d_mags_cap) {
    int cap = std::max(16, e->d_mags_cap * 2);
    while (cap <= m->slot) cap *= 2;
    MagnetDev* nd = nullptr;
    CUDA_TRY(cudaMalloc(&nd, sizeof(MagnetDev) * cap));
    if (e->d_mags) {
      CUDA_TRY(cudaMemcpyAsync(nd, e->d_mags, sizeof(MagnetDev) * e->d_mags_cap, cudaMemcpyDeviceToDevice, e->stream));
      CUDA_TRY(cudaStreamSynchronize(e->stream));
      cudaFree(e->d_mags);
    }
    e->d_mags = nd;
    e->d_mags_cap = cap;
    e->graph_dirty = true;
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_mags + m->slot, &m->dev, sizeof(MagnetDev), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status ensure_group_capacity(mpx_engine* e, int slot) {
  if (slot < e->d_groups_cap) return MPX_OK;
  int cap = std::max(16, e->d_groups_cap * 2);
  while (cap <= slot) cap *= 2;
  GroupDev* nd = nullptr;
  CUDA_TRY(cudaMalloc(&nd, sizeof(GroupDev) * cap));
  CUDA_TRY(cudaMemsetAsync(nd, 0, sizeof(GroupDev) * cap, e->stream));
  if (e->d_groups)
    CUDA_TRY(cudaMemcpyAsync(nd, e->d_groups, sizeof(GroupDev) * e->d_groups_cap, cudaMemcpyDeviceToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (e->d_groups) cudaFree(e->d_groups);
  e->d_groups = nd;
  e->d_groups_cap = cap;
  e->graph_dirty = true;
  return MPX_OK;
}

mpx_status ensure_scratch(mpx_engine* e, size_t bytes) {
  if (bytes <= e->scratch_bytes) return MPX_OK;
  pfree(e, e->d_scratch);
  e->d_scratch = nullptr;
  e->scratch_bytes = 0;
  MPX_TRY(palloc(e, (void**)&e->d_scratch, bytes));
  e->scratch_bytes = bytes;
  return MPX_OK;
}

// Replaces *d by a device copy of v (stream-ordered: kernels queued before
// still read the old table, which returns to the pool after them).
template <typename T>
mpx_status upload_vec(mpx_engine* e, Work** d, const std::vector<T>& v) {
  pfree(e, *d);
  *d = nullptr;
  if (v.empty()) return MPX_OK;
  MPX_TRY(palloc(e, (void**)d, sizeof(T) * v.size()));
  CUDA_TRY(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

// dynamic shared memory: padded rows / columns plus the twiddle table of the length
int x_smem(const Magnet* m) {
  return ((m->ty + (m->ty + 1) / 2) * xrow_stride(m->P[0], m->ty) + m->P[0]) * (int)sizeof(float2);
}
// y lengths of the warp-column y/z pass (k_yzw)
bool yz_warp(int Py) { return Py >= 64 && Py <= 1024; }
// y length 2048 with z lengths up to 8: warp pairs (k_yzw64)
bool yz_pair(int Py, int Pz) { return Py == 2048 && Pz <= 8; }
int yzw_threads_of(int Pz) { return Pz == 16 ? 384 : 256; }
int yz_smem_of(int nz, int nkx, int Py, int Pz) {
  return (nkx * 3 * nz * (yz_warp(Py) || yz_pair(Py, Pz) ? qlen(Py) : plen(Py)) + Py) * (int)sizeof(float2);
}
int yz_smem(const Magnet* m) { return yz_smem_of(m->dev.n[2], m->nkx, m->P[1], m->P[2]); }
// y/z class of a magnet: 20 + log2 Pz for the warp-pair pass of y length 2048
// (z lengths up to 8), 15 + log2 Pz for the warp-column pass of y length 1024,
// 10 + log2 Pz for y lengths 64 .. 512, else log2 Pz, plus 5 for y transforms
// longer than 2048 (which need the radix-16 form).  The FFT plan of a magnet
// depends on its own lengths only, so it computes the same alone and in any
// batch.
int yz_class(const Magnet* m) {
  if (yz_pair(m->P[1], m->P[2])) return 20 + ilog2(m->P[2]);
  if (m->P[1] == 1024) return 15 + ilog2(m->P[2]);
  if (yz_warp(m->P[1])) return 10 + ilog2(m->P[2]);
  return ilog2(m->P[2]) + (m->P[1] > 2048 ? 5 : 0);
}
constexpr int YZ_THREADS = 384;

// Tile shapes.  Row tiles: about 4096 points of the padded x transform per
// tile (4 rows above Px = 1024; up to TY_MAX rows of short transforms), 8 rows
// at Px = 1024 and 16 at Px = 512 (12 units of 1024 values for the 12 warps
// of the warp-row FFT), or
// of the row itself without demag.  y/z blocks: enough consecutive kx that a
// block holds about YZ_VPT * YZ_THREADS points of y transforms.
// Rows per tile are even (or the single row of ny = 1): the x passes pack the
// z components of rows 2k and 2k+1 into one complex FFT, so tiles that start
// on even rows give every magnet the same arithmetic whatever its tiling (the
// same results alone and in any batch).
int even_rows(int t, int ny) { return ny <= 1 ? 1 : std::max(2, t & ~1); }
int choose_ty(int ny, int len) {
  const int t = len == 1024 ? 8 : len == 512 ? 16 : len > 1024 ? 4 : std::min(TY_MAX, std::max(1, 4096 / len));
  return even_rows(std::max(1, std::min(t, ny)), ny);
}
int choose_nkx(int nz, int Py, int Pz, int Fh) {
  // warp pairs (y length 2048): up to 12 columns, two per pair of the 6 pairs
  if (yz_pair(Py, Pz)) return std::max(1, std::min(Fh, 12 / (3 * nz)));
  // warp columns (y lengths 64 .. 1024): 32 values per thread, one 1024-value unit per warp
  const int pts = yz_warp(Py) ? 32 * yzw_threads_of(Pz) : YZ_VPT * YZ_THREADS;
  return std::max(1, std::min(Fh, pts / (3 * nz * Py)));
}

int ycols_smem(const Magnet* m) { return (m->ncy * plen(m->P[1]) + m->P[1]) * (int)sizeof(float2); }
int zmul_smem(const Magnet* m) { return (3 * m->nkz * plen(m->P[2]) + m->P[2]) * (int)sizeof(float2); }

// The three passes of the split y/z path (radix-8 forms when the lengths allow);
// magnets with the tensor-core y transforms take k_ydft_tc (work list tcw)
// instead of k_ycols.
constexpr int TC_GRID_PER_SM = TC_BLOCKS_PER_SM;
mpx_status launch_split(mpx_engine* e, const Work* ycw, int nyc, const Work* zmw, int nzm, int smem_y, int smem_z,
                        int max_py, int max_pz, int stage, int gate, const Work* tcw = nullptr, int ntc = 0) {
  if (nyc <= 0 && ntc <= 0) return MPX_OK;
  const bool ry = max_py <= 2048, rz = max_pz <= 2048;
  const int gtc = std::min(ntc, TC_GRID_PER_SM * e->n_sm);
  if (ntc > 0) {
    k_ydft_tc<-1><<<gtc, 128, TC_SMEM, e->stream>>>(e->d_mags, e->d_groups, tcw, ntc, stage, gate, e->d_dftB);
    e->launches++;
  }
  if (nyc > 0) {
    if (ry)
      k_ycols<-1, 3><<<nyc, YZ_THREADS, smem_y, e->stream>>>(e->d_mags, e->d_groups, ycw, stage, gate, e->d_tw);
    else
      k_ycols<-1, 4><<<nyc, YZ_THREADS, smem_y, e->stream>>>(e->d_mags, e->d_groups, ycw, stage, gate, e->d_tw);
    e->launches++;
  }
  if (rz)
    k_zmul<3><<<nzm, YZ_THREADS, smem_z, e->stream>>>(e->d_mags, e->d_groups, zmw, stage, gate, e->d_tw);
  else
    k_zmul<4><<<nzm, YZ_THREADS, smem_z, e->stream>>>(e->d_mags, e->d_groups, zmw, stage, gate, e->d_tw);
  e->launches++;
  if (nyc > 0) {
    if (ry)
      k_ycols<1, 3><<<nyc, YZ_THREADS, smem_y, e->stream>>>(e->d_mags, e->d_groups, ycw, stage, gate, e->d_tw);
    else
      k_ycols<1, 4><<<nyc, YZ_THREADS, smem_y, e->stream>>>(e->d_mags, e->d_groups, ycw, stage, gate, e->d_tw);
    e->launches++;
  }
  if (ntc > 0) {
    k_ydft_tc<1><<<gtc, 128, TC_SMEM, e->stream>>>(e->d_mags, e->d_groups, tcw, ntc, stage, gate, e->d_dftB);
    e->launches++;
  }
  return MPX_OK;
}

// Launch with programmatic dependent launch allowed: the kernel may start its
// prologue while the previous kernel of the stream finishes (the kernel calls
// pdl_wait before it reads anything the earlier kernels write).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, int smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// y/z launch for one class: warp columns for y lengths 64 .. 1024 (k_yzw);
// else the radix-8 form for z lengths up to 8 and y lengths up to 2048, the
// radix-16 form otherwise (k_yz)
mpx_status launch_yz(mpx_engine* e, int cls, const Work* work, int n, int smem, int stage, int gate) {
  if (n <= 0) return MPX_OK;
#define MPX_YZ(PZ, LR) \
  CUDA_TRY(launch_pdl(k_yz<PZ, LR>, n, YZ_THREADS, smem, e->stream, e->d_mags, e->d_groups, work, stage, gate, e->d_tw))
#define MPX_YZW(PZ) \
  CUDA_TRY(launch_pdl(k_yzw<PZ>, n, yzw_threads<PZ>(), smem, e->stream, e->d_mags, e->d_groups, work, stage, gate, \
                      e->d_tw))
#define MPX_YZW32(PZ) \
  CUDA_TRY(launch_pdl(k_yzw32<PZ>, n, yzw_threads<PZ>(), smem, e->stream, e->d_mags, e->d_groups, work, stage, gate, \
                      e->d_tw))
#define MPX_YZW64(PZ) \
  CUDA_TRY(launch_pdl(k_yzw64<PZ>, n, YZP_THREADS, smem, e->stream, e->d_mags, e->d_groups, work, stage, gate, e->d_tw))
  switch (cls) {
    case 0: MPX_YZ(1, 3); break;
    case 1: MPX_YZ(2, 3); break;
    case 2: MPX_YZ(4, 3); break;
    case 3: MPX_YZ(8, 3); break;
    case 5: MPX_YZ(1, 4); break;
    case 6: MPX_YZ(2, 4); break;
    case 7: MPX_YZ(4, 4); break;
    case 8: MPX_YZ(8, 4); break;
    case 10: MPX_YZW(1); break;
    case 11: MPX_YZW(2); break;
    case 12: MPX_YZW(4); break;
    case 13: MPX_YZW(8); break;
    case 14: MPX_YZW(16); break;
    case 15: MPX_YZW32(1); break;
    case 16: MPX_YZW32(2); break;
    case 17: MPX_YZW32(4); break;
    case 18: MPX_YZW32(8); break;
    case 19: MPX_YZW32(16); break;
    case 20: MPX_YZW64(1); break;
    case 21: MPX_YZW64(2); break;
    case 22: MPX_YZW64(4); break;
    case 23: MPX_YZW64(8); break;
    default: MPX_YZ(16, 4); break;  // 4 and 9 (z length 16)
  }
#undef MPX_YZ
#undef MPX_YZW
#undef MPX_YZW32
#undef MPX_YZW64
  e->launches++;
  return MPX_OK;
}
// The x-pass kernels of a launch: the PAIR forms (2048-point warp-pair rows
// compiled in) when one of its magnets has 2048-point x rows, else the forms
// without them (the shorter lengths keep their registers and code).
using XfwdFn = void (*)(const MagnetDev*, const GroupDev*, const Work*, int, int, const float*, const float2*);
using XinvFn = void (*)(const MagnetDev*, GroupDev*, const Work*, EpiArgs, const float2*);
XfwdFn xfwd_fn(bool combine, bool pair) {
  if (combine) return pair ? k_xfwd<true, true> : k_xfwd<true, false>;
  return pair ? k_xfwd<false, true> : k_xfwd<false, false>;
}
XinvFn xinv_fn(bool pair) { return pair ? k_xinv<true> : k_xinv<false>; }
bool x_pair_of(const Magnet* m) { return m->P[0] == 2048; }

int x_threads(const Magnet* m) {
  int rows = m->ty + (m->ty + 1) / 2;
  int t = (rows * m->P[0] + 7) / 8;  // 8 values per thread in the x FFTs
  t = ((t + 31) / 32) * 32;
  return std::min(X_THREADS_MAX, std::max(64, t));
}

// Tile shapes for magnets launched together: from each magnet's default
// (about 4096 points per x tile, 6144 per y/z block), halve the rows per tile
// and the kx per block, all magnets alike, while the launch would have fewer
// than two blocks per SM; small single solves then spread over the GPU and
// large batches keep their large tiles.
constexpr int SHAPE_MIN_BLOCKS = 2 * 148;
// div_x / div_yz (powers of two, from the autotuner; 1 otherwise) divide the
// default shapes before the rule.
void plan_shapes(const std::vector<Magnet*>& ms, int* ty, int* nkx, int div_x = 1, int div_yz = 1) {
  std::vector<int> t(ms.size()), k(ms.size());
  for (size_t i = 0; i < ms.size(); ++i) {
    t[i] = even_rows(ms[i]->ty_def / div_x, ms[i]->dev.n[1]);
    k[i] = std::max(1, ms[i]->nkx_def / div_yz);
  }
  for (;;) {
    long long blocks = 0;
    bool shrink = false;
    for (size_t i = 0; i < ms.size(); ++i) {
      blocks += (long long)ms[i]->dev.n[2] * ((ms[i]->dev.n[1] + t[i] - 1) / t[i]);
      shrink = shrink || t[i] > even_rows(1, ms[i]->dev.n[1]);
    }
    if (blocks >= SHAPE_MIN_BLOCKS || !shrink) break;
    for (size_t i = 0; i < ms.size(); ++i) t[i] = even_rows(t[i] / 2, ms[i]->dev.n[1]);
  }
  for (;;) {
    long long blocks = 0;
    bool shrink = false;
    for (size_t i = 0; i < ms.size(); ++i) {
      if (!ms[i]->demag || ms[i]->split) continue;
      blocks += (ms[i]->dev.Fh + k[i] - 1) / k[i];
      shrink = shrink || k[i] > 1;
    }
    if (blocks >= SHAPE_MIN_BLOCKS || !shrink) break;
    for (auto& v : k) v = std::max(1, v / 2);
  }
  for (size_t i = 0; i < ms.size(); ++i) {
    ty[i] = t[i];
    nkx[i] = k[i];
  }
}

// Rebuilds the row tiles and y/z work items of m for the given shapes, with its
// own device tables (the per-magnet evaluation path).
mpx_status retile(mpx_engine* e, Magnet* m, int ty, int nkx) {
  const MagnetDev& D = m->dev;
  m->ty = ty;
  m->nkx = nkx;
  m->ver++;  // the launch tables place this magnet's items again
  m->tiles.clear();
  m->kxw.clear();
  for (int z = 0; z < D.n[2]; ++z)
    for (int y0 = 0; y0 < D.n[1]; y0 += m->ty) m->tiles.push_back(Work{m->slot, z, y0, std::min(m->ty, D.n[1] - y0)});
  if (m->demag)
    for (int kx = 0; kx < D.Fh; kx += m->nkx) m->kxw.push_back(Work{m->slot, kx, std::min(m->nkx, D.Fh - kx), 0});
  MPX_TRY(upload_vec(e, &m->d_tiles, m->tiles));
  MPX_TRY(upload_vec(e, &m->d_kxw, m->kxw));
  return MPX_OK;
}

// The magnets of started groups (launched together); returns their total cells.
long long active_set(mpx_engine* e, std::vector<Magnet*>& act) {
  act.clear();
  for (auto& mp : e->mags) {
    if (!mp || mp->probe) continue;
    const Group* g = (mp->group >= 0 && mp->group < (int)e->groups.size()) ? e->groups[mp->group].get() : nullptr;
    if (g && g->active) act.push_back(mp.get());
  }
  long long cells = 0;
  for (Magnet* m : act) cells += m->dev.N;
  return cells;
}

mpx_status rebuild_tables(mpx_engine* e) {
  NvtxRange nvtx_range("rebuild_tables");
  {  // shapes for the set of magnets launched together
    std::vector<Magnet*> act;
    const long long cells = active_set(e, act);
    std::vector<int> ty(act.size()), nkx(act.size());
    // tuned divisors hold while the launched set keeps more than half of the cells
    // it had when they were measured (solves of a batch finish one by one)
    if (2 * cells <= e->tune_cells || cells > e->tune_cells) e->tune_div_x = e->tune_div_yz = 1;
    plan_shapes(act, ty.data(), nkx.data(), e->tune_div_x, e->tune_div_yz);
    for (size_t i = 0; i < act.size(); ++i)
      if (ty[i] != act[i]->ty || nkx[i] != act[i]->nkx) MPX_TRY(retile(e, act[i], ty[i], nkx[i]));
  }
  // the work lists each table should hold: the magnets of started groups
  // (finished and idle solves cost no blocks), in slot order
  const int NT = mpx_engine::TT_YZ0 + YZ_CLASSES;
  std::vector<std::pair<Magnet*, const std::vector<Work>*>> want[mpx_engine::TT_YZ0 + YZ_CLASSES];
  e->smem_ycols = e->smem_zmul = e->maxpy_split = e->maxpz_split = 0;
  e->smem_x = 0;
  e->nt_x = 256;
  e->x_pair = false;
  for (int c = 0; c < YZ_CLASSES; ++c) e->smem_yz[c] = 0;
  for (auto& mp : e->mags) {
    if (!mp || mp->probe) continue;  // probe grids of stray-field evaluations
    Magnet* m = mp.get();
    const Group* g = (m->group >= 0 && m->group < (int)e->groups.size()) ? e->groups[m->group].get() : nullptr;
    if (!g || !g->active) continue;
    if (m->demag) {
      want[mpx_engine::TT_DEMAG].push_back({m, &m->tiles});
      e->smem_x = std::max(e->smem_x, x_smem(m));
      if (m->split) {
        want[mpx_engine::TT_YCOLS].push_back({m, &m->ycw});
        want[mpx_engine::TT_TC].push_back({m, &m->tcw});
        want[mpx_engine::TT_ZMUL].push_back({m, &m->zmw});
        e->smem_ycols = std::max(e->smem_ycols, ycols_smem(m));
        e->smem_zmul = std::max(e->smem_zmul, zmul_smem(m));
        e->maxpy_split = std::max(e->maxpy_split, m->P[1]);
        e->maxpz_split = std::max(e->maxpz_split, m->P[2]);
      } else {
        const int cls = yz_class(m);
        want[mpx_engine::TT_YZ0 + cls].push_back({m, &m->kxw});
        e->smem_yz[cls] = std::max(e->smem_yz[cls], yz_smem(m));
      }
      e->nt_x = std::max(e->nt_x, x_threads(m));
      e->x_pair = e->x_pair || x_pair_of(m);
    } else {
      want[mpx_engine::TT_LOCAL].push_back({m, &m->tiles});
    }
  }
  // each table: holes for the magnets that left (or whose lists changed), the
  // newcomers appended, compaction when the holes outnumber the live entries,
  // and an upload of the changed entries only
  for (int t = 0; t < NT; ++t) {
    SlotTable& T = e->tt[t];
    std::unordered_map<uint64_t, std::pair<Magnet*, const std::vector<Work>*>> w;
    for (auto& pr : want[t])
      if (!pr.second->empty()) w[pr.first->uid] = pr;
    std::vector<uint64_t> gone;
    for (auto& kv : T.place) {
      auto it = w.find(kv.first);
      if (it == w.end() || it->second.first->ver != kv.second.ver) gone.push_back(kv.first);
    }
    for (uint64_t uid : gone) T.remove(uid);
    int add_len = 0;
    for (auto& pr : want[t])
      if (!pr.second->empty() && !T.place.count(pr.first->uid)) add_len += (int)pr.second->size();
    const int used_after = (int)T.items.size() + add_len, live_after = T.live + add_len;
    if (used_after > 64 && used_after - live_after > live_after) {  // compact, in slot order
      T.clear();
      for (auto& pr : want[t])
        if (!pr.second->empty()) T.add(pr.first->uid, pr.first->ver, *pr.second);
    } else {
      for (auto& pr : want[t])
        if (!pr.second->empty() && !T.place.count(pr.first->uid)) T.add(pr.first->uid, pr.first->ver, *pr.second);
    }
    while (!T.items.empty() && T.items.back().mag < 0) T.items.pop_back();  // trailing holes
    const int used = (int)T.items.size();
    if (used > T.cap) {  // grow: a new device array, everything uploaded
      const int nc = std::max({used, 2 * T.cap, 64});
      Work* nd = nullptr;
      MPX_TRY(palloc(e, (void**)&nd, sizeof(Work) * (size_t)nc));
      pfree(e, T.dev);  // stream-ordered after the attempts already queued
      T.dev = nd;
      T.cap = nc;
      T.dirty(0, used);
    }
    const int lo = std::max(0, T.dlo), hi = std::min(used, T.dhi);
    if (hi > lo)
      CUDA_TRY(cudaMemcpyAsync(T.dev + lo, T.items.data() + lo, sizeof(Work) * (size_t)(hi - lo),
                               cudaMemcpyHostToDevice, e->stream));
    T.dlo = 1 << 30;
    T.dhi = -1;
  }
  // groups with thermal noise never reuse k0 (GroupDev::thermal, read by the controller)
  e->any_thermal = false;
  for (auto& gp : e->groups) {
    if (!gp) continue;
    int th = 0;
    for (int id : gp->magnets) {
      Magnet* mm = get_mag(e, id);
      if (mm && (mm->dev.terms & FLAG_THERMAL)) th = 1;
    }
    if (th && gp->active) e->any_thermal = true;
    if (th != gp->thermal) {
      GroupDev G;
      MPX_TRY(read_group(e, gp->slot, &G));
      G.thermal = th;
      MPX_TRY(write_group(e, gp->slot, &G));
      gp->thermal = th;
    }
  }
  e->d_t_demag = e->tt[mpx_engine::TT_DEMAG].dev;
  e->n_t_demag = (int)e->tt[mpx_engine::TT_DEMAG].items.size();
  e->d_t_local = e->tt[mpx_engine::TT_LOCAL].dev;
  e->n_t_local = (int)e->tt[mpx_engine::TT_LOCAL].items.size();
  e->d_t_ycols = e->tt[mpx_engine::TT_YCOLS].dev;
  e->n_t_ycols = (int)e->tt[mpx_engine::TT_YCOLS].items.size();
  e->d_t_zmul = e->tt[mpx_engine::TT_ZMUL].dev;
  e->n_t_zmul = (int)e->tt[mpx_engine::TT_ZMUL].items.size();
  e->d_t_tc = e->tt[mpx_engine::TT_TC].dev;
  e->n_t_tc = (int)e->tt[mpx_engine::TT_TC].items.size();
  for (int c = 0; c < YZ_CLASSES; ++c) {
    e->d_kx_demag[c] = e->tt[mpx_engine::TT_YZ0 + c].dev;
    e->n_kx_demag[c] = (int)e->tt[mpx_engine::TT_YZ0 + c].items.size();
  }
  // Everything the attempt graphs take from the tables: their device arrays,
  // launch sizes and the launch shapes.  A solve that arrives or finishes in
  // an unchanged range of the tables leaves them as they are (no capture); a
  // changed launch size updates the captured graphs in place.
  std::vector<long long> sig;
  for (int t = 0; t < NT; ++t) sig.insert(sig.end(), {(long long)(uintptr_t)e->tt[t].dev, (long long)e->tt[t].items.size()});
  for (int c = 0; c < YZ_CLASSES; ++c) sig.push_back(e->smem_yz[c]);
  sig.insert(sig.end(), {e->smem_x, e->nt_x, e->x_pair ? 1 : 0, e->smem_ycols, e->smem_zmul, e->maxpy_split,
                         e->maxpz_split});
  e->tables_dirty = false;
  if (e->tables_valid && sig == e->tables_sig) return MPX_OK;
  e->tables_sig = std::move(sig);
  e->tables_valid = true;
  e->graph_dirty = true;
  return MPX_OK;
}

// Stray-field pairs: every ordered pair (A, B) of distinct magnets of one group
// with A an enabled source (msat not zero) and B an enabled destination gets
// the FP32 table of the Newell tensor (built in FP64, PBC images included) of
// their displacements; B gets a stray-field buffer and FLAG_STRAY.
mpx_status setup_magnet(mpx_engine* e, Magnet* m, const mpx_magnet_desc* d, bool keep_fields);
void release_all(mpx_engine* e, Magnet* m);

// Pairs whose direct sum would take at least this many cell interactions use
// the FFT form on the pair's kernel grid (periodic images included).
constexpr long long STRAY_FFT_MIN_INTERACTIONS = 1LL << 22;

// The FP32 table of the Newell tensor, with the periodic images of g, at the
// displacements O + j, j < K per axis (k_newell_reflayout's layout).  Where a
// displacement range reaches both signs the tensor is evaluated over the
// absolute displacements only and expanded by the components' parities
// (k_newell_expand_abs): for two overlapping grids a quarter to an eighth of
// the FP64 evaluations.
mpx_status build_pair_table(mpx_engine* e, const KernelGeom& g, const int K[3], const int O[3], float* out) {
  int A[3], L[3];
  long long lt = 1, kt = 1;
  for (int a = 0; a < 3; ++a) {
    const int lo = O[a], hi = O[a] + K[a] - 1;
    if (lo <= 0 && hi >= 0) {
      A[a] = 0;
      L[a] = std::max(-lo, hi) + 1;
    } else {
      A[a] = std::min(std::abs(lo), std::abs(hi));
      L[a] = std::max(std::abs(lo), std::abs(hi)) - A[a] + 1;
    }
    lt *= L[a];
    kt *= K[a];
  }
  if (2 * lt > kt) {
    k_newell_reflayout<<<148 * 8, 128, 0, e->stream>>>(out, g, K[0], K[1], K[2], O[0], O[1], O[2]);
    e->launches++;
  } else {
    float* abs_tab = nullptr;
    MPX_TRY(palloc(e, (void**)&abs_tab, sizeof(float) * 6 * (size_t)lt));
    k_newell_reflayout<<<148 * 8, 128, 0, e->stream>>>(abs_tab, g, L[0], L[1], L[2], A[0], A[1], A[2]);
    k_newell_expand_abs<<<148 * 8, 256, 0, e->stream>>>(out, abs_tab, K[0], K[1], K[2], O[0], O[1], O[2], A[0], A[1],
                                                        A[2], L[0], L[1], L[2]);
    e->launches += 2;
    pfree(e, abs_tab);
  }
  return MPX_OK;
}

// log2 of the FFT lengths of the pair grid n_A + n_B - 1 per axis; false when
// a length exceeds what the pair passes transform (4096 along x and y, 2048
// along z, where six kernel components share one block's shared memory).
bool pair_fft_lengths(const int nA[3], const int nB[3], int logP[3]) {
  for (int a = 0; a < 3; ++a) {
    const long long K = (long long)nA[a] + nB[a] - 1;
    int l = 0;
    while ((1LL << l) < K) ++l;
    if (l > (a == 2 ? 11 : 12)) return false;
    logP[a] = l;
  }
  return true;
}

// Launch shapes of the passes for `ncomp` components with input rows nin and
// output window rows nout (pairfft.cuh); rows per block fill one transform
// group of PF_POINTS points.
void pair_shapes(PairPlan& pl, int ncomp) {
  const PairFft& pf = pl.pf;
  const int Px = 1 << pf.logP[0], Py = 1 << pf.logP[1], Pz = 1 << pf.logP[2], Hx = Px / 2 + 1;
  auto cdiv = [](int a, int b) { return (a + b - 1) / b; };
  const int f2 = (int)sizeof(float2);
  pl.ry_f = std::max(1, std::min(pf.nin[1], PF_POINTS / Px));
  pl.g_xf = ncomp * pf.nin[2] * cdiv(pf.nin[1], pl.ry_f);
  pl.s_xf = (pl.ry_f * plen(Px) + Px) * f2;
  pl.zc_f = std::max(1, std::min(pf.nin[2], PF_POINTS / Py));
  pl.g_yf = Hx * ncomp * cdiv(pf.nin[2], pl.zc_f);
  pl.s_yf = (pl.zc_f * plen(Py) + Py) * f2;
  pl.tky = std::max(1, std::min(Py, PF_POINTS / (ncomp * Pz)));
  pl.g_z = Hx * cdiv(Py, pl.tky);
  pl.s_z = (ncomp * pl.tky * plen(Pz) + Pz) * f2;
  pl.zc_i = std::max(1, std::min(pf.nout[2], PF_POINTS / Py));
  pl.g_yi = Hx * ncomp * cdiv(pf.nout[2], pl.zc_i);
  pl.s_yi = (pl.zc_i * plen(Py) + Py) * f2;
  pl.ry_i = std::max(1, std::min(pf.nout[1], PF_POINTS / Px));
  pl.g_xi = ncomp * pf.nout[2] * cdiv(pf.nout[1], pl.ry_i);
  pl.s_xi = (pl.ry_i * plen(Px) + Px) * f2;
  const int syz = (3 * Pz * plen(Py) + Py) * f2;
  pl.s_yz = (ncomp == 3 && Pz <= 8 && syz <= SMEM_MAX - 8192) ? syz : 0;
}

void free_pair_plan(mpx_engine* e, PairPlan& pl) {
  pfree(e, pl.t);
  pfree(e, pl.ks);
  pl.t = pl.ks = nullptr;
}

// The plan of source A on the destination grid (nB, oB): FFT lengths, the
// buffers, and the kernel spectrum from the FP64-built table of the pair's
// displacements (periodic images of `gimg`: mastergrid and repetitions).
mpx_status build_pair_fft(mpx_engine* e, const Magnet* A, const int nB[3], const int oB[3], const KernelGeom& gimg,
                          PairPlan& pl) {
  PairFft& pf = pl.pf;
  if (!pair_fft_lengths(A->dev.n, nB, pf.logP)) return fail(MPX_ERR_UNSUPPORTED, "stray-field FFT grid too large");
  int K[3], O[3];
  for (int a = 0; a < 3; ++a) {
    K[a] = A->dev.n[a] + nB[a] - 1;
    O[a] = oB[a] - A->dev.o[a] - (A->dev.n[a] - 1);
  }
  const int Px = 1 << pf.logP[0], Py = 1 << pf.logP[1], Pz = 1 << pf.logP[2], Hx = Px / 2 + 1;
  const size_t vol = (size_t)Hx * Pz * Py;
  MPX_TRY(palloc(e, (void**)&pl.t, sizeof(float2) * 3 * vol));
  mpx_status st = palloc(e, (void**)&pl.ks, sizeof(float2) * 6 * vol);
  float* tab = nullptr;
  if (st == MPX_OK) st = palloc(e, (void**)&tab, sizeof(float) * 6 * (size_t)K[0] * K[1] * K[2]);
  if (st != MPX_OK) {
    free_pair_plan(e, pl);
    return st;
  }
  st = build_pair_table(e, gimg, K, O, tab);
  if (st != MPX_OK) {
    pfree(e, tab);
    free_pair_plan(e, pl);
    return st;
  }
  // kernel spectrum: the forward passes over the six tabulated components
  PairPlan kp;
  kp.pf = pf;
  kp.pf.t = pl.ks;
  kp.pf.ks = nullptr;
  for (int a = 0; a < 3; ++a) kp.pf.nin[a] = kp.pf.nout[a] = K[a];
  kp.pf.win[0] = kp.pf.win[1] = kp.pf.win[2] = 0;
  pair_shapes(kp, 6);
  k_pair_xfwd<true><<<kp.g_xf, PF_THREADS, kp.s_xf, e->stream>>>(e->d_mags, e->d_groups, -1, 0, 0, tab, kp.pf, 6,
                                                                  kp.ry_f, e->d_tw);
  k_pair_yfft<-1><<<kp.g_yf, PF_THREADS, kp.s_yf, e->stream>>>(e->d_mags, e->d_groups, -1, 0, 0, kp.pf, 6, kp.zc_f,
                                                                e->d_tw);
  k_pair_zmul<false><<<kp.g_z, PF_THREADS, kp.s_z, e->stream>>>(e->d_mags, e->d_groups, -1, 0, 0, kp.pf, 6, kp.tky,
                                                                 e->d_tw);
  e->launches += 3;
  pfree(e, tab);
  pf.t = pl.t;
  pf.ks = pl.ks;
  for (int a = 0; a < 3; ++a) {
    pf.nin[a] = A->dev.n[a];
    pf.win[a] = A->dev.n[a] - 1;
    pf.nout[a] = nB[a];
  }
  pf.scale = (float)(-1.25663706212e-6 / ((double)Px * Py * Pz));
  pair_shapes(pl, 3);
  const cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    free_pair_plan(e, pl);
    return fail(MPX_ERR_CUDA, std::string("stray-field FFT kernel: ") + cudaGetErrorString(ce));
  }
  return MPX_OK;
}

// The plan of source A on destination grid B with the images of g, from the
// cache of recent evaluations or built (the least recently used of
// PAIR_CACHE_MAX plans is released).  The kernel spectrum depends on the
// geometry only, so repeated evaluations of one StrayField reuse it.
constexpr int PAIR_CACHE_MAX = 2;
mpx_status cached_pair_plan(mpx_engine* e, const Magnet* A, const Magnet* B, const KernelGeom& g, PairPlan** out) {
  int key[18];
  for (int a = 0; a < 3; ++a) {
    key[a] = A->dev.n[a];
    key[3 + a] = A->dev.o[a];
    key[6 + a] = B->dev.n[a];
    key[9 + a] = B->dev.o[a];
    key[12 + a] = g.mg[a];
    key[15 + a] = g.pbc[a];
  }
  for (auto& c : e->pair_cache)
    if (std::memcmp(c.key, key, sizeof key) == 0 && c.cs[0] == g.cs[0] && c.cs[1] == g.cs[1] && c.cs[2] == g.cs[2]) {
      c.used = ++e->pair_cache_tick;
      *out = &c.plan;
      return MPX_OK;
    }
  if ((int)e->pair_cache.size() >= PAIR_CACHE_MAX) {
    auto lru = std::min_element(e->pair_cache.begin(), e->pair_cache.end(),
                                [](const mpx_engine::PairCacheEntry& x, const mpx_engine::PairCacheEntry& y) {
                                  return x.used < y.used;
                                });
    free_pair_plan(e, lru->plan);
    e->pair_cache.erase(lru);
  }
  mpx_engine::PairCacheEntry c;
  std::memcpy(c.key, key, sizeof key);
  for (int a = 0; a < 3; ++a) c.cs[a] = g.cs[a];
  MPX_TRY(build_pair_fft(e, A, B->dev.n, B->dev.o, g, c.plan));
  c.used = ++e->pair_cache_tick;
  e->pair_cache.push_back(c);
  *out = &e->pair_cache.back().plan;
  return MPX_OK;
}

// The five passes of one evaluation: the field of `src`'s state for `stage`
// into out (3 x N of `dst`, added with `add`); `gate` as the stage kernels.
void launch_pair_fft(mpx_engine* e, const PairPlan& pl, int src, int dst, int stage, int gate, int add, float* out) {
  const PairFft& pf = pl.pf;
  k_pair_xfwd<false><<<pl.g_xf, PF_THREADS, pl.s_xf, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, nullptr,
                                                                   pf, 3, pl.ry_f, e->d_tw);
  if (pl.s_yz > 0) {
    const int Hx = (1 << pf.logP[0]) / 2 + 1;
    switch (pf.logP[2]) {
      case 0: k_pair_yz<1><<<Hx, PF_THREADS, pl.s_yz, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, e->d_tw); break;
      case 1: k_pair_yz<2><<<Hx, PF_THREADS, pl.s_yz, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, e->d_tw); break;
      case 2: k_pair_yz<4><<<Hx, PF_THREADS, pl.s_yz, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, e->d_tw); break;
      default: k_pair_yz<8><<<Hx, PF_THREADS, pl.s_yz, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, e->d_tw); break;
    }
  } else {
    k_pair_yfft<-1><<<pl.g_yf, PF_THREADS, pl.s_yf, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, 3,
                                                                  pl.zc_f, e->d_tw);
    k_pair_zmul<true><<<pl.g_z, PF_THREADS, pl.s_z, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, 3,
                                                                  pl.tky, e->d_tw);
    k_pair_yfft<1><<<pl.g_yi, PF_THREADS, pl.s_yi, e->stream>>>(e->d_mags, e->d_groups, src, stage, gate, pf, 3,
                                                                 pl.zc_i, e->d_tw);
  }
  k_pair_xinv<<<pl.g_xi, PF_THREADS, pl.s_xi, e->stream>>>(e->d_mags, e->d_groups, dst, stage, gate, pf, pl.ry_i, add,
                                                           out, e->d_tw);
  e->launches += pl.launches();
}

mpx_status rebuild_pairs(mpx_engine* e) {
  NvtxRange nvtx_range("rebuild_pairs");
  for (auto& p : e->pairs) {
    pfree(e, p.k);
    free_pair_plan(e, p.plan);
  }
  e->pairs.clear();
  std::vector<bool> is_dst(e->mags.size(), false);
  for (auto& gp : e->groups) {
    if (!gp) continue;
    for (int b : gp->magnets)
      for (int a : gp->magnets) {
        if (a == b) continue;
        Magnet* A = get_mag(e, a);
        Magnet* B = get_mag(e, b);
        if (!A->stray_src || A->msat_zero || !B->stray_dst) continue;
        mpx_engine::Pair p;
        p.src = a;
        p.dst = b;
        p.k = nullptr;
        KernelGeom g;
        for (int ax = 0; ax < 3; ++ax) {
          p.tab.K[ax] = A->dev.n[ax] + B->dev.n[ax] - 1;
          p.tab.O[ax] = B->dev.o[ax] - A->dev.o[ax] - (A->dev.n[ax] - 1);
          g.n[ax] = B->dev.n[ax];
          g.mg[ax] = B->dev.mg[ax];
          g.pbc[ax] = B->pbc_rep[ax];
          g.cs[ax] = B->cs_d[ax];
        }
        int logP[3];
        if ((long long)A->dev.N * B->dev.N >= STRAY_FFT_MIN_INTERACTIONS && pair_fft_lengths(A->dev.n, B->dev.n, logP)) {
          MPX_TRY(build_pair_fft(e, A, B->dev.n, B->dev.o, g, p.plan));
          p.fft = true;
          p.launches = p.plan.launches();
          e->pairs.push_back(p);
          is_dst[b] = true;
          continue;
        }
        const size_t KK = (size_t)p.tab.K[0] * p.tab.K[1] * p.tab.K[2];
        MPX_TRY(palloc(e, (void**)&p.k, sizeof(float) * 6 * KK));
        MPX_TRY(build_pair_table(e, g, p.tab.K, p.tab.O, p.k));
        p.tab.k = p.k;
        e->pairs.push_back(p);
        is_dst[b] = true;
      }
  }
  for (size_t i = 0; i < e->mags.size(); ++i) {
    Magnet* m = e->mags[i].get();
    if (!m || m->probe) continue;
    unsigned terms = m->terms_base;
    if (i < is_dst.size() && is_dst[i]) {
      if (!m->hstray) MPX_TRY(palloc(e, (void**)&m->hstray, sizeof(float) * 3 * (size_t)m->dev.N));
      terms |= TERM_EXT | FLAG_STRAY;
    } else if (m->hstray) {
      pfree(e, m->hstray);
      m->hstray = nullptr;
    }
    if (terms != m->dev.terms || m->dev.hstray != m->hstray) {
      m->dev.terms = terms;
      m->dev.hstray = m->hstray;
      MPX_TRY(upload_magnet_desc(e, m));
    }
  }
  e->pairs_dirty = false;
  e->graph_dirty = true;
  const cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("stray-field tables: ") + cudaGetErrorString(ce));
  return MPX_OK;
}

// Stray fields of the sources of `dst` (all destinations when dst < 0) for `stage`.
mpx_status launch_pairs(mpx_engine* e, int dst, int stage, int gate) {
  std::vector<int> seen;
  for (const auto& p : e->pairs) {
    if (dst >= 0 && p.dst != dst) continue;
    const bool add = std::find(seen.begin(), seen.end(), p.dst) != seen.end();
    if (!add) seen.push_back(p.dst);
    Magnet* B = get_mag(e, p.dst);
    if (p.fft) {
      launch_pair_fft(e, p.plan, p.src, p.dst, stage, gate, add ? 1 : 0, B->hstray);
      continue;
    }
    k_stray_pair<<<(B->dev.N + 255) / 256, 256, 0, e->stream>>>(e->d_mags, e->d_groups, p.src, p.dst, p.tab, stage,
                                                                gate, add ? 1 : 0, B->hstray);
    e->launches++;
  }
  return MPX_OK;
}

// ------------------------------------------------ demag kernel construction
mpx_status build_kernel_spectrum(mpx_engine* e, Magnet* m) {
  MagnetDev& d = m->dev;
  KernelGeom g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = d.n[a];
    g.mg[a] = m->kkey_mg[a];
    g.pbc[a] = m->kkey_pbc[a];
    g.cs[a] = m->kkey_cs[a];
  }
  const long long noct = (long long)d.n[0] * d.n[1] * d.n[2];
  const long long PP = (long long)m->P[0] * m->P[1] * m->P[2];
  double* oct = nullptr;
  double2 *f0 = nullptr, *f1 = nullptr;
  mpx_status ast = palloc(e, (void**)&oct, sizeof(double) * 6 * noct);
  if (ast == MPX_OK) ast = palloc(e, (void**)&f0, sizeof(double2) * PP);
  if (ast == MPX_OK) ast = palloc(e, (void**)&f1, sizeof(double2) * PP);
  if (ast != MPX_OK) {
    pfree(e, oct);
    pfree(e, f0);
    return fail(MPX_ERR_NOMEM, "demag kernel construction: out of device memory");
  }
  const int grid = 148 * 8;
  k_newell_octant<<<grid, 128, 0, e->stream>>>(oct, g);
  e->launches++;
  const int kcomp = d.kcomp;
  const int comps6[6] = {0, 1, 2, 3, 4, 5};
  const double pref = -MU0_D / (double)PP;
  for (int kc = 0; kc < kcomp; ++kc) {
    const int c = comps6[kc];
    k_kernel_expand<<<grid, 256, 0, e->stream>>>(f0, oct, c, g, m->P[0], m->P[1], m->P[2]);
    e->launches++;
    double2 *in = f0, *out = f1;
    for (int axis = 0; axis < 3; ++axis) {
      for (int Ns = 1; Ns < m->P[axis]; Ns <<= 1) {
        k_fft64_pass<<<grid, 256, 0, e->stream>>>(in, out, m->P[0], m->P[1], m->P[2], axis, Ns);
        e->launches++;
        std::swap(in, out);
      }
    }
    k_kernel_extract<<<grid, 256, 0, e->stream>>>(m->kspec, in, kc, kcomp, m->P[0], m->P[1], m->P[2], pref);
    e->launches++;
  }
  cudaError_t st = cudaGetLastError();
  pfree(e, oct);
  pfree(e, f0);
  pfree(e, f1);
  cudaError_t st2 = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("kernel build launch: ") + cudaGetErrorString(st));
  if (st2 != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("kernel build: ") + cudaGetErrorString(st2));
  m->kspec_ready = true;
  return MPX_OK;
}

// ------------------------------------------------------- parameter upload
mpx_status load_scalar(mpx_engine* e, Magnet* m, DScalar* out, const mpx_scalar& s, int N) {
  out->u = (float)s.uniform;
  out->p = nullptr;
  if (s.cells) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, sizeof(float) * (size_t)N));
    CUDA_TRY(cudaMemcpyAsync(p, s.cells, sizeof(float) * (size_t)N, cudaMemcpyHostToDevice, e->stream));
    out->p = (const float*)p;
  }
  return MPX_OK;
}
mpx_status load_vector(mpx_engine* e, Magnet* m, DVector* out, const mpx_vector& s, int N) {
  for (int c = 0; c < 3; ++c) out->u[c] = (float)s.uniform[c];
  out->p = nullptr;
  if (s.cells) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, sizeof(float) * 3 * (size_t)N));
    CUDA_TRY(cudaMemcpyAsync(p, s.cells, sizeof(float) * 3 * (size_t)N, cudaMemcpyHostToDevice, e->stream));
    out->p = (const float*)p;
  }
  return MPX_OK;
}

bool scalar_zero(const mpx_scalar& s) { return !s.cells && s.uniform == 0.0; }
bool vector_zero(const mpx_vector& s) {
  return !s.cells && s.uniform[0] == 0.0 && s.uniform[1] == 0.0 && s.uniform[2] == 0.0;
}

mpx_status validate_desc(const mpx_magnet_desc* d) {
  if (!d) return fail(MPX_ERR_INVALID, "null magnet description");
  for (int a = 0; a < 3; ++a) {
    if (d->size[a] <= 0) return fail(MPX_ERR_INVALID, "grid size must be positive");
    if (d->cellsize[a] <= 0) return fail(MPX_ERR_INVALID, "The cell size should be larger than 0");
    if (d->pbc_repetitions[a] < 0) return fail(MPX_ERR_INVALID, "Number of pbcRepetitions should not be negative.");
    if ((d->mastergrid_size[a] == 0) != (d->pbc_repetitions[a] == 0))
      return fail(MPX_ERR_INVALID, "0 in size of mastergrid should match 0 in pbcRepetitions.");
    if (d->mastergrid_size[a] > 0) {  // core/world.cpp inMastergrid
      const int d1 = d->origin[a] - d->mastergrid_origin[a];
      const int d2 = d1 + d->size[a] - d->mastergrid_size[a];
      if (d1 < 0 || d2 > 0)
        return fail(MPX_ERR_RANGE, "Can not add magnet because the grid does not fit in the mastergrid ");
    }
  }
  const long long N = (long long)d->size[0] * d->size[1] * d->size[2];
  if (N >= (1LL << 31) / 3) return fail(MPX_ERR_UNSUPPORTED, "grid too large for 32-bit cell indices");
  return MPX_OK;
}

// Fill the parameter part of the device description from d (allocating per-cell arrays).
mpx_status load_params(mpx_engine* e, Magnet* m, const mpx_magnet_desc* d) {
  MagnetDev& D = m->dev;
  const int N = D.N;
  MPX_TRY(load_scalar(e, m, &D.msat, d->msat, N));
  MPX_TRY(load_scalar(e, m, &D.aex, d->aex, N));
  MPX_TRY(load_scalar(e, m, &D.alpha, d->alpha, N));
  MPX_TRY(load_scalar(e, m, &D.ku1, d->ku1, N));
  MPX_TRY(load_scalar(e, m, &D.ku2, d->ku2, N));
  MPX_TRY(load_scalar(e, m, &D.frozen, d->frozen_spins, N));
  MPX_TRY(load_vector(e, m, &D.anisU, d->anis_u, N));
  MPX_TRY(load_vector(e, m, &D.bias, d->bias_magnetic_field, N));
  MPX_TRY(load_scalar(e, m, &D.kc1, d->kc1, N));
  MPX_TRY(load_scalar(e, m, &D.kc2, d->kc2, N));
  MPX_TRY(load_scalar(e, m, &D.kc3, d->kc3, N));
  MPX_TRY(load_vector(e, m, &D.anisC1, d->anis_c1, N));
  MPX_TRY(load_vector(e, m, &D.anisC2, d->anis_c2, N));
  MPX_TRY(load_scalar(e, m, &D.pol, d->pol, N));
  MPX_TRY(load_scalar(e, m, &D.xi, d->xi, N));
  MPX_TRY(load_scalar(e, m, &D.lambda_, d->lambda, N));
  MPX_TRY(load_scalar(e, m, &D.epsp, d->epsilon_prime, N));
  MPX_TRY(load_scalar(e, m, &D.flt, d->free_layer_thickness, N));
  MPX_TRY(load_vector(e, m, &D.jcur, d->jcur, N));
  MPX_TRY(load_vector(e, m, &D.fixl, d->fixed_layer, N));
  D.fl_below = d->fixed_layer_below ? 1 : 0;
  MPX_TRY(load_scalar(e, m, &D.temp, d->temperature, N));
  D.seed = d->thermal_seed;
  // physics/thermalnoise.cu:60-66: 2 kB gamma_LL / cell volume (KB, GAMMALL of physics/constants.hpp)
  D.noise_pref = (float)(2.0 * 1.38064852e-23 * 1.7595e11 / (d->cellsize[0] * d->cellsize[1] * d->cellsize[2]));
  for (int c = 0; c < 9; ++c) MPX_TRY(load_scalar(e, m, &D.dmi[c], d->dmi[c], N));
  D.inter_u = (float)d->inter_exchange;
  D.scale_u = (float)d->scale_exchange;
  D.inter_lut = nullptr;
  D.scale_lut = nullptr;
  const int L = d->lut_regions * (d->lut_regions - 1) / 2;
  if (d->inter_exchange_lut && L > 0) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, sizeof(float) * L));
    CUDA_TRY(cudaMemcpyAsync(p, d->inter_exchange_lut, sizeof(float) * L, cudaMemcpyHostToDevice, e->stream));
    D.inter_lut = (const float*)p;
  }
  if (d->scale_exchange_lut && L > 0) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, sizeof(float) * L));
    CUDA_TRY(cudaMemcpyAsync(p, d->scale_exchange_lut, sizeof(float) * L, cudaMemcpyHostToDevice, e->stream));
    D.scale_lut = (const float*)p;
  }
  D.geom = nullptr;
  m->ngeo = N;
  if (d->geometry) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, (size_t)N));
    CUDA_TRY(cudaMemcpyAsync(p, d->geometry, (size_t)N, cudaMemcpyHostToDevice, e->stream));
    D.geom = (const unsigned char*)p;
    m->geom = (unsigned char*)p;
    int ng = 0;
    for (int i = 0; i < N; ++i) ng += d->geometry[i] ? 1 : 0;
    m->ngeo = ng;
  } else {
    m->geom = nullptr;
  }
  D.reg = nullptr;
  if (d->regions) {
    void* p;
    MPX_TRY(dalloc(e, m, &p, sizeof(unsigned) * (size_t)N));
    CUDA_TRY(cudaMemcpyAsync(p, d->regions, sizeof(unsigned) * (size_t)N, cudaMemcpyHostToDevice, e->stream));
    D.reg = (const unsigned*)p;
  }
  // terms that are assured zero are skipped (physics/*AssuredZero)
  const bool msat0 = scalar_zero(d->msat);
  unsigned terms = 0;
  const bool inter0 = !d->inter_exchange_lut && d->inter_exchange == 0.0;
  const bool scale0 = !d->scale_exchange_lut && d->scale_exchange == 0.0;
  if (!((scalar_zero(d->aex) && inter0) || scale0 || msat0)) terms |= TERM_EXCH;
  bool dmi0 = true;
  for (int c = 0; c < 9; ++c) dmi0 = dmi0 && scalar_zero(d->dmi[c]);
  if (!(dmi0 || msat0)) terms |= TERM_DMI;
  // physics/anisotropy.cu:9-23: uniaxial unless assured zero, else cubic unless assured zero
  const bool uni0 = (scalar_zero(d->ku1) && scalar_zero(d->ku2)) || vector_zero(d->anis_u) || msat0;
  const bool cub0 = (scalar_zero(d->kc1) && scalar_zero(d->kc2) && scalar_zero(d->kc3)) ||
                    (vector_zero(d->anis_c1) && vector_zero(d->anis_c2)) || msat0;
  if (!uni0) terms |= TERM_ANIS;
  else if (!cub0) terms |= TERM_ANIS | FLAG_CUBIC;
  // physics/stt.cu:9-24: Slonczewski unless assured zero, else Zhang-Li unless assured zero
  const bool j0 = vector_zero(d->jcur);
  const bool zl0 = d->zhang_li_off || msat0 || j0 || scalar_zero(d->pol);
  const bool sl0 = d->slonczewski_off || msat0 || j0 || scalar_zero(d->free_layer_thickness) ||
                   vector_zero(d->fixed_layer) ||
                   (scalar_zero(d->epsilon_prime) && (scalar_zero(d->lambda) || scalar_zero(d->pol)));
  if (!sl0) terms |= FLAG_STT_SL;
  else if (!zl0) terms |= FLAG_STT_ZL;
  if (!scalar_zero(d->temperature) && !msat0) terms |= FLAG_THERMAL;  // physics/thermalnoise.cu:16-18
  const bool wb0 = e->wb[0] == 0 && e->wb[1] == 0 && e->wb[2] == 0;
  if (!(wb0 && vector_zero(d->bias_magnetic_field))) terms |= TERM_EXT;
  if (!vector_zero(d->bias_magnetic_field)) terms |= FLAG_MAGNET_BIAS;
  if (d->enable_demag && !msat0) terms |= TERM_DEMAG;
  if (d->enable_openbc) terms |= FLAG_OPENBC;
  D.terms = terms;
  m->terms_base = terms;
  m->msat_zero = msat0;
  m->stray_src = !d->stray_source_off;
  m->stray_dst = !d->stray_destination_off;
  e->pairs_dirty = true;
  for (int c = 0; c < 3; ++c) D.wb[c] = (float)e->wb[c];
  // fast path: every parameter uniform, no geometry, no regions
  bool uniform = !d->geometry && !d->regions;
  for (const mpx_scalar* s : {&d->msat, &d->aex, &d->alpha, &d->ku1, &d->ku2, &d->frozen_spins, &d->kc1, &d->kc2,
                               &d->kc3})
    uniform = uniform && !s->cells;
  for (int c = 0; c < 9; ++c) uniform = uniform && !d->dmi[c].cells;
  uniform = uniform && !d->anis_u.cells && !d->bias_magnetic_field.cells && !d->anis_c1.cells && !d->anis_c2.cells;
  D.fast = uniform ? 1 : 0;
  if (uniform) {
    const float a = D.aex.u, ms = D.msat.u;
    for (int ax = 0; ax < 3; ++ax) D.fe[ax] = (2 * a) * D.w[ax];  // 2 A w, as physics/exchange.cu:100
    for (int c = 0; c < 9; ++c) D.fd[c] = D.dmi[c].u;
    D.fa = a;
    D.finv_2a = (a == 0.0f) ? 0.0f : 0.5f / a;
    D.finv_ms = (ms == 0.0f) ? 0.0f : 1.0f / ms;
    D.fk1 = D.ku1.u;
    D.fk2 = D.ku2.u;
    const float ux = D.anisU.u[0], uy = D.anisU.u[1], uz = D.anisU.u[2];
    const float nu = std::sqrt(ux * ux + uy * uy + uz * uz);
    const float s = (nu == 0.0f) ? 0.0f : 1.0f / nu;
    D.fu[0] = s * ux;
    D.fu[1] = s * uy;
    D.fu[2] = s * uz;
    for (int c = 0; c < 3; ++c) D.fb[c] = (terms & FLAG_MAGNET_BIAS) ? D.wb[c] + D.bias.u[c] : D.wb[c];
    // cubic axes: normalised c1, c2 and c3 = c1 x c2 (not renormalised), as the reference kernel
    float c1[3], c2[3];
    for (int k = 0; k < 2; ++k) {
      const float* u = k == 0 ? D.anisC1.u : D.anisC2.u;
      const float n = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      const float sc = (n == 0.0f) ? 0.0f : 1.0f / n;
      float* o = k == 0 ? c1 : c2;
      for (int c = 0; c < 3; ++c) o[c] = sc * u[c];
    }
    const float c3[3] = {c1[1] * c2[2] - c1[2] * c2[1], c1[2] * c2[0] - c1[0] * c2[2], c1[0] * c2[1] - c1[1] * c2[0]};
    for (int c = 0; c < 3; ++c) {
      D.fc[0][c] = c1[c];
      D.fc[1][c] = c2[c];
      D.fc[2][c] = c3[c];
    }
    D.fkc[0] = D.kc1.u;
    D.fkc[1] = D.kc2.u;
    D.fkc[2] = D.kc3.u;
  }
  return MPX_OK;
}

mpx_status setup_magnet(mpx_engine* e, Magnet* m, const mpx_magnet_desc* d, bool keep_fields) {
  // keep the state buffers and the spectrum when only parameters change
  MagnetDev& D = m->dev;
  float* old_fields = m->fields;
  float2* old_spec = m->spec;
  float* old_kspec = m->kspec;
  const bool same_grid = keep_fields && D.n[0] == d->size[0] && D.n[1] == d->size[1] && D.n[2] == d->size[2];
  bool kernel_same = same_grid && m->kspec_ready;
  for (int a = 0; a < 3; ++a) {
    kernel_same = kernel_same && m->kkey_mg[a] == d->mastergrid_size[a] && m->kkey_pbc[a] == d->pbc_repetitions[a] &&
                  m->kkey_cs[a] == d->cellsize[a];
  }
  // release parameter allocations (everything except fields/spec/kspec which are tracked separately)
  for (void* p : m->allocs) pfree(e, p);
  e->bytes -= m->bytes;
  m->allocs.clear();
  m->bytes = 0;
  if (!same_grid) {
    pfree(e, old_fields);
    pfree(e, old_spec);
    pfree(e, old_kspec);
    e->bytes -= m->fields_bytes + m->spec_bytes + m->kspec_bytes;
    m->fields_bytes = m->spec_bytes = m->kspec_bytes = 0;
    m->fields = nullptr;
    m->spec = nullptr;
    m->kspec = nullptr;
    m->kspec_ready = false;
    old_fields = nullptr;
    old_spec = nullptr;
    old_kspec = nullptr;
    kernel_same = false;
  }
  for (int a = 0; a < 3; ++a) {
    D.n[a] = d->size[a];
    D.o[a] = d->origin[a];
    D.mg[a] = d->mastergrid_size[a];
    D.mgo[a] = d->mastergrid_origin[a];
    D.cs[a] = (float)d->cellsize[a];
    m->pbc_rep[a] = d->pbc_repetitions[a];
    m->cs_d[a] = d->cellsize[a];
    const float c = (float)d->cellsize[a];
    D.w[a] = 1.0f / (c * c);
    D.inv_cs[a] = 1.0f / c;
  }
  D.N = D.n[0] * D.n[1] * D.n[2];
  D.group = m->group;
  MPX_TRY(load_params(e, m, d));
  const int N = D.N;
  // demag plan
  m->demag = (D.terms & TERM_DEMAG) != 0;
  for (int a = 0; a < 3; ++a) {
    m->P[a] = padded(D.n[a]);
    D.P[a] = m->P[a];
    D.logP[a] = ilog2(m->P[a]);
  }
  D.Fh = m->P[0] / 2 + 1;
  D.kcomp = (m->P[2] == 1) ? 4 : 6;
  m->ty_def = choose_ty(D.n[1], m->demag ? m->P[0] : D.n[0]);
  m->nkx_def = m->demag ? choose_nkx(D.n[2], m->P[1], m->P[2], D.Fh) : 1;
  m->ty = m->ty_def;
  m->nkx = m->nkx_def;
  plan_shapes({m}, &m->ty, &m->nkx);  // alone (plain evaluations, single solves)
  m->split = false;
  if (m->demag) {
    if (m->P[0] > X_VPT * X_THREADS_MAX || m->P[1] > std::min(MAX_FFT, YZ_VPT * YZ_THREADS))
      return fail(MPX_ERR_UNSUPPORTED, "demag: padded FFT length above 2048 along x or 4096 along y "
                                       "(grid side above 1024 along x or 2048 along y)");
    // thick magnets (nz > 8) and long y transforms of many columns take the split y/z path;
    // so do y lengths 1024 and 2048 when the engine runs the tensor-core y transforms
    m->tc = e->dft_mode == MPX_DFT_TF32X3 && (m->P[1] == 1024 || m->P[1] == 2048) && !m->probe;
    m->split = m->tc || m->P[2] > 16 || yz_smem(m) > SMEM_DYN_MAX;
    if (m->split) {
      if (m->P[2] > MAX_FFT) return fail(MPX_ERR_UNSUPPORTED, "demag: padded FFT length above 4096 along z");
      m->ncy = std::max(1, std::min(D.Fh * 3 * D.n[2], (YZ_VPT * YZ_THREADS) / m->P[1]));
      m->nkz = std::max(1, std::min(m->P[1], (YZ_VPT * YZ_THREADS) / (3 * m->P[2])));
      if (ycols_smem(m) > SMEM_DYN_MAX || zmul_smem(m) > SMEM_DYN_MAX)
        return fail(MPX_ERR_UNSUPPORTED, "demag: y/z transforms exceed shared memory");
    }
    if (x_smem(m) > SMEM_DYN_MAX) return fail(MPX_ERR_UNSUPPORTED, "demag: x-pass tile exceeds shared memory");
  }
  // field buffers (9 x 3N floats) and spectrum
  size_t fbytes = sizeof(float) * 9 * 3 * (size_t)N;
  if (!old_fields) {
    MPX_TRY(dalloc(e, nullptr, (void**)&old_fields, fbytes));
    CUDA_TRY(cudaMemsetAsync(old_fields, 0, fbytes, e->stream));
    m->fields_bytes = (int64_t)fbytes;
  }
  m->fields = old_fields;
  for (int b = 0; b < 9; ++b) D.buf[b] = old_fields + (size_t)b * 3 * N;
  const size_t sbytes = sizeof(float2) * (size_t)D.Fh * 3 * D.n[1] * D.n[2];  // S[kx][c][z][y]
  if (m->demag && !old_spec) {
    MPX_TRY(dalloc(e, nullptr, (void**)&old_spec, sbytes));
    m->spec_bytes = (int64_t)sbytes;
  }
  m->spec = old_spec;
  D.spec = old_spec;
  // split path: the y-transformed spectrum (no state kept between evaluations)
  pfree(e, m->tspec);
  e->bytes -= m->tspec_bytes;
  m->tspec = nullptr;
  m->tspec_bytes = 0;
  if (m->demag && m->split) {
    const size_t tb = sizeof(float2) * (size_t)D.Fh * 3 * D.n[2] * m->P[1];
    MPX_TRY(palloc(e, (void**)&m->tspec, tb));
    m->tspec_bytes = (int64_t)tb;
    e->bytes += (int64_t)tb;
  }
  D.tspec = m->tspec;
  const size_t kbytes = sizeof(float) * (size_t)D.Fh * (m->P[1] / 2 + 1) * (m->P[2] / 2 + 1) * D.kcomp;
  if (m->demag && !old_kspec) {
    MPX_TRY(dalloc(e, nullptr, (void**)&old_kspec, kbytes));
    m->kspec_bytes = (int64_t)kbytes;
    kernel_same = false;
  }
  m->kspec = old_kspec;
  D.kspec = old_kspec;
  if (m->demag && !kernel_same) {
    for (int a = 0; a < 3; ++a) {
      m->kkey_n[a] = D.n[a];
      m->kkey_mg[a] = d->mastergrid_size[a];
      m->kkey_pbc[a] = d->pbc_repetitions[a];
      m->kkey_cs[a] = d->cellsize[a];
    }
    m->kspec_ready = false;
    MPX_TRY(build_kernel_spectrum(e, m));
  }
  // tiles
  MPX_TRY(retile(e, m, m->ty, m->nkx));
  m->ycw.clear();
  m->zmw.clear();
  m->tcw.clear();
  if (m->demag && m->split) {
    const int ncols = D.Fh * 3 * D.n[2];
    if (m->tc) {
      const int cpt = 4096 / m->P[1];  // columns per 128-sequence tile: 4 at Py = 1024, 2 at 2048
      for (int c0 = 0; c0 < ncols; c0 += cpt) m->tcw.push_back(Work{m->slot, c0, std::min(cpt, ncols - c0), 0});
    } else {
      for (int c0 = 0; c0 < ncols; c0 += m->ncy) m->ycw.push_back(Work{m->slot, c0, std::min(m->ncy, ncols - c0), 0});
    }
    for (int kx = 0; kx < D.Fh; ++kx)
      for (int ky0 = 0; ky0 < m->P[1]; ky0 += m->nkz)
        m->zmw.push_back(Work{m->slot, kx, ky0, std::min(m->nkz, m->P[1] - ky0)});
  }
  MPX_TRY(upload_vec(e, &m->d_ycw, m->ycw));
  MPX_TRY(upload_vec(e, &m->d_zmw, m->zmw));
  MPX_TRY(upload_vec(e, &m->d_tcw, m->tcw));
  m->ver++;
  MPX_TRY(upload_magnet_desc(e, m));
  e->tables_dirty = true;
  return MPX_OK;
}

// The tableau lives in one __constant__ symbol per device, shared by all
// engines on that device; it is re-uploaded on the engine's stream before
// every run so that engines with different methods never see a stale one.
mpx_status upload_tableau(mpx_engine* e, int method) {
  TableauDev t = make_tableau(method);
  CUDA_TRY(cudaMemcpyToSymbolAsync(c_tab, &t, sizeof(t), 0, cudaMemcpyHostToDevice, e->stream));
  e->tab_method = method;
  return MPX_OK;
}

mpx_status check_launch(mpx_engine* e, const char* what) {
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) return fail(MPX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(st));
  (void)e;
  return MPX_OK;
}

// --------------------------------------------------- field evaluation
// Evaluate quantity q of magnet m into the device buffer out.
mpx_status eval_into(mpx_engine* e, Magnet* m, int q, float* out) {
  // the magnet's own tiles (any tiling gives the same numbers); the attempt
  // tables are not needed here
  if (e->pairs_dirty) MPX_TRY(rebuild_pairs(e));
  const int N = m->dev.N;
  if (q == MPX_Q_MAGNETIZATION) {
    GroupDev G;
    MPX_TRY(read_group(e, m->group, &G));
    CUDA_TRY(cudaMemcpyAsync(out, m->dev.buf[G.map[0]], sizeof(float) * 3 * (size_t)N, cudaMemcpyDeviceToDevice,
                             e->stream));
    return MPX_OK;
  }
  EpiArgs ea;
  ea.mode = EPI_EVAL;
  ea.stage = 0;
  ea.quantity = q;
  ea.fsal_err = 0;
  ea.gate = 0;
  ea.out = out;
  ea.msrc = nullptr;
  const bool needs_demag = (q == MPX_Q_EFFECTIVE_FIELD || q == MPX_Q_DEMAG_FIELD || q == MPX_Q_TORQUE ||
                            q == MPX_Q_LLG_TORQUE || q == MPX_Q_DAMPING_TORQUE || q == MPX_Q_DEMAG_ENERGY_DENSITY ||
                            q == MPX_Q_TOTAL_ENERGY_DENSITY);
  const int ntile = (int)m->tiles.size();
  if (m->hstray) MPX_TRY(launch_pairs(e, m->slot, 0, 0));  // stray fields of the other magnets' states
  if (m->demag && needs_demag) {
    const int sx = x_smem(m), syz = yz_smem(m), nt = x_threads(m);
    xfwd_fn(false, x_pair_of(m))<<<ntile, nt, sx, e->stream>>>(e->d_mags, e->d_groups, m->d_tiles, 0, 0, nullptr,
                                                                e->d_tw);
    if (m->split)
      MPX_TRY(launch_split(e, m->d_ycw, (int)m->ycw.size(), m->d_zmw, (int)m->zmw.size(), ycols_smem(m),
                           zmul_smem(m), m->P[1], m->P[2], 0, 0, m->d_tcw,
                           (int)m->tcw.size()));
    else
      MPX_TRY(launch_yz(e, yz_class(m), m->d_kxw, (int)m->kxw.size(), syz, 0, 0));
    CUDA_TRY(launch_pdl(xinv_fn(x_pair_of(m)), ntile, nt, sx, e->stream, e->d_mags, e->d_groups, m->d_tiles, ea,
                        e->d_tw));
    e->launches += 2;
  } else {
    k_local<<<ntile, 256, 0, e->stream>>>(e->d_mags, e->d_groups, m->d_tiles, ea);
    e->launches += 1;
  }
  return check_launch(e, "eval");
}

// One Runge-Kutta attempt for every running group (core/rungekutta.cpp:39-83).
mpx_status launch_attempt(mpx_engine* e, const TableauDev& T, int first_stage) {
  const int S = T.S;
  for (int s = first_stage; s < S; ++s) {
    EpiArgs ea;
    ea.mode = EPI_STAGE;
    ea.stage = s;
    ea.quantity = 0;
    ea.fsal_err = (T.fsal && s == S - 1) ? 1 : 0;
    ea.gate = 1;
    ea.out = nullptr;
    ea.msrc = nullptr;
    // stage states: combination fused into the x-forward pass, or k_combine
    if (e->n_t_demag > 0) {
      if (s == 0)
        xfwd_fn(false, e->x_pair)<<<e->n_t_demag, e->nt_x, e->smem_x, e->stream>>>(e->d_mags, e->d_groups,
                                                                                    e->d_t_demag, 0, 1, nullptr,
                                                                                    e->d_tw);
      else if (s == first_stage)  // after the step controller: fully serialised
        xfwd_fn(true, e->x_pair)<<<e->n_t_demag, e->nt_x, e->smem_x, e->stream>>>(e->d_mags, e->d_groups,
                                                                                   e->d_t_demag, s, 1, nullptr,
                                                                                   e->d_tw);
      else  // after the previous stage (the group state is constant within an attempt)
        CUDA_TRY(launch_pdl(xfwd_fn(true, e->x_pair), e->n_t_demag, e->nt_x, e->smem_x, e->stream, e->d_mags,
                            e->d_groups, e->d_t_demag, s, 1, (const float*)nullptr, e->d_tw));
      e->launches++;
    }
    if (e->n_t_local > 0 && s > 0) {
      k_combine<<<e->n_t_local, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_local, s, 0);
      e->launches++;
    }
    // stray fields of the stage states of the other magnets
    MPX_TRY(launch_pairs(e, -1, s, 1));
    if (e->n_t_demag > 0) {
      for (int c = 0; c < YZ_CLASSES; ++c)
        MPX_TRY(launch_yz(e, c, e->d_kx_demag[c], e->n_kx_demag[c], e->smem_yz[c], s, 1));
      MPX_TRY(launch_split(e, e->d_t_ycols, e->n_t_ycols, e->d_t_zmul, e->n_t_zmul, e->smem_ycols, e->smem_zmul,
                           e->maxpy_split, e->maxpz_split, s, 1, e->d_t_tc, e->n_t_tc));
      CUDA_TRY(launch_pdl(xinv_fn(e->x_pair), e->n_t_demag, e->nt_x, e->smem_x, e->stream, e->d_mags, e->d_groups,
                          e->d_t_demag, ea, e->d_tw));
      e->launches++;
    }
    if (e->n_t_local > 0) {
      k_local<<<e->n_t_local, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_local, ea);
      e->launches++;
    }
  }
  if (!T.fsal) {
    if (e->n_t_demag > 0) {
      k_combine<<<e->n_t_demag, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_demag, S, 1);
      e->launches++;
    }
    if (e->n_t_local > 0) {
      k_combine<<<e->n_t_local, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_local, S, 1);
      e->launches++;
    }
  }
  const int ng = (int)e->groups.size();
  k_controller<<<(ng + 127) / 128, 128, 0, e->stream>>>(e->d_groups, ng);
  e->launches++;
  // sampled run: <m> of the group's magnets into the rows the controller marked due
  if (e->sampling_group >= 0) {
    Group* sg = get_group(e, e->sampling_group);
    for (size_t j = 0; sg && j < sg->magnets.size(); ++j) {
      const Magnet* m = get_mag(e, sg->magnets[j]);
      if (!m) continue;
      k_sample_partial<<<256, 256, 0, e->stream>>>(e->d_mags, e->d_groups, m->slot, e->d_red);
      k_sample_final<<<1, 32, 0, e->stream>>>(e->d_mags, e->d_groups, m->slot, e->d_red, 256, (long long)m->ngeo,
                                             1 + 3 * (int)j);
      e->launches += 2;
    }
  }
  return check_launch(e, "attempt");
}

mpx_status prepare_run(mpx_engine* e, int method) {
  if (e->pairs_dirty) MPX_TRY(rebuild_pairs(e));
  if (e->tables_dirty) MPX_TRY(rebuild_tables(e));
  MPX_TRY(upload_tableau(e, method));
  return MPX_OK;
}

// Captures one attempt (from `first_stage` on) as an executable graph.
// Captures one attempt into *out.  When *out already holds an attempt graph of
// the same shape (the same kernels in the same order; a solve that arrives or
// finishes changes only grid sizes and table pointers), the executable graph
// is updated in place (cudaGraphExecUpdate) instead of being instantiated
// again.
mpx_status capture_attempt(mpx_engine* e, const TableauDev& T, int first_stage, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const int64_t before = e->launches;
  mpx_status st = launch_attempt(e, T, first_stage);
  cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  e->launches = before;
  if (st != MPX_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ce != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  if (*out) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(*out, g, &info) == cudaSuccess) {
      cudaGraphDestroy(g);
      e->graph_updates++;
      return MPX_OK;
    }
    (void)cudaGetLastError();  // the update was refused: instantiate anew
    cudaGraphExecDestroy(*out);
    *out = nullptr;
  }
  ce = cudaGraphInstantiate(out, g, 0);
  e->graph_instantiations++;
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
  return MPX_OK;
}

// Kernel launches of one attempt from `first_stage` on (for the launch counter).
int attempt_launches(const mpx_engine* e, const TableauDev& T, int first_stage) {
  const int S = T.S, ns = S - first_stage;
  int nyz = 0;
  for (int c = 0; c < YZ_CLASSES; ++c) nyz += e->n_kx_demag[c] > 0 ? 1 : 0;
  if (e->n_t_ycols > 0) nyz += 3;
  int npair = 0;
  for (const auto& p : e->pairs) npair += p.launches;
  int per = 1 + npair * ns + 2 * e->samp_magnets;  // controller, stray-field pairs, samples
  if (e->n_t_demag > 0) per += (2 + nyz) * ns + (T.fsal ? 0 : 1);
  if (e->n_t_local > 0) per += ns + (ns - (first_stage == 0 ? 1 : 0)) + (T.fsal ? 0 : 1);
  return per;
}

// Replays `n` attempts through the CUDA graphs of one attempt.  With an FSAL
// method only the first attempt after a state change evaluates stage 0 (every
// started group then holds its k0); the others replay the graph without it.
mpx_status run_attempts(mpx_engine* e, int method, int n) {
  MPX_TRY(prepare_run(e, method));
  const TableauDev T = make_tableau(method);
  if (e->graph_dirty || e->graph_method != method || !e->graph) {
    MPX_TRY(capture_attempt(e, T, 0, &e->graph));
    if (T.fsal) {
      MPX_TRY(capture_attempt(e, T, 1, &e->graph_nok0));
    } else if (e->graph_nok0) {
      cudaGraphExecDestroy(e->graph_nok0);
      e->graph_nok0 = nullptr;
    }
    e->graph_method = method;
    e->graph_dirty = false;
  }
  const int per_full = attempt_launches(e, T, 0), per_nok0 = attempt_launches(e, T, 1);
  for (int i = 0; i < n; ++i) {
    const bool full = e->need_stage0 || !e->graph_nok0 || e->any_thermal;
    CUDA_TRY(cudaGraphLaunch(full ? e->graph : e->graph_nok0, e->stream));
    e->launches += full ? per_full : per_nok0;
    e->need_stage0 = false;
  }
  return MPX_OK;
}

mpx_status sensible_timestep(mpx_engine* e, Group* g, double* out) {
  // core/timesolver.cpp:37-47: sensibleFactor / max|torque| over the group's magnets
  if (g->magnets.empty()) {
    *out = 0.0;
    return MPX_OK;
  }
  double gmax = 0;
  for (int id : g->magnets) {
    Magnet* m = get_mag(e, id);
    const int N = m->dev.N;
    MPX_TRY(ensure_scratch(e, sizeof(float) * 3 * (size_t)N));
    MPX_TRY(eval_into(e, m, g->torque_kind ? MPX_Q_DAMPING_TORQUE : MPX_Q_TORQUE, e->d_scratch));
    const int nb = 256;
    k_reduce_partial<<<nb, 256, 0, e->stream>>>(e->d_scratch, N, 3, m->geom, 1, e->d_red);
    k_reduce_final<<<1, 32, 0, e->stream>>>(e->d_red, nb, 1, e->d_redout);
    e->launches += 2;
    double r[3];
    CUDA_TRY(cudaMemcpyAsync(r, e->d_redout, sizeof(r), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    gmax = std::max(gmax, r[0]);
  }
  *out = (gmax == 0) ? g->sp.sensible_timestep_default : g->sp.sensible_factor / gmax;
  return MPX_OK;
}

void fill_group_params(GroupDev& G, const mpx_solver_params& sp) {
  G.max_error = sp.max_error;
  G.headroom = sp.headroom;
  G.lower = sp.lower_bound;
  G.upper = sp.upper_bound;
  G.adaptive = sp.adaptive;
}

// Blocks until the group leaves the running state.
mpx_status drive_group(mpx_engine* e, Group* g) {
  NvtxRange nvtx_range("drive_group");
  int chunk = 1;
  for (;;) {
    MPX_TRY(run_attempts(e, g->sp.method, chunk));
    GroupDev G;
    MPX_TRY(read_group(e, g->slot, &G));
    if (G.status != GS_RUNNING) {
      g->active = false;
      e->tables_dirty = true;
    }
    if (G.status == GS_FAILED) {
      G.status = GS_IDLE;
      G.finished_flag = 0;
      MPX_TRY(write_group(e, g->slot, &G));
      return fail(MPX_ERR_RUNTIME, "time integration failed: the error estimate is NaN");
    }
    if (G.status != GS_RUNNING) {
      G.status = GS_IDLE;
      G.finished_flag = 0;
      MPX_TRY(write_group(e, g->slot, &G));
      return MPX_OK;
    }
    // attempts queued after the group has finished launch their kernels for
    // nothing: no more than the steps left of steps(n), or of run() at the
    // current time step (the final shortened step included)
    int left = 16;
    if (G.mode == 1) {
      left = (int)std::min<long long>(16, std::max<long long>(1, G.steps_left));
    } else if (G.mode == 0 && G.dt > 0) {
      const double r = (G.t_stop - G.t) / G.dt;
      left = (G.phase == 1 || r < 1.0) ? 1 : (r < 15.0 ? (int)r + 1 : 16);
    }
    chunk = std::max(1, std::min(std::min(chunk * 2, 16), left));
  }
}

mpx_status set_m_device(mpx_engine* e, Magnet* m, const float* src_dev) {
  GroupDev G;
  MPX_TRY(read_group(e, m->group, &G));
  const int N = m->dev.N;
  k_normalize_into<<<(N + 255) / 256, 256, 0, e->stream>>>(m->dev.buf[G.map[0]], src_dev, N, m->geom);
  e->launches++;
  MPX_TRY(check_launch(e, "set m"));
  G.k0_valid = 0;
  MPX_TRY(write_group(e, m->group, &G));
  return MPX_OK;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

const char* mpx_version(void) { return "mpx 0.1 (sm_100a)"; }
const char* mpx_last_error(void) { return g_last_error.c_str(); }

int mpx_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

mpx_status mpx_engine_create(int device, mpx_engine** out) {
  if (!out) return fail(MPX_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int n = mpx_device_count();
  if (n <= 0) return fail(MPX_ERR_NODEVICE, "no CUDA device available");
  if (device < 0 || device >= n) return fail(MPX_ERR_RANGE, "device index out of range");
  DeviceGuard guard(device);
  auto e = std::make_unique<mpx_engine>();
  e->device = device;
  CUDA_TRY(cudaDeviceGetAttribute(&e->n_sm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
  e->stream = e->own;
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CUDA_TRY(cudaMemPoolCreate(&e->pool, &props));
    uint64_t keep = UINT64_MAX;
    CUDA_TRY(cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  // twiddle table exp(-2 pi i k / 4096), computed in FP64
  std::vector<float2> tw(TW_N);
  for (int k = 0; k < TW_N; ++k) {
    const double a = -2.0 * M_PI * k / TW_N;
    tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  CUDA_TRY(cudaMalloc(&e->d_tw, sizeof(float2) * TW_N));
  CUDA_TRY(cudaMemcpy(e->d_tw, tw.data(), sizeof(float2) * TW_N, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&e->d_red, sizeof(double) * 3 * 1024));
  CUDA_TRY(cudaMalloc(&e->d_redout, sizeof(double) * 4));  // 3 reduction results, or the 4 of k_min_final
  // large dynamic shared memory and the max-shared carveout for the FFT kernels
  const void* fft_kernels[] = {(const void*)k_xfwd<false, false>, (const void*)k_xfwd<true, false>,
                               (const void*)k_xinv<false>, (const void*)k_xfwd<false, true>,
                               (const void*)k_xfwd<true, true>, (const void*)k_xinv<true>,
                               (const void*)k_yz<1, 4>, (const void*)k_yz<2, 4>, (const void*)k_yz<4, 4>,
                               (const void*)k_yz<8, 4>, (const void*)k_yz<16, 4>, (const void*)k_yz<1, 3>,
                               (const void*)k_yz<2, 3>, (const void*)k_yz<4, 3>, (const void*)k_yz<8, 3>,
                               (const void*)k_ycols<-1, 3>, (const void*)k_ycols<-1, 4>, (const void*)k_ycols<1, 3>,
                               (const void*)k_ycols<1, 4>, (const void*)k_zmul<3>, (const void*)k_zmul<4>,
                               (const void*)k_yzw<1>, (const void*)k_yzw<2>, (const void*)k_yzw<4>,
                               (const void*)k_yzw<8>, (const void*)k_yzw<16>, (const void*)k_yzw32<1>,
                               (const void*)k_yzw32<2>, (const void*)k_yzw32<4>, (const void*)k_yzw32<8>,
                               (const void*)k_yzw32<16>, (const void*)k_yzw64<1>, (const void*)k_yzw64<2>,
                               (const void*)k_yzw64<4>, (const void*)k_yzw64<8>, (const void*)k_pair_xfwd<true>,
                               (const void*)k_pair_xfwd<false>, (const void*)k_pair_yfft<-1>,
                               (const void*)k_pair_yfft<1>, (const void*)k_pair_zmul<true>,
                               (const void*)k_pair_zmul<false>, (const void*)k_pair_xinv,
                               (const void*)k_pair_yz<1>, (const void*)k_pair_yz<2>, (const void*)k_pair_yz<4>,
                               (const void*)k_pair_yz<8>};
  // the DFT32 matrix of the tensor-core y transforms in its real 64 x 64 form
  // B[2 k + r][2 n + s] (output k, part r; input n, part s; forward, angle
  // 2 pi k n / 32): re <- cos re + sin im, im <- -sin re + cos im; split into
  // TF32 hi and lo (round to nearest, ties away, as cvt.rna.tf32.f32)
  {
    auto tf32 = [](double v) {
      float f = (float)v;
      uint32_t u;
      std::memcpy(&u, &f, 4);
      u = (u + 0x1000u) & 0xFFFFE000u;
      std::memcpy(&f, &u, 4);
      return f;
    };
    std::vector<float> B(2 * 64 * 64);
    for (int k = 0; k < 32; ++k)
      for (int n = 0; n < 32; ++n) {
        const double a = 2.0 * M_PI * ((k * n) % 32) / 32.0, c = std::cos(a), sn = std::sin(a);
        const double v[2][2] = {{c, sn}, {-sn, c}};
        for (int r = 0; r < 2; ++r)
          for (int q = 0; q < 2; ++q) {
            const int i = (2 * k + r) * 64 + 2 * n + q;
            const float hi = tf32(v[r][q]);
            B[i] = hi;
            B[4096 + i] = tf32(v[r][q] - (double)hi);
          }
      }
    CUDA_TRY(cudaMalloc(&e->d_dftB, sizeof(float) * B.size()));
    CUDA_TRY(cudaMemcpy(e->d_dftB, B.data(), sizeof(float) * B.size(), cudaMemcpyHostToDevice));
  }
  {
    const void* tck[] = {(const void*)k_ydft_tc<-1>, (const void*)k_ydft_tc<1>};
    for (const void* k : tck) CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
  }
  for (const void* k : fft_kernels) {
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, k));
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  SMEM_MAX - (int)fa.sharedSizeBytes));
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  }
  *out = e.release();
  return MPX_OK;
}

mpx_status mpx_engine_destroy(mpx_engine* e) {
  if (!e) return MPX_OK;
  DeviceGuard guard(e->device);
  cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->graph_nok0) cudaGraphExecDestroy(e->graph_nok0);
  for (auto& m : e->mags)
    if (m) release_all(e, m.get());
  for (auto& c : e->pair_cache) free_pair_plan(e, c.plan);
  e->pair_cache.clear();
  cudaFree(e->d_mags);
  cudaFree(e->d_groups);
  cudaFree(e->d_tw);
  cudaFree(e->d_dftB);
  cudaFree(e->d_red);
  cudaFree(e->d_redout);
  pfree(e, e->d_scratch);
  for (auto& t : e->tt) pfree(e, t.dev);  // the launch tables (d_t_* and d_kx_demag alias them)
  cudaStreamSynchronize(e->stream);
  if (e->pool) cudaMemPoolDestroy(e->pool);
  if (e->own) cudaStreamDestroy(e->own);
  delete e;
  return MPX_OK;
}

mpx_status mpx_engine_set_stream(mpx_engine* e, void* stream) {
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  DeviceGuard guard(e->device);
  // pool allocations and frees are ordered on the old stream: let them finish
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->stream = stream ? (cudaStream_t)stream : e->own;
  return MPX_OK;
}

mpx_status mpx_engine_set_dft(mpx_engine* e, int mode) {
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  if (mode != MPX_DFT_FP32 && mode != MPX_DFT_TF32X3) return fail(MPX_ERR_INVALID, "unknown DFT mode");
  for (auto& m : e->mags)
    if (m && !m->probe) return fail(MPX_ERR_INVALID, "set the DFT mode before adding magnets");
  e->dft_mode = mode;
  return MPX_OK;
}

mpx_status mpx_tc_timeout_selftest(unsigned int* timeouts) {
  if (!timeouts) return fail(MPX_ERR_INVALID, "null output");
  unsigned int before = 0;
  MPX_TRY(mpx_tc_status(&before));  // synchronises and clears
  k_tc_timeout_probe<<<1, 128>>>(1 << 14);
  CUDA_TRY(cudaGetLastError());
  MPX_TRY(mpx_tc_status(timeouts));
  return MPX_OK;
}

mpx_status mpx_tc_status(unsigned int* timeouts) {
  if (!timeouts) return fail(MPX_ERR_INVALID, "null output");
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpyFromSymbol(timeouts, g_tc_timeouts, sizeof(unsigned int)));
  const unsigned int zero = 0;
  CUDA_TRY(cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof zero));
  return MPX_OK;
}

mpx_status mpx_engine_synchronize(mpx_engine* e) {
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  DeviceGuard guard(e->device);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status mpx_engine_set_world_bias(mpx_engine* e, const double b[3]) {
  if (!e || !b) return fail(MPX_ERR_INVALID, "null argument");
  DeviceGuard guard(e->device);
  for (int c = 0; c < 3; ++c) e->wb[c] = b[c];
  const bool wb0 = b[0] == 0 && b[1] == 0 && b[2] == 0;
  for (auto& mp : e->mags) {
    if (!mp) continue;
    Magnet* m = mp.get();
    for (int c = 0; c < 3; ++c) m->dev.wb[c] = (float)b[c];
    const bool mb = (m->terms_base & FLAG_MAGNET_BIAS) != 0;
    if (wb0 && !mb) m->terms_base &= ~TERM_EXT;
    else m->terms_base |= TERM_EXT;
    // stray fields keep the external term on
    m->dev.terms = m->terms_base | (m->hstray ? (TERM_EXT | FLAG_STRAY) : 0u);
    for (int c = 0; c < 3; ++c) m->dev.fb[c] = mb ? m->dev.wb[c] + m->dev.bias.u[c] : m->dev.wb[c];
    MPX_TRY(upload_magnet_desc(e, m));
  }
  for (auto& g : e->groups)
    if (g) {
      GroupDev G;
      MPX_TRY(read_group(e, g->slot, &G));
      G.k0_valid = 0;
      MPX_TRY(write_group(e, g->slot, &G));
    }
  return MPX_OK;
}

mpx_status mpx_engine_memory(mpx_engine* e, int64_t* bytes) {
  if (!e || !bytes) return fail(MPX_ERR_INVALID, "null argument");
  *bytes = e->bytes;
  return MPX_OK;
}

mpx_status mpx_engine_graph_stats(mpx_engine* e, int64_t* instantiations, int64_t* updates) {
  if (!e || !instantiations || !updates) return fail(MPX_ERR_INVALID, "null engine / output");
  *instantiations = e->graph_instantiations;
  *updates = e->graph_updates;
  return MPX_OK;
}

mpx_status mpx_engine_launch_count(mpx_engine* e, int64_t* count) {
  if (!e || !count) return fail(MPX_ERR_INVALID, "null argument");
  *count = e->launches;
  return MPX_OK;
}

mpx_status mpx_group_create(mpx_engine* e, int* group) {
  if (!e || !group) return fail(MPX_ERR_INVALID, "null argument");
  DeviceGuard guard(e->device);
  int slot = -1;
  for (int i = 0; i < (int)e->groups.size(); ++i)
    if (!e->groups[i]) { slot = i; break; }
  if (slot < 0) {
    slot = (int)e->groups.size();
    e->groups.emplace_back();
  }
  MPX_TRY(ensure_group_capacity(e, slot));
  auto g = std::make_unique<Group>();
  g->slot = slot;
  GroupDev G;
  std::memset(&G, 0, sizeof(G));
  fill_group_params(G, g->sp);
  for (int b = 0; b < 9; ++b) G.map[b] = b;
  G.status = GS_IDLE;
  MPX_TRY(write_group(e, slot, &G));
  e->groups[slot] = std::move(g);
  e->graph_dirty = true;  // controller grid covers all group slots
  *group = slot;
  return MPX_OK;
}

mpx_status mpx_group_destroy(mpx_engine* e, int group) {
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  std::vector<int> ms = g->magnets;
  for (int id : ms) MPX_TRY(mpx_magnet_remove(e, id));
  GroupDev G;
  std::memset(&G, 0, sizeof(G));
  G.status = GS_IDLE;
  MPX_TRY(write_group(e, group, &G));
  e->groups[group].reset();
  return MPX_OK;
}

// Snapshot layout: header, then per magnet m and k0 (3N floats each).
struct GroupStateHeader {
  char magic[8];  // "MPXSTAT1"
  double t, dt;
  int64_t steps;
  int32_t k0_valid, nmag;
};

static int64_t group_state_bytes(mpx_engine* e, Group* g) {
  int64_t b = sizeof(GroupStateHeader) + sizeof(int64_t) * (int64_t)g->magnets.size();
  for (int id : g->magnets) b += 2 * (int64_t)sizeof(float) * 3 * get_mag(e, id)->dev.N;
  return b;
}

mpx_status mpx_group_state_bytes(mpx_engine* e, int group, int64_t* bytes) {
  Group* g = get_group(e, group);
  if (!g || !bytes) return fail(MPX_ERR_RANGE, "no such group / null output");
  *bytes = group_state_bytes(e, g);
  return MPX_OK;
}

mpx_status mpx_group_save(mpx_engine* e, int group, void* buf, int64_t bytes) {
  Group* g = get_group(e, group);
  if (!g || !buf) return fail(MPX_ERR_RANGE, "no such group / null buffer");
  if (bytes < group_state_bytes(e, g)) return fail(MPX_ERR_INVALID, "state buffer too small");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, g->slot, &G));
  GroupStateHeader h;
  std::memcpy(h.magic, "MPXSTAT1", 8);
  h.t = G.t;
  h.dt = G.dt;
  h.steps = G.steps;
  h.k0_valid = G.k0_valid;
  h.nmag = (int32_t)g->magnets.size();
  char* p = static_cast<char*>(buf);
  std::memcpy(p, &h, sizeof h);
  p += sizeof h;
  for (int id : g->magnets) {
    const int64_t n = get_mag(e, id)->dev.N;
    std::memcpy(p, &n, sizeof n);
    p += sizeof n;
  }
  for (int id : g->magnets) {
    Magnet* m = get_mag(e, id);
    const size_t b = sizeof(float) * 3 * (size_t)m->dev.N;
    CUDA_TRY(cudaMemcpyAsync(p, m->dev.buf[G.map[0]], b, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaMemcpyAsync(p + b, m->dev.buf[G.map[2]], b, cudaMemcpyDeviceToHost, e->stream));
    p += 2 * b;
  }
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status mpx_group_load(mpx_engine* e, int group, const void* buf, int64_t bytes) {
  Group* g = get_group(e, group);
  if (!g || !buf) return fail(MPX_ERR_RANGE, "no such group / null buffer");
  if (bytes < (int64_t)sizeof(GroupStateHeader)) return fail(MPX_ERR_INVALID, "state buffer too small");
  GroupStateHeader h;
  const char* p = static_cast<const char*>(buf);
  std::memcpy(&h, p, sizeof h);
  if (std::memcmp(h.magic, "MPXSTAT1", 8) != 0) return fail(MPX_ERR_INVALID, "not a group state");
  if (h.nmag != (int32_t)g->magnets.size() || bytes < group_state_bytes(e, g))
    return fail(MPX_ERR_INVALID, "the state does not match the magnets of the group");
  p += sizeof h;
  for (int id : g->magnets) {
    int64_t n;
    std::memcpy(&n, p, sizeof n);
    p += sizeof n;
    if (n != get_mag(e, id)->dev.N) return fail(MPX_ERR_INVALID, "the state does not match the magnets of the group");
  }
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, g->slot, &G));
  // a run in progress keeps controller state (the final-step phase, the time
  // step saved before it) that belongs to its own time line: loading another
  // time into it would mix the two
  if (G.status == GS_RUNNING) return fail(MPX_ERR_INVALID, "mpx_group_load: the group is running");
  for (int id : g->magnets) {
    Magnet* m = get_mag(e, id);
    const size_t b = sizeof(float) * 3 * (size_t)m->dev.N;
    CUDA_TRY(cudaMemcpyAsync(m->dev.buf[G.map[0]], p, b, cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(m->dev.buf[G.map[2]], p + b, b, cudaMemcpyHostToDevice, e->stream));
    p += 2 * b;
  }
  G.t = h.t;
  G.dt = h.dt;
  G.steps = h.steps;
  G.k0_valid = h.k0_valid;
  G.phase = 0;  // controller state of an earlier, finished run does not carry over
  G.dt_saved = 0.0;
  MPX_TRY(write_group(e, g->slot, &G));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status mpx_group_info_get(mpx_engine* e, int group, mpx_group_info* out) {
  Group* g = get_group(e, group);
  if (!g || !out) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  out->time = G.t;
  out->timestep = G.dt;
  out->steps = G.steps;
  out->rejected = G.rejected;
  out->evaluations = G.attempts;
  out->status = G.status;
  out->last_error = 0;
  out->max_torque = -1;
  return MPX_OK;
}

// mpx_magnet_add / mpx_magnet_add_state: `m0` (3N floats, host unless
// on_device) is the initial magnetisation, or NULL for the random one.
static mpx_status magnet_add_impl(mpx_engine* e, int group, const mpx_magnet_desc* d, const float* m0, int on_device,
                                  int* magnet) {
  NvtxRange nvtx_range("mpx_magnet_add");
  if (!e || !magnet) return fail(MPX_ERR_INVALID, "null argument");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  MPX_TRY(validate_desc(d));
  DeviceGuard guard(e->device);
  int slot = -1;
  for (int i = 0; i < (int)e->mags.size(); ++i)
    if (!e->mags[i]) { slot = i; break; }
  if (slot < 0) {
    slot = (int)e->mags.size();
    e->mags.emplace_back();
  }
  auto m = std::make_unique<Magnet>();
  std::memset(&m->dev, 0, sizeof(MagnetDev));
  m->slot = slot;
  m->group = group;
  m->uid = e->next_uid++;
  mpx_status st = setup_magnet(e, m.get(), d, false);
  if (st != MPX_OK) {
    std::string msg = g_last_error;
    release_all(e, m.get());
    e->mags[slot].reset();
    g_last_error = msg;
    return st;
  }
  // initial magnetisation: the given one, or normalised random vectors
  // generated on the device (the reference seeds its generator with the clock,
  // ferromagnet.cpp:62-76; here the seed is the magnet slot)
  const int n3 = 3 * m->dev.N;
  const float* src = m0;
  if (!m0 || !on_device) {
    MPX_TRY(ensure_scratch(e, sizeof(float) * (size_t)n3));
    if (m0) {
      CUDA_TRY(cudaMemcpyAsync(e->d_scratch, m0, sizeof(float) * (size_t)n3, cudaMemcpyHostToDevice, e->stream));
    } else {
      k_random_normal<<<std::min((n3 + 255) / 256, 148 * 16), 256, 0, e->stream>>>(
          e->d_scratch, n3, 0x5DEECE66Dull * (unsigned long long)(slot + 1));
      e->launches++;
    }
    src = e->d_scratch;
  }
  Magnet* mp = m.get();
  e->mags[slot] = std::move(m);
  g->magnets.push_back(slot);
  e->tables_dirty = true;
  MPX_TRY(set_m_device(e, mp, src));
  // core/timesolver.cpp:49-52: new equations -> sensible time step (adaptive solvers)
  if (g->sp.adaptive) {
    double dt;
    MPX_TRY(sensible_timestep(e, g, &dt));
    GroupDev G;
    MPX_TRY(read_group(e, group, &G));
    G.dt = dt;
    MPX_TRY(write_group(e, group, &G));
  }
  *magnet = slot;
  return MPX_OK;
}

mpx_status mpx_magnet_add(mpx_engine* e, int group, const mpx_magnet_desc* d, int* magnet) {
  return magnet_add_impl(e, group, d, nullptr, 0, magnet);
}

mpx_status mpx_magnet_add_state(mpx_engine* e, int group, const mpx_magnet_desc* d, const float* m0, int on_device,
                                int* magnet) {
  if (!m0) return fail(MPX_ERR_INVALID, "null initial magnetization");
  return magnet_add_impl(e, group, d, m0, on_device, magnet);
}

mpx_status mpx_magnet_update(mpx_engine* e, int magnet, const mpx_magnet_desc* d) {
  Magnet* m = get_mag(e, magnet);
  if (!m) return fail(MPX_ERR_RANGE, "no such magnet");
  MPX_TRY(validate_desc(d));
  DeviceGuard guard(e->device);
  MPX_TRY(setup_magnet(e, m, d, true));
  GroupDev G;
  MPX_TRY(read_group(e, m->group, &G));
  G.k0_valid = 0;
  MPX_TRY(write_group(e, m->group, &G));
  return MPX_OK;
}

mpx_status mpx_magnet_bytes(const mpx_magnet_desc* d, int64_t* resident, int64_t* transient) {
  if (!resident || !transient) return fail(MPX_ERR_INVALID, "null argument");
  MPX_TRY(validate_desc(d));
  const int64_t N = (int64_t)d->size[0] * d->size[1] * d->size[2];
  int64_t res = 4 * 9 * 3 * N;  // state, stage and scratch buffers (setup_magnet)
  for (const mpx_scalar* sc : {&d->msat, &d->aex, &d->alpha, &d->ku1, &d->ku2, &d->frozen_spins, &d->kc1, &d->kc2,
                                &d->kc3})
    if (sc->cells) res += 4 * N;
  if (d->anis_c1.cells) res += 12 * N;
  if (d->anis_c2.cells) res += 12 * N;
  for (const mpx_scalar* sc : {&d->pol, &d->xi, &d->lambda, &d->epsilon_prime, &d->free_layer_thickness})
    if (sc->cells) res += 4 * N;
  if (d->jcur.cells) res += 12 * N;
  if (d->temperature.cells) res += 4 * N;
  if (d->fixed_layer.cells) res += 12 * N;
  for (int c = 0; c < 9; ++c)
    if (d->dmi[c].cells) res += 4 * N;
  if (d->anis_u.cells) res += 12 * N;
  if (d->bias_magnetic_field.cells) res += 12 * N;
  if (d->geometry) res += N;
  if (d->regions) res += 4 * N;
  const int64_t L = (int64_t)d->lut_regions * (d->lut_regions - 1) / 2;
  if (L > 0) res += 4 * L * ((d->inter_exchange_lut ? 1 : 0) + (d->scale_exchange_lut ? 1 : 0));
  const bool demag = d->enable_demag && !scalar_zero(d->msat);
  const int ty = choose_ty(d->size[1], demag ? padded(d->size[0]) : d->size[0]);
  res += (int64_t)sizeof(Work) * d->size[2] * ((d->size[1] + ty - 1) / ty);
  int64_t tr = 12 * N;  // initial random state (engine scratch)
  if (demag) {
    int P[3];
    for (int a = 0; a < 3; ++a) P[a] = padded(d->size[a]);
    const int64_t Fh = P[0] / 2 + 1;
    const int kc = (P[2] == 1) ? 4 : 6;
    res += 8 * Fh * 3 * d->size[1] * d->size[2];                 // spectrum S[kx][c][z][y]
    res += 4 * Fh * (P[1] / 2 + 1) * (P[2] / 2 + 1) * kc;        // kernel spectrum
    const int nkx = choose_nkx(d->size[2], P[1], P[2], (int)Fh);
    res += (int64_t)sizeof(Work) * ((Fh + nkx - 1) / nkx);       // y/z work items
    const int yzs = yz_smem_of(d->size[2], nkx, P[1], P[2]);
    if (P[2] > 16 || yzs > SMEM_DYN_MAX) {  // split y/z path: T and its work items
      res += 8 * Fh * 3 * d->size[2] * P[1];
      const int64_t ncy = std::max<int64_t>(1, std::min<int64_t>(Fh * 3 * d->size[2], (YZ_VPT * YZ_THREADS) / P[1]));
      const int64_t nkz = std::max(1, std::min(P[1], (YZ_VPT * YZ_THREADS) / (3 * P[2])));
      res += (int64_t)sizeof(Work) * ((Fh * 3 * d->size[2] + ncy - 1) / ncy + Fh * ((P[1] + nkz - 1) / nkz));
    }
    tr += 8 * 6 * N + 2 * 16 * (int64_t)P[0] * P[1] * P[2];    // FP64 octant + two transform buffers
  }
  *resident = res;
  *transient = tr;
  return MPX_OK;
}

mpx_status mpx_magnet_remove(mpx_engine* e, int magnet) {
  Magnet* m = get_mag(e, magnet);
  if (!m || m->probe) return fail(MPX_ERR_RANGE, "no such magnet");
  DeviceGuard guard(e->device);
  // frees are stream-ordered: attempts queued before still see the buffers
  Group* g = get_group(e, m->group);
  if (g) g->magnets.erase(std::remove(g->magnets.begin(), g->magnets.end(), magnet), g->magnets.end());
  release_all(e, m);
  e->mags[magnet].reset();
  e->tables_dirty = true;
  e->pairs_dirty = true;
  return MPX_OK;
}

mpx_status mpx_magnet_set_m(mpx_engine* e, int magnet, const float* src, int on_device) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !src) return fail(MPX_ERR_INVALID, "no such magnet / null data");
  DeviceGuard guard(e->device);
  const size_t bytes = sizeof(float) * 3 * (size_t)m->dev.N;
  const float* dsrc = src;
  if (!on_device) {
    MPX_TRY(ensure_scratch(e, bytes));
    CUDA_TRY(cudaMemcpyAsync(e->d_scratch, src, bytes, cudaMemcpyHostToDevice, e->stream));
    dsrc = e->d_scratch;
  }
  return set_m_device(e, m, dsrc);
}

mpx_status mpx_magnet_get_m(mpx_engine* e, int magnet, float* out, int on_device) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !out) return fail(MPX_ERR_INVALID, "no such magnet / null data");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, m->group, &G));
  const size_t bytes = sizeof(float) * 3 * (size_t)m->dev.N;
  CUDA_TRY(cudaMemcpyAsync(out, m->dev.buf[G.map[0]], bytes,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status mpx_eval(mpx_engine* e, int magnet, int quantity, float* out, int on_device) {
  NvtxRange nvtx_range("mpx_eval");
  Magnet* m = get_mag(e, magnet);
  if (!m || (!out && on_device != 2)) return fail(MPX_ERR_INVALID, "no such magnet / null output");
  if (quantity < 0 || quantity >= MPX_Q_COUNT) return fail(MPX_ERR_INVALID, "unknown quantity");
  DeviceGuard guard(e->device);
  const int nc = MPX_Q_IS_SCALAR(quantity) ? 1 : 3;
  const size_t bytes = sizeof(float) * nc * (size_t)m->dev.N;
  float* dst = out;
  if (on_device == 2) {
    MPX_TRY(ensure_scratch(e, sizeof(float) * 3 * (size_t)m->dev.N));
    MPX_TRY(eval_into(e, m, quantity, e->d_scratch));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return MPX_OK;
  }
  if (!on_device) {
    MPX_TRY(ensure_scratch(e, sizeof(float) * 3 * (size_t)m->dev.N));
    dst = e->d_scratch;
  }
  MPX_TRY(eval_into(e, m, quantity, dst));
  if (!on_device) CUDA_TRY(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

static mpx_status reduce_quantity(mpx_engine* e, Magnet* m, int quantity, int op, double out[3]) {
  const int nc = MPX_Q_IS_SCALAR(quantity) ? 1 : 3;
  const int N = m->dev.N;
  MPX_TRY(ensure_scratch(e, sizeof(float) * 3 * (size_t)N));
  MPX_TRY(eval_into(e, m, quantity, e->d_scratch));
  const int nb = 256;
  k_reduce_partial<<<nb, 256, 0, e->stream>>>(e->d_scratch, N, nc, m->geom, op, e->d_red);
  k_reduce_final<<<1, 32, 0, e->stream>>>(e->d_red, nb, op, e->d_redout);
  e->launches += 2;
  MPX_TRY(check_launch(e, "reduce"));
  CUDA_TRY(cudaMemcpyAsync(out, e->d_redout, sizeof(double) * 3, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return MPX_OK;
}

mpx_status mpx_average(mpx_engine* e, int magnet, int quantity, double out[3]) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !out) return fail(MPX_ERR_INVALID, "no such magnet / null output");
  if (quantity < 0 || quantity >= MPX_Q_COUNT) return fail(MPX_ERR_INVALID, "unknown quantity");
  DeviceGuard guard(e->device);
  double r[3];
  MPX_TRY(reduce_quantity(e, m, quantity, 0, r));
  const int nc = MPX_Q_IS_SCALAR(quantity) ? 1 : 3;
  for (int c = 0; c < 3; ++c) out[c] = (c < nc && m->ngeo > 0) ? r[c] / m->ngeo : 0.0;
  return MPX_OK;
}

mpx_status mpx_max_norm(mpx_engine* e, int magnet, int quantity, double* out) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !out) return fail(MPX_ERR_INVALID, "no such magnet / null output");
  if (quantity < 0 || quantity >= MPX_Q_COUNT) return fail(MPX_ERR_INVALID, "unknown quantity");
  DeviceGuard guard(e->device);
  double r[3];
  MPX_TRY(reduce_quantity(e, m, quantity, 1, r));
  *out = r[0];
  return MPX_OK;
}

mpx_status mpx_energy(mpx_engine* e, int magnet, int quantity, double* out) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !out) return fail(MPX_ERR_INVALID, "no such magnet / null output");
  if (!MPX_Q_IS_SCALAR(quantity))
    return fail(MPX_ERR_INVALID, "energy needs an energy-density quantity");
  double avg[3];
  MPX_TRY(mpx_average(e, magnet, quantity, avg));
  *out = (double)m->dev.N * avg[0] * ((double)m->dev.cs[0] * m->dev.cs[1] * m->dev.cs[2]);
  return MPX_OK;
}

// StrayField(magnet, grid).eval() (physics/strayfield.cpp:45-82) and
// Magnet.stray_field_from_magnet(source).eval() (bindings/wrap_magnet.cpp:45-52):
// the field of `src`'s current state on a destination grid, by direct sum over
// the source cells (METHOD_BRUTE, physics/strayfieldbrute.cu:15-57: the FP64
// Newell tensor of the displacements with the world's periodic images,
// tabulated in FP32) or by FFT convolution of the same table on the pair's
// kernel grid (METHOD_FFT, the default of the reference,
// physics/strayfieldfft.cu; pairfft.cuh).
mpx_status mpx_stray_field(mpx_engine* e, int src, int dst_magnet, const int size[3], const int origin[3], int method,
                           float* out, int on_device) {
  if (!e || !out) return fail(MPX_ERR_INVALID, "null engine / output");
  if (method != MPX_STRAY_FFT && method != MPX_STRAY_BRUTE)
    return fail(MPX_ERR_INVALID, "Method should be \"fft\" or \"brute\"");
  Magnet* A = get_mag(e, src);
  if (!A || A->probe) return fail(MPX_ERR_RANGE, "no such source magnet");
  DeviceGuard guard(e->device);
  int dst = dst_magnet, tmp = -1;
  if (dst_magnet >= 0) {
    Magnet* B0 = get_mag(e, dst_magnet);
    if (!B0 || B0->probe) return fail(MPX_ERR_RANGE, "no such destination magnet");
    if (B0->group != A->group) return fail(MPX_ERR_RUNTIME, "Can not compute the magnetic field of the magnet");
  } else {
    if (!size || !origin) return fail(MPX_ERR_INVALID, "null grid");
    mpx_magnet_desc d;
    std::memset(&d, 0, sizeof d);
    for (int a = 0; a < 3; ++a) {
      if (size[a] <= 0) return fail(MPX_ERR_INVALID, "grid size must be positive");
      d.size[a] = size[a];
      d.origin[a] = origin[a];
      d.cellsize[a] = A->cs_d[a];
    }
    if ((long long)size[0] * size[1] * size[2] >= (1LL << 31) / 3)
      return fail(MPX_ERR_UNSUPPORTED, "grid too large for 32-bit cell indices");
    d.msat.uniform = 1.0;
    d.scale_exchange = 1.0;
    d.stray_source_off = d.stray_destination_off = 1;
    for (int i = 0; i < (int)e->mags.size(); ++i)
      if (!e->mags[i]) { tmp = i; break; }
    if (tmp < 0) {
      tmp = (int)e->mags.size();
      e->mags.emplace_back();
    }
    auto m = std::make_unique<Magnet>();
    std::memset(&m->dev, 0, sizeof(MagnetDev));
    m->slot = tmp;
    m->group = A->group;
    m->probe = true;  // a probe of the destination grid: in no group's tables
    m->uid = e->next_uid++;
    const mpx_status st = setup_magnet(e, m.get(), &d, false);
    if (st != MPX_OK) {
      std::string msg = g_last_error;
      release_all(e, m.get());
      g_last_error = msg;
      return st;
    }
    e->mags[tmp] = std::move(m);
    dst = tmp;
  }
  Magnet* B = get_mag(e, dst);
  const int NB = B->dev.N;
  float* dout = out;
  mpx_status st = MPX_OK;
  auto cleanup = [&]() {
    if (dout != out) pfree(e, dout);
    if (tmp >= 0) {
      release_all(e, e->mags[tmp].get());
      e->mags[tmp].reset();
    }
  };
  if (!on_device && (st = palloc(e, (void**)&dout, sizeof(float) * 3 * (size_t)NB)) != MPX_OK) {
    dout = out;
    cleanup();
    return st;
  }
  if (A->msat_zero) {  // physics/strayfield.cpp:77-80: assuredly zero
    const cudaError_t ce = cudaMemsetAsync(dout, 0, sizeof(float) * 3 * (size_t)NB, e->stream);
    if (ce != cudaSuccess) st = fail(MPX_ERR_CUDA, cudaGetErrorString(ce));
  } else {
    KernelGeom g;  // the source world's periodic images
    for (int ax = 0; ax < 3; ++ax) {
      g.n[ax] = B->dev.n[ax];
      g.mg[ax] = A->dev.mg[ax];
      g.pbc[ax] = A->pbc_rep[ax];
      g.cs[ax] = A->cs_d[ax];
    }
    int logP[3];
    if (method == MPX_STRAY_FFT && pair_fft_lengths(A->dev.n, B->dev.n, logP)) {
      PairPlan* pl = nullptr;
      st = cached_pair_plan(e, A, B, g, &pl);
      if (st == MPX_OK) launch_pair_fft(e, *pl, src, dst, 0, 0, 0, dout);
    } else {  // the direct sum (also the FFT method's form for pair grids beyond the FFT lengths)
      StrayTable tab;
      for (int ax = 0; ax < 3; ++ax) {
        tab.K[ax] = A->dev.n[ax] + B->dev.n[ax] - 1;
        tab.O[ax] = B->dev.o[ax] - A->dev.o[ax] - (A->dev.n[ax] - 1);
      }
      const size_t KK = (size_t)tab.K[0] * tab.K[1] * tab.K[2];
      float* k = nullptr;
      st = palloc(e, (void**)&k, sizeof(float) * 6 * KK);
      if (st == MPX_OK) st = build_pair_table(e, g, tab.K, tab.O, k);
      if (st == MPX_OK) {
        tab.k = k;
        k_stray_pair<<<(NB + 255) / 256, 256, 0, e->stream>>>(e->d_mags, e->d_groups, src, dst, tab, 0, 0, 0, dout);
        e->launches++;
      }
      pfree(e, k);
    }
  }
  if (st == MPX_OK) {
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) st = fail(MPX_ERR_CUDA, std::string("stray field: ") + cudaGetErrorString(ce));
  }
  if (st == MPX_OK && !on_device) {
    cudaError_t ce = cudaMemcpyAsync(out, dout, sizeof(float) * 3 * (size_t)NB, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) st = fail(MPX_ERR_CUDA, cudaGetErrorString(ce));
  }
  cleanup();
  return st;
}

mpx_status mpx_profile_attempt(mpx_engine* e, int method, int reps, double ms[4]) {
  if (!e || !ms || reps <= 0) return fail(MPX_ERR_INVALID, "bad arguments");
  if (method < 0 || method > MPX_RK_DORMAND_PRINCE) return fail(MPX_ERR_INVALID, "unknown method");
  DeviceGuard guard(e->device);
  MPX_TRY(prepare_run(e, method));
  const int s = 1;
  EpiArgs ea;
  ea.mode = EPI_STAGE;
  ea.stage = s;
  ea.quantity = 0;
  ea.fsal_err = 0;
  ea.gate = 1;
  ea.out = nullptr;
  ea.msrc = nullptr;
  cudaEvent_t ev[5];
  for (auto& x : ev) CUDA_TRY(cudaEventCreate(&x));
  double acc[4] = {0, 0, 0, 0};
  for (int r = 0; r <= reps; ++r) {
    CUDA_TRY(cudaEventRecord(ev[0], e->stream));
    if (e->n_t_demag > 0)
      xfwd_fn(true, e->x_pair)<<<e->n_t_demag, e->nt_x, e->smem_x, e->stream>>>(e->d_mags, e->d_groups, e->d_t_demag, s, 1,
                                                                    nullptr, e->d_tw);
    if (e->n_t_local > 0)
      k_combine<<<e->n_t_local, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_local, s, 0);
    CUDA_TRY(cudaEventRecord(ev[1], e->stream));
    MPX_TRY(launch_pairs(e, -1, s, 1));
    CUDA_TRY(cudaEventRecord(ev[2], e->stream));
    if (e->n_t_demag > 0) {
      for (int c = 0; c < YZ_CLASSES; ++c)
        MPX_TRY(launch_yz(e, c, e->d_kx_demag[c], e->n_kx_demag[c], e->smem_yz[c], s, 1));
      MPX_TRY(launch_split(e, e->d_t_ycols, e->n_t_ycols, e->d_t_zmul, e->n_t_zmul, e->smem_ycols, e->smem_zmul,
                           e->maxpy_split, e->maxpz_split, s, 1, e->d_t_tc, e->n_t_tc));
    }
    CUDA_TRY(cudaEventRecord(ev[3], e->stream));
    if (e->n_t_demag > 0)
      CUDA_TRY(launch_pdl(xinv_fn(e->x_pair), e->n_t_demag, e->nt_x, e->smem_x, e->stream, e->d_mags, e->d_groups, e->d_t_demag, ea,
                          e->d_tw));
    if (e->n_t_local > 0) k_local<<<e->n_t_local, 256, 0, e->stream>>>(e->d_mags, e->d_groups, e->d_t_local, ea);
    CUDA_TRY(cudaEventRecord(ev[4], e->stream));
    CUDA_TRY(cudaEventSynchronize(ev[4]));
    MPX_TRY(check_launch(e, "profile attempt"));
    if (r > 0)
      for (int k = 0; k < 4; ++k) {
        float t;
        CUDA_TRY(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
        acc[k] += t;
      }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  for (int k = 0; k < 4; ++k) ms[k] = acc[k] / reps;
  return MPX_OK;
}

mpx_status mpx_autotune(mpx_engine* e, int method, int* div_x, int* div_yz) {
  NvtxRange nvtx_range("mpx_autotune");
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  DeviceGuard guard(e->device);
  std::vector<Magnet*> act;
  const long long cells = active_set(e, act);
  int bx = 1, byz = 1;
  if (!act.empty()) {
    double tx_best = 1e300, tyz_best = 1e300;
    for (int d : {1, 2, 4, 8}) {
      e->tune_cells = cells;
      e->tune_div_x = d;
      e->tune_div_yz = d;
      e->tables_dirty = true;
      double ms[4];
      MPX_TRY(mpx_profile_attempt(e, method, 3, ms));
      if (ms[0] + ms[3] < tx_best) {
        tx_best = ms[0] + ms[3];
        bx = d;
      }
      if (ms[2] < tyz_best) {
        tyz_best = ms[2];
        byz = d;
      }
    }
    e->tune_cells = cells;
    e->tune_div_x = bx;
    e->tune_div_yz = byz;
    e->tables_dirty = true;
  }
  if (div_x) *div_x = bx;
  if (div_yz) *div_yz = byz;
  return MPX_OK;
}

mpx_status mpx_profile_eval(mpx_engine* e, int magnet, int reps, double ms[4]) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !ms || reps <= 0) return fail(MPX_ERR_INVALID, "no such magnet / bad arguments");
  DeviceGuard guard(e->device);
  if (e->tables_dirty) MPX_TRY(rebuild_tables(e));
  MPX_TRY(ensure_scratch(e, sizeof(float) * 3 * (size_t)m->dev.N));
  EpiArgs ea;
  ea.mode = EPI_EVAL;
  ea.stage = 0;
  ea.quantity = MPX_Q_EFFECTIVE_FIELD;
  ea.fsal_err = 0;
  ea.gate = 0;
  ea.out = e->d_scratch;
  ea.msrc = nullptr;
  const int ntile = (int)m->tiles.size();
  const int sx = x_smem(m), syz = yz_smem(m), nt = x_threads(m);
  cudaEvent_t ev[5];
  for (auto& x : ev) CUDA_TRY(cudaEventCreate(&x));
  double acc[4] = {0, 0, 0, 0};
  for (int r = 0; r <= reps; ++r) {  // r == 0 is the warm-up
    float t[4] = {0, 0, 0, 0};
    if (m->demag) {
      CUDA_TRY(cudaEventRecord(ev[0], e->stream));
      xfwd_fn(false, x_pair_of(m))<<<ntile, nt, sx, e->stream>>>(e->d_mags, e->d_groups, m->d_tiles, 0, 0, nullptr, e->d_tw);
      CUDA_TRY(cudaEventRecord(ev[1], e->stream));
      if (m->split)
        MPX_TRY(launch_split(e, m->d_ycw, (int)m->ycw.size(), m->d_zmw, (int)m->zmw.size(), ycols_smem(m),
                             zmul_smem(m), m->P[1], m->P[2], 0, 0, m->d_tcw,
                           (int)m->tcw.size()));
      else
        MPX_TRY(launch_yz(e, yz_class(m), m->d_kxw, (int)m->kxw.size(), syz, 0, 0));
      CUDA_TRY(cudaEventRecord(ev[2], e->stream));
      CUDA_TRY(launch_pdl(xinv_fn(x_pair_of(m)), ntile, nt, sx, e->stream, e->d_mags, e->d_groups, m->d_tiles, ea, e->d_tw));
      CUDA_TRY(cudaEventRecord(ev[3], e->stream));
      e->launches += 2;
      CUDA_TRY(cudaEventSynchronize(ev[3]));
      for (int k = 0; k < 3; ++k) CUDA_TRY(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
    } else {
      CUDA_TRY(cudaEventRecord(ev[3], e->stream));
      k_local<<<ntile, 256, 0, e->stream>>>(e->d_mags, e->d_groups, m->d_tiles, ea);
      CUDA_TRY(cudaEventRecord(ev[4], e->stream));
      e->launches += 1;
      CUDA_TRY(cudaEventSynchronize(ev[4]));
      CUDA_TRY(cudaEventElapsedTime(&t[3], ev[3], ev[4]));
    }
    MPX_TRY(check_launch(e, "profile"));
    if (r > 0)
      for (int k = 0; k < 4; ++k) acc[k] += t[k];
  }
  for (auto& x : ev) cudaEventDestroy(x);
  for (int k = 0; k < 4; ++k) ms[k] = acc[k] / reps;
  return MPX_OK;
}

mpx_status mpx_demag_kernel(mpx_engine* e, int magnet, float* out, int dims[3]) {
  Magnet* m = get_mag(e, magnet);
  if (!m || !dims) return fail(MPX_ERR_INVALID, "no such magnet / null dims");
  DeviceGuard guard(e->device);
  int K[3], O[3];
  for (int a = 0; a < 3; ++a) {
    K[a] = 2 * m->dev.n[a] - 1;
    const int pad = (K[a] > 5 && K[a] % 2 == 1) ? 1 : 0;
    K[a] += pad;
    O[a] = -(m->dev.n[a] - 1) - pad;
    dims[a] = K[a];
  }
  if (!out) return MPX_OK;
  KernelGeom g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = m->dev.n[a];
    g.mg[a] = m->dev.mg[a];
    g.pbc[a] = m->kkey_pbc[a];
    g.cs[a] = m->kkey_cs[a];
  }
  if (!m->kspec_ready) {  // kernel geometry of a magnet without demag
    for (int a = 0; a < 3; ++a) {
      g.pbc[a] = 0;
      g.cs[a] = m->dev.cs[a];
    }
  }
  const size_t KK = (size_t)K[0] * K[1] * K[2];
  float* d = nullptr;
  MPX_TRY(palloc(e, (void**)&d, sizeof(float) * 6 * KK));
  k_newell_reflayout<<<148 * 8, 128, 0, e->stream>>>(d, g, K[0], K[1], K[2], O[0], O[1], O[2]);
  e->launches++;
  cudaError_t st = cudaMemcpyAsync(out, d, sizeof(float) * 6 * KK, cudaMemcpyDeviceToHost, e->stream);
  pfree(e, d);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return fail(MPX_ERR_CUDA, cudaGetErrorString(st));
  return MPX_OK;
}

mpx_status mpx_solver_set_params(mpx_engine* e, int group, const mpx_solver_params* p) {
  Group* g = get_group(e, group);
  if (!g || !p) return fail(MPX_ERR_INVALID, "no such group / null params");
  if (p->method < 0 || p->method > MPX_RK_DORMAND_PRINCE) return fail(MPX_ERR_INVALID, "invalid Runge Kutta method");
  if (p->lower_bound >= p->upper_bound)
    return fail(MPX_ERR_RUNTIME, "The lower bound should be lower than the upper bound.");
  if (p->sensible_timestep_default < 0)
    return fail(MPX_ERR_RUNTIME, "The sensible timestep should be larger than zero.");
  DeviceGuard guard(e->device);
  const bool method_changed = p->method != g->sp.method;
  g->sp = *p;
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  fill_group_params(G, g->sp);
  if (method_changed) G.k0_valid = 0;
  MPX_TRY(write_group(e, group, &G));
  if (method_changed && g->sp.adaptive) {  // core/timesolver.cpp:23-27
    double dt;
    MPX_TRY(sensible_timestep(e, g, &dt));
    MPX_TRY(read_group(e, group, &G));
    G.dt = dt;
    MPX_TRY(write_group(e, group, &G));
  }
  return MPX_OK;
}

mpx_status mpx_solver_get_params(mpx_engine* e, int group, mpx_solver_params* p) {
  Group* g = get_group(e, group);
  if (!g || !p) return fail(MPX_ERR_INVALID, "no such group / null params");
  *p = g->sp;
  return MPX_OK;
}

mpx_status mpx_solver_set_time(mpx_engine* e, int group, double t) {
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  G.t = t;
  MPX_TRY(write_group(e, group, &G));
  return MPX_OK;
}

mpx_status mpx_solver_get_time(mpx_engine* e, int group, double* t) {
  Group* g = get_group(e, group);
  if (!g || !t) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  *t = G.t;
  return MPX_OK;
}

mpx_status mpx_solver_set_timestep(mpx_engine* e, int group, double dt) {
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  G.dt = dt;
  MPX_TRY(write_group(e, group, &G));
  return MPX_OK;
}

mpx_status mpx_solver_get_timestep(mpx_engine* e, int group, double* dt) {
  Group* g = get_group(e, group);
  if (!g || !dt) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  *dt = G.dt;
  return MPX_OK;
}

mpx_status mpx_solver_sensible_timestep(mpx_engine* e, int group, double* dt) {
  Group* g = get_group(e, group);
  if (!g || !dt) return fail(MPX_ERR_RANGE, "no such group");
  DeviceGuard guard(e->device);
  return sensible_timestep(e, g, dt);
}

static mpx_status start_group(mpx_engine* e, Group* g, int mode, long long nsteps, double duration,
                              double torque_stop, bool* nothing_to_do) {
  *nothing_to_do = false;
  GroupDev G;
  MPX_TRY(read_group(e, g->slot, &G));
  if (g->magnets.empty()) {  // core/rungekutta.cpp:26-30: no equations, only time advances
    if (mode == 1) {
      if (!(G.dt > 0)) return fail(MPX_ERR_RUNTIME, "Timesolver can not make a step because the timestep is smaller than or equal to zero.");
      G.t += G.dt * (double)nsteps;
    } else if (duration > 0) {
      const double stop = G.t + duration;
      while (G.t < stop - G.dt) G.t += G.dt;
      G.t = stop;
    }
    MPX_TRY(write_group(e, g->slot, &G));
    *nothing_to_do = true;
    return MPX_OK;
  }
  if (!(G.dt > 0))
    return fail(MPX_ERR_RUNTIME,
                "Timesolver can not make a step because the timestep is smaller than or equal to zero.");
  fill_group_params(G, g->sp);
  G.mode = mode;
  G.phase = 0;
  G.steps_left = nsteps;
  G.torque_stop = torque_stop;
  G.err_bits = 0;
  G.tmax_bits = 0;
  G.finished_flag = 0;
  if (mode == 0 || mode == 2) {
    G.t_stop = G.t + duration;
    if (!(G.t < G.t_stop - G.dt)) {  // core/timesolver.cpp:100-109
      G.phase = 1;
      G.dt_saved = G.dt;
      G.dt = G.t_stop - G.t;
    }
  }
  G.status = GS_RUNNING;
  MPX_TRY(write_group(e, g->slot, &G));
  if (!g->active) {
    g->active = true;
    e->tables_dirty = true;
  }
  return MPX_OK;
}

mpx_status mpx_solver_steps(mpx_engine* e, int group, int nsteps) {
  NvtxRange nvtx_range("mpx_solver_steps");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (nsteps <= 0) return MPX_OK;
  DeviceGuard guard(e->device);
  bool none;
  MPX_TRY(start_group(e, g, 1, nsteps, 0.0, 0.0, &none));
  if (none) return MPX_OK;
  return drive_group(e, g);
}

mpx_status mpx_solver_step(mpx_engine* e, int group) { return mpx_solver_steps(e, group, 1); }

mpx_status mpx_solver_run(mpx_engine* e, int group, double duration) {
  NvtxRange nvtx_range("mpx_solver_run");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (duration <= 0) return MPX_OK;
  DeviceGuard guard(e->device);
  bool none;
  MPX_TRY(start_group(e, g, 0, 0, duration, 0.0, &none));
  if (none) return MPX_OK;
  return drive_group(e, g);
}

mpx_status mpx_solver_run_sampled(mpx_engine* e, int group, const double* times, int n, double* out) {
  NvtxRange nvtx_range("mpx_solver_run_sampled");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (n < 0 || (n > 0 && (!times || !out))) return fail(MPX_ERR_INVALID, "bad time points / output table");
  for (int k = 1; k < n; ++k)
    if (!(times[k - 1] <= times[k])) return fail(MPX_ERR_INVALID, "The list of timepoints should be increasing.");
  if (n == 0) return MPX_OK;
  DeviceGuard guard(e->device);
  const int nmag = (int)g->magnets.size();
  const int row = 1 + 3 * nmag;
  auto record = [&](int k) -> mpx_status {  // row k from the current state, on the host
    MPX_TRY(mpx_solver_get_time(e, group, &out[(size_t)k * row]));
    for (int j = 0; j < nmag; ++j) MPX_TRY(mpx_average(e, g->magnets[j], MPX_Q_MAGNETIZATION, &out[(size_t)k * row + 1 + 3 * j]));
    return MPX_OK;
  };
  double t;
  MPX_TRY(mpx_solver_get_time(e, group, &t));
  if (nmag == 0) {  // no equations: time only advances (start_group)
    for (int k = 0; k < n; ++k) {
      MPX_TRY(mpx_solver_run(e, group, times[k] - t));
      MPX_TRY(record(k));
      t = out[(size_t)k * row];
    }
    return MPX_OK;
  }
  int k0 = 0;  // points that need no step from here: run(t_k - t) would take none
  while (k0 < n && !(times[k0] - t > 0.0)) MPX_TRY(record(k0++));
  if (k0 == n) return MPX_OK;
  double *d_t = nullptr, *d_out = nullptr;
  MPX_TRY(palloc(e, (void**)&d_t, sizeof(double) * n));
  mpx_status st = palloc(e, (void**)&d_out, sizeof(double) * (size_t)n * row);
  if (st == MPX_OK) {
    cudaError_t ce = cudaMemcpyAsync(d_t, times, sizeof(double) * n, cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(d_out, 0, sizeof(double) * (size_t)n * row, e->stream);
    if (ce != cudaSuccess) st = fail(MPX_ERR_CUDA, cudaGetErrorString(ce));
  }
  bool none = false;
  if (st == MPX_OK) st = start_group(e, g, 2, 0, times[k0] - t, 0.0, &none);
  if (st == MPX_OK) {
    GroupDev G;
    st = read_group(e, g->slot, &G);
    if (st == MPX_OK) {
      G.samp_t = d_t;
      G.samp_out = d_out;
      G.samp_n = n;
      G.samp_k = k0;
      G.samp_lo = G.samp_hi = 0;
      G.samp_row = row;
      st = write_group(e, g->slot, &G);
    }
  }
  if (st == MPX_OK) {
    e->sampling_group = group;
    e->samp_magnets = nmag;
    e->graph_dirty = true;
    st = drive_group(e, g);
    e->sampling_group = -1;
    e->samp_magnets = 0;
    e->graph_dirty = true;
    GroupDev G;
    mpx_status s2 = read_group(e, g->slot, &G);
    if (s2 == MPX_OK) {
      G.mode = 0;
      G.samp_t = nullptr;
      G.samp_out = nullptr;
      G.samp_n = G.samp_k = G.samp_lo = G.samp_hi = 0;
      s2 = write_group(e, g->slot, &G);
    }
    if (st == MPX_OK) st = s2;
    if (st == MPX_OK) {
      cudaError_t ce = cudaMemcpyAsync(out + (size_t)k0 * row, d_out + (size_t)k0 * row,
                                       sizeof(double) * (size_t)(n - k0) * row, cudaMemcpyDeviceToHost, e->stream);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
      if (ce != cudaSuccess) st = fail(MPX_ERR_CUDA, cudaGetErrorString(ce));
    }
  }
  pfree(e, d_t);
  pfree(e, d_out);
  return st;
}

// ------------------------------------------------ minimize / relax
// Sum over the group's magnets of the squared norm of the damping torque
// (physics/relaxer.cpp calcTorque: dotSum(torque, torque)), or its largest
// per-cell norm per magnet.
static mpx_status damping_torque_reduce(mpx_engine* e, Magnet* m, int op, double* out) {
  double r[3];
  MPX_TRY(reduce_quantity(e, m, MPX_Q_DAMPING_TORQUE, op, r));
  *out = r[0];
  return MPX_OK;
}

static mpx_status group_energy(mpx_engine* e, Group* g, double* out) {
  double E = 0;
  for (int id : g->magnets) {
    double v;
    MPX_TRY(mpx_energy(e, id, MPX_Q_TOTAL_ENERGY_DENSITY, &v));
    E += v;
  }
  *out = E;
  return MPX_OK;
}

static mpx_status group_torque_sq(mpx_engine* e, Group* g, double* out) {
  double t = 0;
  for (int id : g->magnets) {
    double v;
    MPX_TRY(damping_torque_reduce(e, get_mag(e, id), 2, &v));
    t += v;
  }
  *out = t;
  return MPX_OK;
}

// Iteration bound of the minimize / relax loops, which the reference runs
// without one: a solve that has not converged by then fails instead of hanging.
constexpr long long RELAX_MAX_STEPS = 10000000;

mpx_status mpx_minimize(mpx_engine* e, int group, double tol, int nsamples) {
  NvtxRange nvtx_range("mpx_minimize");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (nsamples <= 0) return fail(MPX_ERR_INVALID, "nsamples must be positive");
  if (g->magnets.empty()) return MPX_OK;
  DeviceGuard guard(e->device);
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  std::vector<Magnet*> ms;
  for (int id : g->magnets) ms.push_back(get_mag(e, id));
  // scratch roles among the stage buffers (the stage values are recomputed after)
  int t0 = 2, t1 = 3;
  const int m0 = 4, m1 = 5;
  for (Magnet* m : ms) MPX_TRY(eval_into(e, m, MPX_Q_DAMPING_TORQUE, m->dev.buf[G.map[t0]]));
  const size_t nkeep = (size_t)nsamples * ms.size();
  std::vector<double> step(ms.size(), 1e-14);
  std::deque<double> diffs;
  const int nb = 256;
  for (long long n = 0;; ++n) {
    if (diffs.size() >= nkeep) {  // Minimizer::converged
      bool conv = true;
      for (double d : diffs) conv = conv && (d <= tol);
      if (conv) break;
    }
    if (n >= RELAX_MAX_STEPS) return fail(MPX_ERR_RUNTIME, "minimize did not converge");
    for (size_t j = 0; j < ms.size(); ++j) {
      MagnetDev& D = ms[j]->dev;
      k_min_step<<<std::min((D.N + 255) / 256, 148 * 8), 256, 0, e->stream>>>(
          D.buf[G.map[0]], D.buf[G.map[m0]], D.buf[G.map[m1]], D.buf[G.map[t0]], D.N, (float)step[j], ms[j]->geom);
      e->launches++;
    }
    for (Magnet* m : ms) MPX_TRY(eval_into(e, m, MPX_Q_DAMPING_TORQUE, m->dev.buf[G.map[t1]]));
    for (size_t j = 0; j < ms.size(); ++j) {
      MagnetDev& D = ms[j]->dev;
      k_min_partial<<<nb, 256, 0, e->stream>>>(D.buf[G.map[m0]], D.buf[G.map[m1]], D.buf[G.map[t0]],
                                               D.buf[G.map[t1]], D.N, e->d_red);
      k_min_final<<<1, 32, 0, e->stream>>>(e->d_red, nb, e->d_redout);
      e->launches += 2;
      MPX_TRY(check_launch(e, "minimize"));
      double r[4];
      CUDA_TRY(cudaMemcpyAsync(r, e->d_redout, sizeof(r), cudaMemcpyDeviceToHost, e->stream));
      CUDA_TRY(cudaStreamSynchronize(e->stream));
      // Barzilai-Borwein step size, alternating its two forms
      const double nom = (n % 2 == 0) ? r[0] : r[1], div = (n % 2 == 0) ? r[1] : r[2];
      step[j] = (div == 0.0) ? 1e-14 : nom / div;
      diffs.push_back(r[3]);
      if (diffs.size() > nkeep) diffs.pop_front();
    }
    std::swap(t0, t1);
  }
  G.k0_valid = 0;
  return write_group(e, group, &G);
}

mpx_status mpx_relax(mpx_engine* e, int group, double tol, double threshold) {
  NvtxRange nvtx_range("mpx_relax");
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (threshold == 0.0) return fail(MPX_ERR_INVALID, "The relax threshold should not be zero.");
  if (g->magnets.empty()) return MPX_OK;
  DeviceGuard guard(e->device);
  const mpx_solver_params saved = g->sp;
  GroupDev G;
  MPX_TRY(read_group(e, group, &G));
  const double t_saved = G.t, dt_saved = G.dt;
  // adaptive Fehlberg on the damping torque, starting from the sensible step for it
  mpx_solver_params p = saved;
  p.method = MPX_RK_FEHLBERG;
  p.adaptive = 1;
  g->sp = p;
  g->torque_kind = 1;
  fill_group_params(G, p);
  G.torque_kind = 1;
  G.k0_valid = 0;
  MPX_TRY(write_group(e, group, &G));
  double dt;
  MPX_TRY(sensible_timestep(e, g, &dt));
  MPX_TRY(mpx_solver_set_timestep(e, group, dt));
  auto set_max_error = [&](double err) -> mpx_status {
    g->sp.max_error = err;
    GroupDev H;
    MPX_TRY(read_group(e, group, &H));
    H.max_error = err;
    return write_group(e, group, &H);
  };
  mpx_status st = MPX_OK;
  long long nsteps = 0;
  auto steps3 = [&]() -> mpx_status {
    nsteps += 3;
    if (nsteps > RELAX_MAX_STEPS) return fail(MPX_ERR_RUNTIME, "relax did not converge");
    return mpx_solver_steps(e, group, 3);
  };
  do {
    // energy phase (physics/relaxer.cpp): steps of 3 while the energy decreases
    double E0, E1;
    if ((st = group_energy(e, g, &E0)) != MPX_OK) break;
    if ((st = steps3()) != MPX_OK) break;
    if ((st = group_energy(e, g, &E1)) != MPX_OK) break;
    while (E1 < E0) {
      if ((st = steps3()) != MPX_OK) break;
      E0 = E1;
      if ((st = group_energy(e, g, &E1)) != MPX_OK) break;
    }
    if (st != MPX_OK) break;
    double err = g->sp.max_error;
    if (threshold < 0) {  // torque phase: lower the error while the torque decreases
      double tq0, tq1;
      if ((st = group_torque_sq(e, g, &tq1)) != MPX_OK) break;
      while (err > tol && st == MPX_OK) {
        err /= std::sqrt(2.0);
        if ((st = set_max_error(err)) != MPX_OK) break;
        if ((st = steps3()) != MPX_OK) break;
        tq0 = tq1;
        if ((st = group_torque_sq(e, g, &tq1)) != MPX_OK) break;
        while (tq1 < tq0) {
          if ((st = steps3()) != MPX_OK) break;
          tq0 = tq1;
          if ((st = group_torque_sq(e, g, &tq1)) != MPX_OK) break;
        }
      }
    } else {  // until every magnet's max torque is at or below the threshold, then lower the error
      while (err > tol && st == MPX_OK) {
        bool conv = true;
        for (int id : g->magnets) {
          double mx;
          if ((st = damping_torque_reduce(e, get_mag(e, id), 1, &mx)) != MPX_OK) break;
          if (mx > threshold) {
            conv = false;
            break;
          }
        }
        if (st != MPX_OK) break;
        if (conv) {
          err /= std::sqrt(2.0);
          if ((st = set_max_error(err)) != MPX_OK) break;
        }
        st = steps3();
      }
    }
  } while (false);
  const std::string msg = g_last_error;
  // restore the solver (physics/relaxer.cpp: method, error, adaptivity, time,
  // time step, then the equations, which for an adaptive solver recompute the
  // sensible time step of the LLG torque)
  g->sp = saved;
  g->torque_kind = 0;
  GroupDev R;
  MPX_TRY(read_group(e, group, &R));
  fill_group_params(R, saved);
  R.torque_kind = 0;
  R.k0_valid = 0;
  R.t = t_saved;
  R.dt = dt_saved;
  MPX_TRY(write_group(e, group, &R));
  if (saved.adaptive) {
    double dt2;
    MPX_TRY(sensible_timestep(e, g, &dt2));
    MPX_TRY(mpx_solver_set_timestep(e, group, dt2));
  }
  if (st != MPX_OK) g_last_error = msg;
  return st;
}

mpx_status mpx_group_start(mpx_engine* e, int group, double duration, double torque_stop) {
  Group* g = get_group(e, group);
  if (!g) return fail(MPX_ERR_RANGE, "no such group");
  if (duration <= 0) return fail(MPX_ERR_INVALID, "duration must be positive");
  if (torque_stop > 0 && g->sp.method != MPX_RK_DORMAND_PRINCE)
    return fail(MPX_ERR_UNSUPPORTED, "the torque stop criterion needs the DormandPrince method");
  // all running groups of an engine advance with one method
  for (auto& og : e->groups)
    if (og && og.get() != g && og->sp.method != g->sp.method) {
      GroupDev G;
      MPX_TRY(read_group(e, og->slot, &G));
      if (G.status == GS_RUNNING) return fail(MPX_ERR_INVALID, "running groups must share one Runge Kutta method");
    }
  DeviceGuard guard(e->device);
  bool none;
  MPX_TRY(start_group(e, g, 0, 0, duration, torque_stop, &none));
  if (none) {
    GroupDev G;
    MPX_TRY(read_group(e, group, &G));
    G.finished_flag = 1;
    G.status = GS_FINISHED;
    MPX_TRY(write_group(e, group, &G));
  }
  return MPX_OK;
}

mpx_status mpx_advance(mpx_engine* e, int attempts) {
  NvtxRange nvtx_range("mpx_advance");
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  if (attempts <= 0) return MPX_OK;
  DeviceGuard guard(e->device);
  int method = -1;
  for (auto& g : e->groups)
    if (g && !g->magnets.empty()) { method = g->sp.method; break; }
  if (method < 0) return MPX_OK;
  return run_attempts(e, method, attempts);
}

mpx_status mpx_poll(mpx_engine* e, int* done, int cap, int* n_done, int* n_running) {
  if (!e) return fail(MPX_ERR_INVALID, "null engine");
  DeviceGuard guard(e->device);
  const int ng = (int)e->groups.size();
  std::vector<GroupDev> G(ng);
  if (ng > 0) {
    CUDA_TRY(cudaMemcpyAsync(G.data(), e->d_groups, sizeof(GroupDev) * ng, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
  }
  int nd = 0, nr = 0;
  for (int i = 0; i < ng; ++i) {
    if (!e->groups[i]) continue;
    if (G[i].status == GS_RUNNING) nr++;
    if (G[i].status != GS_RUNNING && e->groups[i]->active) {  // drop it from the attempt tables
      e->groups[i]->active = false;
      e->tables_dirty = true;
    }
    if (G[i].finished_flag && nd < cap) {
      if (done) done[nd] = i;
      nd++;
      G[i].finished_flag = 0;
      if (G[i].status == GS_FINISHED) G[i].status = GS_IDLE;
      CUDA_TRY(cudaMemcpyAsync(e->d_groups + i, &G[i], sizeof(GroupDev), cudaMemcpyHostToDevice, e->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (n_done) *n_done = nd;
  if (n_running) *n_running = nr;
  return MPX_OK;
}

mpx_status mpx_bounds_check(unsigned long long* first_bad) {
  if (!first_bad) return fail(MPX_ERR_INVALID, "mpx_bounds_check: null output");
  *first_bad = 0;
#ifdef MPX_BOUNDS_CHECK
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpyFromSymbol(first_bad, g_bounds_first_bad, sizeof(unsigned long long)));
  const unsigned long long zero = 0;
  CUDA_TRY(cudaMemcpyToSymbol(g_bounds_first_bad, &zero, sizeof zero));
  return MPX_OK;
#else
  return fail(MPX_ERR_UNSUPPORTED, "mpx_bounds_check: library built without MPX_BOUNDS_CHECK (use libmpx_checked.so)");
#endif
}

}  // extern "C"

// ============================================ allocation-free reduction
// mpx_reduce_noalloc is for callers that may not allocate device memory: a
// diagnostic or monitoring hook running inside another application's time
// loop, whose host gave it a fixed device-memory budget (its own pool, no
// cudaMalloc of its own) and which must not add the device-wide
// synchronisation or the out-of-memory failure a cudaMalloc can bring.  It is
// the sum / max-norm reduction of mpx_average / mpx_max_norm, with the block
// partials and the result kept in the static array below instead of in
// engine-allocated memory, over a field the caller already holds on the device.
namespace {

constexpr int NOALLOC_BLOCKS = 256;   // fixed grid of the partial pass (256 threads each)
constexpr int NOALLOC_RESULT = NOALLOC_BLOCKS * 3;
constexpr long long NOALLOC_MAX_CELLS = 0x7fffffffLL / 3;  // 32-bit cell indices of 3 components

// 256 blocks x 3 partials + 3 results = 6168 bytes.  It is part of the
// library's device image: every GPU that loads libmpx.so holds it until the
// process exits.  All calls share it.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_RESULT + 3];

std::mutex g_noalloc_mutex;
// Device address of the array, per device, looked up by the first call on that
// device.  A cudaDeviceReset (or any re-creation of the device's primary
// context) by the host application unloads the module and would leave the
// cached address stale: the library must not be used across a device reset.
double* g_noalloc_ptr[128] = {nullptr};

}  // namespace

extern "C" mpx_status mpx_reduce_noalloc(const float* field, int ncells, int ncomp,
                                         const unsigned char* geometry, int op, void* stream,
                                         double out[3]) {
  if (!field || !out) return fail(MPX_ERR_INVALID, "mpx_reduce_noalloc: null field or output");
  if (ncomp < 1 || ncomp > 3) return fail(MPX_ERR_INVALID, "mpx_reduce_noalloc: ncomp must be 1, 2 or 3");
  if (op != 0 && op != 1) return fail(MPX_ERR_INVALID, "mpx_reduce_noalloc: op must be 0 (sum) or 1 (max norm)");
  if (ncells < 1 || (long long)ncells > NOALLOC_MAX_CELLS)
    return fail(MPX_ERR_INVALID, "mpx_reduce_noalloc: ncells must be in [1, " + std::to_string(NOALLOC_MAX_CELLS) +
                                     "]");
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(MPX_ERR_RANGE, "mpx_reduce_noalloc: device index out of range");
  double* scratch = nullptr;
  {
    // set-up, once per device with that device current: the array's name is a
    // host-side stand-in, the kernels need its device address
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  // an error left pending by the caller's own earlier work is reported as it
  // is and not cleared, so that the caller still sees it
  {
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
      return fail(MPX_ERR_CUDA, std::string("mpx_reduce_noalloc: CUDA error pending before the call: ") +
                                    cudaGetErrorString(pending));
  }
  // every partial slot the final pass reads is written by this call's partial
  // pass, and the final pass overwrites the results: nothing needs clearing
  k_reduce_partial<<<NOALLOC_BLOCKS, 256, 0, s>>>(field, ncells, ncomp, geometry, op, scratch);
  k_reduce_final<<<1, 32, 0, s>>>(scratch, NOALLOC_BLOCKS, op, scratch + NOALLOC_RESULT);
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) return fail(MPX_ERR_CUDA, std::string("mpx_reduce_noalloc: ") + cudaGetErrorString(st));
  CUDA_TRY(cudaMemcpyAsync(out, scratch + NOALLOC_RESULT, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int c = ncomp; c < 3; ++c)
    if (op == 0) out[c] = 0.0;
  return MPX_OK;
}
