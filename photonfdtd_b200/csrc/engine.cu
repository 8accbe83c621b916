// engine.cu - the C ABI of libpfb200.so (declared in include/pfb200.h).
//
// Device state of one engine (all in HBM for the whole run):
//   fields   2 time levels x 6 components, C-order (nx, ny, nz); a step reads
//            level `cur` and writes level `cur ^ 1` (the fused kernel
//            recomputes H on tile halos, so reads and writes must not alias)
//   ce       one or three per-cell arrays, or a uint32 word per cell + table
//   CPML     b/c per axis and stagger, compact maps (-1 = no psi), psi
//            compacted along its derivative axis; H psi double-buffered
//   ADE      compact polarisation state [level][pole][comp][cells] per medium
//   monitors sample rings + complex128 accumulators (DFT), block partials +
//            float64 accumulators (flux)
#include <algorithm>
#include <type_traits>
#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pfb200.h"
#include "common.cuh"
#include "kernels_adj.cuh"
#include "kernels_aux.cuh"
#include "kernels_fused.cuh"
#include "kernels_split.cuh"
#include "kernels_tma.cuh"

using namespace pfb;

namespace {

constexpr int kRingMax = 32;
constexpr size_t kRingBytesCap = 256u << 20;
thread_local std::string g_create_error;

struct DftMon {
  DftRegion r;
  int n_freq = 0, interval = 1;
  double dt = 0;
  std::vector<double> h_ph_e, h_ph_h;
  long long n_samples = 0;   // samples in the whole run
  long long q_done = 0;      // samples folded into acc
  int pending = 0;           // samples waiting in the ring
  int ring_cap = 1;
  void* ring = nullptr;
  double* acc = nullptr;
  double* ph_e = nullptr;
  double* ph_h = nullptr;
};

struct FluxMon {
  FluxPlane p;
  double dA = 0, dt = 0;
  int pending = 0;
  int ring_cap = kRingMax;
  double* partial = nullptr;
  double* acc = nullptr;
  // adjoint: dJ/dflux and the replay's E plane records (2 * n0 * n1 reals
  // per recorded step, rec_cap steps)
  double cot = 0.0;
  void* rec = nullptr;
  long long rec_cap = 0;
};

struct SrcFamily {
  std::vector<long long> cell;
  std::vector<int> comp, start, wave_row;
  std::vector<double> amp;
  SourceGroups dev{};
};

}  // namespace

struct pf_engine {
  int nx = 0, ny = 0, nz = 0, rb = 4;
  double dl[3] = {1, 1, 1};
  double ch = 0;
  long long n_steps = 0;
  long long ncell = 0;
  int kernel = PF_KERNEL_AUTO;
  bool finalized = false;
  long long step = 0;
  int cur = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  int device = 0;
  size_t dev_bytes = 0;
  std::vector<void*> allocs;

  // staged tables
  int ce_mode = -1;
  std::vector<char> h_ce[3];
  // PF_CE_TABLE: the word goes to the device in pf_set_ce; word_need[m] is
  // 1 + the largest record index its dispersive words give medium m (0: none)
  long long word_need[kMaxMedia] = {};
  std::vector<double> h_table;
  std::vector<char> h_cpml[3][4];  // b_e, c_e, b_h, c_h
  int n_media = 0;
  std::vector<long long> m_count;
  std::vector<int> m_npole;
  std::vector<double> m_coef, m_inv, m_ce;
  std::vector<uint32_t> h_adeword;
  SrcFamily src[2];  // 0 = E family, 1 = H family
  int n_wave = 0;
  std::vector<double> h_wave;
  std::vector<DftMon> dfts;
  std::vector<FluxMon> fluxes;

  // device
  void* E[2][3] = {};
  void* H[2][3] = {};
  void* ce[3] = {};
  uint32_t* word = nullptr;
  void* table = nullptr;
  uint32_t* adeword = nullptr;
  void* cp[3][4] = {};
  int* map_e[3] = {};
  int* map_h[3] = {};
  int npe[3] = {}, nph[3] = {};
  int hb0[3] = {}, hb1[3] = {}, eb0[3] = {}, eb1[3] = {};
  void* psiE[6] = {};
  void* psiH[2][6] = {};
  long long npsiE[6] = {}, npsiH[6] = {};  // reals per psi array
  void* P = nullptr;
  long long plev = 0;  // reals per polarisation level
  void* media = nullptr;
  double* wave = nullptr;
  int* flag = nullptr;
  void* region = nullptr;     // pf_read_region staging buffer (grown on demand)
  size_t region_bytes = 0;
  bool fused = false;
  double rdl[3] = {1, 1, 1};     // RN(1/d) in the real type, per axis
  bool fdiv[3] = {false, false, false};  // reciprocal division verified
  bool tma = false;      // fused path stages planes with TMA
  TmaMaps maps;
  int* tma_err = nullptr;
  int wait_test = 0;     // pf_set_wait_test: one TMA stage wait runs out
  // With env PFB200_INLINE=1 the split E pass adds the E-family sources and
  // writes the DFT samples itself (at most kInlineSrc groups, kInlineDft
  // monitors). Off by default: on config 3 (384^3) the epilogue instantiation
  // of the E pass runs 0.08 ms slower per step than the plain one, more than
  // the 0.024 ms of injection and sampling launches it replaces.
  bool inline_epi = false;
  int isrc_blk[kInlineSrc] = {}, isrc_tid[kInlineSrc] = {};
  long long check_every = 0;  // pf_set_check_every: non-finite scan period
  int fused_ty = 8;      // fused tile height (8 or 16), env PFB200_FUSED_TY
  int fused_chunks = 0;  // x chunks per column (0 = auto), env PFB200_XCHUNKS

  // adjoint (pf_adj_*): adjoint fields, quotient and psi adjoints, the
  // gradient, and the ring of per-step forward records a replay writes
  bool adj = false;
  bool recording = false;
  long long rec_step0 = 0, ring_steps = 0, adj_next = 0;
  void* lamE[3] = {};
  void* lamH[3] = {};
  void* gE[6] = {};
  void* gH[6] = {};
  void* lpE[6] = {};
  void* lpH[6] = {};
  double* grad = nullptr;
  char* rec = nullptr;
  size_t rec_slot = 0;          // bytes per recorded step: H (3 fields) + psi_E
  std::vector<double*> dft_cot;  // per DFT monitor: dJ/d acc on the device, or null
  struct RegionSource {
    long long step;
    int comp;
    DftRegion r;
    double* vals;
  };
  std::vector<RegionSource> rsrc;  // FieldMonitor-frame sources of the loss

  // launch accounting (pf_read_profile)
  long long launches[4] = {};
  double prof_ms[4] = {};
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_pending;  // (kind, first event)
  size_t ev_used = 0;
};

namespace {

int fail(pf_engine* e, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (e)
    e->err = buf;
  else
    g_create_error = buf;
  return code;
}

#define PF_CUDA(e, call)                                                                   \
  do {                                                                                     \
    cudaError_t rc_ = (call);                                                              \
    if (rc_ != cudaSuccess)                                                                \
      return fail((e), rc_ == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA,        \
                  "CUDA error: %s (%s) at %s:%d", cudaGetErrorString(rc_), #call, __FILE__, \
                  __LINE__);                                                               \
  } while (0)

int dalloc(pf_engine* e, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t rc = cudaMalloc(p, bytes);
  if (rc != cudaSuccess)
    return fail(e, PF_ERR_OOM, "CUDA error: cudaMalloc of %zu bytes failed: %s", bytes,
                cudaGetErrorString(rc));
  e->allocs.push_back(*p);
  e->dev_bytes += bytes;
  rc = cudaMemsetAsync(*p, 0, bytes, e->stream);
  if (rc != cudaSuccess) return fail(e, PF_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(rc));
  return PF_OK;
}

int upload(pf_engine* e, void** p, const void* src, size_t bytes) {
  int rc = dalloc(e, p, bytes);
  if (rc) return rc;
  if (bytes) PF_CUDA(e, cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, e->stream));
  return PF_OK;
}

// Whether qdiv's reciprocal division (q0 = a*r, rem = fma(-q0, d, a),
// q = fma(rem, r, q0), r = RN(1/d)) equals IEEE a / d for every float
// significand a in [1, 2). Sign and binade of a do not change the outcome
// while nothing over- or underflows; the device's 2^64 prescaling and the
// range check on d below keep every input of the fast path in that regime.
// About 8.4M fmaf evaluations (~50 ms); the answer per divisor is kept for
// the process, so engines on the same grid spacing check it once.
bool recip_division_exact_scan(float d);
bool recip_division_exact(float d) {
  static std::mutex mu;
  static std::map<uint32_t, bool> known;
  uint32_t key;
  memcpy(&key, &d, 4);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = known.find(key);
    if (it != known.end()) return it->second;
  }
  const bool ok = recip_division_exact_scan(d);
  std::lock_guard<std::mutex> lk(mu);
  known[key] = ok;
  return ok;
}
bool recip_division_exact_scan(float d) {
  if (!(d >= 0x1p-30f && d <= 0x1p-23f)) return false;
  const float r = 1.0f / d;
  for (uint32_t m = 0; m < (1u << 23); ++m) {
    const uint32_t bits = 0x3f800000u | m;
    float a;
    memcpy(&a, &bits, 4);
    volatile float q0 = a * r;
    const float rem = std::fmaf(-q0, d, a);
    const float q = std::fmaf(rem, r, q0);
    volatile float ref = a / d;
    if (q != ref) return false;
  }
  return true;
}

// Bracket one launch of `kind` (0 step, 1 sources, 2 sampling, 3 flush).
struct LaunchScope {
  pf_engine* e;
  int kind;
  LaunchScope(pf_engine* eng, int k) : e(eng), kind(k) {
    e->launches[kind]++;
    if (!e->profiling) return;
    while (e->ev_pool.size() < e->ev_used + 2) {
      cudaEvent_t ev;
      cudaEventCreate(&ev);
      e->ev_pool.push_back(ev);
    }
    cudaEventRecord(e->ev_pool[e->ev_used], e->stream);
  }
  ~LaunchScope() {
    if (!e->profiling) return;
    cudaEventRecord(e->ev_pool[e->ev_used + 1], e->stream);
    e->ev_pending.push_back({kind, (int)e->ev_used});
    e->ev_used += 2;
  }
};

// Fold recorded event pairs into prof_ms (the stream must be idle).
void collect_profile(pf_engine* e) {
  for (auto& pr : e->ev_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e->ev_pool[pr.second], e->ev_pool[pr.second + 1]) == cudaSuccess)
      e->prof_ms[pr.first] += ms;
  }
  e->ev_pending.clear();
  e->ev_used = 0;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// Tiled map over a C-order (nx, ny, nz) array, box (bw along z) x (bh along y)
// x 1 plane. Zero fill outside the array.
bool make_map(CUtensorMap* m, void* ptr, CUtensorMapDataType dt, int elem, int nx, int ny, int nz,
              int bw, int bh) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
  const cuuint64_t strides[2] = {(cuuint64_t)nz * elem, (cuuint64_t)ny * nz * elem};
  const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, dt, 3, ptr, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of the TMA fused path (tile height 8); false if any fails.
template <typename T>
bool build_maps(pf_engine* e) {
  const CUtensorMapDataType dt =
      sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const int S = sizeof(T), TY = 8;
  memset(&e->maps, 0, sizeof e->maps);
  bool ok = true;
  for (int l = 0; l < 2; ++l)
    for (int c = 0; c < 3; ++c) {
      ok = ok && make_map(&e->maps.e[l][c], e->E[l][c], dt, S, e->nx, e->ny, e->nz, kBoxW, TY + 2);
      ok = ok && make_map(&e->maps.h[l][c], e->H[l][c], dt, S, e->nx, e->ny, e->nz, kBoxW, TY + 1);
    }
  void* wptr = e->ce_mode == PF_CE_TABLE ? (void*)e->word : (void*)e->adeword;
  if (wptr)
    ok = ok && make_map(&e->maps.word, wptr, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, e->nx, e->ny,
                        e->nz, 32, TY);
  if (e->ce_mode != PF_CE_TABLE)
    for (int c = 0; c < 3; ++c)
      ok = ok && make_map(&e->maps.ce[c], e->ce[c], dt, S, e->nx, e->ny, e->nz, 32, TY);
  return ok;
}

template <typename T>
int finalize_typed(pf_engine* e) {
  const size_t S = sizeof(T);
  const long long n = e->ncell;
  const int dims[3] = {e->nx, e->ny, e->nz};
  int rc;
  for (int lvl = 0; lvl < 2; ++lvl)
    for (int c = 0; c < 3; ++c) {
      if ((rc = dalloc(e, &e->E[lvl][c], n * S))) return rc;
      if ((rc = dalloc(e, &e->H[lvl][c], n * S))) return rc;
    }
  // E coefficients
  if (e->ce_mode == PF_CE_CELL1) {
    if ((rc = upload(e, &e->ce[0], e->h_ce[0].data(), n * S))) return rc;
    e->ce[1] = e->ce[2] = e->ce[0];
  } else if (e->ce_mode == PF_CE_CELL3) {
    for (int c = 0; c < 3; ++c)
      if ((rc = upload(e, &e->ce[c], e->h_ce[c].data(), n * S))) return rc;
  } else {
    std::vector<T> tab(e->h_table.size());
    for (size_t q = 0; q < tab.size(); ++q) tab[q] = (T)e->h_table[q];
    if ((rc = upload(e, &e->table, tab.data(), tab.size() * S))) return rc;
  }
  // CPML: coefficients, compact maps, psi
  for (int ax = 0; ax < 3; ++ax) {
    const int na = dims[ax];
    std::vector<T> arr[4];
    for (int q = 0; q < 4; ++q) {
      arr[q].assign(na, T(0));
      if (!e->h_cpml[ax][q].empty()) memcpy(arr[q].data(), e->h_cpml[ax][q].data(), na * S);
      if ((rc = upload(e, &e->cp[ax][q], arr[q].data(), na * S))) return rc;
    }
    std::vector<int> me(na, -1), mh(na, -1);
    int ce_n = 0, ch_n = 0;
    for (int t = 0; t < na; ++t) {
      if (arr[1][t] != T(0)) me[t] = ce_n++;
      if (arr[3][t] != T(0)) mh[t] = ch_n++;
    }
    e->npe[ax] = ce_n;
    e->nph[ax] = ch_n;
    // Longest run of cells with no psi and both neighbours present: H needs
    // t <= na-2 (forward difference), E needs t >= 1 (backward difference).
    auto longest = [&](const std::vector<int>& map, int lo, int hi, int& b0, int& b1) {
      b0 = b1 = 0;
      int s0 = -1;
      for (int t = lo; t <= hi; ++t) {
        const bool ok = t < hi && map[t] < 0;
        if (ok && s0 < 0) s0 = t;
        if (!ok && s0 >= 0) {
          if (t - s0 > b1 - b0) { b0 = s0; b1 = t; }
          s0 = -1;
        }
      }
    };
    if (na > 1) {
      longest(mh, 0, na - 1, e->hb0[ax], e->hb1[ax]);
      longest(me, 1, na, e->eb0[ax], e->eb1[ax]);
    }
    if ((rc = upload(e, (void**)&e->map_e[ax], me.data(), na * 4))) return rc;
    if ((rc = upload(e, (void**)&e->map_h[ax], mh.data(), na * 4))) return rc;
  }
  const long long nx = e->nx, ny = e->ny, nz = e->nz;
  // psi extents: the term's derivative axis replaced by its PML cell count
  const long long eE[6] = {nx * e->npe[1] * nz, nx * ny * e->npe[2], nx * ny * e->npe[2],
                           (long long)e->npe[0] * ny * nz, (long long)e->npe[0] * ny * nz,
                           nx * e->npe[1] * nz};
  const long long eH[6] = {nx * e->nph[1] * nz, nx * ny * e->nph[2], nx * ny * e->nph[2],
                           (long long)e->nph[0] * ny * nz, (long long)e->nph[0] * ny * nz,
                           nx * e->nph[1] * nz};
  for (int q = 0; q < 6; ++q) {
    e->npsiE[q] = eE[q];
    e->npsiH[q] = eH[q];
    if ((rc = dalloc(e, &e->psiE[q], eE[q] * S))) return rc;
    for (int lvl = 0; lvl < 2; ++lvl)
      if ((rc = dalloc(e, &e->psiH[lvl][q], eH[q] * S))) return rc;
  }
  // ADE: two levels of per-medium cell records [pole][component]; each
  // medium's block starts 8-real aligned (vector loads, whole-sector stores)
  if (e->n_media > 0) {
    std::vector<MediumT<T>> md(e->n_media);
    long long off = 0;
    size_t ci = 0;
    for (int m = 0; m < e->n_media; ++m) {
      MediumT<T>& M = md[m];
      memset(&M, 0, sizeof M);
      off = (off + 7) & ~7LL;
      M.poff = off;
      M.count = e->m_count[m];
      M.npole = e->m_npole[m];
      M.inv = (T)e->m_inv[m];
      M.ce = e->m_ce.empty() ? T(0) : (T)e->m_ce[m];
      for (int p = 0; p < M.npole; ++p) {
        M.a[p] = (T)e->m_coef[ci++];
        M.b[p] = (T)e->m_coef[ci++];
        M.c[p] = (T)e->m_coef[ci++];
      }
      off += 3LL * M.npole * M.count;
    }
    e->plev = (off + 7) & ~7LL;
    if ((rc = dalloc(e, &e->P, 2 * e->plev * S))) return rc;
    if ((rc = upload(e, &e->media, md.data(), md.size() * sizeof(MediumT<T>)))) return rc;
    if (e->ce_mode == PF_CE_CELL1)
      if ((rc = upload(e, (void**)&e->adeword, e->h_adeword.data(), n * 4))) return rc;
    if (e->ce_mode == PF_CE_TABLE && e->m_ce.size() != (size_t)e->n_media)
      return fail(e, PF_ERR_INVALID, "table mode needs each medium's coefficient");
  }
  // sources
  if (e->n_wave > 0)
    if ((rc = upload(e, (void**)&e->wave, e->h_wave.data(), e->h_wave.size() * 8))) return rc;
  for (int f = 0; f < 2; ++f) {
    SrcFamily& s = e->src[f];
    SourceGroups& d = s.dev;
    d.n_groups = (int)s.cell.size();
    d.n_steps = e->n_steps;
    d.wave = e->wave;
    if (d.n_groups == 0) continue;
    if ((rc = upload(e, (void**)&d.cell, s.cell.data(), s.cell.size() * 8))) return rc;
    if ((rc = upload(e, (void**)&d.comp, s.comp.data(), s.comp.size() * 4))) return rc;
    if ((rc = upload(e, (void**)&d.start, s.start.data(), s.start.size() * 4))) return rc;
    if ((rc = upload(e, (void**)&d.wave_row, s.wave_row.data(), s.wave_row.size() * 4))) return rc;
    if ((rc = upload(e, (void**)&d.amp, s.amp.data(), s.amp.size() * 8))) return rc;
  }
  // monitors
  for (DftMon& m : e->dfts) {
    const size_t per = (size_t)m.r.ncomp * m.r.ncell * S;
    m.ring_cap = (int)std::max<size_t>(1, std::min<size_t>(kRingMax, kRingBytesCap / std::max<size_t>(per, 1)));
    if ((rc = dalloc(e, &m.ring, per * m.ring_cap))) return rc;
    if ((rc = dalloc(e, (void**)&m.acc, (size_t)m.r.ncomp * m.n_freq * m.r.ncell * 16))) return rc;
    if ((rc = upload(e, (void**)&m.ph_e, m.h_ph_e.data(), m.h_ph_e.size() * 8))) return rc;
    if ((rc = upload(e, (void**)&m.ph_h, m.h_ph_h.data(), m.h_ph_h.size() * 8))) return rc;
  }
  for (FluxMon& f : e->fluxes) {
    if ((rc = dalloc(e, (void**)&f.partial, (size_t)f.ring_cap * f.p.nblk * 8))) return rc;
    if ((rc = dalloc(e, (void**)&f.acc, 8))) return rc;
  }
  if ((rc = dalloc(e, (void**)&e->flag, sizeof(int)))) return rc;
  if ((rc = dalloc(e, (void**)&e->tma_err, sizeof(int)))) return rc;
  // TMA staging needs 16-byte row strides (nz * sizeof(T) % 16 == 0)
  if (e->fused && !getenv("PFB200_NO_TMA") && ((long long)e->nz * S) % 16 == 0 &&
      !(e->n_media > 0 && e->ce_mode == PF_CE_CELL3))
    e->tma = build_maps<T>(e);
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

template <typename T>
StepArgs<T> step_args(pf_engine* e) {
  StepArgs<T> a;
  memset(&a, 0, sizeof a);
  a.nx = e->nx;
  a.ny = e->ny;
  a.nz = e->nz;
  a.dx = (T)e->dl[0];
  a.dy = (T)e->dl[1];
  a.dz = (T)e->dl[2];
  a.rdx = (T)e->rdl[0];
  a.rdy = (T)e->rdl[1];
  a.rdz = (T)e->rdl[2];
  a.fdx = e->fdiv[0];
  a.fdy = e->fdiv[1];
  a.fdz = e->fdiv[2];
  a.ch = (T)e->ch;
  for (int ax = 0; ax < 3; ++ax) {
    a.hb0[ax] = e->hb0[ax];
    a.hb1[ax] = e->hb1[ax];
    a.eb0[ax] = e->eb0[ax];
    a.eb1[ax] = e->eb1[ax];
  }
  const int c0 = e->cur, c1 = e->cur ^ 1;
  for (int c = 0; c < 3; ++c) {
    a.Ein[c] = (const T*)e->E[c0][c];
    a.Hin[c] = (const T*)e->H[c0][c];
    a.Eout[c] = (T*)e->E[c1][c];
    a.Hout[c] = (T*)e->H[c1][c];
    a.ce[c] = (const T*)e->ce[c];
  }
  a.word = e->word;
  a.table = (const T*)e->table;
  a.adeword = e->adeword;
  for (int ax = 0; ax < 3; ++ax) {
    a.be[ax] = (const T*)e->cp[ax][0];
    a.cpe[ax] = (const T*)e->cp[ax][1];
    a.bh[ax] = (const T*)e->cp[ax][2];
    a.cph[ax] = (const T*)e->cp[ax][3];
    a.mape[ax] = e->map_e[ax];
    a.maph[ax] = e->map_h[ax];
    a.npe[ax] = e->npe[ax];
    a.nph[ax] = e->nph[ax];
  }
  for (int q = 0; q < 6; ++q) {
    a.psiE[q] = (T*)e->psiE[q];
    a.psiHin[q] = (const T*)e->psiH[c0][q];
    a.psiHout[q] = (T*)e->psiH[c1][q];
  }
  a.media = (const MediumT<T>*)e->media;
  a.n_media = e->n_media;
  a.P = (T*)e->P;
  a.plev = e->plev;
  a.lvl = (int)(e->step & 1);
  a.wait_test = e->wait_test;
  return a;
}

// Scans the six current fields for inf / nan (synchronous).
int scan_finite(pf_engine* e) {
  int* flag = e->flag;
  PF_CUDA(e, cudaMemsetAsync(flag, 0, sizeof(int), e->stream));
  for (int c = 0; c < 6; ++c) {
    const void* f = c < 3 ? e->E[e->cur][c] : e->H[e->cur][c - 3];
    if (e->rb == 4)
      k_nonfinite<float><<<592, 256, 0, e->stream>>>((const float*)f, e->ncell, flag);
    else
      k_nonfinite<double><<<592, 256, 0, e->stream>>>((const double*)f, e->ncell, flag);
  }
  int h = 0;
  PF_CUDA(e, cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return h ? fail(e, PF_ERR_NONFINITE, "non-finite field value at step %lld", e->step) : PF_OK;
}

template <typename T>
void launch_h_split(pf_engine* e, const StepArgs<T>& a, dim3 g, dim3 b) {
  k_h_split<T><<<g, b, 0, e->stream>>>(a);
}

template <typename T, bool EPI>
void launch_e_split_epi(pf_engine* e, const StepArgs<T>& a,
                        const typename EpiParam<T, EPI>::type& ep, dim3 g, dim3 b) {
  const bool ade = e->n_media > 0;
  switch (e->ce_mode) {
    case PF_CE_CELL1:
      if (ade) k_e_split<T, kCeCell1, true, EPI><<<g, b, 0, e->stream>>>(a, ep);
      else k_e_split<T, kCeCell1, false, EPI><<<g, b, 0, e->stream>>>(a, ep);
      break;
    case PF_CE_CELL3:
      k_e_split<T, kCeCell3, false, EPI><<<g, b, 0, e->stream>>>(a, ep);
      break;
    default:
      if (ade) k_e_split<T, kCeTable, true, EPI><<<g, b, 0, e->stream>>>(a, ep);
      else k_e_split<T, kCeTable, false, EPI><<<g, b, 0, e->stream>>>(a, ep);
  }
}

template <typename T>
void launch_e_split(pf_engine* e, const StepArgs<T>& a, const EpiArgs<T>& ep, dim3 g, dim3 b) {
  if (e->inline_epi) launch_e_split_epi<T, true>(e, a, ep, g, b);
  else launch_e_split_epi<T, false>(e, a, NoEpi{}, g, b);
}

template <typename T>
Fields6<T> level_fields(pf_engine* e, int lvl) {
  Fields6<T> f;
  for (int c = 0; c < 3; ++c) {
    f.f[c] = (const T*)e->E[lvl][c];
    f.f[3 + c] = (const T*)e->H[lvl][c];
  }
  return f;
}

template <typename T>
int flush_monitors(pf_engine* e) {
  for (DftMon& m : e->dfts) {
    if (m.pending == 0) continue;
    const long long nt = m.r.ncell * m.r.ncomp;
    const int B = 128;
    LaunchScope ls(e, 3);
    k_dft_flush<T><<<(unsigned)((nt + B - 1) / B), B, 0, e->stream>>>(
        m.r, (const T*)m.ring, m.pending, m.acc, m.ph_e, m.ph_h, m.q_done, m.n_freq, m.dt);
    m.q_done += m.pending;
    m.pending = 0;
  }
  for (FluxMon& f : e->fluxes) {
    if (f.pending == 0) continue;
    LaunchScope ls(e, 3);
    k_flux_flush<T><<<1, 256, 0, e->stream>>>(f.partial, f.p.nblk, f.pending, f.acc, f.dA, f.dt);
    f.pending = 0;
  }
  PF_CUDA(e, cudaGetLastError());
  return PF_OK;
}

// Monitors of step s read the level just written (E at t_e, H at t_h).
template <typename T>
int sample_monitors(pf_engine* e, long long s, int lvl, bool dft = true) {
  if (e->dfts.empty() && e->fluxes.empty()) return PF_OK;
  const Fields6<T> f = level_fields<T>(e, lvl);
  for (DftMon& m : e->dfts) {
    if (!dft) break;  // the E pass sampled them
    if (s % m.interval) continue;
    if (m.pending == m.ring_cap) {
      int rc = flush_monitors<T>(e);
      if (rc) return rc;
    }
    const int B = 256;
    LaunchScope ls(e, 2);
    k_dft_sample<T><<<(unsigned)((m.r.ncell + B - 1) / B), B, 0, e->stream>>>(
        m.r, (T*)m.ring, m.pending, f, e->ny, e->nz);
    m.pending++;
  }
  // every flux plane samples every step: up to kFluxBatch planes per launch
  for (size_t q0 = 0; q0 < e->fluxes.size(); q0 += kFluxBatch) {
    const size_t q1 = std::min(e->fluxes.size(), q0 + (size_t)kFluxBatch);
    for (size_t q = q0; q < q1; ++q)
      if (e->fluxes[q].pending == e->fluxes[q].ring_cap) {
        int rc = flush_monitors<T>(e);
        if (rc) return rc;
        break;
      }
    FluxBatch fb;
    memset(&fb, 0, sizeof fb);
    int maxblk = 1;
    for (size_t q = q0; q < q1; ++q) {
      FluxMon& fl = e->fluxes[q];
      fb.p[q - q0] = fl.p;
      fb.partial[q - q0] = fl.partial;
      fb.slot[q - q0] = fl.pending;
      maxblk = std::max(maxblk, fl.p.nblk);
    }
    LaunchScope ls(e, 2);
    k_flux_sample_batch<T><<<dim3(maxblk, (unsigned)(q1 - q0)), 256, 0, e->stream>>>(fb, f, e->ny,
                                                                                     e->nz);
    for (size_t q = q0; q < q1; ++q) e->fluxes[q].pending++;
  }
  return PF_OK;
}

template <typename T>
int inject(pf_engine* e, int fam, int lvl, long long s) {
  SourceGroups& d = e->src[fam].dev;
  if (d.n_groups == 0) return PF_OK;
  void** F = fam == 0 ? e->E[lvl] : e->H[lvl];
  LaunchScope ls(e, 1);
  k_inject<T><<<(d.n_groups + 127) / 128, 128, 0, e->stream>>>(d, (T*)F[0], (T*)F[1], (T*)F[2], s);
  return PF_OK;
}

// An adjoint replay keeps, per step, H^{n+1/2} and psi_E after the step:
// what the reverse step needs to recompute the gradient's g = curl + psi.
template <typename T>
int record_step(pf_engine* e, long long t) {
  if (t < 0 || t >= e->ring_steps) return fail(e, PF_ERR_STATE, "record slot out of range");
  char* base = e->rec + (size_t)t * e->rec_slot;
  const size_t S = sizeof(T), n = (size_t)e->ncell * S;
  size_t off = 0;
  for (int c = 0; c < 3; ++c, off += n)
    PF_CUDA(e, cudaMemcpyAsync(base + off, e->H[e->cur][c], n, cudaMemcpyDeviceToDevice,
                               e->stream));
  for (int q = 0; q < 6; ++q) {
    const size_t b = (size_t)e->npsiE[q] * S;
    if (b) PF_CUDA(e, cudaMemcpyAsync(base + off, e->psiE[q], b, cudaMemcpyDeviceToDevice, e->stream));
    off += b;
  }
  for (FluxMon& f : e->fluxes) {  // E planes of the flux monitors a loss depends on
    if (f.cot == 0.0) continue;
    if (t >= f.rec_cap) return fail(e, PF_ERR_STATE, "flux record slot out of range");
    const long long np = (long long)f.p.n0 * f.p.n1;
    k_flux_plane_record<T><<<(unsigned)((np + 255) / 256), 256, 0, e->stream>>>(
        f.p, (const T*)e->E[e->cur][0], (const T*)e->E[e->cur][1], (const T*)e->E[e->cur][2],
        (T*)f.rec + (size_t)t * 2 * np, e->ny, e->nz);
  }
  PF_CUDA(e, cudaGetLastError());
  return PF_OK;
}

template <typename T>
int advance_typed(pf_engine* e, long long n_sub) {
  const int nz = e->nz, ny = e->ny, nx = e->nx;
  const dim3 blk = nz > 1 ? dim3(32, 8) : dim3(1, 256);
  const dim3 grd((nz + blk.x - 1) / blk.x, (ny + blk.y - 1) / blk.y, nx);
  for (long long t = 0; t < n_sub; ++t) {
    const long long s = e->step;
    const int nxt = e->cur ^ 1;
    StepArgs<T> a = step_args<T>(e);
    if (e->fused) {
      int rc;
      {
        LaunchScope ls(e, 0);
        if (e->tma)
          rc = launch_tma<T>(e->stream, a, e->maps, e->cur, e->ce_mode, e->n_media > 0,
                             e->fused_chunks, e->tma_err);
        else
          rc = launch_fused<T>(e->stream, a, e->ce_mode, e->n_media > 0, e->fused_ty,
                               e->fused_chunks);
      }
      if (rc) return fail(e, PF_ERR_UNSUPPORTED, "fused kernel does not cover this case");
      // sources of the fused path are injected after its single pass: an H
      // source must reach the E update, so the fused path is only chosen
      // when there are no H-family sources.
      inject<T>(e, 0, nxt, s);
    } else {
      {
        LaunchScope ls(e, 0);
        launch_h_split<T>(e, a, grd, blk);
      }
      inject<T>(e, 1, nxt, s);
      a.Hin[0] = a.Hout[0];
      a.Hin[1] = a.Hout[1];
      a.Hin[2] = a.Hout[2];
      EpiArgs<T> ep;
      memset(&ep, 0, sizeof ep);
      if (e->inline_epi) {
        ep.step = s;
        ep.n_isrc = (int)e->src[0].cell.size();
        for (int g = 0; g < ep.n_isrc; ++g) {
          ep.isrc_blk[g] = e->isrc_blk[g];
          ep.isrc_tid[g] = e->isrc_tid[g];
        }
        ep.isrc = e->src[0].dev;
        // an adjoint replay (recording) samples no monitor
        ep.n_idft = e->recording ? 0 : (int)e->dfts.size();
        // a full ring flushes every monitor, so flush before handing out slots
        for (const DftMon& dm : e->dfts) {
          if (!ep.n_idft) break;
          if (s % dm.interval == 0 && dm.pending == dm.ring_cap) {
            const int frc = flush_monitors<T>(e);
            if (frc) return frc;
            break;
          }
        }
        for (int m = 0; m < ep.n_idft; ++m) {
          DftMon& dm = e->dfts[m];
          ep.idft_slot[m] = -1;
          if (s % dm.interval) continue;
          ep.idft[m] = dm.r;
          ep.idft_ring[m] = (T*)dm.ring;
          ep.idft_slot[m] = dm.pending;
        }
      }
      {
        LaunchScope ls(e, 0);
        launch_e_split<T>(e, a, ep, grd, blk);
      }
      if (e->inline_epi) {
        for (int m = 0; m < ep.n_idft; ++m)
          if (ep.idft_slot[m] >= 0) e->dfts[m].pending++;
      } else {
        inject<T>(e, 0, nxt, s);
      }
    }
    int rc = e->recording ? PF_OK : sample_monitors<T>(e, s, nxt, !(e->inline_epi && !e->fused));
    if (rc) return rc;
    e->cur = nxt;
    e->step++;
    if (e->recording && (rc = record_step<T>(e, s - e->rec_step0))) return rc;
    if (e->check_every > 0 && e->step % e->check_every == 0) {
      PF_CUDA(e, cudaGetLastError());
      if ((rc = scan_finite(e))) {
        collect_profile(e);
        return rc;
      }
    }
  }
  PF_CUDA(e, cudaGetLastError());
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  collect_profile(e);
  if (e->tma) {
    int h = 0;
    PF_CUDA(e, cudaMemcpy(&h, e->tma_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h == 2) return fail(e, PF_ERR_CUDA, "TMA staging buffer misaligned; results are invalid");
    if (h) return fail(e, PF_ERR_TIMEOUT, "a TMA stage wait timed out; results are invalid");
  }
  return PF_OK;
}

bool valid_comp(int c) { return c >= 0 && c < 6; }

}  // namespace

namespace pfb {
bool host_recip_division_exact(float d) { return recip_division_exact(d); }
}  // namespace pfb

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* pf_version(void) { return "pfb200 0.1.0 sm_100a"; }

const char* pf_last_error(const pf_engine* e) {
  return e ? e->err.c_str() : g_create_error.c_str();
}

int pf_create(int nx, int ny, int nz, int real_bytes, double dx, double dy, double dz, double ch,
              int64_t n_steps, pf_engine** out) {
  if (!out) return fail(nullptr, PF_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1)
    return fail(nullptr, PF_ERR_INVALID, "grid shape must be positive, got %d x %d x %d", nx, ny, nz);
  if (real_bytes != 4 && real_bytes != 8)
    return fail(nullptr, PF_ERR_INVALID, "real_bytes must be 4 or 8, got %d", real_bytes);
  if (n_steps < 0) return fail(nullptr, PF_ERR_INVALID, "n_steps must be >= 0");
  if ((long long)nx * ny * nz > 0x7fffffffLL)
    return fail(nullptr, PF_ERR_UNSUPPORTED, "more than 2^31-1 cells");
  if (!(dx > 0 && dy > 0 && dz > 0)) return fail(nullptr, PF_ERR_INVALID, "spacings must be > 0");
  pf_engine* e = new pf_engine();
  e->nx = nx;
  e->ny = ny;
  e->nz = nz;
  e->rb = real_bytes;
  e->dl[0] = dx;
  e->dl[1] = dy;
  e->dl[2] = dz;
  e->ch = ch;
  e->n_steps = n_steps;
  e->ncell = (long long)nx * ny * nz;
  cudaError_t rc = cudaGetDevice(&e->device);
  if (rc == cudaSuccess) rc = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (rc != cudaSuccess) {
    fail(nullptr, PF_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(rc));
    delete e;
    return PF_ERR_CUDA;
  }
  *out = e;
  return PF_OK;
}

int pf_set_ce(pf_engine* e, int mode, const void* ce0, const void* ce1, const void* ce2,
              const uint32_t* word, int n_table, const double* table) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_set_ce after pf_finalize");
  const size_t bytes = (size_t)e->ncell * e->rb;
  for (int c = 0; c < 3; ++c) e->h_ce[c].clear();
  e->h_table.clear();
  if (mode == PF_CE_CELL1) {
    if (!ce0) return fail(e, PF_ERR_INVALID, "PF_CE_CELL1 needs ce0");
    e->h_ce[0].assign((const char*)ce0, (const char*)ce0 + bytes);
  } else if (mode == PF_CE_CELL3) {
    if (!ce0 || !ce1 || !ce2) return fail(e, PF_ERR_INVALID, "PF_CE_CELL3 needs three arrays");
    const void* src[3] = {ce0, ce1, ce2};
    for (int c = 0; c < 3; ++c) e->h_ce[c].assign((const char*)src[c], (const char*)src[c] + bytes);
  } else if (mode == PF_CE_TABLE) {
    if (!word || n_table < 1 || !table) return fail(e, PF_ERR_INVALID, "PF_CE_TABLE needs word and table");
    // one pass: plain words index the table; per medium, the largest record
    // index its dispersive words name (checked against its cell count at
    // pf_finalize). The word then goes to the device straight from the
    // caller's buffer, with no host copy.
    long long need[kMaxMedia] = {};
    for (long long q = 0; q < e->ncell; ++q) {
      const uint32_t w = word[q];
      if (w & kDispersiveBit) {
        const int m = (int)((w >> kMediumShift) & 15u);
        need[m] = std::max(need[m], (long long)(w & kLocMask) + 1);
      } else if (w >= (uint32_t)n_table) {
        return fail(e, PF_ERR_INVALID, "ce word %u at cell %lld exceeds table size %d", w, q, n_table);
      }
    }
    const size_t wb = (size_t)e->ncell * 4;
    PF_CUDA(e, cudaSetDevice(e->device));
    if (!e->word) {
      int rc = dalloc(e, (void**)&e->word, wb);
      if (rc) return rc;
    }
    PF_CUDA(e, cudaMemcpyAsync(e->word, word, wb, cudaMemcpyHostToDevice, e->stream));
    PF_CUDA(e, cudaStreamSynchronize(e->stream));
    memcpy(e->word_need, need, sizeof need);
    e->h_table.assign(table, table + n_table);
  } else {
    return fail(e, PF_ERR_INVALID, "unknown ce mode %d", mode);
  }
  e->ce_mode = mode;
  return PF_OK;
}

int pf_set_cpml(pf_engine* e, int axis, const void* b_e, const void* c_e, const void* b_h,
                const void* c_h) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_set_cpml after pf_finalize");
  if (axis < 0 || axis > 2) return fail(e, PF_ERR_INVALID, "axis must be 0..2");
  const int dims[3] = {e->nx, e->ny, e->nz};
  const size_t bytes = (size_t)dims[axis] * e->rb;
  const void* src[4] = {b_e, c_e, b_h, c_h};
  for (int q = 0; q < 4; ++q) {
    e->h_cpml[axis][q].clear();
    if (src[q]) e->h_cpml[axis][q].assign((const char*)src[q], (const char*)src[q] + bytes);
  }
  return PF_OK;
}

int pf_set_ade(pf_engine* e, int n_media, const int64_t* count, const int32_t* npole,
               const double* coef, const double* inv_eps, const double* ce_m,
               const uint32_t* cell_word) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_set_ade after pf_finalize");
  if (n_media < 0 || n_media > kMaxMedia)
    return fail(e, PF_ERR_UNSUPPORTED, "at most %d dispersive media, got %d", kMaxMedia, n_media);
  e->n_media = n_media;
  e->m_count.assign(count, count + n_media);
  e->m_npole.assign(npole, npole + n_media);
  long long ncoef = 0;
  for (int m = 0; m < n_media; ++m) {
    if (npole[m] < 0 || npole[m] > kMaxPoles)
      return fail(e, PF_ERR_UNSUPPORTED, "at most %d poles per medium, got %d", kMaxPoles, npole[m]);
    if (count[m] < 0 || count[m] > (long long)kLocMask + 1)
      return fail(e, PF_ERR_UNSUPPORTED, "at most 2^%d cells per dispersive medium", kMediumShift);
    ncoef += 3LL * npole[m];
  }
  e->m_coef.assign(coef, coef + ncoef);
  e->m_inv.assign(inv_eps, inv_eps + n_media);
  e->m_ce.clear();
  if (ce_m) e->m_ce.assign(ce_m, ce_m + n_media);
  e->h_adeword.clear();
  if (cell_word) {
    for (long long q = 0; q < e->ncell; ++q) {
      const uint32_t w = cell_word[q];
      if (w && (!(w & kDispersiveBit) || (int)((w >> kMediumShift) & 15u) >= n_media ||
                (long long)(w & kLocMask) >= count[(w >> kMediumShift) & 15u]))
        return fail(e, PF_ERR_INVALID, "bad dispersive word 0x%08x at cell %lld", w, q);
    }
    e->h_adeword.assign(cell_word, cell_word + e->ncell);
  }
  return PF_OK;
}

int pf_rank_dispersive_words(uint32_t* word, int64_t n, int n_media, int64_t* counts,
                             int clear_plain) {
  if (!word || !counts || n < 0) return fail(nullptr, PF_ERR_INVALID, "NULL word or counts");
  if (n_media < 0 || n_media > kMaxMedia)
    return fail(nullptr, PF_ERR_UNSUPPORTED, "at most %d dispersive media, got %d", kMaxMedia,
                n_media);
  long long cnt[kMaxMedia] = {0};
  for (long long q = 0; q < n; ++q) {
    const uint32_t w = word[q];
    if (!(w & kDispersiveBit)) {
      if (clear_plain) word[q] = 0u;
      continue;
    }
    const int m = (int)((w >> kMediumShift) & 15u);
    if (m >= n_media || (w & kLocMask))
      return fail(nullptr, PF_ERR_INVALID, "bad dispersive word 0x%08x at cell %lld", w, q);
    if (cnt[m] > (long long)kLocMask)
      return fail(nullptr, PF_ERR_UNSUPPORTED, "more than 2^%d cells in one dispersive medium",
                  kMediumShift);
    word[q] = w | (uint32_t)cnt[m]++;
  }
  for (int m = 0; m < n_media; ++m) counts[m] = cnt[m];
  return PF_OK;
}

int pf_set_sources(pf_engine* e, int n_src, const int32_t* comp, const int64_t* cell,
                   const int32_t* wave_row, const double* amp, int n_wave, const double* wave) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_set_sources after pf_finalize");
  for (int f = 0; f < 2; ++f) e->src[f] = SrcFamily();
  e->n_wave = n_wave;
  e->h_wave.assign(wave, wave + (size_t)n_wave * e->n_steps);
  // group by (component, cell), keeping list order inside each group
  for (int f = 0; f < 2; ++f) {
    SrcFamily& s = e->src[f];
    std::vector<std::pair<long long, int>> key;  // (comp*ncell + cell, source)
    for (int q = 0; q < n_src; ++q) {
      if (!valid_comp(comp[q])) return fail(e, PF_ERR_INVALID, "source %d: bad component %d", q, comp[q]);
      if (cell[q] < 0 || cell[q] >= e->ncell) return fail(e, PF_ERR_INVALID, "source %d: cell out of range", q);
      if (wave_row[q] < 0 || wave_row[q] >= n_wave) return fail(e, PF_ERR_INVALID, "source %d: bad waveform row", q);
      if ((comp[q] >= 3) != (f == 1)) continue;
      key.push_back({(long long)(comp[q] % 3) * e->ncell + cell[q], q});
    }
    std::stable_sort(key.begin(), key.end(),
                     [](const std::pair<long long, int>& x, const std::pair<long long, int>& y) {
                       return x.first < y.first;
                     });
    for (size_t q = 0; q < key.size(); ++q) {
      if (q == 0 || key[q].first != key[q - 1].first) {
        s.cell.push_back(key[q].first % e->ncell);
        s.comp.push_back((int)(key[q].first / e->ncell));
        s.start.push_back((int)s.wave_row.size());
      }
      s.wave_row.push_back(wave_row[key[q].second]);
      s.amp.push_back(amp[key[q].second]);
    }
    s.start.push_back((int)s.wave_row.size());
  }
  return PF_OK;
}

int pf_add_dft(pf_engine* e, const int32_t start[3], const int32_t stop[3], const int32_t stride[3],
               int comp_mask, int n_freq, int interval, const double* phase_e,
               const double* phase_h, double dt, int* mon) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_add_dft after pf_finalize");
  if (n_freq < 1 || interval < 1 || !(comp_mask & 63) || !phase_e || !phase_h)
    return fail(e, PF_ERR_INVALID, "bad DFT monitor arguments");
  const int dims[3] = {e->nx, e->ny, e->nz};
  DftMon m;
  m.r.ncell = 1;
  for (int a = 0; a < 3; ++a) {
    if (start[a] < 0 || stop[a] > dims[a] || stop[a] <= start[a] || stride[a] < 1)
      return fail(e, PF_ERR_INVALID, "bad DFT region on axis %d", a);
    m.r.start[a] = start[a];
    m.r.stride[a] = stride[a];
    m.r.count[a] = (stop[a] - start[a] + stride[a] - 1) / stride[a];
    m.r.ncell *= m.r.count[a];
  }
  m.r.ncomp = 0;
  for (int c = 0; c < 6; ++c)
    if (comp_mask & (1 << c)) m.r.comps[m.r.ncomp++] = c;
  m.n_freq = n_freq;
  m.interval = interval;
  m.dt = dt;
  m.n_samples = e->n_steps > 0 ? (e->n_steps + interval - 1) / interval : 0;
  m.h_ph_e.assign(phase_e, phase_e + m.n_samples * n_freq * 2);
  m.h_ph_h.assign(phase_h, phase_h + m.n_samples * n_freq * 2);
  e->dfts.push_back(std::move(m));
  if (mon) *mon = (int)e->dfts.size() - 1;
  return PF_OK;
}

int pf_add_flux(pf_engine* e, int axis, int idx, double dA, double dt, int* mon) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_add_flux after pf_finalize");
  const int dims[3] = {e->nx, e->ny, e->nz};
  if (axis < 0 || axis > 2 || idx < 0 || idx >= dims[axis])
    return fail(e, PF_ERR_INVALID, "bad flux plane (axis %d, index %d)", axis, idx);
  FluxMon f;
  f.p.axis = axis;
  f.p.idx = idx;
  f.p.n0 = axis == 0 ? e->ny : e->nx;
  f.p.n1 = axis == 2 ? e->ny : e->nz;
  f.p.nblk = (int)(((long long)f.p.n0 * f.p.n1 + 255) / 256);
  f.dA = dA;
  f.dt = dt;
  e->fluxes.push_back(f);
  if (mon) *mon = (int)e->fluxes.size() - 1;
  return PF_OK;
}

int pf_set_kernel(pf_engine* e, int kernel) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_set_kernel after pf_finalize");
  if (kernel < PF_KERNEL_AUTO || kernel > PF_KERNEL_FUSED)
    return fail(e, PF_ERR_INVALID, "unknown kernel %d", kernel);
  e->kernel = kernel;
  return PF_OK;
}

int pf_finalize(pf_engine* e) {
  if (!e) return PF_ERR_INVALID;
  if (e->finalized) return fail(e, PF_ERR_STATE, "pf_finalize called twice");
  if (e->ce_mode < 0) return fail(e, PF_ERR_INVALID, "pf_set_ce was not called");
  if (e->n_media > 0 && e->ce_mode == PF_CE_CELL3)
    return fail(e, PF_ERR_UNSUPPORTED, "dispersive media with a three-component coefficient");
  if (e->n_media > 0 && e->ce_mode == PF_CE_CELL1 && e->h_adeword.size() != (size_t)e->ncell)
    return fail(e, PF_ERR_INVALID, "PF_CE_CELL1 with dispersive media needs cell_word");
  if (e->ce_mode == PF_CE_TABLE)
    for (int m = 0; m < kMaxMedia; ++m)
      if (e->word_need[m] > 0 && (m >= e->n_media || e->word_need[m] > e->m_count[m]))
        return fail(e, PF_ERR_INVALID,
                    "bad dispersive word: medium %d record %lld, but the medium has %lld cells", m,
                    e->word_need[m] - 1, m < e->n_media ? e->m_count[m] : 0LL);
  const bool has_h_src = !e->src[1].cell.empty();
  const bool fusable = fused_supported(e->nx, e->ny, e->nz) && !has_h_src;
  if (e->kernel == PF_KERNEL_FUSED && !fusable)
    return fail(e, PF_ERR_UNSUPPORTED, "the fused kernel needs a 3D grid without H-family sources");
  // AUTO takes the split passes: on B200 they currently outrun the fused
  // kernel (measured: config-3 384^3 2.05 vs 2.54 ms/step), whose plane loop
  // is latency-bound. PF_KERNEL_FUSED selects it explicitly.
  e->fused = e->kernel == PF_KERNEL_FUSED;
  (void)fusable;
  if (e->fused) {
    if (const char* v = getenv("PFB200_FUSED_TY")) e->fused_ty = atoi(v) == 16 ? 16 : 8;
    const long long tiles = (long long)((e->nz + 31) / 32) * ((e->ny + e->fused_ty - 1) / e->fused_ty);
    // about one resident wave of blocks (148 SMs x 1024 threads), at least
    // 8 planes per chunk
    int nch = (int)std::max<long long>(1, (148LL * 1024 / (32 * e->fused_ty) + tiles / 2) / tiles);
    nch = std::max(nch, (e->nx + 11) / 12);  // short chunks hide the plane-loop latency
    nch = std::min(nch, std::max(1, e->nx / 8));
    if (const char* v = getenv("PFB200_XCHUNKS")) nch = std::max(1, atoi(v));
    e->fused_chunks = nch;
  }
  if (e->rb == 4) {
    const int dims[3] = {e->nx, e->ny, e->nz};
    for (int ax = 0; ax < 3; ++ax) {
      const float d = (float)e->dl[ax];
      e->rdl[ax] = (double)(1.0f / d);
      bool same = false;
      for (int q = 0; q < ax; ++q)
        if (dims[q] > 1 && (float)e->dl[q] == d) {
          e->fdiv[ax] = e->fdiv[q];
          same = true;
        }
      if (!same && dims[ax] > 1 && !getenv("PFB200_IEEE_DIV")) e->fdiv[ax] = recip_division_exact(d);
    }
  }
  int rc = e->rb == 4 ? finalize_typed<float>(e) : finalize_typed<double>(e);
  if (rc) return rc;
  e->inline_epi = !e->fused && getenv("PFB200_INLINE") &&
                  e->src[0].cell.size() <= (size_t)kInlineSrc &&
                  e->dfts.size() <= (size_t)kInlineDft;
  if (e->inline_epi) {
    // each E source group's block and thread in the E pass's grid
    const int bx = e->nz > 1 ? 32 : 1, by = e->nz > 1 ? 8 : 256;
    const long long gx = (e->nz + bx - 1) / bx, gy = (e->ny + by - 1) / by;
    for (size_t g = 0; g < e->src[0].cell.size(); ++g) {
      const long long c = e->src[0].cell[g];
      const long long i = c / ((long long)e->ny * e->nz), j = (c / e->nz) % e->ny, k = c % e->nz;
      e->isrc_blk[g] = (int)((i * gy + j / by) * gx + k / bx);
      e->isrc_tid[g] = (int)((j % by) * bx + k % bx);
    }
  }
  // host staging no longer needed
  for (int c = 0; c < 3; ++c) std::vector<char>().swap(e->h_ce[c]);
  std::vector<uint32_t>().swap(e->h_adeword);
  e->finalized = true;
  return PF_OK;
}

int pf_advance(pf_engine* e, int64_t step0, int64_t n_sub) {
  if (!e) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_advance before pf_finalize");
  if (step0 != e->step)
    return fail(e, PF_ERR_INVALID, "pf_advance(step0=%lld) but the engine is at step %lld",
                (long long)step0, e->step);
  if (n_sub < 0 || e->step + n_sub > e->n_steps)
    return fail(e, PF_ERR_INVALID, "advance past n_steps (%lld)", e->n_steps);
  PF_CUDA(e, cudaSetDevice(e->device));
  return e->rb == 4 ? advance_typed<float>(e, n_sub) : advance_typed<double>(e, n_sub);
}

int pf_read_field(pf_engine* e, int comp, void* dst) {
  if (!e || !dst) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_read_field before pf_finalize");
  if (!valid_comp(comp)) return fail(e, PF_ERR_INVALID, "bad component %d", comp);
  void* src = comp < 3 ? e->E[e->cur][comp] : e->H[e->cur][comp - 3];
  PF_CUDA(e, cudaMemcpyAsync(dst, src, (size_t)e->ncell * e->rb, cudaMemcpyDeviceToHost, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

int pf_read_dft(pf_engine* e, int mon, int comp, double* dst) {
  if (!e || !dst) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_read_dft before pf_finalize");
  if (mon < 0 || mon >= (int)e->dfts.size()) return fail(e, PF_ERR_INVALID, "bad DFT monitor %d", mon);
  DftMon& m = e->dfts[mon];
  int qc = -1;
  for (int q = 0; q < m.r.ncomp; ++q)
    if (m.r.comps[q] == comp) qc = q;
  if (qc < 0) return fail(e, PF_ERR_INVALID, "component %d not recorded by DFT monitor %d", comp, mon);
  int rc = e->rb == 4 ? flush_monitors<float>(e) : flush_monitors<double>(e);
  if (rc) return rc;
  const size_t per = (size_t)m.n_freq * m.r.ncell * 16;
  PF_CUDA(e, cudaMemcpyAsync(dst, (const char*)m.acc + per * qc, per, cudaMemcpyDeviceToHost, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

int pf_read_flux(pf_engine* e, int mon, double* dst) {
  if (!e || !dst) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_read_flux before pf_finalize");
  if (mon < 0 || mon >= (int)e->fluxes.size()) return fail(e, PF_ERR_INVALID, "bad flux monitor %d", mon);
  int rc = e->rb == 4 ? flush_monitors<float>(e) : flush_monitors<double>(e);
  if (rc) return rc;
  PF_CUDA(e, cudaMemcpyAsync(dst, e->fluxes[mon].acc, 8, cudaMemcpyDeviceToHost, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

int pf_read_region(pf_engine* e, int comp, const int32_t start[3], const int32_t stop[3],
                   const int32_t stride[3], void* dst) {
  if (!e || !dst || !start || !stop || !stride) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_read_region before pf_finalize");
  if (!valid_comp(comp)) return fail(e, PF_ERR_INVALID, "bad component %d", comp);
  const int dims[3] = {e->nx, e->ny, e->nz};
  int cnt[3];
  for (int a = 0; a < 3; ++a) {
    if (stride[a] < 1 || start[a] < 0 || stop[a] > dims[a] || start[a] >= stop[a])
      return fail(e, PF_ERR_INVALID, "bad region on axis %d", a);
    cnt[a] = (stop[a] - start[a] + stride[a] - 1) / stride[a];
  }
  const long long n = (long long)cnt[0] * cnt[1] * cnt[2];
  const size_t bytes = (size_t)n * e->rb;
  PF_CUDA(e, cudaSetDevice(e->device));
  const void* src = comp < 3 ? e->E[e->cur][comp] : e->H[e->cur][comp - 3];
  if (n == e->ncell) {  // the whole field: no gather
    PF_CUDA(e, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, e->stream));
    PF_CUDA(e, cudaStreamSynchronize(e->stream));
    return PF_OK;
  }
  if (bytes > e->region_bytes) {
    if (e->region) {
      PF_CUDA(e, cudaStreamSynchronize(e->stream));
      cudaFree(e->region);
      e->dev_bytes -= e->region_bytes;
      e->region = nullptr;
      e->region_bytes = 0;
    }
    const cudaError_t rc = cudaMalloc(&e->region, bytes);
    if (rc != cudaSuccess)
      return fail(e, PF_ERR_OOM, "CUDA error: cudaMalloc of %zu bytes failed", bytes);
    e->region_bytes = bytes;
    e->dev_bytes += bytes;
  }
  const int3 st = make_int3(start[0], start[1], start[2]);
  const int3 sd = make_int3(stride[0], stride[1], stride[2]);
  const int3 ct = make_int3(cnt[0], cnt[1], cnt[2]);
  const unsigned g = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (e->rb == 4)
    k_gather_region<float><<<g, 256, 0, e->stream>>>((const float*)src, e->ny, e->nz, st, sd, ct,
                                                     (float*)e->region);
  else
    k_gather_region<double><<<g, 256, 0, e->stream>>>((const double*)src, e->ny, e->nz, st, sd,
                                                      ct, (double*)e->region);
  PF_CUDA(e, cudaGetLastError());
  PF_CUDA(e, cudaMemcpyAsync(dst, e->region, bytes, cudaMemcpyDeviceToHost, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

int pf_write_field(pf_engine* e, int comp, const void* src) {
  if (!e || !src) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_write_field before pf_finalize");
  if (!valid_comp(comp)) return fail(e, PF_ERR_INVALID, "bad component %d", comp);
  PF_CUDA(e, cudaSetDevice(e->device));
  void* dst = comp < 3 ? e->E[e->cur][comp] : e->H[e->cur][comp - 3];
  PF_CUDA(e, cudaMemcpyAsync(dst, src, (size_t)e->ncell * e->rb, cudaMemcpyHostToDevice, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

namespace {
// The stepping state as a list of (device pointer, bytes) pieces in the
// order of the state blob: the six current field components, the six E psi
// arrays, the six current H psi arrays, then the polarisation level holding
// P^n followed by the one holding P^(n-1) for `step` n.
std::vector<std::pair<char*, size_t>> state_pieces(pf_engine* e, long long step) {
  std::vector<std::pair<char*, size_t>> v;
  const size_t S = e->rb, n = (size_t)e->ncell * S;
  for (int c = 0; c < 3; ++c) v.push_back({(char*)e->E[e->cur][c], n});
  for (int c = 0; c < 3; ++c) v.push_back({(char*)e->H[e->cur][c], n});
  for (int q = 0; q < 6; ++q) v.push_back({(char*)e->psiE[q], (size_t)e->npsiE[q] * S});
  for (int q = 0; q < 6; ++q) v.push_back({(char*)e->psiH[e->cur][q], (size_t)e->npsiH[q] * S});
  if (e->n_media > 0) {
    const size_t lev = (size_t)e->plev * S;
    const int ln = (int)(step & 1);
    v.push_back({(char*)e->P + ln * lev, lev});
    v.push_back({(char*)e->P + (ln ^ 1) * lev, lev});
  }
  return v;
}

int copy_state(pf_engine* e, long long step, void* buf, int64_t bytes, int on_device, bool get) {
  if (!e || !buf) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "state access before pf_finalize");
  const auto pieces = state_pieces(e, step);
  size_t total = 0;
  for (const auto& p : pieces) total += p.second;
  if ((int64_t)total != bytes)
    return fail(e, PF_ERR_INVALID, "state buffer holds %lld bytes, the state is %zu",
                (long long)bytes, total);
  PF_CUDA(e, cudaSetDevice(e->device));
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice
                                        : (get ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice);
  size_t off = 0;
  for (const auto& p : pieces) {
    if (p.second) {
      char* b = (char*)buf + off;
      if (get) PF_CUDA(e, cudaMemcpyAsync(b, p.first, p.second, kind, e->stream));
      else PF_CUDA(e, cudaMemcpyAsync(p.first, b, p.second, kind, e->stream));
    }
    off += p.second;
  }
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}
}  // namespace

int pf_state_bytes(const pf_engine* e, int64_t* bytes) {
  if (!e || !bytes) return PF_ERR_INVALID;
  if (!e->finalized) return PF_ERR_STATE;
  size_t total = 0;
  for (const auto& p : state_pieces(const_cast<pf_engine*>(e), e->step)) total += p.second;
  *bytes = (int64_t)total;
  return PF_OK;
}

int pf_get_state(pf_engine* e, void* dst, int64_t bytes, int dst_on_device) {
  if (!e) return PF_ERR_INVALID;
  return copy_state(e, e->step, dst, bytes, dst_on_device, true);
}

int pf_set_state(pf_engine* e, int64_t step, const void* src, int64_t bytes, int src_on_device) {
  if (!e) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_set_state before pf_finalize");
  if (step < 0 || step > e->n_steps)
    return fail(e, PF_ERR_INVALID, "step %lld outside [0, n_steps]", (long long)step);
  // samples already taken belong to the old timeline: fold them first
  int rc = e->rb == 4 ? flush_monitors<float>(e) : flush_monitors<double>(e);
  if (rc) return rc;
  rc = copy_state(e, step, const_cast<void*>(src), bytes, src_on_device, false);
  if (rc) return rc;
  e->step = step;
  return PF_OK;
}

int pf_step(const pf_engine* e, int64_t* step) {
  if (!e || !step) return PF_ERR_INVALID;
  *step = e->step;
  return PF_OK;
}

int pf_check_finite(pf_engine* e) {
  if (!e) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_check_finite before pf_finalize");
  PF_CUDA(e, cudaSetDevice(e->device));
  return scan_finite(e);
}

int pf_set_check_every(pf_engine* e, int64_t k) {
  if (!e) return PF_ERR_INVALID;
  if (k < 0) return fail(e, PF_ERR_INVALID, "check period must be >= 0");
  e->check_every = k;
  return PF_OK;
}

int pf_set_wait_test(pf_engine* e, int on) {
  if (!e) return PF_ERR_INVALID;
  e->wait_test = on ? 1 : 0;
  return PF_OK;
}

int pf_stream(const pf_engine* e, void** stream) {
  if (!e || !stream) return PF_ERR_INVALID;
  *stream = (void*)e->stream;
  return PF_OK;
}

int pf_set_profiling(pf_engine* e, int on) {
  if (!e) return PF_ERR_INVALID;
  e->profiling = on != 0;
  return PF_OK;
}

int pf_read_profile(pf_engine* e, int64_t launches[4], double ms[4], int reset) {
  if (!e) return PF_ERR_INVALID;
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  collect_profile(e);
  for (int k = 0; k < 4; ++k) {
    if (launches) launches[k] = e->launches[k];
    if (ms) ms[k] = e->prof_ms[k];
    if (reset) {
      e->launches[k] = 0;
      e->prof_ms[k] = 0.0;
    }
  }
  return PF_OK;
}

int pf_info(const pf_engine* e, char* buf, int len) {
  if (!e || !buf || len < 1) return PF_ERR_INVALID;
  snprintf(buf, (size_t)len,
           "kernel=%s fused_ty=%d x_chunks=%d qdiv=%d%d%d ce_mode=%d media=%d real_bytes=%d "
           "tma=%d "
           "shape=%dx%dx%d dft=%zu flux=%zu",
           e->fused ? "fused" : "split", e->fused_ty, e->fused_chunks, (int)e->fdiv[0],
           (int)e->fdiv[1], (int)e->fdiv[2], e->ce_mode, e->n_media, e->rb, (int)e->tma, e->nx,
           e->ny, e->nz,
           e->dfts.size(), e->fluxes.size());
  return PF_OK;
}

int pf_device_bytes(const pf_engine* e, int64_t* bytes) {
  if (!e || !bytes) return PF_ERR_INVALID;
  *bytes = (int64_t)e->dev_bytes;
  return PF_OK;
}

void pf_destroy(pf_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (void* p : e->allocs) cudaFree(p);
  if (e->region) cudaFree(e->region);
  for (cudaEvent_t ev : e->ev_pool) cudaEventDestroy(ev);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of the stepping (value_and_grad_eps, jaxbackend.py:666-722): the
// caller checkpoints the forward run with pf_get_state, hands the loss's
// sensitivities to its outputs to pf_adj_set_dft_cotangent /
// pf_adj_add_field_source, then calls pf_adj_segment on the checkpointed
// segments from the last to the first. Each call restores the segment's
// state, replays it recording H^{n+1/2} and psi_E per step (no monitor
// sampling), and runs its reverse steps (kernels_adj.cuh), accumulating
// dJ/dK per cell.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
AdjState<T> adj_state(pf_engine* e, long long slot) {
  AdjState<T> s;
  memset(&s, 0, sizeof s);
  const char* base = e->rec + (size_t)slot * e->rec_slot;
  const size_t S = sizeof(T), n = (size_t)e->ncell * S;
  size_t off = 0;
  for (int c = 0; c < 3; ++c, off += n) s.Hrec[c] = (const T*)(base + off);
  for (int q = 0; q < 6; ++q) {
    s.psiErec[q] = (const T*)(base + off);
    off += (size_t)e->npsiE[q] * S;
  }
  for (int c = 0; c < 3; ++c) {
    s.lamE[c] = (T*)e->lamE[c];
    s.lamH[c] = (T*)e->lamH[c];
  }
  for (int q = 0; q < 6; ++q) {
    s.gE[q] = (T*)e->gE[q];
    s.gH[q] = (T*)e->gH[q];
    s.lpE[q] = (T*)e->lpE[q];
    s.lpH[q] = (T*)e->lpH[q];
  }
  s.grad = e->grad;
  s.ncell = e->ncell;
  // per-component coefficients are differentiated per component; one
  // coefficient per cell needs only the sum (16 instead of 48 bytes of
  // gradient traffic per cell and reverse step)
  s.gstride = e->ce_mode == PF_CE_CELL3 ? e->ncell : 0;
  for (int a = 0; a < 3; ++a) s.idl[a] = (T)(1.0 / e->dl[a]);
  return s;
}

// The loss's sources on the fields sampled at step m, family fam (0: E^{m+1},
// 1: H^{m+1/2}).
template <typename T>
int adj_sources(pf_engine* e, long long m, int fam, const AdjState<T>& st, long long slot) {
  const int B = 256;
  T* l[3];
  for (int c = 0; c < 3; ++c) l[c] = (T*)(fam == 0 ? e->lamE[c] : e->lamH[c]);
  for (size_t k = 0; k < e->dfts.size(); ++k) {
    const DftMon& dm = e->dfts[k];
    if (!e->dft_cot[k] || m % dm.interval) continue;
    const long long q = m / dm.interval;
    const double* ph = (fam == 0 ? dm.ph_e : dm.ph_h) + q * dm.n_freq * 2;
    const long long nt = dm.r.ncell * dm.r.ncomp;
    k_adj_dft_src<T><<<(unsigned)((nt + B - 1) / B), B, 0, e->stream>>>(
        dm.r, e->dft_cot[k], ph, dm.n_freq, dm.dt, fam, l[0], l[1], l[2], e->ny, e->nz);
  }
  for (const FluxMon& f : e->fluxes) {
    if (f.cot == 0.0) continue;
    const long long np = (long long)f.p.n0 * f.p.n1;
    k_adj_flux_src<T><<<(unsigned)((np + B - 1) / B), B, 0, e->stream>>>(
        f.p, f.cot * f.dA * f.dt, fam, st.Hrec[0], st.Hrec[1], st.Hrec[2],
        (const T*)f.rec + (size_t)slot * 2 * np, l[0], l[1], l[2], e->ny, e->nz);
  }
  for (const auto& rs : e->rsrc) {
    if (rs.step != m || (rs.comp >= 3) != (fam == 1)) continue;
    k_adj_region_src<T><<<(unsigned)((rs.r.ncell + B - 1) / B), B, 0, e->stream>>>(
        rs.r, rs.vals, l[rs.comp % 3], e->ny, e->nz);
  }
  PF_CUDA(e, cudaGetLastError());
  return PF_OK;
}

template <typename T>
int adj_segment_typed(pf_engine* e, long long step0, long long n) {
  e->recording = true;
  e->rec_step0 = step0;
  int rc = advance_typed<T>(e, n);
  e->recording = false;
  if (rc) return rc;
  const int nz = e->nz, ny = e->ny, nx = e->nx;
  const dim3 blk = nz > 1 ? dim3(32, 8) : dim3(1, 256);
  const dim3 grd((nz + blk.x - 1) / blk.x, (ny + blk.y - 1) / blk.y, nx);
  const StepArgs<T> a = step_args<T>(e);
  for (long long m = step0 + n - 1; m >= step0; --m) {
    const AdjState<T> s = adj_state<T>(e, m - step0);
    if ((rc = adj_sources<T>(e, m, 0, s, m - step0))) return rc;
    if (e->ce_mode == PF_CE_CELL1)
      k_adj_e<T, kCeCell1><<<grd, blk, 0, e->stream>>>(a, s);
    else if (e->ce_mode == PF_CE_CELL3)
      k_adj_e<T, kCeCell3><<<grd, blk, 0, e->stream>>>(a, s);
    else
      k_adj_e<T, kCeTable><<<grd, blk, 0, e->stream>>>(a, s);
    if ((rc = adj_sources<T>(e, m, 1, s, m - step0))) return rc;
    k_adj_h<T><<<grd, blk, 0, e->stream>>>(a, s);
  }
  PF_CUDA(e, cudaGetLastError());
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  e->adj_next = step0;
  return PF_OK;
}

int adj_zero(pf_engine* e) {
  const size_t S = e->rb, n = (size_t)e->ncell * S;
  for (int c = 0; c < 3; ++c) {
    PF_CUDA(e, cudaMemsetAsync(e->lamE[c], 0, n, e->stream));
    PF_CUDA(e, cudaMemsetAsync(e->lamH[c], 0, n, e->stream));
  }
  for (int q = 0; q < 6; ++q) {
    PF_CUDA(e, cudaMemsetAsync(e->gE[q], 0, n, e->stream));
    PF_CUDA(e, cudaMemsetAsync(e->gH[q], 0, n, e->stream));
    if (e->npsiE[q]) PF_CUDA(e, cudaMemsetAsync(e->lpE[q], 0, e->npsiE[q] * S, e->stream));
    if (e->npsiH[q]) PF_CUDA(e, cudaMemsetAsync(e->lpH[q], 0, e->npsiH[q] * S, e->stream));
  }
  PF_CUDA(e, cudaMemsetAsync(e->grad, 0, (size_t)e->ncell * 24, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  e->adj_next = e->n_steps;
  return PF_OK;
}

bool make_region(pf_engine* e, const int32_t start[3], const int32_t stop[3],
                 const int32_t stride[3], DftRegion& r) {
  const int dims[3] = {e->nx, e->ny, e->nz};
  r.ncell = 1;
  r.ncomp = 1;
  for (int a = 0; a < 3; ++a) {
    if (start[a] < 0 || stop[a] > dims[a] || stop[a] <= start[a] || stride[a] < 1) return false;
    r.start[a] = start[a];
    r.stride[a] = stride[a];
    r.count[a] = (stop[a] - start[a] + stride[a] - 1) / stride[a];
    r.ncell *= r.count[a];
  }
  return true;
}

}  // namespace

extern "C" {

int pf_adj_init(pf_engine* e, int64_t ring_steps) {
  if (!e) return PF_ERR_INVALID;
  if (!e->finalized) return fail(e, PF_ERR_STATE, "pf_adj_init before pf_finalize");
  if (e->n_media > 0)
    return fail(e, PF_ERR_UNSUPPORTED, "the adjoint does not cover dispersive (ADE) media");
  if (ring_steps < 1 || ring_steps > e->n_steps)
    return fail(e, PF_ERR_INVALID, "ring_steps %lld outside [1, n_steps]", (long long)ring_steps);
  PF_CUDA(e, cudaSetDevice(e->device));
  int rc;
  const size_t S = e->rb, n = (size_t)e->ncell * S;
  if (!e->adj) {
    for (int c = 0; c < 3; ++c) {
      if ((rc = dalloc(e, &e->lamE[c], n))) return rc;
      if ((rc = dalloc(e, &e->lamH[c], n))) return rc;
    }
    for (int q = 0; q < 6; ++q) {
      if ((rc = dalloc(e, &e->gE[q], n))) return rc;
      if ((rc = dalloc(e, &e->gH[q], n))) return rc;
      if ((rc = dalloc(e, &e->lpE[q], e->npsiE[q] * S))) return rc;
      if ((rc = dalloc(e, &e->lpH[q], e->npsiH[q] * S))) return rc;
    }
    if ((rc = dalloc(e, (void**)&e->grad, (size_t)e->ncell * 24))) return rc;
    e->dft_cot.assign(e->dfts.size(), nullptr);
    e->adj = true;
  }
  if (ring_steps > e->ring_steps) {
    size_t slot = 3 * n;
    for (int q = 0; q < 6; ++q) slot += e->npsiE[q] * S;
    e->rec_slot = (slot + 255) & ~(size_t)255;
    // the old ring stays allocated (freed with the engine)
    if ((rc = dalloc(e, (void**)&e->rec, e->rec_slot * (size_t)ring_steps))) return rc;
    e->ring_steps = ring_steps;
  }
  return adj_zero(e);
}

int pf_adj_set_dft_cotangent(pf_engine* e, int mon, const double* cot) {
  if (!e || !cot) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "pf_adj_set_dft_cotangent before pf_adj_init");
  if (mon < 0 || mon >= (int)e->dfts.size()) return fail(e, PF_ERR_INVALID, "bad DFT monitor");
  const DftMon& dm = e->dfts[mon];
  const size_t bytes = (size_t)dm.r.ncomp * dm.n_freq * dm.r.ncell * 16;
  int rc;
  if (!e->dft_cot[mon] && (rc = dalloc(e, (void**)&e->dft_cot[mon], bytes))) return rc;
  PF_CUDA(e, cudaMemcpyAsync(e->dft_cot[mon], cot, bytes, cudaMemcpyHostToDevice, e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  return PF_OK;
}

int pf_adj_set_flux_cotangent(pf_engine* e, int mon, double cot) {
  if (!e) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "pf_adj_set_flux_cotangent before pf_adj_init");
  if (mon < 0 || mon >= (int)e->fluxes.size()) return fail(e, PF_ERR_INVALID, "bad flux monitor");
  if (!std::isfinite(cot)) return fail(e, PF_ERR_INVALID, "flux cotangent must be finite");
  FluxMon& f = e->fluxes[mon];
  if (cot != 0.0 && f.rec_cap < e->ring_steps) {
    int rc;
    const size_t bytes = (size_t)e->ring_steps * 2 * f.p.n0 * f.p.n1 * e->rb;
    if ((rc = dalloc(e, &f.rec, bytes))) return rc;
    f.rec_cap = e->ring_steps;
  }
  f.cot = cot;
  return PF_OK;
}

int pf_adj_add_field_source(pf_engine* e, int64_t step, int comp, const int32_t start[3],
                            const int32_t stop[3], const int32_t stride[3], const double* vals) {
  if (!e || !vals || !start || !stop || !stride) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "pf_adj_add_field_source before pf_adj_init");
  if (!valid_comp(comp) || step < 0 || step >= e->n_steps)
    return fail(e, PF_ERR_INVALID, "bad component or step");
  pf_engine::RegionSource rs;
  rs.step = step;
  rs.comp = comp;
  if (!make_region(e, start, stop, stride, rs.r)) return fail(e, PF_ERR_INVALID, "bad region");
  int rc;
  if ((rc = dalloc(e, (void**)&rs.vals, (size_t)rs.r.ncell * 8))) return rc;
  PF_CUDA(e, cudaMemcpyAsync(rs.vals, vals, (size_t)rs.r.ncell * 8, cudaMemcpyHostToDevice,
                             e->stream));
  PF_CUDA(e, cudaStreamSynchronize(e->stream));
  e->rsrc.push_back(rs);
  return PF_OK;
}

int pf_adj_segment(pf_engine* e, int64_t step0, int64_t n, const void* state, int64_t bytes,
                   int state_on_device) {
  if (!e || !state) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "pf_adj_segment before pf_adj_init");
  if (n < 1 || n > e->ring_steps || step0 < 0 || step0 + n != e->adj_next)
    return fail(e, PF_ERR_STATE,
                "segment [%lld, %lld) must end where the reverse pass stands (%lld) and hold at "
                "most %lld steps",
                (long long)step0, (long long)(step0 + n), e->adj_next, e->ring_steps);
  int rc = e->rb == 4 ? flush_monitors<float>(e) : flush_monitors<double>(e);
  if (rc) return rc;
  if ((rc = copy_state(e, step0, const_cast<void*>(state), bytes, state_on_device, false)))
    return rc;
  e->step = step0;
  return e->rb == 4 ? adj_segment_typed<float>(e, step0, n) : adj_segment_typed<double>(e, step0, n);
}

int pf_adj_read_grad_components(pf_engine* e, double* dst) {
  if (!e || !dst) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "gradient read before pf_adj_init");
  if (e->ce_mode != PF_CE_CELL3)
    return fail(e, PF_ERR_STATE,
                "per-component gradient kept only for per-component coefficients "
                "(PF_CE_CELL3); use pf_adj_read_grad");
  PF_CUDA(e, cudaSetDevice(e->device));
  PF_CUDA(e, cudaMemcpy(dst, e->grad, (size_t)e->ncell * 24, cudaMemcpyDeviceToHost));
  return PF_OK;
}

int pf_adj_read_grad(pf_engine* e, double* dst) {
  if (!e || !dst) return PF_ERR_INVALID;
  if (!e->adj) return fail(e, PF_ERR_STATE, "gradient read before pf_adj_init");
  const size_t n = (size_t)e->ncell;
  if (e->ce_mode != PF_CE_CELL3) {  // accumulated summed over the components
    PF_CUDA(e, cudaSetDevice(e->device));
    PF_CUDA(e, cudaMemcpy(dst, e->grad, n * 8, cudaMemcpyDeviceToHost));
    return PF_OK;
  }
  std::vector<double> g(n * 3);
  int rc = pf_adj_read_grad_components(e, g.data());
  if (rc) return rc;
  for (size_t i = 0; i < n; ++i) dst[i] = (g[i] + g[n + i]) + g[2 * n + i];
  return PF_OK;
}

}  // extern "C"
