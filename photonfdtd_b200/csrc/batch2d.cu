// batch2d.cu - batched 2D TE engine with a hand-written discrete adjoint.
//
// Many uneven 2D instances (xy plane, nz = 1) are stepped together. Their
// fields live in pooled arrays (rows padded to a 32-cell pitch), and every
// kernel walks one work list of tiles drawn from all instances
// (batch2d_kernels.cuh). Only Ex, Ey, Hz are stepped: with TE-only sources
// the other three components of the reference's update
// (src/photonfdtd/simulation.py:1252-1309 with nz = 1) stay exactly zero, so
// Ex, Ey, Hz are the reference's to the bit. Chunks of steps are captured
// once as CUDA graphs and replayed; the chunk's first step lives in device
// memory.
//
// Step n: Hz (curl of E, CPML psi along x and y), H sources, Ex / Ey (curl
// of Hz, psi), E sources, the output-line DFT of Ey accumulated in
// complex128: acc += (exp(i w (n+1) dt) * Ey) * dt (samples kept in a ring
// and folded in step order every 32 steps).
//
// The adjoint is the transpose of that (affine) step, applied backward in
// time. For a real loss L of the line DFT F, the caller passes the
// cotangent G = dL/dRe F + i dL/dIm F; step n's adjoint source on the line is
// dt * sum_f Re(conj(G_f) exp(i w_f (n+1) dt)). The gradient with respect to
// the E coefficient K = dt / (eps eps0) of each design cell is
//   sum_n  aEx^{n+1} * cEx^n + aEy^{n+1} * cEy^n,
// where cE^n is the forward curl (bulk + psi) that multiplied K in step n.
// Those curls are recorded per design cell in a ring of `checkpoint_every`
// (K) steps, slot = n mod K. The forward run stores the full state at the
// start of every K-step segment; the adjoint replays each earlier segment from
// its checkpoint to refill the ring, then runs its K transposed steps. The
// last segment's ring is left by the forward run itself. Memory is
// ceil(N / K) - 1 states + K window rings; K >= N keeps no state and needs no
// replay.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pfb200.h"
#include "batch2d_kernels.cuh"
#include "common.cuh"

using namespace pfb;
using namespace pfb::b2d;

struct pf_batch {
  int n_inst = 0, rb = 4;
  double dx = 1, dy = 1, ch = 0, dt = 0;
  long long n_steps = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  std::vector<Inst> inst;
  std::vector<std::vector<char>> h_ce;
  std::vector<std::vector<char>> h_coef[8];  // bex cex bhx chx bey cey bhy chy
  long long ncell = 0, ncell_real = 0, nx_tot = 0, ny_tot = 0, n_design = 0, nline = 0;
  long long npsi[4] = {};
  int rows = 4;  // rows per thread (tile = 32 columns x 8 * rows)
  int ckpt = 64;
  bool merge_post = true;  // no E-source group sits on an output-line cell
  int n_h_groups = 0;      // source groups on Hz
  bool finalized = false, fwd_done = false, ring_last = false;
  bool fwd_only = false;  // finalized with checkpoint_every = 0: no adjoint state
  bool fd[2] = {false, false};
  double rd[2] = {1, 1};
  std::vector<long long> s_cell;
  std::vector<int> s_comp, s_start, s_row;
  std::vector<double> s_amp, h_wave, h_phase;
  int n_freq = 0;
  // device
  std::vector<void*> allocs;
  Inst* d_inst = nullptr;
  TileRec* d_tiles = nullptr;
  SegRec* d_segs = nullptr;   // marching segments (forward step)
  int nsegs = 0;
  size_t seg_cap = 0;         // SegRec slots of d_segs (the shortest segments)
  bool march = true;          // forward step: marching warps (else kb_step tiles)
  int ntiles = 0;
  int tile_rows = 32;
  size_t tile_cap = 0;  // TileRec slots of d_tiles (the 8-row list, the longest)
  void *Ex = nullptr, *Ey = nullptr, *Hz = nullptr, *ce = nullptr;
  // fused step (no H-family sources): a second level of Ex, Ey, Hz and the
  // H psi; the fields after `field_step` steps are in level_at(field_step)
  bool fused = false;
  void* lvl1[5] = {};  // Ex, Ey, Hz, psi[0], psi[1] of level 1
  long long field_step = 0;
  // fused reverse step: level 1 of aHz, its two psi adjoints, gA and gB
  void* alvl1[5] = {};
  void* coef[8] = {};
  void* psi[4] = {};
  int* maps[4] = {};  // mex mhx mey mhy
  void* aE[3] = {};
  void* apsi[4] = {};
  void* g[4] = {};
  void* design_stage = nullptr;
  double* grad = nullptr;
  void* ring = nullptr;
  void* ckpt_buf = nullptr;
  long long state_elems = 0;
  double* acc = nullptr;
  double* cot = nullptr;
  long long* lcell = nullptr;
  double* phase = nullptr;
  long long* base = nullptr;  // first step of the running chunk
  void* dring = nullptr;      // DFT line samples, kDftRing x line cells
  BSources src{};
  // instantiated graphs and their kernel counts, keyed by (chunk kind, steps)
  std::map<std::pair<int, long long>, std::pair<cudaGraphExec_t, long long>> graphs;
  int64_t launches = 0;
  long long capture_launches = 0;
};

namespace {

int bfail(pf_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return code;
}

#define B_CUDA(b, call)                                                                    \
  do {                                                                                     \
    cudaError_t rc_ = (call);                                                              \
    if (rc_ != cudaSuccess)                                                                \
      return bfail((b), rc_ == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA,       \
                   "CUDA error: %s (%s)", cudaGetErrorString(rc_), #call);                 \
  } while (0)

int balloc(pf_batch* b, void** p, size_t bytes) {
  if (!bytes) bytes = 16;
  cudaError_t rc = cudaMalloc(p, bytes);
  if (rc != cudaSuccess) {
    *p = nullptr;
    return bfail(b, PF_ERR_OOM, "cudaMalloc of %zu bytes failed", bytes);
  }
  b->allocs.push_back(*p);
  rc = cudaMemsetAsync(*p, 0, bytes, b->stream);
  return rc == cudaSuccess ? PF_OK : bfail(b, PF_ERR_CUDA, "%s", cudaGetErrorString(rc));
}

int bup(pf_batch* b, void** p, const void* src, size_t bytes) {
  int rc = balloc(b, p, bytes);
  if (rc) return rc;
  if (bytes) B_CUDA(b, cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, b->stream));
  return PF_OK;
}

template <typename T>
BArgs<T> bargs(pf_batch* b) {
  BArgs<T> a;
  memset(&a, 0, sizeof a);
  a.inst = b->d_inst;
  a.tiles = b->d_tiles;
  a.segs = b->d_segs;
  a.nsegs = b->nsegs;
  a.ntiles = b->ntiles;
  a.Ex = (T*)b->Ex;
  a.Ey = (T*)b->Ey;
  a.Hz = (T*)b->Hz;
  a.ce = (const T*)b->ce;
  const T** cp[8] = {&a.bex, &a.cex, &a.bhx, &a.chx, &a.bey, &a.cey, &a.bhy, &a.chy};
  for (int q = 0; q < 8; ++q) *cp[q] = (const T*)b->coef[q];
  a.mex = b->maps[0];
  a.mhx = b->maps[1];
  a.mey = b->maps[2];
  a.mhy = b->maps[3];
  a.pHzx = (T*)b->psi[0];
  a.pHzy = (T*)b->psi[1];
  a.pExy = (T*)b->psi[2];
  a.pEyx = (T*)b->psi[3];
  a.dx = (T)b->dx;
  a.dy = (T)b->dy;
  a.rdx = (T)b->rd[0];
  a.rdy = (T)b->rd[1];
  a.fdx = b->fd[0];
  a.fdy = b->fd[1];
  a.ch = (T)b->ch;
  a.idx = (T)(1.0 / b->dx);
  a.idy = (T)(1.0 / b->dy);
  a.base = b->base;
  a.ring = (T*)b->ring;
  a.n_design = b->n_design;
  a.ring_len = b->fwd_only ? 1 : b->ckpt;
  T** lv[5] = {a.Ex2, a.Ey2, a.Hz2, a.pHzx2, a.pHzy2};
  void* l0[5] = {b->Ex, b->Ey, b->Hz, b->psi[0], b->psi[1]};
  for (int q = 0; q < 5; ++q) {
    lv[q][0] = (T*)l0[q];
    lv[q][1] = (T*)(b->fused ? b->lvl1[q] : l0[q]);
  }
  return a;
}

template <typename T>
BFields<T> bfields(const BArgs<T>& a, bool flip) {
  BFields<T> f;
  for (int l = 0; l < 2; ++l) {
    f.Ex[l] = a.Ex2[l];
    f.Ey[l] = a.Ey2[l];
    f.Hz[l] = a.Hz2[l];
  }
  f.flip = flip ? 1 : 0;
  return f;
}

// Level holding the fields after `step` steps (always 0 on the split path).
int level_at(const pf_batch* b, long long step) { return b->fused ? (int)(step & 1) : 0; }

template <typename T>
AArgs<T> aargs(pf_batch* b) {
  AArgs<T> d;
  d.aEx = (T*)b->aE[0];
  d.aEy = (T*)b->aE[1];
  d.aHz = (T*)b->aE[2];
  d.aHzx = (T*)b->apsi[0];
  d.aHzy = (T*)b->apsi[1];
  d.aExy = (T*)b->apsi[2];
  d.aEyx = (T*)b->apsi[3];
  d.gA = (T*)b->g[0];
  d.gB = (T*)b->g[1];
  d.hA = (T*)b->g[2];
  d.hB = (T*)b->g[3];
  d.grad = b->grad;
  d.cot = b->cot;
  d.phase = b->phase;
  d.n_freq = b->n_freq;
  d.dt = b->dt;
  T** lv[5] = {d.aHz2, d.aHzx2, d.aHzy2, d.gA2, d.gB2};
  void* l0[5] = {b->aE[2], b->apsi[0], b->apsi[1], b->g[0], b->g[1]};
  for (int q = 0; q < 5; ++q) {
    lv[q][0] = (T*)l0[q];
    lv[q][1] = (T*)(b->fused ? b->alvl1[q] : l0[q]);
  }
  return d;
}

// One tile per block (the kernels also accept a smaller grid).
int grid_blocks(const pf_batch* b) { return std::max(1, b->ntiles); }

template <typename T, int R>
void fwd_kernels(pf_batch* b, long long len, bool dft) {
  const BArgs<T> a = bargs<T>(b);
  const BFields<T> f = bfields<T>(a, b->fused);
  const dim3 blk(32, kWarps);
  const int G = grid_blocks(b);
  const long long ng = b->src.n_groups;
  int pend = 0;
  for (long long t = 0; t < len; ++t) {
    if (b->fused && b->march) {
      kb_march<T><<<(unsigned)((b->nsegs + kMarchWarps - 1) / kMarchWarps), dim3(32, kMarchWarps),
                    0, b->stream>>>(a, (int)t);
      b->capture_launches += 1;
    } else if (b->fused) {
      kb_step<T, R><<<G, blk, 0, b->stream>>>(a, (int)t);
      b->capture_launches += 1;
    } else {
      if (b->n_h_groups) {
        kb_post<T><<<(unsigned)((ng + 127) / 128), 128, 0, b->stream>>>(
            b->src, f, 1, b->base, (int)t, b->lcell, 0, (T*)nullptr);
        ++b->capture_launches;
      }
      kb_h<T, R><<<G, blk, 0, b->stream>>>(a);
      kb_e<T, R><<<G, blk, 0, b->stream>>>(a, (int)t);
      b->capture_launches += 2;
    }
    T* dring = dft ? (T*)b->dring : nullptr;
    if (b->merge_post || !dft) {
      const long long n = ng + (dft ? b->nline : 0);
      if (n) {
        kb_post<T><<<(unsigned)((n + 127) / 128), 128, 0, b->stream>>>(
            b->src, f, 0, b->base, (int)t, b->lcell, b->nline, dring);
        ++b->capture_launches;
      }
    } else {
      if (ng) {
        kb_post<T><<<(unsigned)((ng + 127) / 128), 128, 0, b->stream>>>(
            b->src, f, 0, b->base, (int)t, b->lcell, 0, (T*)nullptr);
        ++b->capture_launches;
      }
      BSources none = b->src;
      none.n_groups = 0;
      kb_post<T><<<(unsigned)((b->nline + 127) / 128), 128, 0, b->stream>>>(
          none, f, 0, b->base, (int)t, b->lcell, b->nline, dring);
      ++b->capture_launches;
    }
    if (dft) {
      ++pend;
      if (pend == kDftRing || t + 1 == len) {
        const long long n = b->nline * b->n_freq;
        kb_dft_flush<T><<<(unsigned)((n + 255) / 256), 256, 0, b->stream>>>(
            (const T*)b->dring, b->nline, b->acc, b->phase, b->n_freq, b->dt, b->base,
            (int)(t + 1 - pend), pend);
        ++b->capture_launches;
        pend = 0;
      }
    }
  }
}

// Reverse pass over chunk steps len-1 .. 0 (n = *base + t): the E transpose
// of the top step, then per step the H transpose and a cell pass that
// finishes that step's E adjoints and, except after the lowest step (whose
// predecessor belongs to the previous segment), runs the next lower step's E
// transpose.
template <typename T, int R>
void adj_kernels(pf_batch* b, long long len) {
  const BArgs<T> a = bargs<T>(b);
  const AArgs<T> d = aargs<T>(b);
  const dim3 blk(32, kWarps);
  const int G = grid_blocks(b);
  if (b->fused && b->march) {
    const dim3 mg((unsigned)((b->nsegs + kMarchWarps - 1) / kMarchWarps)), mb(32, kMarchWarps);
    kb_adj_march<T, false, true><<<mg, mb, 0, b->stream>>>(a, d, (int)(len - 1));
    for (long long t = len - 1; t >= 0; --t) {
      if (t > 0)
        kb_adj_march<T, true, true><<<mg, mb, 0, b->stream>>>(a, d, (int)t);
      else
        kb_adj_march<T, true, false><<<mg, mb, 0, b->stream>>>(a, d, 0);
    }
    b->capture_launches += 1 + len;
    return;
  }
  if (b->fused) {
    kb_adj_step<T, R, false, true><<<G, blk, 0, b->stream>>>(a, d, (int)(len - 1));
    for (long long t = len - 1; t >= 0; --t) {
      if (t > 0)
        kb_adj_step<T, R, true, true><<<G, blk, 0, b->stream>>>(a, d, (int)t);
      else
        kb_adj_step<T, R, true, false><<<G, blk, 0, b->stream>>>(a, d, 0);
    }
    b->capture_launches += 1 + len;
    return;
  }
  kb_adj_cell<T, R, false, true><<<G, blk, 0, b->stream>>>(a, d, (int)(len - 1));
  for (long long t = len - 1; t >= 0; --t) {
    kb_adj_h<T, R><<<G, blk, 0, b->stream>>>(a, d);
    if (t > 0)
      kb_adj_cell<T, R, true, true><<<G, blk, 0, b->stream>>>(a, d, (int)(t - 1));
    else
      kb_adj_cell<T, R, true, false><<<G, blk, 0, b->stream>>>(a, d, 0);
  }
  b->capture_launches += 1 + 2 * len;
}

template <typename T>
void chunk_kernels(pf_batch* b, int kind, long long len) {
  if (kind == 2) {
    if (b->rows == 1) adj_kernels<T, 1>(b, len);
    else if (b->rows == 2) adj_kernels<T, 2>(b, len);
    else adj_kernels<T, 4>(b, len);
  } else {
    if (b->rows == 1) fwd_kernels<T, 1>(b, len, kind == 0);
    else if (b->rows == 2) fwd_kernels<T, 2>(b, len, kind == 0);
    else fwd_kernels<T, 4>(b, len, kind == 0);
  }
}

// Runs `len` steps of kind 0 (forward + DFT + ring), 1 (replay: forward +
// ring) or 2 (adjoint) as one graph launch, chunk step t = 0 at *base. Each
// (kind, len) is captured once; at most two lengths occur per kind (K and
// the last segment's).
template <typename T>
int run_chunk(pf_batch* b, int kind, long long len) {
  if (len > (1LL << 30)) return bfail(b, PF_ERR_INVALID, "chunk too long");
  auto& ent = b->graphs[std::make_pair(kind, len)];
  if (ent.first == nullptr) {
    cudaGraph_t graph = nullptr;
    B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    b->capture_launches = 0;
    chunk_kernels<T>(b, kind, len);
    const cudaError_t e1 = cudaStreamEndCapture(b->stream, &graph);
    if (e1 != cudaSuccess) return bfail(b, PF_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e1));
    const cudaError_t e2 = cudaGraphInstantiate(&ent.first, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
      ent.first = nullptr;
      return bfail(b, PF_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e2));
    }
    ent.second = b->capture_launches;
  }
  B_CUDA(b, cudaGraphLaunch(ent.first, b->stream));
  b->launches += ent.second;
  return PF_OK;
}

// Copies the stepping state (Ex, Ey, Hz, four psi arrays) to / from slot s;
// `step` is the step count the state belongs to (it selects the level).
int state_copy(pf_batch* b, long long s, bool save, long long step) {
  const size_t S = b->rb;
  char* base = (char*)b->ckpt_buf + (size_t)s * b->state_elems * S;
  const bool l1 = level_at(b, step) == 1;
  void* parts[7] = {l1 ? b->lvl1[0] : b->Ex, l1 ? b->lvl1[1] : b->Ey, l1 ? b->lvl1[2] : b->Hz,
                    l1 ? b->lvl1[3] : b->psi[0], l1 ? b->lvl1[4] : b->psi[1], b->psi[2],
                    b->psi[3]};
  const long long n[7] = {b->ncell, b->ncell, b->ncell, b->npsi[0], b->npsi[1], b->npsi[2], b->npsi[3]};
  size_t o = 0;
  for (int q = 0; q < 7; ++q) {
    const size_t bytes = (size_t)n[q] * S;
    if (bytes) {
      void* dst = save ? (void*)(base + o) : parts[q];
      const void* from = save ? parts[q] : (const void*)(base + o);
      B_CUDA(b, cudaMemcpyAsync(dst, from, bytes, cudaMemcpyDeviceToDevice, b->stream));
    }
    o += bytes;
  }
  return PF_OK;
}

int set_base(pf_batch* b, long long s) {
  kb_set<<<1, 1, 0, b->stream>>>(b->base, s);
  b->launches += 1;
  B_CUDA(b, cudaGetLastError());
  return PF_OK;
}

int zero_state(pf_batch* b) {
  const size_t S = b->rb;
  for (void* p : {b->Ex, b->Ey, b->Hz}) B_CUDA(b, cudaMemsetAsync(p, 0, b->ncell * S, b->stream));
  for (int q = 0; q < 4; ++q)
    if (b->npsi[q]) B_CUDA(b, cudaMemsetAsync(b->psi[q], 0, b->npsi[q] * S, b->stream));
  if (b->fused) {
    for (int q = 0; q < 3; ++q) B_CUDA(b, cudaMemsetAsync(b->lvl1[q], 0, b->ncell * S, b->stream));
    for (int q = 0; q < 2; ++q)
      if (b->npsi[q]) B_CUDA(b, cudaMemsetAsync(b->lvl1[3 + q], 0, b->npsi[q] * S, b->stream));
  }
  b->field_step = 0;
  return PF_OK;
}

template <typename T>
int forward_t(pf_batch* b) {
  int rc;
  if ((rc = zero_state(b))) return rc;
  B_CUDA(b, cudaMemsetAsync(b->acc, 0, (size_t)b->nline * b->n_freq * 16, b->stream));
  const long long K = b->ckpt;
  for (long long s0 = 0; s0 < b->n_steps; s0 += K) {
    if (s0 > 0 && !b->fwd_only && (rc = state_copy(b, s0 / K - 1, true, s0)))
      return rc;  // segment 0 starts at zero
    if ((rc = set_base(b, s0))) return rc;
    if ((rc = run_chunk<T>(b, 0, std::min(K, b->n_steps - s0)))) return rc;
  }
  B_CUDA(b, cudaGetLastError());
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  b->field_step = b->n_steps;
  b->fwd_done = true;
  b->ring_last = true;
  return PF_OK;
}

template <typename T>
int adjoint_t(pf_batch* b) {
  const size_t S = b->rb;
  int rc;
  for (int q = 0; q < 3; ++q) B_CUDA(b, cudaMemsetAsync(b->aE[q], 0, b->ncell * S, b->stream));
  for (int q = 0; q < 4; ++q) {
    if (b->npsi[q]) B_CUDA(b, cudaMemsetAsync(b->apsi[q], 0, b->npsi[q] * S, b->stream));
    if (q < 2 || !b->fused) B_CUDA(b, cudaMemsetAsync(b->g[q], 0, b->ncell * S, b->stream));
  }
  if (b->fused) {
    const long long n1[5] = {b->ncell, b->npsi[0], b->npsi[1], b->ncell, b->ncell};
    for (int q = 0; q < 5; ++q)
      if (n1[q]) B_CUDA(b, cudaMemsetAsync(b->alvl1[q], 0, n1[q] * S, b->stream));
  }
  B_CUDA(b, cudaMemsetAsync(b->grad, 0, (size_t)b->n_design * 8, b->stream));
  const long long K = b->ckpt;
  const long long nseg = (b->n_steps + K - 1) / K;
  for (long long sg = nseg - 1; sg >= 0; --sg) {
    const long long s0 = sg * K, len = std::min(K, b->n_steps - s0);
    if (sg < nseg - 1 || !b->ring_last) {  // refill the ring from the segment's checkpoint
      if (sg == 0) {
        if ((rc = zero_state(b))) return rc;
      } else if ((rc = state_copy(b, sg - 1, false, s0))) {
        return rc;
      }
      if ((rc = set_base(b, s0))) return rc;
      if ((rc = run_chunk<T>(b, 1, len))) return rc;
      b->field_step = s0 + len;
    }
    if ((rc = set_base(b, s0))) return rc;
    if ((rc = run_chunk<T>(b, 2, len))) return rc;
  }
  B_CUDA(b, cudaGetLastError());
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  // the replays left the fields and the ring of segment 0 behind; the DFT
  // accumulators still hold the forward result
  b->ring_last = nseg == 1;
  return PF_OK;
}

void destroy_graphs(pf_batch* b) {
  for (auto& kv : b->graphs)
    if (kv.second.first) cudaGraphExecDestroy(kv.second.first);
  b->graphs.clear();
}

}  // namespace

extern "C" {

const char* pfb_last_error(const pf_batch* b) { return b ? b->err.c_str() : "null batch handle"; }

int pfb_create(int n_inst, int real_bytes, double dx, double dy, double ch, double dt,
               int64_t n_steps, pf_batch** out) {
  if (!out) return PF_ERR_INVALID;
  *out = nullptr;
  if (n_inst < 1 || (real_bytes != 4 && real_bytes != 8) || n_steps < 1 || !(dx > 0) || !(dy > 0))
    return PF_ERR_INVALID;
  pf_batch* b = new pf_batch();
  b->n_inst = n_inst;
  b->rb = real_bytes;
  b->dx = dx;
  b->dy = dy;
  b->ch = ch;
  b->dt = dt;
  b->n_steps = n_steps;
  b->inst.resize(n_inst);
  for (Inst& I : b->inst) memset(&I, 0, sizeof I);
  b->h_ce.resize(n_inst);
  for (int q = 0; q < 8; ++q) b->h_coef[q].resize(n_inst);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return PF_ERR_CUDA;
  }
  *out = b;
  return PF_OK;
}

int pfb_set_instance(pf_batch* b, int k, int nx, int ny, const void* ce, const void* const coef[8],
                     int di0, int dj0, int dn, int line_i) {
  if (!b) return PF_ERR_INVALID;
  if (b->finalized) return bfail(b, PF_ERR_STATE, "pfb_set_instance after pfb_finalize");
  if (k < 0 || k >= b->n_inst || nx < 2 || ny < 2 || !ce || !coef)
    return bfail(b, PF_ERR_INVALID, "instance %d: bad arguments", k);
  for (int q = 0; q < 8; ++q)
    if (!coef[q]) return bfail(b, PF_ERR_INVALID, "instance %d: CPML array %d is NULL", k, q);
  if ((long long)nx * ny >= (1LL << 31))
    return bfail(b, PF_ERR_INVALID, "instance %d: 2^31 cells or more", k);
  if (dn < 1 || di0 < 0 || dj0 < 0 || di0 + dn > nx || dj0 + dn > ny)
    return bfail(b, PF_ERR_INVALID, "instance %d: design window outside the grid", k);
  if (line_i < 0 || line_i >= nx)
    return bfail(b, PF_ERR_INVALID, "instance %d: output line outside the grid", k);
  Inst& I = b->inst[k];
  I.nx = nx;
  I.ny = ny;
  I.di0 = di0;
  I.dj0 = dj0;
  I.dn = dn;
  I.line_i = line_i;
  const size_t S = b->rb;
  b->h_ce[k].assign((const char*)ce, (const char*)ce + (size_t)nx * ny * S);
  for (int q = 0; q < 8; ++q) {
    const size_t n = (size_t)(q < 4 ? nx : ny) * S;
    b->h_coef[q][k].assign((const char*)coef[q], (const char*)coef[q] + n);
  }
  return PF_OK;
}

int pfb_set_sources(pf_batch* b, int n_src, const int32_t* inst, const int32_t* comp,
                    const int32_t* i, const int32_t* j, const int32_t* wave_row, const double* amp,
                    int n_wave, const double* wave) {
  if (!b) return PF_ERR_INVALID;
  if (b->finalized) return bfail(b, PF_ERR_STATE, "pfb_set_sources after pfb_finalize");
  if (n_src < 0 || n_wave < 0 ||
      (n_src > 0 && (!inst || !comp || !i || !j || !wave_row || !amp || !wave)))
    return bfail(b, PF_ERR_INVALID, "bad source arrays");
  std::vector<std::pair<std::pair<int, long long>, int>> key;  // ((comp, inst<<32 | cell), src)
  for (int q = 0; q < n_src; ++q) {
    if (inst[q] < 0 || inst[q] >= b->n_inst || comp[q] < 0 || comp[q] > 2)
      return bfail(b, PF_ERR_INVALID, "source %d: bad instance or component", q);
    const Inst& I = b->inst[inst[q]];
    if (I.nx == 0) return bfail(b, PF_ERR_STATE, "source %d: instance %d not set", q, inst[q]);
    if (i[q] < 0 || i[q] >= I.nx || j[q] < 0 || j[q] >= I.ny || wave_row[q] < 0 ||
        wave_row[q] >= n_wave)
      return bfail(b, PF_ERR_INVALID, "source %d out of range", q);
    key.push_back({{comp[q], ((long long)inst[q] << 32) | ((long long)i[q] * I.ny + j[q])}, q});
  }
  std::stable_sort(key.begin(), key.end(),
                   [](const auto& x, const auto& y) { return x.first < y.first; });
  b->s_cell.clear();
  b->s_comp.clear();
  b->s_start.clear();
  b->s_row.clear();
  b->s_amp.clear();
  for (size_t q = 0; q < key.size(); ++q) {
    if (q == 0 || key[q].first != key[q - 1].first) {
      b->s_cell.push_back(key[q].first.second);  // resolved to a pooled cell at finalize
      b->s_comp.push_back(key[q].first.first);
      b->s_start.push_back((int)b->s_row.size());
    }
    b->s_row.push_back(wave_row[key[q].second]);
    b->s_amp.push_back(amp[key[q].second]);
  }
  b->s_start.push_back((int)b->s_row.size());
  b->h_wave.assign(wave, wave + (size_t)n_wave * b->n_steps);
  return PF_OK;
}

int pfb_set_dft(pf_batch* b, int n_freq, const double* phase) {
  if (!b) return PF_ERR_INVALID;
  if (b->finalized) return bfail(b, PF_ERR_STATE, "pfb_set_dft after pfb_finalize");
  if (n_freq < 1 || !phase) return bfail(b, PF_ERR_INVALID, "bad DFT arguments");
  b->n_freq = n_freq;
  b->h_phase.assign(phase, phase + (size_t)b->n_steps * n_freq * 2);
  return PF_OK;
}

}  // extern "C"

namespace {

// The work list at a tile height of tile_rows rows (x) by 32 cells (y),
// every instance's tiles in order.
std::vector<TileRec> make_tiles(const pf_batch* b, int tile_rows) {
  std::vector<TileRec> tiles;
  for (int k = 0; k < b->n_inst; ++k) {
    const Inst& I = b->inst[k];
    for (int i0 = 0; i0 < I.nx; i0 += tile_rows)
      for (int j0 = 0; j0 < I.ny; j0 += 32) {
        TileRec tr;
        tr.base = I.off + (long long)i0 * I.pitch + j0;
        tr.nx = I.nx;
        tr.ny = I.ny;
        tr.pitch = I.pitch;
        tr.i0 = i0;
        tr.j0 = j0;
        tr.ox = I.ox + i0;
        tr.oy = I.oy + j0;
        tr.k = k;
        tr.wdi = I.di0 - i0;
        tr.wdj = I.dj0 - j0;
        tr.wdn = I.dn;
        tr.pad[0] = 0;
        tiles.push_back(tr);
      }
  }
  return tiles;
}

// The marching segments at a height of seg_rows rows: every instance's
// strips of 31 owned columns, each cut into row ranges.
std::vector<SegRec> make_segs(const pf_batch* b, int seg_rows) {
  std::vector<SegRec> segs;
  for (int k = 0; k < b->n_inst; ++k) {
    const Inst& I = b->inst[k];
    for (int j0 = 0; j0 < I.ny; j0 += kMarchCols)
      for (int i0 = 0; i0 < I.nx; i0 += seg_rows) {
        SegRec sg;
        sg.k = k;
        sg.i0 = i0;
        sg.i1 = std::min(I.nx, i0 + seg_rows);
        sg.j0 = j0;
        segs.push_back(sg);
      }
  }
  return segs;
}

int set_tile_rows(pf_batch* b, int tile_rows) {
  const std::vector<TileRec> tiles = make_tiles(b, tile_rows);
  if (tiles.size() > b->tile_cap) return bfail(b, PF_ERR_INVALID, "tile list exceeds its buffer");
  B_CUDA(b, cudaMemcpyAsync(b->d_tiles, tiles.data(), tiles.size() * sizeof(TileRec),
                            cudaMemcpyHostToDevice, b->stream));
  // the marching steps' segments are 2 x tile_rows rows high
  const std::vector<SegRec> segs = make_segs(b, 2 * tile_rows);
  if (segs.size() > b->seg_cap) return bfail(b, PF_ERR_INVALID, "segment list exceeds its buffer");
  B_CUDA(b, cudaMemcpyAsync(b->d_segs, segs.data(), segs.size() * sizeof(SegRec),
                            cudaMemcpyHostToDevice, b->stream));
  b->nsegs = (int)segs.size();
  B_CUDA(b, cudaStreamSynchronize(b->stream));  // before `tiles` and `segs` go
  destroy_graphs(b);  // captured with the old grid and row count
  b->ntiles = (int)tiles.size();
  b->rows = tile_rows / kWarps;
  b->tile_rows = tile_rows;
  return PF_OK;
}

template <typename T>
int tune_tiles_t(pf_batch* b, int trial, float* ms3, int* best) {
  static const int cand[3] = {8, 16, 32};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int rc = PF_OK;
  if (cudaEventCreate(&ev[0]) != cudaSuccess || cudaEventCreate(&ev[1]) != cudaSuccess)
    rc = bfail(b, PF_ERR_CUDA, "cudaEventCreate failed");
  int bi = 2;
  for (int c = 0; c < 3 && !rc; ++c) {
    if ((rc = set_tile_rows(b, cand[c]))) break;
    for (int rep = 0; rep < 2 && !rc; ++rep) {  // rep 0 captures the chunk's graph
      if ((rc = zero_state(b)) || (rc = set_base(b, 0))) break;
      if (rep && cudaEventRecord(ev[0], b->stream) != cudaSuccess) {
        rc = bfail(b, PF_ERR_CUDA, "cudaEventRecord failed");
        break;
      }
      if ((rc = run_chunk<T>(b, 0, trial))) break;
      if (rep && cudaEventRecord(ev[1], b->stream) != cudaSuccess) {
        rc = bfail(b, PF_ERR_CUDA, "cudaEventRecord failed");
        break;
      }
    }
    if (rc) break;
    float ms = 0.f;
    if (cudaEventSynchronize(ev[1]) != cudaSuccess ||
        cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) {
      rc = bfail(b, PF_ERR_CUDA, "tile timing failed");
      break;
    }
    ms3[c] = ms / trial;
    if (ms3[c] < ms3[bi] || c == 0) bi = c;
  }
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  if (rc) return rc;
  if ((rc = set_tile_rows(b, cand[bi]))) return rc;
  // the trial runs left fields, ring and DFT lines behind: start clean
  if ((rc = zero_state(b))) return rc;
  B_CUDA(b, cudaMemsetAsync(b->acc, 0, (size_t)b->nline * b->n_freq * 16, b->stream));
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  b->fwd_done = false;
  b->ring_last = false;
  *best = cand[bi];
  return PF_OK;
}

}  // namespace

extern "C" {

int pfb_set_tile_rows(pf_batch* b, int tile_rows) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized) return bfail(b, PF_ERR_STATE, "pfb_set_tile_rows before pfb_finalize");
  if (tile_rows != 8 && tile_rows != 16 && tile_rows != 32)
    return bfail(b, PF_ERR_INVALID, "tile_rows must be 8, 16 or 32");
  return set_tile_rows(b, tile_rows);
}

int pfb_tune_tiles(pf_batch* b, int trial_steps, float* ms_per_step, int* best_rows) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized) return bfail(b, PF_ERR_STATE, "pfb_tune_tiles before pfb_finalize");
  if (trial_steps < 1 || !ms_per_step || !best_rows)
    return bfail(b, PF_ERR_INVALID, "pfb_tune_tiles: bad arguments");
  const int trial = (int)std::min<long long>(trial_steps, std::min<long long>(b->ckpt, b->n_steps));
  return b->rb == 4 ? tune_tiles_t<float>(b, trial, ms_per_step, best_rows)
                    : tune_tiles_t<double>(b, trial, ms_per_step, best_rows);
}

int pfb_finalize(pf_batch* b, int checkpoint_every, int tile_rows) {
  if (!b) return PF_ERR_INVALID;
  if (b->finalized) return bfail(b, PF_ERR_STATE, "pfb_finalize called twice");
  if (checkpoint_every < 0) return bfail(b, PF_ERR_INVALID, "checkpoint_every must be >= 0");
  if (tile_rows != 8 && tile_rows != 16 && tile_rows != 32)
    return bfail(b, PF_ERR_INVALID, "tile_rows must be 8, 16 or 32");
  if (b->n_freq < 1) return bfail(b, PF_ERR_STATE, "pfb_set_dft must come before pfb_finalize");
  for (int k = 0; k < b->n_inst; ++k)
    if (b->inst[k].nx == 0) return bfail(b, PF_ERR_STATE, "instance %d not set", k);
  b->fwd_only = checkpoint_every == 0;
  // forward-only batches run in graph chunks of at most 512 steps
  b->ckpt = (int)std::min<long long>(b->fwd_only ? 512 : checkpoint_every, b->n_steps);
  b->rows = tile_rows / kWarps;
  const size_t S = b->rb;
  std::vector<int> mp[4];
  std::vector<char> coefp[8], cep;
  std::vector<long long> lcell;
  std::vector<TileRec> tiles;
  for (int k = 0; k < b->n_inst; ++k) {
    Inst& I = b->inst[k];
    I.pitch = (I.ny + 31) / 32 * 32;
    I.off = b->ncell;  // a multiple of 32: every instance holds nx * pitch cells
    I.ox = (int)b->nx_tot;
    I.oy = (int)b->ny_tot;
    I.goff = b->n_design;
    I.loff = b->nline;
    // compact psi maps: a cell has psi along an axis where that axis' c != 0
    auto build = [&](const std::vector<char>& c, int n, std::vector<int>& pool) {
      int cnt = 0;
      for (int t = 0; t < n; ++t) {
        const double v = S == 4 ? (double)((const float*)c.data())[t] : ((const double*)c.data())[t];
        pool.push_back(v != 0.0 ? cnt++ : -1);
      }
      return cnt;
    };
    I.npex = build(b->h_coef[1][k], I.nx, mp[0]);
    I.nphx = build(b->h_coef[3][k], I.nx, mp[1]);
    I.npey = build(b->h_coef[5][k], I.ny, mp[2]);
    I.nphy = build(b->h_coef[7][k], I.ny, mp[3]);
    I.p_hzx = b->npsi[0];
    I.p_hzy = b->npsi[1];
    I.p_exy = b->npsi[2];
    I.p_eyx = b->npsi[3];
    b->npsi[0] += (long long)I.nphx * I.ny;
    b->npsi[1] += (long long)I.nx * I.nphy;
    b->npsi[2] += (long long)I.nx * I.npey;
    b->npsi[3] += (long long)I.npex * I.ny;
    {
      const size_t row = (size_t)I.ny * S, prow = (size_t)I.pitch * S, o = cep.size();
      cep.resize(o + (size_t)I.nx * prow, 0);
      for (int i = 0; i < I.nx; ++i)
        memcpy(cep.data() + o + i * prow, b->h_ce[k].data() + i * row, row);
    }
    for (int q = 0; q < 8; ++q)
      coefp[q].insert(coefp[q].end(), b->h_coef[q][k].begin(), b->h_coef[q][k].end());
    for (int j = 0; j < I.ny; ++j) lcell.push_back(I.off + (long long)I.line_i * I.pitch + j);
    b->ncell += (long long)I.nx * I.pitch;
    b->ncell_real += (long long)I.nx * I.ny;
    b->nx_tot += I.nx;
    b->ny_tot += I.ny;
    b->n_design += (long long)I.dn * I.dn;
    b->nline += I.ny;
    std::vector<char>().swap(b->h_ce[k]);
  }
  tiles = make_tiles(b, tile_rows);
  b->tile_cap = make_tiles(b, 8).size();
  if ((long long)b->tile_cap >= (1LL << 31)) return bfail(b, PF_ERR_INVALID, "too many tiles");
  b->ntiles = (int)tiles.size();
  b->tile_rows = tile_rows;
  int rc;
  if ((rc = bup(b, (void**)&b->d_inst, b->inst.data(), b->inst.size() * sizeof(Inst)))) return rc;
  if ((rc = balloc(b, (void**)&b->d_tiles, b->tile_cap * sizeof(TileRec)))) return rc;
  B_CUDA(b, cudaMemcpyAsync(b->d_tiles, tiles.data(), tiles.size() * sizeof(TileRec),
                            cudaMemcpyHostToDevice, b->stream));
  {
    const std::vector<SegRec> segs = make_segs(b, 2 * tile_rows);
    b->seg_cap = make_segs(b, 16).size();
    if ((long long)b->seg_cap >= (1LL << 31)) return bfail(b, PF_ERR_INVALID, "too many segments");
    b->nsegs = (int)segs.size();
    if ((rc = balloc(b, (void**)&b->d_segs, b->seg_cap * sizeof(SegRec)))) return rc;
    B_CUDA(b, cudaMemcpyAsync(b->d_segs, segs.data(), segs.size() * sizeof(SegRec),
                              cudaMemcpyHostToDevice, b->stream));
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    b->march = !getenv("PFB200_BATCH_TILESTEP");
  }
  if ((rc = bup(b, &b->ce, cep.data(), cep.size()))) return rc;
  for (int q = 0; q < 8; ++q)
    if ((rc = bup(b, &b->coef[q], coefp[q].data(), coefp[q].size()))) return rc;
  for (int q = 0; q < 4; ++q)
    if ((rc = bup(b, (void**)&b->maps[q], mp[q].data(), mp[q].size() * 4))) return rc;
  for (void** p : {&b->Ex, &b->Ey, &b->Hz})
    if ((rc = balloc(b, p, b->ncell * S))) return rc;
  for (int q = 0; q < 4; ++q)
    if ((rc = balloc(b, &b->psi[q], b->npsi[q] * S))) return rc;
  // the fused steps need no H-family source (an Hz source would have to
  // reach the halo recomputation); PFB200_BATCH_SPLIT=1 keeps the split
  // passes
  bool any_h = false;
  for (size_t q = 0; q < b->s_comp.size(); ++q) any_h = any_h || b->s_comp[q] == 2;
  b->fused = !any_h && !getenv("PFB200_BATCH_SPLIT");
  if (b->fused) {
    for (int q = 0; q < 3; ++q)
      if ((rc = balloc(b, &b->lvl1[q], b->ncell * S))) return rc;
    for (int q = 0; q < 2; ++q)
      if ((rc = balloc(b, &b->lvl1[3 + q], b->npsi[q] * S))) return rc;
  }
  if (!b->fwd_only) {
    for (int q = 0; q < 3; ++q)
      if ((rc = balloc(b, &b->aE[q], b->ncell * S))) return rc;
    for (int q = 0; q < 4; ++q) {
      if ((rc = balloc(b, &b->apsi[q], b->npsi[q] * S))) return rc;
      // hA / hB (g[2], g[3]) live in shared memory on the fused path
      const bool need = q < 2 || !b->fused;
      if ((rc = balloc(b, &b->g[q], need ? b->ncell * S : 16))) return rc;
    }
    if (b->fused) {
      const long long n1[5] = {b->ncell, b->npsi[0], b->npsi[1], b->ncell, b->ncell};
      for (int q = 0; q < 5; ++q)
        if ((rc = balloc(b, &b->alvl1[q], n1[q] * S))) return rc;
    }
    if ((rc = balloc(b, (void**)&b->grad, b->n_design * 8))) return rc;
    if ((rc = balloc(b, (void**)&b->cot, (size_t)b->nline * b->n_freq * 16))) return rc;
  }
  if ((rc = balloc(b, &b->design_stage, b->n_design * S))) return rc;
  const long long ring_slots = b->fwd_only ? 1 : b->ckpt;
  if ((rc = balloc(b, &b->ring, (size_t)ring_slots * b->n_design * 2 * S))) return rc;
  b->state_elems = 3 * b->ncell + b->npsi[0] + b->npsi[1] + b->npsi[2] + b->npsi[3];
  const long long nseg = (b->n_steps + b->ckpt - 1) / b->ckpt;
  // checkpoints of segments 1 .. nseg-1 (segment 0 starts from the zero state)
  if (!b->fwd_only &&
      (rc = balloc(b, &b->ckpt_buf, (size_t)(nseg - 1) * b->state_elems * S)))
    return rc;
  if ((rc = balloc(b, (void**)&b->acc, (size_t)b->nline * b->n_freq * 16))) return rc;
  if ((rc = bup(b, (void**)&b->lcell, lcell.data(), lcell.size() * 8))) return rc;
  if ((rc = bup(b, (void**)&b->phase, b->h_phase.data(), b->h_phase.size() * 8))) return rc;
  if ((rc = balloc(b, (void**)&b->base, 8))) return rc;
  if ((rc = balloc(b, &b->dring, (size_t)kDftRing * b->nline * S))) return rc;
  // one launch may inject E sources and sample the lines only if no E group
  // sits on a line cell
  b->merge_post = true;
  b->n_h_groups = 0;
  for (size_t q = 0; q < b->s_cell.size(); ++q) {
    const Inst& I = b->inst[(int)(b->s_cell[q] >> 32)];
    const long long local = b->s_cell[q] & 0xffffffffLL;
    if (b->s_comp[q] == 2) ++b->n_h_groups;
    else if (local / I.ny == I.line_i) b->merge_post = false;
  }
  for (auto& c : b->s_cell) {
    const Inst& I = b->inst[(int)(c >> 32)];
    const long long local = c & 0xffffffffLL;
    c = I.off + local / I.ny * I.pitch + local % I.ny;
  }
  b->src.n_groups = (int)b->s_cell.size();
  b->src.n_steps = b->n_steps;
  if (b->src.n_groups) {
    if ((rc = bup(b, (void**)&b->src.cell, b->s_cell.data(), b->s_cell.size() * 8))) return rc;
    if ((rc = bup(b, (void**)&b->src.comp, b->s_comp.data(), b->s_comp.size() * 4))) return rc;
    if ((rc = bup(b, (void**)&b->src.start, b->s_start.data(), b->s_start.size() * 4))) return rc;
    if ((rc = bup(b, (void**)&b->src.wave_row, b->s_row.data(), b->s_row.size() * 4))) return rc;
    if ((rc = bup(b, (void**)&b->src.amp, b->s_amp.data(), b->s_amp.size() * 8))) return rc;
    void* w = nullptr;
    if ((rc = bup(b, &w, b->h_wave.data(), b->h_wave.size() * 8))) return rc;
    b->src.wave = (const double*)w;
  }
  if (b->rb == 4) {
    for (int ax = 0; ax < 2; ++ax) {
      const float d = (float)(ax == 0 ? b->dx : b->dy);
      b->rd[ax] = (double)(1.0f / d);
      b->fd[ax] = !getenv("PFB200_IEEE_DIV") && host_recip_division_exact(d);
    }
  }
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  b->finalized = true;
  return PF_OK;
}

int pfb_set_design_ce(pf_batch* b, const void* ce_design) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized) return bfail(b, PF_ERR_STATE, "pfb_set_design_ce before pfb_finalize");
  if (!ce_design) return bfail(b, PF_ERR_INVALID, "ce_design is NULL");
  B_CUDA(b, cudaMemcpyAsync(b->design_stage, ce_design, (size_t)b->n_design * b->rb,
                            cudaMemcpyHostToDevice, b->stream));
  const dim3 grid(16, b->n_inst);
  if (b->rb == 4)
    kb_scatter_design<float><<<grid, 256, 0, b->stream>>>(b->d_inst, b->n_inst,
                                                           (const float*)b->design_stage, (float*)b->ce);
  else
    kb_scatter_design<double><<<grid, 256, 0, b->stream>>>(
        b->d_inst, b->n_inst, (const double*)b->design_stage, (double*)b->ce);
  b->launches += 1;
  B_CUDA(b, cudaGetLastError());
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  b->fwd_done = false;
  return PF_OK;
}

int pfb_forward(pf_batch* b) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized) return bfail(b, PF_ERR_STATE, "pfb_forward before pfb_finalize");
  return b->rb == 4 ? forward_t<float>(b) : forward_t<double>(b);
}

int pfb_adjoint(pf_batch* b, const double* cotangent) {
  if (!b) return PF_ERR_INVALID;
  if (b->fwd_only) return bfail(b, PF_ERR_STATE, "forward-only batch (checkpoint_every = 0)");
  if (!b->fwd_done)
    return bfail(b, PF_ERR_STATE, "pfb_adjoint needs a pfb_forward of the current design");
  if (!cotangent) return bfail(b, PF_ERR_INVALID, "cotangent is NULL");
  B_CUDA(b, cudaMemcpyAsync(b->cot, cotangent, (size_t)b->nline * b->n_freq * 16,
                            cudaMemcpyHostToDevice, b->stream));
  return b->rb == 4 ? adjoint_t<float>(b) : adjoint_t<double>(b);
}

int pfb_read_dft(pf_batch* b, double* dst) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized || !dst) return bfail(b, PF_ERR_INVALID, "bad pfb_read_dft");
  B_CUDA(b, cudaMemcpyAsync(dst, b->acc, (size_t)b->nline * b->n_freq * 16, cudaMemcpyDeviceToHost,
                            b->stream));
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  return PF_OK;
}

int pfb_read_grad(pf_batch* b, double* dst) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized || !dst) return bfail(b, PF_ERR_INVALID, "bad pfb_read_grad");
  if (b->fwd_only) return bfail(b, PF_ERR_STATE, "forward-only batch (checkpoint_every = 0)");
  B_CUDA(b, cudaMemcpyAsync(dst, b->grad, (size_t)b->n_design * 8, cudaMemcpyDeviceToHost,
                            b->stream));
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  return PF_OK;
}

int pfb_read_field(pf_batch* b, int k, int comp, void* dst) {
  if (!b) return PF_ERR_INVALID;
  if (!b->finalized || k < 0 || k >= b->n_inst || comp < 0 || comp > 2 || !dst)
    return bfail(b, PF_ERR_INVALID, "bad pfb_read_field");
  const Inst& I = b->inst[k];
  const bool l1 = level_at(b, b->field_step) == 1;
  void* src = comp == 0 ? (l1 ? b->lvl1[0] : b->Ex)
                        : (comp == 1 ? (l1 ? b->lvl1[1] : b->Ey) : (l1 ? b->lvl1[2] : b->Hz));
  B_CUDA(b, cudaMemcpy2DAsync(dst, (size_t)I.ny * b->rb, (char*)src + I.off * b->rb,
                              (size_t)I.pitch * b->rb, (size_t)I.ny * b->rb, I.nx,
                              cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  return PF_OK;
}

int pfb_info(const pf_batch* b, int64_t* out, int n_out) {
  if (!b || !out) return PF_ERR_INVALID;
  const int64_t v[9] = {b->ncell_real,
                        b->nline,
                        b->n_design,
                        b->ntiles,
                        (int64_t)b->ckpt,
                        (int64_t)((b->n_steps + b->ckpt - 1) / b->ckpt),
                        b->state_elems,
                        b->launches,
                        b->fused ? 1 : 0};
  for (int q = 0; q < n_out && q < 9; ++q) out[q] = v[q];
  return PF_OK;
}

void* pfb_stream(pf_batch* b) { return b ? (void*)b->stream : nullptr; }

void pfb_destroy(pf_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  destroy_graphs(b);
  for (void* p : b->allocs) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // extern "C"
