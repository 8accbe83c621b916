// batch2d.cu - batched 2D TE engine with a hand-written discrete adjoint.
//
// Many uneven 2D instances (xy plane, nz = 1) are stepped together. Their
// fields live in pooled arrays, and every kernel walks one work list of
// 32 (y) x TI (x) tiles drawn from all instances (grid-stride, so one launch
// covers the batch whatever the sizes). Only Ex, Ey, Hz are stepped: with
// TE-only sources the other three components of the reference's update
// (src/photonfdtd/simulation.py:1252-1309 with nz = 1) stay exactly zero, so
// Ex, Ey, Hz are the reference's to the bit. The step index lives in device
// memory; chunks of steps are captured once as CUDA graphs and replayed.
//
// Step n: Hz (curl of E, CPML psi along x and y), H sources, Ex / Ey (curl
// of Hz, psi), E sources, the output-line DFT of Ey accumulated in
// complex128: acc += (exp(i w (n+1) dt) * Ey) * dt.
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
// ceil(N / K) states + K window rings; K >= N keeps one state and needs no
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
#include "common.cuh"

using namespace pfb;

namespace {

struct Inst {
  int nx, ny;
  long long off;                         // first cell in the pooled field arrays
  int ox, oy;                            // first entry in the pooled x / y coefficients
  long long p_hzx, p_hzy, p_exy, p_eyx;  // first element of each psi array
  int nphx, nphy, npex, npey;            // compact psi extents along their axes
  int di0, dj0, dn;                      // design window
  long long goff;                        // first design cell (dn * dn per instance)
  int line_i;                            // x index of the output line
  long long loff;                        // first line cell (ny per instance)
};

template <typename T>
struct BArgs {
  const Inst* inst;
  const int4* tiles;  // (instance, i0, j0, -)
  int ntiles;
  T *Ex, *Ey, *Hz;
  const T* ce;
  const T *bex, *cex, *bhx, *chx, *bey, *cey, *bhy, *chy;
  const int *mex, *mhx, *mey, *mhy;
  T *pHzx, *pHzy, *pExy, *pEyx;
  T dx, dy, rdx, rdy, ch;
  T idx, idy;  // 1/dx, 1/dy rounded once (adjoint kernels only)
  bool fdx, fdy;
};

// ---- forward ---------------------------------------------------------------
// Hz^{n+1/2} = Hz - ch (dEy/dx - dEx/dy) - ch psi_x + ch psi_y, where the
// forward differences exist (i < nx-1, j < ny-1).
template <typename T, int TI>
__global__ void __launch_bounds__(32 * TI) kb_h(const __grid_constant__ BArgs<T> a) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int4 tl = a.tiles[t];
    const Inst& I = a.inst[tl.x];
    const int i = tl.y + threadIdx.y, j = tl.z + threadIdx.x;
    if (i >= I.nx - 1 || j >= I.ny - 1) continue;
    const long long id = I.off + (long long)i * I.ny + j;
    const T ey = a.Ey[id], ex = a.Ex[id];
    const T dA = qdiv(sub_rn(a.Ey[id + I.ny], ey), a.dx, a.rdx, a.fdx);
    const T dB = qdiv(sub_rn(a.Ex[id + 1], ex), a.dy, a.rdy, a.fdy);
    const T mch = -a.ch;
    T h = add_rn(a.Hz[id], mul_rn(sub_rn(dA, dB), mch));
    const int mx = a.mhx[I.ox + i];
    if (mx >= 0) {
      const long long q = I.p_hzx + (long long)mx * I.ny + j;
      const T psi = add_rn(mul_rn(a.bhx[I.ox + i], a.pHzx[q]), mul_rn(a.chx[I.ox + i], dA));
      a.pHzx[q] = psi;
      h = add_rn(h, mul_rn(mch, psi));
    }
    const int my = a.mhy[I.oy + j];
    if (my >= 0) {
      const long long q = I.p_hzy + (long long)i * I.nphy + my;
      const T psi = add_rn(mul_rn(a.bhy[I.oy + j], a.pHzy[q]), mul_rn(a.chy[I.oy + j], dB));
      a.pHzy[q] = psi;
      h = add_rn(h, mul_rn(a.ch, psi));
    }
    a.Hz[id] = h;
  }
}

// Ex^{n+1} = Ex + K dHz/dy + K psi_y (j >= 1); Ey^{n+1} = Ey - K dHz/dx -
// K psi_x (i >= 1). With `ring`, design cells store the curls that
// multiplied K: ring[n mod K][cell] = (cEx, cEy).
template <typename T, int TI>
__global__ void __launch_bounds__(32 * TI) kb_e(const __grid_constant__ BArgs<T> a, T* ring,
                                               long long n_design, const long long* step,
                                               int ring_len) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int4 tl = a.tiles[t];
    const Inst& I = a.inst[tl.x];
    const int i = tl.y + threadIdx.y, j = tl.z + threadIdx.x;
    if (i >= I.nx || j >= I.ny) continue;
    const long long id = I.off + (long long)i * I.ny + j;
    const T K = a.ce[id];
    const T hz = a.Hz[id];
    T cx = T(0), cy = T(0);
    if (j >= 1) {
      const T dA = qdiv(sub_rn(hz, a.Hz[id - 1]), a.dy, a.rdy, a.fdy);
      T e = add_rn(a.Ex[id], mul_rn(dA, K));
      cx = dA;
      const int my = a.mey[I.oy + j];
      if (my >= 0) {
        const long long q = I.p_exy + (long long)i * I.npey + my;
        const T psi = add_rn(mul_rn(a.bey[I.oy + j], a.pExy[q]), mul_rn(a.cey[I.oy + j], dA));
        a.pExy[q] = psi;
        e = add_rn(e, mul_rn(K, psi));
        cx = add_rn(dA, psi);
      }
      a.Ex[id] = e;
    }
    if (i >= 1) {
      const T dB = qdiv(sub_rn(hz, a.Hz[id - I.ny]), a.dx, a.rdx, a.fdx);
      T e = add_rn(a.Ey[id], mul_rn(-dB, K));
      cy = -dB;
      const int mx = a.mex[I.ox + i];
      if (mx >= 0) {
        const long long q = I.p_eyx + (long long)mx * I.ny + j;
        const T psi = add_rn(mul_rn(a.bex[I.ox + i], a.pEyx[q]), mul_rn(a.cex[I.ox + i], dB));
        a.pEyx[q] = psi;
        e = add_rn(e, mul_rn(-K, psi));
        cy = sub_rn(cy, psi);
      }
      a.Ey[id] = e;
    }
    if (ring) {
      const int di = i - I.di0, dj = j - I.dj0;
      if (di >= 0 && di < I.dn && dj >= 0 && dj < I.dn) {
        const long long slot = *step % ring_len;
        T* r = ring + (slot * n_design + I.goff + (long long)di * I.dn + dj) * 2;
        r[0] = cx;
        r[1] = cy;
      }
    }
  }
}

struct BSources {
  const long long* cell;  // pooled cell of each group
  const int* comp;        // 0 Ex, 1 Ey, 2 Hz
  const int* start;       // group q owns entries start[q] .. start[q+1]-1
  const int* wave_row;
  const double* amp;
  const double* wave;     // (rows, n_steps) waveform values at the family's times
  long long n_steps;
  int n_groups;
};

// Soft sources: field += amp * waveform, in list order per cell, each term
// added in double and rounded once (numpy's array += python float).
template <typename T>
__global__ void kb_inject(BSources s, T* Ex, T* Ey, T* Hz, int family_h, const long long* step) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n_groups) return;
  const int c = s.comp[g];
  if ((c == 2) != (family_h != 0)) return;
  T* F = c == 0 ? Ex : (c == 1 ? Ey : Hz);
  const long long n = *step;
  T v = F[s.cell[g]];
  for (int q = s.start[g]; q < s.start[g + 1]; ++q)
    v = add_double<T>(v, __dmul_rn(s.amp[q], s.wave[(long long)s.wave_row[q] * s.n_steps + n]));
  F[s.cell[g]] = v;
}

// Line DFT of Ey in the reference's order: acc += (phase * Ey) * dt, per step.
template <typename T>
__global__ void kb_dft(const long long* lcell, long long nline, const T* Ey, double* acc,
                       const double* phase, int n_freq, double dt, const long long* step) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nline) return;
  const double s = (double)Ey[lcell[c]];
  const double* ph = phase + (*step) * n_freq * 2;
  double* A = acc + c * n_freq * 2;
  for (int f = 0; f < n_freq; ++f) {
    A[2 * f] = __dadd_rn(A[2 * f], __dmul_rn(__dmul_rn(ph[2 * f], s), dt));
    A[2 * f + 1] = __dadd_rn(A[2 * f + 1], __dmul_rn(__dmul_rn(ph[2 * f + 1], s), dt));
  }
}

__global__ void kb_tick(long long* step, long long by) { *step += by; }
__global__ void kb_set(long long* step, long long v) { *step = v; }

// Writes packed design-window coefficients into the pooled ce array.
template <typename T>
__global__ void kb_scatter_design(const Inst* inst, int n_inst, const T* src, T* ce) {
  const int k = blockIdx.y;
  if (k >= n_inst) return;
  const Inst& I = inst[k];
  const int n = I.dn * I.dn;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int di = q / I.dn, dj = q % I.dn;
    ce[I.off + (long long)(I.di0 + di) * I.ny + I.dj0 + dj] = src[I.goff + q];
  }
}

// ---- adjoint ---------------------------------------------------------------
template <typename T>
struct AArgs {
  T *aEx, *aEy, *aHz, *aHzx, *aHzy, *aExy, *aEyx;  // adjoint state
  T *gA, *gB, *hA, *hB;                             // adjoints of the per-cell differences
  double* grad;                                     // dL/dK per design cell
  const T* ring;                                    // forward curls, slot = n mod K
  long long n_design;
  int ring_len;
};

// Adjoint source of step n on the output line.
template <typename T>
__global__ void kb_adj_src(const long long* lcell, long long nline, T* aEy, const double* G,
                           const double* phase, int n_freq, double dt, const long long* step) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nline) return;
  const double* ph = phase + (*step) * n_freq * 2;
  const double* g = G + c * n_freq * 2;
  double s = 0.0;
  for (int f = 0; f < n_freq; ++f) s += g[2 * f] * ph[2 * f] + g[2 * f + 1] * ph[2 * f + 1];
  const long long id = lcell[c];
  aEy[id] = (T)((double)aEy[id] + dt * s);
}

// Transpose of the E update of step n (cell-local): the K gradient, the E psi
// adjoints, gA = adjoint of dHz/dy in Ex, gB = adjoint of dHz/dx in Ey.
template <typename T, int TI>
__global__ void __launch_bounds__(32 * TI) kb_adj_e(const __grid_constant__ BArgs<T> a,
                                                   const __grid_constant__ AArgs<T> d,
                                                   const long long* step) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int4 tl = a.tiles[t];
    const Inst& I = a.inst[tl.x];
    const int i = tl.y + threadIdx.y, j = tl.z + threadIdx.x;
    if (i >= I.nx || j >= I.ny) continue;
    const long long id = I.off + (long long)i * I.ny + j;
    const T K = a.ce[id];
    const T lx = d.aEx[id], ly = d.aEy[id];
    const int di = i - I.di0, dj = j - I.dj0;
    if (di >= 0 && di < I.dn && dj >= 0 && dj < I.dn) {
      const long long dc = I.goff + (long long)di * I.dn + dj;
      const T* r = d.ring + ((*step % d.ring_len) * d.n_design + dc) * 2;
      d.grad[dc] += (double)lx * (double)r[0] + (double)ly * (double)r[1];
    }
    T ga = T(0), gb = T(0);
    if (j >= 1) {
      ga = K * lx;
      const int my = a.mey[I.oy + j];
      if (my >= 0) {
        const long long q = I.p_exy + (long long)i * I.npey + my;
        const T ap = d.aExy[q] + K * lx;
        ga += a.cey[I.oy + j] * ap;
        d.aExy[q] = a.bey[I.oy + j] * ap;
      }
    }
    if (i >= 1) {
      gb = -K * ly;
      const int mx = a.mex[I.ox + i];
      if (mx >= 0) {
        const long long q = I.p_eyx + (long long)mx * I.ny + j;
        const T ap = d.aEyx[q] - K * ly;
        gb += a.cex[I.ox + i] * ap;
        d.aEyx[q] = a.bex[I.ox + i] * ap;
      }
    }
    d.gA[id] = ga;
    d.gB[id] = gb;
  }
}

// Transpose of the H update: gathers the E-update terms into aHz, then the H
// psi adjoints and hA = adjoint of dEy/dx, hB = adjoint of dEx/dy.
template <typename T, int TI>
__global__ void __launch_bounds__(32 * TI) kb_adj_h(const __grid_constant__ BArgs<T> a,
                                                   const __grid_constant__ AArgs<T> d) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int4 tl = a.tiles[t];
    const Inst& I = a.inst[tl.x];
    const int i = tl.y + threadIdx.y, j = tl.z + threadIdx.x;
    if (i >= I.nx || j >= I.ny) continue;
    const long long id = I.off + (long long)i * I.ny + j;
    T ah = d.aHz[id];
    T ga = d.gA[id], gb = d.gB[id];
    if (j + 1 < I.ny) ga -= d.gA[id + 1];
    if (i + 1 < I.nx) gb -= d.gB[id + I.ny];
    ah += ga * a.idy + gb * a.idx;
    T ha = T(0), hb = T(0);
    if (i < I.nx - 1 && j < I.ny - 1) {
      ha = -a.ch * ah;
      hb = a.ch * ah;
      const int mx = a.mhx[I.ox + i];
      if (mx >= 0) {
        const long long q = I.p_hzx + (long long)mx * I.ny + j;
        const T ap = d.aHzx[q] - a.ch * ah;
        ha += a.chx[I.ox + i] * ap;
        d.aHzx[q] = a.bhx[I.ox + i] * ap;
      }
      const int my = a.mhy[I.oy + j];
      if (my >= 0) {
        const long long q = I.p_hzy + (long long)i * I.nphy + my;
        const T ap = d.aHzy[q] + a.ch * ah;
        hb += a.chy[I.oy + j] * ap;
        d.aHzy[q] = a.bhy[I.oy + j] * ap;
      }
    }
    d.aHz[id] = ah;
    d.hA[id] = ha;
    d.hB[id] = hb;
  }
}

// E adjoints from the H update's differences (gathered from i-1 / j-1).
template <typename T, int TI>
__global__ void __launch_bounds__(32 * TI) kb_adj_e2(const __grid_constant__ BArgs<T> a,
                                                    const __grid_constant__ AArgs<T> d) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int4 tl = a.tiles[t];
    const Inst& I = a.inst[tl.x];
    const int i = tl.y + threadIdx.y, j = tl.z + threadIdx.x;
    if (i >= I.nx || j >= I.ny) continue;
    const long long id = I.off + (long long)i * I.ny + j;
    T ha = -d.hA[id], hb = -d.hB[id];
    if (i >= 1) ha += d.hA[id - I.ny];
    if (j >= 1) hb += d.hB[id - 1];
    d.aEy[id] += ha * a.idx;
    d.aEx[id] += hb * a.idy;
  }
}

}  // namespace

// ===========================================================================
struct pf_batch {
  int n_inst = 0, rb = 4;
  double dx = 1, dy = 1, ch = 0, dt = 0;
  long long n_steps = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  std::vector<Inst> inst;
  std::vector<std::vector<char>> h_ce;
  std::vector<std::vector<char>> h_coef[8];  // bex cex bhx chx bey cey bhy chy
  long long ncell = 0, nx_tot = 0, ny_tot = 0, n_design = 0, nline = 0;
  long long npsi[4] = {};
  int ti = 8;
  int ckpt = 64;
  bool finalized = false, fwd_done = false, ring_last = false;
  bool fd[2] = {false, false};
  double rd[2] = {1, 1};
  std::vector<long long> s_cell;
  std::vector<int> s_comp, s_start, s_row;
  std::vector<double> s_amp, h_wave, h_phase;
  int n_freq = 0;
  // device
  std::vector<void*> allocs;
  Inst* d_inst = nullptr;
  int4* d_tiles = nullptr;
  int ntiles = 0;
  void *Ex = nullptr, *Ey = nullptr, *Hz = nullptr, *ce = nullptr;
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
  long long* step = nullptr;
  BSources src{};
  // instantiated graphs, keyed by (chunk kind, steps)
  std::map<std::pair<int, long long>, cudaGraphExec_t> graphs;
  int64_t launches = 0;
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
  return a;
}

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
  d.ring = (const T*)b->ring;
  d.n_design = b->n_design;
  d.ring_len = b->ckpt;
  return d;
}

// Persistent-style grid: as many blocks as fit on the 148 SMs walk the tiles.
int grid_blocks(const pf_batch* b) {
  return std::max(1, std::min(b->ntiles, 148 * (2048 / (32 * b->ti))));
}

template <typename T, int TI>
void fwd_kernels(pf_batch* b, bool dft, bool record) {
  const BArgs<T> a = bargs<T>(b);
  const dim3 blk(32, TI);
  const int G = grid_blocks(b);
  kb_h<T, TI><<<G, blk, 0, b->stream>>>(a);
  if (b->src.n_groups)
    kb_inject<T><<<(b->src.n_groups + 127) / 128, 128, 0, b->stream>>>(b->src, a.Ex, a.Ey, a.Hz, 1,
                                                                         b->step);
  kb_e<T, TI><<<G, blk, 0, b->stream>>>(a, record ? (T*)b->ring : nullptr, b->n_design, b->step,
                                        b->ckpt);
  if (b->src.n_groups)
    kb_inject<T><<<(b->src.n_groups + 127) / 128, 128, 0, b->stream>>>(b->src, a.Ex, a.Ey, a.Hz, 0,
                                                                         b->step);
  if (dft && b->nline)
    kb_dft<T><<<(unsigned)((b->nline + 127) / 128), 128, 0, b->stream>>>(
        b->lcell, b->nline, a.Ey, b->acc, b->phase, b->n_freq, b->dt, b->step);
  kb_tick<<<1, 1, 0, b->stream>>>(b->step, 1);
}

template <typename T>
void fwd_step(pf_batch* b, bool dft, bool record) {
  if (b->ti == 4) fwd_kernels<T, 4>(b, dft, record);
  else if (b->ti == 8) fwd_kernels<T, 8>(b, dft, record);
  else fwd_kernels<T, 16>(b, dft, record);
}

template <typename T, int TI>
void adj_kernels(pf_batch* b) {
  const BArgs<T> a = bargs<T>(b);
  const AArgs<T> d = aargs<T>(b);
  const dim3 blk(32, TI);
  const int G = grid_blocks(b);
  if (b->nline)
    kb_adj_src<T><<<(unsigned)((b->nline + 127) / 128), 128, 0, b->stream>>>(
        b->lcell, b->nline, d.aEy, b->cot, b->phase, b->n_freq, b->dt, b->step);
  kb_adj_e<T, TI><<<G, blk, 0, b->stream>>>(a, d, b->step);
  kb_adj_h<T, TI><<<G, blk, 0, b->stream>>>(a, d);
  kb_adj_e2<T, TI><<<G, blk, 0, b->stream>>>(a, d);
  kb_tick<<<1, 1, 0, b->stream>>>(b->step, -1);
}

template <typename T>
void adj_step(pf_batch* b) {
  if (b->ti == 4) adj_kernels<T, 4>(b);
  else if (b->ti == 8) adj_kernels<T, 8>(b);
  else adj_kernels<T, 16>(b);
}

// Kernel launches of one step of each chunk kind.
long long launches_per_step(const pf_batch* b, int kind) {
  if (kind == 2) return 4 + (b->nline ? 1 : 0);
  return 3 + (b->src.n_groups ? 2 : 0) + (kind == 0 && b->nline ? 1 : 0);
}

// Runs `len` steps of kind 0 (forward + DFT + ring), 1 (replay: forward +
// ring) or 2 (adjoint) as one graph launch. Each (kind, len) is captured
// once; at most two lengths occur per kind (K and the last segment's).
template <typename T>
int run_chunk(pf_batch* b, int kind, long long len) {
  cudaGraphExec_t& ex = b->graphs[std::make_pair(kind, len)];
  if (ex == nullptr) {
    cudaGraph_t graph = nullptr;
    B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (long long t = 0; t < len; ++t) {
      if (kind == 2) adj_step<T>(b);
      else fwd_step<T>(b, kind == 0, true);
    }
    const cudaError_t e1 = cudaStreamEndCapture(b->stream, &graph);
    if (e1 != cudaSuccess) return bfail(b, PF_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e1));
    const cudaError_t e2 = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
      ex = nullptr;
      return bfail(b, PF_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e2));
    }
  }
  B_CUDA(b, cudaGraphLaunch(ex, b->stream));
  b->launches += launches_per_step(b, kind) * len;
  return PF_OK;
}

// Copies the stepping state (Ex, Ey, Hz, four psi arrays) to / from slot s.
int state_copy(pf_batch* b, long long s, bool save) {
  const size_t S = b->rb;
  char* base = (char*)b->ckpt_buf + (size_t)s * b->state_elems * S;
  void* parts[7] = {b->Ex, b->Ey, b->Hz, b->psi[0], b->psi[1], b->psi[2], b->psi[3]};
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

int set_step(pf_batch* b, long long s) {
  kb_set<<<1, 1, 0, b->stream>>>(b->step, s);
  b->launches += 1;
  B_CUDA(b, cudaGetLastError());
  return PF_OK;
}

int zero_state(pf_batch* b) {
  const size_t S = b->rb;
  for (void* p : {b->Ex, b->Ey, b->Hz}) B_CUDA(b, cudaMemsetAsync(p, 0, b->ncell * S, b->stream));
  for (int q = 0; q < 4; ++q)
    if (b->npsi[q]) B_CUDA(b, cudaMemsetAsync(b->psi[q], 0, b->npsi[q] * S, b->stream));
  return PF_OK;
}

template <typename T>
int forward_t(pf_batch* b) {
  int rc;
  if ((rc = zero_state(b))) return rc;
  B_CUDA(b, cudaMemsetAsync(b->acc, 0, (size_t)b->nline * b->n_freq * 16, b->stream));
  if ((rc = set_step(b, 0))) return rc;
  const long long K = b->ckpt;
  for (long long s0 = 0; s0 < b->n_steps; s0 += K) {
    if (s0 > 0 && (rc = state_copy(b, s0 / K - 1, true))) return rc;  // segment 0 starts at zero
    if ((rc = run_chunk<T>(b, 0, std::min(K, b->n_steps - s0)))) return rc;
  }
  B_CUDA(b, cudaGetLastError());
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  b->fwd_done = true;
  b->ring_last = true;
  return PF_OK;
}

template <typename T>
int adjoint_t(pf_batch* b) {
  const size_t S = b->rb;
  int rc;
  for (int q = 0; q < 3; ++q) B_CUDA(b, cudaMemsetAsync(b->aE[q], 0, b->ncell * S, b->stream));
  for (int q = 0; q < 4; ++q)
    if (b->npsi[q]) B_CUDA(b, cudaMemsetAsync(b->apsi[q], 0, b->npsi[q] * S, b->stream));
  B_CUDA(b, cudaMemsetAsync(b->grad, 0, (size_t)b->n_design * 8, b->stream));
  const long long K = b->ckpt;
  const long long nseg = (b->n_steps + K - 1) / K;
  for (long long sg = nseg - 1; sg >= 0; --sg) {
    const long long s0 = sg * K, len = std::min(K, b->n_steps - s0);
    if (sg < nseg - 1 || !b->ring_last) {  // refill the ring from the segment's checkpoint
      if (sg == 0) {
        if ((rc = zero_state(b))) return rc;
      } else if ((rc = state_copy(b, sg - 1, false))) {
        return rc;
      }
      if ((rc = set_step(b, s0))) return rc;
      if ((rc = run_chunk<T>(b, 1, len))) return rc;
    }
    if ((rc = set_step(b, s0 + len - 1))) return rc;
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
    if (kv.second) cudaGraphExecDestroy(kv.second);
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

int pfb_finalize(pf_batch* b, int checkpoint_every, int tile_rows) {
  if (!b) return PF_ERR_INVALID;
  if (b->finalized) return bfail(b, PF_ERR_STATE, "pfb_finalize called twice");
  if (checkpoint_every < 1) return bfail(b, PF_ERR_INVALID, "checkpoint_every must be >= 1");
  if (tile_rows != 4 && tile_rows != 8 && tile_rows != 16)
    return bfail(b, PF_ERR_INVALID, "tile_rows must be 4, 8 or 16");
  if (b->n_freq < 1) return bfail(b, PF_ERR_STATE, "pfb_set_dft must come before pfb_finalize");
  for (int k = 0; k < b->n_inst; ++k)
    if (b->inst[k].nx == 0) return bfail(b, PF_ERR_STATE, "instance %d not set", k);
  b->ckpt = (int)std::min<long long>(checkpoint_every, b->n_steps);
  b->ti = tile_rows;
  const size_t S = b->rb;
  std::vector<int> mp[4];
  std::vector<char> coefp[8], cep;
  std::vector<long long> lcell;
  std::vector<int4> tiles;
  for (int k = 0; k < b->n_inst; ++k) {
    Inst& I = b->inst[k];
    I.off = b->ncell;
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
    cep.insert(cep.end(), b->h_ce[k].begin(), b->h_ce[k].end());
    for (int q = 0; q < 8; ++q)
      coefp[q].insert(coefp[q].end(), b->h_coef[q][k].begin(), b->h_coef[q][k].end());
    for (int j = 0; j < I.ny; ++j) lcell.push_back(I.off + (long long)I.line_i * I.ny + j);
    for (int i0 = 0; i0 < I.nx; i0 += b->ti)
      for (int j0 = 0; j0 < I.ny; j0 += 32) tiles.push_back(make_int4(k, i0, j0, 0));
    b->ncell += (long long)I.nx * I.ny;
    b->nx_tot += I.nx;
    b->ny_tot += I.ny;
    b->n_design += (long long)I.dn * I.dn;
    b->nline += I.ny;
    std::vector<char>().swap(b->h_ce[k]);
  }
  if ((long long)tiles.size() >= (1LL << 31)) return bfail(b, PF_ERR_INVALID, "too many tiles");
  b->ntiles = (int)tiles.size();
  int rc;
  if ((rc = bup(b, (void**)&b->d_inst, b->inst.data(), b->inst.size() * sizeof(Inst)))) return rc;
  if ((rc = bup(b, (void**)&b->d_tiles, tiles.data(), tiles.size() * sizeof(int4)))) return rc;
  if ((rc = bup(b, &b->ce, cep.data(), cep.size()))) return rc;
  for (int q = 0; q < 8; ++q)
    if ((rc = bup(b, &b->coef[q], coefp[q].data(), coefp[q].size()))) return rc;
  for (int q = 0; q < 4; ++q)
    if ((rc = bup(b, (void**)&b->maps[q], mp[q].data(), mp[q].size() * 4))) return rc;
  for (void** p : {&b->Ex, &b->Ey, &b->Hz})
    if ((rc = balloc(b, p, b->ncell * S))) return rc;
  for (int q = 0; q < 3; ++q)
    if ((rc = balloc(b, &b->aE[q], b->ncell * S))) return rc;
  for (int q = 0; q < 4; ++q) {
    if ((rc = balloc(b, &b->psi[q], b->npsi[q] * S))) return rc;
    if ((rc = balloc(b, &b->apsi[q], b->npsi[q] * S))) return rc;
    if ((rc = balloc(b, &b->g[q], b->ncell * S))) return rc;
  }
  if ((rc = balloc(b, (void**)&b->grad, b->n_design * 8))) return rc;
  if ((rc = balloc(b, &b->design_stage, b->n_design * S))) return rc;
  if ((rc = balloc(b, &b->ring, (size_t)b->ckpt * b->n_design * 2 * S))) return rc;
  b->state_elems = 3 * b->ncell + b->npsi[0] + b->npsi[1] + b->npsi[2] + b->npsi[3];
  const long long nseg = (b->n_steps + b->ckpt - 1) / b->ckpt;
  // checkpoints of segments 1 .. nseg-1 (segment 0 starts from the zero state)
  if ((rc = balloc(b, &b->ckpt_buf, (size_t)(nseg - 1) * b->state_elems * S))) return rc;
  if ((rc = balloc(b, (void**)&b->acc, (size_t)b->nline * b->n_freq * 16))) return rc;
  if ((rc = balloc(b, (void**)&b->cot, (size_t)b->nline * b->n_freq * 16))) return rc;
  if ((rc = bup(b, (void**)&b->lcell, lcell.data(), lcell.size() * 8))) return rc;
  if ((rc = bup(b, (void**)&b->phase, b->h_phase.data(), b->h_phase.size() * 8))) return rc;
  if ((rc = balloc(b, (void**)&b->step, 8))) return rc;
  for (auto& c : b->s_cell) c = b->inst[(int)(c >> 32)].off + (c & 0xffffffffLL);
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
  void* src = comp == 0 ? b->Ex : (comp == 1 ? b->Ey : b->Hz);
  B_CUDA(b, cudaMemcpyAsync(dst, (char*)src + I.off * b->rb, (size_t)I.nx * I.ny * b->rb,
                            cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(b, cudaStreamSynchronize(b->stream));
  return PF_OK;
}

int pfb_info(const pf_batch* b, int64_t* out, int n_out) {
  if (!b || !out) return PF_ERR_INVALID;
  const int64_t v[8] = {b->ncell,
                        b->nline,
                        b->n_design,
                        b->ntiles,
                        (int64_t)b->ckpt,
                        (int64_t)((b->n_steps + b->ckpt - 1) / b->ckpt),
                        b->state_elems,
                        b->launches};
  for (int q = 0; q < n_out && q < 8; ++q) out[q] = v[q];
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
