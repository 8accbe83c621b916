// batch2d_kernels.cuh - kernels of the batched 2D TE engine (batch2d.cu).
//
// Layout: each instance's rows are padded to a pitch of a multiple of 32
// cells and start 32-aligned, so a warp's row access is one aligned line.
// Work list: tiles of 32 columns (y) x 8R rows (x) drawn from every
// instance; a block of 32 x 8 threads takes one tile, each thread R
// consecutive rows of one column. Every thread issues all its loads before
// its first store (the row it shares with the next row is loaded once), so a
// block keeps 8R cells per column in flight. A tile record carries everything
// needed to address its cells; the instance record is read only for CPML
// psi, design-window and output-line cells.
//
// The step index n of a kernel is *base + t: base is set once per chunk of
// steps, t is baked into the launch, so a captured chunk replays for any
// segment without per-step counter kernels.
#pragma once

#include "common.cuh"

namespace pfb {
namespace b2d {

constexpr int kWarps = 8;     // warps per block
// Minimum resident blocks per SM the fused forward and reverse steps are
// compiled for.
#ifndef PFB_MINB_STEP
#define PFB_MINB_STEP 4
#endif
#ifndef PFB_MINB_ASTEP
#define PFB_MINB_ASTEP 4
#endif
// Minimum resident 128-thread blocks per SM of the marching forward and
// reverse steps (forward at 12: 40 registers, measured 5% faster than at 10;
// the reverse step needs 46-48 registers and slows down at 12).
#ifndef PFB_MINB_MARCH
#define PFB_MINB_MARCH 12
#endif
#ifndef PFB_MINB_AMARCH
#define PFB_MINB_AMARCH 10
#endif
constexpr int kDftRing = 32;  // line samples kept before a DFT flush

struct Inst {
  int nx, ny;
  int pitch;                             // row stride: ny rounded up to 32
  long long off;                         // first cell in the pooled field arrays (32-aligned)
  int ox, oy;                            // first entry in the pooled x / y coefficients
  long long p_hzx, p_hzy, p_exy, p_eyx;  // first element of each psi array
  int nphx, nphy, npex, npey;            // compact psi extents along their axes
  int di0, dj0, dn;                      // design window
  long long goff;                        // first design cell (dn * dn per instance)
  int line_i;                            // x index of the output line
  long long loff;                        // first line cell (ny per instance)
};

struct __align__(16) TileRec {
  long long base;      // pooled index of the tile origin (i0, j0)
  int nx, ny, pitch;   // instance extents, row stride
  int i0, j0;          // tile origin in the instance
  int ox, oy;          // pooled coefficient index of row i0 / column j0
  int k;               // instance
  int wdi, wdj, wdn;   // design window relative to the tile origin, its size
  int pad[1];
};

// A marching segment: instance k, rows [i0, i1), owned columns [j0, j0 + 31).
// Its warp's lane l holds column j0 - 1 + l: lane 0 is the halo column.
struct SegRec {
  int k, i0, i1, j0;
};
constexpr int kMarchCols = 31;  // owned columns per warp
constexpr int kMarchWarps = 4;  // warps (segments) per block

template <typename T>
struct BArgs {
  const Inst* inst;
  const TileRec* tiles;
  int ntiles;
  const SegRec* segs;
  int nsegs;
  T *Ex, *Ey, *Hz;
  const T* ce;
  const T *bex, *cex, *bhx, *chx, *bey, *cey, *bhy, *chy;
  const int *mex, *mhx, *mey, *mhy;
  T *pHzx, *pHzy, *pExy, *pEyx;
  T dx, dy, rdx, rdy, ch;
  T idx, idy;  // 1/dx, 1/dy rounded once (adjoint kernels only)
  bool fdx, fdy;
  const long long* base;  // first step of the running chunk
  T* ring;                // design-window curls, slot = n mod ring_len
  long long n_design;
  int ring_len;
  // The fused step's double-buffered state: step n reads level n & 1 and
  // writes level (n & 1) ^ 1 (level 0 is Ex / Ey / Hz / pHzx / pHzy above).
  T *Ex2[2], *Ey2[2], *Hz2[2], *pHzx2[2], *pHzy2[2];
};

// ---- forward ---------------------------------------------------------------
// Hz^{n+1/2} = Hz - ch (dEy/dx - dEx/dy) - ch psi_x + ch psi_y where both
// forward differences exist (i < nx-1, j < ny-1); the reference's operation
// order (simulation.py:1284-1309).
template <typename T, int R>
__global__ void __launch_bounds__(32 * kWarps) kb_h(const __grid_constant__ BArgs<T> a) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const int r0 = threadIdx.y * R;
    const int i = tr.i0 + r0, j = tr.j0 + threadIdx.x;
    if (j >= tr.ny - 1 || i >= tr.nx - 1) continue;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + threadIdx.x;
    T ey[R + 1], ex0[R], ex1[R], hz[R];
    int mx[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = i + r < tr.nx - 1;  // an H row
      const long long id = id0 + (long long)r * tr.pitch;
      ey[r] = i + r < tr.nx ? a.Ey[id] : T(0);  // also the row after the last H row
      ex0[r] = ok ? a.Ex[id] : T(0);
      ex1[r] = ok ? a.Ex[id + 1] : T(0);
      hz[r] = ok ? a.Hz[id] : T(0);
      mx[r] = ok ? a.mhx[tr.ox + r0 + r] : -1;
    }
    ey[R] = (i + R < tr.nx) ? a.Ey[id0 + (long long)R * tr.pitch] : T(0);
    const int my = a.mhy[tr.oy + threadIdx.x];
    const T mch = -a.ch;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (i + r >= tr.nx - 1) break;
      const T dA = qdiv(sub_rn(ey[r + 1], ey[r]), a.dx, a.rdx, a.fdx);
      const T dB = qdiv(sub_rn(ex1[r], ex0[r]), a.dy, a.rdy, a.fdy);
      T h = add_rn(hz[r], mul_rn(sub_rn(dA, dB), mch));
      if (mx[r] >= 0 || my >= 0) {
        const Inst& I = a.inst[tr.k];
        if (mx[r] >= 0) {
          const long long q = I.p_hzx + (long long)mx[r] * tr.ny + j;
          const int c = tr.ox + r0 + r;
          const T psi = add_rn(mul_rn(a.bhx[c], a.pHzx[q]), mul_rn(a.chx[c], dA));
          a.pHzx[q] = psi;
          h = add_rn(h, mul_rn(mch, psi));
        }
        if (my >= 0) {
          const long long q = I.p_hzy + (long long)(i + r) * I.nphy + my;
          const int c = tr.oy + threadIdx.x;
          const T psi = add_rn(mul_rn(a.bhy[c], a.pHzy[q]), mul_rn(a.chy[c], dB));
          a.pHzy[q] = psi;
          h = add_rn(h, mul_rn(a.ch, psi));
        }
      }
      a.Hz[id0 + (long long)r * tr.pitch] = h;
    }
  }
}

// Ex^{n+1} = Ex + K dHz/dy + K psi_y (j >= 1); Ey^{n+1} = Ey - K dHz/dx -
// K psi_x (i >= 1). Design cells also store the curls that multiplied K:
// ring[n mod ring_len][cell] = (cEx, cEy), n = *base + step_t.
template <typename T, int R>
__global__ void __launch_bounds__(32 * kWarps) kb_e(const __grid_constant__ BArgs<T> a,
                                                   int step_t) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const int r0 = threadIdx.y * R;
    const int i = tr.i0 + r0, j = tr.j0 + threadIdx.x;
    if (j >= tr.ny || i >= tr.nx) continue;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + threadIdx.x;
    T hz[R + 1], hzl[R], ex[R], ey[R], K[R];
    int mx[R];
    hz[0] = i >= 1 ? a.Hz[id0 - tr.pitch] : T(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = i + r < tr.nx;
      const long long id = id0 + (long long)r * tr.pitch;
      hz[r + 1] = ok ? a.Hz[id] : T(0);
      hzl[r] = (ok && j >= 1) ? a.Hz[id - 1] : T(0);
      ex[r] = ok ? a.Ex[id] : T(0);
      ey[r] = ok ? a.Ey[id] : T(0);
      K[r] = ok ? a.ce[id] : T(0);
      mx[r] = ok ? a.mex[tr.ox + r0 + r] : -1;
    }
    const int my = a.mey[tr.oy + threadIdx.x];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (i + r >= tr.nx) break;
      const long long id = id0 + (long long)r * tr.pitch;
      T cx = T(0), cy = T(0);
      if (j >= 1) {
        const T dA = qdiv(sub_rn(hz[r + 1], hzl[r]), a.dy, a.rdy, a.fdy);
        T e = add_rn(ex[r], mul_rn(dA, K[r]));
        cx = dA;
        if (my >= 0) {
          const Inst& I = a.inst[tr.k];
          const long long q = I.p_exy + (long long)(i + r) * I.npey + my;
          const int c = tr.oy + threadIdx.x;
          const T psi = add_rn(mul_rn(a.bey[c], a.pExy[q]), mul_rn(a.cey[c], dA));
          a.pExy[q] = psi;
          e = add_rn(e, mul_rn(K[r], psi));
          cx = add_rn(dA, psi);
        }
        a.Ex[id] = e;
      }
      if (i + r >= 1) {
        const T dB = qdiv(sub_rn(hz[r + 1], hz[r]), a.dx, a.rdx, a.fdx);
        T e = add_rn(ey[r], mul_rn(-dB, K[r]));
        cy = -dB;
        if (mx[r] >= 0) {
          const Inst& I = a.inst[tr.k];
          const long long q = I.p_eyx + (long long)mx[r] * tr.ny + j;
          const int c = tr.ox + r0 + r;
          const T psi = add_rn(mul_rn(a.bex[c], a.pEyx[q]), mul_rn(a.cex[c], dB));
          a.pEyx[q] = psi;
          e = add_rn(e, mul_rn(-K[r], psi));
          cy = sub_rn(cy, psi);
        }
        a.Ey[id] = e;
      }
      const int di = r0 + r - tr.wdi, dj = (int)threadIdx.x - tr.wdj;
      if (di >= 0 && di < tr.wdn && dj >= 0 && dj < tr.wdn) {
        const Inst& I = a.inst[tr.k];
        const long long slot = (*a.base + step_t) % a.ring_len;
        T* rr = a.ring + (slot * a.n_design + I.goff + (long long)di * tr.wdn + dj) * 2;
        rr[0] = cx;
        rr[1] = cy;
      }
    }
  }
}

// ---- fused forward step ------------------------------------------------------
// One launch per step on double-buffered fields: a tile first updates Hz of
// its own cells and, recomputed from the previous level, of the one-cell halo
// its E update needs (the row above, the column to the left), keeping them in
// shared memory; then it updates Ex and Ey of its own cells from there.
// Everything is read from level n & 1 and written to level (n & 1) ^ 1 (the
// E psi, which no other tile reads, in place), so tiles never race and the
// fields cross HBM once per step: Ex, Ey, Hz and ce read, Ex, Ey, Hz written.
// The arithmetic of every cell is kb_h's and kb_e's, operation for operation,
// so the results equal the split passes' bit for bit. Used when no source
// drives Hz (an H source would have to reach the halo recomputation).

// Hz^{n+1/2} of cell (i, j) from its own old value and its E neighbours, as
// kb_h computes it. crow / ccol: pooled x / y coefficient index of the cell;
// psi_out == nullptr recomputes a halo cell without storing its psi.
template <typename T>
__device__ __forceinline__ T hz_value(const BArgs<T>& a, const Inst& I, int i, int j, int ny,
                                      int crow, int ccol, int mx, int my, T hz, T eyp, T ey,
                                      T exp_, T ex, const T* pzx, T* pzxo, const T* pzy,
                                      T* pzyo) {
  const T mch = -a.ch;
  T dA, dB;
  qdiv2(sub_rn(eyp, ey), a.dx, a.rdx, a.fdx, sub_rn(exp_, ex), a.dy, a.rdy, a.fdy, dA, dB);
  T h = add_rn(hz, mul_rn(sub_rn(dA, dB), mch));
  if (mx >= 0) {
    const long long q = I.p_hzx + (long long)mx * ny + j;
    const T psi = add_rn(mul_rn(a.bhx[crow], pzx[q]), mul_rn(a.chx[crow], dA));
    if (pzxo) pzxo[q] = psi;
    h = add_rn(h, mul_rn(mch, psi));
  }
  if (my >= 0) {
    const long long q = I.p_hzy + (long long)i * I.nphy + my;
    const T psi = add_rn(mul_rn(a.bhy[ccol], pzy[q]), mul_rn(a.chy[ccol], dB));
    if (pzyo) pzyo[q] = psi;
    h = add_rn(h, mul_rn(a.ch, psi));
  }
  return h;
}

// Every global load of a tile is issued before its barrier: the own cells'
// E and H values, coefficients and CPML maps (the E update reuses the Ex / Ey
// values the H update loaded), the halo row's inputs (warp 0) and the halo
// column's (warp 1, one row per lane), so a block waits out one memory
// latency per tile.
template <typename T, int R>
__global__ void __launch_bounds__(32 * kWarps, PFB_MINB_STEP) kb_step(
    const __grid_constant__ BArgs<T> a, int step_t) {
  constexpr int TR = kWarps * R;
  static_assert(TR <= 32, "the halo column is one warp's work");
  __shared__ T sH[TR + 1][33];  // [1 + row][1 + column]; row / column 0 = halo
  const long long n = *a.base + step_t;
  const int L = (int)(n & 1);
  const T* Ex = a.Ex2[L];
  const T* Ey = a.Ey2[L];
  const T* Hz = a.Hz2[L];
  T* Exo = a.Ex2[L ^ 1];
  T* Eyo = a.Ey2[L ^ 1];
  T* Hzo = a.Hz2[L ^ 1];
  const T* pzx = a.pHzx2[L];
  const T* pzy = a.pHzy2[L];
  T* pzxo = a.pHzx2[L ^ 1];
  T* pzyo = a.pHzy2[L ^ 1];
  const int lane = threadIdx.x;
  const int r0 = threadIdx.y * R;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const Inst& I = a.inst[tr.k];
    const int i = tr.i0 + r0, j = tr.j0 + lane;
    const bool jv = j < tr.ny;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + lane;
    // ---- loads: own cells
    T ey[R + 1], ex0[R], ex1[R], hz[R], K[R];
    int mxh[R], mxe[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = jv && i + r < tr.nx;
      const long long id = id0 + (long long)r * tr.pitch;
      ey[r] = ok ? Ey[id] : T(0);
      ex0[r] = ok ? Ex[id] : T(0);
      ex1[r] = (ok && j + 1 < tr.ny) ? Ex[id + 1] : T(0);
      hz[r] = ok ? Hz[id] : T(0);
      K[r] = ok ? a.ce[id] : T(0);
      mxh[r] = ok ? a.mhx[tr.ox + r0 + r] : -1;
      mxe[r] = ok ? a.mex[tr.ox + r0 + r] : -1;
    }
    ey[R] = (jv && i + R < tr.nx) ? Ey[id0 + (long long)R * tr.pitch] : T(0);
    const int myh = jv ? a.mhy[tr.oy + lane] : -1;
    const int mye = jv ? a.mey[tr.oy + lane] : -1;
    // ---- loads: the halo cell this thread recomputes, if any (warp 0: row
    // i0 - 1 at column j; warp 1: column j0 - 1 at tile row `lane`)
    int hrole = 0;  // 1 halo row, 2 halo column
    int hi = 0, hj = 0, hcrow = 0, hccol = 0, hmx = -1, hmy = -1;
    T hz_h = T(0), hey1 = T(0), hey0 = T(0), hex1 = T(0), hex0 = T(0);
    if (threadIdx.y == 0 && tr.i0 >= 1 && jv) {
      hrole = 1;
      hi = tr.i0 - 1;
      hj = j;
      hcrow = tr.ox - 1;
      hccol = tr.oy + lane;
    } else if (threadIdx.y == 1 && lane < TR && tr.j0 >= 1 && tr.i0 + lane < tr.nx) {
      hrole = 2;
      hi = tr.i0 + lane;
      hj = tr.j0 - 1;
      hcrow = tr.ox + lane;
      hccol = tr.oy - 1;
    }
    const bool hupd = hrole && hi < tr.nx - 1 && hj < tr.ny - 1;
    if (hrole) {
      const long long id = tr.base + (long long)(hi - tr.i0) * tr.pitch + (hj - tr.j0);
      hz_h = Hz[id];
      if (hupd) {
        hey1 = Ey[id + tr.pitch];
        hey0 = Ey[id];
        hex1 = Ex[id + 1];
        hex0 = Ex[id];
        hmx = a.mhx[hcrow];
        hmy = a.mhy[hccol];
      }
    }
    // ---- Hz of the tile's own cells
#pragma unroll
    for (int r = 0; r < R; ++r) {
      T h = hz[r];
      if (jv && i + r < tr.nx - 1 && j < tr.ny - 1)
        h = hz_value<T>(a, I, i + r, j, tr.ny, tr.ox + r0 + r, tr.oy + lane, mxh[r], myh, hz[r],
                        ey[r + 1], ey[r], ex1[r], ex0[r], pzx, pzxo, pzy, pzyo);
      if (jv && i + r < tr.nx) Hzo[id0 + (long long)r * tr.pitch] = h;
      sH[r0 + r + 1][lane + 1] = h;
    }
    // ---- the halo cell, recomputed from level L (its psi is not stored)
    {
      T h = hz_h;
      if (hupd)
        h = hz_value<T>(a, I, hi, hj, tr.ny, hcrow, hccol, hmx, hmy, hz_h, hey1, hey0, hex1,
                        hex0, pzx, nullptr, pzy, nullptr);
      if (threadIdx.y == 0) sH[0][lane + 1] = hrole == 1 ? h : T(0);
      if (threadIdx.y == 1 && lane < TR) sH[lane + 1][0] = hrole == 2 ? h : T(0);
    }
    __syncthreads();
    // ---- Ex, Ey of the tile's own cells (kb_e's arithmetic, Hz from shared memory)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!(jv && i + r < tr.nx)) break;
      const long long id = id0 + (long long)r * tr.pitch;
      const T hc = sH[r0 + r + 1][lane + 1];
      T cx = T(0), cy = T(0);
      T e = ex0[r];
      if (j >= 1) {
        const T dA = qdiv(sub_rn(hc, sH[r0 + r + 1][lane]), a.dy, a.rdy, a.fdy);
        e = add_rn(ex0[r], mul_rn(dA, K[r]));
        cx = dA;
        if (mye >= 0) {
          const long long q = I.p_exy + (long long)(i + r) * I.npey + mye;
          const int c = tr.oy + lane;
          const T psi = add_rn(mul_rn(a.bey[c], a.pExy[q]), mul_rn(a.cey[c], dA));
          a.pExy[q] = psi;
          e = add_rn(e, mul_rn(K[r], psi));
          cx = add_rn(dA, psi);
        }
      }
      Exo[id] = e;
      e = ey[r];
      if (i + r >= 1) {
        const T dB = qdiv(sub_rn(hc, sH[r0 + r][lane + 1]), a.dx, a.rdx, a.fdx);
        e = add_rn(ey[r], mul_rn(-dB, K[r]));
        cy = -dB;
        if (mxe[r] >= 0) {
          const long long q = I.p_eyx + (long long)mxe[r] * tr.ny + j;
          const int c = tr.ox + r0 + r;
          const T psi = add_rn(mul_rn(a.bex[c], a.pEyx[q]), mul_rn(a.cex[c], dB));
          a.pEyx[q] = psi;
          e = add_rn(e, mul_rn(-K[r], psi));
          cy = sub_rn(cy, psi);
        }
      }
      Eyo[id] = e;
      const int di = r0 + r - tr.wdi, dj = lane - tr.wdj;
      if (di >= 0 && di < tr.wdn && dj >= 0 && dj < tr.wdn) {
        const long long slot = n % a.ring_len;
        T* rr = a.ring + (slot * a.n_design + I.goff + (long long)di * tr.wdn + dj) * 2;
        rr[0] = cx;
        rr[1] = cy;
      }
    }
    __syncthreads();  // sH is rewritten by the next tile
  }
}

// ---- marching forward step ---------------------------------------------------
// One warp per segment marches down its rows: lane l holds column
// j0 - 1 + l, so the left neighbour of every owned column (lanes 1..31) sits
// in the lane below and the right neighbour in the lane above (shuffles);
// lane 0 is a halo column whose Hz it recomputes without storing, and lane 31
// loads the one Ex beyond the strip. The Hz of the previous row stays in a
// register; a segment that starts below row 0 first recomputes its row
// i0 - 1 (Hz only). The next row's loads are issued before the current row is
// computed. As in kb_step, level n & 1 is read and level (n & 1) ^ 1
// written, so segments never race, and every cell's arithmetic is kb_h's and
// kb_e's (hz_value and the E update below), bit for bit. No shared memory,
// no barriers, about four cell loads and three stores per cell and step.
template <typename T>
__global__ void __launch_bounds__(32 * kMarchWarps, PFB_MINB_MARCH) kb_march(
    const __grid_constant__ BArgs<T> a, int step_t) {
  const int w = blockIdx.x * kMarchWarps + threadIdx.y;
  if (w >= a.nsegs) return;  // uniform over the warp
  const SegRec sg = a.segs[w];
  const Inst& I = a.inst[sg.k];
  const long long n = *a.base + step_t;
  const int L = (int)(n & 1);
  const T* Ex = a.Ex2[L];
  const T* Ey = a.Ey2[L];
  const T* Hz = a.Hz2[L];
  T* Exo = a.Ex2[L ^ 1];
  T* Eyo = a.Ey2[L ^ 1];
  T* Hzo = a.Hz2[L ^ 1];
  const T* pzx = a.pHzx2[L];
  const T* pzy = a.pHzy2[L];
  T* pzxo = a.pHzx2[L ^ 1];
  T* pzyo = a.pHzy2[L ^ 1];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  const int nx = I.nx, ny = I.ny;
  const long long pitch = I.pitch;
  const int j = sg.j0 - 1 + lane;
  const bool jv = j >= 0 && j < ny;
  const bool own = lane >= 1 && jv;
  const bool hcol = jv && j < ny - 1;       // Hz is updated in this column
  const bool xr = lane == 31 && j + 1 < ny;  // lane 31 loads Ex one column right
  const long long c0 = I.off + j;           // pooled index of (0, j)
  const int myh = jv ? a.mhy[I.oy + j] : -1;
  const int mye = jv ? a.mey[I.oy + j] : -1;
  const int slot = (int)(n % a.ring_len);
  const int r_first = sg.i0 > 0 ? sg.i0 - 1 : 0;
  // row r_first
  T ex = T(0), hz = T(0), ey = T(0), eyn = T(0), K = T(0), ex31 = T(0);
  {
    const long long id = c0 + r_first * pitch;
    if (jv) {
      ex = Ex[id];
      hz = Hz[id];
      ey = Ey[id];
      if (r_first + 1 < nx) eyn = Ey[id + pitch];
      if (r_first >= sg.i0) K = a.ce[id];
    }
    if (xr) ex31 = Ex[id + 1];
  }
  T hz_prev = T(0);  // Hz^{n+1/2} of the row above
  for (int r = r_first; r < sg.i1; ++r) {
    // the next row's loads first
    const int r1 = r + 1;
    T ex_n = T(0), hz_n = T(0), eyn_n = T(0), K_n = T(0), ex31_n = T(0);
    if (r1 < sg.i1) {
      const long long id = c0 + r1 * pitch;
      if (jv) {
        ex_n = Ex[id];
        hz_n = Hz[id];
        if (r1 + 1 < nx) eyn_n = Ey[id + pitch];
        K_n = a.ce[id];
      }
      if (xr) ex31_n = Ex[id + 1];
    }
    const long long id = c0 + r * pitch;
    const bool body = r >= sg.i0;  // uniform: a row this segment owns
    // Hz of row r (every lane: the halo lane and the prologue row too)
    T exr = __shfl_down_sync(full, ex, 1);
    if (lane == 31) exr = ex31;
    T h = hz;
    if (hcol && r < nx - 1) {
      const bool st = own && body;
      h = hz_value<T>(a, I, r, j, ny, I.ox + r, I.oy + j, a.mhx[I.ox + r], myh, hz, eyn, ey,
                      exr, ex, pzx, st ? pzxo : nullptr, pzy, st ? pzyo : nullptr);
    }
    const T hl = __shfl_up_sync(full, h, 1);  // Hz^{n+1/2} of column j - 1
    if (body && own) {
      Hzo[id] = h;
      // Ex, Ey of (r, j): kb_e's arithmetic (both quotients formed; each is
      // used only where its difference exists)
      T cx = T(0), cy = T(0);
      T e = ex;
      T dA, dBq;
      qdiv2(sub_rn(h, hl), a.dy, a.rdy, a.fdy, sub_rn(h, hz_prev), a.dx, a.rdx, a.fdx, dA, dBq);
      if (j >= 1) {
        e = add_rn(ex, mul_rn(dA, K));
        cx = dA;
        if (mye >= 0) {
          const long long q = I.p_exy + (long long)r * I.npey + mye;
          const int c = I.oy + j;
          const T psi = add_rn(mul_rn(a.bey[c], a.pExy[q]), mul_rn(a.cey[c], dA));
          a.pExy[q] = psi;
          e = add_rn(e, mul_rn(K, psi));
          cx = add_rn(dA, psi);
        }
      }
      Exo[id] = e;
      e = ey;
      if (r >= 1) {
        const T dB = dBq;
        e = add_rn(ey, mul_rn(-dB, K));
        cy = -dB;
        const int mx = a.mex[I.ox + r];
        if (mx >= 0) {
          const long long q = I.p_eyx + (long long)mx * ny + j;
          const int c = I.ox + r;
          const T psi = add_rn(mul_rn(a.bex[c], a.pEyx[q]), mul_rn(a.cex[c], dB));
          a.pEyx[q] = psi;
          e = add_rn(e, mul_rn(-K, psi));
          cy = sub_rn(cy, psi);
        }
      }
      Eyo[id] = e;
      const int di = r - I.di0, dj = j - I.dj0;
      if (di >= 0 && di < I.dn && dj >= 0 && dj < I.dn) {
        T* rr = a.ring + ((long long)slot * a.n_design + I.goff + (long long)di * I.dn + dj) * 2;
        rr[0] = cx;
        rr[1] = cy;
      }
    }
    hz_prev = h;
    ex = ex_n;
    hz = hz_n;
    ey = eyn;
    eyn = eyn_n;
    K = K_n;
    ex31 = ex31_n;
  }
}

// Field pointers kb_post writes through: level 0 for the in-place split
// passes; for the fused step (flip = 1) the level step n has just written.
template <typename T>
struct BFields {
  T* Ex[2];
  T* Ey[2];
  T* Hz[2];
  int flip;
};

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

// Soft sources of one family (field += amp * waveform, in list order per
// cell, each term added in double and rounded once, as numpy's in-place add
// of a float64 scalar does) and, with `dring`, the step's Ey samples of the
// output lines into the DFT ring. Threads [0, n_groups) inject, the next
// nline threads sample: one launch is correct only when no group of this
// family sits on a line cell, which the host checks.
template <typename T>
__global__ void kb_post(BSources s, BFields<T> f, int family_h, const long long* base,
                        int step_t, const long long* lcell, long long nline, T* dring) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = *base + step_t;
  const int lv = f.flip ? (int)((n & 1) ^ 1) : 0;
  T* Ex = f.Ex[lv];
  T* Ey = f.Ey[lv];
  T* Hz = f.Hz[lv];
  if (g < s.n_groups) {
    const int c = s.comp[g];
    if ((c == 2) != (family_h != 0)) return;
    T* F = c == 0 ? Ex : (c == 1 ? Ey : Hz);
    T v = F[s.cell[g]];
    for (int q = s.start[g]; q < s.start[g + 1]; ++q)
      v = add_double<T>(v, __dmul_rn(s.amp[q], s.wave[(long long)s.wave_row[q] * s.n_steps + n]));
    F[s.cell[g]] = v;
    return;
  }
  const long long c = g - s.n_groups;
  if (dring && c < nline) dring[(long long)(step_t % kDftRing) * nline + c] = Ey[lcell[c]];
}

// Folds n_pend ring samples (chunk steps t_first ..) into the line DFT in
// step order, acc += (exp(i w (n+1) dt) * Ey) * dt with the reference's two
// roundings per part (simulation.py:1116-1133). One thread per (cell, freq).
template <typename T>
__global__ void kb_dft_flush(const T* dring, long long nline, double* acc, const double* phase,
                             int n_freq, double dt, const long long* base, int t_first,
                             int n_pend) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nline * n_freq) return;
  const long long c = g / n_freq;
  const int f = (int)(g % n_freq);
  double re = acc[2 * g], im = acc[2 * g + 1];
  const long long n0 = *base;
  for (int q = 0; q < n_pend; ++q) {
    const int tt = t_first + q;
    const double v = (double)dring[(long long)(tt % kDftRing) * nline + c];
    const double* p = phase + ((n0 + tt) * n_freq + f) * 2;
    re = __dadd_rn(re, __dmul_rn(__dmul_rn(p[0], v), dt));
    im = __dadd_rn(im, __dmul_rn(__dmul_rn(p[1], v), dt));
  }
  acc[2 * g] = re;
  acc[2 * g + 1] = im;
}

__global__ void kb_set(long long* v, long long x) { *v = x; }

// Writes packed design-window coefficients into the pooled ce array.
template <typename T>
__global__ void kb_scatter_design(const Inst* inst, int n_inst, const T* src, T* ce) {
  const int k = blockIdx.y;
  if (k >= n_inst) return;
  const Inst& I = inst[k];
  const int n = I.dn * I.dn;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int di = q / I.dn, dj = q % I.dn;
    ce[I.off + (long long)(I.di0 + di) * I.pitch + I.dj0 + dj] = src[I.goff + q];
  }
}

// ---- adjoint ---------------------------------------------------------------
template <typename T>
struct AArgs {
  T *aEx, *aEy, *aHz, *aHzx, *aHzy, *aExy, *aEyx;  // adjoint state
  T *gA, *gB, *hA, *hB;                             // adjoints of the per-cell differences
  double* grad;                                     // dL/dK per design cell
  const double* cot;                                // DFT cotangent, (line cells, n_freq)
  const double* phase;                              // exp(i w (n+1) dt), (n_steps, n_freq)
  int n_freq;
  double dt;
  // The fused reverse step's double-buffered state (level 0 = the arrays
  // above): the E transpose of step m writes gA / gB into level m & 1; the H
  // transpose of step n reads aHz and its psi adjoints from level (n + 1) & 1
  // and writes them into level n & 1.
  T *aHz2[2], *aHzx2[2], *aHzy2[2], *gA2[2], *gB2[2];
};

// The adjoint arithmetic is written with explicitly rounded operations, so
// its result does not depend on the tile shape (no compiler contraction).

// Transpose of the H update: gathers the E-update terms into aHz
// (gA from j and j+1, gB from i and i+1), then the H psi adjoints and
// hA = adjoint of dEy/dx, hB = adjoint of dEx/dy.
template <typename T, int R>
__global__ void __launch_bounds__(32 * kWarps) kb_adj_h(const __grid_constant__ BArgs<T> a,
                                                       const __grid_constant__ AArgs<T> d) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const int r0 = threadIdx.y * R;
    const int i = tr.i0 + r0, j = tr.j0 + threadIdx.x;
    if (j >= tr.ny || i >= tr.nx) continue;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + threadIdx.x;
    const bool jn = j + 1 < tr.ny;
    T ah[R], ga0[R], ga1[R], gb[R + 1];
    int mx[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = i + r < tr.nx;
      const long long id = id0 + (long long)r * tr.pitch;
      ah[r] = ok ? d.aHz[id] : T(0);
      ga0[r] = ok ? d.gA[id] : T(0);
      ga1[r] = (ok && jn) ? d.gA[id + 1] : T(0);
      gb[r] = ok ? d.gB[id] : T(0);
      mx[r] = ok ? a.mhx[tr.ox + r0 + r] : -1;
    }
    gb[R] = (i + R < tr.nx) ? d.gB[id0 + (long long)R * tr.pitch] : T(0);
    const int my = a.mhy[tr.oy + threadIdx.x];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (i + r >= tr.nx) break;
      const long long id = id0 + (long long)r * tr.pitch;
      const T h = fma_rn(sub_rn(gb[r], gb[r + 1]), a.idx, fma_rn(sub_rn(ga0[r], ga1[r]), a.idy, ah[r]));
      T ha = T(0), hb = T(0);
      if (i + r < tr.nx - 1 && j < tr.ny - 1) {
        ha = mul_rn(-a.ch, h);
        hb = mul_rn(a.ch, h);
        if (mx[r] >= 0 || my >= 0) {
          const Inst& I = a.inst[tr.k];
          if (mx[r] >= 0) {
            const long long q = I.p_hzx + (long long)mx[r] * tr.ny + j;
            const int c = tr.ox + r0 + r;
            const T ap = fma_rn(-a.ch, h, d.aHzx[q]);
            ha = fma_rn(a.chx[c], ap, ha);
            d.aHzx[q] = mul_rn(a.bhx[c], ap);
          }
          if (my >= 0) {
            const long long q = I.p_hzy + (long long)(i + r) * I.nphy + my;
            const int c = tr.oy + threadIdx.x;
            const T ap = fma_rn(a.ch, h, d.aHzy[q]);
            hb = fma_rn(a.chy[c], ap, hb);
            d.aHzy[q] = mul_rn(a.bhy[c], ap);
          }
        }
      }
      d.aHz[id] = h;
      d.hA[id] = ha;
      d.hB[id] = hb;
    }
  }
}

// Cell-local part of the reverse pass. With E2, first finishes step n+1's E
// adjoints from the H update's differences (hA from rows i-1 and i, hB from
// columns j-1 and j). With E, then runs the transpose of step n's E update
// (n = *base + step_t): the adjoint source on the output line,
// dt * sum_f Re(conj(G_f) phase_f^n); the K gradient of design cells; the E
// psi adjoints; gA / gB, the adjoints of dHz/dy in Ex and dHz/dx in Ey.
template <typename T, int R, bool E2, bool E>
__global__ void __launch_bounds__(32 * kWarps) kb_adj_cell(const __grid_constant__ BArgs<T> a,
                                                          const __grid_constant__ AArgs<T> d,
                                                          int step_t) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const int r0 = threadIdx.y * R;
    const int i = tr.i0 + r0, j = tr.j0 + threadIdx.x;
    if (j >= tr.ny || i >= tr.nx) continue;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + threadIdx.x;
    T lx[R], ly[R], ha[R + 1], hb0[R], hb1[R], K[R];
    int mx[R];
    if (E2) ha[0] = i >= 1 ? d.hA[id0 - tr.pitch] : T(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = i + r < tr.nx;
      const long long id = id0 + (long long)r * tr.pitch;
      lx[r] = ok ? d.aEx[id] : T(0);
      ly[r] = ok ? d.aEy[id] : T(0);
      if (E2) {
        ha[r + 1] = ok ? d.hA[id] : T(0);
        hb0[r] = ok ? d.hB[id] : T(0);
        hb1[r] = (ok && j >= 1) ? d.hB[id - 1] : T(0);
      }
      if (E) {
        K[r] = ok ? a.ce[id] : T(0);
        mx[r] = ok ? a.mex[tr.ox + r0 + r] : -1;
      }
    }
    const int my = E ? a.mey[tr.oy + threadIdx.x] : -1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (i + r >= tr.nx) break;
      const long long id = id0 + (long long)r * tr.pitch;
      T x = lx[r], y = ly[r];
      if (E2) {
        y = fma_rn(sub_rn(ha[r], ha[r + 1]), a.idx, y);
        x = fma_rn(sub_rn(hb1[r], hb0[r]), a.idy, x);
      }
      if (E) {
        const long long n = *a.base + step_t;
        const Inst& I = a.inst[tr.k];
        if (i + r == I.line_i) {
          const double* ph = d.phase + n * d.n_freq * 2;
          const double* g = d.cot + (I.loff + j) * d.n_freq * 2;
          double s = 0.0;
          for (int f = 0; f < d.n_freq; ++f)
            s = __dadd_rn(s, __dadd_rn(__dmul_rn(g[2 * f], ph[2 * f]),
                                       __dmul_rn(g[2 * f + 1], ph[2 * f + 1])));
          y = (T)__dadd_rn((double)y, __dmul_rn(d.dt, s));
        }
        const int di = r0 + r - tr.wdi, dj = (int)threadIdx.x - tr.wdj;
        if (di >= 0 && di < tr.wdn && dj >= 0 && dj < tr.wdn) {
          const long long dc = I.goff + (long long)di * tr.wdn + dj;
          const T* rr = a.ring + ((n % a.ring_len) * a.n_design + dc) * 2;
          d.grad[dc] = __dadd_rn(d.grad[dc], __dadd_rn(__dmul_rn((double)x, (double)rr[0]),
                                                       __dmul_rn((double)y, (double)rr[1])));
        }
        T ga = T(0), gb = T(0);
        if (j >= 1) {
          ga = mul_rn(K[r], x);
          if (my >= 0) {
            const long long q = I.p_exy + (long long)(i + r) * I.npey + my;
            const int c = tr.oy + threadIdx.x;
            const T ap = fma_rn(K[r], x, d.aExy[q]);
            ga = fma_rn(a.cey[c], ap, ga);
            d.aExy[q] = mul_rn(a.bey[c], ap);
          }
        }
        if (i + r >= 1) {
          gb = mul_rn(-K[r], y);
          if (mx[r] >= 0) {
            const long long q = I.p_eyx + (long long)mx[r] * tr.ny + j;
            const int c = tr.ox + r0 + r;
            const T ap = fma_rn(-K[r], y, d.aEyx[q]);
            gb = fma_rn(a.cex[c], ap, gb);
            d.aEyx[q] = mul_rn(a.bex[c], ap);
          }
        }
        d.gA[id] = ga;
        d.gB[id] = gb;
      }
      d.aEx[id] = x;
      d.aEy[id] = y;
    }
  }
}

// ---- fused reverse step -------------------------------------------------------
// One launch per reverse step n, on double-buffered adjoint state: the H
// transpose of step n (HT: gather gA / gB into aHz, H psi adjoints, hA / hB),
// the gather of hA / hB into step n's E adjoints, then the E transpose of step
// n - 1 (ET: line source, design gradient, E psi adjoints, new gA / gB). hA
// and hB never leave shared memory: a tile recomputes them on its one-cell
// halo (the row above, the column to the left) from the previous level.
// Without HT the launch is the E transpose of step n alone (a chunk's first
// launch); without ET it ends after the gather (its last). Every cell's
// arithmetic is kb_adj_h's and kb_adj_cell's, operation for operation.

// aHz after the H transpose of one cell and its hA / hB (psi adjoints stored
// only when the output pointers are given).
template <typename T>
__device__ __forceinline__ void adj_h_value(const BArgs<T>& a, const Inst& I, int i, int j,
                                            int nx, int ny, int crow, int ccol, int mx, int my,
                                            T ah, T ga0, T ga1, T gb0, T gb1, const T* pzx,
                                            T* pzxo, const T* pzy, T* pzyo, T& h, T& ha,
                                            T& hb) {
  h = fma_rn(sub_rn(gb0, gb1), a.idx, fma_rn(sub_rn(ga0, ga1), a.idy, ah));
  ha = T(0);
  hb = T(0);
  if (i < nx - 1 && j < ny - 1) {
    ha = mul_rn(-a.ch, h);
    hb = mul_rn(a.ch, h);
    if (mx >= 0) {
      const long long q = I.p_hzx + (long long)mx * ny + j;
      const T ap = fma_rn(-a.ch, h, pzx[q]);
      ha = fma_rn(a.chx[crow], ap, ha);
      if (pzxo) pzxo[q] = mul_rn(a.bhx[crow], ap);
    }
    if (my >= 0) {
      const long long q = I.p_hzy + (long long)i * I.nphy + my;
      const T ap = fma_rn(a.ch, h, pzy[q]);
      hb = fma_rn(a.chy[ccol], ap, hb);
      if (pzyo) pzyo[q] = mul_rn(a.bhy[ccol], ap);
    }
  }
}

template <typename T, int R, bool HT, bool ET>
__global__ void __launch_bounds__(32 * kWarps, PFB_MINB_ASTEP) kb_adj_step(
    const __grid_constant__ BArgs<T> a, const __grid_constant__ AArgs<T> d, int step_t) {
  constexpr int TR = kWarps * R;
  static_assert(TR <= 32, "the halo column is one warp's work");
  __shared__ T sA[TR + 1][33];  // hA: [1 + row][1 + column]; row 0 = halo row
  __shared__ T sB[TR + 1][33];  // hB: column 0 = halo column
  const long long n = *a.base + step_t;
  const long long m = HT ? n - 1 : n;  // the step of the E transpose
  const int lg = (int)(n & 1);         // gA / gB level the H transpose reads
  const int lh = (int)((n + 1) & 1);   // aHz / H psi adjoint level it reads
  const T* gA = d.gA2[lg];
  const T* gB = d.gB2[lg];
  T* gAo = d.gA2[(int)(m & 1)];
  T* gBo = d.gB2[(int)(m & 1)];
  const T* aHz = d.aHz2[lh];
  T* aHzo = d.aHz2[lh ^ 1];
  const T* pzx = d.aHzx2[lh];
  const T* pzy = d.aHzy2[lh];
  T* pzxo = d.aHzx2[lh ^ 1];
  T* pzyo = d.aHzy2[lh ^ 1];
  const int lane = threadIdx.x;
  const int r0 = threadIdx.y * R;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const TileRec tr = a.tiles[t];
    const Inst& I = a.inst[tr.k];
    const int i = tr.i0 + r0, j = tr.j0 + lane;
    const bool jv = j < tr.ny;
    const long long id0 = tr.base + (long long)r0 * tr.pitch + lane;
    // ---- loads, all before the barrier: the E adjoints and coefficients of
    // the own cells, then (HT) their H-transpose inputs and the halo's
    T lx[R], ly[R], K[R];
    int mxe[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const bool ok = jv && i + r < tr.nx;
      const long long id = id0 + (long long)r * tr.pitch;
      lx[r] = ok ? d.aEx[id] : T(0);
      ly[r] = ok ? d.aEy[id] : T(0);
      if (ET) {
        K[r] = ok ? a.ce[id] : T(0);
        mxe[r] = ok ? a.mex[tr.ox + r0 + r] : -1;
      }
    }
    const int mye = (ET && jv) ? a.mey[tr.oy + lane] : -1;
    if (HT) {
      T ah[R], ga0[R], ga1[R], gb[R + 1];
      int mxh[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const bool ok = jv && i + r < tr.nx;
        const long long id = id0 + (long long)r * tr.pitch;
        ah[r] = ok ? aHz[id] : T(0);
        ga0[r] = ok ? gA[id] : T(0);
        ga1[r] = (ok && j + 1 < tr.ny) ? gA[id + 1] : T(0);
        gb[r] = ok ? gB[id] : T(0);
        mxh[r] = ok ? a.mhx[tr.ox + r0 + r] : -1;
      }
      gb[R] = (jv && i + R < tr.nx) ? gB[id0 + (long long)R * tr.pitch] : T(0);
      const int myh = jv ? a.mhy[tr.oy + lane] : -1;
      // the halo cell of this thread, if any: warp 0 row i0 - 1 (its hA),
      // warp 1 column j0 - 1 at tile row `lane` (its hB)
      int hrole = 0, hi = 0, hj = 0, hcrow = 0, hccol = 0;
      if (threadIdx.y == 0 && tr.i0 >= 1 && jv) {
        hrole = 1;
        hi = tr.i0 - 1;
        hj = j;
        hcrow = tr.ox - 1;
        hccol = tr.oy + lane;
      } else if (threadIdx.y == 1 && lane < TR && tr.j0 >= 1 && tr.i0 + lane < tr.nx) {
        hrole = 2;
        hi = tr.i0 + lane;
        hj = tr.j0 - 1;
        hcrow = tr.ox + lane;
        hccol = tr.oy - 1;
      }
      T hah = T(0), hga0 = T(0), hga1 = T(0), hgb0 = T(0), hgb1 = T(0);
      int hmx = -1, hmy = -1;
      if (hrole) {
        const long long id = tr.base + (long long)(hi - tr.i0) * tr.pitch + (hj - tr.j0);
        hah = aHz[id];
        hga0 = gA[id];
        hga1 = hj + 1 < tr.ny ? gA[id + 1] : T(0);
        hgb0 = gB[id];
        hgb1 = hi + 1 < tr.nx ? gB[id + tr.pitch] : T(0);
        hmx = a.mhx[hcrow];
        hmy = a.mhy[hccol];
      }
      // ---- H transpose of the own cells
#pragma unroll
      for (int r = 0; r < R; ++r) {
        T h = T(0), ha = T(0), hb = T(0);
        if (jv && i + r < tr.nx) {
          adj_h_value<T>(a, I, i + r, j, tr.nx, tr.ny, tr.ox + r0 + r, tr.oy + lane, mxh[r], myh,
                         ah[r], ga0[r], ga1[r], gb[r], gb[r + 1], pzx, pzxo, pzy, pzyo, h, ha,
                         hb);
          aHzo[id0 + (long long)r * tr.pitch] = h;
        }
        sA[r0 + r + 1][lane + 1] = ha;
        sB[r0 + r + 1][lane + 1] = hb;
      }
      // ---- the halo cell, recomputed from the read level (psi not stored)
      {
        T h = T(0), ha = T(0), hb = T(0);
        if (hrole)
          adj_h_value<T>(a, I, hi, hj, tr.nx, tr.ny, hcrow, hccol, hmx, hmy, hah, hga0, hga1,
                         hgb0, hgb1, pzx, nullptr, pzy, nullptr, h, ha, hb);
        if (threadIdx.y == 0) sA[0][lane + 1] = hrole == 1 ? ha : T(0);
        if (threadIdx.y == 1 && lane < TR) sB[lane + 1][0] = hrole == 2 ? hb : T(0);
      }
      __syncthreads();
    }
    // ---- E adjoints: finish step n's (HT), then the E transpose of step m (ET)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!(jv && i + r < tr.nx)) break;
      const long long id = id0 + (long long)r * tr.pitch;
      T x = lx[r], y = ly[r];
      if (HT) {
        y = fma_rn(sub_rn(sA[r0 + r][lane + 1], sA[r0 + r + 1][lane + 1]), a.idx, y);
        x = fma_rn(sub_rn(sB[r0 + r + 1][lane], sB[r0 + r + 1][lane + 1]), a.idy, x);
      }
      if (ET) {
        if (i + r == I.line_i) {
          const double* ph = d.phase + m * d.n_freq * 2;
          const double* g = d.cot + (I.loff + j) * d.n_freq * 2;
          double sum = 0.0;
          for (int f = 0; f < d.n_freq; ++f)
            sum = __dadd_rn(sum, __dadd_rn(__dmul_rn(g[2 * f], ph[2 * f]),
                                           __dmul_rn(g[2 * f + 1], ph[2 * f + 1])));
          y = (T)__dadd_rn((double)y, __dmul_rn(d.dt, sum));
        }
        const int di = r0 + r - tr.wdi, dj = lane - tr.wdj;
        if (di >= 0 && di < tr.wdn && dj >= 0 && dj < tr.wdn) {
          const long long dc = I.goff + (long long)di * tr.wdn + dj;
          const T* rr = a.ring + ((m % a.ring_len) * a.n_design + dc) * 2;
          d.grad[dc] = __dadd_rn(d.grad[dc], __dadd_rn(__dmul_rn((double)x, (double)rr[0]),
                                                       __dmul_rn((double)y, (double)rr[1])));
        }
        T ga = T(0), gbv = T(0);
        if (j >= 1) {
          ga = mul_rn(K[r], x);
          if (mye >= 0) {
            const long long q = I.p_exy + (long long)(i + r) * I.npey + mye;
            const int c = tr.oy + lane;
            const T ap = fma_rn(K[r], x, d.aExy[q]);
            ga = fma_rn(a.cey[c], ap, ga);
            d.aExy[q] = mul_rn(a.bey[c], ap);
          }
        }
        if (i + r >= 1) {
          gbv = mul_rn(-K[r], y);
          if (mxe[r] >= 0) {
            const long long q = I.p_eyx + (long long)mxe[r] * tr.ny + j;
            const int c = tr.ox + r0 + r;
            const T ap = fma_rn(-K[r], y, d.aEyx[q]);
            gbv = fma_rn(a.cex[c], ap, gbv);
            d.aEyx[q] = mul_rn(a.bex[c], ap);
          }
        }
        gAo[id] = ga;
        gBo[id] = gbv;
      }
      d.aEx[id] = x;
      d.aEy[id] = y;
    }
    if (HT) __syncthreads();  // sA / sB are rewritten by the next tile
  }
}

// ---- marching reverse step ---------------------------------------------------
// kb_adj_step's work on kb_march's segments: one warp marches down its rows;
// gA of the column to the right comes from the lane above (lane 31 loads
// it), gB of the next row is loaded one row ahead, hA of the row above stays
// in a register, and hB of the column to the left comes from the lane below
// (lane 0 recomputes the halo column's H transpose without storing it). A
// segment that starts below row 0 first recomputes hA of row i0 - 1. Same
// levels and arithmetic as kb_adj_step, so the same bits.
template <typename T, bool HT, bool ET>
__global__ void __launch_bounds__(32 * kMarchWarps, PFB_MINB_AMARCH) kb_adj_march(
    const __grid_constant__ BArgs<T> a, const __grid_constant__ AArgs<T> d, int step_t) {
  const int w = blockIdx.x * kMarchWarps + threadIdx.y;
  if (w >= a.nsegs) return;  // uniform over the warp
  const SegRec sg = a.segs[w];
  const Inst& I = a.inst[sg.k];
  const long long n = *a.base + step_t;
  const long long m = HT ? n - 1 : n;  // the step of the E transpose
  const int lg = (int)(n & 1);
  const int lh = (int)((n + 1) & 1);
  const T* gA = d.gA2[lg];
  const T* gB = d.gB2[lg];
  T* gAo = d.gA2[(int)(m & 1)];
  T* gBo = d.gB2[(int)(m & 1)];
  const T* aHz = d.aHz2[lh];
  T* aHzo = d.aHz2[lh ^ 1];
  const T* pzx = d.aHzx2[lh];
  const T* pzy = d.aHzy2[lh];
  T* pzxo = d.aHzx2[lh ^ 1];
  T* pzyo = d.aHzy2[lh ^ 1];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  const int nx = I.nx, ny = I.ny;
  const long long pitch = I.pitch;
  const int j = sg.j0 - 1 + lane;
  const bool jv = j >= 0 && j < ny;
  const bool own = lane >= 1 && jv;
  const bool xr = HT && lane == 31 && j + 1 < ny;
  const long long c0 = I.off + j;
  const int myh = (HT && jv) ? a.mhy[I.oy + j] : -1;
  const int mye = (ET && jv) ? a.mey[I.oy + j] : -1;
  const int r_first = (HT && sg.i0 > 0) ? sg.i0 - 1 : sg.i0;
  // row r_first
  T ah = T(0), ga = T(0), ga31 = T(0), gb = T(0), gbn = T(0), lx = T(0), ly = T(0), K = T(0);
  {
    const long long id = c0 + r_first * pitch;
    if (jv) {
      if (HT) {
        ah = aHz[id];
        ga = gA[id];
        gb = gB[id];
        if (r_first + 1 < nx) gbn = gB[id + pitch];
      }
      if (r_first >= sg.i0) {
        lx = d.aEx[id];
        ly = d.aEy[id];
        if (ET) K = a.ce[id];
      }
    }
    if (xr) ga31 = gA[id + 1];
  }
  T ha_prev = T(0);  // hA of the row above
  for (int r = r_first; r < sg.i1; ++r) {
    const int r1 = r + 1;
    T ah_n = T(0), ga_n = T(0), ga31_n = T(0), gbn_n = T(0), lx_n = T(0), ly_n = T(0), K_n = T(0);
    if (r1 < sg.i1) {
      const long long id = c0 + r1 * pitch;
      if (jv) {
        if (HT) {
          ah_n = aHz[id];
          ga_n = gA[id];
          if (r1 + 1 < nx) gbn_n = gB[id + pitch];
        }
        lx_n = d.aEx[id];
        ly_n = d.aEy[id];
        if (ET) K_n = a.ce[id];
      }
      if (xr) ga31_n = gA[id + 1];
    }
    const long long id = c0 + r * pitch;
    const bool body = r >= sg.i0;  // uniform
    T ha = T(0), hb = T(0);
    if (HT) {
      T ga1 = __shfl_down_sync(full, ga, 1);
      if (lane == 31) ga1 = ga31;
      T h = T(0);
      if (jv) {
        const bool st = own && body;
        adj_h_value<T>(a, I, r, j, nx, ny, I.ox + r, I.oy + j, a.mhx[I.ox + r], myh, ah, ga,
                       ga1, gb, gbn, pzx, st ? pzxo : nullptr, pzy, st ? pzyo : nullptr, h, ha,
                       hb);
        if (st) aHzo[id] = h;
      }
    }
    const T hbl = HT ? __shfl_up_sync(full, hb, 1) : T(0);  // hB of column j - 1
    if (body && own) {
      T x = lx, y = ly;
      if (HT) {
        y = fma_rn(sub_rn(ha_prev, ha), a.idx, y);
        x = fma_rn(sub_rn(hbl, hb), a.idy, x);
      }
      if (ET) {
        if (r == I.line_i) {
          const double* ph = d.phase + m * d.n_freq * 2;
          const double* g = d.cot + (I.loff + j) * d.n_freq * 2;
          double sum = 0.0;
          for (int f = 0; f < d.n_freq; ++f)
            sum = __dadd_rn(sum, __dadd_rn(__dmul_rn(g[2 * f], ph[2 * f]),
                                           __dmul_rn(g[2 * f + 1], ph[2 * f + 1])));
          y = (T)__dadd_rn((double)y, __dmul_rn(d.dt, sum));
        }
        const int di = r - I.di0, dj = j - I.dj0;
        if (di >= 0 && di < I.dn && dj >= 0 && dj < I.dn) {
          const long long dc = I.goff + (long long)di * I.dn + dj;
          const T* rr = a.ring + ((m % a.ring_len) * a.n_design + dc) * 2;
          d.grad[dc] = __dadd_rn(d.grad[dc], __dadd_rn(__dmul_rn((double)x, (double)rr[0]),
                                                       __dmul_rn((double)y, (double)rr[1])));
        }
        T gav = T(0), gbv = T(0);
        if (j >= 1) {
          gav = mul_rn(K, x);
          if (mye >= 0) {
            const long long q = I.p_exy + (long long)r * I.npey + mye;
            const int c = I.oy + j;
            const T ap = fma_rn(K, x, d.aExy[q]);
            gav = fma_rn(a.cey[c], ap, gav);
            d.aExy[q] = mul_rn(a.bey[c], ap);
          }
        }
        if (r >= 1) {
          gbv = mul_rn(-K, y);
          const int mx = a.mex[I.ox + r];
          if (mx >= 0) {
            const long long q = I.p_eyx + (long long)mx * ny + j;
            const int c = I.ox + r;
            const T ap = fma_rn(-K, y, d.aEyx[q]);
            gbv = fma_rn(a.cex[c], ap, gbv);
            d.aEyx[q] = mul_rn(a.bex[c], ap);
          }
        }
        gAo[id] = gav;
        gBo[id] = gbv;
      }
      d.aEx[id] = x;
      d.aEy[id] = y;
    }
    ha_prev = ha;
    ah = ah_n;
    ga = ga_n;
    ga31 = ga31_n;
    gb = gbn;
    gbn = gbn_n;
    lx = lx_n;
    ly = ly_n;
    K = K_n;
  }
}

}  // namespace b2d
}  // namespace pfb
