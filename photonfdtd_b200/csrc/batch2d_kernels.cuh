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

template <typename T>
struct BArgs {
  const Inst* inst;
  const TileRec* tiles;
  int ntiles;
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
__global__ void kb_post(BSources s, T* Ex, T* Ey, T* Hz, int family_h, const long long* base,
                        int step_t, const long long* lcell, long long nline, T* dring) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < s.n_groups) {
    const int c = s.comp[g];
    if ((c == 2) != (family_h != 0)) return;
    T* F = c == 0 ? Ex : (c == 1 ? Ey : Hz);
    const long long n = *base + step_t;
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

}  // namespace b2d
}  // namespace pfb
