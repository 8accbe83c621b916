// kernels_split.cuh - one-thread-per-cell H and E passes for any grid shape.
//
// The split path covers every case the reference covers (1D, 2D in any
// plane, 3D; collapsed axes drop their curl terms) and is the baseline the
// fused 3D kernel is checked against bit for bit. The per-component
// arithmetic lives in cell_update.cuh and is shared with the fused kernel.
// Update order per component (src/photonfdtd/simulation.py:1252-1309):
//   curl = dA - dB (or dA, or -dB when one axis is collapsed)
//   F   += K * curl                          (bulk)
//   psiA = bA*psiA + cA*dA ; F += (+K)*psiA   (only where cA != 0)
//   psiB = bB*psiB + cB*dB ; F += (-K)*psiB   (only where cB != 0)
// with d = (a_hi - a_lo) / dl and K = ce (E) or -ch (H).
//
// A block whose cells all lie in the bulk box (both difference terms, no
// CPML state) takes a straight-line path: the same operations with no
// extent checks, psi lookups or coefficient loads.
#pragma once

#include "cell3d.cuh"

// Minimum resident 256-thread blocks per SM the split passes are compiled
// for (register budget 65536 / (256 * n)). Measured on config 3 (384^3 ADE):
// H at 8 (32 registers, a 12-byte spill) and E at 5 (48 registers) give
// 1.52 ms of step kernels against 1.77 ms at the compiler's choice (48 / 59
// registers); E at 6 spills 28 bytes and is slower.
#ifndef PFB_MINB_H
#define PFB_MINB_H 8
#endif
#ifndef PFB_MINB_E
#define PFB_MINB_E 5
#endif

namespace pfb {

// Load f[id + off] only when the neighbour exists (cond), else 0.
template <typename T>
__device__ __forceinline__ T ld_if(const T* f, long long id, long long off, bool cond) {
  return cond ? f[id + off] : T(0);
}

// Three curl updates sharing one magnitude check of their six numerators:
// out[c] = f[c] + K[c] * (n[2c]/d[2c] - n[2c+1]/d[2c+1]), the divisors in
// axis order ax[0..5]. The fast exact division applies when every numerator
// is within its range, otherwise each division is IEEE.
template <typename T>
__device__ __forceinline__ void bulk3(const StepArgs<T>& a, const T f[3], const T K[3],
                                      const T n[6], const int ax[6], T out[3]) {
  const T dl[3] = {a.dx, a.dy, a.dz};
  const T rl[3] = {a.rdx, a.rdy, a.rdz};
  const bool fl[3] = {a.fdx, a.fdy, a.fdz};
  const T m = absmax(absmax(n[0], n[1]), absmax(absmax(n[2], n[3]), absmax(n[4], n[5])));
  T q[6];
  if (a.fdx && a.fdy && a.fdz && qdiv_ok(m)) {
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = qdiv_fast(n[t], dl[ax[t]], rl[ax[t]]);
  } else {
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = qdiv(n[t], dl[ax[t]], rl[ax[t]], fl[ax[t]]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = bulk(f[c], K[c], q[2 * c], q[2 * c + 1]);
}

__device__ __forceinline__ bool in_box(int i, int j0, int j1, int k0, int k1, const int* b0,
                                       const int* b1) {
  return i >= b0[0] && i < b1[0] && j0 >= b0[1] && j1 <= b1[1] && k0 >= b0[2] && k1 <= b1[2];
}

// H pass: H^{n+1/2} = H^{n-1/2} - ch (curl E^n + psi). One cell; `box`:
// the cell's block lies in the bulk box.
template <typename T>
__device__ __forceinline__ void h_cell(const StepArgs<T>& a, int i, int j, int k, bool box) {
  const long long sy = a.nz, sx = (long long)a.ny * a.nz;
  const long long id = i * sx + j * sy + k;
  const T ex = a.Ein[0][id], ey = a.Ein[1][id], ez = a.Ein[2][id];
  if (box) {
    const T f[3] = {a.Hin[0][id], a.Hin[1][id], a.Hin[2][id]};
    const T mch = -a.ch;
    const T K[3] = {mch, mch, mch};
    // Hx: +dEz/dy - dEy/dz; Hy: +dEx/dz - dEz/dx; Hz: +dEy/dx - dEx/dy
    const T n[6] = {sub_rn(a.Ein[2][id + sy], ez), sub_rn(a.Ein[1][id + 1], ey),
                    sub_rn(a.Ein[0][id + 1], ex), sub_rn(a.Ein[2][id + sx], ez),
                    sub_rn(a.Ein[1][id + sx], ey), sub_rn(a.Ein[0][id + sy], ex)};
    const int ax[6] = {1, 2, 2, 0, 0, 1};
    T h[3];
    bulk3<T>(a, f, K, n, ax, h);
    a.Hout[0][id] = h[0];
    a.Hout[1][id] = h[1];
    a.Hout[2][id] = h[2];
    return;
  }
  const bool hx = i + 1 < a.nx, hy = j + 1 < a.ny, hz = k + 1 < a.nz;
  if (a.nx > 1 && a.ny > 1 && a.nz > 1) {
    const T hold[3] = {a.Hin[0][id], a.Hin[1][id], a.Hin[2][id]};
    const T n[6] = {sub_rn(ld_if(a.Ein[2], id, sy, hy), ez), sub_rn(ld_if(a.Ein[1], id, 1, hz), ey),
                    sub_rn(ld_if(a.Ein[0], id, 1, hz), ex), sub_rn(ld_if(a.Ein[2], id, sx, hx), ez),
                    sub_rn(ld_if(a.Ein[1], id, sx, hx), ey), sub_rn(ld_if(a.Ein[0], id, sy, hy), ex)};
    T h[3];
    h3<T>(a, i, j, k, hold, n, true, h);
    a.Hout[0][id] = h[0];
    a.Hout[1][id] = h[1];
    a.Hout[2][id] = h[2];
    return;
  }
  a.Hout[0][id] = upd_hx<T>(a, i, j, k, a.Hin[0][id], ld_if(a.Ein[2], id, sy, hy), ez,
                            ld_if(a.Ein[1], id, 1, hz), ey, true);
  a.Hout[1][id] = upd_hy<T>(a, i, j, k, a.Hin[1][id], ld_if(a.Ein[0], id, 1, hz), ex,
                            ld_if(a.Ein[2], id, sx, hx), ez, true);
  a.Hout[2][id] = upd_hz<T>(a, i, j, k, a.Hin[2][id], ld_if(a.Ein[1], id, sx, hx), ey,
                            ld_if(a.Ein[0], id, sy, hy), ex, true);
}

template <typename T>
__global__ void __launch_bounds__(256, PFB_MINB_H) k_h_split(const __grid_constant__ StepArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const bool box = in_box(i, blockIdx.y * blockDim.y, (blockIdx.y + 1) * blockDim.y,
                          blockIdx.x * blockDim.x, (blockIdx.x + 1) * blockDim.x, a.hb0, a.hb1);
  if (k >= a.nz || j >= a.ny) return;
  h_cell<T>(a, i, j, k, box);
}

// The E pass's epilogue, after the curl and ADE updates of cell (i, j, k):
// the E-family soft sources of the cell, each group's sources added in list
// order in double and rounded once (k_inject's arithmetic), then the cell's
// samples for the DFT monitors sampled this step (E after the sources, H
// at n + 1/2: the values k_dft_sample reads after the step).
template <typename T>
__device__ __forceinline__ void e_epilogue(const StepArgs<T>& a, const EpiArgs<T>& ep, int i,
                                           int j, int k, long long id, T e[3]) {
  if (ep.n_isrc) {
    const int blk = (int)((blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
    const int tid = (int)(threadIdx.y * blockDim.x + threadIdx.x);
    for (int g = 0; g < ep.n_isrc; ++g) {
      if (blk != ep.isrc_blk[g] || tid != ep.isrc_tid[g]) continue;
      const SourceGroups& s = ep.isrc;
      const int c = s.comp[g];
      T v = e[c];
      for (int q = s.start[g]; q < s.start[g + 1]; ++q)
        v = add_double<T>(v, __dmul_rn(s.amp[q],
                                       s.wave[(long long)s.wave_row[q] * s.n_steps + ep.step]));
      e[c] = v;
    }
  }
  for (int m = 0; m < ep.n_idft; ++m) {
    if (ep.idft_slot[m] < 0) continue;
    const DftRegion& r = ep.idft[m];
    // the bounding box first (unsigned: below start wraps high); the
    // divisions only for cells inside it on a strided axis
    const unsigned di = (unsigned)(i - r.start[0]), dj = (unsigned)(j - r.start[1]),
                   dk = (unsigned)(k - r.start[2]);
    if (di >= (unsigned)((r.count[0] - 1) * r.stride[0] + 1) ||
        dj >= (unsigned)((r.count[1] - 1) * r.stride[1] + 1) ||
        dk >= (unsigned)((r.count[2] - 1) * r.stride[2] + 1))
      continue;
    int ci = (int)di, cj = (int)dj, ck = (int)dk;
    if (r.stride[0] > 1 || r.stride[1] > 1 || r.stride[2] > 1) {
      if (di % r.stride[0] || dj % r.stride[1] || dk % r.stride[2]) continue;
      ci = (int)di / r.stride[0];
      cj = (int)dj / r.stride[1];
      ck = (int)dk / r.stride[2];
      if (ci >= r.count[0] || cj >= r.count[1] || ck >= r.count[2]) continue;
    }
    const long long cell = ((long long)ci * r.count[1] + cj) * r.count[2] + ck;
    T* ring = ep.idft_ring[m] + (long long)ep.idft_slot[m] * r.ncomp * r.ncell;
    for (int q = 0; q < r.ncomp; ++q) {
      // H is reloaded here (a cache hit) rather than kept live through the
      // update for the few cells that sample it
      const int c = r.comps[q];
      ring[(long long)q * r.ncell + cell] = c < 3 ? e[c] : a.Hin[c - 3][id];
    }
  }
}

// Whether block (blockIdx) holds a source cell of this step or cells of a
// DFT region sampled at this step (uniform over the block), so that every
// other block skips the epilogue after one test.
template <typename T>
__device__ __forceinline__ bool epilogue_block(const EpiArgs<T>& a) {
  if (a.n_isrc) {
    const int blk = (int)((blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
    for (int g = 0; g < a.n_isrc; ++g)
      if (blk == a.isrc_blk[g]) return true;
  }
  const int i = blockIdx.z;
  const int j0 = blockIdx.y * blockDim.y, j1 = j0 + blockDim.y;
  const int k0 = blockIdx.x * blockDim.x, k1 = k0 + blockDim.x;
  for (int m = 0; m < a.n_idft; ++m) {
    if (a.idft_slot[m] < 0) continue;
    const DftRegion& r = a.idft[m];
    const int hi0 = r.start[0] + (r.count[0] - 1) * r.stride[0] + 1;
    const int hi1 = r.start[1] + (r.count[1] - 1) * r.stride[1] + 1;
    const int hi2 = r.start[2] + (r.count[2] - 1) * r.stride[2] + 1;
    if (i >= r.start[0] && i < hi0 && j1 > r.start[1] && j0 < hi1 && k1 > r.start[2] && k0 < hi2)
      return true;
  }
  return false;
}

// E pass: E^{n+1} = E^n + ce (curl H^{n+1/2} + psi), then ADE; with EPI the
// epilogue above (a separate instantiation: the plain pass carries none of
// its code).
template <typename T, int CE, bool ADE, bool EPI>
__global__ void __launch_bounds__(256, PFB_MINB_E)
    k_e_split(const __grid_constant__ StepArgs<T> a,
              const __grid_constant__ typename EpiParam<T, EPI>::type ep) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const bool box = in_box(i, blockIdx.y * blockDim.y, (blockIdx.y + 1) * blockDim.y,
                          blockIdx.x * blockDim.x, (blockIdx.x + 1) * blockDim.x, a.eb0, a.eb1);
  const MediumT<T>* media = a.media;
  bool epi = false;
  if constexpr (EPI) epi = (ep.n_isrc || ep.n_idft) && epilogue_block<T>(ep);
  if (k >= a.nz || j >= a.ny) return;
  const long long sy = a.nz, sx = (long long)a.ny * a.nz;
  const long long id = i * sx + j * sy + k;
  // Loads are issued in dependency order: the per-cell word and every field
  // value first, then what the word selects (table coefficient, ADE record),
  // so a warp waits out two memory latencies, not three.
  T K[3];
  uint32_t t, w;
  cell_word<T, CE, ADE>(a, id, K, t);
  const T hx = a.Hin[0][id], hy = a.Hin[1][id], hz = a.Hin[2][id];
  T en[3] = {a.Ein[0][id], a.Ein[1][id], a.Ein[2][id]};
  const bool d3 = a.nx > 1 && a.ny > 1 && a.nz > 1;
  T hn[6];  // Hz(j-1), Hy(k-1), Hx(k-1), Hz(i-1), Hy(i-1), Hx(j-1); 3D grids only
  if (box) {
    hn[0] = a.Hin[2][id - sy];
    hn[1] = a.Hin[1][id - 1];
    hn[2] = a.Hin[0][id - 1];
    hn[3] = a.Hin[2][id - sx];
    hn[4] = a.Hin[1][id - sx];
    hn[5] = a.Hin[0][id - sy];
  } else if (d3) {
    const bool lx = i > 0, ly = j > 0, lz = k > 0;
    hn[0] = ld_if(a.Hin[2], id, -sy, ly);
    hn[1] = ld_if(a.Hin[1], id, -1, lz);
    hn[2] = ld_if(a.Hin[0], id, -1, lz);
    hn[3] = ld_if(a.Hin[2], id, -sx, lx);
    hn[4] = ld_if(a.Hin[1], id, -sx, lx);
    hn[5] = ld_if(a.Hin[0], id, -sy, ly);
  }
  cell_decode<T, CE, ADE>(a, media, t, K, w);
  AdeRec<T> rec;
  if (ADE && w) ade_load<T>(a, media, w, rec);
  T e[3];
  if (box || d3) {
    // Ex: +dHz/dy - dHy/dz; Ey: +dHx/dz - dHz/dx; Ez: +dHy/dx - dHx/dy
    const T n[6] = {sub_rn(hz, hn[0]), sub_rn(hy, hn[1]), sub_rn(hx, hn[2]),
                    sub_rn(hz, hn[3]), sub_rn(hy, hn[4]), sub_rn(hx, hn[5])};
    if (box) {
      const int ax[6] = {1, 2, 2, 0, 0, 1};
      bulk3<T>(a, en, K, n, ax, e);
    } else {
      e3<T>(a, i, j, k, en, K, n, e);
    }
  } else {
    const bool lx = i > 0, ly = j > 0, lz = k > 0;
    e[0] = upd_ex<T>(a, i, j, k, en[0], K[0], hz, ld_if(a.Hin[2], id, -sy, ly), hy,
                     ld_if(a.Hin[1], id, -1, lz));
    e[1] = upd_ey<T>(a, i, j, k, en[1], K[1], hx, ld_if(a.Hin[0], id, -1, lz), hz,
                     ld_if(a.Hin[2], id, -sx, lx));
    e[2] = upd_ez<T>(a, i, j, k, en[2], K[2], hy, ld_if(a.Hin[1], id, -sx, lx), hx,
                     ld_if(a.Hin[0], id, -sy, ly));
  }
  if (ADE && w) ade_update<T>(a, media, rec, en, e);
  if constexpr (EPI) {
    if (epi) e_epilogue<T>(a, ep, i, j, k, id, e);
  }
  a.Eout[0][id] = e[0];
  a.Eout[1][id] = e[1];
  a.Eout[2][id] = e[2];
}

}  // namespace pfb
