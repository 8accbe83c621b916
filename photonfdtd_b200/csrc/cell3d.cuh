// cell3d.cuh - per-cell H and E updates for 3D grids off the bulk path.
//
// For cells in CPML slabs or on a domain face of a 3D grid (every axis
// resolved). Same operations in the same order as curl_term (the
// reference's bulk term, then the CPML correction of each term where its
// coefficient c != 0, simulation.py:1284-1309), organised for a short
// instruction stream: the six divisions of a cell share one range check, a
// component outside the reference's loop extents keeps its old value, and
// psi state is touched only where the per-axis compact map is >= 0.
#pragma once

#include "cell_update.cuh"

namespace pfb {

// Six quotients n[t] / d[ax[t]], exact: the fast reciprocal path when every
// numerator is in its range, IEEE division otherwise.
template <typename T>
__device__ __forceinline__ void divide6(const StepArgs<T>& a, const T n[6], const int ax[6], T q[6]) {
  const T dl[3] = {a.dx, a.dy, a.dz};
  const T rl[3] = {a.rdx, a.rdy, a.rdz};
  const bool fl[3] = {a.fdx, a.fdy, a.fdz};
  const T m = absmax(absmax(n[0], n[1]), absmax(absmax(n[2], n[3]), absmax(n[4], n[5])));
  if (a.fdx && a.fdy && a.fdz && qdiv_ok(m)) {
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = qdiv_fast(n[t], dl[ax[t]], rl[ax[t]]);
  } else {
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = qdiv(n[t], dl[ax[t]], rl[ax[t]], fl[ax[t]]);
  }
}

// psi element of a term on axis AX at (i, j, k) whose axis index maps to m.
template <int AX>
__device__ __forceinline__ int psi_at(int m, int i, int j, int k, int ny, int nz, int np) {
  if (AX == 0) return (m * ny + j) * nz + k;
  if (AX == 1) return (i * np + m) * nz + k;
  return (i * ny + j) * np + m;
}

// f + k*(dA - dB), then psiA (+k) and psiB (-k) corrections where present.
template <typename T, int AXA, int AXB>
__device__ __forceinline__ T curl3(T f, T k, T dA, T dB, int mA, int mB, int i, int j, int k_,
                                   int ny, int nz, const int* np, const T* bA, const T* cA,
                                   const T* bB, const T* cB, const T* psiAin, T* psiAout,
                                   const T* psiBin, T* psiBout, bool write_psi) {
  f = add_rn(f, mul_rn(sub_rn(dA, dB), k));
  const int pos[3] = {i, j, k_};
  if (mA >= 0) {
    const int q = psi_at<AXA>(mA, i, j, k_, ny, nz, np[AXA]);
    const T psi = add_rn(mul_rn(bA[pos[AXA]], psiAin[q]), mul_rn(cA[pos[AXA]], dA));
    if (write_psi) psiAout[q] = psi;
    f = add_rn(f, mul_rn(k, psi));
  }
  if (mB >= 0) {
    const int q = psi_at<AXB>(mB, i, j, k_, ny, nz, np[AXB]);
    const T psi = add_rn(mul_rn(bB[pos[AXB]], psiBin[q]), mul_rn(cB[pos[AXB]], dB));
    if (write_psi) psiBout[q] = psi;
    f = add_rn(f, mul_rn(-k, psi));
  }
  return f;
}

// H^{n+1/2} at (i, j, k) of a 3D grid. n = forward-difference numerators in
// the order Hx (dEz along y, dEy along z), Hy (dEx along z, dEz along x),
// Hz (dEy along x, dEx along y); entries whose neighbour is outside the grid
// are ignored.
template <typename T>
__device__ __forceinline__ void h3(const StepArgs<T>& a, int i, int j, int k, const T hold[3],
                                   const T n[6], bool write_psi, T h[3]) {
  const int ax[6] = {1, 2, 2, 0, 0, 1};
  T d[6];
  divide6<T>(a, n, ax, d);
  const bool fx = i < a.nx - 1, fy = j < a.ny - 1, fz = k < a.nz - 1;
  const int mx = a.maph[0][i], my = a.maph[1][j], mz = a.maph[2][k];
  const T mch = -a.ch;
  h[0] = (fy && fz) ? curl3<T, 1, 2>(hold[0], mch, d[0], d[1], my, mz, i, j, k, a.ny, a.nz, a.nph,
                                     a.bh[1], a.cph[1], a.bh[2], a.cph[2], a.psiHin[0],
                                     a.psiHout[0], a.psiHin[1], a.psiHout[1], write_psi)
                    : hold[0];
  h[1] = (fz && fx) ? curl3<T, 2, 0>(hold[1], mch, d[2], d[3], mz, mx, i, j, k, a.ny, a.nz, a.nph,
                                     a.bh[2], a.cph[2], a.bh[0], a.cph[0], a.psiHin[2],
                                     a.psiHout[2], a.psiHin[3], a.psiHout[3], write_psi)
                    : hold[1];
  h[2] = (fx && fy) ? curl3<T, 0, 1>(hold[2], mch, d[4], d[5], mx, my, i, j, k, a.ny, a.nz, a.nph,
                                     a.bh[0], a.cph[0], a.bh[1], a.cph[1], a.psiHin[4],
                                     a.psiHout[4], a.psiHin[5], a.psiHout[5], write_psi)
                    : hold[2];
}

// E^{n+1} (before ADE) at (i, j, k) of a 3D grid. n = backward-difference
// numerators: Ex (dHz along y, dHy along z), Ey (dHx along z, dHz along x),
// Ez (dHy along x, dHx along y).
template <typename T>
__device__ __forceinline__ void e3(const StepArgs<T>& a, int i, int j, int k, const T eold[3],
                                   const T K[3], const T n[6], T e[3]) {
  const int ax[6] = {1, 2, 2, 0, 0, 1};
  T d[6];
  divide6<T>(a, n, ax, d);
  const bool bx = i >= 1, by = j >= 1, bz = k >= 1;
  const int mx = a.mape[0][i], my = a.mape[1][j], mz = a.mape[2][k];
  e[0] = (by && bz) ? curl3<T, 1, 2>(eold[0], K[0], d[0], d[1], my, mz, i, j, k, a.ny, a.nz, a.npe,
                                     a.be[1], a.cpe[1], a.be[2], a.cpe[2], a.psiE[0], a.psiE[0],
                                     a.psiE[1], a.psiE[1], true)
                    : eold[0];
  e[1] = (bz && bx) ? curl3<T, 2, 0>(eold[1], K[1], d[2], d[3], mz, mx, i, j, k, a.ny, a.nz, a.npe,
                                     a.be[2], a.cpe[2], a.be[0], a.cpe[0], a.psiE[2], a.psiE[2],
                                     a.psiE[3], a.psiE[3], true)
                    : eold[1];
  e[2] = (bx && by) ? curl3<T, 0, 1>(eold[2], K[2], d[4], d[5], mx, my, i, j, k, a.ny, a.nz, a.npe,
                                     a.be[0], a.cpe[0], a.be[1], a.cpe[1], a.psiE[4], a.psiE[4],
                                     a.psiE[5], a.psiE[5], true)
                    : eold[2];
}

}  // namespace pfb
