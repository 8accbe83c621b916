// kernels_split.cuh - one-thread-per-cell H and E passes for any grid shape.
//
// The split path covers every case the reference covers (1D, 2D in any
// plane, 3D; collapsed axes drop their curl terms) and is the bit-exact
// baseline the fused 3D kernel is checked against. Update order per
// component follows src/photonfdtd/simulation.py:1252-1309:
//   curl = dA - dB (or dA, or -dB when one axis is collapsed)
//   F   += K * curl                      (bulk)
//   psiA = bA*psiA + cA*dA ; F += (+K)*psiA   (only where cA != 0)
//   psiB = bB*psiB + cB*dB ; F += (-K)*psiB   (only where cB != 0)
// with d = (a_hi - a_lo) / dl, K = ce (E) or -ch (H). The loop extents are
// the reference's crops: forward differences stop one cell short of the high
// face, backward differences start at index 1 (simulation.py:1180-1199).
#pragma once

#include "common.cuh"

namespace pfb {

// One curl component: bulk update plus the two CPML corrections.
// hasA/hasB: the term's axis is resolved; inA/inB: compact psi index or -1.
template <typename T>
__device__ __forceinline__ T curl_update(T f, T k, bool hasA, T dA, bool hasB, T dB,
                                         long long qA, T bA, T cA, const T* psiAin,
                                         T* psiAout, long long qB, T bB, T cB,
                                         const T* psiBin, T* psiBout) {
  T curl = hasA ? (hasB ? sub_rn(dA, dB) : dA) : -dB;
  f = add_rn(f, mul_rn(curl, k));
  if (hasA && qA >= 0) {
    T psi = add_rn(mul_rn(bA, psiAin[qA]), mul_rn(cA, dA));
    psiAout[qA] = psi;
    f = add_rn(f, mul_rn(k, psi));
  }
  if (hasB && qB >= 0) {
    T psi = add_rn(mul_rn(bB, psiBin[qB]), mul_rn(cB, dB));
    psiBout[qB] = psi;
    f = add_rn(f, mul_rn(-k, psi));
  }
  return f;
}

// H pass: H^{n+1/2} = H^{n-1/2} - ch (curl E^n + psi), forward differences.
template <typename T>
__global__ void __launch_bounds__(256) k_h_split(const __grid_constant__ StepArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long sy = nz, sx = (long long)ny * nz;
  const long long id = i * sx + j * sy + k;
  const bool rx = nx > 1, ry = ny > 1, rz = nz > 1;
  const T mch = -a.ch;
  const bool ix = !rx || i < nx - 1, iy = !ry || j < ny - 1, iz = !rz || k < nz - 1;

  // Hx at (i, j+1/2, k+1/2): +dEz/dy, -dEy/dz
  {
    T h = a.Hin[0][id];
    if (iy && iz && (ry || rz)) {
      T dA = 0, dB = 0;
      long long qA = -1, qB = -1;
      if (ry) {
        dA = div_rn(sub_rn(a.Ein[2][id + sy], a.Ein[2][id]), a.dy);
        int m = a.maph[1][j];
        if (m >= 0) qA = ((long long)i * a.nph[1] + m) * nz + k;
      }
      if (rz) {
        dB = div_rn(sub_rn(a.Ein[1][id + 1], a.Ein[1][id]), a.dz);
        int m = a.maph[2][k];
        if (m >= 0) qB = ((long long)i * ny + j) * a.nph[2] + m;
      }
      h = curl_update<T>(h, mch, ry, dA, rz, dB, qA, ry ? a.bh[1][j] : T(0),
                         ry ? a.cph[1][j] : T(0), a.psiHin[0], a.psiHout[0], qB,
                         rz ? a.bh[2][k] : T(0), rz ? a.cph[2][k] : T(0), a.psiHin[1],
                         a.psiHout[1]);
    }
    a.Hout[0][id] = h;
  }
  // Hy at (i+1/2, j, k+1/2): +dEx/dz, -dEz/dx
  {
    T h = a.Hin[1][id];
    if (iz && ix && (rz || rx)) {
      T dA = 0, dB = 0;
      long long qA = -1, qB = -1;
      if (rz) {
        dA = div_rn(sub_rn(a.Ein[0][id + 1], a.Ein[0][id]), a.dz);
        int m = a.maph[2][k];
        if (m >= 0) qA = ((long long)i * ny + j) * a.nph[2] + m;
      }
      if (rx) {
        dB = div_rn(sub_rn(a.Ein[2][id + sx], a.Ein[2][id]), a.dx);
        int m = a.maph[0][i];
        if (m >= 0) qB = ((long long)m * ny + j) * nz + k;
      }
      h = curl_update<T>(h, mch, rz, dA, rx, dB, qA, rz ? a.bh[2][k] : T(0),
                         rz ? a.cph[2][k] : T(0), a.psiHin[2], a.psiHout[2], qB,
                         rx ? a.bh[0][i] : T(0), rx ? a.cph[0][i] : T(0), a.psiHin[3],
                         a.psiHout[3]);
    }
    a.Hout[1][id] = h;
  }
  // Hz at (i+1/2, j+1/2, k): +dEy/dx, -dEx/dy
  {
    T h = a.Hin[2][id];
    if (ix && iy && (rx || ry)) {
      T dA = 0, dB = 0;
      long long qA = -1, qB = -1;
      if (rx) {
        dA = div_rn(sub_rn(a.Ein[1][id + sx], a.Ein[1][id]), a.dx);
        int m = a.maph[0][i];
        if (m >= 0) qA = ((long long)m * ny + j) * nz + k;
      }
      if (ry) {
        dB = div_rn(sub_rn(a.Ein[0][id + sy], a.Ein[0][id]), a.dy);
        int m = a.maph[1][j];
        if (m >= 0) qB = ((long long)i * a.nph[1] + m) * nz + k;
      }
      h = curl_update<T>(h, mch, rx, dA, ry, dB, qA, rx ? a.bh[0][i] : T(0),
                         rx ? a.cph[0][i] : T(0), a.psiHin[4], a.psiHout[4], qB,
                         ry ? a.bh[1][j] : T(0), ry ? a.cph[1][j] : T(0), a.psiHin[5],
                         a.psiHout[5]);
    }
    a.Hout[2][id] = h;
  }
}

// Locate the medium of compact dispersive index g (media sorted by base).
template <typename T>
__device__ __forceinline__ int find_medium(const MediumT<T>* media, int n, long long g) {
  int m = 0;
  for (int q = 1; q < n; ++q)
    if (g >= media[q].base) m = q;
  return m;
}

// ADE polarisation update and E correction for one dispersive cell
// (simulation.py:645-669): P^{n+1} = a P^n + b P^{n-1} + c E^n per pole and
// component, E -= inv * sum_p (P^{n+1} - P^n). P^{n+1} overwrites P^{n-1}.
template <typename T>
__device__ __forceinline__ void ade_apply(const StepArgs<T>& a, long long g, const T en[3],
                                          T e[3]) {
  const int m = find_medium(a.media, a.n_media, g);
  const MediumT<T>& M = a.media[m];
  const long long loc = g - M.base, cnt = M.count;
  T* P = a.P + M.poff;
  const int np = M.npole;
  const int lc = a.lvl, lp = a.lvl ^ 1;
  for (int c = 0; c < 3; ++c) {
    T delta = T(0);
    for (int p = 0; p < np; ++p) {
      const long long ic = ((long long)(lc * np + p) * 3 + c) * cnt + loc;
      const long long ip = ((long long)(lp * np + p) * 3 + c) * cnt + loc;
      const T pc = P[ic], pp = P[ip];
      const T pn = add_rn(add_rn(mul_rn(M.a[p], pc), mul_rn(M.b[p], pp)), mul_rn(M.c[p], en[c]));
      P[ip] = pn;
      const T inc = sub_rn(pn, pc);
      delta = p == 0 ? inc : add_rn(delta, inc);
    }
    if (np > 0) e[c] = sub_rn(e[c], mul_rn(M.inv, delta));
  }
}

// E pass: E^{n+1} = E^n + ce (curl H^{n+1/2} + psi), backward differences,
// then the ADE correction on dispersive cells.
template <typename T, int CE, bool ADE>
__global__ void __launch_bounds__(256) k_e_split(const __grid_constant__ StepArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long sy = nz, sx = (long long)ny * nz;
  const long long id = i * sx + j * sy + k;
  const bool rx = nx > 1, ry = ny > 1, rz = nz > 1;
  const bool ix = !rx || i >= 1, iy = !ry || j >= 1, iz = !rz || k >= 1;

  T K[3];
  long long g = -1;
  if (CE == kCeCell1) {
    K[0] = K[1] = K[2] = a.ce[0][id];
  } else if (CE == kCeCell3) {
    K[0] = a.ce[0][id];
    K[1] = a.ce[1][id];
    K[2] = a.ce[2][id];
  } else {
    const uint32_t w = a.word[id];
    if (w & kDispersiveBit) {
      g = (long long)(w & ~kDispersiveBit);
      K[0] = K[1] = K[2] = a.media[find_medium(a.media, a.n_media, g)].ce;
    } else {
      K[0] = K[1] = K[2] = a.table[w];
    }
  }
  if (ADE && CE == kCeCell1) {
    const uint32_t w = a.adeword[id];
    if (w) g = (long long)w - 1;
  }

  T en[3] = {a.Ein[0][id], a.Ein[1][id], a.Ein[2][id]};
  T e[3] = {en[0], en[1], en[2]};

  // Ex at (i+1/2, j, k): +dHz/dy, -dHy/dz
  if (iy && iz && (ry || rz)) {
    T dA = 0, dB = 0;
    long long qA = -1, qB = -1;
    if (ry) {
      dA = div_rn(sub_rn(a.Hin[2][id], a.Hin[2][id - sy]), a.dy);
      int m = a.mape[1][j];
      if (m >= 0) qA = ((long long)i * a.npe[1] + m) * nz + k;
    }
    if (rz) {
      dB = div_rn(sub_rn(a.Hin[1][id], a.Hin[1][id - 1]), a.dz);
      int m = a.mape[2][k];
      if (m >= 0) qB = ((long long)i * ny + j) * a.npe[2] + m;
    }
    e[0] = curl_update<T>(e[0], K[0], ry, dA, rz, dB, qA, ry ? a.be[1][j] : T(0),
                          ry ? a.cpe[1][j] : T(0), a.psiE[0], a.psiE[0], qB,
                          rz ? a.be[2][k] : T(0), rz ? a.cpe[2][k] : T(0), a.psiE[1],
                          a.psiE[1]);
  }
  // Ey at (i, j+1/2, k): +dHx/dz, -dHz/dx
  if (iz && ix && (rz || rx)) {
    T dA = 0, dB = 0;
    long long qA = -1, qB = -1;
    if (rz) {
      dA = div_rn(sub_rn(a.Hin[0][id], a.Hin[0][id - 1]), a.dz);
      int m = a.mape[2][k];
      if (m >= 0) qA = ((long long)i * ny + j) * a.npe[2] + m;
    }
    if (rx) {
      dB = div_rn(sub_rn(a.Hin[2][id], a.Hin[2][id - sx]), a.dx);
      int m = a.mape[0][i];
      if (m >= 0) qB = ((long long)m * ny + j) * nz + k;
    }
    e[1] = curl_update<T>(e[1], K[1], rz, dA, rx, dB, qA, rz ? a.be[2][k] : T(0),
                          rz ? a.cpe[2][k] : T(0), a.psiE[2], a.psiE[2], qB,
                          rx ? a.be[0][i] : T(0), rx ? a.cpe[0][i] : T(0), a.psiE[3],
                          a.psiE[3]);
  }
  // Ez at (i, j, k+1/2): +dHy/dx, -dHx/dy
  if (ix && iy && (rx || ry)) {
    T dA = 0, dB = 0;
    long long qA = -1, qB = -1;
    if (rx) {
      dA = div_rn(sub_rn(a.Hin[1][id], a.Hin[1][id - sx]), a.dx);
      int m = a.mape[0][i];
      if (m >= 0) qA = ((long long)m * ny + j) * nz + k;
    }
    if (ry) {
      dB = div_rn(sub_rn(a.Hin[0][id], a.Hin[0][id - sy]), a.dy);
      int m = a.mape[1][j];
      if (m >= 0) qB = ((long long)i * a.npe[1] + m) * nz + k;
    }
    e[2] = curl_update<T>(e[2], K[2], rx, dA, ry, dB, qA, rx ? a.be[0][i] : T(0),
                          rx ? a.cpe[0][i] : T(0), a.psiE[4], a.psiE[4], qB,
                          ry ? a.be[1][j] : T(0), ry ? a.cpe[1][j] : T(0), a.psiE[5],
                          a.psiE[5]);
  }
  if (ADE && g >= 0) ade_apply<T>(a, g, en, e);
  a.Eout[0][id] = e[0];
  a.Eout[1][id] = e[1];
  a.Eout[2][id] = e[2];
}

}  // namespace pfb
