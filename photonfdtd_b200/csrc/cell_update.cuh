// cell_update.cuh - per-cell curl updates shared by the split and fused kernels.
//
// Each function updates one field component at cell (i, j, k) from its
// neighbour values, following src/photonfdtd/simulation.py:1252-1309 exactly
// (see curl_update in kernels_split.cuh for the operation order), and applies
// the reference's loop extents: forward differences (H) stop one cell short
// of the high face, backward differences (E) start at index 1, and a term on
// a collapsed axis is absent. Neighbour values outside those extents are
// never read. write_psi = false computes a halo cell's value without storing
// its CPML state (the owning tile stores it).
#pragma once

#include "common.cuh"

namespace pfb {

template <typename T>
__device__ __forceinline__ T curl_term(T f, T k, bool hasA, T dA, bool hasB, T dB, long long qA,
                                       T bA, T cA, const T* psiAin, T* psiAout, long long qB, T bB,
                                       T cB, const T* psiBin, T* psiBout, bool write_psi) {
  T curl = hasA ? (hasB ? sub_rn(dA, dB) : dA) : -dB;
  f = add_rn(f, mul_rn(curl, k));
  if (hasA && qA >= 0) {
    T psi = add_rn(mul_rn(bA, psiAin[qA]), mul_rn(cA, dA));
    if (write_psi) psiAout[qA] = psi;
    f = add_rn(f, mul_rn(k, psi));
  }
  if (hasB && qB >= 0) {
    T psi = add_rn(mul_rn(bB, psiBin[qB]), mul_rn(cB, dB));
    if (write_psi) psiBout[qB] = psi;
    f = add_rn(f, mul_rn(-k, psi));
  }
  return f;
}

// Bulk curl update: f + K * (dA - dB), the reference's bulk term with no
// CPML correction (simulation.py:1284-1288); curl_term with no psi.
template <typename T>
__device__ __forceinline__ T bulk(T f, T k, T dA, T dB) {
  return add_rn(f, mul_rn(sub_rn(dA, dB), k));
}

// Compact psi index of a term on axis `ax` at (i, j, k), or -1 (bulk).
template <typename T>
__device__ __forceinline__ long long psi_index(const int* map, const int* np, int ax, int i, int j,
                                               int k, int ny, int nz) {
  if (ax == 0) {
    const int m = map[i];
    return m < 0 ? -1 : ((long long)m * ny + j) * nz + k;
  }
  if (ax == 1) {
    const int m = map[j];
    return m < 0 ? -1 : ((long long)i * np[1] + m) * nz + k;
  }
  const int m = map[k];
  return m < 0 ? -1 : ((long long)i * ny + j) * np[2] + m;
}

// ---- H components (forward differences of E^n) ----------------------------
// Hx: +dEz/dy - dEy/dz
template <typename T>
__device__ __forceinline__ T upd_hx(const StepArgs<T>& a, int i, int j, int k, T h, T ez_jp,
                                    T ez, T ey_kp, T ey, bool write_psi) {
  const bool ry = a.ny > 1, rz = a.nz > 1;
  if (!((!ry || j < a.ny - 1) && (!rz || k < a.nz - 1) && (ry || rz))) return h;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (ry) {
    dA = qdiv(sub_rn(ez_jp, ez), a.dy, a.rdy, a.fdy);
    qA = psi_index<T>(a.maph[1], a.nph, 1, i, j, k, a.ny, a.nz);
  }
  if (rz) {
    dB = qdiv(sub_rn(ey_kp, ey), a.dz, a.rdz, a.fdz);
    qB = psi_index<T>(a.maph[2], a.nph, 2, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(h, -a.ch, ry, dA, rz, dB, qA, ry ? a.bh[1][j] : T(0), ry ? a.cph[1][j] : T(0),
                      a.psiHin[0], a.psiHout[0], qB, rz ? a.bh[2][k] : T(0),
                      rz ? a.cph[2][k] : T(0), a.psiHin[1], a.psiHout[1], write_psi);
}

// Hy: +dEx/dz - dEz/dx
template <typename T>
__device__ __forceinline__ T upd_hy(const StepArgs<T>& a, int i, int j, int k, T h, T ex_kp,
                                    T ex, T ez_ip, T ez, bool write_psi) {
  const bool rz = a.nz > 1, rx = a.nx > 1;
  if (!((!rz || k < a.nz - 1) && (!rx || i < a.nx - 1) && (rz || rx))) return h;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (rz) {
    dA = qdiv(sub_rn(ex_kp, ex), a.dz, a.rdz, a.fdz);
    qA = psi_index<T>(a.maph[2], a.nph, 2, i, j, k, a.ny, a.nz);
  }
  if (rx) {
    dB = qdiv(sub_rn(ez_ip, ez), a.dx, a.rdx, a.fdx);
    qB = psi_index<T>(a.maph[0], a.nph, 0, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(h, -a.ch, rz, dA, rx, dB, qA, rz ? a.bh[2][k] : T(0), rz ? a.cph[2][k] : T(0),
                      a.psiHin[2], a.psiHout[2], qB, rx ? a.bh[0][i] : T(0),
                      rx ? a.cph[0][i] : T(0), a.psiHin[3], a.psiHout[3], write_psi);
}

// Hz: +dEy/dx - dEx/dy
template <typename T>
__device__ __forceinline__ T upd_hz(const StepArgs<T>& a, int i, int j, int k, T h, T ey_ip,
                                    T ey, T ex_jp, T ex, bool write_psi) {
  const bool rx = a.nx > 1, ry = a.ny > 1;
  if (!((!rx || i < a.nx - 1) && (!ry || j < a.ny - 1) && (rx || ry))) return h;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (rx) {
    dA = qdiv(sub_rn(ey_ip, ey), a.dx, a.rdx, a.fdx);
    qA = psi_index<T>(a.maph[0], a.nph, 0, i, j, k, a.ny, a.nz);
  }
  if (ry) {
    dB = qdiv(sub_rn(ex_jp, ex), a.dy, a.rdy, a.fdy);
    qB = psi_index<T>(a.maph[1], a.nph, 1, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(h, -a.ch, rx, dA, ry, dB, qA, rx ? a.bh[0][i] : T(0), rx ? a.cph[0][i] : T(0),
                      a.psiHin[4], a.psiHout[4], qB, ry ? a.bh[1][j] : T(0),
                      ry ? a.cph[1][j] : T(0), a.psiHin[5], a.psiHout[5], write_psi);
}

// ---- E components (backward differences of H^{n+1/2}) ----------------------
// Ex: +dHz/dy - dHy/dz
template <typename T>
__device__ __forceinline__ T upd_ex(const StepArgs<T>& a, int i, int j, int k, T e, T K, T hz,
                                    T hz_jm, T hy, T hy_km) {
  const bool ry = a.ny > 1, rz = a.nz > 1;
  if (!((!ry || j >= 1) && (!rz || k >= 1) && (ry || rz))) return e;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (ry) {
    dA = qdiv(sub_rn(hz, hz_jm), a.dy, a.rdy, a.fdy);
    qA = psi_index<T>(a.mape[1], a.npe, 1, i, j, k, a.ny, a.nz);
  }
  if (rz) {
    dB = qdiv(sub_rn(hy, hy_km), a.dz, a.rdz, a.fdz);
    qB = psi_index<T>(a.mape[2], a.npe, 2, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(e, K, ry, dA, rz, dB, qA, ry ? a.be[1][j] : T(0), ry ? a.cpe[1][j] : T(0),
                      a.psiE[0], a.psiE[0], qB, rz ? a.be[2][k] : T(0), rz ? a.cpe[2][k] : T(0),
                      a.psiE[1], a.psiE[1], true);
}

// Ey: +dHx/dz - dHz/dx
template <typename T>
__device__ __forceinline__ T upd_ey(const StepArgs<T>& a, int i, int j, int k, T e, T K, T hx,
                                    T hx_km, T hz, T hz_im) {
  const bool rz = a.nz > 1, rx = a.nx > 1;
  if (!((!rz || k >= 1) && (!rx || i >= 1) && (rz || rx))) return e;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (rz) {
    dA = qdiv(sub_rn(hx, hx_km), a.dz, a.rdz, a.fdz);
    qA = psi_index<T>(a.mape[2], a.npe, 2, i, j, k, a.ny, a.nz);
  }
  if (rx) {
    dB = qdiv(sub_rn(hz, hz_im), a.dx, a.rdx, a.fdx);
    qB = psi_index<T>(a.mape[0], a.npe, 0, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(e, K, rz, dA, rx, dB, qA, rz ? a.be[2][k] : T(0), rz ? a.cpe[2][k] : T(0),
                      a.psiE[2], a.psiE[2], qB, rx ? a.be[0][i] : T(0), rx ? a.cpe[0][i] : T(0),
                      a.psiE[3], a.psiE[3], true);
}

// Ez: +dHy/dx - dHx/dy
template <typename T>
__device__ __forceinline__ T upd_ez(const StepArgs<T>& a, int i, int j, int k, T e, T K, T hy,
                                    T hy_im, T hx, T hx_jm) {
  const bool rx = a.nx > 1, ry = a.ny > 1;
  if (!((!rx || i >= 1) && (!ry || j >= 1) && (rx || ry))) return e;
  T dA = T(0), dB = T(0);
  long long qA = -1, qB = -1;
  if (rx) {
    dA = qdiv(sub_rn(hy, hy_im), a.dx, a.rdx, a.fdx);
    qA = psi_index<T>(a.mape[0], a.npe, 0, i, j, k, a.ny, a.nz);
  }
  if (ry) {
    dB = qdiv(sub_rn(hx, hx_jm), a.dy, a.rdy, a.fdy);
    qB = psi_index<T>(a.mape[1], a.npe, 1, i, j, k, a.ny, a.nz);
  }
  return curl_term<T>(e, K, rx, dA, ry, dB, qA, rx ? a.be[0][i] : T(0), rx ? a.cpe[0][i] : T(0),
                      a.psiE[4], a.psiE[4], qB, ry ? a.be[1][j] : T(0), ry ? a.cpe[1][j] : T(0),
                      a.psiE[5], a.psiE[5], true);
}

// Vector load/store of N consecutive reals (N*sizeof(T) a multiple of the
// vector width, pointer aligned to it).
template <typename T, int N>
__device__ __forceinline__ void ldv(const T* p, T* o) {
  if constexpr (sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
    for (int q = 0; q < N / 4; ++q) {
      const float4 v = reinterpret_cast<const float4*>(p)[q];
      o[4 * q] = v.x; o[4 * q + 1] = v.y; o[4 * q + 2] = v.z; o[4 * q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < N / 2; ++q) {
      if constexpr (sizeof(T) == 4) {
        const float2 v = reinterpret_cast<const float2*>(p)[q];
        o[2 * q] = v.x; o[2 * q + 1] = v.y;
      } else {
        const double2 v = reinterpret_cast<const double2*>(p)[q];
        o[2 * q] = v.x; o[2 * q + 1] = v.y;
      }
    }
  }
}
template <typename T, int N>
__device__ __forceinline__ void stv(T* p, const T* o) {
#pragma unroll
  for (int q = 0; q < N / 2; ++q) {
    if constexpr (sizeof(T) == 4) {
      reinterpret_cast<float2*>(p)[q] = make_float2(o[2 * q], o[2 * q + 1]);
    } else {
      reinterpret_cast<double2*>(p)[q] = make_double2(o[2 * q], o[2 * q + 1]);
    }
  }
}

// Polarisation record of one dispersive cell, loaded ahead of its use.
template <typename T>
struct AdeRec {
  T v[12];   // [level][pole][component] for npole <= 2
  int m;     // medium
  uint32_t loc;
};

template <typename T>
__device__ __forceinline__ void ade_load(const StepArgs<T>& a, const MediumT<T>* media,
                                         uint32_t w, AdeRec<T>& r) {
  r.m = (int)((w >> kMediumShift) & 15u);
  r.loc = w & kLocMask;
  const MediumT<T>& M = media[r.m];
  const T* R0 = a.P + M.poff + (long long)r.loc * (3 * M.npole);
  const T* R1 = R0 + a.plev;
  if (M.npole == 2) {  // 6 reals per level: 8-byte (f32) / 16-byte (f64) aligned
    ldv<T, 6>(R0, r.v);
    ldv<T, 6>(R1, r.v + 6);
  } else if (M.npole == 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r.v[c] = R0[c];
      r.v[3 + c] = R1[c];
    }
  }
}

// ADE polarisation update and E correction for one dispersive cell
// (simulation.py:645-669): P^{n+1} = a P^n + b P^{n-1} + c E^n per pole and
// component, E -= inv * sum_p (P^{n+1} - P^n), with the Python-float
// coefficients rounded to the field type as numpy's weak scalars are.
// P^{n+1} overwrites P^{n-1} (level a.lvl holds P^n). Records with more than
// two poles are read and written in place.
// NP-pole update from a loaded record; out[] receives P^{n+1} per
// [pole][component]. The level of P^n (lc) selects between compile-time
// record slots, so the record stays in registers.
template <typename T, int NP>
__device__ __forceinline__ void ade_np(const MediumT<T>& M, const T* v, int lc, const T en[3],
                                       T e[3], T out[3 * NP]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T delta = T(0);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const T lo = v[p * 3 + c], hi = v[(NP + p) * 3 + c];
      const T pc = lc ? hi : lo, pp = lc ? lo : hi;
      const T pn = add_rn(add_rn(mul_rn(M.a[p], pc), mul_rn(M.b[p], pp)), mul_rn(M.c[p], en[c]));
      out[p * 3 + c] = pn;
      const T inc = sub_rn(pn, pc);
      delta = p == 0 ? inc : add_rn(delta, inc);
    }
    e[c] = sub_rn(e[c], mul_rn(M.inv, delta));
  }
}

template <typename T>
__device__ __forceinline__ void ade_update(const StepArgs<T>& a, const MediumT<T>* media,
                                           const AdeRec<T>& r, const T en[3], T e[3]) {
  const MediumT<T>& M = media[r.m];
  const int np = M.npole;
  T* R = a.P + M.poff + (long long)r.loc * (3 * np);  // level 0 record
  const int lc = a.lvl, lp = a.lvl ^ 1;
  T* Rc = R + lc * a.plev;
  T* Rp = R + lp * a.plev;
  if (np == 2) {
    T out[6];
    ade_np<T, 2>(M, r.v, lc, en, e, out);
    stv<T, 6>(Rp, out);
    return;
  }
  if (np == 1) {
    T out[3];
    ade_np<T, 1>(M, r.v, lc, en, e, out);
    Rp[0] = out[0];
    Rp[1] = out[1];
    Rp[2] = out[2];
    return;
  }
  for (int c = 0; c < 3; ++c) {
    T delta = T(0);
    for (int p = 0; p < np; ++p) {
      const T pc = Rc[p * 3 + c], pp = Rp[p * 3 + c];
      const T pn = add_rn(add_rn(mul_rn(M.a[p], pc), mul_rn(M.b[p], pp)), mul_rn(M.c[p], en[c]));
      Rp[p * 3 + c] = pn;
      const T inc = sub_rn(pn, pc);
      delta = p == 0 ? inc : add_rn(delta, inc);
    }
    if (np > 0) e[c] = sub_rn(e[c], mul_rn(M.inv, delta));
  }
}

// E-update coefficients of one cell and, for a dispersive cell, its ADE
// word (0 for a plain cell).
// cell_coeffs in two halves, so that a kernel can issue its other loads
// between them: cell_word issues the per-cell loads (coefficient or table
// word), cell_decode turns them into K and the ADE word (table lookups).
template <typename T, int CE, bool ADE>
__device__ __forceinline__ void cell_word(const StepArgs<T>& a, long long id, T K[3],
                                          uint32_t& t) {
  t = 0u;
  if (CE == kCeCell1) {
    K[0] = K[1] = K[2] = a.ce[0][id];
    if (ADE) t = a.adeword[id];
  } else if (CE == kCeCell3) {
    K[0] = a.ce[0][id];
    K[1] = a.ce[1][id];
    K[2] = a.ce[2][id];
  } else {
    t = a.word[id];
  }
}
template <typename T, int CE, bool ADE>
__device__ __forceinline__ void cell_decode(const StepArgs<T>& a, const MediumT<T>* media,
                                            uint32_t t, T K[3], uint32_t& w) {
  w = 0u;
  if (CE == kCeCell1) {
    w = t;
  } else if (CE == kCeTable) {
    if (ADE && (t & kDispersiveBit)) {
      w = t;
      K[0] = K[1] = K[2] = media[(t >> kMediumShift) & 15u].ce;
    } else {
      K[0] = K[1] = K[2] = a.table[t & ~kDispersiveBit];
    }
  }
}

template <typename T, int CE, bool ADE>
__device__ __forceinline__ void cell_coeffs(const StepArgs<T>& a, const MediumT<T>* media,
                                            long long id, T K[3], uint32_t& w) {
  w = 0u;
  if (CE == kCeCell1) {
    K[0] = K[1] = K[2] = a.ce[0][id];
    if (ADE) w = a.adeword[id];
  } else if (CE == kCeCell3) {
    K[0] = a.ce[0][id];
    K[1] = a.ce[1][id];
    K[2] = a.ce[2][id];
  } else {
    const uint32_t t = a.word[id];
    if (ADE && (t & kDispersiveBit)) {
      w = t;
      K[0] = K[1] = K[2] = media[(t >> kMediumShift) & 15u].ce;
    } else {
      K[0] = K[1] = K[2] = a.table[t & ~kDispersiveBit];
    }
  }
}

}  // namespace pfb
