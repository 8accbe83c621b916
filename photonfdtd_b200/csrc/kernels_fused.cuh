// kernels_fused.cuh - single-pass fused H + E step for 3D grids.
//
// One launch advances the whole domain by one time step: each field value is
// read once and written once (to the other time level), instead of the
// split path's two passes that read E and H twice. A block owns a 32 (z) x TY
// (y) column of cells and marches along x over a chunk of planes. For each
// plane i it
//   1. stages E^n of plane i+1 (tile + one-cell halo ring) in shared memory
//      (plane i is already there from the previous iteration),
//   2. computes H^{n+1/2} of plane i on the tile plus the low halo row
//      (y = j0-1) and column (z = k0-1), which the E update needs; halo H is
//      recomputed, not exchanged, and its CPML state is read but not stored,
//   3. computes E^{n+1} of plane i on the tile from the staged H, the tile's
//      own H of plane i-1 kept in registers, and applies the ADE update.
// Because halo cells are recomputed from the previous time level, a step
// reads level `cur` and writes level `cur ^ 1` (and the H CPML state is
// double-buffered) so no block sees another block's new values.
//
// Planes where the whole tile (with its halo) is bulk - no CPML term, no
// domain face - take a straight-line path with no extent checks, no CPML
// state and no coefficient lookups; every other plane takes the general
// per-cell path of cell_update.cuh. Both evaluate the same operations in
// the same order, so results equal the split path's bit for bit.
#pragma once

#include "cell_update.cuh"

namespace pfb {

constexpr int kFusedTZ = 32;

inline bool fused_supported(int nx, int ny, int nz) { return nx > 1 && ny > 1 && nz > 1; }

template <typename T, int TY>
struct FusedSmem {
  T e[2][3][TY + 2][kFusedTZ + 2];  // E^n, planes i and i+1, halo ring of 1
  T h[3][TY + 1][kFusedTZ + 1];     // H^{n+1/2}, plane i, low halo row/column
};

template <typename T, int CE, bool ADE, int TY>
__global__ void __launch_bounds__(32 * TY, 1024 / (32 * TY)) k_fused(
    const __grid_constant__ StepArgs<T> a, int xchunk) {
  static_assert(TY >= 4 && TY <= 16, "tile height");
  constexpr int TZ = kFusedTZ, WE = TZ + 2;
  __shared__ FusedSmem<T, TY> sm;
  __shared__ MediumT<T> smed[ADE ? kMaxMedia : 1];
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TY;
  const int k = k0 + tz, j = j0 + ty;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int sy = nz, sx = ny * nz;  // cell count < 2^31 (checked at pf_create)
  const int ib = blockIdx.z * xchunk;
  if (ib >= nx) return;  // whole block: no barrier is skipped by a subset
  const int ie = min(nx, ib + xchunk);
  const bool own = k < nz && j < ny;
  const int jj = ty + 1, kk = tz + 1;
  const int colid = j * sy + k;

  if (ADE) {
    const int t = ty * 32 + tz;
    if (t < a.n_media) smed[t] = a.media[t];
  }
  // Is the tile bulk in y and z? Own cells must lie in both bulk boxes and
  // the low halo row/column in the H box (block-uniform, no barrier needed).
  const bool yz_bulk = j0 - 1 >= a.hb0[1] && j0 + TY <= a.hb1[1] && k0 - 1 >= a.hb0[2] &&
                       k0 + TZ <= a.hb1[2] && j0 >= a.eb0[1] && j0 + TY <= a.eb1[1] &&
                       k0 >= a.eb0[2] && k0 + TZ <= a.eb1[2];
  const int xb0 = max(a.hb0[0], a.eb0[0]), xb1 = min(a.hb1[0], a.eb1[0]);
  if (ADE) __syncthreads();  // media table visible to every thread

  // Stage E of plane i into buffer b (zeros outside the domain).
  auto stage = [&](int b, int i) {
    const bool inx = i < nx;
    const int base = i * sx;
#pragma unroll
    for (int c = 0; c < 3; ++c) sm.e[b][c][jj][kk] = (own && inx) ? a.Ein[c][base + colid] : T(0);
    if (ty < 2) {  // rows y = j0-1 and y = j0+TY, z = k0-1 .. k0+TZ
      const int r = ty == 0 ? 0 : TY + 1;
      const int jr = j0 - 1 + r;
      for (int q = tz; q < WE; q += 32) {
        const int kq = k0 - 1 + q;
        const bool ok = inx && jr >= 0 && jr < ny && kq >= 0 && kq < nz;
        const int id = base + jr * sy + kq;
#pragma unroll
        for (int c = 0; c < 3; ++c) sm.e[b][c][r][q] = ok ? a.Ein[c][id] : T(0);
      }
    } else if (ty == 2) {  // columns z = k0-1 (lanes 0..TY-1), z = k0+TZ (lanes 16..)
      const int t = tz & 15;
      if (t < TY) {
        const int q = tz < 16 ? 0 : WE - 1;
        const int kq = k0 - 1 + q, jr = j0 + t;
        const bool ok = inx && jr < ny && kq >= 0 && kq < nz;
        const int id = base + jr * sy + kq;
#pragma unroll
        for (int c = 0; c < 3; ++c) sm.e[b][c][t + 1][q] = ok ? a.Ein[c][id] : T(0);
      }
    }
  };

  // H of plane ib-1 at this thread's cell (Hy, Hz), for the first E update.
  T hy_prev = T(0), hz_prev = T(0);
  if (ib > 0 && own) {
    const int i = ib - 1;
    const int id = i * sx + colid;
    const T ex = a.Ein[0][id];
    const T ex_kp = k + 1 < nz ? a.Ein[0][id + 1] : T(0);
    const T ex_jp = j + 1 < ny ? a.Ein[0][id + sy] : T(0);
    hy_prev = upd_hy<T>(a, i, j, k, a.Hin[1][id], ex_kp, ex, a.Ein[2][id + sx], a.Ein[2][id], false);
    hz_prev = upd_hz<T>(a, i, j, k, a.Hin[2][id], a.Ein[1][id + sx], a.Ein[1][id], ex_jp, ex, false);
  }

  // Halo roles: warp 0 recomputes H on the row y = j0-1, warp TY-1 (lanes
  // 0..TY-1) on the column z = k0-1.
  const bool row_h = ty == 0 && j0 >= 1 && k < nz;
  const int tcol = tz;
  const bool col_h = ty == TY - 1 && tcol < TY && k0 >= 1 && j0 + tcol < ny;
  const T mch = -a.ch;
  const MediumT<T>* media = ADE ? smed : a.media;
  const bool qfast = a.fdx && a.fdy && a.fdz;
  // The ADE word of the next plane is fetched one plane ahead, so the
  // polarisation loads it addresses can issue at the top of each plane.
  const uint32_t* wsrc = CE == kCeTable ? a.word : a.adeword;
  uint32_t w_next = (ADE && own) ? wsrc[ib * sx + colid] : 0u;

  int cb = 0;
  stage(cb, ib);
  for (int i = ib; i < ie; ++i) {
    const int nb = cb ^ 1;
    const int base = i * sx;
    const int id = base + colid;
    const bool fast = yz_bulk && i >= xb0 && i < xb1;
    // loads whose latency overlaps the staging barrier and the H phase
    T h_old[3] = {T(0), T(0), T(0)};
    T K[3] = {T(0), T(0), T(0)};
    uint32_t w = 0u;
    AdeRec<T> rec;
    if (own) {
      h_old[0] = a.Hin[0][id];
      h_old[1] = a.Hin[1][id];
      h_old[2] = a.Hin[2][id];
      if (ADE) {
        const uint32_t t = w_next;
        if (i + 1 < ie) w_next = wsrc[id + sx];
        if (CE == kCeTable) {
          if (t & kDispersiveBit) {
            w = t;
            K[0] = K[1] = K[2] = media[(t >> kMediumShift) & 15u].ce;
          } else {
            K[0] = K[1] = K[2] = a.table[t];
          }
        } else {
          K[0] = K[1] = K[2] = a.ce[0][id];
          w = t;
        }
        if (w) ade_load<T>(a, media, w, rec);
      } else {
        cell_coeffs<T, CE, false>(a, media, id, K, w);
      }
    }
    T rh[2] = {T(0), T(0)}, chh[2] = {T(0), T(0)};
    if (row_h) {
      const int hid = base + (j0 - 1) * sy + k;
      rh[0] = a.Hin[0][hid];
      rh[1] = a.Hin[2][hid];
    }
    if (col_h) {
      const int hid = base + (j0 + tcol) * sy + (k0 - 1);
      chh[0] = a.Hin[0][hid];
      chh[1] = a.Hin[1][hid];
    }
    stage(nb, i + 1);
    __syncthreads();

    // ---- H^{n+1/2} on plane i ------------------------------------------
    const T(*E0)[TY + 2][WE] = sm.e[cb];
    const T(*E1)[TY + 2][WE] = sm.e[nb];
    T hx = T(0), hy = T(0), hz = T(0);
    if (fast) {
      const T exc = E0[0][jj][kk], eyc = E0[1][jj][kk], ezc = E0[2][jj][kk];
      // numerators of the six forward differences (Hx: y, z; Hy: z, x; Hz: x, y)
      const T n0 = sub_rn(E0[2][jj + 1][kk], ezc), n1 = sub_rn(E0[1][jj][kk + 1], eyc);
      const T n2 = sub_rn(E0[0][jj][kk + 1], exc), n3 = sub_rn(E1[2][jj][kk], ezc);
      const T n4 = sub_rn(E1[1][jj][kk], eyc), n5 = sub_rn(E0[0][jj + 1][kk], exc);
      if (qfast && qdiv_ok(absmax(absmax(n0, n1), absmax(absmax(n2, n3), absmax(n4, n5))))) {
        hx = bulk(h_old[0], mch, qdiv_fast(n0, a.dy, a.rdy), qdiv_fast(n1, a.dz, a.rdz));
        hy = bulk(h_old[1], mch, qdiv_fast(n2, a.dz, a.rdz), qdiv_fast(n3, a.dx, a.rdx));
        hz = bulk(h_old[2], mch, qdiv_fast(n4, a.dx, a.rdx), qdiv_fast(n5, a.dy, a.rdy));
      } else {
        hx = bulk(h_old[0], mch, qdiv(n0, a.dy, a.rdy, a.fdy), qdiv(n1, a.dz, a.rdz, a.fdz));
        hy = bulk(h_old[1], mch, qdiv(n2, a.dz, a.rdz, a.fdz), qdiv(n3, a.dx, a.rdx, a.fdx));
        hz = bulk(h_old[2], mch, qdiv(n4, a.dx, a.rdx, a.fdx), qdiv(n5, a.dy, a.rdy, a.fdy));
      }
      if (row_h) {  // Hx (y, z) and Hz (x, y) at y = j0-1
        const T m0 = sub_rn(E0[2][1][kk], E0[2][0][kk]), m1 = sub_rn(E0[1][0][kk + 1], E0[1][0][kk]);
        const T m2 = sub_rn(E1[1][0][kk], E0[1][0][kk]), m3 = sub_rn(E0[0][1][kk], E0[0][0][kk]);
        sm.h[0][0][kk] = bulk(rh[0], mch, qdiv(m0, a.dy, a.rdy, a.fdy), qdiv(m1, a.dz, a.rdz, a.fdz));
        sm.h[2][0][kk] = bulk(rh[1], mch, qdiv(m2, a.dx, a.rdx, a.fdx), qdiv(m3, a.dy, a.rdy, a.fdy));
      }
      if (col_h) {  // Hx (y, z) and Hy (z, x) at z = k0-1
        const int r = tcol + 1;
        const T m0 = sub_rn(E0[2][r + 1][0], E0[2][r][0]), m1 = sub_rn(E0[1][r][1], E0[1][r][0]);
        const T m2 = sub_rn(E0[0][r][1], E0[0][r][0]), m3 = sub_rn(E1[2][r][0], E0[2][r][0]);
        sm.h[0][r][0] = bulk(chh[0], mch, qdiv(m0, a.dy, a.rdy, a.fdy), qdiv(m1, a.dz, a.rdz, a.fdz));
        sm.h[1][r][0] = bulk(chh[1], mch, qdiv(m2, a.dz, a.rdz, a.fdz), qdiv(m3, a.dx, a.rdx, a.fdx));
      }
    } else {
      if (own) {
        hx = upd_hx<T>(a, i, j, k, h_old[0], E0[2][jj + 1][kk], E0[2][jj][kk], E0[1][jj][kk + 1],
                       E0[1][jj][kk], true);
        hy = upd_hy<T>(a, i, j, k, h_old[1], E0[0][jj][kk + 1], E0[0][jj][kk], E1[2][jj][kk],
                       E0[2][jj][kk], true);
        hz = upd_hz<T>(a, i, j, k, h_old[2], E1[1][jj][kk], E0[1][jj][kk], E0[0][jj + 1][kk],
                       E0[0][jj][kk], true);
      }
      if (row_h) {
        const int jr = j0 - 1;
        sm.h[0][0][kk] = upd_hx<T>(a, i, jr, k, rh[0], E0[2][1][kk], E0[2][0][kk],
                                   E0[1][0][kk + 1], E0[1][0][kk], false);
        sm.h[2][0][kk] = upd_hz<T>(a, i, jr, k, rh[1], E1[1][0][kk], E0[1][0][kk], E0[0][1][kk],
                                   E0[0][0][kk], false);
      }
      if (col_h) {
        const int jr = j0 + tcol, kc = k0 - 1, r = tcol + 1;
        sm.h[0][r][0] = upd_hx<T>(a, i, jr, kc, chh[0], E0[2][r + 1][0], E0[2][r][0],
                                  E0[1][r][1], E0[1][r][0], false);
        sm.h[1][r][0] = upd_hy<T>(a, i, jr, kc, chh[1], E0[0][r][1], E0[0][r][0], E1[2][r][0],
                                  E0[2][r][0], false);
      }
    }
    if (own) {
      a.Hout[0][id] = hx;
      a.Hout[1][id] = hy;
      a.Hout[2][id] = hz;
    }
    sm.h[0][jj][kk] = hx;
    sm.h[1][jj][kk] = hy;
    sm.h[2][jj][kk] = hz;
    __syncthreads();

    // ---- E^{n+1} on plane i --------------------------------------------
    if (own) {
      T en[3] = {E0[0][jj][kk], E0[1][jj][kk], E0[2][jj][kk]};
      T e[3];
      if (fast) {
        // backward differences (Ex: y, z; Ey: z, x; Ez: x, y)
        const T n0 = sub_rn(hz, sm.h[2][jj - 1][kk]), n1 = sub_rn(hy, sm.h[1][jj][kk - 1]);
        const T n2 = sub_rn(hx, sm.h[0][jj][kk - 1]), n3 = sub_rn(hz, hz_prev);
        const T n4 = sub_rn(hy, hy_prev), n5 = sub_rn(hx, sm.h[0][jj - 1][kk]);
        if (qfast && qdiv_ok(absmax(absmax(n0, n1), absmax(absmax(n2, n3), absmax(n4, n5))))) {
          e[0] = bulk(en[0], K[0], qdiv_fast(n0, a.dy, a.rdy), qdiv_fast(n1, a.dz, a.rdz));
          e[1] = bulk(en[1], K[1], qdiv_fast(n2, a.dz, a.rdz), qdiv_fast(n3, a.dx, a.rdx));
          e[2] = bulk(en[2], K[2], qdiv_fast(n4, a.dx, a.rdx), qdiv_fast(n5, a.dy, a.rdy));
        } else {
          e[0] = bulk(en[0], K[0], qdiv(n0, a.dy, a.rdy, a.fdy), qdiv(n1, a.dz, a.rdz, a.fdz));
          e[1] = bulk(en[1], K[1], qdiv(n2, a.dz, a.rdz, a.fdz), qdiv(n3, a.dx, a.rdx, a.fdx));
          e[2] = bulk(en[2], K[2], qdiv(n4, a.dx, a.rdx, a.fdx), qdiv(n5, a.dy, a.rdy, a.fdy));
        }
      } else {
        e[0] = upd_ex<T>(a, i, j, k, en[0], K[0], hz, sm.h[2][jj - 1][kk], hy, sm.h[1][jj][kk - 1]);
        e[1] = upd_ey<T>(a, i, j, k, en[1], K[1], hx, sm.h[0][jj][kk - 1], hz, hz_prev);
        e[2] = upd_ez<T>(a, i, j, k, en[2], K[2], hy, hy_prev, hx, sm.h[0][jj - 1][kk]);
      }
      if (ADE && w) ade_update<T>(a, media, rec, en, e);
      a.Eout[0][id] = e[0];
      a.Eout[1][id] = e[1];
      a.Eout[2][id] = e[2];
    }
    hy_prev = hy;
    hz_prev = hz;
    cb = nb;
  }
}

template <typename T, int CE, bool ADE>
void launch_fused_t(cudaStream_t st, const StepArgs<T>& a, int ty, int nchunk) {
  const int xchunk = (a.nx + nchunk - 1) / nchunk;
  const int nchk = (a.nx + xchunk - 1) / xchunk;
  if (ty == 16) {
    dim3 g((a.nz + kFusedTZ - 1) / kFusedTZ, (a.ny + 15) / 16, nchk);
    k_fused<T, CE, ADE, 16><<<g, dim3(32, 16), 0, st>>>(a, xchunk);
  } else {
    dim3 g((a.nz + kFusedTZ - 1) / kFusedTZ, (a.ny + 7) / 8, nchk);
    k_fused<T, CE, ADE, 8><<<g, dim3(32, 8), 0, st>>>(a, xchunk);
  }
}

// Dispatch on the coefficient mode and ADE; returns 0 when launched.
template <typename T>
int launch_fused(cudaStream_t st, const StepArgs<T>& a, int ce_mode, bool ade, int ty,
                 int nchunk) {
  if (!fused_supported(a.nx, a.ny, a.nz)) return -1;
  switch (ce_mode) {
    case kCeCell1:
      if (ade) launch_fused_t<T, kCeCell1, true>(st, a, ty, nchunk);
      else launch_fused_t<T, kCeCell1, false>(st, a, ty, nchunk);
      return 0;
    case kCeCell3:
      if (ade) return -1;
      launch_fused_t<T, kCeCell3, false>(st, a, ty, nchunk);
      return 0;
    default:
      if (ade) launch_fused_t<T, kCeTable, true>(st, a, ty, nchunk);
      else launch_fused_t<T, kCeTable, false>(st, a, ty, nchunk);
      return 0;
  }
}

}  // namespace pfb
