// kernels_tma.cuh - fused H + E step with TMA-staged planes (sm_100a).
//
// Same per-plane computation as k_fused (kernels_fused.cuh), but the inputs
// of each x-plane - E^n of the plane with its one-cell halo ring, the old H of
// the tile with its low halo row and column, and the per-cell coefficient
// word / arrays - arrive in shared memory by TMA (cp.async.bulk.tensor),
// issued by one thread NS planes ahead of the compute into a ring of NS
// stages, each guarded by an mbarrier. Warps only compute and store, so the
// x-march keeps several planes of loads in flight per block instead of
// exposing one global-memory latency per plane.
//
// Tile boxes (z innermost): E [40 x (TY+2)] from (k0-4, j0-1); old H
// [40 x (TY+1)] from (k0-4, j0-1); word / ce [32 x TY] from (k0, j0). The
// z-start k0-4 keeps every copy's innermost coordinate a multiple of 16
// bytes (k0 is a multiple of 32); boxes that leave the domain read zeros.
// Every wait is bounded: on timeout the block raises an error flag, waits
// (bounded) for its outstanding copies and exits together.
#pragma once

#include <cuda.h>

#include "cell3d.cuh"

namespace pfb {

constexpr int kBoxW = 40;   // z extent of the E / H boxes (k0-4 .. k0+35)
constexpr int kBoxZ0 = 4;   // tile column of k0 inside the box
constexpr long long kWaitLimit = 1LL << 27;  // ~seconds of try_wait polls

struct TmaMaps {
  CUtensorMap e[2][3];  // E components, time levels 0/1
  CUtensorMap h[2][3];  // H components
  CUtensorMap word;     // table word or ADE word (uint32)
  CUtensorMap ce[3];    // per-cell coefficients (CELL1: ce[0]; CELL3: 3)
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          long long limit = kWaitLimit) {
  for (long long t = 0; t < limit; ++t)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                       int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
      "l"((unsigned long long)map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// One TMA destination tile; every tile of a stage starts on a 128-byte
// boundary, as cp.async.bulk.tensor requires of its shared-memory address.
template <typename U, int R, int C>
struct alignas(128) Tile {
  U v[R][C];
};

template <typename T, int TY, int NCE, int NW>
struct TmaStage {
  Tile<T, TY + 2, kBoxW> e[3];
  Tile<T, TY + 1, kBoxW> h[3];
  Tile<uint32_t, NW ? TY : 1, 32> w;
  Tile<T, TY, 32> ce[NCE ? NCE : 1];
  // bytes the copies of one stage deliver (tile payloads, no padding)
  __host__ __device__ static constexpr unsigned bytes() {
    return (unsigned)(sizeof(T) * (3 * (TY + 2) * kBoxW + 3 * (TY + 1) * kBoxW + NCE * TY * 32) +
                      4 * NW * TY * 32);
  }
};

template <int CE, bool ADE>
struct TmaShape {
  static constexpr int NCE = CE == kCeCell1 ? 1 : (CE == kCeCell3 ? 3 : 0);
  static constexpr int NW = (CE == kCeTable || ADE) ? 1 : 0;
};

template <typename T, int CE, bool ADE, int TY, int NS>
__global__ void __launch_bounds__(32 * TY, 1024 / (32 * TY))
    k_fused_tma(const __grid_constant__ StepArgs<T> a, const __grid_constant__ TmaMaps maps,
                int cur, int xchunk, int* err) {
  static_assert(TY >= 4 && TY <= 16, "tile height");
  constexpr int TZ = 32, NCE = TmaShape<CE, ADE>::NCE, NW = TmaShape<CE, ADE>::NW;
  using Stage = TmaStage<T, TY, NCE, NW>;
  extern __shared__ __align__(128) unsigned char dyn[];
  // stages at the first 128-byte boundary of the dynamic window
  Stage* st = reinterpret_cast<Stage*>(((uintptr_t)dyn + 127) & ~(uintptr_t)127);
  __shared__ T sh[3][TY + 1][TZ + 1];
  __shared__ __align__(8) uint64_t full[NS];
  // Test hook (a.wait_test): block (0, 0, 0) waits once on this barrier,
  // which nothing arrives on, with a short limit, and takes the timeout path.
  __shared__ __align__(8) uint64_t never;
  __shared__ MediumT<T> smed[ADE ? kMaxMedia : 1];

  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tz;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TY;
  const int k = k0 + tz, j = j0 + ty;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int sy = nz, sx = ny * nz;
  const int ib = blockIdx.z * xchunk;
  if (ib >= nx) return;  // whole block
  const int ie = min(nx, ib + xchunk);
  const bool own = k < nz && j < ny;
  const int jj = ty + 1, kz = tz + kBoxZ0;
  const int colid = j * sy + k;

  // The producer fills stage (p - ib) % NS with plane p (E up to plane ie).
  auto issue = [&](int p) {
    Stage& S = st[(p - ib) % NS];
    uint64_t* bar = &full[(p - ib) % NS];
    mbar_expect_tx(bar, Stage::bytes());
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tma_3d(&S.e[c].v[0][0], &maps.e[cur][c], bar, k0 - kBoxZ0, j0 - 1, p);
      tma_3d(&S.h[c].v[0][0], &maps.h[cur][c], bar, k0 - kBoxZ0, j0 - 1, p);
    }
    if (NW) tma_3d(&S.w.v[0][0], &maps.word, bar, k0, j0, p);
#pragma unroll
    for (int c = 0; c < NCE; ++c) tma_3d(&S.ce[c].v[0][0], &maps.ce[c], bar, k0, j0, p);
  };
  // Self-check: every copy destination on a 128-byte boundary (else record
  // the error and leave before any copy is issued).
  bool misaligned = false;
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) {
      for (int c = 0; c < 3; ++c)
        misaligned |= ((smem_addr(&st[s].e[c]) | smem_addr(&st[s].h[c])) & 127u) != 0;
      misaligned |= (smem_addr(&st[s].w) & 127u) != 0;
      for (int c = 0; c < NCE; ++c) misaligned |= (smem_addr(&st[s].ce[c]) & 127u) != 0;
    }
    if (misaligned) atomicExch(err, 2);
  }
  if (__syncthreads_or(misaligned)) return;
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    mbar_init(&never, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const bool test_block = a.wait_test && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0;
  if (ADE && tid < a.n_media) smed[tid] = a.media[tid];
  __syncthreads();
  if (tid == 0)
    for (int p = ib; p < min(ib + NS, ie + 1); ++p) issue(p);

  const bool yz_bulk = j0 - 1 >= a.hb0[1] && j0 + TY <= a.hb1[1] && k0 - 1 >= a.hb0[2] &&
                       k0 + TZ <= a.hb1[2] && j0 >= a.eb0[1] && j0 + TY <= a.eb1[1] &&
                       k0 >= a.eb0[2] && k0 + TZ <= a.eb1[2];
  const int xb0 = max(a.hb0[0], a.eb0[0]), xb1 = min(a.hb1[0], a.eb1[0]);
  const bool row_h = ty == 0 && j0 >= 1 && k < nz;
  const int tcol = tz;
  const bool col_h = ty == TY - 1 && tcol < TY && k0 >= 1 && j0 + tcol < ny;
  const T mch = -a.ch;
  const MediumT<T>* media = ADE ? smed : a.media;
  const bool qfast = a.fdx && a.fdy && a.fdz;

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

  for (int i = ib; i < ie; ++i) {
    const int q0 = i - ib, q1 = q0 + 1;
    bool ok;
    if (test_block && i == ib) {
      ok = mbar_wait(&never, 0u, 1 << 12);  // runs out: nothing arrives
    } else {
      ok = mbar_wait(&full[q0 % NS], (unsigned)((q0 / NS) & 1));
      ok = ok && mbar_wait(&full[q1 % NS], (unsigned)((q1 / NS) & 1));
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        // let copies already issued land before the block's shared memory goes
        for (int p = i; p < min(i + NS, ie + 1); ++p)
          mbar_wait(&full[(p - ib) % NS], (unsigned)(((p - ib) / NS) & 1));
      }
      __syncthreads();
      return;
    }
    const Stage& S0 = st[q0 % NS];
    const Stage& S1 = st[q1 % NS];
    const int id = i * sx + colid;

    const bool fast = yz_bulk && i >= xb0 && i < xb1;

    // coefficients and ADE state of plane i
    T K[3] = {T(0), T(0), T(0)};
    uint32_t w = 0u;
    AdeRec<T> rec;
    if (own) {
      if (CE == kCeCell1) {
        K[0] = K[1] = K[2] = S0.ce[0].v[ty][tz];
        if (ADE) w = S0.w.v[ty][tz];
      } else if (CE == kCeCell3) {
        K[0] = S0.ce[0].v[ty][tz];
        K[1] = S0.ce[1].v[ty][tz];
        K[2] = S0.ce[2].v[ty][tz];
      } else {
        const uint32_t t = S0.w.v[ty][tz];
        if (ADE && (t & kDispersiveBit)) {
          w = t;
          K[0] = K[1] = K[2] = media[(t >> kMediumShift) & 15u].ce;
        } else {
          K[0] = K[1] = K[2] = a.table[t & ~kDispersiveBit];
        }
      }
      if (ADE && w) ade_load<T>(a, media, w, rec);
    }

    // ---- H^{n+1/2} on plane i ------------------------------------------
    const T(*E0[3])[kBoxW] = {S0.e[0].v, S0.e[1].v, S0.e[2].v};
    const T(*E1[3])[kBoxW] = {S1.e[0].v, S1.e[1].v, S1.e[2].v};
    const T(*H0[3])[kBoxW] = {S0.h[0].v, S0.h[1].v, S0.h[2].v};
    T hx = T(0), hy = T(0), hz = T(0);
    if (fast) {
      const T exc = E0[0][jj][kz], eyc = E0[1][jj][kz], ezc = E0[2][jj][kz];
      const T n0 = sub_rn(E0[2][jj + 1][kz], ezc), n1 = sub_rn(E0[1][jj][kz + 1], eyc);
      const T n2 = sub_rn(E0[0][jj][kz + 1], exc), n3 = sub_rn(E1[2][jj][kz], ezc);
      const T n4 = sub_rn(E1[1][jj][kz], eyc), n5 = sub_rn(E0[0][jj + 1][kz], exc);
      if (qfast && qdiv_ok(absmax(absmax(n0, n1), absmax(absmax(n2, n3), absmax(n4, n5))))) {
        hx = bulk(H0[0][jj][kz], mch, qdiv_fast(n0, a.dy, a.rdy), qdiv_fast(n1, a.dz, a.rdz));
        hy = bulk(H0[1][jj][kz], mch, qdiv_fast(n2, a.dz, a.rdz), qdiv_fast(n3, a.dx, a.rdx));
        hz = bulk(H0[2][jj][kz], mch, qdiv_fast(n4, a.dx, a.rdx), qdiv_fast(n5, a.dy, a.rdy));
      } else {
        hx = bulk(H0[0][jj][kz], mch, qdiv(n0, a.dy, a.rdy, a.fdy), qdiv(n1, a.dz, a.rdz, a.fdz));
        hy = bulk(H0[1][jj][kz], mch, qdiv(n2, a.dz, a.rdz, a.fdz), qdiv(n3, a.dx, a.rdx, a.fdx));
        hz = bulk(H0[2][jj][kz], mch, qdiv(n4, a.dx, a.rdx, a.fdx), qdiv(n5, a.dy, a.rdy, a.fdy));
      }
      if (row_h) {  // Hx (y, z) and Hz (x, y) at y = j0-1
        const T m0 = sub_rn(E0[2][1][kz], E0[2][0][kz]), m1 = sub_rn(E0[1][0][kz + 1], E0[1][0][kz]);
        const T m2 = sub_rn(E1[1][0][kz], E0[1][0][kz]), m3 = sub_rn(E0[0][1][kz], E0[0][0][kz]);
        sh[0][0][tz + 1] = bulk(H0[0][0][kz], mch, qdiv(m0, a.dy, a.rdy, a.fdy), qdiv(m1, a.dz, a.rdz, a.fdz));
        sh[2][0][tz + 1] = bulk(H0[2][0][kz], mch, qdiv(m2, a.dx, a.rdx, a.fdx), qdiv(m3, a.dy, a.rdy, a.fdy));
      }
      if (col_h) {  // Hx (y, z) and Hy (z, x) at z = k0-1
        const int r = tcol + 1, c3 = kBoxZ0 - 1;
        const T m0 = sub_rn(E0[2][r + 1][c3], E0[2][r][c3]), m1 = sub_rn(E0[1][r][c3 + 1], E0[1][r][c3]);
        const T m2 = sub_rn(E0[0][r][c3 + 1], E0[0][r][c3]), m3 = sub_rn(E1[2][r][c3], E0[2][r][c3]);
        sh[0][r][0] = bulk(H0[0][r][c3], mch, qdiv(m0, a.dy, a.rdy, a.fdy), qdiv(m1, a.dz, a.rdz, a.fdz));
        sh[1][r][0] = bulk(H0[1][r][c3], mch, qdiv(m2, a.dz, a.rdz, a.fdz), qdiv(m3, a.dx, a.rdx, a.fdx));
      }
    } else {
      if (own) {
        const T hold[3] = {H0[0][jj][kz], H0[1][jj][kz], H0[2][jj][kz]};
        const T n[6] = {sub_rn(E0[2][jj + 1][kz], E0[2][jj][kz]), sub_rn(E0[1][jj][kz + 1], E0[1][jj][kz]),
                        sub_rn(E0[0][jj][kz + 1], E0[0][jj][kz]), sub_rn(E1[2][jj][kz], E0[2][jj][kz]),
                        sub_rn(E1[1][jj][kz], E0[1][jj][kz]), sub_rn(E0[0][jj + 1][kz], E0[0][jj][kz])};
        T h[3];
        h3<T>(a, i, j, k, hold, n, true, h);
        hx = h[0];
        hy = h[1];
        hz = h[2];
      }
      if (row_h) {  // Hx and Hz at y = j0-1 (Hy computed and dropped)
        const T hold[3] = {H0[0][0][kz], H0[1][0][kz], H0[2][0][kz]};
        const T n[6] = {sub_rn(E0[2][1][kz], E0[2][0][kz]), sub_rn(E0[1][0][kz + 1], E0[1][0][kz]),
                        sub_rn(E0[0][0][kz + 1], E0[0][0][kz]), sub_rn(E1[2][0][kz], E0[2][0][kz]),
                        sub_rn(E1[1][0][kz], E0[1][0][kz]), sub_rn(E0[0][1][kz], E0[0][0][kz])};
        T h[3];
        h3<T>(a, i, j0 - 1, k, hold, n, false, h);
        sh[0][0][tz + 1] = h[0];
        sh[2][0][tz + 1] = h[2];
      }
      if (col_h) {  // Hx and Hy at z = k0-1 (Hz computed and dropped)
        const int r = tcol + 1, c3 = kBoxZ0 - 1;
        const T hold[3] = {H0[0][r][c3], H0[1][r][c3], H0[2][r][c3]};
        const T n[6] = {sub_rn(E0[2][r + 1][c3], E0[2][r][c3]), sub_rn(E0[1][r][c3 + 1], E0[1][r][c3]),
                        sub_rn(E0[0][r][c3 + 1], E0[0][r][c3]), sub_rn(E1[2][r][c3], E0[2][r][c3]),
                        sub_rn(E1[1][r][c3], E0[1][r][c3]), sub_rn(E0[0][r + 1][c3], E0[0][r][c3])};
        T h[3];
        h3<T>(a, i, j0 + tcol, k0 - 1, hold, n, false, h);
        sh[0][r][0] = h[0];
        sh[1][r][0] = h[1];
      }
    }
    if (own) {
      a.Hout[0][id] = hx;
      a.Hout[1][id] = hy;
      a.Hout[2][id] = hz;
    }
    sh[0][jj][tz + 1] = hx;
    sh[1][jj][tz + 1] = hy;
    sh[2][jj][tz + 1] = hz;
    __syncthreads();

    // ---- E^{n+1} on plane i --------------------------------------------
    if (own) {
      const int kk = tz + 1;
      T en[3] = {E0[0][jj][kz], E0[1][jj][kz], E0[2][jj][kz]};
      T e[3];
      if (fast) {
        const T n0 = sub_rn(hz, sh[2][jj - 1][kk]), n1 = sub_rn(hy, sh[1][jj][kk - 1]);
        const T n2 = sub_rn(hx, sh[0][jj][kk - 1]), n3 = sub_rn(hz, hz_prev);
        const T n4 = sub_rn(hy, hy_prev), n5 = sub_rn(hx, sh[0][jj - 1][kk]);
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
        const T n[6] = {sub_rn(hz, sh[2][jj - 1][kk]), sub_rn(hy, sh[1][jj][kk - 1]),
                        sub_rn(hx, sh[0][jj][kk - 1]), sub_rn(hz, hz_prev),
                        sub_rn(hy, hy_prev), sub_rn(hx, sh[0][jj - 1][kk])};
        e3<T>(a, i, j, k, en, K, n, e);
      }
      if (ADE && w) ade_update<T>(a, media, rec, en, e);
      a.Eout[0][id] = e[0];
      a.Eout[1][id] = e[1];
      a.Eout[2][id] = e[2];
    }
    hy_prev = hy;
    hz_prev = hz;
    __syncthreads();  // stage q0 and sh are free
    if (tid == 0 && i + NS <= ie) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(i + NS);
    }
  }
}

template <typename T, int CE, bool ADE, int TY, int NS>
size_t tma_smem_bytes() {
  using Stage = TmaStage<T, TY, TmaShape<CE, ADE>::NCE, TmaShape<CE, ADE>::NW>;
  return sizeof(Stage) * NS + 128;
}

// Launch one step; returns 0 when launched, -1 when the case is not covered.
template <typename T, int CE, bool ADE>
int launch_tma_t(cudaStream_t st, const StepArgs<T>& a, const TmaMaps& maps, int cur,
                 int nchunk, int* err) {
  constexpr int TY = 8, NS = 4;
  const size_t smem = tma_smem_bytes<T, CE, ADE, TY, NS>();
  auto kern = k_fused_tma<T, CE, ADE, TY, NS>;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return -1;
    configured = true;
  }
  const int xchunk = (a.nx + nchunk - 1) / nchunk;
  const int nchk = (a.nx + xchunk - 1) / xchunk;
  dim3 g((a.nz + 31) / 32, (a.ny + TY - 1) / TY, nchk);
  kern<<<g, dim3(32, TY), smem, st>>>(a, maps, cur, xchunk, err);
  return 0;
}

template <typename T>
int launch_tma(cudaStream_t st, const StepArgs<T>& a, const TmaMaps& maps, int cur, int ce_mode,
               bool ade, int nchunk, int* err) {
  switch (ce_mode) {
    case kCeCell1:
      return ade ? launch_tma_t<T, kCeCell1, true>(st, a, maps, cur, nchunk, err)
                 : launch_tma_t<T, kCeCell1, false>(st, a, maps, cur, nchunk, err);
    case kCeCell3:
      return ade ? -1 : launch_tma_t<T, kCeCell3, false>(st, a, maps, cur, nchunk, err);
    default:
      return ade ? launch_tma_t<T, kCeTable, true>(st, a, maps, cur, nchunk, err)
                 : launch_tma_t<T, kCeTable, false>(st, a, maps, cur, nchunk, err);
  }
}

}  // namespace pfb
