// surrogate.cu - training and inference kernels of the learned surrogate
// (a convolutional encoder-decoder mapping a design density to its complex
// transmission spectrum).
//
// Every layer of the network is expressed with these few device routines,
// all hand-written here:
//   * pfs_gemm_bf16: C = alpha * A B^T + beta * C, A (M x K) and B (N x K)
//     row-major BF16 (K contiguous), C row-major FP32. Tensor cores through
//     mma.sync m16n8k16 (BF16 inputs, FP32 accumulate); 64 x 64 x 32 block
//     tiles, 4 warps of 32 x 32, operands staged in padded shared memory with
//     a register prefetch of the next K slice.
//   * im2col (BF16, K padded with zeros to a multiple of 32) and its adjoint
//     col2im (FP32, a gather over the kernel taps: deterministic);
//   * bias + ReLU with FP32 and BF16 outputs, and its backward with a
//     deterministic column reduction for the bias gradient;
//   * BF16 transposes, FP32 -> BF16 conversion, nearest 2x upsampling along
//     the width and its adjoint, the mean-squared-error loss gradient and an
//     Adam step on FP32 master weights that refreshes their BF16 copies.
// Activations are NHWC. Nothing here allocates: the caller owns every buffer
// and passes its stream (NULL = the default stream).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/pfb200.h"

namespace {

thread_local std::string g_err;

int sfail(int code, const char* msg) {
  g_err = msg;
  return code;
}

int cuda_status(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return PF_OK;
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  g_err = buf;
  return PF_ERR_CUDA;
}

// ---- GEMM ------------------------------------------------------------------
constexpr int BM = 64, BN = 64, BK = 32, PADK = BK + 8;  // padded rows: fewer bank conflicts

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One 16-byte chunk (8 BF16) of row r, columns k0..k0+7 of a row-major
// matrix with `rows` rows and leading dimension ld, or zeros out of range.
__device__ __forceinline__ uint4 ld_chunk(const __nv_bfloat16* p, int rows, int ld, int r, int k0) {
  if (r >= rows) return make_uint4(0, 0, 0, 0);
  return *reinterpret_cast<const uint4*>(p + (long long)r * ld + k0);
}

// C[M x N] = alpha * sum_k A[m][k] B[n][k] + beta * C. K % 32 == 0; lda, ldb
// multiples of 8 (16-byte rows); pointers 16-byte aligned. With split-K
// (gridDim.z > 1) block z sums k in [z * kc, (z + 1) * kc) and writes
// alpha * partial into its own M x N slab of `work` (leading dimension N);
// k_splitk_reduce adds the slabs in order.
__global__ void __launch_bounds__(128) k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* A,
                                                   int lda, const __nv_bfloat16* B, int ldb,
                                                   float* C, int ldc, float alpha, float beta,
                                                   int kc, float* work) {
  const int kbeg = blockIdx.z * kc;
  const int kend = min(K, kbeg + kc);
  if (gridDim.z > 1) {
    C = work + (long long)blockIdx.z * M * N;
    ldc = N;
    beta = 0.f;
  }
  A += kbeg;
  B += kbeg;
  K = max(0, kend - kbeg);
  __shared__ __align__(16) __nv_bfloat16 As[BM][PADK];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][PADK];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, tg = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  // each thread stages two 16-byte chunks of A and two of B per K slice:
  // chunk q = tid + 128 * h -> row q / 4, columns (q % 4) * 8
  uint4 ra[2], rb[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int q = tid + 128 * h, r = q >> 2, kq = (q & 3) * 8;
    ra[h] = K > 0 ? ld_chunk(A, M, lda, m0 + r, kq) : make_uint4(0, 0, 0, 0);
    rb[h] = K > 0 ? ld_chunk(B, N, ldb, n0 + r, kq) : make_uint4(0, 0, 0, 0);
  }
  for (int k0 = 0; k0 < K; k0 += BK) {
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = tid + 128 * h, r = q >> 2, kq = (q & 3) * 8;
      *reinterpret_cast<uint4*>(&As[r][kq]) = ra[h];
      *reinterpret_cast<uint4*>(&Bs[r][kq]) = rb[h];
    }
    __syncthreads();
    if (k0 + BK < K) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = tid + 128 * h, r = q >> 2, kq = (q & 3) * 8;
        ra[h] = ld_chunk(A, M, lda, m0 + r, k0 + BK + kq);
        rb[h] = ld_chunk(B, N, ldb, n0 + r, k0 + BK + kq);
      }
    }
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int r = wm + a * 16 + g;
        af[a][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + tg * 2]);
        af[a][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + tg * 2]);
        af[a][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + tg * 2 + 8]);
        af[a][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + tg * 2 + 8]);
      }
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int n = wn + b * 8 + g;
        bf[b][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + tg * 2]);
        bf[b][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + tg * 2 + 8]);
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) mma_bf16(acc[a][b], af[a], bf[b]);
    }
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int r = m0 + wm + a * 16 + g + (c >= 2 ? 8 : 0);
        const int n = n0 + wn + b * 8 + tg * 2 + (c & 1);
        if (r < M && n < N) {
          float* o = C + (long long)r * ldc + n;
          const float v = alpha * acc[a][b][c];
          *o = beta == 0.f ? v : v + beta * *o;
        }
      }
}

// ---- tcgen05 GEMM ------------------------------------------------------------
// The same contract as k_gemm_bf16 on the 5th-generation tensor cores: a
// 128 x BN output tile per CTA accumulates in tensor memory (TMEM, BN 32-bit
// columns x 128 lanes) from tcgen05.mma.cta_group::1.kind::f16 (BF16 in, FP32
// accumulate). Operand tiles of 64 K-columns (128-byte rows) arrive by TMA
// (cp.async.bulk.tensor, 128-byte swizzle, zeros past the matrix edge) in a
// ring of up to TC_STAGES stages (tc_ring_stages): warp 0 produces (waits
// for a stage's `empty` barrier, posts the byte count on its `full`
// barrier, issues the two loads),
// warp 1 consumes (waits for `full`, lane 0 issues four K = 16 MMAs and
// commits them to `empty`, so the stage is refilled once they have read it).
// A last commit to `done` releases all four warps into the epilogue: each
// reads its 32 TMEM lanes (tile rows) with tcgen05.ld.32x32b, transposes
// 32 x 32 blocks through shared memory and stores whole rows.
// Shared-memory descriptor of a K-major 128-byte-swizzled operand: rows at
// 128 bytes, 8-row groups at 1024 bytes (stride byte offset), leading byte
// offset unused (1), layout type 2; the K = 16 slice ks of a stage starts
// 32 * ks bytes into each row (the swizzle is applied to the full address,
// so stage bases are 1024-byte aligned).
// Every wait is bounded (kTcWaitNs): on a timeout the block sets an abort
// flag, waits (bounded) for its own loads and MMAs in flight, records the
// timeout in *err, skips the epilogue, frees its TMEM and returns.
constexpr int TBM = 128, TBK = 64, TC_STAGES = 4;
constexpr unsigned long long kTcWaitNs = 1000000000ull;  // 1 s per wait

__host__ __device__ constexpr int tc_stage_bytes(int bn) { return (TBM + bn) * TBK * 2; }
__host__ __device__ constexpr int tc_smem_bytes(int bn, int stages = TC_STAGES) {
  return stages * tc_stage_bytes(bn) + 1024;  // + alignment of the ring to 1024 bytes
}
// Ring depth of a launch: no more stages than K tiles in a block's slice, so
// a short-K GEMM (a layer's input gradient: K = 32..256) takes less shared
// memory and several blocks share an SM (one block's epilogue overlapping
// another's loads and MMAs) instead of one block per SM leaving it idle.
// PFB200_TC_FULL_RING=1 keeps the full ring for every launch (comparison).
inline int tc_ring_stages(int kc) {
  static const bool full = getenv("PFB200_TC_FULL_RING") != nullptr;
  return full ? TC_STAGES : std::max(1, std::min(TC_STAGES, (kc + TBK - 1) / TBK));
}

__device__ __forceinline__ unsigned long long tc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool tc_mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.b32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the completion of the phase with the given parity, at most
// limit_ns (and at most 2^30 polls); gives up early once *abort is set.
__device__ __forceinline__ bool tc_mbar_wait(uint32_t bar, uint32_t parity,
                                             const volatile int* abort = nullptr,
                                             unsigned long long limit_ns = kTcWaitNs) {
  const unsigned long long t0 = tc_now();
  for (int i = 0; i < (1 << 30); ++i) {
    if (tc_mbar_try(bar, parity)) return true;
    if ((i & 63) == 63 && (tc_now() - t0 > limit_ns || (abort && *abort))) return false;
  }
  return false;
}

__device__ __forceinline__ uint64_t tc_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// The same for an MN-major operand (stored K x MN, MN contiguous): TMA puts
// each 64-element MN strip of a stage (64 K rows of 128 bytes, swizzled in
// 1024-byte groups of 8 rows) 8192 bytes after the previous one. In the
// descriptor the leading byte offset is the step between MN strips (8192)
// and the stride byte offset the step between 8-row K groups (1024); the
// K = 16 slice ks starts 2048 * ks bytes into the stage.
constexpr uint32_t kMnStrip = 64 * TBK * 2;  // bytes of one 64-wide MN strip of a stage
__device__ __forceinline__ uint64_t tc_desc_mn_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kMnStrip >> 4) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void tc_tma_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                          int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"((unsigned long long)map), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Epilogue of a layer's forward GEMM (EPI): y = act(C + bias) written as
// FP32 (to C) and BF16 (y16, same leading dimension), k_bias_act's
// arithmetic on the value C would have held; beta is 0 and K unsplit.
struct TcEpi {
  const float* bias;
  int relu;
  __nv_bfloat16* y16;
};

// AMN / BMN: the operand is stored MN-major (K x M or K x N, MN contiguous)
// and read as such by the tensor cores (the descriptor's transpose bits), so
// no transposed copy is made; its stage is loaded as 64-wide MN strips.
template <int BN, bool AMN = false, bool BMN = false, bool EPI = false>
__global__ void __launch_bounds__(128, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
              int M, int N, int K, float* C, int ldc, float alpha, float beta, int kc, float* work,
              int* err, int wait_test, TcEpi ep, int nst) {
  static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN");
  static_assert(!BMN || BN >= 64, "an MN-major B needs whole 64-wide strips");
  constexpr uint32_t ABYTES = TBM * TBK * 2, SB = tc_stage_bytes(BN);
  extern __shared__ uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], done;
  // Test hook (pfs_gemm_wait_test): the MMA warp of block (0, 0, 0) first
  // waits 100 us on this barrier, which nothing arrives on, and so takes the
  // timeout path below.
  __shared__ __align__(8) uint64_t never;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag, n_loaded, n_seen;
  volatile int* abort_v = &abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kc;
  const int kend = min(K, kbeg + kc);
  if (gridDim.z > 1) {  // split K (never with the fused epilogue)
    C = work + (long long)blockIdx.z * M * N;
    ldc = N;
    if constexpr (!EPI) beta = 0.f;
  }
  const int nk = (kend - kbeg + TBK - 1) / TBK;  // >= 1 (host guarantees non-empty slices)
  const uint32_t s0 = (smem_u32(tc_smem) + 1023u) & ~1023u;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int i = 0; i < TC_STAGES; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[i])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&done)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&never)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    n_loaded = 0;
    n_seen = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;
  if (warp == 0) {  // producer
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int st = kt % nst;
      bool ok = true;
      if (kt >= nst) ok = tc_mbar_wait(smem_u32(&empty[st]), ((kt / nst) - 1) & 1, abort_v);
      if (!__all_sync(0xffffffffu, ok && !*abort_v)) {
        if (lane == 0) *abort_v = 1;
        break;
      }
      if (lane == 0) {
        const uint32_t fb = smem_u32(&full[st]), dst = s0 + st * SB;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(SB)
                     : "memory");
        if constexpr (AMN) {
#pragma unroll
          for (int q = 0; q < TBM / 64; ++q)
            tc_tma_2d(dst + q * kMnStrip, &ta, fb, m0 + 64 * q, kbeg + kt * TBK);
        } else {
          tc_tma_2d(dst, &ta, fb, kbeg + kt * TBK, m0);
        }
        if constexpr (BMN) {
#pragma unroll
          for (int q = 0; q < BN / 64; ++q)
            tc_tma_2d(dst + ABYTES + q * kMnStrip, &tb, fb, n0 + 64 * q, kbeg + kt * TBK);
        } else {
          tc_tma_2d(dst + ABYTES, &tb, fb, kbeg + kt * TBK, n0);
        }
      }
      __syncwarp();
    }
    if (lane == 0) n_loaded = kt;
  } else if (warp == 1) {  // MMA issue
    constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((AMN ? 1u : 0u) << 15) |
                               ((BMN ? 1u : 0u) << 16) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TBM >> 4) << 24);
    int kt = 0;
    const bool test_block = wait_test && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0;
    for (; kt < nk; ++kt) {
      const int st = kt % nst;
      const bool ok = (test_block && kt == 0)
                          ? tc_mbar_wait(smem_u32(&never), 0, abort_v, 100000ull)
                          : tc_mbar_wait(smem_u32(&full[st]), (kt / nst) & 1, abort_v);
      if (!__all_sync(0xffffffffu, ok && !*abort_v)) {
        if (lane == 0) *abort_v = 1;
        break;
      }
      if (lane == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t a0 = s0 + st * SB, b0 = a0 + ABYTES;
#pragma unroll
        for (int ks = 0; ks < TBK / 16; ++ks) {
          const uint64_t da = AMN ? tc_desc_mn_sw128(a0 + 2048 * ks) : tc_desc_sw128(a0 + 32 * ks);
          const uint64_t db = BMN ? tc_desc_mn_sw128(b0 + 2048 * ks) : tc_desc_sw128(b0 + 32 * ks);
          const uint32_t accum = (kt > 0 || ks > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::
                  "r"(tmem),
              "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&empty[st])));
      }
      __syncwarp();
    }
    if (lane == 0) {
      n_seen = kt;
      // covers every MMA issued above (arrives at once if there were none)
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&done)));
    }
    __syncwarp();
  }
  __syncthreads();
  bool ok = tc_mbar_wait(smem_u32(&done), 0);
  if (__syncthreads_or(!ok || abort_flag)) {
    // loads issued but never consumed are still in flight: wait for them
    if (tid == 0) {
      for (int kt = n_seen; kt < n_loaded; ++kt)
        tc_mbar_wait(smem_u32(&full[kt % nst]), (kt / nst) & 1);
      atomicAdd(err, 1);
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;");
    float* stage = reinterpret_cast<float*>(tc_smem + (s0 - smem_u32(tc_smem))) + warp * 32 * 33;
    const int rbase = m0 + warp * 32;
#pragma unroll 1
    for (int cb = 0; cb < BN / 32; ++cb) {
      if (n0 + cb * 32 >= N) break;  // uniform
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
          "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, "
          "%27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
            "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
            "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) stage[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int n = n0 + cb * 32 + lane;
      for (int rr = 0; rr < 32; ++rr) {
        const int r = rbase + rr;
        if (r < M && n < N) {
          float* o = C + (long long)r * ldc + n;
          const float val = alpha * stage[rr * 33 + lane];
          if constexpr (EPI) {
            float v = val + (ep.bias ? ep.bias[n] : 0.f);
            if (ep.relu) v = fmaxf(v, 0.f);
            *o = v;
            if (ep.y16) ep.y16[(long long)r * ldc + n] = __float2bfloat16(v);
          } else {
            *o = beta == 0.f ? val : val + beta * *o;
          }
        }
      }
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// C = sum over the split slabs, in order, + beta * C.
__global__ void k_splitk_reduce(int M, int N, int splits, const float* work, float* C, int ldc,
                                float beta) {
  const long long total = (long long)M * N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int z = 0; z < splits; ++z) s += work[(long long)z * total + t];
    const long long m = t / N, n = t % N;
    float* o = C + m * ldc + n;
    *o = beta == 0.f ? s : s + beta * *o;
  }
}

// ---- convolution lowering ----------------------------------------------------
// col[(b, oy, ox)][k], k = (ky * kw + kx) * C + c for k < kh*kw*C, zero above.
__global__ void k_im2col(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
                         int Ho, int Wo, const __nv_bfloat16* x, __nv_bfloat16* col, int Kp) {
  const long long total = (long long)nb * Ho * Wo * Kp;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % Kp);
    const long long m = t / Kp;
    __nv_bfloat16 v = __float2bfloat16(0.f);
    if (k < kh * kw * C) {
      const int c = k % C, tap = k / C, kx = tap % kw, ky = tap / kw;
      const int ox = (int)(m % Wo), oy = (int)((m / Wo) % Ho), b = (int)(m / ((long long)Wo * Ho));
      const int iy = oy * stride - ph + ky, ix = ox * stride - pw + kx;
      if (iy >= 0 && iy < H && ix >= 0 && ix < W) v = x[(((long long)b * H + iy) * W + ix) * C + c];
    }
    col[t] = v;
  }
}

// dx[b, iy, ix, c] = sum over the taps (ky, kx) whose output position
// (oy, ox) = ((iy + ph - ky) / stride, (ix + pw - kx) / stride) is integral
// and in range of dcol[(b, oy, ox)][(ky * kw + kx) * C + c].
__global__ void k_col2im(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
                         int Ho, int Wo, const float* dcol, int Kp, float* dx) {
  const long long total = (long long)nb * H * W * C;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const int ix = (int)((t / C) % W), iy = (int)((t / ((long long)C * W)) % H);
    const int b = (int)(t / ((long long)C * W * H));
    float s = 0.f;
    for (int ky = 0; ky < kh; ++ky) {
      const int ny = iy + ph - ky;
      if (ny < 0 || ny % stride) continue;
      const int oy = ny / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < kw; ++kx) {
        const int nx = ix + pw - kx;
        if (nx < 0 || nx % stride) continue;
        const int ox = nx / stride;
        if (ox >= Wo) continue;
        s += dcol[(((long long)b * Ho + oy) * Wo + ox) * Kp + (ky * kw + kx) * C + c];
      }
    }
    dx[t] = s;
  }
}

// Vector forms of the two lowerings (32-bit indices; the host checks the
// sizes and 16-byte alignment). im2col: one thread per 8-column chunk of a
// col row (one 16-byte store); when C % 8 == 0 a chunk is 8 channels of one
// tap, read with one 16-byte load. col2im: one thread per 8 channels of an
// input position (C % 8 == 0), the taps summed in the same order as k_col2im,
// so both forms give identical results.
template <bool VEC>
__global__ void k_im2col8(int rows, int H, int W, int C, int kh, int kw, int stride, int ph,
                          int pw, int Ho, int Wo, const __nv_bfloat16* x, __nv_bfloat16* col,
                          int Kp) {
  const int qn = Kp >> 3, K = kh * kw * C;
  const int total = rows * qn;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int q = t % qn, m = t / qn;
    const int ox = m % Wo, r = m / Wo, oy = r % Ho, b = r / Ho;
    const int k0 = q * 8;
    uint4 out = make_uint4(0, 0, 0, 0);
    if (VEC) {
      if (k0 < K) {
        const int tap = k0 / C, c = k0 - tap * C, kx = tap % kw, ky = tap / kw;
        const int iy = oy * stride - ph + ky, ix = ox * stride - pw + kx;
        if (iy >= 0 && iy < H && ix >= 0 && ix < W)
          out = *reinterpret_cast<const uint4*>(x + ((long long)(b * H + iy) * W + ix) * C + c);
      }
    } else {
      __nv_bfloat16 v[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        v[e] = __float2bfloat16(0.f);
        const int k = k0 + e;
        if (k < K) {
          const int c = k % C, tap = k / C, kx = tap % kw, ky = tap / kw;
          const int iy = oy * stride - ph + ky, ix = ox * stride - pw + kx;
          if (iy >= 0 && iy < H && ix >= 0 && ix < W)
            v[e] = x[((long long)(b * H + iy) * W + ix) * C + c];
        }
      }
      out = *reinterpret_cast<const uint4*>(v);
    }
    *reinterpret_cast<uint4*>(col + (long long)m * Kp + k0) = out;
  }
}

__global__ void k_col2im8(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
                          int Ho, int Wo, const float* dcol, int Kp, float* dx) {
  const int cg = C >> 3;
  const int total = nb * H * W * cg;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int g = t % cg, p = t / cg;
    const int ix = p % W, r = p / W, iy = r % H, b = r / H;
    const int c0 = g * 8;
    float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
    for (int ky = 0; ky < kh; ++ky) {
      const int ny = iy + ph - ky;
      if (ny < 0 || ny % stride) continue;
      const int oy = ny / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < kw; ++kx) {
        const int nx = ix + pw - kx;
        if (nx < 0 || nx % stride) continue;
        const int ox = nx / stride;
        if (ox >= Wo) continue;
        const float4* src = reinterpret_cast<const float4*>(
            dcol + (long long)((b * Ho + oy) * Wo + ox) * Kp + (ky * kw + kx) * C + c0);
        const float4 u = src[0], v = src[1];
        s0.x += u.x; s0.y += u.y; s0.z += u.z; s0.w += u.w;
        s1.x += v.x; s1.y += v.y; s1.z += v.z; s1.w += v.w;
      }
    }
    float4* dst = reinterpret_cast<float4*>(dx + (long long)p * C + c0);
    dst[0] = s0;
    dst[1] = s1;
  }
}

// y = act(x + bias) over an M x N row-major matrix; FP32 and BF16 outputs
// (either may be NULL).
__global__ void k_bias_act(long long M, int N, const float* x, const float* bias, int relu,
                           float* y32, __nv_bfloat16* y16) {
  const long long total = M * N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    float v = x[t] + (bias ? bias[t % N] : 0.f);
    if (relu) v = fmaxf(v, 0.f);
    if (y32) y32[t] = v;
    if (y16) y16[t] = __float2bfloat16(v);
  }
}

// dpre = dy * (y > 0) (or dy), stored FP32 and BF16, and per row block the
// column sums of dpre: part[blockIdx.y][n]. Blocks of 32 columns x 8 row
// lanes; each row block strides the rows, then a fixed-order reduction.
__global__ void k_act_bwd(long long M, int N, const float* dy, const float* y, int relu,
                          float* d32, __nv_bfloat16* d16, float* part) {
  __shared__ float sh[8][33];
  const int n = blockIdx.x * 32 + threadIdx.x;
  float s = 0.f;
  for (long long m = (long long)blockIdx.y * 8 + threadIdx.y; m < M; m += (long long)gridDim.y * 8) {
    if (n < N) {
      const long long t = m * N + n;
      float v = dy[t];
      if (relu && !(y[t] > 0.f)) v = 0.f;
      if (d32) d32[t] = v;
      if (d16) d16[t] = __float2bfloat16(v);
      s += v;
    }
  }
  sh[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && n < N && part) {
    float r = 0.f;
    for (int q = 0; q < 8; ++q) r += sh[q][threadIdx.x];
    part[(long long)blockIdx.y * N + n] = r;
  }
}

// dbias[n] = sum over the row blocks of part[q][n]: one block per column,
// strided partial sums and a fixed-order tree (independent of scheduling).
__global__ void k_colsum(int R, int N, const float* part, float* out) {
  __shared__ float sh[256];
  const int n = blockIdx.x;
  float r = 0.f;
  for (int q = threadIdx.x; q < R; q += blockDim.x) r += part[(long long)q * N + n];
  sh[threadIdx.x] = r;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = sh[0];
}

// out[c][r] = in[r][c] for an R x Cc row-major BF16 matrix; out has leading
// dimension ldo (>= R, extra columns zero-filled up to ldo).
__global__ void k_transpose_bf16(int R, int Cc, const __nv_bfloat16* in, int ldi,
                                 __nv_bfloat16* out, int ldo) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int r = r0 + q, c = c0 + threadIdx.x;
    tile[q][threadIdx.x] = (r < R && c < Cc) ? in[(long long)r * ldi + c] : __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int c = c0 + q, r = r0 + threadIdx.x;
    if (c < Cc && r < ldo) out[(long long)c * ldo + r] = tile[threadIdx.x][q];
  }
}

__global__ void k_to_bf16(long long n, const float* x, __nv_bfloat16* y) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    y[t] = __float2bfloat16(x[t]);
}

// Nearest 2x upsampling along the width of an (nb, W, C) tensor (H = 1):
// y[b, 2w + s, c] = x[b, w, c]; the backward sums the two copies.
__global__ void k_upsample2(long long nb, int W, int C, const __nv_bfloat16* x, __nv_bfloat16* y) {
  const long long total = nb * 2 * W * C;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const long long w2 = (t / C) % (2 * W), b = t / ((long long)C * 2 * W);
    y[t] = x[(b * W + w2 / 2) * C + c];
  }
}

__global__ void k_upsample2_bwd(long long nb, int W, int C, const float* dy, float* dx) {
  const long long total = nb * W * C;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const long long w = (t / C) % W, b = t / ((long long)C * W);
    const long long o = (b * 2 * W + 2 * w) * C + c;
    dx[t] = dy[o] + dy[o + C];
  }
}

// MSE of the first `used` columns of y (rows x ld, FP32) against compact t
// (rows x used): grad (rows x ld) = 2 (y - t) / (rows * used) there, zero in
// the other columns; per-block partial losses in fixed order.
__global__ void k_mse(long long rows, int used, int ld, const float* y, const float* t,
                      float* grad, float* loss) {
  __shared__ float sh[256];
  const long long n = rows * ld;
  const float inv = 1.f / (float)(rows * used);
  float s = 0.f;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % ld);
    if (c < used) {
      const float d = y[q] - t[(q / ld) * used + c];
      grad[q] = 2.f * d * inv;
      s += d * d;
    } else {
      grad[q] = 0.f;
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[blockIdx.x] = sh[0] * inv;
}

// Adam on FP32 master weights (bias-corrected, weight decay decoupled from
// the gradient statistics), then the BF16 copy.
__global__ void k_adam(long long n, float* w, const float* g, float* m, float* v, float lr,
                       float b1, float b2, float eps, float c1, float c2, float wd,
                       __nv_bfloat16* w16) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    const float wn = w[t] - lr * ((mt / c1) / (sqrtf(vt / c2) + eps) + wd * w[t]);
    w[t] = wn;
    if (w16) w16[t] = __float2bfloat16(wn);
  }
}

__device__ int g_tc_err = 0;

typedef CUresult (*TcEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                               const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                               const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// TMA map of a row-major BF16 matrix (rows x cols, leading dimension ld
// elements), box 64 columns x box_rows rows, 128-byte swizzle, zeros outside.
bool tc_map(CUtensorMap* m, const void* ptr, int cols, int rows, int ld, int box_rows) {
  static TcEncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return false;
    fn = (TcEncodeFn)p;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TBK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
int g_gemm_engine = 1;  // 1: tcgen05 (TMEM accumulator), 0: mma.sync m16n8k16
int g_gemm_wait_test = 0;  // pfs_gemm_wait_test

template <int BN, bool AMN, bool BMN, bool EPI = false>
bool tc_prepare() {
  return cudaFuncSetAttribute(k_gemm_tc<BN, AMN, BMN, EPI>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              tc_smem_bytes(BN)) == cudaSuccess;
}

template <bool AMN, bool BMN, bool EPI = false>
void tc_launch(int bn, dim3 grid, cudaStream_t st, const CUtensorMap& ta, const CUtensorMap& tb,
               int M, int N, int K, float* C, int ldc, float alpha, float beta, int kc,
               float* work, int* err, TcEpi ep = TcEpi{}) {
  const int wt = g_gemm_wait_test;
  const int ns = tc_ring_stages(kc);
  switch (bn) {
    case 32:
      if constexpr (!BMN)
        k_gemm_tc<32, AMN, BMN, EPI><<<grid, 128, tc_smem_bytes(32, ns), st>>>(
            ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err, wt, ep, ns);
      break;
    case 64:
      k_gemm_tc<64, AMN, BMN, EPI><<<grid, 128, tc_smem_bytes(64, ns), st>>>(
          ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err, wt, ep, ns);
      break;
    case 128:
      k_gemm_tc<128, AMN, BMN, EPI><<<grid, 128, tc_smem_bytes(128, ns), st>>>(
          ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err, wt, ep, ns);
      break;
    default:
      k_gemm_tc<256, AMN, BMN, EPI><<<grid, 128, tc_smem_bytes(256, ns), st>>>(
          ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err, wt, ep, ns);
  }
}

// Launches the GEMM (split over `sz` K slices of kc when sz > 1). a_mn / b_mn:
// A is stored K x M (lda >= M), B K x N (ldb >= N), read MN-major by the
// tensor cores (tcgen05 engine only).
int launch_gemm(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B,
                int ldb, float* C, int ldc, float alpha, float beta, int kc, int sz, float* work,
                cudaStream_t st, bool a_mn = false, bool b_mn = false,
                const TcEpi* epi = nullptr) {
  if (epi && (g_gemm_engine == 0 || a_mn || b_mn || sz != 1 || beta != 0.f))
    return sfail(PF_ERR_UNSUPPORTED, "pfs_gemm: the fused epilogue needs the tcgen05 engine, "
                                     "K-major operands, one K slice and beta = 0");
  if (g_gemm_engine == 0 && (a_mn || b_mn))
    return sfail(PF_ERR_UNSUPPORTED, "pfs_gemm: MN-major operands need the tcgen05 engine");
  if (g_gemm_engine == 0) {
    const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, sz);
    if (grid.y > 65535) return sfail(PF_ERR_INVALID, "pfs_gemm: M too large");
    k_gemm_bf16<<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, kc, work);
    return PF_OK;
  }
  static int* err = nullptr;
  if (!err && cudaGetSymbolAddress((void**)&err, g_tc_err) != cudaSuccess)
    return sfail(PF_ERR_CUDA, "pfs_gemm: cannot resolve the tensor-core error flag");
  static bool attr = false;
  if (!attr) {
    if (!(tc_prepare<256, false, false>() && tc_prepare<128, false, false>() &&
          tc_prepare<64, false, false>() && tc_prepare<32, false, false>() &&
          tc_prepare<256, true, true>() && tc_prepare<128, true, true>() &&
          tc_prepare<64, true, true>() && tc_prepare<256, false, true>() &&
          tc_prepare<128, false, true>() && tc_prepare<64, false, true>() &&
          tc_prepare<256, true, false>() && tc_prepare<128, true, false>() &&
          tc_prepare<64, true, false>() && tc_prepare<32, true, false>() &&
          tc_prepare<256, false, false, true>() && tc_prepare<128, false, false, true>() &&
          tc_prepare<64, false, false, true>() && tc_prepare<32, false, false, true>()))
      return cuda_status("pfs_gemm: shared memory attribute");
    attr = true;
  }
  if (sz == 1) kc = (K + TBK - 1) / TBK * TBK;  // one slice: the whole K range
  if (kc % TBK) return sfail(PF_ERR_INVALID, "pfs_gemm: K slice not a multiple of 64");
  const long long gy = (M + TBM - 1) / TBM;
  if (gy > 65535) return sfail(PF_ERR_INVALID, "pfs_gemm: M too large");
  // the narrowest tile that covers N, narrowed further (down to 32 columns)
  // while the grid has fewer blocks than SMs
  int bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  while (bn > 32 && gy * ((N + bn - 1) / bn) * sz < 148) bn /= 2;
  if (b_mn && bn < 64) bn = 64;  // an MN-major B is loaded in 64-wide strips
  CUtensorMap ta, tb;
  // K-major: rows of K elements, box 64 (K) x tile rows; MN-major: rows of
  // MN elements, box 64 (MN) x 64 (K)
  const bool ok = (a_mn ? tc_map(&ta, A, M, K, lda, TBK) : tc_map(&ta, A, K, M, lda, TBM)) &&
                  (b_mn ? tc_map(&tb, B, N, K, ldb, TBK) : tc_map(&tb, B, K, N, ldb, bn));
  if (!ok) return sfail(PF_ERR_CUDA, "pfs_gemm: cuTensorMapEncodeTiled failed");
  const dim3 grid((N + bn - 1) / bn, (unsigned)gy, sz);
  if (epi)
    tc_launch<false, false, true>(bn, grid, st, ta, tb, M, N, K, C, ldc, alpha, beta, kc, work,
                                  err, *epi);
  else if (a_mn && b_mn)
    tc_launch<true, true>(bn, grid, st, ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err);
  else if (a_mn)
    tc_launch<true, false>(bn, grid, st, ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err);
  else if (b_mn)
    tc_launch<false, true>(bn, grid, st, ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err);
  else
    tc_launch<false, false>(bn, grid, st, ta, tb, M, N, K, C, ldc, alpha, beta, kc, work, err);
  return PF_OK;
}

unsigned grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g > 148LL * 32) g = 148LL * 32;
  return (unsigned)(g < 1 ? 1 : g);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace

extern "C" {

const char* pfs_last_error(void) { return g_err.c_str(); }

int pfs_gemm_engine(int engine) {
  const int old = g_gemm_engine;
  if (engine == 0 || engine == 1) g_gemm_engine = engine;
  return old;
}

int pfs_gemm_wait_test(int on) {
  const int old = g_gemm_wait_test;
  if (on == 0 || on == 1) g_gemm_wait_test = on;
  return old;
}

int pfs_gemm_timeouts(int* count, int reset) {
  if (!count) return sfail(PF_ERR_INVALID, "pfs_gemm_timeouts: NULL");
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_err, sizeof v) != cudaSuccess) return cuda_status("pfs_gemm_timeouts");
  if (reset) {
    const int z = 0;
    if (cudaMemcpyToSymbol(g_tc_err, &z, sizeof z) != cudaSuccess) return cuda_status("pfs_gemm_timeouts");
  }
  *count = v;
  return PF_OK;
}

int pfs_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C,
                  int ldc, float alpha, float beta, void* stream) {
  if (M < 0 || N < 0 || K < 0 || (M && N && (!A || !B || !C)))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16: bad sizes or NULL operand");
  if (K % 32 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N)
    return sfail(PF_ERR_INVALID,
                 "pfs_gemm_bf16: K must be a multiple of 32, lda/ldb multiples of 8 and >= K");
  if (!aligned16(A) || !aligned16(B))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16: A and B must be 16-byte aligned");
  if (!M || !N) return PF_OK;
  if (K == 0) {
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16: K must be positive");
  }
  const int rc = launch_gemm(M, N, K, (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb,
                             C, ldc, alpha, beta, K, 1, nullptr, (cudaStream_t)stream);
  if (rc) return rc;
  return cuda_status("pfs_gemm_bf16");
}

int pfs_gemm_bf16_splitk(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                         float* C, int ldc, float alpha, float beta, int splits, float* work,
                         int64_t work_floats, void* stream) {
  if (splits <= 1) return pfs_gemm_bf16(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, stream);
  if (M < 0 || N < 0 || K < 1 || (M && N && (!A || !B || !C)) || !work || splits > 65535)
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_splitk: bad sizes or NULL operand");
  if (K % 32 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N)
    return sfail(PF_ERR_INVALID,
                 "pfs_gemm_bf16_splitk: K must be a multiple of 32, lda/ldb multiples of 8");
  if (!aligned16(A) || !aligned16(B))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_splitk: A and B must be 16-byte aligned");
  if ((long long)splits * M * N > work_floats)
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_splitk: work holds fewer than splits*M*N floats");
  if (!M || !N) return PF_OK;
  const int g = g_gemm_engine ? TBK : 32;  // K-tile of the engine
  const int kc = ((K + splits - 1) / splits + g - 1) / g * g;
  const int sz = (K + kc - 1) / kc;  // every slice non-empty
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (sz == 1) {
    rc = launch_gemm(M, N, K, (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C, ldc,
                     alpha, beta, K, 1, nullptr, st);
  } else {
    rc = launch_gemm(M, N, K, (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C, ldc,
                     alpha, beta, kc, sz, work, st);
    if (!rc)
      k_splitk_reduce<<<grid_for((long long)M * N, 256), 256, 0, st>>>(M, N, sz, work, C, ldc,
                                                                        beta);
  }
  if (rc) return rc;
  return cuda_status("pfs_gemm_bf16_splitk");
}

int pfs_gemm_bf16_ex(int M, int N, int K, const void* A, int lda, int a_mn, const void* B,
                     int ldb, int b_mn, float* C, int ldc, float alpha, float beta, int splits,
                     float* work, int64_t work_floats, void* stream) {
  if (!a_mn && !b_mn)
    return pfs_gemm_bf16_splitk(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, splits, work,
                                work_floats, stream);
  if (M < 0 || N < 0 || K < 1 || (M && N && (!A || !B || !C)) || splits < 1 || splits > 65535 ||
      (splits > 1 && !work))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_ex: bad sizes or NULL operand");
  if (K % 32 || lda % 8 || ldb % 8 || ldc < N || lda < (a_mn ? M : K) || ldb < (b_mn ? N : K))
    return sfail(PF_ERR_INVALID,
                 "pfs_gemm_bf16_ex: K must be a multiple of 32, lda/ldb multiples of 8 and at "
                 "least the operand's row length");
  if (!aligned16(A) || !aligned16(B))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_ex: A and B must be 16-byte aligned");
  if (splits > 1 && (long long)splits * M * N > work_floats)
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_ex: work holds fewer than splits*M*N floats");
  if (!M || !N) return PF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int kc = ((K + splits - 1) / splits + TBK - 1) / TBK * TBK;
  const int sz = (K + kc - 1) / kc;
  int rc = launch_gemm(M, N, K, (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C,
                       ldc, alpha, beta, sz == 1 ? K : kc, sz, sz == 1 ? nullptr : work, st,
                       a_mn != 0, b_mn != 0);
  if (!rc && sz > 1)
    k_splitk_reduce<<<grid_for((long long)M * N, 256), 256, 0, st>>>(M, N, sz, work, C, ldc, beta);
  if (rc) return rc;
  return cuda_status("pfs_gemm_bf16_ex");
}

int pfs_gemm_bf16_bias_act(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                           const float* bias, int relu, float* y32, void* y16, int ldy,
                           void* stream) {
  if (M < 0 || N < 0 || K < 1 || (M && N && (!A || !B || !y32)))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_bias_act: bad sizes or NULL operand");
  if (K % 32 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldy < N)
    return sfail(PF_ERR_INVALID,
                 "pfs_gemm_bf16_bias_act: K must be a multiple of 32, lda/ldb multiples of 8 "
                 "and >= K");
  if (!aligned16(A) || !aligned16(B))
    return sfail(PF_ERR_INVALID, "pfs_gemm_bf16_bias_act: A and B must be 16-byte aligned");
  if (!M || !N) return PF_OK;
  const TcEpi ep{bias, relu, (__nv_bfloat16*)y16};
  const int rc = launch_gemm(M, N, K, (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B,
                             ldb, y32, ldy, 1.0f, 0.0f, K, 1, nullptr, (cudaStream_t)stream,
                             false, false, &ep);
  if (rc) return rc;
  return cuda_status("pfs_gemm_bf16_bias_act");
}

int pfs_im2col(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
               const void* x, void* col, int Kp, void* stream) {
  if (nb < 1 || H < 1 || W < 1 || C < 1 || kh < 1 || kw < 1 || stride < 1 || ph < 0 || pw < 0 ||
      !x || !col || Kp < kh * kw * C)
    return sfail(PF_ERR_INVALID, "pfs_im2col: bad arguments");
  const int Ho = (H + 2 * ph - kh) / stride + 1, Wo = (W + 2 * pw - kw) / stride + 1;
  if (Ho < 1 || Wo < 1) return sfail(PF_ERR_INVALID, "pfs_im2col: empty output");
  const long long n = (long long)nb * Ho * Wo * Kp;
  cudaStream_t st = (cudaStream_t)stream;
  if (Kp % 8 == 0 && n / 8 < (1LL << 31) && aligned16(col)) {
    const int rows = nb * Ho * Wo;
    if (C % 8 == 0 && aligned16(x))
      k_im2col8<true><<<grid_for(n / 8, 256), 256, 0, st>>>(rows, H, W, C, kh, kw, stride, ph, pw,
                                                           Ho, Wo, (const __nv_bfloat16*)x,
                                                           (__nv_bfloat16*)col, Kp);
    else
      k_im2col8<false><<<grid_for(n / 8, 256), 256, 0, st>>>(rows, H, W, C, kh, kw, stride, ph,
                                                            pw, Ho, Wo, (const __nv_bfloat16*)x,
                                                            (__nv_bfloat16*)col, Kp);
  } else {
    k_im2col<<<grid_for(n, 256), 256, 0, st>>>(nb, H, W, C, kh, kw, stride, ph, pw, Ho, Wo,
                                               (const __nv_bfloat16*)x, (__nv_bfloat16*)col, Kp);
  }
  return cuda_status("pfs_im2col");
}

int pfs_col2im(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
               const float* dcol, int Kp, float* dx, void* stream) {
  if (nb < 1 || H < 1 || W < 1 || C < 1 || kh < 1 || kw < 1 || stride < 1 || ph < 0 || pw < 0 ||
      !dcol || !dx || Kp < kh * kw * C)
    return sfail(PF_ERR_INVALID, "pfs_col2im: bad arguments");
  const int Ho = (H + 2 * ph - kh) / stride + 1, Wo = (W + 2 * pw - kw) / stride + 1;
  if (Ho < 1 || Wo < 1) return sfail(PF_ERR_INVALID, "pfs_col2im: empty output");
  const long long n = (long long)nb * H * W * C;
  cudaStream_t st = (cudaStream_t)stream;
  if (C % 8 == 0 && Kp % 4 == 0 && n < (1LL << 31) && (long long)nb * Ho * Wo * Kp < (1LL << 31) &&
      aligned16(dcol) && aligned16(dx))
    k_col2im8<<<grid_for(n / 8, 256), 256, 0, st>>>(nb, H, W, C, kh, kw, stride, ph, pw, Ho, Wo,
                                                    dcol, Kp, dx);
  else
    k_col2im<<<grid_for(n, 256), 256, 0, st>>>(nb, H, W, C, kh, kw, stride, ph, pw, Ho, Wo, dcol,
                                               Kp, dx);
  return cuda_status("pfs_col2im");
}

int pfs_bias_act(int64_t M, int N, const float* x, const float* bias, int relu, float* y32,
                 void* y16, void* stream) {
  if (M < 0 || N < 1 || !x || (!y32 && !y16)) return sfail(PF_ERR_INVALID, "pfs_bias_act: bad arguments");
  k_bias_act<<<grid_for(M * N, 256), 256, 0, (cudaStream_t)stream>>>(M, N, x, bias, relu, y32,
                                                                     (__nv_bfloat16*)y16);
  return cuda_status("pfs_bias_act");
}

int pfs_act_bwd(int64_t M, int N, const float* dy, const float* y, int relu, float* d32, void* d16,
                float* dbias, float* part, int row_blocks, void* stream) {
  if (M < 1 || N < 1 || !dy || (relu && !y) || row_blocks < 1 || row_blocks > 65535 ||
      (dbias && !part))
    return sfail(PF_ERR_INVALID, "pfs_act_bwd: bad arguments");
  k_act_bwd<<<dim3((N + 31) / 32, row_blocks), dim3(32, 8), 0, (cudaStream_t)stream>>>(
      M, N, dy, y, relu, d32, (__nv_bfloat16*)d16, dbias ? part : nullptr);
  if (dbias) k_colsum<<<N, 256, 0, (cudaStream_t)stream>>>(row_blocks, N, part, dbias);
  return cuda_status("pfs_act_bwd");
}

int pfs_transpose_bf16(int R, int Cc, const void* in, int ldi, void* out, int ldo, void* stream) {
  if (R < 1 || Cc < 1 || !in || !out || ldi < Cc || ldo < R)
    return sfail(PF_ERR_INVALID, "pfs_transpose_bf16: bad arguments");
  const int rows = (ldo + 31) / 32;  // cover the zero fill up to ldo
  k_transpose_bf16<<<dim3((Cc + 31) / 32, rows), dim3(32, 8), 0, (cudaStream_t)stream>>>(
      R, Cc, (const __nv_bfloat16*)in, ldi, (__nv_bfloat16*)out, ldo);
  return cuda_status("pfs_transpose_bf16");
}

int pfs_to_bf16(int64_t n, const float* x, void* y, void* stream) {
  if (n < 0 || (n && (!x || !y))) return sfail(PF_ERR_INVALID, "pfs_to_bf16: bad arguments");
  if (!n) return PF_OK;
  k_to_bf16<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, x, (__nv_bfloat16*)y);
  return cuda_status("pfs_to_bf16");
}

int pfs_upsample2(int64_t nb, int W, int C, const void* x, void* y, void* stream) {
  if (nb < 1 || W < 1 || C < 1 || !x || !y) return sfail(PF_ERR_INVALID, "pfs_upsample2: bad arguments");
  k_upsample2<<<grid_for(nb * 2 * W * C, 256), 256, 0, (cudaStream_t)stream>>>(
      nb, W, C, (const __nv_bfloat16*)x, (__nv_bfloat16*)y);
  return cuda_status("pfs_upsample2");
}

int pfs_upsample2_bwd(int64_t nb, int W, int C, const float* dy, float* dx, void* stream) {
  if (nb < 1 || W < 1 || C < 1 || !dy || !dx) return sfail(PF_ERR_INVALID, "pfs_upsample2_bwd: bad arguments");
  k_upsample2_bwd<<<grid_for(nb * W * C, 256), 256, 0, (cudaStream_t)stream>>>(nb, W, C, dy, dx);
  return cuda_status("pfs_upsample2_bwd");
}

int pfs_mse(int64_t rows, int used, int ld, const float* y, const float* t, float* grad,
            float* loss_parts, int nparts, void* stream) {
  if (rows < 1 || used < 1 || ld < used || !y || !t || !grad || !loss_parts || nparts < 1)
    return sfail(PF_ERR_INVALID, "pfs_mse: bad arguments");
  k_mse<<<nparts, 256, 0, (cudaStream_t)stream>>>(rows, used, ld, y, t, grad, loss_parts);
  return cuda_status("pfs_mse");
}

int pfs_adam(int64_t n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2,
             float eps, int step, float wd, void* w16, void* stream) {
  if (n < 1 || !w || !g || !m || !v || step < 1) return sfail(PF_ERR_INVALID, "pfs_adam: bad arguments");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, w, g, m, v, lr, b1, b2, eps, c1,
                                                             c2, wd, (__nv_bfloat16*)w16);
  return cuda_status("pfs_adam");
}

}  // extern "C"
