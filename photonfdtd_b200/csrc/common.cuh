// common.cuh - shared types and exactly-rounded arithmetic for the engine.
//
// Every field update in this engine reproduces the reference NumPy path's
// rounding sequence (src/photonfdtd/simulation.py:1138-1309): each add,
// subtract, multiply and divide is one IEEE round-to-nearest operation, and
// none is contracted into an FMA. The *_rn intrinsics below guarantee that
// regardless of -fmad, so a float32 run matches the reference float32 run
// bit for bit wherever the reference's own operation order is used.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pfb {

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// Correctly rounded a / d given r = RN(1/d), by Markstein's correction:
// q0 = RN(a * r), rem = a - q0 * d (exact with one FMA), q = RN(q0 + rem * r).
// The host enables it for a divisor d only after checking that it reproduces
// IEEE a / d for every float significand of a; the identity is invariant
// under scaling a by powers of two while a stays in [2^-100, 2^90) and the
// residual cannot underflow. qdiv_fast first scales a by 2^64 (exact), so
// every |a| < 2^26 - zero and subnormals included - lands in that window,
// and scales the quotient back by 2^-64, which is exact while the quotient
// is normal: guaranteed for d <= 2^-23 (the host requires d in
// [2^-30, 2^-23]). copysign keeps the sign of a zero quotient. The caller
// guarantees |a| < 2^26 (qdiv_ok); qdiv checks it itself.
constexpr float kQdivLimit = 0x1p26f;
__device__ __forceinline__ float qdiv_fast(float a, float d, float r) {
  const float as = __fmul_rn(a, 0x1p64f);
  const float q0 = __fmul_rn(as, r);
  const float rem = __fmaf_rn(-q0, d, as);
  return copysignf(__fmul_rn(__fmaf_rn(rem, r, q0), 0x1p-64f), a);
}
__device__ __forceinline__ float qdiv(float a, float d, float r, bool fast) {
  if (fast && fabsf(a) < kQdivLimit) return qdiv_fast(a, d, r);
  return __fdiv_rn(a, d);
}
__device__ __forceinline__ double qdiv_fast(double a, double d, double) { return __ddiv_rn(a, d); }
__device__ __forceinline__ double qdiv(double a, double d, double, bool) { return __ddiv_rn(a, d); }
// Two exact quotients sharing one range check and one branch: both by the
// reciprocal path when it applies to both, else each by qdiv.
template <typename T>
__device__ __forceinline__ void qdiv2(T a0, T d0, T r0, bool f0, T a1, T d1, T r1, bool f1,
                                      T& q0, T& q1);
// Whether every numerator of a cell may take qdiv_fast.
__device__ __forceinline__ bool qdiv_ok(float m) { return m < kQdivLimit; }
__device__ __forceinline__ bool qdiv_ok(double) { return false; }
__device__ __forceinline__ float absmax(float a, float b) { return fmaxf(fabsf(a), fabsf(b)); }
__device__ __forceinline__ double absmax(double a, double b) { return fmax(fabs(a), fabs(b)); }
template <typename T>
__device__ __forceinline__ void qdiv2(T a0, T d0, T r0, bool f0, T a1, T d1, T r1, bool f1,
                                      T& q0, T& q1) {
  if (f0 && f1 && qdiv_ok(absmax(a0, a1))) {
    q0 = qdiv_fast(a0, d0, r0);
    q1 = qdiv_fast(a1, d1, r1);
  } else {
    q0 = qdiv(a0, d0, r0, f0);
    q1 = qdiv(a1, d1, r1, f1);
  }
}

// Round a double to the field type (round to nearest even).
__device__ __forceinline__ float to_real(double v, float) { return __double2float_rn(v); }
__device__ __forceinline__ double to_real(double v, double) { return v; }

// F += v with v a double: the reference adds a float64 source value to a
// float32 cell in double precision and rounds once on store
// (simulation.py:1371-1372, numpy float32 + float64 -> float64).
template <typename T>
__device__ __forceinline__ T add_double(T f, double v) {
  return to_real(__dadd_rn((double)f, v), T());
}

constexpr int kMaxPoles = 8;
constexpr int kMaxMedia = 16;
constexpr uint32_t kDispersiveBit = 0x80000000u;

// One dispersive medium as the E kernel sees it (simulation.py:572-636).
// Its polarisation state is two arrays, one per time level: level L's record
// of a cell is at P + L * plev + poff + loc * 3 * npole, laid out
// [pole][component]. A step reads both levels and rewrites one, so the
// rewritten records of consecutive cells are contiguous and a warp's stores
// fill whole sectors (each medium's block starts 8-real aligned). A
// dispersive cell's word is kDispersiveBit | medium << kMediumShift | loc.
template <typename T>
struct MediumT {
  long long poff, count;
  int npole;
  T inv;   // 1 / (eps0 * eps_inf), rounded to T as the reference's weak scalar
  T ce;    // dt / (eps_inf * eps0) in table mode
  T a[kMaxPoles], b[kMaxPoles], c[kMaxPoles];
};
constexpr int kMediumShift = 27;
constexpr uint32_t kLocMask = (1u << kMediumShift) - 1u;

// Soft sources of one family (simulation.py:1367-1390). Sources sharing a
// (component, cell) form one group, applied in the reference's list order.
struct SourceGroups {
  const long long* cell;   // flat cell index per group
  const int* comp;         // 0..2 within the family (x, y, z)
  const int* start;        // group g owns sources [start[g], start[g+1])
  const int* wave_row;     // per source
  const double* amp;       // per source
  const double* wave;      // [row][n_steps]
  long long n_steps;
  int n_groups;
};

// A DFT monitor's region: start / stride / count per axis, the components.
struct DftRegion {
  int start[3], stride[3], count[3];
  long long ncell;
  int ncomp;
  int comps[6];
};

// Source groups and DFT monitors the split E pass handles itself.
constexpr int kInlineSrc = 8;
constexpr int kInlineDft = 4;

// Arguments of one H + E step (split or fused kernels).
template <typename T>
struct StepArgs {
  int nx, ny, nz;
  T dx, dy, dz;  // derivative divisors (1 on a collapsed axis)
  T rdx, rdy, rdz;      // RN(1/d) per axis
  bool fdx, fdy, fdz;   // reciprocal division verified exact for that axis
  T ch;          // dt / mu0 rounded to T; the H coefficient is -ch
  const T* Ein[3];
  const T* Hin[3];
  T* Eout[3];
  T* Hout[3];
  // E coefficients: ce[c] per cell (CELL1 repeats one array), or word/table
  const T* ce[3];
  const uint32_t* word;
  const T* table;
  const uint32_t* adeword;  // CELL1 + ADE: 0 = plain, else 1 + compact index
  // CPML: coefficients on the E and H staggers per axis, compact maps
  const T* be[3];
  const T* cpe[3];
  const T* bh[3];
  const T* cph[3];
  const int* mape[3];
  const int* maph[3];
  int npe[3], nph[3];
  // Bulk boxes: cells [b0, b1) per axis where the H (hb) or E (eb) update has
  // both difference terms and no CPML state; they take the straight-line path.
  int hb0[3], hb1[3], eb0[3], eb1[3];
  // psi: E terms Ex_y, Ex_z, Ey_z, Ey_x, Ez_x, Ez_y; H terms Hx_y, Hx_z,
  // Hy_z, Hy_x, Hz_x, Hz_y (rustbackend.py:200-207 order)
  T* psiE[6];
  const T* psiHin[6];
  T* psiHout[6];
  // ADE
  const MediumT<T>* media;
  int n_media;
  T* P;
  long long plev;  // reals per polarisation level
  int lvl;         // polarisation level holding P^n (n & 1)
  int wait_test;   // test hook of the TMA-staged step (pf_set_wait_test)
};

// Arguments of the split E pass's epilogue (the opt-in in-kernel sources
// and DFT sampling): the E-family soft sources of this step (group g at
// block isrc_blk[g], thread isrc_tid[g]) and the samples of the DFT monitors
// sampled at this step (ring slot idft_slot[m], -1: none). A separate kernel
// parameter, so the plain E pass does not carry it.
template <typename T>
struct EpiArgs {
  long long step;
  int n_isrc;
  int isrc_blk[kInlineSrc], isrc_tid[kInlineSrc];
  SourceGroups isrc;
  int n_idft;
  DftRegion idft[kInlineDft];
  T* idft_ring[kInlineDft];
  int idft_slot[kInlineDft];
};
// The epilogue parameter of k_e_split<..., EPI>: EpiArgs, or nothing.
struct NoEpi {};
template <typename T, bool EPI>
struct EpiParam {
  using type = EpiArgs<T>;
};
template <typename T>
struct EpiParam<T, false> {
  using type = NoEpi;
};

enum CeMode { kCeCell1 = 0, kCeCell3 = 1, kCeTable = 2 };

// Host: whether the float reciprocal division of qdiv is exact for divisor d
// (exhaustive check over all significands; defined in engine.cu).
bool host_recip_division_exact(float d);

}  // namespace pfb
