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
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

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

// One dispersive medium as the E kernel sees it (simulation.py:572-636):
// its cells occupy compact indices [base, base + count); its polarisation
// state lives at P + poff as [level 0/1][pole][component][count].
template <typename T>
struct MediumT {
  long long base, count, poff;
  int npole;
  T inv;   // 1 / (eps0 * eps_inf), rounded to T as the reference's weak scalar
  T ce;    // dt / (eps_inf * eps0) in table mode
  T a[kMaxPoles], b[kMaxPoles], c[kMaxPoles];
};

// Arguments of one H + E step (split or fused kernels).
template <typename T>
struct StepArgs {
  int nx, ny, nz;
  T dx, dy, dz;  // derivative divisors (1 on a collapsed axis)
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
  // psi: E terms Ex_y, Ex_z, Ey_z, Ey_x, Ez_x, Ez_y; H terms Hx_y, Hx_z,
  // Hy_z, Hy_x, Hz_x, Hz_y (rustbackend.py:200-207 order)
  T* psiE[6];
  const T* psiHin[6];
  T* psiHout[6];
  // ADE
  const MediumT<T>* media;
  int n_media;
  T* P;
  int lvl;  // polarisation level holding P^n (n & 1)
};

enum CeMode { kCeCell1 = 0, kCeCell3 = 1, kCeTable = 2 };

}  // namespace pfb
