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
#pragma once

#include "cell_update.cuh"

namespace pfb {

// Load f[id + off] only when the neighbour exists (cond), else 0.
template <typename T>
__device__ __forceinline__ T ld_if(const T* f, long long id, long long off, bool cond) {
  return cond ? f[id + off] : T(0);
}

// H pass: H^{n+1/2} = H^{n-1/2} - ch (curl E^n + psi).
template <typename T>
__global__ void __launch_bounds__(256) k_h_split(const __grid_constant__ StepArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const long long sy = a.nz, sx = (long long)a.ny * a.nz;
  const long long id = i * sx + j * sy + k;
  const bool hx = i + 1 < a.nx, hy = j + 1 < a.ny, hz = k + 1 < a.nz;
  const T ex = a.Ein[0][id], ey = a.Ein[1][id], ez = a.Ein[2][id];
  a.Hout[0][id] = upd_hx<T>(a, i, j, k, a.Hin[0][id], ld_if(a.Ein[2], id, sy, hy), ez,
                            ld_if(a.Ein[1], id, 1, hz), ey, true);
  a.Hout[1][id] = upd_hy<T>(a, i, j, k, a.Hin[1][id], ld_if(a.Ein[0], id, 1, hz), ex,
                            ld_if(a.Ein[2], id, sx, hx), ez, true);
  a.Hout[2][id] = upd_hz<T>(a, i, j, k, a.Hin[2][id], ld_if(a.Ein[1], id, sx, hx), ey,
                            ld_if(a.Ein[0], id, sy, hy), ex, true);
}

// E pass: E^{n+1} = E^n + ce (curl H^{n+1/2} + psi), then ADE.
template <typename T, int CE, bool ADE>
__global__ void __launch_bounds__(256) k_e_split(const __grid_constant__ StepArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const long long sy = a.nz, sx = (long long)a.ny * a.nz;
  const long long id = i * sx + j * sy + k;
  T K[3];
  long long g;
  cell_coeffs<T, CE, ADE>(a, id, K, g);
  const T hx = a.Hin[0][id], hy = a.Hin[1][id], hz = a.Hin[2][id];
  const bool lx = i > 0, ly = j > 0, lz = k > 0;
  T en[3] = {a.Ein[0][id], a.Ein[1][id], a.Ein[2][id]};
  T e[3];
  e[0] = upd_ex<T>(a, i, j, k, en[0], K[0], hz, ld_if(a.Hin[2], id, -sy, ly), hy,
                   ld_if(a.Hin[1], id, -1, lz));
  e[1] = upd_ey<T>(a, i, j, k, en[1], K[1], hx, ld_if(a.Hin[0], id, -1, lz), hz,
                   ld_if(a.Hin[2], id, -sx, lx));
  e[2] = upd_ez<T>(a, i, j, k, en[2], K[2], hy, ld_if(a.Hin[1], id, -sx, lx), hx,
                   ld_if(a.Hin[0], id, -sy, ly));
  if (ADE && g >= 0) ade_apply<T>(a, g, en, e);
  a.Eout[0][id] = e[0];
  a.Eout[1][id] = e[1];
  a.Eout[2][id] = e[2];
}

}  // namespace pfb
