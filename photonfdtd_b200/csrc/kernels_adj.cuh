// kernels_adj.cuh - the reverse (adjoint) step of the 3D engine.
//
// The forward step n is linear in the fields for fixed coefficients:
//   H^{n+1/2} = H^{n-1/2} - ch (curl E^n + psi_H)          (H pass)
//   E^{n+1}   = E^n + K (curl H^{n+1/2} + psi_E)           (E pass)
// with psi' = b psi + c d for every CPML term (simulation.py:1252-1309). Its
// transpose runs backwards in time on adjoint fields lamE / lamH and psi
// adjoints, and the gradient of a loss J with respect to the per-cell E
// coefficient K is  dJ/dK(cell) = sum_n sum_c lamE_c^{n+1} * g_c^n  where
// g_c^n = curl + psiA' - psiB' is what K multiplied in step n. Reverse-mode
// differentiation of the reference's step (jaxbackend.py:666-722 differentiates
// the same step with jax.grad) gives exactly these recurrences.
//
// Per reverse step n (k_adj_e, then k_adj_h):
//  * k_adj_e: x_c = lamE_c + (gathered H-term adjoints of step n+1) + the
//    loss's sources on E^{n+1}; grad += sum_c x_c g_c^n (g from the recorded
//    H^{n+1/2} and psi_E of step n); the adjoints of the E update's two
//    difference quotients per component go to gE[6], psi_E adjoints updated.
//  * k_adj_h: y_c = lamH_c + (gathered gE) + sources on H^{n+1/2}; the H
//    update's difference-quotient adjoints go to gH[6], psi_H adjoints.
// A difference d = (f_hi - f_lo) / dl sends +adj(d)/dl to f_hi and -adj(d)/dl
// to f_lo; the gathers read the neighbour cell's quotient adjoint. Terms and
// cells outside the reference's loop extents contribute nothing (their
// quotient adjoints are stored as zero).
#pragma once

#include "cell_update.cuh"
#include "kernels_aux.cuh"

namespace pfb {

template <typename T>
struct AdjState {
  const T* Hrec[3];     // H^{n+1/2} recorded in the replay of step n
  const T* psiErec[6];  // psi_E after step n (compact, like psiE)
  T* lamE[3];
  T* lamH[3];
  T* gE[6];   // quotient adjoints of the E update: Ex A, Ex B, Ey A, Ey B, Ez A, Ez B
  T* gH[6];   // of the H update: Hx A, Hx B, Hy A, Hy B, Hz A, Hz B
  T* lpE[6];  // psi adjoints (compact, like psiE / psiH)
  T* lpH[6];
  double* grad;  // dJ/dK: per component (Ex cells, then Ey, then Ez) or summed
  long long ncell;
  long long gstride;  // ncell: one gradient per component; 0: the three summed
  T idl[3];      // 1 / dl per axis
};

// Term layout of component c (E or H): term A differentiates field comp
// fa[c] along axis axa[c], term B field comp fb[c] along axb[c] (Ex: dHz/dy,
// dHy/dz; Ey: dHx/dz, dHz/dx; Ez: dHy/dx, dHx/dy; H likewise with E).
__device__ __forceinline__ int term_axis_a(int c) { return c == 0 ? 1 : (c == 1 ? 2 : 0); }
__device__ __forceinline__ int term_axis_b(int c) { return c == 0 ? 2 : (c == 1 ? 0 : 1); }
__device__ __forceinline__ int term_comp_a(int c) { return c == 0 ? 2 : (c == 1 ? 0 : 1); }
__device__ __forceinline__ int term_comp_b(int c) { return c == 0 ? 1 : (c == 1 ? 2 : 0); }

// Transpose of one component's curl update f' = f + K (curl + psiA' - psiB')
// given x = adj(f'): quotient adjoints (qa, qb) and the psi adjoint updates.
// mapsA / mapsB: the compact psi index of each term (-1: no CPML state).
template <typename T>
__device__ __forceinline__ void curl_transpose(T x, T K, bool rA, bool rB, long long qA,
                                               long long qB, T bA, T cA, T bB, T cB, T* lpA,
                                               T* lpB, T& qa, T& qb) {
  qa = rA ? mul_rn(K, x) : T(0);
  qb = rB ? mul_rn(-K, x) : T(0);
  if (rA && qA >= 0) {
    const T ap = fma_rn(K, x, lpA[qA]);
    qa = fma_rn(cA, ap, qa);
    lpA[qA] = mul_rn(bA, ap);
  }
  if (rB && qB >= 0) {
    const T ap = fma_rn(-K, x, lpB[qB]);
    qb = fma_rn(cB, ap, qb);
    lpB[qB] = mul_rn(bB, ap);
  }
}

template <typename T, int CE>
__global__ void __launch_bounds__(256) k_adj_e(const __grid_constant__ StepArgs<T> a,
                                               const __grid_constant__ AdjState<T> s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const int n[3] = {a.nx, a.ny, a.nz};
  const int pos[3] = {i, j, k};
  const long long st[3] = {(long long)a.ny * a.nz, a.nz, 1};
  const long long id = i * st[0] + j * st[1] + k;
  const T dl[3] = {a.dx, a.dy, a.dz};
  T K[3];
  uint32_t w;
  cell_coeffs<T, CE, false>(a, nullptr, id, K, w);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // adj(E_c^{n+1}): identity part + the H update of step n+1 (forward
    // differences of E: d(cell) = (E(cell + e) - E(cell)) / dl)
    T x = s.lamE[c][id];
    {
      // H terms reading E_c: Ex <- Hy A (z), Hz B (y); Ey <- Hx B (z), Hz A (x);
      // Ez <- Hx A (y), Hy B (x)
      const int t0 = c == 0 ? 2 : (c == 1 ? 1 : 0), ax0 = c == 0 ? 2 : (c == 1 ? 2 : 1);
      const int t1 = c == 0 ? 5 : (c == 1 ? 4 : 3), ax1 = c == 0 ? 1 : (c == 1 ? 0 : 0);
      const T* g0 = s.gH[t0];
      const T* g1 = s.gH[t1];
      const T lo0 = pos[ax0] >= 1 ? g0[id - st[ax0]] : T(0);
      const T lo1 = pos[ax1] >= 1 ? g1[id - st[ax1]] : T(0);
      x = fma_rn(sub_rn(lo0, g0[id]), s.idl[ax0], x);
      x = fma_rn(sub_rn(lo1, g1[id]), s.idl[ax1], x);
    }
    const int axA = term_axis_a(c), axB = term_axis_b(c);
    const bool rA = n[axA] > 1, rB = n[axB] > 1;
    const bool upd = (!rA || pos[axA] >= 1) && (!rB || pos[axB] >= 1) && (rA || rB);
    T qa = T(0), qb = T(0);
    if (upd) {
      // g = curl + psiA' - psiB' of step n, from the recorded H^{n+1/2}
      const T* HA = s.Hrec[term_comp_a(c)];
      const T* HB = s.Hrec[term_comp_b(c)];
      const T dA = rA ? div_rn(sub_rn(HA[id], HA[id - st[axA]]), dl[axA]) : T(0);
      const T dB = rB ? div_rn(sub_rn(HB[id], HB[id - st[axB]]), dl[axB]) : T(0);
      T g = sub_rn(dA, dB);
      const long long qA = rA ? psi_index<T>(a.mape[axA], a.npe, axA, i, j, k, a.ny, a.nz) : -1;
      const long long qB = rB ? psi_index<T>(a.mape[axB], a.npe, axB, i, j, k, a.ny, a.nz) : -1;
      if (qA >= 0) g = add_rn(g, s.psiErec[2 * c][qA]);
      if (qB >= 0) g = sub_rn(g, s.psiErec[2 * c + 1][qB]);
      const double gc = __dmul_rn((double)x, (double)g);
      if (gc != 0.0) s.grad[c * s.gstride + id] = __dadd_rn(s.grad[c * s.gstride + id], gc);
      curl_transpose<T>(x, K[c], rA, rB, qA, qB, rA ? a.be[axA][pos[axA]] : T(0),
                        rA ? a.cpe[axA][pos[axA]] : T(0), rB ? a.be[axB][pos[axB]] : T(0),
                        rB ? a.cpe[axB][pos[axB]] : T(0), s.lpE[2 * c], s.lpE[2 * c + 1], qa,
                        qb);
    }
    s.gE[2 * c][id] = qa;
    s.gE[2 * c + 1][id] = qb;
    s.lamE[c][id] = x;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_adj_h(const __grid_constant__ StepArgs<T> a,
                                               const __grid_constant__ AdjState<T> s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= a.nz || j >= a.ny) return;
  const int n[3] = {a.nx, a.ny, a.nz};
  const int pos[3] = {i, j, k};
  const long long st[3] = {(long long)a.ny * a.nz, a.nz, 1};
  const long long id = i * st[0] + j * st[1] + k;
  const T K = -a.ch;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // adj(H_c^{n+1/2}): identity part + the E update of step n (backward
    // differences of H: d(cell) = (H(cell) - H(cell - e)) / dl)
    T y = s.lamH[c][id];
    {
      // E terms reading H_c: Hx <- Ey A (z), Ez B (y); Hy <- Ex B (z), Ez A (x);
      // Hz <- Ex A (y), Ey B (x)
      const int t0 = c == 0 ? 2 : (c == 1 ? 1 : 0), ax0 = c == 0 ? 2 : (c == 1 ? 2 : 1);
      const int t1 = c == 0 ? 5 : (c == 1 ? 4 : 3), ax1 = c == 0 ? 1 : (c == 1 ? 0 : 0);
      const T* g0 = s.gE[t0];
      const T* g1 = s.gE[t1];
      const T hi0 = pos[ax0] + 1 < n[ax0] ? g0[id + st[ax0]] : T(0);
      const T hi1 = pos[ax1] + 1 < n[ax1] ? g1[id + st[ax1]] : T(0);
      y = fma_rn(sub_rn(g0[id], hi0), s.idl[ax0], y);
      y = fma_rn(sub_rn(g1[id], hi1), s.idl[ax1], y);
    }
    const int axA = term_axis_a(c), axB = term_axis_b(c);
    const bool rA = n[axA] > 1, rB = n[axB] > 1;
    const bool upd = (!rA || pos[axA] < n[axA] - 1) && (!rB || pos[axB] < n[axB] - 1) && (rA || rB);
    T qa = T(0), qb = T(0);
    if (upd) {
      const long long qA = rA ? psi_index<T>(a.maph[axA], a.nph, axA, i, j, k, a.ny, a.nz) : -1;
      const long long qB = rB ? psi_index<T>(a.maph[axB], a.nph, axB, i, j, k, a.ny, a.nz) : -1;
      curl_transpose<T>(y, K, rA, rB, qA, qB, rA ? a.bh[axA][pos[axA]] : T(0),
                        rA ? a.cph[axA][pos[axA]] : T(0), rB ? a.bh[axB][pos[axB]] : T(0),
                        rB ? a.cph[axB][pos[axB]] : T(0), s.lpH[2 * c], s.lpH[2 * c + 1], qa,
                        qb);
    }
    s.gH[2 * c][id] = qa;
    s.gH[2 * c + 1][id] = qb;
    s.lamH[c][id] = y;
  }
}

// The loss's source on the sampled fields of one DFT monitor at sample q:
// d J / d f(cell) = dt * sum_f (Re G_f Re ph_f + Im G_f Im ph_f) with
// G = dJ/dRe(acc) + i dJ/dIm(acc) per frequency (acc += ph f dt), added to
// the adjoint of every sampled component of family fam (0: E, 1: H).
template <typename T>
__global__ void k_adj_dft_src(DftRegion r, const double* cot, const double* ph, int n_freq,
                              double dt, int fam, T* l0, T* l1, T* l2, int ny, int nz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= r.ncell * r.ncomp) return;
  const long long cell = t % r.ncell;
  const int qc = (int)(t / r.ncell);
  const int c = r.comps[qc];
  if ((c >= 3) != (fam == 1)) return;
  double v = 0.0;
  for (int f = 0; f < n_freq; ++f) {
    const double* g = cot + (((long long)qc * n_freq + f) * r.ncell + cell) * 2;
    v = __dadd_rn(v, __dadd_rn(__dmul_rn(g[0], ph[2 * f]), __dmul_rn(g[1], ph[2 * f + 1])));
  }
  v = __dmul_rn(v, dt);
  const long long ck = cell % r.count[2];
  const long long rest = cell / r.count[2];
  const long long cj = rest % r.count[1];
  const long long ci = rest / r.count[1];
  const long long id = ((long long)(r.start[0] + ci * r.stride[0]) * ny +
                        (r.start[1] + cj * r.stride[1])) * nz +
                       (r.start[2] + ck * r.stride[2]);
  T* l = (c % 3) == 0 ? l0 : ((c % 3) == 1 ? l1 : l2);
  l[id] = to_real(__dadd_rn((double)l[id], v), T());
}

// The loss's source on one recorded field snapshot (a FieldMonitor frame):
// vals[cell] = dJ / d f(cell) over the region, added to the adjoint field.
template <typename T>
__global__ void k_adj_region_src(DftRegion r, const double* vals, T* l, int ny, int nz) {
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= r.ncell) return;
  const long long ck = cell % r.count[2];
  const long long rest = cell / r.count[2];
  const long long cj = rest % r.count[1];
  const long long ci = rest / r.count[1];
  const long long id = ((long long)(r.start[0] + ci * r.stride[0]) * ny +
                        (r.start[1] + cj * r.stride[1])) * nz +
                       (r.start[2] + ck * r.stride[2]);
  l[id] = to_real(__dadd_rn((double)l[id], vals[cell]), T());
}

// ---- flux losses ----------------------------------------------------------
// A flux monitor adds S dA dt per step, S = E_t1 H_t2 - E_t2 H_t1 summed over
// its plane (E at n+1, H at n+1/2; t1, t2 the tangential axes in cyclic
// order, as k_flux_sample_batch). With c = dJ/dflux * dA * dt its sources on
// the adjoint are dS/dE_t1 = H_t2, dS/dE_t2 = -H_t1, dS/dH_t2 = E_t1,
// dS/dH_t1 = -E_t2 at every plane cell.
__device__ __forceinline__ long long flux_cell(const FluxPlane& p, long long t, int ny, int nz) {
  const int u = (int)(t / p.n1), w = (int)(t % p.n1);
  if (p.axis == 0) return ((long long)p.idx * ny + u) * nz + w;
  if (p.axis == 1) return ((long long)u * ny + p.idx) * nz + w;
  return ((long long)u * ny + w) * nz + p.idx;
}

// E_t1, E_t2 of the plane after a step, into a record of 2 * n0 * n1 reals.
template <typename T>
__global__ void k_flux_plane_record(FluxPlane p, const T* E0, const T* E1, const T* E2, T* dst,
                                    int ny, int nz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)p.n0 * p.n1;
  if (t >= np) return;
  const long long id = flux_cell(p, t, ny, nz);
  const T* E[3] = {E0, E1, E2};
  dst[t] = E[(p.axis + 1) % 3][id];
  dst[np + t] = E[(p.axis + 2) % 3][id];
}

// fam 0: lamE_t1 += c H_t2, lamE_t2 -= c H_t1 from the recorded H (full
// fields); fam 1: lamH_t2 += c E_t1, lamH_t1 -= c E_t2 from the plane record.
template <typename T>
__global__ void k_adj_flux_src(FluxPlane p, double c, int fam, const T* H0, const T* H1,
                               const T* H2, const T* erec, T* l0, T* l1, T* l2, int ny, int nz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)p.n0 * p.n1;
  if (t >= np) return;
  const long long id = flux_cell(p, t, ny, nz);
  const int t1 = (p.axis + 1) % 3, t2 = (p.axis + 2) % 3;
  T* l[3] = {l0, l1, l2};
  double a, b;  // sources on component t1, t2
  if (fam == 0) {
    const T* H[3] = {H0, H1, H2};
    a = c * (double)H[t2][id];
    b = -c * (double)H[t1][id];
  } else {
    b = c * (double)erec[t];        // on H_t2
    a = -c * (double)erec[np + t];  // on H_t1
  }
  l[t1][id] = to_real(__dadd_rn((double)l[t1][id], a), T());
  l[t2][id] = to_real(__dadd_rn((double)l[t2][id], b), T());
}

}  // namespace pfb
