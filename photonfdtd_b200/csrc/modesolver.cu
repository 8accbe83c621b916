// modesolver.cu - the full-vectorial waveguide mode operator on the GPU.
//
// The reference's mode solver (src/photonfdtd/mode.py:256-351) assembles the
// transverse-E operator P of Zhu & Brown (Opt. Express 10, 853, 2002) as a
// scipy sparse matrix from staggered difference matrices Uu, Uv (forward
// differences along z and y with a zero neighbour past the last node) and
// Vu = -Uu^T, Vv = -Uv^T, and calls ARPACK in shift-invert mode. Here P is
// applied matrix-free to a block of vectors. Expanding the reference's four
// blocks (P [u; v], u = E_z, v = E_y, flat index iy * nz + iz) and using
// that the y and z difference operators commute gives
//   a = Uv u,  b = Uu v
//   A = eps u + Vv a / k2,   B = eps v + Vu b / k2
//   C = (Vu A + Vv B - Vu Vv (a + b) / k2) / eps
//   P [u; v] = [k2 A - Vv b + Uu C ;  k2 B - Vu a + Uv C]
// (every fourth-order term of the blocks is in C), four stencil passes. The
// Chebyshev filter of the eigensolver (photonfdtd_b200/mode.py) runs its
// three-term recurrence on the device with the last pass fused into the
// recurrence's axpy.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/pfb200.h"

namespace {

thread_local std::string g_mode_error;

int mfail(int code, const char* fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_mode_error = buf;
  return code;
}

struct Grid2 {
  int ny, nz;
  long long n;  // ny * nz
  double idy, idz, ik2, k2;
};

// forward difference along z / y (zero neighbour past the last node)
__device__ __forceinline__ double fz(const double* f, long long id, int iz, const Grid2& g) {
  return ((iz + 1 < g.nz ? f[id + 1] : 0.0) - f[id]) * g.idz;
}
__device__ __forceinline__ double fy(const double* f, long long id, int iy, const Grid2& g) {
  return ((iy + 1 < g.ny ? f[id + g.nz] : 0.0) - f[id]) * g.idy;
}
// backward difference along z / y (zero neighbour before the first node)
__device__ __forceinline__ double bz(const double* f, long long id, int iz, const Grid2& g) {
  return (f[id] - (iz > 0 ? f[id - 1] : 0.0)) * g.idz;
}
__device__ __forceinline__ double by(const double* f, long long id, int iy, const Grid2& g) {
  return (f[id] - (iy > 0 ? f[id - g.nz] : 0.0)) * g.idy;
}

struct Work {
  double *a, *b, *A, *B, *w, *C;  // n * nvec each
};

// Thread t covers cell t % n of vector t / n.
__global__ void k_mode_p1(Grid2 g, const double* x, Work s, int nvec) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n * nvec) return;
  const long long c = t / g.n, id = t - c * g.n;
  const int iy = (int)(id / g.nz), iz = (int)(id - (long long)iy * g.nz);
  const double* u = x + c * 2 * g.n;
  const double* v = u + g.n;
  s.a[t] = fy(u, id, iy, g);
  s.b[t] = fz(v, id, iz, g);
}

__global__ void k_mode_p2(Grid2 g, const double* eps, const double* x, Work s, int nvec) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n * nvec) return;
  const long long c = t / g.n, id = t - c * g.n;
  const int iy = (int)(id / g.nz), iz = (int)(id - (long long)iy * g.nz);
  const double* u = x + c * 2 * g.n;
  const double* v = u + g.n;
  const double* a = s.a + c * g.n;
  const double* b = s.b + c * g.n;
  const double e = eps[id];
  const double vva = by(a, id, iy, g);
  s.A[t] = e * u[id] + vva * g.ik2;
  s.B[t] = e * v[id] + bz(b, id, iz, g) * g.ik2;
  s.w[t] = vva + by(b, id, iy, g);  // Vv (a + b)
}

__global__ void k_mode_p3(Grid2 g, const double* eps, Work s, int nvec) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n * nvec) return;
  const long long c = t / g.n, id = t - c * g.n;
  const int iy = (int)(id / g.nz), iz = (int)(id - (long long)iy * g.nz);
  const double* A = s.A + c * g.n;
  const double* B = s.B + c * g.n;
  const double* w = s.w + c * g.n;
  s.C[t] = (bz(A, id, iz, g) + by(B, id, iy, g) - bz(w, id, iz, g) * g.ik2) / eps[id];
}

// out = al * (P y) + be * y + ga * yprev  (yprev may be null)
__global__ void k_mode_p4(Grid2 g, const double* y, Work s, int nvec, double al, double be,
                          double ga, const double* yprev, double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n * nvec) return;
  const long long c = t / g.n, id = t - c * g.n;
  const int iy = (int)(id / g.nz), iz = (int)(id - (long long)iy * g.nz);
  const double* a = s.a + c * g.n;
  const double* b = s.b + c * g.n;
  const double* C = s.C + c * g.n;
  const double pu = g.k2 * s.A[t] - by(b, id, iy, g) + fz(C, id, iz, g);
  const double pv = g.k2 * s.B[t] - bz(a, id, iz, g) + fy(C, id, iy, g);
  const long long ou = c * 2 * g.n + id, ov = ou + g.n;
  double ru = al * pu + be * y[ou], rv = al * pv + be * y[ov];
  if (yprev) {
    ru += ga * yprev[ou];
    rv += ga * yprev[ov];
  }
  out[ou] = ru;
  out[ov] = rv;
}

Work carve(double* work, long long n, int nvec) {
  const long long m = n * nvec;
  return Work{work, work + m, work + 2 * m, work + 3 * m, work + 4 * m, work + 5 * m};
}

int launch_apply(const Grid2& g, const double* eps, const double* y, Work s, int nvec, double al,
                 double be, double ga, const double* yprev, double* out, cudaStream_t st) {
  const long long tot = g.n * nvec;
  const int B = 256;
  const unsigned grid = (unsigned)((tot + B - 1) / B);
  k_mode_p1<<<grid, B, 0, st>>>(g, y, s, nvec);
  k_mode_p2<<<grid, B, 0, st>>>(g, eps, y, s, nvec);
  k_mode_p3<<<grid, B, 0, st>>>(g, eps, s, nvec);
  k_mode_p4<<<grid, B, 0, st>>>(g, y, s, nvec, al, be, ga, yprev, out);
  const cudaError_t rc = cudaGetLastError();
  if (rc != cudaSuccess) return mfail(PF_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(rc));
  return PF_OK;
}

int make_grid(int ny, int nz, double dy, double dz, double k2, int nvec, Grid2& g) {
  if (ny < 1 || nz < 1 || nvec < 1 || !(dy > 0) || !(dz > 0) || !(k2 > 0))
    return mfail(PF_ERR_INVALID, "bad mode-operator arguments");
  g.ny = ny;
  g.nz = nz;
  g.n = (long long)ny * nz;
  if (g.n * nvec >= (1LL << 40)) return mfail(PF_ERR_INVALID, "block too large");
  g.idy = 1.0 / dy;
  g.idz = 1.0 / dz;
  g.k2 = k2;
  g.ik2 = 1.0 / k2;
  return PF_OK;
}

}  // namespace

extern "C" {

const char* pfm_last_error(void) { return g_mode_error.c_str(); }

int pfm_apply(int ny, int nz, double dy, double dz, double k2, const double* eps, const double* x,
              double* y, int nvec, double* work, void* stream) {
  Grid2 g;
  int rc = make_grid(ny, nz, dy, dz, k2, nvec, g);
  if (rc) return rc;
  if (!eps || !x || !y || !work || x == y) return mfail(PF_ERR_INVALID, "bad mode-operator buffers");
  return launch_apply(g, eps, x, carve(work, g.n, nvec), nvec, 1.0, 0.0, 0.0, nullptr, y,
                      (cudaStream_t)stream);
}

int pfm_chebyshev(int ny, int nz, double dy, double dz, double k2, const double* eps, double* x,
                  int nvec, int degree, double lo, double hi, double* work, void* stream) {
  Grid2 g;
  int rc = make_grid(ny, nz, dy, dz, k2, nvec, g);
  if (rc) return rc;
  if (!eps || !x || !work || degree < 1 || !(hi > lo))
    return mfail(PF_ERR_INVALID, "bad Chebyshev filter arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  const Work s = carve(work, g.n, nvec);
  const long long m = 2 * g.n * nvec;
  double* y0 = work + 6 * g.n * nvec;  // two more vectors of the block
  double* y1 = y0 + m;
  const double e = 0.5 * (hi - lo), c = 0.5 * (hi + lo);
  // T_1: (P x - c x) / e
  if ((rc = launch_apply(g, eps, x, s, nvec, 1.0 / e, -c / e, 0.0, nullptr, y1, st))) return rc;
  double* prev = x;  // T_{j-1}
  double* cur = y1;  // T_j
  double* spare = y0;
  for (int j = 1; j < degree; ++j) {
    // T_{j+1} = 2 (P - c) T_j / e - T_{j-1}
    if ((rc = launch_apply(g, eps, cur, s, nvec, 2.0 / e, -2.0 * c / e, -1.0, prev, spare, st)))
      return rc;
    double* t = prev;
    prev = cur;
    cur = spare;
    spare = t;
  }
  if (cur != x) {
    const cudaError_t r = cudaMemcpyAsync(x, cur, m * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (r != cudaSuccess) return mfail(PF_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(r));
  }
  return PF_OK;
}

}  // extern "C"
