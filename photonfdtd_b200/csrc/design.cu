// design.cu - the density chain of topology optimisation on the GPU.
//
// The reference maps a raw design density rho to the physical density the
// permittivity is built from (src/photonfdtd/design.py):
//   conic_filter (:40-58): y = conv(rho, W) / conv(1, W), W[a, b] =
//     max(0, 1 - sqrt(a^2 + b^2) / R) for |a|, |b| <= r = ceil(R), a
//     same-size convolution with zero padding, normalised per cell so the
//     window edge is not biased toward void; R < 1 leaves rho unchanged;
//   tanh_projection (:61-72): p = (tanh(beta eta) + tanh(beta (y - eta))) /
//     (tanh(beta eta) + tanh(beta (1 - eta))); beta <= 0 leaves y unchanged.
// It differentiates them with JAX. Here both are CUDA kernels over a batch of
// n x n windows (one block per window, the window in shared memory), in
// float64, with a hand-written reverse pass: the projection's derivative
// beta (1 - tanh^2(beta (y - eta))) / den, then the transpose of the
// normalised convolution, which for the symmetric kernel W is the same
// zero-padded convolution applied to g / conv(1, W).
#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/pfb200.h"

namespace {

thread_local std::string g_derr;

int dfail(int code, const char* msg) {
  g_derr = msg;
  return code;
}

constexpr int kMaxWindow = 96;  // n <= 96: two n x n double arrays fit in shared memory
constexpr int kMaxRadius = 32;

struct DensityArgs {
  int n_inst, n, r;
  double R, beta, eta;
};

__device__ __forceinline__ double cone(int a, int b, double R) {
  const double w = 1.0 - sqrt((double)(a * a + b * b)) / R;
  return w > 0.0 ? w : 0.0;
}

// Filter of cell (i, j) of the window in x (shared memory): numerator and
// normaliser, both summed over in-window neighbours in row-major order.
__device__ __forceinline__ void filter_cell(const double* x, int n, int i, int j, int r, double R,
                                            double& num, double& den) {
  num = 0.0;
  den = 0.0;
  for (int a = -r; a <= r; ++a) {
    const int ii = i + a;
    if (ii < 0 || ii >= n) continue;
    for (int b = -r; b <= r; ++b) {
      const int jj = j + b;
      if (jj < 0 || jj >= n) continue;
      const double w = cone(a, b, R);
      num += w * x[ii * n + jj];
      den += w;
    }
  }
}

__device__ __forceinline__ double project(double y, double beta, double eta, double& dproj) {
  const double t0 = tanh(beta * eta);
  const double den = t0 + tanh(beta * (1.0 - eta));
  const double t = tanh(beta * (y - eta));
  dproj = beta * (1.0 - t * t) / den;
  return (t0 + t) / den;
}

__global__ void k_density_forward(DensityArgs p, const double* rho, double* out) {
  extern __shared__ double sm[];
  const int k = blockIdx.x;
  const int nn = p.n * p.n;
  const double* x = rho + (long long)k * nn;
  for (int c = threadIdx.x; c < nn; c += blockDim.x) sm[c] = x[c];
  __syncthreads();
  for (int c = threadIdx.x; c < nn; c += blockDim.x) {
    double y = sm[c];
    if (p.r >= 1) {
      double num, den;
      filter_cell(sm, p.n, c / p.n, c % p.n, p.r, p.R, num, den);
      y = num / den;
    }
    if (p.beta > 0.0) {
      double d;
      y = project(y, p.beta, p.eta, d);
    }
    out[(long long)k * nn + c] = y;
  }
}

__global__ void k_density_backward(DensityArgs p, const double* rho, const double* g_phys,
                                   double* g_rho) {
  extern __shared__ double sm[];
  double* xs = sm;
  double* ws = sm + p.n * p.n;
  const int k = blockIdx.x;
  const int nn = p.n * p.n;
  const double* x = rho + (long long)k * nn;
  const double* g = g_phys + (long long)k * nn;
  for (int c = threadIdx.x; c < nn; c += blockDim.x) xs[c] = x[c];
  __syncthreads();
  // w = dL/dy / conv(1, W) at every output cell (dL/dy through the projection)
  for (int c = threadIdx.x; c < nn; c += blockDim.x) {
    double num = xs[c], den = 1.0;
    if (p.r >= 1) filter_cell(xs, p.n, c / p.n, c % p.n, p.r, p.R, num, den);
    double gy = g[c];
    if (p.beta > 0.0) {
      double d;
      project(num / den, p.beta, p.eta, d);
      gy *= d;
    }
    ws[c] = gy / den;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < nn; c += blockDim.x) {
    double v = ws[c];
    if (p.r >= 1) {
      double unused;
      filter_cell(ws, p.n, c / p.n, c % p.n, p.r, p.R, v, unused);
    }
    g_rho[(long long)k * nn + c] = v;
  }
}

int check_args(int n_inst, int n, double radius, double beta, double eta, DensityArgs& p) {
  if (n_inst < 1 || n < 1) return dfail(PF_ERR_INVALID, "need n_inst >= 1 and n >= 1");
  if (n > kMaxWindow) return dfail(PF_ERR_INVALID, "window side n must be <= 96");
  if (!(radius >= 0.0) || !(beta >= 0.0) || !std::isfinite(eta))
    return dfail(PF_ERR_INVALID, "radius and beta must be >= 0, eta finite");
  p.n_inst = n_inst;
  p.n = n;
  p.R = radius;
  p.r = (int)std::ceil(radius);  // r < 1: no filtering, as the reference
  if (p.r > kMaxRadius) return dfail(PF_ERR_INVALID, "filter radius must be <= 32 cells");
  p.beta = beta;
  p.eta = eta;
  return PF_OK;
}

int launch_status(const char* what) {
  const cudaError_t rc = cudaGetLastError();
  if (rc == cudaSuccess) return PF_OK;
  g_derr = std::string(what) + ": " + cudaGetErrorString(rc);
  return PF_ERR_CUDA;
}

}  // namespace

extern "C" {

const char* pfd_last_error(void) { return g_derr.c_str(); }

int pfd_density_forward(int n_inst, int n, const double* rho, double radius, double beta,
                        double eta, double* rho_phys, void* stream) {
  DensityArgs p;
  int rc = check_args(n_inst, n, radius, beta, eta, p);
  if (rc) return rc;
  if (!rho || !rho_phys) return dfail(PF_ERR_INVALID, "NULL device pointer");
  const size_t smem = (size_t)n * n * sizeof(double);
  static bool attr = false;
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(
        k_density_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
        kMaxWindow * kMaxWindow * (int)sizeof(double));
    if (e != cudaSuccess) return dfail(PF_ERR_CUDA, cudaGetErrorString(e));
    attr = true;
  }
  k_density_forward<<<n_inst, 256, smem, (cudaStream_t)stream>>>(p, rho, rho_phys);
  return launch_status("pfd_density_forward");
}

int pfd_density_backward(int n_inst, int n, const double* rho, double radius, double beta,
                         double eta, const double* grad_phys, double* grad_rho, void* stream) {
  DensityArgs p;
  int rc = check_args(n_inst, n, radius, beta, eta, p);
  if (rc) return rc;
  if (!rho || !grad_phys || !grad_rho) return dfail(PF_ERR_INVALID, "NULL device pointer");
  const size_t smem = 2 * (size_t)n * n * sizeof(double);
  static bool attr = false;
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(
        k_density_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
        2 * kMaxWindow * kMaxWindow * (int)sizeof(double));
    if (e != cudaSuccess) return dfail(PF_ERR_CUDA, cudaGetErrorString(e));
    attr = true;
  }
  k_density_backward<<<n_inst, 256, smem, (cudaStream_t)stream>>>(p, rho, grad_phys, grad_rho);
  return launch_status("pfd_density_backward");
}

}  // extern "C"
