// smoothing.cu - the diagonal subpixel permittivity tensor on the GPU.
//
// The device form of the host precompute in photonfdtd_b200/smoothing.py,
// which follows the reference's smooth_permittivity (src/photonfdtd/
// smoothing.py:87-172) for scenes made of boxes. Per native cell: the
// arithmetic and harmonic means eps_a, eps_h of the permittivity over
// factor sub-cells per resolved axis; the interface normal is the
// normalised np.gradient of eps_a; eps_ii = eps_a + (eps_h - eps_a) * n_i^2.
// Results equal NumPy's bit for bit, because every operation is the same
// IEEE double operation in the same order:
//  - a sub-cell takes the permittivity of the last box whose fine-grid index
//    span holds it (later structures overwrite earlier ones when stamped);
//  - numpy's block mean over the reshaped sub-cell axes adds, for each index
//    of the outer sub-cell axes in order, the sum of the innermost resolved
//    sub-cell axis (started from 0) to a running total started from 0, then
//    divides by the sub-cell count; the harmonic mean does the same on 1/v
//    and takes 1/mean;
//  - np.gradient with a uniform spacing h: (f[p+1] - f[p-1]) / (2.0 * h)
//    inside, one-sided (f[1] - f[0]) / h and (f[n-1] - f[n-2]) / h at the
//    ends, zero along a collapsed axis;
//  - |g| = sqrt((gx^2 + gy^2) + gz^2); cells with |g| <= max(1e-9 max|g|,
//    DBL_MIN) get no normal; eps_ii = eps_a + (eps_h - eps_a) * (n_i * n_i),
//    rounded once to the output type.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/pfb200.h"

namespace {

thread_local std::string g_smooth_err;

int sfail(int code, const std::string& msg) {
  g_smooth_err = msg;
  return code;
}

unsigned blocks_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148LL * 32) g = 148LL * 32;
  return (unsigned)(g < 1 ? 1 : g);
}

struct SmoothDims {
  int n[3];      // native cells per axis
  int f[3];      // sub-cells per native cell per axis (1 on a collapsed axis)
  int inner;     // the innermost axis with f > 1 (2 when none)
  int outer[2];  // the other two axes, ascending
  double h[3];   // gradient spacing per resolved axis
};

__device__ __forceinline__ double sub_eps(int fi, int fj, int fk, double bg, int nbox,
                                          const int* __restrict__ span,
                                          const double* __restrict__ eps) {
  double v = bg;
  for (int s = 0; s < nbox; ++s) {
    const int* p = span + 6 * s;
    if (fi >= p[0] && fi < p[1] && fj >= p[2] && fj < p[3] && fk >= p[4] && fk < p[5])
      v = eps[s];
  }
  return v;
}

__global__ void k_smooth_means(SmoothDims d, double bg, int nbox, const int* __restrict__ span,
                               const double* __restrict__ eps, double* __restrict__ ea,
                               double* __restrict__ eh) {
  const long long total = (long long)d.n[0] * d.n[1] * d.n[2];
  const double cnt = (double)(d.f[0] * d.f[1] * d.f[2]);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c[3] = {(int)(t / ((long long)d.n[1] * d.n[2])), (int)((t / d.n[2]) % d.n[1]),
                      (int)(t % d.n[2])};
    double sa = 0.0, sh = 0.0;
    for (int u = 0; u < d.f[d.outer[0]]; ++u)
      for (int w = 0; w < d.f[d.outer[1]]; ++w) {
        double ta = 0.0, th = 0.0;
        for (int q = 0; q < d.f[d.inner]; ++q) {
          int s[3];
          s[d.outer[0]] = u;
          s[d.outer[1]] = w;
          s[d.inner] = q;
          const double v = sub_eps(c[0] * d.f[0] + s[0], c[1] * d.f[1] + s[1],
                                   c[2] * d.f[2] + s[2], bg, nbox, span, eps);
          ta = __dadd_rn(ta, v);
          th = __dadd_rn(th, __ddiv_rn(1.0, v));
        }
        sa = __dadd_rn(sa, ta);
        sh = __dadd_rn(sh, th);
      }
    ea[t] = __ddiv_rn(sa, cnt);
    eh[t] = __ddiv_rn(1.0, __ddiv_rn(sh, cnt));
  }
}

// np.gradient of f along every axis at flat cell t (zero on collapsed axes).
__device__ __forceinline__ void grad3(const SmoothDims& d, const double* __restrict__ f,
                                      long long t, double g[3]) {
  const long long stride[3] = {(long long)d.n[1] * d.n[2], d.n[2], 1};
  const int c[3] = {(int)(t / stride[0]), (int)((t / d.n[2]) % d.n[1]), (int)(t % d.n[2])};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int n = d.n[a], p = c[a];
    const long long s = stride[a];
    if (n == 1) {
      g[a] = 0.0;
    } else if (p == 0) {
      g[a] = __ddiv_rn(__dsub_rn(f[t + s], f[t]), d.h[a]);
    } else if (p == n - 1) {
      g[a] = __ddiv_rn(__dsub_rn(f[t], f[t - s]), d.h[a]);
    } else {
      g[a] = __ddiv_rn(__dsub_rn(f[t + s], f[t - s]), __dmul_rn(2.0, d.h[a]));
    }
  }
}

__device__ __forceinline__ double norm3(const double g[3]) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(g[0], g[0]), __dmul_rn(g[1], g[1])),
                              __dmul_rn(g[2], g[2])));
}

// |grad eps_a| per cell and its maximum (non-negative doubles order like
// their bit patterns, so an integer atomicMax finds it).
__global__ void k_smooth_gmag(SmoothDims d, const double* __restrict__ ea,
                              double* __restrict__ gm, unsigned long long* gmax) {
  const long long total = (long long)d.n[0] * d.n[1] * d.n[2];
  unsigned long long m = 0ull;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    double g[3];
    grad3(d, ea, t, g);
    const double v = norm3(g);
    gm[t] = v;
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_down_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(gmax, m);
}

template <typename R>
__global__ void k_smooth_out(SmoothDims d, const double* __restrict__ ea,
                             const double* __restrict__ eh, const double* __restrict__ gm,
                             double thr, R* __restrict__ oxx, R* __restrict__ oyy,
                             R* __restrict__ ozz) {
  const long long total = (long long)d.n[0] * d.n[1] * d.n[2];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    double g[3];
    grad3(d, ea, t, g);
    const double gmt = gm[t];
    const double inv = gmt > thr ? __ddiv_rn(1.0, gmt) : 0.0;
    const double a = ea[t], delta = __dsub_rn(eh[t], a);
    R* out[3] = {oxx, oyy, ozz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double nrm = __dmul_rn(g[c], inv);
      out[c][t] = (R)__dadd_rn(a, __dmul_rn(delta, __dmul_rn(nrm, nrm)));
    }
  }
}

}  // namespace

extern "C" {

const char* pf_smooth_last_error(void) { return g_smooth_err.c_str(); }

int pf_smooth_boxes(int nx, int ny, int nz, int factor, double background, int n_box,
                    const int32_t* spans, const double* eps_box, double hx, double hy,
                    double hz, int out_bytes, void* out_xx, void* out_yy, void* out_zz) {
  if (nx < 1 || ny < 1 || nz < 1 || factor < 1 || n_box < 0 || (n_box && (!spans || !eps_box)) ||
      (out_bytes != 4 && out_bytes != 8) || !out_xx || !out_yy || !out_zz)
    return sfail(PF_ERR_INVALID, "pf_smooth_boxes: bad arguments");
  SmoothDims d;
  d.n[0] = nx;
  d.n[1] = ny;
  d.n[2] = nz;
  const double h[3] = {hx, hy, hz};
  int last = 2;
  bool any = false;
  for (int a = 0; a < 3; ++a) {
    d.f[a] = d.n[a] > 1 ? factor : 1;
    d.h[a] = h[a];
    if (d.n[a] > 1 && !(h[a] > 0.0))
      return sfail(PF_ERR_INVALID, "pf_smooth_boxes: spacing must be positive");
    if (d.f[a] > 1) {
      last = a;
      any = true;
    }
    if ((long long)d.n[a] * d.f[a] >= (1LL << 31))
      return sfail(PF_ERR_INVALID, "pf_smooth_boxes: grid too large");
  }
  d.inner = any ? last : 2;
  for (int a = 0, o = 0; a < 3; ++a)
    if (a != d.inner) d.outer[o++] = a;
  const long long n = (long long)nx * ny * nz;
  int* dspan = nullptr;
  double *deps = nullptr, *ea = nullptr, *eh = nullptr, *gm = nullptr;
  unsigned long long* gmax = nullptr;
  void* dout[3] = {nullptr, nullptr, nullptr};
  void* hout[3] = {out_xx, out_yy, out_zz};
  cudaStream_t st = nullptr;
  int rc = PF_OK;
  auto cuda_ok = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    rc = sfail(e == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA,
               std::string("pf_smooth_boxes: ") + what + ": " + cudaGetErrorString(e));
    return false;
  };
  do {
    if (!cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream")) break;
    const size_t nb = (size_t)(n_box ? n_box : 1);
    if (!cuda_ok(cudaMalloc((void**)&dspan, nb * 6 * sizeof(int)), "cudaMalloc")) break;
    if (!cuda_ok(cudaMalloc((void**)&deps, nb * sizeof(double)), "cudaMalloc")) break;
    if (!cuda_ok(cudaMalloc((void**)&ea, (size_t)n * 8), "cudaMalloc")) break;
    if (!cuda_ok(cudaMalloc((void**)&eh, (size_t)n * 8), "cudaMalloc")) break;
    if (!cuda_ok(cudaMalloc((void**)&gm, (size_t)n * 8), "cudaMalloc")) break;
    if (!cuda_ok(cudaMalloc((void**)&gmax, 8), "cudaMalloc")) break;
    bool ok = true;
    for (int c = 0; c < 3 && ok; ++c)
      ok = cuda_ok(cudaMalloc(&dout[c], (size_t)n * out_bytes), "cudaMalloc");
    if (!ok) break;
    if (n_box) {
      if (!cuda_ok(cudaMemcpyAsync(dspan, spans, (size_t)n_box * 6 * sizeof(int),
                                   cudaMemcpyHostToDevice, st), "upload")) break;
      if (!cuda_ok(cudaMemcpyAsync(deps, eps_box, (size_t)n_box * sizeof(double),
                                   cudaMemcpyHostToDevice, st), "upload")) break;
    }
    if (!cuda_ok(cudaMemsetAsync(gmax, 0, 8, st), "memset")) break;
    const unsigned g = blocks_for(n);
    k_smooth_means<<<g, 256, 0, st>>>(d, background, n_box, dspan, deps, ea, eh);
    k_smooth_gmag<<<g, 256, 0, st>>>(d, ea, gm, gmax);
    if (!cuda_ok(cudaGetLastError(), "launch")) break;
    unsigned long long mbits = 0;
    if (!cuda_ok(cudaMemcpyAsync(&mbits, gmax, 8, cudaMemcpyDeviceToHost, st), "read max")) break;
    if (!cuda_ok(cudaStreamSynchronize(st), "means / gradient")) break;
    double gmx;
    memcpy(&gmx, &mbits, 8);
    const double tiny = gmx * 1e-9;
    const double dmin = 2.2250738585072014e-308;  // DBL_MIN, numpy's finfo(float64).tiny
    const double thr = tiny > dmin ? tiny : dmin;
    if (out_bytes == 4)
      k_smooth_out<float><<<g, 256, 0, st>>>(d, ea, eh, gm, thr, (float*)dout[0],
                                             (float*)dout[1], (float*)dout[2]);
    else
      k_smooth_out<double><<<g, 256, 0, st>>>(d, ea, eh, gm, thr, (double*)dout[0],
                                              (double*)dout[1], (double*)dout[2]);
    if (!cuda_ok(cudaGetLastError(), "launch")) break;
    for (int c = 0; c < 3 && ok; ++c)
      ok = cuda_ok(cudaMemcpyAsync(hout[c], dout[c], (size_t)n * out_bytes,
                                   cudaMemcpyDeviceToHost, st), "download");
    if (!ok) break;
    cuda_ok(cudaStreamSynchronize(st), "tensor");
  } while (false);
  if (st) cudaStreamSynchronize(st);
  cudaFree(dspan);
  cudaFree(deps);
  cudaFree(ea);
  cudaFree(eh);
  cudaFree(gm);
  cudaFree(gmax);
  for (void* p : dout) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  return rc;
}

}  // extern "C"
