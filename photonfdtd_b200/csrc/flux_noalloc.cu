// flux_noalloc.cu - plane Poynting flux with no device allocation.
//
// pf_flux_plane_noalloc is the flux monitor's per-step reduction
// (k_flux_sample_batch + the fixed-order fold of k_flux_flush) as a standalone
// call for programs that must not allocate device memory on the call path.
// Typical examples: a process whose device memory is owned by another
// allocator (a framework's caching pool, or a serving process that reserved
// its whole budget up front); code that only borrows field buffers it did not
// create and has no allocator handle; a tight time loop where a cudaMalloc
// would add a device-wide synchronisation. The per-block partial sums that
// the engine keeps in scratch it allocates are kept here in a fixed
// file-scope device array instead.
#include <cstdio>
#include <mutex>

#include "../../include/pfb200.h"
#include "common.cuh"
#include "kernels_aux.cuh"

using namespace pfb;

namespace {

// Partial-sum scratch shared by every call on a device: one double per block
// of 256 plane cells, so at most 65,536 * 256 = 16,777,216 plane cells per
// call (e.g. a 4096 x 4096 plane). 512 KB, held by each GPU that loads this
// library until the process exits.
constexpr int kNoAllocBlocks = 65536;
constexpr int kNoAllocThreads = 256;
static __device__ __align__(256) double g_flux_partials[kNoAllocBlocks];

// Device address of g_flux_partials per device. In host code the array's
// name is only a host-side stand-in, so kernels always get this address.
// It is looked up again on every call made outside a stream capture (the
// lookup allocates nothing), so a module reloaded after cudaDeviceReset is
// followed; a capture uses the address the last uncaptured call on that
// device found. A failed lookup is never kept.
constexpr int kMaxDevices = 64;
double* g_partials_ptr[kMaxDevices];
std::mutex g_ptr_mutex;
thread_local char g_err[256];

// Per-block partial sums of S = E_t1*H_t2 - E_t2*H_t1 over the plane, with
// the same roundings and block layout as the engine's flux sampling.
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_flux_partials_static(FluxPlane p,
                                                                          Fields6<T> f, int ny,
                                                                          int nz, double* part) {
  __shared__ double sh[8];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < (long long)p.n0 * p.n1) {
    const int u = (int)(t / p.n1), w = (int)(t % p.n1);
    long long id;
    int e1, h2, e2, h1;
    if (p.axis == 0) {
      id = ((long long)p.idx * ny + u) * nz + w;
      e1 = 1; h2 = 5; e2 = 2; h1 = 4;
    } else if (p.axis == 1) {
      id = ((long long)u * ny + p.idx) * nz + w;
      e1 = 2; h2 = 3; e2 = 0; h1 = 5;
    } else {
      id = ((long long)u * ny + w) * nz + p.idx;
      e1 = 0; h2 = 4; e2 = 1; h1 = 3;
    }
    v = (double)sub_rn(mul_rn(f.f[e1][id], f.f[h2][id]), mul_rn(f.f[e2][id], f.f[h1][id]));
  }
  v = block_sum<T>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_flux_total_static(const double* part, int nblk,
                                                                       double dA, double dt,
                                                                       double* out) {
  __shared__ double sh[8];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) v += part[b];
  v = block_sum<T>(v, sh);
  if (threadIdx.x == 0) {
    const T s = to_real(v, T());
    *out = __dmul_rn((double)mul_rn(s, (T)dA), dt);
  }
}

int set_error(int code, const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

}  // namespace

extern "C" {

const char* pf_noalloc_last_error(void) { return g_err; }

int pf_flux_plane_noalloc(int real_bytes, int nx, int ny, int nz, const void* const fields[6],
                          int axis, int idx, double dA, double dt, double* out, void* stream) {
  if (real_bytes != 4 && real_bytes != 8) return set_error(PF_ERR_INVALID, "real_bytes must be 4 or 8");
  if (nx < 1 || ny < 1 || nz < 1 || axis < 0 || axis > 2)
    return set_error(PF_ERR_INVALID, "bad grid shape or axis");
  const int dims[3] = {nx, ny, nz};
  if (idx < 0 || idx >= dims[axis]) return set_error(PF_ERR_INVALID, "plane index out of range");
  if (!fields || !out) return set_error(PF_ERR_INVALID, "fields and out must be device pointers");
  for (int c = 0; c < 6; ++c)
    if (!fields[c]) return set_error(PF_ERR_INVALID, "a field pointer is NULL");
  FluxPlane p;
  p.axis = axis;
  p.idx = idx;
  p.n0 = axis == 0 ? ny : nx;
  p.n1 = axis == 2 ? ny : nz;
  const long long cells = (long long)p.n0 * p.n1;
  const long long nblk = (cells + kNoAllocThreads - 1) / kNoAllocThreads;
  if (nblk > kNoAllocBlocks)
    return set_error(PF_ERR_INVALID,
                     "plane has more than 16,777,216 cells (the fixed scratch holds 65,536 "
                     "partial sums of 256 cells)");
  p.nblk = (int)nblk;

  int dev = 0;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess) return set_error(PF_ERR_CUDA, cudaGetErrorString(rc));
  if (dev < 0 || dev >= kMaxDevices) return set_error(PF_ERR_UNSUPPORTED, "device index too large");
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  rc = cudaStreamIsCapturing(st, &cap);
  if (rc != cudaSuccess) return set_error(PF_ERR_CUDA, cudaGetErrorString(rc));
  double* part = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_ptr_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
      // Resolve the scratch array's device address with the device current.
      double* p_dev = nullptr;
      rc = cudaGetSymbolAddress((void**)&p_dev, g_flux_partials);
      if (rc != cudaSuccess) return set_error(PF_ERR_CUDA, cudaGetErrorString(rc));
      g_partials_ptr[dev] = p_dev;
    } else if (g_partials_ptr[dev] == nullptr) {
      return set_error(PF_ERR_STATE,
                       "first call on this device made during a stream capture: call once "
                       "outside the capture first");
    }
    part = g_partials_ptr[dev];
  }
  if (real_bytes == 4) {
    Fields6<float> f;
    for (int c = 0; c < 6; ++c) f.f[c] = (const float*)fields[c];
    k_flux_partials_static<float><<<p.nblk, kNoAllocThreads, 0, st>>>(p, f, ny, nz, part);
    k_flux_total_static<float><<<1, kNoAllocThreads, 0, st>>>(part, p.nblk, dA, dt, out);
  } else {
    Fields6<double> f;
    for (int c = 0; c < 6; ++c) f.f[c] = (const double*)fields[c];
    k_flux_partials_static<double><<<p.nblk, kNoAllocThreads, 0, st>>>(p, f, ny, nz, part);
    k_flux_total_static<double><<<1, kNoAllocThreads, 0, st>>>(part, p.nblk, dA, dt, out);
  }
  rc = cudaGetLastError();
  return rc == cudaSuccess ? PF_OK : set_error(PF_ERR_CUDA, cudaGetErrorString(rc));
}

}  // extern "C"
