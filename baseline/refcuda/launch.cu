// launch.cu - host harness for the reference's own CUDA stepping kernels.
//
// The reference (rust/src/cuda.rs:29-265) keeps its Yee+CPML kernels as CUDA C
// source text compiled at run time by NVRTC with -DREAL=float|double. The
// build recipe next to this file extracts that text from the reference tree
// into a temporary file and compiles it, with REF_KERNEL_SRC naming it, into
// this translation unit; nothing of the reference is stored here. The host
// side below is this project's restatement of the reference's driver
// (Inner::run_steps, cuda.rs:298-341, and the constructor, cuda.rs:436-500):
// same buffers, same argument lists, same launch shape (cudarc's
// LaunchConfig::for_num_elems: 1024 threads, ceil(n / 1024) blocks), same
// per-step order H pass, H sources, E pass, E sources.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

#ifndef REAL
#error "REAL must be float or double"
#endif
#include REF_KERNEL_SRC

namespace {

struct RefCuda {
  int nx = 0, ny = 0, nz = 0;
  long long n = 0;
  real* f[6] = {};      // Ex, Ey, Ez, Hx, Hy, Hz
  real* psi[12] = {};   // E terms 0-5, H terms 6-11 (cuda.rs:457-461 order)
  real* be[3] = {};
  real* cpe[3] = {};
  real* bh[3] = {};
  real* cph[3] = {};
  int* me[3] = {};
  int* mh[3] = {};
  real* ce_field = nullptr;
  int* src_comp = nullptr;
  int* src_idx = nullptr;
  int* src_rows = nullptr;
  real* src_vals = nullptr;
  int pe[3] = {}, ph[3] = {};
  real ch = 0, inv_d[3] = {};
  int n_src = 0;
  long long n_steps_total = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[2] = {};
};

char g_err[512];

int fail(cudaError_t e, const char* what) {
  snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
  return -1;
}

template <typename U>
int upload(U** dst, const U* src, size_t count) {
  const size_t bytes = (count ? count : 1) * sizeof(U);
  cudaError_t e = cudaMalloc((void**)dst, bytes);
  if (e != cudaSuccess) return fail(e, "cudaMalloc");
  if (src && count) e = cudaMemcpy(*dst, src, count * sizeof(U), cudaMemcpyHostToDevice);
  else e = cudaMemset(*dst, 0, bytes);
  return e == cudaSuccess ? 0 : fail(e, "upload");
}

int count_pml(const int* map, int len) {
  int c = 0;
  for (int i = 0; i < len; ++i) c += map[i] >= 0;
  return c;
}

}  // namespace

extern "C" {

const char* refcuda_last_error(void) { return g_err; }

int refcuda_real_size(void) { return (int)sizeof(real); }

// Tables as rustbackend._build_tables makes them (rustbackend.py:135-166):
// ce_field (nx*ny*nz), per axis b/c for E and H (length = that axis' size),
// compact CPML maps (int32, -1 in the bulk), sources as component code
// (0-5 = Ex..Hz), (i, j, k) and a value table (n_src x n_steps_total).
int refcuda_create(int nx, int ny, int nz, const real* ce_field, const real* const* b_e,
                   const real* const* c_e, const real* const* b_h, const real* const* c_h,
                   const int* const* maps_e, const int* const* maps_h, real ch_field, real dx,
                   real dy, real dz, int n_src, const int* src_comp, const int* src_idx,
                   const real* src_vals, long long n_steps_total, void** out) {
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || n_src < 1 || n_steps_total < 1) {
    snprintf(g_err, sizeof g_err, "refcuda_create: bad sizes");
    return -1;
  }
  RefCuda* r = new RefCuda;
  r->nx = nx;
  r->ny = ny;
  r->nz = nz;
  r->n = (long long)nx * ny * nz;
  const int dims[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    r->pe[a] = count_pml(maps_e[a], dims[a]);
    r->ph[a] = count_pml(maps_h[a], dims[a]);
  }
  const long long X = nx, Y = ny, Z = nz;
  const long long sizes[12] = {X * r->pe[1] * Z, X * Y * r->pe[2], X * Y * r->pe[2],
                               r->pe[0] * Y * Z, r->pe[0] * Y * Z, X * r->pe[1] * Z,
                               X * r->ph[1] * Z, X * Y * r->ph[2], X * Y * r->ph[2],
                               r->ph[0] * Y * Z, r->ph[0] * Y * Z, X * r->ph[1] * Z};
  int rc = 0;
  for (int c = 0; c < 6 && !rc; ++c) rc = upload<real>(&r->f[c], nullptr, r->n);
  for (int q = 0; q < 12 && !rc; ++q) rc = upload<real>(&r->psi[q], nullptr, sizes[q]);
  for (int a = 0; a < 3 && !rc; ++a) {
    rc = upload(&r->be[a], b_e[a], dims[a]);
    if (!rc) rc = upload(&r->cpe[a], c_e[a], dims[a]);
    if (!rc) rc = upload(&r->bh[a], b_h[a], dims[a]);
    if (!rc) rc = upload(&r->cph[a], c_h[a], dims[a]);
    if (!rc) rc = upload(&r->me[a], maps_e[a], dims[a]);
    if (!rc) rc = upload(&r->mh[a], maps_h[a], dims[a]);
  }
  if (!rc) rc = upload(&r->ce_field, ce_field, r->n);
  if (!rc) rc = upload(&r->src_comp, src_comp, n_src);
  if (!rc) rc = upload(&r->src_idx, src_idx, 3 * (size_t)n_src);
  if (!rc) {
    int* rows = new int[n_src];
    for (int s = 0; s < n_src; ++s) rows[s] = s;  // cuda.rs:484-488
    rc = upload(&r->src_rows, rows, n_src);
    delete[] rows;
  }
  if (!rc) rc = upload(&r->src_vals, src_vals, (size_t)n_src * n_steps_total);
  r->ch = ch_field;
  r->inv_d[0] = (real)1 / dx;  // cuda.rs:494-495
  r->inv_d[1] = (real)1 / dy;
  r->inv_d[2] = (real)1 / dz;
  r->n_src = n_src;
  r->n_steps_total = n_steps_total;
  cudaError_t e;
  if (!rc && (e = cudaStreamCreate(&r->st)) != cudaSuccess) rc = fail(e, "stream");
  if (!rc && (e = cudaEventCreate(&r->ev[0])) != cudaSuccess) rc = fail(e, "event");
  if (!rc && (e = cudaEventCreate(&r->ev[1])) != cudaSuccess) rc = fail(e, "event");
  if (rc) {
    *out = r;  // the caller destroys it
    return rc;
  }
  *out = r;
  return 0;
}

// Steps [step0, step0 + n_sub) as Inner::run_steps does; when ms is given,
// the device time of the whole loop by CUDA events on the stream.
int refcuda_run(void* h, long long step0, long long n_sub, float* ms) {
  RefCuda* r = (RefCuda*)h;
  if (!r || step0 < 0 || n_sub < 0 || step0 + n_sub > r->n_steps_total) {
    snprintf(g_err, sizeof g_err, "refcuda_run: steps out of range");
    return -1;
  }
  const unsigned threads = 1024;
  const unsigned blocks = (unsigned)((r->n + threads - 1) / threads);
  const unsigned sblocks = (unsigned)((r->n_src + threads - 1) / threads);
  if (ms) cudaEventRecord(r->ev[0], r->st);
  for (long long step = step0; step < step0 + n_sub; ++step) {
    update_h<<<blocks, threads, 0, r->st>>>(
        r->f[0], r->f[1], r->f[2], r->f[3], r->f[4], r->f[5], r->psi[6], r->psi[7], r->psi[8],
        r->psi[9], r->psi[10], r->psi[11], r->bh[0], r->cph[0], r->bh[1], r->cph[1], r->bh[2],
        r->cph[2], r->mh[0], r->mh[1], r->mh[2], r->nx, r->ny, r->nz, r->ph[1], r->ph[2], r->ch,
        r->inv_d[0], r->inv_d[1], r->inv_d[2]);
    inject<<<sblocks, threads, 0, r->st>>>(r->f[0], r->f[1], r->f[2], r->f[3], r->f[4], r->f[5],
                                           r->src_comp, r->src_idx, r->src_rows, r->src_vals,
                                           r->n_src, r->n_steps_total, step, 0, r->ny, r->nz);
    update_e<<<blocks, threads, 0, r->st>>>(
        r->f[0], r->f[1], r->f[2], r->f[3], r->f[4], r->f[5], r->psi[0], r->psi[1], r->psi[2],
        r->psi[3], r->psi[4], r->psi[5], r->be[0], r->cpe[0], r->be[1], r->cpe[1], r->be[2],
        r->cpe[2], r->me[0], r->me[1], r->me[2], r->ce_field, r->nx, r->ny, r->nz, r->pe[1],
        r->pe[2], r->inv_d[0], r->inv_d[1], r->inv_d[2]);
    inject<<<sblocks, threads, 0, r->st>>>(r->f[0], r->f[1], r->f[2], r->f[3], r->f[4], r->f[5],
                                           r->src_comp, r->src_idx, r->src_rows, r->src_vals,
                                           r->n_src, r->n_steps_total, step, 1, r->ny, r->nz);
  }
  if (ms) cudaEventRecord(r->ev[1], r->st);
  cudaError_t e = cudaStreamSynchronize(r->st);
  if (e != cudaSuccess) return fail(e, "refcuda_run");
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "refcuda_run launch");
  if (ms && (e = cudaEventElapsedTime(ms, r->ev[0], r->ev[1])) != cudaSuccess)
    return fail(e, "refcuda_run timing");
  return 0;
}

int refcuda_read(void* h, int comp, real* dst) {
  RefCuda* r = (RefCuda*)h;
  if (!r || comp < 0 || comp > 5 || !dst) {
    snprintf(g_err, sizeof g_err, "refcuda_read: bad arguments");
    return -1;
  }
  cudaError_t e = cudaMemcpy(dst, r->f[comp], r->n * sizeof(real), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : fail(e, "refcuda_read");
}

void refcuda_destroy(void* h) {
  RefCuda* r = (RefCuda*)h;
  if (!r) return;
  for (auto* p : r->f) cudaFree(p);
  for (auto* p : r->psi) cudaFree(p);
  for (int a = 0; a < 3; ++a) {
    cudaFree(r->be[a]);
    cudaFree(r->cpe[a]);
    cudaFree(r->bh[a]);
    cudaFree(r->cph[a]);
    cudaFree(r->me[a]);
    cudaFree(r->mh[a]);
  }
  cudaFree(r->ce_field);
  cudaFree(r->src_comp);
  cudaFree(r->src_idx);
  cudaFree(r->src_rows);
  cudaFree(r->src_vals);
  if (r->ev[0]) cudaEventDestroy(r->ev[0]);
  if (r->ev[1]) cudaEventDestroy(r->ev[1]);
  if (r->st) cudaStreamDestroy(r->st);
  delete r;
}

}  // extern "C"
