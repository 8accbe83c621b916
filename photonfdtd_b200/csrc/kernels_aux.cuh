// kernels_aux.cuh - soft-source injection and the DFT / flux monitor kernels.
#pragma once

#include "common.cuh"

namespace pfb {

// ---------------------------------------------------------------------------
// Soft sources (simulation.py:1367-1390). Sources sharing a (component, cell)
// form one group; a group's sources are applied in the reference's list order,
// each as a double add rounded to the field type, so coincident dipoles round
// exactly as the reference's successive `F[i,j,k] += val` do.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_inject(SourceGroups s, T* f0, T* f1, T* f2, long long step) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n_groups) return;
  T* F = s.comp[g] == 0 ? f0 : (s.comp[g] == 1 ? f1 : f2);
  const long long c = s.cell[g];
  T v = F[c];
  for (int q = s.start[g]; q < s.start[g + 1]; ++q)
    v = add_double<T>(v, __dmul_rn(s.amp[q], s.wave[(long long)s.wave_row[q] * s.n_steps + step]));
  F[c] = v;
}

// ---------------------------------------------------------------------------
// DFT monitor (simulation.py:1116-1133). Each sampled step writes the region's
// values into a ring of pending samples; a flush folds the pending samples,
// oldest first, into the complex128 accumulators:
//   acc += (phase * f) * dt   per frequency, per cell
// with the same two roundings per real and imaginary part as numpy's
// complex128 * float32 -> complex128 product followed by * dt. Summation order
// over steps is the reference's, so the accumulators match bit for bit.
// ---------------------------------------------------------------------------
// The six field components of one time level, by component code.
template <typename T>
struct Fields6 {
  const T* f[6];
};

template <typename T>
__global__ void k_dft_sample(DftRegion r, T* ring, int slot, Fields6<T> fields, int ny,
                             int nz) {
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= r.ncell) return;
  const long long ck = cell % r.count[2];
  const long long rest = cell / r.count[2];
  const long long cj = rest % r.count[1];
  const long long ci = rest / r.count[1];
  const long long id = ((long long)(r.start[0] + ci * r.stride[0]) * ny +
                        (r.start[1] + cj * r.stride[1])) * nz +
                       (r.start[2] + ck * r.stride[2]);
  for (int q = 0; q < r.ncomp; ++q)
    ring[((long long)slot * r.ncomp + q) * r.ncell + cell] = fields.f[r.comps[q]][id];
}

template <typename T>
__global__ void k_dft_flush(DftRegion r, const T* ring, int n_pending, double* acc,
                            const double* ph_e, const double* ph_h, long long q0, int n_freq,
                            double dt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= r.ncell * r.ncomp) return;
  const long long cell = t % r.ncell;
  const int qc = (int)(t / r.ncell);
  const double* ph = r.comps[qc] < 3 ? ph_e : ph_h;
  constexpr int F = 8;
  for (int f0 = 0; f0 < n_freq; f0 += F) {
    double re[F], im[F];
    const int nf = min(F, n_freq - f0);
#pragma unroll
    for (int f = 0; f < F; ++f) {
      if (f < nf) {
        const long long o = (((long long)qc * n_freq + f0 + f) * r.ncell + cell) * 2;
        re[f] = acc[o];
        im[f] = acc[o + 1];
      }
    }
    for (int q = 0; q < n_pending; ++q) {
      const double s = (double)ring[((long long)q * r.ncomp + qc) * r.ncell + cell];
      const double* row = ph + ((q0 + q) * n_freq + f0) * 2;
#pragma unroll
      for (int f = 0; f < F; ++f) {
        if (f < nf) {
          re[f] = __dadd_rn(re[f], __dmul_rn(__dmul_rn(row[2 * f], s), dt));
          im[f] = __dadd_rn(im[f], __dmul_rn(__dmul_rn(row[2 * f + 1], s), dt));
        }
      }
    }
#pragma unroll
    for (int f = 0; f < F; ++f) {
      if (f < nf) {
        const long long o = (((long long)qc * n_freq + f0 + f) * r.ncell + cell) * 2;
        acc[o] = re[f];
        acc[o + 1] = im[f];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Flux monitor (simulation.py:1440-1459). Per step, S = E_t1*H_t2 - E_t2*H_t1
// in the field type at every cell of the plane (the same three roundings as
// the reference), summed in double per block; block partials go to a ring.
// The flush reduces each step's partials in a fixed order and accumulates
// flux += double(T(sum) * T(dA)) * dt, as the reference's float32 run does.
// ---------------------------------------------------------------------------
struct FluxPlane {
  int axis, idx;
  int n0, n1;  // plane extents (the two other axes, in order)
  int nblk;
};

template <typename T>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Flux planes sampled by one launch (up to kFluxBatch): blockIdx.y picks
// the plane; block x of a plane sums S = E_t1 H_t2 - E_t2 H_t1 (rounded in
// the field type, simulation.py:1440-1459) over the plane's cells
// [256 x, 256 x + 256) in row-major (n0, n1) order with block_sum, and
// stores the partial in the plane's ring slot; k_flux_flush folds the
// partials in block order. Blocks past a plane's own count return before
// any barrier, as a whole.
constexpr int kFluxBatch = 8;
struct FluxBatch {
  FluxPlane p[kFluxBatch];
  double* partial[kFluxBatch];
  int slot[kFluxBatch];
};

template <typename T>
__global__ void __launch_bounds__(256) k_flux_sample_batch(FluxBatch b, Fields6<T> fields, int ny,
                                                           int nz) {
  __shared__ double sh[8];
  const FluxPlane& p = b.p[blockIdx.y];
  if ((int)blockIdx.x >= p.nblk) return;  // uniform over the block
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < (long long)p.n0 * p.n1) {
    const int u = (int)(t / p.n1), w = (int)(t % p.n1);
    long long id;
    int e1, h2, e2, h1;
    if (p.axis == 0) {  // S = Ey*Hz - Ez*Hy
      id = ((long long)p.idx * ny + u) * nz + w;
      e1 = 1; h2 = 5; e2 = 2; h1 = 4;
    } else if (p.axis == 1) {  // S = Ez*Hx - Ex*Hz
      id = ((long long)u * ny + p.idx) * nz + w;
      e1 = 2; h2 = 3; e2 = 0; h1 = 5;
    } else {  // S = Ex*Hy - Ey*Hx
      id = ((long long)u * ny + w) * nz + p.idx;
      e1 = 0; h2 = 4; e2 = 1; h1 = 3;
    }
    const T s = sub_rn(mul_rn(fields.f[e1][id], fields.f[h2][id]),
                       mul_rn(fields.f[e2][id], fields.f[h1][id]));
    v = (double)s;
  }
  v = block_sum<T>(v, sh);
  if (threadIdx.x == 0) b.partial[blockIdx.y][(long long)b.slot[blockIdx.y] * p.nblk + blockIdx.x] = v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_flux_flush(const double* partial, int nblk, int n_pending,
                                                    double* acc, double dA, double dt) {
  __shared__ double sh[8];
  double total = *acc;
  for (int q = 0; q < n_pending; ++q) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) v += partial[(long long)q * nblk + b];
    v = block_sum<T>(v, sh);
    __syncthreads();
    if (threadIdx.x == 0) {
      const T s = to_real(v, T());
      const T sa = mul_rn(s, (T)dA);
      total = __dadd_rn(total, __dmul_rn((double)sa, dt));
    }
  }
  if (threadIdx.x == 0) *acc = total;
}

// Strided sub-block of one field into a compact C-order buffer (the
// FieldMonitor snapshot: every stride-th cell per axis, or one z plane).
template <typename T>
__global__ void k_gather_region(const T* f, int ny, int nz, int3 start, int3 stride,
                                int3 count, T* out) {
  const long long n = (long long)count.x * count.y * count.z;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long ck = t % count.z, rest = t / count.z;
    const long long cj = rest % count.y, ci = rest / count.y;
    out[t] = f[((long long)(start.x + ci * stride.x) * ny + (start.y + cj * stride.y)) * nz +
               (start.z + ck * stride.z)];
  }
}

// Non-finite scan over a field: sets *flag when any value is inf or nan.
template <typename T>
__global__ void k_nonfinite(const T* f, long long n, int* flag) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    if (!isfinite(f[t])) {
      *flag = 1;
      return;
    }
}

}  // namespace pfb
