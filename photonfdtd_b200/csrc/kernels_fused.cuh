// kernels_fused.cuh - single-pass fused H + E step for 3D grids.
#pragma once

#include "common.cuh"

namespace pfb {

inline bool fused_supported(int nx, int ny, int nz) { return false; }

template <typename T>
int launch_fused(cudaStream_t stream, const StepArgs<T>& a, int ce_mode, bool ade) {
  return -1;
}

}  // namespace pfb
