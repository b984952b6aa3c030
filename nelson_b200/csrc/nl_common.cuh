// nl_common.cuh -- shared device helpers for the nelson_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "../../include/nelson_b200.h"

namespace nl {

// Padded element strides of the per-block Hessian storage.  Blocks are
// row-major and padded to a multiple of 16 bytes so they move as 16-byte
// vectors.
template <typename T>
__host__ __device__ constexpr int pad16(int n) {
  return ((n * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T);
}
template <typename T, int BC>
struct Layout {
  static constexpr int W = pad16<T>(BC * 3);   // W / Y (= W V^-1) block, BC x 3
  static constexpr int U = pad16<T>(BC * BC);  // U block, BC x BC
  static constexpr int V = pad16<T>(9);        // V / V^-1 block, 3 x 3
};

// Host-side NVTX range over the enqueue of one phase (named like the phases
// of SolverCholeskySchurIterationTimeStat, nelson/SolverCholeskySchur.h:25-38),
// so a profiler timeline groups each phase's kernel launches.  Costs nothing
// when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device-side error / status word bits (nl_status in the C ABI).
enum : int {
  ST_VINV_FAIL = 1,      // a damped 3x3 point block was not positive definite
  ST_CHOL_FAIL = 2,      // a pivot of the reduced camera system was <= 0 or not finite
  ST_SPIN_TIMEOUT = 4,   // a bounded wait between blocks gave up
  ST_NONFINITE = 8,      // a non-finite cost or increment was produced
};

// Deterministic block reduction of one double: every thread passes its value,
// thread 0 gets the total (warp shuffles then a fixed-order sum over warps).
template <int NT>
__device__ inline double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; i++) s += sh[i];
  }
  __syncthreads();
  return s;
}

__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Left SO(3) increment exp(w) by Rodrigues' formula (FP64).
__device__ inline void so3_exp(const double* w, double* R) {
  const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double A, B;
  if (th2 < 1e-8) {
    A = 1.0 - th2 / 6.0 + th2 * th2 / 120.0;
    B = 0.5 - th2 / 24.0 + th2 * th2 / 720.0;
  } else {
    const double th = sqrt(th2);
    double s, c;
    sincos(th, &s, &c);
    A = s / th;
    B = (1.0 - c) / th2;
  }
  const double K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double k2 = K[i * 3 + 0] * K[0 * 3 + j] + K[i * 3 + 1] * K[1 * 3 + j] + K[i * 3 + 2] * K[2 * 3 + j];
      R[i * 3 + j] = A * K[i * 3 + j] + B * k2 + (i == j ? 1.0 : 0.0);
    }
}

}  // namespace nl
