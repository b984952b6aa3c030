// tc_syrk.h -- tensor-core trailing update of the mixed-precision Cholesky.
#pragma once
#include <cuda_runtime.h>

namespace nl {

// Sets the kernel attributes the tensor-core update needs on the current
// device (call before capturing launches into a CUDA graph).
cudaError_t tc_prepare();

// Scratch the tensor-core update needs for a trailing matrix of n_pad rows:
// the current panel split into BF16 hi/lo halves in UMMA canonical layout.
size_t tc_syrk_scratch_bytes(int n_pad);

// Pack rows (k+1)*128 + r_first .. + nrows - 1 of panel k into `pack` (packed
// tile t holds rows (k+1+t)*128 ..; r_first is a multiple of 128).
cudaError_t tc_pack_f32(const float* S, int ld, int k, int r_first, int nrows, void* pack, const int* active,
                        cudaStream_t st);
// Up to four packed panels of one update.
constexpr int kTcMaxPanels = 4;
struct TcPacks {
  const void* p[kTcMaxPanels];
  int n;
};
// Update with packed panels k .. k + packs.n - 1: packs.p[i] holds panel k + i
// (rows from (k+1+i)*128), so the update has K = 128 packs.n.  ncols = 0
// updates the lower triangle of tiles t0 .. t0+nt-1; ncols > 0 only its first
// ncols tile columns from relative row rb on (tiles (I, J),
// t0 <= J < t0 + ncols, max(J, t0 + rb) <= I < t0 + nt).
cudaError_t tc_update_f32(float* S, int ld, int k, int t0, int nt, int ncols, int rb, const TcPacks& packs,
                          const int* active, int* status, cudaStream_t st);

// S[I][J] -= X_I X_J' for the lower 128x128 tiles I >= J of the trailing
// matrix (tiles t0 .. t0 + nt - 1), X = columns [k*128, (k+1)*128) of S
// (FP32, row-major, leading dimension ld).  The product runs as three BF16
// tcgen05 MMAs (hi*hi + hi*lo + lo*hi) accumulating in TMEM (FP32).
cudaError_t tc_syrk_f32(float* S, int ld, int k, int t0, int nt, void* scratch,
                        const int* active, int* status, cudaStream_t st);

}  // namespace nl
