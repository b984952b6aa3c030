// tc_syrk.cu -- tensor-core (tcgen05) trailing update of the mixed Cholesky.
#include "tc_syrk.h"

namespace nl {

size_t tc_syrk_scratch_bytes(int n_pad) { return (size_t)n_pad * 128 * 2 * 2; }

cudaError_t tc_syrk_f32(float*, int, int, int, int, void*, const int*, int*, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace nl
