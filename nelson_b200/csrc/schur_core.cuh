// schur_core.cuh -- device state of SolverCholeskySchur for one structure.
//
// Owns the Hessian blocks (U, V, W, bU, bV in T), the Schur work buffers and
// the dense factor, and enqueues computeIncrement
// (nelson/SolverCholeskySchur.hpp:91-157) on a stream.  The BA problem
// writes the Hessian blocks directly; the solver-only drop-in uploads them
// from the host.
#pragma once

#include <cublas_v2.h>

#include <algorithm>
#include <cstdio>
#include <memory>
#include <vector>

#include "cholesky.cuh"
#include "lm_kernels.cuh"
#include "nl_common.cuh"
#include "schur_kernels.cuh"
#include "tc_syrk.h"

namespace nl {

#define NL_CUDA(x)                                                                        \
  do {                                                                                    \
    cudaError_t _e = (x);                                                                 \
    if (_e != cudaSuccess) {                                                              \
      fprintf(stderr, "nelson_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(_e), \
              __FILE__, __LINE__);                                                        \
      return NL_ERR_CUDA;                                                                 \
    }                                                                                     \
  } while (0)

// Device allocation owned by a handle.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  nl_status alloc(size_t b) {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = b;
    if (b == 0) return NL_OK;
    if (cudaMalloc(&p, b) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return NL_ERR_NOMEM;
    }
    return NL_OK;
  }
  template <typename X>
  X* as() const {
    return static_cast<X*>(p);
  }
};

template <typename X>
nl_status upload(DevBuf& b, const std::vector<X>& v, cudaStream_t st) {
  nl_status s = b.alloc(std::max<size_t>(v.size(), 1) * sizeof(X));
  if (s != NL_OK) return s;
  if (!v.empty()) NL_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st));
  return NL_OK;
}

// Structure the core is built from (internal indices, reference UID order).
struct SchurStructure {
  int bc = 0, nci = 0, np = 0;
  std::vector<int> u_r, u_c;  // nU, upper (r <= c), CSC order
  std::vector<int> v_uid;     // np, -1 if no block (V is block diagonal)
  std::vector<int> w_r, w_c;  // nW, CSR order
};

class SchurCore {
 public:
  virtual ~SchurCore() {}
  virtual nl_status setup(const SchurStructure& st, cudaStream_t stream) = 0;
  // computeIncrement with lam = device (rel, abs); `active` predicates every kernel.
  virtual nl_status enqueue_increment(const double* lam, int* status, const int* active) = 0;
  // Solve with the factorisation of the last enqueue_increment for the
  // current bU / bV (same V^-1, W V^-1 and factor of S): incU / incV get
  // -(J'WJ + damping)^-1 b.
  virtual nl_status enqueue_resolve(int* status) = 0;
  // Test of the bounded waits: a forward solve in which one tile's flag is
  // never published, so every wait runs out after wait_limit polls.
  virtual nl_status enqueue_solve_withheld(int* status) = 0;
  virtual nl_status enqueue_hdiag(double* out) = 0;
  virtual nl_status enqueue_maxabs_b(double* out, const int* active) = 0;
  virtual nl_status enqueue_inc_dot(const LmDev* s, double* part, int* nparts) = 0;
  virtual int n() const = 0;
  virtual int ld() const = 0;
  virtual nl_status get_hessian(double* U, double* V, double* W, double* bU, double* bV) = 0;
  virtual nl_status set_hessian(const double* U, const double* V, const double* W, const double* bU,
                                const double* bV) = 0;
  virtual nl_status get_schur(double* S, double* bS) = 0;
  // raw device buffers
  virtual void* dU() = 0;
  virtual void* dV() = 0;
  virtual void* dW() = 0;
  virtual void* dbU() = 0;
  virtual void* dbV() = 0;
  double* incU = nullptr;  // device, n_pad
  double* incV = nullptr;  // device, 3 np
  int keep_schur = 0;      // keep an undamaged copy of S for nl_get_schur
  int refine_sweeps = 0;
  int use_tc = 1;          // tensor-core trailing update (mixed)
  nl_phase_times times{};
  long long launches = 0;
  int timing = 0;          // record per-phase CUDA events
  int envelope = 0;        // envelope solver: skip the tiles of S outside the Cholesky envelope
  long long wait_limit = kSpinLimit;  // polls before a flag wait of the solves gives up
  int timing_detail = 0;   // with timing: also per-panel events on the factorisation's critical path
                           // (costly on the host: one record per kernel boundary, and no early launch)
};

std::unique_ptr<SchurCore> make_schur_core(int precision, int bc, cublasHandle_t cublas);

}  // namespace nl
