// noalloc.cu -- the bundle-adjustment cost on caller-owned device buffers,
// with no device allocation at all.
//
// Why it exists: a caller that cannot allocate device memory while it runs
// cannot create an nl_problem (a handle owns scratch buffers that it allocates
// with cudaMalloc).  Such callers include code inside a pre-sized memory pool
// that has already taken the whole device, real-time loops that must not touch
// the allocator between frames, and host code in a context that forbids
// allocation calls.  nl_ba_cost_noalloc evaluates the same FP64 cost
// chi2 = sum_e w_e |r_e|^2 as nl_update, but takes every input and its output as
// device pointers and keeps its only scratch (the per-chunk partial sums) in a
// fixed array compiled into the library.
//
// The scratch array: NL_NOALLOC_MAX_EDGES / kChunk partial sums (32 KB of
// doubles), a file-scope __device__ array.  Every GPU that loads the library
// holds it until the process exits.  All calls share it and it keeps the last
// call's contents; each call writes every partial it later reads, so nothing
// needs clearing.  Two calls whose kernels overlap on the GPU (different
// streams, or different host threads on the same device) race on it and may
// return wrong sums: serialise them.
//
// Device address of the array: the name `noalloc_partials` in host code is
// only a host-side handle for the symbol.  The first call on each device looks
// up the real address with cudaGetSymbolAddress, with that device current, and
// caches it; that first call should come before any stream capture.  The
// cached address belongs to the device's primary context: a program that
// calls cudaDeviceReset (or otherwise tears that context down) must not call
// nl_ba_cost_noalloc on that device afterwards, since the cache would still
// hold the old context's address.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/nelson_b200.h"
#include "ba_kernels.cuh"

namespace nl {
namespace {

constexpr int kNoallocNT = 256;
constexpr int kChunk = 4096;  // edges per partial sum (16 per thread)
constexpr int kMaxPartials = NL_NOALLOC_MAX_EDGES / kChunk;
static_assert(NL_NOALLOC_MAX_EDGES % kChunk == 0, "edge limit must be a whole number of chunks");

static __device__ __align__(256) double noalloc_partials[kMaxPartials];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// One CTA per chunk of kChunk edges: partial[c] = sum over the chunk, summed in
// a fixed order (per thread in edge order, then the CTA tree), so the result
// depends only on the inputs and ne.
template <int BC>
__global__ void __launch_bounds__(kNoallocNT)
cost_chunk_kernel(int ne, const double* __restrict__ cam, const double* __restrict__ pt,
                  const int* __restrict__ e_cam, const int* __restrict__ e_pt,
                  const double* __restrict__ obs, const double* __restrict__ w, double f, double cx,
                  double cy, double* __restrict__ partial) {
  __shared__ double sh[kNoallocNT / 32];
  const int e0 = blockIdx.x * kChunk;
  const int e1 = min(ne, e0 + kChunk);
  double acc = 0.0;
  for (int e = e0 + threadIdx.x; e < e1; e += kNoallocNT) {
    const double* cs = cam + (size_t)__ldg(e_cam + e) * 16;
    const double* X = pt + (size_t)__ldg(e_pt + e) * 3;
    double r0, r1;
    ba_project<double, BC, false, false>(cs, X, __ldg(obs + 2 * e), __ldg(obs + 2 * e + 1), f, cx, cy,
                                         r0, r1, nullptr, nullptr);
    acc += (w ? __ldg(w + e) : 1.0) * (r0 * r0 + r1 * r1);
  }
  const double s = block_sum<kNoallocNT>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Device address of the scratch array on the current device (looked up once
// per device).
nl_status scratch_address(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return NL_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return NL_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, noalloc_partials) != cudaSuccess || !p) return NL_ERR_CUDA;
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return NL_OK;
}

}  // namespace
}  // namespace nl

extern "C" nl_status nl_ba_cost_noalloc(int bc, int ne, const double* d_cam_state, const double* d_pts,
                                        const int* d_edge_cam, const int* d_edge_pt, const double* d_obs,
                                        const double* d_weight, double f, double cx, double cy,
                                        double* d_chi2, void* stream) {
  using namespace nl;
  if ((bc != 6 && bc != 9) || ne < 0 || ne > NL_NOALLOC_MAX_EDGES || !d_chi2) return NL_ERR_ARG;
  if (ne > 0 && (!d_cam_state || !d_pts || !d_edge_cam || !d_edge_pt || !d_obs)) return NL_ERR_ARG;
  double* partial = nullptr;
  nl_status s = scratch_address(&partial);
  if (s != NL_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nparts = (ne + kChunk - 1) / kChunk;
  if (nparts > 0) {
    if (bc == 9)
      cost_chunk_kernel<9><<<nparts, kNoallocNT, 0, st>>>(ne, d_cam_state, d_pts, d_edge_cam, d_edge_pt, d_obs,
                                                          d_weight, f, cx, cy, partial);
    else
      cost_chunk_kernel<6><<<nparts, kNoallocNT, 0, st>>>(ne, d_cam_state, d_pts, d_edge_cam, d_edge_pt, d_obs,
                                                          d_weight, f, cx, cy, partial);
  }
  // nparts == 0 writes 0 to *d_chi2
  sum_partials_kernel<256><<<1, 256, 0, st>>>(partial, nparts, d_chi2, nullptr);
  return cudaGetLastError() == cudaSuccess ? NL_OK : NL_ERR_CUDA;
}
