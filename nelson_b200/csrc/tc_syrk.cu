// tc_syrk.cu -- tensor-core (tcgen05) trailing update of the mixed Cholesky.
//
// For panel k the trailing lower triangle of S receives C_IJ -= X_I X_J',
// X = S[(k+1)128:, k 128:(k+1) 128] (FP32).  This is the one dense
// contraction of the reduced-camera-system factorisation
// (SolverCholeskyEigenDense::factorize, nelson/SolverCholeskyDense.hpp:15-18).
//
// tc_pack_kernel   splits X into BF16 hi = bf16(x) and lo = bf16(x - hi) and
//                  stores each 128-row tile as four K-chunks of 32 columns,
//                  each chunk (8 KB) contiguous in the UMMA canonical K-major
//                  no-swizzle layout: 8x8 core matrices (128 contiguous bytes),
//                  core (m-group g, k-group h') at byte (4 g + h') * 128 of the
//                  chunk, i.e. LBO (K step) = 128 B, SBO (M step) = 512 B.
// tc_syrk_kernel   one CTA per lower 128x128 output tile.  One thread runs a
//                  two-stage pipeline over the K-chunks (K = 128 per panel,
//                  up to four panels per update): one cp.async.bulk per
//                  operand chunk (A hi, A lo, B hi, B lo) lands on the
//                  stage's mbarrier while the previous chunk's six
//                  tcgen05.mma (M = N = 128, K = 16, kind::f16, BF16 in, FP32
//                  accumulate in TMEM: hi*hi + hi*lo + lo*hi) run; each chunk
//                  commits to the stage's MMA mbarrier, which frees the stage.
//                  Eight warps then read the accumulator with tcgen05.ld
//                  (32x32b), stage it in shared memory and subtract it from the
//                  tile with coalesced accesses.
// Every wait is bounded: on expiry the kernel records ST_SPIN_TIMEOUT, waits
// (bounded) for what it issued, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <stdint.h>

#include "nl_common.cuh"
#include "tc_pack_layout.cuh"
#include "tc_syrk.h"

namespace nl {

namespace {

constexpr int TB = 128;                  // tile rows / cols / K of one panel
constexpr int kTileBytes = TB * TB * 2;  // one BF16 operand tile (32 KB)
constexpr int kPackTile = 2 * kTileBytes;  // hi + lo
constexpr int kChunkK = 32;                // K columns per pipeline chunk
constexpr int kChunkBytes = TB * kChunkK * 2;  // one operand chunk: 8 KB
static_assert(kChunkBytes == kPackChunkBytes && kTileBytes == kPackHalfBytes, "pack layout");
constexpr int kChunksPerPanel = TB / kChunkK;  // 4
constexpr long long kWaitLimit = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; returns false when the limit is hit
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long it = 0; it < kWaitLimit; it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 64) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(p);
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;               // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: kind::f16, A = B = BF16, D = F32, K-major, M = N = 128
constexpr uint32_t kIdesc = (1u << 4)           // D format F32
                            | (1u << 7)         // A format BF16
                            | (1u << 10)        // B format BF16
                            | ((TB >> 3) << 17) // N >> 3
                            | ((TB >> 4) << 24);// M >> 4

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// X rows (k+1)*TB + r_first .. + nrows - 1 (columns k*TB ..) -> packed hi / lo
// tiles; packed tile t holds rows (k+1+t)*TB ...
// One thread per (row, 8-column group).
__global__ void tc_pack_kernel(const float* __restrict__ S, int ld, int k, int r_first, int nrows,
                               uint8_t* __restrict__ pack, const int* __restrict__ active) {
  if (active && !*active) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nrows * 16) return;
  const int r = r_first + (int)(t >> 4), h = (int)(t & 15);
  const float* src = S + (size_t)((k + 1) * TB + r) * ld + (size_t)k * TB + 8 * h;
  const float4 a = *reinterpret_cast<const float4*>(src);
  const float4 b = *reinterpret_cast<const float4*>(src + 4);
  const float x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  tc_pack_store8(pack, tc_pack_offset(r, h), x);
}

// ---------------------------------------------------------------------------
// 256 threads.  K = 128 in two chunks of 64 through one 64 KB operand buffer
// (A hi, A lo, B hi, B lo: 16 KB each), so three CTAs fit on an SM and
// overlap each other's copies, MMAs and epilogues.  The accumulator is
// staged through shared memory so the read-modify-write of the FP32 C tile
// is coalesced (a warp covers a 512-byte row).
constexpr int kStageBytes = 4 * kChunkBytes;   // A hi, A lo, B hi, B lo of one chunk
constexpr int kStages = 2;
constexpr int kStageLd = TB + 4;               // floats per staged accumulator row
constexpr int kSmemBytes = TB * kStageLd * 4;  // 67,584 B >= 2 stages x 32 KB operands
static_assert(kStages * kStageBytes <= kSmemBytes, "operand stages alias the epilogue staging");

__global__ void __launch_bounds__(256) tc_syrk_kernel(float* __restrict__ S, int ld, int k, int t0, int nt,
                                                      int ncols, int rb, const TcPacks packs,
                                                      const int* __restrict__ active, int* __restrict__ status) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar_load[2], bar_mma[2];
  __shared__ uint32_t tmem_base;
  __shared__ int ok_s;
  if (active && !*active) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int q = blockIdx.x;
  int I, J;
  if (ncols > 0) {
    // the first ncols tile columns of the trailing triangle: column j holds
    // tiles max(j, rb) .. nt - 1
    J = 0;
    while (J + 1 < ncols && q >= nt - max(J, rb)) {
      q -= nt - max(J, rb);
      J++;
    }
    I = max(J, rb) + q;
  } else {
    I = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
    while ((I + 1) * (I + 2) / 2 <= q) I++;
    while (I * (I + 1) / 2 > q) I--;
    J = q - I * (I + 1) / 2;
  }
  const bool diag = I == J;

  // start pulling the output tile into L2 now; the epilogue reads it last
  {
    const float* crow0 = S + (size_t)((t0 + I) * TB) * ld + (size_t)(t0 + J) * TB;
    if (tid < TB)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(crow0 + (size_t)tid * ld), "r"(TB * 4)
                   : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TB));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < kStages; st++) {
      mbar_init(&bar_load[st], 1);
      mbar_init(&bar_mma[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = tmem_base;

  if (tid == 0) {
    int ok = 1;
    const int nch = kChunksPerPanel * packs.n;
    // chunk c: stage c & 1, its (c >> 1)-th use of that stage
    auto issue_load = [&](int c) {
      uint8_t* st = smem + (size_t)(c & 1) * kStageBytes;
      const int panel = c / kChunksPerPanel, cc = c % kChunksPerPanel;
      const uint8_t* pk = static_cast<const uint8_t*>(packs.p[panel]);
      const int first = k + 1 + panel;  // first tile row of that pack
      const uint8_t* pa = pk + (size_t)(t0 + I - first) * kPackTile + (size_t)cc * kChunkBytes;
      const uint8_t* pb = pk + (size_t)(t0 + J - first) * kPackTile + (size_t)cc * kChunkBytes;
      mbar_expect_tx(&bar_load[c & 1], (diag ? 2 : 4) * kChunkBytes);
      bulk_g2s(st, pa, kChunkBytes, &bar_load[c & 1]);
      bulk_g2s(st + kChunkBytes, pa + kTileBytes, kChunkBytes, &bar_load[c & 1]);
      if (!diag) {
        bulk_g2s(st + 2 * kChunkBytes, pb, kChunkBytes, &bar_load[c & 1]);
        bulk_g2s(st + 3 * kChunkBytes, pb + kTileBytes, kChunkBytes, &bar_load[c & 1]);
      }
    };
    int last_load = 0, last_commit = -1;
    issue_load(0);
    for (int c = 0; c < nch && ok; c++) {
      if (c + 1 < nch) {
        // stage (c + 1) & 1 was last read by the MMAs of chunk c - 1
        if (c >= 1 && !mbar_wait(&bar_mma[(c + 1) & 1], ((c - 1) >> 1) & 1)) {
          ok = 0;
          break;
        }
        issue_load(c + 1);
        last_load = c + 1;
      }
      if (!mbar_wait(&bar_load[c & 1], (c >> 1) & 1)) {
        ok = 0;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint8_t* st = smem + (size_t)(c & 1) * kStageBytes;
      const uint8_t* ah = st;
      const uint8_t* al = st + kChunkBytes;
      const uint8_t* bh = diag ? ah : st + 2 * kChunkBytes;
      const uint8_t* bl = diag ? al : st + 3 * kChunkBytes;
      const uint8_t* as[3] = {ah, ah, al};
      const uint8_t* bs[3] = {bh, bl, bh};
#pragma unroll
      for (int p = 0; p < 3; p++) {
#pragma unroll
        for (int s2 = 0; s2 < kChunkK / 16; s2++) {
          // K = 16 = two core columns: 256 B along K; chunk SBO = 4 * 128 B
          const uint64_t da = umma_desc(as[p] + s2 * 256, 128, 512);
          const uint64_t db = umma_desc(bs[p] + s2 * 256, 128, 512);
          umma_bf16(tmem_d, da, db, (c > 0 || p > 0 || s2 > 0) ? 1u : 0u);
        }
      }
      umma_commit(&bar_mma[c & 1]);
      last_commit = c;
    }
    // the last commit tracks every MMA issued before it
    if (ok && !mbar_wait(&bar_mma[(nch - 1) & 1], ((nch - 1) >> 1) & 1)) ok = 0;
    if (!ok) {
      // a wait gave up: give what was issued a bounded chance to land before
      // the shared memory and TMEM are reused / freed
      if (last_commit >= 0) mbar_wait(&bar_mma[last_commit & 1], (last_commit >> 1) & 1);
      mbar_wait(&bar_load[last_load & 1], (last_load >> 1) & 1);
    }
    ok_s = ok;
    if (!ok) atomicOr(status, ST_SPIN_TIMEOUT);
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int ok = ok_s;
  float* stage = reinterpret_cast<float*>(smem);  // operands are consumed: reuse
  if (ok) {
    // warps w and w + 4 share TMEM lanes 32 (w % 4) ..; they split the columns
    const int row = 32 * (warp & 3) + lane;
    const int cbase = 64 * (warp >> 2);
#pragma unroll 1
    for (int c = 0; c < 2; c++) {
      float d[32];
      tmem_ld32(tmem_d + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cbase + 32 * c), d);
      float4* dst = reinterpret_cast<float4*>(stage + row * kStageLd + cbase + 32 * c);
#pragma unroll
      for (int i = 0; i < 8; i++) dst[i] = make_float4(d[4 * i], d[4 * i + 1], d[4 * i + 2], d[4 * i + 3]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(TB));
  }
  if (ok) {
    // coalesced read-modify-write: warp w takes rows w, w + 8, ...; lane = 4 columns
    float* base = S + (size_t)((t0 + I) * TB) * ld + (size_t)(t0 + J) * TB + 4 * lane;
#pragma unroll 4
    for (int r = warp; r < TB; r += 8) {
      float4 v = *reinterpret_cast<float4*>(base + (size_t)r * ld);
      const float4 dd = *reinterpret_cast<const float4*>(stage + r * kStageLd + 4 * lane);
      const int col = 4 * lane;
      if (!diag || col + 0 <= r) v.x -= dd.x;
      if (!diag || col + 1 <= r) v.y -= dd.y;
      if (!diag || col + 2 <= r) v.z -= dd.z;
      if (!diag || col + 3 <= r) v.w -= dd.w;
      *reinterpret_cast<float4*>(base + (size_t)r * ld) = v;
    }
  }
}

}  // namespace

size_t tc_syrk_scratch_bytes(int n_pad) { return (size_t)(n_pad / TB + 1) * kPackTile; }

cudaError_t tc_pack_f32(const float* S, int ld, int k, int r_first, int nrows, void* pack, const int* active,
                        cudaStream_t st) {
  const long long nthr = (long long)nrows * 16;
  if (nthr <= 0) return cudaSuccess;
  tc_pack_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>(S, ld, k, r_first, nrows,
                                                                  static_cast<uint8_t*>(pack), active);
  return cudaGetLastError();
}

cudaError_t tc_prepare() {
  return cudaFuncSetAttribute(tc_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
}

cudaError_t tc_update_f32(float* S, int ld, int k, int t0, int nt, int ncols, int rb, const TcPacks& packs,
                          const int* active, int* status, cudaStream_t st) {
  if (packs.n < 1 || packs.n > kTcMaxPanels) return cudaErrorInvalidValue;
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(tc_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_dev = dev;
  }
  int grid = 0;
  if (ncols > 0) {
    for (int j = 0; j < ncols && j < nt; j++) grid += nt - std::max(j, rb) > 0 ? nt - std::max(j, rb) : 0;
  } else {
    grid = nt * (nt + 1) / 2;
  }
  if (grid <= 0) return cudaSuccess;
  tc_syrk_kernel<<<grid, 256, kSmemBytes, st>>>(S, ld, k, t0, nt, ncols > nt ? nt : ncols, ncols > 0 ? rb : 0,
                                                packs, active, status);
  return cudaGetLastError();
}

cudaError_t tc_syrk_f32(float* S, int ld, int k, int t0, int nt, void* scratch, const int* active, int* status,
                        cudaStream_t st) {
  cudaError_t e = tc_pack_f32(S, ld, k, 0, nt * TB, scratch, active, st);
  if (e != cudaSuccess) return e;
  TcPacks pk{{scratch, nullptr, nullptr, nullptr}, 1};
  return tc_update_f32(S, ld, k, t0, nt, 0, 0, pk, active, status, st);
}

}  // namespace nl
