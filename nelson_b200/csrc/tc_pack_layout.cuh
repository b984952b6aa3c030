// tc_pack_layout.cuh -- byte layout of the BF16 hi/lo panel packs read by the
// tensor-core trailing update (tc_syrk.cu).  A pack holds the rows below the
// diagonal tile of one 128-wide panel, one 64 KB entry per 128-row tile:
// 32 KB of hi = bf16(x), then 32 KB of lo = bf16(x - hi).  Each half is four
// K-chunks of 32 columns (8 KB each) in the UMMA canonical K-major no-swizzle
// layout: 8x8 core matrices of 128 contiguous bytes, core (row group g,
// column group h') at byte (4 g + h') * 128 of the chunk.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace nl {

constexpr int kPackRows = 128;
constexpr int kPackHalfBytes = kPackRows * kPackRows * 2;  // 32 KB
constexpr int kPackEntryBytes = 2 * kPackHalfBytes;        // hi + lo
constexpr int kPackChunkBytes = kPackRows * 32 * 2;        // 8 KB

// Offset of the 16-byte hi vector of packed row `rel_row` (counted from the
// pack's first row), columns 8 h .. 8 h + 7; lo is kPackHalfBytes further on.
__host__ __device__ inline size_t tc_pack_offset(int rel_row, int h) {
  const int tile = rel_row / kPackRows, rr = rel_row % kPackRows;
  const int g = rr >> 3, ri = rr & 7, c = h >> 2, hh = h & 3;
  return (size_t)tile * kPackEntryBytes + (size_t)c * kPackChunkBytes + (size_t)((4 * g + hh) * 128 + ri * 16);
}

// Splits 8 FP32 values into BF16 hi / lo and stores both 16-byte vectors.
__device__ inline void tc_pack_store8(uint8_t* pack, size_t off, const float* x) {
  __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    hi[i] = __float2bfloat16_rn(x[i]);
    lo[i] = __float2bfloat16_rn(x[i] - __bfloat162float(hi[i]));
  }
  *reinterpret_cast<uint4*>(pack + off) = *reinterpret_cast<const uint4*>(hi);
  *reinterpret_cast<uint4*>(pack + off + kPackHalfBytes) = *reinterpret_cast<const uint4*>(lo);
}

}  // namespace nl
