// Device memory layouts of the tensor-core decode-GEMM operands (kernels_gemm_tc.cu).
//
// A (packed genotype codes), "tiled": for every window, the rows (SNPs for Z^T Omega, samples
// for Z G) are cut into 128-row tiles and the K codes into 64-code chunks; block (tile, chunk)
// is 2048 contiguous bytes = 128 rows x 16 bytes (64 codes of one row, PLINK bit order).
// Blocks are stored chunk-fastest: block (t, kc) of a window starts at (t * C + kc) * 2048 for
// the window's chunk stride C. One CTA streams consecutive chunks of one tile, i.e. one
// contiguous range, with one 2048-byte bulk copy per chunk.
//
// B (split-BF16 sketch operand), "swizzled chunk-major": for 64-code chunk kc, NP rows of 128
// bytes (64 BF16 values in the permuted K order of the decode) are stored exactly as the
// tensor core reads them from shared memory with the 128-byte swizzle: the 16-byte unit u of
// row n sits at unit u ^ (n & 7). One chunk is one contiguous NP * 128-byte bulk copy.
#pragma once

#include <cstdint>

namespace pg {

constexpr int kTcTileRows = 128;
constexpr int kTcChunk = 64;          // codes per K chunk
constexpr int kTcBlockBytes = 2048;   // 128 rows x 16 bytes

// Code index k -> its position in the decode order of its 64-code chunk: decode_word emits
// the pairs (c0,c4) (c8,c12) (c1,c5) (c9,c13) ... of each 16-code word, so code
// c = 16q + r lands at 2 * (8q + 2 (r & 3) + (r >> 3)) + ((r >> 2) & 1).
__host__ __device__ __forceinline__ int64_t tc_pos(int64_t k) {
  const int c = (int)(k & 63), q = c >> 4, r16 = c & 15;
  return (k & ~(int64_t)63) + 2 * (8 * q + 2 * (r16 & 3) + (r16 >> 3)) + ((r16 >> 2) & 1);
}

// Element index of (row n, permuted position kpos) in the swizzled chunk-major B layout.
__host__ __device__ __forceinline__ int64_t bt_elem(int n, int64_t kpos, int np) {
  const int w = (int)(kpos & 63);
  return (kpos >> 6) * (int64_t)np * 64 + (int64_t)n * 64 + ((((w >> 3) ^ (n & 7))) << 3) + (w & 7);
}

}  // namespace pg
