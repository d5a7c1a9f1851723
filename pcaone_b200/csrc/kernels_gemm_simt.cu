// SIMT decode-GEMM (FP32 or FP64 FMA): the plain-precision GPU path.
//
//   out[s][r][c] = sum_{k in split s} val(code[r][k]) * B[k][c]
//
// with val(00, 01, 10, 11) = (2, 0, 1, 0): the A1 allele count, missing as 0. This is the
// raw product of the reference's G^T * Omega and G * G (src/Halko.cpp:123-124, 193-202);
// centring, scaling and the missing-entry terms are applied by the epilogue kernels.
//
// Tiling: a CTA owns 128 rows; each thread owns 4 rows x 8 columns of the output; K is
// streamed in chunks of 64 codes (16 packed bytes per row) staged in shared memory together
// with the matching 64 rows of B.
#include <algorithm>

#include "internal.hpp"
#include "rsvd.hpp"

namespace pg {

namespace {

constexpr int kTR = 128;  // rows per CTA
constexpr int kKC = 64;   // codes per K chunk
constexpr int kRPT = 4;   // rows per thread
constexpr int kCW = 8;    // columns per thread

// Map 16 packed codes to their 2-bit values v = (1-b0)(2-b1): 00->2, 01->0, 10->1, 11->0.
__device__ __forceinline__ uint32_t map_values(uint32_t w) {
  uint32_t b0 = w & 0x55555555u, b1 = (w >> 1) & 0x55555555u;
  uint32_t v0 = b1 & ~b0;                 // het -> 1
  uint32_t v1 = ~(b0 | b1) & 0x55555555u; // hom A1 -> 2
  return v0 | (v1 << 1);
}

template <typename T>
__device__ __forceinline__ T small_to_real(uint32_t x);
template <>
__device__ __forceinline__ float small_to_real<float>(uint32_t x) {
  return __int_as_float(0x4B400000u | x) - 12582912.0f;
}
template <>
__device__ __forceinline__ double small_to_real<double>(uint32_t x) {
  return __longlong_as_double(0x4338000000000000ull | x) - 6755399441055744.0;
}

template <typename T, int G>
__global__ void __launch_bounds__(32 * G)
k_decode_gemm(const uint8_t* __restrict__ codes, uint32_t pitch, int64_t rows, int64_t K,
              const T* __restrict__ B, int ldb, int l, int64_t kchunks_per_split,
              T* __restrict__ out) {
  constexpr int LDS = G * kCW;              // padded B columns in shared memory
  __shared__ uint32_t pk[kTR * 5];          // 128 rows x 4 words, row stride 5 words
  __shared__ __align__(16) T bs[kKC * LDS];

  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int64_t r0 = (int64_t)blockIdx.x * kTR;
  const int64_t kc_begin = (int64_t)blockIdx.y * kchunks_per_split;
  const int64_t kc_total = (K + kKC - 1) / kKC;
  const int64_t kc_end = min(kc_begin + kchunks_per_split, kc_total);

  T acc[kRPT][kCW];
#pragma unroll
  for (int q = 0; q < kRPT; ++q)
#pragma unroll
    for (int c = 0; c < kCW; ++c) acc[q][c] = T(0);

  for (int64_t kc = kc_begin; kc < kc_end; ++kc) {
    const int64_t k0 = kc * kKC;
    // packed codes: 128 rows x 16 bytes
    for (int t = threadIdx.x; t < kTR * 4; t += 32 * G) {
      int r = t >> 2, wq = t & 3;
      const uint32_t* src = reinterpret_cast<const uint32_t*>(codes + (r0 + r) * (int64_t)pitch + (k0 >> 2));
      pk[r * 5 + wq] = map_values(__ldg(src + wq));
    }
    // B chunk: 64 rows x LDS columns (zero beyond l and beyond K)
    for (int t = threadIdx.x; t < kKC * LDS; t += 32 * G) {
      int kk = t / LDS, cc = t - kk * LDS;
      int64_t k = k0 + kk;
      bs[t] = (cc < l && k < K) ? B[k * ldb + cc] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int wq = 0; wq < 4; ++wq) {
      uint32_t w[kRPT];
#pragma unroll
      for (int q = 0; q < kRPT; ++q) w[q] = pk[(lane + 32 * q) * 5 + wq];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const T* brow = bs + (wq * 16 + e) * LDS + g * kCW;
        T b[kCW];
#pragma unroll
        for (int c = 0; c < kCW; ++c) b[c] = brow[c];
#pragma unroll
        for (int q = 0; q < kRPT; ++q) {
          T v = small_to_real<T>((w[q] >> (2 * e)) & 3u);
#pragma unroll
          for (int c = 0; c < kCW; ++c) acc[q][c] = fma(v, b[c], acc[q][c]);
        }
      }
    }
    __syncthreads();
  }
  T* o = out + (int64_t)blockIdx.y * rows * l;
#pragma unroll
  for (int q = 0; q < kRPT; ++q) {
    int64_t r = r0 + lane + 32 * q;
    if (r >= rows) continue;
#pragma unroll
    for (int c = 0; c < kCW; ++c) {
      int col = g * kCW + c;
      if (col < l) o[r * l + col] = acc[q][c];
    }
  }
}

template <typename T, int G>
void launch_g(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t rows, int64_t K,
              const T* B, int ldb, int l, int ksplit, T* out) {
  int64_t kc_total = (K + kKC - 1) / kKC;
  int64_t per = (kc_total + ksplit - 1) / ksplit;
  dim3 grid((unsigned)((rows + kTR - 1) / kTR), (unsigned)ksplit);
  k_decode_gemm<T, G><<<grid, 32 * G, 0, c->stream>>>(codes, pitch, rows, K, B, ldb, l, per, out);
  PG_CHECK_LAUNCH();
}

}  // namespace

template <typename T>
void launch_decode_gemm_simt(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t rows,
                             int64_t K, const T* B, int ldb, int l, int ksplit, T* out) {
  PG_REQUIRE(l >= 1 && l <= kLmax, PCAONE_EBADARG, "sketch width out of range");
  int G = (l + kCW - 1) / kCW;
  switch (G) {
    case 1: launch_g<T, 1>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 2: launch_g<T, 2>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 3: launch_g<T, 3>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 4: launch_g<T, 4>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 5: launch_g<T, 5>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 6: launch_g<T, 6>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    case 7: launch_g<T, 7>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
    default: launch_g<T, 8>(c, codes, pitch, rows, K, B, ldb, l, ksplit, out); break;
  }
  c->launches++;
  c->gemm_launches++;
}

namespace {
template <typename T>
void simt_gemm(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t, int64_t rows, int64_t K,
               const T* B, int l, int ks, T* out) {
  launch_decode_gemm_simt<T>(c, codes, pitch, rows, K, B, l, l, ks, out);
}
int simt_ksplit(pcaone_ctx* c, int64_t rows, int64_t K, int) {
  int64_t tiles = (rows + kTR - 1) / kTR;
  int64_t chunks = (K + kKC - 1) / kKC;
  int64_t want = (2 * (int64_t)c->sm_count + tiles - 1) / tiles;
  int64_t ks = std::max<int64_t>(1, std::min<int64_t>(want, chunks / 4));
  return (int)std::min<int64_t>(ks, 64);
}
void no_omega(pcaone_ctx*, const double*, int, int64_t) {}
template <typename T>
void no_b2(pcaone_ctx*, const T*, int, int64_t) {}
}  // namespace

GemmFnT<float> gemm_simt_float() {
  return GemmFnT<float>{simt_ksplit, simt_gemm<float>, simt_gemm<float>, no_omega, no_b2<float>};
}
GemmFnT<double> gemm_simt_double() {
  return GemmFnT<double>{simt_ksplit, simt_gemm<double>, simt_gemm<double>, no_omega, no_b2<double>};
}

template void launch_decode_gemm_simt<float>(pcaone_ctx*, const uint8_t*, uint32_t, int64_t,
                                             int64_t, const float*, int, int, int, float*);
template void launch_decode_gemm_simt<double>(pcaone_ctx*, const uint8_t*, uint32_t, int64_t,
                                              int64_t, const double*, int, int, int, double*);

}  // namespace pg
