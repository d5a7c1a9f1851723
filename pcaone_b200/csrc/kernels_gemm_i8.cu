// tcgen05 (sm_100a) int8 decode-GEMM: the mixed-precision back end of the two sketch
// products G = Z^T Omega and H = Z G.
//
//   out[s][r][c] = sum_{k in split s} val(code[r][k]) * B[k][c]
//
// val(00, 01, 10, 11) = (2, 0, 1, 0) is exact as an unsigned 8-bit integer. The FP64 sketch
// operand B (Omega, or s/2 * G of the current window) enters as three signed 8-bit fixed-point
// pieces per column,
//
//   B[k][c] ~= sig0_c * q0[k][c] + sig1_c * q1[k][c] + sig2_c * q2[k][c],
//   sig0_c = max_k |B[k][c]| / 127,  sig1_c = sig0_c / 254,  sig2_c = sig1_c / 254,
//
// each piece the rounded residual of the previous ones (|q| <= 127). The absolute error of an
// entry is at most sig2_c / 2 = max_k |B[k][c]| / (2 * 127 * 254^2): 21 bits below the column
// maximum, finer than a split BF16 hi+lo pair for the entries that carry the product. The
// tensor core accumulates each piece exactly in int32 (|acc| <= 254 K); the readout combines
// the pieces in FP64 and stores FP32 partial sums. The epilogue kernels (kernels_epilogue.cu)
// add the rank-1 centring term and the sparse missing-entry term in FP64.
//
// Work split: rows are cut into 128-row tiles and tiles into pairs; a unit is one tile pair x
// UC consecutive 128-code K chunks. Both tiles of a pair multiply the same B chunk, so each B
// chunk crosses L2 once for 256 rows. Units are in pair-major order and CTA j of G (one CTA per
// SM, the whole tensor memory) owns units [j U / G, (j+1) U / G) (stream-K). Segment q of a
// pair writes its partial sums to output slot q and the CTA holding a pair's last unit
// zero-fills the slots the pair does not use, so every row has exactly `ks` slots that the
// epilogue sums in a fixed order (deterministic, no atomics).
//
// Roles (15 warps):
//   * warps 0-7 (decoders): warp w owns the 32 rows 32 (w % 4) .. of tile w / 4 = its TMEM
//     lanes; a thread decodes its row's 128 codes of a chunk with four PRMT byte lookups per
//     16 codes and writes the 128 int8 values with one tcgen05.st into an A slot of its tile;
//   * warp 8 (producer): lane 0 copies a unit's tiled codes (UC x 8 KB, contiguous) and lane
//     1 its B chunks (UC x NP x 128 bytes, already in the 128-byte-swizzled shared-memory
//     image) with 1-D bulk copies into a ring of S shared-memory stages;
//   * warps 9 and 10 (MMA): lane 0 of warp 9 + t issues the 128 x NP x 32 kind::i8 MMAs of
//     tile t (A from TMEM, B from shared memory) into the tile's TMEM accumulator and one
//     tcgen05.commit per unit, which frees the stage once both tiles' MMAs have read it;
//   * warps 11-14 (readout): at the end of a segment, move both accumulators to registers
//     with tcgen05.ld, combine the three pieces, store the FP32 partial sums.
// Tensor memory (512 columns): accumulator of tile t in [t NP, (t+1) NP); A slots (one
// 128-code chunk of one tile = 32 columns) from 2 NP on, RA per tile.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on timeout the CTA sets
// an error flag, stops issuing work, waits (bounded) for its copies and MMAs in flight, frees
// its tensor memory and returns, and the host reports PCAONE_ETIMEOUT.
#include <algorithm>
#include <array>
#include <cstdlib>

#include "internal.hpp"
#include "rsvd.hpp"
#include "tc_ptx.hpp"

namespace pg {

namespace {

using tc::bulk_load;
using tc::mbar_arrive;
using tc::mbar_arrive_tx;
using tc::mbar_drain;
using tc::mbar_init;
using tc::mbar_wait;
using tc::smem_desc_sw128;
using tc::smem_u32;

constexpr int kRows = 128;                       // rows per tile
constexpr int kChunk = 128;                      // codes per K chunk (32 packed bytes per row)
constexpr int kPairChunkBytes = 2 * kRows * 32;  // one chunk of a tile pair: 8192 bytes
constexpr int kHalfBytes = kRows * 16;           // 64 codes of one tile: 2048 bytes
constexpr int kThreads = 480;                    // 8 decoders + producer + 2 MMA + 4 readout warps
constexpr int kTmemCols = 512;
constexpr int kMinUnitsPerCta = 2;

// Column layout of the quantised operand: piece p of column c is row p * LP + c of B (and
// column p * LP + c of the accumulator), LP = l rounded up to 8.
__host__ __device__ constexpr int lp_of(int l) { return (l + 7) / 8 * 8; }
__host__ __device__ constexpr int np_of(int l) { return (3 * lp_of(l) + 15) / 16 * 16; }

// Pipeline shape of variant V (chosen per product shape by the autotuner in run_i8):
// bit 0 clear: units of two K chunks, two units in flight in tensor memory per tile; set:
// units of one chunk, four in flight (finer stream-K split, half the MMAs per commit). Wide
// sketches (NP > 128) take one-chunk units only. Bit 1 (AG): the decoders load the packed
// codes straight from global memory, one unit ahead in registers, instead of through the
// shared-memory ring, which then carries B alone (less shared-memory traffic per MMA).
template <int NP, int V = 0>
struct Cfg {
  static constexpr bool AG = (V & 2) != 0;
  static constexpr int UC = (NP <= 128 && (V & 1) == 0) ? 2 : 1;  // K chunks per unit
  static constexpr int RA = NP <= 128 ? 4 : 2;                    // A slots per tile (one chunk each)
  static constexpr int NU = RA / UC;  // units in flight in tensor memory per tile
  static constexpr int SB = NP * 128;  // B bytes per chunk
  static constexpr int STAGE = UC * ((AG ? 0 : kPairChunkBytes) + SB);
  static constexpr int S = (192 * 1024) / STAGE < 8 ? (192 * 1024) / STAGE : 8;
  static constexpr int ACOL = 2 * NP;
  static_assert(2 * NP + 2 * RA * 32 <= kTmemCols, "tensor memory over-subscribed");
  static_assert(S >= 2, "shared-memory ring too shallow");
};

// Decode one 32-bit word (16 codes c0..c15, 2 bits each, LSB first) into 16 unsigned bytes:
// o[0] = (c0, c2, c4, c6), o[1] = (c8, .., c14), o[2] = (c1, .., c7), o[3] = (c9, .., c15),
// i.e. code c lands at byte position 8 (c & 1) + (c >> 1). Byte value: 00 -> 2, 01 -> 0
// (missing), 10 -> 1, 11 -> 0; each PRMT selector nibble holds one code.
__device__ __forceinline__ void decode_word_i8(uint32_t w, uint32_t* o) {
  constexpr uint32_t kLut = 0x00010002u;
  const uint32_t x = w & 0x33333333u, y = (w >> 2) & 0x33333333u;
  o[0] = __byte_perm(kLut, 0u, x);
  o[1] = __byte_perm(kLut, 0u, x >> 16);
  o[2] = __byte_perm(kLut, 0u, y);
  o[3] = __byte_perm(kLut, 0u, y >> 16);
}

struct I8Args {
  const uint8_t* a_tiles;  // tiled codes: block (pair, chunk) of 8192 bytes, chunk-fastest
  const int8_t* bq;        // quantised B, per chunk NP rows x 128 bytes (swizzled)
  const float* sig;        // 3 x LP piece scales
  int64_t a_stride;        // chunks per pair in a_tiles (>= cpw)
  int64_t cpw;             // K chunks per window: chunk g lies in window g / cpw of a_tiles
  int64_t win_bytes;       // bytes per window of a_tiles (0 for a single window)
  int64_t rows;            // valid rows (outputs written for r < rows)
  int64_t chunks;          // K chunks (C)
  int64_t upp;             // units per pair (P = ceil(C / UC))
  int64_t units;           // pairs x P
  int grid, ks, l, lp;
  float* out;  // [ks][rows][l]
  int* err;
};

__device__ __forceinline__ int64_t unit_begin(int64_t j, const I8Args& a) { return j * a.units / a.grid; }
__device__ __forceinline__ int64_t cta_of_unit(int64_t x, const I8Args& a) {
  return ((x + 1) * a.grid + a.units - 1) / a.units - 1;
}

template <int NP, int V>
__global__ void __launch_bounds__(kThreads, 1) k_decode_gemm_i8(const __grid_constant__ I8Args args) {
  using C = Cfg<NP, V>;
  constexpr int S = C::S, UC = C::UC, RA = C::RA, NU = C::NU;
  constexpr uint32_t kStageA = C::AG ? 0 : UC * kPairChunkBytes, kStageB = UC * C::SB;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sB = smem;                      // S x kStageB (1024-byte aligned swizzle atoms)
  uint8_t* sA = smem + S * kStageB;        // S x kStageA
  uint64_t* bars = (uint64_t*)(sA + S * kStageA);
  uint64_t* full = bars;                   // [S]  bulk copies landed
  uint64_t* empty = bars + S;              // [S]  both tiles' MMAs done with the stage
  uint64_t* dec_full = bars + 2 * S;       // [2][NU] a unit of tile t decoded into TMEM
  uint64_t* acc_full = dec_full + 2 * NU;  // [2]  accumulator of tile t complete
  uint64_t* acc_empty = acc_full + 2;      // [2]  accumulator of tile t read out
  uint64_t* done = acc_full + 4;           // [2]  every MMA of issuer t complete
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(acc_full + 6);
  volatile int* abort_flag = (volatile int*)(acc_full + 7);
  float* sig_s = (float*)(acc_full + 8);  // [3 * lp]
  float* stg_all = sig_s + 3 * 64;        // [4 readout warps][32 rows][9]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t u0 = unit_begin(blockIdx.x, args), u1 = unit_begin(blockIdx.x + 1, args);
  const int n = (int)(u1 - u0);
  const int64_t P = args.upp, Cn = args.chunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 2);
    }
    for (int b = 0; b < 2 * NU; ++b) mbar_init(smem_u32(&dec_full[b]), 4);
    for (int t = 0; t < 2; ++t) {
      mbar_init(smem_u32(&acc_full[t]), 1);
      mbar_init(smem_u32(&acc_empty[t]), 4);
      mbar_init(smem_u32(&done[t]), 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = threadIdx.x; i < 3 * args.lp; i += blockDim.x) sig_s[i] = args.sig[i];
  if (warp == 9) tc::tmem_alloc(smem_u32((const void*)tmem_slot), kTmemCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < 8) {
    // ---------------- decoders: tile t, row r = 32 q + lane, TMEM lanes 32 q ..
    const int t = warp >> 2, q = warp & 3, r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    int64_t p = u0 % P;
    if constexpr (C::AG) {
      // this row's 32 code bytes of every chunk of unit i, read from global memory
      auto load = [&](int i, uint4 (&dst)[UC][2]) {
        const int64_t u = u0 + i, pair = u / P, kc = (u - pair * P) * UC;
#pragma unroll
        for (int ch = 0; ch < UC; ++ch) {
          const int64_t g = kc + ch;
          if (g < Cn) {
            const int64_t w = g / args.cpw;
            const uint8_t* base = args.a_tiles + w * args.win_bytes +
                                  (pair * args.a_stride + (g - w * args.cpw)) * kPairChunkBytes +
                                  t * (2 * kHalfBytes) + r * 16;
            dst[ch][0] = __ldg(reinterpret_cast<const uint4*>(base));
            dst[ch][1] = __ldg(reinterpret_cast<const uint4*>(base + kHalfBytes));
          }
        }
      };
      uint4 cur[UC][2], nxt[UC][2];
      if (n > 0) load(0, cur);
      for (int i = 0; i < n; ++i) {
        const int ua = i % NU;
        const int nch = (int)(Cn - p * UC < UC ? Cn - p * UC : UC);
        if (i + 1 < n) load(i + 1, nxt);  // in flight while this unit is decoded
        if (i >= NU) {  // the MMAs of unit i - NU have released this tile's A slots
          const int j = i - NU;
          if (!mbar_wait(smem_u32(&empty[j % S]), (j / S) & 1, abort_flag, args.err, 8)) break;
        }
        tc::fence_after();
#pragma unroll
        for (int ch = 0; ch < UC; ++ch) {
          if (ch >= nch) break;
          uint32_t v[32];
          decode_word_i8(cur[ch][0].x, v + 0);
          decode_word_i8(cur[ch][0].y, v + 4);
          decode_word_i8(cur[ch][0].z, v + 8);
          decode_word_i8(cur[ch][0].w, v + 12);
          decode_word_i8(cur[ch][1].x, v + 16);
          decode_word_i8(cur[ch][1].y, v + 20);
          decode_word_i8(cur[ch][1].z, v + 24);
          decode_word_i8(cur[ch][1].w, v + 28);
          tc::tmem_st32(tmem + lane_base + C::ACOL + t * (RA * 32) + (ua * UC + ch) * 32, v);
        }
        tc::tmem_wait_st();
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&dec_full[t * NU + ua]));
#pragma unroll
        for (int ch = 0; ch < UC; ++ch) {
          cur[ch][0] = nxt[ch][0];
          cur[ch][1] = nxt[ch][1];
        }
        if (++p == P) p = 0;
      }
    } else
    for (int i = 0; i < n; ++i) {
      const int s = i % S, ua = i % NU;
      const int nch = (int)(Cn - p * UC < UC ? Cn - p * UC : UC);
      if (!mbar_wait(smem_u32(&full[s]), (i / S) & 1, abort_flag, args.err, 8)) break;
      if (i >= NU) {  // the MMAs of unit i - NU have released this tile's A slots
        const int j = i - NU;
        if (!mbar_wait(smem_u32(&empty[j % S]), (j / S) & 1, abort_flag, args.err, 8)) break;
      }
      tc::fence_after();
      for (int ch = 0; ch < nch; ++ch) {
        const uint8_t* base = sA + s * kStageA + ch * kPairChunkBytes + t * (2 * kHalfBytes) + r * 16;
        const uint4 h0 = *reinterpret_cast<const uint4*>(base);
        const uint4 h1 = *reinterpret_cast<const uint4*>(base + kHalfBytes);
        uint32_t v[32];
        decode_word_i8(h0.x, v + 0);
        decode_word_i8(h0.y, v + 4);
        decode_word_i8(h0.z, v + 8);
        decode_word_i8(h0.w, v + 12);
        decode_word_i8(h1.x, v + 16);
        decode_word_i8(h1.y, v + 20);
        decode_word_i8(h1.z, v + 24);
        decode_word_i8(h1.w, v + 28);
        tc::tmem_st32(tmem + lane_base + C::ACOL + t * (RA * 32) + (ua * UC + ch) * 32, v);
      }
      tc::tmem_wait_st();
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&dec_full[t * NU + ua]));
      if (++p == P) p = 0;
    }
  } else if (warp == 8) {
    // ---------------- producer: lane 0 the codes, lane 1 the B chunks of each unit
    if (lane < 2) {  // the two lanes move in lockstep, so every issued unit has its arrive
      int issued = 0;
      int64_t pair = u0 / P, p = u0 - pair * P;
      for (int i = 0; i < n; ++i) {
        const int s = i % S;
        int ok = 1;
        if (lane == 0) ok = mbar_wait(smem_u32(&empty[s]), ((i / S) & 1) ^ 1, abort_flag, args.err, 1);
        ok = __shfl_sync(0x3u, ok, 0);
        if (!ok) break;
        const int64_t kc = p * UC;
        const uint32_t nch = (uint32_t)(Cn - kc < UC ? Cn - kc : UC);
        const uint32_t bar = smem_u32(&full[s]);
        if (lane == 0) {
          if constexpr (C::AG) {  // B alone: the decoders read the codes from global memory
            mbar_arrive_tx(bar, nch * C::SB);
            bulk_load(smem_u32(sB + s * kStageB), args.bq + kc * C::SB, nch * C::SB, bar);
          } else {
            mbar_arrive_tx(bar, nch * (kPairChunkBytes + C::SB));
            for (uint32_t ch = 0; ch < nch; ++ch) {  // chunk by chunk: a unit may straddle two windows
              const int64_t g = kc + ch, w = g / args.cpw;
              bulk_load(smem_u32(sA + s * kStageA + ch * kPairChunkBytes),
                        args.a_tiles + w * args.win_bytes +
                            (pair * args.a_stride + (g - w * args.cpw)) * kPairChunkBytes,
                        kPairChunkBytes, bar);
            }
          }
        } else if (!C::AG) {
          bulk_load(smem_u32(sB + s * kStageB), args.bq + kc * C::SB, nch * C::SB, bar);
        }
        issued = i + 1;
        if (++p == P) {
          p = 0;
          ++pair;
        }
      }
      if (*abort_flag && lane == 0) {  // drain copies in flight before the CTA exits
        for (int i = max(0, issued - S); i < issued; ++i) mbar_drain(smem_u32(&full[i % S]), (i / S) & 1);
      }
    }
  } else if (warp == 9 || warp == 10) {
    // ---------------- MMA issuer of tile t
    const int t = warp - 9;
    if (lane == 0) {
      constexpr uint32_t idesc = (2u << 4)                 // D: S32
                                 | (0u << 7) | (1u << 10)  // A: unsigned 8-bit, B: signed 8-bit
                                 | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
      int seg = 0;
      int64_t p = u0 % P;
      const uint32_t d_col = tmem + t * NP;
      for (int i = 0; i < n; ++i) {
        const int s = i % S, ua = i % NU;
        const bool first = (i == 0 || p == 0), last = (i == n - 1 || p == P - 1);
        const int nch = (int)(Cn - p * UC < UC ? Cn - p * UC : UC);
        if (first) {
          if (!mbar_wait(smem_u32(&acc_empty[t]), (seg & 1) ^ 1, abort_flag, args.err, 2)) break;
        }
        if (!mbar_wait(smem_u32(&full[s]), (i / S) & 1, abort_flag, args.err, 2)) break;
        if (!mbar_wait(smem_u32(&dec_full[t * NU + ua]), (i / NU) & 1, abort_flag, args.err, 4)) break;
        tc::fence_after();
        const uint32_t b_addr = smem_u32(sB + s * kStageB);
        const uint32_t a_col = tmem + C::ACOL + t * (RA * 32) + ua * UC * 32;
        for (int ch = 0; ch < nch; ++ch) {
#pragma unroll
          for (int kk = 0; kk < kChunk / 32; ++kk)
            tc::mma_i8(d_col, a_col + ch * 32 + kk * 8, smem_desc_sw128(b_addr + ch * C::SB + kk * 32), idesc,
                       (first && ch == 0 && kk == 0) ? 0u : 1u);
        }
        tc::commit(smem_u32(&empty[s]));
        if (last) {
          tc::commit(smem_u32(&acc_full[t]));
          ++seg;
        }
        if (++p == P) p = 0;
      }
      tc::commit(smem_u32(&done[t]));  // tracks every MMA issued above
      mbar_drain(smem_u32(&done[t]), 0);
    }
  } else {
    // ---------------- readout warps 11-14: TMEM lanes 32 (warp % 4) .. + 31 of both tiles
    const int q4 = warp & 3;
    const uint32_t lane_base = (uint32_t)(q4 * 32) << 16;
    const int l = args.l, lp = args.lp;
    float* stg = stg_all + q4 * 32 * 9;
    int64_t u = u0;
    bool ok = true;
    for (int seg = 0; u < u1 && ok; ++seg) {
      const int64_t pair = u / P;
      const int64_t seg_end = min(u1, (pair + 1) * P);
      const bool pair_end = seg_end == (pair + 1) * P;
      const int slot = (int)(blockIdx.x - cta_of_unit(pair * P, args));
      for (int t = 0; t < 2; ++t) {
        if (!mbar_wait(smem_u32(&acc_full[t]), seg & 1, abort_flag, args.err, 16)) {
          ok = false;
          break;
        }
        tc::fence_after();
        const int64_t row0 = (pair * 2 + t) * kRows + q4 * 32;
        const int nvalid = (int)(args.rows - row0 < 32 ? (args.rows - row0 > 0 ? args.rows - row0 : 0) : 32);
        float* o = args.out + ((int64_t)slot * args.rows + row0) * l;
        const uint32_t acc = tmem + lane_base + t * NP;
        for (int c0 = 0; c0 < lp; c0 += 8) {
          uint32_t v0[8], v1[8], v2[8];
          tc::tmem_ld8(acc + c0, v0);
          tc::tmem_ld8(acc + lp + c0, v1);
          tc::tmem_ld8(acc + 2 * lp + c0, v2);
          tc::tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int c = c0 + j;
            const double x = (double)(int)v0[j] * (double)sig_s[c] + (double)(int)v1[j] * (double)sig_s[lp + c] +
                             (double)(int)v2[j] * (double)sig_s[2 * lp + c];
            stg[lane * 9 + j] = (float)x;
          }
          __syncwarp();
          // each store instruction writes 4 rows x 8 columns
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int rr = 4 * k + (lane >> 3), e = lane & 7;
            if (rr < nvalid && c0 + e < l) o[(int64_t)rr * l + c0 + e] = stg[rr * 9 + e];
          }
          __syncwarp();
        }
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&acc_empty[t]));
        if (pair_end) {  // zero the slots this pair does not use: nvalid contiguous rows each
          for (int sl = slot + 1; sl < args.ks; ++sl) {
            float* z = args.out + ((int64_t)sl * args.rows + row0) * l;
            for (int e = lane; e < nvalid * l; e += 32) z[e] = 0.0f;
          }
        }
      }
      u = seg_end;
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 9) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// Tiled copy of one window's codes for this kernel: block (pair, chunk) = [tile 2p: codes
// 0-63 of the chunk (128 rows x 16 bytes), codes 64-127][tile 2p+1: same]. src holds `rows`
// valid rows of `pitch` bytes; rows past `rows` and bytes past the pitch are code 11 (value
// 0). One thread per (row, 16-byte half chunk).
__global__ void k_tile_codes_i8(const uint8_t* __restrict__ src, uint32_t pitch, int64_t rows, int64_t pairs,
                                int64_t chunks, uint8_t* __restrict__ dst) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t halves = 2 * chunks;
  if (t >= pairs * 2 * kRows * halves) return;
  const int64_t hc = t % halves, row = t / halves;
  uint4 v = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
  if (row < rows && (hc + 1) * 16 <= (int64_t)pitch)
    v = *reinterpret_cast<const uint4*>(src + row * (int64_t)pitch + hc * 16);
  const int64_t pair = row / (2 * kRows), rin2 = row - pair * 2 * kRows;
  const int64_t tile = rin2 / kRows, rin = rin2 - tile * kRows;
  const int64_t kc = hc >> 1, h = hc & 1;
  *reinterpret_cast<uint4*>(dst + (pair * chunks + kc) * kPairChunkBytes + tile * 2 * kHalfBytes + h * kHalfBytes +
                            rin * 16) = v;
}

// Largest |X[k][c]| over the K rows of a row-major K x l matrix, as the bits of a double
// (monotone in |x|, so atomicMax is order-independent and the result deterministic).
template <typename T>
__global__ void k_colmax(const T* __restrict__ X, int64_t K, int l, unsigned long long* __restrict__ qmax) {
  __shared__ unsigned long long sm[64];
  for (int c = threadIdx.x; c < l; c += blockDim.x) sm[c] = 0ull;
  __syncthreads();
  const int64_t tot = K * l;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const double x = fabs((double)X[e]);
    atomicMax(&sm[e % l], (unsigned long long)__double_as_longlong(x));
  }
  __syncthreads();
  for (int c = threadIdx.x; c < l; c += blockDim.x)
    if (sm[c]) atomicMax(&qmax[c], sm[c]);
}

// Piece scales of column c from its maximum: sig0 = max / 127, sig1 = sig0 / 254,
// sig2 = sig1 / 254, in FP32 (the same values in the quantiser and in the GEMM readout).
__device__ __forceinline__ void piece_scales(unsigned long long bits, float* s) {
  const double mx = __longlong_as_double((long long)bits);
  s[0] = mx > 0.0 ? (float)(mx / 127.0) : 1.0f;
  s[1] = s[0] / 254.0f;
  s[2] = s[1] / 254.0f;
}

// Quantised B of one chunk per CTA: every byte of the chunk's NP x 128 image is written
// (piece rows, zero rows past 3 LP and past l, zero K positions that hold no operand row).
// The image is assembled in shared memory: thread task = one (K position kk, column c)
// element, whose three pieces (each the rounded residual of the previous ones, |q| <= 127) go
// to rows c, LP + c, 2 LP + c at the byte that the decoder's order gives code kk (16-byte
// unit u = kk / 16, byte 8 (o & 1) + (o >> 1) for o = kk % 16, units 128-byte swizzled); the
// image then leaves as 16-byte stores. Operand row k is present when it lies in the first
// wlen rows of its window of kpw rows (windows w = k / kpw) and w * wlen + (k % kpw) < mtot.
// CTA 0 also writes the 3 x LP scales.
template <typename T>
__global__ void __launch_bounds__(256) k_quant(const T* __restrict__ X, int64_t kpw, int64_t wlen, int64_t mtot,
                                               int l, int lp, int np, const unsigned long long* __restrict__ qmax,
                                               int8_t* __restrict__ bq, float* __restrict__ sig) {
  __shared__ __align__(16) uint8_t img[192 * 128];
  __shared__ float sc[3][64];
  const int64_t kc = blockIdx.x;
  for (int c = threadIdx.x; c < lp; c += blockDim.x) {
    float s[3] = {1.0f, 1.0f, 1.0f};
    if (c < l) piece_scales(qmax[c], s);
    sc[0][c] = s[0];
    sc[1][c] = s[1];
    sc[2][c] = s[2];
    if (kc == 0) {
      sig[c] = s[0];
      sig[lp + c] = s[1];
      sig[2 * lp + c] = s[2];
    }
  }
  uint4* img4 = reinterpret_cast<uint4*>(img);
  for (int t = threadIdx.x; t < np * 8; t += blockDim.x) img4[t] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  for (int e = threadIdx.x; e < kChunk * l; e += blockDim.x) {
    const int kk = e / l, c = e - kk * l;
    const int64_t k = kc * kChunk + kk, w = k / kpw, r = k - w * kpw;
    if (r >= wlen || w * wlen + r >= mtot) continue;
    double x = (double)X[k * l + c];
    const int u = kk >> 4, o = kk & 15, pp = 8 * (o & 1) + (o >> 1);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const double s = (double)sc[p][c];
      const double q = fmin(127.0, fmax(-127.0, rint(x / s)));
      x -= q * s;
      const int n = p * lp + c;
      img[n * 128 + ((u ^ (n & 7)) << 4) + pp] = (uint8_t)(int8_t)(int)q;
    }
  }
  __syncthreads();
  uint4* dst = reinterpret_cast<uint4*>(bq + kc * (int64_t)np * 128);
  for (int t = threadIdx.x; t < np * 8; t += blockDim.x) dst[t] = img4[t];
}

// ------------------------------------------------------------------ host side
template <int NP, int V>
constexpr size_t smem_of() {
  using C = Cfg<NP, V>;
  return (size_t)1024 + (size_t)C::S * C::STAGE + (size_t)(2 * C::S + 2 * C::NU + 8) * 8 + (3 * 64 + 4 * 32 * 9) * 4;
}

int uc_of(int np, int v) { return (np <= 128 && (v & 1) == 0) ? 2 : 1; }
// the distinct variants of a sketch width: {0, 1, 2, 3}, or {0, 2} when NP > 128 (one-chunk
// units only)
int variants_of(int np) { return np <= 128 ? 4 : 2; }
int variant_id(int np, int idx) { return np <= 128 ? idx : 2 * idx; }

struct I8Plan {
  int64_t tiles = 0, pairs = 0, chunks = 0, upp = 0, units = 0;
  int grid = 0, ks = 1;
};

int64_t plan_cta_of_unit(int64_t x, int64_t units, int grid) { return ((x + 1) * grid + units - 1) / units - 1; }

I8Plan make_plan(const pcaone_ctx* c, int64_t rows, int64_t K, int np, int v) {
  I8Plan p;
  p.tiles = (rows + kRows - 1) / kRows;
  p.pairs = (p.tiles + 1) / 2;
  p.chunks = (K + kChunk - 1) / kChunk;
  p.upp = (p.chunks + uc_of(np, v) - 1) / uc_of(np, v);
  p.units = p.pairs * p.upp;
  if (p.units == 0) return p;
  p.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)c->sm_count, p.units / kMinUnitsPerCta));
  int ks = 1;
  for (int64_t t = 0; t < p.pairs; ++t) {
    const int64_t a = plan_cta_of_unit(t * p.upp, p.units, p.grid);
    const int64_t b = plan_cta_of_unit(t * p.upp + p.upp - 1, p.units, p.grid);
    ks = std::max<int>(ks, (int)(b - a + 1));
  }
  p.ks = ks;
  return p;
}

// Output slots every variant can fill: the largest split count over the variants (a variant
// that uses fewer zero-fills the rest).
int ks_all(const pcaone_ctx* c, int64_t rows, int64_t K, int np) {
  int ks = 1;
  for (int v = 0; v < variants_of(np); ++v) ks = std::max(ks, make_plan(c, rows, K, np, variant_id(np, v)).ks);
  return ks;
}

template <int NP, int V>
void launch_np(pcaone_ctx* c, const I8Args& a) {
  constexpr size_t smem = smem_of<NP, V>();
  static_assert(smem <= 227 * 1024, "shared memory above the per-CTA limit");
  if (c->smem_attr_set.insert((const void*)k_decode_gemm_i8<NP, V>).second)
    PG_CUDA(cudaFuncSetAttribute(k_decode_gemm_i8<NP, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_decode_gemm_i8<NP, V><<<a.grid, kThreads, smem, c->stream>>>(a);
  PG_CHECK_LAUNCH();
}

template <int NP>
void launch_v(pcaone_ctx* c, const I8Args& a, int v) {
  if constexpr (NP <= 128) {
    if (v == 1) return launch_np<NP, 1>(c, a);
    if (v == 3) return launch_np<NP, 3>(c, a);
  }
  if (v == 2) return launch_np<NP, 2>(c, a);
  launch_np<NP, 0>(c, a);
}

// The autotuner: the first product of a given shape (NP, rows, K and window layout of K)
// times each pipeline variant (after a warm-up launch, the fastest of three launches, CUDA
// events on the library's stream) and keeps the faster for every later product of that
// shape. Every variant writes the same product (to the rounding of the partial sums), so the
// launches that time them are the product itself. While the stream is being captured into a
// graph an unknown shape runs variant 0 untimed.
// PCAONE_I8_VARIANT=v pins variant v (when the sketch width has it) instead, for tests.
template <typename F>
int tune_variant(pcaone_ctx* c, const std::array<int64_t, 5>& key, int nvar, F&& launch) {
  if (const char* pin = std::getenv("PCAONE_I8_VARIANT")) {
    const int v = std::atoi(pin);
    for (int idx = 0; idx < nvar; ++idx)
      if (variant_id((int)key[0], idx) == v) return v;
  }
  auto it = c->i8_tune.find(key);
  if (it != c->i8_tune.end()) return it->second;
  if (nvar <= 1) return c->i8_tune[key] = 0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PG_CUDA(cudaStreamIsCapturing(c->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) return 0;
  cudaEvent_t e0, e1;
  PG_CUDA(cudaEventCreate(&e0));
  PG_CUDA(cudaEventCreate(&e1));
  int best = 0;
  float best_ms = 0.f;
  for (int idx = 0; idx < nvar; ++idx) {
    const int v = variant_id((int)key[0], idx);
    launch(v);  // warm-up (first use of the variant)
    float vbest = 0.f;
    for (int rep = 0; rep < 3; ++rep) {  // the fastest of three timed launches
      PG_CUDA(cudaEventRecord(e0, c->stream));
      launch(v);
      PG_CUDA(cudaEventRecord(e1, c->stream));
      PG_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep == 0 || ms < vbest) vbest = ms;
    }
    if (idx == 0 || vbest < best_ms) {
      best = v;
      best_ms = vbest;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return c->i8_tune[key] = best;
}

// One product over tiled codes (a_stride chunks per pair row, rows valid, K codes) and the
// quantised B (kpad K positions); out holds ks = make_plan(rows, K).ks slots of rows x l
// partial sums. With cpw > 0 the K chunks run over consecutive windows of a_tiles, cpw chunks
// and win_bytes bytes per window (a run of windows as one product).
void run_i8(pcaone_ctx* c, const uint8_t* a_tiles, int64_t a_stride, int64_t rows, int64_t K, const int8_t* bq,
            const float* sig, int64_t kpad, int l, int ks, float* out, int64_t cpw = 0, int64_t win_bytes = 0) {
  const int np = np_of(l);
  PG_REQUIRE(np <= 192, PCAONE_EBADARG, "sketch width too large for the int8 tensor-core path");
  PG_REQUIRE(ks == ks_all(c, rows, K, np), PCAONE_EBADARG, "output slot count does not match the product plan");
  const I8Plan p0 = make_plan(c, rows, K, np, 0);
  if (p0.units == 0) {
    PG_CUDA(cudaMemsetAsync(out, 0, (size_t)ks * rows * l * sizeof(float), c->stream));
    return;
  }
  if (cpw <= 0) {
    cpw = p0.chunks;
    win_bytes = 0;
  }
  PG_REQUIRE(cpw <= a_stride && p0.chunks * kChunk <= kpad, PCAONE_EBADARG, "K padding too small");
  PG_REQUIRE(((uintptr_t)a_tiles & 15) == 0 && ((uintptr_t)bq & 15) == 0, PCAONE_EBADARG,
             "operands not 16-byte aligned");
  auto launch = [&](int v) {
    const I8Plan p = make_plan(c, rows, K, np, v);
    I8Args a;
    a.a_tiles = a_tiles;
    a.bq = bq;
    a.sig = sig;
    a.a_stride = a_stride;
    a.cpw = cpw;
    a.win_bytes = win_bytes;
    a.rows = rows;
    a.chunks = p.chunks;
    a.upp = p.upp;
    a.units = p.units;
    a.grid = p.grid;
    a.ks = ks;
    a.l = l;
    a.lp = lp_of(l);
    a.out = out;
    a.err = (int*)scratch(c, "tc_err", sizeof(int));
    switch (np) {
      case 32: launch_v<32>(c, a, v); break;
      case 48: launch_v<48>(c, a, v); break;
      case 64: launch_v<64>(c, a, v); break;
      case 80: launch_v<80>(c, a, v); break;
      case 96: launch_v<96>(c, a, v); break;
      case 112: launch_v<112>(c, a, v); break;
      case 128: launch_v<128>(c, a, v); break;
      case 144: launch_v<144>(c, a, v); break;
      case 160: launch_v<160>(c, a, v); break;
      case 176: launch_v<176>(c, a, v); break;
      default: launch_v<192>(c, a, v); break;
    }
    c->launches++;
    c->gemm_launches++;
  };
  launch(tune_variant(c, {np, rows, K, cpw, win_bytes}, variants_of(np), launch));
}

// Tiled copies of the codes for the current window layout: "i8_tile1" (per window: SNP
// pairs x sample chunks, for Z^T Omega) from the SNP-major matrix and "i8_tile2" (per window:
// sample pairs x SNP chunks, for Z G) from the per-window transposed copy. Rebuilt when the
// matrix (load, permutation) or the window layout changes.
struct TileGeom {
  int64_t p1, c1, p2, c2;  // pairs per window and chunk stride of tile1 / tile2
};
TileGeom tile_geom(const pcaone_ctx* c) {
  const int64_t bs = (int64_t)c->win.blocksize, N = (int64_t)c->N;
  return TileGeom{((bs + kRows - 1) / kRows + 1) / 2, (N + kChunk - 1) / kChunk, ((N + kRows - 1) / kRows + 1) / 2,
                  (bs + kChunk - 1) / kChunk};
}
void ensure_tiles(pcaone_ctx* c) {
  if (c->streamed) return;  // the window run's tiles are built in its device slot
  PG_REQUIRE(c->bedT_valid, PCAONE_ESTATE, "transposed copy not built");
  const uint64_t key = (c->generation << 24) ^ ((uint64_t)c->win.bands << 44) ^ (uint64_t)c->win.blocksize;
  const TileGeom g = tile_geom(c);
  const int bands = c->win.bands;
  const size_t w1 = (size_t)g.p1 * g.c1 * kPairChunkBytes, w2 = (size_t)g.p2 * g.c2 * kPairChunkBytes;
  uint8_t* d1 = (uint8_t*)scratch(c, "i8_tile1", (size_t)bands * w1);
  uint8_t* d2 = (uint8_t*)scratch(c, "i8_tile2", (size_t)bands * w2);
  if (c->tiles8_valid && c->tiles8_key == key && c->tile81_ptr == d1 && c->tile82_ptr == d2) return;
  for (int b = 0; b < bands; ++b) {
    const int64_t s = (int64_t)c->win.start[b], m = (int64_t)c->win.stop[b] - s;
    const int64_t n1 = g.p1 * 2 * kRows * 2 * g.c1, n2 = g.p2 * 2 * kRows * 2 * g.c2;
    k_tile_codes_i8<<<(unsigned)((n1 + 255) / 256), 256, 0, c->stream>>>(c->d_bed + s * c->pitch, c->pitch, m, g.p1,
                                                                       g.c1, d1 + (size_t)b * w1);
    PG_CHECK_LAUNCH();
    k_tile_codes_i8<<<(unsigned)((n2 + 255) / 256), 256, 0, c->stream>>>(
        c->d_bedT + (int64_t)b * c->Npad * c->win.pitch, c->win.pitch, (int64_t)c->N, g.p2, g.c2, d2 + (size_t)b * w2);
    PG_CHECK_LAUNCH();
    c->launches += 2;
  }
  c->tiles8_key = key;
  c->tiles8_valid = true;
  c->tile81_ptr = d1;
  c->tile82_ptr = d2;
}

// Tiles of windows [b0, b1) for the first (which = 1) or the second product: the resident
// tiled copies, or the current slot of streamed genotypes (which must hold the windows).
const uint8_t* tiles_of(pcaone_ctx* c, int which, int64_t b0, int64_t b1) {
  const TileGeom g = tile_geom(c);
  const size_t w = which == 1 ? (size_t)g.p1 * g.c1 * kPairChunkBytes : (size_t)g.p2 * g.c2 * kPairChunkBytes;
  if (c->streamed) {
    PG_REQUIRE(c->cur_slot >= 0, PCAONE_ESTATE, "no window slot staged");
    const auto& S = c->slot[c->cur_slot];
    PG_REQUIRE(S.t1 && b0 >= S.b0 && b1 <= S.b1, PCAONE_ESTATE, "windows not in the staged slot");
    return (which == 1 ? S.t1 : S.t2) + (size_t)(b0 - S.b0) * w;
  }
  return (const uint8_t*)(which == 1 ? c->tile81_ptr : c->tile82_ptr) + (size_t)b0 * w;
}

// Quantise a row-major operand of kpad rows x l into the chunked piece layout (kpad / 128
// chunks); rows that hold no operand (see k_quant: windows of kpw rows with wlen present, mtot
// in all) quantise to zero. have_max: the column maxima in "i8_qmax<tag>" were already
// accumulated (by the first epilogue); otherwise they are computed here over the first K rows.
template <typename T>
void quantize(pcaone_ctx* c, const T* X, int64_t K, int l, int64_t kpad, const char* tag, bool have_max,
              int64_t kpw = 0, int64_t wlen = 0, int64_t mtot = 0) {
  const int np = np_of(l), lp = lp_of(l);
  const std::string t(tag);
  auto* qmax = (unsigned long long*)scratch(c, "i8_qmax" + t, 64 * sizeof(unsigned long long));
  auto* bq = (int8_t*)scratch(c, "i8_bq" + t, (size_t)kpad * np);
  auto* sig = (float*)scratch(c, "i8_sig" + t, 3 * 64 * sizeof(float));
  if (!have_max) {
    PG_CUDA(cudaMemsetAsync(qmax, 0, (size_t)l * sizeof(unsigned long long), c->stream));
    const int64_t tot = K * l;
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(2 * c->sm_count, (tot + 1023) / 1024));
    k_colmax<T><<<nblk, 256, 0, c->stream>>>(X, K, l, qmax);
    PG_CHECK_LAUNCH();
    c->launches++;
  }
  if (kpw <= 0) {
    kpw = kpad;
    wlen = mtot = K;
  }
  k_quant<T><<<(unsigned)(kpad / kChunk), 256, 0, c->stream>>>(X, kpw, wlen, mtot, l, lp, np, qmax, bq, sig);
  PG_CHECK_LAUNCH();
  c->launches++;
}

int i8_ksplit(pcaone_ctx* c, int64_t rows, int64_t K, int l) { return ks_all(c, rows, K, np_of(l)); }

void i8_omega(pcaone_ctx* c, const double* omega, int l, int64_t npad) {
  quantize<double>(c, omega, (int64_t)c->N, l, npad, "1", false);
}

void i8_b2(pcaone_ctx* c, const float* B2, int l, int64_t m) {
  quantize<float>(c, B2, m, l, (int64_t)round_up(c->win.blocksize, 256), "2", c->i8_b2_max_ready);
  c->i8_b2_max_ready = false;
}

unsigned long long* i8_b2_qmax(pcaone_ctx* c, int) {
  auto* qmax = (unsigned long long*)scratch(c, "i8_qmax2", 64 * sizeof(unsigned long long));
  PG_CUDA(cudaMemsetAsync(qmax, 0, 64 * sizeof(unsigned long long), c->stream));
  c->i8_b2_max_ready = true;
  return qmax;
}

void i8_p1(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t row_off, int64_t rows, int64_t K, const float*, int l,
           int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  const int64_t b = row_off / (int64_t)c->win.blocksize;
  PG_REQUIRE(b < c->win.bands && (uint64_t)row_off == c->win.start[b] && K == (int64_t)c->N, PCAONE_EBADARG,
             "first product must cover one window");
  const int np = np_of(l);
  auto* bq = (const int8_t*)scratch(c, "i8_bq1", (size_t)c->Npad * np);
  auto* sig = (const float*)scratch(c, "i8_sig1", 3 * 64 * sizeof(float));
  run_i8(c, tiles_of(c, 1, b, b + 1), g.c1, rows, K, bq, sig,
         c->Npad, l, ks, out);
}

void i8_p2(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t window, int64_t rows, int64_t K, const float*, int l,
           int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  PG_REQUIRE(window < c->win.bands && rows == (int64_t)c->N, PCAONE_EBADARG, "second product must cover one window");
  const int64_t kpad = round_up(c->win.blocksize, 256);
  const int np = np_of(l);
  auto* bq = (const int8_t*)scratch(c, "i8_bq2", (size_t)kpad * np);
  auto* sig = (const float*)scratch(c, "i8_sig2", 3 * 64 * sizeof(float));
  run_i8(c, tiles_of(c, 2, window, window + 1), g.c2, rows, K, bq, sig,
         kpad, l, ks, out);
}

// ---- runs of consecutive windows [b0, b1) as one product each (the tiled copies of the
// windows are contiguous): the first product's rows are the windows' SNP pairs, each window
// padded to p1 pairs (padding rows decode to zero); the second product's K runs over the
// windows' chunks, each window padded to c2 chunks, with B2 in the same padded row layout.
int64_t i8_seg_rows1(pcaone_ctx* c) { return tile_geom(c).p1 * 2 * kRows; }
int64_t i8_seg_k2(pcaone_ctx* c) { return tile_geom(c).c2 * kChunk; }

int i8_ksplit_seg(pcaone_ctx* c, int which, int nw, int l) {
  const TileGeom g = tile_geom(c);
  return which == 1 ? ks_all(c, (int64_t)nw * g.p1 * 2 * kRows, (int64_t)c->N, np_of(l))
                    : ks_all(c, (int64_t)c->N, (int64_t)nw * g.c2 * kChunk, np_of(l));
}

void i8_p1_seg(pcaone_ctx* c, int b0, int b1, const float*, int l, int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  PG_REQUIRE(b0 >= 0 && b0 < b1 && b1 <= c->win.bands, PCAONE_EBADARG, "bad window run");
  const int np = np_of(l);
  auto* bq = (const int8_t*)scratch(c, "i8_bq1", (size_t)c->Npad * np);
  auto* sig = (const float*)scratch(c, "i8_sig1", 3 * 64 * sizeof(float));
  run_i8(c, tiles_of(c, 1, b0, b1), g.c1,
         (int64_t)(b1 - b0) * g.p1 * 2 * kRows, (int64_t)c->N, bq, sig, c->Npad, l, ks, out);
}

void i8_b2_seg(pcaone_ctx* c, const float* B2, int l, int b0, int b1) {
  const TileGeom g = tile_geom(c);
  const int64_t kpw = g.c2 * kChunk, kpad = (int64_t)(b1 - b0) * kpw;
  const int64_t mtot = (int64_t)(c->win.stop[b1 - 1] - c->win.start[b0]);
  PG_REQUIRE(c->i8_b2_max_ready, PCAONE_ESTATE, "column maxima of the window operand not gathered");
  quantize<float>(c, B2, kpad, l, kpad, "2", c->i8_b2_max_ready, kpw, (int64_t)c->win.blocksize, mtot);
  c->i8_b2_max_ready = false;
}

void i8_p2_seg(pcaone_ctx* c, int b0, int b1, const float*, int l, int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  PG_REQUIRE(b0 >= 0 && b0 < b1 && b1 <= c->win.bands, PCAONE_EBADARG, "bad window run");
  const int64_t kpad = (int64_t)(b1 - b0) * g.c2 * kChunk;
  const int np = np_of(l);
  auto* bq = (const int8_t*)scratch(c, "i8_bq2", (size_t)kpad * np);
  auto* sig = (const float*)scratch(c, "i8_sig2", 3 * 64 * sizeof(float));
  run_i8(c, tiles_of(c, 2, b0, b1), g.c2, (int64_t)c->N, kpad,
         bq, sig, kpad, l, ks, out, g.c2, g.p2 * g.c2 * kPairChunkBytes);
}

}  // namespace

void i8_tile_bytes(const pcaone_ctx* c, size_t* w1, size_t* w2) {
  const TileGeom g = tile_geom(c);
  *w1 = (size_t)g.p1 * g.c1 * kPairChunkBytes;
  *w2 = (size_t)g.p2 * g.c2 * kPairChunkBytes;
}

void i8_tile_window(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, int64_t m, const uint8_t* recT, uint8_t* t1,
                    uint8_t* t2) {
  const TileGeom g = tile_geom(c);
  const int64_t n1 = g.p1 * 2 * kRows * 2 * g.c1, n2 = g.p2 * 2 * kRows * 2 * g.c2;
  k_tile_codes_i8<<<(unsigned)((n1 + 255) / 256), 256, 0, st>>>(rec, c->pitch, m, g.p1, g.c1, t1);
  PG_CHECK_LAUNCH();
  k_tile_codes_i8<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(recT, c->win.pitch, (int64_t)c->N, g.p2, g.c2, t2);
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

GemmFnT<float> gemm_i8() {
  GemmFnT<float> f{i8_ksplit, i8_p1, i8_p2, i8_omega, i8_b2, nullptr, nullptr, i8_b2_qmax};
  f.seg_rows1 = i8_seg_rows1;
  f.seg_k2 = i8_seg_k2;
  f.ksplit_seg = i8_ksplit_seg;
  f.p1_seg = i8_p1_seg;
  f.b2_seg = i8_b2_seg;
  f.p2_seg = i8_p2_seg;
  return f;
}

}  // namespace pg
