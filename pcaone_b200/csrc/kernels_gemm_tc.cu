// tcgen05 (sm_100a) decode-GEMM: the mixed-precision back end of the two sketch products.
//
//   out[s][r][c] = sum_{k in split s} val(code[r][k]) * (B_hi[k][c] + B_lo[k][c])
//
// val(00, 01, 10, 11) = (2, 0, 1, 0) is exact in BF16; B = B_hi + B_lo is the split-BF16 form
// of the FP32/FP64 sketch operand (Omega for G = Z^T Omega, s/2 * G for H = Z G); the tensor
// core accumulates in FP32 in tensor memory. The epilogue kernels (kernels_epilogue.cu) then
// add the rank-1 centring term and the sparse missing-entry term in FP64.
//
// Work split (stream-K): a unit is one 128-row tile x two consecutive 64-code K chunks (the
// last unit of a tile has one chunk when the tile has an odd number of chunks); units are in
// tile-major order and CTA j of G owns units [j U / G, (j+1) U / G). A CTA therefore covers
// one or more contiguous K ranges ("segments") of one or two tiles; segment q of a tile
// writes its FP32 partial sums to output slot q, and the CTA holding a tile's last unit
// zero-fills the slots that tile does not use, so every row has exactly `ks` slots summed by
// the epilogue in a fixed order (deterministic, no atomics). The grid is two CTAs per SM.
//
// Issue costs set the unit size: a tcgen05.commit costs the issuing thread about as much as
// three or four MMAs and a bulk copy about as much as a commit, so one unit carries eight
// 128 x NP x 16 MMAs, one commit and two copies.
//
// Roles (10 warps):
//   * warp 4 (producer): lane 0 copies the unit's tiled codes (2048 contiguous bytes per
//     chunk) and lane 1 its B chunks (NP rows x 128 bytes per chunk, BF16, already in the
//     128B-swizzled shared-memory image) with 1-D bulk copies (cp.async.bulk) into a ring of
//     ring_stages(NP) shared-memory stages (operand layouts: tc_layout.hpp);
//   * warps 0-3 (decoders) each own 32 rows = the 32 TMEM lanes of their sub-partition: a
//     thread decodes its row's codes in registers (PRMT table lookup) into BF16 pairs and
//     writes them with tcgen05.st into one of two TMEM A stages (A operand in TMEM);
//   * warp 5 (MMA) issues 128 x NP x 16 tcgen05.mma (A from TMEM, B from shared memory) into
//     one of two TMEM accumulators (one when NP > 64); one tcgen05.commit per unit frees the
//     shared-memory stage and, for the decoders two units later, the TMEM A stage;
//   * warps 6-9 (readout) move a finished accumulator to registers with tcgen05.ld, free it
//     for the next segment and store hi + lo sums to the segment's output slot.
// B is [B_hi | B_lo] stacked along N (NP = round_up(2l, 16) columns) so each A tile is read
// by the tensor core once for both halves. The decode emits K pairs in a fixed permuted
// order inside each 64-code chunk; the B operand is written in the same order.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on timeout the CTA sets
// an error flag, stops issuing work, waits (bounded) for its copies and MMAs in flight, frees
// its tensor memory and returns, and the host reports PCAONE_ETIMEOUT.
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.hpp"
#include "rsvd.hpp"
#include "tc_layout.hpp"
#include "tc_ptx.hpp"

namespace pg {

namespace {

constexpr int kTileRows = kTcTileRows;
constexpr int kChunk = kTcChunk;  // codes per K chunk (16 packed bytes per row)
constexpr int kUnitChunks = 2;    // K chunks per unit
constexpr int kAStages = 2;       // decoded A units in TMEM (kUnitChunks x 32 columns each)
constexpr int kThreads = 320;     // 4 decoder warps + producer + MMA + 4 readout warps
constexpr int kTmemCols = 256;    // accumulators in [0, 128), A stages in [128, 256)
constexpr int kAColBase = 128;
constexpr int kMinUnitsPerCta = 4;

// Shared-memory ring depth for NP accumulator columns: about 104 KB of stages, so two CTAs
// (and their 2 x 256 TMEM columns) fit on one SM and a third cannot become resident.
__host__ __device__ constexpr int stage_bytes(int np) { return kUnitChunks * (np * kChunk * 2 + kTileRows * 16); }
__host__ __device__ constexpr int ring_stages(int np) {
  return (104 * 1024) / stage_bytes(np) < 8 ? (104 * 1024) / stage_bytes(np) : 8;
}
__host__ __device__ constexpr int acc_bufs(int np) { return np <= 64 ? 2 : 1; }
static_assert(kAColBase + kAStages * kUnitChunks * 32 <= kTmemCols, "TMEM A stages exceed the allocation");

using tc::bulk_load;
using tc::mbar_arrive;
using tc::mbar_arrive_tx;
using tc::mbar_drain;
using tc::mbar_init;
using tc::mbar_wait;
using tc::smem_desc_sw128;
using tc::smem_u32;
using tc::tmem_ld8;
using tc::tmem_st32;
using tc::tmem_wait_ld;
using tc::tmem_wait_st;
__device__ __forceinline__ void tc_fence_before() { tc::fence_before(); }
__device__ __forceinline__ void tc_fence_after() { tc::fence_after(); }
__device__ __forceinline__ void tc_commit(uint32_t bar) { tc::commit(bar); }
__device__ __forceinline__ void tc_mma(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  tc::mma_f16(d, a, b, idesc, acc);
}

// Decode one 32-bit word (16 codes c0..c15) into 8 BF16 pairs. Output word order:
// (c0,c4) (c8,c12) (c1,c5) (c9,c13) (c2,c6) (c10,c14) (c3,c7) (c11,c15); low half first.
// BF16 bytes per code: 00 -> 2.0 (0x4000), 01 -> 0, 10 -> 1.0 (0x3F80), 11 -> 0.
// prmt selector nibble n in 0..3 picks byte n of kLoTab, 4..7 byte n-4 of kHiTab.
__device__ __forceinline__ void decode_word(uint32_t w, uint32_t* o) {
  constexpr uint32_t kLoTab = 0x00800000u;  // low bytes  (c=0,1,2,3): 00 00 80 00
  constexpr uint32_t kHiTab = 0x003F0040u;  // high bytes (c=0,1,2,3): 40 00 3F 00
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    uint32_t t = (w >> (2 * p)) & 0x03030303u;      // bytes: c_p, c_p+4, c_p+8, c_p+12
    uint32_t s = t * 0x11u + 0x40404040u;           // byte = c | (c + 4) << 4
    uint32_t s2 = __umulhi(t, 0x110000u) + 0x4040u; // bytes 2,3 of t, same mapping
    o[2 * p] = __byte_perm(kLoTab, kHiTab, s);
    o[2 * p + 1] = __byte_perm(kLoTab, kHiTab, s2);
  }
}

struct TcArgs {
  const uint8_t* a_tiles;   // tiled codes of this product (tc_layout.hpp)
  const __nv_bfloat16* bt;  // swizzled chunk-major B (tc_layout.hpp)
  int64_t a_stride;         // chunk stride of the tiled codes (>= chunks)
  int64_t rows;    // valid rows (outputs written for r < rows)
  int64_t chunks;  // K chunks (C)
  int64_t pairs;   // units per tile (P = ceil(C / kUnitChunks))
  int64_t units;   // tiles x P
  int grid;        // CTAs (G)
  int ks;          // output slots per row
  int l;
  float* out;      // [ks][rows][l]
  int* err;
};

__device__ __forceinline__ int64_t unit_begin(int64_t j, const TcArgs& a) { return j * a.units / a.grid; }
// The CTA whose unit range holds unit x.
__device__ __forceinline__ int64_t cta_of_unit(int64_t x, const TcArgs& a) {
  return ((x + 1) * a.grid + a.units - 1) / a.units - 1;
}

template <int NP>
__global__ void __launch_bounds__(kThreads, 2)
k_decode_gemm_tc(const __grid_constant__ TcArgs args) {
  constexpr int S = ring_stages(NP);
  constexpr int NACC = acc_bufs(NP);
  constexpr uint32_t kBChunkBytes = NP * kChunk * 2;  // NP rows x 128 bytes
  constexpr uint32_t kAChunkBytes = kTileRows * 16;
  constexpr uint32_t kBStageBytes = kUnitChunks * kBChunkBytes;
  constexpr uint32_t kAStageBytes = kUnitChunks * kAChunkBytes;
  static_assert(S >= 2, "shared-memory ring too shallow");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the 128B-swizzled B stages
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sB = smem;                          // S x kBStageBytes
  uint8_t* sA = smem + S * kBStageBytes;       // S x kAStageBytes
  uint64_t* bars = (uint64_t*)(sA + S * kAStageBytes);
  uint64_t* full = bars;                       // [S]  bulk copies landed
  uint64_t* empty = bars + S;                  // [S]  MMA done with the unit (stage + TMEM A)
  uint64_t* dec_full = bars + 2 * S;           // [2]  A unit decoded into TMEM
  uint64_t* acc_full = bars + 2 * S + 2;       // [2]  accumulator complete
  uint64_t* acc_empty = acc_full + 2;          // [2]  accumulator read out
  uint64_t* done = acc_full + 4;               // [1]  every MMA of this CTA complete
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(acc_full + 5);
  volatile int* abort_flag = (volatile int*)(acc_full + 6);
  float* stg_all = (float*)(acc_full + 8);       // [4 readout warps][32 rows][9] output staging

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t u0 = unit_begin(blockIdx.x, args), u1 = unit_begin(blockIdx.x + 1, args);
  const int n = (int)(u1 - u0);
  const int64_t P = args.pairs, C = args.chunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&dec_full[b]), 4);
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), 4);
    }
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {  // allocate tensor memory (warp-wide)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32((const void*)tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // ---------------- producer: lane 0 the codes, lane 1 the B chunks of each unit
    if (lane < 2) {  // the two lanes move in lockstep, so every issued unit has its arrive
      int issued = 0;
      int64_t tile = u0 / P, p = u0 - tile * P;
      for (int i = 0; i < n; ++i) {
        const int s = i % S;
        int ok = 1;
        if (lane == 0) ok = mbar_wait(smem_u32(&empty[s]), ((i / S) & 1) ^ 1, abort_flag, args.err, 1);
        ok = __shfl_sync(0x3u, ok, 0);
        if (!ok) break;
        const int64_t kc = p * kUnitChunks;
        const uint32_t nch = (uint32_t)(C - kc < kUnitChunks ? C - kc : kUnitChunks);
        const uint32_t bar = smem_u32(&full[s]);
        if (lane == 0) {
          mbar_arrive_tx(bar, nch * (kAChunkBytes + kBChunkBytes));
          bulk_load(smem_u32(sA + s * kAStageBytes), args.a_tiles + (tile * args.a_stride + kc) * kAChunkBytes,
                    nch * kAChunkBytes, bar);
        } else {
          bulk_load(smem_u32(sB + s * kBStageBytes), args.bt + kc * (int64_t)NP * kChunk, nch * kBChunkBytes, bar);
        }
        issued = i + 1;
        if (++p == P) {
          p = 0;
          ++tile;
        }
      }
      if (*abort_flag && lane == 0) {  // drain copies in flight before the CTA exits
        for (int i = max(0, issued - S); i < issued; ++i) mbar_drain(smem_u32(&full[i % S]), (i / S) & 1);
      }
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = (1u << 4)                 // D: FP32
                                 | (1u << 7) | (1u << 10)  // A, B: BF16
                                 | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(kTileRows >> 4) << 24);
      int seg = 0;
      int64_t p = u0 % P;
      for (int i = 0; i < n; ++i) {
        const int s = i % S, t = i & 1, b = seg % NACC;
        const bool first = (i == 0 || p == 0), last = (i == n - 1 || p == P - 1);
        const int nch = (int)(C - p * kUnitChunks < kUnitChunks ? C - p * kUnitChunks : kUnitChunks);
        if (first) {
          if (!mbar_wait(smem_u32(&acc_empty[b]), ((seg / NACC) & 1) ^ 1, abort_flag, args.err, 2)) break;
        }
        if (!mbar_wait(smem_u32(&full[s]), (i / S) & 1, abort_flag, args.err, 2)) break;
        if (!mbar_wait(smem_u32(&dec_full[t]), (i >> 1) & 1, abort_flag, args.err, 4)) break;
        tc_fence_after();
        const uint32_t b_addr = smem_u32(sB + s * kBStageBytes);
        const uint32_t a_col = tmem + kAColBase + t * (kUnitChunks * 32);  // t < kAStages
        const uint32_t d_col = tmem + b * NP;
        for (int ch = 0; ch < nch; ++ch) {
#pragma unroll
          for (int kk = 0; kk < kChunk / 16; ++kk)
            tc_mma(d_col, a_col + ch * 32 + kk * 8, smem_desc_sw128(b_addr + ch * kBChunkBytes + kk * 32), idesc,
                   (first && ch == 0 && kk == 0) ? 0u : 1u);
        }
        tc_commit(smem_u32(&empty[s]));
        if (last) {
          tc_commit(smem_u32(&acc_full[b]));
          ++seg;
        }
        if (++p == P) p = 0;
      }
      tc_commit(smem_u32(done));  // tracks every MMA issued above
      mbar_drain(smem_u32(done), 0);
    }
  } else if (warp < 4) {
    // ---------------- decoders: row r = 32 * warp + lane, TMEM lanes of this warp
    const int r = warp * 32 + lane;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    int64_t p = u0 % P;
    for (int i = 0; i < n; ++i) {
      const int s = i % S, t = i & 1;
      const int nch = (int)(C - p * kUnitChunks < kUnitChunks ? C - p * kUnitChunks : kUnitChunks);
      if (!mbar_wait(smem_u32(&full[s]), (i / S) & 1, abort_flag, args.err, 8)) break;
      if (i >= 2) {  // the MMAs of unit i - 2 have released TMEM A stage t
        const int j = i - 2;
        if (!mbar_wait(smem_u32(&empty[j % S]), (j / S) & 1, abort_flag, args.err, 8)) break;
      }
      tc_fence_after();
      for (int ch = 0; ch < nch; ++ch) {
        const uint4 q = *reinterpret_cast<const uint4*>(sA + s * kAStageBytes + ch * kAChunkBytes + r * 16);
        uint32_t v[32];
        decode_word(q.x, v);
        decode_word(q.y, v + 8);
        decode_word(q.z, v + 16);
        decode_word(q.w, v + 24);
        tmem_st32(tmem + lane_base + kAColBase + t * (kUnitChunks * 32) + ch * 32, v);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&dec_full[t]));
      if (++p == P) p = 0;
    }
  } else {
    // ---------------- readout warps 6-9: TMEM lanes 32 * (warp % 4) .. + 31
    const int q4 = warp & 3;
    const uint32_t lane_base = (uint32_t)(q4 * 32) << 16;
    int64_t u = u0;
    for (int seg = 0; u < u1; ++seg) {
      const int64_t tile = u / P;
      const int64_t seg_end = min(u1, (tile + 1) * P);
      const bool tile_end = seg_end == (tile + 1) * P;
      const int b = seg % NACC;
      if (!mbar_wait(smem_u32(&acc_full[b]), (seg / NACC) & 1, abort_flag, args.err, 16)) break;
      tc_fence_after();
      const int64_t first_cta = cta_of_unit(tile * P, args);
      const int slot = (int)(blockIdx.x - first_cta);
      // rows row0 .. row0 + nvalid - 1 of this warp are contiguous in the output slot
      const int64_t row0 = tile * kTileRows + q4 * 32;
      const int nvalid = (int)(args.rows - row0 < 32 ? (args.rows - row0 > 0 ? args.rows - row0 : 0) : 32);
      float* stg = stg_all + q4 * 32 * 9;
      float* o = args.out + ((int64_t)slot * args.rows + row0) * args.l;
#pragma unroll
      for (int c0 = 0; c0 < NP / 2; c0 += 8) {  // hi columns c0.., lo columns NP/2 + c0..
        uint32_t hv[8], lv[8];
        tmem_ld8(tmem + lane_base + b * NP + c0, hv);
        tmem_ld8(tmem + lane_base + b * NP + NP / 2 + c0, lv);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 8; ++j) stg[lane * 9 + j] = __uint_as_float(hv[j]) + __uint_as_float(lv[j]);
        __syncwarp();
        // each store instruction writes 4 rows x 8 columns = four full 32-byte sectors
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int rr = 4 * k + (lane >> 3), e = lane & 7;
          if (rr < nvalid && c0 + e < args.l) o[(int64_t)rr * args.l + c0 + e] = stg[rr * 9 + e];
        }
        __syncwarp();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
      if (tile_end) {  // zero the slots this tile does not use: nvalid contiguous rows each
        for (int sl = slot + 1; sl < args.ks; ++sl) {
          float* z = args.out + ((int64_t)sl * args.rows + row0) * args.l;
          for (int t = lane; t < nvalid * args.l; t += 32) z[t] = 0.0f;
        }
      }
      u = seg_end;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// Permuted K position -> code index inside a 64-code chunk (see decode_word).
__host__ __device__ __forceinline__ int chunk_code_of_pos(int pos) {
  const int base[8] = {0, 8, 1, 9, 2, 10, 3, 11};
  int j = pos >> 1, h = pos & 1;
  int q = j >> 3, rr = j & 7;
  return q * 16 + base[rr] + 4 * h;
}

// B operand in the swizzled chunk-major layout (tc_layout.hpp): row n < l holds hi = bf16(x),
// row NP/2 + n holds bf16(x - hi), other rows zero; x = B[k][col] for the code index k of
// permuted position kpos (zero past K). The fixed NP/2 offset of the lo half lets the readout
// add the halves with compile-time register indices.
template <typename T>
__global__ void k_split_bf16(const T* __restrict__ B, int64_t K, int l, int np, int64_t kpad,
                             __nv_bfloat16* __restrict__ Bt) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= kpad * np) return;
  const int n = (int)(t / kpad);
  const int64_t kp = t - (int64_t)n * kpad;
  const int64_t k = (kp / kChunk) * kChunk + chunk_code_of_pos((int)(kp % kChunk));
  float v = 0.0f;
  const int half = np >> 1;
  const bool is_hi = n < l, is_lo = n >= half && n < half + l;
  if ((is_hi || is_lo) && k < K) {
    const int col = is_hi ? n : n - half;
    const float x = (float)B[k * l + col];
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    v = is_hi ? __bfloat162float(hi) : x - __bfloat162float(hi);
  }
  Bt[bt_elem(n, kp, np)] = __float2bfloat16_rn(v);
}

// Tiled copy of one window's codes (tc_layout.hpp): src holds `rows` valid rows of `pitch`
// bytes; tile rows past `rows` are filled with code 11 (value 0). One thread per (row, chunk).
__global__ void k_tile_codes(const uint8_t* __restrict__ src, uint32_t pitch, int64_t rows, int64_t tiles,
                             int64_t chunks, uint8_t* __restrict__ dst) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t total = tiles * kTileRows * chunks;
  if (t >= total) return;
  const int64_t kc = t % chunks, r = t / chunks;  // r: row of the window (tile * 128 + row in tile)
  uint4 v = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
  if (r < rows) v = *reinterpret_cast<const uint4*>(src + r * (int64_t)pitch + kc * 16);
  const int64_t tile = r / kTileRows, rin = r - tile * kTileRows;
  *reinterpret_cast<uint4*>(dst + (tile * chunks + kc) * kTcBlockBytes + rin * 16) = v;
}

// ------------------------------------------------------------------ host side
int np_of(int l) { return (int)round_up(2 * l, 16); }

// At most two CTAs per SM: each allocates 256 of the SM's 512 TMEM columns, so the request is
// at least 100 KB to keep a third CTA from becoming resident.
size_t smem_bytes(int np) {
  const int S = ring_stages(np);
  const size_t need = 1024 + (size_t)S * stage_bytes(np) + (2 * S + 16) * 8 + 4 * 32 * 9 * sizeof(float);
  return std::max<size_t>(need, 100 * 1024);
}

// Stream-K plan of one product: G CTAs over tiles x C units, and the output slots per row
// (the largest number of CTAs that share one tile).
struct TcPlan {
  int64_t tiles = 0, chunks = 0, pairs = 0, units = 0;
  int grid = 0, ks = 1;
};

int64_t plan_cta_of_unit(int64_t x, int64_t units, int grid) { return ((x + 1) * grid + units - 1) / units - 1; }

TcPlan make_plan(const pcaone_ctx* c, int64_t rows, int64_t K) {
  TcPlan p;
  p.tiles = (rows + kTileRows - 1) / kTileRows;
  p.chunks = (K + kChunk - 1) / kChunk;
  p.pairs = (p.chunks + kUnitChunks - 1) / kUnitChunks;
  p.units = p.tiles * p.pairs;
  if (p.units == 0) return p;
  p.grid = (int)std::max<int64_t>(1, std::min<int64_t>(2 * (int64_t)c->sm_count, p.units / kMinUnitsPerCta));
  int ks = 1;
  for (int64_t t = 0; t < p.tiles; ++t) {
    const int64_t a = plan_cta_of_unit(t * p.pairs, p.units, p.grid);
    const int64_t b = plan_cta_of_unit(t * p.pairs + p.pairs - 1, p.units, p.grid);
    ks = std::max<int>(ks, (int)(b - a + 1));
  }
  p.ks = ks;
  return p;
}

template <int NP>
void launch_np(pcaone_ctx* c, const TcArgs& a) {
  const size_t smem = smem_bytes(NP);
  // the attribute belongs to the device's context: set once per library context (one device)
  if (c->smem_attr_set.insert((const void*)k_decode_gemm_tc<NP>).second)
    PG_CUDA(cudaFuncSetAttribute(k_decode_gemm_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_decode_gemm_tc<NP><<<a.grid, kThreads, smem, c->stream>>>(a);
  PG_CHECK_LAUNCH();
}

// One product over the tiled codes of one window (a_stride chunks per tile row, rows valid,
// K codes) and the swizzled B (np x kpad BF16); out holds ks = make_plan(rows, K).ks slots of
// rows x l partial sums.
void run_tc(pcaone_ctx* c, const uint8_t* a_tiles, int64_t a_stride, int64_t rows, int64_t K,
            const __nv_bfloat16* Bt, int64_t kpad, int l, int ks, float* out) {
  const int np = np_of(l);
  PG_REQUIRE(np <= 128, PCAONE_EBADARG, "sketch width too large for the tensor-core path");
  const TcPlan p = make_plan(c, rows, K);
  PG_REQUIRE(ks == p.ks, PCAONE_EBADARG, "output slot count does not match the product plan");
  if (p.units == 0) {
    PG_CUDA(cudaMemsetAsync(out, 0, (size_t)ks * rows * l * sizeof(float), c->stream));
    return;
  }
  PG_REQUIRE(p.chunks <= a_stride && p.chunks * kChunk <= kpad, PCAONE_EBADARG, "K padding too small");
  PG_REQUIRE(((uintptr_t)a_tiles & 15) == 0 && ((uintptr_t)Bt & 15) == 0, PCAONE_EBADARG,
             "operands not 16-byte aligned");
  TcArgs a;
  a.a_tiles = a_tiles;
  a.bt = Bt;
  a.a_stride = a_stride;
  a.rows = rows;
  a.chunks = p.chunks;
  a.pairs = p.pairs;
  a.units = p.units;
  a.grid = p.grid;
  a.ks = p.ks;
  a.l = l;
  a.out = out;
  a.err = (int*)scratch(c, "tc_err", sizeof(int));
  switch (np) {
    case 16: launch_np<16>(c, a); break;
    case 32: launch_np<32>(c, a); break;
    case 48: launch_np<48>(c, a); break;
    case 64: launch_np<64>(c, a); break;
    case 80: launch_np<80>(c, a); break;
    case 96: launch_np<96>(c, a); break;
    case 112: launch_np<112>(c, a); break;
    default: launch_np<128>(c, a); break;
  }
  c->launches++;
  c->gemm_launches++;
}

// Tiled copies of the codes for the current window layout: "tc_tile1" (per window: SNP rows x
// sample chunks, for Z^T Omega) from the SNP-major matrix and "tc_tile2" (per window: sample
// rows x SNP chunks, for Z G) from the per-window transposed copy. Rebuilt when the matrix
// (load, permutation) or the window layout changes.
struct TileGeom {
  int64_t t1, c1, t2, c2;  // tiles per window and chunk stride of tile1 / tile2
};
TileGeom tile_geom(const pcaone_ctx* c) {
  const int64_t bs = (int64_t)c->win.blocksize;
  return TileGeom{(bs + kTileRows - 1) / kTileRows, ((int64_t)c->N + kChunk - 1) / kChunk,
                  ((int64_t)c->N + kTileRows - 1) / kTileRows, (bs + kChunk - 1) / kChunk};
}
void ensure_tiles(pcaone_ctx* c) {
  PG_REQUIRE(c->bedT_valid, PCAONE_ESTATE, "transposed copy not built");
  const uint64_t key = (c->generation << 24) ^ ((uint64_t)c->win.bands << 44) ^ (uint64_t)c->win.blocksize;
  const TileGeom g = tile_geom(c);
  const int bands = c->win.bands;
  const size_t b1 = (size_t)bands * g.t1 * g.c1 * kTcBlockBytes, b2 = (size_t)bands * g.t2 * g.c2 * kTcBlockBytes;
  uint8_t* d1 = (uint8_t*)scratch(c, "tc_tile1", b1);
  uint8_t* d2 = (uint8_t*)scratch(c, "tc_tile2", b2);
  if (c->tiles_valid && c->tiles_key == key && c->tile1_ptr == d1 && c->tile2_ptr == d2) return;
  for (int b = 0; b < bands; ++b) {
    const int64_t s = (int64_t)c->win.start[b], m = (int64_t)c->win.stop[b] - s;
    const int64_t n1 = g.t1 * kTileRows * g.c1, n2 = g.t2 * kTileRows * g.c2;
    k_tile_codes<<<(unsigned)((n1 + 255) / 256), 256, 0, c->stream>>>(
        c->d_bed + s * c->pitch, c->pitch, m, g.t1, g.c1, d1 + (size_t)b * g.t1 * g.c1 * kTcBlockBytes);
    PG_CHECK_LAUNCH();
    k_tile_codes<<<(unsigned)((n2 + 255) / 256), 256, 0, c->stream>>>(
        c->d_bedT + (int64_t)b * c->Npad * c->win.pitch, c->win.pitch, (int64_t)c->N, g.t2, g.c2,
        d2 + (size_t)b * g.t2 * g.c2 * kTcBlockBytes);
    PG_CHECK_LAUNCH();
    c->launches += 2;
  }
  c->tiles_key = key;
  c->tiles_valid = true;
  c->tile1_ptr = d1;
  c->tile2_ptr = d2;
}

template <typename T>
void split_bf16(pcaone_ctx* c, const T* B, int64_t K, int l, int64_t kpad, __nv_bfloat16* Bt) {
  const int np = np_of(l);
  const int64_t tot = kpad * np;
  k_split_bf16<T><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(B, K, l, np, kpad, Bt);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// ---- back-end state kept in named scratch buffers
int tc_ksplit(pcaone_ctx* c, int64_t rows, int64_t K, int) { return make_plan(c, rows, K).ks; }

void tc_omega(pcaone_ctx* c, const double* omega, int l, int64_t npad) {
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt1", (size_t)npad * np_of(l) * 2);
  split_bf16<double>(c, omega, c->N, l, npad, Bt);
}

void tc_b2(pcaone_ctx* c, const float* B2, int l, int64_t m) {
  const int64_t kpad = round_up(c->win.blocksize, 256);
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt2", (size_t)kpad * np_of(l) * 2);
  split_bf16<float>(c, B2, m, l, kpad, Bt);
}

void check_err(pcaone_ctx* c) {
  int* err = (int*)scratch(c, "tc_err", sizeof(int));
  int h = 0;
  PG_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  PG_REQUIRE(h == 0, PCAONE_ETIMEOUT, "tensor-core decode-GEMM: bounded wait expired (code " + std::to_string(h) + ")");
}

void tc_p1(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t row_off, int64_t rows, int64_t K,
           const float*, int l, int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  const int64_t b = row_off / (int64_t)c->win.blocksize;
  PG_REQUIRE(b < c->win.bands && (uint64_t)row_off == c->win.start[b] && K == (int64_t)c->N, PCAONE_EBADARG,
             "first product must cover one window");
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt1", (size_t)c->Npad * np_of(l) * 2);
  run_tc(c, (const uint8_t*)c->tile1_ptr + (size_t)b * g.t1 * g.c1 * kTcBlockBytes, g.c1, rows, K, Bt, c->Npad, l,
         ks, out);
}

void tc_p2(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t window, int64_t rows, int64_t K,
           const float*, int l, int ks, float* out) {
  ensure_tiles(c);
  const TileGeom g = tile_geom(c);
  PG_REQUIRE(window < c->win.bands && rows == (int64_t)c->N, PCAONE_EBADARG, "second product must cover one window");
  const int64_t kpad = round_up(c->win.blocksize, 256);
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt2", (size_t)kpad * np_of(l) * 2);
  run_tc(c, (const uint8_t*)c->tile2_ptr + (size_t)window * g.t2 * g.c2 * kTcBlockBytes, g.c2, rows, K, Bt, kpad,
         l, ks, out);
}

}  // namespace

bool tc_supported(pcaone_ctx* c) { return c->cc_major == 10; }

void tc_clear_error(pcaone_ctx* c) {
  int* err = (int*)scratch(c, "tc_err", sizeof(int));
  PG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
}

void tc_check_error(pcaone_ctx* c) { check_err(c); }

namespace {
__nv_bfloat16* tc_omega_bt(pcaone_ctx* c, int l, int* half) {
  *half = np_of(l) / 2;
  return (__nv_bfloat16*)scratch(c, "tc_bt1", (size_t)c->Npad * np_of(l) * 2);
}
// The split window operand written by the first epilogue. Its unused rows stay zero: the
// buffer is cleared whenever its shape changes.
__nv_bfloat16* tc_b2_bt(pcaone_ctx* c, int l, int64_t* kpad, int* half) {
  *kpad = round_up(c->win.blocksize, 256);
  *half = np_of(l) / 2;
  const size_t bytes = (size_t)(*kpad) * np_of(l) * 2;
  auto* p = (__nv_bfloat16*)scratch(c, "tc_bt2", bytes);
  int64_t& shape = c->bt2_shape;
  const int64_t key = (*kpad) * 1024 + l;
  if (shape != key || (void*)p != c->bt2_ptr) {
    PG_CUDA(cudaMemsetAsync(p, 0, bytes, c->stream));
    shape = key;
    c->bt2_ptr = p;
  }
  return p;
}
}  // namespace

GemmFnT<float> gemm_tc() { return GemmFnT<float>{tc_ksplit, tc_p1, tc_p2, tc_omega, tc_b2, tc_omega_bt, tc_b2_bt}; }

}  // namespace pg
