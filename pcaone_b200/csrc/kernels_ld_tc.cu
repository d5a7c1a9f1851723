// Windowed LD r2 (flow A) on the tcgen05 tensor cores: the band of the SNP x SNP Gram matrix
// that the windows cover, as exact integer products of decoded genotype tiles.
//
// The centred cross product of two SNPs needs four integer sums over the samples (the same
// identity as the bit-plane kernel in kernels_ld.cu):
//
//   4 Gc_i.Gc_k = RR - 2 F_k RN - 2 F_i NR + 4 F_i F_k NN,
//   RR = sum r_i r_k, RN = sum r_i n_k, NR = sum n_i r_k, NN = sum n_i n_k,
//
// with r the A1 count (00 -> 2, 10 -> 1, 11 -> 0, missing 01 -> 0) and n the non-missing
// indicator. For a 128 x 128 tile of SNP pairs (lead tile I, partner tile K) two kind::i8 MMAs
// per 32 samples give all four at once: D0 = R_I [R_K; N_K]^T and D1 = N_I [R_K; N_K]^T
// (M = 128, N = 256, unsigned 8-bit operands, exact int32 accumulation; the two accumulators
// fill the 512 tensor-memory columns). The residualisation and the normalisation are FP64
// in the readout: r_ik = (Gc_i.Gc_k - W_i . Y_k) / sqrt(d_i d_k).
//
// The band is one persistent launch over a host-built list of (I, K) tiles: every lead tile
// pairs with the partner tiles its windows reach, whatever their uneven lengths, and CTA j
// takes tiles j, j + G, ... (all tiles cost the same K loop).
//
// Roles (14 warps, one CTA per SM):
//   * warp 0 (producer): lane 0 copies the packed codes of both tiles for one 128-sample chunk
//     (2 x 4 KB, tiled by k_ld_tile_codes) with 1-D bulk copies into a ring of raw stages;
//   * warps 1-8 (decoders): warp 1 + 4 s + q decodes the rows 32 q .. of tile s (0 = I,
//     1 = K): one thread per SNP row turns 128 codes into 128 bytes of r and 128 bytes of n
//     (PRMT lookups; both operands share the same in-chunk sample order, which a dot product
//     does not see) and stores them 128-byte-swizzled into a decoded stage, then makes the
//     stores visible to the tensor core (fence.proxy.async);
//   * warp 9 (MMA): lane 0 issues the 8 MMAs of a chunk and one tcgen05.commit that frees the
//     decoded stage; after the last chunk of a tile a commit signals the readout;
//   * warps 10-13 (readout): lanes = the 128 lead SNPs; each thread reads its row of both
//     accumulators with tcgen05.ld and writes r2 for the pairs inside its SNP's window.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on timeout the CTA sets
// an error flag, stops issuing work, drains its copies and MMAs in flight, frees its tensor
// memory and returns, and the host reports PCAONE_ETIMEOUT.
#include <algorithm>

#include "internal.hpp"
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

constexpr int kTile = 128;                     // SNPs per tile
constexpr int kChunk = 128;                    // samples per K chunk
constexpr int kRawTile = kTile * kChunk / 4;   // packed bytes of one tile chunk: 4096
constexpr int kImg = kTile * kChunk;           // one decoded operand image (r or n): 16384
constexpr int kRS = 2;                         // raw stages (codes of both tiles)
constexpr int kDS = 3;                         // decoded stages (r_I, n_I, r_K, n_K)
constexpr int kStageD = 4 * kImg;              // 65536
constexpr int kThreads = 448;
constexpr int kTmemCols = 512;
constexpr int kMaxProj = 16;                   // largest projection width k of this kernel

// Decode one 32-bit word (16 codes) into 16 bytes with the lookup table lut (one byte per
// code value); byte order c0, c2, c4, c6 | c8 .. c14 | c1, c3, c5, c7 | c9 .. c15.
__device__ __forceinline__ void decode_word(uint32_t w, uint32_t lut, uint32_t* o) {
  const uint32_t x = w & 0x33333333u, y = (w >> 2) & 0x33333333u;
  o[0] = __byte_perm(lut, 0u, x);
  o[1] = __byte_perm(lut, 0u, x >> 16);
  o[2] = __byte_perm(lut, 0u, y);
  o[3] = __byte_perm(lut, 0u, y >> 16);
}

// Warp-uniform bounded wait: lane 0 waits, the outcome is broadcast and the warp
// re-converges (its other lanes then see what lane 0 acquired).
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          int code) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort_flag, err, code) ? 1 : 0;
  ok = __shfl_sync(0xffffffffu, ok, 0);
  __syncwarp();
  return ok != 0;
}

struct LdArgs {
  const uint8_t* tiles;    // [tile][chunk] blocks of 128 rows x 32 bytes
  const int2* list;        // (lead tile, partner tile) pairs
  int ntiles, nchunks;
  uint64_t M;
  const double* F;         // M
  const double* isd;       // M, 1 / |G_i| of the residualised columns (inf / NaN kept: r is NaN then)
  const double* W;         // M x k row-major, or null
  const double* Y;         // M x k row-major, or null
  int k;
  const int64_t* win_of;   // M: window led by SNP i, or -1
  const int32_t* we;       // window lengths (lead included)
  const int64_t* off;      // first pair of each window in r2
  void* r2;                // float, or double with f64
  int f64;
  int* err;
};

__global__ void __launch_bounds__(kThreads, 1) k_ld_gram_i8(const __grid_constant__ LdArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sD = smem;                          // kDS x [r_I | n_I | r_K | n_K]
  uint8_t* sR = sD + kDS * kStageD;            // kRS x [I codes | K codes]
  uint64_t* bars = (uint64_t*)(sR + kRS * 2 * kRawTile);
  uint64_t* raw_full = bars;                   // [kRS]
  uint64_t* raw_empty = bars + kRS;            // [kRS] 8 decoder warps
  uint64_t* dec_full = bars + 2 * kRS;         // [kDS] 8 decoder warps
  uint64_t* dec_empty = dec_full + kDS;        // [kDS] MMA commit
  uint64_t* acc_full = dec_empty + kDS;        // MMA commit
  uint64_t* acc_empty = acc_full + 1;          // 4 readout warps
  uint64_t* done = acc_full + 2;               // every MMA complete
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(acc_full + 3);
  volatile int* abort_flag = (volatile int*)(acc_full + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int my_tiles = a.ntiles > (int)blockIdx.x ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nc = a.nchunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kRS; ++s) {
      mbar_init(smem_u32(&raw_full[s]), 1);
      mbar_init(smem_u32(&raw_empty[s]), 8);
    }
    for (int s = 0; s < kDS; ++s) {
      mbar_init(smem_u32(&dec_full[s]), 8);
      mbar_init(smem_u32(&dec_empty[s]), 1);
    }
    mbar_init(smem_u32(acc_full), 1);
    mbar_init(smem_u32(acc_empty), 4);
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 9) tc::tmem_alloc(smem_u32((const void*)tmem_slot), kTmemCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;
  const int64_t total = (int64_t)my_tiles * nc;  // chunks this CTA runs

  if (warp == 0) {
    // ---------------- producer
    if (lane == 0) {
      int64_t issued = 0;
      for (int64_t g = 0; g < total; ++g) {
        const int s = (int)(g % kRS);
        if (!mbar_wait(smem_u32(&raw_empty[s]), (uint32_t)(((g / kRS) & 1) ^ 1), abort_flag, a.err, 1)) break;
        const int t = (int)blockIdx.x + (int)(g / nc) * (int)gridDim.x, c = (int)(g % nc);
        const int2 tk = a.list[t];
        const uint32_t bar = smem_u32(&raw_full[s]);
        mbar_arrive_tx(bar, 2 * kRawTile);
        bulk_load(smem_u32(sR + s * 2 * kRawTile), a.tiles + ((int64_t)tk.x * nc + c) * kRawTile, kRawTile, bar);
        bulk_load(smem_u32(sR + s * 2 * kRawTile + kRawTile), a.tiles + ((int64_t)tk.y * nc + c) * kRawTile, kRawTile,
                  bar);
        issued = g + 1;
      }
      if (*abort_flag)
        for (int64_t g = issued > kRS ? issued - kRS : 0; g < issued; ++g)
          mbar_drain(smem_u32(&raw_full[g % kRS]), (uint32_t)((g / kRS) & 1));
    }
  } else if (warp >= 1 && warp <= 8) {
    // ---------------- decoders: tile side sd (0 = I, 1 = K), rows 32 q + lane
    const int dw = warp - 1, sd = dw >> 2, q = dw & 3, r = q * 32 + lane;
    constexpr uint32_t kLutR = 0x00010002u;  // 00 -> 2, 01 -> 0, 10 -> 1, 11 -> 0
    constexpr uint32_t kLutN = 0x01010001u;  // 00 -> 1, 01 -> 0, 10 -> 1, 11 -> 1
    for (int64_t g = 0; g < total; ++g) {
      const int s = (int)(g % kRS), sdec = (int)(g % kDS);
      if (!warp_wait(smem_u32(&raw_full[s]), (uint32_t)((g / kRS) & 1), abort_flag, a.err, 8)) break;
      if (!warp_wait(smem_u32(&dec_empty[sdec]), (uint32_t)(((g / kDS) & 1) ^ 1), abort_flag, a.err, 8)) break;
      const uint8_t* src = sR + s * 2 * kRawTile + sd * kRawTile + r * 32;
      const uint4 h0 = *reinterpret_cast<const uint4*>(src);
      const uint4 h1 = *reinterpret_cast<const uint4*>(src + 16);
      const uint32_t wd[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
      uint8_t* imgR = sD + sdec * kStageD + (2 * sd) * kImg;
      uint8_t* imgN = imgR + kImg;
      const int rowoff = (r >> 3) * 1024 + (r & 7) * 128;
#pragma unroll
      for (int u = 0; u < 8; ++u) {  // 16 codes -> one 16-byte unit of the row
        uint32_t vr[4], vn[4];
        decode_word(wd[u], kLutR, vr);
        decode_word(wd[u], kLutN, vn);
        const int o = rowoff + ((u ^ (r & 7)) << 4);
        *reinterpret_cast<uint4*>(imgR + o) = make_uint4(vr[0], vr[1], vr[2], vr[3]);
        *reinterpret_cast<uint4*>(imgN + o) = make_uint4(vn[0], vn[1], vn[2], vn[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> tensor core
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(smem_u32(&raw_empty[s]));
        mbar_arrive(smem_u32(&dec_full[sdec]));
      }
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = (2u << 4)                 // D: S32
                                 | (0u << 7) | (0u << 10)  // A, B: unsigned 8-bit
                                 | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
      for (int64_t g = 0; g < total; ++g) {
        const int sdec = (int)(g % kDS), c = (int)(g % nc);
        const int64_t tt = g / nc;
        if (c == 0 && !mbar_wait(smem_u32(acc_empty), (uint32_t)((tt & 1) ^ 1), abort_flag, a.err, 2)) break;
        if (!mbar_wait(smem_u32(&dec_full[sdec]), (uint32_t)((g / kDS) & 1), abort_flag, a.err, 2)) break;
        tc::fence_after();
        const uint32_t base = smem_u32(sD + sdec * kStageD);
#pragma unroll
        for (int kk = 0; kk < kChunk / 32; ++kk) {
          const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
          const uint64_t bdesc = smem_desc_sw128(base + 2 * kImg + kk * 32);  // [r_K; n_K]: N = 256
          tc::mma_i8_ss(tmem, smem_desc_sw128(base + kk * 32), bdesc, idesc, acc);              // r_I
          tc::mma_i8_ss(tmem + 256, smem_desc_sw128(base + kImg + kk * 32), bdesc, idesc, acc);  // n_I
        }
        tc::commit(smem_u32(&dec_empty[sdec]));
        if (c == nc - 1) tc::commit(smem_u32(acc_full));
      }
      tc::commit(smem_u32(done));
      mbar_drain(smem_u32(done), 0);
    }
  } else {
    // ---------------- readout warps 10-13: lead rows 32 q4 + lane
    const int q4 = warp & 3;
    const int rw = q4 * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q4 * 32) << 16;
    const int k = a.k;
    for (int tt = 0; tt < my_tiles; ++tt) {
      if (!warp_wait(smem_u32(acc_full), (uint32_t)(tt & 1), abort_flag, a.err, 16)) break;
      tc::fence_after();
      const int2 tk = a.list[(int)blockIdx.x + tt * (int)gridDim.x];
      const uint64_t i = (uint64_t)tk.x * kTile + rw, k0 = (uint64_t)tk.y * kTile;
      int64_t w = -1;
      double Fi = 0.0, isdi = 1.0;
      double wi[kMaxProj];
#pragma unroll
      for (int t = 0; t < kMaxProj; ++t) wi[t] = 0.0;
      if (i < a.M) {
        w = a.win_of[i];
        Fi = a.F[i];
        isdi = a.isd[i];
        if (a.W)
#pragma unroll
          for (int t = 0; t < kMaxProj; ++t)
            if (t < k) wi[t] = a.W[i * k + t];
      }
      const int len = w >= 0 ? a.we[w] : 0;
      const int64_t base_out = w >= 0 ? a.off[w] : 0;
      // columns of this tile that can be inside the window: k - i in [1, len)
      const int64_t lo = (int64_t)i + 1 - (int64_t)k0, hi = (int64_t)i + len - 1 - (int64_t)k0;
      const bool any = w >= 0 && hi >= 0 && lo < kTile;
      // every lane must join the collective TMEM loads: a warp reads a column chunk when
      // one of its lanes needs it
      const int clo = any ? (int)(lo > 0 ? lo : 0) : kTile, chi = any ? (int)(hi < kTile - 1 ? hi : kTile - 1) : -1;
      int wlo = clo, whi = chi;
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        wlo = min(wlo, __shfl_xor_sync(0xffffffffu, wlo, o));
        whi = max(whi, __shfl_xor_sync(0xffffffffu, whi, o));
      }
      for (int c0 = (wlo / 8) * 8; c0 <= whi; c0 += 8) {
        uint32_t rr[8], rn[8], nr[8], nn[8];
        tc::tmem_ld8(tmem + lane_base + c0, rr);
        tc::tmem_ld8(tmem + lane_base + 128 + c0, rn);
        tc::tmem_ld8(tmem + lane_base + 256 + c0, nr);
        tc::tmem_ld8(tmem + lane_base + 384 + c0, nn);
        tc::tmem_wait_ld();
        // the chunk's partner values, the same for every lane (broadcast loads)
        double Fk8[8], isk8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint64_t kk = k0 + c0 + j;
          Fk8[j] = kk < a.M ? __ldg(a.F + kk) : 0.0;
          isk8[j] = kk < a.M ? __ldg(a.isd + kk) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int col = c0 + j;
          if (col < clo || col > chi) continue;
          const uint64_t kk = k0 + col;
          if (kk >= a.M) continue;
          const double Fk = Fk8[j];
          double num = 0.25 * ((double)(int)rr[j] - 2.0 * Fk * (double)(int)rn[j] - 2.0 * Fi * (double)(int)nr[j]) +
                       Fi * Fk * (double)(int)nn[j];
          if (a.W) {  // the lanes of a warp read the same partner row: broadcast loads
            const double* yk = a.Y + kk * k;
#pragma unroll
            for (int t = 0; t < kMaxProj; ++t)
              if (t < k) num -= wi[t] * __ldg(yk + t);
          }
          const double rv = num * isdi * isk8[j];
          const int64_t o = base_out + (int64_t)(kk - i) - 1;
          if (a.f64)
            ((double*)a.r2)[o] = rv * rv;
          else
            ((float*)a.r2)[o] = (float)(rv * rv);
        }
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(acc_empty));
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 9) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// Tiled codes for the Gram kernel: block (SNP tile t, sample chunk c) = 128 rows x 32 bytes,
// row = the chunk's 128 codes of SNP 128 t + row. Samples past N and rows past M are code 01
// (missing: r = n = 0), so padding adds nothing to any sum. Thread per (row, 16-byte half).
__global__ void k_ld_tile_codes(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t M, uint32_t N,
                                int64_t ntile, int nchunks, uint8_t* __restrict__ dst) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t halves = 2 * (int64_t)nchunks;
  if (t >= ntile * kTile * halves) return;
  const int64_t row = t / halves, hc = t - row * halves;
  const int64_t c = hc >> 1, h = hc & 1;
  uint32_t w[4] = {0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u};
  const int64_t s0 = c * kChunk + h * 64;  // first sample of these 64 codes
  if ((uint64_t)row < M) {
    const uint8_t* src = bed + (uint64_t)row * pitch;
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // 16 samples per word
      const int64_t sq = s0 + 16 * q;
      if (sq >= (int64_t)N) break;
      uint32_t x = 0;
      if (sq + 16 <= (int64_t)N) {
        x = *reinterpret_cast<const uint32_t*>(src + sq / 4);
      } else {
        for (int b = 0; b < 4; ++b)
          if (sq + 4 * b < (int64_t)N) x |= (uint32_t)src[sq / 4 + b] << (8 * b);
        const int valid = (int)((int64_t)N - sq);  // 1..15 codes
        const uint32_t keep = (1u << (2 * valid)) - 1u;
        x = (x & keep) | (0x55555555u & ~keep);
      }
      w[q] = x;
    }
  }
  const int64_t tile = row / kTile, rin = row - tile * kTile;
  *reinterpret_cast<uint4*>(dst + (tile * nchunks + c) * kRawTile + rin * 32 + h * 16) = make_uint4(w[0], w[1], w[2], w[3]);
}

constexpr size_t ld_smem_bytes() { return 1024 + (size_t)kDS * kStageD + (size_t)kRS * 2 * kRawTile + 16 * 8; }

// Warp per SNP: 1 / |G_i| with |G_i|^2 = d_i of the residualised column from the code counts
// of its first N samples (RR = 4 n00 + n10, RN = NR = 2 n00 + n10, NN = non-missing) minus
// W_i . Y_i; a zero or negative d_i gives inf or NaN, so r is NaN as the reference's 0 / 0.
__global__ void k_ld_diag_codes(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t M, uint32_t N,
                                const double* __restrict__ F, const double* __restrict__ W,
                                const double* __restrict__ Y, int k, double* __restrict__ isd) {
  const uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= M) return;
  const uint8_t* rec = bed + i * pitch;
  long long n00 = 0, n10 = 0, nm = 0;
  for (uint32_t b = lane; b < (N + 3) / 4; b += 32) {
    const uint32_t x = rec[b];
    for (int q = 0; q < 4; ++q) {
      if (4 * b + q >= N) break;
      const uint32_t code = (x >> (2 * q)) & 3u;
      n00 += code == 0;
      n10 += code == 2;
      nm += code != 1;
    }
  }
  double wy = 0.0;
  if (W)
    for (int t = lane; t < k; t += 32) wy += W[i * k + t] * Y[i * k + t];
  for (int o = 16; o; o >>= 1) {
    n00 += __shfl_xor_sync(0xffffffffu, n00, o);
    n10 += __shfl_xor_sync(0xffffffffu, n10, o);
    nm += __shfl_xor_sync(0xffffffffu, nm, o);
    wy += __shfl_xor_sync(0xffffffffu, wy, o);
  }
  if (lane == 0) {
    const double f = F[i], rr = (double)(4 * n00 + n10), rn = (double)(2 * n00 + n10);
    const double d = 0.25 * (rr - 4.0 * f * rn) + f * f * (double)nm - wy;
    isd[i] = 1.0 / sqrt(d);
  }
}

}  // namespace

bool ld_tc_usable(pcaone_ctx* c, int k) { return tc_supported(c) && k <= kMaxProj; }

void ld_r2_tc(pcaone_ctx* c, const double* W, const double* Y, int k, const int64_t* ws, const int32_t* we,
              uint64_t nwin, const int64_t* d_win_of, const int32_t* d_we, const int64_t* d_off, void* d_r2, bool f64) {
  PG_REQUIRE(k <= kMaxProj, PCAONE_EBADARG, "projection too wide for the tensor-core LD kernel");
  const uint64_t M = c->M;
  cudaEvent_t ev[3];
  for (auto& e : ev) PG_CUDA(cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  PG_CUDA(cudaEventRecord(ev[0], c->stream));
  double* isd = (double*)scratch(c, "ld_isd", M * 8);
  k_ld_diag_codes<<<(unsigned)((M * 32 + 255) / 256), 256, 0, c->stream>>>(c->d_bed, c->pitch, M, c->N, c->d_F,
                                                                           k > 0 ? W : nullptr, Y, k, isd);
  PG_CHECK_LAUNCH();
  c->launches++;
  const int64_t ntile = (int64_t)((M + kTile - 1) / kTile);
  const int nchunks = (int)((c->N + kChunk - 1) / kChunk);
  // tile list: lead tile b pairs with the partner tiles its windows reach
  std::vector<int64_t> reach(ntile, -1);
  for (uint64_t w = 0; w < nwin; ++w) {
    if (we[w] < 2) continue;
    const int64_t b = ws[w] / kTile;
    reach[b] = std::max<int64_t>(reach[b], ws[w] + we[w] - 1);
  }
  std::vector<int2> list;
  for (int64_t b = 0; b < ntile; ++b)
    if (reach[b] >= 0)
      for (int64_t q = b; q <= reach[b] / kTile; ++q) list.push_back(make_int2((int)b, (int)q));
  if (list.empty()) {
    c->ld_device_ms = c->ld_gram_ms = 0.0;
    return;
  }
  PG_REQUIRE(ntile < (1ll << 31), PCAONE_EBADARG, "LD band too large");
  const size_t tile_bytes = (size_t)ntile * nchunks * kRawTile;
  uint8_t* tiles = (uint8_t*)scratch(c, "ld_tc_tiles", tile_bytes);
  {
    const int64_t n = ntile * kTile * 2 * nchunks;
    k_ld_tile_codes<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_bed, c->pitch, M, c->N, ntile, nchunks,
                                                                      tiles);
    PG_CHECK_LAUNCH();
  }
  int2* d_list = (int2*)scratch(c, "ld_tc_list", list.size() * sizeof(int2));
  PG_CUDA(cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  LdArgs a;
  a.tiles = tiles;
  a.list = d_list;
  a.ntiles = (int)list.size();
  a.nchunks = nchunks;
  a.M = M;
  a.F = c->d_F;
  a.isd = isd;
  a.W = k > 0 ? W : nullptr;
  a.Y = k > 0 ? Y : nullptr;
  a.k = k;
  a.win_of = d_win_of;
  a.we = d_we;
  a.off = d_off;
  a.r2 = d_r2;
  a.f64 = f64 ? 1 : 0;
  a.err = (int*)scratch(c, "tc_err", sizeof(int));
  constexpr size_t smem = ld_smem_bytes();
  static_assert(smem <= 227 * 1024, "shared memory above the per-CTA limit");
  if (c->smem_attr_set.insert((const void*)k_ld_gram_i8).second)
    PG_CUDA(cudaFuncSetAttribute(k_ld_gram_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>((int64_t)c->sm_count, (int64_t)list.size());
  PG_CUDA(cudaEventRecord(ev[1], c->stream));
  k_ld_gram_i8<<<grid, kThreads, smem, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  PG_CUDA(cudaEventRecord(ev[2], c->stream));
  c->launches += 2;
  PG_CUDA(cudaEventSynchronize(ev[2]));
  float t_all = 0.f, t_gram = 0.f;
  PG_CUDA(cudaEventElapsedTime(&t_all, ev[0], ev[2]));
  PG_CUDA(cudaEventElapsedTime(&t_gram, ev[1], ev[2]));
  c->ld_device_ms = t_all;
  c->ld_gram_ms = t_gram;
}

}  // namespace pg
