// tcgen05 (sm_100a) decode-GEMM: the mixed-precision back end of the two sketch products.
//
//   out[s][r][c] = sum_{k in split s} val(code[r][k]) * (B_hi[k][c] + B_lo[k][c])
//
// val(00, 01, 10, 11) = (2, 0, 1, 0) is exact in BF16; B = B_hi + B_lo is the split-BF16 form
// of the FP32/FP64 sketch operand (Omega for G = Z^T Omega, s/2 * G for H = Z G); the tensor
// core accumulates in FP32 in tensor memory. The epilogue kernels (kernels_epilogue.cu) then
// add the rank-1 centring term and the sparse missing-entry term in FP64.
//
// One CTA owns a 128-row tile and one K split. Per 64-code K chunk:
//   * warp 4 (producer) TMA-loads the packed 2-bit codes of the 128 rows (128 x 16 bytes) and
//     the B chunk (NP rows x 64 K, BF16, 128B swizzle) into a shared-memory stage;
//   * warps 0-3 (decoders) each own 32 rows = the 32 TMEM lanes of their sub-partition: a
//     thread decodes its row's 64 codes in registers (PRMT table lookup) into 32 BF16 pairs
//     and writes them with tcgen05.st to the stage's 32 TMEM columns (A operand in TMEM);
//   * warp 5 (MMA) issues four 128 x NP x 16 tcgen05.mma (A from TMEM, B from shared memory)
//     accumulating in TMEM, and tcgen05.commit frees the stage.
// B is [B_hi | B_lo] stacked along N (NP = round_up(2l, 16) columns) so each A tile is read
// by the tensor core once for both halves. The decode emits K pairs in a fixed permuted
// order inside each 64-code chunk; the B operand is written in the same order.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on timeout the CTA sets
// an error flag, stops issuing work, waits (bounded) for its copies in flight, frees its
// tensor memory and returns, and the host reports PCAONE_ETIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "internal.hpp"
#include "rsvd.hpp"

namespace pg {

namespace {

constexpr int kTileRows = 128;
constexpr int kChunk = 64;        // codes per K chunk (16 packed bytes per row)
constexpr int kStages = 4;
constexpr int kThreads = 192;     // 4 decoder warps + producer + MMA
constexpr int kTmemCols = 256;    // accumulator in [0, NP), A stages from column 128
constexpr int kAColBase = 128;
constexpr uint64_t kWaitNs = 1000000000ull;  // bounded waits: 1 s

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait. Returns false (and raises the CTA abort flag / global error) on timeout or
// when another role already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          int* err, int code) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 0) {
      if (*abort_flag) return false;
      if (globaltimer() - t0 > kWaitNs) {
        *abort_flag = 1;
        atomicOr(err, code);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

// Eight 32-bit TMEM columns per call would need eight calls per chunk; one .x32 store
// writes this thread's 32 columns (lane = row) in one instruction.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31, %32};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
      "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
      "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
      "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
        "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128B swizzle, 8-row atoms of 1024 bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
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
  int64_t rows;              // valid rows (outputs written for r < rows)
  int64_t kchunks_total;     // K chunks of the whole problem
  int64_t kchunks_per_split;
  int l;
  float* out;                // [split][rows][l]
  int* err;
};

template <int NP>
__global__ void __launch_bounds__(kThreads, 2)
k_decode_gemm_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 TcArgs args) {
  constexpr uint32_t kBStageBytes = NP * kChunk * 2;  // NP rows x 128 bytes
  constexpr uint32_t kAStageBytes = kTileRows * 16;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the 128B-swizzled B stages
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sB = smem;                                  // kStages x kBStageBytes
  uint8_t* sA = smem + kStages * kBStageBytes;         // kStages x kAStageBytes
  uint64_t* bars = (uint64_t*)(sA + kStages * kAStageBytes);
  uint64_t* tma_full = bars;                 // [kStages]
  uint64_t* dec_full = bars + kStages;       // [kStages]
  uint64_t* empty = bars + 2 * kStages;      // [kStages]
  uint64_t* acc_full = bars + 3 * kStages;   // [1]
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(bars + 3 * kStages + 1);
  volatile int* abort_flag = (volatile int*)(bars + 3 * kStages + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t kc0 = (int64_t)blockIdx.y * args.kchunks_per_split;
  const int64_t kc1 = min(kc0 + args.kchunks_per_split, args.kchunks_total);
  const int nk = kc1 > kc0 ? (int)(kc1 - kc0) : 0;
  const int row0 = blockIdx.x * kTileRows;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&tma_full[s]), 1);
      mbar_init(smem_u32(&dec_full[s]), 4);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(acc_full), 1);
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
    // ---------------- producer: packed codes + B chunk per stage
    if (lane == 0) {
      int issued = 0;
      for (int i = 0; i < nk; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1, abort_flag, args.err, 1)) break;
        const uint32_t bar = smem_u32(&tma_full[s]);
        mbar_arrive_tx(bar, kAStageBytes + kBStageBytes);
        const int kc = (int)(kc0 + i);
        tma_load_2d(smem_u32(sA + s * kAStageBytes), &tmA, kc * 16, row0, bar);
        tma_load_2d(smem_u32(sB + s * kBStageBytes), &tmB, kc * kChunk, 0, bar);
        issued = i + 1;
      }
      if (*abort_flag) {  // drain copies in flight before the CTA exits
        for (int i = max(0, issued - kStages); i < issued; ++i)
          mbar_wait(smem_u32(&tma_full[i % kStages]), (i / kStages) & 1, abort_flag, args.err, 0);
      }
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = (1u << 4)                 // D: FP32
                                 | (1u << 7) | (1u << 10)  // A, B: BF16
                                 | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(kTileRows >> 4) << 24);
      bool ok = true;
      for (int i = 0; i < nk && ok; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        ok = mbar_wait(smem_u32(&tma_full[s]), ph, abort_flag, args.err, 2) &&
             mbar_wait(smem_u32(&dec_full[s]), ph, abort_flag, args.err, 4);
        if (!ok) break;
        tc_fence_after();
        const uint32_t b_addr = smem_u32(sB + s * kBStageBytes);
        const uint32_t a_col = tmem + kAColBase + s * 32;
#pragma unroll
        for (int kk = 0; kk < kChunk / 16; ++kk)
          tc_mma(tmem, a_col + kk * 8, smem_desc_sw128(b_addr + kk * 32), idesc, (i > 0 || kk > 0) ? 1u : 0u);
        tc_commit(smem_u32(&empty[s]));
      }
      tc_commit(smem_u32(acc_full));  // also drains every MMA issued above
    }
  } else {
    // ---------------- decoders (warps 0-3): row r = 32 * warp + lane, TMEM lanes of this warp
    const int r = warp * 32 + lane;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (i / kStages) & 1;
      if (!mbar_wait(smem_u32(&tma_full[s]), ph, abort_flag, args.err, 8)) break;
      const uint4 q = *reinterpret_cast<const uint4*>(sA + s * kAStageBytes + r * 16);
      uint32_t v[32];
      decode_word(q.x, v);
      decode_word(q.y, v + 8);
      decode_word(q.z, v + 16);
      decode_word(q.w, v + 24);
      tmem_st32(tmem + lane_base + kAColBase + s * 32, v);
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&dec_full[s]));
    }
    // ---------------- epilogue: sum hi and lo halves of the accumulator
    const bool ok = mbar_wait(smem_u32(acc_full), 0, abort_flag, args.err, 16);
    tc_fence_after();
    if (ok) {
      float acc[NP];
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        uint32_t t[16];
        tmem_ld16(tmem + lane_base + c0, t);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c0 + j] = nk > 0 ? __uint_as_float(t[j]) : 0.0f;
      }
      const int64_t row = row0 + r;
      if (row < args.rows) {
        float* o = args.out + ((int64_t)blockIdx.y * args.rows + row) * args.l;
        for (int c = 0; c < args.l; ++c) o[c] = acc[c] + acc[args.l + c];
      }
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

// Bt[n][kpos] (NP x kpad, BF16): rows n < l hold bf16(x), rows l..2l-1 hold bf16(x - hi),
// others zero; x = B[k][n] for the code index k of permuted position kpos (zero past K).
template <typename T>
__global__ void k_split_bf16(const T* __restrict__ B, int64_t K, int l, int np, int64_t kpad,
                             __nv_bfloat16* __restrict__ Bt) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= kpad * np) return;
  const int n = (int)(t / kpad);
  const int64_t kp = t - (int64_t)n * kpad;
  const int64_t k = (kp / kChunk) * kChunk + chunk_code_of_pos((int)(kp % kChunk));
  float v = 0.0f;
  if (n < 2 * l && k < K) {
    const int col = n < l ? n : n - l;
    const float x = (float)B[k * l + col];
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    v = n < l ? __bfloat162float(hi) : x - __bfloat162float(hi);
  }
  Bt[t] = __float2bfloat16_rn(v);
}

// ------------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    PG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    PG_REQUIRE(p && q == cudaDriverEntryPointSuccess, PCAONE_ENODEV, "cuTensorMapEncodeTiled unavailable");
    fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

CUtensorMap make_map(CUtensorMapDataType dt, void* base, uint64_t inner, uint64_t outer,
                     uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle sw) {
  PG_REQUIRE(((uintptr_t)base & 15) == 0 && row_bytes % 16 == 0, PCAONE_EBADARG,
             "tensor map base/stride not 16-byte aligned");
  CUtensorMap m;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {row_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PG_REQUIRE(r == CUDA_SUCCESS, PCAONE_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

int np_of(int l) { return (int)round_up(2 * l, 16); }

// At most two CTAs per SM: each allocates 256 of the SM's 512 TMEM columns, so the
// shared-memory request is padded to keep a third CTA from becoming resident.
size_t smem_bytes(int np) {
  size_t need = 1024 + kStages * ((size_t)np * kChunk * 2 + kTileRows * 16) + (3 * kStages + 4) * 8;
  return std::max<size_t>(need, 100 * 1024);
}

template <int NP>
void launch_np(pcaone_ctx* c, const CUtensorMap& ta, const CUtensorMap& tb, const TcArgs& a,
               dim3 grid) {
  static bool attr = false;
  const size_t smem = smem_bytes(NP);
  if (!attr) {
    PG_CUDA(cudaFuncSetAttribute(k_decode_gemm_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  k_decode_gemm_tc<NP><<<grid, kThreads, smem, c->stream>>>(ta, tb, a);
  PG_CHECK_LAUNCH();
}

// One product: codes (rows_alloc x pitch bytes, rows valid), K codes; Bt (np x kpad BF16).
void run_tc(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t rows, int64_t rows_alloc,
            int64_t K, const __nv_bfloat16* Bt, int64_t kpad, int l, int ks, float* out) {
  const int np = np_of(l);
  PG_REQUIRE(np <= 128, PCAONE_EBADARG, "sketch width too large for the tensor-core path");
  PG_REQUIRE((int64_t)round_up(rows, kTileRows) <= rows_alloc, PCAONE_EBADARG, "row padding too small");
  const int64_t nkc = (K + kChunk - 1) / kChunk;
  PG_REQUIRE(nkc * 16 <= (int64_t)pitch && nkc * kChunk <= kpad, PCAONE_EBADARG, "K padding too small");
  CUtensorMap ta = make_map(CU_TENSOR_MAP_DATA_TYPE_UINT8, (void*)codes, pitch, rows_alloc, pitch, 16,
                            kTileRows, CU_TENSOR_MAP_SWIZZLE_NONE);
  CUtensorMap tb = make_map(CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (void*)Bt, kpad, np, kpad * 2, kChunk, np,
                            CU_TENSOR_MAP_SWIZZLE_128B);
  int* err = (int*)scratch(c, "tc_err", sizeof(int));
  TcArgs a;
  a.rows = rows;
  a.kchunks_total = nkc;
  a.kchunks_per_split = (nkc + ks - 1) / ks;
  a.l = l;
  a.out = out;
  a.err = err;
  dim3 grid((unsigned)((rows + kTileRows - 1) / kTileRows), (unsigned)ks);
  switch (np) {
    case 16: launch_np<16>(c, ta, tb, a, grid); break;
    case 32: launch_np<32>(c, ta, tb, a, grid); break;
    case 48: launch_np<48>(c, ta, tb, a, grid); break;
    case 64: launch_np<64>(c, ta, tb, a, grid); break;
    case 80: launch_np<80>(c, ta, tb, a, grid); break;
    case 96: launch_np<96>(c, ta, tb, a, grid); break;
    case 112: launch_np<112>(c, ta, tb, a, grid); break;
    default: launch_np<128>(c, ta, tb, a, grid); break;
  }
  c->launches++;
  c->gemm_launches++;
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
int tc_ksplit(pcaone_ctx* c, int64_t rows, int64_t K) {
  const int64_t tiles = (rows + kTileRows - 1) / kTileRows;
  const int64_t chunks = (K + kChunk - 1) / kChunk;
  const int64_t want = (2 * (int64_t)c->sm_count + tiles - 1) / tiles;
  return (int)std::max<int64_t>(1, std::min<int64_t>({want, chunks / 8, 64}));
}

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

void tc_p1(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t row_off, int64_t rows, int64_t K,
           const float*, int l, int ks, float* out) {
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt1", (size_t)c->Npad * np_of(l) * 2);
  run_tc(c, codes, pitch, rows, (int64_t)c->Mpad - row_off, K, Bt, c->Npad, l, ks, out);
}

void tc_p2(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t, int64_t rows, int64_t K,
           const float*, int l, int ks, float* out) {
  const int64_t kpad = round_up(c->win.blocksize, 256);
  auto* Bt = (__nv_bfloat16*)scratch(c, "tc_bt2", (size_t)kpad * np_of(l) * 2);
  run_tc(c, codes, pitch, rows, c->Npad, K, Bt, kpad, l, ks, out);
}

}  // namespace

bool tc_supported(pcaone_ctx* c) { return c->cc_major == 10; }

void tc_clear_error(pcaone_ctx* c) {
  int* err = (int*)scratch(c, "tc_err", sizeof(int));
  PG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
}

void tc_check_error(pcaone_ctx* c) { check_err(c); }

GemmFnT<float> gemm_tc() { return GemmFnT<float>{tc_ksplit, tc_p1, tc_p2, tc_omega, tc_b2}; }

}  // namespace pg
