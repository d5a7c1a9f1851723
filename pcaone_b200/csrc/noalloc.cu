// Allocation-free variant of the FP32 product Z^T B (pcaone_gpu_product_t_noalloc).
//
// Some callers cannot let a library call cudaMalloc: code that runs inside another
// framework's memory pool (the framework owns all device memory and a private cudaMalloc
// would fragment or oversubscribe it), or a solver loop that must not allocate on its hot
// path, such as an outer eigensolver calling this product as its matrix-vector operator
// thousands of times. This entry point takes the caller's device buffers for B and the
// result and keeps all of its own scratch in one file-scope device array.
//
// Scratch: kScratchBytes = 64 MiB in `g_noalloc_scratch`. Every GPU that loads the library
// holds this array until the process exits. Calls whose scratch need exceeds it are
// rejected with PCAONE_EBADARG. All calls share the array and every call overwrites what it
// uses before reading it, so nothing has to start at zero; calls that overlap on the GPU
// (several host threads, or several streams) race on it and must be serialised by the caller.
#include <algorithm>
#include <mutex>

#include "internal.hpp"

namespace pg {

namespace {

constexpr size_t kScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device, resolved once with that device current.
// In host code the array's name is only a host-side stand-in for the device symbol.
std::mutex g_addr_mu;
void* g_addr[64] = {nullptr};

void* scratch_address(int device) {
  PG_REQUIRE(device >= 0 && device < 64, PCAONE_EBADARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    PG_REQUIRE(e == cudaSuccess && p, PCAONE_ECUDA,
               std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") + cudaGetErrorString(e));
    g_addr[device] = p;
  }
  return g_addr[device];
}

// B (N x l column-major FP64, device) -> Bf (N x l row-major float) and Bd (row-major FP64).
__global__ void k_pack_b(const double* __restrict__ B, uint32_t N, int l, float* __restrict__ Bf,
                         double* __restrict__ Bd) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= (uint64_t)N * l) return;
  const uint64_t i = t / l;
  const int c = (int)(t - i * l);
  const double v = B[(uint64_t)c * N + i];
  Bf[t] = (float)v;
  Bd[t] = v;
}

// wsum[c] = sum_i B[i][c]; one block per column, fixed-order tree reduction.
__global__ void k_colsum(const double* __restrict__ Bd, uint32_t N, int l, double* __restrict__ wsum) {
  __shared__ double sm[256];
  const int c = blockIdx.x;
  double s = 0.0;
  for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) s += Bd[(uint64_t)i * l + c];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st; st >>= 1) {
    if (threadIdx.x < st) sm[threadIdx.x] += sm[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) wsum[c] = sm[0];
}

// out[c * M + j] = s_j (0.5 sum_split D1 - F_j wsum_c + sum_{i miss} (e_ij + F_j) B_ic)
__global__ void k_epilogue(const float* __restrict__ D1, int ks, uint64_t M, int l, const double* __restrict__ F,
                           const double* __restrict__ scale, const double* __restrict__ wsum,
                           const double* __restrict__ Bd, const int64_t* __restrict__ mptr,
                           const int32_t* __restrict__ midx, const double* __restrict__ mval,
                           double* __restrict__ out) {
  const uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= M) return;
  const double f = F[j], s = scale[j];
  const int64_t e0 = mptr[j], e1 = mptr[j + 1];
  for (int c = lane; c < l; c += 32) {
    double d = 0.0;
    for (int sp = 0; sp < ks; ++sp) d += (double)D1[((uint64_t)sp * M + j) * l + c];
    double sparse = 0.0;
    for (int64_t e = e0; e < e1; ++e) sparse += ((mval ? mval[e] : 0.0) + f) * Bd[(uint64_t)midx[e] * l + c];
    out[(uint64_t)c * M + j] = s * (0.5 * d - f * wsum[c] + sparse);
  }
}

}  // namespace

void product_t_noalloc(pcaone_ctx* c, int standardize, int ploidy, const double* d_B, int l, double* d_out) {
  PG_REQUIRE(c->loaded && !c->dense, PCAONE_ESTATE, "no packed genotypes loaded");
  PG_REQUIRE(d_B && d_out && l >= 1 && l <= kLmax, PCAONE_EBADARG, "bad product operands");
  PG_REQUIRE(ploidy == 1 || ploidy == 2, PCAONE_EBADARG, "ploidy must be 1 or 2");
  PG_REQUIRE(c->miss_snp_valid, PCAONE_ESTATE,
             "the missing-genotype list is not built yet: call pcaone_gpu_product (or pcaone_gpu_rsvd) "
             "once on this matrix before the allocation-free product");
  // scratch plan: Bf | Bd | wsum | D1 partials, each 256-byte aligned
  const uint64_t N = c->N, M = c->M;
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t bf = up(N * l * 4), bd = up(N * l * 8), ws = up((size_t)l * 8);
  const size_t per_split = up(M * l * 4);
  const size_t fixed = bf + bd + ws;
  PG_REQUIRE(fixed + per_split <= kScratchBytes, PCAONE_EBADARG,
             "pcaone_gpu_product_t_noalloc: problem needs " + std::to_string(fixed + per_split) +
                 " bytes of scratch, above its fixed maximum of " + std::to_string(kScratchBytes) +
                 " bytes (nsamples*ncols*12 + nsnps*ncols*4); use pcaone_gpu_product");
  // K splits: enough CTAs to fill the GPU, as many as fit in the scratch
  const int64_t tiles = (int64_t)((M + 127) / 128), chunks = (int64_t)((N + 63) / 64);
  int64_t ks = std::max<int64_t>(1, std::min<int64_t>({(2 * (int64_t)c->sm_count + tiles - 1) / tiles,
                                                       chunks / 4, 64}));
  ks = std::min<int64_t>(ks, (int64_t)((kScratchBytes - fixed) / per_split));
  unsigned char* base = (unsigned char*)scratch_address(c->device);
  float* Bf = (float*)base;
  double* Bd = (double*)(base + bf);
  double* wsum = (double*)(base + bf + bd);
  float* D1 = (float*)(base + fixed);

  k_pack_b<<<(unsigned)((N * l + 255) / 256), 256, 0, c->stream>>>(d_B, (uint32_t)N, l, Bf, Bd);
  PG_CHECK_LAUNCH();
  k_colsum<<<l, 256, 0, c->stream>>>(Bd, (uint32_t)N, l, wsum);
  PG_CHECK_LAUNCH();
  compute_scale(c, standardize, ploidy);
  launch_decode_gemm_simt<float>(c, c->d_bed, c->pitch, (int64_t)M, (int64_t)N, Bf, l, l, (int)ks, D1);
  k_epilogue<<<(unsigned)((M * 32 + 255) / 256), 256, 0, c->stream>>>(
      D1, (int)ks, M, l, c->d_F, c->d_scale, wsum, Bd, c->d_miss_snp_ptr, c->d_miss_snp_idx,
      c->imputed ? c->d_miss_snp_val : nullptr, d_out);
  PG_CHECK_LAUNCH();
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->launches += 3;
}

}  // namespace pg

extern "C" int pcaone_gpu_product_t_noalloc(pcaone_ctx* c, int standardize, int ploidy, const double* d_B,
                                            uint32_t ncols, double* d_out) {
  if (!c) return PCAONE_EBADARG;
  try {
    PG_CUDA(cudaSetDevice(c->device));
    pg::require_resident(c, "the allocation-free product");
    pg::product_t_noalloc(c, standardize, ploidy, d_B, (int)ncols, d_out);
    c->err.clear();
    return PCAONE_OK;
  } catch (const pg::Error& e) {
    c->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return PCAONE_ECUDA;
  }
}
