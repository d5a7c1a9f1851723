// EM support kernels: the per-SNP standardisation scale and the EMU imputation of missing
// entries (Data::fit_with_pi EMU branch, src/Data.cpp:272-287; Data::standardize_E,
// src/Data.cpp:290-299).
//
// Reference index semantics: after the in-core SNP shuffle the reference keeps F in the
// original SNP order while G's columns are permuted, so the EMU clip bounds and the
// standardisation of the final EMU run read F at the permuted column's position
// (F_load[j] for SNP j of the current order) rather than that SNP's own frequency. With
// imputed_compat the same arrays are used here; without it the SNP's own F is used.
#include "internal.hpp"

namespace pg {

namespace {

__global__ void k_scale(const double* __restrict__ F, uint64_t M, int standardize, int ploidy,
                        double* __restrict__ scale) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= M) return;
  double s = 1.0;
  if (standardize) {
    double sd = sqrt((double)ploidy * F[j] * (1.0 - F[j]));
    if (sd > 1e-9) s = 1.0 / sd;
  }
  scale[j] = s;
}

// e = clip(sum_t US_it V_jt, -Fc, 1 - Fc) with one factor row in registers (`own`, the row
// every entry of the thread's CSR row shares) and the other gathered (`row`, 16-byte loads
// when k is even: the row then starts 16-byte aligned). KM >= k is a compile-time bound.
template <int KM>
__device__ __forceinline__ double imputed_dot(const double* own, const double* __restrict__ row, int k) {
  double g = 0.0;
  if ((k & 1) == 0) {
    const double2* r2 = reinterpret_cast<const double2*>(row);
#pragma unroll
    for (int t = 0; t < KM; t += 2)
      if (t < k) {
        const double2 v = __ldg(r2 + t / 2);
        g += own[t] * v.x;  // sum_k U S V^T, in the order t = 0, 1, ...
        g += own[t + 1] * v.y;
      }
  } else {
#pragma unroll
    for (int t = 0; t < KM; ++t)
      if (t < k) g += own[t] * __ldg(row + t);
  }
  return g;
}

// by-SNP list: warp per SNP row (V_j in registers), lanes over its entries (US_i gathered)
template <int KM>
__global__ void k_impute_snp(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, uint64_t M,
                             const double* __restrict__ US, const double* __restrict__ V, int k,
                             const double* __restrict__ Fc, double* __restrict__ val) {
  uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (j >= M) return;
  double v[KM];
#pragma unroll
  for (int t = 0; t < KM; ++t) v[t] = t < k ? V[j * k + t] : 0.0;
  const double fc = Fc[j];
  for (int64_t e = ptr[j] + lane; e < ptr[j + 1]; e += 32) {
    // same products and order as US_i . V_j
    double g = 0.0;
    const double* us = US + (int64_t)idx[e] * k;
    if ((k & 1) == 0) {
      const double2* u2 = reinterpret_cast<const double2*>(us);
#pragma unroll
      for (int t = 0; t < KM; t += 2)
        if (t < k) {
          const double2 u = __ldg(u2 + t / 2);
          g += u.x * v[t];
          g += u.y * v[t + 1];
        }
    } else {
#pragma unroll
      for (int t = 0; t < KM; ++t)
        if (t < k) g += __ldg(us + t) * v[t];
    }
    val[e] = fmin(fmax(g, -fc), 1.0 - fc);
  }
}

// (window, sample) list: CSR row r = i * nwin + b holds the SNPs of window b missing in sample
// i; warp per row (US_i in registers), lanes over its entries (V_j gathered)
template <int KM>
__global__ void k_impute_ws(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, uint64_t rows,
                            uint32_t nwin, const double* __restrict__ US, const double* __restrict__ V,
                            int k, const double* __restrict__ Fc, double* __restrict__ val) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (r >= rows) return;
  const int64_t i = (int64_t)(r / nwin), e0 = ptr[r], e1 = ptr[r + 1];
  if (e0 == e1) return;
  double us[KM];
#pragma unroll
  for (int t = 0; t < KM; ++t) us[t] = t < k ? US[i * k + t] : 0.0;
  for (int64_t e = e0 + lane; e < e1; e += 32) {
    const int64_t j = idx[e];
    const double g = imputed_dot<KM>(us, V + j * k, k);
    const double fc = Fc[j];
    val[e] = fmin(fmax(g, -fc), 1.0 - fc);
  }
}

// entry weights of the (window, sample) list: the SNP of entry e is idx[e]
__global__ void k_ws_weights(const int32_t* __restrict__ idx, int64_t n, const double* __restrict__ val,
                             const double* __restrict__ scale, const double* __restrict__ F,
                             double* __restrict__ w) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j = idx[e];
    w[e] = scale[j] * (val[e] + F[j]);
  }
}

}  // namespace

void compute_ws_weights(pcaone_ctx* c, const double* F, double* w) {
  PG_REQUIRE(c->miss_ws_valid && c->miss_ws_val_valid, PCAONE_ESTATE, "imputed values not set");
  if (c->n_missing == 0) return;
  const unsigned nblk = (unsigned)std::min<int64_t>(8 * (int64_t)c->sm_count, (c->n_missing + 255) / 256);
  k_ws_weights<<<nblk, 256, 0, c->stream>>>(c->d_miss_ws_idx, c->n_missing, c->d_miss_ws_val, c->d_scale, F, w);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void compute_scale(pcaone_ctx* c, int standardize, int ploidy) {
  const double* Fs = (c->imputed && c->imputed_compat) ? c->d_F_load : c->d_F;
  k_scale<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(Fs, c->M, standardize, ploidy, c->d_scale);
  PG_CHECK_LAUNCH();
  c->launches++;
}

static const double* clip_freq(pcaone_ctx* c) { return c->imputed_compat ? c->d_F_load : c->d_F; }

void compute_imputed_snp(pcaone_ctx* c) {
  PG_REQUIRE(c->miss_snp_valid, PCAONE_ESTATE, "missing-entry list not built");
  c->d_miss_snp_val = (double*)scratch(c, "d_miss_snp_val", std::max<int64_t>(c->n_missing, 1) * 8);
  uint64_t threads = c->M * 32;
  auto go = [&](auto kern) {
    kern<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(c->d_miss_snp_ptr, c->d_miss_snp_idx, c->M,
                                                                   c->d_imp_US, c->d_imp_V, c->imp_k, clip_freq(c),
                                                                   c->d_miss_snp_val);
  };
  if (c->imp_k <= 8) go(k_impute_snp<8>);
  else if (c->imp_k <= 16) go(k_impute_snp<16>);
  else if (c->imp_k <= 32) go(k_impute_snp<32>);
  else go(k_impute_snp<64>);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void compute_imputed_ws(pcaone_ctx* c) {
  if (c->miss_ws_val_valid) return;
  PG_REQUIRE(c->miss_ws_valid, PCAONE_ESTATE, "missing-entry list not built");
  c->d_miss_ws_val = (double*)scratch(c, "d_miss_ws_val", std::max<int64_t>(c->n_missing, 1) * 8);
  const uint64_t rows = (uint64_t)c->win.bands * c->Npad;
  uint64_t threads = rows * 32;
  auto go = [&](auto kern) {
    kern<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(c->d_miss_ws_ptr, c->d_miss_ws_idx, rows,
                                                                   (uint32_t)c->win.bands, c->d_imp_US, c->d_imp_V,
                                                                   c->imp_k, clip_freq(c), c->d_miss_ws_val);
  };
  if (c->imp_k <= 8) go(k_impute_ws<8>);
  else if (c->imp_k <= 16) go(k_impute_ws<16>);
  else if (c->imp_k <= 32) go(k_impute_ws<32>);
  else go(k_impute_ws<64>);
  PG_CHECK_LAUNCH();
  c->launches++;
  c->miss_ws_val_valid = true;
}

}  // namespace pg
