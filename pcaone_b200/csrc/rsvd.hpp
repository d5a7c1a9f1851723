// RSVD driver and the decode-GEMM back ends it can run on.
#pragma once

#include <cuda_bf16.h>

#include "internal.hpp"

namespace pg {

// A decode-GEMM back end. p1/p2 compute out[s][r][c] = sum_k val(code[r][k]) * B[k][c]
// over K split into `ks` ranges (see kernels_gemm_simt.cu); B is row-major K x l.
// omega_changed / b2_ready let a back end re-pack the B operands into its own layout.
template <typename T>
struct GemmFnT {
  int (*ksplit)(pcaone_ctx* c, int64_t rows, int64_t K, int l);
  // p1: rows = SNPs row0..row0+rows of the SNP-major matrix; p2: rows = samples of window
  // `window` of the sample-major copy. `codes` points at the first row of the packed data.
  void (*p1)(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t row0, int64_t rows,
             int64_t K, const T* B, int l, int ks, T* out);
  void (*p2)(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t window, int64_t rows,
             int64_t K, const T* B, int l, int ks, T* out);
  void (*omega_changed)(pcaone_ctx* c, const double* omega, int l, int64_t npad);
  void (*b2_ready)(pcaone_ctx* c, const T* B2, int l, int64_t m);
  // Split-BF16 operand buffers in the tensor-core layout (nullptr for the SIMT back ends):
  // when non-null, the fused Omega update and the first epilogue write them directly.
  // *half receives the row offset of the lo halves.
  __nv_bfloat16* (*omega_bt)(pcaone_ctx* c, int l, int* half) = nullptr;
  __nv_bfloat16* (*b2_bt)(pcaone_ctx* c, int l, int64_t* kpad, int* half) = nullptr;
  // Zeroed per-column maxima of |B2| for the first epilogue to fill (int8 back end), or null.
  unsigned long long* (*b2_qmax)(pcaone_ctx* c, int l) = nullptr;
  // Runs of consecutive windows [b0, b1) as one product each (null: one window at a time).
  // The first product writes seg_rows1 rows per window (SNP rows, zero padding rows); the
  // second reads B2 with seg_k2 rows per window (window SNPs first, zero rows after);
  // ksplit_seg(which = 1 or 2, windows, l) is the split count of either product.
  int64_t (*seg_rows1)(pcaone_ctx* c) = nullptr;
  int64_t (*seg_k2)(pcaone_ctx* c) = nullptr;
  int (*ksplit_seg)(pcaone_ctx* c, int which, int nw, int l) = nullptr;
  // B: the first product's operand (Omega, engine layout) / the run's B2 (seg_k2 rows per
  // window); back ends that keep their own packed copy ignore it.
  void (*p1_seg)(pcaone_ctx* c, int b0, int b1, const T* B, int l, int ks, T* out) = nullptr;
  void (*b2_seg)(pcaone_ctx* c, const T* B2, int l, int b0, int b1) = nullptr;
  void (*p2_seg)(pcaone_ctx* c, int b0, int b1, const T* B2, int l, int ks, T* out) = nullptr;
};

GemmFnT<float> gemm_simt_float();
GemmFnT<double> gemm_simt_double();
GemmFnT<float> gemm_tc();
GemmFnT<float> gemm_i8();  // int8 three-piece tensor-core back end, kernels_gemm_i8.cu
GemmFnT<float> gemm_dense_float();  // dense float E (PCAngsd), kernels_gl.cu

// PCAngsd device steps (kernels_gl.cu)
void gl_em_maf(pcaone_ctx* c, int maxiter, double tolmaf, int* iters);
// The loaded packed genotypes (current SNP order) -> likelihood mode: pseudo-likelihoods, the
// initial centred matrix E and F = the genotype allele frequencies (pcaone_gpu_bed_to_gl).
void gl_from_bed(pcaone_ctx* c);
// FP32 likelihoods on the host -> FP64 on the device, through a bounded staging buffer
void gl_widen_f32(pcaone_ctx* c, const float* P, size_t n, double* dP);
void gl_posterior(pcaone_ctx* c, const double* US, const double* V, int k);
// PCAngsd GRM (pcaone_gpu_gl_grm): C (host N x N, or null), its singular vectors (host N x N
// column-major, or null) and values (host N, or null); US, V as for gl_posterior.
void gl_grm(pcaone_ctx* c, const double* US, const double* V, int k, double* C, double* evecs, double* svals);
// Frees the context's cuSOLVER handle.
void gl_release(pcaone_ctx* c);

void omega_host(int seed, int rand, uint64_t nrow, uint32_t ncol, double* out);
void jacobi_svd(int n, const double* A, double* U, double* s, double* V);
void run_product(pcaone_ctx* c, int precision, int transpose, int standardize, int ploidy,
                 const double* B, int l, double* out);
void run_gram(pcaone_ctx* c, int precision, int standardize, int ploidy, const double* X, int l, double* Y);
void run_rsvd(pcaone_ctx* c, const pcaone_rsvd_opts& o, double* U, double* S, double* V,
              pcaone_rsvd_report* rep);

}  // namespace pg
