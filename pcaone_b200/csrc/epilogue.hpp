// Parameters and launchers of the decode-GEMM epilogues (kernels_epilogue.cu).
#pragma once

#include <cuda_bf16.h>

#include "internal.hpp"

namespace pg {

struct EpiP1 {          // after the Z^T Omega product of one window
  int64_t start = 0;    // first SNP of the window, or of a run of windows (current SNP order)
  int64_t m = 0;        // SNPs in the window (run)
  // Padded layout of a run of windows: SNP jl of the run lies in window w = jl / wlen at
  // row w * d1_ws + jl % wlen of D1 (d1_rows rows per split) and row w * b2_ws + jl % wlen of
  // B2. 0 = one window: wlen = d1_ws = b2_ws = d1_rows = m.
  int64_t wlen = 0, d1_ws = 0, b2_ws = 0, d1_rows = 0;
  int l = 0, ksplit = 1;
  const double* F = nullptr;         // M, centring frequencies
  const double* scale = nullptr;     // M, per-SNP scale s_j
  const double* wsum = nullptr;      // l: column sums of Omega
  const double* omega = nullptr;     // Npad x l
  const float* omega_f = nullptr;    // FP32 copy of omega: when set, the sparse gather reads it
  const int64_t* miss_ptr = nullptr; // by-SNP CSR
  const int32_t* miss_idx = nullptr;
  const double* miss_val = nullptr;  // e_ij per entry (EM-imputed), or null for 0
  double* G = nullptr;               // M x l (rows start..start+m written)
  float* Gf = nullptr;               // when set: FP32 rows of the window (run) for the second
                                     // gather: G, or s F G when miss_val is null (window-local)
  unsigned long long* qmax = nullptr;  // when set: atomicMax of |B2| per column (double bits)
  __nv_bfloat16* bt2 = nullptr;      // when set: B2 written as split BF16 (tc_layout.hpp)
  int64_t kpad2 = 0;                 // K extent of bt2 (multiple of 64)
  int bt_half = 0;                   // row offset of the lo half in bt2 (= NP / 2)
};

struct EpiP2 {          // after the Z * G product of one window or of a run of windows
  int b0 = 0, b1 = 1;   // windows [b0, b1)
  int nwin = 1;         // windows of the layout (the (window, sample) list has nwin rows per sample)
  int64_t n = 0, npad = 0;
  int l = 0, ksplit = 1;
  const double* F = nullptr;
  const double* scale = nullptr;
  const double* G = nullptr;         // M x l
  const float* Gf = nullptr;         // when set: window-local FP32 rows (see EpiP1::Gf) read by the gather
  int64_t g_start = 0;               // first SNP of window b0 (row 0 of Gf)
  const double* h0 = nullptr;        // l
  const int64_t* miss_ptr = nullptr; // (window, sample) CSR, row i * nwin + b
  const int32_t* miss_idx = nullptr;
  const double* miss_val = nullptr;
  const double* miss_w = nullptr;    // when set: per-entry weights s_j (e_ij + F_j) (replaces the
                                     // per-entry gathers of s and F)
  double* H = nullptr;               // Npad x l accumulator
};

template <typename T>
void launch_prep(pcaone_ctx* c, const EpiP1& p, const T* D1, T* B2, double* h0);
// B2 = s/2 G and h0 = sum s F G for the rows [start, start+m) of p.G (no product).
template <typename T>
void launch_scale_g(pcaone_ctx* c, const EpiP1& p, T* B2, double* h0);
template <typename T>
void launch_accum(pcaone_ctx* c, const EpiP2& p, const T* D2);
void zero(pcaone_ctx* c, double* a, int64_t n);

}  // namespace pg
