// FP64 sketch-width linear algebra launchers (kernels_linalg.cu). Tall matrices are
// row-major n x l.
#pragma once

#include "internal.hpp"

namespace pg {

// out (la x lb, row-major) = A^T B for A: n x la, B: n x lb.
void cross(pcaone_ctx* c, const double* A, int la, const double* B, int lb, int64_t n, double* out);
// W = R^T R; R upper. When Rprev is given, Racc = R * Rprev; when Rinv is given, R^-1 (upper,
// zeros below). d_status gets 1+j on failure.
void cholesky(pcaone_ctx* c, const double* W, int l, double* R, const double* Rprev, double* Racc,
              int* d_status, double* Rinv = nullptr);
// Q = A R^-1 (may alias A == Q).
void trsm_right_upper(pcaone_ctx* c, const double* A, const double* R, int l, int64_t n, double* Q);
// CholeskyQR2: A = Q R with Q orthonormal (Q may alias A).
void cholqr2(pcaone_ctx* c, const double* A, int l, int64_t n, double* Q, double* R, int* d_status);
// out (l x l) = (A Rinv)^T (A Rinv) for Rinv = R^-1 (upper), without writing A Rinv.
void cross_solved(pcaone_ctx* c, const double* A, const double* Rinv, int l, int64_t n, double* out);
// The R factor of CholeskyQR2 of A (A = Q R), without Q: Q = A R^-1 when needed.
void cholqr2_r(pcaone_ctx* c, const double* A, int l, int64_t n, double* R, int* d_status);
void colsum(pcaone_ctx* c, const double* A, int l, int64_t n, double* out);
// Y (n x kc) = X (n x l) * C[:, :kc] with C l x ldc row-major.
void rowmat(pcaone_ctx* c, const double* X, int l, const double* C, int ldc, int kc, int64_t n, double* Y);

// Forward substitution for one row: x R = a with R upper l x l staged by stage_r (row stride
// LMAX, so every R address is a constant offset; the diagonal slots hold 1 / R_jj, so the
// dependent chain has no division), x kept in registers (LMAX >= l; the loops unroll over LMAX
// and skip j >= l). Every element of a is read before out is written, so out may alias a.
template <int LMAX>
__device__ __forceinline__ void solve_row_upper(const double* a, const double* Rs, int l, double* out) {
  double x[LMAX];
#pragma unroll
  for (int j = 0; j < LMAX; ++j) {
    if (j < l) {
      double v = a[j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= x[k] * Rs[k * LMAX + j];
      x[j] = v * Rs[j * LMAX + j];
    } else {
      x[j] = 0.0;
    }
  }
#pragma unroll
  for (int j = 0; j < LMAX; ++j)
    if (j < l) out[j] = x[j];
}

// Copy R (l x l row-major, upper) into shared memory with row stride LMAX for
// solve_row_upper: the diagonal slots get 1 / R_jj.
template <int LMAX>
__device__ __forceinline__ void stage_r(const double* R, int l, double* Rs) {
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) {
    const int i = t / l, j = t - i * l;
    Rs[i * LMAX + j] = i == j ? 1.0 / R[t] : R[t];
  }
}

}  // namespace pg
