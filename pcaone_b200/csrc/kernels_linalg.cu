// FP64 kernels for the (k+p)-wide sketch outside the fused Omega update: Gram matrices,
// Cholesky and triangular solves (CholeskyQR2 of the epoch tail), column sums and small
// products.
//
// Tall matrices are row-major n x l (one sample or SNP per row, l <= kLmax columns).
// All reductions run in a fixed order (per-CTA or per-cluster partials, then a fixed-order
// sum), so results are deterministic run to run.
#include "gram.hpp"
#include "internal.hpp"
#include "linalg.hpp"

namespace pg {

namespace {

// A^T B over rows: each CTA of a cluster streams its contiguous row block through two
// shared-memory stages (cp.async, the next batch in flight while the current one is summed
// into 4 x 4 register tiles, gram.hpp), sums its thread groups, and the cluster adds its CTAs'
// sums through distributed shared memory into gpart[cluster] (ntiles * 16 values in tile
// layout). SYM (A == B): only the tiles on and above the diagonal, one staged copy.
constexpr int kCrossThreads = 256;
constexpr int kCrossMaxClusters = kGramMaxParts;
constexpr int kCrossSmemBudget = 96 * 1024;  // two CTAs an SM

__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}

template <bool SYM>
__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kCrossThreads)
    k_cross(const double* __restrict__ A, int la, const double* __restrict__ Bm, int lb, int64_t n, int rows,
            double* __restrict__ gpart) {
  extern __shared__ double sm[];
  const GramTiling g = gram_tiling(la, lb, SYM, blockDim.x);
  const int w = g.la4 + (SYM ? 0 : g.lb4);  // staged doubles per row: A rows (la4), then B rows (lb4)
  double* red = sm + 2 * rows * w;  // stages: sm and sm + rows * w
  double* cpart = red + g.ngrp * g.ntiles * 16;
  for (int t = threadIdx.x; t < 2 * rows; t += blockDim.x) {  // zero padding columns, never copied
    double* base = sm + (t / rows) * rows * w;
    const int r = t % rows;
    for (int cc = la; cc < g.la4; ++cc) base[r * g.la4 + cc] = 0.0;
    if (!SYM)
      for (int cc = lb; cc < g.lb4; ++cc) base[rows * g.la4 + r * g.lb4 + cc] = 0.0;
  }
  int64_t r0, r1;
  row_range(n, r0, r1);
  auto issue = [&](int64_t b, double* dst) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    for (int t = threadIdx.x; t < nr * la; t += blockDim.x) {
      const int r = t / la;
      cp_async8(dst + r * g.la4 + (t - r * la), A + b * la + t);
    }
    if (!SYM)
      for (int t = threadIdx.x; t < nr * lb; t += blockDim.x) {
        const int r = t / lb;
        cp_async8(dst + rows * g.la4 + r * g.lb4 + (t - r * lb), Bm + b * lb + t);
      }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  GramThread gt;
  gt.init(g);
  int s = 0;
  if (r0 < r1) issue(r0, sm);
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    if (b + rows < r1) {
      issue(b + rows, sm + (s ^ 1) * rows * w);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();  // stage s complete (and the padding zeroed) for every thread
    const double* sa = sm + s * rows * w;
    gt.add_rows(sa, SYM ? sa : sa + rows * g.la4, nr, g);
    __syncthreads();  // stage s is consumed before it is refilled
    s ^= 1;
  }
  gt.finish(g, red, cpart);
  cluster_sum(cpart, g.ntiles * 16, gpart);
}

// Gram of Q1 = A R^{-1} without writing Q1 (the second pass of CholeskyQR2 when only its R
// is needed): k_cross<true> with a product step. Each staged batch of rows (row stride
// la4 + 2, 16-byte aligned) is multiplied by Rinv = R^{-1} (upper, staged in shared memory
// with row stride LMAX and zeros outside l x l) in 4 x 4 register tiles, a thread per tile
// (the host sizes the batch so that one pass of the CTA covers it), written back in place
// and then summed into the Gram tiles.
template <int LMAX>
__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kCrossThreads)
    k_cross_solved(const double* __restrict__ A, const double* __restrict__ Rinv, int l, int64_t n, int rows,
                   double* __restrict__ gpart) {
  extern __shared__ double sm[];
  const GramTiling g = gram_tiling(l, l, true, blockDim.x);
  GramTiling gs = g;  // the tile reads with the staged row stride
  gs.la4 = gs.lb4 = g.la4 + 2;
  const int w = gs.la4;
  double* Rs = sm;  // LMAX x LMAX
  double* st = Rs + LMAX * LMAX;
  double* red = st + 2 * rows * w;
  double* cpart = red + g.ngrp * g.ntiles * 16;
  for (int t = threadIdx.x; t < LMAX * LMAX; t += blockDim.x) {
    const int i = t / LMAX, j = t - i * LMAX;
    Rs[t] = (i < l && j < l) ? Rinv[i * l + j] : 0.0;
  }
  for (int t = threadIdx.x; t < 2 * rows; t += blockDim.x)  // padding columns, never copied or written
    for (int cc = l; cc < w; ++cc) st[t * w + cc] = 0.0;
  int64_t r0, r1;
  row_range(n, r0, r1);
  auto issue = [&](int64_t b, double* dst) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    for (int t = threadIdx.x; t < nr * l; t += blockDim.x) {
      const int r = t / l;
      cp_async8(dst + r * w + (t - r * l), A + b * l + t);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  GramThread gt;
  gt.init(g);
  int s = 0;
  if (r0 < r1) issue(r0, st);
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    if (b + rows < r1) {
      issue(b + rows, st + (s ^ 1) * rows * w);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();  // stage s complete, R staged, padding zeroed
    double* sa = st + s * rows * w;
    {
      const int nbc = g.la4 >> 2, nbr = (nr + 3) >> 2;
      const bool act = (int)threadIdx.x < nbr * nbc;
      const int rb = act ? (int)threadIdx.x / nbc : 0, cb = act ? (int)threadIdx.x - rb * nbc : 0;
      const int rr0 = 4 * rb, cc0 = 4 * cb;
      double q[4][4];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) q[x][y] = 0.0;
      if (act) {
        const int kend = l < cc0 + 4 ? l : cc0 + 4;  // Rinv is upper: rows past the tile's last column add 0
        for (int kk = 0; kk < kend; ++kk) {
          const double2 r01 = *reinterpret_cast<const double2*>(Rs + kk * LMAX + cc0);
          const double2 r23 = *reinterpret_cast<const double2*>(Rs + kk * LMAX + cc0 + 2);
          const double rv[4] = {r01.x, r01.y, r23.x, r23.y};
          double av[4];
#pragma unroll
          for (int x = 0; x < 4; ++x) av[x] = rr0 + x < nr ? sa[(rr0 + x) * w + kk] : 0.0;
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) q[x][y] = fma(av[x], rv[y], q[x][y]);
        }
      }
      __syncthreads();  // every row of the batch read before any is overwritten
      if (act)
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y)
            if (rr0 + x < nr && cc0 + y < l) sa[(rr0 + x) * w + cc0 + y] = q[x][y];
    }
    __syncthreads();
    gt.add_rows(sa, sa, nr, gs);
    __syncthreads();  // stage s is consumed before it is refilled
    s ^= 1;
  }
  gt.finish(g, red, cpart);
  cluster_sum(cpart, g.ntiles * 16, gpart);
}

// out (la x lb, global) = sum of the nparts cluster sums of k_cross.
__global__ void __launch_bounds__(kCrossThreads) k_cross_final(const double* __restrict__ gpart, int nparts, int la,
                                                               int lb, int sym, double* __restrict__ out) {
  const GramTiling g = gram_tiling(la, lb, sym != 0, kCrossThreads);
  gram_final(g, gpart, nparts, la, lb, out);
}

__global__ void k_cholesky(const double* __restrict__ W, int l, double* __restrict__ R,
                           const double* __restrict__ Rprev, double* __restrict__ Racc,
                           double* __restrict__ Rinv, int* __restrict__ status) {
  extern __shared__ double s[];  // l x l, then l x l for R^-1
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) s[t] = W[t];
  const int bad = chol_upper_smem(s, l);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) R[t] = s[t];
  if (Rinv) {  // column j of R^-1 by back substitution (thread j), zeros below the diagonal
    double* si = s + l * l;
    for (int j = threadIdx.x; j < l; j += blockDim.x) {
      for (int i = l - 1; i > j; --i) si[i * l + j] = 0.0;
      si[j * l + j] = 1.0 / s[j * l + j];
      for (int i = j - 1; i >= 0; --i) {
        double acc = 0.0;
        for (int m = i + 1; m <= j; ++m) acc = fma(s[i * l + m], si[m * l + j], acc);
        si[i * l + j] = -acc / s[i * l + i];
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < l * l; t += blockDim.x) Rinv[t] = si[t];
  }
  __syncthreads();
  if (Rprev) {
    for (int t = threadIdx.x; t < l * l; t += blockDim.x) {
      int i = t / l, j = t % l;
      double acc = 0.0;
      for (int k = i; k <= j; ++k) acc += R[i * l + k] * Rprev[k * l + j];
      Racc[t] = (j >= i) ? acc : 0.0;
    }
  }
  if (threadIdx.x == 0 && bad && status) atomicMax(status, bad);
}

// Q = A R^{-1} (row-wise forward substitution x R = a), R upper l x l. One thread per row;
// the row's unknowns stay in registers (LMAX >= l, loops unrolled over LMAX).
template <int LMAX>
__global__ void __launch_bounds__(128) k_trsm_right_upper(const double* A, const double* __restrict__ R, int l,
                                                          int64_t n, double* Q) {  // A may alias Q
  extern __shared__ double sr[];  // LMAX x LMAX
  stage_r<LMAX>(R, l, sr);
  __syncthreads();
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  solve_row_upper<LMAX>(A + r * l, sr, l, Q + r * l);
}

// Column sums of A (n x l) into partials (grid.y = column).
__global__ void k_colsum_partial(const double* __restrict__ A, int l, int64_t n,
                                 double* __restrict__ part) {
  __shared__ double sm[256];
  const int col = blockIdx.y;
  double s = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x)
    s += A[r * l + col];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st; st >>= 1) {
    if (threadIdx.x < st) sm[threadIdx.x] += sm[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(int64_t)col * gridDim.x + blockIdx.x] = sm[0];
}

__global__ void k_colsum_final(const double* __restrict__ part, int nblk, int l,
                               double* __restrict__ out) {
  int col = threadIdx.x;
  if (col >= l) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(int64_t)col * nblk + b];
  out[col] = s;
}

// Y (n x kc) = X (n x l) * C (l x ldc, first kc columns), row-major; X row in registers.
template <int LMAX>
__global__ void __launch_bounds__(128) k_rowmat(const double* __restrict__ X, int l, const double* __restrict__ C,
                                                int ldc, int kc, int64_t n, double* __restrict__ Y) {
  extern __shared__ double sc[];
  for (int t = threadIdx.x; t < l * kc; t += blockDim.x) sc[t] = C[(t / kc) * ldc + t % kc];
  __syncthreads();
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double* x = X + r * l;
  double xr[LMAX];
#pragma unroll
  for (int j = 0; j < LMAX; ++j) xr[j] = j < l ? x[j] : 0.0;
  for (int c = 0; c < kc; ++c) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < LMAX; ++j)
      if (j < l) s = fma(xr[j], sc[j * kc + c], s);
    Y[r * kc + c] = s;
  }
}

}  // namespace

void cross(pcaone_ctx* c, const double* A, int la, const double* B, int lb, int64_t n, double* out) {
  PG_REQUIRE(la >= 1 && lb >= 1 && la <= kLmax && lb <= kLmax, PCAONE_EBADARG, "cross product too wide");
  const bool sym = A == B && la == lb;
  const GramTiling g = gram_tiling(la, lb, sym, kCrossThreads);
  const int w = g.la4 + (sym ? 0 : g.lb4);
  const int fixed = gram_smem_doubles(g) * 8;
  const int rows = std::max(8, std::min(128, (kCrossSmemBudget - fixed) / (2 * w * 8)));
  const size_t smem = (size_t)fixed + (size_t)2 * rows * w * 8;
  const int64_t want = (n + (int64_t)kGramCluster * 4 * rows - 1) / ((int64_t)kGramCluster * 4 * rows);
  int cap = std::max(1, std::min(kCrossMaxClusters, 2 * c->sm_count / kGramCluster));
  const void* kern = sym ? (const void*)k_cross<true> : (const void*)k_cross<false>;
  PG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int resident = resident_clusters(c, kern, ((uint64_t)la << 32) | (uint64_t)lb, kCrossThreads, smem);
  if (resident > 0) cap = std::min(cap, resident);
  const int ncl = (int)std::max<int64_t>(1, std::min<int64_t>(cap, want));
  double* gpart = (double*)scratch(c, "cross_part", (size_t)ncl * g.ntiles * 16 * 8);
  if (sym) {
    k_cross<true><<<ncl * kGramCluster, kCrossThreads, smem, c->stream>>>(A, la, A, lb, n, rows, gpart);
  } else {
    k_cross<false><<<ncl * kGramCluster, kCrossThreads, smem, c->stream>>>(A, la, B, lb, n, rows, gpart);
  }
  PG_CHECK_LAUNCH();
  k_cross_final<<<1, kCrossThreads, 0, c->stream>>>(gpart, ncl, la, lb, sym ? 1 : 0, out);
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

void cross_solved(pcaone_ctx* c, const double* A, const double* Rinv, int l, int64_t n, double* out) {
  PG_REQUIRE(l >= 1 && l <= kLmax, PCAONE_EBADARG, "cross product too wide");
  const GramTiling g = gram_tiling(l, l, true, kCrossThreads);
  const int lmax = l <= 16 ? 16 : l <= 32 ? 32 : l <= 48 ? 48 : 64;
  const int w = g.la4 + 2;
  const int fixed = (gram_smem_doubles(g) + lmax * lmax) * 8;
  // one 4 x 4 product tile per thread covers a batch of rows
  const int rows_tiles = 4 * (kCrossThreads / (g.la4 / 4));
  const int rows = std::max(4, std::min(std::min(128, rows_tiles), (kCrossSmemBudget - fixed) / (2 * w * 8)));
  const size_t smem = (size_t)fixed + (size_t)2 * rows * w * 8;
  const int64_t want = (n + (int64_t)kGramCluster * 4 * rows - 1) / ((int64_t)kGramCluster * 4 * rows);
  int cap = std::max(1, std::min(kCrossMaxClusters, 2 * c->sm_count / kGramCluster));
  auto go = [&](auto kern) {
    PG_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int resident = resident_clusters(c, (const void*)kern, ((uint64_t)l << 32) | 0x5u, kCrossThreads, smem);
    if (resident > 0) cap = std::min(cap, resident);
    const int ncl = (int)std::max<int64_t>(1, std::min<int64_t>(cap, want));
    double* gpart = (double*)scratch(c, "cross_part", (size_t)ncl * g.ntiles * 16 * 8);
    kern<<<ncl * kGramCluster, kCrossThreads, smem, c->stream>>>(A, Rinv, l, n, rows, gpart);
    PG_CHECK_LAUNCH();
    k_cross_final<<<1, kCrossThreads, 0, c->stream>>>(gpart, ncl, l, l, 1, out);
    PG_CHECK_LAUNCH();
  };
  if (lmax == 16)
    go(k_cross_solved<16>);
  else if (lmax == 32)
    go(k_cross_solved<32>);
  else if (lmax == 48)
    go(k_cross_solved<48>);
  else
    go(k_cross_solved<64>);
  c->launches += 2;
}

void cholqr2_r(pcaone_ctx* c, const double* A, int l, int64_t n, double* R, int* d_status) {
  double* W = (double*)scratch(c, "cq_W", (size_t)l * l * 8);
  double* R1 = (double*)scratch(c, "cq_R1", (size_t)l * l * 8);
  double* R2 = (double*)scratch(c, "cq_R2", (size_t)l * l * 8);
  double* R1i = (double*)scratch(c, "cq_R1i", (size_t)l * l * 8);
  cross(c, A, l, A, l, n, W);
  cholesky(c, W, l, R1, nullptr, nullptr, d_status, R1i);
  cross_solved(c, A, R1i, l, n, W);
  cholesky(c, W, l, R2, R1, R, d_status);
}

void cholesky(pcaone_ctx* c, const double* W, int l, double* R, const double* Rprev, double* Racc,
              int* d_status, double* Rinv) {
  k_cholesky<<<1, 256, (size_t)(Rinv ? 2 : 1) * l * l * 8, c->stream>>>(W, l, R, Rprev, Racc, Rinv, d_status);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void trsm_right_upper(pcaone_ctx* c, const double* A, const double* R, int l, int64_t n, double* Q) {
  const dim3 grid((unsigned)((n + 127) / 128));
  if (l <= 16)
    k_trsm_right_upper<16><<<grid, 128, 16 * 16 * 8, c->stream>>>(A, R, l, n, Q);
  else if (l <= 32)
    k_trsm_right_upper<32><<<grid, 128, 32 * 32 * 8, c->stream>>>(A, R, l, n, Q);
  else if (l <= 48)
    k_trsm_right_upper<48><<<grid, 128, 48 * 48 * 8, c->stream>>>(A, R, l, n, Q);
  else
    k_trsm_right_upper<64><<<grid, 128, 64 * 64 * 8, c->stream>>>(A, R, l, n, Q);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void cholqr2(pcaone_ctx* c, const double* A, int l, int64_t n, double* Q, double* R, int* d_status) {
  double* W = (double*)scratch(c, "cq_W", (size_t)l * l * 8);
  double* R1 = (double*)scratch(c, "cq_R1", (size_t)l * l * 8);
  double* R2 = (double*)scratch(c, "cq_R2", (size_t)l * l * 8);
  cross(c, A, l, A, l, n, W);
  cholesky(c, W, l, R1, nullptr, nullptr, d_status);
  trsm_right_upper(c, A, R1, l, n, Q);
  cross(c, Q, l, Q, l, n, W);
  cholesky(c, W, l, R2, R1, R, d_status);
  trsm_right_upper(c, Q, R2, l, n, Q);
}

void colsum(pcaone_ctx* c, const double* A, int l, int64_t n, double* out) {
  const int nblk = 64;
  double* part = (double*)scratch(c, "colsum_part", (size_t)l * nblk * 8);
  k_colsum_partial<<<dim3(nblk, l), 256, 0, c->stream>>>(A, l, n, part);
  PG_CHECK_LAUNCH();
  k_colsum_final<<<1, 128, 0, c->stream>>>(part, nblk, l, out);
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

void rowmat(pcaone_ctx* c, const double* X, int l, const double* C, int ldc, int kc, int64_t n, double* Y) {
  const dim3 grid((unsigned)((n + 127) / 128));
  const size_t smem = (size_t)l * kc * 8;
  if (l <= 16)
    k_rowmat<16><<<grid, 128, smem, c->stream>>>(X, l, C, ldc, kc, n, Y);
  else if (l <= 32)
    k_rowmat<32><<<grid, 128, smem, c->stream>>>(X, l, C, ldc, kc, n, Y);
  else if (l <= 48)
    k_rowmat<48><<<grid, 128, smem, c->stream>>>(X, l, C, ldc, kc, n, Y);
  else
    k_rowmat<64><<<grid, 128, smem, c->stream>>>(X, l, C, ldc, kc, n, Y);
  PG_CHECK_LAUNCH();
  c->launches++;
}

}  // namespace pg
