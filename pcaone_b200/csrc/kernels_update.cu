// Fused Omega update: Omega = flipOmg(Omega2, thin Q of H) in four launches.
//
// Reference: the Householder QR + householderQ() + flipOmg block of the winSVD window loop
// (src/Halko.cpp:213-216) and of the Halko epochs (src/Halko.cpp:118-122, src/RSVD.hpp:81-90).
//
//   K1  H = H1 + H2 (winSVD), W1 = H^T H                     last CTA: R1 = chol(W1)
//   K2  Q1 = H R1^-1, W2 = Q1^T Q1                          last CTA: R2 = chol(W2)
//   K3  Q = Q1 R2^-1, flip sums |O2 - Q|, |O2 + Q|          last CTA: signs D, multipliers m = +-D
//   K4  Omega = Q m, Omega2 = Omega, operand copies, column sums  last CTA: sum of Omega
//
// Each kernel runs as clusters of kGramCluster CTAs that own fixed row ranges. A CTA stages
// its rows in shared memory and sums them into a CTA partial (Gram matrices: 4 x 4 register
// tiles of the upper triangle, thread groups over rows, gram.hpp); the cluster adds its CTAs'
// partials through distributed shared memory, and the CTA that finishes last (atomic ticket
// after a __threadfence) adds the cluster sums in cluster order, so the result is
// deterministic. The Householder column signs D come from the modified LU of the top l x l
// block of Q (Ballard et al. 2015): pivot s -> D = -sign(s), sign(0) = +. Row solves keep the
// row in registers (kernels templated on LMAX >= l).
#include <cuda_bf16.h>

#include <algorithm>

#include "gram.hpp"
#include "internal.hpp"
#include "linalg.hpp"
#include "tc_layout.hpp"
#include "update.hpp"

namespace pg {

namespace {

constexpr int kThreads = 256;

// rows staged per batch: a batch of rows, the group sums and R fit in about 100 KB, so two
// CTAs (two clusters' worth per 8 SMs) fit on an SM
__host__ __device__ constexpr int stage_rows(int l) { return l <= 48 ? 128 : 64; }

// Column-strided pass over this CTA's rows: thread t owns column t % l of rows
// r0 + t / l, r0 + t / l + T / l, ... with T = l * (blockDim / l) threads.
__device__ __forceinline__ int col_threads(int l) { return l * (blockDim.x / l); }

// Shared memory of the Gram kernels: [LMAX x LMAX R] | group sums | CTA sum | staged rows
// (stage_rows(l) x l4, at least l x l).
__host__ __device__ inline int upd_gram_smem_doubles(int l, int rmax) {
  const GramTiling g = gram_tiling(l, l, true, kThreads);
  const int l4 = (l + 3) & ~3;
  return rmax * rmax + gram_smem_doubles(g) + std::max(stage_rows(l) * l4, l * l);
}

__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kThreads) k_upd1(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  const GramTiling g = gram_tiling(l, l, true, blockDim.x);
  double* red = sm;
  double* cpart = red + g.ngrp * g.ntiles * 16;
  double* stage = cpart + g.ntiles * 16;
  const int rows = stage_rows(l);
  GramThread gt;
  gt.init(g);
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    __syncthreads();
#pragma unroll 4
    for (int t = threadIdx.x; t < nr * g.la4; t += blockDim.x) {
      const int r = t / g.la4, cc = t - r * g.la4;
      double v = 0.0;
      if (cc < l) {
        const int64_t o = (b + r) * l + cc;
        if (a.H2) {
          v = a.H1[o] + a.H2[o];
          a.H[o] = v;
        } else {
          v = a.H[o];
        }
      }
      stage[t] = v;
    }
    __syncthreads();
    gt.add_rows(stage, stage, nr, g);
  }
  gt.finish(g, red, cpart);
  cluster_sum(cpart, g.ntiles * 16, a.part);
  if (!last_cta(&a.counters[0])) return;
  gram_final(g, a.part, gridDim.x / kGramCluster, l, l, stage);
  const int bad = chol_upper_smem(stage, l);
  if (bad && threadIdx.x == 0) atomicMax(a.status, bad);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R1[t] = stage[t];
  if (threadIdx.x == 0) a.counters[0] = 0;
}

template <int LMAX>
__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kThreads) k_upd2(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  const GramTiling g = gram_tiling(l, l, true, blockDim.x);
  double* R = sm;  // LMAX x LMAX (row stride LMAX)
  double* red = R + LMAX * LMAX;
  double* cpart = red + g.ngrp * g.ntiles * 16;
  double* stage = cpart + g.ntiles * 16;
  const int rows = stage_rows(l);
  stage_r<LMAX>(a.R1, l, R);
  {
    GramThread gt;
    gt.init(g);
    gt.park(g, red);  // the tiles live in red between batches (registers go to the row solves)
  }
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    __syncthreads();  // R staged; the previous batch's rows are consumed
    for (int r = threadIdx.x; r < nr; r += blockDim.x)
      solve_row_upper<LMAX>(a.H + (b + r) * l, R, l, stage + r * g.la4);
    __syncthreads();
#pragma unroll 4
    for (int t = threadIdx.x; t < nr * g.la4; t += blockDim.x) {
      const int r = t / g.la4, cc = t - r * g.la4;
      if (cc < l)
        a.Q[(b + r) * l + cc] = stage[t];
      else
        stage[t] = 0.0;
    }
    __syncthreads();
    GramThread gt;
    gt.init(g);
    gt.unpark(g, red);
    gt.add_rows(stage, stage, nr, g);
    gt.park(g, red);
  }
  __syncthreads();
  {
    const int n = g.ntiles * 16;  // CTA sum of the groups' tiles, fixed group order
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      double s = 0.0;
      for (int q = 0; q < g.ngrp; ++q) s += red[q * n + e];
      cpart[e] = s;
    }
    __syncthreads();
  }
  cluster_sum(cpart, g.ntiles * 16, a.part);
  if (!last_cta(&a.counters[1])) return;
  double* Rn = stage;  // W2, then R2 (row stride l)
  gram_final(g, a.part, gridDim.x / kGramCluster, l, l, Rn);
  const int bad = chol_upper_smem(Rn, l);
  if (bad && threadIdx.x == 0) atomicMax(a.status, bad);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R2[t] = Rn[t];
  if (threadIdx.x == 0) a.counters[1] = 0;
}

// K3. The flip sums are taken without the signs: A_c = sum |O2 - Q| and B_c = sum |O2 + Q|
// per column; with D_c = +1 they are |O2 - Q D| and |O2 + Q D|, with D_c = -1 swapped (the
// same values bit for bit). The last CTA reads the top l x l block of the final Q for D.
template <int LMAX>
__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kThreads) k_upd3(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  const int rows = stage_rows(l);
  double* R = sm;                      // LMAX x LMAX (row stride LMAX)
  double* sq = R + LMAX * LMAX;        // rows x l: Q
  double* so = sq + rows * l;          // rows x l: Omega2
  double* red = so + rows * l;         // kThreads x 2
  double* cpart = red + kThreads * 2;  // 2 l
  stage_r<LMAX>(a.R2, l, R);
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  const int T = col_threads(l);
  const int c = threadIdx.x % l;
  double sa = 0.0, sb = 0.0;
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    __syncthreads();  // R staged; the previous batch is consumed
    for (int r = threadIdx.x; r < nr; r += blockDim.x) solve_row_upper<LMAX>(a.Q + (b + r) * l, R, l, sq + r * l);
#pragma unroll 4
    for (int t = threadIdx.x; t < nr * l; t += blockDim.x) so[t] = a.Omg2[b * l + t];
    __syncthreads();
#pragma unroll 4
    for (int t = threadIdx.x; t < nr * l; t += blockDim.x) a.Q[b * l + t] = sq[t];
    if (threadIdx.x < T) {
      for (int r = threadIdx.x / l; r < nr; r += T / l) {
        const double o = so[r * l + c], q = sq[r * l + c];
        sa += fabs(o - q);
        sb += fabs(o + q);
      }
    }
  }
  red[threadIdx.x * 2] = sa;
  red[threadIdx.x * 2 + 1] = sb;
  __syncthreads();
  for (int j = threadIdx.x; j < l; j += blockDim.x) {  // fixed-order sum over this column's threads
    double m = 0.0, p = 0.0;
    for (int t = j; t < T; t += l) {
      m += red[t * 2];
      p += red[t * 2 + 1];
    }
    cpart[j] = m;
    cpart[l + j] = p;
  }
  cluster_sum(cpart, 2 * l, a.part);
  if (!last_cta(&a.counters[2])) return;
  double* top = R;  // the top l x l block of Q, written by this kernel's CTAs
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) top[t] = a.Q[t];
  householder_signs_smem(top, l, a.D);
  const int ncl = gridDim.x / kGramCluster;
  for (int j = threadIdx.x; j < l; j += blockDim.x) {
    const double A = sum_all<kGramMaxParts>(a.part + j, ncl, 2 * l);
    const double B = sum_all<kGramMaxParts>(a.part + l + j, ncl, 2 * l);
    const double d = a.D[j];
    const double m = d > 0.0 ? A : B, p = d > 0.0 ? B : A;
    a.mult[j] = (m > 2.0 * p) ? -d : d;  // src/RSVD.hpp:85
  }
  if (threadIdx.x == 0) a.counters[2] = 0;
}

// K4. Writes in row-major order (coalesced), column sums from the staged batch.
__global__ void __cluster_dims__(kGramCluster, 1, 1) __launch_bounds__(kThreads) k_upd4(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  const int rows = stage_rows(l);
  double* red = sm;                // kThreads
  double* cpart = red + kThreads;  // l
  double* st = cpart + l;          // rows x l
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  const int T = col_threads(l);
  double cs = 0.0;
  for (int64_t b = r0; b < r1; b += rows) {
    const int nr = (int)(r1 - b < rows ? r1 - b : rows);
    __syncthreads();  // the previous batch is summed
#pragma unroll 4
    for (int t = threadIdx.x; t < nr * l; t += blockDim.x) {
      const int rr = t / l, j = t - rr * l;
      const int64_t r = b + rr, o = b * l + t;
      const double v = a.Q[o] * a.mult[j];
      a.Omg[o] = v;
      a.Omg2[o] = v;
      st[t] = v;
      if (a.Omgf) a.Omgf[o] = (float)v;
      if (a.bt1) {
        const int64_t kp = tc_pos(r);
        const float x = (float)v;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        a.bt1[bt_elem(j, kp, 2 * a.bt_half)] = hi;
        a.bt1[bt_elem(a.bt_half + j, kp, 2 * a.bt_half)] = __float2bfloat16_rn(x - __bfloat162float(hi));
      }
    }
    __syncthreads();
    if (threadIdx.x < T)
      for (int rr = threadIdx.x / l; rr < nr; rr += T / l) cs += st[rr * l + threadIdx.x % l];
  }
  red[threadIdx.x] = cs;
  __syncthreads();
  for (int j = threadIdx.x; j < l; j += blockDim.x) {
    double s = 0.0;
    for (int t = j; t < T; t += l) s += red[t];
    cpart[j] = s;
  }
  cluster_sum(cpart, l, a.part);
  if (!last_cta(&a.counters[3])) return;
  const int ncl = gridDim.x / kGramCluster;
  for (int j = threadIdx.x; j < l; j += blockDim.x) a.wsum[j] = sum_all<kGramMaxParts>(a.part + j, ncl, l);
  if (threadIdx.x == 0) a.counters[3] = 0;
}

// CTAs of the update kernels: whole clusters, about 64 rows or more per CTA, at most
// kMaxClusters clusters (two CTAs an SM; the last CTA reads one partial per cluster).
constexpr int kMaxClusters = kGramMaxParts;

int update_ctas(pcaone_ctx* c, int64_t N, int resident) {
  const int64_t want = (N + kGramCluster * 64 - 1) / (kGramCluster * 64);
  int cap = std::max(1, std::min(kMaxClusters, 2 * c->sm_count / kGramCluster));
  if (resident > 0) cap = std::min(cap, resident);
  return (int)std::max<int64_t>(1, std::min<int64_t>(cap, want)) * kGramCluster;
}

template <int LMAX>
void launch_all(pcaone_ctx* c, const UpdateArgs& a) {
  const int l = a.l, rows = stage_rows(l);
  const size_t s1 = (size_t)upd_gram_smem_doubles(l, 0) * 8;
  const size_t s2 = (size_t)upd_gram_smem_doubles(l, LMAX) * 8;
  const size_t s3 = ((size_t)LMAX * LMAX + 2 * (size_t)rows * l + 2 * kThreads + 2 * l) * 8;
  const size_t s4 = ((size_t)kThreads + l + (size_t)rows * l) * 8;
  PG_CUDA(cudaFuncSetAttribute(k_upd1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
  PG_CUDA(cudaFuncSetAttribute(k_upd2<LMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2));
  PG_CUDA(cudaFuncSetAttribute(k_upd3<LMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s3));
  // every cluster of every kernel resident at once: the tightest of the four bounds
  int resident = 0;
  const void* ks[4] = {(const void*)k_upd1, (const void*)k_upd2<LMAX>, (const void*)k_upd3<LMAX>, (const void*)k_upd4};
  const size_t ss[4] = {s1, s2, s3, s4};
  for (int i = 0; i < 4; ++i) {
    const int n = resident_clusters(c, ks[i], (uint64_t)l, kThreads, ss[i]);
    if (n > 0) resident = resident > 0 ? std::min(resident, n) : n;
  }
  const int nblk = update_ctas(c, a.N, resident);
  k_upd1<<<nblk, kThreads, s1, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd2<LMAX><<<nblk, kThreads, s2, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd3<LMAX><<<nblk, kThreads, s3, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd4<<<nblk, kThreads, s4, c->stream>>>(a);
  PG_CHECK_LAUNCH();
}

}  // namespace

size_t update_part_doubles(int l) {
  const GramTiling g = gram_tiling(l, l, true, kThreads);
  return (size_t)kMaxClusters * std::max(g.ntiles * 16, 2 * l);
}

void fused_update(pcaone_ctx* c, UpdateArgs a) {
  PG_REQUIRE(a.l >= 1 && a.l <= kLmax, PCAONE_EBADARG, "sketch width out of range");
  if (a.l <= 16)
    launch_all<16>(c, a);
  else if (a.l <= 32)
    launch_all<32>(c, a);
  else if (a.l <= 48)
    launch_all<48>(c, a);
  else
    launch_all<64>(c, a);
  c->launches += 4;
}

}  // namespace pg
