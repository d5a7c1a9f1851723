// Fused Omega update: Omega = flipOmg(Omega2, thin Q of H) in four launches.
//
// Reference: the Householder QR + householderQ() + flipOmg block of the winSVD window loop
// (src/Halko.cpp:213-216) and of the Halko epochs (src/Halko.cpp:118-122, src/RSVD.hpp:81-90).
//
//   K1  H = H1 + H2 (winSVD), W1 = H^T H                     last CTA: R1 = chol(W1)
//   K2  Q1 = H R1^-1, W2 = Q1^T Q1                          last CTA: R2 = chol(W2), signs D
//   K3  Q = Q1 R2^-1, flip sums |O2 - Q D|, |O2 + Q D|      last CTA: multipliers m = +-D
//   K4  Omega = Q m, Omega2 = Omega, operand copies, column sums  last CTA: sum of Omega
//
// Each kernel's CTAs own fixed row ranges and write per-CTA partial sums; the CTA that
// finishes last (atomic ticket after a __threadfence) reduces the partials in CTA order, so
// the result is deterministic. The Householder column signs D come from the modified LU of
// the top l x l block of Q (Ballard et al. 2015): pivot s -> D = -sign(s), sign(0) = +.
// Row solves keep the row in registers (kernels templated on LMAX >= l); Gram matrices use
// 4 x 4 register tiles; column sums use a column-strided thread layout.
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.hpp"
#include "linalg.hpp"
#include "tc_layout.hpp"
#include "update.hpp"

namespace pg {

namespace {

constexpr int kThreads = 256;
constexpr int kStageRows = 32;

// Shared-memory Cholesky of an l x l SPD matrix (upper R, W = R^T R), in place in s.
__device__ void chol_smem(double* s, int l, int* status) {
  for (int j = 0; j < l; ++j) {
    if (threadIdx.x == 0) {
      double d = s[j * l + j];
      if (!(d > 0.0) || !isfinite(d)) {
        atomicMax(status, j + 1);
        d = 1.0;
      }
      s[j * l + j] = sqrt(d);
    }
    __syncthreads();
    const double djj = s[j * l + j];
    for (int i = j + 1 + threadIdx.x; i < l; i += blockDim.x) s[j * l + i] /= djj;
    __syncthreads();
    const int w = l - j - 1;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int a = j + 1 + t / w, b = j + 1 + t % w;
      if (b >= a) s[a * l + b] -= s[j * l + a] * s[j * l + b];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < l * l; t += blockDim.x)
    if (t % l < t / l) s[t] = 0.0;
  __syncthreads();
}

// This CTA's rows [r0, r1) of A^T A (A: n x l row-major) added into a 4 x 4 register tile per
// thread; stage holds kStageRows x l4 doubles. Threads past the (l4/4)^2 tiles only stage.
__device__ void gram_rows(const double* A, int l, int64_t r0, int64_t r1, double* stage, double (&acc)[4][4]) {
  const int l4 = (l + 3) & ~3, nb = l4 / 4;
  const bool active = threadIdx.x < nb * nb;
  const int i0 = active ? (threadIdx.x / nb) * 4 : 0, j0 = active ? (threadIdx.x % nb) * 4 : 0;
  for (int64_t b = r0; b < r1; b += kStageRows) {
    const int nr = (int)(r1 - b < kStageRows ? r1 - b : kStageRows);
    __syncthreads();
    for (int t = threadIdx.x; t < nr * l4; t += blockDim.x) {
      const int r = t / l4, c = t - r * l4;
      stage[t] = c < l ? A[(b + r) * l + c] : 0.0;
    }
    __syncthreads();
    if (active) {
      for (int r = 0; r < nr; ++r) {
        const double2 a01 = *reinterpret_cast<const double2*>(stage + r * l4 + i0);
        const double2 a23 = *reinterpret_cast<const double2*>(stage + r * l4 + i0 + 2);
        const double2 b01 = *reinterpret_cast<const double2*>(stage + r * l4 + j0);
        const double2 b23 = *reinterpret_cast<const double2*>(stage + r * l4 + j0 + 2);
        const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) acc[x][y] = fma(av[x], bv[y], acc[x][y]);
      }
    }
  }
}

__device__ void store_gram_part(const double (&acc)[4][4], int l, double* part) {
  const int l4 = (l + 3) & ~3, nb = l4 / 4;
  if (threadIdx.x >= nb * nb) return;
  const int i0 = (threadIdx.x / nb) * 4, j0 = (threadIdx.x % nb) * 4;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y)
      if (i0 + x < l && j0 + y < l) part[(int64_t)blockIdx.x * l * l + (i0 + x) * l + j0 + y] = acc[x][y];
}

__device__ bool last_cta(unsigned* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// sum_{b < n} x[b * stride], added in b order (the same result as the plain loop); the loads
// of eight terms are issued before their adds, so they overlap instead of paying one L2
// round trip per term.
__device__ __forceinline__ double sum_strided(const double* x, int n, int64_t stride) {
  double s = 0.0;
  int b = 0;
  for (; b + 8 <= n; b += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = x[(int64_t)(b + k) * stride];
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
  }
  for (; b < n; ++b) s += x[(int64_t)b * stride];
  return s;
}

__device__ void reduce_pairs(const double* part, int nblk, int npairs, double* out_smem) {
  for (int p = threadIdx.x; p < npairs; p += blockDim.x) out_smem[p] = sum_strided(part + p, nblk, npairs);
  __syncthreads();
}

__device__ __forceinline__ void row_range(int64_t N, int64_t& r0, int64_t& r1) {
  const int64_t rpb = (N + gridDim.x - 1) / gridDim.x;
  r0 = blockIdx.x * rpb;
  r1 = (N < r0 + rpb ? N : r0 + rpb);
  if (r0 > r1) r0 = r1;
}

// Column-strided pass over this CTA's rows: thread t owns column t % l of rows
// r0 + t / l, r0 + t / l + T / l, ... with T = l * (blockDim / l) threads.
__device__ __forceinline__ int col_threads(int l) { return l * (blockDim.x / l); }

__global__ void __launch_bounds__(kThreads) k_upd1(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* stage = sm;  // max(kStageRows, l) x l4
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  if (a.H2) {
    for (int64_t t = r0 * l + threadIdx.x; t < r1 * l; t += blockDim.x) a.H[t] = a.H1[t] + a.H2[t];
    __syncthreads();
  }
  double acc[4][4] = {};
  gram_rows(a.H, l, r0, r1, stage, acc);
  store_gram_part(acc, l, a.part);
  if (!last_cta(&a.counters[0])) return;
  reduce_pairs(a.part, gridDim.x, l * l, stage);
  chol_smem(stage, l, a.status);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R1[t] = stage[t];
  if (threadIdx.x == 0) a.counters[0] = 0;
}

template <int LMAX>
__global__ void __launch_bounds__(kThreads) k_upd2(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* R = sm;                    // LMAX x LMAX (row stride LMAX)
  double* stage = sm + LMAX * LMAX;  // max(kStageRows, l) x l4
  stage_r<LMAX>(a.R1, l, R);
  __syncthreads();
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) solve_row_upper<LMAX>(a.H + r * l, R, l, a.Q + r * l);
  __syncthreads();
  double acc[4][4] = {};
  gram_rows(a.Q, l, r0, r1, stage, acc);
  store_gram_part(acc, l, a.part);
  if (!last_cta(&a.counters[1])) return;
  double* Rn = R;
  reduce_pairs(a.part, gridDim.x, l * l, Rn);  // Rn <- W2 (row stride l; R1 no longer needed)
  chol_smem(Rn, l, a.status);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R2[t] = Rn[t];
  __syncthreads();
  // top l x l block of Q = Q1[0:l] R2^-1 (substitution in shared memory), then the modified
  // LU for the Householder signs
  double* top = stage;
  for (int r = threadIdx.x; r < l; r += blockDim.x) {
    const double* q = a.Q + (int64_t)r * l;
    for (int j = 0; j < l; ++j) {
      double v = q[j];
      for (int k = 0; k < j; ++k) v -= top[r * l + k] * Rn[k * l + j];
      top[r * l + j] = v / Rn[j * l + j];
    }
  }
  __syncthreads();
  for (int i = 0; i < l; ++i) {
    const double piv = top[i * l + i];
    const double di = piv >= 0.0 ? -1.0 : 1.0;
    const double p = piv - di;
    __syncthreads();
    if (threadIdx.x == 0) {
      a.D[i] = di;
      top[i * l + i] = p;
    }
    for (int r = i + 1 + threadIdx.x; r < l; r += blockDim.x) top[r * l + i] /= p;
    __syncthreads();
    const int w = l - i - 1;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int r = i + 1 + t / w, cc = i + 1 + t % w;
      top[r * l + cc] -= top[r * l + i] * top[i * l + cc];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) a.counters[1] = 0;
}

template <int LMAX>
__global__ void __launch_bounds__(kThreads) k_upd3(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* R = sm;                  // LMAX x LMAX (row stride LMAX)
  double* red = sm + LMAX * LMAX;  // kThreads x 2
  stage_r<LMAX>(a.R2, l, R);
  __syncthreads();
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) solve_row_upper<LMAX>(a.Q + r * l, R, l, a.Q + r * l);
  __syncthreads();  // this CTA's rows of Q are written
  const int T = col_threads(l);
  double dm = 0.0, dp = 0.0;
  if (threadIdx.x < T) {
    const int c = threadIdx.x % l;
    const double d = a.D[c];
    for (int64_t r = r0 + threadIdx.x / l; r < r1; r += T / l) {
      const double o = a.Omg2[r * l + c], q = a.Q[r * l + c] * d;
      dm += fabs(o - q);
      dp += fabs(o + q);
    }
  }
  red[threadIdx.x * 2] = dm;
  red[threadIdx.x * 2 + 1] = dp;
  __syncthreads();
  for (int c = threadIdx.x; c < l; c += blockDim.x) {  // fixed-order sum over this column's threads
    double m = 0.0, p = 0.0;
    for (int t = c; t < T; t += l) {
      m += red[t * 2];
      p += red[t * 2 + 1];
    }
    a.part[(int64_t)blockIdx.x * 2 * l + c] = m;
    a.part[(int64_t)blockIdx.x * 2 * l + l + c] = p;
  }
  if (!last_cta(&a.counters[2])) return;
  for (int j = threadIdx.x; j < l; j += blockDim.x) {
    const double m = sum_strided(a.part + j, gridDim.x, 2 * l);
    const double p = sum_strided(a.part + l + j, gridDim.x, 2 * l);
    a.mult[j] = (m > 2.0 * p) ? -a.D[j] : a.D[j];  // src/RSVD.hpp:85
  }
  if (threadIdx.x == 0) a.counters[2] = 0;
}

__global__ void __launch_bounds__(kThreads) k_upd4(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* red = sm;  // kThreads
  int64_t r0, r1;
  row_range(a.N, r0, r1);
  const int T = col_threads(l);
  double cs = 0.0;
  if (threadIdx.x < T) {
    const int j = threadIdx.x % l;
    const double mj = a.mult[j];
    for (int64_t r = r0 + threadIdx.x / l; r < r1; r += T / l) {
      const double v = a.Q[r * l + j] * mj;
      a.Omg[r * l + j] = v;
      a.Omg2[r * l + j] = v;
      cs += v;
      if (a.Omgf) a.Omgf[r * l + j] = (float)v;
      if (a.bt1) {
        const int64_t kp = tc_pos(r);
        const float x = (float)v;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        a.bt1[bt_elem(j, kp, 2 * a.bt_half)] = hi;
        a.bt1[bt_elem(a.bt_half + j, kp, 2 * a.bt_half)] = __float2bfloat16_rn(x - __bfloat162float(hi));
      }
    }
  }
  red[threadIdx.x] = cs;
  __syncthreads();
  for (int c = threadIdx.x; c < l; c += blockDim.x) {
    double s = 0.0;
    for (int t = c; t < T; t += l) s += red[t];
    a.part[(int64_t)blockIdx.x * l + c] = s;
  }
  if (!last_cta(&a.counters[3])) return;
  for (int j = threadIdx.x; j < l; j += blockDim.x) a.wsum[j] = sum_strided(a.part + j, gridDim.x, l);
  if (threadIdx.x == 0) a.counters[3] = 0;
}

template <int LMAX>
void launch_all(pcaone_ctx* c, const UpdateArgs& a) {
  const int l4 = (a.l + 3) & ~3;
  const size_t sstage = (size_t)std::max(kStageRows, a.l) * l4 * 8;  // staged rows or an l x l matrix
  const size_t s1 = sstage;
  const size_t s2 = (size_t)LMAX * LMAX * 8 + sstage;
  const size_t s3 = (size_t)LMAX * LMAX * 8 + (size_t)kThreads * 2 * 8;
  const size_t s4 = (size_t)kThreads * 8;
  static bool attr = false;  // shared memory above 48 KB for the widest sketches
  if (!attr) {
    PG_CUDA(cudaFuncSetAttribute(k_upd2<LMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)LMAX * LMAX * 8 + (size_t)std::max(kStageRows, LMAX) * LMAX * 8)));
    attr = true;
  }
  k_upd1<<<a.nblk, kThreads, s1, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd2<LMAX><<<a.nblk, kThreads, s2, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd3<LMAX><<<a.nblk, kThreads, s3, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd4<<<a.nblk, kThreads, s4, c->stream>>>(a);
  PG_CHECK_LAUNCH();
}

}  // namespace

void fused_update(pcaone_ctx* c, UpdateArgs a) {
  PG_REQUIRE(a.l >= 1 && a.l <= kLmax, PCAONE_EBADARG, "sketch width out of range");
  PG_REQUIRE(((a.l + 3) / 4) * ((a.l + 3) / 4) <= kThreads, PCAONE_EBADARG, "sketch width too large for the update");
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
