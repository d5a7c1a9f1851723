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
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.hpp"
#include "tc_layout.hpp"
#include "update.hpp"

namespace pg {

namespace {

constexpr int kThreads = 512;
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

// Accumulate this CTA's rows of A^T A into per-thread pairs (staging rows in shared memory).
__device__ void gram_rows(const double* A, int l, int64_t r0, int64_t r1, double* stage, double (&acc)[8]) {
  const int npairs = l * l;
  for (int64_t b = r0; b < r1; b += kStageRows) {
    const int nr = (int)(r1 - b < kStageRows ? r1 - b : kStageRows);
    __syncthreads();
    for (int t = threadIdx.x; t < nr * l; t += blockDim.x) stage[t] = A[b * l + t];
    __syncthreads();
    for (int q = 0; q < 8; ++q) {
      const int p = threadIdx.x + q * blockDim.x;
      if (p >= npairs) break;
      const int i = p / l, j = p - i * l;
      double s = acc[q];
      for (int r = 0; r < nr; ++r) s = fma(stage[r * l + i], stage[r * l + j], s);
      acc[q] = s;
    }
  }
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

__device__ void reduce_pairs(const double* part, int nblk, int npairs, double* out_smem) {
  for (int p = threadIdx.x; p < npairs; p += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * npairs + p];
    out_smem[p] = s;
  }
  __syncthreads();
}

__device__ void trsm_row(const double* a, const double* R, int l, double* x) {
  for (int j = 0; j < l; ++j) {
    double v = a[j];
    for (int k = 0; k < j; ++k) v -= x[k] * R[k * l + j];
    x[j] = v / R[j * l + j];
  }
}

__global__ void __launch_bounds__(kThreads) k_upd1(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* stage = sm;  // kStageRows * l (also reused for the l*l reduction)
  const int64_t rpb = (a.N + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rpb, r1 = (a.N < r0 + rpb ? a.N : r0 + rpb);
  if (a.H2) {
    for (int64_t t = r0 * l + threadIdx.x; t < r1 * l; t += blockDim.x) a.H[t] = a.H1[t] + a.H2[t];
    __syncthreads();
    __threadfence_block();
  }
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  gram_rows(a.H, l, r0, r1, stage, acc);
  for (int q = 0; q < 8; ++q) {
    const int p = threadIdx.x + q * blockDim.x;
    if (p < l * l) a.part[(int64_t)blockIdx.x * l * l + p] = acc[q];
  }
  if (!last_cta(&a.counters[0])) return;
  reduce_pairs(a.part, gridDim.x, l * l, stage);
  chol_smem(stage, l, a.status);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R1[t] = stage[t];
  if (threadIdx.x == 0) a.counters[0] = 0;
}

__global__ void __launch_bounds__(kThreads) k_upd2(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* R = sm;            // l*l
  double* stage = sm + l * l;  // kStageRows * l
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) R[t] = a.R1[t];
  __syncthreads();
  const int64_t rpb = (a.N + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rpb, r1 = (a.N < r0 + rpb ? a.N : r0 + rpb);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double x[kLmax];
    trsm_row(a.H + r * l, R, l, x);
    for (int j = 0; j < l; ++j) a.Q[r * l + j] = x[j];
  }
  __syncthreads();
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  gram_rows(a.Q, l, r0, r1, stage, acc);
  for (int q = 0; q < 8; ++q) {
    const int p = threadIdx.x + q * blockDim.x;
    if (p < l * l) a.part[(int64_t)blockIdx.x * l * l + p] = acc[q];
  }
  if (!last_cta(&a.counters[1])) return;
  double* W = stage;  // the stage area holds max(kStageRows, l) * l doubles
  double* Rn = R;
  reduce_pairs(a.part, gridDim.x, l * l, Rn);  // Rn <- W2 (R1 no longer needed)
  chol_smem(Rn, l, a.status);
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) a.R2[t] = Rn[t];
  __syncthreads();
  // top l x l block of Q = Q1[0:l] R2^-1, then the modified LU for the Householder signs
  double* top = W;  // l*l doubles in the stage area
  for (int r = threadIdx.x; r < l; r += blockDim.x) {
    double x[kLmax];
    trsm_row(a.Q + (int64_t)r * l, Rn, l, x);
    for (int j = 0; j < l; ++j) top[r * l + j] = x[j];
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

__global__ void __launch_bounds__(kThreads) k_upd3(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  double* R = sm;                // l*l
  double* red = sm + l * l;      // 2 * l sums per warp slot: [nwarps][2l]
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) R[t] = a.R2[t];
  const int nwarps = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < nwarps * 2 * l; t += blockDim.x) red[t] = 0.0;
  __syncthreads();
  const int64_t rpb = (a.N + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rpb, r1 = (a.N < r0 + rpb ? a.N : r0 + rpb);
  double dm[kLmax], dp[kLmax];
  for (int j = 0; j < l; ++j) dm[j] = dp[j] = 0.0;
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double x[kLmax];
    trsm_row(a.Q + r * l, R, l, x);
    for (int j = 0; j < l; ++j) {
      a.Q[r * l + j] = x[j];
      const double o = a.Omg2[r * l + j], q = x[j] * a.D[j];
      dm[j] += fabs(o - q);
      dp[j] += fabs(o + q);
    }
  }
  // block reduction of dm, dp (warp shuffle, then fixed-order sum over warps)
  for (int j = 0; j < l; ++j) {
    double u = dm[j], v = dp[j];
    for (int o = 16; o; o >>= 1) {
      u += __shfl_xor_sync(0xffffffffu, u, o);
      v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    if (lane == 0) {
      red[warp * 2 * l + j] = u;
      red[warp * 2 * l + l + j] = v;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 2 * l; t += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; ++w) s += red[w * 2 * l + t];
    a.part[(int64_t)blockIdx.x * 2 * l + t] = s;
  }
  if (!last_cta(&a.counters[2])) return;
  for (int j = threadIdx.x; j < l; j += blockDim.x) {
    double m = 0.0, p = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) {
      m += a.part[(int64_t)b * 2 * l + j];
      p += a.part[(int64_t)b * 2 * l + l + j];
    }
    a.mult[j] = (m > 2.0 * p) ? -a.D[j] : a.D[j];  // src/RSVD.hpp:85
  }
  if (threadIdx.x == 0) a.counters[2] = 0;
}

__global__ void __launch_bounds__(kThreads) k_upd4(UpdateArgs a) {
  extern __shared__ double sm[];
  const int l = a.l;
  const int nwarps = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  double* red = sm;  // [nwarps][l]
  const int64_t rpb = (a.N + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rpb, r1 = (a.N < r0 + rpb ? a.N : r0 + rpb);
  double cs[kLmax];
  for (int j = 0; j < l; ++j) cs[j] = 0.0;
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int64_t kp = tc_pos(r);
    for (int j = 0; j < l; ++j) {
      const double v = a.Q[r * l + j] * a.mult[j];
      a.Omg[r * l + j] = v;
      a.Omg2[r * l + j] = v;
      cs[j] += v;
      if (a.Omgf) a.Omgf[r * l + j] = (float)v;
      if (a.bt1) {
        const float x = (float)v;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        a.bt1[bt_elem(j, kp, 2 * a.bt_half)] = hi;
        a.bt1[bt_elem(a.bt_half + j, kp, 2 * a.bt_half)] = __float2bfloat16_rn(x - __bfloat162float(hi));
      }
    }
  }
  for (int j = 0; j < l; ++j) {
    double u = cs[j];
    for (int o = 16; o; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
    if (lane == 0) red[warp * l + j] = u;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < l; t += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; ++w) s += red[w * l + t];
    a.part[(int64_t)blockIdx.x * l + t] = s;
  }
  if (!last_cta(&a.counters[3])) return;
  for (int j = threadIdx.x; j < l; j += blockDim.x) {
    double s = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) s += a.part[(int64_t)b * l + j];
    a.wsum[j] = s;
  }
  if (threadIdx.x == 0) a.counters[3] = 0;
}

}  // namespace

void fused_update(pcaone_ctx* c, UpdateArgs a) {
  PG_REQUIRE(a.l >= 1 && a.l <= kLmax, PCAONE_EBADARG, "sketch width out of range");
  const int nblk = a.nblk;
  const size_t s1 = (size_t)std::max(kStageRows, a.l) * a.l * 8;  // staged rows or an l x l matrix
  const size_t s2 = (size_t)a.l * a.l * 8 + s1;
  const size_t s3 = (size_t)a.l * a.l * 8 + (size_t)(kThreads / 32) * 2 * a.l * 8;
  const size_t s4 = (size_t)(kThreads / 32) * a.l * 8;
  k_upd1<<<nblk, kThreads, s1, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd2<<<nblk, kThreads, s2, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd3<<<nblk, kThreads, s3, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  k_upd4<<<nblk, kThreads, s4, c->stream>>>(a);
  PG_CHECK_LAUNCH();
  c->launches += 4;
}

}  // namespace pg
