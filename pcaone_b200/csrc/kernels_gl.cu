// PCAngsd on genotype likelihoods: allele-frequency EM, posterior expected genotypes and the
// standardised posterior matrix with its diagonal, plus the dense-matrix decode-GEMM back end
// the RSVD uses on that matrix.
//
//  * emMAF_with_GL (src/Utils.cpp:501-531)
//  * FileBeagle::read_all initial E (src/FileBeagle.cpp:121-143) and Data::fit_with_pi PCAngsd
//    branch (src/Data.cpp:249-270): E_ij = (p1 + 2 p2)/(p0 + p1 + p2) - 2 F_j with
//    p0 = P0 (1-pt)^2, p1 = P1 2 pt (1-pt), p2 = (1 - P0 - P1) pt^2 and pt = F_j initially or
//    clip((U S V^T + 2F)/2, 1e-4, 1 - 1e-4) in the EM steps
//  * Data::pcangsd_standardize_E (src/Data.cpp:301-343)
//
// Layout: GL pairs are SNP-major floats, P[j][2i + {0,1}] (the reference's 2N x M column-major
// P); E is SNP-major floats E[j][i] with rows padded to Npad samples (zeros beyond N).
// Posterior arithmetic is FP64 in registers.
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "internal.hpp"
#include "rsvd.hpp"

namespace pg {

namespace {

__device__ __forceinline__ void posterior(double P0, double P1, double pt, double& p0, double& p1, double& p2) {
  p0 = P0 * (1.0 - pt) * (1.0 - pt);
  p1 = P1 * 2 * pt * (1.0 - pt);
  p2 = (1 - P0 - P1) * pt * pt;
}

// One EM sweep of the allele frequencies: warp per SNP. diff2[j] = (F_new - F_old)^2.
__global__ void k_em_maf(const double* __restrict__ P, uint64_t M, uint32_t N, uint32_t ldp,
                         double* __restrict__ F, double* __restrict__ diff2) {
  const uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= M) return;
  const double f = F[j];
  const double2* row = reinterpret_cast<const double2*>(P + j * ldp);
  double acc = 0.0;
  for (uint32_t i = lane; i < N; i += 32) {
    const double2 gl = __ldg(row + i);
    double p0, p1, p2;
    posterior(gl.x, gl.y, f, p0, p1, p2);
    acc += (p1 + 2.0 * p2) / (p0 + p1 + p2);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    const double fn = acc * (1.0 / (2.0 * N));
    diff2[j] = (fn - f) * (fn - f);
    F[j] = fn;
  }
}

// E_ij = E[g | likelihoods, pt_ij] - 2 F_j for SNP rows (fit_with_pi, src/Data.cpp:249-270);
// the standardised E of the GRM stage is k_grm_e. Thread per sample: the sample's row of
// US (U diag S, N x k row-major) stays in registers (KM >= k is a compile-time bound) and the
// thread walks the sites of its CTA's slice; the loading row V[j] (M x k row-major) and F_j
// are the same for every thread of the CTA (broadcast loads), the likelihood pair (one
// double2) and the E entry are coalesced over the samples. Each sample-site is one 16-byte
// read and one 4-byte write, eight sites in flight per thread.
template <int KM>
__global__ void __launch_bounds__(128) k_posterior_e(const double* __restrict__ P, uint64_t M, uint32_t N, uint32_t ldp,
                                                     const double* __restrict__ F, const double* __restrict__ US,
                                                     const double* __restrict__ V, int k, float* __restrict__ E,
                                                     uint32_t lde) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint64_t per = (M + gridDim.y - 1) / gridDim.y;
  const uint64_t ja = (uint64_t)blockIdx.y * per, jb = ja + per < M ? ja + per : M;
  double us[KM];
#pragma unroll
  for (int t = 0; t < KM; ++t) us[t] = (V && t < k) ? US[(uint64_t)i * k + t] : 0.0;
  constexpr int U4 = 8;
  uint64_t j = ja;
  for (; j + U4 <= jb; j += U4) {
    double2 gl[U4];
#pragma unroll
    for (int u = 0; u < U4; ++u) gl[u] = __ldcs(reinterpret_cast<const double2*>(P + (j + u) * ldp) + i);
#pragma unroll
    for (int u = 0; u < U4; ++u) {
      const double f = __ldg(F + j + u);
      double pt = f;
      if (V) {
        double pred = 0.0;
        const double* v = V + (j + u) * k;
#pragma unroll
        for (int t = 0; t < KM; ++t)
          if (t < k) pred += us[t] * __ldg(v + t);
        pt = fmin(fmax((pred + 2.0 * f) / 2.0, 1e-4), 1.0 - 1e-4);
      }
      double p0, p1, p2;
      posterior(gl[u].x, gl[u].y, pt, p0, p1, p2);
      __stcs(E + (j + u) * lde + i, (float)((p1 + 2.0 * p2) / (p0 + p1 + p2) - 2.0 * f));
    }
  }
  for (; j < jb; ++j) {
    const double2 gl = __ldcs(reinterpret_cast<const double2*>(P + j * ldp) + i);
    const double f = __ldg(F + j);
    double pt = f;
    if (V) {
      double pred = 0.0;
      const double* v = V + j * k;
#pragma unroll
      for (int t = 0; t < KM; ++t)
        if (t < k) pred += us[t] * __ldg(v + t);
      pt = fmin(fmax((pred + 2.0 * f) / 2.0, 1e-4), 1.0 - 1e-4);
    }
    double p0, p1, p2;
    posterior(gl.x, gl.y, pt, p0, p1, p2);
    __stcs(E + j * lde + i, (float)((p1 + 2.0 * p2) / (p0 + p1 + p2) - 2.0 * f));
  }
}

// PLINK input with --pcangsd (FileBed::read_all, src/FilePlink.cpp:89-115): pseudo-likelihood
// pairs from the genotype codes, 11 (RR) -> (1, 0), 00 (AA) -> (0, 0), 10 (RA) -> (0, 1),
// 01 (missing) -> (0.333333, 0.333333), and the initial matrix E = BED2GENO - F_j with
// BED2GENO = {1, -, 0.5, 0} and missing -> 0. Warp per SNP row of the packed codes.
__global__ void k_bed_pseudo_gl(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t M, uint32_t N,
                                const double* __restrict__ F, double* __restrict__ P, uint32_t ldp,
                                float* __restrict__ E, uint32_t lde) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (uint64_t j = (uint64_t)blockIdx.x * nwarps + warp; j < M; j += (uint64_t)gridDim.x * nwarps) {
    const double f = F[j];
    const uint8_t* rec = bed + j * pitch;
    for (uint32_t i = lane; i < N; i += 32) {
      const int code = (rec[i >> 2] >> (2 * (i & 3))) & 3;
      double p0 = 0.0, p1 = 0.0;
      float e = 0.0f;
      if (code == 3) {
        p0 = 1.0;
        e = (float)(0.0 - f);
      } else if (code == 0) {
        e = (float)(1.0 - f);
      } else if (code == 2) {
        p1 = 1.0;
        e = (float)(0.5 - f);
      } else {
        p0 = p1 = 0.333333;
      }
      P[j * ldp + 2 * i] = p0;
      P[j * ldp + 2 * i + 1] = p1;
      E[j * lde + i] = e;
    }
  }
}

// Dense SIMT GEMM: out[s][r][c] = sum_{k in split s} A(r, k) * B[k][c]. A(r, k) is
// A[r * lda + k] when !AT (rows = SNPs, K = samples) and A[k * lda + r] when AT (rows =
// samples of E's rows, K = SNPs). Same tiling as the decode-GEMM: 128 rows x 8 columns per
// warp group, 4 rows x 8 columns per thread.
template <bool AT, int G>
__global__ void __launch_bounds__(32 * G)
k_dense_gemm(const float* __restrict__ A, uint64_t lda, int64_t rows, int64_t K, const float* __restrict__ B,
             int l, int64_t kchunks_per_split, float* __restrict__ out) {
  constexpr int TR = 128, KC = 32, LDSB = G * 8;
  __shared__ float as[KC][TR + 1];
  __shared__ __align__(16) float bs[KC * LDSB];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int64_t r0 = (int64_t)blockIdx.x * TR;
  const int64_t kc_total = (K + KC - 1) / KC;
  const int64_t kc0 = (int64_t)blockIdx.y * kchunks_per_split;
  const int64_t kc1 = min(kc0 + kchunks_per_split, kc_total);
  float acc[4][8];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[q][c] = 0.f;
  for (int64_t kc = kc0; kc < kc1; ++kc) {
    const int64_t k0 = kc * KC;
    for (int t = threadIdx.x; t < KC * TR; t += 32 * G) {
      int kk, r;
      if (AT) {
        kk = t / TR;
        r = t - kk * TR;
      } else {
        r = t / KC;
        kk = t - r * KC;
      }
      const int64_t row = r0 + r, k = k0 + kk;
      float v = 0.f;
      if (row < rows && k < K) v = AT ? A[(uint64_t)k * lda + row] : A[(uint64_t)row * lda + k];
      as[kk][r] = v;
    }
    for (int t = threadIdx.x; t < KC * LDSB; t += 32 * G) {
      int kk = t / LDSB, cc = t - kk * LDSB;
      int64_t k = k0 + kk;
      bs[t] = (cc < l && k < K) ? B[k * l + cc] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KC; ++kk) {
      float b[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) b[c] = bs[kk * LDSB + g * 8 + c];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float a = as[kk][lane + 32 * q];
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[q][c] = fmaf(a, b[c], acc[q][c]);
      }
    }
    __syncthreads();
  }
  float* o = out + (int64_t)blockIdx.y * rows * l;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int64_t r = r0 + lane + 32 * q;
    if (r >= rows) continue;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int col = g * 8 + c;
      if (col < l) o[r * l + col] = acc[q][c];
    }
  }
}

// Register-tiled form for sketch widths l <= 48 (the PCAngsd RSVD: l = k + max(10, k)):
// CTA = 128 rows x CN columns (CN = l rounded up to 16), 256 threads; thread (ty, tx) owns
// rows 4 ty .. 4 ty + 3 and columns tx CN/8 .. (tx + 1) CN/8 - 1. K runs in chunks of 32
// through two shared-memory buffers (k-major A tile, so one 16-byte load gives the thread's
// four rows); the next chunk's global loads are issued (16 bytes per thread and load) before
// the current chunk is multiplied. The product is bound by reading A once from HBM.
template <bool AT, int CN>
__global__ void __launch_bounds__(256)
k_dense_gemm2(const float* __restrict__ A, uint64_t lda, int64_t rows, int64_t K, const float* __restrict__ B,
              int l, int64_t kchunks_per_split, float* __restrict__ out) {
  constexpr int TR = 128, KC = 32, CW = CN / 8;
  __shared__ __align__(16) float as[2][KC][TR + 4];
  __shared__ __align__(16) float bs[2][KC][CN];
  const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
  const int64_t r0 = (int64_t)blockIdx.x * TR;
  const int64_t kc_total = (K + KC - 1) / KC;
  const int64_t kc0 = (int64_t)blockIdx.y * kchunks_per_split;
  const int64_t kc1 = min(kc0 + kchunks_per_split, kc_total);
  float acc[4][CW];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < CW; ++c) acc[q][c] = 0.f;
  // global -> registers: A is 4096 floats a chunk (four float4 per thread), B KC x CN
  float4 ra[4];
  float rb[(KC * CN + 255) / 256];
  auto load = [&](int64_t kc) {
    const int64_t k0 = kc * KC;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + 256 * u;  // float4 index within the tile
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (AT) {  // A[k][r]: 32 k-rows of 128 r, 32 float4 per k-row
        const int kk = e >> 5, r4 = (e & 31) * 4;
        const int64_t k = k0 + kk, r = r0 + r4;
        if (k < K) {
          const float* src = A + (uint64_t)k * lda + r;
          if (r + 3 < rows && ((uintptr_t)src & 15) == 0)
            v = *reinterpret_cast<const float4*>(src);
          else {
            v.x = r < rows ? src[0] : 0.f;
            v.y = r + 1 < rows ? src[1] : 0.f;
            v.z = r + 2 < rows ? src[2] : 0.f;
            v.w = r + 3 < rows ? src[3] : 0.f;
          }
        }
      } else {  // A[r][k]: 128 rows of 32 k, 8 float4 per row
        const int rr = e >> 3, k4 = (e & 7) * 4;
        const int64_t r = r0 + rr, k = k0 + k4;
        if (r < rows) {
          const float* src = A + (uint64_t)r * lda + k;
          if (k + 3 < K && ((uintptr_t)src & 15) == 0)
            v = *reinterpret_cast<const float4*>(src);
          else {
            v.x = k < K ? src[0] : 0.f;
            v.y = k + 1 < K ? src[1] : 0.f;
            v.z = k + 2 < K ? src[2] : 0.f;
            v.w = k + 3 < K ? src[3] : 0.f;
          }
        }
      }
      ra[u] = v;
    }
#pragma unroll
    for (int u = 0; u < (KC * CN + 255) / 256; ++u) {
      const int e = tid + 256 * u, kk = e / CN, cc = e - kk * CN;
      const int64_t k = k0 + kk;
      rb[u] = (e < KC * CN && cc < l && k < K) ? B[k * l + cc] : 0.f;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + 256 * u;
      if (AT) {
        const int kk = e >> 5, r4 = (e & 31) * 4;
        *reinterpret_cast<float4*>(&as[buf][kk][r4]) = ra[u];
      } else {
        const int rr = e >> 3, k4 = (e & 7) * 4;
        as[buf][k4][rr] = ra[u].x;
        as[buf][k4 + 1][rr] = ra[u].y;
        as[buf][k4 + 2][rr] = ra[u].z;
        as[buf][k4 + 3][rr] = ra[u].w;
      }
    }
#pragma unroll
    for (int u = 0; u < (KC * CN + 255) / 256; ++u) {
      const int e = tid + 256 * u;
      if (e < KC * CN) (&bs[buf][0][0])[e] = rb[u];
    }
  };
  if (kc0 < kc1) {
    load(kc0);
    store(0);
  }
  __syncthreads();
  int buf = 0;
  for (int64_t kc = kc0; kc < kc1; ++kc) {
    const bool more = kc + 1 < kc1;
    if (more) load(kc + 1);  // in flight during this chunk's products
#pragma unroll 8
    for (int kk = 0; kk < KC; ++kk) {
      const float4 a = *reinterpret_cast<const float4*>(&as[buf][kk][4 * ty]);
      float b[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) b[c] = bs[buf][kk][tx * CW + c];
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        acc[0][c] = fmaf(a.x, b[c], acc[0][c]);
        acc[1][c] = fmaf(a.y, b[c], acc[1][c]);
        acc[2][c] = fmaf(a.z, b[c], acc[2][c]);
        acc[3][c] = fmaf(a.w, b[c], acc[3][c]);
      }
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
  float* o = out + (int64_t)blockIdx.y * rows * l;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int64_t r = r0 + 4 * ty + q;
    if (r >= rows) continue;
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      const int col = tx * CW + c;
      if (col < l) o[r * l + col] = acc[q][c];
    }
  }
}

template <bool AT, int G>
void launch_dense_g(pcaone_ctx* c, const float* A, uint64_t lda, int64_t rows, int64_t K, const float* B, int l,
                    int ks, float* out) {
  const int64_t kct = (K + 31) / 32;
  const int64_t per = (kct + ks - 1) / ks;
  dim3 grid((unsigned)((rows + 127) / 128), (unsigned)ks);
  k_dense_gemm<AT, G><<<grid, 32 * G, 0, c->stream>>>(A, lda, rows, K, B, l, per, out);
  PG_CHECK_LAUNCH();
}

template <bool AT, int CN>
void launch_dense2(pcaone_ctx* c, const float* A, uint64_t lda, int64_t rows, int64_t K, const float* B, int l,
                   int ks, float* out) {
  const int64_t kct = (K + 31) / 32;
  const int64_t per = (kct + ks - 1) / ks;
  dim3 grid((unsigned)((rows + 127) / 128), (unsigned)ks);
  k_dense_gemm2<AT, CN><<<grid, 256, 0, c->stream>>>(A, lda, rows, K, B, l, per, out);
  PG_CHECK_LAUNCH();
}

template <bool AT>
void launch_dense(pcaone_ctx* c, const float* A, uint64_t lda, int64_t rows, int64_t K, const float* B, int l,
                  int ks, float* out) {
  if (l <= 48) {
    switch ((l + 15) / 16) {
      case 1: launch_dense2<AT, 16>(c, A, lda, rows, K, B, l, ks, out); break;
      case 2: launch_dense2<AT, 32>(c, A, lda, rows, K, B, l, ks, out); break;
      default: launch_dense2<AT, 48>(c, A, lda, rows, K, B, l, ks, out); break;
    }
    c->launches++;
    c->gemm_launches++;
    return;
  }
  switch ((l + 7) / 8) {
    case 1: launch_dense_g<AT, 1>(c, A, lda, rows, K, B, l, ks, out); break;
    case 2: launch_dense_g<AT, 2>(c, A, lda, rows, K, B, l, ks, out); break;
    case 3: launch_dense_g<AT, 3>(c, A, lda, rows, K, B, l, ks, out); break;
    case 4: launch_dense_g<AT, 4>(c, A, lda, rows, K, B, l, ks, out); break;
    case 5: launch_dense_g<AT, 5>(c, A, lda, rows, K, B, l, ks, out); break;
    case 6: launch_dense_g<AT, 6>(c, A, lda, rows, K, B, l, ks, out); break;
    case 7: launch_dense_g<AT, 7>(c, A, lda, rows, K, B, l, ks, out); break;
    default: launch_dense_g<AT, 8>(c, A, lda, rows, K, B, l, ks, out); break;
  }
  c->launches++;
  c->gemm_launches++;
}

// Back end for the RSVD engine: "codes" are the float rows of E (the engine passes the row
// offset through the pointer), "pitch" is unused.
int dense_ksplit(pcaone_ctx* c, int64_t rows, int64_t K, int) {
  // enough CTAs for four a SM, each split at least four K chunks long
  int64_t tiles = (rows + 127) / 128, chunks = (K + 31) / 32;
  int64_t want = (4 * (int64_t)c->sm_count + tiles - 1) / tiles;
  return (int)std::max<int64_t>(1, std::min<int64_t>({want, chunks / 4, 64}));
}
void dense_p1(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t row0, int64_t rows, int64_t K, const float* B,
              int l, int ks, float* out) {
  launch_dense<false>(c, c->d_E + (uint64_t)row0 * c->Npad, c->Npad, rows, K, B, l, ks, out);
}
void dense_p2(pcaone_ctx* c, const uint8_t*, uint32_t, int64_t window, int64_t rows, int64_t K, const float* B,
              int l, int ks, float* out) {
  launch_dense<true>(c, c->d_E + c->win.start[window] * (uint64_t)c->Npad, c->Npad, rows, K, B, l, ks, out);
}
// Window runs on the dense matrix: a run's windows are contiguous rows of E (blocksize each,
// the last one shorter), so both products are plain products over the run's rows.
int64_t dense_seg_rows(pcaone_ctx* c) { return (int64_t)c->win.blocksize; }
int dense_ksplit_seg(pcaone_ctx* c, int which, int nw, int l) {
  const int64_t m = (int64_t)nw * (int64_t)c->win.blocksize;
  return which == 1 ? dense_ksplit(c, m, (int64_t)c->N, l) : dense_ksplit(c, (int64_t)c->N, m, l);
}
void dense_p1_seg(pcaone_ctx* c, int b0, int b1, const float* B, int l, int ks, float* out) {
  const int64_t s = (int64_t)c->win.start[b0], m = (int64_t)c->win.stop[b1 - 1] - s;
  launch_dense<false>(c, c->d_E + (uint64_t)s * c->Npad, c->Npad, m, (int64_t)c->N, B, l, ks, out);
}
void dense_p2_seg(pcaone_ctx* c, int b0, int b1, const float* B2, int l, int ks, float* out) {
  const int64_t s = (int64_t)c->win.start[b0], m = (int64_t)c->win.stop[b1 - 1] - s;
  launch_dense<true>(c, c->d_E + (uint64_t)s * c->Npad, c->Npad, (int64_t)c->N, m, B2, l, ks, out);
}
void dense_seg_b2(pcaone_ctx*, const float*, int, int, int) {}
void dense_none_omega(pcaone_ctx*, const double*, int, int64_t) {}
void dense_none_b2(pcaone_ctx*, const float*, int, int64_t) {}

// Standardised posterior E of Data::pcangsd_standardize_E (src/Data.cpp:301-343) for the
// sites [j0, j0 + mc) in FP64, with the per-sample diagonal terms. Thread (i, slice): sample
// i over the slice's sites of the chunk, in site order; e is written to E[(j - j0) * lde + i]
// and the slice's diagonal sum is added to dpart[slice * N + i] (each entry has one owner and
// the chunks run in stream order, so the sums are deterministic). US: N x k (U diag S) and
// V: M x k row-major as in k_posterior_e; V null: pt = F_j.
__global__ void __launch_bounds__(128) k_grm_e(const double* __restrict__ P, uint32_t N, uint32_t ldp,
                                               const double* __restrict__ F, const double* __restrict__ US,
                                               const double* __restrict__ V, int k, uint64_t j0, uint64_t mc,
                                               double* __restrict__ E, uint32_t lde, double* __restrict__ dpart) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint64_t per = (mc + gridDim.y - 1) / gridDim.y;
  const uint64_t a = (uint64_t)blockIdx.y * per, b = (a + per < mc ? a + per : mc);
  double dc = 0.0;
  for (uint64_t jl = a; jl < b; ++jl) {
    const uint64_t j = j0 + jl;
    const double f = F[j];
    double pt = f;
    if (V) {
      double pred = 0.0;
      for (int t = 0; t < k; ++t) pred += US[(uint64_t)i * k + t] * V[j * k + t];
      pt = fmin(fmax((pred + 2.0 * f) / 2.0, 1e-4), 1.0 - 1e-4);
    }
    const double2 pp = *reinterpret_cast<const double2*>(P + j * ldp + 2 * i);
    double p0, p1, p2;
    posterior(pp.x, pp.y, pt, p0, p1, p2);
    const double sum = p0 + p1 + p2;
    double e = (p1 + 2.0 * p2) / sum - 2.0 * f;
    const double norm = sqrt(2.0 * f * (1.0 - f));
    if (norm > 1e-9) e /= norm;
    const double f2 = 2.0 * f;
    double t = (0.0 - f2) * (0.0 - f2) * (p0 / sum);
    t += (1.0 - f2) * (1.0 - f2) * (p1 / sum);
    t += (2.0 - f2) * (2.0 - f2) * (p2 / sum);
    dc += t / (2.0 * f * (1.0 - f));
    E[jl * lde + i] = e;
  }
  dpart[(uint64_t)blockIdx.y * N + i] += dc;
}

// C (N x N, column-major, full) = the lower triangle of L (E E^T from the SYRK) mirrored,
// divided by M, with the diagonal replaced by Dc / M, Dc_i = sum over slices of dpart in
// slice order (src/Halko.cpp:322-324).
__global__ void k_grm_finish(const double* __restrict__ L, const double* __restrict__ dpart, int nsl, uint32_t N,
                             double M, double* __restrict__ C) {
  const uint64_t n2 = (uint64_t)N * N;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = (uint32_t)(t / N), i = (uint32_t)(t - (uint64_t)j * N);
    double v;
    if (i == j) {
      v = 0.0;
      for (int sl = 0; sl < nsl; ++sl) v += dpart[(uint64_t)sl * N + i];
    } else {
      v = i > j ? L[t] : L[(uint64_t)i * N + j];
    }
    C[t] = v / M;
  }
}

// Lower-triangular tiles of L = E E^T (N x N, column-major, ld N) over the sites of one
// chunk of the standardised posterior matrix (E: site-major, column j = site j, ld lde): the
// O(N^2 M) product of the GRM (src/Halko.cpp:320, G G^T). One CTA per 128 x 128 tile (I, J)
// with I >= J, 256 threads, each owning an 8 x 8 block (rows 4 ty + {0..3} and 64 + 4 ty +
// {0..3}, columns likewise from tx) accumulated in FP64 registers, site by site in order, so
// the result is deterministic. The two 128-row panels of 16 sites stream through a
// three-stage ring of 16-byte asynchronous copies (zero-filled past N and past the chunk).
// accumulate: add to L (later chunks) instead of overwriting it.
constexpr int kSyrkT = 128, kSyrkKC = 16, kSyrkStages = 3;
constexpr size_t kSyrkSmem = (size_t)kSyrkStages * 2 * kSyrkKC * kSyrkT * sizeof(double);

__device__ __forceinline__ void cp_async16_zfill(double* sdst, const double* gsrc, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(256, 1) k_syrk_lower(const double* __restrict__ E, uint32_t lde, uint32_t N,
                                                       uint64_t mc, double* __restrict__ L, int accumulate) {
  extern __shared__ __align__(16) double smem_syrk[];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const uint32_t t = blockIdx.x;
  uint32_t I = (uint32_t)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  while (I * (I + 1) / 2 > t) --I;
  const uint32_t J = t - I * (I + 1) / 2;
  const uint32_t r0 = I * kSyrkT, c0 = J * kSyrkT;
  const int64_t nk = (int64_t)((mc + kSyrkKC - 1) / kSyrkKC);
  auto issue = [&](int64_t kc, int stage) {
    double* a = smem_syrk + (size_t)stage * 2 * kSyrkKC * kSyrkT;
    double* b = a + kSyrkKC * kSyrkT;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + 256 * u;  // 1024 16-byte pieces per panel: site kk, rows p, p + 1
      const int kk = e >> 6, p = (e & 63) * 2;
      const uint64_t site = (uint64_t)kc * kSyrkKC + kk;
      const bool in = site < mc;
      const uint32_t ra = r0 + p, rb = c0 + p;
      const int ba = in && ra < N ? (int)min(16u, (N - ra) * 8u) : 0;
      const int bb = in && rb < N ? (int)min(16u, (N - rb) * 8u) : 0;
      cp_async16_zfill(a + kk * kSyrkT + p, ba ? E + site * lde + ra : E, ba);
      cp_async16_zfill(b + kk * kSyrkT + p, bb ? E + site * lde + rb : E, bb);
    }
  };
  double acc[8][8];
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[q][c] = 0.0;
#pragma unroll
  for (int st = 0; st < kSyrkStages - 1; ++st) {
    if (st < nk) issue(st, st);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int64_t kc = 0; kc < nk; ++kc) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kSyrkStages - 2) : "memory");
    __syncthreads();  // stage kc landed for every thread; stage kc - 1 is no longer read
    if (kc + kSyrkStages - 1 < nk) issue(kc + kSyrkStages - 1, (int)((kc + kSyrkStages - 1) % kSyrkStages));
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const double* a = smem_syrk + (size_t)(kc % kSyrkStages) * 2 * kSyrkKC * kSyrkT;
    const double* b = a + kSyrkKC * kSyrkT;
#pragma unroll 4
    for (int kk = 0; kk < kSyrkKC; ++kk) {
      double av[8], bv[8];
      const double2* ap = reinterpret_cast<const double2*>(a + kk * kSyrkT);
      const double2* bp = reinterpret_cast<const double2*>(b + kk * kSyrkT);
      const double2 a0 = ap[2 * ty], a1 = ap[2 * ty + 1], a2 = ap[32 + 2 * ty], a3 = ap[33 + 2 * ty];
      const double2 b0 = bp[2 * tx], b1 = bp[2 * tx + 1], b2 = bp[32 + 2 * tx], b3 = bp[33 + 2 * tx];
      av[0] = a0.x; av[1] = a0.y; av[2] = a1.x; av[3] = a1.y;
      av[4] = a2.x; av[5] = a2.y; av[6] = a3.x; av[7] = a3.y;
      bv[0] = b0.x; bv[1] = b0.y; bv[2] = b1.x; bv[3] = b1.y;
      bv[4] = b2.x; bv[5] = b2.y; bv[6] = b3.x; bv[7] = b3.y;
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[q][c] = fma(av[q], bv[c], acc[q][c]);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const uint32_t col = c0 + (c < 4 ? 4 * tx + c : 64 + 4 * tx + c - 4);
    if (col >= N) continue;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t row = r0 + (q < 4 ? 4 * ty + q : 64 + 4 * ty + q - 4);
      if (row >= N) continue;
      double* dst = L + (uint64_t)col * N + row;
      *dst = accumulate ? *dst + acc[q][c] : acc[q][c];
    }
  }
}

}  // namespace

GemmFnT<float> gemm_dense_float() {
  GemmFnT<float> f{dense_ksplit, dense_p1, dense_p2, dense_none_omega, dense_none_b2};
  f.seg_rows1 = dense_seg_rows;
  f.seg_k2 = dense_seg_rows;
  f.ksplit_seg = dense_ksplit_seg;
  f.p1_seg = dense_p1_seg;
  f.b2_seg = dense_seg_b2;
  f.p2_seg = dense_p2_seg;
  return f;
}

__global__ void k_widen(const float* __restrict__ in, size_t n, double* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    out[t] = in[t];
}

void gl_widen_f32(pcaone_ctx* c, const float* P, size_t n, double* dP) {
  const size_t chunk = size_t(16) << 20;  // floats per staging pass (64 MB)
  float* stage = (float*)scratch(c, "gl_stage", std::min(n, chunk) * 4);
  for (size_t a = 0; a < n; a += chunk) {
    const size_t m = std::min(chunk, n - a);
    PG_CUDA(cudaMemcpyAsync(stage, P + a, m * 4, cudaMemcpyHostToDevice, c->stream));
    const unsigned nblk = (unsigned)std::min<size_t>(4 * (size_t)c->sm_count, (m + 255) / 256);
    k_widen<<<nblk, 256, 0, c->stream>>>(stage, m, dP + a);
    PG_CHECK_LAUNCH();
    c->launches++;
  }
}

void gl_from_bed(pcaone_ctx* c) {
  PG_REQUIRE(c->loaded && !c->dense && c->d_bed, PCAONE_ESTATE, "no packed genotypes loaded");
  const size_t np = (size_t)c->M * 2 * c->N;
  double* P = (double*)scratch(c, "d_P", np * 8);
  float* E = (float*)scratch(c, "d_E", (size_t)c->Mpad * c->Npad * 4);
  PG_CUDA(cudaMemsetAsync(E, 0, (size_t)c->Mpad * c->Npad * 4, c->stream));
  const int threads = 256, nwarps = threads / 32;
  const int nblk = (int)std::min<uint64_t>(8 * (uint64_t)c->sm_count, (c->M + nwarps - 1) / nwarps);
  k_bed_pseudo_gl<<<nblk, threads, 0, c->stream>>>(c->d_bed, c->pitch, c->M, c->N, c->d_F, P, 2 * c->N, E, c->Npad);
  PG_CHECK_LAUNCH();
  c->launches++;
  c->d_zero = (double*)scratch(c, "d_zero", c->M * 8);
  PG_CUDA(cudaMemsetAsync(c->d_zero, 0, c->M * 8, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->d_P = P;
  c->d_E = E;
  c->dense = true;
  c->generation++;
  c->bedT_valid = c->miss_snp_valid = c->miss_ws_valid = false;
  c->imputed = false;
}

void gl_em_maf(pcaone_ctx* c, int maxiter, double tolmaf, int* iters) {
  double* diff2 = (double*)scratch(c, "gl_diff2", c->M * 8);
  std::vector<double> h(c->M);
  const double init = 0.25;
  std::vector<double> f0(c->M, init);
  PG_CUDA(cudaMemcpyAsync(c->d_F, f0.data(), c->M * 8, cudaMemcpyHostToDevice, c->stream));
  int it = 0;
  for (it = 0; it < maxiter; ++it) {
    k_em_maf<<<(unsigned)((c->M * 32 + 255) / 256), 256, 0, c->stream>>>(c->d_P, c->M, c->N, 2 * c->N, c->d_F,
                                                                         diff2);
    PG_CHECK_LAUNCH();
    c->launches++;
    PG_CUDA(cudaMemcpyAsync(h.data(), diff2, c->M * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    double sum = 0.0;
    for (uint64_t j = 0; j < c->M; ++j) sum += h[j];
    if (std::sqrt(sum / c->M) < tolmaf) break;
  }
  if (iters) *iters = std::min(it + 1, maxiter);
}

void gl_posterior(pcaone_ctx* c, const double* US, const double* V, int k) {
  PG_REQUIRE(k <= kLmax, PCAONE_EBADARG, "too many factors for the posterior");
  // grid: sample blocks of 128 x site slices, about 16 CTAs an SM (two waves or more of the
  // resident CTAs, so that the slices finish close together)
  const unsigned bx = (c->N + 127) / 128;
  const uint64_t want = (16ull * c->sm_count + bx - 1) / bx;
  const unsigned by = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (c->M + 63) / 64));
  const dim3 grid(bx, by);
  if (k <= 8)
    k_posterior_e<8><<<grid, 128, 0, c->stream>>>(c->d_P, c->M, c->N, 2 * c->N, c->d_F, US, V, k, c->d_E, c->Npad);
  else if (k <= 16)
    k_posterior_e<16><<<grid, 128, 0, c->stream>>>(c->d_P, c->M, c->N, 2 * c->N, c->d_F, US, V, k, c->d_E, c->Npad);
  else if (k <= 32)
    k_posterior_e<32><<<grid, 128, 0, c->stream>>>(c->d_P, c->M, c->N, 2 * c->N, c->d_F, US, V, k, c->d_E, c->Npad);
  else
    k_posterior_e<64><<<grid, 128, 0, c->stream>>>(c->d_P, c->M, c->N, 2 * c->N, c->d_F, US, V, k, c->d_E, c->Npad);
  PG_CHECK_LAUNCH();
  c->launches++;
}

#define PG_SOLVER(call)                                                                          \
  do {                                                                                         \
    const int st_ = (int)(call);                                                               \
    PG_REQUIRE(st_ == 0, PCAONE_ECUDA, std::string(#call) + " failed with status " + std::to_string(st_)); \
  } while (0)

void gl_grm(pcaone_ctx* c, const double* US, const double* V, int k, double* C, double* evecs, double* svals) {
  const uint32_t N = c->N;
  const uint64_t M = c->M;
  const uint32_t ntile = (N + kSyrkT - 1) / kSyrkT;
  PG_CUDA(cudaFuncSetAttribute(k_syrk_lower, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyrkSmem));
  // E in chunks of sites: at most 2^27 doubles (1 GiB) a chunk
  const uint32_t lde = c->Npad;
  uint64_t mc_max = std::max<uint64_t>(1, std::min<uint64_t>(M, (1ull << 27) / lde));
  if (const char* pin = std::getenv("PCAONE_GRM_CHUNK_SITES"))  // smaller chunks, for tests
    mc_max = std::max<uint64_t>(1, std::min<uint64_t>(mc_max, std::strtoull(pin, nullptr, 10)));
  const int nsl = (int)std::max<uint64_t>(1, std::min<uint64_t>(64, (4ull * c->sm_count * 128 + N - 1) / N));
  double* E = (double*)scratch(c, "grm_E", (size_t)mc_max * lde * 8);
  double* dpart = (double*)scratch(c, "grm_dpart", (size_t)nsl * N * 8);
  double* L = (double*)scratch(c, "grm_L", (size_t)N * N * 8);
  double* dC = (double*)scratch(c, "grm_C", (size_t)N * N * 8);
  PG_CUDA(cudaMemsetAsync(dpart, 0, (size_t)nsl * N * 8, c->stream));
  for (uint64_t j0 = 0; j0 < M; j0 += mc_max) {
    const uint64_t mc = std::min<uint64_t>(mc_max, M - j0);
    k_grm_e<<<dim3((N + 127) / 128, nsl), 128, 0, c->stream>>>(c->d_P, N, 2 * N, c->d_F, US, V, k, j0, mc, E, lde,
                                                              dpart);
    PG_CHECK_LAUNCH();
    c->launches++;
    k_syrk_lower<<<ntile * (ntile + 1) / 2, 256, kSyrkSmem, c->stream>>>(E, lde, N, mc, L, j0 == 0 ? 0 : 1);
    PG_CHECK_LAUNCH();
    c->launches++;
  }
  const uint64_t n2 = (uint64_t)N * N;
  k_grm_finish<<<(unsigned)std::min<uint64_t>(8ull * c->sm_count, (n2 + 255) / 256), 256, 0, c->stream>>>(
      L, dpart, nsl, N, (double)M, dC);
  PG_CHECK_LAUNCH();
  c->launches++;
  if (C) PG_CUDA(cudaMemcpyAsync(C, dC, n2 * 8, cudaMemcpyDeviceToHost, c->stream));
  if (evecs || svals) {
    // singular vectors of the symmetric C (JacobiSVD in the reference, src/Halko.cpp:328):
    // eigenvectors ordered by decreasing |eigenvalue|
    if (!c->solver) {
      cusolverDnHandle_t h = nullptr;
      PG_SOLVER(cusolverDnCreate(&h));
      c->solver = h;
    }
    cusolverDnHandle_t sol = (cusolverDnHandle_t)c->solver;
    PG_SOLVER(cusolverDnSetStream(sol, c->stream));
    double* W = (double*)scratch(c, "grm_W", (size_t)N * 8);
    int* info = (int*)scratch(c, "grm_info", sizeof(int));
    int lwork = 0;
    PG_SOLVER(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)N, dC, (int)N, W,
                                        &lwork));
    double* work = (double*)scratch(c, "grm_work", (size_t)std::max(lwork, 1) * 8);
    PG_SOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)N, dC, (int)N, W, work,
                             lwork, info));
    std::vector<double> w(N), vec(evecs ? n2 : 0);
    int hinfo = 0;
    PG_CUDA(cudaMemcpyAsync(w.data(), W, (size_t)N * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    if (evecs) PG_CUDA(cudaMemcpyAsync(vec.data(), dC, n2 * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    PG_REQUIRE(hinfo == 0, PCAONE_ENUMERIC, "eigendecomposition of the PCAngsd GRM failed (info " +
                                                std::to_string(hinfo) + ")");
    std::vector<uint32_t> ord(N);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return std::fabs(w[x]) > std::fabs(w[y]); });
    for (uint32_t r = 0; r < N; ++r) {
      if (svals) svals[r] = std::fabs(w[ord[r]]);
      if (evecs) std::memcpy(evecs + (size_t)r * N, vec.data() + (size_t)ord[r] * N, (size_t)N * 8);
    }
  }
  PG_CUDA(cudaStreamSynchronize(c->stream));
}

void gl_release(pcaone_ctx* c) {
  if (c->solver) cusolverDnDestroy((cusolverDnHandle_t)c->solver);
  c->solver = nullptr;
}

}  // namespace pg
