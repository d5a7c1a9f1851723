// Windowed LD r2 on PC-residualised genotypes (LD flow A of run_ld_stuff with --read-U,
// src/LD.cpp:444-468 and ld_r2_big, src/LD.cpp:419-442).
//
// The reference forms G = (I - U U^T) G_c with G_c the centred genotypes (missing -> 0) and
// prints r_ik^2 with r_ik = G_i.G_k / (|G_i| |G_k|) for every pair of a window. Here
//
//   G_i.G_k = Gc_i.Gc_k - W_i . Y_k,   W = U^T Gc (per SNP, k values), Y = (2I - U^T U) W
//
// and the genotype part is integer-exact: with r = A1 count (missing 0) and nm = non-missing,
// 4 Gc_i.Gc_k = RR - 2 F_k RN - 2 F_i NR + 4 F_i F_k NN, where RR = sum r_i r_k,
// RN = sum r_i nm_k, NR = sum nm_i r_k and NN = sum nm_i nm_k (the pairwise non-missing count)
// are popcounts over bit planes of the packed codes (h = two A1 copies, e = one copy,
// n = non-missing; r = 2h + e), 32 samples per 32-bit word.
#include "internal.hpp"

namespace pg {

namespace {

// Bit planes of one SNP record: word t holds samples 32t..32t+31. planes: [3][M][nw].
__global__ void k_bitplanes(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t M, uint32_t nw,
                            uint32_t* __restrict__ ph, uint32_t* __restrict__ pe, uint32_t* __restrict__ pn) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= M * nw) return;
  const uint64_t j = t / nw;
  const uint32_t w = (uint32_t)(t - j * nw);
  const uint64_t x = *reinterpret_cast<const uint64_t*>(bed + j * pitch + (uint64_t)w * 8);  // 32 codes
  uint32_t h = 0, e = 0, n = 0;
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    uint32_t c = (uint32_t)(x >> (2 * s)) & 3u;
    h |= (uint32_t)(c == 0) << s;   // 00: two A1
    e |= (uint32_t)(c == 2) << s;   // 10: one A1
    n |= (uint32_t)(c != 1) << s;   // padding codes are 11: counted non-missing, r = 0
  }
  ph[t] = h;
  pe[t] = e;
  pn[t] = n;
}

struct PairSums {
  long long rr, rn, nr, nn;
};

__device__ __forceinline__ PairSums pair_sums(const uint32_t* __restrict__ hi, const uint32_t* __restrict__ ei,
                                              const uint32_t* __restrict__ ni, const uint32_t* __restrict__ hk,
                                              const uint32_t* __restrict__ ek, const uint32_t* __restrict__ nk,
                                              uint32_t nw, int lane) {
  int rr = 0, rn = 0, nr = 0, nn = 0;
  for (uint32_t w = lane; w < nw; w += 32) {
    const uint32_t a = hi[w], b = ei[w], c = ni[w], d = hk[w], f = ek[w], g = nk[w];
    rr += 4 * __popc(a & d) + 2 * (__popc(a & f) + __popc(b & d)) + __popc(b & f);
    rn += 2 * __popc(a & g) + __popc(b & g);
    nr += 2 * __popc(c & d) + __popc(c & f);
    nn += __popc(c & g);
  }
  for (int o = 16; o; o >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, o);
    rn += __shfl_xor_sync(0xffffffffu, rn, o);
    nr += __shfl_xor_sync(0xffffffffu, nr, o);
    nn += __shfl_xor_sync(0xffffffffu, nn, o);
  }
  return {rr, rn, nr, nn};
}

// Centred genotype cross product from the integer sums; npad samples (code 11) have r = 0
// and are counted in NN, which is corrected by subtracting them (they carry F_i F_k each).
__device__ __forceinline__ double centred_dot(PairSums s, double Fi, double Fk, long long npad) {
  const double nn = (double)(s.nn - npad);
  return 0.25 * ((double)s.rr - 2.0 * Fk * (double)s.rn - 2.0 * Fi * (double)s.nr) + Fi * Fk * nn;
}

// Warp per SNP: d_i = |G_i|^2 of the residualised column.
__global__ void k_ld_diag(const uint32_t* __restrict__ ph, const uint32_t* __restrict__ pe,
                          const uint32_t* __restrict__ pn, uint64_t M, uint32_t nw, long long npad,
                          const double* __restrict__ F, const double* __restrict__ W,
                          const double* __restrict__ Y, int k, double* __restrict__ d) {
  const uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= M) return;
  const uint32_t *h = ph + i * nw, *e = pe + i * nw, *n = pn + i * nw;
  PairSums s = pair_sums(h, e, n, h, e, n, nw, lane);
  double wy = 0.0;
  if (W)
    for (int t = lane; t < k; t += 32) wy += W[i * k + t] * Y[i * k + t];
  for (int o = 16; o; o >>= 1) wy += __shfl_xor_sync(0xffffffffu, wy, o);
  if (lane == 0) d[i] = centred_dot(s, F[i], F[i], npad) - wy;
}

// CTA per window: warp per follower k of the lead SNP i; writes r^2 in pair order (as float
// for the .ld.gz text, or as double for the pruning and clumping decisions).
template <typename OutT>
__global__ void k_ld_pairs(const uint32_t* __restrict__ ph, const uint32_t* __restrict__ pe,
                           const uint32_t* __restrict__ pn, uint32_t nw, long long npad,
                           const double* __restrict__ F, const double* __restrict__ W,
                           const double* __restrict__ Y, int k, const double* __restrict__ d,
                           const int64_t* __restrict__ ws, const int32_t* __restrict__ we,
                           const int64_t* __restrict__ off, OutT* __restrict__ r2) {
  const int64_t w = blockIdx.x;
  const int64_t i = ws[w];
  const int cnt = we[w];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t *hi = ph + i * nw, *ei = pe + i * nw, *ni = pn + i * nw;
  for (int t = 1 + warp; t < cnt; t += nwarps) {
    const int64_t kk = i + t;
    PairSums s = pair_sums(hi, ei, ni, ph + kk * nw, pe + kk * nw, pn + kk * nw, nw, lane);
    double wy = 0.0;
    if (W)
      for (int q = lane; q < k; q += 32) wy += W[i * k + q] * Y[kk * k + q];
    for (int o = 16; o; o >>= 1) wy += __shfl_xor_sync(0xffffffffu, wy, o);
    if (lane == 0) {
      const double num = centred_dot(s, F[i], F[kk], npad) - wy;
      const double r = num / sqrt(d[i] * d[kk]);
      r2[off[w] + t - 1] = (OutT)(r * r);
    }
  }
}

// ---------------------------------------------------------------- LD flow B
// Residual matrix of Data::write_residuals (src/Data.cpp:196-245): R_ij = Gc_ij - sum_t US_it
// V_jt with Gc the centred genotypes (BED2GENO - F_j, missing -> 0; ld_stats 0) or Gc itself
// without factors (ld_stats 1), then every SNP column centred over the samples (FP64), stored
// as float, SNP-major (row jj = SNP snp0 + jj of the current order). Warp per SNP; the
// residual is recomputed in the second pass instead of being stored.
__global__ void k_residuals(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t snp0, uint64_t nsnp,
                            uint32_t N, const double* __restrict__ F, const double* __restrict__ US,
                            const double* __restrict__ V, int k, float* __restrict__ out) {
  __shared__ double vs[8][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t jj = (uint64_t)blockIdx.x * 8 + warp;
  if (jj >= nsnp) return;
  const uint64_t j = snp0 + jj;
  const double f = F[j];
  if (V)
    for (int t = lane; t < k; t += 32) vs[warp][t] = V[jj * k + t];
  __syncwarp();
  const uint8_t* rec = bed + j * pitch;
  auto resid = [&](uint32_t i) {
    const int code = (rec[i >> 2] >> (2 * (i & 3))) & 3;
    double g = code == 1 ? 0.0 : (code == 0 ? 1.0 : (code == 2 ? 0.5 : 0.0)) - f;
    if (V)
      for (int t = 0; t < k; ++t) g -= US[(uint64_t)i * k + t] * vs[warp][t];
    return g;
  };
  double s = 0.0;
  for (uint32_t i = lane; i < N; i += 32) s += resid(i);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const double mean = s / N;
  for (uint32_t i = lane; i < N; i += 32) out[jj * N + i] = (float)(resid(i) - mean);
}

// Dense matrix X (SNP-major floats, row stride ldx) -> column-centred copy in place (FP64
// mean, FileBin::read_all, src/FileBinary.cpp:21-30) and the squared norms d_j of the centred
// columns (calc_sds, src/LD.cpp:20-23, without the common 1/(N-1)). Warp per SNP.
__global__ void k_dense_center(float* __restrict__ X, uint32_t ldx, uint64_t M, uint32_t N, double* __restrict__ d) {
  const uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= M) return;
  float* row = X + j * ldx;
  double s = 0.0;
  for (uint32_t i = lane; i < N; i += 32) s += (double)row[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const double mean = s / N;
  double q = 0.0;
  for (uint32_t i = lane; i < N; i += 32) {
    const double v = (double)row[i] - mean;
    row[i] = (float)v;
    q += (double)row[i] * (double)row[i];
  }
  for (int o = 16; o; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  if (lane == 0) d[j] = q;
}

// Band Gram of the centred dense matrix for LD flow B (ld_r2_big, src/LD.cpp:419-442): CTA
// (lead block b of 32 SNPs, partner tile q of 32 SNPs starting at 32 b + 32 q); the 32 x 32
// dot products are accumulated in FP64 from the float values (each product exact in FP64),
// over sample chunks of 64 staged in shared memory; thread t owns lead row t / 8 and four
// partner columns. Pairs (i, k) with 1 <= k - i < we[w] of the lead's window w are written
// as r^2 = (X_i.X_k)^2 / (d_i d_k) to r2[off[w] + k - i - 1].
constexpr int kLdTile = 32, kLdChunk = 64;
template <typename OutT>
__global__ void __launch_bounds__(256) k_ld_dense(const float* __restrict__ X, uint32_t ldx, uint64_t M, uint32_t N,
                                                  const double* __restrict__ d, const int64_t* __restrict__ win_of,
                                                  const int32_t* __restrict__ we, const int64_t* __restrict__ off,
                                                  const int32_t* __restrict__ span, OutT* __restrict__ r2) {
  __shared__ double A[kLdTile][kLdChunk + 1], B[kLdTile][kLdChunk + 1];
  const uint64_t i0 = (uint64_t)blockIdx.x * kLdTile;
  const uint64_t k0 = i0 + (uint64_t)blockIdx.y * kLdTile;
  if (k0 >= M || (int64_t)blockIdx.y * kLdTile > span[blockIdx.x]) return;
  const int t = threadIdx.x, r = t >> 3, c0 = (t & 7) * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t s0 = 0; s0 < N; s0 += kLdChunk) {
    __syncthreads();
    for (int e = t; e < kLdTile * kLdChunk; e += 256) {
      const int rr = e / kLdChunk, ss = e - rr * kLdChunk;
      const uint64_t ia = i0 + rr, ib = k0 + rr;
      const uint32_t s = s0 + ss;
      A[rr][ss] = (ia < M && s < N) ? (double)X[ia * ldx + s] : 0.0;
      B[rr][ss] = (ib < M && s < N) ? (double)X[ib * ldx + s] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int ss = 0; ss < kLdChunk; ++ss) {
      const double a = A[r][ss];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(a, B[c0 + q][ss], acc[q]);
    }
  }
  const uint64_t i = i0 + r;
  if (i >= M) return;
  const int64_t w = win_of[i];
  if (w < 0) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint64_t kk = k0 + c0 + q;
    const int64_t dist = (int64_t)kk - (int64_t)i;
    if (kk < M && dist >= 1 && dist < we[w]) {
      const double rr = acc[q] / sqrt(d[i] * d[kk]);
      r2[off[w] + dist - 1] = (OutT)(rr * rr);
    }
  }
}

}  // namespace

void residuals(pcaone_ctx* c, const double* US, const double* V, int k, uint64_t snp0, uint64_t nsnp, float* out) {
  k_residuals<<<(unsigned)((nsnp + 7) / 8), 256, 0, c->stream>>>(c->d_bed, c->pitch, snp0, nsnp, c->N, c->d_F, US,
                                                                  V, k, out);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void dense_center(pcaone_ctx* c, double* d) {
  k_dense_center<<<(unsigned)((c->M * 32 + 255) / 256), 256, 0, c->stream>>>(c->d_E, c->Npad, c->M, c->N, d);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void ld_r2_dense(pcaone_ctx* c, const double* d, const int64_t* d_win_of, const int32_t* d_we, const int64_t* d_off,
                 const int32_t* d_span, int max_span, void* d_r2, bool f64) {
  const uint64_t blocks = (c->M + kLdTile - 1) / kLdTile;
  const unsigned tiles = (unsigned)((max_span + kLdTile) / kLdTile);
  PG_REQUIRE(blocks < (1ull << 31) && tiles < 65536, PCAONE_EBADARG, "LD band too large");
  if (f64)
    k_ld_dense<double><<<dim3((unsigned)blocks, tiles), 256, 0, c->stream>>>(c->d_E, c->Npad, c->M, c->N, d, d_win_of,
                                                                             d_we, d_off, d_span, (double*)d_r2);
  else
    k_ld_dense<float><<<dim3((unsigned)blocks, tiles), 256, 0, c->stream>>>(c->d_E, c->Npad, c->M, c->N, d, d_win_of,
                                                                            d_we, d_off, d_span, (float*)d_r2);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void ld_r2(pcaone_ctx* c, const double* W, const double* Y, int k, const int64_t* d_ws,
           const int32_t* d_we, const int64_t* d_off, int64_t nwin, void* d_r2, bool f64) {
  const uint32_t nw = (c->N + 31) / 32;  // 32 samples per word; pitch covers ceil(N/32)*8 bytes
  PG_REQUIRE((uint64_t)nw * 8 <= c->pitch, PCAONE_EBADARG, "pitch too small for bit planes");
  const long long npad = (long long)nw * 32 - c->N;
  const size_t plane = (size_t)c->M * nw;
  uint32_t* ph = (uint32_t*)scratch(c, "ld_planes", plane * 3 * 4);
  uint32_t* pe = ph + plane;
  uint32_t* pn = pe + plane;
  k_bitplanes<<<(unsigned)((plane + 255) / 256), 256, 0, c->stream>>>(c->d_bed, c->pitch, c->M, nw, ph, pe, pn);
  PG_CHECK_LAUNCH();
  double* d = (double*)scratch(c, "ld_diag", c->M * 8);
  k_ld_diag<<<(unsigned)((c->M * 32 + 255) / 256), 256, 0, c->stream>>>(ph, pe, pn, c->M, nw, npad, c->d_F, W,
                                                                         Y, k, d);
  PG_CHECK_LAUNCH();
  if (nwin > 0) {
    if (f64)
      k_ld_pairs<double><<<(unsigned)nwin, 256, 0, c->stream>>>(ph, pe, pn, nw, npad, c->d_F, W, Y, k, d, d_ws, d_we,
                                                               d_off, (double*)d_r2);
    else
      k_ld_pairs<float><<<(unsigned)nwin, 256, 0, c->stream>>>(ph, pe, pn, nw, npad, c->d_F, W, Y, k, d, d_ws, d_we,
                                                              d_off, (float*)d_r2);
    PG_CHECK_LAUNCH();
  }
  c->launches += 3;
}

}  // namespace pg
