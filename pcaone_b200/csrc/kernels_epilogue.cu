// Epilogues of the two decode-GEMMs of one window.
//
// The reference multiplies the dense FP64 matrix Z_ij = s_j (x_ij - F_j) (missing -> e_ij,
// 0 before any EM update) by Omega and by G (src/FilePlink.cpp:106-114, src/Data.cpp:290-299,
// src/Halko.cpp:193-202). Here x_ij = r_ij / 2 with r the raw A1 count decoded from the packed
// codes (missing decodes to r = 0), so
//
//   Z_ij = (s_j/2) r_ij - s_j F_j + [missing] s_j (e_ij + F_j)
//
// and the two products become a raw decode-GEMM plus a rank-1 term plus a sparse term over
// the missing entries:
//
//   G_j = s_j/2 (R^T Omega)_j - s_j F_j sum_i Omega_i + sum_{i miss} s_j (e_ij + F_j) Omega_i
//   H_i = (R B2)_i - h0 + sum_{j miss} s_j (e_ij + F_j) G_j,  B2_j = s_j/2 G_j,
//                                                             h0 = sum_j s_j F_j G_j
#include "epilogue.hpp"
#include "tc_layout.hpp"

namespace pg {

namespace {

// Warp-cooperative sparse gather: out[c] = sum_{e in [e0, e1)} w_e * rows[idx_e][c] for all
// c < l. The warp loads 32 entries (index and weight) at once; then four 8-lane groups each
// take one entry per step (two steps unrolled, so eight rows are in flight), and lane q of
// a group owns the columns q, q + 8, ..., so each load instruction reads one contiguous
// 64-byte segment of a row per group and each entry costs a few warp instructions. The
// groups' sums are combined with two shuffle levels in a fixed order (deterministic) and
// written to out (shared memory of this warp). CPL = ceil(l / 8).
template <int CPL, typename R, typename Wt>
__device__ __forceinline__ void gather_rows(int64_t e0, int64_t e1, const int32_t* __restrict__ idx,
                                            const R* __restrict__ rows, int64_t row0, int l, Wt weight,
                                            double* out) {
  constexpr int kSteps = 2;
  const int lane = threadIdx.x & 31, grp = lane >> 3, q = lane & 7;
  double acc[CPL];
#pragma unroll
  for (int k = 0; k < CPL; ++k) acc[k] = 0.0;
  for (int64_t base = e0; base < e1; base += 32) {
    const int64_t e = base + lane;
    int my_i = 0;
    double my_w = 0.0;
    if (e < e1) {
      my_i = idx[e];
      my_w = weight(e, my_i);
    }
    const int cnt = (int)(e1 - base < 32 ? e1 - base : 32);
    for (int t = 0; t < cnt; t += 4 * kSteps) {
      int it[kSteps];
      double wt[kSteps], v[kSteps][CPL];
#pragma unroll
      for (int h = 0; h < kSteps; ++h) {
        const int src = t + 4 * h + grp;
        it[h] = __shfl_sync(0xffffffffu, my_i, src & 31);
        wt[h] = __shfl_sync(0xffffffffu, my_w, src & 31);
        if (src >= cnt) wt[h] = 0.0;
      }
#pragma unroll
      for (int h = 0; h < kSteps; ++h) {
        const R* r = rows + ((int64_t)it[h] - row0) * l + q;
        const bool ok = t + 4 * h + grp < cnt;
#pragma unroll
        for (int k = 0; k < CPL; ++k) v[h][k] = (ok && q + 8 * k < l) ? (double)r[8 * k] : 0.0;
      }
#pragma unroll
      for (int h = 0; h < kSteps; ++h)
#pragma unroll
        for (int k = 0; k < CPL; ++k) acc[k] = fma(wt[h], v[h][k], acc[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < CPL; ++k) {
    acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], 8);
    acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], 16);
  }
  if (grp == 0) {
#pragma unroll
    for (int k = 0; k < CPL; ++k)
      if (q + 8 * k < l) out[q + 8 * k] = acc[k];
  }
  __syncwarp();
}

// Unweighted warp-cooperative gather for rows of l = 4 G FP32 values (16-byte aligned rows):
// out[c] = sum_{e in [e0, e1)} rows[idx_e - row0][c]. The warp takes kSumBatch entries at a
// time (lane t loads the index of entry t); the rows of the batch are then split over
// R = 32 / G row groups of G lanes, lane g of a group owning columns 4g .. 4g + 3, and each
// lane issues all its float4 loads of the batch (ceil(kSumBatch / R) rows) before it adds
// them. FP64 sums; the row groups are combined in a fixed order (deterministic) into out
// (shared memory of this warp). The batch is sized so that the kernels keep three CTAs of
// 256 threads per SM (registers) with 16 rows in flight per warp.
// With kWeighted, entry e's row is scaled by weight(e), a per-entry value loaded by the lane
// that loads the index and passed along with it. The indices and weights of the next batch
// are loaded while the current batch's rows are in flight, so a batch waits for one load
// latency, not two.
constexpr int kSumBatch = 16;
template <int G, bool kWeighted = false, typename Wt = double (*)(int64_t)>
__device__ __forceinline__ void sum_rows4(int64_t e0, int64_t e1, const int32_t* __restrict__ idx,
                                          const float* __restrict__ rows, int64_t row0, double* out,
                                          Wt weight = nullptr) {
  // batch size by row width, so that the kernels stay within three CTAs an SM without
  // spilling: rows of up to 20 values take 24 entries a batch (18 weighted), 24-32 values 16
  // (12), 36-64 values 12 (9)
  constexpr int B = G >= 9 ? (kWeighted ? 9 : 12) : G >= 6 ? (kWeighted ? 12 : kSumBatch) : (kWeighted ? 18 : 24),
                R = 32 / G, T = (B + R - 1) / R;
  const int lane = threadIdx.x & 31, grp = lane / G, cg = lane - grp * G;
  const bool active = grp < R;
  const float4* rows4 = reinterpret_cast<const float4*>(rows);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int32_t nxt = 0;
  double nxtw = 0.0;
  if (e0 + lane < e1) {
    nxt = idx[e0 + lane];
    if constexpr (kWeighted) nxtw = weight(e0 + lane);
  }
  for (int64_t base = e0; base < e1; base += B) {
    const int cnt = (int)(e1 - base < B ? e1 - base : B);
    const int64_t my = (int64_t)nxt - row0;
    const double myw = nxtw;
    float4 v[T];
    double w[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {  // every row load of the batch first
      const int src = grp + R * t;
      const int64_t ii = __shfl_sync(0xffffffffu, my, src & 31);
      v[t] = (active && src < cnt) ? __ldg(rows4 + ii * G + cg) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    nxt = 0;
    nxtw = 0.0;
    if (base + B + lane < e1) {  // the next batch's index and weight, in flight with the rows
      nxt = idx[base + B + lane];
      if constexpr (kWeighted) nxtw = weight(base + B + lane);
    }
    if constexpr (kWeighted) {
#pragma unroll
      for (int t = 0; t < T; ++t) w[t] = __shfl_sync(0xffffffffu, myw, (grp + R * t) & 31);
    }
#pragma unroll
    for (int t = 0; t < T; ++t) {
      if constexpr (kWeighted) {
        acc[0] = fma(w[t], (double)v[t].x, acc[0]);
        acc[1] = fma(w[t], (double)v[t].y, acc[1]);
        acc[2] = fma(w[t], (double)v[t].z, acc[2]);
        acc[3] = fma(w[t], (double)v[t].w, acc[3]);
      } else {
        acc[0] += (double)v[t].x;
        acc[1] += (double)v[t].y;
        acc[2] += (double)v[t].z;
        acc[3] += (double)v[t].w;
      }
    }
  }
  for (int g = 0; g < R; ++g) {
    if (active && grp == g)
#pragma unroll
      for (int j = 0; j < 4; ++j) out[4 * cg + j] = (g == 0 ? 0.0 : out[4 * cg + j]) + acc[j];
    __syncwarp();
  }
}

// out = sum of the rows for l % 4 == 0 and ceil(l / 8) = CPL, i.e. G = l / 4 = 2 CPL - 1 or
// 2 CPL (the two instantiations a kernel of that CPL can meet).
template <int CPL, bool kWeighted = false, typename Wt = double (*)(int64_t)>
__device__ __forceinline__ void sum_rows(int64_t e0, int64_t e1, const int32_t* __restrict__ idx,
                                         const float* __restrict__ rows, int64_t row0, int l, double* out,
                                         Wt weight = nullptr) {
  if ((l >> 2) == 2 * CPL)
    sum_rows4<2 * CPL, kWeighted>(e0, e1, idx, rows, row0, out, weight);
  else
    sum_rows4<(2 * CPL - 1 > 0 ? 2 * CPL - 1 : 1), kWeighted>(e0, e1, idx, rows, row0, out, weight);
}

// Warp per SNP of the window. Writes G (global rows), B2 (window-local rows, type T) and
// per-CTA partials of h0; with p.Gf also the FP32 rows the second gather reads (G, or
// s F G when no imputed values are set, which makes that gather unweighted), with p.qmax the
// column maxima of |B2| the int8 quantiser needs. The sparse gather reads the FP32 copy of
// Omega when p.omega_f is set (half the L2 bytes of the FP64 rows); without imputed values
// its weight is F_j for every entry, so it sums the rows unweighted (sum_rows, l % 4 == 0).
// kMode picks the sparse gather at compile time, so that each form keeps its own register
// budget: 0 = the generic 8-lane-group gather (any l, FP64 or FP32 rows; weighted when
// imputed values are set), 1 = unweighted float4 row sums (no imputed values, FP32 rows,
// l % 4 == 0), 2 = weighted float4 row sums (imputed values, FP32 rows, l % 4 == 0).
template <typename T, int CPL, int kMode>
__global__ void __launch_bounds__(256, CPL <= 5 ? 3 : 2) k_prep(EpiP1 p, const T* __restrict__ D1, T* __restrict__ B2,
                       double* __restrict__ h0_part) {
  extern __shared__ double sh0[];  // warps x l partial h0, then warps x l sparse sums
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double* ssp = sh0 + nwarps * p.l + warp * p.l;
  unsigned long long* smax = (unsigned long long*)(sh0 + 2 * nwarps * p.l);  // l column maxima
  for (int c = lane; c < p.l; c += 32) sh0[warp * p.l + c] = 0.0;
  if (p.qmax) {
    for (int c = threadIdx.x; c < p.l; c += blockDim.x) smax[c] = 0ull;
    __syncthreads();
  }
  const int64_t wl = p.wlen ? p.wlen : p.m, d1ws = p.d1_ws ? p.d1_ws : p.m, b2ws = p.b2_ws ? p.b2_ws : p.m;
  const int64_t d1rows = p.d1_rows ? p.d1_rows : p.m;
  for (int64_t jl = (int64_t)blockIdx.x * nwarps + warp; jl < p.m; jl += (int64_t)gridDim.x * nwarps) {
    const int64_t j = p.start + jl;
    const int64_t wi = jl / wl, r = jl - wi * wl, d1row = wi * d1ws + r, b2row = wi * b2ws + r;
    const double F = p.F[j];
    const double s = p.scale[j];
    const int64_t e0 = p.miss_ptr[j], e1 = p.miss_ptr[j + 1];
    const double* mv = p.miss_val;
    auto w = [&](int64_t e, int) { return (mv ? mv[e] : 0.0) + F; };
    constexpr bool plain = kMode == 1;
    if constexpr (kMode == 1)
      sum_rows<CPL>(e0, e1, p.miss_idx, p.omega_f, 0, p.l, ssp);
    else if constexpr (kMode == 2)
      sum_rows<CPL, true>(e0, e1, p.miss_idx, p.omega_f, 0, p.l, ssp, [&](int64_t e) { return mv[e] + F; });
    else if (p.omega_f)
      gather_rows<CPL>(e0, e1, p.miss_idx, p.omega_f, 0, p.l, w, ssp);
    else
      gather_rows<CPL>(e0, e1, p.miss_idx, p.omega, 0, p.l, w, ssp);
    for (int c = lane; c < p.l; c += 32) {
      double d = 0.0;
      for (int sp = 0; sp < p.ksplit; ++sp) d += (double)D1[((int64_t)sp * d1rows + d1row) * p.l + c];
      const double sparse = plain ? F * ssp[c] : ssp[c];
      double g = s * (0.5 * d - F * p.wsum[c] + sparse);
      p.G[j * p.l + c] = g;
      if (p.Gf) p.Gf[jl * p.l + c] = (float)(mv ? g : s * F * g);
      const T b2 = (T)(0.5 * s * g);
      if (p.qmax) atomicMax(&smax[c], (unsigned long long)__double_as_longlong(fabs((double)b2)));
      if (p.bt2) {
        const float x = (float)b2;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const int64_t kp = tc_pos(jl);
        const int np = 2 * p.bt_half;
        p.bt2[bt_elem(c, kp, np)] = hi;
        p.bt2[bt_elem(p.bt_half + c, kp, np)] = __float2bfloat16_rn(x - __bfloat162float(hi));
      } else {
        B2[b2row * p.l + c] = b2;
      }
      sh0[warp * p.l + c] += s * F * g;
    }
    __syncwarp();  // ssp is rewritten for the next SNP
  }
  if (p.bt2) {  // positions m..kpad2 of the split operand: zero (a shorter window follows a longer one)
    const int64_t tail = p.kpad2 - p.m, tot = tail * 2 * p.l;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
      const int64_t r = t / tail, jl = p.m + (t - r * tail);
      const int row = (int)(r < p.l ? r : p.bt_half + (r - p.l));
      p.bt2[bt_elem(row, tc_pos(jl), 2 * p.bt_half)] = __float2bfloat16_rn(0.0f);
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < p.l; c += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < nwarps; ++w) acc += sh0[w * p.l + c];
    h0_part[(int64_t)blockIdx.x * p.l + c] = acc;
    if (p.qmax && smax[c]) atomicMax(&p.qmax[c], smax[c]);
  }
}

// B2_j = s_j/2 G_j and per-CTA partials of h0 = sum_j s_j F_j G_j, for a given G.
template <typename T>
__global__ void k_scale_g(int64_t start, int64_t m, int l, const double* __restrict__ scale,
                          const double* __restrict__ F, const double* __restrict__ G,
                          T* __restrict__ B2, double* __restrict__ h0_part) {
  extern __shared__ double sh0[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int c = lane; c < l; c += 32) sh0[warp * l + c] = 0.0;
  for (int64_t jl = (int64_t)blockIdx.x * nwarps + warp; jl < m; jl += (int64_t)gridDim.x * nwarps) {
    const int64_t j = start + jl;
    const double f = F[j], s = scale[j];
    for (int c = lane; c < l; c += 32) {
      const double g = G[j * l + c];
      B2[jl * l + c] = (T)(0.5 * s * g);
      sh0[warp * l + c] += s * f * g;
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < l; c += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < nwarps; ++w) acc += sh0[w * l + c];
    h0_part[(int64_t)blockIdx.x * l + c] = acc;
  }
}

// out[c] = sum_b part[b][c]: one CTA of kRedThreads per column; thread t sums the rows
// t, t + kRedThreads, ... (eight loads in flight), then a fixed shuffle tree and a fixed
// combination of the warps' sums (deterministic).
constexpr int kRedThreads = 128;
__global__ void __launch_bounds__(kRedThreads) k_reduce_cols(const double* __restrict__ part, int nblk, int l,
                                                             double* __restrict__ out) {
  __shared__ double ws[kRedThreads / 32];
  const int c = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int b = threadIdx.x + u * kRedThreads;
    v[u] = b < nblk ? part[(int64_t)b * l + c] : 0.0;
  }
  double t = 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) t += v[u];
  for (int b = threadIdx.x + 8 * kRedThreads; b < nblk; b += kRedThreads) t += part[(int64_t)b * l + c];
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) ws[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) acc += ws[w];
    out[c] = acc;
  }
}

// Warp per sample: H[i] += sum_split D2 - h0 + sparse, the sparse term over the sample's
// missing entries in the windows [b0, b1).
template <typename T, int CPL, int kMode>
__global__ void __launch_bounds__(256, CPL <= 5 ? 3 : 2) k_accum(EpiP2 p, const T* __restrict__ D2) {
  extern __shared__ double ssm[];  // warps x l sparse sums
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double* ssp = ssm + warp * p.l;
  for (int64_t i = (int64_t)blockIdx.x * nwarps + warp; i < p.n; i += (int64_t)gridDim.x * nwarps) {
    const int64_t e0 = p.miss_ptr[i * p.nwin + p.b0], e1 = p.miss_ptr[i * p.nwin + p.b1];
    const double* mv = p.miss_val;
    const double *sc = p.scale, *F = p.F, *mw = p.miss_w;
    auto w = [&](int64_t e, int j) { return mw ? mw[e] : sc[j] * ((mv ? mv[e] : 0.0) + F[j]); };
    if constexpr (kMode == 1)  // Gf holds s F G: the sparse term is a plain row sum
      sum_rows<CPL>(e0, e1, p.miss_idx, p.Gf, p.g_start, p.l, ssp);
    else if constexpr (kMode == 2)
      sum_rows<CPL, true>(e0, e1, p.miss_idx, p.Gf, p.g_start, p.l, ssp, [&](int64_t e) { return mw[e]; });
    else if (p.Gf && !mv)
      gather_rows<CPL>(e0, e1, p.miss_idx, p.Gf, p.g_start, p.l, [](int64_t, int) { return 1.0; }, ssp);
    else if (p.Gf)
      gather_rows<CPL>(e0, e1, p.miss_idx, p.Gf, p.g_start, p.l, w, ssp);
    else
      gather_rows<CPL>(e0, e1, p.miss_idx, p.G, 0, p.l, w, ssp);
    for (int c = lane; c < p.l; c += 32) {
      double d = 0.0;
      for (int sp = 0; sp < p.ksplit; ++sp) d += (double)D2[((int64_t)sp * p.n + i) * p.l + c];
      const double sparse = ssp[c];
      p.H[i * p.l + c] += d - p.h0[c] + sparse;
    }
    __syncwarp();  // ssp is rewritten for the next row
  }
}

// CTAs of `threads` threads that fit on one SM at once for kernel fn with `smem` dynamic
// shared memory (at least 1): the grid-stride epilogues launch exactly one resident wave.
int resident_ctas(const void* fn, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    n = 1;
  }
  return std::max(1, n);
}

}  // namespace

template <typename T>
void launch_prep(pcaone_ctx* c, const EpiP1& p, const T* D1, T* B2, double* h0) {
  const int threads = 256, nwarps = threads / 32;
  const size_t smem = (size_t)2 * nwarps * p.l * 8 + (size_t)p.l * 8;
  const int mode = (p.omega_f && (p.l & 3) == 0) ? (p.miss_val ? 2 : 1) : 0;
  auto go = [&](auto kern) {
    const int per_sm = resident_ctas((const void*)kern, threads, smem);
    const int nblk = (int)std::min<int64_t>((int64_t)per_sm * c->sm_count,
                                            std::max<int64_t>(1, (p.m + nwarps - 1) / nwarps));
    double* part = (double*)scratch(c, "h0_part", (size_t)nblk * p.l * 8);
    kern<<<nblk, threads, smem, c->stream>>>(p, D1, B2, part);
    PG_CHECK_LAUNCH();
    k_reduce_cols<<<p.l, kRedThreads, 0, c->stream>>>(part, nblk, p.l, h0);
  };
  switch ((p.l + 7) / 8) {
    case 1: mode == 1 ? go(k_prep<T, 1, 1>) : mode == 2 ? go(k_prep<T, 1, 2>) : go(k_prep<T, 1, 0>); break;
    case 2: mode == 1 ? go(k_prep<T, 2, 1>) : mode == 2 ? go(k_prep<T, 2, 2>) : go(k_prep<T, 2, 0>); break;
    case 3: mode == 1 ? go(k_prep<T, 3, 1>) : mode == 2 ? go(k_prep<T, 3, 2>) : go(k_prep<T, 3, 0>); break;
    case 4: mode == 1 ? go(k_prep<T, 4, 1>) : mode == 2 ? go(k_prep<T, 4, 2>) : go(k_prep<T, 4, 0>); break;
    case 5: mode == 1 ? go(k_prep<T, 5, 1>) : mode == 2 ? go(k_prep<T, 5, 2>) : go(k_prep<T, 5, 0>); break;
    case 6: mode == 1 ? go(k_prep<T, 6, 1>) : mode == 2 ? go(k_prep<T, 6, 2>) : go(k_prep<T, 6, 0>); break;
    case 7: mode == 1 ? go(k_prep<T, 7, 1>) : mode == 2 ? go(k_prep<T, 7, 2>) : go(k_prep<T, 7, 0>); break;
    default: mode == 1 ? go(k_prep<T, 8, 1>) : mode == 2 ? go(k_prep<T, 8, 2>) : go(k_prep<T, 8, 0>); break;
  }
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

template <typename T>
void launch_accum(pcaone_ctx* c, const EpiP2& p, const T* D2) {
  const int threads = 256, nwarps = threads / 32;
  const size_t smem = (size_t)nwarps * p.l * 8;
  // the weighted row sums read the per-entry weights p.miss_w; without them the generic gather
  const int mode = (p.Gf && (p.l & 3) == 0) ? (p.miss_val ? (p.miss_w ? 2 : 0) : 1) : 0;
  auto go = [&](auto kern) {
    const int per_sm = resident_ctas((const void*)kern, threads, smem);
    const int nblk = (int)std::min<int64_t>((int64_t)per_sm * c->sm_count, (p.n + nwarps - 1) / nwarps);
    kern<<<nblk, threads, smem, c->stream>>>(p, D2);
  };
  switch ((p.l + 7) / 8) {
    case 1: mode == 1 ? go(k_accum<T, 1, 1>) : mode == 2 ? go(k_accum<T, 1, 2>) : go(k_accum<T, 1, 0>); break;
    case 2: mode == 1 ? go(k_accum<T, 2, 1>) : mode == 2 ? go(k_accum<T, 2, 2>) : go(k_accum<T, 2, 0>); break;
    case 3: mode == 1 ? go(k_accum<T, 3, 1>) : mode == 2 ? go(k_accum<T, 3, 2>) : go(k_accum<T, 3, 0>); break;
    case 4: mode == 1 ? go(k_accum<T, 4, 1>) : mode == 2 ? go(k_accum<T, 4, 2>) : go(k_accum<T, 4, 0>); break;
    case 5: mode == 1 ? go(k_accum<T, 5, 1>) : mode == 2 ? go(k_accum<T, 5, 2>) : go(k_accum<T, 5, 0>); break;
    case 6: mode == 1 ? go(k_accum<T, 6, 1>) : mode == 2 ? go(k_accum<T, 6, 2>) : go(k_accum<T, 6, 0>); break;
    case 7: mode == 1 ? go(k_accum<T, 7, 1>) : mode == 2 ? go(k_accum<T, 7, 2>) : go(k_accum<T, 7, 0>); break;
    default: mode == 1 ? go(k_accum<T, 8, 1>) : mode == 2 ? go(k_accum<T, 8, 2>) : go(k_accum<T, 8, 0>); break;
  }
  PG_CHECK_LAUNCH();
  c->launches++;
}

template <typename T>
void launch_scale_g(pcaone_ctx* c, const EpiP1& p, T* B2, double* h0) {
  const int threads = 256, nwarps = threads / 32;
  int nblk = (int)std::min<int64_t>(4 * c->sm_count, std::max<int64_t>(1, (p.m + nwarps - 1) / nwarps));
  double* part = (double*)scratch(c, "h0_part", (size_t)nblk * p.l * 8);
  k_scale_g<T><<<nblk, threads, (size_t)nwarps * p.l * 8, c->stream>>>(p.start, p.m, p.l, p.scale,
                                                                       p.F, p.G, B2, part);
  PG_CHECK_LAUNCH();
  k_reduce_cols<<<p.l, kRedThreads, 0, c->stream>>>(part, nblk, p.l, h0);
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

void zero(pcaone_ctx* c, double* a, int64_t n) {
  PG_CUDA(cudaMemsetAsync(a, 0, n * sizeof(double), c->stream));
}

template void launch_prep<float>(pcaone_ctx*, const EpiP1&, const float*, float*, double*);
template void launch_prep<double>(pcaone_ctx*, const EpiP1&, const double*, double*, double*);
template void launch_scale_g<float>(pcaone_ctx*, const EpiP1&, float*, double*);
template void launch_scale_g<double>(pcaone_ctx*, const EpiP1&, double*, double*);
template void launch_accum<float>(pcaone_ctx*, const EpiP2&, const float*);
template void launch_accum<double>(pcaone_ctx*, const EpiP2&, const double*);

}  // namespace pg
