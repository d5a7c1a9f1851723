// Gram products of tall row-major matrices (A^T B, n x la and n x lb, or the symmetric A^T A)
// for the sketch-width kernels: register tiles, thread groups over rows, and a deterministic
// two-level reduction (8-CTA clusters through distributed shared memory, then one CTA over
// the cluster sums).
#pragma once

#include <cooperative_groups.h>

#include "internal.hpp"

namespace pg {

namespace cg = cooperative_groups;

constexpr int kGramCluster = 8;    // CTAs per cluster of the Gram kernels
constexpr int kGramMaxParts = 36;  // cluster sums read at once by the final reductions

// The la4 x lb4 output (widths rounded up to 4) is cut into 4 x 4 tiles; a symmetric product
// keeps the tiles on and above the diagonal. The CTA's threads form ngrp groups of ntiles
// threads; group g adds the staged rows g, g + ngrp, ... into its tiles.
struct GramTiling {
  int la4, lb4, nbi, nbj, ntiles, ngrp;
  bool sym;
};

__host__ __device__ inline GramTiling gram_tiling(int la, int lb, bool sym, int threads) {
  GramTiling g;
  g.la4 = (la + 3) & ~3;
  g.lb4 = (lb + 3) & ~3;
  g.nbi = g.la4 / 4;
  g.nbj = g.lb4 / 4;
  g.sym = sym;
  g.ntiles = sym ? g.nbi * (g.nbi + 1) / 2 : g.nbi * g.nbj;
  g.ngrp = threads / g.ntiles > 0 ? threads / g.ntiles : 1;
  return g;
}

// Tile index -> first row / column of the tile.
__device__ __forceinline__ void gram_tile_origin(const GramTiling& g, int tile, int& i0, int& j0) {
  int bi = 0, bj;
  if (g.sym) {
    int t = tile;
    while (t >= g.nbi - bi) {
      t -= g.nbi - bi;
      ++bi;
    }
    bj = bi + t;
  } else {
    bi = tile / g.nbj;
    bj = tile - bi * g.nbj;
  }
  i0 = bi * 4;
  j0 = bj * 4;
}

// Shared-memory doubles the Gram helpers need beside the staged rows: group sums and the
// CTA sum.
__host__ __device__ inline int gram_smem_doubles(const GramTiling& g) { return (g.ngrp + 1) * g.ntiles * 16; }

struct GramThread {
  int i0 = 0, j0 = 0, grp = 0, tile = 0;
  bool active = false;
  double acc[4][4];

  __device__ void init(const GramTiling& g) {
    tile = threadIdx.x % g.ntiles;
    grp = threadIdx.x / g.ntiles;
    active = grp < g.ngrp;
    gram_tile_origin(g, tile, i0, j0);
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
  }

  // sa: nr x la4, sb: nr x lb4 staged rows (columns past la / lb zero)
  __device__ void add_rows(const double* sa, const double* sb, int nr, const GramTiling& g) {
    if (!active) return;
    for (int r = grp; r < nr; r += g.ngrp) {
      const double2 a01 = *reinterpret_cast<const double2*>(sa + r * g.la4 + i0);
      const double2 a23 = *reinterpret_cast<const double2*>(sa + r * g.la4 + i0 + 2);
      const double2 b01 = *reinterpret_cast<const double2*>(sb + r * g.lb4 + j0);
      const double2 b23 = *reinterpret_cast<const double2*>(sb + r * g.lb4 + j0 + 2);
      const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(av[x], bv[y], acc[x][y]);
    }
  }

  // Keeping the tile in red (ngrp * ntiles * 16 doubles of shared memory) between batches
  // frees its registers for other work of the kernel: park() stores it, unpark() reloads it.
  __device__ void park(const GramTiling& g, double* red) const {
    if (!active) return;
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) red[(grp * g.ntiles + tile) * 16 + x * 4 + y] = acc[x][y];
  }
  __device__ void unpark(const GramTiling& g, const double* red) {
    if (!active) return;
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = red[(grp * g.ntiles + tile) * 16 + x * 4 + y];
  }

  // CTA sum of the groups' tiles (fixed group order) into out[ntiles * 16] (shared memory);
  // red holds ngrp * ntiles * 16 doubles.
  __device__ void finish(const GramTiling& g, double* red, double* out) {
    park(g, red);
    __syncthreads();
    const int n = g.ntiles * 16;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      double s = 0.0;
      for (int q = 0; q < g.ngrp; ++q) s += red[q * n + e];
      out[e] = s;
    }
    __syncthreads();
  }
};

// sum_{b < n} x[b * stride] in b order; W loads are issued before their adds.
template <int W = 8>
__device__ __forceinline__ double sum_strided(const double* x, int n, int64_t stride) {
  double s = 0.0;
  int b = 0;
  for (; b + W <= n; b += W) {
    double v[W];
#pragma unroll
    for (int k = 0; k < W; ++k) v[k] = x[(int64_t)(b + k) * stride];
#pragma unroll
    for (int k = 0; k < W; ++k) s += v[k];
  }
  for (; b < n; ++b) s += x[(int64_t)b * stride];
  return s;
}

// sum_{b < n} x[b * stride] in b order with every load issued before the adds (n <= WMAX);
// longer sums go to sum_strided.
template <int WMAX>
__device__ __forceinline__ double sum_all(const double* x, int n, int64_t stride) {
  if (n > WMAX) return sum_strided<16>(x, n, stride);
  double v[WMAX];
#pragma unroll
  for (int k = 0; k < WMAX; ++k) v[k] = k < n ? x[(int64_t)k * stride] : 0.0;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < WMAX; ++k)
    if (k < n) s += v[k];
  return s;
}

// Cluster sum of the CTAs' part[n] (shared memory), in rank order, written to
// gout[cluster index * n + e]. Every CTA of the cluster calls it; the rank-r CTA sums the
// elements r * blockDim + t, ... through distributed shared memory. The second cluster barrier
// keeps each CTA's shared memory alive until the others have read it.
__device__ __forceinline__ void cluster_sum(const double* part, int n, double* gout) {
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  const int rank = (int)cl.block_rank();
  const int64_t cid = blockIdx.x / kGramCluster;
  for (int e = rank * blockDim.x + threadIdx.x; e < n; e += kGramCluster * blockDim.x) {
    double v[kGramCluster];
#pragma unroll
    for (int q = 0; q < kGramCluster; ++q) v[q] = cl.map_shared_rank(part, q)[e];
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kGramCluster; ++q) s += v[q];
    gout[cid * n + e] = s;
  }
  cl.sync();
}

// W (la x lb row-major, shared or global memory) = sum over nparts cluster sums of the tile
// layout in gpart; a symmetric product is mirrored below the diagonal.
__device__ __forceinline__ void gram_final(const GramTiling& g, const double* gpart, int nparts, int la, int lb,
                                           double* W) {
  const int n = g.ntiles * 16;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const double v = sum_all<kGramMaxParts>(gpart + e, nparts, n);
    int i0, j0;
    gram_tile_origin(g, e / 16, i0, j0);
    const int i = i0 + (e % 16) / 4, j = j0 + e % 4;
    if (i < la && j < lb) {
      W[i * lb + j] = v;
      if (g.sym) W[j * lb + i] = v;
    }
  }
  __syncthreads();
}

// Ticket: true in the CTA that finishes last (after a fence, so it sees every CTA's writes).
__device__ __forceinline__ bool last_cta(unsigned* counter) {
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

// One elimination step on the l x l matrix s (shared memory, row-major): for the rows
// a = j + 1, ..., l - 1 (a warp per row, eight rows a warp in flight) and the columns b > j
// (b >= a when upper; lanes over columns, two a lane for l <= 64),
//   s[a][b] -= (s[a][j] or s[j][a]) * inv * s[j][b],
// with the multiplier from column j (lu) or row j (upper). All loads of a batch of rows are
// issued before its stores, so the step costs about one shared-memory round trip.
template <bool kUpper>
__device__ __forceinline__ void elim_step(double* s, int l, int j, double inv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int b0 = lane, b1 = lane + 32;
  const double rj0 = (b0 > j && b0 < l) ? s[j * l + b0] : 0.0;
  const double rj1 = (b1 > j && b1 < l) ? s[j * l + b1] : 0.0;
  for (int a0 = j + 1 + warp; a0 < l; a0 += 8 * nw) {
    double f[8], v0[8], v1[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int a = a0 + k * nw;
      const bool ok = a < l;
      const int lo = kUpper ? a : j + 1;  // first column updated in row a
      f[k] = ok ? (kUpper ? s[j * l + a] : s[a * l + j]) * inv : 0.0;
      v0[k] = (ok && b0 >= lo && b0 < l) ? s[a * l + b0] : 0.0;
      v1[k] = (ok && b1 >= lo && b1 < l) ? s[a * l + b1] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int a = a0 + k * nw;
      if (a >= l) break;
      const int lo = kUpper ? a : j + 1;
      if (b0 >= lo && b0 < l) s[a * l + b0] = v0[k] - f[k] * rj0;
      if (b1 >= lo && b1 < l) s[a * l + b1] = v1[k] - f[k] * rj1;
    }
  }
}

// In-place Cholesky of the SPD l x l matrix in s (shared memory, row-major; the upper triangle
// is read; l <= 64): on return s holds the upper factor R (W = R^T R) with zeros below the
// diagonal. Right-looking with the row scaling deferred: step j subtracts
// s[j][a] s[j][b] / s[j][j] from the trailing upper triangle (elim_step; one reciprocal of the
// pivot a step), one barrier a step; row j is divided by sqrt(s[j][j]) at the end. A pivot
// that is not positive and finite is replaced by 1. Returns 1 + the first such column, else 0
// (the same in every thread).
__device__ __forceinline__ int chol_upper_smem(double* s, int l) {
  int bad = 0;
  __syncthreads();
  for (int j = 0; j < l; ++j) {
    double p = s[j * l + j];
    if (!(p > 0.0) || !isfinite(p)) {
      if (!bad) bad = j + 1;
      p = 1.0;
    }
    elim_step<true>(s, l, j, __drcp_rn(p));
    __syncthreads();
  }
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) {  // off-diagonal first: diagonals still pivots
    const int i = t / l, j = t - i * l;
    if (j > i) {
      const double p = s[i * l + i];
      s[t] /= (p > 0.0 && isfinite(p)) ? sqrt(p) : 1.0;
    } else if (j < i) {
      s[t] = 0.0;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < l; i += blockDim.x) {
    const double p = s[i * l + i];
    s[i * l + i] = (p > 0.0 && isfinite(p)) ? sqrt(p) : 1.0;
  }
  __syncthreads();
  return bad;
}

// Householder column signs D (l) from the modified LU of the l x l block T (shared memory,
// overwritten; l <= 64): step i takes the pivot s = T[i][i], D_i = -sign(s) with
// sign(0) = +, and eliminates below it with the shifted pivot s - D_i (Ballard et al. 2015);
// the multipliers T[r][i] / (s - D_i) are used, not stored. One barrier a step. D is
// written by thread 0 and visible to the CTA on return.
__device__ __forceinline__ void householder_signs_smem(double* T, int l, double* D) {
  __syncthreads();
  for (int i = 0; i < l; ++i) {
    const double piv = T[i * l + i];
    const double di = piv >= 0.0 ? -1.0 : 1.0;
    if (threadIdx.x == 0) D[i] = di;
    elim_step<false>(T, l, i, __drcp_rn(piv - di));
    __syncthreads();
  }
}

// Clusters of kGramCluster CTAs of kernel (threads, smem bytes) that fit on the device at
// once, cached in the context by (kernel, key); 0 when the runtime cannot tell.
inline int resident_clusters(pcaone_ctx* c, const void* kernel, uint64_t key, int threads, size_t smem) {
  const auto k = std::make_pair(kernel, key);
  auto it = c->cluster_occupancy.find(k);
  if (it != c->cluster_occupancy.end()) return it->second;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kGramCluster * 64);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kGramCluster;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    n = 0;
  }
  c->cluster_occupancy[k] = n;
  return n;
}

// Row range of this CTA when n rows are split over the grid in contiguous blocks.
__device__ __forceinline__ void row_range(int64_t n, int64_t& r0, int64_t& r1) {
  const int64_t rpb = (n + gridDim.x - 1) / gridDim.x;
  r0 = blockIdx.x * rpb;
  r1 = (n < r0 + rpb ? n : r0 + rpb);
  if (r0 > r1) r0 = r1;
}

}  // namespace pg
