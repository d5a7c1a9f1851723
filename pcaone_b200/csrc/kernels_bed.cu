// Device-side PLINK genotype handling: padding, integer allele counts, SNP permutation,
// the sample-major (transposed) packed copy per window, and the sparse lists of missing
// entries. Replaces FileBed::read_all (src/FilePlink.cpp:29-131) and the in-core column
// permutation permute_matrix (src/RSVD.hpp:63-79).
//
// Packed code of sample j in a SNP record: bits 2*(j%4) of byte j/4 (LSB first);
// 00 = two A1 copies, 10 = one, 11 = none, 01 = missing (src/Common.hpp:49-58).
// Padding (samples >= N inside the last byte, bytes beyond the record, rows beyond M) is set
// to code 11, which decodes to zero and is never counted as missing.
#include <numeric>

#include "internal.hpp"

namespace pg {

namespace {

__global__ void k_fix_padding(uint8_t* bed, uint64_t M, uint32_t bpr, uint32_t pitch, uint32_t N) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= M) return;
  uint32_t r = N & 3u;
  if (r) bed[j * pitch + bpr - 1] |= (uint8_t)(0xFFu << (2 * r));
}

// Warp per SNP record. n00 = code 00 (two A1), n10 = code 10 (het), n01 = code 01 (missing).
__global__ void k_counts(const uint8_t* __restrict__ bed, uint64_t M, uint32_t pitch, uint32_t N,
                         uint32_t* __restrict__ a1x2, uint32_t* __restrict__ nonmiss) {
  uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (j >= M) return;
  const uint32_t* row = reinterpret_cast<const uint32_t*>(bed + j * pitch);
  uint32_t nwords = pitch >> 2;
  uint32_t c00 = 0, c10 = 0, c01 = 0;
  for (uint32_t w = lane; w < nwords; w += 32) {
    uint32_t x = __ldg(row + w);
    uint32_t b0 = x & 0x55555555u, b1 = (x >> 1) & 0x55555555u;
    c00 += __popc(~(b0 | b1) & 0x55555555u);
    c10 += __popc(b1 & ~b0);
    c01 += __popc(b0 & ~b1);
  }
  for (int o = 16; o; o >>= 1) {
    c00 += __shfl_xor_sync(0xffffffffu, c00, o);
    c10 += __shfl_xor_sync(0xffffffffu, c10, o);
    c01 += __shfl_xor_sync(0xffffffffu, c01, o);
  }
  if (lane == 0) {
    a1x2[j] = 2 * c00 + c10;
    nonmiss[j] = N - c01;
  }
}

// F_j = (sum of {1, 0.5, 0} over non-missing) / count, with the FP64 sum formed exactly as
// (a1x2 * 0.5) so the division reproduces the reference bit-for-bit (src/FilePlink.cpp:53-56).
__global__ void k_freq(const uint32_t* a1x2, const uint32_t* nonmiss, uint64_t M, double* F) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= M) return;
  uint32_t c = nonmiss[j];
  F[j] = c == 0 ? 0.0 : ((double)a1x2[j] * 0.5) / (double)c;
}

// out row j = in row perm[j]; 16-byte copies (pitch is a multiple of 64).
__global__ void k_permute(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                          const int32_t* __restrict__ perm, uint64_t M, uint32_t pitch) {
  uint64_t j = blockIdx.y * (uint64_t)gridDim.x + blockIdx.x;
  if (j >= M) return;
  const uint4* src = reinterpret_cast<const uint4*>(in + (uint64_t)perm[j] * pitch);
  uint4* dst = reinterpret_cast<uint4*>(out + j * pitch);
  for (uint32_t t = threadIdx.x; t < pitch / 16; t += blockDim.x) dst[t] = src[t];
}

// Sample-major packed copy of one 64 SNP x 64 sample tile of window `b`.
// grid = (snp tiles per window, Npad / 64, bands), block = 256.
__global__ void k_transpose(const uint8_t* __restrict__ bed, uint32_t pitch, uint64_t M,
                            uint64_t blocksize, uint8_t* __restrict__ bedT, uint32_t pitchT,
                            uint32_t Npad) {
  __shared__ uint8_t tile[64][17];
  const uint32_t b = blockIdx.z;
  const uint64_t w0 = (uint64_t)b * blocksize;
  const uint64_t w1 = min((uint64_t)(b + 1) * blocksize, M);
  const uint64_t jl0 = (uint64_t)blockIdx.x * 64;  // local SNP offset inside the window
  if (w0 + jl0 >= w1) return;
  const uint32_t i0 = blockIdx.y * 64;  // first sample
  // load 64 SNP rows x 16 bytes (64 samples)
  for (int t = threadIdx.x; t < 64 * 16; t += blockDim.x) {
    int r = t >> 4, cb = t & 15;
    uint64_t j = w0 + jl0 + r;
    tile[r][cb] = (j < w1) ? bed[j * pitch + (i0 >> 2) + cb] : (uint8_t)0xFF;
  }
  __syncthreads();
  // each thread: one output word = 16 SNPs of one sample
  const int si = threadIdx.x >> 2, wq = threadIdx.x & 3;
  uint32_t word = 0;
#pragma unroll
  for (int t = 0; t < 16; ++t) {
    uint32_t code = (tile[wq * 16 + t][si >> 2] >> (2 * (si & 3))) & 3u;
    word |= code << (2 * t);
  }
  uint8_t* dst = bedT + ((uint64_t)b * Npad + i0 + si) * pitchT + (jl0 >> 2) + wq * 4;
  *reinterpret_cast<uint32_t*>(dst) = word;
}

// Warp per packed row: count missing codes (01) in a row of `nbytes` bytes.
// CSR row of packed row r: r itself (by-SNP list, nwin = 0), or for the (window, sample)
// list, where packed row r = b * npad + i, the sample-major row i * nwin + b, so that the
// entries of sample i over a run of consecutive windows [b0, b1) are one contiguous range.
__device__ __forceinline__ uint64_t csr_row(uint64_t r, uint32_t npad, uint32_t nwin) {
  return nwin ? (r % npad) * nwin + r / npad : r;
}

__global__ void k_count_missing_rows(const uint8_t* __restrict__ base, uint32_t pitch, uint64_t nrows,
                                     uint32_t nwords, uint32_t npad, uint32_t nwin, int64_t* __restrict__ cnt) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (r >= nrows) return;
  const uint32_t* row = reinterpret_cast<const uint32_t*>(base + r * pitch);
  uint32_t n = 0;
  for (uint32_t w = lane; w < nwords; w += 32) {
    uint32_t x = row[w];
    n += __popc((x & 0x55555555u) & ~((x >> 1) & 0x55555555u));
  }
  for (int o = 16; o; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) cnt[csr_row(r, npad, nwin)] = n;
}

// ---- exclusive prefix sum of int64 counts on the device (CSR row pointers): per 1024-element
// block a shuffle scan, then one block scans the block totals, then the offsets are added.
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock) k_scan_local(const int64_t* __restrict__ cnt, uint64_t n,
                                                           int64_t* __restrict__ ptr, int64_t* __restrict__ bsum) {
  __shared__ int64_t wsum[32];
  const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t v = i < n ? cnt[i] : 0;
  int64_t x = v;  // inclusive scan within the warp
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t t = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    wsum[lane] = t;
  }
  __syncthreads();
  const int64_t excl = (w > 0 ? wsum[w - 1] : 0) + x - v;
  if (i < n) ptr[i] = excl;
  if (threadIdx.x == kScanBlock - 1) bsum[blockIdx.x] = excl + v;
}

// In place exclusive scan of nb block totals (one block); bsum[nb] = the grand total.
__global__ void __launch_bounds__(kScanBlock) k_scan_bsums(int64_t* bsum, int64_t nb) {
  __shared__ int64_t part[kScanBlock];
  const int64_t per = (nb + kScanBlock - 1) / kScanBlock;
  const int64_t b0 = threadIdx.x * per, b1 = b0 + per < nb ? b0 + per : nb;
  int64_t s = 0;
  for (int64_t b = b0; b < b1; ++b) s += bsum[b];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t run = 0;
    for (int t = 0; t < kScanBlock; ++t) {
      const int64_t v = part[t];
      part[t] = run;
      run += v;
    }
    bsum[nb] = run;
  }
  __syncthreads();
  int64_t run = part[threadIdx.x];
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = bsum[b];
    bsum[b] = run;
    run += v;
  }
}

__global__ void k_scan_add(int64_t* __restrict__ ptr, uint64_t n, const int64_t* __restrict__ bsum, int64_t nb) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ptr[i] += bsum[i / kScanBlock];
  if (i == 0) ptr[n] = bsum[nb];
}

// counts of missing codes per SNP from the non-missing counts
__global__ void k_missing_counts(const uint32_t* __restrict__ nonmiss, uint64_t M, uint32_t N,
                                 int64_t* __restrict__ cnt) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < M) cnt[j] = (int64_t)(N - nonmiss[j]);
}

// Warp per packed row: write the positions of missing codes in increasing order.
// idx_out[ptr[csr_row(r)] + t] = pos_offset(r) + position. pos_base is added to every
// position; for the (window, sample) lists, row r = b * Npad + i and pos_base = window start
// of b (rows_per_base = npad).
__global__ void k_fill_missing_rows(const uint8_t* __restrict__ base, uint32_t pitch,
                                    uint64_t nrows, uint32_t nwords,
                                    const int64_t* __restrict__ ptr, int32_t* __restrict__ idx,
                                    const uint64_t* __restrict__ row_pos_base, uint32_t rows_per_base,
                                    uint32_t nwin) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (r >= nrows) return;
  const uint32_t* row = reinterpret_cast<const uint32_t*>(base + r * pitch);
  int64_t out = ptr[csr_row(r, rows_per_base, nwin)];
  uint64_t pbase = row_pos_base ? row_pos_base[r / rows_per_base] : 0;
  for (uint32_t w0 = 0; w0 < nwords; w0 += 32) {
    uint32_t w = w0 + lane;
    uint32_t m = 0;
    if (w < nwords) {
      uint32_t x = row[w];
      m = (x & 0x55555555u) & ~((x >> 1) & 0x55555555u);
    }
    uint32_t n = __popc(m);
    uint32_t incl = n;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    int64_t pos = out + incl - n;
    while (m) {
      int bit = __ffs(m) - 1;
      idx[pos++] = (int32_t)(pbase + (uint64_t)w * 16 + (bit >> 1));
      m &= m - 1;
    }
    out += total;
  }
}

}  // namespace

void launch_fix_padding(pcaone_ctx* c) {
  if ((c->N & 3u) == 0) return;
  k_fix_padding<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(c->d_bed, c->M, c->bpr,
                                                                         c->pitch, c->N);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void launch_counts(pcaone_ctx* c) {
  uint64_t threads = c->M * 32;
  k_counts<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(c->d_bed, c->M, c->pitch, c->N,
                                                                      c->d_a1x2, c->d_nonmiss);
  PG_CHECK_LAUNCH();
  k_freq<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(c->d_a1x2, c->d_nonmiss, c->M, c->d_F);
  PG_CHECK_LAUNCH();
  c->launches += 2;
}

void launch_permute(pcaone_ctx* c, const int32_t* d_perm, uint8_t* d_out) {
  dim3 grid((unsigned)std::min<uint64_t>(c->M, 65535), (unsigned)((c->M + 65534) / 65535));
  k_permute<<<grid, 128, 0, c->stream>>>(c->d_bed, d_out, d_perm, c->M, c->pitch);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// ---- launchers for streamed genotypes: the same kernels on rows staged in a device slot
void launch_counts_rows(pcaone_ctx* c, cudaStream_t st, const uint8_t* rows, uint64_t nrows, uint64_t row0) {
  const uint64_t threads = nrows * 32;
  k_counts<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(rows, nrows, c->pitch, c->N, c->d_a1x2 + row0,
                                                               c->d_nonmiss + row0);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void launch_freq(pcaone_ctx* c) {
  k_freq<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(c->d_a1x2, c->d_nonmiss, c->M, c->d_F);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// Sample-major copies of nwin consecutive windows of the current layout whose nsnp records
// start at rec (the first window at rec); recT: nwin x Npad x win.pitch.
void launch_transpose_run(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, uint64_t nsnp, int nwin,
                          uint8_t* recT) {
  PG_CUDA(cudaMemsetAsync(recT, 0xFF, (size_t)nwin * c->Npad * c->win.pitch, st));
  dim3 grid((unsigned)((c->win.blocksize + 63) / 64), c->Npad / 64, (unsigned)nwin);
  k_transpose<<<grid, 256, 0, st>>>(rec, c->pitch, nsnp, c->win.blocksize, recT, c->win.pitch, c->Npad);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// By-SNP missing entries of the staged records of SNPs row0 .. row0 + nrows (row pointers set).
void launch_missing_snp_rows(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, uint64_t nrows, uint64_t row0) {
  const uint64_t threads = nrows * 32;
  k_fill_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      rec, c->pitch, nrows, c->pitch / 4, c->d_miss_snp_ptr + row0, c->d_miss_snp_idx, nullptr, 1, 0);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// (window, sample) missing counts / entries of the staged sample-major copies of the windows
// b0 .. b0 + nw: row r of the copies is sample r % Npad of window b0 + r / Npad, whose CSR row
// (i * bands + b) is reached by offsetting the count / pointer array by b0.
void launch_missing_ws_count(pcaone_ctx* c, cudaStream_t st, const uint8_t* recT, int b0, int nw, int64_t* cnt) {
  const uint64_t rows = (uint64_t)nw * c->Npad, threads = rows * 32;
  k_count_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      recT, c->win.pitch, rows, c->win.pitch / 4, c->Npad, (uint32_t)c->win.bands, cnt + b0);
  PG_CHECK_LAUNCH();
  c->launches++;
}

void launch_missing_ws_fill(pcaone_ctx* c, cudaStream_t st, const uint8_t* recT, int b0, int nw,
                            const uint64_t* d_base) {
  const uint64_t rows = (uint64_t)nw * c->Npad, threads = rows * 32;
  k_fill_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      recT, c->win.pitch, rows, c->win.pitch / 4, c->d_miss_ws_ptr + b0, c->d_miss_ws_idx, d_base + b0, c->Npad,
      (uint32_t)c->win.bands);
  PG_CHECK_LAUNCH();
  c->launches++;
}

// bands windows of blocksize SNPs; blocksize 0 = ceil(M / bands) (src/Halko.cpp:178), else the
// blocks of the out-of-core plan (src/Data.cpp:56-71, bands = ceil(M / blocksize)).
static WindowLayout make_layout(pcaone_ctx* c, int bands, uint64_t blocksize) {
  WindowLayout w;
  w.bands = bands;
  w.blocksize = blocksize ? blocksize : (uint64_t)std::ceil((double)c->M / bands);
  PG_REQUIRE(w.blocksize > 0, PCAONE_EBADARG, "empty windows");
  w.pitch = (uint32_t)round_up((w.blocksize + 3) / 4, kPitchAlign);
  for (int b = 0; b < bands; ++b) {
    uint64_t s = (uint64_t)b * w.blocksize;
    uint64_t e = std::min<uint64_t>((uint64_t)(b + 1) * w.blocksize, c->M);
    PG_REQUIRE(s < e, PCAONE_EBADARG,
               "window " + std::to_string(b) + " is empty: fewer SNPs than windows");
    w.start.push_back(s);
    w.stop.push_back(e);
  }
  return w;
}

void set_window_layout(pcaone_ctx* c, int bands, uint64_t blocksize) {
  const uint64_t bs = blocksize ? blocksize : (uint64_t)std::ceil((double)c->M / bands);
  if (c->win.bands == bands && c->win.blocksize == bs && !c->win.start.empty()) return;
  c->win = make_layout(c, bands, blocksize);
  c->miss_ws_valid = false;
}

void build_empty_missing(pcaone_ctx* c) {
  const uint64_t rows = (uint64_t)c->win.bands * c->Npad;
  if (!c->miss_snp_valid) {
    c->d_miss_snp_ptr = (int64_t*)scratch(c, "d_miss_snp_ptr", (c->M + 1) * 8);
    c->d_miss_snp_idx = (int32_t*)scratch(c, "d_miss_snp_idx", 4);
    PG_CUDA(cudaMemsetAsync(c->d_miss_snp_ptr, 0, (c->M + 1) * 8, c->stream));
    c->n_missing = 0;
    c->miss_snp_valid = true;
  }
  if (!c->miss_ws_valid) {
    c->d_miss_ws_ptr = (int64_t*)scratch(c, "d_miss_ws_ptr", (rows + 1) * 8);
    c->d_miss_ws_idx = (int32_t*)scratch(c, "d_miss_ws_idx", 4);
    PG_CUDA(cudaMemsetAsync(c->d_miss_ws_ptr, 0, (rows + 1) * 8, c->stream));
    c->miss_ws_valid = true;
  }
}

void build_transposed(pcaone_ctx* c, int bands, uint64_t blocksize) {
  const uint64_t bs = blocksize ? blocksize : (uint64_t)std::ceil((double)c->M / bands);
  if (c->bedT_valid && c->win.bands == bands && c->win.blocksize == bs) return;
  WindowLayout w = make_layout(c, bands, blocksize);
  size_t bytes = (size_t)bands * c->Npad * w.pitch;
  c->d_bedT = (uint8_t*)scratch(c, "d_bedT", bytes);
  PG_CUDA(cudaMemsetAsync(c->d_bedT, 0xFF, bytes, c->stream));
  dim3 grid((unsigned)((w.blocksize + 63) / 64), c->Npad / 64, bands);
  k_transpose<<<grid, 256, 0, c->stream>>>(c->d_bed, c->pitch, c->M, w.blocksize, c->d_bedT,
                                           w.pitch, c->Npad);
  PG_CHECK_LAUNCH();
  c->launches++;
  c->win = w;
  c->bedT_valid = true;
  c->miss_ws_valid = false;
}

// ptr[0..n] = exclusive prefix sum of cnt[0..n) on the device; returns ptr[n].
static int64_t device_exclusive_scan(pcaone_ctx* c, const int64_t* cnt, uint64_t n, int64_t* ptr) {
  const int64_t nb = (int64_t)((n + kScanBlock - 1) / kScanBlock);
  int64_t* bsum = (int64_t*)scratch(c, "scan_bsum", (size_t)(nb + 1) * 8);
  k_scan_local<<<(unsigned)std::max<int64_t>(nb, 1), kScanBlock, 0, c->stream>>>(cnt, n, ptr, bsum);
  PG_CHECK_LAUNCH();
  k_scan_bsums<<<1, kScanBlock, 0, c->stream>>>(bsum, nb);
  PG_CHECK_LAUNCH();
  k_scan_add<<<(unsigned)((n + 255) / 256 + 1), 256, 0, c->stream>>>(ptr, n, bsum, nb);
  PG_CHECK_LAUNCH();
  c->launches += 3;
  int64_t total = 0;
  PG_CUDA(cudaMemcpyAsync(&total, ptr + n, 8, cudaMemcpyDeviceToHost, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  return total;
}

int64_t scan_counts(pcaone_ctx* c, const int64_t* cnt, uint64_t n, int64_t* ptr) {
  return device_exclusive_scan(c, cnt, n, ptr);
}

// Row pointers of the by-SNP list from the non-missing counts, and its index array (sized).
int64_t missing_snp_scan(pcaone_ctx* c) {
  int64_t* d_cnt = (int64_t*)scratch(c, "miss_snp_cnt", c->M * 8);
  k_missing_counts<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(c->d_nonmiss, c->M, c->N, d_cnt);
  PG_CHECK_LAUNCH();
  c->launches++;
  c->d_miss_snp_ptr = (int64_t*)scratch(c, "d_miss_snp_ptr", (c->M + 1) * 8);
  c->n_missing = device_exclusive_scan(c, d_cnt, c->M, c->d_miss_snp_ptr);
  c->d_miss_snp_idx = (int32_t*)scratch(c, "d_miss_snp_idx", std::max<int64_t>(c->n_missing, 1) * 4);
  return c->n_missing;
}

void build_missing_by_snp(pcaone_ctx* c) {
  if (c->miss_snp_valid) return;
  if (c->streamed) {
    stream_missing_snp(c);
    return;
  }
  int64_t* d_cnt = (int64_t*)scratch(c, "miss_snp_cnt", c->M * 8);
  k_missing_counts<<<(unsigned)((c->M + 255) / 256), 256, 0, c->stream>>>(c->d_nonmiss, c->M, c->N, d_cnt);
  PG_CHECK_LAUNCH();
  c->d_miss_snp_ptr = (int64_t*)scratch(c, "d_miss_snp_ptr", (c->M + 1) * 8);
  c->n_missing = device_exclusive_scan(c, d_cnt, c->M, c->d_miss_snp_ptr);
  c->d_miss_snp_idx = (int32_t*)scratch(c, "d_miss_snp_idx", std::max<int64_t>(c->n_missing, 1) * 4);
  uint64_t threads = c->M * 32;
  k_fill_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
      c->d_bed, c->pitch, c->M, c->pitch / 4, c->d_miss_snp_ptr, c->d_miss_snp_idx, nullptr, 1, 0);
  PG_CHECK_LAUNCH();
  c->launches += 2;
  c->miss_snp_valid = true;
}

void build_missing_by_window_sample(pcaone_ctx* c) {
  if (c->miss_ws_valid) return;
  require_resident(c, "the (window, sample) list outside an RSVD");
  PG_REQUIRE(c->bedT_valid, PCAONE_ESTATE, "transposed copy not built");
  const uint64_t rows = (uint64_t)c->win.bands * c->Npad;
  int64_t* d_cnt = (int64_t*)scratch(c, "miss_ws_cnt", rows * 8);
  uint64_t threads = rows * 32;
  k_count_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
      c->d_bedT, c->win.pitch, rows, c->win.pitch / 4, c->Npad, (uint32_t)c->win.bands, d_cnt);
  PG_CHECK_LAUNCH();
  c->d_miss_ws_ptr = (int64_t*)scratch(c, "d_miss_ws_ptr", (rows + 1) * 8);
  const int64_t total = device_exclusive_scan(c, d_cnt, rows, c->d_miss_ws_ptr);
  c->d_miss_ws_idx = (int32_t*)scratch(c, "d_miss_ws_idx", std::max<int64_t>(total, 1) * 4);
  uint64_t* d_base = (uint64_t*)scratch(c, "miss_ws_base", c->win.bands * 8);
  PG_CUDA(cudaMemcpyAsync(d_base, c->win.start.data(), c->win.bands * 8, cudaMemcpyHostToDevice,
                          c->stream));
  k_fill_missing_rows<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
      c->d_bedT, c->win.pitch, rows, c->win.pitch / 4, c->d_miss_ws_ptr, c->d_miss_ws_idx, d_base,
      c->Npad, (uint32_t)c->win.bands);
  PG_CHECK_LAUNCH();
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->launches += 2;
  c->miss_ws_valid = true;
}

}  // namespace pg
