// Internal declarations shared by the CUDA translation units of libpcaone_gpu.so.
// Nothing here crosses the C ABI (include/pcaone_gpu.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <array>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pcaone_gpu.h"

namespace pg {

// ---------------------------------------------------------------- errors
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PG_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      throw ::pg::Error(e_ == cudaErrorMemoryAllocation ? PCAONE_EOOM : PCAONE_ECUDA,     \
                        std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +     \
                            __FILE__ + ":" + std::to_string(__LINE__));                   \
    }                                                                                    \
  } while (0)

#define PG_CHECK_LAUNCH() PG_CUDA(cudaGetLastError())

#define PG_REQUIRE(cond, code, msg)                 \
  do {                                              \
    if (!(cond)) throw ::pg::Error((code), (msg));  \
  } while (0)

// ---------------------------------------------------------------- device buffers
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Layout constants of the device-resident genotype matrices.
constexpr int kPitchAlign = 64;   // bytes; row pitch of packed matrices (TMA needs 16)
constexpr int kRowPad = 256;      // rows are padded to a multiple of this (sample / SNP tiles)
constexpr int kLmax = 64;         // largest sketch width l = k + oversamples supported

inline uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Window layout of the transposed (sample-major) packed copy used by the X * G product.
struct WindowLayout {
  int bands = 0;           // number of windows (1 for Halko)
  uint64_t blocksize = 0;  // SNPs per window (last may be shorter)
  uint32_t pitch = 0;      // bytes per sample row inside one window block
  std::vector<uint64_t> start, stop;  // [start, stop) SNP range of each window
};

}  // namespace pg

struct pcaone_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  // device time of the last LD r2 call (CUDA events on the stream): all of its device work
  // (diagonal, tiling, band Gram) and the band-Gram launch alone; pairs it produced
  double ld_device_ms = 0.0, ld_gram_ms = 0.0;
  double gl_post_ms = 0.0;  // device time of the last posterior kernel (pcaone_gpu_gl_update)
  int64_t ld_pairs = 0;
  // int8 decode-GEMM autotuner: pipeline variant per product shape (NP, rows, K, K chunks per
  // window, bytes per window)
  std::map<std::array<int64_t, 5>, int> i8_tune;

  // genotypes
  bool loaded = false;
  uint32_t N = 0;       // samples
  uint64_t M = 0;       // SNPs
  uint32_t bpr = 0;     // bytes per SNP record = ceil(N/4)
  uint32_t pitch = 0;   // device row pitch of the SNP-major copy
  uint32_t Npad = 0;    // samples rounded up to kRowPad
  uint64_t Mpad = 0;    // SNPs rounded up to kRowPad
  uint8_t* d_bed = nullptr;  // Mpad x pitch, SNP-major (current SNP order)
  uint32_t* d_a1x2 = nullptr;
  uint32_t* d_nonmiss = nullptr;
  double* d_F = nullptr;
  double* d_F_load = nullptr;  // F in the SNP order of load time (before any permutation)
  double* d_scale = nullptr;   // per-SNP multiplier of the centred genotypes (current order)

  // Streamed genotypes (pcaone_gpu_load_bed_host): the SNP-major records (M x pitch, padding
  // codes set) stay in a pinned host buffer and d_bed is null. The RSVD copies each run of
  // windows into one of two device slots on the copy stream, builds the run's transposed copy
  // (and the int8 back end's tiles) there, and the products read the slot; the other slot
  // takes the next windows meanwhile. The missing-entry lists and per-SNP vectors stay
  // resident (built by streaming passes).
  bool streamed = false;
  uint8_t* h_bed = nullptr;
  size_t h_bed_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  size_t slot_budget = 0;  // device bytes per slot (records, transposed copy, tiles)
  struct StreamSlot {
    int b0 = -1, b1 = -1;  // windows held, once `ready` has completed on the copy stream
    uint64_t key = 0;      // data generation, window layout and tile kind of the contents
    uint8_t *rec = nullptr, *recT = nullptr, *t1 = nullptr, *t2 = nullptr;
    cudaEvent_t ready = nullptr;  // contents complete (copy stream)
    cudaEvent_t idle = nullptr;   // last product reading the slot (main stream)
  } slot[2];
  int slot_windows = 0;   // windows a slot holds for the current layout
  int cur_slot = -1;      // slot the products of the current run read
  uint64_t streamed_h2d = 0;  // bytes copied to the device by window staging (cumulative)

  // PCAngsd (genotype-likelihood) mode: no packed codes; the RSVD runs on the dense float
  // posterior matrix E (SNP-major, Npad floats per SNP), rebuilt from the GL pairs P.
  bool dense = false;
  double* d_dense_norm = nullptr;  // pcaone_gpu_load_dense: squared norms of the centred rows
  double* d_P = nullptr;      // M x 2N doubles (P0, P1 per sample)
  float* d_E = nullptr;       // M x Npad floats
  double* d_zero = nullptr;   // M zeros (centring frequencies of E, already centred)

  // transposed copy for the current window layout
  pg::WindowLayout win;
  uint8_t* d_bedT = nullptr;  // bands x Npad x win.pitch
  bool bedT_valid = false;

  // missing entries: by SNP (CSR over current SNP order) and by (window, sample)
  int64_t n_missing = 0;
  int64_t* d_miss_snp_ptr = nullptr;   // M + 1
  int32_t* d_miss_snp_idx = nullptr;   // sample index per entry
  int64_t* d_miss_ws_ptr = nullptr;    // bands * Npad + 1, sample-major: row i * bands + b
  int32_t* d_miss_ws_idx = nullptr;    // SNP index (global, current order) per entry
  bool miss_snp_valid = false, miss_ws_valid = false;

  // EM imputation (EMU): centred values e_ij of the missing entries, aligned with the two
  // lists, computed from factors U diag(S) V^T kept on the device
  bool imputed = false;        // use e_ij instead of 0 for missing entries
  bool imputed_compat = true;  // reference index semantics for F after the permutation
  int imp_k = 0;
  double* d_imp_US = nullptr;  // N x k (U diag S)
  double* d_imp_V = nullptr;   // M x k (current SNP order)
  double* d_miss_snp_val = nullptr;
  double* d_miss_ws_val = nullptr;
  bool miss_ws_val_valid = false;

  // key (N, l, bands, data generation) of the winSVD window sums kept between calls
  uint64_t h12_key = 0;
  uint64_t generation = 0;  // bumped by every load / permutation
  int bed_slot = 0;         // which of the scratch buffers "d_bed_0" / "d_bed_1" holds d_bed
  // shape key and address of the zeroed split-BF16 window operand (tensor-core back end)
  int64_t bt2_shape = -1;
  void* bt2_ptr = nullptr;
  // tiled copies of the codes for the tensor-core back end, valid for (generation, windows)
  bool tiles_valid = false;
  uint64_t tiles_key = 0;
  void* tile1_ptr = nullptr;
  void* tile2_ptr = nullptr;
  // the same for the tiled copies of the int8 tensor-core back end (kernels_gemm_i8.cu)
  bool tiles8_valid = false;
  uint64_t tiles8_key = 0;
  void* tile81_ptr = nullptr;
  void* tile82_ptr = nullptr;
  bool i8_b2_max_ready = false;  // the first epilogue filled the window operand's column maxima

  // cuSOLVER handle of the PCAngsd GRM's N x N eigendecomposition (created on first use)
  void* solver = nullptr;

  // named scratch buffers (grown on demand, freed with the context)
  std::map<std::string, pg::DevBuf> bufs;

  // kernels whose dynamic shared-memory limit was raised on this context's device
  std::set<const void*> smem_attr_set;

  // resident clusters of the cluster kernels, by kernel and shape (gram.hpp)
  std::map<std::pair<const void*, uint64_t>, int> cluster_occupancy;

  // timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // pinned host buffer and event of the epoch tail's small read-backs (kept between calls)
  void* h_pin = nullptr;
  size_t h_pin_bytes = 0;
  cudaEvent_t ev_tail = nullptr;
  double gemm_ms_accum = 0.0;
  int64_t launches = 0, gemm_launches = 0;
};

namespace pg {

void* scratch(pcaone_ctx* c, const std::string& name, size_t bytes);
void free_all(pcaone_ctx* c);

// ---------------------------------------------------------------- bed kernels (kernels_bed.cu)
void launch_fix_padding(pcaone_ctx* c);
void launch_counts(pcaone_ctx* c);
void launch_permute(pcaone_ctx* c, const int32_t* d_perm, uint8_t* d_out);
// Window layout: bands windows of ceil(M / bands) SNPs, or of blocksize SNPs when it is set
// (the out-of-core block plan); the transposed copy is built per window.
void build_transposed(pcaone_ctx* c, int bands, uint64_t blocksize = 0);
void set_window_layout(pcaone_ctx* c, int bands, uint64_t blocksize = 0);  // layout only (dense mode)
void build_empty_missing(pcaone_ctx* c);           // dense mode: no missing entries
void build_missing_by_snp(pcaone_ctx* c);
void build_missing_by_window_sample(pcaone_ctx* c);
// e_ij = clip(sum_k US_ik V_jk, -Fc_j, 1 - Fc_j) for every entry of the by-SNP list (and of
// the (window, sample) list when it exists); Fc = F at load time under reference index
// semantics, else the current F (Data::fit_with_pi EMU branch, src/Data.cpp:272-287).
void compute_imputed_snp(pcaone_ctx* c);
void compute_imputed_ws(pcaone_ctx* c);
// w[e] = scale_j (val[e] + F_j) for every entry e of the (window, sample) list (j its SNP)
void compute_ws_weights(pcaone_ctx* c, const double* F, double* w);
// LD r2 of every window pair (kernels_ld.cu). W, Y: M x k row-major device arrays (or null).
// d_r2 holds float values, or double with f64.
void ld_r2(pcaone_ctx* c, const double* W, const double* Y, int k, const int64_t* d_ws,
           const int32_t* d_we, const int64_t* d_off, int64_t nwin, void* d_r2, bool f64);
// The same on the tcgen05 tensor cores (kernels_ld_tc.cu): the band Gram of the windows as
// exact int8 products, one persistent launch; usable for projections of at most 16 columns.
// ws, we: host window arrays; d_win_of (M: window led by SNP i or -1), d_we, d_off: device.
bool ld_tc_usable(pcaone_ctx* c, int k);
void ld_r2_tc(pcaone_ctx* c, const double* W, const double* Y, int k, const int64_t* ws, const int32_t* we,
              uint64_t nwin, const int64_t* d_win_of, const int32_t* d_we, const int64_t* d_off, void* d_r2, bool f64);
// LD flow B (kernels_ld.cu): residual rows of snp0..snp0+nsnp (US N x k, V nsnp x k
// row-major device arrays, or null for the centred genotypes), the in-place centring of the
// dense matrix with its squared column norms d, and r2 of the window pairs on it.
void residuals(pcaone_ctx* c, const double* US, const double* V, int k, uint64_t snp0, uint64_t nsnp, float* out);
void dense_center(pcaone_ctx* c, double* d);
void ld_r2_dense(pcaone_ctx* c, const double* d, const int64_t* d_win_of, const int32_t* d_we, const int64_t* d_off,
                 const int32_t* d_span, int max_span, void* d_r2, bool f64);
// d_scale_j = 1/sqrt(ploidy Fs_j (1 - Fs_j)) (or 1 when not standardising / sd <= 1e-9).
void compute_scale(pcaone_ctx* c, int standardize, int ploidy);

// ---------------------------------------------------------------- streamed genotypes (stream.cu)
// Counts and F of the host records (staged through the device), at load.
void stream_counts(pcaone_ctx* c);
// By-SNP missing-entry list from one staging pass.
void stream_missing_snp(pcaone_ctx* c);
// Window layout, and the two missing-entry lists built from two staging passes.
void stream_prepare(pcaone_ctx* c, int bands, uint64_t blocksize, bool tiles);
// Pinned host copy of the records at the device pitch (padding set), copy stream; counts at load.
void stream_load(pcaone_ctx* c, const uint8_t* packed, size_t slot_bytes);
// Host records in the order perm (row j = old row perm[j]).
void stream_permute(pcaone_ctx* c, const int32_t* perm);
// Make the slot holding window b current (staging [b, b + slot_windows) if no slot holds it;
// the main stream waits for its contents); tiles: also the int8 back end's tiled copies.
// Returns the last window + 1 the slot holds.
int stream_acquire(pcaone_ctx* c, int b, bool tiles);
// Stage the windows from b on into the slot that is not current, unless a slot holds b.
void stream_prefetch(pcaone_ctx* c, int b, bool tiles);
// The products of the current run are queued: the slot may be refilled after them.
void stream_release(pcaone_ctx* c);
// Packed rows of window b in the current slot: SNP-major records / sample-major copy.
const uint8_t* stream_codes(const pcaone_ctx* c, int b);
const uint8_t* stream_codesT(const pcaone_ctx* c, int b);
void stream_free(pcaone_ctx* c);
// Fails with PCAONE_ESTATE when the genotypes are streamed (calls that need them resident).
void require_resident(const pcaone_ctx* c, const char* what);
// Launchers used by the staging (kernels_bed.cu, kernels_gemm_i8.cu)
void launch_counts_rows(pcaone_ctx* c, cudaStream_t st, const uint8_t* rows, uint64_t nrows, uint64_t row0);
void launch_freq(pcaone_ctx* c);
void launch_transpose_run(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, uint64_t nsnp, int nwin, uint8_t* recT);
void launch_missing_snp_rows(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, uint64_t nrows, uint64_t row0);
void launch_missing_ws_count(pcaone_ctx* c, cudaStream_t st, const uint8_t* recT, int b0, int nw, int64_t* cnt);
void launch_missing_ws_fill(pcaone_ctx* c, cudaStream_t st, const uint8_t* recT, int b0, int nw,
                            const uint64_t* d_base);
int64_t missing_snp_scan(pcaone_ctx* c);  // by-SNP row pointers from the counts; total
int64_t scan_counts(pcaone_ctx* c, const int64_t* cnt, uint64_t n, int64_t* ptr);
// int8 back end: tile bytes per window (first, second product) and the tiling of one window
void i8_tile_bytes(const pcaone_ctx* c, size_t* w1, size_t* w2);
void i8_tile_window(pcaone_ctx* c, cudaStream_t st, const uint8_t* rec, int64_t m, const uint8_t* recT,
                    uint8_t* t1, uint8_t* t2);

// ---------------------------------------------------------------- SIMT decode-GEMM
// out[s][r][c] = sum_{k in split s} val(code[r][k]) * B[k][c], val(00,01,10,11) = (2,0,1,0)
// codes: rows x pitch bytes; B: row-major K x ldb (T); out: ksplit x rows x l (T).
template <typename T>
void launch_decode_gemm_simt(pcaone_ctx* c, const uint8_t* codes, uint32_t pitch, int64_t rows,
                             int64_t K, const T* B, int ldb, int l, int ksplit, T* out);

// ---------------------------------------------------------------- tcgen05 decode-GEMM
// Same contract with BF16 hi/lo split of B; see kernels_gemm_tc.cu.
bool tc_supported(pcaone_ctx* c);
void tc_clear_error(pcaone_ctx* c);
void tc_check_error(pcaone_ctx* c);

}  // namespace pg
