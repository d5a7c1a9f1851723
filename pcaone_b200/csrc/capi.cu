// C ABI entry points (include/pcaone_gpu.h). Every call catches pg::Error and returns its
// status code; the message is kept on the context for pcaone_gpu_last_error().
#include <algorithm>
#include <cstring>
#include <numeric>
#include <random>

#include "internal.hpp"
#include "rsvd.hpp"

namespace pg {

void* scratch(pcaone_ctx* c, const std::string& name, size_t bytes) {
  DevBuf& b = c->bufs[name];
  if (b.bytes < bytes) {
    if (b.p) PG_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    size_t alloc = round_up(std::max<size_t>(bytes, 256), 256);
    PG_CUDA(cudaMalloc(&b.p, alloc));
    b.bytes = alloc;
  }
  return b.p;
}

static void free_ptr(void* p) {
  if (p) cudaFree(p);
}

// Forget the loaded data. Every data buffer is a named scratch buffer of the context (kept,
// with its capacity, for the next load of the same or a smaller problem; freed by free_all).
void free_data(pcaone_ctx* c) {
  c->d_P = nullptr;
  c->d_E = nullptr;
  c->d_dense_norm = nullptr;
  c->d_zero = nullptr;
  c->dense = false;
  c->win = WindowLayout();
  c->d_F_load = c->d_scale = c->d_imp_US = c->d_imp_V = c->d_miss_snp_val = c->d_miss_ws_val = nullptr;
  c->imputed = false;
  c->miss_ws_val_valid = false;
  c->d_bed = c->d_bedT = nullptr;
  c->d_a1x2 = c->d_nonmiss = nullptr;
  c->d_F = nullptr;
  c->d_miss_snp_ptr = c->d_miss_ws_ptr = nullptr;
  c->d_miss_snp_idx = c->d_miss_ws_idx = nullptr;
  c->loaded = c->bedT_valid = c->miss_snp_valid = c->miss_ws_valid = false;
  // streamed genotypes: the pinned host buffer and the slots are kept for reuse; their
  // contents are forgotten (a copy still in flight completes first)
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  c->streamed = false;
  c->slot[0].key = c->slot[1].key = 0;
  c->cur_slot = -1;
  c->slot_windows = 0;
}

void free_all(pcaone_ctx* c) {
  free_data(c);
  for (auto& kv : c->bufs) free_ptr(kv.second.p);
  c->bufs.clear();
  c->bt2_shape = -1;
  c->bt2_ptr = nullptr;
  c->tiles_valid = false;
  c->tiles8_valid = false;
  c->tile1_ptr = c->tile2_ptr = nullptr;
}

}  // namespace pg

using namespace pg;

namespace {

template <typename F>
int guarded(pcaone_ctx* c, F&& f) {
  if (!c) return PCAONE_EBADARG;
  try {
    PG_CUDA(cudaSetDevice(c->device));
    f();
    c->err.clear();
    return PCAONE_OK;
  } catch (const Error& e) {
    c->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return PCAONE_ECUDA;
  }
}

}  // namespace

namespace {

// U diag(S) (N x k) and V (M x k), both row-major, on the device for the posterior kernels;
// U and V are column-major host matrices.
void upload_factors(pcaone_ctx* c, const double* U, const double* S, const double* V, uint32_t k, double** dUS,
                    double** dV) {
  PG_REQUIRE(S && V && k >= 1 && k <= (uint32_t)pg::kLmax, PCAONE_EBADARG, "bad factors");
  std::vector<double> us((size_t)c->N * k), v((size_t)c->M * k);
  // column by column: sequential reads of the column-major inputs
  for (uint32_t t = 0; t < k; ++t)
    for (uint32_t i = 0; i < c->N; ++i) us[(size_t)i * k + t] = U[(size_t)t * c->N + i] * S[t];
  for (uint32_t t = 0; t < k; ++t)
    for (uint64_t j = 0; j < c->M; ++j) v[(size_t)j * k + t] = V[(size_t)t * c->M + j];
  *dUS = (double*)pg::scratch(c, "gl_US", us.size() * 8);
  *dV = (double*)pg::scratch(c, "gl_V", v.size() * 8);
  PG_CUDA(cudaMemcpyAsync(*dUS, us.data(), us.size() * 8, cudaMemcpyHostToDevice, c->stream));
  PG_CUDA(cudaMemcpyAsync(*dV, v.data(), v.size() * 8, cudaMemcpyHostToDevice, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace

extern "C" {

int pcaone_gpu_create(int device, pcaone_ctx** out) {
  if (!out) return PCAONE_EBADARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return PCAONE_ENODEV;
  auto* c = new pcaone_ctx();
  c->device = device;
  int st = guarded(c, [&] {
    cudaDeviceProp prop;
    PG_CUDA(cudaGetDeviceProperties(&prop, device));
    c->sm_count = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    PG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    PG_CUDA(cudaEventCreate(&c->ev0));
    PG_CUDA(cudaEventCreate(&c->ev1));
  });
  if (st != PCAONE_OK) {
    delete c;
    return st;
  }
  *out = c;
  return PCAONE_OK;
}

int pcaone_gpu_destroy(pcaone_ctx* c) {
  if (!c) return PCAONE_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  pg::gl_release(c);
  free_all(c);
  pg::stream_free(c);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_tail) cudaEventDestroy(c->ev_tail);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return PCAONE_OK;
}

const char* pcaone_gpu_last_error(const pcaone_ctx* c) { return c ? c->err.c_str() : "null context"; }

int pcaone_gpu_load_bed(pcaone_ctx* c, const uint8_t* packed, uint64_t nsnps, uint32_t nsamples) {
  return guarded(c, [&] {
    PG_REQUIRE(packed && nsnps > 0 && nsamples > 0, PCAONE_EBADARG, "empty genotype matrix");
    PG_REQUIRE(nsnps < (1ull << 31) && nsamples < (1u << 30), PCAONE_EBADARG, "genotype matrix too large");
    free_data(c);
    c->generation++;
    c->N = nsamples;
    c->M = nsnps;
    c->bpr = (nsamples + 3) / 4;
    c->Npad = (uint32_t)round_up(nsamples, kRowPad);
    c->pitch = c->Npad / 4;  // == round_up(bpr, kPitchAlign)
    c->Mpad = round_up(nsnps, kRowPad) + kRowPad;
    const size_t bytes = (size_t)c->Mpad * c->pitch;
    c->bed_slot = 0;
    c->d_bed = (uint8_t*)scratch(c, "d_bed_0", bytes);
    c->d_a1x2 = (uint32_t*)scratch(c, "d_a1x2", c->M * 4);
    c->d_nonmiss = (uint32_t*)scratch(c, "d_nonmiss", c->M * 4);
    c->d_F = (double*)scratch(c, "d_F", c->M * 8);
    c->d_F_load = (double*)scratch(c, "d_F_load", c->M * 8);
    c->d_scale = (double*)scratch(c, "d_scale", c->M * 8);
    PG_CUDA(cudaMemsetAsync(c->d_bed, 0xFF, bytes, c->stream));
    PG_CUDA(cudaMemcpy2DAsync(c->d_bed, c->pitch, packed, c->bpr, c->bpr, c->M,
                              cudaMemcpyHostToDevice, c->stream));
    launch_fix_padding(c);
    launch_counts(c);
    PG_CUDA(cudaMemcpyAsync(c->d_F_load, c->d_F, c->M * 8, cudaMemcpyDeviceToDevice, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    c->loaded = true;
  });
}

int pcaone_gpu_load_bed_host(pcaone_ctx* c, const uint8_t* packed, uint64_t nsnps, uint32_t nsamples,
                             uint64_t slot_bytes) {
  return guarded(c, [&] {
    PG_REQUIRE(packed && nsnps > 0 && nsamples > 0, PCAONE_EBADARG, "empty genotype matrix");
    PG_REQUIRE(nsnps < (1ull << 31) && nsamples < (1u << 30), PCAONE_EBADARG, "genotype matrix too large");
    free_data(c);
    c->generation++;
    c->N = nsamples;
    c->M = nsnps;
    c->bpr = (nsamples + 3) / 4;
    c->Npad = (uint32_t)round_up(nsamples, kRowPad);
    c->pitch = c->Npad / 4;
    c->Mpad = round_up(nsnps, kRowPad) + kRowPad;
    c->d_bed = nullptr;
    c->d_a1x2 = (uint32_t*)scratch(c, "d_a1x2", c->M * 4);
    c->d_nonmiss = (uint32_t*)scratch(c, "d_nonmiss", c->M * 4);
    c->d_F = (double*)scratch(c, "d_F", c->M * 8);
    c->d_F_load = (double*)scratch(c, "d_F_load", c->M * 8);
    c->d_scale = (double*)scratch(c, "d_scale", c->M * 8);
    stream_load(c, packed, (size_t)slot_bytes);
    stream_counts(c);
    PG_CUDA(cudaMemcpyAsync(c->d_F_load, c->d_F, c->M * 8, cudaMemcpyDeviceToDevice, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    c->loaded = true;
  });
}

int pcaone_gpu_counts(pcaone_ctx* c, uint32_t* a1x2, uint32_t* nonmiss) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
    if (a1x2) PG_CUDA(cudaMemcpyAsync(a1x2, c->d_a1x2, c->M * 4, cudaMemcpyDeviceToHost, c->stream));
    if (nonmiss)
      PG_CUDA(cudaMemcpyAsync(nonmiss, c->d_nonmiss, c->M * 4, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int pcaone_gpu_allele_freq(pcaone_ctx* c, double* F) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
    PG_REQUIRE(F, PCAONE_EBADARG, "null output");
    PG_CUDA(cudaMemcpyAsync(F, c->d_F, c->M * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int pcaone_gpu_permute(pcaone_ctx* c, const int32_t* perm) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
    PG_REQUIRE(perm, PCAONE_EBADARG, "null permutation");
    std::vector<char> seen(c->M, 0);
    for (uint64_t j = 0; j < c->M; ++j) {
      PG_REQUIRE(perm[j] >= 0 && (uint64_t)perm[j] < c->M && !seen[perm[j]], PCAONE_EBADARG,
                 "perm is not a permutation of 0..nsnps-1");
      seen[perm[j]] = 1;
    }
    if (c->streamed) {  // the host records are permuted, then counted again
      PG_CUDA(cudaStreamSynchronize(c->stream));
      if (c->copy_stream) PG_CUDA(cudaStreamSynchronize(c->copy_stream));
      stream_permute(c, perm);
      stream_counts(c);
    } else {
      int32_t* d_perm = (int32_t*)scratch(c, "perm", c->M * 4);
      PG_CUDA(cudaMemcpyAsync(d_perm, perm, c->M * 4, cudaMemcpyHostToDevice, c->stream));
      // permute into the other of the two packed-matrix slots, then swap
      const size_t bytes = (size_t)c->Mpad * c->pitch;
      uint8_t* out = (uint8_t*)scratch(c, c->bed_slot ? "d_bed_0" : "d_bed_1", bytes);
      PG_CUDA(cudaMemsetAsync(out, 0xFF, bytes, c->stream));
      launch_permute(c, d_perm, out);
      PG_CUDA(cudaStreamSynchronize(c->stream));
      c->d_bed = out;
      c->bed_slot ^= 1;
      launch_counts(c);
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
    c->bedT_valid = c->miss_snp_valid = c->miss_ws_valid = false;
    c->generation++;
    c->imputed = false;  // imputed values are tied to the SNP order of the lists
    c->miss_ws_val_valid = false;
  });
}

int pcaone_shuffle_perm(uint64_t n, int32_t* perm) {
  if (!perm) return PCAONE_EBADARG;
  std::iota(perm, perm + n, 0);
  auto rng = std::default_random_engine{};
  std::shuffle(perm, perm + n, rng);
  return PCAONE_OK;
}

int pcaone_plink_perm(uint64_t nsnps, uint32_t nsamples, uint32_t buffer_gb, uint32_t nbands, int32_t* perm) {
  // permute_plink (src/FilePlink.cpp:298-405) without its file copies: the input is read in
  // buffers of a multiple of nbands SNPs (buffer_gb GB at most); within a buffer SNP
  // j * nbands + b goes to band b, whose SNPs are stored contiguously from bandidx[b]
  // (bands as equal as possible, the first M % nbands one SNP longer); the last, shorter
  // buffer deals its SNPs round-robin to the first bands. perm[new] = old.
  if (!perm || nsnps == 0 || nbands == 0 || nsamples == 0) return PCAONE_EBADARG;
  const uint64_t M = nsnps, bpr = (nsamples + 3) >> 2, nb = nbands;
  uint64_t two = (uint64_t)std::floor(1073741824.0 * buffer_gb / (double)bpr);
  if (two > M) two = M;
  uint64_t bufsize = two / nb;
  if (bufsize == 0) return PCAONE_EBADARG;
  two = bufsize * nb;
  const uint64_t nblocks = (M + two - 1) / two;
  uint64_t modr2 = M % two;
  const uint64_t bufidx = bufsize;
  std::vector<uint64_t> bandidx(nb);
  const uint64_t modr = M % nb, bandsize = (M + nb - 1) / nb;
  for (uint64_t b = 0; b < nb; ++b)
    bandidx[b] = (modr == 0 || b < modr) ? b * bandsize : modr * bandsize + (bandsize - 1) * (b - modr);
  std::vector<char> seen(M, 0);
  for (uint64_t i = 0; i < nblocks; ++i) {
    if (i == nblocks - 1 && modr2 != 0) {
      const uint64_t two2 = M - (nblocks - 1) * two;
      bufsize = (two2 + nb - 1) / nb;
      modr2 = two2 % nb;
    }
    for (uint64_t b = 0; b < nb; ++b) {
      uint64_t j = 0;
      auto put = [&](uint64_t jj) {
        const uint64_t ia = i * two + jj * nb + b, ib = i * bufidx + bandidx[b] + jj;
        if (ia < M && ib < M) {
          perm[ib] = (int32_t)ia;
          seen[ib] = 1;
        }
      };
      for (; j + 1 < bufsize; ++j) put(j);
      if (i != nblocks - 1 || b < modr2 || modr2 == 0) put(j);
    }
  }
  for (uint64_t t = 0; t < M; ++t)
    if (!seen[t]) return PCAONE_EBADARG;
  return PCAONE_OK;
}

int pcaone_omega(int seed, int rand, uint64_t nrow, uint32_t ncol, double* out) {
  if (!out) return PCAONE_EBADARG;
  omega_host(seed, rand, nrow, ncol, out);
  return PCAONE_OK;
}

int pcaone_gpu_rsvd(pcaone_ctx* c, const pcaone_rsvd_opts* opts, double* U, double* S, double* V,
                    pcaone_rsvd_report* report) {
  return guarded(c, [&] {
    PG_REQUIRE(opts, PCAONE_EBADARG, "null options");
    run_rsvd(c, *opts, U, S, V, report);
  });
}

int pcaone_gpu_gram_product(pcaone_ctx* c, int precision, int standardize, int ploidy, const double* X,
                            uint32_t ncols, double* Y) {
  return guarded(c, [&] { run_gram(c, precision, standardize, ploidy, X, (int)ncols, Y); });
}

int pcaone_gpu_product(pcaone_ctx* c, int precision, int transpose, int standardize, int ploidy,
                       const double* B, uint32_t ncols, double* out) {
  return guarded(c, [&] { run_product(c, precision, transpose, standardize, ploidy, B, (int)ncols, out); });
}

int pcaone_gpu_fit_emu(pcaone_ctx* c, const double* U, const double* S, const double* V,
                       uint32_t k, int reference_index) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
    PG_REQUIRE(U && S && V && k >= 1 && k <= (uint32_t)kLmax, PCAONE_EBADARG, "bad EMU factors");
    build_missing_by_snp(c);
    // US = U diag(S), row-major N x k; V row-major M x k
    std::vector<double> us((size_t)c->N * k), v((size_t)c->M * k);
    for (uint32_t t = 0; t < k; ++t)  // column by column: sequential reads of the inputs
      for (uint32_t i = 0; i < c->N; ++i) us[(size_t)i * k + t] = U[(size_t)t * c->N + i] * S[t];
    for (uint32_t t = 0; t < k; ++t)
      for (uint64_t j = 0; j < c->M; ++j) v[(size_t)j * k + t] = V[(size_t)t * c->M + j];
    c->d_imp_US = (double*)scratch(c, "d_imp_US", us.size() * 8);
    c->d_imp_V = (double*)scratch(c, "d_imp_V", v.size() * 8);
    PG_CUDA(cudaMemcpyAsync(c->d_imp_US, us.data(), us.size() * 8, cudaMemcpyHostToDevice, c->stream));
    PG_CUDA(cudaMemcpyAsync(c->d_imp_V, v.data(), v.size() * 8, cudaMemcpyHostToDevice, c->stream));
    c->imp_k = (int)k;
    c->imputed_compat = reference_index != 0;
    compute_imputed_snp(c);
    c->miss_ws_val_valid = false;
    if (c->miss_ws_valid) compute_imputed_ws(c);
    c->imputed = true;
    PG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int pcaone_gpu_clear_imputed(pcaone_ctx* c) {
  return guarded(c, [&] { c->imputed = false; });
}

}  // extern "C"

namespace {
// r2 of the window pairs into the host array r2 (float, or double with f64).
void ld_r2_impl(pcaone_ctx* c, const double* U, uint32_t k, const int64_t* ws, const int32_t* we, uint64_t nwin,
                void* r2, bool f64) {
  {
    const size_t esz = f64 ? 8 : 4;
    c->ld_device_ms = c->ld_gram_ms = -1.0;
    PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
    PG_REQUIRE(ws && we && (r2 || nwin == 0), PCAONE_EBADARG, "null window arrays");
    PG_REQUIRE(!U || (k >= 1 && k <= (uint32_t)kLmax), PCAONE_EBADARG, "bad U width");
    PG_REQUIRE(!c->imputed, PCAONE_ESTATE, "clear the EMU imputation before LD");
    std::vector<int64_t> off(nwin + 1, 0);
    for (uint64_t w = 0; w < nwin; ++w) {
      PG_REQUIRE(ws[w] >= 0 && we[w] >= 1 && (uint64_t)ws[w] + we[w] <= c->M, PCAONE_EBADARG,
                 "window " + std::to_string(w) + " out of range");
      off[w + 1] = off[w] + (we[w] - 1);
    }
    if (c->dense) {
      // LD flow B: r2 on the centred dense matrix of pcaone_gpu_load_dense
      PG_REQUIRE(!U && c->d_dense_norm, PCAONE_ESTATE,
                 "LD on a dense matrix needs pcaone_gpu_load_dense and no U (the residuals are already adjusted)");
      std::vector<int64_t> win_of(c->M, -1);
      const uint64_t blocks = (c->M + 31) / 32;
      std::vector<int32_t> span(blocks, -1);
      int max_span = 0;
      for (uint64_t w = 0; w < nwin; ++w) {
        win_of[ws[w]] = (int64_t)w;
        const uint64_t b = (uint64_t)ws[w] / 32;
        const int s = (int)((uint64_t)ws[w] - b * 32) + we[w] - 1;
        span[b] = std::max(span[b], s);
        max_span = std::max(max_span, s);
      }
      int64_t* d_win_of = (int64_t*)scratch(c, "ld_win_of", c->M * 8);
      int32_t* d_span = (int32_t*)scratch(c, "ld_span", blocks * 4);
      int32_t* d_we = (int32_t*)scratch(c, "ld_we", std::max<uint64_t>(nwin, 1) * 4);
      int64_t* d_off = (int64_t*)scratch(c, "ld_off", (nwin + 1) * 8);
      void* d_r2 = scratch(c, "ld_r2", std::max<int64_t>(off[nwin], 1) * esz);
      PG_CUDA(cudaMemcpyAsync(d_win_of, win_of.data(), c->M * 8, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaMemcpyAsync(d_span, span.data(), blocks * 4, cudaMemcpyHostToDevice, c->stream));
      if (nwin) {
        PG_CUDA(cudaMemcpyAsync(d_we, we, nwin * 4, cudaMemcpyHostToDevice, c->stream));
        PG_CUDA(cudaMemcpyAsync(d_off, off.data(), (nwin + 1) * 8, cudaMemcpyHostToDevice, c->stream));
        ld_r2_dense(c, c->d_dense_norm, d_win_of, d_we, d_off, d_span, max_span, d_r2, f64);
      }
      if (off[nwin] > 0)
        PG_CUDA(cudaMemcpyAsync(r2, d_r2, off[nwin] * esz, cudaMemcpyDeviceToHost, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
      return;
    }
    double *dW = nullptr, *dY = nullptr;
    if (U) {
      // W = Gc^T U (M x k) through the FP64 product path; Y = (2I - U^T U) W on the host
      std::vector<double> W((size_t)c->M * k), C((size_t)k * k, 0.0), Wr((size_t)c->M * k), Yr((size_t)c->M * k);
      run_product(c, PCAONE_PREC_FP64, 0, 0, 2, U, (int)k, W.data());
      for (uint32_t a = 0; a < k; ++a)
        for (uint32_t b = 0; b < k; ++b) {
          double acc = 0;
          for (uint32_t i = 0; i < c->N; ++i) acc += U[(size_t)a * c->N + i] * U[(size_t)b * c->N + i];
          C[(size_t)a * k + b] = (a == b ? 2.0 : 0.0) - acc;
        }
      for (uint64_t j = 0; j < c->M; ++j)
        for (uint32_t a = 0; a < k; ++a) {
          Wr[j * k + a] = W[(size_t)a * c->M + j];
          double acc = 0;
          for (uint32_t b = 0; b < k; ++b) acc += C[(size_t)a * k + b] * W[(size_t)b * c->M + j];
          Yr[j * k + a] = acc;
        }
      dW = (double*)scratch(c, "ld_W", Wr.size() * 8);
      dY = (double*)scratch(c, "ld_Y", Yr.size() * 8);
      PG_CUDA(cudaMemcpyAsync(dW, Wr.data(), Wr.size() * 8, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaMemcpyAsync(dY, Yr.data(), Yr.size() * 8, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
    int64_t* d_ws = (int64_t*)scratch(c, "ld_ws", std::max<uint64_t>(nwin, 1) * 8);
    int32_t* d_we = (int32_t*)scratch(c, "ld_we", std::max<uint64_t>(nwin, 1) * 4);
    int64_t* d_off = (int64_t*)scratch(c, "ld_off", (nwin + 1) * 8);
    void* d_r2 = scratch(c, "ld_r2", std::max<int64_t>(off[nwin], 1) * esz);
    if (nwin) {
      PG_CUDA(cudaMemcpyAsync(d_ws, ws, nwin * 8, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaMemcpyAsync(d_we, we, nwin * 4, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaMemcpyAsync(d_off, off.data(), (nwin + 1) * 8, cudaMemcpyHostToDevice, c->stream));
    }
    if (ld_tc_usable(c, U ? (int)k : 0)) {
      // band Gram on the tensor cores: windows located by their lead SNP
      std::vector<int64_t> win_of(c->M, -1);
      for (uint64_t w = 0; w < nwin; ++w) win_of[ws[w]] = (int64_t)w;
      int64_t* d_win_of = (int64_t*)scratch(c, "ld_win_of", c->M * 8);
      PG_CUDA(cudaMemcpyAsync(d_win_of, win_of.data(), c->M * 8, cudaMemcpyHostToDevice, c->stream));
      tc_clear_error(c);
      ld_r2_tc(c, dW, dY, U ? (int)k : 0, ws, we, nwin, d_win_of, d_we, d_off, d_r2, f64);
      tc_check_error(c);
    } else {
      ld_r2(c, dW, dY, U ? (int)k : 0, d_ws, d_we, d_off, (int64_t)nwin, d_r2, f64);
    }
    if (off[nwin] > 0)
      PG_CUDA(cudaMemcpyAsync(r2, d_r2, off[nwin] * esz, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
  }
}
}  // namespace

extern "C" {

int pcaone_gpu_ld_r2(pcaone_ctx* c, const double* U, uint32_t k, const int64_t* ws, const int32_t* we,
                     uint64_t nwin, float* r2) {
  return guarded(c, [&] {
    require_resident(c, "LD r2");
    ld_r2_impl(c, U, k, ws, we, nwin, r2, false);
  });
}

int pcaone_gpu_ld_r2_f64(pcaone_ctx* c, const double* U, uint32_t k, const int64_t* ws, const int32_t* we,
                         uint64_t nwin, double* r2) {
  return guarded(c, [&] {
    require_resident(c, "LD r2");
    ld_r2_impl(c, U, k, ws, we, nwin, r2, true);
  });
}

int pcaone_gpu_ld_timing(pcaone_ctx* c, double* device_ms, double* gram_ms) {
  return guarded(c, [&] {
    PG_REQUIRE(device_ms && gram_ms, PCAONE_EBADARG, "null timing outputs");
    *device_ms = c->ld_device_ms;
    *gram_ms = c->ld_gram_ms;
  });
}


}  // extern "C"

namespace {
// Likelihood pairs (FP64 or FP32 host, 2N x M column-major) -> the context's FP64 device copy.
template <typename T>
void load_gl_impl(pcaone_ctx* c, const T* P, uint64_t nsnps, uint32_t nsamples) {
  PG_REQUIRE(P && nsnps > 0 && nsamples > 0, PCAONE_EBADARG, "empty likelihood matrix");
  PG_REQUIRE(nsnps < (1ull << 31) && nsamples < (1u << 29), PCAONE_EBADARG, "likelihood matrix too large");
  free_data(c);
  c->generation++;
  c->dense = true;
  c->N = nsamples;
  c->M = nsnps;
  c->Npad = (uint32_t)round_up(nsamples, kRowPad);
  c->Mpad = round_up(nsnps, kRowPad) + kRowPad;
  c->pitch = 1;
  const size_t np = (size_t)nsnps * 2 * nsamples;
  // kept in FP64 as the reference keeps it: under the shuffle's index semantics the EM
  // updates amplify FP32 rounding of the likelihoods to about 1e-6 of the singular values
  c->d_P = (double*)scratch(c, "d_P", np * 8);
  if (std::is_same<T, double>::value)
    PG_CUDA(cudaMemcpyAsync(c->d_P, P, np * 8, cudaMemcpyHostToDevice, c->stream));
  else
    gl_widen_f32(c, reinterpret_cast<const float*>(P), np, c->d_P);
  c->d_E = (float*)scratch(c, "d_E", (size_t)c->Mpad * c->Npad * 4);
  PG_CUDA(cudaMemsetAsync(c->d_E, 0, (size_t)c->Mpad * c->Npad * 4, c->stream));
  c->d_F = (double*)scratch(c, "d_F", c->M * 8);
  c->d_F_load = (double*)scratch(c, "d_F_load", c->M * 8);
  c->d_scale = (double*)scratch(c, "d_scale", c->M * 8);
  c->d_zero = (double*)scratch(c, "d_zero", c->M * 8);
  PG_CUDA(cudaMemsetAsync(c->d_zero, 0, c->M * 8, c->stream));
  std::vector<double> q(c->M, 0.25);
  PG_CUDA(cudaMemcpyAsync(c->d_F, q.data(), c->M * 8, cudaMemcpyHostToDevice, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->loaded = true;
}
}  // namespace

extern "C" {

int pcaone_gpu_load_gl(pcaone_ctx* c, const double* P, uint64_t nsnps, uint32_t nsamples) {
  return guarded(c, [&] { load_gl_impl<double>(c, P, nsnps, nsamples); });
}

int pcaone_gpu_load_gl_f32(pcaone_ctx* c, const float* P, uint64_t nsnps, uint32_t nsamples) {
  return guarded(c, [&] { load_gl_impl<float>(c, P, nsnps, nsamples); });
}

int pcaone_gpu_load_dense(pcaone_ctx* c, const float* X, uint64_t nsnps, uint32_t nsamples) {
  return guarded(c, [&] {
    PG_REQUIRE(X && nsnps > 0 && nsamples > 1, PCAONE_EBADARG, "empty dense matrix");
    PG_REQUIRE(nsnps < (1ull << 31) && nsamples < (1u << 29), PCAONE_EBADARG, "dense matrix too large");
    free_data(c);
    c->generation++;
    c->dense = true;
    c->N = nsamples;
    c->M = nsnps;
    c->Npad = (uint32_t)round_up(nsamples, kRowPad);
    c->Mpad = round_up(nsnps, kRowPad) + kRowPad;
    c->pitch = 1;
    c->d_E = (float*)scratch(c, "d_E", (size_t)c->Mpad * c->Npad * 4);
    PG_CUDA(cudaMemsetAsync(c->d_E, 0, (size_t)c->Mpad * c->Npad * 4, c->stream));
    PG_CUDA(cudaMemcpy2DAsync(c->d_E, (size_t)c->Npad * 4, X, (size_t)nsamples * 4, (size_t)nsamples * 4, nsnps,
                              cudaMemcpyHostToDevice, c->stream));
    c->d_dense_norm = (double*)scratch(c, "d_dense_norm", c->M * 8);
    dense_center(c, c->d_dense_norm);
    c->d_F = (double*)scratch(c, "d_F", c->M * 8);
    c->d_F_load = (double*)scratch(c, "d_F_load", c->M * 8);
    c->d_scale = (double*)scratch(c, "d_scale", c->M * 8);
    c->d_zero = (double*)scratch(c, "d_zero", c->M * 8);
    PG_CUDA(cudaMemsetAsync(c->d_zero, 0, c->M * 8, c->stream));
    PG_CUDA(cudaMemsetAsync(c->d_F, 0, c->M * 8, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    c->loaded = true;
  });
}

int pcaone_gpu_residuals(pcaone_ctx* c, const double* U, const double* S, const double* V, uint32_t k,
                         uint64_t snp0, uint64_t nsnp, float* out) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded && !c->dense, PCAONE_ESTATE, "residuals need packed genotypes (load_bed)");
    require_resident(c, "residuals");
    PG_REQUIRE(out && snp0 + nsnp <= c->M, PCAONE_EBADARG, "residual rows out of range");
    PG_REQUIRE(!U || (S && V && k >= 1 && k <= (uint32_t)kLmax), PCAONE_EBADARG, "bad factors");
    double *dUS = nullptr, *dV = nullptr;
    if (U) {
      std::vector<double> us((size_t)c->N * k), v((size_t)nsnp * k);
      for (uint32_t i = 0; i < c->N; ++i)
        for (uint32_t t = 0; t < k; ++t) us[(size_t)i * k + t] = U[(size_t)t * c->N + i] * S[t];
      for (uint64_t j = 0; j < nsnp; ++j)
        for (uint32_t t = 0; t < k; ++t) v[(size_t)j * k + t] = V[(size_t)t * nsnp + j];
      dUS = (double*)scratch(c, "res_US", us.size() * 8);
      dV = (double*)scratch(c, "res_V", std::max<size_t>(v.size(), 1) * 8);
      PG_CUDA(cudaMemcpyAsync(dUS, us.data(), us.size() * 8, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaMemcpyAsync(dV, v.data(), v.size() * 8, cudaMemcpyHostToDevice, c->stream));
    }
    float* d_out = (float*)scratch(c, "res_out", std::max<uint64_t>(nsnp, 1) * c->N * 4);
    if (nsnp) residuals(c, dUS, dV, U ? (int)k : 0, snp0, nsnp, d_out);
    if (nsnp) PG_CUDA(cudaMemcpyAsync(out, d_out, nsnp * c->N * 4, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int pcaone_gpu_bed_to_gl(pcaone_ctx* c) {
  return guarded(c, [&] {
    require_resident(c, "pseudo-likelihoods");
    gl_from_bed(c);
  });
}

int pcaone_gpu_gl_freq(pcaone_ctx* c, int maxiter, double tolmaf, double* F, int* iters) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded && c->dense, PCAONE_ESTATE, "no likelihoods loaded");
    PG_REQUIRE(maxiter >= 1, PCAONE_EBADARG, "maxiter must be >= 1");
    gl_em_maf(c, maxiter, tolmaf, iters);
    if (F) PG_CUDA(cudaMemcpyAsync(F, c->d_F, c->M * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int pcaone_gpu_gl_update(pcaone_ctx* c, const double* U, const double* S, const double* V, uint32_t k) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded && c->dense, PCAONE_ESTATE, "no likelihoods loaded");
    double *dUS = nullptr, *dV = nullptr;
    if (U) upload_factors(c, U, S, V, k, &dUS, &dV);
    PG_CUDA(cudaEventRecord(c->ev0, c->stream));
    gl_posterior(c, dUS, dV, U ? (int)k : 0);
    PG_CUDA(cudaEventRecord(c->ev1, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    PG_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->gl_post_ms = ms;
  });
}

int pcaone_gpu_gl_timing(pcaone_ctx* c, double* posterior_ms) {
  return guarded(c, [&] {
    PG_REQUIRE(posterior_ms, PCAONE_EBADARG, "null timing output");
    *posterior_ms = c->gl_post_ms;
  });
}

int pcaone_gpu_gl_grm(pcaone_ctx* c, const double* U, const double* S, const double* V, uint32_t k, double* C,
                      double* evecs, double* svals) {
  return guarded(c, [&] {
    PG_REQUIRE(c->loaded && c->dense && c->d_P, PCAONE_ESTATE, "no likelihoods loaded");
    PG_REQUIRE(U, PCAONE_EBADARG, "the GRM needs the factors U, S, V");
    double *dUS = nullptr, *dV = nullptr;
    upload_factors(c, U, S, V, k, &dUS, &dV);
    gl_grm(c, dUS, dV, (int)k, C, evecs, svals);
  });
}

}  // extern "C"
