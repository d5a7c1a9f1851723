// Streamed genotypes: the packed matrix stays in pinned host memory and the RSVD copies it
// to the device one run of windows at a time, for matrices beyond device memory. This is the
// device side of the reference's out-of-core mode (-m; FileBed::read_block_initial /
// read_block_update, src/FilePlink.cpp:133-294, over the block plan of Data::prepare,
// src/Data.cpp:16-72): each window is one block of the plan, read again in every epoch.
//
// Two device slots each hold up to slot_windows consecutive windows: their SNP-major records
// (a plain copy of host rows), the sample-major copy per window and, for the int8 back end,
// the tiled copies of both products. While the products of one slot run on the library's
// stream, the copy stream fills the other slot with the next windows (H2D copy, transposition
// and tiling), ordered by two events per slot: `ready` (contents complete) and `idle` (the
// last product reading the slot). The missing-entry lists and the per-SNP vectors stay on
// the device; they are built from two staging passes when the window layout is set.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.hpp"

namespace pg {

void require_resident(const pcaone_ctx* c, const char* what) {
  PG_REQUIRE(!c->streamed, PCAONE_ESTATE,
             std::string(what) + " needs the genotypes resident on the device (pcaone_gpu_load_bed); "
                                 "they are streamed from host memory");
}

namespace {

uint64_t slot_key(const pcaone_ctx* c, bool tiles) {
  return (c->generation << 24) ^ ((uint64_t)c->win.bands << 44) ^ (uint64_t)c->win.blocksize ^
         (tiles ? (1ull << 63) : 0ull);
}

struct SlotSizes {
  size_t rec, recT, t1, t2;  // bytes per window
};

SlotSizes slot_sizes(const pcaone_ctx* c, bool tiles) {
  SlotSizes z{(size_t)c->win.blocksize * c->pitch, (size_t)c->Npad * c->win.pitch, 0, 0};
  if (tiles) i8_tile_bytes(c, &z.t1, &z.t2);
  return z;
}

// Stage windows [b0, b1) into slot s on the copy stream.
void stage(pcaone_ctx* c, int s, int b0, int b1, bool tiles) {
  auto& S = c->slot[s];
  const SlotSizes z = slot_sizes(c, tiles);
  const uint64_t s0 = c->win.start[b0], s1 = c->win.stop[b1 - 1];
  PG_CUDA(cudaStreamWaitEvent(c->copy_stream, S.idle, 0));
  S.key = 0;  // invalid until the host has queued the whole fill
  PG_CUDA(cudaMemcpyAsync(S.rec, c->h_bed + s0 * c->pitch, (size_t)(s1 - s0) * c->pitch, cudaMemcpyHostToDevice,
                          c->copy_stream));
  launch_transpose_run(c, c->copy_stream, S.rec, s1 - s0, b1 - b0, S.recT);
  if (tiles)
    for (int b = b0; b < b1; ++b)
      i8_tile_window(c, c->copy_stream, S.rec + (size_t)(c->win.start[b] - s0) * c->pitch,
                     (int64_t)(c->win.stop[b] - c->win.start[b]), S.recT + (size_t)(b - b0) * z.recT,
                     S.t1 + (size_t)(b - b0) * z.t1, S.t2 + (size_t)(b - b0) * z.t2);
  PG_CUDA(cudaEventRecord(S.ready, c->copy_stream));
  S.b0 = b0;
  S.b1 = b1;
  S.key = slot_key(c, tiles);
  c->streamed_h2d += (s1 - s0) * c->pitch;
}

int slot_holding(const pcaone_ctx* c, int b, bool tiles) {
  const uint64_t key = slot_key(c, tiles);
  for (int s = 0; s < 2; ++s)
    if (c->slot[s].key == key && c->slot[s].b0 <= b && b < c->slot[s].b1) return s;
  return -1;
}

}  // namespace

void stream_counts(pcaone_ctx* c) {
  // staged through slot 0's record buffer (at least 256 MB here; the RSVD may grow it)
  if (c->copy_stream) PG_CUDA(cudaStreamSynchronize(c->copy_stream));
  const uint64_t rows = std::max<uint64_t>(1, std::min<uint64_t>(c->M, (uint64_t(256) << 20) / c->pitch));
  uint8_t* buf = (uint8_t*)scratch(c, "stream_rec0", rows * c->pitch);
  c->slot[0].key = 0;
  c->slot[0].rec = buf;
  for (uint64_t r0 = 0; r0 < c->M; r0 += rows) {
    const uint64_t n = std::min(rows, c->M - r0);
    PG_CUDA(cudaMemcpyAsync(buf, c->h_bed + r0 * c->pitch, n * c->pitch, cudaMemcpyHostToDevice, c->stream));
    launch_counts_rows(c, c->stream, buf, n, r0);
  }
  launch_freq(c);
  PG_CUDA(cudaStreamSynchronize(c->stream));
}

void stream_missing_snp(pcaone_ctx* c) {
  if (c->miss_snp_valid) return;
  if (c->copy_stream) PG_CUDA(cudaStreamSynchronize(c->copy_stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  missing_snp_scan(c);
  const uint64_t rows = std::max<uint64_t>(1, std::min<uint64_t>(c->M, (uint64_t(256) << 20) / c->pitch));
  uint8_t* buf = (uint8_t*)scratch(c, "stream_rec0", rows * c->pitch);
  c->slot[0].key = 0;
  c->slot[0].rec = buf;
  for (uint64_t r0 = 0; r0 < c->M; r0 += rows) {
    const uint64_t n = std::min(rows, c->M - r0);
    PG_CUDA(cudaMemcpyAsync(buf, c->h_bed + r0 * c->pitch, n * c->pitch, cudaMemcpyHostToDevice, c->stream));
    launch_missing_snp_rows(c, c->stream, buf, n, r0);
  }
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->miss_snp_valid = true;
}

void stream_prepare(pcaone_ctx* c, int bands, uint64_t blocksize, bool tiles) {
  PG_REQUIRE(c->streamed && c->h_bed, PCAONE_ESTATE, "no streamed genotypes");
  // buffers may be reallocated below: no fill of a slot may still be in flight
  if (c->copy_stream) PG_CUDA(cudaStreamSynchronize(c->copy_stream));
  set_window_layout(c, bands, blocksize);
  const int nwin = c->win.bands;
  const SlotSizes z = slot_sizes(c, tiles);
  const size_t per = z.rec + z.recT + z.t1 + z.t2;
  const int W = (int)std::max<size_t>(1, std::min<size_t>((size_t)nwin, c->slot_budget / per));
  if (W != c->slot_windows) {
    c->slot_windows = W;
    c->slot[0].key = c->slot[1].key = 0;
  }
  for (int s = 0; s < 2; ++s) {
    auto& S = c->slot[s];
    const std::string t = std::to_string(s);
    uint8_t* rec = (uint8_t*)scratch(c, "stream_rec" + t, (size_t)W * z.rec);
    uint8_t* recT = (uint8_t*)scratch(c, "stream_recT" + t, (size_t)W * z.recT);
    uint8_t* t1 = tiles ? (uint8_t*)scratch(c, "stream_t1" + t, (size_t)W * z.t1) : S.t1;
    uint8_t* t2 = tiles ? (uint8_t*)scratch(c, "stream_t2" + t, (size_t)W * z.t2) : S.t2;
    if (rec != S.rec || recT != S.recT || t1 != S.t1 || t2 != S.t2) S.key = 0;  // reallocated
    S.rec = rec;
    S.recT = recT;
    S.t1 = t1;
    S.t2 = t2;
    if (!S.ready) PG_CUDA(cudaEventCreateWithFlags(&S.ready, cudaEventDisableTiming));
    if (!S.idle) PG_CUDA(cudaEventCreateWithFlags(&S.idle, cudaEventDisableTiming));
  }
  if (c->miss_snp_valid && c->miss_ws_valid) return;
  // The lists from two passes over the windows through slot 0 (on the library's stream, after
  // any fill or product of the slot): pass 1 fills the by-SNP entries and counts the (window,
  // sample) entries, pass 2 fills those.
  PG_CUDA(cudaStreamWaitEvent(c->stream, c->slot[0].ready, 0));
  PG_CUDA(cudaStreamWaitEvent(c->stream, c->slot[0].idle, 0));
  auto& S = c->slot[0];
  S.key = 0;
  const bool snp = !c->miss_snp_valid;
  if (snp) missing_snp_scan(c);
  const uint64_t rows = (uint64_t)nwin * c->Npad;
  int64_t* cnt = (int64_t*)scratch(c, "miss_ws_cnt", rows * 8);
  uint64_t* d_base = (uint64_t*)scratch(c, "miss_ws_base", nwin * 8);
  PG_CUDA(cudaMemcpyAsync(d_base, c->win.start.data(), nwin * 8, cudaMemcpyHostToDevice, c->stream));
  for (int pass = 0; pass < 2; ++pass) {
    for (int b0 = 0; b0 < nwin; b0 += W) {
      const int b1 = std::min(nwin, b0 + W);
      const uint64_t s0 = c->win.start[b0], s1 = c->win.stop[b1 - 1];
      PG_CUDA(cudaMemcpyAsync(S.rec, c->h_bed + s0 * c->pitch, (size_t)(s1 - s0) * c->pitch,
                              cudaMemcpyHostToDevice, c->stream));
      if (pass == 0 && snp) launch_missing_snp_rows(c, c->stream, S.rec, s1 - s0, s0);
      launch_transpose_run(c, c->stream, S.rec, s1 - s0, b1 - b0, S.recT);
      if (pass == 0)
        launch_missing_ws_count(c, c->stream, S.recT, b0, b1 - b0, cnt);
      else
        launch_missing_ws_fill(c, c->stream, S.recT, b0, b1 - b0, d_base);
    }
    if (pass == 0) {
      c->d_miss_ws_ptr = (int64_t*)scratch(c, "d_miss_ws_ptr", (rows + 1) * 8);
      const int64_t total = scan_counts(c, cnt, rows, c->d_miss_ws_ptr);
      c->d_miss_ws_idx = (int32_t*)scratch(c, "d_miss_ws_idx", std::max<int64_t>(total, 1) * 4);
    }
  }
  PG_CUDA(cudaStreamSynchronize(c->stream));
  c->miss_snp_valid = c->miss_ws_valid = true;
  c->miss_ws_val_valid = false;
}

int stream_acquire(pcaone_ctx* c, int b, bool tiles) {
  int s = slot_holding(c, b, tiles);
  if (s < 0) {
    s = c->cur_slot == 0 ? 1 : 0;
    stage(c, s, b, std::min(c->win.bands, b + c->slot_windows), tiles);
  }
  PG_CUDA(cudaStreamWaitEvent(c->stream, c->slot[s].ready, 0));
  c->cur_slot = s;
  return c->slot[s].b1;
}

void stream_prefetch(pcaone_ctx* c, int b, bool tiles) {
  if (b >= c->win.bands) b = 0;  // the next epoch starts again at the first window
  if (slot_holding(c, b, tiles) >= 0) return;
  const int s = c->cur_slot == 0 ? 1 : 0;
  stage(c, s, b, std::min(c->win.bands, b + c->slot_windows), tiles);
}

void stream_release(pcaone_ctx* c) {
  if (c->cur_slot >= 0) PG_CUDA(cudaEventRecord(c->slot[c->cur_slot].idle, c->stream));
}

const uint8_t* stream_codes(const pcaone_ctx* c, int b) {
  const auto& S = c->slot[c->cur_slot];
  return S.rec + (size_t)(c->win.start[b] - c->win.start[S.b0]) * c->pitch;
}

const uint8_t* stream_codesT(const pcaone_ctx* c, int b) {
  const auto& S = c->slot[c->cur_slot];
  return S.recT + (size_t)(b - S.b0) * c->Npad * c->win.pitch;
}

void stream_load(pcaone_ctx* c, const uint8_t* packed, size_t slot_bytes) {
  if (c->copy_stream) PG_CUDA(cudaStreamSynchronize(c->copy_stream));
  const size_t bytes = (size_t)c->M * c->pitch;
  if (c->h_bed_bytes < bytes) {
    if (c->h_bed) PG_CUDA(cudaFreeHost(c->h_bed));
    c->h_bed = nullptr;
    c->h_bed_bytes = 0;
    PG_CUDA(cudaMallocHost(&c->h_bed, bytes));
    c->h_bed_bytes = bytes;
  }
  if (!c->copy_stream) PG_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  // records at the device pitch, padding codes 11 past the samples (as k_fix_padding sets
  // them in the resident copy), copied by a few host threads
  const uint32_t bpr = c->bpr, pitch = c->pitch, r = c->N & 3u;
  const uint8_t last_or = r ? (uint8_t)(0xFFu << (2 * r)) : 0;
  const uint64_t M = c->M;
  const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (uint64_t j = M * t / nt; j < M * (t + 1) / nt; ++j) {
        uint8_t* dst = c->h_bed + j * pitch;
        std::memcpy(dst, packed + j * bpr, bpr);
        dst[bpr - 1] |= last_or;
        std::memset(dst + bpr, 0xFF, pitch - bpr);
      }
    });
  for (auto& x : th) x.join();
  c->slot_budget = slot_bytes ? slot_bytes : (size_t(1) << 30);
  c->slot[0].key = c->slot[1].key = 0;
  c->cur_slot = -1;
  c->streamed = true;
}

// In-core shuffle of streamed records: row j of the new order = row perm[j] of the old one.
void stream_permute(pcaone_ctx* c, const int32_t* perm) {
  const size_t bytes = (size_t)c->M * c->pitch;
  std::vector<uint8_t> old(c->h_bed, c->h_bed + bytes);
  const uint64_t M = c->M;
  const uint32_t pitch = c->pitch;
  const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (uint64_t j = M * t / nt; j < M * (t + 1) / nt; ++j)
        std::memcpy(c->h_bed + j * pitch, old.data() + (size_t)perm[j] * pitch, pitch);
    });
  for (auto& x : th) x.join();
  c->slot[0].key = c->slot[1].key = 0;
}

void stream_free(pcaone_ctx* c) {
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  for (auto& S : c->slot) {
    if (S.ready) cudaEventDestroy(S.ready);
    if (S.idle) cudaEventDestroy(S.idle);
    S = pcaone_ctx::StreamSlot();
  }
  if (c->h_bed) cudaFreeHost(c->h_bed);
  c->h_bed = nullptr;
  c->h_bed_bytes = 0;
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  c->copy_stream = nullptr;
}

}  // namespace pg
