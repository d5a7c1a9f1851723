// Randomized SVD driver on device-resident packed genotypes: the epoch loop of
// RsvdOpData::computeUSV (src/Halko.cpp:45-95) with the Halko schedule of
// NormalRsvdOpData::computeGandH (src/Halko.cpp:97-125) or the window schedule of
// FancyRsvdOpData::computeGandH (src/Halko.cpp:153-226).
//
// Differences of form (not of result) from the reference:
//  * thin QR is CholeskyQR2 in FP64 instead of Householder; the Householder column signs,
//    which steer the winSVD trajectory through flipOmg, are recovered exactly from the
//    final Q of each Omega update (kernels_update.cu, modified LU of its top block);
//  * B = R^-T H^T is never formed: its SVD comes from CholeskyQR2 of B^T = H R^-1 and a
//    one-sided Jacobi SVD of the l x l triangular factor on the host.
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <random>

#include "epilogue.hpp"
#include "linalg.hpp"
#include "rsvd.hpp"
#include "update.hpp"

namespace pg {

namespace {
// Omega column-major N x l (host layout of the reference) -> row-major Npad x l FP64 copies
// (padding rows zero) and an optional FP32 copy.
__global__ void k_omega_layout(const double* __restrict__ cm, int64_t N, int l, int64_t npad, double* __restrict__ O,
                               double* __restrict__ O2, float* __restrict__ Of) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= npad * l) return;
  const int64_t i = t / l, j = t - i * l;
  const double v = i < N ? cm[j * N + i] : 0.0;
  O[t] = v;
  O2[t] = v;
  if (Of) Of[t] = (float)v;
}

// Row-major n x k (row stride ld) -> column-major n x k.
__global__ void k_to_colmajor(const double* __restrict__ X, int64_t n, int k, int ld, double* __restrict__ Y) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t j = t / n, i = t - j * n;
  Y[t] = X[i * ld + j];
}
}  // namespace

// ---------------------------------------------------------------- host helpers
// One-sided Jacobi SVD of a small square matrix A (n x n, row-major): A = U diag(s) V^T,
// singular values sorted in decreasing order. U, V row-major n x n.
void jacobi_svd(int n, const double* A, double* U, double* s, double* V) {
  // work on column-major copies so every column is contiguous; the three dot products of a
  // pair use four partial sums each, which breaks the add-latency chains
  std::vector<double> a((size_t)n * n), v((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) a[(size_t)j * n + i] = A[(size_t)i * n + j];
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n - 1; ++p) {
      double* ap = a.data() + (size_t)p * n;
      double* vp = v.data() + (size_t)p * n;
      for (int q = p + 1; q < n; ++q) {
        double* aq = a.data() + (size_t)q * n;
        double* vq = v.data() + (size_t)q * n;
        double al[4] = {0, 0, 0, 0}, be[4] = {0, 0, 0, 0}, ga[4] = {0, 0, 0, 0};
        int i = 0;
        for (; i + 4 <= n; i += 4)
          for (int u = 0; u < 4; ++u) {
            al[u] += ap[i + u] * ap[i + u];
            be[u] += aq[i + u] * aq[i + u];
            ga[u] += ap[i + u] * aq[i + u];
          }
        for (; i < n; ++i) {
          al[0] += ap[i] * ap[i];
          be[0] += aq[i] * aq[i];
          ga[0] += ap[i] * aq[i];
        }
        const double alpha = (al[0] + al[1]) + (al[2] + al[3]), beta = (be[0] + be[1]) + (be[2] + be[3]);
        const double gamma = (ga[0] + ga[1]) + (ga[2] + ga[3]);
        if (gamma == 0.0) continue;
        double conv = std::fabs(gamma) / std::sqrt(alpha * beta);
        off = std::max(off, conv);
        if (conv < 1e-15) continue;
        double zeta = (beta - alpha) / (2.0 * gamma);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
        for (int r = 0; r < n; ++r) {
          const double x = ap[r], y = aq[r];
          ap[r] = cs * x - sn * y;
          aq[r] = sn * x + cs * y;
          const double xv = vp[r], yv = vq[r];
          vp[r] = cs * xv - sn * yv;
          vq[r] = sn * xv + cs * yv;
        }
      }
    }
    if (off < 1e-15) break;
  }
  std::vector<double> norms(n);
  for (int j = 0; j < n; ++j) {
    double acc = 0;
    for (int i = 0; i < n; ++i) acc += a[(size_t)j * n + i] * a[(size_t)j * n + i];
    norms[j] = std::sqrt(acc);
  }
  std::vector<int> ord(n);
  for (int j = 0; j < n; ++j) ord[j] = j;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return norms[x] > norms[y]; });
  for (int jj = 0; jj < n; ++jj) {
    int j = ord[jj];
    s[jj] = norms[j];
    for (int i = 0; i < n; ++i) {
      U[(size_t)i * n + jj] = norms[j] > 0 ? a[(size_t)j * n + i] / norms[j] : (i == jj ? 1.0 : 0.0);
      V[(size_t)i * n + jj] = v[(size_t)j * n + i];
    }
  }
}

// ---------------------------------------------------------------- engine
template <typename T>
struct Engine {
  pcaone_ctx* c;
  pcaone_rsvd_opts o;
  int N, l, k;
  int64_t M, Npad;
  GemmFnT<T> gemm;

  double *Omg, *Omg2, *wsum, *G, *H, *H1, *H2, *Tb, *Rg, *Rb, *Dsig, *Ucur, *Upre, *Ck;
  // epoch tail outputs kept apart from the epoch body's buffers (so the next body may run
  // while the host finishes the tail): Q of the sketch B^T and Q_B^T U_pre (l x k)
  double *Tq, *Xk;
  // G of the even and the odd epochs: the epoch body writes G of its parity, so an epoch body
  // queued ahead of the host's decision leaves the previous epoch's G (the output V needs it)
  double* Gbuf[2];
  T* OmgT;   // Omega as the B operand of the first product (alias of Omg for FP64)
  int* d_status;
  unsigned* upd_cnt;
  const double* Fcent;  // centring frequencies of the epilogues (zeros for the dense E)

  Engine(pcaone_ctx* c_, const pcaone_rsvd_opts& o_, GemmFnT<T> g) : c(c_), o(o_), gemm(g) {
    N = (int)c->N;
    M = (int64_t)c->M;
    Npad = c->Npad;
    Fcent = c->dense ? c->d_zero : c->d_F;
    k = o.k;
    l = o.k + o.oversamples;
    auto d = [&](const char* name, size_t n) { return (double*)scratch(c, name, n * sizeof(double)); };
    Omg = d("r_omg", Npad * l);
    Omg2 = d("r_omg2", Npad * l);
    wsum = d("r_wsum", l);
    Gbuf[0] = G = d("r_G", (size_t)c->Mpad * l);
    Gbuf[1] = d("r_G1", (size_t)c->Mpad * l);
    H = d("r_H", Npad * l);
    H1 = d("r_H1", Npad * l);
    H2 = d("r_H2", Npad * l);
    Tb = d("r_Tb", Npad * l);
    Tq = d("r_Tq", Npad * l);
    Xk = d("r_Xk", (size_t)kLmax * kLmax);
    Rg = d("r_Rg", l * l);
    Rb = d("r_Rb", l * l);
    Dsig = d("r_D", l);
    Ucur = d("r_Ucur", Npad * k);
    Upre = d("r_Upre", Npad * k);
    Ck = d("r_Ck", (size_t)kLmax * kLmax);
    d_status = (int*)scratch(c, "r_status", sizeof(int));
    PG_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), c->stream));
    upd_cnt = (unsigned*)scratch(c, "upd_cnt", 4 * sizeof(unsigned));
    PG_CUDA(cudaMemsetAsync(upd_cnt, 0, 4 * sizeof(unsigned), c->stream));
    if (std::is_same<T, double>::value)
      OmgT = reinterpret_cast<T*>(Omg);
    else
      OmgT = (T*)scratch(c, "r_omgT", Npad * l * sizeof(T));
  }

  float* omg_float() { return std::is_same<T, float>::value ? reinterpret_cast<float*>(OmgT) : nullptr; }

  void init_omega() {
    std::vector<double> cm((size_t)N * l);
    omega_host(o.seed, o.rand, N, l, cm.data());
    double* d_cm = (double*)scratch(c, "r_omg_cm", cm.size() * 8);
    PG_CUDA(cudaMemcpyAsync(d_cm, cm.data(), cm.size() * 8, cudaMemcpyHostToDevice, c->stream));
    const int64_t tot = Npad * l;
    k_omega_layout<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(d_cm, N, l, Npad, Omg, Omg2, omg_float());
    PG_CHECK_LAUNCH();
    c->launches++;
    colsum(c, Omg, l, N, wsum);
    PG_CUDA(cudaStreamSynchronize(c->stream));  // the host vector goes out of scope
    gemm.omega_changed(c, Omg, l, Npad);
  }

  // Y = Z (Z^T X) over the windows of the current layout (the Gram product of streamed
  // genotypes, window run by window run): X (N x l, column-major host) takes Omega's place,
  // the window sums go to H, and Y (column-major host) is read back.
  void gram_windows(const double* X, double* Y, double* Gt = nullptr) {
    std::vector<double> cm(X, X + (size_t)N * l);
    double* d_cm = (double*)scratch(c, "r_omg_cm", cm.size() * 8);
    PG_CUDA(cudaMemcpyAsync(d_cm, cm.data(), cm.size() * 8, cudaMemcpyHostToDevice, c->stream));
    const int64_t tot = Npad * l;
    k_omega_layout<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(d_cm, N, l, Npad, Omg, Omg2, omg_float());
    PG_CHECK_LAUNCH();
    c->launches++;
    colsum(c, Omg, l, N, wsum);
    gemm.omega_changed(c, Omg, l, Npad);
    G = Gbuf[0];
    zero(c, H, Npad * l);
    process_windows(0, c->win.bands, H);
    double* cmaj = (double*)scratch(c, "r_out_cm", (size_t)Npad * l * 8);
    k_to_colmajor<<<(unsigned)(((int64_t)N * l + 255) / 256), 256, 0, c->stream>>>(H, N, l, l, cmaj);
    PG_CHECK_LAUNCH();
    c->launches++;
    if (Y) PG_CUDA(cudaMemcpyAsync(Y, cmaj, (size_t)N * l * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));  // cm (host) and Y complete
    if (Gt) {  // Z^T X of every window (G rows, current SNP order), column-major
      double* gm = (double*)scratch(c, "r_out_g", (size_t)M * l * 8);
      k_to_colmajor<<<(unsigned)((M * l + 255) / 256), 256, 0, c->stream>>>(G, M, l, l, gm);
      PG_CHECK_LAUNCH();
      c->launches++;
      PG_CUDA(cudaMemcpyAsync(Gt, gm, (size_t)M * l * 8, cudaMemcpyDeviceToHost, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
  }

  // Omega = flipOmg(Omega2, thinQ(Householder QR of H)); Omega2 = Omega. With H2, the sketch
  // is H = H1 + H2 (written to H); otherwise H1 is the sketch itself.
  void update_omega(double* H1in, const double* H2in) {
    UpdateArgs a;
    a.H1 = H2in ? H1in : nullptr;
    a.H2 = H2in;
    a.H = H2in ? H : H1in;
    a.Q = Tb;
    a.Omg = Omg;
    a.Omg2 = Omg2;
    a.Omgf = omg_float();
    a.bt1 = gemm.omega_bt ? gemm.omega_bt(c, l, &a.bt_half) : nullptr;
    a.kpad = Npad;
    a.wsum = wsum;
    a.part = (double*)scratch(c, "upd_part", update_part_doubles(l) * 8);
    a.R1 = (double*)scratch(c, "upd_R1", (size_t)l * l * 8);
    a.R2 = (double*)scratch(c, "upd_R2", (size_t)l * l * 8);
    a.D = Dsig;
    a.mult = (double*)scratch(c, "upd_mult", (size_t)l * 8);
    a.counters = upd_cnt;
    a.status = d_status;
    a.N = N;
    a.l = l;
    fused_update(c, a);
    if (!a.bt1) gemm.omega_changed(c, Omg, l, Npad);
  }

  // G rows of window b and accumulation of Z_b G_b into Ht.
  void process_window(int b, double* Ht) {
    const int64_t s = (int64_t)c->win.start[b], e = (int64_t)c->win.stop[b], m = e - s;
    // product 1: D1 = R_b^T Omega
    int ks1 = gemm.ksplit(c, m, N, l);
    T* D1 = (T*)scratch(c, "r_D1", (size_t)ks1 * m * l * sizeof(T));
    const uint8_t* codes = c->dense ? nullptr : c->streamed ? stream_codes(c, b) : c->d_bed + s * (int64_t)c->pitch;
    timed([&] { gemm.p1(c, codes, c->pitch, s, m, N, OmgT, l, ks1, D1); });
    EpiP1 p1;
    p1.start = s;
    p1.m = m;
    p1.l = l;
    p1.ksplit = ks1;
    p1.F = Fcent;
    p1.scale = c->d_scale;
    p1.wsum = wsum;
    p1.omega = Omg;
    p1.omega_f = omg_float();
    p1.miss_ptr = c->d_miss_snp_ptr;
    p1.miss_idx = c->d_miss_snp_idx;
    p1.miss_val = c->imputed ? c->d_miss_snp_val : nullptr;
    p1.G = G;
    T* B2 = (T*)scratch(c, "r_B2", (size_t)round_up(c->win.blocksize, 256) * l * sizeof(T));
    double* h0 = (double*)scratch(c, "r_h0", l * 8);
    if (gemm.b2_bt) p1.bt2 = gemm.b2_bt(c, l, &p1.kpad2, &p1.bt_half);
    if (gemm.b2_qmax) p1.qmax = gemm.b2_qmax(c, l);
    // FP32 copy of the window's G rows for the second gather (FP32 engines)
    float* Gf = std::is_same<T, float>::value
                    ? (float*)scratch(c, "r_Gf", (size_t)round_up(c->win.blocksize, 256) * l * sizeof(float))
                    : nullptr;
    p1.Gf = Gf;
    timed([&] {
      launch_prep<T>(c, p1, D1, B2, h0);
      if (!p1.bt2) gemm.b2_ready(c, B2, l, m);
    }, 1);
    // product 2: D2 = R_b B2
    int ks2 = gemm.ksplit(c, N, m, l);
    T* D2 = (T*)scratch(c, "r_D2", (size_t)ks2 * N * l * sizeof(T));
    const uint8_t* codesT = c->dense      ? nullptr
                            : c->streamed ? stream_codesT(c, b)
                                          : c->d_bedT + (int64_t)b * Npad * c->win.pitch;
    timed([&] { gemm.p2(c, codesT, c->win.pitch, b, N, m, B2, l, ks2, D2); });
    EpiP2 p2;
    p2.b0 = b;
    p2.b1 = b + 1;
    p2.nwin = c->win.bands;
    p2.n = N;
    p2.npad = Npad;
    p2.l = l;
    p2.ksplit = ks2;
    p2.F = Fcent;
    p2.scale = c->d_scale;
    p2.G = G;
    p2.Gf = Gf;
    p2.g_start = s;
    p2.h0 = h0;
    p2.miss_ptr = c->d_miss_ws_ptr;
    p2.miss_idx = c->d_miss_ws_idx;
    p2.miss_val = c->imputed ? c->d_miss_ws_val : nullptr;
    p2.miss_w = ws_weights();
    p2.H = Ht;
    timed([&] { launch_accum<T>(c, p2, D2); }, 1);
  }

  // Windows [b0, b1) into Ht as one pair of products (back ends with window runs): the
  // first product covers the run's SNPs, its epilogue writes G, the FP32 rows of the second
  // gather and the run's window operand B2 in the padded layout of the second product, whose
  // K then runs over all the run's SNPs. The same sums as window by window, in another order.
  void process_run(int b0, int b1, double* Ht) {
    const int64_t s = (int64_t)c->win.start[b0], e = (int64_t)c->win.stop[b1 - 1], m = e - s;
    const int nw = b1 - b0;
    const int64_t rows1 = gemm.seg_rows1(c), k2 = gemm.seg_k2(c);
    const int ks1 = gemm.ksplit_seg(c, 1, nw, l);
    // D1 rows per split: the padded windows of the back end, or exactly the run's SNPs for the
    // dense matrix (whose windows are contiguous rows without padding)
    const int64_t d1rows = c->dense ? m : nw * rows1;
    T* D1 = (T*)scratch(c, "r_D1", (size_t)ks1 * std::max<int64_t>(d1rows, nw * rows1) * l * sizeof(T));
    timed([&] { gemm.p1_seg(c, b0, b1, OmgT, l, ks1, D1); });
    EpiP1 p1;
    p1.start = s;
    p1.m = m;
    p1.l = l;
    p1.ksplit = ks1;
    p1.wlen = (int64_t)c->win.blocksize;
    p1.d1_ws = rows1;
    p1.b2_ws = k2;
    p1.d1_rows = d1rows;
    p1.F = Fcent;
    p1.scale = c->d_scale;
    p1.wsum = wsum;
    p1.omega = Omg;
    p1.omega_f = omg_float();
    p1.miss_ptr = c->d_miss_snp_ptr;
    p1.miss_idx = c->d_miss_snp_idx;
    p1.miss_val = c->imputed ? c->d_miss_snp_val : nullptr;
    p1.G = G;
    T* B2 = (T*)scratch(c, "r_B2", (size_t)nw * k2 * l * sizeof(T));
    double* h0 = (double*)scratch(c, "r_h0", l * 8);
    p1.qmax = gemm.b2_qmax ? gemm.b2_qmax(c, l) : nullptr;
    float* Gf = (float*)scratch(c, "r_Gf", (size_t)round_up(m, 256) * l * sizeof(float));
    p1.Gf = Gf;
    timed([&] {
      launch_prep<T>(c, p1, D1, B2, h0);
      gemm.b2_seg(c, B2, l, b0, b1);
    }, 1);
    const int ks2 = gemm.ksplit_seg(c, 2, nw, l);
    T* D2 = (T*)scratch(c, "r_D2", (size_t)ks2 * N * l * sizeof(T));
    timed([&] { gemm.p2_seg(c, b0, b1, B2, l, ks2, D2); });
    EpiP2 p2;
    p2.b0 = b0;
    p2.b1 = b1;
    p2.nwin = c->win.bands;
    p2.n = N;
    p2.npad = Npad;
    p2.l = l;
    p2.ksplit = ks2;
    p2.F = Fcent;
    p2.scale = c->d_scale;
    p2.G = G;
    p2.Gf = Gf;
    p2.g_start = s;
    p2.h0 = h0;
    p2.miss_ptr = c->d_miss_ws_ptr;
    p2.miss_idx = c->d_miss_ws_idx;
    p2.miss_val = c->imputed ? c->d_miss_ws_val : nullptr;
    p2.miss_w = ws_weights();
    p2.H = Ht;
    timed([&] { launch_accum<T>(c, p2, D2); }, 1);
  }

  // Windows [b0, b1) into Ht: as runs of at most kRunRows padded rows of the first product
  // when the back end batches windows, else one window at a time.
  static constexpr int64_t kRunRows = int64_t(1) << 22;
  void process_windows(int b0, int b1, double* Ht) {
    if (c->streamed) {  // by device slots: the windows of one slot, while the next is filled
      const bool tiles = o.precision == PCAONE_PREC_MIXED;
      for (int b = b0; b < b1;) {
        const int held = stream_acquire(c, b, tiles), e = std::min(b1, held);
        stream_prefetch(c, held, tiles);
        if (gemm.p1_seg) {
          const int per = (int)std::max<int64_t>(1, kRunRows / gemm.seg_rows1(c));
          for (int r = b; r < e; r += per) process_run(r, std::min(e, r + per), Ht);
        } else {
          for (int r = b; r < e; ++r) process_window(r, Ht);
        }
        stream_release(c);
        b = e;
      }
      return;
    }
    if (!gemm.p1_seg) {
      for (int b = b0; b < b1; ++b) process_window(b, Ht);
      return;
    }
    const int per = (int)std::max<int64_t>(1, kRunRows / gemm.seg_rows1(c));
    for (int b = b0; b < b1; b += per) process_run(b, std::min(b1, b + per), Ht);
  }

  // Weights s_j (e_ij + F_j) of the (window, sample) missing entries for the accumulation
  // gather, built once a run when imputed values are set (scale and F are fixed within it).
  double* ws_w = nullptr;
  const double* ws_weights() {
    if (!c->imputed || !c->miss_ws_val_valid || c->n_missing == 0) return nullptr;
    if (!ws_w) {
      ws_w = (double*)scratch(c, "r_ws_w", (size_t)c->n_missing * 8);
      compute_ws_weights(c, Fcent, ws_w);
    }
    return ws_w;
  }

  int bandsize = 1;
  int updates = 0;

  // With opts.profile, bracket each decode-GEMM launch with CUDA events on the launching
  // stream; the elapsed times are summed into gemm_ms after each epoch.
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  std::vector<int> ev_cat;
  size_t ev_used = 0;
  double cat_ms[4] = {0, 0, 0, 0};
  template <typename F>
  void timed(F&& f, int cat = 0) {
    if (!o.profile) {
      f();
      return;
    }
    if (ev_cat.size() <= ev_used) ev_cat.resize(ev_used + 1);
    ev_cat[ev_used] = cat;
    if (ev_used == evs.size()) {
      cudaEvent_t a, b;
      PG_CUDA(cudaEventCreate(&a));
      PG_CUDA(cudaEventCreate(&b));
      evs.push_back({a, b});
    }
    PG_CUDA(cudaEventRecord(evs[ev_used].first, c->stream));
    f();
    PG_CUDA(cudaEventRecord(evs[ev_used].second, c->stream));
    ev_used++;
  }
  void collect_times() {
    if (!ev_used) return;
    PG_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < ev_used; ++i) {
      float ms = 0.f;
      PG_CUDA(cudaEventElapsedTime(&ms, evs[i].first, evs[i].second));
      cat_ms[ev_cat[i]] += ms;
      if (ev_cat[i] == 0) c->gemm_ms_accum += ms;
    }
    ev_used = 0;
  }
  ~Engine() {
    for (auto& e : evs) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    for (auto& e : steady_exec)
      if (e) cudaGraphExecDestroy(e);
  }

  // Steady epochs as one CUDA graph. Once the schedule stops depending on the epoch (the
  // winSVD from 2^pi >= bands on: every window run and every Omega update the same; Halko from
  // its second update on), the epoch body is launched as a graph: run once directly (buffers
  // sized), then captured once for each epoch parity (each writes G of its parity) and
  // replayed after that. The epoch tail, with its host round
  // trip, stays outside. Used by the tensor-core back ends when no per-launch profile is asked.
  cudaGraphExec_t steady_exec[2] = {nullptr, nullptr};  // by epoch parity (G of that parity)
  int steady_seen = 0, steady_updates = 0;
  uint64_t steady_launches = 0, steady_gemm_launches = 0;
  bool graphs_failed = false;
  bool graphs_on() const {
    static const bool disabled = std::getenv("PCAONE_NO_GRAPHS") != nullptr;
    return !disabled && !graphs_failed && !o.profile &&
           (o.precision == PCAONE_PREC_MIXED || o.precision == PCAONE_PREC_BF16) && !c->dense && !c->streamed;
  }
  bool steady_epoch(int pi) const {
    return o.svd == 1 ? pi >= 2 : (std::pow(2.0, pi) >= o.bands && o.block_snps == 0);
  }
  void run_epoch(int pi) {
    auto body = [&] {
      if (o.svd == 1)
        epoch_halko(pi);
      else
        epoch_winsvd(pi);
    };
    const int par = pi & 1;
    G = Gbuf[par];
    if (!graphs_on() || !steady_epoch(pi)) {
      body();
      return;
    }
    if (steady_exec[par]) {  // replay, with the host-side counters the body would have advanced
      PG_CUDA(cudaGraphLaunch(steady_exec[par], c->stream));
      updates += steady_updates;
      c->launches += steady_launches;
      c->gemm_launches += steady_gemm_launches;
      return;
    }
    if (steady_seen++ == 0) {  // first steady epoch: direct, sizes every buffer it touches
      body();
      return;
    }
    const int u0 = updates;
    const int64_t l0 = c->launches, g0 = c->gemm_launches;
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        body();
      } catch (...) {
        ok = false;
      }
      cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
      ok = ok && e == cudaSuccess && graph;
      if (ok) ok = cudaGraphInstantiate(&steady_exec[par], graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
    }
    if (!ok) {  // capture refused: run this epoch and the rest directly (nothing was executed)
      (void)cudaGetLastError();
      for (auto& ex : steady_exec) {
        if (ex) cudaGraphExecDestroy(ex);
        ex = nullptr;
      }
      graphs_failed = true;
      updates = u0;
      c->launches = l0;
      c->gemm_launches = g0;
      body();
      return;
    }
    steady_updates = updates - u0;
    steady_launches = c->launches - l0;
    steady_gemm_launches = c->gemm_launches - g0;
    PG_CUDA(cudaGraphLaunch(steady_exec[par], c->stream));
  }

  void epoch_halko(int pi) {
    if (pi == 0)
      init_omega();
    else {
      timed([&] { update_omega(H, nullptr); }, 2);
      updates++;
    }
    zero(c, H, Npad * l);
    process_windows(0, c->win.bands, H);  // one window, or the blocks of streamed genotypes
  }

  // The in-core schedule runs over the o.bands windows; with the out-of-core block plan the
  // windows are the nblocks blocks and bands start at band_factor blocks (src/Halko.cpp:228-
  // 269); the two coincide for band_factor = 1 and nblocks = bands.
  void epoch_winsvd(int pi) {
    const int bands = o.bands, nwin = c->win.bands, bf = o.block_snps > 0 ? std::max(1, o.band_factor) : 1;
    if (pi == 0) init_omega();
    if (std::pow(2.0, pi) >= bands) {
      zero(c, H1, Npad * l);
      zero(c, H2, Npad * l);
    }
    if (pi == 0) bandsize = bf;
    bandsize = std::min(bandsize * 2, nwin);
    // windows are gathered into runs that share the target sum and end at the next Omega
    // update; each run is processed as a whole before the update reads H1 / H2
    int run0 = 0;
    double* run_target = nullptr;
    for (int b = 0, i = 1; b < nwin; ++b, ++i) {
      double* target = i <= bandsize / 2 ? H1 : H2;
      if (b > run0 && target != run_target) {
        process_windows(run0, b, run_target);
        run0 = b;
      }
      run_target = target;
      const bool adjacent = pi > 0 && (b + 1) == (int)std::pow(2.0, pi - 1) * bf && std::pow(2.0, pi) < bands;
      if ((b + 1) < bandsize && !adjacent) continue;
      if (!((i == bandsize) || (i == bandsize / 2) || adjacent)) continue;
      process_windows(run0, b + 1, run_target);
      run0 = b + 1;
      timed([&] { update_omega(H1, H2); }, 2);
      updates++;
      if (i == bandsize) {
        zero(c, H1, Npad * l);
        i = 0;
      } else {
        zero(c, H2, Npad * l);
      }
    }
    if (run0 < nwin) process_windows(run0, nwin, run_target);
  }

  void run(double* U, double* S, double* V, pcaone_rsvd_report* rep) {
    // zero the FP64 work buffers once so padded rows stay zero; the winSVD window sums are
    // kept from the previous call when asked to and still valid for this shape and data
    const uint64_t key = ((uint64_t)N * 131 + (uint64_t)l) * 1031 + (uint64_t)o.bands + ((uint64_t)o.block_snps << 20) +
                         (c->generation << 40);
    zero(c, H, Npad * l);
    if (!(o.svd == 2 && o.carry_window_state && c->h12_key == key)) {
      zero(c, H1, Npad * l);
      zero(c, H2, Npad * l);
    }
    c->h12_key = o.svd == 2 ? key : 0;
    zero(c, Tb, Npad * l);
    zero(c, Ucur, Npad * k);
    zero(c, Upre, Npad * k);
    int p = o.maxp;
    std::vector<double> ur((size_t)l * l), vr((size_t)l * l), sv(l), ck((size_t)k * k);
    // pinned host copies of the tail's small results (read while the next body may run),
    // kept on the context with their event
    struct {
      double* rb;
      double* xk;
      int* st;
    } pin;
    const size_t pin_bytes = ((size_t)l * l + (size_t)l * k) * 8 + 16;
    if (c->h_pin_bytes < pin_bytes) {
      if (c->h_pin) PG_CUDA(cudaFreeHost(c->h_pin));
      c->h_pin = nullptr;
      c->h_pin_bytes = 0;
      PG_CUDA(cudaMallocHost(&c->h_pin, pin_bytes));
      c->h_pin_bytes = pin_bytes;
    }
    pin.rb = (double*)c->h_pin;
    pin.xk = pin.rb + (size_t)l * l;
    pin.st = (int*)(pin.xk + (size_t)l * k);
    if (!c->ev_tail) PG_CUDA(cudaEventCreateWithFlags(&c->ev_tail, cudaEventDisableTiming));
    cudaEvent_t ev_tail = c->ev_tail;
    double diff = 0.0;
    int epochs = 0;
    bool done = false;
    // Overlap of the epoch tail with the next epoch body. The body of epoch pi + 1 does not
    // read the tail's results (they only decide whether to stop), so once the tail of epoch pi
    // and the read-back of its small results are queued, the body of epoch pi + 1 is queued
    // too and the host runs the l x l SVD and the convergence test meanwhile. If the run stops
    // at pi that body is discarded: the outputs come from the tail's own buffers (Tq, R_G) and
    // from G of epoch pi, which the body of epoch pi + 1 does not write (other parity). The winSVD window sums H1 / H2, which a later call may carry on
    // from, are saved before the body runs ahead and put back when it is discarded. Not with
    // opts.profile (the breakdown measures the waits); PCAONE_NO_OVERLAP turns it off.
    static const bool no_overlap = std::getenv("PCAONE_NO_OVERLAP") != nullptr;
    const bool overlap = !o.profile && !no_overlap;
    bool ran_ahead = false;
    const size_t hbytes = (size_t)Npad * l * 8;
    double* H1s = o.svd == 2 && overlap ? (double*)scratch(c, "r_H1s", hbytes) : nullptr;
    double* H2s = o.svd == 2 && overlap ? (double*)scratch(c, "r_H2s", hbytes) : nullptr;
    // with opts.profile: event pairs around the stretches in which the device waits for the
    // host (the small SVD, and the convergence test up to the next epoch's first launch)
    std::vector<cudaEvent_t> gap_ev;
    bool gap_open = false;
    auto gap_mark = [&](bool begin) {
      if (!o.profile || gap_open == begin) return;
      cudaEvent_t e;
      PG_CUDA(cudaEventCreate(&e));
      PG_CUDA(cudaEventRecord(e, c->stream));
      gap_ev.push_back(e);
      gap_open = begin;
    };
    for (int pi = 0; pi <= p && !done; ++pi) {
      gap_mark(false);  // the previous epoch's host decisions end here
      if (!ran_ahead) run_epoch(pi);
      ran_ahead = false;
      // tail of computeUSV: QR(G) twice, B = R^-T H^T, SVD(B); Q_B^T U_pre for the test
      timed([&] {
        cholqr2_r(c, G, l, M, Rg, d_status);  // Q_G itself only for the output V
        trsm_right_upper(c, H, Rg, l, N, Tq);
        cholqr2(c, Tq, l, N, Tq, Rb, d_status);
        if (pi > 0) cross(c, Tq, l, Upre, k, N, Xk);
      }, 3);
      gap_mark(true);
      const bool tc = o.precision == PCAONE_PREC_MIXED || o.precision == PCAONE_PREC_BF16;
      PG_CUDA(cudaMemcpyAsync(pin.rb, Rb, (size_t)l * l * 8, cudaMemcpyDeviceToHost, c->stream));
      if (pi > 0) PG_CUDA(cudaMemcpyAsync(pin.xk, Xk, (size_t)l * k * 8, cudaMemcpyDeviceToHost, c->stream));
      PG_CUDA(cudaMemcpyAsync(pin.st, d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      pin.st[1] = 0;
      if (tc)  // the tensor-core kernels' bounded-wait flag
        PG_CUDA(cudaMemcpyAsync(pin.st + 1, scratch(c, "tc_err", sizeof(int)), sizeof(int), cudaMemcpyDeviceToHost,
                                c->stream));
      PG_CUDA(cudaEventRecord(ev_tail, c->stream));
      const int updates_before = updates;
      const int64_t launches_before = c->launches, gemm_launches_before = c->gemm_launches;
      const bool may_continue = pi < p || (o.svd == 2 && std::pow(2.0, pi) < o.bands);
      if (overlap && may_continue) {
        if (H1s) {
          PG_CUDA(cudaMemcpyAsync(H1s, H1, hbytes, cudaMemcpyDeviceToDevice, c->stream));
          PG_CUDA(cudaMemcpyAsync(H2s, H2, hbytes, cudaMemcpyDeviceToDevice, c->stream));
        }
        run_epoch(pi + 1);
        ran_ahead = true;
      }
      PG_CUDA(cudaEventSynchronize(ev_tail));
      collect_times();
      PG_REQUIRE(pin.st[1] == 0, PCAONE_ETIMEOUT,
                 "tensor-core decode-GEMM: bounded wait expired (code " + std::to_string(pin.st[1]) + ")");
      PG_REQUIRE(*pin.st == 0, PCAONE_ENUMERIC,
                 "Cholesky factorisation of a sketch Gram matrix failed at column " + std::to_string(*pin.st - 1));
      jacobi_svd(l, pin.rb, ur.data(), sv.data(), vr.data());
      gap_mark(false);
      // Ucur = Q_B Ur[:, :k] (queued after the body that ran ahead; Tq is not one of its buffers)
      PG_CUDA(cudaMemcpyAsync(Ck, ur.data(), ur.size() * 8, cudaMemcpyHostToDevice, c->stream));
      rowmat(c, Tq, l, Ck, l, k, N, Ucur);
      epochs = pi + 1;
      bool keep_going = true, new_pre = true;  // U_pre is kept when the winSVD runs on past convergence
      if (pi > 0) {
        // mev (src/Utils.cpp:192-198) of U = Q_B Ur_k against U_pre: U^T U_pre = Ur_k^T (Q_B^T U_pre)
        // ck (k x k, row-major) = U^T U_pre: ck[i][j] = sum_t Ur[t][i] X[t][j], X = Q_B^T U_pre
        for (int i = 0; i < k; ++i)
          for (int j = 0; j < k; ++j) {
            double acc = 0.0;
            for (int t = 0; t < l; ++t) acc += ur[(size_t)t * l + i] * pin.xk[(size_t)t * k + j];
            ck[(size_t)i * k + j] = acc;
          }
        double acc = 0.0;
        for (int j = 0; j < k; ++j) {
          double nrm = 0.0;
          for (int i = 0; i < k; ++i) nrm += ck[(size_t)i * k + j] * ck[(size_t)i * k + j];
          acc += std::sqrt(nrm);
        }
        diff = 1.0 - acc / k;
        if (o.verbose) printf("running of epoch = %d, diff = %g\n", pi, diff);
        if (diff < o.tol || pi == p) {
          new_pre = false;
          if (o.svd == 2 && std::pow(2.0, pi) < o.bands)
            p = (int)std::log2((double)o.bands);
          else
            keep_going = false;
        }
      }
      if (!keep_going) {
        done = true;
        if (ran_ahead) {  // the body queued ahead is discarded: count only the kept epochs
          updates = updates_before;
          c->launches = launches_before;
          c->gemm_launches = gemm_launches_before;
          if (H1s) {
            PG_CUDA(cudaMemcpyAsync(H1, H1s, hbytes, cudaMemcpyDeviceToDevice, c->stream));
            PG_CUDA(cudaMemcpyAsync(H2, H2s, hbytes, cudaMemcpyDeviceToDevice, c->stream));
          }
        }
        break;
      }
      if (new_pre)
        PG_CUDA(cudaMemcpyAsync(Upre, Ucur, (size_t)Npad * k * 8, cudaMemcpyDeviceToDevice, c->stream));
    }
    // outputs: U = Ucur, S = sigma[:k], V = Q_G Vr[:, :k]
    if (S)
      for (int j = 0; j < k; ++j) S[j] = sv[j];
    // U and V leave the device already column-major (the host layout of the outputs)
    double* cmaj = (double*)scratch(c, "r_out_cm", (size_t)std::max<int64_t>(M, N) * k * 8);
    if (U) {
      k_to_colmajor<<<(unsigned)(((int64_t)N * k + 255) / 256), 256, 0, c->stream>>>(Ucur, N, k, k, cmaj);
      PG_CHECK_LAUNCH();
      PG_CUDA(cudaMemcpyAsync(U, cmaj, (size_t)N * k * 8, cudaMemcpyDeviceToHost, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
    if (V) {
      double* Vd = (double*)scratch(c, "r_V", (size_t)c->Mpad * k * 8);
      PG_CUDA(cudaMemcpyAsync(Ck, vr.data(), vr.size() * 8, cudaMemcpyHostToDevice, c->stream));
      double* Gl = Gbuf[(epochs - 1) & 1];  // G of the last epoch kept; Q_G = G R_G^-1 in place
      trsm_right_upper(c, Gl, Rg, l, M, Gl);
      rowmat(c, Gl, l, Ck, l, k, M, Vd);
      k_to_colmajor<<<(unsigned)((M * k + 255) / 256), 256, 0, c->stream>>>(Vd, M, k, k, cmaj);
      PG_CHECK_LAUNCH();
      PG_CUDA(cudaMemcpyAsync(V, cmaj, (size_t)M * k * 8, cudaMemcpyDeviceToHost, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
    if (rep) {
      rep->epochs = epochs;
      rep->omega_updates = updates;
      rep->last_diff = diff;
      rep->epilogue_ms = cat_ms[1];
      rep->update_ms = cat_ms[2];
      rep->tail_ms = cat_ms[3];
      rep->host_ms = 0.0;
      gap_mark(false);
      if (!gap_ev.empty()) {
        PG_CUDA(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i + 1 < gap_ev.size(); i += 2) {  // (begin, end) pairs
          float ms = 0.f;
          PG_CUDA(cudaEventElapsedTime(&ms, gap_ev[i], gap_ev[i + 1]));
          rep->host_ms += ms;
        }
      }
    }
    for (auto e : gap_ev) cudaEventDestroy(e);
  }
};

// One standardised product through the same kernels as the RSVD (single window).
template <typename T>
void product_t(pcaone_ctx* c, GemmFnT<T> gemm, int transpose, int standardize, int ploidy,
               const double* B, int l, double* out) {
  const int N = (int)c->N;
  const int64_t M = (int64_t)c->M, Npad = c->Npad;
  auto d = [&](const char* name, size_t n) { return (double*)scratch(c, name, n * sizeof(double)); };
  double* G = d("r_G", (size_t)c->Mpad * l);
  double* H = d("r_H", Npad * l);
  double* Bd = d("r_omg", Npad * l);
  double* wsum = d("r_wsum", l);
  double* h0 = d("r_h0", l);
  T* B2 = (T*)scratch(c, "r_B2", (size_t)round_up(c->win.blocksize, 256) * l * sizeof(T));
  std::vector<double> rm;
  if (transpose == 0) {
    rm.assign((size_t)Npad * l, 0.0);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < l; ++j) rm[(size_t)i * l + j] = B[(size_t)j * N + i];
    PG_CUDA(cudaMemcpyAsync(Bd, rm.data(), rm.size() * 8, cudaMemcpyHostToDevice, c->stream));
    T* BT = std::is_same<T, double>::value ? reinterpret_cast<T*>(Bd) : (T*)scratch(c, "r_omgT", Npad * l * sizeof(T));
    if (!std::is_same<T, double>::value) {
      std::vector<float> f(rm.begin(), rm.end());
      PG_CUDA(cudaMemcpyAsync(BT, f.data(), f.size() * 4, cudaMemcpyHostToDevice, c->stream));
      PG_CUDA(cudaStreamSynchronize(c->stream));
    }
    colsum(c, Bd, l, N, wsum);
    gemm.omega_changed(c, Bd, l, Npad);
    const int ks = gemm.ksplit(c, M, N, l);
    T* D1 = (T*)scratch(c, "r_D1", (size_t)ks * M * l * sizeof(T));
    gemm.p1(c, c->d_bed, c->pitch, 0, M, N, BT, l, ks, D1);
    EpiP1 p1;
    p1.start = 0; p1.m = M; p1.l = l; p1.ksplit = ks;
    p1.F = c->d_F; p1.scale = c->d_scale; p1.wsum = wsum; p1.omega = Bd; p1.miss_ptr = c->d_miss_snp_ptr;
    p1.miss_idx = c->d_miss_snp_idx; p1.miss_val = c->imputed ? c->d_miss_snp_val : nullptr; p1.G = G;
    launch_prep<T>(c, p1, D1, B2, h0);
    rm.resize((size_t)M * l);
    PG_CUDA(cudaMemcpyAsync(rm.data(), G, rm.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < M; ++i)
      for (int j = 0; j < l; ++j) out[(size_t)j * M + i] = rm[(size_t)i * l + j];
  } else {
    rm.assign((size_t)M * l, 0.0);
    for (int64_t i = 0; i < M; ++i)
      for (int j = 0; j < l; ++j) rm[(size_t)i * l + j] = B[(size_t)j * M + i];
    PG_CUDA(cudaMemcpyAsync(G, rm.data(), rm.size() * 8, cudaMemcpyHostToDevice, c->stream));
    EpiP1 p1;
    p1.start = 0; p1.m = M; p1.l = l;
    p1.F = c->d_F; p1.scale = c->d_scale; p1.G = G;
    launch_scale_g<T>(c, p1, B2, h0);
    gemm.b2_ready(c, B2, l, M);
    const int ks = gemm.ksplit(c, N, M, l);
    T* D2 = (T*)scratch(c, "r_D2", (size_t)ks * N * l * sizeof(T));
    gemm.p2(c, c->d_bedT, c->win.pitch, 0, N, M, B2, l, ks, D2);
    zero(c, H, Npad * l);
    EpiP2 p2;
    p2.b0 = 0; p2.b1 = 1; p2.nwin = c->win.bands; p2.n = N; p2.npad = Npad; p2.l = l; p2.ksplit = ks;
    p2.F = c->d_F; p2.scale = c->d_scale; p2.G = G; p2.h0 = h0; p2.miss_ptr = c->d_miss_ws_ptr;
    p2.miss_idx = c->d_miss_ws_idx; p2.miss_val = c->imputed ? c->d_miss_ws_val : nullptr; p2.H = H;
    launch_accum<T>(c, p2, D2);
    rm.resize((size_t)N * l);
    PG_CUDA(cudaMemcpyAsync(rm.data(), H, rm.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < l; ++j) out[(size_t)j * N + i] = rm[(size_t)i * l + j];
  }
}

// Y = Z (Z^T X) on the device: the first product and its epilogue give G = Z^T X and the
// window operand s/2 G, which the second product and its epilogue turn into Z G, with no host
// round trip between the two (the matrix operation of ArnoldiOpData::perform_op,
// src/Arnoldi.cpp:18-46, over the whole matrix as one window).
template <typename T>
void gram_t(pcaone_ctx* c, GemmFnT<T> gemm, const double* X, int l, double* Y) {
  const int N = (int)c->N;
  const int64_t M = (int64_t)c->M, Npad = c->Npad;
  auto d = [&](const char* name, size_t n) { return (double*)scratch(c, name, n * sizeof(double)); };
  double* G = d("r_G", (size_t)c->Mpad * l);
  double* H = d("r_H", Npad * l);
  double* Bd = d("r_omg", Npad * l);
  double* wsum = d("r_wsum", l);
  double* h0 = d("r_h0", l);
  T* B2 = (T*)scratch(c, "r_B2", (size_t)round_up(c->win.blocksize, 256) * l * sizeof(T));
  std::vector<double> rm((size_t)Npad * l, 0.0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < l; ++j) rm[(size_t)i * l + j] = X[(size_t)j * N + i];
  PG_CUDA(cudaMemcpyAsync(Bd, rm.data(), rm.size() * 8, cudaMemcpyHostToDevice, c->stream));
  T* BT = std::is_same<T, double>::value ? reinterpret_cast<T*>(Bd) : (T*)scratch(c, "r_omgT", Npad * l * sizeof(T));
  std::vector<float> f;
  if (!std::is_same<T, double>::value) {
    f.assign(rm.begin(), rm.end());
    PG_CUDA(cudaMemcpyAsync(BT, f.data(), f.size() * 4, cudaMemcpyHostToDevice, c->stream));
  }
  colsum(c, Bd, l, N, wsum);
  gemm.omega_changed(c, Bd, l, Npad);
  const int ks1 = gemm.ksplit(c, M, N, l);
  T* D1 = (T*)scratch(c, "r_D1", (size_t)ks1 * M * l * sizeof(T));
  gemm.p1(c, c->d_bed, c->pitch, 0, M, N, BT, l, ks1, D1);
  EpiP1 p1;
  p1.start = 0; p1.m = M; p1.l = l; p1.ksplit = ks1;
  p1.F = c->d_F; p1.scale = c->d_scale; p1.wsum = wsum; p1.omega = Bd; p1.miss_ptr = c->d_miss_snp_ptr;
  p1.miss_idx = c->d_miss_snp_idx; p1.miss_val = c->imputed ? c->d_miss_snp_val : nullptr; p1.G = G;
  if (gemm.b2_bt) p1.bt2 = gemm.b2_bt(c, l, &p1.kpad2, &p1.bt_half);
  if (gemm.b2_qmax) p1.qmax = gemm.b2_qmax(c, l);
  launch_prep<T>(c, p1, D1, B2, h0);
  if (!p1.bt2) gemm.b2_ready(c, B2, l, M);
  const int ks2 = gemm.ksplit(c, N, M, l);
  T* D2 = (T*)scratch(c, "r_D2", (size_t)ks2 * N * l * sizeof(T));
  gemm.p2(c, c->d_bedT, c->win.pitch, 0, N, M, B2, l, ks2, D2);
  zero(c, H, Npad * l);
  EpiP2 p2;
  p2.b0 = 0; p2.b1 = 1; p2.nwin = c->win.bands; p2.n = N; p2.npad = Npad; p2.l = l; p2.ksplit = ks2;
  p2.F = c->d_F; p2.scale = c->d_scale; p2.G = G; p2.h0 = h0; p2.miss_ptr = c->d_miss_ws_ptr;
  p2.miss_idx = c->d_miss_ws_idx; p2.miss_val = c->imputed ? c->d_miss_ws_val : nullptr; p2.H = H;
  launch_accum<T>(c, p2, D2);
  rm.resize((size_t)N * l);
  PG_CUDA(cudaMemcpyAsync(rm.data(), H, rm.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  PG_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < l; ++j) Y[(size_t)j * N + i] = rm[(size_t)i * l + j];
}

// The Gram product on streamed genotypes (the out-of-core matvec of ArnoldiOpData::perform_op,
// src/Arnoldi.cpp:18-46, block by block): the blocks of the Halko plan on streamed data
// (blocks whose slot contents fit the slot budget), each window run staged into a device slot.
// Y = Z Z^T X (Y may be null) and, with Gt, Z^T X itself (the single product on streamed
// genotypes comes out of the same pass over the windows).
void run_gram_streamed(pcaone_ctx* c, int precision, int standardize, int ploidy, const double* X, int l,
                       double* Y, double* Gt = nullptr) {
  PG_REQUIRE(precision != PCAONE_PREC_BF16, PCAONE_EBADARG,
             "the split-BF16 back end needs the genotypes resident on the device");
  PG_REQUIRE((uint32_t)l <= c->N, PCAONE_EBADARG, "more columns than samples");
  uint64_t blocksize = std::max<uint64_t>(kRowPad, c->slot_budget / (4ull * c->pitch) / kRowPad * kRowPad);
  blocksize = std::min<uint64_t>(blocksize, c->M);
  const int bands = (int)((c->M + blocksize - 1) / blocksize);
  stream_prepare(c, bands, blocksize, precision == PCAONE_PREC_MIXED);
  if (c->imputed) compute_imputed_ws(c);
  compute_scale(c, standardize, ploidy);
  pcaone_rsvd_opts o{};
  o.k = l;
  o.oversamples = 0;
  o.svd = 1;
  o.bands = bands;
  o.precision = precision;
  o.ploidy = ploidy;
  if (precision == PCAONE_PREC_FP64) {
    Engine<double> e(c, o, gemm_simt_double());
    e.gram_windows(X, Y, Gt);
  } else if (precision == PCAONE_PREC_FP32) {
    Engine<float> e(c, o, gemm_simt_float());
    e.gram_windows(X, Y, Gt);
  } else if (precision == PCAONE_PREC_MIXED) {
    PG_REQUIRE(tc_supported(c), PCAONE_ENODEV, "tcgen05 path needs an sm_100 device");
    tc_clear_error(c);
    Engine<float> e(c, o, gemm_i8());
    e.gram_windows(X, Y, Gt);
    tc_check_error(c);
  } else {
    throw Error(PCAONE_EBADARG, "unknown precision");
  }
}

void run_gram(pcaone_ctx* c, int precision, int standardize, int ploidy, const double* X, int l, double* Y) {
  PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
  PG_REQUIRE(X && Y && l >= 1 && l <= kLmax, PCAONE_EBADARG, "bad gram-product operands");
  PG_REQUIRE(ploidy == 1 || ploidy == 2, PCAONE_EBADARG, "ploidy must be 1 or 2");
  PG_REQUIRE(!c->dense, PCAONE_ESTATE, "products need packed genotypes (load_bed)");
  if (c->streamed) {
    run_gram_streamed(c, precision, standardize, ploidy, X, l, Y);
    return;
  }
  build_transposed(c, 1);
  build_missing_by_snp(c);
  build_missing_by_window_sample(c);
  if (c->imputed) compute_imputed_ws(c);
  compute_scale(c, standardize, ploidy);
  if (precision == PCAONE_PREC_FP64) {
    gram_t<double>(c, gemm_simt_double(), X, l, Y);
  } else if (precision == PCAONE_PREC_FP32) {
    gram_t<float>(c, gemm_simt_float(), X, l, Y);
  } else if (precision == PCAONE_PREC_MIXED || precision == PCAONE_PREC_BF16) {
    PG_REQUIRE(tc_supported(c), PCAONE_ENODEV, "tcgen05 path needs an sm_100 device");
    tc_clear_error(c);
    gram_t<float>(c, precision == PCAONE_PREC_MIXED ? gemm_i8() : gemm_tc(), X, l, Y);
    tc_check_error(c);
  } else {
    throw Error(PCAONE_EBADARG, "unknown precision");
  }
}

void run_product(pcaone_ctx* c, int precision, int transpose, int standardize, int ploidy,
                 const double* B, int l, double* out) {
  PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
  PG_REQUIRE(B && out && l >= 1 && l <= kLmax, PCAONE_EBADARG, "bad product operands");
  PG_REQUIRE(transpose == 0 || transpose == 1, PCAONE_EBADARG, "transpose must be 0 or 1");
  PG_REQUIRE(ploidy == 1 || ploidy == 2, PCAONE_EBADARG, "ploidy must be 1 or 2");
  PG_REQUIRE(!c->dense, PCAONE_ESTATE, "products need packed genotypes (load_bed)");
  if (c->streamed) {  // Z^T B from a pass over the streamed windows; Z B needs them resident
    if (transpose == 1) require_resident(c, "the product Z B");
    run_gram_streamed(c, precision, standardize, ploidy, B, l, nullptr, out);
    return;
  }
  build_transposed(c, 1);
  build_missing_by_snp(c);
  build_missing_by_window_sample(c);
  if (c->imputed) compute_imputed_ws(c);
  compute_scale(c, standardize, ploidy);
  if (precision == PCAONE_PREC_FP64) {
    product_t<double>(c, gemm_simt_double(), transpose, standardize, ploidy, B, l, out);
  } else if (precision == PCAONE_PREC_FP32) {
    product_t<float>(c, gemm_simt_float(), transpose, standardize, ploidy, B, l, out);
  } else if (precision == PCAONE_PREC_MIXED || precision == PCAONE_PREC_BF16) {
    PG_REQUIRE(tc_supported(c), PCAONE_ENODEV, "tcgen05 path needs an sm_100 device");
    tc_clear_error(c);
    product_t<float>(c, precision == PCAONE_PREC_MIXED ? gemm_i8() : gemm_tc(), transpose, standardize, ploidy, B, l,
                     out);
    tc_check_error(c);
  } else {
    throw Error(PCAONE_EBADARG, "unknown precision");
  }
}

void run_rsvd(pcaone_ctx* c, const pcaone_rsvd_opts& o, double* U, double* S, double* V,
              pcaone_rsvd_report* rep) {
  PG_REQUIRE(c->loaded, PCAONE_ESTATE, "no genotypes loaded");
  PG_REQUIRE(o.k >= 1 && o.oversamples >= 0, PCAONE_EBADARG, "bad k / oversamples");
  const int l = o.k + o.oversamples;
  PG_REQUIRE(l <= kLmax, PCAONE_EBADARG, "k + oversamples must be <= " + std::to_string(kLmax));
  PG_REQUIRE((uint32_t)l <= c->N, PCAONE_EBADARG, "k + oversamples must not exceed the number of samples");
  PG_REQUIRE(o.svd == 1 || o.svd == 2, PCAONE_EBADARG, "svd must be 1 (Halko) or 2 (winSVD)");
  PG_REQUIRE(o.svd == 1 || (o.bands >= 4 && o.bands % 2 == 0), PCAONE_EBADARG,
             "the -w/--batches must be a power of 2 and the minimun is 4.");
  PG_REQUIRE(o.maxp >= 0, PCAONE_EBADARG, "maxp must be >= 0");
  PG_REQUIRE(o.ploidy == 1 || o.ploidy == 2, PCAONE_EBADARG, "ploidy must be 1 or 2");
  PG_REQUIRE(o.block_snps >= 0 && o.band_factor >= 0, PCAONE_EBADARG, "bad block plan");
  // the out-of-core block plan changes only the winSVD windows; Halko's result does not depend
  // on the blocks
  const bool blocks = o.svd == 2 && o.block_snps > 0;
  int bands = o.svd == 1 ? 1 : (blocks ? (int)((c->M + o.block_snps - 1) / o.block_snps) : o.bands);
  uint64_t blocksize = blocks ? (uint64_t)o.block_snps : 0;
  if (c->streamed && o.svd == 1) {
    // Halko on streamed genotypes sums the product over blocks: those of the out-of-core plan
    // when given, else blocks whose slot contents (records, transposed copy, tiles: about
    // four bytes per SNP per packed byte) fit the slot budget
    blocksize = o.block_snps > 0 ? (uint64_t)o.block_snps
                                 : std::max<uint64_t>(kRowPad, c->slot_budget / (4ull * c->pitch) / kRowPad * kRowPad);
    blocksize = std::min<uint64_t>(blocksize, c->M);
    bands = (int)((c->M + blocksize - 1) / blocksize);
  }
  if (c->dense) {
    // dense posterior matrix: already centred and not standardised in the EM steps; the
    // epilogues see F = 0 and s = 2 so that G = E^T Omega and B2 = G exactly
    set_window_layout(c, bands, blocksize);
    build_empty_missing(c);
    std::vector<double> two(c->M, 2.0);
    PG_CUDA(cudaMemcpyAsync(c->d_scale, two.data(), c->M * 8, cudaMemcpyHostToDevice, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    PG_REQUIRE(o.precision != PCAONE_PREC_FP64, PCAONE_EBADARG, "the PCAngsd matrix is FP32");
  } else if (c->streamed) {
    PG_REQUIRE(o.precision != PCAONE_PREC_BF16, PCAONE_EBADARG,
               "the split-BF16 back end needs the genotypes resident on the device");
    stream_prepare(c, bands, blocksize, o.precision == PCAONE_PREC_MIXED);
    if (c->imputed) compute_imputed_ws(c);
    compute_scale(c, o.standardize, o.ploidy);
  } else {
    build_transposed(c, bands, blocksize);
    build_missing_by_snp(c);
    build_missing_by_window_sample(c);
    if (c->imputed) compute_imputed_ws(c);
    compute_scale(c, o.standardize, o.ploidy);
  }
  c->gemm_ms_accum = 0.0;
  const int64_t l0 = c->launches, g0 = c->gemm_launches;
  const uint64_t h2d0 = c->streamed_h2d;
  PG_CUDA(cudaEventRecord(c->ev0, c->stream));
  if (c->dense) {
    Engine<float> e(c, o, gemm_dense_float());
    e.run(U, S, V, rep);
  } else if (o.precision == PCAONE_PREC_FP64) {
    Engine<double> e(c, o, gemm_simt_double());
    e.run(U, S, V, rep);
  } else if (o.precision == PCAONE_PREC_FP32) {
    Engine<float> e(c, o, gemm_simt_float());
    e.run(U, S, V, rep);
  } else if (o.precision == PCAONE_PREC_MIXED || o.precision == PCAONE_PREC_BF16) {
    PG_REQUIRE(tc_supported(c), PCAONE_ENODEV, "tcgen05 path needs an sm_100 device");
    tc_clear_error(c);
    Engine<float> e(c, o, o.precision == PCAONE_PREC_MIXED ? gemm_i8() : gemm_tc());
    e.run(U, S, V, rep);
    tc_check_error(c);  // also covers an epoch body queued ahead and discarded
  } else {
    throw Error(PCAONE_EBADARG, "unknown precision");
  }
  PG_CUDA(cudaEventRecord(c->ev1, c->stream));
  PG_CUDA(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  PG_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  if (rep) {
    rep->gpu_ms = ms;
    rep->gemm_ms = c->gemm_ms_accum;
    rep->kernel_launches = c->launches - l0;
    rep->gemm_launches = c->gemm_launches - g0;
    rep->h2d_bytes = c->streamed_h2d - h2d0;
  }
}

}  // namespace pg
