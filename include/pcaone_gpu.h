/*
 * pcaone_gpu.h -- C ABI of the B200 (sm_100a) implementation of PCAone's randomized-SVD
 * hot path.
 *
 * The reference PCAone is a C++ command-line tool with no library or FFI; its internal
 * seams on this path are the Data readers (src/Data.hpp:15-20), the RSVD operators
 * RsvdOpData::computeGandH / computeUSV (src/Halko.hpp:7-42, src/Halko.cpp:45-270), the EM
 * updates Data::fit_with_pi / pcangsd_standardize_E (src/Data.cpp:247-343) and the LD r2
 * loop (src/LD.cpp:419-442). Each entry point below replaces one of those seams; the
 * comment on each names the reference code it stands in for.
 *
 * Conventions
 *  - Every function returns an int status (pcaone_status); 0 is success. No exception or
 *    C++ type crosses this boundary. pcaone_gpu_last_error() returns the message of the
 *    last failure on a context.
 *  - Host buffers are owned by the caller. Matrices are column-major FP64 (as Eigen's
 *    Mat2D in the reference). No host pointer is retained after a call returns.
 *  - The context owns all device memory, streams and CUDA graphs on one GPU. Calls on one
 *    context must be serialised by the caller (one context per host thread).
 *  - "SNP order" after pcaone_gpu_permute() is the permuted order: SNP j of the context is
 *    original SNP perm[j] (as G = G * P in src/RSVD.hpp:63-79).
 */
#ifndef PCAONE_GPU_H_
#define PCAONE_GPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pcaone_ctx pcaone_ctx;

typedef enum {
  PCAONE_OK = 0,
  PCAONE_EBADARG = 1,   /* invalid argument or size (e.g. k + oversamples > samples) */
  PCAONE_EOOM = 2,      /* device allocation failed */
  PCAONE_ECUDA = 3,     /* CUDA runtime / launch error */
  PCAONE_ETIMEOUT = 4,  /* a bounded device wait gave up */
  PCAONE_ENUMERIC = 5,  /* factorisation failed (non-positive Gram matrix) */
  PCAONE_ESTATE = 6,    /* call out of order (e.g. rsvd before load_bed) */
  PCAONE_ENODEV = 7     /* no usable sm_100 device / extension not built for it */
} pcaone_status;

typedef enum {
  PCAONE_PREC_FP32 = 0,  /* FP32 SIMT decode-GEMMs (the plain FP32 GPU path) */
  PCAONE_PREC_MIXED = 1, /* tcgen05 int8 decode-GEMMs: genotypes as exact unsigned 8-bit
                            integers, the sketch as three signed 8-bit fixed-point pieces per
                            column (21 bits below the column maximum), exact int32 accumulation */
  PCAONE_PREC_FP64 = 2,  /* FP64 SIMT decode-GEMMs (algorithm-matched FP64 run) */
  PCAONE_PREC_BF16 = 3   /* tcgen05 BF16 decode-GEMMs, split BF16 hi+lo sketch, FP32 accum */
} pcaone_precision;

/* Create / destroy a context on CUDA device `device`. Replaces nothing in the reference
 * (the reference has no device); errors here map to cao.error (src/Logger.hpp:96-105). */
int pcaone_gpu_create(int device, pcaone_ctx** out);
int pcaone_gpu_destroy(pcaone_ctx* ctx);
const char* pcaone_gpu_last_error(const pcaone_ctx* ctx);

/* Upload the packed SNP-major PLINK records (nsnps x ceil(nsamples/4) bytes, the .bed body
 * without its 3-byte magic) and compute the integer allele counts on the device.
 * Replaces FileBed::read_all (src/FilePlink.cpp:29-131) up to the F estimate. */
int pcaone_gpu_load_bed(pcaone_ctx* ctx, const uint8_t* packed, uint64_t nsnps,
                        uint32_t nsamples);

/* The same genotypes kept in host memory: the records are copied into a pinned host buffer
 * owned by the context (the caller's array is not retained) and the counts are computed
 * from them. pcaone_gpu_rsvd (Halko and winSVD at the FP32, FP64 and mixed precisions) then
 * copies one run of windows at a time into one of two device slots of slot_bytes each
 * (0: 1 GiB) on a copy stream, while the products of the other slot run; the missing-entry
 * lists and per-SNP vectors stay on the device. For matrices beyond device memory.
 * Replaces the out-of-core reader FileBed::read_block_initial / read_block_update
 * (src/FilePlink.cpp:133-294) over the block plan of Data::prepare (src/Data.cpp:16-72); the
 * winSVD windows are the plan's blocks when pcaone_rsvd_opts.block_snps is set, and Halko
 * sums its products over blocks. pcaone_gpu_permute permutes the host records.
 * pcaone_gpu_gram_product and pcaone_gpu_product with transpose = 0 (Z^T B) also run over
 * the streamed blocks (FP32, FP64, mixed; the IRAM operator of the out-of-core Arnoldi,
 * src/Arnoldi.cpp:18-46). Z B (transpose = 1), LD, residual, pseudo-likelihood and the
 * allocation-free product need resident genotypes and return PCAONE_ESTATE on a streamed
 * matrix. */
int pcaone_gpu_load_bed_host(pcaone_ctx* ctx, const uint8_t* packed, uint64_t nsnps,
                             uint32_t nsamples, uint64_t slot_bytes);

/* Per-SNP integer counts in the current SNP order: a1x2[j] = 2*n(00) + n(10) (twice the sum
 * of BED2GENO over non-missing entries, src/FilePlink.cpp:36-57) and nonmiss[j] = number of
 * non-missing samples. Bit-exact. */
int pcaone_gpu_counts(pcaone_ctx* ctx, uint32_t* a1x2, uint32_t* nonmiss);

/* Allele frequencies F_j = (a1x2/2)/nonmiss as FP64 (src/FilePlink.cpp:53-56), bit-exact
 * with the reference's accumulation. */
int pcaone_gpu_allele_freq(pcaone_ctx* ctx, double* F);

/* Permute SNP records on the device (or in the host buffer of streamed genotypes): new SNP
 * j = old SNP perm[j] (src/RSVD.hpp:63-79 for the in-core winSVD shuffle). perm is a host
 * array of nsnps int32 indices. */
int pcaone_gpu_permute(pcaone_ctx* ctx, const int32_t* perm);

/* The reference's in-core SNP shuffle (std::shuffle of 0..n-1 with a default-seeded
 * std::default_random_engine, src/RSVD.hpp:67-70), written to perm (host, n int32). */
int pcaone_shuffle_perm(uint64_t n, int32_t* perm);

/* The structured SNP order of the reference's out-of-core winSVD (-m with --svd 2 without -S):
 * permute_plink (src/FilePlink.cpp:298-405) deals the SNPs of each read buffer (buffer_gb GB,
 * --buffer, default 2) round-robin to nbands contiguous bands. perm[new] = old, n int32, for
 * pcaone_gpu_permute. */
int pcaone_plink_perm(uint64_t nsnps, uint32_t nsamples, uint32_t buffer_gb, uint32_t nbands, int32_t* perm);

/* The reference's sketch Omega (nrow x ncol, column-major FP64) drawn from
 * std::default_random_engine seeded with `seed` through std::normal_distribution (rand=1)
 * or uniform(-1,1) (rand=0), as RsvdOpData::initOmg (src/Halko.cpp:14-22). */
int pcaone_omega(int seed, int rand, uint64_t nrow, uint32_t ncol, double* out);

typedef struct {
  int32_t k;            /* -k/--pc */
  int32_t oversamples;  /* effective oversampling (the reference uses max(--oversamples,k)) */
  int32_t maxp;         /* -p/--maxp: epochs 0..maxp */
  int32_t svd;          /* 1 = Halko sSVD (--svd 1), 2 = window-based winSVD (--svd 2) */
  int32_t bands;        /* -w/--batches (winSVD windows); ignored for svd = 1 */
  int32_t precision;    /* pcaone_precision */
  int32_t standardize;  /* divide by sqrt(ploidy F (1-F)) (Data::standardize_E) */
  int32_t ploidy;       /* 2, or 1 with --haploid */
  int32_t seed;         /* --seed for Omega */
  int32_t rand;         /* --rand: 1 Gaussian, 0 uniform */
  double tol;           /* --tol-rsvd */
  int32_t verbose;      /* print per-epoch "running of epoch" lines to stdout */
  int32_t profile;      /* time every decode-GEMM launch with CUDA events (gemm_ms) */
  int32_t carry_window_state; /* winSVD: keep the window sums H1/H2 of the previous call on
                                 this context, as successive computeUSV calls on one
                                 FancyRsvdOpData do (src/Halko.hpp:68, src/Halko.cpp:159-163);
                                 0 starts from zero like a fresh process */
  int32_t block_snps;   /* winSVD with the out-of-core block plan of -m (src/Data.cpp:27-71):
                           windows of block_snps SNPs (the reference's blocks) and band_factor
                           blocks per band (FancyRsvdOpData::computeGandH out-of-core,
                           src/Halko.cpp:228-269); 0 = the in-core windows of ceil(M / bands) */
  int32_t band_factor;
} pcaone_rsvd_opts;

typedef struct {
  int32_t epochs;        /* epochs run (the reference's "stops at epoch") */
  int32_t omega_updates; /* Omega re-orthonormalisations performed */
  double last_diff;      /* last 1 - mev(U, Upre) */
  double gpu_ms;         /* device time of the whole call (CUDA events) */
  double gemm_ms;        /* device time inside the decode-GEMM kernels (with opts.profile) */
  int64_t kernel_launches;
  int64_t gemm_launches;
  double epilogue_ms;    /* with opts.profile: centring/sparse epilogues and B-operand packing */
  double update_ms;      /* with opts.profile: Omega re-orthonormalisations (QR, signs, flip) */
  double tail_ms;        /* with opts.profile: per-epoch QR of G, B, small SVD, mev */
  double host_ms;        /* with opts.profile: device idle while the host runs the epoch tail's
                            small SVD and convergence test */
  uint64_t h2d_bytes;    /* streamed genotypes (pcaone_gpu_load_bed_host): record bytes copied
                            to the device slots by the call; 0 when resident */
} pcaone_rsvd_report;

/* Run Halko (svd=1) or window-based (svd=2) RSVD on the loaded genotypes: the epoch loop of
 * RsvdOpData::computeUSV (src/Halko.cpp:45-95) with NormalRsvdOpData::computeGandH
 * (src/Halko.cpp:97-126) or FancyRsvdOpData::computeGandH (src/Halko.cpp:153-226).
 * Outputs (host, column-major): U (nsamples x k), S (k), V (nsnps x k, current SNP order).
 * Any output pointer may be NULL. report may be NULL. */
int pcaone_gpu_rsvd(pcaone_ctx* ctx, const pcaone_rsvd_opts* opts, double* U, double* S,
                    double* V, pcaone_rsvd_report* report);

/* One standardised product on the loaded genotypes, the blockwise matvec of
 * ArnoldiOpData::perform_op (src/Arnoldi.cpp:18-46) and each half of
 * NormalRsvdOpData::computeGandH (src/Halko.cpp:123-124):
 *   transpose = 0: out (nsnps x ncols)    = Z^T B, B is nsamples x ncols;
 *   transpose = 1: out (nsamples x ncols) = Z B,   B is nsnps x ncols;
 * Z_ij = s_j (x_ij - F_j), missing -> 0, s_j = 1/sqrt(ploidy F_j (1-F_j)) when standardize
 * (src/Data.cpp:290-299) else 1. Column-major FP64 host buffers; ncols <= 64. */
int pcaone_gpu_product(pcaone_ctx* ctx, int precision, int transpose, int standardize,
                       int ploidy, const double* B, uint32_t ncols, double* out);

/* Y = Z (Z^T X) for X (nsamples x ncols, column-major FP64 host), Y the same shape: the
 * matrix operation of the IRAM solver, ArnoldiOpData::perform_op (src/Arnoldi.cpp:18-46),
 * summed over the whole matrix as one block. Both decode-GEMMs and their centring/missing-
 * entry epilogues run back to back on the device (Z^T X never leaves it); Z, precision,
 * standardize and ploidy as for pcaone_gpu_product; ncols <= 64. */
int pcaone_gpu_gram_product(pcaone_ctx* ctx, int precision, int standardize, int ploidy,
                            const double* X, uint32_t ncols, double* Y);

/* EMU imputation step, Data::fit_with_pi EMU branch (src/Data.cpp:272-287): every missing
 * genotype of the loaded matrix takes the centred value
 *   e_ij = clip(sum_t U_it S_t V_jt, -F_j, 1 - F_j)
 * in place of 0 in all later products and RSVD runs, until pcaone_gpu_clear_imputed or a
 * new load/permutation. U (nsamples x k), S (k), V (nsnps x k, current SNP order) are host
 * column-major buffers, e.g. the outputs of the previous pcaone_gpu_rsvd call.
 * reference_index = 1 reproduces the reference's index semantics after the in-core
 * shuffle: the clip bounds, and the standardisation of later runs while imputation is
 * active, read F at the SNP's permuted position (F in load order) as src/Data.cpp:283 and
 * :296 do; 0 uses each SNP's own F. */
int pcaone_gpu_fit_emu(pcaone_ctx* ctx, const double* U, const double* S, const double* V,
                       uint32_t k, int reference_index);
int pcaone_gpu_clear_imputed(pcaone_ctx* ctx);

/* Windowed LD r2 on the loaded genotypes (current SNP order, normally unpermuted):
 * run_ld_stuff flow A (src/LD.cpp:444-468) with ld_r2_big (src/LD.cpp:419-442). The centred
 * genotypes (missing -> 0) are projected off U when U is given, G = (I - U U^T) G, and for
 * window w (lead SNP ws[w], we[w] SNPs including the lead) r2[off_w + t - 1] =
 * (G_i.G_{i+t} / (|G_i| |G_{i+t}|))^2 for t = 1..we[w]-1, off_w = sum_{v<w} (we[v] - 1).
 * U: nsamples x k column-major host matrix as read by the caller, or NULL (no projection).
 * r2: host array of sum_w (we[w] - 1) floats. The genotype cross products are exact
 * integer counts (bit-plane popcounts); the projection is FP64. */
int pcaone_gpu_ld_r2(pcaone_ctx* ctx, const double* U, uint32_t k, const int64_t* ws,
                     const int32_t* we, uint64_t nwin, float* r2);

/* The same pairs as pcaone_gpu_ld_r2 with r2 in FP64: the values the pruning
 * (ld_prune_big / ld_prune_small, src/LD.cpp:141-242: r2 > --ld-r2) and clumping
 * (ld_clump_single_pheno, src/LD.cpp:299-367: r2 >= --clump-r2, on the unprojected matrix,
 * U = NULL) decisions compare. */
int pcaone_gpu_ld_r2_f64(pcaone_ctx* ctx, const double* U, uint32_t k, const int64_t* ws,
                         const int32_t* we, uint64_t nwin, double* r2);

/* Device time (CUDA events on the context's stream) of the last pcaone_gpu_ld_r2 /
 * pcaone_gpu_ld_r2_f64 call on packed genotypes through the tensor-core band Gram: all its
 * device work after the projection factors are in place (diagonal, code tiling, band Gram)
 * and the band-Gram launch alone, in ms; -1 when that call took another path. */
int pcaone_gpu_ld_timing(pcaone_ctx* ctx, double* device_ms, double* gram_ms);

/* LD flow B, first half: the residual matrix of Data::write_residuals (src/Data.cpp:196-245)
 * for the SNPs snp0 .. snp0 + nsnp - 1 of the current order. R_ij = Gc_ij - sum_t U_it S_t
 * V_jt with Gc the centred genotypes (BED2GENO - F_j, missing -> 0; not standardised), or Gc
 * itself when U is NULL (--ld-stats 1); every SNP's residuals are then centred over the
 * samples (FP64) and stored as float. U (nsamples x k), S (k) and V (nsnp x k, the loadings
 * of those SNPs) are column-major host matrices; out (host) receives nsnp rows of nsamples
 * floats, the layout of the .residuals body. */
int pcaone_gpu_residuals(pcaone_ctx* ctx, const double* U, const double* S, const double* V, uint32_t k,
                         uint64_t snp0, uint64_t nsnp, float* out);

/* LD flow B, second half: load a dense SNP-major float matrix (nsnps rows of nsamples, the
 * .residuals body after its 8-byte header) and centre every row in FP64 as FileBin::read_all
 * does (src/FileBinary.cpp:21-30). pcaone_gpu_ld_r2 with U = NULL then gives the r2 of
 * ld_r2_big (src/LD.cpp:419-442) on it. */
int pcaone_gpu_load_dense(pcaone_ctx* ctx, const float* X, uint64_t nsnps, uint32_t nsamples);

/* PCAngsd on genotype likelihoods (Beagle input). Load the likelihood pairs: P is the
 * reference's 2N x M column-major FP64 matrix of the first two likelihoods per sample and
 * site (FileBeagle::read_all, src/FileBeagle.cpp:121-143; the third is implied as
 * 1 - P0 - P1). The context then holds no packed codes; pcaone_gpu_rsvd runs on the dense
 * posterior matrix E built by pcaone_gpu_gl_update. */
int pcaone_gpu_load_gl(pcaone_ctx* ctx, const double* P, uint64_t nsnps, uint32_t nsamples);
/* The same from FP32 likelihood pairs (the device keeps them in FP32 either way); half the
 * host memory of the FP64 form for large inputs. */
int pcaone_gpu_load_gl_f32(pcaone_ctx* ctx, const float* P, uint64_t nsnps, uint32_t nsamples);

/* PCAngsd on PLINK input (-b with --pcangsd): switch the loaded packed genotypes, in the
 * current SNP order (after any pcaone_gpu_permute), to the likelihood mode as
 * FileBed::read_all does with --pcangsd (src/FilePlink.cpp:89-115): pseudo-likelihood pairs
 * per genotype (RR -> (1, 0), AA -> (0, 0), RA -> (0, 1), missing -> (0.333333, 0.333333)),
 * F = the genotype allele frequencies (src/FilePlink.cpp:36-64, no likelihood EM), and the
 * initial matrix E = BED2GENO - F with missing -> 0 (not standardised). pcaone_gpu_rsvd and
 * pcaone_gpu_gl_update then run the PCAngsd EM loop on it. */
int pcaone_gpu_bed_to_gl(pcaone_ctx* ctx);

/* Allele frequencies by EM from the likelihoods, emMAF_with_GL (src/Utils.cpp:501-531):
 * F0 = 0.25, at most maxiter sweeps, stops when sqrt(mean((F - F_prev)^2)) < tolmaf.
 * F (host, nsnps) and iters (number of sweeps run) may be NULL. */
int pcaone_gpu_gl_freq(pcaone_ctx* ctx, int maxiter, double tolmaf, double* F, int* iters);

/* Rebuild E_ij = E[g | likelihoods, pt_ij] - 2 F_j for every sample and site:
 * pt_ij = F_j when U is NULL (initial E, src/FileBeagle.cpp:121-143), else
 * pt_ij = clip((sum_t U_it S_t V_jt + 2 F_j) / 2, 1e-4, 1 - 1e-4), Data::fit_with_pi
 * PCAngsd branch (src/Data.cpp:249-270). V (nsnps x k) row j is the loading used for
 * site j (the caller applies the reference's index semantics). */
int pcaone_gpu_gl_update(pcaone_ctx* ctx, const double* U, const double* S, const double* V,
                         uint32_t k);

/* Device time in ms of the posterior kernel of the last pcaone_gpu_gl_update call (CUDA
 * events on the context's stream; the factor upload excluded). Measurement only; no
 * reference counterpart. */
int pcaone_gpu_gl_timing(pcaone_ctx* ctx, double* posterior_ms);

/* PCAngsd genetic relationship matrix, the stage after the EM loop (src/Halko.cpp:317-331
 * with Data::pcangsd_standardize_E, src/Data.cpp:301-343). The posterior E is rebuilt in FP64
 * from U, S and V as pcaone_gpu_gl_update does (same arguments and index semantics), site j
 * divided by sqrt(2 F_j (1 - F_j)) when that exceeds 1e-9, and per sample
 * Dc_i = sum_j sum_g (g - 2F_j)^2 P(g) / (2 F_j (1 - F_j)). Then C = E E^T / M with
 * diag(C) = Dc / M: nsamples x nsamples, column-major FP64 host (symmetric), or NULL.
 * evecs (nsamples x nsamples column-major host, or NULL) and svals (nsamples, or NULL): the
 * singular vectors and values of C that the reference's JacobiSVD gives, i.e. the
 * eigenvectors of the symmetric C ordered by decreasing |eigenvalue| and those |eigenvalues|.
 * The sign of each vector is arbitrary, as in any SVD. */
int pcaone_gpu_gl_grm(pcaone_ctx* ctx, const double* U, const double* S, const double* V, uint32_t k,
                      double* C, double* evecs, double* svals);

/* Allocation-free Z^T B for callers that cannot let a library call cudaMalloc: code running
 * inside another framework's device memory pool, or an outer solver loop that must not
 * allocate per call (e.g. an eigensolver using this product as its operator). It has no
 * counterpart in the reference. Same result as pcaone_gpu_product(ctx, PCAONE_PREC_FP32,
 * 0, standardize, ploidy, ...) but B (nsamples x ncols) and out (nsnps x ncols) are
 * column-major FP64 DEVICE buffers owned by the caller, and the call allocates nothing: its
 * scratch is one fixed 64 MiB device array inside the library (held by every GPU that loads
 * the library until exit). Problems needing more than that (nsamples*ncols*12 +
 * nsnps*ncols*4 bytes plus alignment) are rejected with PCAONE_EBADARG. The matrix must be
 * loaded and pcaone_gpu_product or pcaone_gpu_rsvd must have been called on it once (that
 * builds the missing-genotype list; PCAONE_ESTATE otherwise). The first call on a device
 * resolves the array's device address (cudaGetSymbolAddress), so make that first call before
 * any stream capture. All calls share the array and overwrite what they use; calls that
 * overlap on the GPU race and must be serialised by the caller.
 * Stream semantics: the call runs on the context's own stream, which is created non-blocking
 * and is not ordered after any of the caller's streams. Every kernel that writes d_B must
 * therefore be complete before the call (e.g. synchronise the producing stream first); the
 * call synchronises its stream before returning, so d_out is complete when it returns. */
int pcaone_gpu_product_t_noalloc(pcaone_ctx* ctx, int standardize, int ploidy, const double* B,
                                 uint32_t ncols, double* out);

#ifdef __cplusplus
}
#endif

#endif /* PCAONE_GPU_H_ */
