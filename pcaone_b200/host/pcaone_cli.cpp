// PCAone command-line front end for the B200 implementation: the same flags and output
// files as the reference CLI (src/Cmd.cpp:28-111, src/Main.cpp:44-165) for the modes this
// build covers, with all compute going through the C ABI in include/pcaone_gpu.h.
//
// Covered: PLINK input (-b) with --svd 0 (IRAM: restarted Lanczos on the device gram
// product, host/iram.hpp), --svd 1 (Halko) and --svd 2 (winSVD, in-core shuffle unless
// -S), -k, -p, --ncv, --imaxiter, --itol, -w/--batches/--windows, --oversamples, --seed, --rand, --tol-rsvd, --maf,
// -C/--scale 0 (no standardisation), --haploid, -V, -o, -v; outputs .sigvals .eigvals
// .eigvecs [.loadings .mbim] .eigvecs2 and .log. Options of the reference that belong to
// modes outside this build are recognised and rejected with a clear message and exit 1.
#include <sys/utsname.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>
#include <zlib.h>

#include "../../include/pcaone_gpu.h"
#include "iram.hpp"

namespace {

// ------------------------------------------------------------------ logging (src/Logger.hpp)
struct Log {
  std::ofstream file;
  bool screen = true;
  template <typename... A>
  void print(const A&... a) {
    std::ostringstream s;
    s.precision(6);
    s.setf(std::ios::fixed, std::ios::floatfield);
    (..., (s << a << " "));
    std::string line = s.str();
    if (!line.empty()) line.pop_back();
    if (file.is_open()) file << line << "\n" << std::flush;
    if (screen) std::cout << line << std::endl;
  }
};
Log g_log;

std::string date() {
  auto now = std::chrono::system_clock::now();
  auto t = std::chrono::system_clock::to_time_t(now);
  std::stringstream ss;
  ss << std::put_time(std::localtime(&t), "[%d/%m/%Y-%X]");
  return ss.str();
}

[[noreturn]] void fail(const std::string& msg) {
  if (g_log.file.is_open()) g_log.file << "error: " << msg << "\n";
  std::cerr << "error: " << msg << "\n";
  std::exit(EXIT_FAILURE);
}

// ------------------------------------------------------------------ options (src/Cmd.cpp)
struct Params {
  std::string bfile, beagle, fileout = "pcaone";
  double tolmaf = 1e-6;
  int svd = 2;
  unsigned k = 10, maxp = 20, bands = 64, oversamples = 10, rand = 1, verbose = 1, threads = 12;
  int seed = 101, scale = -1;
  bool noshuffle = false, printv = false, haploid = false, emu = false, pcangsd = false;
  double tol = 1e-4, maf = 0.0, memory = 0.0, tolem = 1e-5;
  unsigned buffer = 2;  // --buffer: GB per read buffer of the out-of-core permutation
  unsigned maxiter = 100;
  unsigned ncv = 20, imaxiter = 1000;  // IRAM (--svd 0): ncv = max(20, 2k + 1) (src/Cmd.cpp:189)
  double itol = 1e-6;
  bool ncv_set = false;
  bool fix_index = false;
  bool print_r2 = false, fix_read_u = false;
  unsigned ld_bp = 0;
  double ld_r2 = 0.0;  // --ld-r2: LD pruning threshold
  // --clump (comma-separated assoc-like files) and its options (src/Cmd.hpp:57-66)
  std::string clump, clump_names = "CHR,BP,P";
  double clump_p1 = 0.0001, clump_p2 = 0.01, clump_r2 = 0.5;
  unsigned clump_bp = 250000;
  std::string fileU, filebim;
  std::string binfile;  // -B/--binary: float32 .residuals matrix (LD flow B input)
  bool ld_write = false;  // -D/--ld: write the .residuals matrix after the PCA
  int ld_stats = 0;       // --ld-stats: 0 ancestry-adjusted residuals, 1 centred genotypes
  int precision = PCAONE_PREC_MIXED;
  bool precision_set = false;
  int device = 0;
  std::string cmdline;
};

const std::set<std::string> kUnsupported = {
    "-c", "--csv", "-g", "--bgen", "--project",
    "--inbreed", "--USV", "--read-V", "--read-S", "--M", "--N",
    "--scale-factor", "--buffer"};

void usage() {
  std::cout << "PCAone (B200 build)\n"
               "Usage: PCAone -b plink [-k 10] [-d 2] [-w 64] [-p 20] [-o pcaone] [-V] [-S]\n"
               "  -b, --bfile      prefix of PLINK .bed/.bim/.fam files\n"
               "  -k, --pc         top k principal components [10]\n"
               "  -d, --svd        1: single-pass RSVD (Halko), 2: window-based RSVD [2]\n"
               "  -p, --maxp       maximum number of power iterations [20]\n"
               "  -w, --batches    number of windows for --svd 2 (alias --windows) [64]\n"
               "  -S, --no-shuffle do not shuffle SNPs for --svd 2\n"
               "      --oversamples, --seed, --rand, --tol-rsvd, --maf, --haploid\n"
               "      --emu        EMU imputation of missing genotypes (--maxiter, --tol-em)\n"
               "      --fix-perm-index  EM steps read each SNP's own F after the shuffle\n"
               "  -C, --scale      0: centre only, 1: standardise (default for PLINK)\n"
               "  LD r2 (flow A): -b plink --read-U pcs.eigvecs -f pcs.mbim --ld-bp BP -R\n"
               "  LD r2 (flow B): -b plink -k K -D (writes .residuals), then\n"
               "                  -B out.residuals -f out.mbim --ld-bp BP -R\n"
               "  LD pruning:     either flow with --ld-r2 R2 instead of -R (.ld.prune.in/.out)\n"
               "  LD clumping:    either flow with --clump a.assoc[,b.assoc] (--clump-names,\n"
               "                  --clump-p1, --clump-p2, --clump-r2, --clump-bp; .pN.clump)\n"
               "      --fix-read-u read U row by row (the reference views it column-major)\n"
               "  -V, --printv     write .loadings and .mbim\n"
               "  -o, --out        output prefix [pcaone]\n"
               "  -v, --verbose    0 silent, 1 screen\n"
               "      --precision  mixed (int8 tensor cores, three-piece sketch; default), bf16 (split\n"
               "                   BF16 tensor cores), fp32 or fp64\n"
               "      --device     CUDA device index [0]\n";
}

Params parse(int argc, char** argv) {
  Params p;
  for (int i = 0; i < argc; ++i) p.cmdline += std::string(argv[i]) + " ";
  if (argc == 1) {
    usage();
    std::exit(EXIT_SUCCESS);
  }
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], val;
    auto eq = a.find('=');
    bool has_eq = a.rfind("--", 0) == 0 && eq != std::string::npos;
    if (has_eq) {
      val = a.substr(eq + 1);
      a = a.substr(0, eq);
    }
    auto next = [&]() -> std::string {
      if (has_eq) return val;
      if (i + 1 >= argc) {
        std::cerr << "Invalid Option Exception: missing_argument\noption: " << a << "\n";
        std::exit(EXIT_FAILURE);
      }
      return argv[++i];
    };
    auto num = [&](const std::string& s) -> double {
      char* end = nullptr;
      double v = std::strtod(s.c_str(), &end);
      if (!end || *end) {
        std::cerr << "Invalid Option Exception: invalid_argument\noption: " << a << "\nvalue:  " << s << "\n";
        std::exit(EXIT_FAILURE);
      }
      return v;
    };
    if (a == "-h" || a == "--help") {
      usage();
      std::exit(EXIT_SUCCESS);
    } else if (a == "-b" || a == "--bfile") p.bfile = next();
    else if (a == "-G" || a == "--beagle") p.beagle = next();
    else if (a == "--pcangsd") p.pcangsd = true;  // implied by Beagle input (src/Cmd.cpp:205)
    else if (a == "--tol-maf") p.tolmaf = num(next());
    else if (a == "-o" || a == "--out") p.fileout = next();
    else if (a == "-k" || a == "--pc") p.k = (unsigned)num(next());
    else if (a == "-d" || a == "--svd") p.svd = (int)num(next());
    else if (a == "--ncv") {
      p.ncv = (unsigned)num(next());
      p.ncv_set = true;
    } else if (a == "--imaxiter") p.imaxiter = (unsigned)num(next());
    else if (a == "--itol") p.itol = num(next());
    else if (a == "-p" || a == "--maxp") p.maxp = (unsigned)num(next());
    else if (a == "-w" || a == "--batches" || a == "--windows") p.bands = (unsigned)num(next());
    else if (a == "-S" || a == "--no-shuffle") p.noshuffle = true;
    else if (a == "--seed") p.seed = (int)num(next());
    else if (a == "--oversamples") p.oversamples = (unsigned)num(next());
    else if (a == "--rand") p.rand = (unsigned)num(next());
    else if (a == "--tol-rsvd") p.tol = num(next());
    else if (a == "--maf") p.maf = num(next());
    else if (a == "-C" || a == "--scale") p.scale = (int)num(next());
    else if (a == "--haploid") p.haploid = true;
    else if (a == "--emu") p.emu = true;
    else if (a == "--maxiter") p.maxiter = (unsigned)num(next());
    else if (a == "--tol-em") p.tolem = num(next());
    else if (a == "--fix-perm-index") p.fix_index = true;
    else if (a == "-R" || a == "--print-r2") p.print_r2 = true;
    else if (a == "--ld-bp") p.ld_bp = (unsigned)num(next());
    else if (a == "--ld-r2") p.ld_r2 = num(next());
    else if (a == "--clump") p.clump = next();
    else if (a == "--clump-names") p.clump_names = next();
    else if (a == "--clump-p1") p.clump_p1 = num(next());
    else if (a == "--clump-p2") p.clump_p2 = num(next());
    else if (a == "--clump-r2") p.clump_r2 = num(next());
    else if (a == "--clump-bp") p.clump_bp = (unsigned)num(next());
    else if (a == "--read-U") p.fileU = next();
    else if (a == "-B" || a == "--binary") p.binfile = next();
    else if (a == "-D" || a == "--ld") p.ld_write = true;
    else if (a == "--ld-stats") p.ld_stats = (int)num(next());
    else if (a == "-f" || a == "--match-bim") p.filebim = next();
    else if (a == "--fix-read-u") p.fix_read_u = true;
    else if (a == "-V" || a == "--printv") p.printv = true;
    else if (a == "-v" || a == "--verbose") p.verbose = (unsigned)num(next());
    else if (a == "-n" || a == "--threads") p.threads = (unsigned)num(next());
    else if (a == "-m" || a == "--memory") p.memory = num(next());
    else if (a == "--buffer") p.buffer = (unsigned)num(next());
    else if (a == "--device") p.device = (int)num(next());
    else if (a == "--precision") {
      p.precision_set = true;
      std::string v = next();
      if (v == "mixed" || v == "int8") p.precision = PCAONE_PREC_MIXED;
      else if (v == "bf16") p.precision = PCAONE_PREC_BF16;
      else if (v == "fp32") p.precision = PCAONE_PREC_FP32;
      else if (v == "fp64") p.precision = PCAONE_PREC_FP64;
      else fail("--precision must be mixed, bf16, fp32 or fp64");
    } else if (kUnsupported.count(a)) {
      fail("option " + a + " belongs to a mode this build does not provide");
    } else {
      std::cerr << "unknown option: " << a << "\n";  // src/Cmd.cpp:125-128
      std::exit(EXIT_FAILURE);
    }
  }
  if (p.bfile.empty() && p.beagle.empty() && p.binfile.empty())
    fail("no input: use -b/--bfile, -G/--beagle or -B/--binary");
  if (p.ld_write && (p.emu || p.pcangsd || p.bfile.empty()))
    fail("-D/--ld writes residuals of a plain PCA of PLINK input in this build");
  if (p.svd != 0 && p.svd != 1 && p.svd != 2) fail("--svd must be 0, 1 or 2 in this build");
  if (!p.ncv_set) p.ncv = std::max(20u, 2 * p.k + 1);
  // the reference's EM modes with --svd 0 fail (src/Data.cpp:277 reads an empty permutation)
  if (p.svd == 0 && (p.emu || p.pcangsd)) fail("--emu / --pcangsd need --svd 1 or 2 in this build");
  if (p.bands < 4 || p.bands % 2 != 0) fail("the -w/--batches must be a power of 2 and the minimun is 4.");
  if (p.maf > 0.5) {
    std::cerr << "warning: '--maf' with a value greater than 0.5 will be converted to 1 - maf.\n";
    p.maf = 1 - p.maf;
  }
  p.oversamples = std::max(p.oversamples, p.k);  // src/Cmd.cpp:190
  // -m/--memory: the reference's out-of-core mode. The packed genotypes stay in host memory and
  // the RSVD streams them to the device by blocks (pcaone_gpu_load_bed_host); what -m changes
  // in the results (the permute_plink SNP order and the block-granular winSVD windows) is
  // reproduced. The reference's own restrictions apply (src/Cmd.cpp:201-212).
  if (p.memory > 0 && p.maf > 0) fail("does not support --maf filters for out-of-core mode yet! ");
  if (p.memory > 0 && (p.emu || p.pcangsd || p.bfile.empty()))
    fail("-m/--memory applies to a plain PCA of PLINK input in this build");
  return p;
}

std::vector<std::string> split(const std::string& s, const char* seps) {
  std::vector<std::string> out;
  size_t b = 0;
  for (size_t q = 0; q <= s.size(); ++q)
    if (q == s.size() || std::strchr(seps, s[q])) {
      out.push_back(s.substr(b, q - b));
      b = q + 1;
    }
  return out;
}

// read_usv (src/Utils.cpp:255-286): values are read row by row into one vector that the
// reference then views as a column-major rows x cols matrix. Returned column-major.
std::vector<double> read_usv(const std::string& path, size_t& rows, size_t& cols, bool row_major) {
  std::ifstream f(path);
  if (!f.is_open()) fail("can not open " + path);
  std::vector<double> v;
  std::string line;
  rows = 0;
  cols = 0;
  while (std::getline(f, line)) {
    auto tok = split(line, "\t");
    if (rows == 0) cols = tok.size();
    else if (tok.size() != cols) fail("the columns are not aligned!\n =>" + path);
    for (auto& t : tok) v.push_back(std::stod(t));
    ++rows;
  }
  if (!row_major) return v;  // reinterpreted column-major, as the reference does
  std::vector<double> cm(v.size());
  for (size_t i = 0; i < rows; ++i)
    for (size_t j = 0; j < cols; ++j) cm[j * rows + i] = v[i * cols + j];
  return cm;
}

size_t count_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f.is_open()) fail("can not open " + path);
  size_t n = 0;
  std::string line;
  while (std::getline(f, line)) ++n;
  return n;
}

void check(pcaone_ctx* ctx, int st, const char* what) {
  if (st != PCAONE_OK) fail(std::string(what) + ": " + pcaone_gpu_last_error(ctx));
}

// Eigen::IOFormat(6, DontAlignCols, "\t", "\n") of a column-major matrix (src/Data.cpp:181).
void write_matrix(std::ostream& o, const double* a, size_t rows, size_t cols) {
  std::ostringstream s;
  s.precision(6);
  for (size_t i = 0; i < rows; ++i) {
    for (size_t j = 0; j < cols; ++j) {
      if (j) s << '\t';
      s << a[j * rows + i];
    }
    if (i + 1 < rows) s << '\n';
  }
  o << s.str();
}

// A coefficient as a stream of precision 6 prints it (std::num_put formats with "%.*g").
inline int fmt_g6(char* b, double v) { return std::snprintf(b, 32, "%.6g", v); }

// Eigen's default `stream << matrix` (IOFormat(): stream precision, aligned columns): every
// coefficient right-aligned to the widest one of the whole matrix, " " between coefficients,
// "\n" between rows, nothing after the last row. rows x cols, element (i, j) at a[i + j * ld].
// The .cov matrix and the rows of the PCAngsd .eigvecs2 are written this way
// (src/Halko.cpp:325, src/Utils.cpp:435).
void write_aligned(std::ostream& o, const double* a, size_t rows, size_t cols, size_t ld) {
  int width = 0;
#pragma omp parallel for reduction(max : width) schedule(static)
  for (long j = 0; j < (long)cols; ++j) {
    char b[32];
    for (size_t i = 0; i < rows; ++i) width = std::max(width, fmt_g6(b, a[i + (size_t)j * ld]));
  }
  std::vector<std::string> lines(rows);
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < (long)rows; ++i) {
    std::string& s = lines[i];
    s.reserve(cols * (width + 1));
    char b[32];
    for (size_t j = 0; j < cols; ++j) {
      if (j) s.push_back(' ');
      const int n = fmt_g6(b, a[i + j * ld]);
      s.append((size_t)(width - n), ' ');
      s.append(b, (size_t)n);
    }
  }
  for (size_t i = 0; i < rows; ++i) {
    o << lines[i];
    if (i + 1 < rows) o << '\n';
  }
}

// Sample names of a Beagle file: every third header token from the fourth on
// (parse_beagle_samples, src/Utils.cpp:407-424).
std::vector<std::string> beagle_samples(const std::string& path) {
  gzFile gz = gzopen(path.c_str(), "rb");
  if (!gz) fail("can not open " + path);
  std::string head;
  std::vector<char> buf(1 << 20);
  while (gzgets(gz, buf.data(), (int)buf.size())) {
    head += buf.data();
    if (!head.empty() && head.back() == '\n') break;
  }
  gzclose(gz);
  std::vector<std::string> names;
  std::istringstream hs(head);
  std::string t;
  for (size_t idx = 0; hs >> t; ++idx)
    if (idx >= 3 && idx % 3 == 0) names.push_back(t);
  return names;
}

}  // namespace

// ---------------------------------------------------------------- LD: r2, pruning, clumping
// SNPld (src/LD.hpp:8-15) of a .bim / .mbim or of an assoc-like file, as get_snp_pos_bim
// reads it (src/LD.cpp:51-77): chromosome runs, positions, the "chr\tpos\tid" strings of the
// .ld.gz text, the raw lines and, from 7-column (.mbim) files, the allele frequencies.
struct SnpLd {
  std::vector<long> pos;
  std::vector<int> end_pos;
  std::vector<std::string> chr, bims, lines;
  std::vector<double> af;
  std::vector<int64_t> ws;  // divide_pos_by_window: lead SNP of each window
  std::vector<int32_t> we;  // and its SNP count (lead included)
};

SnpLd read_snp_ld(const std::string& file, bool header, int ic, int ip, std::string* head = nullptr) {
  std::ifstream fb(file);
  if (!fb.is_open()) fail("can not open " + file);
  SnpLd s;
  std::string line, prev;
  if (header) {
    std::getline(fb, line);
    if (head) *head = line;
  }
  while (std::getline(fb, line)) {
    auto tok = split(line, " \t");
    if ((int)tok.size() <= std::max(ic, ip)) fail("the input file is not valid!\n => " + file);
    if (tok.size() == 7 && !header) s.af.push_back(std::stod(tok[6]));
    if (prev.empty()) s.chr.push_back(tok[ic]);
    if (!prev.empty() && prev != tok[ic]) {
      s.end_pos.push_back((int)s.pos.size() - 1);
      s.chr.push_back(tok[ic]);
    }
    prev = tok[ic];
    s.pos.push_back(std::stol(tok[ip]));
    if (!header) s.bims.push_back(tok[0] + "\t" + tok[3] + "\t" + tok[1]);
    s.lines.push_back(line);
  }
  s.end_pos.push_back((int)s.pos.size() - 1);
  return s;
}

// divide_pos_by_window (src/LD.cpp:125-139): for each SNP not at its chromosome's last
// position, the window of the following SNPs of that chromosome within bp (lead included).
void divide_by_window(SnpLd& s, long bp) {
  s.ws.clear();
  s.we.clear();
  for (size_t i = 0, c = 0; i < s.pos.size(); ++i) {
    if (s.pos[i] == s.pos[s.end_pos[c]]) {
      ++c;
      continue;
    }
    size_t j = i;
    for (; j <= (size_t)s.end_pos[c]; ++j)
      if (s.pos[j] - s.pos[i] > bp) break;
    s.ws.push_back((int64_t)i);
    s.we.push_back((int32_t)(j - i));
  }
}

std::vector<int64_t> pair_offsets(const std::vector<int32_t>& we) {
  std::vector<int64_t> off(we.size() + 1, 0);
  for (size_t w = 0; w < we.size(); ++w) off[w + 1] = off[w] + (we[w] - 1);
  return off;
}

// r2 (FP64) of every window pair on the device: flow A (packed genotypes, projected off U when
// given) or flow B (the dense matrix loaded into ctx).
std::vector<double> device_r2_f64(pcaone_ctx* ctx, const std::vector<double>* U, size_t uc,
                                  const std::vector<int64_t>& ws, const std::vector<int32_t>& we) {
  const auto off = pair_offsets(we);
  std::vector<double> r2(std::max<int64_t>(off.back(), 1));
  auto t0 = std::chrono::steady_clock::now();
  check(ctx, pcaone_gpu_ld_r2_f64(ctx, U ? U->data() : nullptr, (uint32_t)(U ? uc : 0), ws.data(), we.data(),
                                  ws.size(), r2.data()),
        "ld_r2_f64");
  g_log.print(date(), "LD r2 of", off.back(), "pairs computed in",
              std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(), "seconds");
  return r2;
}

// ld_prune_big / ld_prune_small (src/LD.cpp:141-242): windows in order; a lead SNP that is
// still kept compares every kept follower of its window; r2 > tol drops the follower, or the
// lead when the .mbim frequencies give the follower the larger MAF.
void ld_prune(const Params& p, const SnpLd& s, const std::vector<double>& r2) {
  const bool pick_random_one = s.af.empty();
  g_log.print(date(), "LD pruning, choose sites to be kept randomly or with high MAF? 1(random) : 0(high MAF). =>",
              pick_random_one);
  auto maf = [](double a) { return a > 0.5 ? 1 - a : a; };
  std::vector<char> keep(s.pos.size(), 1);
  const auto off = pair_offsets(s.we);
  for (size_t w = 0; w < s.ws.size(); ++w) {
    const int64_t i = s.ws[w];
    if (!keep[i]) continue;
    for (int j = 1; j < s.we[w]; ++j) {
      const int64_t k = i + j;
      if (!keep[k]) continue;
      if (r2[off[w] + j - 1] > p.ld_r2) {
        int64_t o = k;
        if (!pick_random_one) o = maf(s.af[k]) > maf(s.af[i]) ? i : k;
        keep[o] = 0;
      }
    }
  }
  std::ofstream out(p.fileout + ".ld.prune.out"), in(p.fileout + ".ld.prune.in");
  for (size_t i = 0; i < s.lines.size(); ++i) (keep[i] ? in : out) << s.lines[i] << std::endl;
}

// std::sort of the indices by value (sortidx, src/Common.hpp:68-73): the same algorithm on
// the same sequence gives the reference's order of ties.
std::vector<size_t> sortidx(const std::vector<double>& v) {
  std::vector<size_t> idx(v.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&v](size_t a, size_t b) { return v[a] < v[b]; });
  return idx;
}

// LD clumping of each assoc-like file (src/LD.cpp:245-367, 474-505): the targets with
// p <= clump_p2 per chromosome (map_index_snps, whose first line of a chromosome is filed
// under the previous one), matched by position to the LD matrix (get_target_snp_idx); index
// SNPs in increasing p take the unclumped targets within clump_bp (backward, then forward)
// with r2 >= clump_r2. The r2 of every pair within clump_bp comes from one device call per
// file (windows led by the matched targets).
void ld_clump(const Params& p, pcaone_ctx* ctx, const SnpLd& snp, const std::vector<double>* U, size_t uc) {
  using Pds = std::pair<double, std::string>;
  const auto files = split(p.clump, ",");
  const auto want = split(p.clump_names, ",");
  if (want.size() != 3) fail("--clump-names needs three column names");
  for (size_t fi = 0; fi < files.size(); ++fi) {
    g_log.print(date(), "LD-based clumping for associated file:", files[fi]);
    std::ifstream fa(files[fi]);
    if (!fa.is_open()) fail("can not open " + files[fi]);
    std::string line;
    std::getline(fa, line);
    const auto fields = split(line, "\t");
    int colidx[3] = {-1, -1, -1};
    for (size_t j = 0; j < fields.size(); ++j)
      for (int t = 0; t < 3; ++t)
        if (fields[j] == want[t]) colidx[t] = (int)j;
    for (int t = 0; t < 3; ++t)
      if (colidx[t] < 0) fail("the assoc-like file has no " + want[t] + " column");
    std::string head;
    const SnpLd tgt = read_snp_ld(files[fi], true, colidx[0], colidx[1], &head);
    // map_index_snps
    std::vector<std::unordered_map<int, Pds>> vm;
    {
      std::unordered_map<int, Pds> m;
      std::string prev;
      for (const auto& l : tgt.lines) {
        const auto tok = split(l, "\t");
        const std::string cur = tok[colidx[0]];
        const int bp = std::stoi(tok[colidx[1]]);
        const double pval = std::stod(tok[colidx[2]]);
        if (pval <= p.clump_p2) m.insert({bp, {pval, l}});
        if (!prev.empty() && prev != cur) {
          vm.push_back(m);
          m.clear();
        }
        prev = cur;
      }
      vm.push_back(m);
    }
    // get_target_snp_idx
    std::vector<std::vector<int>> idx_per_chr(tgt.chr.size()), bp_per_chr(tgt.chr.size());
    {
      std::vector<size_t> ord;
      for (const auto& ch : snp.chr) {
        size_t i = 0;
        while (i < tgt.chr.size() && tgt.chr[i] != ch) ++i;
        ord.push_back(i);
      }
      if (!std::is_sorted(ord.begin(), ord.end()))
        fail("the association file may be not sorted, hence not matching the bimfile ");
      for (size_t tc = 0; tc < tgt.chr.size(); ++tc) {
        size_t c = 0;
        while (c < snp.chr.size() && snp.chr[c] != tgt.chr[tc]) ++c;
        if (c == snp.chr.size()) continue;
        std::unordered_map<long, int> mpos;
        const int e = snp.end_pos[c], s0 = c > 0 ? snp.end_pos[c - 1] : 0;
        for (int i = s0; i <= e; ++i) mpos[snp.pos[i]] = i;
        const int te = tgt.end_pos[tc], ts = tc > 0 ? tgt.end_pos[tc - 1] : 0;
        for (int i = ts; i <= te; ++i) {
          auto it = mpos.find(tgt.pos[i]);
          if (it != mpos.end()) {
            bp_per_chr[tc].push_back((int)tgt.pos[i]);
            idx_per_chr[tc].push_back(it->second);
          }
        }
      }
    }
    // r2 of the pairs within clump_bp: one window per matched target, up to its farthest
    // matched partner on the right
    std::vector<int64_t> ws;
    std::vector<int32_t> we;
    std::unordered_map<int64_t, size_t> win_of;
    for (size_t c = 0; c < idx_per_chr.size(); ++c) {
      const auto& idx = idx_per_chr[c];
      const auto& bp = bp_per_chr[c];
      for (size_t j = 0; j < idx.size(); ++j) {
        size_t kmax = j;
        while (kmax + 1 < idx.size() && bp[kmax + 1] <= (long)bp[j] + (long)p.clump_bp) ++kmax;
        const int64_t a = idx[j];
        int32_t len = 1;
        for (size_t k = j + 1; k <= kmax; ++k) len = std::max<int32_t>(len, (int32_t)(idx[k] - a + 1));
        auto it = win_of.find(a);
        if (it == win_of.end()) {
          win_of[a] = ws.size();
          ws.push_back(a);
          we.push_back(len);
        } else {
          we[it->second] = std::max(we[it->second], len);
        }
      }
    }
    const auto off = pair_offsets(we);
    const std::vector<double> r2 = ws.empty() ? std::vector<double>() : device_r2_f64(ctx, U, uc, ws, we);
    auto r2_of = [&](int64_t a, int64_t b) {
      if (a > b) std::swap(a, b);
      const size_t w = win_of.at(a);
      if (b - a >= we[w]) fail("internal error: clumping pair outside its window");
      return r2[off[w] + (b - a) - 1];
    };
    // ld_clump_single_pheno
    std::ofstream ofs(p.fileout + ".p" + std::to_string(fi) + ".clump");
    ofs << head + "\tSP2" << std::endl;
    for (size_t c = 0; c < bp_per_chr.size() && c < vm.size(); ++c) {
      const auto& idx = idx_per_chr[c];
      const auto& bp = bp_per_chr[c];
      std::unordered_map<int, int> mbp;
      for (size_t i = 0; i < bp.size(); ++i) mbp.insert({bp[i], (int)i});
      auto mpp = vm[c];
      std::vector<double> pp;
      std::vector<int> ps;
      for (auto it = mpp.begin(); it != mpp.end(); ++it)
        if (it->second.first <= p.clump_p1) {
          ps.push_back(it->first);
          pp.push_back(it->second.first);
        }
      for (size_t oi : sortidx(pp)) {
        const int pos = ps[oi];
        if (mpp.count(pos) == 0) continue;
        if (mbp.count(pos) == 0) continue;
        std::vector<int> clumped;
        const int j = mbp.at(pos);
        int k = j;
        bool backward = true;
        while (true) {
          if (backward) {
            --k;
            if (k < 0 || bp[k] < (long)pos - (long)p.clump_bp) {
              backward = false;
              k = j;
              continue;
            }
          } else {
            ++k;
            if (k >= (int)bp.size() || bp[k] > (long)pos + (long)p.clump_bp) break;
          }
          const int p2 = bp[k];
          if (mpp.count(p2) == 0) continue;
          if (r2_of(idx[j], idx[k]) >= p.clump_r2) {
            clumped.push_back(p2);
            mpp.erase(p2);
          }
        }
        ofs << vm[c].at(pos).second << "\t";
        if (clumped.empty()) {
          ofs << "NONE";
        } else {
          std::vector<double> opp;
          for (int op : clumped) opp.push_back(vm[c].at(op).first);
          size_t t = 0;
          for (size_t q : sortidx(opp)) {
            ofs << clumped[q] << (t + 1 == opp.size() ? "" : ",");
            ++t;
          }
        }
        ofs << std::endl;
      }
    }
  }
}

// run_ld_stuff (src/LD.cpp:444-507): clumping when --clump is given, else the windows of
// --ld-bp with -R (.ld.gz of every pair's r2) or --ld-r2 (pruning). Flow A: packed genotypes
// projected off the --read-U factors (clumping reads them unprojected); flow B (dense): the
// .residuals matrix loaded into ctx.
int run_ld(const Params& p, pcaone_ctx* ctx, size_t N, size_t M, bool dense) {
  const std::string filebim = !p.filebim.empty() ? p.filebim : (dense ? p.binfile : p.bfile) + ".bim";
  SnpLd snp = read_snp_ld(filebim, false, 0, 3);
  if (snp.pos.size() != M) fail("The number of variants is not matching the LD matrix");
  size_t ur = 0, uc = 0;
  std::vector<double> U;
  if (!dense) {
    U = read_usv(p.fileU, ur, uc, p.fix_read_u);
    if (ur != N) fail("the number of rows of --read-U differs from the samples");
  }
  if (!p.clump.empty()) {
    ld_clump(p, ctx, snp, nullptr, 0);
    return 0;
  }
  divide_by_window(snp, (long)p.ld_bp);
  const auto& ws = snp.ws;
  const auto& we = snp.we;
  if (!p.print_r2) {
    ld_prune(p, snp, device_r2_f64(ctx, dense ? nullptr : &U, uc, ws, we));
    return 0;
  }
  const auto off = pair_offsets(we);
  const auto& bims = snp.bims;
  std::vector<float> r2(std::max<int64_t>(off.back(), 1));
  auto t0 = std::chrono::steady_clock::now();
  check(ctx, pcaone_gpu_ld_r2(ctx, dense ? nullptr : U.data(), (uint32_t)uc, ws.data(), we.data(), ws.size(),
                              r2.data()),
        "ld_r2");
  double gpu_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  g_log.print(date(), "LD r2 of", off.back(), "pairs computed in", gpu_s, "seconds");
  // format and deflate chunks of windows in parallel; concatenated gzip members are one file
  const size_t nw = ws.size(), chunk = 4096;
  const size_t nchunks = (nw + chunk - 1) / chunk;
  std::vector<std::string> gz(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
  for (long q = 0; q < (long)nchunks; ++q) {
    std::string text;
    if (q == 0) text = "CHR_A\tBP_A\tSNP_A\tCHR_B\tBP_B\tSNP_B\tR2\n";
    for (size_t w = q * chunk; w < std::min(nw, (q + 1) * chunk); ++w) {
      const size_t i = ws[w];
      for (int t = 1; t < we[w]; ++t) {
        text += bims[i];
        text += '\t';
        text += bims[i + t];
        text += '\t';
        text += std::to_string((double)r2[off[w] + t - 1]);
        text += '\n';
      }
    }
    z_stream zs{};
    deflateInit2(&zs, Z_DEFAULT_COMPRESSION, Z_DEFLATED, 15 + 16, 8, Z_DEFAULT_STRATEGY);
    std::string out(deflateBound(&zs, text.size()) + 64, '\0');
    zs.next_in = (Bytef*)text.data();
    zs.avail_in = (uInt)text.size();
    zs.next_out = (Bytef*)&out[0];
    zs.avail_out = (uInt)out.size();
    deflate(&zs, Z_FINISH);
    out.resize(zs.total_out);
    deflateEnd(&zs);
    gz[q] = std::move(out);
  }
  std::ofstream o(p.fileout + ".ld.gz", std::ios::binary);
  for (auto& g : gz) o.write(g.data(), (std::streamsize)g.size());
  return 0;
}

// ---------------------------------------------------------------- PCAngsd (Beagle input)
// parse_beagle_file (src/Utils.cpp:377-405): header gives N = columns/3 - 1; each site line
// holds marker, allele1, allele2 and three likelihoods per sample, of which the first two
// are used. Lines are parsed in parallel after the whole gz file is inflated.
std::vector<double> read_beagle(const std::string& path, size_t& N, size_t& M) {
  gzFile gz = gzopen(path.c_str(), "rb");
  if (!gz) fail("can not open " + path);
  std::string text;
  std::vector<char> buf(1 << 24);
  int n;
  while ((n = gzread(gz, buf.data(), (unsigned)buf.size())) > 0) text.append(buf.data(), n);
  gzclose(gz);
  std::vector<size_t> starts;
  size_t b = 0;
  while (b < text.size()) {
    starts.push_back(b);
    size_t e = text.find('\n', b);
    if (e == std::string::npos) e = text.size();
    b = e + 1;
  }
  if (starts.size() < 2) fail("the Beagle file has no sites");
  {
    std::string head = text.substr(starts[0], (starts.size() > 1 ? starts[1] - 1 : text.size()) - starts[0]);
    size_t cols = 0;
    std::istringstream hs(head);
    std::string t;
    while (hs >> t) ++cols;
    if (cols % 3) fail("Number of columns should be a multiple of 3.");
    N = cols / 3 - 1;
  }
  M = starts.size() - 1;
  std::vector<double> P(2 * N * M);
  bool bad = false;
#pragma omp parallel for schedule(dynamic, 256)
  for (long j = 0; j < (long)M; ++j) {
    const char* q = text.data() + starts[j + 1];
    char* end = nullptr;
    for (int f = 0; f < 3; ++f) {  // marker, allele1, allele2
      while (*q == ' ' || *q == '\t') ++q;
      while (*q && *q != ' ' && *q != '\t' && *q != '\n') ++q;
    }
    for (size_t i = 0; i < N; ++i) {
      double v[3];
      for (int f = 0; f < 3; ++f) {
        v[f] = std::strtod(q, &end);
        if (end == q) {
          bad = true;
          v[f] = 0;
        }
        q = end;
      }
      P[(size_t)j * 2 * N + 2 * i] = v[0];
      P[(size_t)j * 2 * N + 2 * i + 1] = v[1];
    }
  }
  if (bad) fail("something wrong parsing beagle");
  return P;
}

// The EM loop of run_pca_with_halko for PCAngsd (src/Halko.cpp:294-316) on the likelihood
// matrix of ctx: a first RSVD, then alternate the posterior update and the RSVD until
// 1 - mev(V, Vpre) < tolem. perm is the in-core SNP order (identity without the shuffle).
void pcangsd_em(const Params& p, pcaone_ctx* ctx, pcaone_rsvd_opts& o, size_t M, const std::vector<int32_t>& perm,
                std::vector<double>& U, std::vector<double>& S, std::vector<double>& V) {
  std::vector<double> Vpre, Vuse(M * p.k);
  pcaone_rsvd_report rep{};
  check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
  g_log.print(date(), "run EM-PCA. maxiter =", p.maxiter);
  o.carry_window_state = 1;
  for (unsigned it = 0; it < p.maxiter; ++it) {
    Vpre = V;
    // reference index semantics after the shuffle: position j is predicted from loading row
    // perm[j] (src/Data.cpp:249-270 indexes P, F and V^T by the permuted column)
    for (unsigned t = 0; t < p.k; ++t)
      for (size_t j = 0; j < M; ++j) Vuse[t * M + j] = p.fix_index ? V[t * M + j] : V[t * M + perm[j]];
    check(ctx, pcaone_gpu_gl_update(ctx, U.data(), S.data(), Vuse.data(), p.k), "gl_update");
    check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
    double acc = 0;
    for (unsigned b2 = 0; b2 < p.k; ++b2) {
      double nrm = 0;
      for (unsigned a = 0; a < p.k; ++a) {
        double d = 0;
        for (size_t j = 0; j < M; ++j) d += V[a * M + j] * Vpre[b2 * M + j];
        nrm += d * d;
      }
      acc += std::sqrt(nrm);
    }
    const double diff = 1.0 - acc / p.k;
    g_log.print(date(), "individual allele frequencies estimated iter =", it + 1, ", diff =", diff);
    if (diff < p.tolem) {
      g_log.print(date(), "come to convergence!");
      break;
    }
  }
}

int run_pcangsd(const Params& p, std::chrono::steady_clock::time_point t_start) {
  g_log.print(date(), "start parsing BEAGLE format");
  size_t N = 0, M = 0;
  std::vector<double> P = read_beagle(p.beagle, N, M);
  g_log.print(date(), "N (# samples):", N, ", M (# SNPs):", M);
  if (p.k + p.oversamples > N) fail("k + oversamples must not exceed the number of samples");
  const bool perm_on = p.svd == 2 && !p.noshuffle;
  std::vector<int32_t> perm(M);
  if (perm_on) pcaone_shuffle_perm(M, perm.data());
  else for (size_t j = 0; j < M; ++j) perm[j] = (int32_t)j;
  std::vector<double> Pp(P.size());  // sites in the RSVD's column order
  for (size_t j = 0; j < M; ++j) std::memcpy(&Pp[j * 2 * N], &P[(size_t)perm[j] * 2 * N], 2 * N * sizeof(double));
  pcaone_ctx* ctx = nullptr;
  if (pcaone_gpu_create(p.device, &ctx) != PCAONE_OK) fail("no usable CUDA device");
  check(ctx, pcaone_gpu_load_gl(ctx, Pp.data(), M, (uint32_t)N), "load_gl");
  g_log.print(date(), "begin to estimate allele frequencies");
  int fit = 0;
  check(ctx, pcaone_gpu_gl_freq(ctx, (int)p.maxiter, p.tolmaf, nullptr, &fit), "gl_freq");
  g_log.print(date(), fit < (int)p.maxiter ? "EM (MAF) converged at iteration:" : "EM (MAF) did not converge", fit);
  check(ctx, pcaone_gpu_gl_update(ctx, nullptr, nullptr, nullptr, 0), "gl_update");
  pcaone_rsvd_opts o{};
  o.k = (int)p.k;
  o.oversamples = (int)p.oversamples;
  o.maxp = (int)p.maxp;
  o.svd = p.svd;
  o.bands = (int)p.bands;
  o.precision = PCAONE_PREC_FP32;  // the posterior matrix is dense FP32
  o.standardize = 0;
  o.ploidy = 2;
  o.seed = p.seed;
  o.rand = (int)p.rand;
  o.tol = p.tol;
  o.verbose = p.verbose > 0;
  std::vector<double> U(N * p.k), S(p.k), V(M * p.k), Vuse(M * p.k);
  pcangsd_em(p, ctx, o, M, perm, U, S, V);
  // GRM stage (src/Halko.cpp:317-331): standardised posterior from the final factors, with the
  // same index semantics as the EM updates; C = E E^T / M with diag Dc / M, and its singular
  // vectors written with the sample names
  g_log.print(date(), "estimate GRM for pcangsd");
  g_log.print(date(), "begin to standardize the matrix for pcangsd procedure");
  for (unsigned t = 0; t < p.k; ++t)
    for (size_t j = 0; j < M; ++j) Vuse[t * M + j] = p.fix_index ? V[t * M + j] : V[t * M + perm[j]];
  {
    std::vector<double> C(N * N), Ev(N * N);
    check(ctx, pcaone_gpu_gl_grm(ctx, U.data(), S.data(), Vuse.data(), p.k, C.data(), Ev.data(), nullptr),
          "gl_grm");
    std::ofstream fcov(p.fileout + ".cov");
    write_aligned(fcov, C.data(), N, N, N);
    fcov << '\n';
    std::ofstream feig2(p.fileout + ".eigvecs2");
    feig2 << "#FID\tIID";
    for (size_t i = 0; i < N; ++i) feig2 << "\tPC" << i + 1;
    feig2 << '\n';
    size_t i = 0;
    for (const auto& s : beagle_samples(p.beagle)) {
      if (i >= N) break;
      feig2 << s << '\t' << s << '\t';
      write_aligned(feig2, Ev.data() + i, 1, N, N);
      feig2 << '\n';
      ++i;
    }
  }
  pcaone_gpu_destroy(ctx);
  std::vector<double> Vo(V.size());
  for (size_t j = 0; j < M; ++j)
    for (unsigned c = 0; c < p.k; ++c) Vo[c * M + perm[j]] = V[c * M + j];
  std::ofstream outs(p.fileout + ".sigvals"), oute(p.fileout + ".eigvals"), outu(p.fileout + ".eigvecs");
  outs << '#' << N << ',' << M << '\n';
  write_matrix(outs, S.data(), p.k, 1);
  outs << '\n';
  std::vector<double> E(p.k);
  for (unsigned c = 0; c < p.k; ++c) E[c] = S[c] * S[c] / (double)M * 2;
  write_matrix(oute, E.data(), p.k, 1);
  oute << '\n';
  write_matrix(outu, U.data(), N, p.k);
  outu << '\n';
  if (p.printv) {
    std::ofstream ov(p.fileout + ".loadings");
    write_matrix(ov, Vo.data(), M, p.k);
    ov << '\n';
  }
  g_log.print(date(), "eigen vectors and values saved");
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  g_log.print(date(), "total elapsed wall time:", wall, " seconds");
  return 0;
}

// -B/--binary input (FileBin, src/FileBinary.cpp): the float32 matrix written by -D (header:
// uint32 nsnps, uint32 nsamples; then nsnps rows of nsamples floats), LD r2 only.
int run_binary(const Params& p, std::chrono::steady_clock::time_point t_start) {
  std::ifstream f(p.binfile, std::ios::binary);
  if (!f.is_open()) fail("Cannot open " + p.binfile);
  uint32_t hdr[2] = {0, 0};
  f.read((char*)hdr, 8);
  const size_t M = hdr[0], N = hdr[1];
  g_log.print(date(), "shape of input matrix (features x samples) is", M, "x", N);
  if (!(p.print_r2 || p.ld_r2 > 0 || !p.clump.empty()))
    fail("-B/--binary input supports the LD modes (-R, --ld-r2, --clump) in this build");
  std::vector<float> X(M * N);
  f.read((char*)X.data(), (std::streamsize)(X.size() * 4));
  if ((size_t)f.gcount() != X.size() * 4) fail("the binary file is shorter than its header implies");
  pcaone_ctx* ctx = nullptr;
  if (pcaone_gpu_create(p.device, &ctx) != PCAONE_OK) fail("no usable CUDA device");
  check(ctx, pcaone_gpu_load_dense(ctx, X.data(), M, (uint32_t)N), "load_dense");
  g_log.print(date(), "run LD stuff");
  run_ld(p, ctx, N, M, true);
  pcaone_gpu_destroy(ctx);
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  g_log.print(date(), "total elapsed wall time:", wall, " seconds");
  return 0;
}

int main(int argc, char** argv) {
  Params p = parse(argc, argv);
  auto t_start = std::chrono::steady_clock::now();
  g_log.file.open(p.fileout + ".log");
  g_log.screen = p.verbose > 0;
  {
    struct utsname u;
    uname(&u);
    g_log.print(std::string("Machine name: ") + u.machine + "\nNode name: " + u.nodename +
                "\nOperating system release: " + u.release + "\n");
    g_log.print("PCAone (B200 build)\nOptions in effect:\n" + p.cmdline);
  }
  g_log.print(date(), "program started");
  if (!p.beagle.empty()) return run_pcangsd(p, t_start);
  if (!p.binfile.empty()) return run_binary(p, t_start);
  g_log.print(date(), "start parsing PLINK format");
  const size_t N = count_lines(p.bfile + ".fam"), M0 = count_lines(p.bfile + ".bim");
  g_log.print(date(), "N (# samples):", N, ", M (# SNPs):", M0);
  const size_t bpr = (N + 3) >> 2;
  std::vector<uint8_t> packed;
  {
    std::ifstream f(p.bfile + ".bed", std::ios::binary);
    if (!f.is_open()) fail("Cannot open bed file.");
    unsigned char h[3] = {0, 0, 0};
    f.read((char*)h, 3);
    if (h[0] != 0x6c || h[1] != 0x1b || h[2] != 0x01) fail("Incorrect magic number in plink bed file.");
    packed.resize(bpr * M0);
    f.read((char*)packed.data(), (std::streamsize)packed.size());
    if ((size_t)f.gcount() != packed.size()) fail("the .bed file is shorter than the .bim/.fam imply");
  }
  if (p.k + p.oversamples > N) fail("k + oversamples must not exceed the number of samples");
  if (p.pcangsd && p.emu) fail("--emu and --pcangsd are exclusive");
  // with --maf the reference indexes the filtered pseudo-likelihoods by unfiltered SNP index
  // (src/Data.cpp:255 with src/FilePlink.cpp:67-105), reading past them: not reproduced
  if (p.pcangsd && p.maf > 0) fail("--pcangsd with PLINK input does not support --maf");

  pcaone_ctx* ctx = nullptr;
  if (pcaone_gpu_create(p.device, &ctx) != PCAONE_OK) fail("no usable CUDA device");
  // out-of-core mode (-m): the genotypes are streamed from host memory for the RSVD (-d 1, 2)
  // and for IRAM (-d 0) when its operator is Z Z^T (samples <= SNPs); LD and the residual
  // writer read them resident
  const bool ld_mode = p.print_r2 || p.ld_r2 > 0 || !p.clump.empty();
  const bool streamed = p.memory > 0 && !p.ld_write && !ld_mode && (p.svd != 0 || N <= M0);
  if (streamed)
    check(ctx, pcaone_gpu_load_bed_host(ctx, packed.data(), M0, (uint32_t)N, 0), "load_bed_host");
  else
    check(ctx, pcaone_gpu_load_bed(ctx, packed.data(), M0, (uint32_t)N), "load_bed");
  std::vector<double> F(M0);
  check(ctx, pcaone_gpu_allele_freq(ctx, F.data()), "allele_freq");
  for (size_t j = 0; j < M0; ++j)
    if (F[j] == 0.0 || F[j] == 1.0) {
      std::cout << "\x1B[33m" << "sites with MAF=0 found! remove them first!" << "\033[0m\n";
      break;
    }
  // --maf filter (src/Data.cpp:74-91): keep SNPs with MAF > maf, re-upload the kept records
  std::vector<int> keep;
  size_t M = M0;
  if (p.maf > 0) {
    for (size_t j = 0; j < M0; ++j) {
      double maf = F[j] > 0.5 ? 1 - F[j] : F[j];
      if (maf > p.maf) keep.push_back((int)j);
    }
    M = keep.size();
    g_log.print(date(), "number of SNPs after filtering by MAF >", p.maf, ":", M);
    if (M < 1) fail("no SNPs left after filtering!");
    std::vector<uint8_t> kept(bpr * M);
    std::vector<double> Fk(M);
    for (size_t i = 0; i < M; ++i) {
      std::memcpy(&kept[i * bpr], &packed[(size_t)keep[i] * bpr], bpr);
      Fk[i] = F[keep[i]];
    }
    packed.swap(kept);
    F.swap(Fk);
    check(ctx, pcaone_gpu_load_bed(ctx, packed.data(), M, (uint32_t)N), "load_bed");
  }
  g_log.print(date(), "done reading all data");

  if (ld_mode) {  // LD mode (src/Main.cpp:64-77)
    if (p.fileU.empty()) fail("LD from PLINK input needs --read-U (flow A)");
    g_log.print(date(), "run LD stuff");
    run_ld(p, ctx, N, M, false);
    pcaone_gpu_destroy(ctx);
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    g_log.print(date(), "total elapsed wall time:", wall, " seconds");
    return 0;
  }

  const bool perm_on = p.svd == 2 && !p.noshuffle;  // src/Cmd.cpp:216
  // out-of-core plan (Data::prepare, src/Data.cpp:27-71): blocks of blocksize SNPs and, for the
  // winSVD, band_factor blocks per band
  int block_snps = 0, band_factor = 0;
  if (p.memory > 0) {
    const double l = p.k + p.oversamples;
    double bs;
    if (p.svd == 0) {
      bs = std::ceil(p.memory * 134217728 / N);
    } else {
      double m = (3 * N * l + 2 * M * l + 5 * M) / 134217728;
      if (p.memory > 1.1 * m) m = 0;
      else std::cout << "\x1B[33m" << "minimum RAM required is " << m << " GB. trying to allocate more RAM." << "\033[0m\n";
      bs = std::ceil(((m + p.memory) * 134217728 - 3 * N * l - 2 * M * l - 5 * M) / N);
    }
    long nblocks = (long)std::ceil((double)M / bs);
    int factor = 1;
    g_log.print(date(), "initial setting by -m/--memory: blocksize =", (long)bs, ", nblocks =", nblocks,
                ", factor =", factor);
    if (nblocks == 1) fail("only one block exists. please remove -m option");
    if (p.svd == 2) {
      if (nblocks < (long)p.bands) {
        bs = std::ceil((double)M / p.bands);
      } else {
        factor = (int)std::ceil((double)nblocks / p.bands);
        bs = std::ceil((double)M / (p.bands * factor));
      }
      nblocks = (long)std::ceil((double)M / bs);
      g_log.print(date(), "after adjustment by PCAone: -w =", p.bands, ", blocksize =", (long)bs, ", nblocks =",
                  nblocks, ", factor =", factor);
      block_snps = (int)bs;
      band_factor = factor;
    }
  }
  std::vector<int32_t> perm;
  if (perm_on) {
    perm.resize(M);
    if (p.memory > 0) {  // the structured order of permute_plink (src/FilePlink.cpp:298-405)
      g_log.print(date(), "permute plink files. nsnps:", M, ", nsamples:", N);
      if (pcaone_plink_perm(M, (uint32_t)N, p.buffer, p.bands, perm.data()) != PCAONE_OK)
        fail("cannot plan the out-of-core permutation");
      // the reference leaves the permuted fileset beside its outputs (src/FilePlink.cpp:339-403)
      std::ofstream ob(p.fileout + ".perm.bed", std::ios::binary);
      const char magic[3] = {0x6c, 0x1b, 0x01};
      ob.write(magic, 3);
      for (size_t i = 0; i < M; ++i) ob.write((const char*)&packed[(size_t)perm[i] * bpr], (std::streamsize)bpr);
      std::vector<std::string> bims;
      std::ifstream ib(p.bfile + ".bim");
      for (std::string line; std::getline(ib, line);) bims.push_back(line);
      std::ofstream obim(p.fileout + ".perm.bim");
      for (size_t i = 0; i < M; ++i) obim << bims[perm[i]] << "\n";
      std::ifstream ifam(p.bfile + ".fam");
      std::ofstream ofam(p.fileout + ".perm.fam");
      ofam << ifam.rdbuf();
    } else {
      pcaone_shuffle_perm(M, perm.data());
      g_log.print(date(), "permuting data matrix by columns in place");
    }
    check(ctx, pcaone_gpu_permute(ctx, perm.data()), "permute");
  }
  if (p.svd != 0)
    g_log.print(date(), p.svd == 2 ? "initialize window-based RSVD (winSVD) with" : "initialize single-pass RSVD (sSVD) with",
                streamed ? "out-of-core" : "in-core");
  pcaone_rsvd_opts o{};
  o.k = (int)p.k;
  o.oversamples = (int)p.oversamples;
  o.maxp = (int)p.maxp;
  o.svd = p.svd;
  o.bands = (int)p.bands;
  o.precision = p.precision;
  // with -D the reference runs the PCA on the centred, unstandardised genotypes
  // (src/Halko.cpp:285-288)
  o.standardize = (p.scale == 0 || p.ld_write) ? 0 : 1;
  o.ploidy = p.haploid ? 1 : 2;
  o.seed = p.seed;
  o.rand = (int)p.rand;
  o.tol = p.tol;
  o.verbose = p.verbose > 0;
  o.block_snps = block_snps;
  o.band_factor = band_factor;
  std::vector<double> U(N * p.k), S(p.k), V(M * p.k);
  pcaone_rsvd_report rep{};
  double gpu_s = 0;
  if (p.svd == 0) {
    // IRAM (run_pca_with_arnoldi in-core, src/Arnoldi.cpp:48-87): the largest k eigenpairs of
    // Z Z^T by restarted Lanczos, each operator application one device gram product; then
    // S = sqrt(eigenvalues), U = eigenvectors, V = Z^T U / S. FP64 products unless --precision
    // is given (the Lanczos residuals need the operator to full precision).
    g_log.print(date(), streamed ? "running IRAM SVD with out-of-core mode." : "running IRAM SVD with in-core mode.");
    const int prec = p.precision_set ? p.precision : PCAONE_PREC_FP64;
    const int stdz = (p.scale == 0 || p.ld_write) ? 0 : 1, ploidy = p.haploid ? 1 : 2;
    auto op = [&](const double* x, double* y) {
      if (N <= M) {
        check(ctx, pcaone_gpu_gram_product(ctx, prec, stdz, ploidy, x, 1, y), "gram_product");
      } else {  // tall matrix: Z^T Z x on the SNP side
        std::vector<double> t(N);
        check(ctx, pcaone_gpu_product(ctx, prec, 1, stdz, ploidy, x, 1, t.data()), "product");
        check(ctx, pcaone_gpu_product(ctx, prec, 0, stdz, ploidy, t.data(), 1, y), "product");
      }
    };
    const size_t n = N <= M ? N : M;
    auto res = iram::largest(op, n, (int)p.k, (int)p.ncv, (int)p.imaxiter, p.itol);
    if (!res.converged) fail("the nconv is not equal to k.");
    g_log.print(date(), "IRAM converged after", res.restarts, "restarts and", res.matvecs, "operator applications");
    for (unsigned c = 0; c < p.k; ++c) S[c] = std::sqrt(std::max(res.evals[c], 0.0));
    std::vector<double>& small = N <= M ? U : V;  // eigenvectors live on the smaller side
    std::vector<double>& big = N <= M ? V : U;
    small = res.evecs;
    check(ctx, pcaone_gpu_product(ctx, prec, N <= M ? 0 : 1, stdz, ploidy, small.data(), p.k, big.data()),
          "product");
    const size_t nb = N <= M ? M : N;
    for (unsigned c = 0; c < p.k; ++c)
      for (size_t j = 0; j < nb; ++j) big[c * nb + j] /= S[c];
    g_log.print(date(), "PCAone - IRAM SVD done");
  } else if (p.pcangsd) {
    // PCAngsd on PLINK input (src/FilePlink.cpp:89-115, src/Halko.cpp:294-316): pseudo-
    // likelihoods from the genotypes, F from the genotype counts, the first RSVD on the
    // centred unstandardised genotypes; no GRM stage (Beagle input only)
    std::vector<int32_t> order(perm);
    if (order.empty())
      for (size_t j = 0; j < M; ++j) order.push_back((int32_t)j);
    check(ctx, pcaone_gpu_bed_to_gl(ctx), "bed_to_gl");
    o.precision = PCAONE_PREC_FP32;  // the posterior matrix is dense FP32
    o.standardize = 0;
    o.carry_window_state = 0;
    pcangsd_em(p, ctx, o, M, order, U, S, V);
  } else if (!p.emu) {
    check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
    gpu_s += rep.gpu_ms / 1e3;
    g_log.print(date(), "stops at epoch =", rep.epochs);
  } else {
    // run_pca_with_halko impute branch with --emu (src/Halko.cpp:294-336)
    o.standardize = 0;
    o.carry_window_state = 0;
    check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
    gpu_s += rep.gpu_ms / 1e3;
    g_log.print(date(), "run EM-PCA. maxiter =", p.maxiter);
    o.carry_window_state = 1;
    const int compat = p.fix_index ? 0 : 1;
    std::vector<double> Vpre;
    for (unsigned it = 0; it < p.maxiter; ++it) {
      Vpre = V;
      check(ctx, pcaone_gpu_fit_emu(ctx, U.data(), S.data(), V.data(), p.k, compat), "fit_emu");
      check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
      gpu_s += rep.gpu_ms / 1e3;
      double acc = 0;  // 1 - mev(V, Vpre) (src/Utils.cpp:192-198)
      for (unsigned b = 0; b < p.k; ++b) {
        double nrm = 0;
        for (unsigned a = 0; a < p.k; ++a) {
          double d = 0;
          for (size_t j = 0; j < M; ++j) d += V[a * M + j] * Vpre[b * M + j];
          nrm += d * d;
        }
        acc += std::sqrt(nrm);
      }
      const double diff = 1.0 - acc / p.k;
      g_log.print(date(), "individual allele frequencies estimated iter =", it + 1, ", diff =", diff);
      if (diff < p.tolem) {
        g_log.print(date(), "come to convergence!");
        break;
      }
    }
    g_log.print(date(), "standardize the final matrix for EMU");
    check(ctx, pcaone_gpu_fit_emu(ctx, U.data(), S.data(), V.data(), p.k, compat), "fit_emu");
    o.standardize = p.scale == 0 ? 0 : 1;
    check(ctx, pcaone_gpu_rsvd(ctx, &o, U.data(), S.data(), V.data(), &rep), "rsvd");
    gpu_s += rep.gpu_ms / 1e3;
  }
  g_log.print(date(), "PCAone - Randomized SVD done; GPU time", gpu_s, "seconds");
  if (p.ld_write) {
    // Data::write_residuals (src/Data.cpp:196-245): header uint32 nsnps, uint32 nsamples, then
    // each SNP's centred residuals as float at its input position (perm undoes the shuffle);
    // rows are computed on the device in chunks of the current SNP order
    g_log.print(date(), p.ld_stats == 1 ? "ld-stats=1: calculate standardized genotype matrix!"
                                        : "ld-stats=0: calculate the ancestry adjusted LD matrix!");
    std::FILE* fr = std::fopen((p.fileout + ".residuals").c_str(), "wb");
    if (!fr) fail("cannot write " + p.fileout + ".residuals");
    const uint32_t hdr[2] = {(uint32_t)M, (uint32_t)N};
    std::fwrite(hdr, 4, 2, fr);
    const size_t chunk = std::max<size_t>(1, ((size_t)1 << 28) / (N * 4));
    std::vector<float> rows;
    std::vector<double> Vc;
    for (size_t s0 = 0; s0 < M; s0 += chunk) {
      const size_t n = std::min(chunk, M - s0);
      rows.resize(n * N);
      Vc.resize(n * p.k);
      for (unsigned c = 0; c < p.k; ++c)
        for (size_t j = 0; j < n; ++j) Vc[c * n + j] = V[c * M + s0 + j];
      if (p.ld_stats == 1)
        check(ctx, pcaone_gpu_residuals(ctx, nullptr, nullptr, nullptr, 0, s0, n, rows.data()), "residuals");
      else
        check(ctx, pcaone_gpu_residuals(ctx, U.data(), S.data(), Vc.data(), p.k, s0, n, rows.data()), "residuals");
      for (size_t j = 0; j < n; ++j) {
        const size_t dst = perm_on ? (size_t)perm[s0 + j] : s0 + j;
        std::fseek(fr, (long)(8 + dst * N * 4), SEEK_SET);
        std::fwrite(rows.data() + j * N, 4, N, fr);
      }
    }
    std::fclose(fr);
  }
  pcaone_gpu_destroy(ctx);

  // loadings back to the input SNP order (data->perm * V, src/Halko.cpp:340)
  if (perm_on) {
    std::vector<double> Vo(V.size());
    for (size_t j = 0; j < M; ++j)
      for (unsigned c = 0; c < p.k; ++c) Vo[c * M + perm[j]] = V[c * M + j];
    V.swap(Vo);
  }
  // outputs (src/Data.cpp:177-194)
  {
    std::ofstream outs(p.fileout + ".sigvals"), oute(p.fileout + ".eigvals"), outu(p.fileout + ".eigvecs");
    outs << '#' << N << ',' << M << '\n';
    write_matrix(outs, S.data(), p.k, 1);
    outs << '\n';
    std::vector<double> E(p.k);
    const int ploidy = p.haploid ? 1 : 2;
    for (unsigned c = 0; c < p.k; ++c) E[c] = S[c] * S[c] / (double)M * ploidy;
    write_matrix(oute, E.data(), p.k, 1);
    oute << '\n';
    write_matrix(outu, U.data(), N, p.k);
    outu << '\n';
  }
  if (p.printv || p.ld_write) {
    // .mbim: .bim line + tab + F (src/Data.cpp:96-136); -D saves it too (write_residuals)
    g_log.print(date(), "save matched sites in .mbim file and permutation mode is", perm_on ? 1 : 0);
    std::ifstream ib(p.bfile + ".bim");
    std::ofstream ob(p.fileout + ".mbim");
    std::string line;
    size_t j = 0, i = 0;
    while (std::getline(ib, line)) {
      if (!keep.empty()) {
        if (i < keep.size() && keep[i] == (int)j) {
          ob << line << "\t" << F[i] << "\n";
          ++i;
        }
      } else {
        ob << line << "\t" << F[j] << "\n";
      }
      ++j;
    }
  }
  if (p.printv) {
    std::ofstream ov(p.fileout + ".loadings");
    write_matrix(ov, V.data(), M, p.k);
    ov << '\n';
  }
  g_log.print(date(), "eigen vectors and values saved");
  {
    // .eigvecs2 (src/Utils.cpp:223-236)
    std::ifstream ifam(p.bfile + ".fam"), iev(p.fileout + ".eigvecs");
    std::ofstream o2(p.fileout + ".eigvecs2");
    o2 << "#FID\tIID";
    for (unsigned c = 0; c < p.k; ++c) o2 << "\tPC" << c + 1;
    o2 << "\n";
    std::string l1, l2;
    while (std::getline(ifam, l1)) {
      std::vector<std::string> tok;
      size_t b = 0;
      for (size_t q = 0; q <= l1.size(); ++q)
        if (q == l1.size() || l1[q] == ' ' || l1[q] == '\t') {
          tok.push_back(l1.substr(b, q - b));
          b = q + 1;
        }
      std::getline(iev, l2);
      o2 << tok[0] + "\t" + (tok.size() > 1 ? tok[1] : "") + "\t" << l2 << std::endl;
    }
  }
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  g_log.print(date(), "total elapsed wall time:", wall, " seconds");
  g_log.print(date(), "have a nice day. bye!");
  return 0;
}
