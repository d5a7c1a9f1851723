// Seeded synthetic PLINK .bed/.bim/.fam and Beagle genotype-likelihood generator.
//
// Population models (all per-SNP independent random streams, so the output does not
// depend on the number of OpenMP threads):
//   * Balding-Nichols: ancestral p ~ U(pmin, pmax); population k frequency
//     p_k ~ Beta(p (1-F_k)/F_k, (1-p)(1-F_k)/F_k); samples assigned to populations in
//     contiguous blocks; genotype (A1 dosage) ~ Binomial(2, p_k) (HWE).
//   * Admixed: per-sample ancestry proportions q_i ~ Dirichlet(alpha); the individual
//     frequency is sum_k q_ik p_k.
//   * Missingness: MCAR with a global rate, or a per-sample rate ~ Beta(a, b).
//   * Beagle: true genotypes as above, read depth ~ Poisson(depth), reads ~ Binomial with
//     sequencing error; GL triple P(reads | g) normalised to sum 1 per sample-site.
//   * Block LD (--ld-switch s): each population has H founder haplotypes whose alleles at SNP
//     j are Bernoulli(p_k); every sample haplotype copies one founder of its population and
//     switches to a uniformly drawn founder before each SNP with probability s (a Markov
//     copying model), so nearby SNPs are correlated. Genotype = sum of two haplotypes.
//
// The .bed coding follows the PLINK 1 SNP-major format: magic 6c 1b 01, then per SNP
// ceil(N/4) bytes, sample j at bits 2*(j%4) of byte j/4 (LSB first), codes
// 00 = two copies of A1, 10 = one copy, 11 = zero copies, 01 = missing.
//
// Usage: pcaone-sim --out PREFIX --n N --m M [--pops K] [--fst F | --fst-lo a --fst-hi b]
//                   [--pmin a --pmax b] [--miss r | --miss-beta a,b] [--admix alpha]
//                   [--seed s] [--beagle depth,err] [--chroms C] [--bp-spacing S]
//                   [--ld-switch s [--founders H]] [--gl-bin]
// --gl-bin (with --beagle): instead of the gz text, write PREFIX.gl.f32 = the first two
// normalised likelihoods per sample and site as float32, site-major (M x 2N), the layout of
// the reference's 2N x M column-major P, plus PREFIX.gl.bim.
#include <omp.h>
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Rng {  // xoshiro256** seeded by splitmix64
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  Rng(uint64_t seed, uint64_t stream) {
    uint64_t x = seed * 0xD1B54A32D192ED03ull ^ (stream + 0x632BE59BD9B4E019ull);
    for (auto& v : s) v = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uni() { return (next() >> 11) * 0x1.0p-53; }  // [0,1)
  double normal() {                                       // Box-Muller
    double u1 = uni(), u2 = uni();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  double gamma(double a) {  // Marsaglia-Tsang
    if (a < 1.0) {
      double u = uni();
      if (u < 1e-300) u = 1e-300;
      return gamma(a + 1.0) * std::pow(u, 1.0 / a);
    }
    double d = a - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
    for (;;) {
      double x = normal(), v = 1.0 + c * x;
      if (v <= 0) continue;
      v = v * v * v;
      double u = uni();
      if (u < 1.0 - 0.0331 * x * x * x * x) return d * v;
      if (std::log(u) < 0.5 * x * x + d * (1.0 - v + std::log(v))) return d * v;
    }
  }
  double beta(double a, double b) {
    double x = gamma(a), y = gamma(b);
    return x / (x + y);
  }
  int poisson(double lam) {  // Knuth, fine for small lambda
    double L = std::exp(-lam), p = 1.0;
    int k = 0;
    do { ++k; p *= uni(); } while (p > L);
    return k - 1;
  }
};

struct Opts {
  std::string out = "sim";
  long n = 1000, m = 10000;
  int pops = 3;
  double fst_lo = 0.05, fst_hi = 0.05;
  double pmin = 0.05, pmax = 0.5;
  double miss = 0.0, miss_a = 0.0, miss_b = 0.0;
  double admix = 0.0;
  uint64_t seed = 1;
  double depth = 0.0, err = 0.01;
  int chroms = 1;
  double bp_spacing = 100.0;  // mean spacing between SNPs (bp)
  double ld_switch = 0.0;     // > 0: Markov haplotype-copying model
  int founders = 40;          // founder haplotypes per population
  bool gl_bin = false;        // binary float32 likelihood pairs instead of Beagle text
};

void die(const char* msg) {
  fprintf(stderr, "pcaone-sim: %s\n", msg);
  exit(1);
}

}  // namespace

int main(int argc, char** argv) {
  Opts o;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto val = [&]() -> const char* {
      if (i + 1 >= argc) die(("missing value for " + a).c_str());
      return argv[++i];
    };
    if (a == "--out") o.out = val();
    else if (a == "--n") o.n = atol(val());
    else if (a == "--m") o.m = atol(val());
    else if (a == "--pops") o.pops = atoi(val());
    else if (a == "--fst") o.fst_lo = o.fst_hi = atof(val());
    else if (a == "--fst-lo") o.fst_lo = atof(val());
    else if (a == "--fst-hi") o.fst_hi = atof(val());
    else if (a == "--pmin") o.pmin = atof(val());
    else if (a == "--pmax") o.pmax = atof(val());
    else if (a == "--miss") o.miss = atof(val());
    else if (a == "--miss-beta") { if (sscanf(val(), "%lf,%lf", &o.miss_a, &o.miss_b) != 2) die("bad --miss-beta"); }
    else if (a == "--admix") o.admix = atof(val());
    else if (a == "--seed") o.seed = strtoull(val(), nullptr, 10);
    else if (a == "--beagle") { if (sscanf(val(), "%lf,%lf", &o.depth, &o.err) != 2) die("bad --beagle"); }
    else if (a == "--chroms") o.chroms = atoi(val());
    else if (a == "--bp-spacing") o.bp_spacing = atof(val());
    else if (a == "--ld-switch") o.ld_switch = atof(val());
    else if (a == "--founders") o.founders = atoi(val());
    else if (a == "--gl-bin") o.gl_bin = true;
    else die(("unknown option " + a).c_str());
  }
  if (o.n < 1 || o.m < 1 || o.pops < 1) die("bad sizes");
  const long N = o.n, M = o.m, K = o.pops;

  // Population-level draws: per-population Fst, per-sample population / admixture and
  // per-sample missing rate. Stream 0 is reserved for these.
  Rng g(o.seed, 0);
  std::vector<double> fst(K);
  for (long k = 0; k < K; ++k) fst[k] = o.fst_lo + (o.fst_hi - o.fst_lo) * g.uni();
  std::vector<double> q(N * K, 0.0);  // ancestry proportions
  for (long i = 0; i < N; ++i) {
    if (o.admix > 0) {
      double s = 0;
      for (long k = 0; k < K; ++k) s += (q[i * K + k] = g.gamma(o.admix));
      for (long k = 0; k < K; ++k) q[i * K + k] /= s;
    } else {
      q[i * K + (i * K) / N] = 1.0;
    }
  }
  std::vector<double> srate(N, o.miss);
  if (o.miss_a > 0 && o.miss_b > 0)
    for (long i = 0; i < N; ++i) srate[i] = g.beta(o.miss_a, o.miss_b);

  const long bpr = (N + 3) / 4;
  const bool beagle = o.depth > 0;
  if (o.ld_switch > 0 && (beagle || o.admix > 0 || o.founders < 1))
    die("--ld-switch needs PLINK output, no --admix and --founders >= 1");
  std::vector<uint8_t> bed;
  if (!beagle) bed.assign((size_t)bpr * M, 0);
  const bool glbin = beagle && o.gl_bin;
  std::vector<std::string> gl_lines(beagle && !glbin ? M : 0);
  std::vector<float> glf(glbin ? (size_t)M * 2 * N : 0);

  if (o.ld_switch > 0) {
    // founder alleles: founder f of population k at SNP j, per-SNP streams
    const long H = o.founders;
    std::vector<uint8_t> fa((size_t)M * K * H);
#pragma omp parallel for schedule(dynamic, 64)
    for (long j = 0; j < M; ++j) {
      Rng r(o.seed, (uint64_t)j + 1);
      const double panc = o.pmin + (o.pmax - o.pmin) * r.uni();
      for (long k = 0; k < K; ++k) {
        const double F = fst[k];
        double pkk = r.beta(panc * (1 - F) / F, (1 - panc) * (1 - F) / F);
        pkk = std::min(std::max(pkk, 1e-6), 1 - 1e-6);
        for (long f = 0; f < H; ++f) fa[((size_t)j * K + k) * H + f] = r.uni() < pkk;
      }
    }
    // haplotype paths: one thread per 4 samples (one byte column of the .bed)
    bed.assign((size_t)bpr * M, 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (long b = 0; b < bpr; ++b) {
      for (long i = 4 * b; i < std::min(N, 4 * b + 4); ++i) {
        Rng r(o.seed, (uint64_t)(M + 1000 + i));
        const long k = (i * K) / N;
        long h0 = (long)(r.uni() * H) % H, h1 = (long)(r.uni() * H) % H;
        for (long j = 0; j < M; ++j) {
          if (r.uni() < o.ld_switch) h0 = (long)(r.uni() * H) % H;
          if (r.uni() < o.ld_switch) h1 = (long)(r.uni() * H) % H;
          const int d = fa[((size_t)j * K + k) * H + h0] + fa[((size_t)j * K + k) * H + h1];
          const bool missing = r.uni() < srate[i];
          const uint8_t code = missing ? 1 : (d == 2 ? 0 : (d == 1 ? 2 : 3));
          bed[(size_t)j * bpr + b] |= (uint8_t)(code << (2 * (i & 3)));
        }
      }
    }
  }

#pragma omp parallel for schedule(dynamic, 64)
  for (long j = 0; j < (o.ld_switch > 0 ? 0 : M); ++j) {
    Rng r(o.seed, (uint64_t)j + 1);
    double panc = o.pmin + (o.pmax - o.pmin) * r.uni();
    double pk[64];
    for (long k = 0; k < K && k < 64; ++k) {
      double F = fst[k];
      pk[k] = r.beta(panc * (1 - F) / F, (1 - panc) * (1 - F) / F);
      pk[k] = std::min(std::max(pk[k], 1e-6), 1 - 1e-6);
    }
    uint8_t* row = beagle ? nullptr : &bed[(size_t)j * bpr];
    std::string line;
    if (beagle && !glbin) {
      char head[64];
      snprintf(head, sizeof head, "%d_%ld\t0\t1", 1 + (int)(j * o.chroms / M), j + 1);
      line = head;
      line.reserve(line.size() + N * 24);
    }
    for (long i = 0; i < N; ++i) {
      double p = 0;
      for (long k = 0; k < K; ++k) p += q[i * K + k] * pk[k];
      int d = (r.uni() < p) + (r.uni() < p);  // A1 dosage
      bool missing = r.uni() < srate[i];
      if (!beagle) {
        uint8_t code = missing ? 1 : (d == 2 ? 0 : (d == 1 ? 2 : 3));
        row[i >> 2] |= (uint8_t)(code << (2 * (i & 3)));
      } else {
        // reads: allele A1 with prob d/2, flipped by sequencing error
        int depth = r.poisson(o.depth);
        int na1 = 0;
        for (int t = 0; t < depth; ++t) {
          bool a1 = r.uni() < d / 2.0;
          if (r.uni() < o.err) a1 = !a1;
          na1 += a1;
        }
        int na2 = depth - na1;
        // P(reads | genotype) with genotypes ordered (A1A1, A1A2, A2A2)
        double e = o.err;
        double l0 = std::pow(1 - e, na1) * std::pow(e, na2);
        double l1 = std::pow(0.5, depth);
        double l2 = std::pow(e, na1) * std::pow(1 - e, na2);
        double s = l0 + l1 + l2;
        if (glbin) {
          glf[((size_t)j * N + i) * 2] = (float)(l0 / s);
          glf[((size_t)j * N + i) * 2 + 1] = (float)(l1 / s);
        } else {
          char buf[96];
          snprintf(buf, sizeof buf, "\t%.6f\t%.6f\t%.6f", l0 / s, l1 / s, l2 / s);
          line += buf;
        }
      }
    }
    if (beagle && !glbin) gl_lines[j] = std::move(line);
  }

  // Positions: strictly increasing within a chromosome, gaps ~ Exp(mean spacing) with a
  // slowly varying density so fixed-bp windows hold uneven numbers of SNPs.
  std::vector<long> pos(M);
  std::vector<int> chr(M);
  {
    Rng pr(o.seed, (uint64_t)M + 7);
    long p = 0;
    int c = 0;
    for (long j = 0; j < M; ++j) {
      int cj = 1 + (int)(j * o.chroms / M);
      if (cj != c) { c = cj; p = 0; }
      double dens = 1.0 + 0.9 * std::sin(6.283185307179586 * j / 20000.0);
      double gap = -std::log(std::max(pr.uni(), 1e-12)) * o.bp_spacing / dens;
      p += 1 + (long)gap;
      pos[j] = p;
      chr[j] = c;
    }
  }

  if (!beagle) {
    FILE* f = fopen((o.out + ".bed").c_str(), "wb");
    if (!f) die("cannot write .bed");
    const uint8_t magic[3] = {0x6c, 0x1b, 0x01};
    fwrite(magic, 1, 3, f);
    fwrite(bed.data(), 1, bed.size(), f);
    fclose(f);
    FILE* b = fopen((o.out + ".bim").c_str(), "w");
    for (long j = 0; j < M; ++j) fprintf(b, "%d\tsnp%ld\t0\t%ld\tA\tG\n", chr[j], j + 1, pos[j]);
    fclose(b);
    FILE* fa = fopen((o.out + ".fam").c_str(), "w");
    for (long i = 0; i < N; ++i) fprintf(fa, "fam%ld\tind%ld\t0\t0\t0\t-9\n", i + 1, i + 1);
    fclose(fa);
  } else if (glbin) {
    FILE* f = fopen((o.out + ".gl.f32").c_str(), "wb");
    if (!f) die("cannot write .gl.f32");
    fwrite(glf.data(), sizeof(float), glf.size(), f);
    fclose(f);
    FILE* b = fopen((o.out + ".gl.bim").c_str(), "w");
    for (long j = 0; j < M; ++j) fprintf(b, "%d\t%d_%ld\t0\t%ld\tA\tG\n", chr[j], chr[j], j + 1, pos[j]);
    fclose(b);
  } else {
    gzFile gz = gzopen((o.out + ".beagle.gz").c_str(), "wb1");
    if (!gz) die("cannot write .beagle.gz");
    std::string head = "marker\tallele1\tallele2";
    for (long i = 0; i < N; ++i) {
      char buf[96];
      snprintf(buf, sizeof buf, "\tInd%ld\tInd%ld\tInd%ld", i, i, i);
      head += buf;
    }
    head += "\n";
    gzwrite(gz, head.data(), head.size());
    for (long j = 0; j < M; ++j) {
      gl_lines[j] += "\n";
      gzwrite(gz, gl_lines[j].data(), gl_lines[j].size());
    }
    gzclose(gz);
    FILE* b = fopen((o.out + ".beagle.gz.bim").c_str(), "w");
    for (long j = 0; j < M; ++j) fprintf(b, "%d\t%d_%ld\t0\t%ld\tA\tG\n", chr[j], chr[j], j + 1, pos[j]);
    fclose(b);
  }
  return 0;
}
