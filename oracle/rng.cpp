// ORACLE (test infrastructure only; never part of the product path).
//
// libstdc++ random draws that the reference makes, exposed to the numpy oracle:
//  * oracle_omega: the sketch Omega (nrow x ncol, column-major) drawn from
//    std::default_random_engine seeded with --seed, through std::normal_distribution<double>
//    (--rand 1) or std::uniform_real_distribution<double>(-1, 1) (--rand 0), filled in
//    column-major order. Follows RsvdOpData::initOmg (src/Halko.cpp:14-22) and
//    StandardNormalRandom / UniformRandom (src/RSVD.hpp:20-61).
//  * oracle_shuffle: the in-core SNP permutation, std::shuffle of 0..n-1 with a
//    default-constructed std::default_random_engine (seed not taken from --seed),
//    following permute_matrix (src/RSVD.hpp:63-79).
#include <algorithm>
#include <numeric>
#include <random>

extern "C" {

void oracle_omega(int seed, int rand, long nrow, long ncol, double* out) {
  std::default_random_engine rng;
  rng.seed(seed);
  if (rand) {
    std::normal_distribution<double> d{0, 1};
    for (long i = 0; i < nrow * ncol; ++i) out[i] = d(rng);
  } else {
    std::uniform_real_distribution<double> d{-1, 1};
    for (long i = 0; i < nrow * ncol; ++i) out[i] = d(rng);
  }
}

void oracle_shuffle(long n, int* out) {
  std::iota(out, out + n, 0);
  auto rng = std::default_random_engine{};
  std::shuffle(out, out + n, rng);
}
}
