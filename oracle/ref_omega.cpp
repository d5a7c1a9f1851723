// ORACLE pin (test infrastructure only). Compiled by oracle/ref.mk against the reference's
// own headers (src/RSVD.hpp, vendored Eigen) to dump the reference's Omega and in-core SNP
// permutation, so that the restated draws in oracle/rng.cpp and in the product host code
// can be checked bit-for-bit.
//
//   omega_ref SEED RAND NROW NCOL PERM_N > out.bin
//   writes NROW*NCOL doubles (column-major) then PERM_N int32 permutation indices.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "RSVD.hpp"

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: omega_ref SEED RAND NROW NCOL PERM_N\n");
    return 1;
  }
  int seed = atoi(argv[1]), rand = atoi(argv[2]);
  long nrow = atol(argv[3]), ncol = atol(argv[4]), pn = atol(argv[5]);
  using Mat2D = Eigen::MatrixXd;
  auto rng = std::default_random_engine{};
  rng.seed(seed);
  Mat2D Omg = rand ? PCAone::StandardNormalRandom<Mat2D, std::default_random_engine>(nrow, ncol, rng)
                   : PCAone::UniformRandom<Mat2D, std::default_random_engine>(nrow, ncol, rng);
  fwrite(Omg.data(), sizeof(double), nrow * ncol, stdout);
  Mat2D G = Mat2D::Zero(1, pn);
  Eigen::PermutationMatrix<Eigen::Dynamic, Eigen::Dynamic> P;
  PCAone::permute_matrix(G, P);
  for (long i = 0; i < pn; ++i) {
    int v = P.indices()[i];
    fwrite(&v, sizeof(int), 1, stdout);
  }
  return 0;
}
