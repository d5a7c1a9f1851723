// Restarted Lanczos for the largest eigenpairs of a symmetric operator: the role of the
// reference's IRAM solver (--svd 0: Spectra::PartialSVDSolver / SymEigsSolver with the
// sort rule "largest algebraic", src/Arnoldi.cpp:48-87).
//
// Thick restart (Wu and Simon, 2000): a Krylov basis of ncv vectors is built with full
// reorthogonalisation; the Rayleigh quotient T = V^T A V (ncv x ncv) is diagonalised; the
// nev wanted Ritz pairs are accepted when every residual |beta * y_last| is at most
// tol * max(eps^(2/3), |theta|) (the convergence test of Spectra's SymEigsSolver); otherwise
// the basis restarts from the kept Ritz vectors and the residual direction, which spans the
// same space as an implicitly restarted Lanczos with exact shifts. The operator is applied
// to one vector at a time through a callback (here the device gram product Z Z^T x).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <random>
#include <vector>

namespace iram {

// Cyclic Jacobi eigen-decomposition of a small symmetric matrix (n x n, column-major, taken
// as (A + A^T) / 2). Eigenvalues in decreasing order; eigenvectors as columns of Q.
inline void sym_eig(int n, const std::vector<double>& A0, std::vector<double>& w, std::vector<double>& Q) {
  std::vector<double> A((size_t)n * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) A[(size_t)j * n + i] = 0.5 * (A0[(size_t)j * n + i] + A0[(size_t)i * n + j]);
  std::vector<double> V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const double a = A[(size_t)j * n + i] * A[(size_t)j * n + i];
        tot += a;
        if (i != j) off += a;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)q * n + p];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {  // A = J^T A J, columns then rows
          const double akp = A[(size_t)p * n + k], akq = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = cs * akp - sn * akq;
          A[(size_t)q * n + k] = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[(size_t)k * n + p], aqk = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = cs * apk - sn * aqk;
          A[(size_t)k * n + q] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
          V[(size_t)p * n + k] = cs * vkp - sn * vkq;
          V[(size_t)q * n + k] = sn * vkp + cs * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return A[(size_t)a * n + a] > A[(size_t)b * n + b]; });
  w.assign(n, 0.0);
  Q.assign((size_t)n * n, 0.0);
  for (int c = 0; c < n; ++c) {
    w[c] = A[(size_t)ord[c] * n + ord[c]];
    for (int i = 0; i < n; ++i) Q[(size_t)c * n + i] = V[(size_t)ord[c] * n + i];
  }
}

struct Result {
  std::vector<double> evals;  // nev, decreasing
  std::vector<double> evecs;  // n x nev column-major
  int restarts = 0;
  long matvecs = 0;
  bool converged = false;
};

// Largest nev eigenpairs of the symmetric n x n operator op (y = A x). ncv > nev basis
// vectors, at most maxit restarts, relative tolerance tol.
inline Result largest(const std::function<void(const double*, double*)>& op, size_t n, int nev, int ncv, int maxit,
                      double tol, uint64_t seed = 1) {
  Result r;
  ncv = std::min<int>(ncv, (int)n);
  nev = std::min(nev, ncv - 1);
  std::vector<double> V(n * (size_t)(ncv + 1), 0.0), T((size_t)ncv * ncv, 0.0), w(n), h(ncv + 1);
  auto col = [&](int j) { return V.data() + (size_t)j * n; };
  auto dot = [&](const double* a, const double* b) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  };
  // orthogonalise w against columns 0..j (twice, classical Gram-Schmidt); h accumulates
  auto orth = [&](int j) {
    std::fill(h.begin(), h.end(), 0.0);
    for (int pass = 0; pass < 2; ++pass)
      for (int i = 0; i <= j; ++i) {
        const double c = dot(col(i), w.data());
        h[i] += c;
        const double* vi = col(i);
        for (size_t t = 0; t < n; ++t) w[t] -= c * vi[t];
      }
  };
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> uni(-0.5, 0.5);
  auto random_into = [&](int j) {  // a random unit vector orthogonal to columns 0..j-1
    for (size_t t = 0; t < n; ++t) w[t] = uni(rng);
    if (j > 0) orth(j - 1);
    const double nr = std::sqrt(dot(w.data(), w.data()));
    for (size_t t = 0; t < n; ++t) col(j)[t] = w[t] / nr;
  };
  random_into(0);
  const double eps23 = std::pow(std::numeric_limits<double>::epsilon(), 2.0 / 3.0);
  int kept = 0;
  double beta = 0.0;
  std::vector<double> theta, Y;
  for (int it = 0; it <= maxit; ++it) {
    for (int j = kept; j < ncv; ++j) {
      op(col(j), w.data());
      r.matvecs++;
      orth(j);
      for (int i = 0; i <= j; ++i) {
        T[(size_t)j * ncv + i] = h[i];
        T[(size_t)i * ncv + j] = h[i];
      }
      beta = std::sqrt(dot(w.data(), w.data()));
      if (beta < 1e-12 * std::fabs(h[j]) || beta == 0.0) {  // invariant subspace: continue randomly
        random_into(j + 1);
        beta = 0.0;
      } else {
        for (size_t t = 0; t < n; ++t) col(j + 1)[t] = w[t] / beta;
      }
      if (j + 1 < ncv) {
        T[(size_t)j * ncv + j + 1] = beta;
        T[(size_t)(j + 1) * ncv + j] = beta;
      }
    }
    sym_eig(ncv, T, theta, Y);
    int nconv = 0;
    for (int i = 0; i < nev; ++i)
      if (std::fabs(beta * Y[(size_t)i * ncv + ncv - 1]) <= tol * std::max(eps23, std::fabs(theta[i]))) ++nconv;
    r.restarts = it;
    if (nconv == nev || it == maxit) {
      r.converged = nconv == nev;
      r.evals.assign(theta.begin(), theta.begin() + nev);
      r.evecs.assign(n * (size_t)nev, 0.0);
      for (int c = 0; c < nev; ++c)
        for (int j = 0; j < ncv; ++j) {
          const double y = Y[(size_t)c * ncv + j];
          const double* vj = col(j);
          double* out = r.evecs.data() + (size_t)c * n;
          for (size_t t = 0; t < n; ++t) out[t] += y * vj[t];
        }
      return r;
    }
    // thick restart: keep the leading Ritz vectors plus the residual direction
    kept = std::min(ncv - 1, nev + std::max(1, (ncv - nev) / 2));
    std::vector<double> Vn(n * (size_t)(kept + 1), 0.0);
    for (int c = 0; c < kept; ++c)
      for (int j = 0; j < ncv; ++j) {
        const double y = Y[(size_t)c * ncv + j];
        const double* vj = col(j);
        double* out = Vn.data() + (size_t)c * n;
        for (size_t t = 0; t < n; ++t) out[t] += y * vj[t];
      }
    std::copy(col(ncv), col(ncv) + n, Vn.data() + (size_t)kept * n);
    std::copy(Vn.begin(), Vn.end(), V.begin());
    std::fill(T.begin(), T.end(), 0.0);
    for (int c = 0; c < kept; ++c) {
      T[(size_t)c * ncv + c] = theta[c];
      const double s = beta * Y[(size_t)c * ncv + ncv - 1];
      T[(size_t)kept * ncv + c] = s;
      T[(size_t)c * ncv + kept] = s;
    }
  }
  return r;
}

}  // namespace iram
