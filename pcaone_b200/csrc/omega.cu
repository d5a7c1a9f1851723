// The reference's sketch Omega (RsvdOpData::initOmg, src/Halko.cpp:14-22): a
// std::default_random_engine (libstdc++ minstd_rand0) seeded with --seed, filled column-major
// with std::normal_distribution<double>(0, 1) draws (or uniform_real_distribution(-1, 1) with
// --rand 0). The result must be bit-identical to that sequential fill; it is generated here in
// parallel without changing a single draw:
//
//  * minstd_rand0 is x_{k+1} = 16807 x_k mod (2^31 - 1), so the state after d draws is
//    16807^d x_0 mod (2^31 - 1) (square-and-multiply), and an engine seeded with that state
//    continues the stream exactly;
//  * each uniform is std::generate_canonical<double, 53> of two draws, so a candidate pair of
//    the polar method (libstdc++ normal_distribution) consumes exactly four draws, and a
//    uniform_real_distribution value exactly two;
//  * the polar method keeps a candidate pair when 0 < x^2 + y^2 <= 1 and then returns y*m
//    followed by the saved x*m. So segments of candidate pairs are processed independently
//    (same expressions as libstdc++), and the accepted pairs are concatenated in segment
//    order, which is the sequential output order.
#include <algorithm>
#include <cmath>
#include <random>
#include <thread>
#include <vector>

#include "rsvd.hpp"

namespace pg {

namespace {

constexpr uint64_t kM = 2147483647ull;  // minstd_rand0 modulus
constexpr uint64_t kA = 16807ull;       // minstd_rand0 multiplier

uint64_t pow_mod(uint64_t b, uint64_t e) {
  uint64_t r = 1;
  b %= kM;
  while (e) {
    if (e & 1) r = r * b % kM;
    b = b * b % kM;
    e >>= 1;
  }
  return r;
}

// Engine whose next draw is draw number d + 1 of the stream that starts at state x0.
std::minstd_rand0 engine_at(uint64_t x0, uint64_t d) {
  return std::minstd_rand0((std::minstd_rand0::result_type)(pow_mod(kA, d) * x0 % kM));
}

int worker_count() {
  const unsigned hc = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(hc ? hc : 1u, 32u));
}

}  // namespace

void omega_host(int seed, int rand, uint64_t nrow, uint32_t ncol, double* out) {
  const uint64_t n = nrow * (uint64_t)ncol;
  if (n == 0) return;
  // libstdc++ linear_congruential_engine::seed: x0 = s mod m, or 1 when that is 0 (c = 0)
  const uint64_t s = (uint64_t)(std::minstd_rand0::result_type)seed;
  const uint64_t x0 = (s % kM) ? (s % kM) : 1;
  const int T = worker_count();
  if (!rand) {  // uniform_real_distribution(-1, 1): value i = canonical(draws 2i+1, 2i+2) * 2 - 1
    const uint64_t per = (n + T - 1) / T;
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
      const uint64_t b = (uint64_t)t * per, e = std::min<uint64_t>(n, b + per);
      if (b >= e) break;
      th.emplace_back([=] {
        std::minstd_rand0 eng = engine_at(x0, 2 * b);
        std::uniform_real_distribution<double> d{-1, 1};
        for (uint64_t i = b; i < e; ++i) out[i] = d(eng);
      });
    }
    for (auto& x : th) x.join();
    return;
  }
  if (n < (1u << 16)) {  // small fills: the sequential distribution itself
    std::minstd_rand0 eng = engine_at(x0, 0);
    std::normal_distribution<double> d{0, 1};
    for (uint64_t i = 0; i < n; ++i) out[i] = d(eng);
    return;
  }
  // normal: one segment of candidate pairs per thread and round (4 draws per pair), sized so
  // that one round usually covers the n values (acceptance pi/4); further rounds continue
  // the stream where the last one stopped
  const uint64_t seg = ((uint64_t)((double)n / 2 / 0.75) / T) + 1024;
  std::vector<std::vector<double>> seg_out(T);
  uint64_t written = 0, next_pair = 0;
  while (written < n) {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
      const uint64_t p0 = next_pair + (uint64_t)t * seg;
      th.emplace_back([&, t, p0] {
        std::vector<double>& o = seg_out[t];
        o.clear();
        o.reserve(2 * seg);
        std::minstd_rand0 eng = engine_at(x0, p0 * 4);
        for (uint64_t p = 0; p < seg; ++p) {
          // the polar step of libstdc++ normal_distribution::operator(), same expressions
          const double x = 2.0 * std::generate_canonical<double, 53>(eng) - 1.0;
          const double y = 2.0 * std::generate_canonical<double, 53>(eng) - 1.0;
          const double r2 = x * x + y * y;
          if (r2 > 1.0 || r2 == 0.0) continue;
          const double mult = std::sqrt(-2 * std::log(r2) / r2);
          o.push_back(y * mult * 1.0 + 0.0);  // returned value, then the saved one
          o.push_back(x * mult * 1.0 + 0.0);
        }
      });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < T && written < n; ++t) {
      const uint64_t take = std::min<uint64_t>(n - written, seg_out[t].size());
      std::copy(seg_out[t].begin(), seg_out[t].begin() + take, out + written);
      written += take;
    }
    next_pair += (uint64_t)T * seg;
  }
}

}  // namespace pg
