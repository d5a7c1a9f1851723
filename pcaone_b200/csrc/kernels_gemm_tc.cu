// tcgen05 (sm_100a) decode-GEMM back end: placeholder until the kernel lands.
#include "internal.hpp"
#include "rsvd.hpp"

namespace pg {

bool tc_supported(pcaone_ctx* c) { return c->cc_major == 10; }

namespace {
int tc_ksplit(pcaone_ctx*, int64_t, int64_t) { return 1; }
void tc_gemm(pcaone_ctx*, const uint8_t*, uint32_t, int64_t, int64_t, const float*, int, int, float*) {
  throw Error(PCAONE_ENODEV, "mixed-precision path not built");
}
void tc_omega(pcaone_ctx*, const double*, int, int64_t) {}
void tc_b2(pcaone_ctx*, const float*, int, int64_t) {}
}  // namespace

GemmFnT<float> gemm_tc() { return GemmFnT<float>{tc_ksplit, tc_gemm, tc_gemm, tc_omega, tc_b2}; }

}  // namespace pg
