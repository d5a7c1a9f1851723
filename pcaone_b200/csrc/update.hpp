// Fused Omega update (kernels_update.cu).
#pragma once

#include <cuda_bf16.h>

#include "internal.hpp"

namespace pg {

struct UpdateArgs {
  const double* H1 = nullptr;  // winSVD: H = H1 + H2; Halko: H1 = nullptr, H2 = nullptr
  const double* H2 = nullptr;
  double* H = nullptr;         // N x l: written when H2 is given, else the input sketch
  double* Q = nullptr;         // N x l work (Q1 then Q)
  double* Omg = nullptr;       // N x l outputs
  double* Omg2 = nullptr;
  float* Omgf = nullptr;       // FP32 operand copy (SIMT path) or null
  __nv_bfloat16* bt1 = nullptr;  // split-BF16 operand (tc_layout.hpp) or null
  int64_t kpad = 0;
  int bt_half = 0;               // row offset of the lo half in bt1 (= NP / 2)
  double* wsum = nullptr;      // l
  double* part = nullptr;      // update_part_doubles(l) work
  double* R1 = nullptr;        // l x l work
  double* R2 = nullptr;
  double* D = nullptr;         // l
  double* mult = nullptr;      // l
  unsigned* counters = nullptr;  // 4 tickets, zero between calls
  int* status = nullptr;
  int64_t N = 0;
  int l = 0;
};

// doubles of UpdateArgs::part for sketch width l
size_t update_part_doubles(int l);
void fused_update(pcaone_ctx* c, UpdateArgs a);

}  // namespace pg
