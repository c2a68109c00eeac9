// mlp_types.cuh -- sizes, parameter layout and launch arguments of the proposal network
// (kernels in kernels_mlp.cuh, compiled in proposal.cu only).
#pragma once
#include <cstdint>

namespace rbmd {

constexpr int kMlpIn = 16, kMlpHid = 64, kMlpRows = 256;
// parameter vector: W1 [64][16], b1 [64], W2 [64][64], b2 [64], w3 [64], b3
constexpr int kOW1 = 0, kOB1 = 1024, kOW2 = 1088, kOB2 = 5184, kOW3 = 5248, kOB3 = 5312;
constexpr int kMlpNParam = 5313;
constexpr uint32_t kFlagMlpTimeout = 0x80u;   // an mbarrier wait of the MLP kernel gave up

struct MlpArgs {
  int groups;                  // CTAs; rows = groups * 256
  int train;                   // 0: forward only (h); 1: also loss and parameter gradients
  float gscale;                // d(total loss)/d(group loss), e.g. 1/groups
  const float* params;         // [kMlpNParam] FP32 master copy
  const float* x;              // [rows][16] features (rounded to BF16 on load)
  const float* wbin;           // [rows] W_b (train)
  const float* cbin;           // [rows] C_b (train)
  float* h;                    // [rows] output h (may be null in training)
  double* loss;                // [groups] l per group (train)
  float* grad_partial;         // [groups][kMlpNParam] per-group gradient (train)
  uint32_t* status;
};

}  // namespace rbmd
