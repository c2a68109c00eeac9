// mlp_forward.cuh -- forward pass of the proposal network for one row on four lanes of a warp,
// on the CUDA cores (the per-step evaluation of the sampler; training runs k_mlp on the tensor
// cores).  Same BF16 roundings as k_mlp (inputs, W1, W2 and the layer-1 activations), FP32 sums.
#pragma once
#include <cuda_bf16.h>

#include "mlp_types.cuh"

namespace rbmd {

__device__ __forceinline__ float mlp_bf16(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// h of the row whose 16 inputs are x[0..15], computed by the four lanes (lane & ~3) .. (lane | 3)
// of the calling warp, all of which must call it (with part = lane & 3): lane `part` evaluates
// hidden units 16 part .. 16 part + 15 of both layers; the layer-1 activations are exchanged by
// shuffles and the four partial outputs summed.  Every calling lane gets h.
__device__ __forceinline__ float mlp_row_forward4(const float* __restrict__ P, const float* x, int part) {
  const int base = (threadIdx.x & 31) & ~3;
  float xb[kMlpIn];
#pragma unroll
  for (int f = 0; f < kMlpIn; ++f) xb[f] = mlp_bf16(x[f]);
  float a1[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int j = 16 * part + u;
    float z = 0.f;
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) z = fmaf(xb[f], mlp_bf16(__ldg(P + kOW1 + j * kMlpIn + f)), z);
    a1[u] = mlp_bf16(tanhf(z + __ldg(P + kOB1 + j)));
  }
  float z2[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) z2[u] = 0.f;
#pragma unroll
  for (int i = 0; i < kMlpHid; ++i) {
    const float ai = __shfl_sync(0xffffffffu, a1[i & 15], base | (i >> 4));
#pragma unroll
    for (int u = 0; u < 16; ++u) z2[u] = fmaf(ai, mlp_bf16(__ldg(P + kOW2 + (16 * part + u) * kMlpHid + i)), z2[u]);
  }
  float hp = 0.f;
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int j = 16 * part + u;
    hp = fmaf(tanhf(z2[u] + __ldg(P + kOB2 + j)), __ldg(P + kOW3 + j), hp);
  }
  hp += __shfl_xor_sync(0xffffffffu, hp, 1);
  hp += __shfl_xor_sync(0xffffffffu, hp, 2);
  return __ldg(P + kOB3) + hp;
}

}  // namespace rbmd
