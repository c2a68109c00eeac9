// mlp_forward.cuh -- forward pass of the proposal network for one row on four lanes of a warp,
// on the CUDA cores (the per-step evaluation of the sampler; training runs k_mlp on the tensor
// cores).  Same BF16 roundings as k_mlp (inputs, W1, W2 and the layer-1 activations), FP32 sums.
#pragma once
#include <cuda_bf16.h>

#include "mlp_types.cuh"

namespace rbmd {

__device__ __forceinline__ float mlp_bf16(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// h of the row whose 16 inputs are x[0..15], computed by G consecutive lanes of the calling warp
// (G = 2 .. 32, a power of two), all of which must call it with part = lane % G: lane `part`
// evaluates hidden units U part .. U part + U - 1 (U = 64 / G) of both layers; the layer-1
// activations are exchanged by shuffles and the G partial outputs summed by a butterfly.  Every
// calling lane gets h.
template <int G>
__device__ __forceinline__ float mlp_row_forward(const float* __restrict__ P, const float* x, int part) {
  static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "G lanes per row, a power of two");
  constexpr int U = kMlpHid / G;
  const int base = (threadIdx.x & 31) & ~(G - 1);
  float xb[kMlpIn];
#pragma unroll
  for (int f = 0; f < kMlpIn; ++f) xb[f] = mlp_bf16(x[f]);
  float a1[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int j = U * part + u;
    float z = 0.f;
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) z = fmaf(xb[f], mlp_bf16(__ldg(P + kOW1 + j * kMlpIn + f)), z);
    a1[u] = mlp_bf16(tanhf(z + __ldg(P + kOB1 + j)));
  }
  float z2[U];
#pragma unroll
  for (int u = 0; u < U; ++u) z2[u] = 0.f;
#pragma unroll
  for (int i = 0; i < kMlpHid; ++i) {
    const float ai = __shfl_sync(0xffffffffu, a1[i % U], base | (i / U));
#pragma unroll
    for (int u = 0; u < U; ++u) z2[u] = fmaf(ai, mlp_bf16(__ldg(P + kOW2 + (U * part + u) * kMlpHid + i)), z2[u]);
  }
  float hp = 0.f;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int j = U * part + u;
    hp = fmaf(tanhf(z2[u] + __ldg(P + kOB2 + j)), __ldg(P + kOW3 + j), hp);
  }
#pragma unroll
  for (int o = 1; o < G; o <<= 1) hp += __shfl_xor_sync(0xffffffffu, hp, o);
  return __ldg(P + kOB3) + hp;
}

// lanes per row of the sampler's per-step evaluation (k_prop_h, k_mlp_infer)
constexpr int kMlpLanes = 16;

}  // namespace rbmd
