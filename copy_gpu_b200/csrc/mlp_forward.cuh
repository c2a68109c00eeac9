// mlp_forward.cuh -- forward pass of the proposal network for one row on four lanes of a warp,
// on the CUDA cores (the per-step evaluation of the sampler; training runs k_mlp on the tensor
// cores).  Same BF16 roundings as k_mlp (inputs, W1, W2 and the layer-1 activations), FP32 sums.
#pragma once
#include <cuda_bf16.h>

#include "mlp_types.cuh"

namespace rbmd {

__device__ __forceinline__ float mlp_bf16(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Layout of the prepared weights T[kMlpNParam] (k_mlp_prep, once per parameter change): the
// parameter vector's offsets, with W1 and W2 transposed and rounded to BF16,
// T[kTW1 + f * 64 + j] = W1[j][f] and T[kTW2 + i * 64 + j] = W2[j][i]; b1, b2, w3 and b3 as they
// are.  Lanes that hold consecutive hidden units j read consecutive words.
constexpr int kTW1 = kOW1, kTW2 = kOW2;

// h of the row whose 16 inputs are x[0..15], computed by G consecutive lanes of the calling warp
// (G = 2 .. 32, a power of two), all of which must call it with part = lane % G: lane `part`
// evaluates hidden units j = part + G u (u < 64 / G) of both layers, so the lanes of a group read
// consecutive words of T; the layer-1 activations are exchanged by shuffles and the G partial
// outputs summed by a butterfly.  Every calling lane gets h.
template <int G>
__device__ __forceinline__ float mlp_row_forward(const float* __restrict__ T, const float* x, int part) {
  static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "G lanes per row, a power of two");
  constexpr int U = kMlpHid / G;
  const int base = (threadIdx.x & 31) & ~(G - 1);
  float xb[kMlpIn];
#pragma unroll
  for (int f = 0; f < kMlpIn; ++f) xb[f] = mlp_bf16(x[f]);
  float a1[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int j = part + G * u;
    float z = 0.f;
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) z = fmaf(xb[f], __ldg(T + kTW1 + f * kMlpHid + j), z);
    a1[u] = mlp_bf16(tanhf(z + __ldg(T + kOB1 + j)));
  }
  float z2[U];
#pragma unroll
  for (int u = 0; u < U; ++u) z2[u] = 0.f;
#pragma unroll
  for (int i = 0; i < kMlpHid; ++i) {
    const float ai = __shfl_sync(0xffffffffu, a1[i / G], base | (i % G));
#pragma unroll
    for (int u = 0; u < U; ++u) z2[u] = fmaf(ai, __ldg(T + kTW2 + i * kMlpHid + part + G * u), z2[u]);
  }
  float hp = 0.f;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int j = part + G * u;
    hp = fmaf(tanhf(z2[u] + __ldg(T + kOB2 + j)), __ldg(T + kOW3 + j), hp);
  }
#pragma unroll
  for (int o = 1; o < G; o <<= 1) hp += __shfl_xor_sync(0xffffffffu, hp, o);
  return __ldg(T + kOB3) + hp;
}

// lanes per row of the sampler's per-step evaluation (k_prop_h, k_mlp_infer)
constexpr int kMlpLanes = 16;

}  // namespace rbmd
