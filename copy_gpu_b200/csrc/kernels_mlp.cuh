// kernels_mlp.cuh -- the k-proposal network of the learned RBE sampler on the 5th-generation
// tensor cores: a 16 -> 64 -> 64 -> 1 perceptron (tanh hidden units, BF16 operands, FP32
// accumulation) evaluated and trained on groups of 256 rows, one CTA per group.
//
// Per CTA: the operands of every GEMM are staged in shared memory in the canonical K-major
// "core matrix" layout without swizzle (8 rows x 16 bytes per core matrix; core matrices along K
// 128 bytes apart, 8-row groups K*16 bytes apart), one thread issues tcgen05.mma (kind::f16,
// M = 128, N = 64, K = 16 per instruction) for each of the two 128-row tiles, the accumulators
// live in 128 TMEM columns (tile t in columns [64t, 64t + 64)), tcgen05.commit arrives on an
// mbarrier, and each thread reads its own row back with tcgen05.ld (warp w reads TMEM lanes
// 32 (w % 4) .. 32 (w % 4) + 31, i.e. thread t owns row t).  GEMMs on the tensor cores:
// Z1 = X W1^T, Z2 = A1 W2^T (forward) and dA1 = dZ2 W2 (backward).  The weight gradients
// (sums over the 256 rows) are FP32 reductions on the CUDA cores.
//
// Training loss of a group (one snapshot): l = log sum_b W_b e^{h_b} + log sum_b C_b e^{-h_b},
// the logarithm of the RBE force variance sum_b C_b / q_b of the proposal q_b = W_b e^{h_b} / Z
// (W_b: Gaussian mass of bin b, C_b: variance weight of bin b); it is minimised by
// e^{h_b} ~ sqrt(C_b / W_b) and does not change when a constant is added to h.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

#include "common.cuh"
#include "mlp_forward.cuh"
#include "mlp_types.cuh"

namespace rbmd {

struct __align__(1024) MlpSmem {
  uint16_t x[kMlpRows * kMlpIn];        //  8 KB  X    [256][16]   (A of layer 1)
  uint16_t w1[kMlpHid * kMlpIn];        //  2 KB  W1   [64][16]    (B of layer 1)
  uint16_t w2[kMlpHid * kMlpHid];       //  8 KB  W2   [64][64]    (B of layer 2)
  uint16_t w2t[kMlpHid * kMlpHid];      //  8 KB  W2^T [64][64]    (B of dA1 = dZ2 W2)
  uint16_t a1[kMlpRows * kMlpHid];      // 32 KB  A1   [256][64]   (A of layer 2)
  uint16_t dz2[kMlpRows * kMlpHid];     // 32 KB  dZ2  [256][64]   (A of dA1); then dZ1 FP32 over a1+dz2
  float red[8][kMlpHid];                // per-warp partial sums
  float gsum[8][4];
  float par_b1[kMlpHid], par_b2[kMlpHid], par_w3[kMlpHid];
  float scal[8];
  unsigned long long mbar;
  uint32_t tmem;
};

// element offset of (row r, column k) in a [rows][K] K-major core-matrix layout
__device__ __forceinline__ int core_off(int r, int k, int K) {
  return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint16_t to_bf16(float v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
__device__ __forceinline__ float from_bf16(uint16_t v) { return __bfloat162float(__ushort_as_bfloat16(v)); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor (SWIZZLE_NONE, K-major): start address, leading byte offset
// (between core matrices along K) = 128 B, stride byte offset (between 8-row groups) = K * 16 B,
// all in 16-byte units; bits 46-47 = 1 (descriptor version of this architecture)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 64, M = 128
constexpr uint32_t kMlpIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(kMlpIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(unsigned long long* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(mbar))
               : "memory");
}

// bounded wait on an mbarrier phase; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long* mbar, uint32_t parity) {
  const uint32_t a = smem_u32(mbar);
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum the per-thread values v[64] over the block's 256 rows into out[64] (fixed order).
__device__ __forceinline__ void block_colsum(MlpSmem& S, const float* v, float* out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kMlpHid; ++j) {
    const float s = warp_sum(v[j]);
    if (lane == 0) S.red[w][j] = s;
  }
  __syncthreads();
  if (threadIdx.x < kMlpHid) {
    float s = 0;
    for (int k = 0; k < 8; ++k) s += S.red[k][threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// One CTA = one group of 256 rows, 256 threads (thread t = row t).
__global__ void __launch_bounds__(256, 1) k_mlp(MlpArgs args) {
  extern __shared__ unsigned char smem_raw[];
  MlpSmem& S = *reinterpret_cast<MlpSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int g = blockIdx.x;
  const size_t row = (size_t)g * kMlpRows + t;
  const float* P = args.params;

  // ---- stage operands (generic proxy) ----
#pragma unroll
  for (int f = 0; f < kMlpIn; ++f) S.x[core_off(t, f, kMlpIn)] = to_bf16(args.x[row * kMlpIn + f]);
  for (int e = t; e < kMlpHid * kMlpIn; e += 256) {
    const int j = e / kMlpIn, f = e % kMlpIn;
    S.w1[core_off(j, f, kMlpIn)] = to_bf16(P[kOW1 + e]);
  }
  for (int e = t; e < kMlpHid * kMlpHid; e += 256) {
    const int j = e / kMlpHid, i = e % kMlpHid;   // W2[j][i]: output j, input i
    const uint16_t v = to_bf16(P[kOW2 + e]);
    S.w2[core_off(j, i, kMlpHid)] = v;
    S.w2t[core_off(i, j, kMlpHid)] = v;
  }
  if (t < kMlpHid) {
    S.par_b1[t] = P[kOB1 + t];
    S.par_b2[t] = P[kOB2 + t];
    S.par_w3[t] = P[kOW3 + t];
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(smem_u32(&S.tmem)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const int tile = t >> 7;
  const uint32_t my_lane_addr = tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)(64 * tile);
  uint32_t parity = 0;
  bool ok = true;
  const uint32_t xa = smem_u32(S.x), w1a = smem_u32(S.w1), w2a = smem_u32(S.w2), w2ta = smem_u32(S.w2t);
  const uint32_t a1a = smem_u32(S.a1), dz2a = smem_u32(S.dz2);

  // ---- layer 1: Z1 = X W1^T (K = 16: one instruction per tile) ----
  if (t == 0) {
    tc_fence_after();
    for (int tl = 0; tl < 2; ++tl)
      mma_bf16(tmem + 64 * tl, smem_desc(xa + tl * 16 * (kMlpIn * 16), kMlpIn * 16), smem_desc(w1a, kMlpIn * 16), 0);
    mma_commit(&S.mbar);
  }
  ok = mbar_wait(&S.mbar, parity);
  parity ^= 1;
  if (!__syncthreads_and(ok)) goto fail;
  tc_fence_after();
  {
    float z[16];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      tmem_ld16(my_lane_addr + 16 * c, z);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int j = 16 * c + k;
        S.a1[core_off(t, j, kMlpHid)] = to_bf16(tanhf(z[k] + S.par_b1[j]));
      }
    }
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();

  // ---- layer 2: Z2 = A1 W2^T (K = 64: four instructions per tile) ----
  if (t == 0) {
    tc_fence_after();
    for (int tl = 0; tl < 2; ++tl)
      for (int ks = 0; ks < 4; ++ks)
        mma_bf16(tmem + 64 * tl, smem_desc(a1a + tl * 16 * (kMlpHid * 16) + ks * 256, kMlpHid * 16),
                 smem_desc(w2a + ks * 256, kMlpHid * 16), ks > 0);
    mma_commit(&S.mbar);
  }
  ok = mbar_wait(&S.mbar, parity);
  parity ^= 1;
  if (!__syncthreads_and(ok)) goto fail;
  tc_fence_after();
  {
    float a2[kMlpHid];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float z[16];
      tmem_ld16(my_lane_addr + 16 * c, z);
#pragma unroll
      for (int k = 0; k < 16; ++k) a2[16 * c + k] = tanhf(z[k] + S.par_b2[16 * c + k]);
    }
    float h = P[kOB3];
#pragma unroll
    for (int j = 0; j < kMlpHid; ++j) h = fmaf(a2[j], S.par_w3[j], h);
    if (args.h) args.h[row] = h;
    if (!args.train) goto done;

    // ---- loss of the group and dl/dh of each row ----
    float hmax = h, hmin = h;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      hmax = fmaxf(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
      hmin = fminf(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
    }
    if (lane == 0) { S.gsum[w][0] = hmax; S.gsum[w][1] = hmin; }
    __syncthreads();
    if (t == 0) {
      float a = S.gsum[0][0], b = S.gsum[0][1];
      for (int k = 1; k < 8; ++k) { a = fmaxf(a, S.gsum[k][0]); b = fminf(b, S.gsum[k][1]); }
      S.scal[0] = a;
      S.scal[1] = b;
    }
    __syncthreads();
    hmax = S.scal[0];
    hmin = S.scal[1];
    const float wb = args.wbin[row], cb = args.cbin[row];
    const float ep = wb * __expf(h - hmax), em = cb * __expf(hmin - h);
    const float sp = warp_sum(ep), sm = warp_sum(em);
    if (lane == 0) { S.gsum[w][2] = sp; S.gsum[w][3] = sm; }
    __syncthreads();
    if (t == 0) {
      float a = 0, b = 0;
      for (int k = 0; k < 8; ++k) { a += S.gsum[k][2]; b += S.gsum[k][3]; }
      S.scal[2] = a;
      S.scal[3] = b;
      args.loss[g] = (double)hmax + log((double)a) - (double)hmin + log((double)b);
    }
    __syncthreads();
    const float dh = args.gscale * (ep / S.scal[2] - em / S.scal[3]);

    // ---- output layer and layer-2 gradients ----
    float* G = args.grad_partial + (size_t)g * kMlpNParam;
    {
      const float db3 = warp_sum(dh);
      if (lane == 0) S.gsum[w][0] = db3;
      __syncthreads();
      if (t == 0) {
        float s = 0;
        for (int k = 0; k < 8; ++k) s += S.gsum[k][0];
        G[kOB3] = s;
      }
    }
    float v[kMlpHid];
#pragma unroll
    for (int j = 0; j < kMlpHid; ++j) v[j] = dh * a2[j];
    block_colsum(S, v, G + kOW3);                      // dw3
#pragma unroll
    for (int j = 0; j < kMlpHid; ++j) {
      v[j] = dh * S.par_w3[j] * (1.0f - a2[j] * a2[j]);   // dZ2
      S.dz2[core_off(t, j, kMlpHid)] = to_bf16(v[j]);
    }
    block_colsum(S, v, G + kOB2);                      // db2 (block_colsum synchronises)
  }
  // ---- dA1 = dZ2 W2 on the tensor cores, dW2 = dZ2^T A1 on the CUDA cores meanwhile ----
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  if (t == 0) {
    tc_fence_after();
    for (int tl = 0; tl < 2; ++tl)
      for (int ks = 0; ks < 4; ++ks)
        mma_bf16(tmem + 64 * tl, smem_desc(dz2a + tl * 16 * (kMlpHid * 16) + ks * 256, kMlpHid * 16),
                 smem_desc(w2ta + ks * 256, kMlpHid * 16), ks > 0);
    mma_commit(&S.mbar);
  }
  {
    float* G = args.grad_partial + (size_t)g * kMlpNParam;
    const int j = t >> 2, i0 = (t & 3) * 16;
    float acc[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k] = 0.f;
    for (int r = 0; r < kMlpRows; ++r) {
      const float d = from_bf16(S.dz2[core_off(r, j, kMlpHid)]);
#pragma unroll
      for (int k = 0; k < 16; ++k) acc[k] = fmaf(d, from_bf16(S.a1[core_off(r, i0 + k, kMlpHid)]), acc[k]);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) G[kOW2 + j * kMlpHid + i0 + k] = acc[k];
  }
  ok = mbar_wait(&S.mbar, parity);
  parity ^= 1;
  if (!__syncthreads_and(ok)) goto fail;
  tc_fence_after();
  {
    float dz1[kMlpHid];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float z[16];
      tmem_ld16(my_lane_addr + 16 * c, z);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int i = 16 * c + k;
        const float a = from_bf16(S.a1[core_off(t, i, kMlpHid)]);
        dz1[i] = z[k] * (1.0f - a * a);
      }
    }
    float* G = args.grad_partial + (size_t)g * kMlpNParam;
    block_colsum(S, dz1, G + kOB1);                    // db1 (synchronises: A1 and dZ2 are free now)
    float* dz1s = reinterpret_cast<float*>(S.a1);      // [256][64] FP32 over a1 + dz2
#pragma unroll
    for (int i = 0; i < kMlpHid; ++i) dz1s[t * kMlpHid + ((i + t) & 63)] = dz1[i];
    __syncthreads();
    const int i = t >> 2, f0 = (t & 3) * 4;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int r = 0; r < kMlpRows; ++r) {
      const float d = dz1s[r * kMlpHid + ((i + r) & 63)];
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = fmaf(d, from_bf16(S.x[core_off(r, f0 + k, kMlpIn)]), acc[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) G[kOW1 + i * kMlpIn + f0 + k] = acc[k];
  }
  goto done;
fail:
  if (t == 0) atomicOr(args.status, kFlagMlpTimeout);
done:
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem));
  }
}

// Sum of the per-group gradients in group order (deterministic), one thread per parameter.
// T from the parameter vector P (layout in mlp_forward.cuh), one thread per word
__global__ void k_mlp_prep(const float* __restrict__ P, float* __restrict__ T) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kMlpNParam) return;
  if (e >= kTW1 && e < kTW1 + kMlpHid * kMlpIn) {          // T[kTW1 + f * 64 + j] = W1[j][f]
    const int k = e - kTW1, f = k / kMlpHid, j = k % kMlpHid;
    T[e] = mlp_bf16(P[kOW1 + j * kMlpIn + f]);
  } else if (e >= kTW2 && e < kTW2 + kMlpHid * kMlpHid) {   // T[kTW2 + i * 64 + j] = W2[j][i]
    const int k = e - kTW2, i = k / kMlpHid, j = k % kMlpHid;
    T[e] = mlp_bf16(P[kOW2 + j * kMlpHid + i]);
  } else {
    T[e] = P[e];
  }
}

// Forward pass alone on the CUDA cores (mlp_row_forward, kMlpLanes lanes per row, prepared weights
// T): the entry point's train < 0 evaluation, the same arithmetic as the sampler's per-step
// evaluation k_prop_h.
__global__ void __launch_bounds__(256) k_mlp_infer(int rows, const float* __restrict__ T,
                                                  const float* __restrict__ x, float* __restrict__ h) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = gt / kMlpLanes, part = gt % kMlpLanes;
  const int r = row < rows ? row : rows - 1;   // every lane joins the shuffles
  const float v = mlp_row_forward<kMlpLanes>(T, x + (size_t)r * kMlpIn, part);
  if (row < rows && part == 0) h[row] = v;
}

__global__ void k_mlp_grad_sum(int groups, const float* __restrict__ partial, float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpNParam) return;
  float s = 0;
  for (int g = 0; g < groups; ++g) s += partial[(size_t)g * kMlpNParam + p];
  grad[p] = s;
}

// Adam (Kingma & Ba, ICLR 2015) on the FP32 master parameters.
__global__ void k_adam(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, int step) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpNParam) return;
  const float gr = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * gr;
  const float vv = b2 * v[p] + (1.f - b2) * gr * gr;
  m[p] = mm;
  v[p] = vv;
  const float mh = mm / (1.f - powf(b1, (float)step)), vh = vv / (1.f - powf(b2, (float)step));
  params[p] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace rbmd
