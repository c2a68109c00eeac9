// rhok_noalloc.cu -- structure factors without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need k-space structure
// factors: an MD engine that owns every device allocation through its own pool or a fixed
// budget handed out at start-up (a library-side cudaMalloc would fail near capacity or
// fragment that pool), or a time-step loop that keeps several streams busy and cannot take
// the device-wide synchronisation that cudaFree implies.  For them this file provides one
// entry point, rbmd_rhok_noalloc, that computes rho_k = sum_j q_j exp(i k.r_j) with the same
// fixed-point phase arithmetic as the force path but keeps all of its scratch (fixed-point
// coordinates and per-block partial sums) in a file-scope static device array of fixed size.
// The caller still passes the inputs and the output.
//
// Limits and sharing rules:
//   * scratch is kNoAllocScratchBytes (8 MiB) per device, held by every GPU that loads the
//     library until the process exits;
//   * n <= kNoAllocMaxAtoms and P <= kNoAllocMaxK, otherwise RBMD_ERR_ARG (nothing launched);
//   * every call on a device shares the one array and leaves its contents behind; all of it is
//     overwritten before it is read, so nothing needs clearing between calls, but calls that
//     overlap on the GPU (different streams, or different host threads) race on it;
//   * the array's device address comes from cudaGetSymbolAddress (in host code the array's
//     name is only a host-side stand-in).  Each call made while its stream is not capturing
//     looks the address up again in the current context, so a device reset or another context
//     on the device never leaves a stale address behind; the first call on a device (and after a
//     reset) does this set-up, so make it before any stream capture begins.  A call made during
//     capture reuses the address recorded for the current context and refuses (RBMD_ERR_CUDA)
//     when none is recorded;
//   * a NaN position gives unspecified structure factors (its fixed-point turn is undefined).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/rbmd_force.h"
#include "common.cuh"

namespace rbmd_internal {
extern char g_last_error[512];   // shared with rbmd_force.cu (rbmd_last_error)
}

namespace {

constexpr int kNoAllocMaxAtoms = 262144;                 // fixed-point coordinates: 4 MiB
constexpr int kNoAllocMaxK = 1024;
constexpr int kNoAllocChunk = 2048;                      // atoms per structure-factor block
constexpr size_t kNoAllocFracBytes = (size_t)kNoAllocMaxAtoms * sizeof(rbmd::Frac32);
constexpr size_t kNoAllocScratchBytes = 8u << 20;        // 8 MiB in total
constexpr int kMaxDevices = 64;

// The scratch array.  Host code must not pass `g_noalloc_scratch` to a kernel: in host code the
// name is a stand-in, the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Per device: the scratch address and the id of the context it was looked up in.
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

void set_error(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(rbmd_internal::g_last_error, sizeof rbmd_internal::g_last_error, fmt, ap);
  va_end(ap);
}

// Unique id of the calling thread's current context (cuCtxGetId, CUDA 12.0+), reached through
// the runtime's driver entry points so that the library needs no link to libcuda.  0 if unknown.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

__global__ void k_na_frac(int n, const double* __restrict__ pos, const double* __restrict__ charge,
                          double lo0, double lo1, double lo2, double L0, double L1, double L2,
                          rbmd::Frac32* __restrict__ frac) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lo[3] = {lo0, lo1, lo2}, L[3] = {L0, L1, L2};
  uint32_t U[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double u = (pos[3 * i + d] - lo[d]) / L[d];
    U[d] = rbmd::turn32(u - floor(u));   // a whole turn wraps to 0
  }
  frac[i] = rbmd::Frac32{U[0], U[1], U[2], (float)charge[i]};
}

// One sample per lane (up to 32 per warp, P <= 32 * warps), the block's chunk of atoms staged
// in shared memory and read by broadcast; partial[(chunk * P + k) * 2 + {0,1}] in FP32.
__global__ void __launch_bounds__(1024) k_na_rho(int n, int P, const rbmd::Frac32* __restrict__ frac,
                                                 const int* __restrict__ m, float* __restrict__ partial) {
  __shared__ rbmd::Frac32 stage[256];
  const int k = threadIdx.x;
  const bool ok = k < P;
  const uint32_t mx = ok ? (uint32_t)m[3 * k] : 0u, my = ok ? (uint32_t)m[3 * k + 1] : 0u,
                 mz = ok ? (uint32_t)m[3 * k + 2] : 0u;
  const int a0 = blockIdx.x * kNoAllocChunk, a1 = min(n, a0 + kNoAllocChunk);
  float re = 0.f, im = 0.f;
  for (int base = a0; base < a1; base += 256) {
    const int cnt = min(256, a1 - base);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) stage[t] = frac[base + t];
    __syncthreads();
    if (!ok) continue;
    for (int a = 0; a < cnt; ++a) {
      const rbmd::Frac32 f = stage[a];
      const uint32_t ph = mx * f.x + my * f.y + mz * f.z;
      // top 23 bits -> float in [1, 2); angle 2 pi (t - 1/2) in [-pi, pi)
      const float tf = __uint_as_float((ph >> 9) | 0x3F800000u) - 1.5f;
      float s, c;
      __sincosf(tf * 6.28318530717958647692f, &s, &c);
      re = fmaf(f.q, c, re);
      im = fmaf(f.q, s, im);
    }
  }
  if (ok) {
    partial[((size_t)blockIdx.x * P + k) * 2] = re;
    partial[((size_t)blockIdx.x * P + k) * 2 + 1] = im;
  }
}

// One warp per sample: fixed-order FP64 sum of the chunk partials; the angle was shifted by half
// a turn, which negates both components.
__global__ void k_na_finish(int P, int nchunks, const float* __restrict__ partial, double* __restrict__ rho) {
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= P) return;
  double re = 0, im = 0;
  for (int c = lane; c < nchunks; c += 32) {
    re += (double)partial[((size_t)c * P + k) * 2];
    im += (double)partial[((size_t)c * P + k) * 2 + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane == 0) {
    rho[2 * k] = -re;
    rho[2 * k + 1] = -im;
  }
}

}  // namespace

extern "C" {

RBMD_API rbmd_status rbmd_rhok_noalloc(const double* pos_dev, const double* charge_dev, int32_t n,
                                       const rbmd_box* box, const int32_t* m_dev, int32_t P,
                                       double* rho_dev, void* stream) {
  if (!pos_dev || !charge_dev || !box || !m_dev || !rho_dev || n < 1 || P < 1) {
    set_error("rbmd_rhok_noalloc: null pointer or non-positive size (n=%d, P=%d)", n, P);
    return RBMD_ERR_ARG;
  }
  const int nchunks = (n + kNoAllocChunk - 1) / kNoAllocChunk;
  const size_t partial_bytes = (size_t)nchunks * P * 2 * sizeof(float);
  if (n > kNoAllocMaxAtoms || P > kNoAllocMaxK || kNoAllocFracBytes + partial_bytes > kNoAllocScratchBytes) {
    set_error("rbmd_rhok_noalloc: n=%d, P=%d exceed the fixed scratch (n <= %d, P <= %d)", n, P,
              kNoAllocMaxAtoms, kNoAllocMaxK);
    return RBMD_ERR_ARG;
  }
  double L[3];
  for (int d = 0; d < 3; ++d) {
    L[d] = box->hi[d] - box->lo[d];
    if (!(L[d] > 0)) {
      set_error("rbmd_rhok_noalloc: box length %g along axis %d is not positive", L[d], d);
      return RBMD_ERR_ARG;
    }
  }
  // an error left pending by the caller's earlier work is reported as such, not as ours
  const cudaError_t pending = cudaGetLastError();
  if (pending != cudaSuccess) {
    set_error("rbmd_rhok_noalloc: a CUDA error from earlier work was pending (nothing launched): %s",
              cudaGetErrorString(pending));
    return RBMD_ERR_CUDA;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("rbmd_rhok_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return RBMD_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("rbmd_rhok_noalloc: device %d is beyond the %d devices this entry point serves", dev, kMaxDevices);
    return RBMD_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();                       // the query's own error; treat as capturing
    cap = cudaStreamCaptureStatusActive;
  }
  const unsigned long long ctx = current_context_id();
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      // with the device current: the static array's address in the current context
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_error("rbmd_rhok_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return RBMD_ERR_CUDA;
      }
      g_scratch_ptr[dev] = p;
      g_scratch_ctx[dev] = ctx;
    } else if (!g_scratch_ptr[dev] || ctx == 0 || g_scratch_ctx[dev] != ctx) {
      set_error("rbmd_rhok_noalloc: called during stream capture before any call in this context "
                "(make the first call outside capture)");
      return RBMD_ERR_CUDA;
    }
    base = g_scratch_ptr[dev];
  }
  rbmd::Frac32* frac = reinterpret_cast<rbmd::Frac32*>(base);
  float* partial = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + kNoAllocFracBytes);
  k_na_frac<<<(n + 255) / 256, 256, 0, s>>>(n, pos_dev, charge_dev, box->lo[0], box->lo[1], box->lo[2], L[0],
                                           L[1], L[2], frac);
  const int threads = ((P + 31) / 32) * 32;
  k_na_rho<<<nchunks, threads, 0, s>>>(n, P, frac, m_dev, partial);
  k_na_finish<<<(P + 3) / 4, 128, 0, s>>>(P, nchunks, partial, rho_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("rbmd_rhok_noalloc: launch failed: %s", cudaGetErrorString(e));
    return RBMD_ERR_CUDA;
  }
  return RBMD_OK;
}

}  // extern "C"
