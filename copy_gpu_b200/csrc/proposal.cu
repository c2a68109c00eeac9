// proposal.cu -- host side of the learned k-proposal network: launches of the tcgen05 MLP
// kernel (evaluation, gradients, Adam) shared by the training driver and the sampler.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <set>

#include "../../include/rbmd_force.h"
#include "kernels_mlp.cuh"
#include "proposal.hpp"

namespace rbmd_internal {
extern char g_last_error[512];
}

namespace rbmd {

cudaError_t mlp_launch(const MlpArgs& a, cudaStream_t s) {
  // the shared-memory limit is a per-device attribute of the kernel: set once on each device
  static std::mutex mu;
  static std::set<int> devices_set;
  const size_t smem = sizeof(MlpSmem) + 1024;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!devices_set.count(dev)) {
      e = cudaFuncSetAttribute(k_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      devices_set.insert(dev);
    }
  }
  k_mlp<<<a.groups, 256, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t mlp_prepare(const float* params, float* prepared, cudaStream_t s) {
  k_mlp_prep<<<(kMlpNParam + 255) / 256, 256, 0, s>>>(params, prepared);
  return cudaGetLastError();
}

cudaError_t mlp_infer(int groups, const float* prepared, const float* x, float* h, cudaStream_t s) {
  const int rows = groups * kMlpRows;
  k_mlp_infer<<<(kMlpLanes * rows + 255) / 256, 256, 0, s>>>(rows, prepared, x, h);
  return cudaGetLastError();
}

cudaError_t mlp_grad_sum(int groups, const float* partial, float* grad, cudaStream_t s) {
  k_mlp_grad_sum<<<(kMlpNParam + 255) / 256, 256, 0, s>>>(groups, partial, grad);
  return cudaGetLastError();
}

cudaError_t mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int step, cudaStream_t s) {
  k_adam<<<(kMlpNParam + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, 0.9f, 0.999f, 1e-8f, step);
  return cudaGetLastError();
}

}  // namespace rbmd

extern "C" {

RBMD_API rbmd_status rbmd_proposal_mlp_eval(const float* params, const float* x, const float* wbin,
                                            const float* cbin, int32_t groups, int32_t train, float* h,
                                            double* loss, float* grad, uint32_t* status, void* stream) {
  using namespace rbmd;
  if (!params || !x || groups < 1 || !status || (train > 0 && (!wbin || !cbin || !loss || !grad)) ||
      (train < 0 && !h))
    return RBMD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (train < 0) {   // the sampler's per-step forward pass on the CUDA cores
    float* prepared = nullptr;
    if (cudaMalloc(&prepared, sizeof(float) * kMlpNParam) != cudaSuccess) return RBMD_ERR_CUDA;
    cudaError_t e = mlp_prepare(params, prepared, s);
    if (e == cudaSuccess) e = mlp_infer(groups, prepared, x, h, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(prepared);
    if (e != cudaSuccess) {
      std::snprintf(rbmd_internal::g_last_error, sizeof rbmd_internal::g_last_error, "mlp_eval: %s",
                    cudaGetErrorString(e));
      return RBMD_ERR_CUDA;
    }
    return RBMD_OK;
  }
  float* partial = nullptr;
  if (train && cudaMalloc(&partial, sizeof(float) * (size_t)groups * kMlpNParam) != cudaSuccess)
    return RBMD_ERR_CUDA;
  MlpArgs a{};
  a.groups = groups;
  a.train = train > 0;
  a.gscale = 1.0f / (float)groups;
  a.params = params;
  a.x = x;
  a.wbin = wbin;
  a.cbin = cbin;
  a.h = h;
  a.loss = loss;
  a.grad_partial = partial;
  a.status = status;
  cudaError_t e = mlp_launch(a, s);
  if (e == cudaSuccess && train) e = mlp_grad_sum(groups, partial, grad, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (partial) cudaFree(partial);
  if (e != cudaSuccess) {
    std::snprintf(rbmd_internal::g_last_error, sizeof rbmd_internal::g_last_error, "mlp_eval: %s",
                  cudaGetErrorString(e));
    return RBMD_ERR_CUDA;
  }
  return RBMD_OK;
}

}  // extern "C"
