// proposal.hpp -- launch helpers of the learned k-proposal network (proposal.cu).
#pragma once
#include <cuda_runtime.h>

#include "mlp_types.cuh"

namespace rbmd {
cudaError_t mlp_launch(const MlpArgs& a, cudaStream_t s);
// the CUDA-core forward pass's weight layout (k_mlp_prep) from the parameter vector
cudaError_t mlp_prepare(const float* params, float* prepared, cudaStream_t s);
// forward pass on the CUDA cores (k_mlp_infer): h[groups * 256] from x, prepared weights
cudaError_t mlp_infer(int groups, const float* prepared, const float* x, float* h, cudaStream_t s);
cudaError_t mlp_grad_sum(int groups, const float* partial, float* grad, cudaStream_t s);
cudaError_t mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int step, cudaStream_t s);
}  // namespace rbmd
