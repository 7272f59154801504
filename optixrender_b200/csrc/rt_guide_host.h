// rt_guide_host.h - host launchers of the guiding network (rt_guide.cu).
#pragma once

#include <cuda_runtime.h>

#include "rt_guide.cuh"

namespace rtgh {

size_t forward_smem();
size_t backward_smem();
cudaError_t set_resolutions(const int* res);
cudaError_t prepare_kernels();
// mode 0: raw outputs (n x 32 floats); mode 1: one Mixture per position.
void launch_forward(const rtg::NetView& net, const float* pos, int n, int mode, float* raw, rtg::Mixture* mix, int sms,
                    cudaStream_t st);
void launch_backward(const rtg::NetView& net, const float* pos, const float* dir, const float* weight, int n,
                     float scale, float* grad_table, float* grad_mlp, float* loss, int sms, cudaStream_t st);
void launch_adam(float* p, __half* p16, float* grad, float* m, float* v, int64_t n, float lr, int step,
                 cudaStream_t st);
void launch_to_half(const float* p, __half* p16, int64_t n, cudaStream_t st);
void launch_pdf_sample(const rtg::Mixture* mix, const float* dir, const float* u, int n, float* out_dir, float* pdf,
                       cudaStream_t st);

// Level resolutions floor(16 * b^l), b = exp((ln 2048 - ln 16) / 15).
void level_resolutions(int* res);

}  // namespace rtgh
