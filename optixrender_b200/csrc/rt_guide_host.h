// rt_guide_host.h - host launchers of the guiding network (rt_guide.cu).
#pragma once

#include <cuda_runtime.h>

#include "rt_guide.cuh"
#include "rt_kernels.cuh"

namespace rtgh {

size_t backward_smem();
cudaError_t prepare_kernels();
// Inference CTAs that gave up waiting on their tensor-core work since the
// last call (the counter is cleared); each is reported as a watchdog error.
int take_tc_timeouts();
// mode 0: raw outputs (n x 32 floats); mode 1: one Mixture per position.
void launch_forward(const rtg::NetView& net, const float* pos, int n, int mode, float* raw, rtg::Mixture* mix, int sms,
                    cudaStream_t st);
// `weight_sum` (device, may be null) replaces `scale` by 1 / *weight_sum.
// Bytes of training fragments per 16-sample tile (the scratch `frags` of
// launch_backward holds frag_tiles tiles).
size_t frag_bytes_per_tile();
void launch_backward(const rtg::NetView& net, const float* pos, const float* dir, const float* weight, int n,
                     float scale, const float* weight_sum, float* grad_table, float* grad_mlp, float* loss,
                     uint32_t* frags, int frag_tiles, int sms, cudaStream_t st);
// Renderer side: mixtures of a bounce's guided vertices, training samples of
// a wave, training batches (strided subsets from a random start).
void launch_infer(const rtd::Ctx& c, const rtg::NetView& net, int sms, cudaStream_t st);
void launch_collect(const rtd::Ctx& c, float4* buf, int* count, int cap, cudaStream_t st);
void launch_batch(const float4* buf, const int* count, int cap, int n, uint32_t seed, float* pos, float* dir,
                  float* w, float* weight_sum, cudaStream_t st);
void launch_adam(float* p, __half* p16, float* grad, float* m, float* v, int64_t n, float lr, int step,
                 cudaStream_t st);
// Adam on the hash table's first level_entries[l] entries of every level l.
void launch_adam_table(float* p, __half* p16, float* grad, float* m, float* v, const int64_t* level_entries, float lr,
                       int step, cudaStream_t st);
void launch_to_half(const float* p, __half* p16, int64_t n, cudaStream_t st);
void launch_pdf_sample(const rtg::Mixture* mix, const float* dir, const float* u, int n, float* out_dir, float* pdf,
                       cudaStream_t st);

// Level resolutions floor(n_min * b^l + 1e-6), b = exp((ln n_max - ln n_min) / 15), n_min = min(16, n_max).
void level_resolutions(int n_max, int* res);

}  // namespace rtgh

namespace rti {
rt_status guide_create(const rt_guide_options* o, rt_guide** out);
rtg::NetView guide_view(const rt_guide* g, float3 lo, float3 inv_ext);
// Gradient of n device samples (scale multiplies every weight; a non-null
// weight_sum replaces it by 1 / *weight_sum) followed by one Adam step.
rt_status guide_train_device(rt_guide* g, const float* pos, const float* dir, const float* weight, int n, float scale,
                             const float* weight_sum, cudaStream_t st);
int guide_sms(const rt_guide* g);
// Device memory of the network, its optimiser state and its training scratch.
int64_t guide_device_bytes(const rt_guide* g);
}  // namespace rti
