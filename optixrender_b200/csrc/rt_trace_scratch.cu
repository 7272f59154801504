// rt_trace_scratch.cu - ray queries staged in a fixed device array.
//
// rt_renderer_trace_noalloc answers the same queries as rt_renderer_trace
// with host buffers, but allocates nothing: the rays and hits pass through
// g_trace_scratch, one file-scope device array per device of
// kTraceScratchRays rays (32 bytes in + 16 bytes out each: 3 MiB).
#include <cuda_runtime.h>

#include <cfloat>

#include "rt_kernels.cuh"
#include "rt_traverse.cuh"

namespace rtd {

constexpr int64_t kTraceScratchRays = 65536;

// Rays (2 float4 each) in the first 2 * kTraceScratchRays entries, hits
// (1 float4 each) in the last kTraceScratchRays.  Nothing in it needs to start
// at zero: a call copies in the n rays the kernel reads and copies out only
// the n hits the kernel wrote.
static __device__ __align__(256) float4 g_trace_scratch[3 * kTraceScratchRays];

// k_trace (rt_kernels.cu) reading its rays from, and writing its hits to,
// the scratch array passed in by the host.
template <bool AnyHit>
__global__ void __launch_bounds__(128) k_trace_scratch(SceneView sc, float4* scratch, int n, int* overflow) {
    const int i = int(blockIdx.x) * int(blockDim.x) + int(threadIdx.x);
    if (i >= n) return;
    const float4* rays = scratch;
    float4* hits = scratch + 2 * kTraceScratchRays;
    float4 a = rays[2 * i], b = rays[2 * i + 1];
    TravRay r;
    r.o = xyz(a);
    r.d = xyz(b);
    r.tmin = a.w;
    r.tmax = b.w;
    prepare_ray(r);
    float t = FLT_MAX, b1 = 0.f, b2 = 0.f;
    uint32_t nv = 0, nt = 0, ovf = 0;
    int tri = traverse<AnyHit, false>(sc, r, t, b1, b2, nv, nt, ovf);
    if (ovf) atomicAdd(overflow, int(ovf));
    float4 out;
    if (tri < 0) {
        out = make_float4(FLT_MAX, 0.f, 0.f, __int_as_float(-1));
    } else if (AnyHit) {
        out = make_float4(t, b1, b2, __int_as_float(1));
    } else {
        int orig = __float_as_int(__ldg(sc.tri_v + size_t(tri) * 3).w);
        out = make_float4(t, b1, b2, __int_as_float(orig));
    }
    hits[i] = out;
}

}  // namespace rtd

namespace rth {

int64_t trace_scratch_rays() { return rtd::kTraceScratchRays; }

// Device address of the scratch array on `device`, which must be the calling
// thread's current device (the entry point makes the renderer's device
// current).  Looked up on every call: cudaGetSymbolAddress allocates nothing
// and is cheap, and a cached address would go stale after a device reset.
cudaError_t trace_scratch_address(int device, void** ptr) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev != device) return cudaErrorInvalidDevice;
    return cudaGetSymbolAddress(ptr, rtd::g_trace_scratch);
}

void launch_trace_scratch(const rtd::SceneView& sc, bool any_hit, void* scratch, int n, int* overflow, cudaStream_t st) {
    if (n <= 0) return;
    const int block = 128, grid = (n + block - 1) / block;
    float4* s = static_cast<float4*>(scratch);
    if (any_hit)
        rtd::k_trace_scratch<true><<<grid, block, 0, st>>>(sc, s, n, overflow);
    else
        rtd::k_trace_scratch<false><<<grid, block, 0, st>>>(sc, s, n, overflow);
}

}  // namespace rth
