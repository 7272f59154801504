// rt_bvh.h - host build of the compressed 8-wide BVH.
#pragma once

#include <string>
#include <vector>

#include "rt_device.cuh"

namespace rth {

struct BuiltBvh {
    std::vector<rtd::CwNode> nodes;  // node 0 is the root
    std::vector<int> order;          // triangle slot -> original triangle index
    int depth;                       // number of wide levels
};

// tv: ntri * 9 floats (three vertices per triangle).  Host build, validated.
bool build_cwbvh(const float* tv, int64_t ntri, BuiltBvh& out, std::string& err);
// The same rules built on the current device (rt_bvh_gpu.cu); tv is host memory.
bool build_cwbvh_gpu(const float* tv, int64_t ntri, BuiltBvh& out, std::string& err, cudaStream_t st);
// Checks a wide BVH against its triangles: every index a traversal can form is
// in range, the triangle order is a permutation and every quantised child box
// contains what it stands for.
bool validate_cwbvh(const BuiltBvh& bvh, const float* tv, int64_t ntri, std::string& err);

// Host tables shared with the device (rt_tables.cpp).
void kulla_conty_tables(float* bsdf_avg, float* albedo_avg);
void env_sampling_cache(const float* rgba, int width, int height, float* cache);

}  // namespace rth
