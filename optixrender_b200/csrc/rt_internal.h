// rt_internal.h - host-side objects behind the opaque handles of rt_capi.h.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <string>
#include <vector>

#include "../../include/rt_capi.h"
#include "rt_kernels.cuh"

// Scene: the reference's Scene (core/include/Scene.h:195-214) with meshes
// de-indexed as TriangleMesh::LoadMesh does (core/src/Scene.cpp:167-174).
struct rt_scene {
    std::vector<float> tv;   // 9 floats per triangle
    std::vector<float> tn;   // 9 floats per triangle
    std::vector<float> tuv;  // 6 floats per triangle
    std::vector<int> tri_mesh;
    std::vector<rt_material> mesh_mat;
    std::vector<int> mesh_out, mesh_in;
    std::vector<rt_light> lights;
    std::vector<rt_medium> media;
    std::vector<std::vector<float>> media_density;
    std::vector<float> env;
    int env_w = 0, env_h = 0;
    std::vector<uint32_t> tex;       // RGBA8 texels of every texture, row 0 at v = 0
    std::vector<int32_t> tex_info;   // offset, width, height per texture
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
};

namespace rti {

extern thread_local std::string g_error;
rt_status fail(rt_status code, const std::string& msg);
rt_status cuda_fail(cudaError_t e, const char* what);
// RT_ERR_UNSUPPORTED when a wide BVH is deeper than the traversal stack.
rt_status check_bvh_depth(int depth);

// Makes `dev` the calling thread's current device for the guard's scope and
// restores the previous device afterwards.  Renderers and servers remember
// the device they were created on; every entry point that touches device
// memory or launches work takes this guard, so a call from a thread whose
// current device is another GPU still works on the object's own device.
struct DeviceGuard {
    int prev = -1;
    cudaError_t status = cudaSuccess;
    explicit DeviceGuard(int dev) {
        int cur = -1;
        status = cudaGetDevice(&cur);
        if (status == cudaSuccess && cur != dev) {
            status = cudaSetDevice(dev);
            if (status == cudaSuccess) prev = cur;
        }
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t alloc(size_t n);
    cudaError_t upload(const void* src, size_t n, cudaStream_t st);
    void release();
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
};

const float* kc_tables(const float** avg);
rtd::DevMaterial to_dev(const rt_material& m);
rtd::DevLight to_dev(const rt_light& l);
rtd::DevMedium to_dev(const rt_medium& m);
rtd::CameraView camera_view(const rt_camera& c, int w, int h);

// Everything of a scene that lives on the device.
struct DeviceScene {
    DevBuf nodes, tri_v, tri_a, meshes, materials, lights, media, env, env_cache, lut, lut_avg, tex, tex_info;
    std::vector<DevBuf*> grids;
    rtd::SceneView view{};
    int bvh_depth = 0;
    size_t bytes = 0;
    ~DeviceScene();
};
// Builds the wide BVH (on the device unless host_build) and uploads everything.
rt_status upload_scene(const rt_scene& s, DeviceScene& ds, cudaStream_t st, bool host_build = false);
void grid_majorants(const float* dens, const int res[3], int mres, std::vector<float>& out);

}  // namespace rti
