// rt_capi.cpp - implementation of include/rt_capi.h.
//
// Scene (core/include/Scene.h:195-214) and Renderer (core/include/Renderer.h)
// of the reference, as opaque handles.  The renderer owns every device
// allocation it makes and frees them in rt_renderer_destroy; nothing throws
// across the ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "rt_bvh.h"
#include "rt_internal.h"
#include "rt_kernels.cuh"

using namespace rtd;

namespace rti {

thread_local std::string g_error;

rt_status fail(rt_status code, const std::string& msg) {
    g_error = msg;
    return code;
}

rt_status check_bvh_depth(int depth) {
    static_assert(RT_MAX_BVH_DEPTH == rtd::kStackSize, "the traversal stack bounds the BVH depth");
    if (depth <= RT_MAX_BVH_DEPTH) return RT_OK;
    return fail(RT_ERR_UNSUPPORTED, "BVH too deep for the traversal stack (" + std::to_string(depth) + " levels, at most " +
                                        std::to_string(RT_MAX_BVH_DEPTH) + ")");
}

rt_status cuda_fail(cudaError_t e, const char* what) {
    g_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? RT_ERR_OUT_OF_MEMORY : RT_ERR_CUDA;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

cudaError_t DevBuf::alloc(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

cudaError_t DevBuf::upload(const void* src, size_t n, cudaStream_t st) {
    cudaError_t e = alloc(n);
    if (e != cudaSuccess || n == 0) return e;
    e = cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

const float* kc_tables(const float** avg) {
    static float lut[64 * 64];
    static float lavg[64];
    static std::once_flag once;
    std::call_once(once, [] { rth::kulla_conty_tables(lut, lavg); });
    if (avg) *avg = lavg;
    return lut;
}

DevMaterial to_dev(const rt_material& m) {
    DevMaterial d;
    std::memset(&d, 0, sizeof(d));
    d.type = m.type;
    for (int a = 0; a < 3; a++) {
        d.albedo[a] = m.albedo[a];
        d.eta[a] = m.eta[a];
        d.k[a] = m.k[a];
        d.specular[a] = m.specular[a];
    }
    d.roughness = m.roughness;
    d.anisotropy = m.anisotropy;
    d.int_ior = m.int_ior;
    d.ext_ior = m.ext_ior;
    d.metallic = m.metallic;
    d.coat_weight = m.coat_weight;
    d.nonlinear = m.nonlinear;
    d.coat_roughness_u = m.coat_roughness_u;
    d.coat_roughness_v = m.coat_roughness_v;
    for (int t = 0; t < 8; t++) {
        d.tex[t] = m.texture_ids[t];
        if (d.tex[t] >= 0) d.textured = 1;
    }
    return d;
}

DevLight to_dev(const rt_light& l) {
    DevLight d;
    std::memset(&d, 0, sizeof(d));
    d.type = l.type;
    d.double_side = l.double_side;
    d.radius = l.radius;
    d.medium = l.medium;
    for (int a = 0; a < 3; a++) {
        d.radiance[a] = l.radiance[a];
        d.position[a] = l.position[a];
        d.u[a] = l.u[a];
        d.v[a] = l.v[a];
    }
    return d;
}

DevMedium to_dev(const rt_medium& m) {
    DevMedium d;
    std::memset(&d, 0, sizeof(d));
    d.type = m.type;
    d.phase = m.phase;
    d.scale = m.scale;
    d.majorant_res = m.majorant_res > 0 ? m.majorant_res : 8;
    for (int a = 0; a < 3; a++) {
        d.g[a] = m.g[a];
        d.sigma_s[a] = m.sigma_s[a];
        d.sigma_a[a] = m.sigma_a[a];
        d.bmin[a] = m.bounds_min[a];
        d.bmax[a] = m.bounds_max[a];
        d.res[a] = m.grid_res[a];
    }
    return d;
}

// Renderer::SetCamera, core/src/Renderer.cpp:796-813
CameraView camera_view(const rt_camera& c, int w, int h) {
    CameraView v;
    v3 from = ld3(c.from), at = ld3(c.at), up = ld3(c.up);
    v3 dir = normalize(at - from);
    float cos_fovy = 0.66f;
    if (c.fov_y_deg > 0.0f) cos_fovy = 2.0f * std::tan(0.5f * c.fov_y_deg * 3.14159265358979323846f / 180.0f);
    float aspect = float(w) / float(h > 0 ? h : 1);
    v3 hor = cos_fovy * aspect * normalize(cross(dir, up));
    v3 ver = cos_fovy * normalize(cross(hor, dir));
    const v3* src[4] = {&from, &dir, &hor, &ver};
    float* dst[4] = {v.pos, v.dir, v.hor, v.ver};
    for (int i = 0; i < 4; i++) {
        dst[i][0] = src[i]->x;
        dst[i][1] = src[i]->y;
        dst[i][2] = src[i]->z;
    }
    v.medium = c.medium;
    return v;
}

}  // namespace rti

using namespace rti;

// ====================================================================== defaults
extern "C" {

const char* rt_last_error_message(void) { return g_error.c_str(); }
int32_t rt_version(void) { return 10000; }

void rt_material_default(rt_material* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->type = RT_MAT_METAL_WORKFLOW;
    for (int a = 0; a < 3; a++) {
        m->albedo[a] = 1.0f;
        m->specular[a] = 1.0f;
    }
    m->roughness = 0.1f;
    m->anisotropy = 0.0f;
    const float eta[3] = {0.14282f, 0.37414f, 1.43944f}, k[3] = {3.97472f, 2.38066f, 1.59981f};
    for (int a = 0; a < 3; a++) {
        m->eta[a] = eta[a];
        m->k[a] = k[a];
    }
    m->int_ior = 1.5f;
    m->ext_ior = 1.0f;
    m->nonlinear = 1;
    m->metallic = 0.8f;
    m->coat_weight = 2.0f;
    m->coat_roughness_u = 0.1f;
    m->coat_roughness_v = 0.1f;
    for (int t = 0; t < 8; t++) m->texture_ids[t] = -1;
}

void rt_light_default(rt_light* l) {
    if (!l) return;
    std::memset(l, 0, sizeof(*l));
    l->type = RT_LIGHT_SPHERE;
    l->double_side = 0;
    for (int a = 0; a < 3; a++) l->radiance[a] = 3.0f;
    l->position[0] = 6.0f;
    l->position[1] = 2.0f;
    l->position[2] = 0.0f;
    l->u[2] = 6.0f;
    l->v[0] = 6.0f;
    l->radius = 3.0f;
    l->medium = -1;
}

void rt_medium_default(rt_medium* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->type = RT_MEDIUM_HOMOGENEOUS;
    m->phase = RT_PHASE_ISOTROPIC;
    const float ss[3] = {0.74f, 0.88f, 1.01f}, sa[3] = {0.032f, 0.17f, 0.48f};
    for (int a = 0; a < 3; a++) {
        m->sigma_s[a] = ss[a];
        m->sigma_a[a] = sa[a];
    }
    m->scale = 500.0f;
    m->majorant_res = 8;
}

void rt_camera_default(rt_camera* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->from[2] = -1.0f;
    c->up[1] = 1.0f;
    c->medium = -1;
    c->fov_y_deg = 0.0f;
}

void rt_options_default(rt_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->width = 0;
    o->height = 0;
    o->spp = 1;            // LaunchParams.h:29
    o->max_depth = 25;     // LaunchParams.h:30
    o->filter = RT_FILTER_GAUSSIAN;  // LaunchParams.h:66
    o->rng = RT_RNG_LCG;
    o->rr_depth = 0;
    o->progressive = 0;    // Renderer.h:140
    o->seed = 1;
    o->tonemap = RT_TONEMAP_REINHARD;
    o->wave_paths = 0;
    o->collect_stats = 0;
    o->exposure = 1.0f;
    o->guided = 0;
    o->guide_train_spp = 32;
    o->guide_prob = 0.5f;
    o->guide_steps = 4;
    o->bvh_build = RT_BVH_GPU;
}

// ====================================================================== scene
rt_status rt_scene_create(rt_scene** out) {
    if (!out) return fail(RT_ERR_INVALID_ARG, "rt_scene_create: out is NULL");
    rt_scene* s = new (std::nothrow) rt_scene();
    if (!s) return fail(RT_ERR_OUT_OF_MEMORY, "rt_scene_create: out of host memory");
    *out = s;
    return RT_OK;
}

rt_status rt_scene_destroy(rt_scene* s) {
    delete s;
    return RT_OK;
}

rt_status rt_scene_add_mesh(rt_scene* s, const rt_mesh_desc* m, const rt_material* mat, int32_t out_medium,
                            int32_t in_medium, int32_t* out_mesh_id) {
    if (!s || !m || !mat) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh: NULL argument");
    if (m->num_triangles < 0 || !m->positions) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh: no positions");
    if (mat->type < RT_MAT_DIFFUSE || mat->type > RT_MAT_DIFFUSE_TRANSMITTER)
        return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh: unknown material type");
    const int64_t nt = m->num_triangles;
    if (m->indices) {
        for (int64_t i = 0; i < nt * 3; i++)
            if (m->indices[i] < 0 || m->indices[i] >= m->num_vertices)
                return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh: index out of range");
    } else if (m->num_vertices < nt * 3) {
        return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh: de-indexed mesh needs 3 vertices per triangle");
    }
    try {
        int mesh = int(s->mesh_mat.size());
        size_t base = s->tv.size() / 9;
        s->tv.resize(s->tv.size() + size_t(nt) * 9);
        s->tn.resize(s->tn.size() + size_t(nt) * 9);
        s->tuv.resize(s->tuv.size() + size_t(nt) * 6);
        s->tri_mesh.resize(s->tri_mesh.size() + size_t(nt), mesh);
        for (int64_t t = 0; t < nt; t++) {
            int64_t idx[3];
            for (int k = 0; k < 3; k++) idx[k] = m->indices ? m->indices[t * 3 + k] : t * 3 + k;
            float* pv = &s->tv[(base + size_t(t)) * 9];
            float* pn = &s->tn[(base + size_t(t)) * 9];
            float* pt = &s->tuv[(base + size_t(t)) * 6];
            for (int k = 0; k < 3; k++)
                for (int a = 0; a < 3; a++) pv[k * 3 + a] = m->positions[idx[k] * 3 + a];
            if (m->normals) {
                // normalize(vec3f(nx, ny, nz)), Scene.cpp:136
                for (int k = 0; k < 3; k++) {
                    v3 n = normalize(ld3(m->normals + idx[k] * 3));
                    pn[k * 3 + 0] = n.x;
                    pn[k * 3 + 1] = n.y;
                    pn[k * 3 + 2] = n.z;
                }
            } else {
                // face normal, Scene.cpp:150-158
                v3 v0 = ld3(pv), v1 = ld3(pv + 3), v2 = ld3(pv + 6);
                v3 n = normalize(cross(normalize(v1 - v0), normalize(v2 - v0)));
                for (int k = 0; k < 3; k++) {
                    pn[k * 3 + 0] = n.x;
                    pn[k * 3 + 1] = n.y;
                    pn[k * 3 + 2] = n.z;
                }
            }
            if (m->texcoords) {
                for (int k = 0; k < 3; k++) {
                    pt[k * 2 + 0] = m->texcoords[idx[k] * 2 + 0];
                    pt[k * 2 + 1] = m->texcoords[idx[k] * 2 + 1];
                }
            } else {
                const float def[6] = {0.f, 0.f, 1.f, 0.f, 0.f, 1.f};  // Scene.cpp:160-165
                for (int k = 0; k < 6; k++) pt[k] = def[k];
            }
            for (int k = 0; k < 3; k++) {
                for (int a = 0; a < 3; a++) {
                    s->lo[a] = std::min(s->lo[a], pv[k * 3 + a]);
                    s->hi[a] = std::max(s->hi[a], pv[k * 3 + a]);
                }
            }
        }
        s->mesh_mat.push_back(*mat);
        s->mesh_out.push_back(out_medium);
        s->mesh_in.push_back(in_medium);
        if (out_mesh_id) *out_mesh_id = mesh;
    } catch (const std::bad_alloc&) {
        return fail(RT_ERR_OUT_OF_MEMORY, "rt_scene_add_mesh: out of host memory");
    }
    return RT_OK;
}

rt_status rt_scene_add_light(rt_scene* s, const rt_light* l) {
    if (!s || !l) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_light: NULL argument");
    if (l->type < RT_LIGHT_QUAD || l->type > RT_LIGHT_POINT) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_light: unknown type");
    s->lights.push_back(*l);
    return RT_OK;
}

rt_status rt_scene_add_medium(rt_scene* s, const rt_medium* m) {
    if (!s || !m) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_medium: NULL argument");
    if (m->type != RT_MEDIUM_HOMOGENEOUS && m->type != RT_MEDIUM_GRID)
        return fail(RT_ERR_INVALID_ARG, "rt_scene_add_medium: unknown type");
    rt_medium c = *m;
    std::vector<float> dens;
    if (m->type == RT_MEDIUM_GRID) {
        int64_t n = int64_t(m->grid_res[0]) * m->grid_res[1] * m->grid_res[2];
        if (n <= 0 || !m->density) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_medium: grid medium needs a density grid");
        dens.assign(m->density, m->density + n);
    }
    c.density = nullptr;
    s->media.push_back(c);
    s->media_density.push_back(std::move(dens));
    return RT_OK;
}

rt_status rt_scene_set_env(rt_scene* s, const float* rgba, int32_t w, int32_t h, float scale) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_set_env: NULL scene");
    if (!rgba || w <= 0 || h <= 0) {
        s->env.clear();
        s->env_w = s->env_h = 0;
        return RT_OK;
    }
    s->env.assign(rgba, rgba + size_t(w) * h * 4);
    if (scale != 1.0f)
        for (float& v : s->env) v *= scale;
    s->env_w = w;
    s->env_h = h;
    return RT_OK;
}

rt_status rt_scene_get_bounds(const rt_scene* s, float lo[3], float hi[3]) {
    if (!s || !lo || !hi) return fail(RT_ERR_INVALID_ARG, "rt_scene_get_bounds: NULL argument");
    for (int a = 0; a < 3; a++) {
        lo[a] = s->lo[a];
        hi[a] = s->hi[a];
    }
    return RT_OK;
}

rt_status rt_scene_counts(const rt_scene* s, int64_t* tris, int32_t* meshes, int32_t* lights, int32_t* media) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_counts: NULL scene");
    if (tris) *tris = int64_t(s->tri_mesh.size());
    if (meshes) *meshes = int32_t(s->mesh_mat.size());
    if (lights) *lights = int32_t(s->lights.size());
    if (media) *media = int32_t(s->media.size());
    return RT_OK;
}

rt_status rt_scene_build_bvh(const rt_scene* s, int64_t* num_nodes, int32_t* depth) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_build_bvh: NULL scene");
    rth::BuiltBvh bvh;
    std::string err;
    if (!rth::build_cwbvh(s->tv.data(), int64_t(s->tri_mesh.size()), bvh, err))
        return fail(RT_ERR_UNSUPPORTED, "BVH build failed: " + err);
    if (num_nodes) *num_nodes = int64_t(bvh.nodes.size());
    if (depth) *depth = bvh.depth;
    return check_bvh_depth(bvh.depth);
}

rt_status rt_scene_build_bvh_gpu(const rt_scene* s, int64_t* num_nodes, int32_t* depth) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_build_bvh_gpu: NULL scene");
    rth::BuiltBvh bvh;
    std::string err;
    const int64_t nt = int64_t(s->tri_mesh.size());
    if (!rth::build_cwbvh_gpu(s->tv.data(), nt, bvh, err, nullptr)) return fail(RT_ERR_CUDA, err);
    if (!rth::validate_cwbvh(bvh, s->tv.data(), nt, err)) return fail(RT_ERR_UNSUPPORTED, "GPU BVH invalid: " + err);
    if (num_nodes) *num_nodes = int64_t(bvh.nodes.size());
    if (depth) *depth = bvh.depth;
    return check_bvh_depth(bvh.depth);
}

// ====================================================================== tables
rt_status rt_kulla_conty_lut(float* bsdf, float* avg) {
    if (!bsdf || !avg) return fail(RT_ERR_INVALID_ARG, "rt_kulla_conty_lut: NULL argument");
    const float* a = nullptr;
    const float* l = kc_tables(&a);
    std::memcpy(bsdf, l, sizeof(float) * 64 * 64);
    std::memcpy(avg, a, sizeof(float) * 64);
    return RT_OK;
}

rt_status rt_env_sampling_cache(const float* rgba, int32_t w, int32_t h, float* cache) {
    if (!rgba || !cache || w <= 0 || h <= 0) return fail(RT_ERR_INVALID_ARG, "rt_env_sampling_cache: bad argument");
    rth::env_sampling_cache(rgba, w, h, cache);
    return RT_OK;
}

}  // extern "C"
