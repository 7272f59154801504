// rt_renderer.cpp - the Renderer handle: scene upload, per-pixel and per-wave
// buffers, and the host loop that issues the wavefront kernels for one
// Renderer::Render() (core/src/Renderer.cpp:635-793).
#include <cuda_runtime.h>

#include <cstddef>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "rt_bvh.h"
#include "rt_guide_host.h"
#include "rt_image.h"
#include "rt_internal.h"

using namespace rtd;
using namespace rti;

namespace rti {

DeviceScene::~DeviceScene() {
    for (DevBuf* g : grids) delete g;
}

#define RT_CUDA(call, what)                        \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// The renderer's device current for the rest of the calling scope.
#define RT_ON_DEVICE(rr, what)                                         \
    DeviceGuard dg_((rr)->device);                                     \
    if (dg_.status != cudaSuccess) return cuda_fail(dg_.status, what)

// Per majorant cell, the largest density any trilinear lookup inside the cell
// can return: the maximum over the voxels within one voxel of the cell.
void grid_majorants(const float* dens, const int res[3], int mres, std::vector<float>& out) {
    out.assign(size_t(mres) * mres * mres, 0.0f);
    for (int cz = 0; cz < mres; cz++)
        for (int cy = 0; cy < mres; cy++)
            for (int cx = 0; cx < mres; cx++) {
                int c[3] = {cx, cy, cz}, lo[3], hi[3];
                for (int a = 0; a < 3; a++) {
                    lo[a] = std::max(0, int(std::floor(double(c[a]) * res[a] / mres)) - 1);
                    hi[a] = std::min(res[a] - 1, int(std::ceil(double(c[a] + 1) * res[a] / mres)) + 1);
                }
                float m = 0.0f;
                for (int z = lo[2]; z <= hi[2]; z++)
                    for (int y = lo[1]; y <= hi[1]; y++)
                        for (int x = lo[0]; x <= hi[0]; x++)
                            m = std::max(m, dens[(size_t(z) * res[1] + y) * res[0] + x]);
                out[(size_t(cz) * mres + cy) * mres + cx] = m;
            }
}

rt_status upload_scene(const rt_scene& s, DeviceScene& ds, cudaStream_t st, bool host_build) {
    const int64_t nt = int64_t(s.tri_mesh.size());
    rth::BuiltBvh bvh;
    std::string err;
    if (host_build) {
        if (!rth::build_cwbvh(s.tv.data(), nt, bvh, err)) return fail(RT_ERR_UNSUPPORTED, "BVH build failed: " + err);
    } else if (!rth::build_cwbvh_gpu(s.tv.data(), nt, bvh, err, st)) {
        return fail(RT_ERR_CUDA, err);
    } else if (!rth::validate_cwbvh(bvh, s.tv.data(), nt, err)) {
        // The device build is checked like the host build checks its own
        // tree (every index in range, every quantised box containing what it
        // bounds).  Inputs it gets wrong - coordinates spanning the whole
        // float range - are built again on the host.
        if (!rth::build_cwbvh(s.tv.data(), nt, bvh, err)) return fail(RT_ERR_UNSUPPORTED, "BVH build failed: " + err);
    }
    if (rt_status dst = check_bvh_depth(bvh.depth)) return dst;
    ds.bvh_depth = bvh.depth;
    std::vector<float4> tv(size_t(nt) * 3), ta(size_t(nt) * 4);
    for (int64_t t = 0; t < nt; t++) {
        int o = bvh.order[size_t(t)];
        const float* p = &s.tv[size_t(o) * 9];
        const float* n = &s.tn[size_t(o) * 9];
        const float* uv = &s.tuv[size_t(o) * 6];
        float4 id;
        std::memcpy(&id.x, &o, 4);
        tv[size_t(t) * 3 + 0] = make_float4(p[0], p[1], p[2], id.x);
        // v1.w: the shade bucket (material type) of the triangle's mesh
        int mt = s.mesh_mat[size_t(s.tri_mesh[size_t(o)])].type;
        int key = (mt >= 0 && mt < kMissBucket) ? mt : 0;
        float kf;
        std::memcpy(&kf, &key, 4);
        tv[size_t(t) * 3 + 1] = make_float4(p[3], p[4], p[5], kf);
        tv[size_t(t) * 3 + 2] = make_float4(p[6], p[7], p[8], 0.0f);
        int mesh = s.tri_mesh[size_t(o)];
        float mf;
        std::memcpy(&mf, &mesh, 4);
        ta[size_t(t) * 4 + 0] = make_float4(n[0], n[1], n[2], uv[0]);
        ta[size_t(t) * 4 + 1] = make_float4(n[3], n[4], n[5], uv[1]);
        ta[size_t(t) * 4 + 2] = make_float4(n[6], n[7], n[8], uv[2]);
        ta[size_t(t) * 4 + 3] = make_float4(uv[3], uv[4], uv[5], mf);
    }
    const int ntex = int(s.tex_info.size() / 3);
    for (size_t i = 0; i < s.mesh_mat.size(); i++)
        for (int t = 0; t < 8; t++)
            if (s.mesh_mat[i].texture_ids[t] >= ntex)
                return fail(RT_ERR_INVALID_ARG, "mesh " + std::to_string(i) + " refers to texture " +
                                                    std::to_string(s.mesh_mat[i].texture_ids[t]) + " of " +
                                                    std::to_string(ntex));
    std::vector<MeshInfo> meshes(s.mesh_mat.size());
    std::vector<DevMaterial> mats(s.mesh_mat.size());
    for (size_t i = 0; i < meshes.size(); i++) {
        meshes[i].material = int(i);
        meshes[i].in_medium = s.mesh_in[i];
        meshes[i].out_medium = s.mesh_out[i];
        meshes[i].pad = 0;
        mats[i] = to_dev(s.mesh_mat[i]);
    }
    std::vector<DevLight> lights;
    for (auto& l : s.lights) lights.push_back(to_dev(l));
    std::vector<DevMedium> media;
    for (size_t i = 0; i < s.media.size(); i++) media.push_back(to_dev(s.media[i]));
    RT_CUDA(ds.nodes.upload(bvh.nodes.data(), bvh.nodes.size() * sizeof(CwNode), st), "upload BVH nodes");
    RT_CUDA(ds.tri_v.upload(tv.data(), tv.size() * sizeof(float4), st), "upload triangles");
    RT_CUDA(ds.tri_a.upload(ta.data(), ta.size() * sizeof(float4), st), "upload triangle attributes");
    RT_CUDA(ds.meshes.upload(meshes.data(), meshes.size() * sizeof(MeshInfo), st), "upload meshes");
    RT_CUDA(ds.materials.upload(mats.data(), mats.size() * sizeof(DevMaterial), st), "upload materials");
    RT_CUDA(ds.lights.upload(lights.data(), lights.size() * sizeof(DevLight), st), "upload lights");
    if (ntex > 0) {
        std::vector<int4> info(static_cast<size_t>(ntex));
        for (int t = 0; t < ntex; t++)
            info[size_t(t)] = make_int4(s.tex_info[3 * size_t(t)], s.tex_info[3 * size_t(t) + 1],
                                        s.tex_info[3 * size_t(t) + 2], 0);
        RT_CUDA(ds.tex.upload(s.tex.data(), s.tex.size() * sizeof(uint32_t), st), "upload textures");
        RT_CUDA(ds.tex_info.upload(info.data(), info.size() * sizeof(int4), st), "upload textures");
    }
    const float* avg = nullptr;
    const float* lut = kc_tables(&avg);
    RT_CUDA(ds.lut.upload(lut, 64 * 64 * sizeof(float), st), "upload LUT");
    RT_CUDA(ds.lut_avg.upload(avg, 64 * sizeof(float), st), "upload LUT");
    if (s.env_w > 0) {
        std::vector<float> cache(s.env.size());
        rth::env_sampling_cache(s.env.data(), s.env_w, s.env_h, cache.data());
        RT_CUDA(ds.env.upload(s.env.data(), s.env.size() * sizeof(float), st), "upload environment");
        RT_CUDA(ds.env_cache.upload(cache.data(), cache.size() * sizeof(float), st), "upload environment cache");
    }
    for (size_t i = 0; i < media.size(); i++) {
        if (s.media[i].type != RT_MEDIUM_GRID) continue;
        const std::vector<float>& d = s.media_density[i];
        DevBuf* g = new DevBuf();
        ds.grids.push_back(g);
        RT_CUDA(g->upload(d.data(), d.size() * sizeof(float), st), "upload density grid");
        media[i].density = g->as<float>();
        float mx = 0.0f;
        for (float v : d) mx = std::max(mx, v);
        media[i].max_density = mx;
        std::vector<float> maj;
        grid_majorants(d.data(), s.media[i].grid_res, media[i].majorant_res, maj);
        DevBuf* mb = new DevBuf();
        ds.grids.push_back(mb);
        RT_CUDA(mb->upload(maj.data(), maj.size() * sizeof(float), st), "upload majorant grid");
        media[i].majorant = mb->as<float>();
    }
    RT_CUDA(ds.media.upload(media.data(), media.size() * sizeof(DevMedium), st), "upload media");
    SceneView& v = ds.view;
    v.nodes = ds.nodes.as<CwNode>();
    v.tri_v = ds.tri_v.as<float4>();
    v.tri_a = ds.tri_a.as<float4>();
    v.num_nodes = int(bvh.nodes.size());
    v.bvh_depth = bvh.depth;
    v.num_tris = int(nt);
    v.meshes = ds.meshes.as<MeshInfo>();
    v.materials = ds.materials.as<DevMaterial>();
    v.lights = ds.lights.as<DevLight>();
    v.num_lights = int(lights.size());
    v.media = ds.media.as<DevMedium>();
    v.num_media = int(media.size());
    v.env = ds.env.as<float4>();
    v.env_cache = ds.env_cache.as<float4>();
    v.env_w = s.env_w;
    v.env_h = s.env_h;
    v.lut = ds.lut.as<float>();
    v.lut_avg = ds.lut_avg.as<float>();
    v.tex = ds.tex.as<uint32_t>();
    v.tex_info = ds.tex_info.as<int4>();
    v.num_tex = ntex;
    ds.bytes = ds.nodes.bytes + ds.tri_v.bytes + ds.tri_a.bytes + ds.env.bytes + ds.env_cache.bytes + ds.tex.bytes;
    for (DevBuf* g : ds.grids) ds.bytes += g->bytes;
    return RT_OK;
}

}  // namespace rti

struct KernelTimer {
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<std::pair<int, size_t>> marks;  // (class, event index of the start)
    cudaEvent_t next() {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    void reset() {
        used = 0;
        marks.clear();
    }
    ~KernelTimer() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

struct rt_renderer {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    rth::WaveFork fork{};  // side stream and events: k_shadow beside the next k_extend
    bool have_fork = false;
    DeviceScene ds;
    rt_options opt{};
    rt_camera cam{};
    int frame = 0;
    int pw = 0, ph = 0;
    DevBuf acc_color, acc_albedo, acc_normal, lcg_state, color, albedo, normal, rgba8;
    int capacity = 0;
    DevBuf slots, aov_a, aov_n, rng, q0, q1, sq, sh_o, sh_d, ctl, segs, job;  // slots: kSlotRecord bytes per slot
    DevBuf sorted;            // shade queue by material type
    DevBuf dn_tmp0, dn_tmp1, dn_out;  // denoiser scratch and output (rt_options.denoise)
    int dn_pixels = 0;                // pixels covered by the denoiser buffers
    bool denoised = false;            // dn_out holds the last render's denoised colour
    DevBuf mat_tex;           // per-slot textured materials (scenes with textures)
    bool sort_shade = true;   // RT_SORT_SHADE=0 keeps the shade queue in extend order
    int wave_paths = 0;       // slots per wave of the last render
    int64_t h2d_bytes = 0;    // host-to-device bytes of the last render
    DevBuf wave_index;
    DevBuf q_job, q_wave, q_index, q_ctl;  // rt_renderer_trace_wavefront: its job, wave table and counters
    // one captured wave (raygen, (extend, shade, shadow) x depth, resolve, advance)
    cudaGraphExec_t graph = nullptr;
    int graph_capacity = -1, graph_depth = -1, graph_ring = -1;
    const void* graph_waves = nullptr;
    rth::LaunchShape shape{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    KernelTimer timer;
    bool rendered = false;
    int launches = 0;
    int waves = 0;
    int extend_launches = 0;
    int64_t paths = 0;
    // path guiding
    float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {1.f, 1.f, 1.f};  // scene bounds
    rt_guide* guide = nullptr;
    DevBuf g_mix, g_rec, g_buf, g_count, g_bpos, g_bdir, g_bw, g_wsum;
    int g_cap = 0;             // slots covered by g_mix
    int64_t guide_trained = 0; // samples per pixel rendered while training
    uint32_t guide_seed = 1;
    bool graph_guided = false;
    const void* graph_mix = nullptr;
    // Pinned staging of each Render()'s launch parameters and wave table, so
    // that their copies are true asynchronous DMA; a ring, so that the host
    // can queue a few frames ahead before it waits for a buffer's last copy.
    struct HostStage {
        void* ptr = nullptr;
        size_t bytes = 0;
        cudaEvent_t copied = nullptr;  // recorded after the copies that read ptr
    };
    static constexpr int kStages = 3;
    HostStage stage[kStages];
    int stage_next = 0;
};

namespace {

constexpr int kGuideBatch = 1 << 18;
constexpr int kGuidedWaveMax = 1 << 24;

rt_status ensure_pixels(rt_renderer* r, int w, int h) {
    if (r->pw == w && r->ph == h) return RT_OK;
    size_t n = size_t(w) * h;
    DevBuf* f4s[] = {&r->acc_color, &r->acc_albedo, &r->acc_normal, &r->color, &r->albedo, &r->normal};
    for (DevBuf* b : f4s) {
        b->release();
        RT_CUDA(b->alloc(n * sizeof(float4)), "allocate frame buffers");
        RT_CUDA(cudaMemsetAsync(b->ptr, 0, n * sizeof(float4), r->stream), "clear frame buffers");
    }
    r->lcg_state.release();
    r->rgba8.release();
    RT_CUDA(r->lcg_state.alloc(n * 4), "allocate frame buffers");
    RT_CUDA(r->rgba8.alloc(n * 4), "allocate frame buffers");
    RT_CUDA(cudaMemsetAsync(r->rgba8.ptr, 0, n * 4, r->stream), "clear frame buffers");
    r->pw = w;
    r->ph = h;
    r->denoised = false;
    return RT_OK;
}

rt_status ensure_denoiser(rt_renderer* r) {
    const int n = r->pw * r->ph;
    if (r->dn_pixels == n) return RT_OK;
    DevBuf* bufs[] = {&r->dn_tmp0, &r->dn_tmp1, &r->dn_out};
    for (DevBuf* b : bufs) {
        b->release();
        RT_CUDA(b->alloc(size_t(n) * sizeof(float4)), "allocate denoiser buffers");
    }
    r->dn_pixels = n;
    return RT_OK;
}

rt_status ensure_waves(rt_renderer* r, int cap) {
    if (cap <= r->capacity) return RT_OK;
    size_t n = size_t(cap);
    RT_CUDA(r->slots.alloc(n * kSlotRecord), "allocate path state");
    RT_CUDA(r->aov_a.alloc(n * sizeof(float4)), "allocate path state");
    RT_CUDA(r->aov_n.alloc(n * sizeof(float2)), "allocate path state");
    RT_CUDA(r->rng.alloc(n * sizeof(uint2)), "allocate path state");
    RT_CUDA(r->q0.alloc(n * sizeof(int)), "allocate queues");
    RT_CUDA(r->q1.alloc(n * sizeof(int)), "allocate queues");
    RT_CUDA(r->sq.alloc(n * sizeof(int)), "allocate queues");
    RT_CUDA(r->sh_o.alloc(2 * n * sizeof(float4)), "allocate shadow queue");
    RT_CUDA(r->sh_d.alloc(2 * n * sizeof(float4)), "allocate shadow queue");
    if (r->sort_shade) RT_CUDA(r->sorted.alloc(size_t(kShadeBuckets) * n * sizeof(int)), "allocate shade buckets");
    if (r->ds.view.num_tex > 0) RT_CUDA(r->mat_tex.alloc(n * sizeof(DevMaterial)), "allocate textured materials");
    r->capacity = cap;
    return RT_OK;
}

// The renderer's per-slot path state as the kernels see it.
void wave_bufs(rt_renderer* r, WaveBufs& b) {
    b.ray_o = slot_field(r->slots.ptr, kRecRayO);
    b.ray_d = slot_field(r->slots.ptr, kRecRayD);
    b.hit = slot_field(r->slots.ptr, kRecHit);
    b.thr = slot_field(r->slots.ptr, kRecThr);
    b.rad = slot_field(r->slots.ptr, kRecRad);
    b.nee0 = slot_field(r->slots.ptr, kRecNee0);
    b.nee1 = slot_field(r->slots.ptr, kRecNee1);
    b.stale = slot_field(r->slots.ptr, kRecStale);
    b.aov_a = r->aov_a.as<float4>();
    b.aov_n = r->aov_n.as<float2>();
    b.rng = r->rng.as<uint2>();
    b.queue[0] = r->q0.as<int>();
    b.queue[1] = r->q1.as<int>();
    b.squeue = r->sq.as<int>();
    b.sh_o = r->sh_o.as<float4>();
    b.sh_d = r->sh_d.as<float4>();
    b.sorted = r->sort_shade ? r->sorted.as<int>() : nullptr;
    b.mat_tex = r->ds.view.num_tex > 0 ? r->mat_tex.as<DevMaterial>() : nullptr;
    b.ctl = r->ctl.as<WaveCtl>();
    b.capacity = r->capacity;
}

int auto_capacity(const rt_options& o, int64_t npix, int64_t total, int64_t allocated) {
    // Large waves: the last bounces of a wave carry few paths and run at the
    // latency of a handful of rays, so fewer, larger waves spend less time
    // there.  Automatic: up to 2^26 slots (272 B each, 18 GB), at most a
    // quarter of the free device memory.  The free memory is asked for only
    // when the renderer's wave buffers (`allocated` slots) are too small for
    // the frame: the query goes to the driver and, on a busy host, took tens
    // of milliseconds, which a Render() that only launches work must not spend.
    int64_t cap = o.wave_paths > 0 ? int64_t(o.wave_paths) : std::max<int64_t>(npix, int64_t(1) << 26);
    auto clamp = [&](int64_t c) {
        c = std::min<int64_t>(c, int64_t(1) << 26);
        if (o.rng == RT_RNG_LCG) c = std::min<int64_t>(c, npix);
        return std::max<int64_t>(std::min<int64_t>(c, total), 1);
    };
    if (o.wave_paths <= 0 && clamp(cap) > allocated) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            cap = std::min<int64_t>(cap, std::max<int64_t>(std::max<int64_t>(int64_t(1) << 20, allocated),
                                                           int64_t(fr / 4) / 400));
    }
    return int(clamp(cap));
}

// Guiding network and its per-slot buffers: mixtures for `cap` slots, and
// for training waves of `train_slots` paths the records, the sample buffer
// and one batch.
rt_status ensure_guide(rt_renderer* r, int cap, int64_t train_slots) {
    if (!r->guide) {
        rt_guide_options go;
        rt_guide_options_default(&go);
        go.seed = r->opt.seed;
        rt_status st = guide_create(&go, &r->guide);
        if (st) return st;
    }
    if (r->g_cap < cap) {
        RT_CUDA(r->g_mix.alloc(size_t(cap) * sizeof(rtg::Mixture)), "allocate guide mixtures");
        r->g_cap = cap;
    }
    if (train_slots > 0) {
        const size_t rec = size_t(rtg::kGuideRec) * 4 * size_t(r->capacity) * sizeof(float4);
        if (r->g_rec.bytes < rec) RT_CUDA(r->g_rec.alloc(rec), "allocate guide records");
        const size_t buf = size_t(rtg::kGuideRec) * size_t(train_slots) * 32;
        if (r->g_buf.bytes < buf) RT_CUDA(r->g_buf.alloc(buf), "allocate guide samples");
        if (!r->g_count.ptr) RT_CUDA(r->g_count.alloc(sizeof(int)), "allocate guide samples");
        if (!r->g_wsum.ptr) RT_CUDA(r->g_wsum.alloc(sizeof(float)), "allocate guide batch");
        if (!r->g_bw.ptr) {
            RT_CUDA(r->g_bpos.alloc(size_t(kGuideBatch) * 12), "allocate guide batch");
            RT_CUDA(r->g_bdir.alloc(size_t(kGuideBatch) * 12), "allocate guide batch");
            RT_CUDA(r->g_bw.alloc(size_t(kGuideBatch) * 4), "allocate guide batch");
        }
    }
    return RT_OK;
}

// The traversal stack-overflow counter of the renderer's control block.
int* overflow_counter(rt_renderer* r) {
    return reinterpret_cast<int*>(static_cast<char*>(r->ctl.ptr) + offsetof(WaveCtl, overflow));
}

rt_status overflow_status(int n, const char* what) {
    if (n <= 0) return RT_OK;
    return fail(RT_ERR_DEVICE_WATCHDOG, std::string(what) + ": " + std::to_string(n) +
                                            " traversal node groups found the " + std::to_string(kStackSize) +
                                            "-entry stack full; their subtrees were not visited");
}

rt_status check_options(const rt_options* o) {
    if (o->spp < 1 || o->max_depth < 1) return fail(RT_ERR_INVALID_ARG, "spp and max_depth must be >= 1");
    if (o->width < 0 || o->height < 0) return fail(RT_ERR_INVALID_ARG, "negative frame size");
    if (int64_t(o->width) * o->height > (int64_t(1) << 28)) return fail(RT_ERR_INVALID_ARG, "frame too large");
    if (o->rng != RT_RNG_LCG && o->rng != RT_RNG_PCG32) return fail(RT_ERR_INVALID_ARG, "unknown rng");
    if (o->bvh_build != RT_BVH_GPU && o->bvh_build != RT_BVH_HOST) return fail(RT_ERR_INVALID_ARG, "unknown bvh_build");
    if (o->guided && o->rng != RT_RNG_PCG32)
        return fail(RT_ERR_INVALID_ARG, "guided rendering needs PCG32 streams (rng = RT_RNG_PCG32)");
    if (o->guided && (!(o->guide_prob > 0.0f) || o->guide_prob > 1.0f || o->guide_train_spp < 0 || o->guide_steps < 0))
        return fail(RT_ERR_INVALID_ARG, "guide_prob must be in (0, 1], guide_train_spp and guide_steps >= 0");
    if (o->filter < RT_FILTER_BOX || o->filter > RT_FILTER_GAUSSIAN) return fail(RT_ERR_INVALID_ARG, "unknown filter");
    return RT_OK;
}

}  // namespace

extern "C" {

rt_status rt_renderer_create(const rt_scene* s, const rt_options* opts, rt_renderer** out) {
    if (!s || !out) return fail(RT_ERR_INVALID_ARG, "rt_renderer_create: NULL argument");
    rt_options o;
    rt_options_default(&o);
    if (opts) o = *opts;
    rt_status st = check_options(&o);
    if (st) return st;
    rt_renderer* r = new (std::nothrow) rt_renderer();
    if (!r) return fail(RT_ERR_OUT_OF_MEMORY, "rt_renderer_create: out of host memory");
    cudaError_t e = cudaGetDevice(&r->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = rth::create_fork(r->fork);
    if (e != cudaSuccess) {
        if (r->stream) cudaStreamDestroy(r->stream);
        delete r;
        return cuda_fail(e, "rt_renderer_create");
    }
    r->have_fork = true;
    r->own_stream = true;
    r->opt = o;
    if (const char* v = std::getenv("RT_SORT_SHADE")) r->sort_shade = std::atoi(v) != 0;
    rt_camera_default(&r->cam);
    st = upload_scene(*s, r->ds, r->stream, o.bvh_build == RT_BVH_HOST);
    for (int a = 0; a < 3; a++) {
        r->lo[a] = s->lo[a];
        r->hi[a] = s->hi[a];
    }
    if (st == RT_OK) {
        e = cudaEventCreate(&r->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&r->ev1);
        if (e == cudaSuccess) e = cudaMalloc(&r->ctl.ptr, sizeof(WaveCtl));
        if (e == cudaSuccess) {
            r->ctl.bytes = sizeof(WaveCtl);
            e = cudaMemset(r->ctl.ptr, 0, sizeof(WaveCtl));
        }
        if (e == cudaSuccess) e = r->job.alloc(sizeof(JobDesc));
        if (e != cudaSuccess) st = cuda_fail(e, "rt_renderer_create");
    }
    if (st == RT_OK) rth::query_shape(r->shape);
    if (st == RT_OK && o.width > 0 && o.height > 0) st = ensure_pixels(r, o.width, o.height);
    if (st) {
        rt_renderer_destroy(r);
        return st;
    }
    *out = r;
    return RT_OK;
}

rt_status rt_renderer_destroy(rt_renderer* r) {
    if (!r) return RT_OK;
    RT_ON_DEVICE(r, "rt_renderer_destroy");
    if (r->stream) cudaStreamSynchronize(r->stream);
    if (r->graph) cudaGraphExecDestroy(r->graph);
    if (r->guide) rt_guide_destroy(r->guide);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->fork.side) cudaStreamSynchronize(r->fork.side);
    rth::destroy_fork(r->fork);
    for (auto& hs : r->stage) {
        if (hs.copied) cudaEventDestroy(hs.copied);
        if (hs.ptr) cudaFreeHost(hs.ptr);
    }
    if (r->own_stream && r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return RT_OK;
}

rt_status rt_renderer_set_options(rt_renderer* r, const rt_options* o) {
    if (!r || !o) return fail(RT_ERR_INVALID_ARG, "rt_renderer_set_options: NULL argument");
    RT_ON_DEVICE(r, "rt_renderer_set_options");
    rt_status st = check_options(o);
    if (st) return st;
    int w = r->opt.width, h = r->opt.height;
    r->opt = *o;
    if (o->width != w || o->height != h) return rt_renderer_resize(r, o->width, o->height);
    return RT_OK;
}

rt_status rt_renderer_get_options(const rt_renderer* r, rt_options* o) {
    if (!r || !o) return fail(RT_ERR_INVALID_ARG, "rt_renderer_get_options: NULL argument");
    *o = r->opt;
    return RT_OK;
}

rt_status rt_renderer_resize(rt_renderer* r, int32_t w, int32_t h) {
    if (!r || w < 0 || h < 0) return fail(RT_ERR_INVALID_ARG, "rt_renderer_resize: bad argument");
    RT_ON_DEVICE(r, "rt_renderer_resize");
    r->opt.width = w;
    r->opt.height = h;
    if (w > 0 && h > 0) {
        rt_status st = ensure_pixels(r, w, h);
        if (st) return st;
    }
    r->frame = 0;  // SetCamera(lastSetCamera), Renderer.cpp:874
    return RT_OK;
}

rt_status rt_renderer_set_camera(rt_renderer* r, const rt_camera* c) {
    if (!r || !c) return fail(RT_ERR_INVALID_ARG, "rt_renderer_set_camera: NULL argument");
    r->cam = *c;
    r->frame = 0;  // Renderer.cpp:799
    return RT_OK;
}

rt_status rt_renderer_set_stream(rt_renderer* r, void* s) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "rt_renderer_set_stream: NULL renderer");
    RT_ON_DEVICE(r, "rt_renderer_set_stream");
    cudaStreamSynchronize(r->stream);
    if (r->own_stream) cudaStreamDestroy(r->stream);
    if (s) {
        r->stream = static_cast<cudaStream_t>(s);
        r->own_stream = false;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "rt_renderer_set_stream");
        r->own_stream = true;
    }
    return RT_OK;
}

rt_status rt_renderer_render(rt_renderer* r) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "rt_renderer_render: NULL renderer");
    RT_ON_DEVICE(r, "rt_renderer_render");
    const rt_options& o = r->opt;
    if (o.width <= 0 || o.height <= 0) return RT_OK;  // Renderer.cpp:638-640
    rt_status st = ensure_pixels(r, o.width, o.height);
    if (st) return st;
    const int64_t npix = int64_t(o.width) * o.height;
    const int64_t total = npix * o.spp;
    const bool guided = o.guided != 0;
    int cap = auto_capacity(o, npix, total, r->capacity);
    if (guided) cap = std::min(cap, kGuidedWaveMax);
    // guided: the first training samples run one sample per pixel per wave
    const int64_t train_waves =
        guided && npix <= int64_t(kGuidedWaveMax)
            ? std::min<int64_t>(o.spp, std::max<int64_t>(0, int64_t(o.guide_train_spp) - r->guide_trained))
            : 0;
    const int wave_cap = train_waves > 0 ? std::max<int>(cap, int(npix)) : cap;
    r->wave_paths = cap;
    st = ensure_waves(r, wave_cap);
    if (st) return st;
    if (guided) {
        st = ensure_guide(r, wave_cap, train_waves > 0 ? npix : 0);
        if (st) return st;
    }
    if (!o.progressive) r->frame = 0;  // Renderer.cpp:642-644
    JobDesc hj;
    std::memset(&hj, 0, sizeof(hj));
    hj.sc = r->ds.view;
    hj.cam = camera_view(r->cam, o.width, o.height);
    JobParams& j = hj.job;
    j.width = o.width;
    j.height = o.height;
    j.spp = o.spp;
    j.max_depth = o.max_depth;
    j.filter = o.filter;
    j.rng = o.rng;
    j.rr_depth = o.rr_depth;
    j.frame = r->frame;
    j.seed = o.seed;
    j.npix = npix;
    j.tonemap = o.tonemap;
    j.exposure = o.exposure;
    j.acc_color = r->acc_color.as<float4>();
    j.acc_albedo = r->acc_albedo.as<float4>();
    j.acc_normal = r->acc_normal.as<float4>();
    j.lcg_state = r->lcg_state.as<uint32_t>();
    j.color = r->color.as<float4>();
    j.albedo = r->albedo.as<float4>();
    j.normal = r->normal.as<float4>();
    j.rgba8 = r->rgba8.as<uint32_t>();
    r->frame++;
    cudaStream_t s = r->stream;
    const int64_t trained_paths = train_waves * npix;
    const int64_t nwaves = train_waves + (total - trained_paths + cap - 1) / cap;
    std::vector<WaveParams> waves(static_cast<size_t>(nwaves));
    int64_t begin = 0;
    for (int64_t w = 0; w < nwaves; w++) {
        WaveParams& wp = waves[size_t(w)];
        std::memset(&wp, 0, sizeof(wp));
        wp.num_seg = 1;
        wp.wave_count = int(std::min<int64_t>(w < train_waves ? npix : cap, total - begin));
        wp.seg[0].job = 0;
        wp.seg[0].slot_begin = 0;
        wp.seg[0].count = wp.wave_count;
        wp.seg[0].path_begin = begin;
        begin += wp.wave_count;
    }
    RT_CUDA(r->segs.alloc(waves.size() * sizeof(WaveParams)), "allocate wave table");
    {  // launch parameters and wave table through the next pinned staging buffer
        rt_renderer::HostStage& hs = r->stage[r->stage_next];
        r->stage_next = (r->stage_next + 1) % rt_renderer::kStages;
        const size_t wbytes = waves.size() * sizeof(WaveParams), need = sizeof(hj) + wbytes;
        if (hs.copied) RT_CUDA(cudaEventSynchronize(hs.copied), "staging buffer reuse");
        if (hs.bytes < need) {
            if (hs.ptr) cudaFreeHost(hs.ptr);
            hs.ptr = nullptr;
            hs.bytes = 0;
            RT_CUDA(cudaHostAlloc(&hs.ptr, need, cudaHostAllocDefault), "allocate pinned staging");
            hs.bytes = need;
        }
        if (!hs.copied) RT_CUDA(cudaEventCreateWithFlags(&hs.copied, cudaEventDisableTiming), "staging event");
        char* h = static_cast<char*>(hs.ptr);
        std::memcpy(h, &hj, sizeof(hj));
        std::memcpy(h + sizeof(hj), waves.data(), wbytes);
        RT_CUDA(cudaMemcpyAsync(r->job.ptr, h, sizeof(hj), cudaMemcpyHostToDevice, s), "upload launch parameters");
        RT_CUDA(cudaMemcpyAsync(r->segs.ptr, h + sizeof(hj), wbytes, cudaMemcpyHostToDevice, s), "upload wave table");
        RT_CUDA(cudaEventRecord(hs.copied, s), "staging event");
    }
    r->h2d_bytes = int64_t(sizeof(hj) + waves.size() * sizeof(WaveParams));
    if (!r->wave_index.ptr) RT_CUDA(r->wave_index.alloc(sizeof(int)), "allocate wave counter");
    RT_CUDA(cudaMemsetAsync(r->wave_index.ptr, 0, sizeof(int), s), "clear wave counter");
    RT_CUDA(cudaMemsetAsync(r->ctl.ptr, 0, sizeof(WaveCtl), s), "clear counters");
    const bool stats = o.collect_stats != 0;
    r->timer.reset();
    RT_CUDA(cudaEventRecord(r->ev0, s), "record event");
    const JobDesc* dj = r->job.as<JobDesc>();
    rth::launch_begin(hj, dj, s);
    int launches = 1;
    int ext = 0;
    Ctx c;
    std::memset(&c, 0, sizeof(c));
    c.jobs = dj;
    wave_bufs(r, c.wb);
    c.waves = r->segs.as<WaveParams>();
    c.wave_index = r->wave_index.as<int>();
    c.wave_ring = int(nwaves);
    c.max_depth = o.max_depth;
    c.features = (r->ds.view.num_media > 0 ? kFeatureMedia : 0) | (guided ? kFeatureGuide : 0) |
                 (r->ds.view.num_tex > 0 ? kFeatureTextures : 0);
    rtg::NetView net{};
    if (guided) {
        float3 lo, inv;
        for (int a = 0; a < 3; a++) {  // 1% margin around the scene bounds
            const float ext = std::max(r->hi[a] - r->lo[a], 1e-6f);
            (&lo.x)[a] = r->lo[a] - 0.01f * ext;
            (&inv.x)[a] = 1.0f / (1.02f * ext);
        }
        net = guide_view(r->guide, lo, inv);
        c.G.mix = r->g_mix.as<rtg::Mixture>();
        c.G.prob = o.guide_prob;
        c.G.min_rough = 0.3f;
        c.G.lo = lo;
        c.G.inv_ext = inv;
    }
    const int gsms = guided ? guide_sms(r->guide) : 0;
    auto issue_wave = [&](bool timed, bool training) {
        c.G.rec = training ? r->g_rec.as<float4>() : nullptr;
        if (training) cudaMemsetAsync(r->g_count.ptr, 0, sizeof(int), s);
        c.bounce = 0;
        rth::launch_raygen(c, s);
        if (timed) {  // one kernel after the other, each between two timing events
            for (int bnc = 0; bnc < o.max_depth; bnc++) {
                c.bounce = bnc;
                size_t i0 = r->timer.used;
                cudaEventRecord(r->timer.next(), s);
                rth::launch_extend(c, r->shape, true, s);
                cudaEventRecord(r->timer.next(), s);
                if (guided) rtgh::launch_infer(c, net, gsms, s);
                rth::launch_shade(c, r->shape, true, s);
                cudaEventRecord(r->timer.next(), s);
                rth::launch_sample(c, r->shape, true, s);
                cudaEventRecord(r->timer.next(), s);
                rth::launch_shadow(c, r->shape, true, s);
                cudaEventRecord(r->timer.next(), s);
                r->timer.marks.push_back({0, i0});
                r->timer.marks.push_back({1, i0 + 1});
                r->timer.marks.push_back({3, i0 + 2});
                r->timer.marks.push_back({2, i0 + 3});
            }
        } else {  // a bounce's k_shadow beside its k_sample and the next bounce's k_extend
            rth::launch_extend(c, r->shape, false, s);
            for (int bnc = 0; bnc < o.max_depth; bnc++) {
                c.bounce = bnc;
                if (guided) rtgh::launch_infer(c, net, gsms, s);
                rth::launch_shade(c, r->shape, false, s);
                if (bnc + 1 < o.max_depth) {
                    rth::launch_sample_shadow_and_next_extend(c, r->shape, s, r->have_fork ? &r->fork : nullptr);
                } else {
                    rth::launch_sample(c, r->shape, false, s);
                    rth::launch_shadow(c, r->shape, false, s);
                }
            }
        }
        rth::launch_resolve(c, s);
        if (training) rtgh::launch_collect(c, r->g_buf.as<float4>(), r->g_count.as<int>(), int(r->g_buf.bytes / 32), s);
        rth::launch_next_wave(c, s);
    };
    // training waves, each followed by guide_steps Adam steps on batches of its samples
    for (int64_t w = 0; w < train_waves; w++) {
        issue_wave(stats, true);
        for (int k = 0; k < o.guide_steps; k++) {
            RT_CUDA(cudaMemsetAsync(r->g_wsum.ptr, 0, sizeof(float), s), "guide batch");
            rtgh::launch_batch(r->g_buf.as<float4>(), r->g_count.as<int>(), int(r->g_buf.bytes / 32), kGuideBatch,
                               r->guide_seed++ * 0x9E3779B9u, r->g_bpos.as<float>(), r->g_bdir.as<float>(),
                               r->g_bw.as<float>(), r->g_wsum.as<float>(), s);
            st = guide_train_device(r->guide, r->g_bpos.as<float>(), r->g_bdir.as<float>(), r->g_bw.as<float>(),
                                    kGuideBatch, 1.0f, r->g_wsum.as<float>(), s);
            if (st) return st;
        }
    }
    r->guide_trained += train_waves;
    const int64_t plain_waves = nwaves - train_waves;
    // graph capture is not possible on the legacy default stream
    if (stats || s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
        for (int64_t w = 0; w < plain_waves; w++) issue_wave(stats, false);
    } else if (plain_waves > 0) {
        if (!r->graph || r->graph_capacity != r->capacity || r->graph_depth != o.max_depth ||
            r->graph_waves != r->segs.ptr || r->graph_ring != int(nwaves) || r->graph_guided != guided ||
            r->graph_mix != r->g_mix.ptr) {
            if (r->graph) cudaGraphExecDestroy(r->graph);
            r->graph = nullptr;
            cudaGraph_t g = nullptr;
            RT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin graph capture");
            issue_wave(false, false);
            RT_CUDA(cudaStreamEndCapture(s, &g), "end graph capture");
            cudaError_t e = cudaGraphInstantiate(&r->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "instantiate wave graph");
            r->graph_capacity = r->capacity;
            r->graph_depth = o.max_depth;
            r->graph_waves = r->segs.ptr;
            r->graph_ring = int(nwaves);
            r->graph_guided = guided;
            r->graph_mix = r->g_mix.ptr;
        }
        for (int64_t w = 0; w < plain_waves; w++) RT_CUDA(cudaGraphLaunch(r->graph, s), "launch wave graph");
    }
    launches += int(nwaves) * (4 * o.max_depth + 3) + (guided ? int(nwaves) * o.max_depth : 0) +
                int(train_waves) * (1 + 3 * o.guide_steps);
    ext = int(nwaves) * o.max_depth;
    rth::launch_finalize(hj, dj, s);
    launches++;
    r->denoised = false;
    if (o.denoise) {  // Renderer.cpp:660-785: the displayed image is the denoised colour
        st = ensure_denoiser(r);
        if (st) return st;
        rth::DenoiseArgs d;
        d.color = r->color.as<float4>();
        d.albedo = r->albedo.as<float4>();
        d.normal = r->normal.as<float4>();
        d.tmp0 = r->dn_tmp0.as<float4>();
        d.tmp1 = r->dn_tmp1.as<float4>();
        d.out = r->dn_out.as<float4>();
        d.rgba8 = r->rgba8.as<uint32_t>();
        d.w = r->pw;
        d.h = r->ph;
        d.tonemap = o.tonemap;
        d.exposure = o.exposure;
        launches += rth::launch_denoise(d, s);
        r->denoised = true;
    }
    RT_CUDA(cudaEventRecord(r->ev1, s), "record event");
    RT_CUDA(cudaGetLastError(), "launch");
    r->rendered = true;
    r->launches = launches;
    r->waves = int(nwaves);
    r->extend_launches = ext;
    r->paths = total;
    return RT_OK;
}

rt_status rt_renderer_guide(rt_renderer* r, rt_guide** guide) {
    if (!r || !guide) return fail(RT_ERR_INVALID_ARG, "rt_renderer_guide: NULL argument");
    RT_ON_DEVICE(r, "rt_renderer_guide");
    if (!r->guide) {
        rt_status st = ensure_guide(r, 0, 0);
        if (st) return st;
    }
    *guide = r->guide;
    return RT_OK;
}

rt_status rt_renderer_guide_samples(rt_renderer* r, float* out, int64_t max_samples, int64_t* count) {
    if (!r || !count) return fail(RT_ERR_INVALID_ARG, "rt_renderer_guide_samples: NULL argument");
    RT_ON_DEVICE(r, "rt_renderer_guide_samples");
    *count = 0;
    if (!r->g_count.ptr) return RT_OK;
    int n = 0;
    RT_CUDA(cudaMemcpyAsync(&n, r->g_count.ptr, sizeof(int), cudaMemcpyDeviceToHost, r->stream), "guide samples");
    RT_CUDA(cudaStreamSynchronize(r->stream), "guide samples");
    const int64_t cap = int64_t(r->g_buf.bytes / 32);
    *count = std::min<int64_t>(n, cap);
    const int64_t k = std::min<int64_t>(*count, max_samples);
    if (out && k > 0) {
        RT_CUDA(cudaMemcpyAsync(out, r->g_buf.ptr, size_t(k) * 32, cudaMemcpyDeviceToHost, r->stream), "guide samples");
        RT_CUDA(cudaStreamSynchronize(r->stream), "guide samples");
    }
    return RT_OK;
}

rt_status rt_renderer_synchronize(rt_renderer* r) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "rt_renderer_synchronize: NULL renderer");
    RT_ON_DEVICE(r, "rt_renderer_synchronize");
    RT_CUDA(cudaStreamSynchronize(r->stream), "rt_renderer_synchronize");
    if (r->rendered && r->ctl.ptr) {  // the device-side step budget of media walks, traversal stack overflows
        int hits[2] = {0, 0};
        static_assert(offsetof(WaveCtl, overflow) == offsetof(WaveCtl, error) + sizeof(int), "counter layout");
        RT_CUDA(cudaMemcpy(hits, static_cast<char*>(r->ctl.ptr) + offsetof(WaveCtl, error), 2 * sizeof(int),
                           cudaMemcpyDeviceToHost),
                "rt_renderer_synchronize");
        if (hits[0] > 0)
            return fail(RT_ERR_DEVICE_WATCHDOG,
                        std::to_string(hits[0]) + " medium walks of the last render ran out of their " +
                            std::to_string(kMaxTrackingSteps) + "-step budget and were ended with zero weight");
        if (hits[1] > 0) return overflow_status(hits[1], "the last render");
    }
    if (r->opt.guided) {  // bounded waits of the guide network's tensor-core inference
        const int n = rtgh::take_tc_timeouts();
        if (n > 0)
            return fail(RT_ERR_DEVICE_WATCHDOG,
                        std::to_string(n) + " guide inference blocks gave up waiting for their tensor-core work");
    }
    return RT_OK;
}

static rt_status download(rt_renderer* r, const DevBuf& b, void* dst, size_t bytes) {
    if (!r || !dst) return fail(RT_ERR_INVALID_ARG, "download: NULL argument");
    RT_ON_DEVICE(r, "download");
    if (!b.ptr) return fail(RT_ERR_STATE, "download: nothing rendered at this size");
    RT_CUDA(cudaMemcpyAsync(dst, b.ptr, bytes, cudaMemcpyDeviceToHost, r->stream), "download");
    RT_CUDA(cudaStreamSynchronize(r->stream), "download");
    return RT_OK;
}

rt_status rt_renderer_download_rgba8(rt_renderer* r, uint32_t* px) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "NULL renderer");
    return download(r, r->rgba8, px, size_t(r->pw) * r->ph * 4);
}

rt_status rt_renderer_download_linear(rt_renderer* r, float* rgba) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "NULL renderer");
    return download(r, r->color, rgba, size_t(r->pw) * r->ph * 16);
}

rt_status rt_renderer_download_aov(rt_renderer* r, int32_t kind, float* rgba) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "NULL renderer");
    size_t n = size_t(r->pw) * r->ph * 16;
    if (kind == RT_AOV_COLOR) return download(r, r->color, rgba, n);
    if (kind == RT_AOV_ALBEDO) return download(r, r->albedo, rgba, n);
    if (kind == RT_AOV_NORMAL) return download(r, r->normal, rgba, n);
    if (kind == RT_AOV_DENOISED) {
        if (!r->denoised) return fail(RT_ERR_STATE, "rt_renderer_download_aov: the last render was not denoised");
        return download(r, r->dn_out, rgba, n);
    }
    return fail(RT_ERR_INVALID_ARG, "rt_renderer_download_aov: unknown kind");
}

rt_status rt_renderer_device_buffers(rt_renderer* r, void** color, void** rgba8) {
    if (!r) return fail(RT_ERR_INVALID_ARG, "NULL renderer");
    if (color) *color = r->color.ptr;
    if (rgba8) *rgba8 = r->rgba8.ptr;
    return RT_OK;
}

rt_status rt_renderer_frame_index(const rt_renderer* r, int32_t* f) {
    if (!r || !f) return fail(RT_ERR_INVALID_ARG, "NULL argument");
    *f = r->frame;
    return RT_OK;
}

rt_status rt_renderer_get_stats(const rt_renderer* rc, rt_render_stats* out) {
    rt_renderer* r = const_cast<rt_renderer*>(rc);
    if (!r || !out) return fail(RT_ERR_INVALID_ARG, "rt_renderer_get_stats: NULL argument");
    RT_ON_DEVICE(r, "rt_renderer_get_stats");
    std::memset(out, 0, sizeof(*out));
    if (!r->rendered) return RT_OK;
    RT_CUDA(cudaStreamSynchronize(r->stream), "rt_renderer_get_stats");
    WaveCtl ctl;
    RT_CUDA(cudaMemcpy(&ctl, r->ctl.ptr, sizeof(ctl), cudaMemcpyDeviceToHost), "read counters");
    out->paths = r->paths;
    out->extend_rays = int64_t(ctl.stats[0]);
    out->shadow_rays = int64_t(ctl.stats[1]);
    out->extend_nodes = int64_t(ctl.stats[2]);
    out->extend_tris = int64_t(ctl.stats[3]);
    out->nodes_visited = int64_t(ctl.stats[2] + ctl.stats[4]);
    out->tris_tested = int64_t(ctl.stats[3] + ctl.stats[5]);
    out->nan_samples = int64_t(ctl.stats[6]);
    out->nan_throughput_paths = int64_t(ctl.stats[7]);
    out->watchdog_walks = int64_t(ctl.error);
    out->stack_overflows = int64_t(ctl.overflow);
    out->waves = r->waves;
    out->launches = r->launches;
    out->extend_launches = r->extend_launches;
    out->wave_paths = r->wave_paths;
    out->h2d_bytes = r->h2d_bytes;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    out->ms_total = ms;
    float cls[4] = {0.f, 0.f, 0.f, 0.f};
    for (auto& m : r->timer.marks) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, r->timer.pool[m.second], r->timer.pool[m.second + 1]);
        cls[m.first] += t;
    }
    out->ms_extend = cls[0];
    out->ms_shade = cls[1];
    out->ms_shadow = cls[2];
    out->ms_sample = cls[3];
    out->ms_other = r->timer.marks.empty() ? 0.0f : ms - cls[0] - cls[1] - cls[2] - cls[3];
    return RT_OK;
}

rt_status rt_renderer_trace(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n, float* hits,
                            int32_t device_ptrs) {
    if (!r || (n > 0 && (!rays || !hits)) || n < 0) return fail(RT_ERR_INVALID_ARG, "rt_renderer_trace: bad argument");
    RT_ON_DEVICE(r, "rt_renderer_trace");
    if (n == 0) return RT_OK;
    int* ovf = overflow_counter(r);
    int h_ovf = 0;
    RT_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int), r->stream), "rt_renderer_trace");
    if (device_ptrs) {
        rth::launch_trace(r->ds.view, any_hit != 0, rays, n, hits, ovf, r->stream);
        RT_CUDA(cudaGetLastError(), "rt_renderer_trace");
        RT_CUDA(cudaMemcpyAsync(&h_ovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, r->stream), "rt_renderer_trace");
        RT_CUDA(cudaStreamSynchronize(r->stream), "rt_renderer_trace");
        return overflow_status(h_ovf, "rt_renderer_trace");
    }
    DevBuf dr, dh;
    RT_CUDA(dr.alloc(size_t(n) * 32), "rt_renderer_trace: allocate");
    RT_CUDA(dh.alloc(size_t(n) * 16), "rt_renderer_trace: allocate");
    RT_CUDA(cudaMemcpyAsync(dr.ptr, rays, size_t(n) * 32, cudaMemcpyHostToDevice, r->stream), "rt_renderer_trace");
    rth::launch_trace(r->ds.view, any_hit != 0, dr.as<float>(), n, dh.as<float>(), ovf, r->stream);
    RT_CUDA(cudaGetLastError(), "rt_renderer_trace");
    RT_CUDA(cudaMemcpyAsync(hits, dh.ptr, size_t(n) * 16, cudaMemcpyDeviceToHost, r->stream), "rt_renderer_trace");
    RT_CUDA(cudaMemcpyAsync(&h_ovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, r->stream), "rt_renderer_trace");
    RT_CUDA(cudaStreamSynchronize(r->stream), "rt_renderer_trace");
    return overflow_status(h_ovf, "rt_renderer_trace");
}

// Ray queries through the path tracer's own persistent traversal kernels:
// the batch is staged as the extend queue (closest hit) or the shadow queue
// (any hit) of a one-bounce wave and k_extend / k_shadow run on it with the
// launch shape of Render(), so these hits come from exactly the loop that
// renders images (lane refill, triangle postponing, near-to-far order).
rt_status rt_renderer_trace_wavefront(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n, float* hits,
                                      int64_t* counters) {
    if (!r || n < 0 || (n > 0 && (!rays || !hits)))
        return fail(RT_ERR_INVALID_ARG, "rt_renderer_trace_wavefront: bad argument");
    RT_ON_DEVICE(r, "rt_renderer_trace_wavefront");
    if (counters) counters[0] = counters[1] = counters[2] = 0;
    for (int64_t i = 0; i < n; i++) {  // the kernels' own ray extents
        const float tmin = rays[i * 8 + 3], tmax = rays[i * 8 + 7];
        if (tmin != kEps || std::isnan(tmax) || (!any_hit && tmax < FLT_MAX))
            return fail(RT_ERR_INVALID_ARG, "rt_renderer_trace_wavefront: ray " + std::to_string(i) +
                                                " must have tmin = 1e-4 (the integrator's ray offset) and, for "
                                                "closest-hit queries, tmax = FLT_MAX or infinity");
    }
    if (n == 0) return RT_OK;
    constexpr int kChunk = 1 << 22;
    const int chunk = int(std::min<int64_t>(n, kChunk));
    rt_status st = ensure_waves(r, chunk);
    if (st) return st;
    if (!r->q_job.ptr) {
        RT_CUDA(r->q_job.alloc(sizeof(JobDesc)), "rt_renderer_trace_wavefront: allocate");
        RT_CUDA(r->q_wave.alloc(sizeof(WaveParams)), "rt_renderer_trace_wavefront: allocate");
        RT_CUDA(r->q_index.alloc(sizeof(int)), "rt_renderer_trace_wavefront: allocate");
        RT_CUDA(r->q_ctl.alloc(sizeof(WaveCtl)), "rt_renderer_trace_wavefront: allocate");
    }
    cudaStream_t s = r->stream;
    JobDesc hj;
    std::memset(&hj, 0, sizeof(hj));
    hj.sc = r->ds.view;
    RT_CUDA(cudaMemcpyAsync(r->q_job.ptr, &hj, sizeof(hj), cudaMemcpyHostToDevice, s), "rt_renderer_trace_wavefront");
    RT_CUDA(cudaMemsetAsync(r->q_index.ptr, 0, sizeof(int), s), "rt_renderer_trace_wavefront");
    DevBuf dr, dh;
    RT_CUDA(dr.alloc(size_t(chunk) * 32), "rt_renderer_trace_wavefront: allocate");
    RT_CUDA(dh.alloc(size_t(chunk) * 16), "rt_renderer_trace_wavefront: allocate");
    Ctx c;
    std::memset(&c, 0, sizeof(c));
    c.jobs = r->q_job.as<JobDesc>();
    wave_bufs(r, c.wb);
    c.wb.ctl = r->q_ctl.as<WaveCtl>();
    c.waves = r->q_wave.as<WaveParams>();
    c.wave_index = r->q_index.as<int>();
    c.wave_ring = 1;
    c.bounce = 0;
    c.max_depth = 1;
    const bool stats = counters != nullptr;
    int overflows = 0;
    for (int64_t b0 = 0; b0 < n; b0 += chunk) {
        const int m = int(std::min<int64_t>(chunk, n - b0));
        WaveParams wp;
        std::memset(&wp, 0, sizeof(wp));
        wp.num_seg = 1;
        wp.wave_count = m;
        wp.seg[0].count = m;
        RT_CUDA(cudaMemcpyAsync(r->q_wave.ptr, &wp, sizeof(wp), cudaMemcpyHostToDevice, s), "rt_renderer_trace_wavefront");
        RT_CUDA(cudaMemcpyAsync(dr.ptr, rays + b0 * 8, size_t(m) * 32, cudaMemcpyHostToDevice, s),
                "rt_renderer_trace_wavefront");
        rth::launch_query_stage(c, dr.as<float>(), m, any_hit != 0, s);
        if (any_hit)
            rth::launch_shadow(c, r->shape, stats, s);
        else
            rth::launch_extend(c, r->shape, stats, s);
        rth::launch_query_collect(c, r->ds.view, dh.as<float>(), m, any_hit != 0, s);
        RT_CUDA(cudaGetLastError(), "rt_renderer_trace_wavefront");
        RT_CUDA(cudaMemcpyAsync(hits + b0 * 4, dh.ptr, size_t(m) * 16, cudaMemcpyDeviceToHost, s),
                "rt_renderer_trace_wavefront");
        WaveCtl ctl;
        RT_CUDA(cudaMemcpyAsync(&ctl, r->q_ctl.ptr, sizeof(ctl), cudaMemcpyDeviceToHost, s), "rt_renderer_trace_wavefront");
        RT_CUDA(cudaStreamSynchronize(s), "rt_renderer_trace_wavefront");
        overflows += ctl.overflow;
        if (counters) {
            const int o = any_hit ? 1 : 0;  // stats: extend rays, shadow rays, ext nodes, ext tris, sh nodes, sh tris
            counters[0] += int64_t(ctl.stats[o]);
            counters[1] += int64_t(ctl.stats[2 + 2 * o]);
            counters[2] += int64_t(ctl.stats[3 + 2 * o]);
        }
    }
    return overflow_status(overflows, "rt_renderer_trace_wavefront");
}

// Same queries as rt_renderer_trace with host buffers, staged in the fixed
// device array of rt_trace_scratch.cu instead of buffers allocated per call.
rt_status rt_renderer_trace_noalloc(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n, float* hits) {
    if (!r || n < 0 || (n > 0 && (!rays || !hits)))
        return fail(RT_ERR_INVALID_ARG, "rt_renderer_trace_noalloc: bad argument");
    RT_ON_DEVICE(r, "rt_renderer_trace_noalloc");
    const int64_t cap = rth::trace_scratch_rays();
    if (n > cap)
        return fail(RT_ERR_INVALID_ARG, "rt_renderer_trace_noalloc: " + std::to_string(n) + " rays exceed the " +
                                            std::to_string(cap) +
                                            " of the static scratch; split the batch or use rt_renderer_trace");
    if (n == 0) return RT_OK;
    void* scratch = nullptr;
    RT_CUDA(rth::trace_scratch_address(r->device, &scratch), "rt_renderer_trace_noalloc: scratch address");
    float4* sc = static_cast<float4*>(scratch);
    int* ovf = overflow_counter(r);  // the renderer's own control block: nothing allocated
    int h_ovf = 0;
    RT_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int), r->stream), "rt_renderer_trace_noalloc");
    RT_CUDA(cudaMemcpyAsync(sc, rays, size_t(n) * 32, cudaMemcpyHostToDevice, r->stream), "rt_renderer_trace_noalloc");
    rth::launch_trace_scratch(r->ds.view, any_hit != 0, scratch, int(n), ovf, r->stream);
    RT_CUDA(cudaGetLastError(), "rt_renderer_trace_noalloc");
    RT_CUDA(cudaMemcpyAsync(hits, sc + 2 * cap, size_t(n) * 16, cudaMemcpyDeviceToHost, r->stream),
            "rt_renderer_trace_noalloc");
    RT_CUDA(cudaMemcpyAsync(&h_ovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, r->stream), "rt_renderer_trace_noalloc");
    RT_CUDA(cudaStreamSynchronize(r->stream), "rt_renderer_trace_noalloc");
    return overflow_status(h_ovf, "rt_renderer_trace_noalloc");
}

rt_status rt_write_png(const char* path, const uint32_t* rgba8, int32_t w, int32_t h) {
    if (!path || !rgba8 || w <= 0 || h <= 0) return fail(RT_ERR_INVALID_ARG, "rt_write_png: bad argument");
    std::string err;
    if (!rti::write_png(path, rgba8, w, h, err)) return fail(RT_ERR_IO, "rt_write_png: " + err);
    return RT_OK;
}

rt_status rt_denoise_image(const float* color, const float* albedo, const float* normal, int32_t w, int32_t h,
                           float* out) {
    if (!color || !albedo || !normal || !out || w <= 0 || h <= 0 || int64_t(w) * h > (int64_t(1) << 28))
        return fail(RT_ERR_INVALID_ARG, "rt_denoise_image: bad argument");
    const size_t bytes = size_t(w) * h * sizeof(float4);
    DevBuf c, a, n, t0, t1, o;
    DevBuf* all[] = {&c, &a, &n, &t0, &t1, &o};
    for (DevBuf* b : all) RT_CUDA(b->alloc(bytes), "rt_denoise_image");
    RT_CUDA(cudaMemcpy(c.ptr, color, bytes, cudaMemcpyHostToDevice), "rt_denoise_image");
    RT_CUDA(cudaMemcpy(a.ptr, albedo, bytes, cudaMemcpyHostToDevice), "rt_denoise_image");
    RT_CUDA(cudaMemcpy(n.ptr, normal, bytes, cudaMemcpyHostToDevice), "rt_denoise_image");
    rth::DenoiseArgs d;
    d.color = c.as<float4>();
    d.albedo = a.as<float4>();
    d.normal = n.as<float4>();
    d.tmp0 = t0.as<float4>();
    d.tmp1 = t1.as<float4>();
    d.out = o.as<float4>();
    d.rgba8 = nullptr;
    d.w = w;
    d.h = h;
    d.tonemap = RT_TONEMAP_REINHARD;
    d.exposure = 1.0f;
    rth::launch_denoise(d, nullptr);
    RT_CUDA(cudaGetLastError(), "rt_denoise_image");
    RT_CUDA(cudaMemcpy(out, o.ptr, bytes, cudaMemcpyDeviceToHost), "rt_denoise_image");
    return RT_OK;
}

rt_status rt_verify_shading(int32_t op, const rt_material* materials, int32_t nmat, const rt_light* lights, int32_t nl,
                            const rt_medium* media, int32_t nm, const float* in, int64_t n, float* out) {
    if (!in || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "rt_verify_shading: bad argument");
    if (op < RT_VERIFY_BSDF_EVAL || op > RT_VERIFY_BSDF_SAMPLE_PDF)
        return fail(RT_ERR_INVALID_ARG, "rt_verify_shading: unknown op");
    for (int64_t i = 0; i < n; i++) {
        const float* x = in + i * 16;
        int idx = (op == RT_VERIFY_BSDF_EVAL || op == RT_VERIFY_BSDF_SAMPLE_PDF) ? int(x[10])
                  : op == RT_VERIFY_BSDF_SAMPLE ? int(x[13])
                  : op == RT_VERIFY_LIGHT_SAMPLE ? int(x[5])
                  : op == RT_VERIFY_LIGHT_EVAL ? int(x[7])
                  : op == RT_VERIFY_MEDIUM_SAMPLE ? int(x[3])
                  : op == RT_VERIFY_PHASE_SAMPLE ? int(x[7])
                                                  : int(x[6]);
        int lim = (op <= RT_VERIFY_BSDF_SAMPLE || op == RT_VERIFY_BSDF_SAMPLE_PDF) ? nmat
                  : (op <= RT_VERIFY_LIGHT_EVAL ? nl : nm);
        if (idx < 0 || idx >= lim) return fail(RT_ERR_INVALID_ARG, "rt_verify_shading: index out of range");
    }
    if (n == 0) return RT_OK;
    cudaStream_t s = nullptr;
    DevBuf dm, dl, dmed, dlut, davg, din, dout;
    std::vector<DevMaterial> m;
    for (int i = 0; i < nmat; i++) m.push_back(to_dev(materials[i]));
    std::vector<DevLight> l;
    for (int i = 0; i < nl; i++) l.push_back(to_dev(lights[i]));
    std::vector<DevMedium> md;
    for (int i = 0; i < nm; i++) md.push_back(to_dev(media[i]));
    const float* avg = nullptr;
    const float* lut = kc_tables(&avg);
    RT_CUDA(dm.upload(m.data(), m.size() * sizeof(DevMaterial), s), "rt_verify_shading");
    RT_CUDA(dl.upload(l.data(), l.size() * sizeof(DevLight), s), "rt_verify_shading");
    RT_CUDA(dmed.upload(md.data(), md.size() * sizeof(DevMedium), s), "rt_verify_shading");
    RT_CUDA(dlut.upload(lut, 64 * 64 * 4, s), "rt_verify_shading");
    RT_CUDA(davg.upload(avg, 64 * 4, s), "rt_verify_shading");
    RT_CUDA(din.upload(in, size_t(n) * 64, s), "rt_verify_shading");
    RT_CUDA(dout.alloc(size_t(n) * 32), "rt_verify_shading");
    SceneView v;
    std::memset(&v, 0, sizeof(v));
    v.materials = dm.as<DevMaterial>();
    v.lut = dlut.as<float>();
    v.lut_avg = davg.as<float>();
    rth::launch_verify(op, v, dl.as<DevLight>(), dmed.as<DevMedium>(), din.as<float>(), n, dout.as<float>(), s);
    RT_CUDA(cudaGetLastError(), "rt_verify_shading");
    RT_CUDA(cudaMemcpy(out, dout.ptr, size_t(n) * 32, cudaMemcpyDeviceToHost), "rt_verify_shading");
    return RT_OK;
}

}  // extern "C"
