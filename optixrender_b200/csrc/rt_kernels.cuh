// rt_kernels.cuh - host-visible declarations of the wavefront pipeline.
//
// One Renderer::Render() (core/src/Renderer.cpp:635-793) becomes, per wave of
// paths: raygen -> [extend -> shade -> shadow] x max_depth -> resolve, and
// finally finalize (running mean, AOVs, tonemap).  The megakernel loop of
// core/cuda/devicePrograms.cu:213-516 is split at every optixTrace call.
#pragma once

#include "rt_device.cuh"
#include "rt_guide.cuh"

namespace rtd {

constexpr int kMaxSegments = 16;
// Shade queue buckets: the material type of the hit surface (0..7), or a miss.
constexpr int kShadeBuckets = 9;
constexpr int kMissBucket = 8;

// Per-render parameters and per-pixel buffers of one job.
struct JobParams {
    int width, height, spp, max_depth;
    int filter, rng, rr_depth, frame;
    uint64_t seed;
    int64_t npix;
    int tonemap;
    float exposure;
    float4* acc_color;   // per pixel: running sum of the launch (w: aborted flag)
    float4* acc_albedo;
    float4* acc_normal;
    uint32_t* lcg_state; // per pixel (RT_RNG_LCG)
    float4* color;       // running mean across Render() calls
    float4* albedo;
    float4* normal;
    uint32_t* rgba8;
};

struct JobDesc {
    SceneView sc;
    CameraView cam;
    JobParams job;
};

// A contiguous run of one job's paths inside a wave.
struct Segment {
    int job;
    int slot_begin;
    int count;
    int pad;
    int64_t path_begin;
};

struct WaveCtl {
    int count[2];
    // shadow rays queued by k_shade at bounces of parity 0 / 1: k_shadow of
    // bounce b reads entry b & 1 while k_sample of bounce b clears entry
    // (b + 1) & 1 for the next k_shade, so the two kernels may run side by side
    int shadow_count[2];
    int fetch_ext;
    int fetch_shade;
    int fetch_shadow;
    int error;     // media walks that exhausted their step budget in this render
    int overflow;  // traversal node groups that found the stack full (the BVH depth check keeps this 0)
    unsigned long long stats[8];  // extend rays, shadow rays, ext nodes, ext tris, sh nodes, sh tris,
                                  // NaN samples, paths ended by a NaN throughput
    int bucket[kShadeBuckets];    // extend results per shade bucket
    int sample_count;             // paths k_shade left at BSDF sampling (k_sample's queue)
    int fetch_sample;
};

// Per-slot path state of a wave.  A slot's eight float4 fields of path state lie together in one 128-byte
// record (one cache line), so that the shade and sample kernels, which touch
// most of a slot's state, read one line per slot instead of eight lines of
// eight arrays; the slots are visited in the scattered order of the material
// sort.  A field is the record array at the field's byte offset.
constexpr size_t kSlotRecord = 128;
enum SlotOffset : size_t {
    kRecRayO = 0, kRecRayD = 16, kRecHit = 32, kRecThr = 48, kRecRad = 64, kRecNee0 = 80, kRecNee1 = 96, kRecStale = 112
};
struct SlotField {
    char* base;  // record array + the field's offset
    RT_HD float4& operator[](size_t slot) const { return *reinterpret_cast<float4*>(base + slot * kSlotRecord); }
};
RT_HD SlotField slot_field(void* records, SlotOffset off) { return SlotField{static_cast<char*>(records) + off}; }

struct WaveBufs {
    SlotField ray_o;   // origin
    SlotField ray_d;   // direction
    SlotField hit;     // t, b1, b2, triangle (bits; -1 = miss)
    SlotField thr;     // throughput (history), pre_pdf
    SlotField rad;     // radiance
    SlotField nee0;    // pending environment NEE contribution
    SlotField nee1;    // pending light NEE contribution
    SlotField stale;   // shading normal and mesh of the last hit
    float4* aov_a;   // albedo, normal.x
    float2* aov_n;   // normal.y, normal.z
    uint2* rng;      // random state
    int* queue[2];   // active slots
    int* squeue;     // slots waiting for BSDF sampling (k_sample)
    float4* sh_o;    // shadow ray origin, tmax
    float4* sh_d;    // shadow ray direction, slot * 2 + channel (bits)
    int* sorted;     // kShadeBuckets regions of `capacity` slots: extend results by material type (or null)
    DevMaterial* mat_tex;  // per slot: the textured copy of the last hit's material (null: no textures)
    WaveCtl* ctl;
    int capacity;
};

// The per-wave part of a launch, in device memory so that one captured graph
// serves every wave: kernels read waves[*wave_index].
struct WaveParams {
    Segment seg[kMaxSegments];
    int num_seg;
    int wave_count;
    int pad[2];
};

struct Ctx {
    const JobDesc* jobs;
    WaveBufs wb;
    const WaveParams* waves;
    int* wave_index;  // advanced by k_next_wave at the end of each wave
    int wave_ring;    // number of WaveParams entries; the index wraps around
    int bounce;
    int max_depth;  // largest max_depth of the jobs in the wave
    rtg::GuideCtx G;  // path guiding (G.mix null: not guided)
    int features;     // kFeature* bits of the wave's scenes and jobs (host side: picks the shade kernel)
};

// Scene and job features that need the full shade kernel.
constexpr int kFeatureMedia = 1, kFeatureGuide = 2, kFeatureTextures = 4;

#ifdef __CUDACC__
RT_D const WaveParams& wave_of(const Ctx& c) { return c.waves[*c.wave_index]; }

// The segment of a wave that holds `slot`.
RT_D int find_segment(const WaveParams& w, int slot) {
    int s = w.num_seg - 1;
    while (s > 0 && slot < w.seg[s].slot_begin) s--;
    return s;
}
#endif

}  // namespace rtd

// Host launchers (rt_kernels.cu).
namespace rth {
struct LaunchShape {
    int sms;
    int blocks_extend, blocks_shade, blocks_shadow;
    int blocks_shade_plain;  // the shade kernel without media, guiding and textures
    int blocks_sample;
};
void query_shape(LaunchShape& s);
// The a-trous denoiser: colour, albedo and normal AOVs (W x H float4) in;
// denoised linear colour (and, when rgba8 is not null, its tonemapped RGBA8)
// out; tmp0 / tmp1 are W x H float4 scratch.  Returns the kernels launched.
constexpr int kDenoisePasses = 5;
constexpr float kDenoiseSigmaColor = 1.0f;   // irradiance difference relative to the centre's luminance
constexpr float kDenoiseSigmaNormal = 0.3f;
constexpr float kDenoiseSigmaAlbedo = 0.1f;
struct DenoiseArgs {
    const float4* color;
    const float4* albedo;
    const float4* normal;
    float4* tmp0;
    float4* tmp1;
    float4* out;
    uint32_t* rgba8;
    int w, h;
    int tonemap;
    float exposure;
};
int launch_denoise(const DenoiseArgs& d, cudaStream_t st);
void launch_begin(const rtd::JobDesc& host_job, const rtd::JobDesc* dev_job, cudaStream_t st);
void launch_raygen(const rtd::Ctx& c, cudaStream_t st);
void launch_extend(const rtd::Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st);
void launch_shade(const rtd::Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st);
// BSDF sampling of the paths k_shade left at a surface (runs between shade and shadow).
void launch_sample(const rtd::Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st);
void launch_shadow(const rtd::Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st);
// A second stream and two events (created with cudaEventDisableTiming) for
// the two branches of a wave below.
struct WaveFork {
    cudaStream_t side;
    cudaEvent_t fork, join;
};
// After k_shade of bounce c.bounce: its shadow rays, and its BSDF sampling
// followed by the next bounce's closest hits, share no data: k_shadow reads
// the shadow queue and its length (shadow_count[bounce & 1]) and clears the
// NEE fields of occluded slots; k_sample reads and writes the other fields of
// the slots it samples and clears shadow_count[(bounce + 1) & 1] and the
// shade buckets; k_extend reads the path queue and writes the hit fields,
// the shade buckets and the counters of the next k_shade and k_sample.  So
// with `f` k_shadow runs on f->side as a parallel branch of the stream (or of
// the wave's graph when capturing), joined back before the next k_shade, and
// the kernels fill each other's tails.  Without `f` the three run one after
// the other on `st`.
void launch_sample_shadow_and_next_extend(rtd::Ctx c, const LaunchShape& s, cudaStream_t st, const WaveFork* f);
cudaError_t create_fork(WaveFork& f);  // on the current device; on failure nothing stays allocated
void destroy_fork(WaveFork& f);
void launch_resolve(const rtd::Ctx& c, cudaStream_t st);
void launch_next_wave(const rtd::Ctx& c, cudaStream_t st);
void launch_finalize(const rtd::JobDesc& host_job, const rtd::JobDesc* dev_job, cudaStream_t st);
void launch_begin_n(const rtd::JobDesc* dev_job, int64_t npix, cudaStream_t st);
void launch_finalize_n(const rtd::JobDesc* dev_job, int64_t npix, cudaStream_t st);
// Per-thread ray queries; `overflow` (device int) counts traversal stack overflows.
void launch_trace(const rtd::SceneView& sc, bool any_hit, const float* rays, int64_t n, float* hits, int* overflow,
                  cudaStream_t st);
// Ray queries through the wavefront kernels: stage n rays (8 floats each, device)
// as the extend queue (closest hit) or the shadow queue (any hit) of a wave,
// run launch_extend / launch_shadow, then collect the hits (4 floats each, device).
void launch_query_stage(const rtd::Ctx& c, const float* rays, int n, bool any_hit, cudaStream_t st);
void launch_query_collect(const rtd::Ctx& c, const rtd::SceneView& sc, float* hits, int n, bool any_hit,
                          cudaStream_t st);
void launch_verify(int op, const rtd::SceneView& sc, const rtd::DevLight* lights, const rtd::DevMedium* media,
                   const float* in, int64_t n, float* out, cudaStream_t st);
// rt_trace_scratch.cu: ray queries staged in a fixed device array.
int64_t trace_scratch_rays();
cudaError_t trace_scratch_address(int device, void** ptr);
void launch_trace_scratch(const rtd::SceneView& sc, bool any_hit, void* scratch, int n, int* overflow, cudaStream_t st);
}  // namespace rth
