// rt_server.cpp - continuous-batching render server.
//
// Scenes are uploaded once and stay resident.  Jobs are admitted in arrival
// order while the device-memory budget and the job table allow; each
// admitted job owns its accumulation and output buffers.  Every wave the
// scheduler fills the shared path slots with contiguous path ranges taken
// from the admitted jobs in admission order (up to kMaxSegments jobs per
// wave), so a job that arrives while others run joins the next wave.  A wave
// is one replay of a captured CUDA graph (raygen, (extend, shade, shadow) x
// depth, resolve, advance) whose parameters come from a device ring.  A job
// whose paths have all been issued gets its finalize kernel and an event; the
// host marks it done when the event completes.
//
// Nothing on the job path synchronises the device: a job's buffers are one
// stream-ordered allocation from the server's memory pool (freed the same
// way, so a release never waits for waves in flight), its descriptor is
// copied from pinned staging memory, and downloads use their own stream.
//
// Paths draw PCG32 streams keyed by (job seed, path index) and each pixel's
// samples are summed in sample order, so a plain job's image does not depend
// on which jobs share its waves.
//
// Guided jobs: every resident scene owns one guiding network.  A wave holds
// either plain jobs of any scenes or the guided jobs of one scene (the
// network a wave samples is fixed while it runs, so the estimate stays
// unbiased); the scene's first guide_train_waves guided waves record training
// samples and are followed by guide_steps Adam steps, and every later guided
// job on the scene samples the trained network without training again.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "rt_guide_host.h"
#include "rt_internal.h"
#include "rt_schedule.h"

static_assert(int(RT_SERVE_FAIR) == int(rti::kPlanFair) && int(RT_SERVE_FIFO) == int(rti::kPlanFifo) &&
                  int(RT_SERVE_SRPT) == int(rti::kPlanSrpt),
              "policy numbering");

using namespace rtd;
using namespace rti;

namespace {

#define SV_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// The server's device current for the rest of the calling scope.
#define SV_ON_DEVICE(srv, what)                                        \
    DeviceGuard dg_((srv)->device);                                    \
    if (dg_.status != cudaSuccess) return cuda_fail(dg_.status, what)

struct Job {
    int64_t id;
    rt_job_desc desc;
    int state = RT_JOB_QUEUED;
    double submit_ms = 0, admit_ms = 0, done_ms = 0;
    int slot = -1;
    int64_t npix = 0, total = 0, issued = 0;
    int64_t bytes = 0;
    // one pool allocation: acc_color, acc_albedo, acc_normal, color, albedo,
    // normal (float4 per pixel), then lcg and rgba8 (4 bytes per pixel)
    char* mem = nullptr;
    cudaEvent_t done_ev = nullptr;
    float4* f4(int k) const { return reinterpret_cast<float4*>(mem) + size_t(k) * size_t(npix); }
    uint32_t* u32(int k) const { return reinterpret_cast<uint32_t*>(mem + size_t(npix) * 96) + size_t(k) * size_t(npix); }
    bool finalize_issued = false;
};

int64_t job_bytes(int64_t npix) { return npix * (6 * 16 + 2 * 4); }

constexpr int kGuideBatch = 1 << 18;  // training samples per Adam step

// The guiding network of one resident scene.
struct SceneGuide {
    rt_guide* net = nullptr;
    float3 lo{}, inv{};  // position normalisation: scene bounds with a 1% margin
    int64_t train_waves = 0;
    uint32_t seed = 1;
};

}  // namespace

struct rt_server {
    rt_server_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t dl_stream = nullptr;  // downloads of finished images
    rth::WaveFork fork{};              // side stream and events: k_shadow beside the next k_extend
    cudaMemPool_t pool = nullptr;      // job buffers, stream-ordered on `stream`
    JobDesc* host_jobs = nullptr;      // pinned staging of the job table
    std::chrono::steady_clock::time_point t0;
    std::vector<std::unique_ptr<DeviceScene>> scenes;
    std::vector<SceneGuide> guides;  // one per scene; networks created at the first guided wave
    int64_t scene_bytes = 0;
    std::vector<int> scene_features;  // per scene: kFeatureMedia / kFeatureTextures
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    std::deque<int64_t> queued;
    std::vector<int64_t> running;  // admission order
    std::vector<int> free_slots;
    int64_t next_id = 1;
    PlanState plan;  // rotation state of the fair-share policy
    int64_t bytes_in_use = 0;
    // device state
    DevBuf job_table, ring, wave_index, ctl;
    DevBuf slots, aov_a, aov_n, rng, q0, q1, sq, sh_o, sh_d, sorted;  // slots: kSlotRecord bytes per slot
    DevBuf mat_tex;  // per-slot textured materials, once a scene with textures is resident
    // guiding: per-slot mixtures, training records and samples, one batch
    DevBuf g_mix, g_rec, g_buf, g_count, g_wsum, g_bpos, g_bdir, g_bw;
    int64_t guide_bytes = 0;
    int capacity = 0;
    int ring_size = 0;
    int ring_pos = 0;
    WaveParams* host_ring = nullptr;   // pinned
    std::vector<cudaEvent_t> ring_ev;     // end of the wave in each ring slot
    std::vector<cudaEvent_t> ring_start;  // its start, for the device-busy time
    std::vector<char> ring_timed;         // slot holds a wave not yet added to busy_ms
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // by (bounce count, guided scene + 1 or 0)
    rth::LaunchShape shape{};
    // stats
    int64_t waves = 0, paths = 0, done = 0, submitted = 0, depth_sum = 0, guided_waves = 0, training_waves = 0;
    int max_segments = 0;
    double busy_ms = 0.0;
    // background thread
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    int worker_device = -1;  // current device of the background thread, once it runs
    bool stop = false;
    std::string bg_error;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

rt_status setup(rt_server* s) {
    SV_CUDA(cudaGetDevice(&s->device), "rt_server_create");
    SV_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "rt_server_create");
    SV_CUDA(cudaStreamCreateWithFlags(&s->dl_stream, cudaStreamNonBlocking), "rt_server_create");
    SV_CUDA(rth::create_fork(s->fork), "rt_server_create");
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = s->device;
    SV_CUDA(cudaMemPoolCreate(&s->pool, &pp), "create job memory pool");
    const int n = s->opt.max_jobs;
    SV_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s->host_jobs), size_t(n) * sizeof(JobDesc)),
            "allocate pinned job table");
    SV_CUDA(s->job_table.alloc(size_t(n) * sizeof(JobDesc)), "allocate job table");
    SV_CUDA(cudaMemset(s->job_table.ptr, 0, size_t(n) * sizeof(JobDesc)), "clear job table");
    s->ring_size = std::max(2, s->opt.waves_in_flight + 1);
    SV_CUDA(s->ring.alloc(size_t(s->ring_size) * sizeof(WaveParams)), "allocate wave ring");
    SV_CUDA(s->wave_index.alloc(sizeof(int)), "allocate wave counter");
    SV_CUDA(cudaMemset(s->wave_index.ptr, 0, sizeof(int)), "clear wave counter");
    SV_CUDA(s->ctl.alloc(sizeof(WaveCtl)), "allocate counters");
    SV_CUDA(cudaMemset(s->ctl.ptr, 0, sizeof(WaveCtl)), "clear counters");
    SV_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s->host_ring), size_t(s->ring_size) * sizeof(WaveParams)),
            "allocate pinned wave ring");
    for (int i = 0; i < s->ring_size; i++) {
        cudaEvent_t e, b;
        SV_CUDA(cudaEventCreate(&e), "create event");
        SV_CUDA(cudaEventCreate(&b), "create event");
        s->ring_ev.push_back(e);
        s->ring_start.push_back(b);
        s->ring_timed.push_back(0);
    }
    const size_t cap = size_t(s->opt.wave_paths);
    SV_CUDA(s->slots.alloc(cap * kSlotRecord), "allocate path state");
    SV_CUDA(s->aov_a.alloc(cap * sizeof(float4)), "allocate path state");
    SV_CUDA(s->aov_n.alloc(cap * sizeof(float2)), "allocate path state");
    SV_CUDA(s->rng.alloc(cap * sizeof(uint2)), "allocate path state");
    SV_CUDA(s->q0.alloc(cap * sizeof(int)), "allocate queues");
    SV_CUDA(s->q1.alloc(cap * sizeof(int)), "allocate queues");
    SV_CUDA(s->sq.alloc(cap * sizeof(int)), "allocate queues");
    SV_CUDA(s->sh_o.alloc(2 * cap * sizeof(float4)), "allocate shadow queue");
    SV_CUDA(s->sh_d.alloc(2 * cap * sizeof(float4)), "allocate shadow queue");
    SV_CUDA(s->sorted.alloc(size_t(kShadeBuckets) * cap * sizeof(int)), "allocate shade buckets");
    s->capacity = int(cap);
    for (int i = n - 1; i >= 0; i--) s->free_slots.push_back(i);
    rth::query_shape(s->shape);
    if (s->opt.hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        SV_CUDA(cudaMemGetInfo(&fr, &tot), "query device memory");
        s->opt.hbm_budget_bytes = int64_t(double(fr) * 0.8);
    }
    // freed job memory stays in the pool, up to the budget, for the next admissions
    uint64_t keep = uint64_t(s->opt.hbm_budget_bytes);
    SV_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep), "configure job memory pool");
    return RT_OK;
}

// Per-slot guiding buffers, allocated with the first guided job.
rt_status ensure_guide_buffers(rt_server* s) {
    if (s->g_mix.ptr) return RT_OK;
    const size_t cap = size_t(s->capacity);
    SV_CUDA(s->g_mix.alloc(cap * sizeof(rtg::Mixture)), "allocate guide mixtures");
    SV_CUDA(s->g_rec.alloc(size_t(rtg::kGuideRec) * 4 * cap * sizeof(float4)), "allocate guide records");
    SV_CUDA(s->g_buf.alloc(size_t(rtg::kGuideRec) * cap * 32), "allocate guide samples");
    SV_CUDA(s->g_count.alloc(sizeof(int)), "allocate guide samples");
    SV_CUDA(s->g_wsum.alloc(sizeof(float)), "allocate guide batch");
    SV_CUDA(s->g_bpos.alloc(size_t(kGuideBatch) * 12), "allocate guide batch");
    SV_CUDA(s->g_bdir.alloc(size_t(kGuideBatch) * 12), "allocate guide batch");
    SV_CUDA(s->g_bw.alloc(size_t(kGuideBatch) * 4), "allocate guide batch");
    s->guide_bytes = int64_t(s->g_mix.bytes + s->g_rec.bytes + s->g_buf.bytes + 3 * size_t(kGuideBatch) * 12);
    return RT_OK;
}

// The network of scene `k`, created at its first guided wave.
rt_status ensure_scene_guide(rt_server* s, int k) {
    SceneGuide& g = s->guides[size_t(k)];
    if (g.net) return RT_OK;
    rt_guide_options go;
    rt_guide_options_default(&go);
    go.seed = uint64_t(k) + 1;
    rt_status st = guide_create(&go, &g.net);
    if (!st) s->guide_bytes += guide_device_bytes(g.net);  // counted against the budget from now on
    return st;
}

// Wave groups (rt_schedule.h): plain jobs of scenes without media or
// textures (the plain shade kernel), plain jobs of scenes with them and the
// guided jobs of each scene (the full shade kernel).
constexpr int kGroupPlain = 0, kGroupFull = 1, kGroupGuided0 = 2;
int job_group(const rt_server* s, const rt_job_desc& d) {
    if (d.guided) return kGroupGuided0 + d.scene;
    return s->scene_features[size_t(d.scene)] != 0 ? kGroupFull : kGroupPlain;
}

// `group`: the wave's group; a guided group's wave samples the guiding
// network of its scene.
Ctx make_ctx(rt_server* s, int group) {
    const int gscene = group >= kGroupGuided0 ? group - kGroupGuided0 : -1;
    Ctx c;
    std::memset(&c, 0, sizeof(c));
    c.jobs = s->job_table.as<JobDesc>();
    WaveBufs& b = c.wb;
    b.ray_o = slot_field(s->slots.ptr, kRecRayO);
    b.ray_d = slot_field(s->slots.ptr, kRecRayD);
    b.hit = slot_field(s->slots.ptr, kRecHit);
    b.thr = slot_field(s->slots.ptr, kRecThr);
    b.rad = slot_field(s->slots.ptr, kRecRad);
    b.nee0 = slot_field(s->slots.ptr, kRecNee0);
    b.nee1 = slot_field(s->slots.ptr, kRecNee1);
    b.stale = slot_field(s->slots.ptr, kRecStale);
    b.aov_a = s->aov_a.as<float4>();
    b.aov_n = s->aov_n.as<float2>();
    b.rng = s->rng.as<uint2>();
    b.queue[0] = s->q0.as<int>();
    b.queue[1] = s->q1.as<int>();
    b.squeue = s->sq.as<int>();
    b.sh_o = s->sh_o.as<float4>();
    b.sh_d = s->sh_d.as<float4>();
    b.sorted = s->sorted.as<int>();
    b.mat_tex = s->mat_tex.ptr ? s->mat_tex.as<DevMaterial>() : nullptr;
    b.ctl = s->ctl.as<WaveCtl>();
    b.capacity = s->capacity;
    c.waves = s->ring.as<WaveParams>();
    c.wave_index = s->wave_index.as<int>();
    c.wave_ring = s->ring_size;
    c.max_depth = s->opt.max_depth;
    c.features = group == kGroupPlain ? 0 : group == kGroupFull ? kFeatureMedia | kFeatureTextures : kFeatureGuide;
    if (gscene >= 0) {
        const SceneGuide& g = s->guides[size_t(gscene)];
        c.G.mix = s->g_mix.as<rtg::Mixture>();
        c.G.prob = s->opt.guide_prob;
        c.G.min_rough = 0.3f;
        c.G.lo = g.lo;
        c.G.inv_ext = g.inv;
    }
    return c;
}

// One wave's launches: raygen, (extend, [guide inference,] shade, shadow) x
// depth, resolve, [training samples,] advance of the wave ring.
void issue_wave(rt_server* s, const Ctx& c0, int depth, int gscene, bool training) {
    Ctx c = c0;
    c.max_depth = depth;
    c.G.rec = training ? s->g_rec.as<float4>() : nullptr;
    rtg::NetView net{};
    int gsms = 0;
    if (gscene >= 0) {
        const SceneGuide& g = s->guides[size_t(gscene)];
        net = guide_view(g.net, g.lo, g.inv);
        gsms = guide_sms(g.net);
    }
    if (training) cudaMemsetAsync(s->g_count.ptr, 0, sizeof(int), s->stream);
    c.bounce = 0;
    rth::launch_raygen(c, s->stream);
    rth::launch_extend(c, s->shape, false, s->stream);
    for (int b = 0; b < depth; b++) {
        c.bounce = b;
        if (gscene >= 0) rtgh::launch_infer(c, net, gsms, s->stream);
        rth::launch_shade(c, s->shape, false, s->stream);
        if (b + 1 < depth) {  // this bounce's k_shadow beside its k_sample and the next bounce's k_extend
            rth::launch_sample_shadow_and_next_extend(c, s->shape, s->stream, &s->fork);
        } else {
            rth::launch_sample(c, s->shape, false, s->stream);
            rth::launch_shadow(c, s->shape, false, s->stream);
        }
    }
    rth::launch_resolve(c, s->stream);
    if (training)
        rtgh::launch_collect(c, s->g_buf.as<float4>(), s->g_count.as<int>(), int(s->g_buf.bytes / 32), s->stream);
    rth::launch_next_wave(c, s->stream);
}

// One captured wave per bounce count: raygen, (extend, shade, shadow) x depth,
// resolve, advance of the wave ring.  A wave uses the graph of the deepest
// job in it; each path still stops at its own job's max_depth.
rt_status wave_graph(rt_server* s, int depth, int group, cudaGraphExec_t* out) {
    const int gscene = group >= kGroupGuided0 ? group - kGroupGuided0 : -1;
    const std::pair<int, int> key(depth, group);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return RT_OK;
    }
    cudaGraph_t g = nullptr;
    SV_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin graph capture");
    issue_wave(s, make_ctx(s, group), depth, gscene, false);
    SV_CUDA(cudaStreamEndCapture(s->stream, &g), "end graph capture");
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "instantiate wave graph");
    s->graphs[key] = ge;
    *out = ge;
    return RT_OK;
}

rt_status admit(rt_server* s, Job& j) {
    const rt_job_desc& d = j.desc;
    j.npix = int64_t(d.width) * d.height;
    j.total = j.npix * d.spp;
    j.bytes = job_bytes(j.npix);
    SV_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&j.mem), size_t(j.bytes), s->pool, s->stream),
            "allocate job buffers");
    SV_CUDA(cudaEventCreateWithFlags(&j.done_ev, cudaEventDisableTiming), "create event");
    j.slot = s->free_slots.back();
    s->free_slots.pop_back();
    // A slot's staging entry is rewritten only after its previous job was
    // released, i.e. after that job's upload and waves completed.
    JobDesc& hj = s->host_jobs[j.slot];
    std::memset(&hj, 0, sizeof(hj));
    hj.sc = s->scenes[size_t(d.scene)]->view;
    hj.cam = camera_view(d.camera, d.width, d.height);
    JobParams& p = hj.job;
    p.width = d.width;
    p.height = d.height;
    p.spp = d.spp;
    p.max_depth = d.max_depth;
    p.filter = d.filter;
    p.rng = RT_RNG_PCG32;
    p.rr_depth = d.rr_depth;
    p.frame = 0;
    p.seed = d.seed;
    p.npix = j.npix;
    p.tonemap = d.tonemap;
    p.exposure = d.exposure;
    p.acc_color = j.f4(0);
    p.acc_albedo = j.f4(1);
    p.acc_normal = j.f4(2);
    p.color = j.f4(3);
    p.albedo = j.f4(4);
    p.normal = j.f4(5);
    p.lcg_state = j.u32(0);
    p.rgba8 = j.u32(1);
    JobDesc* dj = s->job_table.as<JobDesc>() + j.slot;
    SV_CUDA(cudaMemcpyAsync(dj, &hj, sizeof(hj), cudaMemcpyHostToDevice, s->stream), "upload job");
    rth::launch_begin_n(dj, j.npix, s->stream);
    j.state = RT_JOB_RUNNING;
    j.admit_ms = s->now_ms();
    s->bytes_in_use += j.bytes;
    return RT_OK;
}

// Adds the device time of every finished wave not yet counted.
void account_busy(rt_server* s) {
    for (size_t i = 0; i < s->ring_ev.size(); i++) {
        if (!s->ring_timed[i] || cudaEventQuery(s->ring_ev[i]) != cudaSuccess) continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, s->ring_start[i], s->ring_ev[i]) == cudaSuccess) s->busy_ms += double(ms);
        s->ring_timed[i] = 0;
    }
}

void free_job(rt_server* s, Job& j) {
    if (j.mem) cudaFreeAsync(j.mem, s->stream);  // after every wave issued so far
    j.mem = nullptr;
    if (j.done_ev) cudaEventDestroy(j.done_ev);
    j.done_ev = nullptr;
    if (j.slot >= 0) s->free_slots.push_back(j.slot);
    j.slot = -1;
    s->bytes_in_use -= j.bytes;
    j.bytes = 0;
}

// One scheduling step with the lock held.  When the next slot of the wave
// ring is still read by a queued wave, nothing is issued and *blocked names
// the event to wait for (outside the lock).
rt_status step_locked(rt_server* s, int32_t* did_work, cudaEvent_t* blocked) {
    int work = 0;
    *blocked = nullptr;
    // retire finished jobs
    for (size_t i = 0; i < s->running.size();) {
        Job& j = *s->jobs[s->running[i]];
        if (j.finalize_issued && cudaEventQuery(j.done_ev) == cudaSuccess) {
            j.state = RT_JOB_DONE;
            j.done_ms = s->now_ms();
            s->done++;
            s->running.erase(s->running.begin() + long(i));
            work = 1;
        } else {
            i++;
        }
    }
    // admission in arrival order by memory budget and free slots (a finished
    // job holds its memory and slot until it is released)
    while (!s->queued.empty() && !s->free_slots.empty()) {
        Job& j = *s->jobs[s->queued.front()];
        int64_t need = job_bytes(int64_t(j.desc.width) * j.desc.height);
        if (s->bytes_in_use + s->scene_bytes + s->guide_bytes + need > s->opt.hbm_budget_bytes) break;
        s->queued.pop_front();
        rt_status st = admit(s, j);
        if (st) {
            j.state = RT_JOB_FAILED;
            free_job(s, j);
            return st;
        }
        s->running.push_back(j.id);
        work = 1;
    }
    // fill a wave from the running jobs
    if (cudaEventQuery(s->ring_ev[size_t(s->ring_pos)]) == cudaErrorNotReady) {
        *blocked = s->ring_ev[size_t(s->ring_pos)];
        if (did_work) *did_work = 1;
        return RT_OK;
    }
    account_busy(s);
    // The group this wave serves and the paths each of its jobs gets
    // (rt_schedule.h).
    std::vector<Job*> active;
    std::vector<PlanJob> pj;
    for (int64_t id : s->running) {
        Job& j = *s->jobs[id];
        if (j.issued < j.total) {
            active.push_back(&j);
            pj.push_back({j.total - j.issued, job_group(s, j.desc)});
        }
    }
    std::vector<std::pair<Job*, int64_t>> plan;
    for (const auto& seg : plan_wave(pj, s->opt.policy, s->capacity, kMaxSegments, s->plan))
        plan.emplace_back(active[seg.first], seg.second);
    WaveParams wp;
    std::memset(&wp, 0, sizeof(wp));
    int filled = 0, depth = 1;
    const int group = plan.empty() ? kGroupPlain : job_group(s, plan.front().first->desc);
    const int gscene = group >= kGroupGuided0 ? group - kGroupGuided0 : -1;
    std::vector<Job*> completing;
    for (auto& pj : plan) {
        Job& j = *pj.first;
        Segment& g = wp.seg[wp.num_seg++];
        g.job = j.slot;
        g.slot_begin = filled;
        g.count = int(pj.second);
        g.path_begin = j.issued;
        j.issued += pj.second;
        filled += int(pj.second);
        depth = std::max(depth, j.desc.max_depth);
        if (j.issued >= j.total) completing.push_back(&j);
    }
    if (filled > 0) {
        wp.wave_count = filled;
        bool training = false;
        if (gscene >= 0) {
            rt_status gs = ensure_guide_buffers(s);
            if (!gs) gs = ensure_scene_guide(s, gscene);
            if (gs) return gs;
            training = s->guides[size_t(gscene)].train_waves < s->opt.guide_train_waves;
        }
        cudaGraphExec_t graph = nullptr;
        if (!training) {
            rt_status gs = wave_graph(s, depth, group, &graph);
            if (gs) return gs;
        }
        int pos = s->ring_pos;
        SV_CUDA(cudaEventRecord(s->ring_start[size_t(pos)], s->stream), "record event");
        s->host_ring[pos] = wp;
        SV_CUDA(cudaMemcpyAsync(s->ring.as<WaveParams>() + pos, &s->host_ring[pos], sizeof(WaveParams),
                                cudaMemcpyHostToDevice, s->stream),
                "upload wave");
        if (training) {
            // launched directly: the wave records training samples, then the
            // scene's network takes guide_steps Adam steps on batches of them
            SceneGuide& g = s->guides[size_t(gscene)];
            issue_wave(s, make_ctx(s, group), depth, gscene, true);
            for (int k = 0; k < s->opt.guide_steps; k++) {
                SV_CUDA(cudaMemsetAsync(s->g_wsum.ptr, 0, sizeof(float), s->stream), "guide batch");
                rtgh::launch_batch(s->g_buf.as<float4>(), s->g_count.as<int>(), int(s->g_buf.bytes / 32),
                                   kGuideBatch, g.seed++ * 0x9E3779B9u, s->g_bpos.as<float>(), s->g_bdir.as<float>(),
                                   s->g_bw.as<float>(), s->g_wsum.as<float>(), s->stream);
                rt_status ts = guide_train_device(g.net, s->g_bpos.as<float>(), s->g_bdir.as<float>(),
                                                  s->g_bw.as<float>(), kGuideBatch, 1.0f, s->g_wsum.as<float>(),
                                                  s->stream);
                if (ts) return ts;
            }
            g.train_waves++;
            s->training_waves++;
            SV_CUDA(cudaGetLastError(), "launch training wave");
        } else {
            SV_CUDA(cudaGraphLaunch(graph, s->stream), "launch wave");
        }
        if (gscene >= 0) s->guided_waves++;
        SV_CUDA(cudaEventRecord(s->ring_ev[size_t(pos)], s->stream), "record event");
        s->ring_timed[size_t(pos)] = 1;
        s->ring_pos = (pos + 1) % s->ring_size;
        s->waves++;
        s->depth_sum += depth;
        s->paths += filled;
        s->max_segments = std::max(s->max_segments, wp.num_seg);
        for (Job* j : completing) {
            JobDesc* dj = s->job_table.as<JobDesc>() + j->slot;
            rth::launch_finalize_n(dj, j->npix, s->stream);
            SV_CUDA(cudaEventRecord(j->done_ev, s->stream), "record event");
            j->finalize_issued = true;
        }
        work = 1;
    } else if (!s->running.empty()) {
        work = 1;  // waiting for finalize events
    }
    if (did_work) *did_work = work;
    return RT_OK;
}

void worker_loop(rt_server* s) {
    // A new thread starts on device 0: the events, graphs and launches below
    // belong to the device the server was created on.
    cudaError_t de = cudaSetDevice(s->device);
    int dev = -1;
    if (de == cudaSuccess) de = cudaGetDevice(&dev);
    std::unique_lock<std::mutex> lk(s->mu);
    s->worker_device = dev;
    if (de != cudaSuccess) {  // every job fails with the reason
        s->bg_error = std::string("background thread: cudaSetDevice failed: ") + cudaGetErrorString(de);
        while (!s->stop) {
            for (int64_t id : s->queued) s->jobs[id]->state = RT_JOB_FAILED;
            s->queued.clear();
            s->cv.notify_all();
            s->cv.wait(lk);
        }
        return;
    }
    while (!s->stop) {
        if (s->queued.empty() && s->running.empty()) {
            s->cv.wait(lk);
            continue;
        }
        int32_t w = 0;
        cudaEvent_t blocked = nullptr;
        rt_status st = step_locked(s, &w, &blocked);
        if (blocked) {
            lk.unlock();
            cudaEventSynchronize(blocked);
            lk.lock();
            continue;
        }
        if (st) {
            s->bg_error = g_error;
            for (int64_t id : s->running) s->jobs[id]->state = RT_JOB_FAILED;
            s->running.clear();
        }
        bool waiting_only = true;
        for (int64_t id : s->running)
            if (s->jobs[id]->issued < s->jobs[id]->total) waiting_only = false;
        s->cv.notify_all();
        if (waiting_only && s->queued.empty()) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        }
    }
}

void fill_status(const rt_server* s, const Job& j, rt_job_status* st) {
    std::memset(st, 0, sizeof(*st));
    st->state = j.state;
    st->submit_ms = j.submit_ms;
    st->admit_ms = j.admit_ms;
    st->done_ms = j.done_ms;
    st->paths = j.total ? j.total : int64_t(j.desc.width) * j.desc.height * j.desc.spp;
    st->bytes = j.bytes;
    (void)s;
}

}  // namespace

extern "C" {

void rt_server_options_default(rt_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->wave_paths = 1 << 23;
    o->max_jobs = 256;
    o->max_depth = 32;
    o->background = 1;
    o->waves_in_flight = 2;
    o->guide_train_waves = 32;
    o->guide_steps = 4;
    o->guide_prob = 0.5f;
}

rt_status rt_server_create(const rt_server_options* o, rt_server** out) {
    if (!out) return fail(RT_ERR_INVALID_ARG, "rt_server_create: out is NULL");
    rt_server* s = new (std::nothrow) rt_server();
    if (!s) return fail(RT_ERR_OUT_OF_MEMORY, "rt_server_create: out of host memory");
    rt_server_options_default(&s->opt);
    if (o) {
        s->opt = *o;
        if (s->opt.wave_paths <= 0) s->opt.wave_paths = 1 << 23;
        if (s->opt.max_jobs <= 0) s->opt.max_jobs = 256;
        if (s->opt.max_depth <= 0) s->opt.max_depth = 32;
        if (s->opt.waves_in_flight <= 0) s->opt.waves_in_flight = 2;
        if (s->opt.guide_train_waves <= 0) s->opt.guide_train_waves = 32;
        if (s->opt.guide_steps <= 0) s->opt.guide_steps = 4;
        if (s->opt.guide_prob == 0.0f) s->opt.guide_prob = 0.5f;
    }
    if (!(s->opt.guide_prob > 0.0f && s->opt.guide_prob <= 1.0f)) {
        delete s;
        return fail(RT_ERR_INVALID_ARG, "rt_server_create: guide_prob must be in (0, 1]");
    }
    if (s->opt.policy != RT_SERVE_FAIR && s->opt.policy != RT_SERVE_FIFO && s->opt.policy != RT_SERVE_SRPT) {
        delete s;
        return fail(RT_ERR_INVALID_ARG, "rt_server_create: unknown policy");
    }
    if (s->opt.max_jobs > 256 || s->opt.wave_paths > (1 << 26)) {
        delete s;
        return fail(RT_ERR_INVALID_ARG, "rt_server_create: max_jobs <= 256 and wave_paths <= 2^26");
    }
    s->t0 = std::chrono::steady_clock::now();
    rt_status st = setup(s);
    if (st) {
        rt_server_destroy(s);
        return st;
    }
    if (s->opt.background) s->worker = std::thread(worker_loop, s);
    *out = s;
    return RT_OK;
}

rt_status rt_server_destroy(rt_server* s) {
    if (!s) return RT_OK;
    SV_ON_DEVICE(s, "rt_server_destroy");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& kv : s->jobs) free_job(s, *kv.second);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    for (SceneGuide& g : s->guides)
        if (g.net) rt_guide_destroy(g.net);
    for (cudaEvent_t e : s->ring_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : s->ring_start) cudaEventDestroy(e);
    if (s->host_ring) cudaFreeHost(s->host_ring);
    if (s->host_jobs) cudaFreeHost(s->host_jobs);
    if (s->fork.side) cudaStreamSynchronize(s->fork.side);
    rth::destroy_fork(s->fork);
    if (s->dl_stream) cudaStreamDestroy(s->dl_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return RT_OK;
}

rt_status rt_server_add_scene(rt_server* s, const rt_scene* scene, int32_t* id) {
    if (!s || !scene) return fail(RT_ERR_INVALID_ARG, "rt_server_add_scene: NULL argument");
    SV_ON_DEVICE(s, "rt_server_add_scene");
    std::lock_guard<std::mutex> lk(s->mu);
    std::unique_ptr<DeviceScene> ds(new DeviceScene());
    rt_status st = upload_scene(*scene, *ds, s->stream);
    if (st) return st;
    if (ds->view.num_tex > 0 && !s->mat_tex.ptr) {
        SV_CUDA(cudaStreamSynchronize(s->stream), "rt_server_add_scene");
        SV_CUDA(s->mat_tex.alloc(size_t(s->capacity) * sizeof(DevMaterial)), "allocate textured materials");
        for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);  // captured without the buffer
        s->graphs.clear();
    }
    s->scene_features.push_back((ds->view.num_media > 0 ? kFeatureMedia : 0) |
                                (ds->view.num_tex > 0 ? kFeatureTextures : 0));
    s->scene_bytes += int64_t(ds->bytes);
    s->scenes.push_back(std::move(ds));
    SceneGuide g;
    for (int a = 0; a < 3; a++) {  // 1% margin around the scene bounds
        const float ext = std::max(scene->hi[a] - scene->lo[a], 1e-6f);
        (&g.lo.x)[a] = scene->lo[a] - 0.01f * ext;
        (&g.inv.x)[a] = 1.0f / (1.02f * ext);
    }
    s->guides.push_back(g);
    if (id) *id = int32_t(s->scenes.size()) - 1;
    return RT_OK;
}

rt_status rt_server_submit(rt_server* s, const rt_job_desc* d, int64_t* id) {
    if (!s || !d) return fail(RT_ERR_INVALID_ARG, "rt_server_submit: NULL argument");
    SV_ON_DEVICE(s, "rt_server_submit");
    std::lock_guard<std::mutex> lk(s->mu);
    if (d->scene < 0 || d->scene >= int(s->scenes.size())) return fail(RT_ERR_INVALID_ARG, "rt_server_submit: unknown scene");
    if (d->width <= 0 || d->height <= 0 || d->spp <= 0 || d->max_depth <= 0 || d->max_depth > s->opt.max_depth)
        return fail(RT_ERR_INVALID_ARG, "rt_server_submit: bad size, spp or max_depth (<= the server's max_depth)");
    if (d->guided) {  // the per-slot guiding buffers count against the budget from the first guided job on
        rt_status gs = ensure_guide_buffers(s);
        if (gs) return gs;
    }
    if (job_bytes(int64_t(d->width) * d->height) + s->scene_bytes + s->guide_bytes > s->opt.hbm_budget_bytes)
        return fail(RT_ERR_OUT_OF_MEMORY, "rt_server_submit: the job alone exceeds the memory budget");
    std::unique_ptr<Job> j(new Job());
    j->id = s->next_id++;
    j->desc = *d;
    j->submit_ms = s->now_ms();
    int64_t jid = j->id;
    s->jobs[jid] = std::move(j);
    s->queued.push_back(jid);
    s->submitted++;
    if (id) *id = jid;
    s->cv.notify_all();
    return RT_OK;
}

rt_status rt_server_cancel(rt_server* s, int64_t id) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_server_cancel: NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(RT_ERR_INVALID_ARG, "rt_server_cancel: unknown job");
    Job& j = *it->second;
    if (j.state != RT_JOB_QUEUED) return fail(RT_ERR_STATE, "rt_server_cancel: only queued jobs can be cancelled");
    s->queued.erase(std::find(s->queued.begin(), s->queued.end(), id));
    j.state = RT_JOB_CANCELLED;
    return RT_OK;
}

rt_status rt_server_poll(rt_server* s, int64_t id, rt_job_status* st) {
    if (!s || !st) return fail(RT_ERR_INVALID_ARG, "rt_server_poll: NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(RT_ERR_INVALID_ARG, "rt_server_poll: unknown job");
    fill_status(s, *it->second, st);
    return RT_OK;
}

rt_status rt_server_wait(rt_server* s, int64_t id, double timeout_ms, rt_job_status* st) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_server_wait: NULL server");
    SV_ON_DEVICE(s, "rt_server_wait");
    const auto t_end = std::chrono::steady_clock::now() + std::chrono::microseconds(int64_t(timeout_ms * 1000.0));
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        auto it = s->jobs.find(id);
        if (it == s->jobs.end()) return fail(RT_ERR_INVALID_ARG, "rt_server_wait: unknown job");
        Job& j = *it->second;
        if (j.state == RT_JOB_DONE || j.state == RT_JOB_FAILED || j.state == RT_JOB_CANCELLED) {
            if (st) fill_status(s, j, st);
            if (j.state == RT_JOB_FAILED) return fail(RT_ERR_CUDA, "job failed: " + s->bg_error);
            return RT_OK;
        }
        if (timeout_ms >= 0 && std::chrono::steady_clock::now() >= t_end)
            return fail(RT_ERR_TIMEOUT, "rt_server_wait: timed out");
        if (!s->opt.background) {  // manual mode: the caller's thread drives the loop
            int32_t w = 0;
            cudaEvent_t blocked = nullptr;
            rt_status e = step_locked(s, &w, &blocked);
            if (e) return e;
            if (blocked) SV_CUDA(cudaEventSynchronize(blocked), "rt_server_wait");
            if (!w)
                return fail(RT_ERR_STATE, "rt_server_wait: the job can make no progress (memory budget or job slots "
                                          "held by finished jobs that were not released)");
        } else if (timeout_ms >= 0) {
            s->cv.wait_until(lk, t_end);
        } else {
            s->cv.wait(lk);
        }
    }
}

static rt_status download_job(rt_server* s, int64_t id, void* dst, bool rgba8) {
    if (!s || !dst) return fail(RT_ERR_INVALID_ARG, "rt_server_download: NULL argument");
    SV_ON_DEVICE(s, "rt_server_download");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(RT_ERR_INVALID_ARG, "rt_server_download: unknown job");
    Job& j = *it->second;
    if (j.state != RT_JOB_DONE) return fail(RT_ERR_STATE, "rt_server_download: job not done");
    if (!j.mem) return fail(RT_ERR_STATE, "rt_server_download: job released");
    // the job's finalize has completed (its event did), so the copy need not
    // wait behind the waves queued on the server stream
    const void* src = rgba8 ? static_cast<const void*>(j.u32(1)) : static_cast<const void*>(j.f4(3));
    SV_CUDA(cudaMemcpyAsync(dst, src, size_t(j.npix) * (rgba8 ? 4 : 16), cudaMemcpyDeviceToHost, s->dl_stream),
            "rt_server_download");
    SV_CUDA(cudaStreamSynchronize(s->dl_stream), "rt_server_download");
    return RT_OK;
}

rt_status rt_server_download(rt_server* s, int64_t id, float* rgba) { return download_job(s, id, rgba, false); }

rt_status rt_server_download_rgba8(rt_server* s, int64_t id, uint32_t* pixels) {
    return download_job(s, id, pixels, true);
}

rt_status rt_server_release(rt_server* s, int64_t id) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_server_release: NULL server");
    SV_ON_DEVICE(s, "rt_server_release");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(RT_ERR_INVALID_ARG, "rt_server_release: unknown job");
    Job& j = *it->second;
    if (j.state == RT_JOB_RUNNING) return fail(RT_ERR_STATE, "rt_server_release: job still running");
    if (j.state == RT_JOB_QUEUED) s->queued.erase(std::find(s->queued.begin(), s->queued.end(), id));
    free_job(s, j);
    s->jobs.erase(it);
    s->cv.notify_all();
    return RT_OK;
}

rt_status rt_server_step(rt_server* s, int32_t* did_work) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_server_step: NULL server");
    if (s->opt.background) return fail(RT_ERR_STATE, "rt_server_step: server runs in the background");
    SV_ON_DEVICE(s, "rt_server_step");
    std::lock_guard<std::mutex> lk(s->mu);
    cudaEvent_t blocked = nullptr;
    rt_status st = step_locked(s, did_work, &blocked);
    if (st) return st;
    if (blocked) SV_CUDA(cudaEventSynchronize(blocked), "rt_server_step");
    return RT_OK;
}

rt_status rt_server_get_stats(rt_server* s, rt_server_stats* st) {
    if (!s || !st) return fail(RT_ERR_INVALID_ARG, "rt_server_get_stats: NULL argument");
    SV_ON_DEVICE(s, "rt_server_get_stats");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->jobs_submitted = s->submitted;
    st->jobs_done = s->done;
    st->jobs_queued = int64_t(s->queued.size());
    st->jobs_running = int64_t(s->running.size());
    st->waves = s->waves;
    st->paths = s->paths;
    st->bytes_in_use = s->bytes_in_use + s->scene_bytes + s->guide_bytes;
    st->bytes_budget = s->opt.hbm_budget_bytes;
    st->max_segments_in_a_wave = s->max_segments;
    account_busy(s);
    st->busy_ms = s->busy_ms;
    st->mean_wave_depth = s->waves ? double(s->depth_sum) / double(s->waves) : 0.0;
    st->guided_waves = s->guided_waves;
    st->training_waves = s->training_waves;
    st->device = s->device;
    st->worker_device = s->opt.background ? s->worker_device : -1;
    return RT_OK;
}

}  // extern "C"
