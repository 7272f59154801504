// rt_kernels.cu - wavefront path-tracing kernels for sm_100a.
//
// The per-path control flow is the reference integrator
// (core/cuda/devicePrograms.cu:170-532) cut at its optixTrace calls:
//   raygen   devicePrograms.cu:220-253  camera ray, filter jitter, RNG state
//   extend   devicePrograms.cu:258-269  closest hit through the wide BVH
//   shade    devicePrograms.cu:71-132, 148-159, 270-497  hit attributes,
//            analytic-light test, media, emission, NEE (shadow rays are queued
//            with their contribution), BSDF sampling, Russian roulette
//   shadow   devicePrograms.cu:303-319, 389-405, 437-453  any-hit; an occluded
//            ray zeroes its pending contribution
//   resolve  devicePrograms.cu:499-516  NaN handling and per-pixel sums
//   finalize devicePrograms.cu:518-531 + PostProcessing.cu:26-48
// Pending NEE contributions are folded into the path radiance at the start of
// the next shade (or in resolve) in the reference's order: environment, then
// light.  extend/shade/shadow are persistent kernels: each warp takes 32
// queue entries at a time with one atomicAdd.
#include <algorithm>
#include <cstdio>

#include "rt_kernels.cuh"
#include "rt_media.cuh"
#include "rt_shading.cuh"
#include "rt_traverse.cuh"

namespace rtd {

constexpr int kBlock = 128;
static_assert(kBlock == kTravBlock, "the traversal stack is laid out for this block size");
// 8 resident blocks per SM (64 registers) beat 6 (80 registers) by 11%.
constexpr int kTravMinBlocks = 8;
constexpr int kStaleTextured = 1 << 30;  // stale.w flag: the slot's mat_tex holds the last hit's material


RT_D int warp_fetch(int* counter, int lane) {
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, 32);
    return __shfl_sync(0xffffffffu, base, 0);
}

// Appends `flag` lanes of a converged warp to a queue; returns the position.
RT_D int warp_append(int* counter, bool flag, int lane) {
    unsigned m = __ballot_sync(0xffffffffu, flag);
    if (m == 0) return -1;
    int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return flag ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

RT_D void warp_stat(unsigned long long* dst, unsigned v) {
    unsigned long long x = v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(dst, x);
}

// ------------------------------------------------------------------ begin
__global__ void k_begin(const JobDesc* __restrict__ jd) {
    const JobParams& j = jd->job;
    int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= j.npix) return;
    j.acc_color[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    j.acc_albedo[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    j.acc_normal[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (j.rng == RT_RNG_LCG) j.lcg_state[p] = lcg_seed(uint32_t(p), uint32_t(j.frame));  // devicePrograms.cu:179-180
}

// ------------------------------------------------------------------ raygen
// The camera ray of the path in `slot` (devicePrograms.cu:178-180, 214-227): its slot
// record goes to `rec`, its random state and queue entry to their arrays.
RT_D void raygen_slot(const Ctx& c, const WaveParams& W, int slot, float4* rec) {
    const WaveBufs& b = c.wb;
    const Segment sg = W.seg[find_segment(W, slot)];
    const JobDesc* jd = c.jobs + sg.job;
    const JobParams& j = jd->job;
    const CameraView& cam = jd->cam;
    int64_t p = sg.path_begin + (slot - sg.slot_begin);
    int pix = int(p % j.npix);
    int ix = pix % j.width, iy = pix / j.width;
    Rng rng;
    if (j.rng == RT_RNG_LCG) {
        rng.inc = 0;
        rng.state = j.lcg_state[pix];
    } else {
        rng.inc = pcg_inc(uint64_t(p));
        rng.state = pcg_seed(pcg_frame_state(j.seed, j.frame), uint64_t(p));
    }
    float u0 = rng.next(), u1 = rng.next();
    float jx, jy;
    filter_jitter(j.filter, u0, u1, jx, jy);
    float sx = (float(ix) + 0.5f + jx) / float(j.width);
    float sy = (float(iy) + 0.5f + jy) / float(j.height);
    v3 dir = normalize(ld3(cam.dir) + (sx - 0.5f) * ld3(cam.hor) + (sy - 0.5f) * ld3(cam.ver));
    rec[kRecRayO / 16] = f4(ld3(cam.pos), 0.0f);
    rec[kRecRayD / 16] = f4(dir, 0.0f);
    rec[kRecHit / 16] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    rec[kRecThr / 16] = make_float4(1.f, 1.f, 1.f, 0.f);
    rec[kRecRad / 16] = make_float4(0.f, 0.f, 0.f, 0.f);
    rec[kRecNee0 / 16] = make_float4(0.f, 0.f, 0.f, 0.f);
    rec[kRecNee1 / 16] = make_float4(0.f, 0.f, 0.f, 0.f);
    rec[kRecStale / 16] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    b.rng[slot] = make_uint2(uint32_t(rng.state), uint32_t(rng.state >> 32));
    b.queue[0][slot] = slot;
    if (c.G.rec != nullptr)
        for (int r = 0; r < rtg::kGuideRec; r++)
            c.G.rec[(size_t(r) * 4 + 1) * size_t(b.capacity) + slot] = make_float4(0.f, 0.f, 0.f, 0.f);
}

constexpr int kRaygenBlock = 256;
constexpr int kRecF4 = int(kSlotRecord / 16);  // float4s per slot record
constexpr int kStagePad = kRecF4 + 1;          // per staged record: the 16-byte stores of a warp hit distinct banks
__global__ void __launch_bounds__(kRaygenBlock) k_raygen(Ctx c) {
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    WaveCtl* ctl = c.wb.ctl;
    const WaveParams& W = wave_of(c);
    if (slot == 0) {
        ctl->count[0] = W.wave_count;
        ctl->count[1] = 0;
        ctl->shadow_count[0] = 0;
        ctl->shadow_count[1] = 0;
        ctl->fetch_ext = 0;
        ctl->fetch_shade = 0;
        ctl->fetch_shadow = 0;
        ctl->sample_count = 0;
        ctl->fetch_sample = 0;
        for (int b = 0; b < kShadeBuckets; b++) ctl->bucket[b] = 0;
    }
    // A warp's 32 slot records are 4 KB of contiguous memory: they are built
    // in shared memory and stored as 16-byte pieces by consecutive lanes, so
    // that every store instruction writes whole lines.
    __shared__ float4 stage[kRaygenBlock / 32][32 * kStagePad];
    const int lane = threadIdx.x & 31;
    const int slot0 = slot - lane;
    if (slot0 >= W.wave_count) return;  // the whole warp
    float4* st = stage[threadIdx.x >> 5];
    if (slot < W.wave_count) raygen_slot(c, W, slot, st + lane * kStagePad);
    __syncwarp();
    float4* dst = reinterpret_cast<float4*>(c.wb.ray_o.base - kRecRayO) + size_t(slot0) * kRecF4;
#pragma unroll
    for (int k = 0; k < kRecF4; k++) {
        const int idx = k * 32 + lane;  // float4 index in the warp's records
        const int r = idx / kRecF4;
        if (slot0 + r < W.wave_count) dst[idx] = st[r * kStagePad + idx % kRecF4];
    }
}

// ------------------------------------------------------------------ extend
struct ExtendSrc {
    const Ctx* c;
    const int* q;
    RT_D void load(int i, TravRay& r, const SceneView*& sc) {
        int slot = q[i];
        const WaveParams& W = wave_of(*c);
        sc = &c->jobs[W.seg[find_segment(W, slot)].job].sc;
        float4 o = c->wb.ray_o[slot], d = c->wb.ray_d[slot];
        r.o = xyz(o);
        r.d = xyz(d);
        r.tmin = kEps;
        r.tmax = FLT_MAX;
    }
    // Stores the hit and, when the shade queue is sorted, appends the slot to
    // the bucket of the hit surface's material type (tri_v[1].w of the
    // triangle) with one atomicAdd per bucket present in the warp.
    RT_D void finish(bool fin, int i, int tri, float t, float b1, float b2, const float4* tri_v) {
        int slot = fin ? q[i] : 0;
        if (fin) c->wb.hit[slot] = make_float4(tri >= 0 ? t : FLT_MAX, b1, b2, __int_as_float(tri));
        int* sorted = c->wb.sorted;
        if (sorted == nullptr || __ballot_sync(0xffffffffu, fin) == 0u) return;
        int key = -1;
        if (fin) key = tri >= 0 ? __float_as_int(__ldg(reinterpret_cast<const float*>(tri_v + size_t(tri) * 3 + 1) + 3))
                                : kMissBucket;
        const int lane = threadIdx.x & 31;
        unsigned peers = __match_any_sync(0xffffffffu, key);
        int leader = __ffs(peers) - 1;
        int base = 0;
        if (fin && lane == leader) base = atomicAdd(&c->wb.ctl->bucket[key], __popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (fin) sorted[size_t(key) * size_t(c->wb.capacity) + size_t(base + __popc(peers & ((1u << lane) - 1u)))] = slot;
    }
};

template <bool Stats>
__global__ void __launch_bounds__(kBlock, kTravMinBlocks) k_extend(Ctx c) {
    WaveCtl* ctl = c.wb.ctl;
    const int cur = c.bounce & 1, nxt = cur ^ 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->count[nxt] = 0;
        ctl->fetch_shade = 0;
        ctl->sample_count = 0;
        ctl->fetch_sample = 0;
    }
    const int total = ctl->count[cur];
    uint32_t nodes = 0, tris = 0, rays = 0, overflows = 0;
    ExtendSrc src{&c, c.wb.queue[cur]};
    traverse_queue<false, Stats>(src, &ctl->fetch_ext, total, nodes, tris, rays, overflows);
    if (overflows) atomicAdd(&ctl->overflow, int(overflows));
    if (Stats) {
        warp_stat(&ctl->stats[0], rays);
        warp_stat(&ctl->stats[2], nodes);
        warp_stat(&ctl->stats[3], tris);
    }
}

// lightTrace, devicePrograms.cu:192-211: the nearest analytic light closer
// than `closest`; `lpdf` ends as the pdf of the last light evaluated.
RT_D bool light_trace(const SceneView& sc, v3 o, v3 d, float& closest, v3& lrad, float& lpdf, int& medium) {
    bool hit = false;
    for (int i = 0; i < sc.num_lights; i++) {
        LightParams l = load_light(sc.lights + i);
        float ld = 0.0f;
        v3 Li = evaluate_light(l, o, d, closest, lpdf, ld);
        if (lpdf == 0.0f) continue;
        hit = true;
        lrad = Li;
        closest = ld;
        medium = l.medium;
    }
    return hit;
}

RT_D bool nee_pdf_ok(float p) { return p > 0.0f && p < FLT_MAX; }

// SampleMediumDistance (Medium.h:233-244) for either medium type.
template <class RNG>
RT_D bool medium_sample(const DevMedium* mp, const MedParams& med, v3 o, v3 d, float maxd, float& dist, float& tp,
                        v3& tr, RNG& rng, int& budget_hits) {
    if (med.type == RT_MEDIUM_GRID) {
        tp = 1.0f;
        return grid_sample_distance(load_grid(mp), o, d, maxd, rng, dist, tr, budget_hits);
    }
    return sample_medium_distance(med, maxd, dist, tp, tr, rng);
}
// EvaluateMediumDistance(medium, false, ...) (Medium.h:222-231): the
// transmittance of a next-event segment; ratio tracking for a grid.
template <class RNG>
RT_D v3 medium_transmittance(const DevMedium* mp, const MedParams& med, v3 o, v3 d, float dist, float& tp, RNG& rng,
                             int& budget_hits) {
    if (med.type == RT_MEDIUM_GRID) {
        tp = 1.0f;
        return v3(grid_transmittance(load_grid(mp), o, d, dist, rng, budget_hits));
    }
    return eval_medium_distance(med, false, dist, tp);
}

// ------------------------------------------------------------------ shade
// Full = false compiles the kernel without the participating-media,
// path-guiding and material-texture branches, for waves whose scenes have
// none of them (the host picks it from Ctx::features): those branches set
// the register budget of the whole kernel, so the common path runs at a
// lower occupancy when they are compiled in.
template <bool Stats, bool Full>
__global__ void __launch_bounds__(kBlock) k_shade(Ctx c) {
    WaveCtl* ctl = c.wb.ctl;
    const int cur = c.bounce & 1, nxt = cur ^ 1;
    const int bounce = c.bounce;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->fetch_shadow = 0;
        ctl->fetch_ext = 0;
    }
    const int total = ctl->count[cur];
    const int* __restrict__ q = c.wb.queue[cur];
    const WaveBufs& B = c.wb;
    const WaveParams& W = wave_of(c);
    const int lane = threadIdx.x & 31;
    uint32_t nan_paths = 0;
    int budget_hits = 0;  // media walks that ran out of steps (reported as a watchdog error)
    // Sorted queue: item i lies in the bucket whose prefix range holds it.
    __shared__ int prefix[kShadeBuckets + 1];
    const bool sorted = B.sorted != nullptr;
    if (sorted && threadIdx.x == 0) {
        int acc = 0;
        for (int b = 0; b < kShadeBuckets; b++) {
            prefix[b] = acc;
            acc += ctl->bucket[b];
        }
        prefix[kShadeBuckets] = acc;
    }
    __syncthreads();
    while (true) {
        int base = warp_fetch(&ctl->fetch_shade, lane);
        if (base >= total) break;
        int i = base + lane;
        bool cont = false, defer = false;
        bool sh0 = false, sh1 = false;
        int slot = 0;
        v3 s0o, s0d, s1o, s1d;
        float s0t = 0.f, s1t = 0.f;
        if (i < total) {
            if (sorted) {
                int b = 0;
                while (b < kShadeBuckets - 1 && i >= prefix[b + 1]) b++;
                slot = B.sorted[size_t(b) * size_t(B.capacity) + size_t(i - prefix[b])];
            } else {
                slot = q[i];
            }
            const Segment& sgm = W.seg[find_segment(W, slot)];
            const JobDesc* jd = c.jobs + sgm.job;
            const SceneView& sc = jd->sc;
            const JobParams& jp = jd->job;
            float4 o4 = B.ray_o[slot], d4 = B.ray_d[slot], th = B.thr[slot], h4 = B.hit[slot];
            float4 r4 = B.rad[slot];
            float4 n0 = B.nee0[slot], n1 = B.nee1[slot];
            uint2 rs = B.rng[slot];
            Rng rng;
            rng.state = uint64_t(rs.x) | (uint64_t(rs.y) << 32);
            if (jp.rng == RT_RNG_LCG) {
                rng.inc = 0;
            } else {
                rng.inc = pcg_inc(uint64_t(sgm.path_begin + (slot - sgm.slot_begin)));
            }
            v3 o = xyz(o4), d = xyz(d4);
            v3 history = xyz(th);
            float pre_pdf = th.w;
            v3 radiance = xyz(r4);
            radiance += xyz(n0);
            radiance += xyz(n1);
            const rtg::GuideCtx& G = c.G;
            const size_t cap = size_t(B.capacity);
            if (Full && G.rec != nullptr && bounce >= 1 && bounce - 1 < rtg::kGuideRec)  // radiance before the next vertex
                G.rec[(size_t(bounce - 1) * 4 + 3) * cap + slot] = f4(radiance, 0.0f);
            v3 V = -d, L = d;
            float gp = 0.0f;  // probability of sampling the guiding mixture at this vertex
            float rec_pdf = 0.0f, rec_cos = 0.0f;
            float3 gin = make_float3(0.f, 0.f, 0.f);  // network input of this vertex
            // ---- closest hit / miss programs (devicePrograms.cu:71-132, 148-159)
            int tri = __float_as_int(h4.w);
            Surf s;
            v3 pos = o;
            float closest;
            int in_m, out_m;
            if (tri >= 0) {
                const float4* tv = sc.tri_v + size_t(tri) * 3;
                const float4* ta = sc.tri_a + size_t(tri) * 4;
                float4 p0 = __ldg(tv), p1 = __ldg(tv + 1), p2 = __ldg(tv + 2);
                float4 a0 = __ldg(ta), a1 = __ldg(ta + 1), a2 = __ldg(ta + 2), a3 = __ldg(ta + 3);
                float u = h4.y, v = h4.z;
                float w0 = 1.0f - u - v;
                v3 Ns = normalize(w0 * xyz(a0) + u * xyz(a1) + v * xyz(a2));
                int mesh = __float_as_int(a3.w);
                MeshInfo mi = sc.meshes[mesh];
                s.mat = sc.materials + mi.material;
                int stale_mesh = mesh;
                const int4* mt = reinterpret_cast<const int4*>(s.mat);
                if (Full && __ldg(mt + 5).z != 0 && B.mat_tex != nullptr) {
                    // texture overrides of the closest-hit program (devicePrograms.cu:84-115)
                    float tcx = w0 * a0.w + u * a2.w + v * a3.y;
                    float tcy = w0 * a1.w + u * a3.x + v * a3.z;
                    const int4 ta = __ldg(mt + 6), tb = __ldg(mt + 7);
                    DevMaterial* dm = B.mat_tex + slot;
                    const float4* src = reinterpret_cast<const float4*>(s.mat);
                    float4* dst = reinterpret_cast<float4*>(dm);
#pragma unroll
                    for (int w = 0; w < 6; w++) dst[w] = __ldg(src + w);
                    if (ta.x >= 0) {
                        float4 t = tex_lookup(sc, ta.x, tcx, tcy);
                        dm->albedo[0] = t.x, dm->albedo[1] = t.y, dm->albedo[2] = t.z;
                    }
                    if (ta.y >= 0) dm->roughness = tex_lookup(sc, ta.y, tcx, tcy).x;
                    if (ta.z >= 0) dm->anisotropy = tex_lookup(sc, ta.z, tcx, tcy).x;
                    if (ta.w >= 0) {
                        float4 t = tex_lookup(sc, ta.w, tcx, tcy);
                        dm->specular[0] = t.x, dm->specular[1] = t.y, dm->specular[2] = t.z;
                    }
                    if (tb.x >= 0) dm->metallic = tex_lookup(sc, tb.x, tcx, tcy).x;
                    if (tb.y >= 0) dm->coat_roughness_u = tex_lookup(sc, tb.y, tcx, tcy).x;
                    if (tb.z >= 0) dm->coat_roughness_v = tex_lookup(sc, tb.z, tcx, tcy).x;
                    if (tb.w >= 0) Ns = normal_from_tangent(Ns, xyz(tex_lookup(sc, tb.w, tcx, tcy)));
                    s.mat = dm;
                    stale_mesh = mesh | kStaleTextured;
                }
                v3 P = w0 * xyz(p0) + u * xyz(p1) + v * xyz(p2);
                if (Full && G.rec != nullptr) gin = rtg::guide_input(o + h4.x * d, xyz(p0), xyz(p1), xyz(p2), d, G);
                s.front = dot(d, Ns) < 0.0f;
                s.sn = s.front ? Ns : -Ns;
                closest = length(P - o);
                pos = P;
                in_m = mi.in_medium;
                out_m = mi.out_medium;
                B.stale[slot] = make_float4(s.sn.x, s.sn.y, s.sn.z, __int_as_float(stale_mesh));
                if (bounce == 0) {
                    B.aov_a[slot] = make_float4(s.mat->albedo[0], s.mat->albedo[1], s.mat->albedo[2], Ns.x);
                    B.aov_n[slot] = make_float2(Ns.y, Ns.z);
                }
            } else {
                float4 st = B.stale[slot];
                int mesh = __float_as_int(st.w);
                s.sn = xyz(st);
                s.front = true;
                if (mesh < 0)
                    s.mat = nullptr;
                else if (Full && (mesh & kStaleTextured))  // the last hit's textured material stays, as isect.material does
                    s.mat = B.mat_tex + slot;
                else
                    s.mat = sc.materials + sc.meshes[mesh].material;
                closest = FLT_MAX;
                in_m = out_m = jd->cam.medium;
                if (bounce == 0) {
                    B.aov_a[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
                    B.aov_n[slot] = make_float2(0.f, 0.f);
                }
            }
            const rtg::Mixture* gmix = nullptr;
            if (Full && G.mix != nullptr && tri >= 0 && s.mat != nullptr) {
                const float* mw = reinterpret_cast<const float*>(s.mat);  // type, roughness (plain loads)
                const int mtype = __float_as_int(mw[0]);
                const bool glossy = mtype == RT_MAT_CONDUCTOR || mtype == RT_MAT_CLEARCOATED_CONDUCTOR;
                if (rtg::guided_type(mtype) && (!glossy || mw[4] >= G.min_rough)) {
                    gp = G.prob;
                    gmix = G.mix + slot;
                }
            }
            // ---- analytic lights (devicePrograms.cu:270-271)
            v3 light_rad(0.0f);
            float light_pdf = 0.0f;
            int lm = 0;
            bool hit_light = light_trace(sc, o, d, closest, light_rad, light_pdf, lm);
            if (hit_light) in_m = out_m = lm;

            bool alive = true;
            bool scattered = false;
            int medium_index = -1;
            float mult_trans_pdf = 1.0f;
            v3 nee_e(0.0f), nee_l(0.0f);
            // ---- media (devicePrograms.cu:274-338)
            if (Full && sc.num_media != 0) {
                medium_index = (hit_light || s.front) ? out_m : in_m;
                if (medium_index != -1) {
                    const DevMedium* mp = sc.media + medium_index;
                    const MedParams med = load_medium(mp);
                    float distance = 0.0f, trans_pdf = 0.0f;
                    v3 tr;
                    scattered = medium_sample(mp, med, o, d, closest, distance, trans_pdf, tr, rng, budget_hits);
                    history *= (tr / trans_pdf);
                    mult_trans_pdf *= trans_pdf;
                    if (scattered) {
                        pos = o + distance * d;
                        const int nl = sc.num_lights;
                        if (nl != 0) {
                            int idx = min(max(int(float(nl) * rng.next()), 0), nl - 1);
                            LightParams l = load_light(sc.lights + idx);
                            float ld = 0.0f, lp = 0.0f;
                            v3 sd;
                            float u0 = rng.next(), u1 = rng.next();
                            v3 lr = sample_light(l, pos, u0, u1, sd, ld, lp);
                            lp *= (1.0f / float(nl));
                            float cl = ld - kEps;
                            v3 tvv;
                            float tpdf;
                            int tm;
                            if (!light_trace(sc, pos, sd, cl, tvv, tpdf, tm) && nee_pdf_ok(lp)) {
                                float tp2, phase_pdf;
                                v3 tr2 = medium_transmittance(mp, med, pos, sd, cl, tp2, rng, budget_hits);
                                v3 att = evaluate_phase(med, V, sd, phase_pdf);
                                float w = l.type == RT_LIGHT_POINT ? 1.0f : power_heuristic(lp, phase_pdf * tp2);
                                nee_l = w * (tr2 / tp2) * lr * att * history / lp;
                                sh1 = !(nee_l.x == 0.0f && nee_l.y == 0.0f && nee_l.z == 0.0f);
                                s1o = pos;
                                s1d = sd;
                                s1t = ld - kEps;
                            }
                        }
                        float phase_pdf = 0.0f;
                        v3 att = sample_phase(med, rng, V, L, phase_pdf);
                        history *= (att / phase_pdf);
                        pre_pdf = phase_pdf;
                    }
                }
            }
            if (!scattered) {
                if (hit_light) {  // devicePrograms.cu:342-351
                    float w = 1.0f;
                    if (bounce != 0) {
                        pre_pdf *= mult_trans_pdf;
                        w = power_heuristic(pre_pdf, light_pdf);
                    }
                    radiance += w * history * light_rad;
                    alive = false;
                } else if (closest == FLT_MAX && medium_index == -1) {  // devicePrograms.cu:354-373
                    if (sc.env_w > 0) {
                        float u, v;
                        sphere_to_plane(d, u, v);
                        float lp = float(sc.env_w * sc.env_h) / (2.0f * sqr(kPi));
                        float4 e = tex_bilinear(sc.env, sc.env_w, sc.env_h, u, v);
                        lp *= tex_bilinear(sc.env_cache, sc.env_w, sc.env_h, u, v).z;
                        float w = 1.0f;
                        if (bounce != 0) {
                            pre_pdf *= mult_trans_pdf;
                            w = power_heuristic(pre_pdf, lp);
                        }
                        radiance += w * history * xyz(e);
                    }
                    alive = false;
                } else {
                    if (sc.env_w > 0) {  // environment NEE, devicePrograms.cu:376-424
                        float r0 = rng.next(), r1 = rng.next();
                        float4 cs = tex_bilinear(sc.env_cache, sc.env_w, sc.env_h, r0, r1);
                        v3 sd = plane_to_sphere(cs.x, cs.y);
                        float lp = float(sc.env_w * sc.env_h) / (2.0f * sqr(kPi));
                        lp *= tex_bilinear(sc.env_cache, sc.env_w, sc.env_h, cs.x, cs.y).z;
                        v3 lr = xyz(tex_bilinear(sc.env, sc.env_w, sc.env_h, cs.x, cs.y));
                        float cl = FLT_MAX;
                        v3 tvv;
                        float tpdf;
                        int tm;
                        if (!light_trace(sc, pos, sd, cl, tvv, tpdf, tm) && nee_pdf_ok(lp)) {
                            float bpdf;
                            v3 f = eval_material(sc, s, V, sd, bpdf);
                            if (Full && gp > 0.0f) bpdf = gp * rtg::mixture_pdf(gmix, sd) + (1.0f - gp) * bpdf;
                            float ct = fabsf(dot(s.sn, sd));
                            float w = power_heuristic(lp, bpdf);
                            v3 thh(1.0f);
                            if (Full && medium_index != -1) {
                                const DevMedium* mp = sc.media + medium_index;
                                const MedParams med = load_medium(mp);
                                float tp2;
                                v3 tr2 = medium_transmittance(mp, med, pos, sd, cl, tp2, rng, budget_hits);
                                thh = tr2 / tp2;
                                w = power_heuristic(lp, bpdf * tp2);
                            }
                            nee_e = w * thh * lr * f * ct * history / lp;
                            // a shadow ray only decides whether its contribution counts:
                            // one with none (the light below the horizon, f = 0) is not
                            // traced (it halves the shadow rays of the benchmark frame)
                            sh0 = !(nee_e.x == 0.0f && nee_e.y == 0.0f && nee_e.z == 0.0f);
                            s0o = pos;
                            s0d = sd;
                            s0t = FLT_MAX;
                        }
                    }
                    const int nl = sc.num_lights;
                    if (nl != 0) {  // light NEE, devicePrograms.cu:426-471
                        int idx = min(max(int(float(nl) * rng.next()), 0), nl - 1);
                        LightParams l = load_light(sc.lights + idx);
                        float ld = 0.0f, lp = 0.0f;
                        v3 sd;
                        float u0 = rng.next(), u1 = rng.next();
                        v3 lr = sample_light(l, pos, u0, u1, sd, ld, lp);
                        lp *= (1.0f / float(nl));
                        float cl = ld - kEps;
                        v3 tvv;
                        float tpdf;
                        int tm;
                        if (!light_trace(sc, pos, sd, cl, tvv, tpdf, tm) && nee_pdf_ok(lp)) {
                            float bpdf;
                            v3 f = eval_material(sc, s, V, sd, bpdf);
                            if (Full && gp > 0.0f) bpdf = gp * rtg::mixture_pdf(gmix, sd) + (1.0f - gp) * bpdf;
                            float ct = fabsf(dot(s.sn, sd));
                            float w = l.type == RT_LIGHT_POINT ? 1.0f : power_heuristic(lp, bpdf);
                            v3 thh(1.0f);
                            if (Full && medium_index != -1) {
                                const DevMedium* mp = sc.media + medium_index;
                                const MedParams med = load_medium(mp);
                                float tp2;
                                v3 tr2 = medium_transmittance(mp, med, pos, sd, cl, tp2, rng, budget_hits);
                                thh = tr2 / tp2;
                                if (l.type != RT_LIGHT_POINT) w = power_heuristic(lp, bpdf * tp2);
                            }
                            nee_l = w * thh * lr * f * ct * history / lp;
                            sh1 = !(nee_l.x == 0.0f && nee_l.y == 0.0f && nee_l.z == 0.0f);
                            s1o = pos;
                            s1d = sd;
                            s1t = ld - kEps;
                        }
                    }
                    // BSDF sampling, devicePrograms.cu:474-477
                    if (Full && gp > 0.0f) {
                        // one-sample MIS of the mixture and the BSDF: the direction comes
                        // from the mixture with probability gp, and is weighted by the
                        // combined density gp * q + (1 - gp) * p_bsdf
                        if (rng.next() < gp) {
                            float u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
                            L = rtg::mixture_sample(gmix, u0, u1, u2);
                        } else {
                            // only the direction is used (the weight comes from
                            // guide_bsdf), so the FP32 sampler serves here
                            float unused;
                            sample_material_t<float>(sc, s, rng, V, L, unused);
                        }
                        // weighted by what plain BSDF sampling integrates over the combined
                        // real density; the emission MIS weight at the next vertex uses the
                        // pdf plain sampling reports (guide_bsdf)
                        v3 fd;
                        float p_true, p_rep;
                        guide_bsdf(sc, s, V, L, fd, p_true, p_rep);
                        const float q = rtg::mixture_pdf(gmix, L);
                        const float pm = gp * q + (1.0f - gp) * p_true;
                        float ct = fabsf(dot(s.sn, L));
                        history *= (fd * ct / pm);
                        pre_pdf = gp * q + (1.0f - gp) * p_rep;
                        rec_pdf = pm;
                        rec_cos = ct;
                    } else {
                        // SampleMaterial, the path weight, Russian roulette and
                        // the next ray follow in k_sample
                        defer = true;
                    }
                }
            }
            if (alive && !defer) {
                // Russian roulette, devicePrograms.cu:480-489
                if (bounce >= jp.rr_depth) {
                    float prr = fminf((history.x + history.y + history.z) / 3.0f, 0.95f);
                    if (rng.next() > prr) {
                        alive = false;
                    } else {
                        history /= prr;
                    }
                }
                if (alive && any_nan(history)) {
                    alive = false;
                    nan_paths++;
                }
            }
            cont = alive && !defer && (bounce + 1 < jp.max_depth);
            if (Full && G.rec != nullptr && cont && rec_pdf > 0.0f && rec_cos > 0.0f && bounce < rtg::kGuideRec) {
                // training record: network input, pdf, direction, |cos|, throughput after this vertex
                float4* R = G.rec + size_t(bounce) * 4 * cap + slot;
                R[0] = make_float4(gin.x, gin.y, gin.z, rec_pdf);
                R[cap] = f4(L, rec_cos);
                R[2 * cap] = f4(history, 0.0f);
            }
            B.rad[slot] = f4(radiance, 0.0f);
            B.nee0[slot] = f4(nee_e, 0.0f);
            B.nee1[slot] = f4(nee_l, 0.0f);
            B.rng[slot] = make_uint2(uint32_t(rng.state), uint32_t(rng.state >> 32));
            if (cont) {
                B.ray_o[slot] = f4(pos, 0.0f);
                B.ray_d[slot] = f4(L, 0.0f);
                B.thr[slot] = f4(history, pre_pdf);
            } else if (defer) {  // k_sample's inputs: origin of the next ray and the front-face flag
                B.ray_o[slot] = f4(pos, s.front ? 1.0f : 0.0f);
                B.thr[slot] = f4(history, pre_pdf);
            }
        }
        int qp = warp_append(&ctl->count[nxt], cont, lane);
        if (cont) B.queue[nxt][qp] = slot;
        int sp = warp_append(&ctl->sample_count, defer, lane);
        if (defer) B.squeue[sp] = slot;
        int p0 = warp_append(&ctl->shadow_count[cur], sh0, lane);
        if (sh0) {
            B.sh_o[p0] = f4(s0o, s0t);
            B.sh_d[p0] = f4(s0d, __int_as_float(slot * 2 + 0));
        }
        int p1 = warp_append(&ctl->shadow_count[cur], sh1, lane);
        if (sh1) {
            B.sh_o[p1] = f4(s1o, s1t);
            B.sh_d[p1] = f4(s1d, __int_as_float(slot * 2 + 1));
        }
    }
    if (Stats) warp_stat(&ctl->stats[7], nan_paths);
    if (budget_hits) atomicAdd(&ctl->error, budget_hits);
}

// ------------------------------------------------------------------ BSDF sampling
// The paths k_shade leaves at a surface's BSDF sampling (devicePrograms.cu:
// 474-489): SampleMaterial in double precision (sample_material), the path
// weight, Russian roulette and the next ray.  A kernel of its own, so that
// the double-precision sampler's registers do not lower the occupancy of the
// much larger shade kernel.  Per slot it reads the origin of the next ray and
// the front-face flag (ray_o), the incoming direction (ray_d), the
// throughput and pdf (thr), the shading normal and mesh of the hit (stale)
// and the random state, which continues where k_shade left it.
template <bool Stats>
__global__ void __launch_bounds__(kBlock, 4) k_sample(Ctx c) {
    WaveCtl* ctl = c.wb.ctl;
    const int nxt = (c.bounce & 1) ^ 1;
    const int bounce = c.bounce;
    const int total = ctl->sample_count;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the next k_shade appends its shadow rays to entry nxt (k_shadow of
        // the bounce before it has finished), the next k_extend its paths to
        // the shade buckets; this bounce's k_shadow, which may run beside this
        // kernel, reads entry bounce & 1 only
        ctl->shadow_count[nxt] = 0;
        for (int b = 0; b < kShadeBuckets; b++) ctl->bucket[b] = 0;
    }
    const WaveBufs& B = c.wb;
    const WaveParams& W = wave_of(c);
    const int lane = threadIdx.x & 31;
    uint32_t nan_paths = 0;
    while (true) {
        const int base = warp_fetch(&ctl->fetch_sample, lane);
        if (base >= total) break;
        const int i = base + lane;
        bool cont = false;
        int slot = 0;
        if (i < total) {
            slot = B.squeue[i];
            const Segment& sgm = W.seg[find_segment(W, slot)];
            const JobDesc* jd = c.jobs + sgm.job;
            const SceneView& sc = jd->sc;
            const JobParams& jp = jd->job;
            const float4 o4 = B.ray_o[slot], d4 = B.ray_d[slot], th = B.thr[slot], st = B.stale[slot];
            const uint2 rs = B.rng[slot];
            Rng rng;
            rng.state = uint64_t(rs.x) | (uint64_t(rs.y) << 32);
            rng.inc = jp.rng == RT_RNG_LCG ? 0 : pcg_inc(uint64_t(sgm.path_begin + (slot - sgm.slot_begin)));
            Surf s;
            s.sn = xyz(st);
            s.front = o4.w != 0.0f;
            const int mesh = __float_as_int(st.w);
            if (mesh < 0)
                s.mat = nullptr;
            else if (mesh & kStaleTextured)
                s.mat = B.mat_tex + slot;
            else
                s.mat = sc.materials + sc.meshes[mesh].material;
            const v3 d = xyz(d4);
            const v3 V = -d;
            v3 L = d, history = xyz(th);
            float bpdf = 0.0f;
            const v3 f = sample_material(sc, s, rng, V, L, bpdf);
            const float ct = fabsf(dot(s.sn, L));
            history *= (f * ct / bpdf);
            bool alive = true;
            // Russian roulette, devicePrograms.cu:480-489
            if (bounce >= jp.rr_depth) {
                float prr = fminf((history.x + history.y + history.z) / 3.0f, 0.95f);
                if (rng.next() > prr) {
                    alive = false;
                } else {
                    history /= prr;
                }
            }
            if (alive && any_nan(history)) {
                alive = false;
                nan_paths++;
            }
            cont = alive && (bounce + 1 < jp.max_depth);
            B.rng[slot] = make_uint2(uint32_t(rng.state), uint32_t(rng.state >> 32));
            if (cont) {
                B.ray_d[slot] = f4(L, 0.0f);
                B.thr[slot] = f4(history, bpdf);
            }
        }
        const int qp = warp_append(&ctl->count[nxt], cont, lane);
        if (cont) B.queue[nxt][qp] = slot;
    }
    if (Stats) warp_stat(&ctl->stats[7], nan_paths);
}

// ------------------------------------------------------------------ shadow
// Shadow rays whose tmax is not above tmin cannot hit anything (the reference
// traces [EPS, light_distance - EPS]); they keep their contribution.
struct ShadowSrc {
    const Ctx* c;
    RT_D void load(int i, TravRay& r, const SceneView*& sc) {
        float4 o = c->wb.sh_o[i], d = c->wb.sh_d[i];
        int slot = __float_as_int(d.w) >> 1;
        const WaveParams& W = wave_of(*c);
        sc = &c->jobs[W.seg[find_segment(W, slot)].job].sc;
        r.o = xyz(o);
        r.d = xyz(d);
        r.tmin = kEps;
        r.tmax = o.w;
    }
    RT_D void finish(bool fin, int i, int tri, float, float, float, const float4*) {
        if (!fin || tri < 0) return;
        int code = __float_as_int(c->wb.sh_d[i].w);
        int slot = code >> 1;
        (code & 1 ? c->wb.nee1 : c->wb.nee0)[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
};

template <bool Stats>
__global__ void __launch_bounds__(kBlock, kTravMinBlocks) k_shadow(Ctx c) {
    WaveCtl* ctl = c.wb.ctl;
    const int total = ctl->shadow_count[c.bounce & 1];
    uint32_t nodes = 0, tris = 0, rays = 0, overflows = 0;
    ShadowSrc src{&c};
    traverse_queue<true, Stats>(src, &ctl->fetch_shadow, total, nodes, tris, rays, overflows);
    if (overflows) atomicAdd(&ctl->overflow, int(overflows));
    if (Stats) {
        warp_stat(&ctl->stats[1], rays);
        warp_stat(&ctl->stats[4], nodes);
        warp_stat(&ctl->stats[5], tris);
    }
}

// ------------------------------------------------------------------ resolve
// Folds the last pending NEE and adds each path to its pixel's sum in sample
// order.  With RT_RNG_LCG a wave holds at most one sample per pixel and a NaN
// sample ends the pixel's launch (devicePrograms.cu:499-501); with PCG32 the
// first sample of a pixel in the wave sums all of them and a NaN sample is
// dropped alone.
// The slots resolve works on, segment after segment: every slot of an LCG
// segment (at most one sample per pixel), the first npix slots of a PCG32
// segment (the first sample of each of its pixels).  Item t lies in segment
// *sgi at slot *slot; false once t is past the last item.
RT_D bool resolve_item(const Ctx& c, const WaveParams& W, int t, int* sgi, int* slot) {
    for (int i = 0; i < W.num_seg; i++) {
        const Segment& sg = W.seg[i];
        const JobParams& j = c.jobs[sg.job].job;
        const int items = j.rng == RT_RNG_LCG ? sg.count : int(min(int64_t(sg.count), j.npix));
        if (t < items) {
            *sgi = i;
            *slot = sg.slot_begin + t;
            return true;
        }
        t -= items;
    }
    return false;
}

// One path's sample: radiance, the two pending NEE terms, first-hit AOVs.
struct ResolveSample {
    float4 r, e, f, a;
    float2 n;
};
RT_D ResolveSample resolve_load(const WaveBufs& B, int sl) {
    return ResolveSample{B.rad[sl], B.nee0[sl], B.nee1[sl], B.aov_a[sl], B.aov_n[sl]};
}
// Adds the sample to the sums; a NaN sample is left out (returns false).
RT_D bool resolve_add(const ResolveSample& x, float4& acc, float4& aa, float4& an) {
    v3 r = xyz(x.r);
    r += xyz(x.e);
    r += xyz(x.f);
    if (any_nan(r)) return false;
    acc.x += r.x;
    acc.y += r.y;
    acc.z += r.z;
    aa.x += x.a.x;
    aa.y += x.a.y;
    aa.z += x.a.z;
    an.x += x.a.w;
    an.y += x.n.x;
    an.z += x.n.y;
    return true;
}

// A grid-stride loop over the wave's resolve items (a fixed grid: launching
// a thread per slot left all but the first sample's threads of a PCG32
// wave, 31 of 32 on the benchmark frame, to be scheduled only to return).
__global__ void __launch_bounds__(256) k_resolve(Ctx c) {
    const WaveParams& W = wave_of(c);
    const WaveBufs& B = c.wb;
    unsigned nans = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x;; t += gridDim.x * blockDim.x) {
        int sgi = 0, slot = 0;
        if (!resolve_item(c, W, t, &sgi, &slot)) break;
        const Segment& sg = W.seg[sgi];
        const JobParams& j = c.jobs[sg.job].job;
        const int64_t p = sg.path_begin + (slot - sg.slot_begin);
        const int pix = int(p % j.npix);
        if (j.rng == RT_RNG_LCG) {
            uint2 rs = B.rng[slot];
            j.lcg_state[pix] = rs.x;
            float4 acc = j.acc_color[pix];
            if (acc.w != 0.0f) continue;
            v3 r = xyz(B.rad[slot]);
            r += xyz(B.nee0[slot]);
            r += xyz(B.nee1[slot]);
            if (any_nan(r)) {
                j.acc_color[pix].w = 1.0f;
                nans++;
                continue;
            }
            float4 a = B.aov_a[slot];
            float2 n = B.aov_n[slot];
            j.acc_color[pix] = make_float4(acc.x + r.x, acc.y + r.y, acc.z + r.z, 0.0f);
            float4 aa = j.acc_albedo[pix], an = j.acc_normal[pix];
            j.acc_albedo[pix] = make_float4(aa.x + a.x, aa.y + a.y, aa.z + a.z, 0.f);
            j.acc_normal[pix] = make_float4(an.x + a.w, an.y + n.x, an.z + n.y, 0.f);
            continue;
        }
        // PCG32: this pixel's samples in the segment, in sample order
        float4 acc = j.acc_color[pix], aa = j.acc_albedo[pix], an = j.acc_normal[pix];
        const int64_t end = sg.path_begin + sg.count;
        const int step = int(j.npix);
        int sl = slot;
        int64_t q = p;
        // four samples' loads in flight at a time; the sums keep sample order
        for (; q + 3 * j.npix < end; q += 4 * j.npix, sl += 4 * step) {
            const ResolveSample x0 = resolve_load(B, sl), x1 = resolve_load(B, sl + step),
                                x2 = resolve_load(B, sl + 2 * step), x3 = resolve_load(B, sl + 3 * step);
            nans += resolve_add(x0, acc, aa, an) ? 0u : 1u;
            nans += resolve_add(x1, acc, aa, an) ? 0u : 1u;
            nans += resolve_add(x2, acc, aa, an) ? 0u : 1u;
            nans += resolve_add(x3, acc, aa, an) ? 0u : 1u;
        }
        for (; q < end; q += j.npix, sl += step) nans += resolve_add(resolve_load(B, sl), acc, aa, an) ? 0u : 1u;
        j.acc_color[pix] = acc;
        j.acc_albedo[pix] = aa;
        j.acc_normal[pix] = an;
    }
    if (nans) atomicAdd(&B.ctl->stats[6], (unsigned long long)nans);
}

__global__ void k_next_wave(int* wave_index, int ring) { *wave_index = (*wave_index + 1) % ring; }

// ------------------------------------------------------------------ finalize
RT_D uint32_t tonemap_pixel(float4 c, int mode, float exposure) {
    float x = c.x * exposure, y = c.y * exposure, z = c.z * exposure;
    if (mode == RT_TONEMAP_REINHARD) {  // PostProcessing.cu:18-48
        float lum = 0.299f * x + 0.587f * y + 0.114f * z;
        float f = 1.0f / (1.0f + lum / 1.5f);
        float v0 = powf(x * f, 1.0f / 2.2f), v1 = powf(y * f, 1.0f / 2.2f), v2 = powf(z * f, 1.0f / 2.2f);
        v0 = fminf(1.0f, fmaxf(0.0f, v0));
        v1 = fminf(1.0f, fmaxf(0.0f, v1));
        v2 = fminf(1.0f, fmaxf(0.0f, v2));
        return uint32_t(v0 * 255.9f) | (uint32_t(v1 * 255.9f) << 8) | (uint32_t(v2 * 255.9f) << 16) | (255u << 24);
    }
    float v[3] = {x, y, z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float t = v[k];
        if (mode == RT_TONEMAP_ACES_SRGB) {  // ACES filmic fit (Narkowicz 2015), then sRGB encoding
            t = (t * (2.51f * t + 0.03f)) / (t * (2.43f * t + 0.59f) + 0.14f);
            t = fminf(1.0f, fmaxf(0.0f, t));
            t = t <= 0.0031308f ? 12.92f * t : 1.055f * powf(t, 1.0f / 2.4f) - 0.055f;
        }
        v[k] = fminf(1.0f, fmaxf(0.0f, t));
    }
    return uint32_t(v[0] * 255.0f + 0.5f) | (uint32_t(v[1] * 255.0f + 0.5f) << 8) |
           (uint32_t(v[2] * 255.0f + 0.5f) << 16) | (255u << 24);
}

__global__ void k_finalize(const JobDesc* __restrict__ jd) {
    const JobParams& j = jd->job;
    int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= j.npix) return;
    float spp = float(j.spp);
    float4 a = j.acc_color[p];
    float4 rgba = make_float4(a.x / spp, a.y / spp, a.z / spp, 1.0f);
    if (j.frame > 0) {  // devicePrograms.cu:524-528
        float fr = float(j.frame);
        float4 old = j.color[p];
        rgba.x = (rgba.x + fr * old.x) / (fr + 1.0f);
        rgba.y = (rgba.y + fr * old.y) / (fr + 1.0f);
        rgba.z = (rgba.z + fr * old.z) / (fr + 1.0f);
        rgba.w = (rgba.w + fr * old.w) / (fr + 1.0f);
    }
    j.color[p] = rgba;
    float4 al = j.acc_albedo[p], nm = j.acc_normal[p];
    j.albedo[p] = make_float4(al.x / spp, al.y / spp, al.z / spp, 1.0f);
    j.normal[p] = make_float4(nm.x / spp, nm.y / spp, nm.z / spp, 1.0f);
    j.rgba8[p] = tonemap_pixel(rgba, j.tonemap, j.exposure);
}

// ------------------------------------------------------------------ denoiser
// Replaces the OptiX AI denoiser of Renderer::Render (core/src/Renderer.cpp:
// 660-785), a closed library: an edge-avoiding a-trous wavelet filter
// (Dammertz, Sewtz, Hanika and Lensch, HPG 2010).  It runs on irradiance
// (colour divided by the first-hit albedo AOV, so texture detail is not
// blurred), stops at edges of the normal and albedo AOVs - the guide layers
// the reference gives its denoiser - and at irradiance differences relative
// to the centre's luminance; the result is multiplied back by the albedo and
// tonemapped.  Before the passes, a pixel brighter than kDnFirefly times the
// brightest of its 8 neighbours is scaled down to that bound (an isolated
// firefly would otherwise survive the edge-stopping weights).  Five passes
// with tap spacings 1, 2, 4, 8, 16 (5 x 5 B3-spline taps each, 65 x 65 pixels
// reach), the irradiance tolerance halving per pass.
constexpr float kDnAlbedoMin = 1e-3f;
constexpr float kDnFirefly = 4.0f;

RT_D float dn_lum(float4 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

RT_D float3 dn_factor(float4 al) {
    return make_float3(al.x > kDnAlbedoMin ? al.x : 1.0f, al.y > kDnAlbedoMin ? al.y : 1.0f,
                       al.z > kDnAlbedoMin ? al.z : 1.0f);
}

__global__ void k_dn_demod(const float4* __restrict__ color, const float4* __restrict__ albedo,
                           float4* __restrict__ irr, int64_t n) {
    int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 c = color[p];
    const float3 f = dn_factor(albedo[p]);
    irr[p] = make_float4(c.x / f.x, c.y / f.y, c.z / f.z, 1.0f);
}

__global__ void k_dn_clamp(const float4* __restrict__ in, float4* __restrict__ out, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int64_t p = int64_t(y) * w + x;
    const float4 c = in[p];
    float lmax = 0.0f;
    for (int j = -1; j <= 1; j++)
        for (int i = -1; i <= 1; i++) {
            const int xx = x + i, yy = y + j;
            if ((i | j) == 0 || xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
            lmax = fmaxf(lmax, dn_lum(__ldg(in + int64_t(yy) * w + xx)));
        }
    const float lc = dn_lum(c), bound = kDnFirefly * lmax;
    const float s = lc > bound && lc > 0.0f ? bound / lc : 1.0f;
    out[p] = make_float4(c.x * s, c.y * s, c.z * s, 1.0f);
}

__global__ void k_dn_atrous(const float4* __restrict__ in, float4* __restrict__ out,
                            const float4* __restrict__ albedo, const float4* __restrict__ normal, int w, int h,
                            int step, float inv_sc2, float inv_sn2, float inv_sa2) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int64_t p = int64_t(y) * w + x;
    const float4 c = in[p], n = normal[p], a = albedo[p];
    const float lp = dn_lum(c);
    const float cs = inv_sc2 / (lp * lp + 1e-4f);
    const float hk[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    float sx = 0.f, sy = 0.f, sz = 0.f, ws = 0.f;
#pragma unroll
    for (int j = -2; j <= 2; j++) {
        const int yy = y + j * step;
        if (yy < 0 || yy >= h) continue;
#pragma unroll
        for (int i = -2; i <= 2; i++) {
            const int xx = x + i * step;
            if (xx < 0 || xx >= w) continue;
            const int64_t q = int64_t(yy) * w + xx;
            const float4 cq = __ldg(in + q), nq = __ldg(normal + q), aq = __ldg(albedo + q);
            const float dc = (cq.x - c.x) * (cq.x - c.x) + (cq.y - c.y) * (cq.y - c.y) + (cq.z - c.z) * (cq.z - c.z);
            const float dn = (nq.x - n.x) * (nq.x - n.x) + (nq.y - n.y) * (nq.y - n.y) + (nq.z - n.z) * (nq.z - n.z);
            const float da = (aq.x - a.x) * (aq.x - a.x) + (aq.y - a.y) * (aq.y - a.y) + (aq.z - a.z) * (aq.z - a.z);
            const float wq = hk[i + 2] * hk[j + 2] * __expf(-(dc * cs + dn * inv_sn2 + da * inv_sa2));
            sx += wq * cq.x;
            sy += wq * cq.y;
            sz += wq * cq.z;
            ws += wq;
        }
    }
    // the centre tap always has weight 9/64, so ws > 0 unless c is not finite
    out[p] = ws > 0.0f ? make_float4(sx / ws, sy / ws, sz / ws, 1.0f) : c;
}

__global__ void k_dn_remod(const float4* __restrict__ irr, const float4* __restrict__ albedo,
                           float4* __restrict__ out, uint32_t* __restrict__ rgba8, int64_t n, int tonemap,
                           float exposure) {
    int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 e = irr[p];
    const float3 f = dn_factor(albedo[p]);
    const float4 c = make_float4(e.x * f.x, e.y * f.y, e.z * f.z, 1.0f);
    out[p] = c;
    if (rgba8) rgba8[p] = tonemap_pixel(c, tonemap, exposure);
}

// ------------------------------------------------------------------ ray queries
template <bool AnyHit>
__global__ void __launch_bounds__(kBlock) k_trace(SceneView sc, const float* __restrict__ rays, int64_t n,
                                                  float* __restrict__ hits, int* overflow) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4* rr = reinterpret_cast<const float4*>(rays) + i * 2;
    float4 a = rr[0], b = rr[1];
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
    reinterpret_cast<float4*>(hits)[i] = out;
}

// ------------------------------------------------------------------ wavefront ray queries
// Stages n query rays (2 float4 each: origin + tmin, direction + tmax) as one
// wave of the path-tracing kernels: closest-hit queries become the extend
// queue of bounce 0 (slot i = ray i), any-hit queries become the shadow queue
// with a unit pending contribution in nee0[i] that k_shadow clears when the
// ray is occluded.  Resets the wave's counters as k_raygen does.
__global__ void k_query_stage(Ctx c, const float4* __restrict__ rays, int n, int any_hit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const WaveBufs& b = c.wb;
    WaveCtl* ctl = b.ctl;
    if (i == 0) {
        ctl->count[0] = any_hit ? 0 : n;
        ctl->count[1] = 0;
        ctl->shadow_count[0] = any_hit ? n : 0;
        ctl->shadow_count[1] = 0;
        ctl->fetch_ext = 0;
        ctl->fetch_shade = 0;
        ctl->fetch_shadow = 0;
        ctl->error = 0;
        ctl->overflow = 0;
        for (int k = 0; k < 8; k++) ctl->stats[k] = 0ull;
        for (int k = 0; k < kShadeBuckets; k++) ctl->bucket[k] = 0;
    }
    if (i >= n) return;
    const float4 o = rays[2 * i], d = rays[2 * i + 1];
    if (!any_hit) {
        b.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
        b.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
        b.queue[0][i] = i;
    } else {
        b.sh_o[i] = make_float4(o.x, o.y, o.z, d.w);
        b.sh_d[i] = make_float4(d.x, d.y, d.z, __int_as_float(i * 2));
        b.nee0[i] = make_float4(1.f, 1.f, 1.f, 0.f);
    }
}

// Hits of a query wave in the layout of k_trace: (t, b1, b2, original
// triangle id) for closest hits, (0, 0, 0, 1) for an occluded any-hit ray and
// (FLT_MAX, 0, 0, -1) for a miss.
__global__ void k_query_collect(Ctx c, SceneView sc, float4* __restrict__ out, int n, int any_hit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const WaveBufs& b = c.wb;
    const float4 miss = make_float4(FLT_MAX, 0.f, 0.f, __int_as_float(-1));
    if (any_hit) {
        out[i] = b.nee0[i].x == 0.0f ? make_float4(0.f, 0.f, 0.f, __int_as_float(1)) : miss;
        return;
    }
    const float4 h = b.hit[i];
    const int tri = __float_as_int(h.w);
    if (tri < 0) {
        out[i] = miss;
        return;
    }
    out[i] = make_float4(h.x, h.y, h.z, __ldg(sc.tri_v + size_t(tri) * 3).w);
}

// ------------------------------------------------------------------ verification
struct ListRng {
    const float* u;
    int n, used;
    RT_D float next() {
        used++;
        return (used - 1) < n ? u[used - 1] : 0.5f;
    }
};

__global__ void k_verify(int op, SceneView sc, const DevLight* lights, const DevMedium* media,
                         const float* __restrict__ in, int64_t n, float* __restrict__ out) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* x = in + i * 16;
    float* y = out + i * 8;
    float r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    ListRng rng;
    rng.used = 0;
    if (op == RT_VERIFY_BSDF_SAMPLE_PDF) {
        Surf s;
        s.sn = ld3(x);
        s.front = x[9] != 0.0f;
        s.mat = sc.materials + int(x[10]);
        float epdf = 0.0f;
        eval_material(sc, s, ld3(x + 3), ld3(x + 6), epdf);
        v3 fd;
        float p_true, p_rep;
        guide_bsdf(sc, s, ld3(x + 3), ld3(x + 6), fd, p_true, p_rep);
        r[0] = p_true;
        r[1] = epdf;
        r[2] = p_rep;
        r[3] = fd.x;
        r[4] = fd.y;
        r[5] = fd.z;
    } else if (op == RT_VERIFY_BSDF_EVAL || op == RT_VERIFY_BSDF_SAMPLE) {
        bool sample = op == RT_VERIFY_BSDF_SAMPLE;
        Surf s;
        s.sn = ld3(x);
        s.front = (sample ? x[12] : x[9]) != 0.0f;
        s.mat = sc.materials + int(sample ? x[13] : x[10]);
        v3 V = ld3(x + 3);
        float pdf = 0.0f;
        v3 f;
        if (!sample) {
            f = eval_material(sc, s, V, ld3(x + 6), pdf);
        } else {
            rng.u = x + 6;
            rng.n = 6;
            v3 L(0.0f);
            f = sample_material(sc, s, rng, V, L, pdf);
            r[4] = L.x;
            r[5] = L.y;
            r[6] = L.z;
            r[7] = float(rng.used);
        }
        r[0] = f.x;
        r[1] = f.y;
        r[2] = f.z;
        r[3] = pdf;
    } else if (op == RT_VERIFY_LIGHT_SAMPLE) {
        LightParams l = load_light(lights + int(x[5]));
        v3 L(0.0f);
        float dist = 0.0f, pdf = 0.0f;
        v3 Li = sample_light(l, ld3(x), x[3], x[4], L, dist, pdf);
        r[0] = Li.x; r[1] = Li.y; r[2] = Li.z; r[3] = pdf;
        r[4] = L.x; r[5] = L.y; r[6] = L.z; r[7] = dist;
    } else if (op == RT_VERIFY_LIGHT_EVAL) {
        LightParams l = load_light(lights + int(x[7]));
        float pdf = 0.0f, ld = 0.0f;
        v3 Li = evaluate_light(l, ld3(x), ld3(x + 3), x[6], pdf, ld);
        r[0] = Li.x; r[1] = Li.y; r[2] = Li.z; r[3] = pdf; r[4] = ld;
    } else if (op == RT_VERIFY_MEDIUM_SAMPLE) {
        MedParams m = load_medium(media + int(x[3]));
        rng.u = x + 1;
        rng.n = 2;
        float dist = 0.0f, tp = 0.0f;
        v3 tr;
        bool sc_ = sample_medium_distance(m, x[0], dist, tp, tr, rng);
        r[0] = tr.x; r[1] = tr.y; r[2] = tr.z; r[3] = tp; r[4] = dist; r[5] = sc_ ? 1.0f : 0.0f;
        r[6] = float(rng.used);
    } else if (op == RT_VERIFY_PHASE_SAMPLE) {
        MedParams m = load_medium(media + int(x[7]));
        rng.u = x + 3;
        rng.n = 4;
        v3 L(0.0f);
        float pdf = 0.0f;
        v3 a = sample_phase(m, rng, ld3(x), L, pdf);
        r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = pdf;
        r[4] = L.x; r[5] = L.y; r[6] = L.z; r[7] = float(rng.used);
    } else if (op == RT_VERIFY_PHASE_EVAL) {
        MedParams m = load_medium(media + int(x[6]));
        float pdf = 0.0f;
        v3 a = evaluate_phase(m, ld3(x), ld3(x + 3), pdf);
        r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = pdf;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) y[k] = r[k];
}

}  // namespace rtd

// ====================================================================== host
namespace rth {
using namespace rtd;

void query_shape(LaunchShape& s) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_extend<false>, kBlock, 0);
    s.blocks_extend = s.sms * (b > 0 ? b : 1);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<false, true>, kBlock, 0);
    s.blocks_shade = s.sms * (b > 0 ? b : 1);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<false, false>, kBlock, 0);
    s.blocks_shade_plain = s.sms * (b > 0 ? b : 1);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shadow<false>, kBlock, 0);
    s.blocks_shadow = s.sms * (b > 0 ? b : 1);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sample<false>, kBlock, 0);
    s.blocks_sample = s.sms * (b > 0 ? b : 1);
}

static unsigned grid_for(int64_t n, int block) { return unsigned((n + block - 1) / block); }

void launch_begin(const JobDesc& hj, const JobDesc* dj, cudaStream_t st) {
    k_begin<<<grid_for(hj.job.npix, 256), 256, 0, st>>>(dj);
}
void launch_sample_shadow_and_next_extend(Ctx c, const LaunchShape& s, cudaStream_t st, const WaveFork* f) {
    if (f == nullptr) {
        launch_sample(c, s, false, st);
        launch_shadow(c, s, false, st);
        c.bounce += 1;
        launch_extend(c, s, false, st);
        return;
    }
    cudaEventRecord(f->fork, st);
    cudaStreamWaitEvent(f->side, f->fork, 0);
    launch_shadow(c, s, false, f->side);
    cudaEventRecord(f->join, f->side);
    launch_sample(c, s, false, st);
    c.bounce += 1;
    launch_extend(c, s, false, st);
    cudaStreamWaitEvent(st, f->join, 0);
}

cudaError_t create_fork(WaveFork& f) {
    f = WaveFork{};
    cudaError_t e = cudaStreamCreateWithFlags(&f.side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming);
    if (e != cudaSuccess) destroy_fork(f);
    return e;
}

void destroy_fork(WaveFork& f) {
    if (f.side) cudaStreamDestroy(f.side);
    if (f.fork) cudaEventDestroy(f.fork);
    if (f.join) cudaEventDestroy(f.join);
    f = WaveFork{};
}

void launch_raygen(const Ctx& c, cudaStream_t st) { k_raygen<<<grid_for(c.wb.capacity, kRaygenBlock), kRaygenBlock, 0, st>>>(c); }
void launch_extend(const Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st) {
    if (stats)
        k_extend<true><<<s.blocks_extend, kBlock, 0, st>>>(c);
    else
        k_extend<false><<<s.blocks_extend, kBlock, 0, st>>>(c);
}
void launch_shade(const Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st) {
    const bool full = c.features != 0;
    const int blocks = full ? s.blocks_shade : s.blocks_shade_plain;
    if (stats) {
        if (full)
            k_shade<true, true><<<blocks, kBlock, 0, st>>>(c);
        else
            k_shade<true, false><<<blocks, kBlock, 0, st>>>(c);
    } else {
        if (full)
            k_shade<false, true><<<blocks, kBlock, 0, st>>>(c);
        else
            k_shade<false, false><<<blocks, kBlock, 0, st>>>(c);
    }
}
void launch_sample(const Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st) {
    if (stats)
        k_sample<true><<<s.blocks_sample, kBlock, 0, st>>>(c);
    else
        k_sample<false><<<s.blocks_sample, kBlock, 0, st>>>(c);
}
void launch_shadow(const Ctx& c, const LaunchShape& s, bool stats, cudaStream_t st) {
    if (stats)
        k_shadow<true><<<s.blocks_shadow, kBlock, 0, st>>>(c);
    else
        k_shadow<false><<<s.blocks_shadow, kBlock, 0, st>>>(c);
}
void launch_resolve(const Ctx& c, cudaStream_t st) {
    // enough threads for a few items each on the benchmark frame (2M pixels)
    k_resolve<<<std::min(grid_for(c.wb.capacity, 256), 2048u), 256, 0, st>>>(c);
}
void launch_next_wave(const Ctx& c, cudaStream_t st) { k_next_wave<<<1, 1, 0, st>>>(c.wave_index, c.wave_ring); }
void launch_finalize(const JobDesc& hj, const JobDesc* dj, cudaStream_t st) {
    k_finalize<<<grid_for(hj.job.npix, 256), 256, 0, st>>>(dj);
}
void launch_begin_n(const JobDesc* dj, int64_t npix, cudaStream_t st) { k_begin<<<grid_for(npix, 256), 256, 0, st>>>(dj); }
void launch_finalize_n(const JobDesc* dj, int64_t npix, cudaStream_t st) {
    k_finalize<<<grid_for(npix, 256), 256, 0, st>>>(dj);
}
int launch_denoise(const DenoiseArgs& d, cudaStream_t st) {
    const int64_t n = int64_t(d.w) * d.h;
    if (n <= 0) return 0;
    k_dn_demod<<<grid_for(n, 256), 256, 0, st>>>(d.color, d.albedo, d.tmp0, n);
    const dim3 blk(16, 16), grd(unsigned((d.w + 15) / 16), unsigned((d.h + 15) / 16));
    k_dn_clamp<<<grd, blk, 0, st>>>(d.tmp0, d.tmp1, d.w, d.h);
    float4* src = d.tmp1;
    float4* dst = d.tmp0;
    float inv_sc2 = 1.0f / (kDenoiseSigmaColor * kDenoiseSigmaColor);
    for (int it = 0; it < kDenoisePasses; it++) {
        k_dn_atrous<<<grd, blk, 0, st>>>(src, dst, d.albedo, d.normal, d.w, d.h, 1 << it, inv_sc2,
                                         1.0f / (kDenoiseSigmaNormal * kDenoiseSigmaNormal),
                                         1.0f / (kDenoiseSigmaAlbedo * kDenoiseSigmaAlbedo));
        inv_sc2 *= 4.0f;  // sigma halves per pass
        float4* t = src;
        src = dst;
        dst = t;
    }
    k_dn_remod<<<grid_for(n, 256), 256, 0, st>>>(src, d.albedo, d.out, d.rgba8, n, d.tonemap, d.exposure);
    return kDenoisePasses + 3;
}
void launch_trace(const SceneView& sc, bool any_hit, const float* rays, int64_t n, float* hits, int* overflow,
                  cudaStream_t st) {
    if (n <= 0) return;
    if (any_hit)
        k_trace<true><<<grid_for(n, kBlock), kBlock, 0, st>>>(sc, rays, n, hits, overflow);
    else
        k_trace<false><<<grid_for(n, kBlock), kBlock, 0, st>>>(sc, rays, n, hits, overflow);
}
void launch_query_stage(const Ctx& c, const float* rays, int n, bool any_hit, cudaStream_t st) {
    k_query_stage<<<grid_for(std::max(n, 1), 256), 256, 0, st>>>(c, reinterpret_cast<const float4*>(rays), n,
                                                                  any_hit ? 1 : 0);
}
void launch_query_collect(const Ctx& c, const SceneView& sc, float* hits, int n, bool any_hit, cudaStream_t st) {
    if (n <= 0) return;
    k_query_collect<<<grid_for(n, 256), 256, 0, st>>>(c, sc, reinterpret_cast<float4*>(hits), n, any_hit ? 1 : 0);
}
void launch_verify(int op, const SceneView& sc, const DevLight* lights, const DevMedium* media, const float* in,
                   int64_t n, float* out, cudaStream_t st) {
    if (n <= 0) return;
    k_verify<<<grid_for(n, 128), 128, 0, st>>>(op, sc, lights, media, in, n, out);
}
}  // namespace rth
