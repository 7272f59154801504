// rt_bvh_gpu.cu - the acceleration structure built on the device (replaces
// optixAccelBuild, core/src/Renderer.cpp:146-285), with the rules of the host
// build in rt_bvh.cpp:
//
// 1. Binned SAH binary BVH, 32 bins per axis on the triangle centroids, leaves
//    of at most three triangles (a node of up to three may stay a leaf when
//    SAH prefers it).  Nodes of more than kSmall triangles are split level by
//    level by all SMs: blocks bin chunks of 4096 positions in shared memory
//    and add their bins to the node's with atomics, one warp per node picks the
//    split, and the chunks are partitioned through a scratch permutation.
//    Smaller nodes are finished by one warp each, a lane per bin.
// 2. Collapse into compressed 8-wide nodes, one thread per wide node, level by
//    level: open the largest-area child until there are eight, assign slots by
//    the octant of each child's centre, quantise the child boxes outwards.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "rt_bvh.h"
#include "rt_device.cuh"

namespace rtbg {

constexpr int kBins = 32;
constexpr int kMaxLeaf = 3;
constexpr int kSmall = 256;    // nodes of at most this many triangles are built by one warp
constexpr int kChunk = 4096;   // positions binned / partitioned by one block
constexpr int kStack = 256;    // per-warp range stack of the small builds (at most one entry per triangle)

struct Node2 {
    float lo[3];
    int left;   // first child (the second is left + 1), -1 for a leaf
    float hi[3];
    int first;  // range of the permutation
    int count;
    int pad[3];
};

struct Task {
    int node, first, count, pad;
    float cmin[4], cmax[4];  // centroid bounds
};

// Bins of one large node: per axis and bin a count, the box and the centroid
// box, as order-preserving integers so that atomicMin/Max can combine them.
struct Bins {
    int cnt[3][kBins];
    int lo[3][kBins][3], hi[3][kBins][3];
    int clo[3][kBins][3], chi[3][kBins][3];
};
constexpr int kBinWords = int(sizeof(Bins) / 4);  // cnt 96, then four blocks of 288

struct Split {
    int axis;  // -1: split the range in the middle
    int bin;   // first bin of the right child
    int nl;    // triangles in the left child
    int lcur, rcur;  // partition cursors
};

RT_D int f2o(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
RT_D float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

RT_D float area_of(const float lo[3], const float hi[3]) {
    float d0 = fmaxf(0.f, hi[0] - lo[0]), d1 = fmaxf(0.f, hi[1] - lo[1]), d2 = fmaxf(0.f, hi[2] - lo[2]);
    return 2.0f * (d0 * d1 + d1 * d2 + d2 * d0);
}

RT_D int bin_of(float c, float cmin, float scale) { return min(kBins - 1, max(0, int((c - cmin) * scale))); }

// Initial value of word w of a Bins record: 0 for counts, +-FLT_MAX for bounds.
RT_D int bin_init(int w) {
    if (w < 96) return 0;
    const int part = (w - 96) / 288;  // 0 lo, 1 hi, 2 clo, 3 chi
    return (part == 0 || part == 2) ? f2o(FLT_MAX) : f2o(-FLT_MAX);
}

// ------------------------------------------------------------------ primitives
__global__ void k_prims(const float* __restrict__ tv, int n, float4* __restrict__ plo, float4* __restrict__ phi,
                        int* __restrict__ ids, int* __restrict__ root_c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int c[6];
    for (int a = 0; a < 3; a++) {
        c[a] = f2o(FLT_MAX);
        c[3 + a] = f2o(-FLT_MAX);
    }
    if (i < n) {
        const float* t = tv + size_t(i) * 9;
        float lo[3], hi[3];
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(fminf(t[a], t[3 + a]), t[6 + a]);
            hi[a] = fmaxf(fmaxf(t[a], t[3 + a]), t[6 + a]);
            const float cc = 0.5f * (lo[a] + hi[a]);
            c[a] = f2o(cc);
            c[3 + a] = f2o(cc);
        }
        plo[i] = make_float4(lo[0], lo[1], lo[2], 0.f);
        phi[i] = make_float4(hi[0], hi[1], hi[2], 0.f);
        ids[i] = i;
    }
    for (int a = 0; a < 3; a++) {
        int mn = c[a], mx = c[3 + a];
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(root_c + a, mn);
            atomicMax(root_c + 3 + a, mx);
        }
    }
}

__global__ void k_root_task(const int* __restrict__ root_c, int n, Task* __restrict__ tasks) {
    Task t;
    t.node = 0;
    t.first = 0;
    t.count = n;
    t.pad = 0;
    for (int a = 0; a < 3; a++) {
        t.cmin[a] = o2f(root_c[a]);
        t.cmax[a] = o2f(root_c[3 + a]);
    }
    t.cmin[3] = t.cmax[3] = 0.f;
    tasks[0] = t;
}

// ------------------------------------------------------------------ large nodes
// Chunk list of this level: chunk k covers positions [start, start + kChunk) of task `task`.
__global__ void k_chunks(const Task* __restrict__ tasks, const int* __restrict__ ntasks, int2* __restrict__ chunks,
                         int* __restrict__ nchunks, int max_chunks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int k = 0;
    for (int t = 0; t < *ntasks; t++)
        for (int s = 0; s < tasks[t].count && k < max_chunks; s += kChunk) chunks[k++] = make_int2(t, s);
    *nchunks = k;
}

__global__ void k_clear_bins(Bins* __restrict__ bins, const int* __restrict__ ntasks) {
    const int total = *ntasks * kBinWords;
    int* b = reinterpret_cast<int*>(bins);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        b[i] = bin_init(i % kBinWords);
}

__global__ void __launch_bounds__(256) k_bin(const int2* __restrict__ chunks, const int* __restrict__ nchunks,
                                             const Task* __restrict__ tasks, const int* __restrict__ ids,
                                             const float4* __restrict__ plo, const float4* __restrict__ phi,
                                             Bins* __restrict__ bins) {
    __shared__ Bins sb;
    const int nc = *nchunks;
    int* s = reinterpret_cast<int*>(&sb);
    for (int ck = blockIdx.x; ck < nc; ck += gridDim.x) {
        for (int w = threadIdx.x; w < kBinWords; w += blockDim.x) s[w] = bin_init(w);
        __syncthreads();
        const int2 c = chunks[ck];
        const Task t = tasks[c.x];
        const int end = min(t.count, c.y + kChunk);
        float scale[3];
        for (int a = 0; a < 3; a++) {
            const float ext = t.cmax[a] - t.cmin[a];
            scale[a] = ext > 0.f ? float(kBins) / ext : 0.f;
        }
        for (int i = c.y + threadIdx.x; i < end; i += blockDim.x) {
            const int p = ids[t.first + i];
            const float4 lo = plo[p], hi = phi[p];
            const float cc[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
            const float l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z};
            for (int a = 0; a < 3; a++) {
                const int b = bin_of(cc[a], t.cmin[a], scale[a]);
                atomicAdd(&sb.cnt[a][b], 1);
                for (int k = 0; k < 3; k++) {
                    atomicMin(&sb.lo[a][b][k], f2o(l3[k]));
                    atomicMax(&sb.hi[a][b][k], f2o(h3[k]));
                    atomicMin(&sb.clo[a][b][k], f2o(cc[k]));
                    atomicMax(&sb.chi[a][b][k], f2o(cc[k]));
                }
            }
        }
        __syncthreads();
        Bins* g = bins + c.x;
        for (int w = threadIdx.x; w < 3 * kBins; w += blockDim.x) {
            const int a = w / kBins, b = w % kBins;
            if (sb.cnt[a][b] == 0) continue;
            atomicAdd(&g->cnt[a][b], sb.cnt[a][b]);
            for (int k = 0; k < 3; k++) {
                atomicMin(&g->lo[a][b][k], sb.lo[a][b][k]);
                atomicMax(&g->hi[a][b][k], sb.hi[a][b][k]);
                atomicMin(&g->clo[a][b][k], sb.clo[a][b][k]);
                atomicMax(&g->chi[a][b][k], sb.chi[a][b][k]);
            }
        }
        __syncthreads();
    }
}

// Warp helpers over lanes = bins.
struct Box3 {
    float lo[3], hi[3];
};
RT_D Box3 box_shfl_up(const Box3& b, int d) {
    Box3 r;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = __shfl_up_sync(0xffffffffu, b.lo[k], d);
        r.hi[k] = __shfl_up_sync(0xffffffffu, b.hi[k], d);
    }
    return r;
}
RT_D Box3 box_shfl_down(const Box3& b, int d) {
    Box3 r;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = __shfl_down_sync(0xffffffffu, b.lo[k], d);
        r.hi[k] = __shfl_down_sync(0xffffffffu, b.hi[k], d);
    }
    return r;
}
RT_D void box_grow(Box3& a, const Box3& b) {
    for (int k = 0; k < 3; k++) {
        a.lo[k] = fminf(a.lo[k], b.lo[k]);
        a.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
}
RT_D Box3 empty_box() {
    Box3 b;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = FLT_MAX;
        b.hi[k] = -FLT_MAX;
    }
    return b;
}
RT_D void box_reduce_all(Box3& b) {
    for (int o = 16; o > 0; o >>= 1) box_grow(b, box_shfl_down(b, o));
    for (int k = 0; k < 3; k++) {
        b.lo[k] = __shfl_sync(0xffffffffu, b.lo[k], 0);
        b.hi[k] = __shfl_sync(0xffffffffu, b.hi[k], 0);
    }
}

// SAH over one axis with lane = bin: the axis' best cost, split (first bin of
// the right side) and left count, the same on all lanes.
RT_D void sah_axis(int cnt, Box3 box, float& best_cost, int& best_split, int& best_nl) {
    const int lane = threadIdx.x & 31;
    int cl = cnt, cr = cnt;
    Box3 bl = box, br = box;
    for (int d = 1; d < 32; d <<= 1) {
        const int ul = __shfl_up_sync(0xffffffffu, cl, d);
        const Box3 xl = box_shfl_up(bl, d);
        const int ur = __shfl_down_sync(0xffffffffu, cr, d);
        const Box3 xr = box_shfl_down(br, d);
        if (lane >= d) {
            cl += ul;
            box_grow(bl, xl);
        }
        if (lane + d < 32) {
            cr += ur;
            box_grow(br, xr);
        }
    }
    // split after bin `lane`: left = bins 0..lane, right = bins lane+1..31
    const int rc = __shfl_down_sync(0xffffffffu, cr, 1);
    const Box3 rb = box_shfl_down(br, 1);
    float cost = FLT_MAX;
    if (lane < 31 && cl > 0 && rc > 0) cost = area_of(bl.lo, bl.hi) * float(cl) + area_of(rb.lo, rb.hi) * float(rc);
    best_cost = cost;
    best_split = lane + 1;
    best_nl = cl;
    for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_down_sync(0xffffffffu, best_cost, o);
        const int os = __shfl_down_sync(0xffffffffu, best_split, o);
        const int on = __shfl_down_sync(0xffffffffu, best_nl, o);
        if (oc < best_cost || (oc == best_cost && os < best_split)) {
            best_cost = oc;
            best_split = os;
            best_nl = on;
        }
    }
    best_cost = __shfl_sync(0xffffffffu, best_cost, 0);
    best_split = __shfl_sync(0xffffffffu, best_split, 0);
    best_nl = __shfl_sync(0xffffffffu, best_nl, 0);
}

// One warp per large node: the split, the node's box, its two children and
// where they go next (the next level's large nodes or the small list).  A
// large node (more than kSmall > kMaxLeaf triangles) always splits.
__global__ void k_split(const Task* __restrict__ tasks, const int* __restrict__ ntasks, const Bins* __restrict__ bins,
                        Split* __restrict__ splits, Node2* __restrict__ nodes, int* __restrict__ node_count,
                        Task* __restrict__ next, int* __restrict__ nnext, Task* __restrict__ small,
                        int* __restrict__ nsmall) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= *ntasks) return;
    const Task t = tasks[warp];
    const Bins& b = bins[warp];
    float best = FLT_MAX;
    int axis = -1, split = 0, nl = 0;
    for (int a = 0; a < 3; a++) {
        if (!(t.cmax[a] - t.cmin[a] > 0.f)) continue;
        Box3 bx;
        for (int k = 0; k < 3; k++) {
            bx.lo[k] = o2f(b.lo[a][lane][k]);
            bx.hi[k] = o2f(b.hi[a][lane][k]);
        }
        float c;
        int s, n;
        sah_axis(b.cnt[a][lane], bx, c, s, n);
        if (c < best) {
            best = c;
            axis = a;
            split = s;
            nl = n;
        }
    }
    // node box: the bins of any one axis hold every triangle
    Box3 nodebox;
    {
        const int a = axis >= 0 ? axis : 0;
        for (int k = 0; k < 3; k++) {
            nodebox.lo[k] = b.cnt[a][lane] ? o2f(b.lo[a][lane][k]) : FLT_MAX;
            nodebox.hi[k] = b.cnt[a][lane] ? o2f(b.hi[a][lane][k]) : -FLT_MAX;
        }
        box_reduce_all(nodebox);
    }
    if (axis < 0 || nl <= 0 || nl >= t.count) {  // identical centroids: split the range
        axis = -1;
        nl = t.count / 2;
    }
    Box3 cl = empty_box(), cr = empty_box();
    if (axis >= 0) {
        if (b.cnt[axis][lane]) {
            Box3 cb;
            for (int k = 0; k < 3; k++) {
                cb.lo[k] = o2f(b.clo[axis][lane][k]);
                cb.hi[k] = o2f(b.chi[axis][lane][k]);
            }
            box_grow(lane < split ? cl : cr, cb);
        }
        box_reduce_all(cl);
        box_reduce_all(cr);
    } else {
        for (int k = 0; k < 3; k++) {
            cl.lo[k] = cr.lo[k] = t.cmin[k];
            cl.hi[k] = cr.hi[k] = t.cmax[k];
        }
    }
    if (lane != 0) return;
    Node2 nd;
    for (int k = 0; k < 3; k++) {
        nd.lo[k] = nodebox.lo[k];
        nd.hi[k] = nodebox.hi[k];
    }
    const int c = atomicAdd(node_count, 2);
    nd.left = c;
    nd.first = t.first;
    nd.count = t.count;
    nd.pad[0] = nd.pad[1] = nd.pad[2] = 0;
    nodes[t.node] = nd;
    Split sp;
    sp.axis = axis;
    sp.bin = split;
    sp.nl = nl;
    sp.lcur = t.first;
    sp.rcur = t.first + nl;
    splits[warp] = sp;
    const int counts[2] = {nl, t.count - nl};
    const int firsts[2] = {t.first, t.first + nl};
    for (int h = 0; h < 2; h++) {
        Task ct;
        ct.node = c + h;
        ct.first = firsts[h];
        ct.count = counts[h];
        ct.pad = 0;
        const Box3& cb = h ? cr : cl;
        for (int k = 0; k < 3; k++) {
            ct.cmin[k] = cb.lo[k];
            ct.cmax[k] = cb.hi[k];
        }
        ct.cmin[3] = ct.cmax[3] = 0.f;
        if (ct.count > kSmall)
            next[atomicAdd(nnext, 1)] = ct;
        else
            small[atomicAdd(nsmall, 1)] = ct;
    }
}

__global__ void __launch_bounds__(256) k_partition(const int2* __restrict__ chunks, const int* __restrict__ nchunks,
                                                   const Task* __restrict__ tasks, Split* __restrict__ splits,
                                                   const int* __restrict__ ids, int* __restrict__ tmp,
                                                   const float4* __restrict__ plo, const float4* __restrict__ phi) {
    const int nc = *nchunks;
    const int lane = threadIdx.x & 31;
    for (int ck = blockIdx.x; ck < nc; ck += gridDim.x) {
        const int2 c = chunks[ck];
        const Task t = tasks[c.x];
        Split* sp = splits + c.x;
        const int axis = sp->axis, sbin = sp->bin, nl = sp->nl;
        const float ext = axis >= 0 ? t.cmax[axis] - t.cmin[axis] : 0.f;
        const float scale = ext > 0.f ? float(kBins) / ext : 0.f;
        const float cmin = axis >= 0 ? t.cmin[axis] : 0.f;
        const int end = min(t.count, c.y + kChunk);
        for (int base = c.y; base < end; base += blockDim.x) {
            const int i = base + int(threadIdx.x);
            const bool valid = i < end;
            int p = 0;
            bool left = false;
            if (valid) {
                p = ids[t.first + i];
                if (axis >= 0) {
                    const float4 lo = plo[p], hi = phi[p];
                    const float cc = 0.5f * ((&lo.x)[axis] + (&hi.x)[axis]);
                    left = bin_of(cc, cmin, scale) < sbin;
                } else {
                    left = i < nl;
                }
            }
            const unsigned ml = __ballot_sync(0xffffffffu, valid && left);
            const unsigned mr = __ballot_sync(0xffffffffu, valid && !left);
            int bl = 0, br = 0;
            if (lane == 0) {
                if (ml) bl = atomicAdd(&sp->lcur, __popc(ml));
                if (mr) br = atomicAdd(&sp->rcur, __popc(mr));
            }
            bl = __shfl_sync(0xffffffffu, bl, 0);
            br = __shfl_sync(0xffffffffu, br, 0);
            const unsigned lt = (1u << lane) - 1u;
            if (valid) tmp[left ? bl + __popc(ml & lt) : br + __popc(mr & lt)] = p;
        }
    }
}

__global__ void k_copy_back(const int2* __restrict__ chunks, const int* __restrict__ nchunks,
                            const Task* __restrict__ tasks, const int* __restrict__ tmp, int* __restrict__ ids) {
    const int nc = *nchunks;
    for (int ck = blockIdx.x; ck < nc; ck += gridDim.x) {
        const int2 c = chunks[ck];
        const Task t = tasks[c.x];
        const int end = min(t.count, c.y + kChunk);
        for (int i = c.y + threadIdx.x; i < end; i += blockDim.x) ids[t.first + i] = tmp[t.first + i];
    }
}

// ------------------------------------------------------------------ small nodes
// One warp builds the whole subtree of a node of at most kSmall triangles.
__global__ void __launch_bounds__(128) k_small(const Task* __restrict__ tasks, const int* __restrict__ ntasks,
                                               int* __restrict__ ids, int* __restrict__ tmp,
                                               const float4* __restrict__ plo, const float4* __restrict__ phi,
                                               Node2* __restrict__ nodes, int* __restrict__ node_count,
                                               int* __restrict__ error) {
    __shared__ int3 stack[4][kStack];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int ti = warp; ti < *ntasks; ti += nwarps) {
        if (lane == 0) stack[wib][0] = make_int3(tasks[ti].node, tasks[ti].first, tasks[ti].count);
        int sp = 1;
        __syncwarp();
        while (sp > 0) {
            const int3 e = stack[wib][--sp];
            __syncwarp();
            const int node = e.x, first = e.y, count = e.z;
            Box3 bb = empty_box(), cb = empty_box();
            for (int i = lane; i < count; i += 32) {
                const int p = ids[first + i];
                const float4 lo = plo[p], hi = phi[p];
                Box3 x;
                x.lo[0] = lo.x, x.lo[1] = lo.y, x.lo[2] = lo.z;
                x.hi[0] = hi.x, x.hi[1] = hi.y, x.hi[2] = hi.z;
                box_grow(bb, x);
                Box3 cc;
                for (int k = 0; k < 3; k++) cc.lo[k] = cc.hi[k] = 0.5f * (x.lo[k] + x.hi[k]);
                box_grow(cb, cc);
            }
            box_reduce_all(bb);
            box_reduce_all(cb);
            float best = FLT_MAX;
            int axis = -1, split = 0, nl = 0;
            if (count > 1) {
                for (int a = 0; a < 3; a++) {
                    const float ext = cb.hi[a] - cb.lo[a];
                    if (!(ext > 0.f)) continue;
                    const float scale = float(kBins) / ext;
                    int cnt = 0;
                    Box3 bx = empty_box();
                    for (int i = 0; i < count; i++) {
                        const int p = ids[first + i];
                        const float4 lo = plo[p], hi = phi[p];
                        const float cc = 0.5f * ((&lo.x)[a] + (&hi.x)[a]);
                        if (bin_of(cc, cb.lo[a], scale) == lane) {
                            cnt++;
                            Box3 x;
                            x.lo[0] = lo.x, x.lo[1] = lo.y, x.lo[2] = lo.z;
                            x.hi[0] = hi.x, x.hi[1] = hi.y, x.hi[2] = hi.z;
                            box_grow(bx, x);
                        }
                    }
                    float c;
                    int s, n;
                    sah_axis(cnt, bx, c, s, n);
                    if (c < best) {
                        best = c;
                        axis = a;
                        split = s;
                        nl = n;
                    }
                }
            }
            const float parent_area = fmaxf(area_of(bb.lo, bb.hi), 1e-30f);
            const bool leaf =
                count <= 1 || (count <= kMaxLeaf && (axis < 0 || float(count) <= 1.0f + best / parent_area));
            Node2 nd;
            for (int k = 0; k < 3; k++) {
                nd.lo[k] = bb.lo[k];
                nd.hi[k] = bb.hi[k];
            }
            nd.first = first;
            nd.count = count;
            nd.left = -1;
            nd.pad[0] = nd.pad[1] = nd.pad[2] = 0;
            if (!leaf) {
                if (axis < 0 || nl <= 0 || nl >= count) {  // identical centroids: split the range
                    axis = -1;
                    nl = count / 2;
                } else {
                    // stable partition of [first, first + count) through tmp
                    const float scale = float(kBins) / (cb.hi[axis] - cb.lo[axis]);
                    int lbase = 0, rbase = nl;
                    for (int base = 0; base < count; base += 32) {
                        const int i = base + lane;
                        const bool valid = i < count;
                        int p = 0;
                        bool left = false;
                        if (valid) {
                            p = ids[first + i];
                            const float4 lo = plo[p], hi = phi[p];
                            left = bin_of(0.5f * ((&lo.x)[axis] + (&hi.x)[axis]), cb.lo[axis], scale) < split;
                        }
                        const unsigned ml = __ballot_sync(0xffffffffu, valid && left);
                        const unsigned mr = __ballot_sync(0xffffffffu, valid && !left);
                        const unsigned lt = (1u << lane) - 1u;
                        if (valid) tmp[first + (left ? lbase + __popc(ml & lt) : rbase + __popc(mr & lt))] = p;
                        lbase += __popc(ml);
                        rbase += __popc(mr);
                    }
                    __syncwarp();
                    for (int i = lane; i < count; i += 32) ids[first + i] = tmp[first + i];
                    __syncwarp();
                }
                if (sp + 2 > kStack) {
                    if (lane == 0) atomicExch(error, 1);  // left as an oversized leaf; the build fails
                } else {
                    int c = 0;
                    if (lane == 0) c = atomicAdd(node_count, 2);
                    c = __shfl_sync(0xffffffffu, c, 0);
                    nd.left = c;
                    if (lane == 0) {
                        stack[wib][sp] = make_int3(c + 1, first + nl, count - nl);
                        stack[wib][sp + 1] = make_int3(c, first, nl);
                    }
                    sp += 2;
                }
            }
            if (lane == 0) nodes[node] = nd;
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------ collapse
struct WideItem {
    int wide, node;
};

RT_D int ilog2ceil_scale(float ext) {
    // smallest e with 255 * 2^e >= ext
    if (!(ext > 0.0f)) return -126;
    int e = int(ceil(log2(double(ext) / 255.0)));
    while (ldexp(255.0, e) < double(ext)) e++;
    while (e > -126 && ldexp(255.0, e - 1) >= double(ext)) e--;
    return max(e, -126);
}

__global__ void k_collapse(const WideItem* __restrict__ items, const int* __restrict__ nitems,
                           const Node2* __restrict__ nodes, const int* __restrict__ ids, rtd::CwNode* __restrict__ out,
                           int* __restrict__ order, int* __restrict__ wide_count, int* __restrict__ tri_count,
                           WideItem* __restrict__ next, int* __restrict__ nnext, int* __restrict__ error, int max_wide,
                           int max_tris) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= *nitems) return;
    const WideItem w = items[it];
    int ch[8];
    int nch = 0;
    const Node2 root = nodes[w.node];
    if (root.left < 0 || root.count <= kMaxLeaf) {
        ch[nch++] = w.node;
    } else {
        ch[nch++] = root.left;
        ch[nch++] = root.left + 1;
        while (nch < 8) {
            int best = -1;
            float ba = -1.0f;
            for (int i = 0; i < nch; i++) {
                const Node2& c = nodes[ch[i]];
                if (c.left < 0) continue;
                const float a = area_of(c.lo, c.hi);
                if (a > ba) {
                    ba = a;
                    best = i;
                }
            }
            if (best < 0) break;
            const int c = ch[best];
            ch[best] = nodes[c].left;
            ch[nch++] = nodes[c].left + 1;
        }
    }
    float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < nch; i++) {
        const Node2& c = nodes[ch[i]];
        for (int a = 0; a < 3; a++) {
            nlo[a] = fminf(nlo[a], c.lo[a]);
            nhi[a] = fmaxf(nhi[a], c.hi[a]);
        }
    }
    float pc[3];
    for (int a = 0; a < 3; a++) pc[a] = 0.5f * (nlo[a] + nhi[a]);
    int slot_of[8];
    unsigned used = 0, done = 0;
    for (int k = 0; k < nch; k++) {
        float best = -FLT_MAX;
        int bi = -1, bs = -1;
        for (int i = 0; i < nch; i++) {
            if ((done >> i) & 1u) continue;
            const Node2& c = nodes[ch[i]];
            float d[3];
            for (int a = 0; a < 3; a++) d[a] = 0.5f * (c.lo[a] + c.hi[a]) - pc[a];
            for (int s = 0; s < 8; s++) {
                if ((used >> s) & 1u) continue;
                const float v = ((s & 1) ? d[0] : -d[0]) + ((s & 2) ? d[1] : -d[1]) + ((s & 4) ? d[2] : -d[2]);
                if (v > best) {
                    best = v;
                    bi = i;
                    bs = s;
                }
            }
        }
        done |= 1u << bi;
        used |= 1u << bs;
        slot_of[bi] = bs;
    }
    int child_at[8];
    for (int s = 0; s < 8; s++) child_at[s] = -1;
    for (int i = 0; i < nch; i++) child_at[slot_of[i]] = ch[i];
    rtd::CwNode node;
    memset(&node, 0, sizeof(node));
    node.px = nlo[0];
    node.py = nlo[1];
    node.pz = nlo[2];
    int e[3];
    for (int a = 0; a < 3; a++) e[a] = ilog2ceil_scale(nhi[a] - nlo[a]);
    node.ex = uint8_t(e[0] + 127);
    node.ey = uint8_t(e[1] + 127);
    node.ez = uint8_t(e[2] + 127);
    int n_internal = 0, n_tris = 0;
    for (int s = 0; s < 8; s++) {
        const int c = child_at[s];
        if (c < 0) continue;
        const Node2& cn = nodes[c];
        if (cn.left < 0 || cn.count <= kMaxLeaf)
            n_tris += cn.count;
        else
            n_internal++;
    }
    const int cb = atomicAdd(wide_count, n_internal);
    const int tb = atomicAdd(tri_count, n_tris);
    if (cb + n_internal > max_wide || tb + n_tris > max_tris || n_tris > 24) {
        atomicExch(error, 2);
        return;
    }
    node.child_base = uint32_t(cb);
    node.tri_base = uint32_t(tb);
    const float p[3] = {node.px, node.py, node.pz};
    uint8_t* qlo[3] = {node.qlox, node.qloy, node.qloz};
    uint8_t* qhi[3] = {node.qhix, node.qhiy, node.qhiz};
    int tri_off = 0, next_child = 0;
    for (int s = 0; s < 8; s++) {
        const int c = child_at[s];
        if (c < 0) {
            node.meta[s] = 0;
            continue;
        }
        const Node2& cn = nodes[c];
        for (int a = 0; a < 3; a++) {
            const double sc = ldexp(1.0, e[a]);
            double lo = floor((double(cn.lo[a]) - double(p[a])) / sc);
            double hi = ceil((double(cn.hi[a]) - double(p[a])) / sc);
            lo = fmin(255.0, fmax(0.0, lo));
            hi = fmin(255.0, fmax(0.0, hi));
            while (lo > 0 && double(p[a]) + lo * sc > double(cn.lo[a])) lo -= 1;
            while (hi < 255 && double(p[a]) + hi * sc < double(cn.hi[a])) hi += 1;
            qlo[a][s] = uint8_t(lo);
            qhi[a][s] = uint8_t(hi);
        }
        if (cn.left < 0 || cn.count <= kMaxLeaf) {
            const int k = cn.count;
            const uint32_t unary = k == 1 ? 1u : (k == 2 ? 3u : 7u);
            node.meta[s] = uint8_t((unary << 5) | uint32_t(tri_off));
            for (int i = 0; i < k; i++) order[tb + tri_off + i] = ids[cn.first + i];
            tri_off += k;
        } else {
            node.imask |= uint8_t(1u << s);
            node.meta[s] = uint8_t((1u << 5) | uint32_t(24 + s));
            next[atomicAdd(nnext, 1)] = WideItem{cb + next_child, c};
            next_child++;
        }
    }
    out[w.wide] = node;
}

}  // namespace rtbg

namespace rth {

namespace {

struct Buf {
    void* p = nullptr;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

#define BG_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            err = std::string("GPU BVH build: ") + cudaGetErrorString(e_);     \
            return false;                                                      \
        }                                                                      \
    } while (0)

int f2o_host(float f) {
    int i;
    std::memcpy(&i, &f, 4);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}

}  // namespace

bool build_cwbvh_gpu(const float* tv, int64_t ntri, BuiltBvh& res, std::string& err, cudaStream_t st) {
    using namespace rtbg;
    res.nodes.clear();
    res.order.clear();
    res.depth = 0;
    if (ntri <= 0) return true;
    if (ntri > (int64_t(1) << 30)) {
        err = "too many triangles for one acceleration structure";
        return false;
    }
    const int n = int(ntri);
    int dev = 0, sms = 148;
    BG_CUDA(cudaGetDevice(&dev));
    BG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int max_large = n / kSmall + 2;
    const int max_chunks = n / kChunk + max_large + 1;
    const int max_nodes = 2 * n + 1;
    Buf d_tv, plo, phi, ids, tmp, nodes, tasks0, tasks1, small, bins, splits, chunks, counters, rootc;
    BG_CUDA(cudaMalloc(&d_tv.p, size_t(n) * 9 * 4));
    BG_CUDA(cudaMalloc(&plo.p, size_t(n) * 16));
    BG_CUDA(cudaMalloc(&phi.p, size_t(n) * 16));
    BG_CUDA(cudaMalloc(&ids.p, size_t(n) * 4));
    BG_CUDA(cudaMalloc(&tmp.p, size_t(n) * 4));
    BG_CUDA(cudaMalloc(&nodes.p, size_t(max_nodes) * sizeof(Node2)));
    BG_CUDA(cudaMalloc(&tasks0.p, size_t(max_large) * sizeof(Task)));
    BG_CUDA(cudaMalloc(&tasks1.p, size_t(max_large) * sizeof(Task)));
    BG_CUDA(cudaMalloc(&small.p, size_t(n) * sizeof(Task)));
    BG_CUDA(cudaMalloc(&bins.p, size_t(max_large) * sizeof(Bins)));
    BG_CUDA(cudaMalloc(&splits.p, size_t(max_large) * sizeof(Split)));
    BG_CUDA(cudaMalloc(&chunks.p, size_t(max_chunks) * sizeof(int2)));
    // counters: 0 node count, 1 large nodes this level, 2 large nodes next level, 3 small nodes, 4 chunks,
    // 5 error, 6 wide nodes, 7 triangles placed, 8 wide items this level, 9 next level, 10 collapse error
    BG_CUDA(cudaMalloc(&counters.p, 16 * 4));
    BG_CUDA(cudaMalloc(&rootc.p, 6 * 4));
    int* cnt = counters.as<int>();
    BG_CUDA(cudaMemcpyAsync(d_tv.p, tv, size_t(n) * 9 * 4, cudaMemcpyHostToDevice, st));
    BG_CUDA(cudaMemsetAsync(counters.p, 0, 16 * 4, st));
    int init[6];
    for (int a = 0; a < 3; a++) {
        init[a] = f2o_host(FLT_MAX);
        init[3 + a] = f2o_host(-FLT_MAX);
    }
    BG_CUDA(cudaMemcpyAsync(rootc.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_prims<<<(n + 255) / 256, 256, 0, st>>>(d_tv.as<float>(), n, plo.as<float4>(), phi.as<float4>(), ids.as<int>(),
                                            rootc.as<int>());
    const int one = 1;
    BG_CUDA(cudaMemcpyAsync(cnt + 0, &one, 4, cudaMemcpyHostToDevice, st));  // node 0 is the root
    if (n > kSmall) {
        k_root_task<<<1, 1, 0, st>>>(rootc.as<int>(), n, tasks0.as<Task>());
        BG_CUDA(cudaMemcpyAsync(cnt + 1, &one, 4, cudaMemcpyHostToDevice, st));
    } else {
        k_root_task<<<1, 1, 0, st>>>(rootc.as<int>(), n, small.as<Task>());
        BG_CUDA(cudaMemcpyAsync(cnt + 3, &one, 4, cudaMemcpyHostToDevice, st));
    }
    Task* cur = tasks0.as<Task>();
    Task* nxt = tasks1.as<Task>();
    int ncur = n > kSmall ? 1 : 0;
    int levels = 0;
    while (ncur > 0) {
        if (++levels > 256) {
            err = "GPU BVH build: too many levels";
            return false;
        }
        BG_CUDA(cudaMemsetAsync(cnt + 2, 0, 4, st));
        k_chunks<<<1, 32, 0, st>>>(cur, cnt + 1, chunks.as<int2>(), cnt + 4, max_chunks);
        k_clear_bins<<<sms * 4, 256, 0, st>>>(bins.as<Bins>(), cnt + 1);
        k_bin<<<sms * 4, 256, 0, st>>>(chunks.as<int2>(), cnt + 4, cur, ids.as<int>(), plo.as<float4>(),
                                       phi.as<float4>(), bins.as<Bins>());
        k_split<<<(ncur * 32 + 127) / 128, 128, 0, st>>>(cur, cnt + 1, bins.as<Bins>(), splits.as<Split>(),
                                                         nodes.as<Node2>(), cnt + 0, nxt, cnt + 2, small.as<Task>(),
                                                         cnt + 3);
        k_partition<<<sms * 4, 256, 0, st>>>(chunks.as<int2>(), cnt + 4, cur, splits.as<Split>(), ids.as<int>(),
                                             tmp.as<int>(), plo.as<float4>(), phi.as<float4>());
        k_copy_back<<<sms * 4, 256, 0, st>>>(chunks.as<int2>(), cnt + 4, cur, tmp.as<int>(), ids.as<int>());
        BG_CUDA(cudaGetLastError());
        BG_CUDA(cudaMemcpyAsync(cnt + 1, cnt + 2, 4, cudaMemcpyDeviceToDevice, st));
        BG_CUDA(cudaMemcpyAsync(&ncur, cnt + 2, 4, cudaMemcpyDeviceToHost, st));
        BG_CUDA(cudaStreamSynchronize(st));
        std::swap(cur, nxt);
    }
    int nsmall = 0;
    BG_CUDA(cudaMemcpyAsync(&nsmall, cnt + 3, 4, cudaMemcpyDeviceToHost, st));
    BG_CUDA(cudaStreamSynchronize(st));
    if (nsmall > 0) {
        const int blocks = (nsmall + 3) / 4 < sms * 16 ? (nsmall + 3) / 4 : sms * 16;
        k_small<<<blocks, 128, 0, st>>>(small.as<Task>(), cnt + 3, ids.as<int>(), tmp.as<int>(), plo.as<float4>(),
                                        phi.as<float4>(), nodes.as<Node2>(), cnt + 0, cnt + 5);
        BG_CUDA(cudaGetLastError());
    }
    int h[6] = {0, 0, 0, 0, 0, 0};
    BG_CUDA(cudaMemcpyAsync(h, cnt, 6 * 4, cudaMemcpyDeviceToHost, st));
    BG_CUDA(cudaStreamSynchronize(st));
    if (h[5]) {
        err = "GPU BVH build: a small subtree is deeper than the build stack";
        return false;
    }
    const int nbvh2 = h[0];
    // collapse, level by level
    Buf wide, order, items0, items1;
    const int max_wide = nbvh2;  // at most one wide node per binary node
    BG_CUDA(cudaMalloc(&wide.p, size_t(max_wide) * sizeof(rtd::CwNode)));
    BG_CUDA(cudaMalloc(&order.p, size_t(n) * 4));
    BG_CUDA(cudaMalloc(&items0.p, size_t(max_wide) * sizeof(WideItem)));
    BG_CUDA(cudaMalloc(&items1.p, size_t(max_wide) * sizeof(WideItem)));
    const WideItem root{0, 0};
    BG_CUDA(cudaMemcpyAsync(items0.p, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    const int init2[5] = {1, 0, 1, 0, 0};  // wide nodes, triangles, items, next items, error
    BG_CUDA(cudaMemcpyAsync(cnt + 6, init2, sizeof(init2), cudaMemcpyHostToDevice, st));
    WideItem* icur = items0.as<WideItem>();
    WideItem* inxt = items1.as<WideItem>();
    int nitems = 1, depth = 0;
    while (nitems > 0) {
        if (++depth > 64) {
            err = "GPU BVH build: collapse too deep";
            return false;
        }
        BG_CUDA(cudaMemsetAsync(cnt + 9, 0, 4, st));
        k_collapse<<<(nitems + 127) / 128, 128, 0, st>>>(icur, cnt + 8, nodes.as<Node2>(), ids.as<int>(),
                                                         wide.as<rtd::CwNode>(), order.as<int>(), cnt + 6, cnt + 7,
                                                         inxt, cnt + 9, cnt + 10, max_wide, n);
        BG_CUDA(cudaGetLastError());
        BG_CUDA(cudaMemcpyAsync(cnt + 8, cnt + 9, 4, cudaMemcpyDeviceToDevice, st));
        BG_CUDA(cudaMemcpyAsync(&nitems, cnt + 9, 4, cudaMemcpyDeviceToHost, st));
        BG_CUDA(cudaStreamSynchronize(st));
        std::swap(icur, inxt);
    }
    int tail[5];
    BG_CUDA(cudaMemcpyAsync(tail, cnt + 6, sizeof(tail), cudaMemcpyDeviceToHost, st));
    BG_CUDA(cudaStreamSynchronize(st));
    if (tail[4]) {
        err = "GPU BVH build: collapse ran out of room";
        return false;
    }
    if (tail[1] != n) {
        err = "GPU BVH build: triangle count mismatch after collapse";
        return false;
    }
    res.nodes.resize(size_t(tail[0]));
    res.order.resize(size_t(n));
    BG_CUDA(cudaMemcpyAsync(res.nodes.data(), wide.p, res.nodes.size() * sizeof(rtd::CwNode), cudaMemcpyDeviceToHost,
                            st));
    BG_CUDA(cudaMemcpyAsync(res.order.data(), order.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st));
    BG_CUDA(cudaStreamSynchronize(st));
    res.depth = depth;
    return true;
}

}  // namespace rth
