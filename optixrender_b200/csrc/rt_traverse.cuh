// rt_traverse.cuh - ray traversal of the compressed 8-wide BVH.
//
// Replaces optixTrace (core/cuda/devicePrograms.cu:258-269 closest hit,
// :303-319 terminate-on-first-hit shadow rays).  Traversal follows Ylitie,
// Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs" (HPG 2017): a node is read as five 16-byte loads, its
// eight quantised child boxes are tested at once, and the hits become a
// 32-bit group mask (bits 24..31 internal children in near-to-far order,
// bits 0..23 triangles) kept on a short per-thread stack.  Triangles use the
// watertight test of Woop, Benthin and Wald (JCGT 2013).
#pragma once

#include "rt_device.cuh"

namespace rtd {

struct TravRay {
    v3 o, d;
    float tmin, tmax;
    v3 idir;        // 1 / d with tiny components clamped
    uint32_t oct;   // bit a set when d[a] < 0: slot index of the nearest child
    int kx, ky, kz; // watertight shear axes
    float Sx, Sy, Sz;
};

RT_D void prepare_ray(TravRay& r) {
    const float tiny = 1e-20f;
    float dx = fabsf(r.d.x) > tiny ? r.d.x : copysignf(tiny, r.d.x);
    float dy = fabsf(r.d.y) > tiny ? r.d.y : copysignf(tiny, r.d.y);
    float dz = fabsf(r.d.z) > tiny ? r.d.z : copysignf(tiny, r.d.z);
    r.idir = v3(1.0f / dx, 1.0f / dy, 1.0f / dz);
    r.oct = (r.d.x < 0.0f ? 1u : 0u) | (r.d.y < 0.0f ? 2u : 0u) | (r.d.z < 0.0f ? 4u : 0u);
    float ax = fabsf(r.d.x), ay = fabsf(r.d.y), az = fabsf(r.d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dkz = r.d[kz];
    if (dkz < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.Sx = __fdiv_rn(r.d[kx], dkz);
    r.Sy = __fdiv_rn(r.d[ky], dkz);
    r.Sz = __fdiv_rn(1.0f, dkz);
}

RT_D float comp(v3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Watertight ray/triangle test.  Products are rounded individually (no FMA
// contraction) so the edge functions match a plain FP32 evaluation.  The
// distance range is tested on the unnormalised T against tmin/tmax * |det|;
// the one division happens only for an accepted hit.
RT_D bool intersect_tri(const TravRay& r, float4 a, float4 b, float4 c, float tmax, float& t, float& b1, float& b2) {
    v3 A = v3(a.x, a.y, a.z) - r.o, B = v3(b.x, b.y, b.z) - r.o, C = v3(c.x, c.y, c.z) - r.o;
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.Sx, Akz)), Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.Sy, Akz));
    float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.Sx, Bkz)), By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.Sy, Bkz));
    float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.Sx, Ckz)), Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
    float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float adet = fabsf(det);
    const float sT = det < 0.0f ? -T : T;
    if (!(sT > 0.99999f * r.tmin * adet && sT < 1.00001f * tmax * adet)) return false;
    float inv = __fdiv_rn(1.0f, det);
    float tt = __fmul_rn(T, inv);
    if (!(tt > r.tmin && tt < tmax)) return false;
    t = tt;
    b1 = __fmul_rn(V, inv);
    b2 = __fmul_rn(W, inv);
    return true;
}

// Byte `byte` of w as the float 2^15 + byte, by one byte permute: the byte
// lands in mantissa bits 8..15 of 2^15 (0x47000000), where one unit is 1.
RT_D float u8f15(uint32_t w, int byte) {
    const uint32_t sel = 4u | (uint32_t(byte) << 4) | (5u << 8) | (7u << 12);
    return __uint_as_float(__byte_perm(w, 0x47000000u, sel));
}

// Byte `byte` of w, zero-extended.
RT_D uint32_t byte_of(uint32_t w, int byte) { return __byte_perm(w, 0u, 0x4440u | uint32_t(byte)); }

// Three-input minimum / maximum (PTX ISA 8.8, sm_100).
RT_D float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
RT_D float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Tests the eight children of `node`; returns the hit mask of internal
// children (bits 24..31, near-to-far) with the node's imask in bits 0..7,
// and the triangle hit mask (bits 0..23) in `tri_bits`.
RT_D uint32_t intersect_children(const CwNode* nodes, uint32_t idx, const TravRay& r, float tmax, uint32_t& child_base,
                                 uint32_t& tri_base, uint32_t& tri_bits) {
    const float4* q = reinterpret_cast<const float4*>(nodes + idx);
    float4 n0 = __ldg(q + 0), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3), n4 = __ldg(q + 4);
    uint32_t e = __float_as_uint(n0.w);
    uint32_t ex = e & 0xFFu, ey = (e >> 8) & 0xFFu, ez = (e >> 16) & 0xFFu, imask = e >> 24;
    child_base = __float_as_uint(n1.x);
    tri_base = __float_as_uint(n1.y);
    uint32_t meta_lo = __float_as_uint(n1.z), meta_hi = __float_as_uint(n1.w);
    // per axis: t = q * (2^e * idir) + (p - o) * idir
    float sx = __uint_as_float(ex << 23) * r.idir.x, sy = __uint_as_float(ey << 23) * r.idir.y,
          sz = __uint_as_float(ez << 23) * r.idir.z;
    float ox = (n0.x - r.o.x) * r.idir.x, oy = (n0.y - r.o.y) * r.idir.y, oz = (n0.z - r.o.z) * r.idir.z;
    // lo / hi planes per axis packed as bytes: qlox n2.xy, qloy n2.zw, qloz n3.xy, qhix n3.zw, qhiy n4.xy, qhiz n4.zw
    uint32_t lox[2] = {__float_as_uint(n2.x), __float_as_uint(n2.y)};
    uint32_t loy[2] = {__float_as_uint(n2.z), __float_as_uint(n2.w)};
    uint32_t loz[2] = {__float_as_uint(n3.x), __float_as_uint(n3.y)};
    uint32_t hix[2] = {__float_as_uint(n3.z), __float_as_uint(n3.w)};
    uint32_t hiy[2] = {__float_as_uint(n4.x), __float_as_uint(n4.y)};
    uint32_t hiz[2] = {__float_as_uint(n4.z), __float_as_uint(n4.w)};
    // near plane = lo when the direction is positive
    const bool nx = r.idir.x >= 0.0f, ny = r.idir.y >= 0.0f, nz = r.idir.z >= 0.0f;
    // t = (2^15 + q) * s + (o - 2^15 s): one FFMA per plane after the byte
    // permute.  The folded offset carries a rounding error of at most
    // |2^15 s| * 2^-24 = |s| / 512 per rounding (plus an |o|-relative part
    // the far-distance epsilon below covers), so near planes move in and far
    // planes out by |s| / 128, 1/128 of a quantisation step (+1.4% paths/s).
    const float cx = fmaf(-32768.0f, sx, ox), cy = fmaf(-32768.0f, sy, oy), cz = fmaf(-32768.0f, sz, oz);
    const float wx = fabsf(sx) * (1.0f / 128.0f), wy = fabsf(sy) * (1.0f / 128.0f), wz = fabsf(sz) * (1.0f / 128.0f);
    const float cxn = cx - wx, cxf = cx + wx, cyn = cy - wy, cyf = cy + wy, czn = cz - wz, czf = cz + wz;
    uint32_t hits = 0;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        // A child's meta byte is (bits << 5) | index: an internal child has
        // bits 1 and index 24 + slot, a leaf child its triangles' unary mask
        // and the bit of its first triangle (< 24), an empty slot 0.  Internal
        // children (index >= 24: bits 3 and 4 set, which no leaf index has)
        // get the ray octant XORed into the slot, so bits 24..31 of the hit
        // mask come out in near-to-far order.  Four children per 32-bit word.
        const uint32_t m = half == 0 ? meta_lo : meta_hi;
        const uint32_t inner = m & (m << 1) & 0x10101010u;
        const uint32_t idx4 = (m ^ ((inner >> 4) * r.oct)) & 0x1F1F1F1Fu;
        const uint32_t bits4 = (m >> 5) & 0x07070707u;
        uint32_t xn = nx ? lox[half] : hix[half], xf = nx ? hix[half] : lox[half];
        uint32_t yn = ny ? loy[half] : hiy[half], yf = ny ? hiy[half] : loy[half];
        uint32_t zn = nz ? loz[half] : hiz[half], zf = nz ? hiz[half] : loz[half];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            float tx0 = fmaf(u8f15(xn, b), sx, cxn), tx1 = fmaf(u8f15(xf, b), sx, cxf);
            float ty0 = fmaf(u8f15(yn, b), sy, cyn), ty1 = fmaf(u8f15(yf, b), sy, cyf);
            float tz0 = fmaf(u8f15(zn, b), sz, czn), tz1 = fmaf(u8f15(zf, b), sz, czf);
            float tn = max3f(tx0, ty0, fmaxf(tz0, r.tmin));
            float tf = min3f(tx1, ty1, fminf(tz1, tmax));
            // conservative: the far distance is widened by 1.6e-6 relative
            // (tn >= tmin >= 0), covering the rounding of the slab distances;
            // an empty slot adds no bits whatever its planes
            if (tn <= tf * 1.0000016f) hits |= byte_of(bits4, b) << byte_of(idx4, b);
        }
    }
    tri_bits = hits & 0x00FFFFFFu;
    return (hits & 0xFF000000u) | imask;
}

// Returns the index of the closest hit triangle (or -1) in [tmin, tmax).
// `nodes_visited` / `tris_tested` are only updated when Stats is true.
// `overflows` counts node groups that found the stack full (their subtrees
// are not visited); the renderer rejects BVHs deeper than the stack, so it
// stays zero unless that check is broken, and callers report it as an error.
template <bool AnyHit, bool Stats>
RT_D int traverse(const SceneView& sc, TravRay& r, float& t_hit, float& b1, float& b2, uint32_t& nodes_visited,
                  uint32_t& tris_tested, uint32_t& overflows) {
    int hit_tri = -1;
    float tmax = r.tmax;
    if (sc.num_nodes <= 0) return -1;
    uint2 stack[kStackSize];
    int sp = 0;
    // node group: x = base node index, y = internal hit bits (24..31) | parent imask (0..7)
    uint2 g = make_uint2(0u, 1u << (24 + r.oct));
    // Invariant at the top of the loop: g holds at least one internal-child bit.
    while (true) {
        uint32_t bit = __ffs(g.y >> 24) - 1u;
        g.y &= ~(1u << (24 + bit));
        uint32_t slot = bit ^ r.oct;
        uint32_t idx = g.x + __popc((g.y & 0xFFu) & ((1u << slot) - 1u));
        if (g.y & 0xFF000000u) {
            if (sp < kStackSize)
                stack[sp++] = g;
            else
                overflows++;
        }
        uint32_t cb, tb, tbits;
        uint32_t nb = intersect_children(sc.nodes, idx, r, tmax, cb, tb, tbits);
        if (Stats) nodes_visited++;
        g = make_uint2(cb, nb);
        while (tbits) {
            uint32_t b = __ffs(tbits) - 1u;
            tbits &= ~(1u << b);
            uint32_t ti = tb + b;
            const float4* tv = sc.tri_v + size_t(ti) * 3;
            float4 a = __ldg(tv), bb = __ldg(tv + 1), c = __ldg(tv + 2);
            if (Stats) tris_tested++;
            float t, u, v;
            if (intersect_tri(r, a, bb, c, tmax, t, u, v)) {
                hit_tri = int(ti);
                tmax = t;
                t_hit = t;
                b1 = u;
                b2 = v;
                if (AnyHit) return hit_tri;
            }
        }
        while (!(g.y & 0xFF000000u)) {
            if (sp == 0) return hit_tri;
            g = stack[--sp];
        }
    }
    return hit_tri;
}

// ------------------------------------------------------------------ persistent traversal
// Lane-refill ("while-while with dynamic fetch", Aila and Laine, HPG 2009):
// every lane traverses its own ray one wide node at a time; when enough lanes
// of a warp have finished, they take new rays from the queue with a single
// warp-aggregated atomicAdd, so a warp never waits for its slowest ray while
// work remains.  `src.load(i, ray, scene)` fetches queue entry i;
// `src.finish(fin, i, tri, t, b1, b2, tri_v)` is called by the whole warp after
// every step and stores the result of the lanes whose `fin` is set.
// Measured on the 2.59M-triangle scene: with one setting for both kernels,
// refilling at 12 idle lanes beat 4, 8 and 16 and postponing triangles below
// 20% of the lanes beat 10, 15, 30 and 40.  Apart (per benchmark step):
// closest-hit rays do best at 12 lanes and 12% (k_extend 63.6 -> 63.0 ms;
// 8% or 16 lanes 63.5 ms), shadow rays at 8 lanes and 30% (k_shadow 20.2 ->
// 19.5 ms).
constexpr int kRefillLanesClosest = 12;
constexpr int kRefillLanesAny = 8;
constexpr int kPostponePercentClosest = 12;
constexpr int kPostponePercentAny = 30;
// Threads per block of the persistent traversal kernels.
constexpr int kTravBlock = 128;
// Stack entries with this bit in x are postponed triangle groups
// (x = first triangle, y = triangle hit bits), not node groups.
constexpr uint32_t kTriGroup = 0x80000000u;

// The per-thread traversal stack (local memory; a shared-memory stack
// measured no faster).
struct TravStack {
    uint2 e[kStackSize];
    int sp;
    RT_D void push(uint2 v) { e[sp++] = v; }
    RT_D uint2 pop() { return e[--sp]; }
};

struct TravState {
    TravRay r;
    const CwNode* nodes;
    const float4* tri_v;
    // Postponed triangle groups may fill the stack only up to kStackSize -
    // BVH depth: node groups on the stack are at most one per level of the
    // current path, so they always find room.
    int tri_room;
    uint2 g;
    float tmax;
    float t, b1, b2;
    int hit;
};

// One wide node (or one postponed triangle group) and its triangles; returns
// true when the ray is finished.  `overflows` as in traverse().
template <bool AnyHit, bool Stats>
RT_D bool trav_step(TravState& s, TravStack& st, uint32_t& nodes_visited, uint32_t& tris_tested, uint32_t& overflows) {
    uint32_t tb, tbits;
    if (s.g.x & kTriGroup) {
        tb = s.g.x & ~kTriGroup;
        tbits = s.g.y;
        s.g = make_uint2(0u, 0u);
    } else {
        uint32_t bit = __ffs(s.g.y >> 24) - 1u;
        s.g.y &= ~(1u << (24 + bit));
        uint32_t slot = bit ^ s.r.oct;
        uint32_t idx = s.g.x + __popc((s.g.y & 0xFFu) & ((1u << slot) - 1u));
        if (s.g.y & 0xFF000000u) {
            if (st.sp < kStackSize)
                st.push(s.g);
            else
                overflows++;
        }
        uint32_t cb;
        uint32_t nb = intersect_children(s.nodes, idx, s.r, s.tmax, cb, tb, tbits);
        if (Stats) nodes_visited++;
        s.g = make_uint2(cb, nb);
    }
    // Triangle postponing (Ylitie et al. 2017): when fewer than the
    // postponing percentage of the lanes in this step still test triangles,
    // the rest of the group goes on the stack and the lane returns to node
    // traversal with the others (+7% paths/s on the 2.59M-triangle scene).
    constexpr int kPostpone = AnyHit ? kPostponePercentAny : kPostponePercentClosest;
    const int n_step = __popc(__activemask());
    while (tbits) {
        if (__popc(__activemask()) * 100 < kPostpone * n_step && st.sp < s.tri_room) {
            st.push(make_uint2(tb | kTriGroup, tbits));
            break;
        }
        uint32_t b = __ffs(tbits) - 1u;
        tbits &= ~(1u << b);
        uint32_t ti = tb + b;
        const float4* tv = s.tri_v + size_t(ti) * 3;
        float4 a = __ldg(tv), bb = __ldg(tv + 1), c = __ldg(tv + 2);
        if (Stats) tris_tested++;
        float t, u, v;
        if (intersect_tri(s.r, a, bb, c, s.tmax, t, u, v)) {
            s.hit = int(ti);
            s.tmax = t;
            s.t = t;
            s.b1 = u;
            s.b2 = v;
            if (AnyHit) return true;
        }
    }
    while (!(s.g.x & kTriGroup) && !(s.g.y & 0xFF000000u)) {
        if (st.sp == 0) return true;
        s.g = st.pop();
    }
    return false;
}

template <bool AnyHit, bool Stats, class Src>
RT_D void traverse_queue(Src& src, int* fetch_counter, int total, uint32_t& nodes_visited, uint32_t& tris_tested,
                         uint32_t& rays, uint32_t& overflows) {
    constexpr int kRefillLanes = AnyHit ? kRefillLanesAny : kRefillLanesClosest;
    const int lane = threadIdx.x & 31;
    TravStack st;
    st.sp = 0;
    TravState s;
    int item = -1;
    bool active = false, exhausted = false;
    while (true) {
        bool fin = false;
        unsigned idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && idle && (__popc(idle) >= kRefillLanes || idle == 0xffffffffu)) {
            int leader = __ffs(idle) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(fetch_counter, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= total) exhausted = true;
            if (!active) {
                int my = base + __popc(idle & ((1u << lane) - 1u));
                if (my < total) {
                    item = my;
                    const SceneView* sc = nullptr;
                    src.load(item, s.r, sc);
                    prepare_ray(s.r);
                    s.nodes = sc->nodes;
                    s.tri_v = sc->tri_v;
                    s.tri_room = kStackSize - sc->bvh_depth;
                    s.tmax = s.r.tmax;
                    s.hit = -1;
                    st.sp = 0;
                    s.g = make_uint2(0u, 1u << (24 + s.r.oct));
                    rays++;
                    if (sc->num_nodes > 0)
                        active = true;
                    else
                        fin = true;  // empty scene: a miss
                }
            }
        }
        if (active && trav_step<AnyHit, Stats>(s, st, nodes_visited, tris_tested, overflows)) {
            fin = true;
            active = false;
        }
        // called by the whole warp; lanes with `fin` store their result
        src.finish(fin, item, s.hit, s.t, s.b1, s.b2, s.tri_v);
        if (__ballot_sync(0xffffffffu, active) == 0 && exhausted) break;
    }
}

}  // namespace rtd
