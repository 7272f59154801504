// rt_bvh.cpp - acceleration structure build (replaces optixAccelBuild +
// optixAccelCompact, core/src/Renderer.cpp:146-285).
//
// 1. Binned SAH binary BVH (32 bins per axis, 3 axes, leaves of at most three
//    triangles), built top-down with OpenMP tasks.
// 2. Collapse into 8-wide nodes: a node opens its largest-area children until
//    it has eight slots; subtrees of at most three triangles become leaf slots.
// 3. Children are assigned to slots so that slot s holds the child furthest
//    along the octant direction of s; traversal visits slots in the order
//    slot ^ ray_octant, which is approximately near to far.
// 4. Child boxes are quantised to 8 bits per plane relative to the node box,
//    rounded outwards (Ylitie, Karras, Laine, HPG 2017).
#include "rt_bvh.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

namespace rth {
namespace {

struct Box {
    float lo[3], hi[3];
    void reset() {
        for (int a = 0; a < 3; a++) {
            lo[a] = INFINITY;
            hi[a] = -INFINITY;
        }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    float area() const {
        float d[3];
        for (int a = 0; a < 3; a++) d[a] = std::max(0.0f, hi[a] - lo[a]);
        return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct Node2 {
    Box box;
    int left, right;  // -1 for leaves
    int first, count;
};

constexpr int kBins = 32;
constexpr int kMaxLeaf = 3;

// Bin of a centroid coordinate, saturating like the device build's float to
// int conversion: a node whose centroid extent is so small that kBins / extent
// overflows to infinity gives NaN (c == cmin) or infinity here, and both must
// land in a valid bin.
inline int bin_of(float c, float cmin, float scale) {
    const float f = (c - cmin) * scale;
    if (!(f > 0.0f)) return 0;  // also NaN
    if (f >= float(kBins - 1)) return kBins - 1;
    return int(f);
}

struct Builder {
    const float* tv;
    std::vector<Box> pbox;
    std::vector<float> cen;  // 3 per prim
    std::vector<int> prims;
    std::vector<Node2> nodes;
    std::atomic<int> next{1};

    int alloc2() { return next.fetch_add(2); }

    void bounds(int first, int count, Box& b, Box& cb) {
        b.reset();
        cb.reset();
        if (count > 65536) {
            int nt = omp_get_max_threads();
            std::vector<Box> pb(nt), pc(nt);
            for (int t = 0; t < nt; t++) {
                pb[t].reset();
                pc[t].reset();
            }
#pragma omp parallel for schedule(static)
            for (int i = first; i < first + count; i++) {
                int t = omp_get_thread_num();
                int p = prims[size_t(i)];
                pb[t].grow(pbox[size_t(p)]);
                pc[t].grow(&cen[size_t(p) * 3]);
            }
            for (int t = 0; t < nt; t++) {
                b.grow(pb[t]);
                cb.grow(pc[t]);
            }
            return;
        }
        for (int i = first; i < first + count; i++) {
            int p = prims[size_t(i)];
            b.grow(pbox[size_t(p)]);
            cb.grow(&cen[size_t(p) * 3]);
        }
    }

    void build(int ni, int first, int count) {
        Box b, cb;
        bounds(first, count, b, cb);
        Node2& n = nodes[size_t(ni)];
        n.box = b;
        n.first = first;
        n.count = count;
        n.left = n.right = -1;
        if (count <= 1) return;
        // binned SAH over the three axes
        float best_cost = INFINITY;
        int best_axis = -1, best_split = -1;
        for (int a = 0; a < 3; a++) {
            float ext = cb.hi[a] - cb.lo[a];
            if (!(ext > 0.0f)) continue;
            float scale = float(kBins) / ext;
            Box bb[kBins];
            int bc[kBins];
            for (int k = 0; k < kBins; k++) {
                bb[k].reset();
                bc[k] = 0;
            }
            for (int i = first; i < first + count; i++) {
                int p = prims[size_t(i)];
                int k = bin_of(cen[size_t(p) * 3 + a], cb.lo[a], scale);
                bb[k].grow(pbox[size_t(p)]);
                bc[k]++;
            }
            float ra[kBins];
            int rc[kBins];
            Box acc;
            acc.reset();
            int cnt = 0;
            for (int k = kBins - 1; k > 0; k--) {
                acc.grow(bb[k]);
                cnt += bc[k];
                ra[k] = acc.area();
                rc[k] = cnt;
            }
            acc.reset();
            cnt = 0;
            for (int k = 0; k < kBins - 1; k++) {
                acc.grow(bb[k]);
                cnt += bc[k];
                if (cnt == 0 || rc[k + 1] == 0) continue;
                float c = acc.area() * float(cnt) + ra[k + 1] * float(rc[k + 1]);
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_split = k + 1;
                }
            }
        }
        float parent_area = std::max(b.area(), 1e-30f);
        float leaf_cost = float(count);
        float split_cost = 1.0f + best_cost / parent_area;
        if (count <= kMaxLeaf && (best_axis < 0 || leaf_cost <= split_cost)) return;
        int mid;
        if (best_axis < 0) {
            mid = first + count / 2;  // identical centroids: split the range
        } else {
            int a = best_axis;
            float scale = float(kBins) / (cb.hi[a] - cb.lo[a]);
            float lo = cb.lo[a];
            auto it = std::partition(prims.begin() + first, prims.begin() + first + count, [&](int p) {
                return bin_of(cen[size_t(p) * 3 + a], lo, scale) < best_split;
            });
            mid = int(it - prims.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        }
        int l = alloc2();
        n.left = l;
        n.right = l + 1;
        int lc = mid - first, rcnt = first + count - mid;
        if (count > 4096) {
#pragma omp task default(shared) firstprivate(l, first, lc)
            build(l, first, lc);
#pragma omp task default(shared) firstprivate(l, mid, rcnt)
            build(l + 1, mid, rcnt);
#pragma omp taskwait
        } else {
            build(l, first, lc);
            build(l + 1, mid, rcnt);
        }
    }
};

int ilog2ceil_scale(float ext) {
    // smallest e with 255 * 2^e >= ext
    if (!(ext > 0.0f)) return -126;
    int e = int(std::ceil(std::log2(double(ext) / 255.0)));
    while (std::ldexp(255.0, e) < double(ext)) e++;
    while (e > -126 && std::ldexp(255.0, e - 1) >= double(ext)) e--;
    return std::max(e, -126);
}

struct Collapser {
    const Builder& b;
    std::vector<rtd::CwNode>& out;
    std::vector<int>& order;
    std::vector<Box> wbox;  // true bounds of each wide node
    int max_depth = 0;

    Collapser(const Builder& bb, std::vector<rtd::CwNode>& o, std::vector<int>& ord) : b(bb), out(o), order(ord) {}

    void gather(int ni, std::vector<int>& tris) const {
        const Node2& n = b.nodes[size_t(ni)];
        for (int i = n.first; i < n.first + n.count; i++) tris.push_back(b.prims[size_t(i)]);
    }

    // Fills wide node `wi` from binary node `ni`; returns the binary nodes of
    // its internal children (in slot order) so the caller can recurse.
    void fill(int wi, int ni, std::vector<std::pair<int, int>>& todo) {
        std::vector<int> ch;
        const Node2& root = b.nodes[size_t(ni)];
        if (root.left < 0 || root.count <= kMaxLeaf) {
            ch.push_back(ni);
        } else {
            ch.push_back(root.left);
            ch.push_back(root.right);
            while (ch.size() < 8) {
                int best = -1;
                float ba = -1.0f;
                for (size_t i = 0; i < ch.size(); i++) {
                    const Node2& c = b.nodes[size_t(ch[i])];
                    if (c.left < 0) continue;
                    float a = c.box.area();
                    if (a > ba) {
                        ba = a;
                        best = int(i);
                    }
                }
                if (best < 0) break;
                int c = ch[size_t(best)];
                ch[size_t(best)] = b.nodes[size_t(c)].left;
                ch.push_back(b.nodes[size_t(c)].right);
            }
        }
        // node box and octant slot assignment
        Box nb;
        nb.reset();
        for (int c : ch) nb.grow(b.nodes[size_t(c)].box);
        float pc[3];
        for (int a = 0; a < 3; a++) pc[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
        int slot_of[8];
        bool used_slot[8] = {false, false, false, false, false, false, false, false};
        bool done[8] = {false, false, false, false, false, false, false, false};
        for (size_t it = 0; it < ch.size(); it++) {
            float best = -INFINITY;
            int bi = -1, bs = -1;
            for (size_t i = 0; i < ch.size(); i++) {
                if (done[i]) continue;
                const Box& cbx = b.nodes[size_t(ch[i])].box;
                float d[3];
                for (int a = 0; a < 3; a++) d[a] = 0.5f * (cbx.lo[a] + cbx.hi[a]) - pc[a];
                for (int s = 0; s < 8; s++) {
                    if (used_slot[s]) continue;
                    float v = ((s & 1) ? d[0] : -d[0]) + ((s & 2) ? d[1] : -d[1]) + ((s & 4) ? d[2] : -d[2]);
                    if (v > best) {
                        best = v;
                        bi = int(i);
                        bs = s;
                    }
                }
            }
            done[bi] = true;
            used_slot[bs] = true;
            slot_of[bi] = bs;
        }
        int child_at[8];
        for (int s = 0; s < 8; s++) child_at[s] = -1;
        for (size_t i = 0; i < ch.size(); i++) child_at[slot_of[i]] = ch[i];

        rtd::CwNode node;
        std::memset(&node, 0, sizeof(node));
        node.px = nb.lo[0];
        node.py = nb.lo[1];
        node.pz = nb.lo[2];
        int e[3];
        for (int a = 0; a < 3; a++) e[a] = ilog2ceil_scale(nb.hi[a] - nb.lo[a]);
        node.ex = uint8_t(e[0] + 127);
        node.ey = uint8_t(e[1] + 127);
        node.ez = uint8_t(e[2] + 127);
        // internal children first (contiguous), then leaf triangles
        int n_internal = 0;
        for (int s = 0; s < 8; s++) {
            int c = child_at[s];
            if (c < 0) continue;
            const Node2& cn = b.nodes[size_t(c)];
            if (!(cn.left < 0 || cn.count <= kMaxLeaf)) n_internal++;
        }
        node.child_base = uint32_t(out.size());
        node.tri_base = uint32_t(order.size());
        out.resize(out.size() + size_t(n_internal));
        int tri_off = 0;
        int next_child = 0;
        const float p[3] = {node.px, node.py, node.pz};
        uint8_t* qlo[3] = {node.qlox, node.qloy, node.qloz};
        uint8_t* qhi[3] = {node.qhix, node.qhiy, node.qhiz};
        for (int s = 0; s < 8; s++) {
            int c = child_at[s];
            if (c < 0) {
                node.meta[s] = 0;
                continue;
            }
            const Node2& cn = b.nodes[size_t(c)];
            for (int a = 0; a < 3; a++) {
                double sc = std::ldexp(1.0, e[a]);
                double lo = std::floor((double(cn.box.lo[a]) - double(p[a])) / sc);
                double hi = std::ceil((double(cn.box.hi[a]) - double(p[a])) / sc);
                lo = std::min(255.0, std::max(0.0, lo));
                hi = std::min(255.0, std::max(0.0, hi));
                while (lo > 0 && double(p[a]) + lo * sc > double(cn.box.lo[a])) lo -= 1;
                while (hi < 255 && double(p[a]) + hi * sc < double(cn.box.hi[a])) hi += 1;
                qlo[a][s] = uint8_t(lo);
                qhi[a][s] = uint8_t(hi);
            }
            if (cn.left < 0 || cn.count <= kMaxLeaf) {
                std::vector<int> tris;
                gather(c, tris);
                int k = int(tris.size());
                uint32_t unary = k == 1 ? 1u : (k == 2 ? 3u : 7u);
                node.meta[s] = uint8_t((unary << 5) | uint32_t(tri_off));
                for (int t : tris) order.push_back(t);
                tri_off += k;
            } else {
                node.imask |= uint8_t(1u << s);
                node.meta[s] = uint8_t((1u << 5) | uint32_t(24 + s));
                todo.push_back({int(node.child_base) + next_child, c});
                next_child++;
            }
        }
        out[size_t(wi)] = node;
        if (wbox.size() < out.size()) wbox.resize(out.size());
        wbox[size_t(wi)] = nb;
        for (int s = 0; s < 8; s++) {
            int c = child_at[s];
            if (c >= 0 && ((node.imask >> s) & 1u)) {
                int rank = 0;
                for (int q = 0; q < s; q++) rank += (node.imask >> q) & 1u;
                wbox[size_t(node.child_base) + size_t(rank)] = b.nodes[size_t(c)].box;
            }
        }
    }
};

// Checks that every index a traversal can form stays in range and that each
// quantised child box contains the child it stands for.
bool validate(const std::vector<rtd::CwNode>& nodes, const std::vector<int>& order, const std::vector<Box>& wbox,
              const float* tv, std::string& err) {
    const size_t nn = nodes.size(), nt = order.size();
    for (size_t i = 0; i < nn; i++) {
        const rtd::CwNode& n = nodes[i];
        const float p[3] = {n.px, n.py, n.pz};
        const int e[3] = {int(n.ex) - 127, int(n.ey) - 127, int(n.ez) - 127};
        const uint8_t* qlo[3] = {n.qlox, n.qloy, n.qloz};
        const uint8_t* qhi[3] = {n.qhix, n.qhiy, n.qhiz};
        int rank = 0;
        for (int s = 0; s < 8; s++) {
            if (n.meta[s] == 0) {
                if ((n.imask >> s) & 1u) {
                    err = "internal slot without meta";
                    return false;
                }
                continue;
            }
            double lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
                lo[a] = double(p[a]) + std::ldexp(double(qlo[a][s]), e[a]);
                hi[a] = double(p[a]) + std::ldexp(double(qhi[a][s]), e[a]);
            }
            auto inside = [&](const float* v) {
                for (int a = 0; a < 3; a++)
                    if (double(v[a]) < lo[a] || double(v[a]) > hi[a]) return false;
                return true;
            };
            if ((n.imask >> s) & 1u) {
                size_t c = size_t(n.child_base) + size_t(rank++);
                if (c >= nn || c == i) {
                    err = "child index out of range";
                    return false;
                }
                const Box& cb = wbox[c];
                if (!inside(cb.lo) || !inside(cb.hi)) {
                    err = "quantised box does not contain its child node";
                    return false;
                }
                if ((n.meta[s] & 31u) != uint32_t(24 + s) || (n.meta[s] >> 5) != 1u) {
                    err = "bad internal meta";
                    return false;
                }
            } else {
                uint32_t unary = n.meta[s] >> 5, off = n.meta[s] & 31u;
                int cnt = unary == 1 ? 1 : unary == 3 ? 2 : unary == 7 ? 3 : 0;
                if (cnt == 0 || off + uint32_t(cnt) > 24 || size_t(n.tri_base) + off + size_t(cnt) > nt) {
                    err = "leaf triangle range out of bounds";
                    return false;
                }
                for (int k = 0; k < cnt; k++) {
                    const float* t = tv + size_t(order[size_t(n.tri_base) + off + size_t(k)]) * 9;
                    if (!inside(t) || !inside(t + 3) || !inside(t + 6)) {
                        err = "quantised box does not contain its triangles";
                        return false;
                    }
                }
            }
        }
    }
    return true;
}

// True bounds of wide node i from its triangles and children (post-order).
void wide_bounds(const std::vector<rtd::CwNode>& nodes, const std::vector<int>& order, const float* tv, size_t i,
                 std::vector<Box>& wbox, std::vector<char>& done, int depth, bool& ok) {
    if (depth > 64 || i >= nodes.size()) {
        ok = false;
        return;
    }
    const rtd::CwNode& n = nodes[i];
    Box b;
    b.reset();
    int rank = 0;
    for (int s = 0; s < 8; s++) {
        if (n.meta[s] == 0) continue;
        if ((n.imask >> s) & 1u) {
            size_t c = size_t(n.child_base) + size_t(rank++);
            if (c >= nodes.size() || c == i) {
                ok = false;
                return;
            }
            if (!done[c]) wide_bounds(nodes, order, tv, c, wbox, done, depth + 1, ok);
            if (!ok) return;
            b.grow(wbox[c]);
        } else {
            uint32_t unary = n.meta[s] >> 5, off = n.meta[s] & 31u;
            int cnt = unary == 1 ? 1 : unary == 3 ? 2 : unary == 7 ? 3 : 0;
            for (int k = 0; k < cnt; k++) {
                size_t slot = size_t(n.tri_base) + off + size_t(k);
                if (slot >= order.size()) {
                    ok = false;
                    return;
                }
                const float* t = tv + size_t(order[slot]) * 9;
                b.grow(t);
                b.grow(t + 3);
                b.grow(t + 6);
            }
        }
    }
    wbox[i] = b;
    done[i] = 1;
}

}  // namespace

bool validate_cwbvh(const BuiltBvh& bvh, const float* tv, int64_t ntri, std::string& err) {
    if (int64_t(bvh.order.size()) != ntri) {
        err = "triangle count mismatch";
        return false;
    }
    std::vector<char> seen(size_t(ntri), 0);
    for (int t : bvh.order) {
        if (t < 0 || t >= ntri || seen[size_t(t)]) {
            err = "triangle order is not a permutation";
            return false;
        }
        seen[size_t(t)] = 1;
    }
    if (bvh.nodes.empty()) return ntri == 0;
    std::vector<Box> wbox(bvh.nodes.size());
    std::vector<char> done(bvh.nodes.size(), 0);
    bool ok = true;
    wide_bounds(bvh.nodes, bvh.order, tv, 0, wbox, done, 0, ok);
    if (!ok) {
        err = "child or triangle index out of range";
        return false;
    }
    for (size_t i = 0; i < done.size(); i++)
        if (!done[i]) {
            err = "unreachable wide node";
            return false;
        }
    return validate(bvh.nodes, bvh.order, wbox, tv, err);
}

bool build_cwbvh(const float* tv, int64_t ntri, BuiltBvh& res, std::string& err) {
    res.nodes.clear();
    res.order.clear();
    res.depth = 0;
    if (ntri <= 0) return true;
    if (ntri > (int64_t(1) << 30)) {
        err = "too many triangles for one acceleration structure";
        return false;
    }
    Builder b;
    b.tv = tv;
    b.pbox.resize(size_t(ntri));
    b.cen.resize(size_t(ntri) * 3);
    b.prims.resize(size_t(ntri));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ntri; i++) {
        Box bx;
        bx.reset();
        bx.grow(tv + i * 9);
        bx.grow(tv + i * 9 + 3);
        bx.grow(tv + i * 9 + 6);
        b.pbox[size_t(i)] = bx;
        for (int a = 0; a < 3; a++) b.cen[size_t(i) * 3 + a] = 0.5f * (bx.lo[a] + bx.hi[a]);
        b.prims[size_t(i)] = int(i);
    }
    b.nodes.resize(size_t(2 * ntri + 1));
#pragma omp parallel
#pragma omp single
    b.build(0, 0, int(ntri));
    b.nodes.resize(size_t(b.next.load()));

    Collapser c(b, res.nodes, res.order);
    res.nodes.resize(1);
    std::vector<std::pair<int, int>> todo, next;
    todo.push_back({0, 0});
    int depth = 0;
    while (!todo.empty()) {
        depth++;
        next.clear();
        for (auto& w : todo) c.fill(w.first, w.second, next);
        todo.swap(next);
    }
    res.depth = depth;
    if (int64_t(res.order.size()) != ntri) {
        err = "internal error: triangle count mismatch after collapse";
        return false;
    }
    std::vector<char> seen(size_t(ntri), 0);
    for (int t : res.order) {
        if (t < 0 || t >= ntri || seen[size_t(t)]) {
            err = "internal error: triangle order is not a permutation";
            return false;
        }
        seen[size_t(t)] = 1;
    }
    return validate(res.nodes, res.order, c.wbox, tv, err);
}

}  // namespace rth
