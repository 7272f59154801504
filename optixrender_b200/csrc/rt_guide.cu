// rt_guide.cu - fused kernels of the path-guiding network.
//
// Inference (the renderer's per-vertex mixtures and rt_guide_forward) runs
// on the 5th-generation tensor cores: tcgen05.mma with FP32 accumulators in
// tensor memory, 128 queries per CTA (k_guide_forward_tc, k_guide_infer_tc).
// Training runs on warp-level MMA as follows.
//
// One warp runs 16 queries at a time through the whole network with
// mma.sync.m16n8k16 (FP16 operands, FP32 accumulation): the hash-grid
// features are gathered straight into the A fragments of the first layer,
// every layer's accumulators are repacked in registers as the next layer's A
// fragments, and the weights sit in shared memory (rows padded by 8 halves so
// that a fragment load hits 32 different banks).  Training runs forward, loss
// gradient, backward and weight gradients in the same kernel: deltas stay in
// registers, the weight gradients are products of transposed fragments
// (movmatrix), accumulated in shared memory and added to global memory once
// per block, and the hash-grid gradient is scattered with float2 atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "rt_guide.cuh"
#include "rt_guide_host.h"
#include "rt_kernels.cuh"

namespace rtg {

namespace {

constexpr int kBwdWarps = 8;  // training pass: 2 blocks of 8 warps per SM (registers, shared weights)
// padded shared-memory rows (halves)
constexpr int kS32 = kIn + 8;   // rows of 32 inputs
constexpr int kS64 = kHid + 8;  // rows of 64 inputs
// forward weights: W0 [64][40], W1 [64][72], W2 [64][72], W3 [32][72]
constexpr int kOffW0 = 0, kOffW1 = kOffW0 + kHid * kS32, kOffW2 = kOffW1 + kHid * kS64, kOffW3 = kOffW2 + kHid * kS64;
constexpr int kFwdHalves = kOffW3 + kOut * kS64;
// transposed weights for the backward pass: W3T [64][40], W2T [64][72], W1T [64][72], W0T [32][72]
constexpr int kOffT3 = 0, kOffT2 = kOffT3 + kHid * kS32, kOffT1 = kOffT2 + kHid * kS64, kOffT0 = kOffT1 + kHid * kS64;
constexpr int kBwdHalves = kOffT0 + kIn * kS64;
constexpr int kTileStride = kOut + 1;  // per-warp 16 x 33 float staging tile
constexpr int kShadeBucketsG = 6;      // shade buckets of guided material types

RT_D void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

RT_D uint32_t pack_h2(float lo, float hi) {
    __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}
RT_D float2 unpack_h2(uint32_t x) { return __half22float2(*reinterpret_cast<__half2*>(&x)); }

RT_D uint32_t trans8x8(uint32_t x) {
    uint32_t y;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(y) : "r"(x));
    return y;
}

// Two 8x8 FP16 matrices from shared memory in mma fragment order: lane i
// (and i + 8) gives the address of row i & 7 of matrix (i >> 3) & 1; register
// m receives matrix m's fragment (row g, columns 2 tig and 2 tig + 1 for
// lane 4 g + tig).
RT_D void ldsm_x2(const __half* p, uint32_t& r0, uint32_t& r1) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}

// d[j] = A (16 x K) * W^T (K x N) for the weight W [N][K] in shared memory,
// row stride S halves (a multiple of 8, so every row starts on 16 bytes).
// One ldmatrix.x2 brings the B fragments of output block j for one mma
// k-step: matrix 0 holds rows 8j..8j+7, columns 16t..16t+7, matrix 1 the
// next 8 columns.  (The x4 form would halve the loads again but makes the
// compiler hoist twice the registers.)
template <int K, int N, int S>
RT_D void layer(const uint32_t (&a)[K / 16][4], const __half* W, float (&d)[N / 8][4]) {
    static_assert(K % 16 == 0 && S % 8 == 0, "ldmatrix layout");
    const int lane = threadIdx.x & 31;
    const __half* base = W + (lane & 7) * S + 8 * ((lane >> 3) & 1);
#pragma unroll
    for (int j = 0; j < N / 8; j++) {
        d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.0f;
#pragma unroll
        for (int t = 0; t < K / 16; t++) {
            uint32_t b0, b1;
            ldsm_x2(base + 8 * j * S + 16 * t, b0, b1);
            mma16816(d[j], a[t], b0, b1);
        }
    }
}

// Accumulators of N columns -> A fragments (N / 16 k-tiles), with ReLU.
template <int N>
RT_D void pack_relu(const float (&d)[N / 8][4], uint32_t (&a)[N / 16][4]) {
#pragma unroll
    for (int t = 0; t < N / 16; t++) {
        a[t][0] = pack_h2(fmaxf(d[2 * t][0], 0.f), fmaxf(d[2 * t][1], 0.f));
        a[t][1] = pack_h2(fmaxf(d[2 * t][2], 0.f), fmaxf(d[2 * t][3], 0.f));
        a[t][2] = pack_h2(fmaxf(d[2 * t + 1][0], 0.f), fmaxf(d[2 * t + 1][1], 0.f));
        a[t][3] = pack_h2(fmaxf(d[2 * t + 1][2], 0.f), fmaxf(d[2 * t + 1][3], 0.f));
    }
}

// ReLU mask of N / 16 A fragments: bit 8t + 2r + i is set where half i of
// word a[t][r] is positive (32 bits for a 64-wide layer).
template <int N>
RT_D uint32_t relu_mask(const uint32_t (&h)[N / 16][4]) {
    static_assert(N / 16 * 8 <= 32, "mask wider than a word");
    uint32_t m = 0;
#pragma unroll
    for (int t = 0; t < N / 16; t++)
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const float2 hv = unpack_h2(h[t][r]);
            m |= (hv.x > 0.f ? 1u : 0u) << (8 * t + 2 * r);
            m |= (hv.y > 0.f ? 1u : 0u) << (8 * t + 2 * r + 1);
        }
    return m;
}

// Deltas masked by the ReLU of the forward activations (relu_mask bits), packed to A fragments.
template <int N>
RT_D void pack_masked(const float (&d)[N / 8][4], uint32_t mask, uint32_t (&a)[N / 16][4]) {
#pragma unroll
    for (int t = 0; t < N / 16; t++) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const float* src = d[2 * t + (r >> 1)] + 2 * (r & 1);
            const int b = 8 * t + 2 * r;
            a[t][r] = pack_h2((mask >> b) & 1u ? src[0] : 0.f, (mask >> (b + 1)) & 1u ? src[1] : 0.f);
        }
    }
}

// Training stores, per 16-sample tile, the fragments the weight gradients
// need: output delta (2 x 4 words), then the input and delta of each hidden
// layer, then the encoded input.  Word w of lane l sits at
// [w / 4][l][w % 4], so one A fragment (4 words) is one 16-byte store or
// load per lane and 512 contiguous bytes per warp.  k_guide_wgrad_tc forms
// dW_l = E^T X from them.
constexpr int kFragAdo = 0, kFragH3 = 8, kFragE3 = 24, kFragH2 = 40, kFragE2 = 56, kFragH1 = 72, kFragE1 = 88,
              kFragAx = 104, kFragWords = 112;
static_assert(kFragH3 % 4 == 0 && kFragE3 % 4 == 0 && kFragH2 % 4 == 0 && kFragE2 % 4 == 0 && kFragH1 % 4 == 0 &&
                  kFragE1 % 4 == 0 && kFragAx % 4 == 0 && kFragWords % 4 == 0,
              "fragments start on 16-byte boundaries");

template <int T>
RT_D void frag_store(uint32_t* tile_frags, int off, const uint32_t (&f)[T][4], int lane) {
    uint4* q = reinterpret_cast<uint4*>(tile_frags) + (off / 4) * 32 + lane;
#pragma unroll
    for (int t = 0; t < T; t++) q[32 * t] = make_uint4(f[t][0], f[t][1], f[t][2], f[t][3]);
}

RT_D void frag_load(const uint32_t* tile_frags, int off, int lane, uint32_t (&f)[4]) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(tile_frags) + (off / 4) * 32 + lane);
    f[0] = v.x;
    f[1] = v.y;
    f[2] = v.z;
    f[3] = v.w;
}

struct Corners {
    uint32_t idx[8];
    float w[8];
};

// net.res[base + q], q = 0..3 a runtime lane index and base a constant
// after unrolling: selecting among four constant indices keeps the
// parameter array out of local memory (a runtime index into a kernel
// parameter array makes the compiler copy it there).
RT_D int level_res(const NetView& net, int base, int q) {
    return q == 0 ? net.res[base] : q == 1 ? net.res[base + 1] : q == 2 ? net.res[base + 2] : net.res[base + 3];
}

RT_D void level_corners(int res, float3 x, Corners& c) {
    const float fr = float(res);
    float px = x.x * fr, py = x.y * fr, pz = x.z * fr;
    float cx = fminf(floorf(px), fr - 1.0f), cy = fminf(floorf(py), fr - 1.0f), cz = fminf(floorf(pz), fr - 1.0f);
    const float fx = px - cx, fy = py - cy, fz = pz - cz;
    const uint32_t ix = uint32_t(cx), iy = uint32_t(cy), iz = uint32_t(cz);
    const uint32_t r1 = uint32_t(res) + 1u;
    // A level whose (res + 1)^3 grid points fit the table indexes them
    // directly, a finer one hashes them.  Branching (rather than selecting
    // per corner) spares the dense levels the hash arithmetic; the condition
    // is the same for every lane on the same level.
    if (uint64_t(r1) * r1 * r1 <= uint64_t(kT)) {
        const uint32_t r2 = r1 * r1, base = ix + iy * r1 + iz * r2;
#pragma unroll
        for (int k = 0; k < 8; k++) c.idx[k] = base + (k & 1) + ((k >> 1) & 1) * r1 + ((k >> 2) & 1) * r2;
    } else {
        const uint32_t hx[2] = {ix, ix + 1u}, hy[2] = {iy * kPrime1, (iy + 1u) * kPrime1},
                       hz[2] = {iz * kPrime2, (iz + 1u) * kPrime2};
#pragma unroll
        for (int k = 0; k < 8; k++)
            c.idx[k] = (hx[k & 1] ^ hy[(k >> 1) & 1] ^ hz[(k >> 2) & 1]) & uint32_t(kT - 1);
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
        c.w[k] = ((k & 1) ? fx : 1.0f - fx) * (((k >> 1) & 1) ? fy : 1.0f - fy) * (((k >> 2) & 1) ? fz : 1.0f - fz);
}

RT_D uint32_t encode_level(const __half2* __restrict__ table, int res, int l, float3 x) {
    Corners c;
    level_corners(res, x, c);
    const __half2* t = table + size_t(l) * kT;
    float f0 = 0.f, f1 = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float2 v = __half22float2(__ldg(t + c.idx[k]));
        f0 += c.w[k] * v.x;
        f1 += c.w[k] * v.y;
    }
    return pack_h2(f0, f1);
}

// A fragments of the 16 x 32 input: this thread's rows g and g + 8, levels
// tig, tig + 4, tig + 8, tig + 12 (feature pairs 2l, 2l + 1).
RT_D void encode_tile(const NetView& net, float3 xg, float3 xg8, bool vg, bool vg8, uint32_t (&a)[2][4]) {
    const int tig = threadIdx.x & 3;
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int l0 = 8 * t + tig, l1 = 8 * t + 4 + tig;
        const int r0 = level_res(net, 8 * t, tig), r1 = level_res(net, 8 * t + 4, tig);
        a[t][0] = vg ? encode_level(net.table, r0, l0, xg) : 0u;
        a[t][1] = vg8 ? encode_level(net.table, r0, l0, xg8) : 0u;
        a[t][2] = vg ? encode_level(net.table, r1, l1, xg) : 0u;
        a[t][3] = vg8 ? encode_level(net.table, r1, l1, xg8) : 0u;
    }
}

RT_D void load_weights(const __half* __restrict__ mlp, __half* fw, __half* bw) {
    const __half* W0 = mlp;
    const __half* W1 = W0 + kW0;
    const __half* W2 = W1 + kW1;
    const __half* W3 = W2 + kW2;
    for (int i = threadIdx.x; i < kW0; i += blockDim.x) {
        int o = i / kIn, k = i % kIn;
        fw[kOffW0 + o * kS32 + k] = W0[i];
        if (bw) bw[kOffT0 + k * kS64 + o] = W0[i];
    }
    for (int i = threadIdx.x; i < kW1; i += blockDim.x) {
        int o = i / kHid, k = i % kHid;
        fw[kOffW1 + o * kS64 + k] = W1[i];
        fw[kOffW2 + o * kS64 + k] = W2[i];
        if (bw) {
            bw[kOffT1 + k * kS64 + o] = W1[i];
            bw[kOffT2 + k * kS64 + o] = W2[i];
        }
    }
    for (int i = threadIdx.x; i < kW3; i += blockDim.x) {
        int o = i / kHid, k = i % kHid;
        fw[kOffW3 + o * kS64 + k] = W3[i];
        if (bw) bw[kOffT3 + k * kS32 + o] = W3[i];
    }
}

RT_D float3 ld_pos(const float* p, int64_t i) { return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

RT_D void stage_outputs(const float (&out)[4][4], float* tile) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float* p = tile + g * kTileStride + 8 * j + 2 * tig;
        p[0] = out[j][0];
        p[1] = out[j][1];
        p[8 * kTileStride] = out[j][2];
        p[8 * kTileStride + 1] = out[j][3];
    }
}

}  // namespace

// One vMF lobe of a row's raw outputs o4 = (weight logit, log kappa, theta
// and phi logits), evaluated at the unit direction d: everything the loss and
// its gradient need except the mixture weight.  The angles lie in [0, 2 pi],
// where the fast sine / cosine / exponential intrinsics are accurate to a
// few ulp - far inside the FP16 rounding of the network around them.
struct LobeTerms {
    float kap, st, sp;   // concentration, sigmoid(theta logit), sigmoid(phi logit)
    float c;             // cos(mean direction, d)
    float dens;          // vMF density at d
    float dth_d, dph_d;  // d . d(mean)/d(theta), d . d(mean)/d(phi)
    bool inr;            // log kappa inside [kKappaLo, kappa_hi] (gradient passes the clamp)
};

RT_D LobeTerms lobe_terms(float kr, float tl, float pl, float3 d, float kappa_hi) {
    LobeTerms t;
    t.inr = kr >= kKappaLo && kr <= kappa_hi;
    t.kap = __expf(fminf(fmaxf(kr, kKappaLo), kappa_hi));
    t.st = 1.f / (1.f + __expf(-tl));
    t.sp = 1.f / (1.f + __expf(-pl));
    float s_t, c_t, s_p, c_p;
    __sincosf(3.14159265358979f * t.st, &s_t, &c_t);
    __sincosf(6.28318530717959f * t.sp, &s_p, &c_p);
    t.c = s_t * c_p * d.x + s_t * s_p * d.y + c_t * d.z;
    t.dth_d = c_t * c_p * d.x + c_t * s_p * d.y - s_t * d.z;
    t.dph_d = -s_t * s_p * d.x + s_t * c_p * d.y;
    t.dens = t.kap / (6.28318530717959f * -expm1f(-2.f * t.kap)) * __expf(t.kap * (t.c - 1.f));
    return t;
}

// Loss gradient of a warp's 16-row output tile (staged in shared memory,
// row stride kTileStride), in place: for row r the loss is -s_r log q(d_r)
// with s_r = weight[r] * scale, and the 32 raw outputs are replaced by its
// gradient.  Lane 2i + h takes row i's lobes 4h..4h+3; the two lanes of a
// row combine the softmax and mixture sums with one shuffle each, so all 32
// lanes work and every lobe is evaluated once.  Rows at or past n get zero
// gradients.  Returns this lane's share of the tile's loss.
RT_D float loss_grad_tile(float* tile, int row0, int n, const float* __restrict__ dir,
                          const float* __restrict__ weight, float scale, float kappa_hi) {
    const int lane = threadIdx.x & 31, i = lane >> 1, h = lane & 1;
    const int row = row0 + i;
    const bool valid = row < n;
    float* o = tile + i * kTileStride + 16 * h;
    const float3 d = valid ? ld_pos(dir, row) : make_float3(0.f, 0.f, 1.f);
    const float s = valid ? weight[row] * scale : 0.f;
    float mx = o[0];
#pragma unroll
    for (int j = 1; j < 4; j++) mx = fmaxf(mx, o[4 * j]);
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    LobeTerms t[4];
    float e[4], sum = 0.f, qsum = 0.f;  // softmax normaliser; sum of e^(logit - mx) * density
#pragma unroll
    for (int j = 0; j < 4; j++) {
        t[j] = lobe_terms(o[4 * j + 1], o[4 * j + 2], o[4 * j + 3], d, kappa_hi);
        e[j] = __expf(o[4 * j] - mx);
        sum += e[j];
        qsum += e[j] * t[j].dens;
    }
    sum += __shfl_xor_sync(0xffffffffu, sum, 1);
    qsum += __shfl_xor_sync(0xffffffffu, qsum, 1);
    const float inv_sum = 1.f / sum;
    const float q = fmaxf(qsum * inv_sum, 1e-30f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float w = e[j] * inv_sum;
        const float r = w * t[j].dens / q;
        const float dlogk = 1.f / t[j].kap - 2.f / expm1f(2.f * t[j].kap) + (t[j].c - 1.f);
        const float sr = s * -r * t[j].kap;
        o[4 * j] = valid ? s * (w - r) : 0.f;
        o[4 * j + 1] = valid && t[j].inr ? sr * dlogk : 0.f;
        o[4 * j + 2] = valid ? sr * t[j].dth_d * 3.14159265358979f * t[j].st * (1.f - t[j].st) : 0.f;
        o[4 * j + 3] = valid ? sr * t[j].dph_d * 6.28318530717959f * t[j].sp * (1.f - t[j].sp) : 0.f;
    }
    return valid && h == 0 ? -s * logf(q) : 0.f;
}

// Forward + loss + backward of n samples (position, unit direction, weight);
// `scale` multiplies every sample weight (1 / batch).  Adds the gradients to
// grad_table / grad_mlp and the loss to *loss.
__global__ void __launch_bounds__(kBwdWarps * 32, 2) k_guide_backward(NetView net, const float* __restrict__ pos,
                                                           const float* __restrict__ dir,
                                                           const float* __restrict__ weight, int n, float scale,
                                                           const float* __restrict__ weight_sum,
                                                           float* __restrict__ grad_table,
                                                           uint32_t* __restrict__ frags, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (weight_sum) {  // scale = 1 / (sum of the batch's weights), computed on the device
        const float ws = *weight_sum;
        scale = ws > 0.f ? 1.0f / ws : 0.f;
    }
    __half* sw = reinterpret_cast<__half*>(smem);
    __half* sb = sw + kFwdHalves;
    float* tiles = reinterpret_cast<float*>(smem + (kFwdHalves + kBwdHalves) * sizeof(__half));
    int* sres = reinterpret_cast<int*>(tiles + kBwdWarps * 16 * (kTileStride + 3));
    load_weights(net.mlp, sw, sb);
    if (threadIdx.x == 0) {  // constant indices: a runtime index would copy net.res to local memory
#pragma unroll
        for (int q = 0; q < kLevels; q++) sres[q] = net.res[q];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    float* tile = tiles + warp * 16 * kTileStride;
    float* ptile = tiles + kBwdWarps * 16 * kTileStride + warp * 48;  // the tile's 16 positions
    const int lres = sres[lane >> 1];  // resolution of this lane's level in the gradient scatter
    float lsum = 0.f;
    const int tiles_total = (n + 15) / 16;
    for (int tt = blockIdx.x * kBwdWarps + warp; tt < tiles_total; tt += gridDim.x * kBwdWarps) {
        const int r0 = tt * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        const float3 x0 = v0 ? ld_pos(pos, r0) : make_float3(0.f, 0.f, 0.f);
        const float3 x1 = v1 ? ld_pos(pos, r1) : make_float3(0.f, 0.f, 0.f);
        // forward: each layer's input goes to the fragments as soon as it
        // exists; only its ReLU mask stays in registers for the backward
        uint32_t* tf = frags + size_t(tt) * kFragWords * 32;
        uint32_t ax[2][4], h[4][4];
        encode_tile(net, x0, x1, v0, v1, ax);
        frag_store<2>(tf, kFragAx, ax, lane);
        float d64[8][4], out[4][4];
        layer<kIn, kHid, kS32>(ax, sw + kOffW0, d64);
        pack_relu<kHid>(d64, h);
        frag_store<4>(tf, kFragH1, h, lane);
        const uint32_t m1 = relu_mask<kHid>(h);
        layer<kHid, kHid, kS64>(h, sw + kOffW1, d64);
        pack_relu<kHid>(d64, h);
        frag_store<4>(tf, kFragH2, h, lane);
        const uint32_t m2 = relu_mask<kHid>(h);
        layer<kHid, kHid, kS64>(h, sw + kOffW2, d64);
        pack_relu<kHid>(d64, h);
        frag_store<4>(tf, kFragH3, h, lane);
        const uint32_t m3 = relu_mask<kHid>(h);
        layer<kHid, kOut, kS64>(h, sw + kOffW3, out);
        stage_outputs(out, tile);
        __syncwarp();
        lsum += loss_grad_tile(tile, tt * 16, n, dir, weight, scale, net.kappa_hi);
        __syncwarp();
        // dO as A fragments (fp16)
        uint32_t ado[2][4];
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const float* p = tile + g * kTileStride + 16 * t + 2 * tig;
            ado[t][0] = pack_h2(p[0], p[1]);
            ado[t][1] = pack_h2(p[8 * kTileStride], p[8 * kTileStride + 1]);
            ado[t][2] = pack_h2(p[8], p[9]);
            ado[t][3] = pack_h2(p[8 * kTileStride + 8], p[8 * kTileStride + 9]);
        }
        __syncwarp();
        frag_store<2>(tf, kFragAdo, ado, lane);
        uint32_t e[4][4];
        layer<kOut, kHid, kS32>(ado, sb + kOffT3, d64);
        pack_masked<kHid>(d64, m3, e);
        frag_store<4>(tf, kFragE3, e, lane);
        layer<kHid, kHid, kS64>(e, sb + kOffT2, d64);
        pack_masked<kHid>(d64, m2, e);
        frag_store<4>(tf, kFragE2, e, lane);
        layer<kHid, kHid, kS64>(e, sb + kOffT1, d64);
        pack_masked<kHid>(d64, m1, e);
        frag_store<4>(tf, kFragE1, e, lane);
        float dx[4][4];
        layer<kHid, kIn, kS64>(e, sb + kOffT0, dx);
        // hash-grid gradient.  The 16 x 32 input gradient goes through the
        // staging tile so that lane 2l + hh owns level l for rows 8hh..8hh+7.
        // Consecutive batch rows are neighbouring samples: a corner that the
        // next row shares is summed in registers and leaves as one reduction,
        // which spares the contended coarse levels most of their atomics.
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float* p = tile + g * kTileStride + 8 * j + 2 * tig;
            p[0] = dx[j][0];
            p[1] = dx[j][1];
            p[8 * kTileStride] = dx[j][2];
            p[8 * kTileStride + 1] = dx[j][3];
        }
        if (tig == 0) {
            float* q = ptile + 3 * g;
            q[0] = x0.x, q[1] = x0.y, q[2] = x0.z;
            q[24] = x1.x, q[25] = x1.y, q[26] = x1.z;
        }
        __syncwarp();
        {
            const int l = lane >> 1, rbase = 8 * (lane & 1);
            const int rows = min(8, n - tt * 16 - rbase);
            float2* gt = reinterpret_cast<float2*>(grad_table) + size_t(l) * kT;
            uint32_t pidx[8];
            float2 pg[8];
#pragma unroll
            for (int r = 0; r < 8; r++) {
                if (r >= rows) break;
                const int row = rbase + r;
                const float3 x = make_float3(ptile[3 * row], ptile[3 * row + 1], ptile[3 * row + 2]);
                const float g0 = tile[row * kTileStride + 2 * l], g1 = tile[row * kTileStride + 2 * l + 1];
                Corners c;
                level_corners(lres, x, c);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const float2 v = make_float2(c.w[k] * g0, c.w[k] * g1);
                    if (r > 0 && c.idx[k] == pidx[k]) {
                        pg[k].x += v.x;
                        pg[k].y += v.y;
                    } else {
                        if (r > 0) atomicAdd(gt + pidx[k], pg[k]);
                        pidx[k] = c.idx[k];
                        pg[k] = v;
                    }
                }
            }
            if (rows > 0) {
#pragma unroll
                for (int k = 0; k < 8; k++) atomicAdd(gt + pidx[k], pg[k]);
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0 && lsum != 0.f) atomicAdd(loss, lsum);
}

// ------------------------------------------------------------------ renderer side
// Items of the sorted shade queue whose material type is guided, in bucket order.
struct GuidedItems {
    int bucket[kShadeBucketsG], count[kShadeBucketsG], n;
};

RT_D GuidedItems guided_items(const rtd::WaveCtl* ctl) {
    GuidedItems gi;
    int m = 0;  // a constant at every step once both loops are unrolled, so gi stays in registers
    gi.n = 0;
#pragma unroll
    for (int b = 0; b < rtd::kShadeBuckets; b++) {
        if (b == rtd::kMissBucket || !guided_type(b)) continue;
        gi.bucket[m] = b;
        gi.count[m] = ctl->bucket[b];
        gi.n += gi.count[m];
        m++;
    }
#pragma unroll
    for (; m < kShadeBucketsG; m++) gi.bucket[m] = gi.count[m] = 0;
    return gi;
}

// The slot of guided item i: bucket m holds items [base_m, base_m + count_m).
// Unrolled with constant indices (a runtime index would put gi in local memory).
RT_D int guided_slot(const GuidedItems& gi, const rtd::WaveBufs& B, int i) {
    int bucket = gi.bucket[0], base = 0;
    bool found = false;
#pragma unroll
    for (int m = 0; m < kShadeBucketsG - 1; m++) {
        if (!found && i >= base + gi.count[m]) {
            base += gi.count[m];
            bucket = gi.bucket[m + 1];
        } else {
            found = true;
        }
    }
    return B.sorted[size_t(bucket) * size_t(B.capacity) + size_t(i - base)];
}

RT_D float3 hit_position(const rtd::Ctx& c, int slot) {
    const rtd::WaveBufs& B = c.wb;
    const float4 o = B.ray_o[slot], d = B.ray_d[slot], h = B.hit[slot];
    const rtd::WaveParams& W = c.waves[*c.wave_index];
    const rtd::SceneView& sc = c.jobs[W.seg[rtd::find_segment(W, slot)].job].sc;
    const float4* tv = sc.tri_v + size_t(__float_as_int(h.w)) * 3;
    const float4 p0 = __ldg(tv), p1 = __ldg(tv + 1), p2 = __ldg(tv + 2);
    const rtd::v3 dd(d.x, d.y, d.z);
    const rtd::v3 p(o.x + h.x * d.x, o.y + h.x * d.y, o.z + h.x * d.z);
    return guide_input(p, rtd::v3(p0.x, p0.y, p0.z), rtd::v3(p1.x, p1.y, p1.z), rtd::v3(p2.x, p2.y, p2.z), dd, c.G);
}

// ======================================================================
// Inference on the 5th-generation tensor cores (tcgen05, accumulators in
// tensor memory).  A CTA of kTcRows = 128 threads runs 128 queries, one per
// thread and per TMEM lane, through the 32-64-64-64-32 MLP:
//   * thread t gathers its query's 16 hash-grid levels and writes row t of
//     the A operand in shared memory: K-major, the canonical no-swizzle
//     layout of 8-row x 16-byte core matrices (LBO = 128 B between the two
//     core matrices of a 16-wide K step, SBO = K * 2 * 8 B between 8-row
//     groups);
//   * thread 0 issues the layer's tcgen05.mma.kind::f16 (M = 128, N = 64 or
//     32, K = 16 per instruction, FP16 operands from shared memory, FP32
//     accumulators in 64 TMEM columns) and commits them to an mbarrier;
//   * every warp reads its 32 TMEM lanes back (tcgen05.ld 32x32b), applies
//     ReLU, rounds to FP16 and writes the next layer's A rows;
//   * the last layer's 32 outputs, in registers, become the mixture.
// The weights (B operands, [out][in] = N x K, K-major) are written once per
// CTA in the same layout.  Every wait on the mbarrier is bounded: a timeout
// is counted in g_tc_timeouts (reported by the host as a watchdog error),
// and the CTA stops issuing, frees its TMEM and returns.
// ======================================================================
constexpr int kTcRows = 128;
constexpr int kTcCols = 64;  // TMEM columns: the widest layer's accumulators
constexpr uint32_t kTcA = 0, kTcW0 = kTcA + kTcRows * kHid * 2, kTcW1 = kTcW0 + kHid * kIn * 2,
                   kTcW2 = kTcW1 + kHid * kHid * 2, kTcW3 = kTcW2 + kHid * kHid * 2, kTcBar = kTcW3 + kOut * kHid * 2,
                   kTcSlot = kTcBar + 8, kTcSmem = kTcSlot + 8;
constexpr long long kTcWaitLimit = 1ll << 22;  // mbarrier polls before a wait is given up
__device__ int g_tc_timeouts;

// Byte offset of element (row r, column k) of an R x K FP16 operand in the
// canonical K-major no-swizzle layout.
RT_D uint32_t tc_off(int r, int k, int K) {
    return uint32_t(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// Shared-memory matrix descriptor (sm_100): start, leading (K) and stride
// (row-group) byte offsets >> 4, descriptor version 1, no swizzle.
RT_D uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulators, FP16 A and B, both
// K-major, M = 128, N.
RT_HD constexpr uint32_t tc_idesc(int n) { return (1u << 4) | (uint32_t(n >> 3) << 17) | (uint32_t(kTcRows >> 4) << 24); }

RT_D uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

RT_D void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
RT_D void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}
RT_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
RT_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// generic-proxy writes of shared memory made visible to the tensor cores' reads
RT_D void tc_fence_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
RT_D bool tc_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kTcWaitLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
RT_D void tmem_ld_x64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}

RT_D void tmem_ld_x32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}


// Weights -> shared memory, B operands in the canonical layout.
RT_D void tc_load_weights(const __half* __restrict__ mlp, unsigned char* sm) {
    const __half* W[4] = {mlp, mlp + kW0, mlp + kW0 + kW1, mlp + kW0 + kW1 + kW2};
    const uint32_t off[4] = {kTcW0, kTcW1, kTcW2, kTcW3};
    const int rows[4] = {kHid, kHid, kHid, kOut}, cols[4] = {kIn, kHid, kHid, kHid};
#pragma unroll
    for (int l = 0; l < 4; l++)
        for (int i = threadIdx.x; i < rows[l] * cols[l]; i += blockDim.x) {
            const int o = i / cols[l], k = i % cols[l];
            *reinterpret_cast<__half*>(sm + off[l] + tc_off(o, k, cols[l])) = W[l][i];
        }
}

// Row `row` of the first layer's A operand: the 16 levels' features of x.
RT_D void tc_encode_row(const NetView& net, float3 x, bool valid, unsigned char* sm, int row) {
    uint32_t f[kLevels];
#pragma unroll
    for (int l = 0; l < kLevels; l++) f[l] = valid ? encode_level(net.table, net.res[l], l, x) : 0u;
#pragma unroll
    for (int j = 0; j < kIn / 8; j++)
        *reinterpret_cast<uint4*>(sm + kTcA + tc_off(row, 8 * j, kIn)) =
            make_uint4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
}

// The four layers for the 128 rows staged in A; this thread's 32 outputs.
// Returns false when a wait timed out (outputs undefined).
RT_D bool tc_mlp(unsigned char* sm, uint32_t tmem, uint32_t& parity, float (&out)[kOut]) {
    const uint32_t bar = smem_u32(sm + kTcBar), a_base = smem_u32(sm + kTcA);
    const uint32_t taddr = tmem + (uint32_t(threadIdx.x >> 5) * 32u << 16);
    const uint32_t w_off[4] = {kTcW0, kTcW1, kTcW2, kTcW3};
#pragma unroll
    for (int layer = 0; layer < 4; layer++) {
        const int K = layer == 0 ? kIn : kHid, N = layer == 3 ? kOut : kHid;
        tc_fence_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (threadIdx.x == 0) {
            const uint32_t w_base = smem_u32(sm + w_off[layer]);
#pragma unroll
            for (int ks = 0; ks < K / 16; ks++)
                tc_mma(tmem, tc_desc(a_base + 256u * ks, 128u, uint32_t(K) * 16u),
                       tc_desc(w_base + 256u * ks, 128u, uint32_t(K) * 16u), tc_idesc(N), ks > 0 ? 1u : 0u);
            tc_commit(bar);
        }
        // the CTA agrees on the outcome, so no thread is left at a barrier
        const bool ok = __syncthreads_and(tc_wait(bar, parity)) != 0;
        parity ^= 1u;
        if (!ok) return false;
        tc_fence_after();
        if (layer < 3) {
            float v[kHid];
            tmem_ld_x64(taddr, v);
#pragma unroll
            for (int j = 0; j < kHid / 8; j++)
                *reinterpret_cast<uint4*>(sm + kTcA + tc_off(threadIdx.x, 8 * j, kHid)) = make_uint4(
                    pack_h2(fmaxf(v[8 * j], 0.f), fmaxf(v[8 * j + 1], 0.f)),
                    pack_h2(fmaxf(v[8 * j + 2], 0.f), fmaxf(v[8 * j + 3], 0.f)),
                    pack_h2(fmaxf(v[8 * j + 4], 0.f), fmaxf(v[8 * j + 5], 0.f)),
                    pack_h2(fmaxf(v[8 * j + 6], 0.f), fmaxf(v[8 * j + 7], 0.f)));
        } else {
            tmem_ld_x32(taddr, out);
        }
    }
    return true;
}

// Set-up shared by the kernels: weights, mbarrier, TMEM columns.
RT_D uint32_t tc_setup(const NetView& net, unsigned char* sm) {
    tc_load_weights(net.mlp, sm);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(sm + kTcBar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     ::"r"(smem_u32(sm + kTcSlot)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *reinterpret_cast<volatile uint32_t*>(sm + kTcSlot);
}
RT_D void tc_teardown(uint32_t tmem, bool ok) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcCols) : "memory");
    if (!ok && threadIdx.x == 0) atomicAdd(&g_tc_timeouts, 1);
}

// ----------------------------------------------------------- weight gradients
// dW_l = E_l^T X_l, summed over the samples of a training pass, on the
// tensor cores.  For layer l, E_l holds the output deltas and X_l the inputs
// of every sample (k_guide_backward stores both per 16-sample tile as mma
// fragments: word r of lane 4g + t of a 16-unit block is units 8(r >> 1) +
// 2t, +1 of sample g + 8(r & 1); a tile is 28 such blocks, "pieces").  One
// CTA of 16 warps per SM takes four tiles (64 samples, a chunk) at a time,
// in a pipeline over two staging buffers and two operand buffers:
//   * chunk c + 2 is copied to shared memory with cp.async while chunk c is
//     transposed (56 KB per SM always in flight from HBM);
//   * warp w transposes 7 pieces of tile w & 3 (w >> 2 chooses which), each
//     8x8 block with movmatrix (lane 4g + t then holds unit g, samples 2t and
//     2t + 1) and one 32-bit store into the K-major canonical operands of
//     chunk c's buffer (K = the chunk's 64 samples):
//       A_l = E_l^T, the layer's 32 or 64 output units as rows;
//       B_l = X_l^T, the layer's 64 (or 32) input units as rows;
//   * one thread issues, per layer, four tcgen05.mma.kind::f16 (M = 128,
//     N = 64 or 32, K = 16) accumulating into the layer's TMEM columns
//     (layer 3 in 0..63, 2 in 64..127, 1 in 128..191, 0 in 192..223) and
//     commits them to the buffer's mbarrier; the warps go on to chunk c + 1
//     in the other buffer, and wait for that mbarrier only before they
//     overwrite this buffer with chunk c + 2.
// The MMA's rows are independent, so A rows past the layer's outputs are
// whatever follows in shared memory (the next operand): they only make
// accumulator rows that are never read.  At the end warps 0 and 1 read rows
// 0..63 back (tcgen05.ld 32x32b) and add them to the FP32 gradients.  Waits
// on the mbarriers are bounded as in the inference kernel: a CTA that gives
// up adds nothing, frees its TMEM and is counted in g_tc_timeouts.
constexpr int kWgK = 64;                   // samples per chunk
constexpr int kWgTiles = kWgK / 16;        // tiles per chunk
constexpr int kWgParts = 4;                // warps per tile
constexpr int kWgWarps = kWgTiles * kWgParts;
constexpr int kWgCols = 256;               // TMEM columns (224 used)
constexpr int kWgPieces = kFragWords / 4;  // 16-byte pieces of a tile per lane
constexpr int kWgPartPieces = kWgPieces / kWgParts;
static_assert(kWgPieces % kWgParts == 0, "pieces per warp");
constexpr uint32_t kWgTileBytes = uint32_t(kFragWords) * 32u * 4u;
constexpr uint32_t kWgRow = kWgK * 2u;  // bytes per operand row
// operands of one buffer, in fragment order; an M = 128 A operand reads 128
// rows from its start, so A0 needs 128 rows of shared memory after it
constexpr uint32_t kWgA3 = 0, kWgB3 = kWgA3 + kOut * kWgRow, kWgA2 = kWgB3 + kHid * kWgRow,
                   kWgB2 = kWgA2 + kHid * kWgRow, kWgA1 = kWgB2 + kHid * kWgRow, kWgB1 = kWgA1 + kHid * kWgRow,
                   kWgA0 = kWgB1 + kHid * kWgRow, kWgB0 = kWgA0 + kHid * kWgRow, kWgOps = kWgB0 + kIn * kWgRow;
constexpr uint32_t kWgStage = 2 * kWgOps, kWgBar = kWgStage + 2u * kWgTiles * kWgTileBytes, kWgSlot = kWgBar + 16,
                   kWgSmem = kWgSlot + 8;
static_assert(kWgStage % 16 == 0 && kWgBar % 8 == 0 && kWgSmem <= 227 * 1024, "shared memory layout");
static_assert(kWgOps + kWgA0 + 128 * kWgRow <= kWgBar, "the second buffer's A0 reads 128 rows inside the allocation");

RT_D void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
RT_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
RT_D void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Operand offset of fragment piece i (the operands follow the fragment order:
// A3 2 pieces, B3 4, A2 4, B2 4, A1 4, B1 4, A0 4, B0 2; a piece is a
// 16-unit block, 16 rows of its operand).
RT_D uint32_t wg_piece_rows(int i) {
    static_assert(kFragAdo == 0 && kFragH3 == 8 && kFragE3 == 24 && kFragH2 == 40 && kFragE2 == 56 &&
                      kFragH1 == 72 && kFragE1 == 88 && kFragAx == 104,
                  "fragment order");
    return uint32_t(i) * 16u * kWgRow;  // every piece is 16 rows of K-major operand in fragment order
}

// The staged pieces [p0, p0 + kWgPartPieces) of one tile (or zeros) into
// the operand buffer `ops`, samples 16 * tile .. 16 * tile + 15.  Rows m
// of piece i's operand: 16 (i - first piece of the operand) + 0..15; as the
// operands are stored back to back in fragment order and a piece is a
// 16-row block, the canonical offset of (operand row, k) within the buffer
// is that of the piece's own 16-row block.
RT_D void wg_stage(const unsigned char* stage, int p0, unsigned char* ops, int tile, int lane, bool valid) {
#pragma unroll
    for (int j = 0; j < kWgPartPieces; j++) {
        const int i = p0 + j;
        const uint4 q = valid ? *reinterpret_cast<const uint4*>(stage + (i * 32 + lane) * 16) : make_uint4(0u, 0u, 0u, 0u);
        const uint32_t f[4] = {q.x, q.y, q.z, q.w};
        unsigned char* blk = ops + wg_piece_rows(i);
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int m = 8 * (r >> 1) + (lane >> 2);
            const int k = 16 * tile + 8 * (r & 1) + 2 * (lane & 3);
            *reinterpret_cast<uint32_t*>(blk + tc_off(m, k, kWgK)) = trans8x8(f[r]);
        }
    }
}

// Rows 32 w .. 32 w + 31 of one layer's accumulators (N columns from `col`)
// added to gW [M][N]; rows >= M are not the layer's.
template <int M, int N>
RT_D void wg_flush(uint32_t tmem, int col, int warp, int lane, float* __restrict__ gW) {
    float v[N];
    const uint32_t taddr = tmem + (uint32_t(32 * warp) << 16) + uint32_t(col);
    if constexpr (N == 64)
        tmem_ld_x64(taddr, v);
    else
        tmem_ld_x32(taddr, v);
    const int m = 32 * warp + lane;
    if (m >= M) return;
    // one 16-byte reduction per four columns: the CTAs of the grid all add
    // their partial sums at about the same time, and scalar atomics made
    // this a third of the kernel's time
#pragma unroll
    for (int n = 0; n < N; n += 4)
        if (v[n] != 0.f || v[n + 1] != 0.f || v[n + 2] != 0.f || v[n + 3] != 0.f)
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(gW + m * N + n), "f"(v[n]),
                         "f"(v[n + 1]), "f"(v[n + 2]), "f"(v[n + 3])
                         : "memory");
}

__global__ void __launch_bounds__(kWgWarps * 32, 1) k_guide_wgrad_tc(const uint32_t* __restrict__ frags, int tiles,
                                                                     int chunk, float* __restrict__ grad_mlp) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int t0 = blockIdx.x * chunk, t1 = min(tiles, t0 + chunk);
    if (t0 >= t1) return;  // the whole CTA
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = warp % kWgTiles, p0 = (warp / kWgTiles) * kWgPartPieces;
    const uint32_t bar0 = smem_u32(sm + kWgBar), stage0 = smem_u32(sm + kWgStage);
    auto stage_off = [&](int c) { return (uint32_t(c & 1) * kWgTiles + uint32_t(tile)) * kWgTileBytes; };
    auto copy = [&](int c, int nchunks) {  // this lane's pieces of its tile of chunk c
        const int tl = t0 + c * kWgTiles + tile;
        if (c < nchunks && tl < t1) {
            const uint4* src = reinterpret_cast<const uint4*>(frags + size_t(tl) * kFragWords * 32);
            const uint32_t dst = stage0 + stage_off(c);
            for (int i = p0; i < p0 + kWgPartPieces; i++) cp_async16(dst + uint32_t(i * 32 + lane) * 16u, src + i * 32 + lane);
        }
        cp_async_commit();  // one group per chunk, empty or not
    };
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0 + 8u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     ::"r"(smem_u32(sm + kWgSlot)), "r"(kWgCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    const int nchunks = (t1 - t0 + kWgTiles - 1) / kWgTiles;
    copy(0, nchunks);
    copy(1, nchunks);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kWgSlot);
    bool ok = true;
    for (int c = 0; c < nchunks && ok; c++) {
        const int b = c & 1;
        if (c >= 2) {  // the MMAs of chunk c - 2 have read this operand buffer
            ok = __syncthreads_and(tc_wait(bar0 + 8u * uint32_t(b), uint32_t((c / 2 - 1) & 1))) != 0;
            if (!ok) break;
            tc_fence_after();
        }
        cp_async_wait_1();  // this lane's copies of chunk c have landed
        wg_stage(sm + kWgStage + stage_off(c), p0, sm + b * kWgOps, tile, lane, t0 + c * kWgTiles + tile < t1);
        copy(c + 2, nchunks);  // into the staging buffer this lane has just read
        tc_fence_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (threadIdx.x == 0) {
            const uint32_t ops = smem_u32(sm + b * kWgOps);
            const uint32_t a[4] = {kWgA3, kWgA2, kWgA1, kWgA0}, bo[4] = {kWgB3, kWgB2, kWgB1, kWgB0};
            const int n[4] = {kHid, kHid, kHid, kIn};
#pragma unroll
            for (int l = 0; l < 4; l++)
#pragma unroll
                for (int ks = 0; ks < kWgK / 16; ks++)
                    tc_mma(tmem + uint32_t(64 * l), tc_desc(ops + a[l] + 256u * ks, 128u, kWgK * 16u),
                           tc_desc(ops + bo[l] + 256u * ks, 128u, kWgK * 16u), tc_idesc(n[l]),
                           (c > 0 || ks > 0) ? 1u : 0u);
            tc_commit(bar0 + 8u * uint32_t(b));
        }
    }
    if (ok) {  // the last commit arrives once every MMA of the CTA is done
        const int last = nchunks - 1;
        ok = __syncthreads_and(tc_wait(bar0 + 8u * uint32_t(last & 1), uint32_t((last / 2) & 1))) != 0;
        tc_fence_after();
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy outlives the CTA
    if (ok && warp < 2) {
        wg_flush<kOut, kHid>(tmem, 0, warp, lane, grad_mlp + kW0 + kW1 + kW2);
        wg_flush<kHid, kHid>(tmem, 64, warp, lane, grad_mlp + kW0 + kW1);
        wg_flush<kHid, kHid>(tmem, 128, warp, lane, grad_mlp + kW0);
        wg_flush<kHid, kIn>(tmem, 192, warp, lane, grad_mlp);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kWgCols) : "memory");
    if (!ok && threadIdx.x == 0) atomicAdd(&g_tc_timeouts, 1);
}

// Raw outputs (mode 0) or mixtures (mode 1) of n normalised positions.
__global__ void __launch_bounds__(kTcRows) k_guide_forward_tc(NetView net, const float* __restrict__ pos, int n,
                                                              int mode, float* __restrict__ raw,
                                                              Mixture* __restrict__ mix) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t tmem = tc_setup(net, sm);
    uint32_t parity = 0;
    bool ok = true;
    const int tiles = (n + kTcRows - 1) / kTcRows;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int row = t * kTcRows + int(threadIdx.x);
        const bool valid = row < n;
        tc_encode_row(net, valid ? ld_pos(pos, row) : make_float3(0.f, 0.f, 0.f), valid, sm, threadIdx.x);
        float out[kOut];
        ok = tc_mlp(sm, tmem, parity, out);
        if (ok && valid) {
            if (mode == 0) {
#pragma unroll
                for (int k = 0; k < kOut; k++) raw[int64_t(row) * kOut + k] = out[k];
            } else {
                Mixture m;
                head_from_outputs(out, m, net.kappa_hi);
                mix[row] = m;
            }
        }
    }
    tc_teardown(tmem, ok);
}

// Mixtures of this bounce's guided vertices (surface hits of guided material
// types), written per slot for the shade kernel.
__global__ void __launch_bounds__(kTcRows) k_guide_infer_tc(rtd::Ctx c, NetView net) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t tmem = tc_setup(net, sm);
    const rtd::WaveBufs& B = c.wb;
    const GuidedItems gi = guided_items(B.ctl);
    const int n = gi.n;
    uint32_t parity = 0;
    bool ok = true;
    const int tiles = (n + kTcRows - 1) / kTcRows;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int r = t * kTcRows + int(threadIdx.x);
        const bool valid = r < n;
        const int slot = valid ? guided_slot(gi, B, r) : 0;
        tc_encode_row(net, valid ? hit_position(c, slot) : make_float3(0.f, 0.f, 0.f), valid, sm, threadIdx.x);
        float out[kOut];
        ok = tc_mlp(sm, tmem, parity, out);
        if (ok && valid) {
            Mixture m;
            head_from_outputs(out, m, net.kappa_hi);
            c.G.mix[slot] = m;
        }
    }
    tc_teardown(tmem, ok);
}

// End of a training wave: turns each path's records into training samples
// (position, direction, weight = luminance of the incident-radiance estimate
// (R_end - R_i) / T_i times |cos| over the sampling pdf: the mixture is fitted
// to incident radiance times the cosine), appended to `buf`.
__global__ void k_guide_collect(rtd::Ctx c, float4* __restrict__ buf, int* __restrict__ count, int cap) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const rtd::WaveParams& W = c.waves[*c.wave_index];
    const rtd::WaveBufs& B = c.wb;
    const int lane = threadIdx.x & 31;
    const bool in_wave = slot < W.wave_count;
    float4 re = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in_wave) {
        const float4 a = B.rad[slot], e = B.nee0[slot], l = B.nee1[slot];
        re = make_float4(a.x + e.x + l.x, a.y + e.y + l.y, a.z + e.z + l.z, 0.f);
    }
    const size_t C = size_t(B.capacity);
    for (int r = 0; r < kGuideRec; r++) {
        bool ok = false;
        float4 xp = make_float4(0.f, 0.f, 0.f, 0.f), dv = xp;
        float wgt = 0.f;
        if (in_wave) {
            const float4* R = c.G.rec + size_t(r) * 4 * C + slot;
            dv = R[C];
            if (dv.w != 0.f) {
                xp = R[0];
                const float4 t = R[2 * C], rr = R[3 * C];
                const float lx = t.x > 0.f ? (re.x - rr.x) / t.x : 0.f;
                const float ly = t.y > 0.f ? (re.y - rr.y) / t.y : 0.f;
                const float lz = t.z > 0.f ? (re.z - rr.z) / t.z : 0.f;
                wgt = (lx + ly + lz) * (1.0f / 3.0f) * dv.w / xp.w;  // target: L_in |cos|
                ok = wgt > 0.f && wgt < 3.0e38f;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (!m) continue;
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        const int pos = base + __popc(m & ((1u << lane) - 1u));
        if (ok && pos < cap) {
            buf[2 * size_t(pos)] = make_float4(xp.x, xp.y, xp.z, wgt);
            buf[2 * size_t(pos) + 1] = make_float4(dv.x, dv.y, dv.z, 1.0f);
        }
    }
}

// A training batch of `n` samples: all collected ones when they fit, else
// every (count / n)-th one from a start drawn from `seed`; accumulates the
// batch's weight sum for the loss scale.
__global__ void k_guide_batch(const float4* __restrict__ buf, const int* __restrict__ count, int cap, int n,
                              uint32_t seed, float* __restrict__ pos, float* __restrict__ dir, float* __restrict__ w,
                              float* __restrict__ weight_sum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cnt = min(*count, cap);
    float wi = 0.f;
    if (i < n) {
        float4 a = make_float4(0.5f, 0.5f, 0.5f, 0.f), b = make_float4(0.f, 0.f, 1.f, 0.f);
        if (cnt > n) {
            // every (cnt / n)-th sample from a start drawn per step: each
            // sample at most once, and neighbouring batch rows are samples
            // written close together (in slot order, so close in space), so
            // the hash-grid gradient of a 16-row tile merges repeated corners
            uint32_t h = seed * 0x9E3779B9u;
            h ^= h >> 16;
            h *= 0x85EBCA6Bu;
            h ^= h >> 13;
            h *= 0xC2B2AE35u;
            h ^= h >> 16;
            const uint64_t start = uint64_t(h) * uint64_t(cnt) >> 32;
            const int j = int((start + uint64_t(i) * uint64_t(cnt) / uint64_t(n)) % uint64_t(cnt));
            a = buf[2 * size_t(j)];
            b = buf[2 * size_t(j) + 1];
        } else if (i < cnt) {  // every sample once; the rest of the batch weighs nothing
            a = buf[2 * size_t(i)];
            b = buf[2 * size_t(i) + 1];
        }
        pos[3 * i] = a.x;
        pos[3 * i + 1] = a.y;
        pos[3 * i + 2] = a.z;
        dir[3 * i] = b.x;
        dir[3 * i + 1] = b.y;
        dir[3 * i + 2] = b.z;
        wi = a.w;
        w[i] = wi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wi += __shfl_down_sync(0xffffffffu, wi, o);
    if ((threadIdx.x & 31) == 0 && wi != 0.f) atomicAdd(weight_sum, wi);
}

// Adam over one parameter array: p -= lr * mhat / (sqrt(vhat) + eps); the
// gradient is cleared and the fp16 copy refreshed.
__global__ void k_adam(float* __restrict__ p, __half* __restrict__ p16, float* __restrict__ grad,
                       float* __restrict__ m, float* __restrict__ v, int64_t n, float lr, float b1, float b2, float c1,
                       float c2, float eps) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float gr = grad[i];
        grad[i] = 0.f;
        const float mi = b1 * m[i] + (1.f - b1) * gr;
        const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        p16[i] = __float2half_rn(pi);
    }
}

// Adam on the hash table, level l = blockIdx.y over its first n_l entries
// (one entry = kFeats = 2 parameters, moved as float2 / half2).  Entries past
// n_l have never had a gradient (m = v = 0), for which Adam's update is 0,
// so leaving them out changes nothing.
struct LevelExtents {
    int32_t n[kLevels];  // entries of each level that any resolution so far has used
};
__global__ void __launch_bounds__(256) k_adam_table(float2* __restrict__ p, __half2* __restrict__ p16,
                                                    float2* __restrict__ grad, float2* __restrict__ m,
                                                    float2* __restrict__ v, LevelExtents ext, float lr, float b1,
                                                    float b2, float c1, float c2, float eps) {
    __shared__ int32_t s_n;
    if (threadIdx.x == 0) {  // constant indices only: a runtime index would copy ext to local memory
        int32_t n = 0;
#pragma unroll
        for (int q = 0; q < kLevels; q++)
            if (int(blockIdx.y) == q) n = ext.n[q];
        s_n = n;
    }
    __syncthreads();
    const int32_t n = s_n;
    const size_t base = size_t(blockIdx.y) * kT;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = base + size_t(i);
        const float2 gr = grad[k], mo = m[k], vo = v[k], po = p[k];
        grad[k] = make_float2(0.f, 0.f);
        const float2 mi = make_float2(b1 * mo.x + (1.f - b1) * gr.x, b1 * mo.y + (1.f - b1) * gr.y);
        const float2 vi = make_float2(b2 * vo.x + (1.f - b2) * gr.x * gr.x, b2 * vo.y + (1.f - b2) * gr.y * gr.y);
        m[k] = mi;
        v[k] = vi;
        const float2 pi = make_float2(po.x - lr * (mi.x * c1) / (sqrtf(vi.x * c2) + eps),
                                      po.y - lr * (mi.y * c1) / (sqrtf(vi.y * c2) + eps));
        p[k] = pi;
        p16[k] = __floats2half2_rn(pi.x, pi.y);
    }
}

__global__ void k_to_half(const float* __restrict__ p, __half* __restrict__ p16, int64_t n) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p16[i] = __float2half_rn(p[i]);
}

// Mixture pdf of (position, direction) pairs and samples from (position, u0..u2).
__global__ void k_guide_pdf_sample(const Mixture* __restrict__ mix, const float* __restrict__ dir,
                                   const float* __restrict__ u, int n, float* __restrict__ out_dir,
                                   float* __restrict__ pdf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Mixture* m = mix + i;
    rtd::v3 d;
    if (u) {
        d = mixture_sample(m, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
        out_dir[3 * i] = d.x;
        out_dir[3 * i + 1] = d.y;
        out_dir[3 * i + 2] = d.z;
    } else {
        d = rtd::v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    }
    pdf[i] = mixture_pdf(m, d);
}

}  // namespace rtg

namespace rtgh {

size_t backward_smem() {
    return size_t(rtg::kFwdHalves + rtg::kBwdHalves) * 2 + size_t(rtg::kBwdWarps) * 16 * (rtg::kTileStride + 3) * 4 +
           size_t(rtg::kLevels) * 4;
}

cudaError_t prepare_kernels() {
    cudaError_t e = cudaFuncSetAttribute(rtg::k_guide_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(backward_smem()));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(rtg::k_guide_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(rtg::kWgSmem));
    return e;
}

// Inference CTAs per SM: 4 of 128 threads (122 registers each); with 64 TMEM
// columns a CTA, at most 256 of the SM's 512 columns are allocated, so no
// CTA waits for tensor memory.
constexpr int kTcBlocksPerSm = 4;

void launch_forward(const rtg::NetView& net, const float* pos, int n, int mode, float* raw, rtg::Mixture* mix, int sms,
                    cudaStream_t st) {
    if (n <= 0) return;
    const int tiles = (n + rtg::kTcRows - 1) / rtg::kTcRows;
    rtg::k_guide_forward_tc<<<std::min(tiles, sms * kTcBlocksPerSm), rtg::kTcRows, rtg::kTcSmem, st>>>(net, pos, n,
                                                                                                      mode, raw, mix);
}

int take_tc_timeouts() {
    int n = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&n, rtg::g_tc_timeouts, sizeof(int)) != cudaSuccess) return 0;
    if (n) cudaMemcpyToSymbol(rtg::g_tc_timeouts, &zero, sizeof(int));
    return n;
}

size_t frag_bytes_per_tile() { return size_t(rtg::kFragWords) * 32 * 4; }

void launch_backward(const rtg::NetView& net, const float* pos, const float* dir, const float* weight, int n,
                     float scale, const float* weight_sum, float* grad_table, float* grad_mlp, float* loss,
                     uint32_t* frags, int frag_tiles, int sms, cudaStream_t st) {
    // chunks of at most frag_tiles tiles: the fused pass stores their
    // fragments, then k_guide_wgrad_tc turns them into weight gradients
    for (int begin = 0; begin < n; begin += frag_tiles * 16) {
        const int m = std::min(n - begin, frag_tiles * 16);
        const int tiles = (m + 15) / 16;
        int blocks = (tiles + rtg::kBwdWarps - 1) / rtg::kBwdWarps;
        if (blocks > sms * 2) blocks = sms * 2;  // 2 resident per SM: <= 128 registers, ~73 KB shared each
        rtg::k_guide_backward<<<blocks, rtg::kBwdWarps * 32, backward_smem(), st>>>(
            net, pos + size_t(begin) * 3, dir + size_t(begin) * 3, weight + begin, m, scale, weight_sum, grad_table,
            frags, loss);
        // one CTA per SM (224 KB of operands and staging, 256 TMEM columns),
        // a multiple of four tiles each
        int chunk = (tiles + sms - 1) / sms;
        chunk = std::max(rtg::kWgTiles, (chunk + rtg::kWgTiles - 1) / rtg::kWgTiles * rtg::kWgTiles);
        rtg::k_guide_wgrad_tc<<<(tiles + chunk - 1) / chunk, rtg::kWgWarps * 32, rtg::kWgSmem, st>>>(frags, tiles,
                                                                                                    chunk, grad_mlp);
    }
}

void launch_infer(const rtd::Ctx& c, const rtg::NetView& net, int sms, cudaStream_t st) {
    rtg::k_guide_infer_tc<<<sms * kTcBlocksPerSm, rtg::kTcRows, rtg::kTcSmem, st>>>(c, net);
}

void launch_collect(const rtd::Ctx& c, float4* buf, int* count, int cap, cudaStream_t st) {
    rtg::k_guide_collect<<<(c.wb.capacity + 255) / 256, 256, 0, st>>>(c, buf, count, cap);
}

void launch_batch(const float4* buf, const int* count, int cap, int n, uint32_t seed, float* pos, float* dir,
                  float* w, float* weight_sum, cudaStream_t st) {
    rtg::k_guide_batch<<<(n + 255) / 256, 256, 0, st>>>(buf, count, cap, n, seed, pos, dir, w, weight_sum);
}

static constexpr float kAdamB1 = 0.9f, kAdamB2 = 0.99f, kAdamEps = 1e-10f;

void launch_adam(float* p, __half* p16, float* grad, float* m, float* v, int64_t n, float lr, int step,
                 cudaStream_t st) {
    const float b1 = kAdamB1, b2 = kAdamB2, eps = kAdamEps;
    const float c1 = 1.0f / (1.0f - powf(b1, float(step))), c2 = 1.0f / (1.0f - powf(b2, float(step)));
    int blocks = int((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    rtg::k_adam<<<blocks, 256, 0, st>>>(p, p16, grad, m, v, n, lr, b1, b2, c1, c2, eps);
}

void launch_adam_table(float* p, __half* p16, float* grad, float* m, float* v, const int64_t* level_entries, float lr,
                       int step, cudaStream_t st) {
    const float b1 = kAdamB1, b2 = kAdamB2, eps = kAdamEps;
    const float c1 = 1.0f / (1.0f - powf(b1, float(step))), c2 = 1.0f / (1.0f - powf(b2, float(step)));
    rtg::LevelExtents ext;
    int64_t most = 1;
    for (int l = 0; l < rtg::kLevels; l++) {
        ext.n[l] = int32_t(std::min<int64_t>(level_entries[l], rtg::kT));
        most = std::max<int64_t>(most, ext.n[l]);
    }
    const int gx = int(std::min<int64_t>((most + 255) / 256, 256));
    rtg::k_adam_table<<<dim3(gx, rtg::kLevels), 256, 0, st>>>(
        reinterpret_cast<float2*>(p), reinterpret_cast<__half2*>(p16), reinterpret_cast<float2*>(grad),
        reinterpret_cast<float2*>(m), reinterpret_cast<float2*>(v), ext, lr, b1, b2, c1, c2, eps);
}

void launch_to_half(const float* p, __half* p16, int64_t n, cudaStream_t st) {
    int blocks = int((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    rtg::k_to_half<<<blocks, 256, 0, st>>>(p, p16, n);
}

void launch_pdf_sample(const rtg::Mixture* mix, const float* dir, const float* u, int n, float* out_dir, float* pdf,
                       cudaStream_t st) {
    if (n <= 0) return;
    rtg::k_guide_pdf_sample<<<(n + 127) / 128, 128, 0, st>>>(mix, dir, u, n, out_dir, pdf);
}

}  // namespace rtgh
