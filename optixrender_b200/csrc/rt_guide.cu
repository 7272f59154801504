// rt_guide.cu - fused kernels of the path-guiding network.
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

constexpr int kWarps = 4;
constexpr int kBlock = kWarps * 32;
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

// d[j] = A (16 x K) * W^T (K x N) for the weight W [N][K] in shared memory, row stride S.
template <int K, int N, int S>
RT_D void layer(const uint32_t (&a)[K / 16][4], const __half* W, float (&d)[N / 8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < N / 8; j++) {
        d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.0f;
        const __half* row = W + (8 * j + g) * S + 2 * tig;
#pragma unroll
        for (int t = 0; t < K / 16; t++) {
            uint32_t b0 = *reinterpret_cast<const uint32_t*>(row + 16 * t);
            uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + 16 * t + 8);
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

// Deltas masked by the ReLU of the forward activations `h` (A fragments), packed to A fragments.
template <int N>
RT_D void pack_masked(const float (&d)[N / 8][4], const uint32_t (&h)[N / 16][4], uint32_t (&a)[N / 16][4]) {
#pragma unroll
    for (int t = 0; t < N / 16; t++) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const float* src = d[2 * t + (r >> 1)] + 2 * (r & 1);
            float2 hv = unpack_h2(h[t][r]);
            a[t][r] = pack_h2(hv.x > 0.f ? src[0] : 0.f, hv.y > 0.f ? src[1] : 0.f);
        }
    }
}

// Training stores, per 16-sample tile, the fragments the weight gradients
// need, word-major ([word][lane], so every store and load is one 128-byte
// line): output delta (2 x 4 words), then the input and delta of each hidden
// layer, then the encoded input.  k_guide_wgrad forms dW_l = E^T X from them.
constexpr int kFragAdo = 0, kFragH3 = 8, kFragE3 = 24, kFragH2 = 40, kFragE2 = 56, kFragH1 = 72, kFragE1 = 88,
              kFragAx = 104, kFragWords = 112;

template <int T>
RT_D void frag_store(uint32_t* tile_frags, int off, const uint32_t (&f)[T][4], int lane) {
#pragma unroll
    for (int t = 0; t < T; t++)
#pragma unroll
        for (int r = 0; r < 4; r++) tile_frags[(off + 4 * t + r) * 32 + lane] = f[t][r];
}

struct Corners {
    uint32_t idx[8];
    float w[8];
};

RT_D void level_corners(const int* res_table, int l, float3 x, Corners& c) {
    const int res = res_table[l];
    const float fr = float(res);
    float px = x.x * fr, py = x.y * fr, pz = x.z * fr;
    float cx = fminf(floorf(px), fr - 1.0f), cy = fminf(floorf(py), fr - 1.0f), cz = fminf(floorf(pz), fr - 1.0f);
    const float fx = px - cx, fy = py - cy, fz = pz - cz;
    const uint32_t ix = uint32_t(cx), iy = uint32_t(cy), iz = uint32_t(cz);
    const uint32_t r1 = uint32_t(res) + 1u;
    const bool dense = uint64_t(r1) * r1 * r1 <= uint64_t(kT);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t gx = ix + (k & 1), gy = iy + ((k >> 1) & 1), gz = iz + ((k >> 2) & 1);
        c.idx[k] = dense ? gx + gy * r1 + gz * r1 * r1 : ((gx * 1u) ^ (gy * kPrime1) ^ (gz * kPrime2)) & uint32_t(kT - 1);
        c.w[k] = ((k & 1) ? fx : 1.0f - fx) * (((k >> 1) & 1) ? fy : 1.0f - fy) * (((k >> 2) & 1) ? fz : 1.0f - fz);
    }
}

RT_D uint32_t encode_level(const __half2* __restrict__ table, const int* res, int l, float3 x) {
    Corners c;
    level_corners(res, l, x, c);
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
        a[t][0] = vg ? encode_level(net.table, net.res, l0, xg) : 0u;
        a[t][1] = vg8 ? encode_level(net.table, net.res, l0, xg8) : 0u;
        a[t][2] = vg ? encode_level(net.table, net.res, l1, xg) : 0u;
        a[t][3] = vg8 ? encode_level(net.table, net.res, l1, xg8) : 0u;
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

// Forward of 16 rows: returns the output accumulators (4 n-tiles of 8 outputs).
RT_D void forward_tile(const __half* sw, const uint32_t (&ax)[2][4], float (&out)[4][4]) {
    float d64[8][4];
    uint32_t h[4][4];
    layer<kIn, kHid, kS32>(ax, sw + kOffW0, d64);
    pack_relu<kHid>(d64, h);
    layer<kHid, kHid, kS64>(h, sw + kOffW1, d64);
    pack_relu<kHid>(d64, h);
    layer<kHid, kHid, kS64>(h, sw + kOffW2, d64);
    pack_relu<kHid>(d64, h);
    layer<kHid, kOut, kS64>(h, sw + kOffW3, out);
}

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

// Raw outputs (mode 0) or mixtures (mode 1) of n normalised positions.
__global__ void __launch_bounds__(kBlock) k_guide_forward(NetView net, const float* __restrict__ pos, int n, int mode,
                                                          float* __restrict__ raw, Mixture* __restrict__ mix) {
    extern __shared__ __align__(16) unsigned char smem[];
    __half* sw = reinterpret_cast<__half*>(smem);
    float* tiles = reinterpret_cast<float*>(smem + kFwdHalves * sizeof(__half));
    load_weights(net.mlp, sw, nullptr);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2;
    float* tile = tiles + warp * 16 * kTileStride;
    const int tiles_total = (n + 15) / 16;
    for (int tt = blockIdx.x * kWarps + warp; tt < tiles_total; tt += gridDim.x * kWarps) {
        const int r0 = tt * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        float3 x0 = v0 ? ld_pos(pos, r0) : make_float3(0.f, 0.f, 0.f);
        float3 x1 = v1 ? ld_pos(pos, r1) : make_float3(0.f, 0.f, 0.f);
        uint32_t ax[2][4];
        encode_tile(net, x0, x1, v0, v1, ax);
        float out[4][4];
        forward_tile(sw, ax, out);
        stage_outputs(out, tile);
        __syncwarp();
        if (lane < 16 && tt * 16 + lane < n) {
            const int64_t row = int64_t(tt) * 16 + lane;
            const float* o = tile + lane * kTileStride;
            if (mode == 0) {
                for (int k = 0; k < kOut; k++) raw[row * kOut + k] = o[k];
            } else {
                Mixture m;
                head_from_outputs(o, m, net.kappa_hi);
                mix[row] = m;
            }
        }
        __syncwarp();
    }
}

// Loss gradient of one row with respect to its 32 raw outputs (in place),
// for -s * log q(d); returns the row's loss term.
RT_D float loss_grad_row(float* o, float3 d, float s, float kappa_hi) {
    float w[kLobes], kap[kLobes], dens[kLobes];
    float3 mu[kLobes], dth[kLobes], dph[kLobes];
    float st[kLobes], sp[kLobes];
    bool inr[kLobes];
    float mx = o[0];
    for (int k = 1; k < kLobes; k++) mx = fmaxf(mx, o[4 * k]);
    float sum = 0.f;
    for (int k = 0; k < kLobes; k++) {
        w[k] = expf(o[4 * k] - mx);
        sum += w[k];
    }
    float q = 0.f;
    for (int k = 0; k < kLobes; k++) {
        w[k] /= sum;
        const float kr = o[4 * k + 1];
        inr[k] = kr >= kKappaLo && kr <= kappa_hi;
        kap[k] = expf(fminf(fmaxf(kr, kKappaLo), kappa_hi));
        st[k] = 1.f / (1.f + expf(-o[4 * k + 2]));
        sp[k] = 1.f / (1.f + expf(-o[4 * k + 3]));
        const float th = 3.14159265358979f * st[k], ph = 6.28318530717959f * sp[k];
        const float s_t = sinf(th), c_t = cosf(th), s_p = sinf(ph), c_p = cosf(ph);
        mu[k] = make_float3(s_t * c_p, s_t * s_p, c_t);
        dth[k] = make_float3(c_t * c_p, c_t * s_p, -s_t);
        dph[k] = make_float3(-s_t * s_p, s_t * c_p, 0.f);
        const float c = mu[k].x * d.x + mu[k].y * d.y + mu[k].z * d.z;
        dens[k] = kap[k] / (6.28318530717959f * -expm1f(-2.f * kap[k])) * expf(kap[k] * (c - 1.f));
        q += w[k] * dens[k];
    }
    q = fmaxf(q, 1e-30f);
    for (int k = 0; k < kLobes; k++) {
        const float r = w[k] * dens[k] / q;
        const float c = mu[k].x * d.x + mu[k].y * d.y + mu[k].z * d.z;
        const float dlogk = 1.f / kap[k] - 2.f / expm1f(2.f * kap[k]) + (c - 1.f);
        o[4 * k] = s * (w[k] - r);
        o[4 * k + 1] = inr[k] ? s * -r * dlogk * kap[k] : 0.f;
        o[4 * k + 2] = s * -r * kap[k] * (dth[k].x * d.x + dth[k].y * d.y + dth[k].z * d.z) * 3.14159265358979f *
                       st[k] * (1.f - st[k]);
        o[4 * k + 3] = s * -r * kap[k] * (dph[k].x * d.x + dph[k].y * d.y + dph[k].z * d.z) * 6.28318530717959f *
                       sp[k] * (1.f - sp[k]);
    }
    return -s * logf(q);
}

// Forward + loss + backward of n samples (position, unit direction, weight);
// `scale` multiplies every sample weight (1 / batch).  Adds the gradients to
// grad_table / grad_mlp and the loss to *loss.
__global__ void __launch_bounds__(kBlock) k_guide_backward(NetView net, const float* __restrict__ pos,
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
    load_weights(net.mlp, sw, sb);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    float* tile = tiles + warp * 16 * kTileStride;
    float lsum = 0.f;
    const int tiles_total = (n + 15) / 16;
    for (int tt = blockIdx.x * kWarps + warp; tt < tiles_total; tt += gridDim.x * kWarps) {
        const int r0 = tt * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        const float3 x0 = v0 ? ld_pos(pos, r0) : make_float3(0.f, 0.f, 0.f);
        const float3 x1 = v1 ? ld_pos(pos, r1) : make_float3(0.f, 0.f, 0.f);
        uint32_t ax[2][4], h1[4][4], h2[4][4], h3[4][4];
        encode_tile(net, x0, x1, v0, v1, ax);
        float d64[8][4], out[4][4];
        layer<kIn, kHid, kS32>(ax, sw + kOffW0, d64);
        pack_relu<kHid>(d64, h1);
        layer<kHid, kHid, kS64>(h1, sw + kOffW1, d64);
        pack_relu<kHid>(d64, h2);
        layer<kHid, kHid, kS64>(h2, sw + kOffW2, d64);
        pack_relu<kHid>(d64, h3);
        layer<kHid, kOut, kS64>(h3, sw + kOffW3, out);
        stage_outputs(out, tile);
        __syncwarp();
        if (lane < 16) {
            const int row = tt * 16 + lane;
            float* o = tile + lane * kTileStride;
            if (row < n) {
                const float3 dd = ld_pos(dir, row);
                lsum += loss_grad_row(o, dd, weight[row] * scale, net.kappa_hi);
            } else {
                for (int k = 0; k < kOut; k++) o[k] = 0.f;
            }
        }
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
        uint32_t* tf = frags + size_t(tt) * kFragWords * 32;
        frag_store<2>(tf, kFragAdo, ado, lane);
        frag_store<4>(tf, kFragH3, h3, lane);
        frag_store<4>(tf, kFragH2, h2, lane);
        frag_store<4>(tf, kFragH1, h1, lane);
        frag_store<2>(tf, kFragAx, ax, lane);
        uint32_t e[4][4];
        layer<kOut, kHid, kS32>(ado, sb + kOffT3, d64);
        pack_masked<kHid>(d64, h3, e);
        frag_store<4>(tf, kFragE3, e, lane);
        layer<kHid, kHid, kS64>(e, sb + kOffT2, d64);
        pack_masked<kHid>(d64, h2, e);
        frag_store<4>(tf, kFragE2, e, lane);
        layer<kHid, kHid, kS64>(e, sb + kOffT1, d64);
        pack_masked<kHid>(d64, h1, e);
        frag_store<4>(tf, kFragE1, e, lane);
        float dx[4][4];
        layer<kHid, kIn, kS64>(e, sb + kOffT0, dx);
        // hash-grid gradient: this thread's levels 4j + tig for rows g (dx[j][0..1]) and g + 8 (dx[j][2..3])
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int l = 4 * j + tig;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (!(h ? v1 : v0)) continue;
                Corners c;
                level_corners(net.res, l, h ? x1 : x0, c);
                float2* gt = reinterpret_cast<float2*>(grad_table) + size_t(l) * kT;
                const float g0 = dx[j][2 * h], g1 = dx[j][2 * h + 1];
#pragma unroll
                for (int k = 0; k < 8; k++) atomicAdd(gt + c.idx[k], make_float2(c.w[k] * g0, c.w[k] * g1));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0 && lsum != 0.f) atomicAdd(loss, lsum);
}

// Weight gradients dW_l[M][N] += E^T X from the fragments of `tiles` tiles.
// Warp w of a block plays role w: a 16-row block of one layer's outputs
// (layer 3: 2 blocks, layers 2, 1, 0: 4 each), whose 16 x N gradient stays in
// registers across the block's chunk of tiles and is added to global memory
// once.  The 14 warps of a block read the same tiles, so those loads hit L1.
constexpr int kWgradRoles = 14;
template <int M, int N>
RT_D void wgrad_role(const uint32_t* __restrict__ frags, int t0, int t1, int offE, int offX, int mt, float* gW) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    float acc[N / 8][4];
#pragma unroll
    for (int j = 0; j < N / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    for (int tt = t0; tt < t1; tt++) {
        const uint32_t* tf = frags + size_t(tt) * kFragWords * 32 + lane;
        uint32_t x[N / 16][4];
#pragma unroll
        for (int t = 0; t < N / 16; t++)
#pragma unroll
            for (int r = 0; r < 4; r++) x[t][r] = __ldg(tf + (offX + 4 * t + r) * 32);
        uint32_t e4[4];
#pragma unroll
        for (int r = 0; r < 4; r++) e4[r] = __ldg(tf + (offE + 4 * mt + r) * 32);
        const uint32_t at[4] = {trans8x8(e4[0]), trans8x8(e4[2]), trans8x8(e4[1]), trans8x8(e4[3])};
#pragma unroll
        for (int j = 0; j < N / 8; j++) {
            const int t = j >> 1, hi = j & 1;
            mma16816(acc[j], at, trans8x8(x[t][hi ? 2 : 0]), trans8x8(x[t][hi ? 3 : 1]));
        }
    }
#pragma unroll
    for (int j = 0; j < N / 8; j++) {
        float* p = gW + (16 * mt + g) * N + 8 * j + 2 * tig;
        if (acc[j][0] != 0.f) atomicAdd(p, acc[j][0]);
        if (acc[j][1] != 0.f) atomicAdd(p + 1, acc[j][1]);
        if (acc[j][2] != 0.f) atomicAdd(p + 8 * N, acc[j][2]);
        if (acc[j][3] != 0.f) atomicAdd(p + 8 * N + 1, acc[j][3]);
    }
}

__global__ void __launch_bounds__(kWgradRoles * 32) k_guide_wgrad(const uint32_t* __restrict__ frags, int tiles,
                                                                  int chunk, float* __restrict__ grad_mlp) {
    const int role = threadIdx.x >> 5;
    const int t0 = blockIdx.x * chunk, t1 = min(tiles, t0 + chunk);
    if (t0 >= t1) return;
    if (role < 2)
        wgrad_role<kOut, kHid>(frags, t0, t1, kFragAdo, kFragH3, role, grad_mlp + kW0 + kW1 + kW2);
    else if (role < 6)
        wgrad_role<kHid, kHid>(frags, t0, t1, kFragE3, kFragH2, role - 2, grad_mlp + kW0 + kW1);
    else if (role < 10)
        wgrad_role<kHid, kHid>(frags, t0, t1, kFragE2, kFragH1, role - 6, grad_mlp + kW0);
    else
        wgrad_role<kHid, kIn>(frags, t0, t1, kFragE1, kFragAx, role - 10, grad_mlp);
}

// ------------------------------------------------------------------ renderer side
// Items of the sorted shade queue whose material type is guided, in bucket order.
struct GuidedItems {
    int bucket[kShadeBucketsG], count[kShadeBucketsG], n;
};

RT_D GuidedItems guided_items(const rtd::WaveCtl* ctl) {
    GuidedItems gi;
    int m = 0;
    gi.n = 0;
    for (int b = 0; b < rtd::kShadeBuckets; b++) {
        if (b == rtd::kMissBucket || !guided_type(b)) continue;
        gi.bucket[m] = b;
        gi.count[m] = ctl->bucket[b];
        gi.n += gi.count[m];
        m++;
    }
    for (; m < kShadeBucketsG; m++) gi.bucket[m] = gi.count[m] = 0;
    return gi;
}

RT_D int guided_slot(const GuidedItems& gi, const rtd::WaveBufs& B, int i) {
    int m = 0, base = 0;
    while (m < kShadeBucketsG - 1 && i >= base + gi.count[m]) base += gi.count[m++];
    return B.sorted[size_t(gi.bucket[m]) * size_t(B.capacity) + size_t(i - base)];
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

// Mixtures of this bounce's guided vertices (surface hits of guided material
// types), written per slot for the shade kernel.
// Warps per block of k_guide_infer, which share the weights in shared memory.
// 16 warps x 2 blocks per SM (register-limited) keep 32 warps per SM in the
// latency-bound hash-grid gathers: 25% less time per guided sample than
// 4 x 4 or 4 x 6, on the portal scene.
constexpr int kInferWarps = 16;
constexpr int kInferBlocksPerSm = 2;
__global__ void __launch_bounds__(kInferWarps * 32) k_guide_infer(rtd::Ctx c, NetView net) {
    extern __shared__ __align__(16) unsigned char smem[];
    __half* sw = reinterpret_cast<__half*>(smem);
    float* tiles = reinterpret_cast<float*>(smem + kFwdHalves * sizeof(__half));
    load_weights(net.mlp, sw, nullptr);
    __syncthreads();
    const rtd::WaveBufs& B = c.wb;
    const GuidedItems gi = guided_items(B.ctl);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2;
    float* tile = tiles + warp * 16 * kTileStride;
    const int n = gi.n;
    const int tiles_total = (n + 15) / 16;
    for (int tt = blockIdx.x * kInferWarps + warp; tt < tiles_total; tt += gridDim.x * kInferWarps) {
        const int r0 = tt * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        const int s0 = v0 ? guided_slot(gi, B, r0) : 0, s1 = v1 ? guided_slot(gi, B, r1) : 0;
        const float3 x0 = v0 ? hit_position(c, s0) : make_float3(0.f, 0.f, 0.f);
        const float3 x1 = v1 ? hit_position(c, s1) : make_float3(0.f, 0.f, 0.f);
        uint32_t ax[2][4];
        encode_tile(net, x0, x1, v0, v1, ax);
        float out[4][4];
        forward_tile(sw, ax, out);
        stage_outputs(out, tile);
        __syncwarp();
        if (lane < 16 && tt * 16 + lane < n) {
            const int slot = guided_slot(gi, B, tt * 16 + lane);
            Mixture m;
            head_from_outputs(tile + lane * kTileStride, m, net.kappa_hi);
            c.G.mix[slot] = m;
        }
        __syncwarp();
    }
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

// A training batch of `n` samples: all collected ones when they fit, else a
// uniform random subset (with replacement); accumulates the batch's weight sum
// for the loss scale.
__global__ void k_guide_batch(const float4* __restrict__ buf, const int* __restrict__ count, int cap, int n,
                              uint32_t seed, float* __restrict__ pos, float* __restrict__ dir, float* __restrict__ w,
                              float* __restrict__ weight_sum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cnt = min(*count, cap);
    float wi = 0.f;
    if (i < n) {
        float4 a = make_float4(0.5f, 0.5f, 0.5f, 0.f), b = make_float4(0.f, 0.f, 1.f, 0.f);
        if (cnt > n) {  // a random subset (with replacement)
            uint32_t h = uint32_t(i) * 0x9E3779B9u ^ seed;
            h ^= h >> 16;
            h *= 0x85EBCA6Bu;
            h ^= h >> 13;
            h *= 0xC2B2AE35u;
            h ^= h >> 16;
            const int j = int(uint64_t(h) * uint64_t(cnt) >> 32);
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
    const Mixture m = mix[i];
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

size_t forward_smem() { return size_t(rtg::kFwdHalves) * 2 + size_t(rtg::kWarps) * 16 * rtg::kTileStride * 4; }
static size_t infer_smem() {
    return size_t(rtg::kFwdHalves) * 2 + size_t(rtg::kInferWarps) * 16 * rtg::kTileStride * 4;
}
size_t backward_smem() {
    return size_t(rtg::kFwdHalves + rtg::kBwdHalves) * 2 + size_t(rtg::kWarps) * 16 * rtg::kTileStride * 4;
}

cudaError_t prepare_kernels() {
    cudaError_t e = cudaFuncSetAttribute(rtg::k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(forward_smem()));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(rtg::k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, int(infer_smem()));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(rtg::k_guide_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(backward_smem()));
}

static int grid_for_tiles(int n, int sms) {
    const int tiles = (n + 15) / 16;
    const int blocks = (tiles + rtg::kWarps - 1) / rtg::kWarps;
    return blocks < sms * 8 ? (blocks > 0 ? blocks : 1) : sms * 8;
}

void launch_forward(const rtg::NetView& net, const float* pos, int n, int mode, float* raw, rtg::Mixture* mix, int sms,
                    cudaStream_t st) {
    if (n <= 0) return;
    rtg::k_guide_forward<<<grid_for_tiles(n, sms), rtg::kBlock, forward_smem(), st>>>(net, pos, n, mode, raw, mix);
}

size_t frag_bytes_per_tile() { return size_t(rtg::kFragWords) * 32 * 4; }

void launch_backward(const rtg::NetView& net, const float* pos, const float* dir, const float* weight, int n,
                     float scale, const float* weight_sum, float* grad_table, float* grad_mlp, float* loss,
                     uint32_t* frags, int frag_tiles, int sms, cudaStream_t st) {
    // chunks of at most frag_tiles tiles: the fused pass stores their
    // fragments, then k_guide_wgrad turns them into weight gradients
    for (int begin = 0; begin < n; begin += frag_tiles * 16) {
        const int m = std::min(n - begin, frag_tiles * 16);
        const int tiles = (m + 15) / 16;
        int blocks = (tiles + rtg::kWarps - 1) / rtg::kWarps;
        if (blocks > sms * 3) blocks = sms * 3;  // shared weights and transposes, ~64 KB per block
        rtg::k_guide_backward<<<blocks, rtg::kBlock, backward_smem(), st>>>(
            net, pos + size_t(begin) * 3, dir + size_t(begin) * 3, weight + begin, m, scale, weight_sum, grad_table,
            frags, loss);
        const int chunk = std::max(4, (tiles + 2 * sms - 1) / (2 * sms));
        rtg::k_guide_wgrad<<<(tiles + chunk - 1) / chunk, rtg::kWgradRoles * 32, 0, st>>>(frags, tiles, chunk,
                                                                                          grad_mlp);
    }
}

void launch_infer(const rtd::Ctx& c, const rtg::NetView& net, int sms, cudaStream_t st) {
    rtg::k_guide_infer<<<sms * rtg::kInferBlocksPerSm, rtg::kInferWarps * 32, infer_smem(), st>>>(c, net);
}

void launch_collect(const rtd::Ctx& c, float4* buf, int* count, int cap, cudaStream_t st) {
    rtg::k_guide_collect<<<(c.wb.capacity + 255) / 256, 256, 0, st>>>(c, buf, count, cap);
}

void launch_batch(const float4* buf, const int* count, int cap, int n, uint32_t seed, float* pos, float* dir,
                  float* w, float* weight_sum, cudaStream_t st) {
    rtg::k_guide_batch<<<(n + 255) / 256, 256, 0, st>>>(buf, count, cap, n, seed, pos, dir, w, weight_sum);
}

void launch_adam(float* p, __half* p16, float* grad, float* m, float* v, int64_t n, float lr, int step,
                 cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-10f;
    const float c1 = 1.0f / (1.0f - powf(b1, float(step))), c2 = 1.0f / (1.0f - powf(b2, float(step)));
    int blocks = int((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    rtg::k_adam<<<blocks, 256, 0, st>>>(p, p16, grad, m, v, n, lr, b1, b2, c1, c2, eps);
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
