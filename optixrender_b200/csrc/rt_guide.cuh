// rt_guide.cuh - the path-guiding network: constants, the per-query mixture
// record, and the von Mises-Fisher mixture used by the shade kernel.
//
// Network (no counterpart in the reference renderer): a multiresolution hash
// encoding of the position (Mueller et al., "Instant Neural Graphics
// Primitives", 2022: 16 levels x 2 features, 2^19 entries per level) feeding a
// 32-64-64-64-32 MLP without biases (ReLU hidden layers, FP16 weights, FP32
// accumulation), whose 32 outputs are an 8-lobe vMF mixture over incident
// directions: lobe k reads (weight logit, log concentration, polar angle,
// azimuth) from outputs 4k..4k+3.
#pragma once

#include <cuda_fp16.h>

#include "rt_device.cuh"

namespace rtg {

constexpr int kLevels = 16;
constexpr int kFeats = 2;
constexpr int kLog2T = 19;
constexpr int kT = 1 << kLog2T;
constexpr int kIn = kLevels * kFeats;  // 32
constexpr int kHid = 64;
constexpr int kOut = 32;
constexpr int kLobes = 8;
constexpr int kW0 = kHid * kIn, kW1 = kHid * kHid, kW2 = kHid * kHid, kW3 = kOut * kHid;
constexpr int kMlpParams = kW0 + kW1 + kW2 + kW3;  // 12288
constexpr int64_t kTableParams = int64_t(kLevels) * kT * kFeats;
constexpr float kKappaLo = -2.0f;  // lowest log-concentration (the highest is per network)
constexpr uint32_t kPrime1 = 2654435761u, kPrime2 = 805459861u;

// Mixture of one query: lobe k = (mu.xyz, kappa) and the normalised weights.
struct __align__(16) Mixture {
    float4 lobe[kLobes];
    float w[kLobes];
};

// Device view of the network's parameters.
struct NetView {
    const __half2* table;  // kLevels * kT entries (fp16 features)
    const __half* mlp;     // kMlpParams, W0 W1 W2 W3 row-major [out][in]
    float3 lo, inv_ext;    // position normalisation: (x - lo) * inv_ext in [0, 1]
    int res[kLevels];      // grid resolution of each level
    float kappa_hi;        // highest log-concentration of a lobe
};

// Guiding state of a wave, read by the wavefront kernels.
constexpr int kGuideRec = 3;  // training records per path (the first bounces)
struct GuideCtx {
    Mixture* mix;        // per slot: this bounce's mixture (null: the wave is not guided)
    float4* rec;         // training records, [kGuideRec][4][capacity] float4 (null: no training)
    float prob;          // probability of sampling the mixture at a guided vertex
    float min_rough;     // conductors and clear coats rougher than this are guided
    float3 lo, inv_ext;  // position normalisation of the scene
};

#ifdef __CUDACC__
// Raw network outputs -> mixture (softmax weights, kappa = exp(clamped),
// mu from theta = pi * sigmoid, phi = 2 pi * sigmoid).
RT_D void head_from_outputs(const float* o, Mixture& m, float kappa_hi) {
    float mx = o[0];
#pragma unroll
    for (int k = 1; k < kLobes; k++) mx = fmaxf(mx, o[4 * k]);
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; k++) {
        m.w[k] = __expf(o[4 * k] - mx);
        sum += m.w[k];
    }
    const float inv = 1.0f / sum;
#pragma unroll
    for (int k = 0; k < kLobes; k++) {
        m.w[k] *= inv;
        float kap = __expf(fminf(fmaxf(o[4 * k + 1], kKappaLo), kappa_hi));
        float th = 3.14159265358979f / (1.0f + __expf(-o[4 * k + 2]));
        float ph = 6.28318530717959f / (1.0f + __expf(-o[4 * k + 3]));
        float st, ct, sp, cp;
        __sincosf(th, &st, &ct);
        __sincosf(ph, &sp, &cp);
        m.lobe[k] = make_float4(st * cp, st * sp, ct, kap);
    }
}

// vMF density kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.d - 1)).
RT_D float vmf_pdf(float4 l, rtd::v3 d) {
    const float c = l.x * d.x + l.y * d.y + l.z * d.z;
    return l.w / (6.28318530717959f * -expm1f(-2.0f * l.w)) * __expf(l.w * (c - 1.0f));
}

// Lobe of a mixture picked by u0: the first k with u0 < w_0 + ... + w_k (the
// last lobe when rounding leaves u0 above the running sum).  Constant indices
// only, so the weights stay in registers.
RT_D int pick_lobe(const float (&w)[kLobes], float u0) {
    int k = kLobes - 1;
    float acc = 0.0f;
    bool found = false;
#pragma unroll
    for (int j = 0; j < kLobes - 1; j++) {
        acc += w[j];
        if (!found && u0 < acc) {
            k = j;
            found = true;
        }
    }
    return k;
}

// Samples the vMF lobe l = (mu, kappa) with (u1, u2): the cosine to mu is
// 1 + log(u1 + (1 - u1) e^{-2 kappa}) / kappa (Jakob, "Numerically stable
// sampling of the von Mises Fisher distribution on S2", 2012).
RT_D rtd::v3 vmf_sample(float4 l, float u1, float u2) {
    float w = 1.0f + __logf(u1 + (1.0f - u1) * __expf(-2.0f * l.w)) / l.w;
    w = fminf(fmaxf(w, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float sp, cp;
    __sincosf(6.28318530717959f * u2, &sp, &cp);
    const rtd::v3 mu(l.x, l.y, l.z);
    // orthonormal basis around mu (Duff et al., "Building an orthonormal basis, revisited", 2017)
    const float sg = copysignf(1.0f, mu.z);
    const float a = -1.0f / (sg + mu.z), b = mu.x * mu.y * a;
    const rtd::v3 t1(1.0f + sg * mu.x * mu.x * a, sg * b, -sg * mu.x);
    const rtd::v3 t2(b, sg + mu.y * mu.y * a, -mu.y);
    return normalize(t1 * (s * cp) + t2 * (s * sp) + mu * w);
}

// Density and sampling of a mixture in global memory (read-only for the kernel).
RT_D float mixture_pdf(const Mixture* m, rtd::v3 d) {
    const float4* w4 = reinterpret_cast<const float4*>(m->w);
    const float4 wa = __ldg(w4), wb = __ldg(w4 + 1);
    const float w[kLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    float p = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; k++) p += w[k] * vmf_pdf(__ldg(m->lobe + k), d);
    return p;
}
// Picks a lobe with u0 and samples it with (u1, u2).
RT_D rtd::v3 mixture_sample(const Mixture* m, float u0, float u1, float u2) {
    const float4* w4 = reinterpret_cast<const float4*>(m->w);
    const float4 wa = __ldg(w4), wb = __ldg(w4 + 1);
    const float w[kLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    return vmf_sample(__ldg(m->lobe + pick_lobe(w, u0)), u1, u2);
}

// Network input of a surface point: the position moved by kSideOffset (in
// normalised scene units) along the geometric normal turned towards the
// incoming ray, so that the two sides of a thin wall read different hash
// cells at the fine levels; then normalised and clamped to [0, 1]^3.
constexpr float kSideOffset = 1.0f / 512.0f;
RT_D float3 guide_input(rtd::v3 p, rtd::v3 p0, rtd::v3 p1, rtd::v3 p2, rtd::v3 d, const GuideCtx& G) {
    rtd::v3 ng = cross(p1 - p0, p2 - p0);
    const float len = sqrtf(dot(ng, ng));
    ng = len > 0.0f ? ng * (1.0f / len) : rtd::v3(0.0f);
    if (dot(ng, d) > 0.0f) ng = -ng;
    float3 x;
    x.x = fminf(fmaxf((p.x - G.lo.x) * G.inv_ext.x + kSideOffset * ng.x, 0.f), 1.f);
    x.y = fminf(fmaxf((p.y - G.lo.y) * G.inv_ext.y + kSideOffset * ng.y, 0.f), 1.f);
    x.z = fminf(fmaxf((p.z - G.lo.z) * G.inv_ext.z + kSideOffset * ng.z, 0.f), 1.f);
    return x;
}

// Material types whose vertices are guided (dielectrics never; conductors and
// clear coats only above the roughness threshold).
RT_D bool guided_type(int type) { return type != RT_MAT_DIELECTRIC && type != RT_MAT_THIN_DIELECTRIC; }
#endif

}  // namespace rtg
