// pt_oracle.hpp - CPU oracle for the B200 path tracer.
//
// TEST INFRASTRUCTURE ONLY.  This is a restatement, in plain C++ templated on
// the scalar type, of the reference renderer's device code
// (GraphicsEnthusiast/OptiXRender, core/cuda/*.h and
// core/cuda/devicePrograms.cu).  R = double is the FP64 oracle used to check
// the GPU's FP32 shading; R = float follows the GPU arithmetic closely enough
// that, fed the same random streams, it traces the same paths and is the
// per-pixel image oracle.  Every function cites the reference lines it
// follows.  Nothing in the product links or calls this file.
//
// Deliberate difference from the reference (applied identically on the GPU):
// a next-event-estimation sample whose light pdf is zero or not finite adds
// nothing.  In the reference such a sample evaluates 0*x/0 = NaN, which then
// drops the pixel's remaining samples (devicePrograms.cu:329,422,469,499-501).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/rt_capi.h"

namespace orc {

// ---------------------------------------------------------------- vectors
// gdt vec_t<float,3> semantics (common/gdt/gdt/math/vec.h:299-316):
// dot is left to right, length = sqrt(dot), normalize divides each component.
template <class R>
struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a) : x(a), y(a), z(a) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R& operator[](int i) { return (&x)[i]; }
    const R& operator[](int i) const { return (&x)[i]; }
};
template <class R> inline V3<R> operator+(const V3<R>& a, const V3<R>& b) { return V3<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R> inline V3<R> operator-(const V3<R>& a, const V3<R>& b) { return V3<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R> inline V3<R> operator*(const V3<R>& a, const V3<R>& b) { return V3<R>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class R> inline V3<R> operator/(const V3<R>& a, const V3<R>& b) { return V3<R>(a.x / b.x, a.y / b.y, a.z / b.z); }
template <class R> inline V3<R> operator*(const V3<R>& a, R s) { return V3<R>(a.x * s, a.y * s, a.z * s); }
template <class R> inline V3<R> operator*(R s, const V3<R>& a) { return V3<R>(s * a.x, s * a.y, s * a.z); }
template <class R> inline V3<R> operator/(const V3<R>& a, R s) { return V3<R>(a.x / s, a.y / s, a.z / s); }
template <class R> inline V3<R> operator/(R s, const V3<R>& a) { return V3<R>(s / a.x, s / a.y, s / a.z); }
template <class R> inline V3<R> operator+(const V3<R>& a, R s) { return V3<R>(a.x + s, a.y + s, a.z + s); }
template <class R> inline V3<R> operator+(R s, const V3<R>& a) { return V3<R>(s + a.x, s + a.y, s + a.z); }
template <class R> inline V3<R> operator-(const V3<R>& a, R s) { return V3<R>(a.x - s, a.y - s, a.z - s); }
template <class R> inline V3<R> operator-(R s, const V3<R>& a) { return V3<R>(s - a.x, s - a.y, s - a.z); }
template <class R> inline V3<R> operator-(const V3<R>& a) { return V3<R>(-a.x, -a.y, -a.z); }
template <class R> inline V3<R>& operator+=(V3<R>& a, const V3<R>& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
template <class R> inline V3<R>& operator*=(V3<R>& a, const V3<R>& b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
template <class R> inline V3<R>& operator/=(V3<R>& a, const V3<R>& b) { a.x /= b.x; a.y /= b.y; a.z /= b.z; return a; }
template <class R> inline V3<R>& operator*=(V3<R>& a, R s) { a.x *= s; a.y *= s; a.z *= s; return a; }
template <class R> inline V3<R>& operator/=(V3<R>& a, R s) { a.x /= s; a.y /= s; a.z /= s; return a; }
template <class R> inline R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(const V3<R>& a, const V3<R>& b) {
    return V3<R>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <class R> inline R length(const V3<R>& v) { return std::sqrt(dot(v, v)); }
template <class R> inline V3<R> normalize(const V3<R>& v) { return v / std::sqrt(dot(v, v)); }
template <class R> inline V3<R> vabs(const V3<R>& v) { return V3<R>(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }
template <class R> inline bool is_nan3(const V3<R>& v) { return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z); }
template <class R> inline V3<R> from3(const float* p) { return V3<R>(R(p[0]), R(p[1]), R(p[2])); }

// Device min/max (fminf/fmaxf): a NaN operand yields the other one.
template <class R> inline R dmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R dmax(R a, R b) { return std::fmax(a, b); }
template <class R> inline R clampr(R v, R lo, R hi) { return dmin(hi, dmax(lo, v)); }
template <class R> inline R sqr(R x) { return x * x; }
template <class R> inline R mixr(R x, R y, R t) { return x * (R(1) - t) + y * t; }

template <class R> struct K {
    static constexpr R EPS = R(1e-4f);                                  // core/cuda/Utils.h:10
    static constexpr R PI = R(3.14159265358979323846);                  // Utils.h:11
    static constexpr R TWO_PI = R(6.28318530717958647692);              // Utils.h:14
    static constexpr R INV_PI = R(0.318309886183790671538);             // Utils.h:13
};

// ---------------------------------------------------------------- random
// gdt::LCG<16>, common/gdt/gdt/random/random.h:54-87: TEA-16 seed, 24-bit LCG.
struct LCG {
    uint32_t state;
    void init(uint32_t val0, uint32_t val1) {
        uint32_t v0 = val0, v1 = val1, s0 = 0;
        for (int n = 0; n < 16; n++) {
            s0 += 0x9e3779b9u;
            v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
            v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
        }
        state = v0;
    }
    float next() {
        state = 1664525u * state + 1013904223u;
        return float(state & 0x00FFFFFFu) / float(0x01000000);
    }
};

// PCG32 (O'Neill, pcg-random.org, "pcg32_random_r"); one stream per path.
struct PCG {
    uint64_t state, inc;
    void seed(uint64_t initstate, uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        step();
        state += initstate;
        step();
    }
    void step() { state = state * 6364136223846793005ULL + inc; }
    uint32_t next_u32() {
        uint64_t old = state;
        step();
        uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    float next() { return float(next_u32() >> 8) * (1.0f / 16777216.0f); }
};

// A random source: either stream, or a fixed list of numbers (verification).
struct Rng {
    int kind = 0;  // 0 LCG, 1 PCG, 2 list
    LCG lcg;
    PCG pcg;
    const float* list = nullptr;
    int list_n = 0, used = 0;
    float next() {
        used++;
        if (kind == 0) return lcg.next();
        if (kind == 1) return pcg.next();
        return (used - 1) < list_n ? list[used - 1] : 0.5f;
    }
};

inline uint64_t pcg_frame_state(uint64_t seed, int frame) {
    return seed ^ (uint64_t(uint32_t(frame)) * 0x9E3779B97F4A7C15ULL);
}

// ---------------------------------------------------------------- sampling
// core/cuda/Sampling.h:5-10
template <class R> inline R power_heuristic(R p1, R p2) {
    R a = p1 * p1, b = p2 * p2;
    return a / (a + b);
}
// Sampling.h:12-24
template <class R> inline V3<R> plane_to_sphere(R u, R v) {
    R phi = K<R>::TWO_PI * (u - R(0.5f));
    R theta = K<R>::PI * (v - R(0.5f));
    return normalize(V3<R>(std::cos(theta) * std::cos(phi), std::sin(theta), std::cos(theta) * std::sin(phi)));
}
// Sampling.h:26-33
template <class R> inline void sphere_to_plane(const V3<R>& d, R& u, R& v) {
    u = std::atan2(d.z, d.x);
    v = std::asin(d.y);
    u /= K<R>::TWO_PI;
    v /= K<R>::PI;
    u += R(0.5f);
    v += R(0.5f);
}
// Sampling.h:36-52
template <class R> inline V3<R> uniform_sample_cone(R s0, R s1, R cos_angle) {
    R phi = K<R>::TWO_PI * s0;
    R cos_theta = mixr(cos_angle, R(1), s1);
    R sin_theta = std::sqrt(R(1) - cos_theta * cos_theta);
    return normalize(V3<R>(sin_theta * std::cos(phi), sin_theta * std::sin(phi), cos_theta));
}
template <class R> inline R uniform_pdf_cone(R cos_angle) { return R(1) / (K<R>::TWO_PI * (R(1) - cos_angle)); }
// Sampling.h:56-73
template <class R> inline V3<R> cosine_sample_hemisphere(R s0, R s1) {
    R r = std::sqrt(s0);
    R phi = K<R>::TWO_PI * s1;
    V3<R> p(r * std::cos(phi), r * std::sin(phi), R(0));
    p.z = std::sqrt(dmax(R(0), R(1) - p.x * p.x - p.y * p.y));
    return normalize(p);
}
template <class R> inline R cosine_pdf_hemisphere(R ndotl) { return ndotl * K<R>::INV_PI; }
// Sampling.h:76-88
template <class R> inline V3<R> uniform_sample_sphere(R s0, R s1) {
    R phi = K<R>::TWO_PI * s0;
    R cos_theta = R(1) - R(2) * s1;
    R sin_theta = std::sqrt(R(1) - cos_theta * cos_theta);
    return normalize(V3<R>(sin_theta * std::cos(phi), sin_theta * std::sin(phi), cos_theta));
}

// ---------------------------------------------------------------- frames
// core/cuda/Utils.h:28-38
template <class R> inline V3<R> reflect(const V3<R>& v, const V3<R>& n) { return normalize(v - R(2) * dot(v, n) * n); }
template <class R> inline V3<R> refract(const V3<R>& v, const V3<R>& n, R eta) {
    R cos_theta = dmin(dot(-v, n), R(1));
    V3<R> perp = eta * (v + cos_theta * n);
    V3<R> par = -std::sqrt(std::fabs(R(1) - dot(perp, perp))) * n;
    return normalize(perp + par);
}
// Utils.h:99-112
template <class R> inline V3<R> to_local(const V3<R>& dir, const V3<R>& up) {
    V3<R> C;
    if (std::fabs(up.x) > std::fabs(up.y)) {
        R inv = R(1) / std::sqrt(up.x * up.x + up.z * up.z);
        C = V3<R>(up.z * inv, R(0), -up.x * inv);
    } else {
        R inv = R(1) / std::sqrt(up.y * up.y + up.z * up.z);
        C = V3<R>(R(0), up.z * inv, -up.y * inv);
    }
    V3<R> B = cross(C, up);
    return V3<R>(dot(dir, B), dot(dir, C), dot(dir, up));
}
// Utils.h:117-129
template <class R> inline V3<R> to_world(const V3<R>& dir, const V3<R>& up) {
    V3<R> C;
    if (std::fabs(up.x) > std::fabs(up.y)) {
        R inv = R(1) / std::sqrt(up.x * up.x + up.z * up.z);
        C = V3<R>(up.z * inv, R(0), -up.x * inv);
    } else {
        R inv = R(1) / std::sqrt(up.y * up.y + up.z * up.z);
        C = V3<R>(R(0), up.z * inv, -up.y * inv);
    }
    V3<R> B = cross(C, up);
    return normalize(dir.x * B + dir.y * C + dir.z * up);
}
// Utils.h:76-78
template <class R> inline R luminance(const V3<R>& c) { return dot(V3<R>(R(0.299f), R(0.587f), R(0.114f)), c); }

// ---------------------------------------------------------------- microfacet
// core/cuda/Microfacet.h:22-46
template <class R> inline V3<R> fresnel_conductor(const V3<R>& V, const V3<R>& H, const V3<R>& er, const V3<R>& ei) {
    R c = dot(V, H), c2 = c * c, s2 = R(1) - c2, s4 = s2 * s2;
    V3<R> t1 = er * er - ei * ei - s2;
    V3<R> a2pb2 = t1 * t1 + R(4) * ei * ei * er * er;
    for (int i = 0; i < 3; i++) a2pb2[i] = std::sqrt(dmax(R(0), a2pb2[i]));
    V3<R> a = R(0.5f) * (a2pb2 + t1);
    for (int i = 0; i < 3; i++) a[i] = std::sqrt(dmax(R(0), a[i]));
    V3<R> term1 = a2pb2 + s2, term2 = R(2) * c * a, term3 = a2pb2 * c2 + s4, term4 = term2 * s2;
    V3<R> rs = (term1 - term2) / (term1 + term2);
    V3<R> rp = rs * (term3 - term4) / (term3 + term4);
    return R(0.5f) * (rs + rp);
}
// Microfacet.h:48-70
template <class R> inline V3<R> average_fresnel_conductor(const V3<R>& eta, const V3<R>& k) {
    V3<R> refl, edge;
    for (int i = 0; i < 3; i++) {
        refl[i] = (sqr(eta[i] - R(1)) + sqr(k[i])) / (sqr(eta[i] + R(1)) + sqr(k[i]));
        R t1 = R(1) + std::sqrt(refl[i]);
        R t2 = R(1) - std::sqrt(refl[i]);
        R t3 = (R(1) - refl[i]) / (R(1) + refl[i]);
        edge[i] = (t1 - eta[i] * t2) / (t1 - t3 * t2);
    }
    return V3<R>(R(0.087237f)) + R(0.0230685f) * edge - R(0.0864902f) * edge * edge +
           R(0.0774594f) * edge * edge * edge + R(0.782654f) * refl - R(0.136432f) * refl * refl +
           R(0.278708f) * refl * refl * refl + R(0.19744f) * edge * refl + R(0.0360605f) * edge * edge * refl -
           R(0.2586f) * edge * refl * refl;
}
// Microfacet.h:72-85
template <class R> inline R fresnel_dielectric(const V3<R>& V, const V3<R>& H, R eta_inv) {
    R ci = std::fabs(dot(V, H));
    R ct2 = R(1) - sqr(eta_inv) * (R(1) - sqr(ci));
    if (ct2 <= R(0)) return R(1);
    R ct = std::sqrt(ct2);
    R rs = (eta_inv * ci - ct) / (eta_inv * ci + ct);
    R rp = (ci - eta_inv * ct) / (ci + eta_inv * ct);
    return (rs * rs + rp * rp) / R(2);
}
// Microfacet.h:87-113
template <class R> inline R average_fresnel_dielectric(R eta) {
    if (eta < R(1)) return R(-1.4399f) * (eta * eta) + R(0.7099f) * eta + R(0.6681f) + R(0.0636f) / eta;
    R i1 = R(1) / eta, i2 = i1 * i1, i3 = i2 * i1, i4 = i3 * i1, i5 = i4 * i1;
    return R(0.919317f) - R(3.4793f) * i1 + R(6.75335f) * i2 - R(7.80989f) * i3 + R(4.98554f) * i4 -
           R(1.36881f) * i5;
}
// Microfacet.h:117-142
template <class R> inline R smith_g1(const V3<R>& V, const V3<R>& H, const V3<R>& N, R au, R av) {
    R cvn = dot(V, N);
    if (cvn * dot(V, H) <= R(0)) return R(0);
    if (std::fabs(cvn - R(1)) < K<R>::EPS) return R(1);
    if (au == av) {
        R c2 = sqr(cvn), t2 = (R(1) - c2) / c2, a2 = au * au;
        return R(2) / (R(1) + std::sqrt(R(1) + a2 * t2));
    }
    V3<R> d = to_local(V, N);
    R xy = sqr(au * d.x) + sqr(av * d.y), t = xy / sqr(d.z);
    return R(2) / (R(1) + std::sqrt(R(1) + t));
}
// Microfacet.h:144-160
template <class R> inline R ggx_d(const V3<R>& H, const V3<R>& N, R au, R av) {
    R c = dot(H, N);
    if (c <= R(0)) return R(0);
    R c2 = sqr(c), t2 = (R(1) - c2) / c2, a2 = au * av;
    if (au == av) return a2 / (K<R>::PI * std::pow(c, R(2)) * sqr(a2 + t2));
    V3<R> d = to_local(H, N);
    return R(1) / (K<R>::PI * a2 * sqr(sqr(d.x / au) + sqr(d.y / av) + sqr(d.z)));
}
// Microfacet.h:162-164
template <class R> inline R ggx_dv(const V3<R>& V, const V3<R>& H, const V3<R>& N, R au, R av) {
    return smith_g1(V, H, N, au, av) * dot(V, H) * ggx_d(H, N, au, av) / dot(N, V);
}
// Microfacet.h:166-186
template <class R> inline V3<R> sample_ggx(R au, R av, R s0, R s1) {
    R sp, cp, a2;
    if (au == av) {
        R phi = K<R>::TWO_PI * s1;
        cp = std::cos(phi);
        sp = std::sin(phi);
        a2 = au * au;
    } else {
        R phi = std::atan(av / au * std::tan(K<R>::PI + K<R>::TWO_PI * s1)) + K<R>::PI * std::floor(R(2) * s1 + R(0.5f));
        cp = std::cos(phi);
        sp = std::sin(phi);
        a2 = R(1) / (sqr(cp / au) + sqr(sp / av));
    }
    R t2 = a2 * s0 / (R(1) - s0), ct = R(1) / std::sqrt(R(1) + t2), st = std::sqrt(R(1) - ct * ct);
    return normalize(V3<R>(st * cp, st * sp, ct));
}
// Microfacet.h:188-214 (returns H in the local frame of N)
template <class R> inline V3<R> sample_vndf(const V3<R>& N, const V3<R>& Ve, R au, R av, R s0, R s1) {
    V3<R> V = to_local(Ve, N);
    V3<R> Vh = normalize(V3<R>(au * V.x, av * V.y, V.z));
    R len2 = sqr(Vh.x) + sqr(Vh.y);
    V3<R> T1 = len2 > R(0) ? V3<R>(-Vh.y, Vh.x, R(0)) * std::sqrt(R(1) / len2) : V3<R>(R(1), R(0), R(0));
    V3<R> T2 = cross(Vh, T1);
    R r = std::sqrt(s0), phi = s1 * K<R>::TWO_PI;
    R t1 = r * std::cos(phi), t2 = r * std::sin(phi);
    R s = R(0.5f) * (R(1) + Vh.z);
    t2 = (R(1) - s) * std::sqrt(R(1) - sqr(t1)) + s * t2;
    V3<R> Nh = t1 * T1 + t2 * T2 + std::sqrt(dmax(R(0), R(1) - sqr(t1) - sqr(t2))) * Vh;
    return normalize(V3<R>(au * Nh.x, av * Nh.y, dmax(R(0), Nh.z)));
}

// Kulla-Conty tables, Microfacet.h:218-291.  Always computed in float: the
// renderer uploads the float table and both precisions read it.
constexpr int kLut = 64;
inline void hammersley(uint32_t i, uint32_t N, float& a, float& b) {
    uint32_t bits = (i << 16u) | (i >> 16u);
    bits = ((bits & 0x55555555u) << 1u) | ((bits & 0xAAAAAAAAu) >> 1u);
    bits = ((bits & 0x33333333u) << 2u) | ((bits & 0xCCCCCCCCu) >> 2u);
    bits = ((bits & 0x0F0F0F0Fu) << 4u) | ((bits & 0xF0F0F0F0u) >> 4u);
    bits = ((bits & 0x00FF00FFu) << 8u) | ((bits & 0xFF00FF00u) >> 8u);
    b = static_cast<float>(float(bits) * 2.3283064365386963e-10f);
    a = float(i) / float(N);
}
inline void kulla_conty(float* bsdf, float* albedo_avg) {
    using R = float;
    const V3<R> N(0.f, 0.f, 1.f);
    auto integrate_bsdf = [&](const V3<R>& V, float rough) {
        const uint32_t n = 128;
        const float step = 1.0f / n;
        float acc = 0.f;
        for (uint32_t i = 0; i < n; ++i) {
            float a, b;
            hammersley(i + 1, n + 1, a, b);
            V3<R> H = sample_ggx<R>(rough, rough, a, b);
            V3<R> L = reflect(-V, H);
            float G = smith_g1(L, H, N, rough, rough) * smith_g1(V, H, N, rough, rough);
            float NdotV = dot(N, V), NdotL = dot(N, L), NdotH = dot(N, H), HdotV = dot(H, V);
            if (NdotL > 0.f && NdotH > 0.f && HdotV > 0.f) acc += (HdotV * G) / (NdotV * NdotH);
        }
        return std::min(acc * step, 1.0f);
    };
    auto integrate_albedo = [&](const V3<R>& V, float rough, float bs) {
        const uint32_t n = 128;
        const float step = 1.0f / n;
        float acc = 0.f;
        for (uint32_t i = 0; i < n; ++i) {
            float a, b;
            hammersley(i + 1, n + 1, a, b);
            V3<R> H = sample_ggx<R>(rough, rough, a, b);
            V3<R> L = reflect(-V, H);
            float HdotV = dot(H, V), NdotL = dot(N, L), NdotH = dot(N, H);
            if (NdotL > 0.f && NdotH > 0.f && HdotV > 0.f) acc += bs * NdotL;
        }
        return acc * 2.0f * step;
    };
    float step = 1.0f / kLut;
    for (int i = kLut - 1; i >= 0; --i) {
        float acc = 0.f;
        float rough = step * (static_cast<float>(i) + 0.5f);
        for (int j = kLut - 1; j >= 0; --j) {
            float NdotV = step * (static_cast<float>(j) + 0.5f);
            V3<R> V(std::sqrt(1.0f - NdotV * NdotV), 0.0f, NdotV);
            float avg = integrate_bsdf(V, rough);
            bsdf[i * kLut + j] = avg;
            acc += integrate_albedo(V, rough, avg);
        }
        albedo_avg[i] = acc * step;
    }
}
// Microfacet.h:293-324
template <class R> inline R get_bsdf_avg(R cos_theta, R rough, const float* t) {
    R o1 = sqr(rough) * R(kLut), o2 = cos_theta * R(kLut);
    int i1 = static_cast<int>(o1), i2 = static_cast<int>(o2);
    auto at = [&](int r, int c) { return R(t[r * kLut + c]); };
    if (i1 >= kLut - 1) {
        if (i2 >= kLut - 1) return at(kLut - 1, kLut - 1);
        return mixr(at(kLut - 1, i2), at(kLut - 1, i2 + 1), o2 - R(i2));
    }
    if (i2 >= kLut - 1) return mixr(at(i1, kLut - 1), at(i1 + 1, kLut - 1), o1 - R(i1));
    return mixr(mixr(at(i1, i2), at(i1 + 1, i2), o1 - R(i1)), mixr(at(i1, i2 + 1), at(i1 + 1, i2 + 1), o1 - R(i1)),
                o2 - R(i2));
}
// Microfacet.h:326-335
template <class R> inline R get_albedo_avg(R rough, const float* t) {
    R o = sqr(rough) * R(kLut);
    int i = static_cast<int>(o);
    if (i >= kLut - 1) return R(t[kLut - 1]);
    return mixr(R(t[i]), R(t[i + 1]), o - R(i));
}

// ---------------------------------------------------------------- materials
template <class R> struct Mat {
    int type;
    V3<R> albedo, eta, k, specular;
    R roughness, anisotropy, int_ior, ext_ior, metallic, coat_weight, cru, crv;
    bool nonlinear;
    int tex[8];      // texture ids (-1 = constant), rt_material.texture_ids order
    bool textured;
    void set(const rt_material& m) {
        type = m.type;
        textured = false;
        for (int t = 0; t < 8; t++) {
            tex[t] = m.texture_ids[t];
            textured = textured || tex[t] >= 0;
        }
        albedo = from3<R>(m.albedo);
        eta = from3<R>(m.eta);
        k = from3<R>(m.k);
        specular = from3<R>(m.specular);
        roughness = R(m.roughness);
        anisotropy = R(m.anisotropy);
        int_ior = R(m.int_ior);
        ext_ior = R(m.ext_ior);
        metallic = R(m.metallic);
        coat_weight = R(m.coat_weight);
        cru = R(m.coat_roughness_u);
        crv = R(m.coat_roughness_v);
        nonlinear = m.nonlinear != 0;
    }
};

// struct Interaction, core/cuda/Utils.h:62-74
template <class R> struct Isect {
    R distance;
    V3<R> position, sn;
    bool front;
    const Mat<R>* mat;
    int in_medium, out_medium;
    void set_face_normal(const V3<R>& dir, const V3<R>& n) {
        front = dot(dir, n) < R(0);
        sn = front ? n : -n;
    }
};

template <class R> struct Lut {
    const float* bsdf;
    const float* avg;
};

// Microfacet.h:337-346
template <class R> inline V3<R> multiple_scatter(const Lut<R>& lut, R NdotL, R NdotV, R rough, const V3<R>& Favg) {
    R bl = get_bsdf_avg(NdotL, rough, lut.bsdf), bv = get_bsdf_avg(NdotV, rough, lut.bsdf);
    R ea = get_albedo_avg(rough, lut.avg);
    R fms = (R(1) - bl) * (R(1) - bv) / (K<R>::PI * (R(1) - ea));
    V3<R> fadd = Favg * Favg * ea / (R(1) - Favg * (R(1) - ea));
    return fms * fadd;
}

// Diffuse, core/cuda/Material.h:7-72
template <class R> inline V3<R> diffuse_brdf(const Mat<R>& m, const V3<R>& N, const V3<R>& V, const V3<R>& L, R NdotL,
                                             R& pdf, bool& ok) {
    V3<R> H = normalize(V + L);
    R NdotV = dot(N, V), VdotH = dot(V, H);
    ok = !(NdotL <= R(0) || NdotV <= R(0));
    if (!ok) return V3<R>(R(0));
    R a = m.roughness * m.roughness, s2 = a * a;
    R VdotL = R(2) * VdotH * VdotH - R(1);
    R cosri = VdotL - NdotV * NdotL;
    R C1 = R(1) - R(0.5f) * s2 / (s2 + R(0.33f));
    R C2 = R(0.45f) * s2 / (s2 + R(0.09f)) * cosri * (cosri >= R(0) ? dmax(NdotL, NdotV) : R(1));
    pdf = cosine_pdf_hemisphere(NdotL);
    return m.albedo * K<R>::INV_PI * (C1 + C2) * (R(1) + m.roughness * R(0.5f));
}
template <class R> inline V3<R> eval_diffuse(const Isect<R>& it, const V3<R>& V, const V3<R>& L, R& pdf) {
    V3<R> lL = to_local(L, it.sn);
    bool ok;
    return diffuse_brdf(*it.mat, it.sn, V, L, lL.z, pdf, ok);
}
template <class R> inline V3<R> sample_diffuse(const Isect<R>& it, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    R u0 = rng.next(), u1 = rng.next();
    V3<R> lL = cosine_sample_hemisphere(u0, u1);
    L = to_world(lL, it.sn);
    bool ok;
    return diffuse_brdf(*it.mat, it.sn, V, L, lL.z, pdf, ok);
}

// Conductor, Material.h:76-146
template <class R> inline V3<R> conductor_common(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L,
                                                 const V3<R>& H, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    V3<R> Favg = average_fresnel_conductor(m.eta, m.k);
    const V3<R>& N = it.sn;
    R Dv = ggx_dv(V, H, N, au, av);
    pdf = Dv * std::fabs(R(1) / (R(4) * dot(V, H)));
    R NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= R(0) || NdotL <= R(0)) return V3<R>(R(0));
    V3<R> F = fresnel_conductor(V, H, m.eta, m.k);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    return m.albedo * (F * D * G / (R(4) * NdotV * NdotL) + multiple_scatter(lut, NdotL, NdotV, m.roughness, Favg));
}
template <class R> inline V3<R> eval_conductor(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L,
                                               R& pdf) {
    return conductor_common(it, lut, V, L, normalize(V + L), pdf);
}
template <class R> inline V3<R> sample_conductor(const Isect<R>& it, const Lut<R>& lut, Rng& rng, const V3<R>& V, V3<R>& L,
                                                 R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    R u0 = rng.next(), u1 = rng.next();
    V3<R> H = to_world(sample_vndf(it.sn, V, au, av, u0, u1), it.sn);
    L = reflect(-V, H);
    return conductor_common(it, lut, V, L, H, pdf);
}

// Dielectric, Material.h:150-269
template <class R> inline V3<R> eval_dielectric(const Isect<R>& it, const V3<R>& V, const V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    R eta = m.int_ior / m.ext_ior;
    R e = it.front ? (R(1) / eta) : eta;
    const V3<R>& N = it.sn;
    V3<R> H;
    bool refl = dot(N, L) * dot(N, V) > R(0);
    if (refl) {
        H = normalize(V + L);
    } else {
        H = -normalize(e * V + L);
        if (dot(N, H) < R(0)) H = -H;
    }
    R Dv = ggx_dv(V, H, N, au, av);
    pdf = Dv * std::fabs(R(1) / (R(4) * dot(V, H)));
    R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
    R F = fresnel_dielectric(V, H, e);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    if (refl) {
        R dwh = std::fabs(R(1) / (R(4) * dot(V, H)));
        pdf = F * Dv * dwh;
        return m.albedo * F * D * G / (R(4) * NdotV * NdotL);
    }
    R HdotV = dot(H, V), HdotL = dot(H, L);
    R sd = e * HdotV + HdotL;
    R factor = std::fabs(HdotL * HdotV / (NdotL * NdotV));
    R dwh = std::fabs(HdotL) / sqr(sd);
    pdf = (R(1) - F) * Dv * dwh;
    V3<R> f = m.albedo * (R(1) - F) * D * G * factor / sqr(sd);
    f *= sqr(R(1) / e);
    return f;
}
template <class R> inline V3<R> sample_dielectric(const Isect<R>& it, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    R eta = m.int_ior / m.ext_ior;
    R e = it.front ? (R(1) / eta) : eta;
    const V3<R>& N = it.sn;
    R u0 = rng.next(), u1 = rng.next();
    V3<R> H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
    R Dv = ggx_dv(V, H, N, au, av);
    R F = fresnel_dielectric(V, H, e);
    R D = ggx_d(H, N, au, av);
    if (R(rng.next()) < F) {
        L = reflect(-V, H);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
        R dwh = std::fabs(R(1) / (R(4) * dot(V, H)));
        pdf = F * Dv * dwh;
        R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
        R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
        return m.albedo * F * D * G / (R(4) * NdotV * NdotL);
    }
    L = refract(-V, H, e);
    if (dot(N, L) * dot(N, V) >= R(0)) return V3<R>(R(0));
    R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R HdotV = dot(H, V), HdotL = dot(H, L);
    R sd = e * HdotV + HdotL;
    R factor = std::fabs(HdotL * HdotV / (NdotL * NdotV));
    R dwh = std::fabs(HdotL) / sqr(sd);
    pdf = (R(1) - F) * Dv * dwh;
    V3<R> f = m.albedo * (R(1) - F) * D * G * factor / sqr(sd);
    f *= sqr(R(1) / e);
    return f;
}

// Plastic, Material.h:273-403
template <class R> inline V3<R> plastic_brdf(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L,
                                             const V3<R>& H, R Fo, R Fi, R pdf_spec, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    R eta = m.int_ior / m.ext_ior;
    R Favg = average_fresnel_dielectric(eta);
    const V3<R>& N = it.sn;
    R NdotV = dot(N, V), NdotL = dot(N, L);
    R Dv = ggx_dv(V, H, N, au, av);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    V3<R> F(fresnel_dielectric(L, H, R(1) / eta));
    V3<R> f = m.nonlinear ? m.albedo / (R(1) - m.albedo * Favg) : m.albedo / (R(1) - Favg);
    f *= (R(1) - Fi) * (R(1) - Fo) * K<R>::INV_PI;
    f += m.specular * (F * D * G / (R(4) * NdotL * NdotV) + multiple_scatter(lut, NdotL, NdotV, m.roughness, V3<R>(Favg)));
    pdf = pdf_spec * Dv * std::fabs(R(1) / (R(4) * dot(V, H))) + (R(1) - pdf_spec) * cosine_pdf_hemisphere(NdotL);
    return f;
}
template <class R> inline R plastic_spec_weight(const Mat<R>& m) {
    R d = m.albedo.x + m.albedo.y + m.albedo.z, s = m.specular.x + m.specular.y + m.specular.z;
    return s / (s + d);
}
template <class R> inline V3<R> eval_plastic(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R eta = m.int_ior / m.ext_ior;
    const V3<R>& N = it.sn;
    V3<R> H = normalize(V + L);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= R(0) || NdotL <= R(0)) return V3<R>(R(0));
    R Fo = fresnel_dielectric(V, N, R(1) / eta), Fi = fresnel_dielectric(L, N, R(1) / eta);
    R w = plastic_spec_weight(m);
    R ps = Fi * w, pd = (R(1) - Fi) * (R(1) - w);
    ps = ps / (ps + pd);
    return plastic_brdf(it, lut, V, L, H, Fo, Fi, ps, pdf);
}
template <class R> inline V3<R> sample_plastic(const Isect<R>& it, const Lut<R>& lut, Rng& rng, const V3<R>& V, V3<R>& L,
                                               R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    R eta = m.int_ior / m.ext_ior;
    const V3<R>& N = it.sn;
    R NdotV = dot(N, V);
    if (NdotV <= R(0)) return V3<R>(R(0));
    R Fo = fresnel_dielectric(V, N, R(1) / eta), Fi = Fo;
    R w = plastic_spec_weight(m);
    R ps = Fi * w, pd = (R(1) - Fi) * (R(1) - w);
    ps = ps / (ps + pd);
    V3<R> H;
    if (R(rng.next()) < ps) {
        R u0 = rng.next(), u1 = rng.next();
        H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
        L = reflect(-V, H);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
    } else {
        R u0 = rng.next(), u1 = rng.next();
        L = to_world(cosine_sample_hemisphere(u0, u1), N);
        H = normalize(V + L);
        Fi = fresnel_dielectric(L, N, R(1) / eta);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
    }
    return plastic_brdf(it, lut, V, L, H, Fo, Fi, ps, pdf);
}

// Metal workflow, Material.h:407-516
template <class R> inline V3<R> metal_brdf(const Isect<R>& it, const V3<R>& V, const V3<R>& L, const V3<R>& H, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    const V3<R>& N = it.sn;
    R NdotV = dot(N, V), NdotL = dot(N, L);
    R diel = R(1) - m.metallic;
    R spec = m.metallic + diel;
    R pdiff = diel / (diel + spec);
    R Dv = ggx_dv(V, H, N, au, av);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    V3<R> F0 = V3<R>(R(0.04f)) * (R(1) - m.metallic) + m.albedo * m.metallic;
    R vdh = dot(V, H);
    R tmp = R(1) - clampr(vdh, R(0), R(1));
    R tmp2 = tmp * tmp;
    R Fc = tmp2 * tmp2 * tmp;
    V3<R> F = F0 + (R(1) - F0) * Fc;
    V3<R> sb = D * F * G / (R(4) * NdotL * NdotV);
    V3<R> db = m.albedo * K<R>::INV_PI;
    pdf = (R(1) - pdiff) * Dv * std::fabs(R(1) / (R(4) * vdh)) + pdiff * cosine_pdf_hemisphere(NdotL);
    return pdiff * db + (R(1) - pdiff) * sb;
}
template <class R> inline V3<R> eval_metal(const Isect<R>& it, const V3<R>& V, const V3<R>& L, R& pdf) {
    const V3<R>& N = it.sn;
    V3<R> H = normalize(L + V);
    if (dot(N, V) <= R(0) || dot(N, L) <= R(0)) return V3<R>(R(0));
    return metal_brdf(it, V, L, H, pdf);
}
template <class R> inline V3<R> sample_metal(const Isect<R>& it, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.roughness) * (R(1) + m.anisotropy), av = sqr(m.roughness) * (R(1) - m.anisotropy);
    const V3<R>& N = it.sn;
    if (dot(N, V) <= R(0)) return V3<R>(R(0));
    R diel = R(1) - m.metallic, spec = m.metallic + diel, pdiff = diel / (diel + spec);
    V3<R> H;
    if (R(rng.next()) < pdiff) {
        R u0 = rng.next(), u1 = rng.next();
        L = to_world(cosine_sample_hemisphere(u0, u1), N);
        H = normalize(V + L);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
    } else {
        R u0 = rng.next(), u1 = rng.next();
        H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
        L = reflect(-V, H);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
    }
    return metal_brdf(it, V, L, H, pdf);
}

// Thin dielectric, Material.h:520-630
template <class R> inline R thin_fresnel(const V3<R>& V, const V3<R>& H, R eta) {
    R F = fresnel_dielectric(V, H, R(1) / eta);
    if (F < R(1)) F *= R(2) / (R(1) + F);
    return F;
}
template <class R> inline V3<R> eval_thin(const Isect<R>& it, const V3<R>& V, const V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R eta = m.int_ior / m.ext_ior, a = sqr(m.roughness);
    const V3<R>& N = it.sn;
    V3<R> H;
    bool refl = dot(N, L) * dot(N, V) > R(0);
    if (refl) {
        H = normalize(V + L);
    } else {
        V3<R> Vr = to_world(to_local(V, -N), N);
        H = normalize(Vr + L);
        if (dot(N, H) < R(0)) H = -H;
    }
    R Dv = ggx_dv(V, H, N, a, a);
    R F = thin_fresnel(V, H, eta);
    R D = ggx_d(H, N, a, a);
    R dwh = std::fabs(R(1) / (R(4) * dot(V, H)));
    R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
    R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
    if (refl) {
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
        pdf = F * Dv * dwh;
        return m.albedo * F * D * G / (R(4) * NdotV * NdotL);
    }
    if (dot(N, L) * dot(N, V) >= R(0)) return V3<R>(R(0));
    pdf = (R(1) - F) * Dv * dwh;
    return m.albedo * (R(1) - F) * D * G / (R(4) * NdotV * NdotL);
}
template <class R> inline V3<R> sample_thin(const Isect<R>& it, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R eta = m.int_ior / m.ext_ior, a = sqr(m.roughness);
    const V3<R>& N = it.sn;
    R u0 = rng.next(), u1 = rng.next();
    V3<R> H = to_world(sample_vndf(N, V, a, a, u0, u1), N);
    R Dv = ggx_dv(V, H, N, a, a);
    R F = thin_fresnel(V, H, eta);
    R D = ggx_d(H, N, a, a);
    if (R(rng.next()) < F) {
        L = reflect(-V, H);
        if (dot(N, L) <= R(0)) return V3<R>(R(0));
        R dwh = std::fabs(R(1) / (R(4) * dot(V, H)));
        R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
        R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
        pdf = F * Dv * dwh;
        return m.albedo * F * D * G / (R(4) * NdotV * NdotL);
    }
    L = -V;
    if (dot(N, L) * dot(N, V) >= R(0)) return V3<R>(R(0));
    R NdotV = std::fabs(dot(N, V)), NdotL = std::fabs(dot(N, L));
    R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
    R dwh = std::fabs(R(1) / (R(4) * dot(V, H)));
    pdf = (R(1) - F) * Dv * dwh;
    return m.albedo * (R(1) - F) * D * G / (R(4) * NdotV * NdotL);
}

// Clear-coated conductor, Material.h:634-734
template <class R> inline V3<R> eval_clearcoat(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L, R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.cru), av = sqr(m.crv);
    const V3<R>& N = it.sn;
    V3<R> H = normalize(V + L);
    R Dv = ggx_dv(V, H, N, au, av);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= R(0) || NdotL <= R(0)) return V3<R>(R(0));
    R F = fresnel_dielectric(V, H, R(1) / R(1.5f));
    R cw = m.coat_weight * F;
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    R cpdf = R(0);
    R coat_pdf = Dv * std::fabs(R(1) / (R(4) * dot(V, H)));
    V3<R> cond = eval_conductor(it, lut, V, L, cpdf);
    V3<R> coat(D * G / (R(4) * NdotV * NdotL));
    pdf = cw * coat_pdf + (R(1) - cw) * cpdf;
    return cw * coat + (R(1) - cw) * cond;
}
template <class R> inline V3<R> sample_clearcoat(const Isect<R>& it, const Lut<R>& lut, Rng& rng, const V3<R>& V, V3<R>& L,
                                                 R& pdf) {
    const Mat<R>& m = *it.mat;
    R au = sqr(m.cru), av = sqr(m.crv);
    const V3<R>& N = it.sn;
    R F = fresnel_dielectric(V, N, R(1) / R(1.5f));
    R cw = m.coat_weight * F;
    if (R(rng.next()) < cw) {
        R u0 = rng.next(), u1 = rng.next();
        V3<R> H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
        L = reflect(-V, H);
        R NdotV = dot(N, V), NdotL = dot(N, L);
        if (NdotV <= R(0) || NdotL <= R(0)) return V3<R>(R(0));
        R Dv = ggx_dv(V, H, N, au, av);
        F = fresnel_dielectric(V, H, R(1) / R(1.5f));
        cw = m.coat_weight * F;
        R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
        R D = ggx_d(H, N, au, av);
        R coat_pdf = Dv * std::fabs(R(1) / (R(4) * dot(V, H)));
        R cpdf = R(0);
        V3<R> cond = eval_conductor(it, lut, V, L, cpdf);
        V3<R> coat(D * G / (R(4) * NdotV * NdotL));
        pdf = cw * coat_pdf + (R(1) - cw) * cpdf;
        return cw * coat + (R(1) - cw) * cond;
    }
    R cpdf = R(0);
    V3<R> cond = sample_conductor(it, lut, rng, V, L, cpdf);
    V3<R> H = normalize(V + L);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= R(0) || NdotL <= R(0)) return V3<R>(R(0));
    R Dv = ggx_dv(V, H, N, au, av);
    F = fresnel_dielectric(V, H, R(1) / R(1.5f));
    cw = m.coat_weight * F;
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    R coat_pdf = Dv * std::fabs(R(1) / (R(4) * dot(V, H)));
    V3<R> coat(D * G / (R(4) * NdotV * NdotL));
    pdf = cw * coat_pdf + (R(1) - cw) * cpdf;
    return cw * coat + (R(1) - cw) * cond;
}

// Diffuse transmitter, Material.h:738-779
template <class R> inline V3<R> eval_transmitter(const Isect<R>& it, const V3<R>& V, const V3<R>& L, R& pdf) {
    V3<R> N = -it.sn;
    V3<R> lL = to_local(L, N);
    R NdotL = lL.z, NdotV = dot(N, V);
    if (NdotL * NdotV >= R(0)) return V3<R>(R(0));
    pdf = cosine_pdf_hemisphere(std::fabs(NdotL));
    return it.mat->albedo * K<R>::INV_PI;
}
template <class R> inline V3<R> sample_transmitter(const Isect<R>& it, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    R u0 = rng.next(), u1 = rng.next();
    V3<R> lL = cosine_sample_hemisphere(u0, u1);
    V3<R> N = -it.sn;
    L = to_world(lL, N);
    R NdotL = lL.z, NdotV = dot(N, V);
    if (NdotL * NdotV >= R(0)) return V3<R>(R(0));
    pdf = cosine_pdf_hemisphere(std::fabs(NdotL));
    return it.mat->albedo * K<R>::INV_PI;
}

// Material.h:783-813
template <class R> inline V3<R> eval_material(const Isect<R>& it, const Lut<R>& lut, const V3<R>& V, const V3<R>& L, R& pdf) {
    pdf = R(0);
    if (!it.mat) return V3<R>(R(0));
    switch (it.mat->type) {
        case RT_MAT_DIFFUSE: return eval_diffuse(it, V, L, pdf);
        case RT_MAT_CONDUCTOR: return eval_conductor(it, lut, V, L, pdf);
        case RT_MAT_DIELECTRIC: return eval_dielectric(it, V, L, pdf);
        case RT_MAT_PLASTIC: return eval_plastic(it, lut, V, L, pdf);
        case RT_MAT_METAL_WORKFLOW: return eval_metal(it, V, L, pdf);
        case RT_MAT_THIN_DIELECTRIC: return eval_thin(it, V, L, pdf);
        case RT_MAT_CLEARCOATED_CONDUCTOR: return eval_clearcoat(it, lut, V, L, pdf);
        case RT_MAT_DIFFUSE_TRANSMITTER: return eval_transmitter(it, V, L, pdf);
    }
    return V3<R>(R(0));
}
// Material.h:815-845
template <class R> inline V3<R> sample_material(const Isect<R>& it, const Lut<R>& lut, Rng& rng, const V3<R>& V, V3<R>& L,
                                                R& pdf) {
    pdf = R(0);
    if (!it.mat) return V3<R>(R(0));
    switch (it.mat->type) {
        case RT_MAT_DIFFUSE: return sample_diffuse(it, rng, V, L, pdf);
        case RT_MAT_CONDUCTOR: return sample_conductor(it, lut, rng, V, L, pdf);
        case RT_MAT_DIELECTRIC: return sample_dielectric(it, rng, V, L, pdf);
        case RT_MAT_PLASTIC: return sample_plastic(it, lut, rng, V, L, pdf);
        case RT_MAT_METAL_WORKFLOW: return sample_metal(it, rng, V, L, pdf);
        case RT_MAT_THIN_DIELECTRIC: return sample_thin(it, rng, V, L, pdf);
        case RT_MAT_CLEARCOATED_CONDUCTOR: return sample_clearcoat(it, lut, rng, V, L, pdf);
        case RT_MAT_DIFFUSE_TRANSMITTER: return sample_transmitter(it, rng, V, L, pdf);
    }
    return V3<R>(R(0));
}

// The renderer's BSDF sampler: SampleMaterial evaluated in double precision on
// the FP32 inputs and random numbers, rounded once (optixrender_b200's
// sample_material).  The FP32 render oracle samples with it so that the same
// random streams trace the same paths; the FP32 shading ops keep the
// reference's own FP32 sampler (the golden-vector pins).
inline V3<double> sample_material_device(const Isect<double>& it, const Lut<double>& lut, Rng& rng,
                                         const V3<double>& V, V3<double>& L, double& pdf) {
    return sample_material(it, lut, rng, V, L, pdf);
}
inline V3<float> sample_material_device(const Isect<float>& it, const Lut<float>& lut, Rng& rng, const V3<float>& V,
                                        V3<float>& L, float& pdf) {
    auto d3 = [](const V3<float>& v) { return V3<double>(double(v.x), double(v.y), double(v.z)); };
    Mat<double> md;
    if (it.mat) {
        const Mat<float>& m = *it.mat;
        md.type = m.type;
        md.albedo = d3(m.albedo);
        md.eta = d3(m.eta);
        md.k = d3(m.k);
        md.specular = d3(m.specular);
        md.roughness = m.roughness, md.anisotropy = m.anisotropy, md.int_ior = m.int_ior, md.ext_ior = m.ext_ior;
        md.metallic = m.metallic, md.coat_weight = m.coat_weight, md.cru = m.cru, md.crv = m.crv;
        md.nonlinear = m.nonlinear;
        for (int t = 0; t < 8; t++) md.tex[t] = m.tex[t];
        md.textured = m.textured;
    }
    Isect<double> id;
    id.distance = it.distance;
    id.position = d3(it.position);
    id.sn = d3(it.sn);
    id.front = it.front;
    id.mat = it.mat ? &md : nullptr;
    id.in_medium = it.in_medium;
    id.out_medium = it.out_medium;
    const Lut<double> ld{lut.bsdf, lut.avg};
    V3<double> Ld = d3(L);
    double pd = 0.0;
    const V3<double> f = sample_material(id, ld, rng, d3(V), Ld, pd);
    L = V3<float>(float(Ld.x), float(Ld.y), float(Ld.z));
    pdf = float(pd);
    return V3<float>(float(f.x), float(f.y), float(f.z));
}

// ---------------------------------------------------------------- lights
template <class R> struct Lt {
    int type;
    bool two_sided;
    V3<R> radiance, position, u, v;
    R radius;
    int medium;
    void set(const rt_light& l) {
        type = l.type;
        two_sided = l.double_side != 0;
        radiance = from3<R>(l.radiance);
        position = from3<R>(l.position);
        u = from3<R>(l.u);
        v = from3<R>(l.v);
        radius = R(l.radius);
        medium = l.medium;
    }
};
// core/cuda/Light.h:6-26
template <class R> inline R intersect_quad(const V3<R>& o, const V3<R>& d, const V3<R>& corner, const V3<R>& u_, const V3<R>& v_) {
    V3<R> n = normalize(cross(u_, v_));
    V3<R> u = u_ * (R(1) / dot(u_, u_));
    V3<R> v = v_ * (R(1) / dot(v_, v_));
    R dt = dot(d, n);
    R t = (dot(n, corner) - dot(n, o)) / dt;
    if (t > K<R>::EPS) {
        V3<R> p = o + d * t;
        V3<R> vi = p - corner;
        R a1 = dot(u, vi);
        if (a1 >= R(0) && a1 <= R(1)) {
            R a2 = dot(v, vi);
            if (a2 >= R(0) && a2 <= R(1)) return t;
        }
    }
    return R(FLT_MAX);
}
// Light.h:78-98
template <class R> inline R intersect_sphere(const V3<R>& o, const V3<R>& d, const V3<R>& c, R radius) {
    V3<R> co = c - o;
    R b = dot(co, d);
    R det = b * b - dot(co, co) + radius * radius;
    if (det < R(0)) return R(FLT_MAX);
    det = std::sqrt(det);
    R t1 = b - det;
    if (t1 > K<R>::EPS) return t1;
    R t2 = b + det;
    if (t2 > K<R>::EPS) return t2;
    return R(FLT_MAX);
}
// EvaluateLight, Light.h:28-52, 100-116, 145-156.  A point light cannot be hit.
template <class R> inline V3<R> evaluate_light(const Lt<R>& l, const V3<R>& o, const V3<R>& d, R distance, R& pdf, R& ld) {
    if (l.type == RT_LIGHT_QUAD) {
        V3<R> n = normalize(cross(l.u, l.v));
        R ct = dot(d, n);
        if (!l.two_sided && ct < R(0)) {
            pdf = R(0);
            return V3<R>(R(0));
        }
        ld = intersect_quad(o, d, l.position, l.u, l.v);
        R area = length(l.u) * length(l.v);
        if (ld < distance) {
            pdf = R(1) / area;
            pdf *= sqr(ld) / std::fabs(ct);
            return l.radiance;
        }
        pdf = R(0);
        return V3<R>(R(0));
    }
    if (l.type == RT_LIGHT_SPHERE) {
        ld = intersect_sphere(o, d, l.position, l.radius);
        if (ld < distance) {
            V3<R> dir = l.position - o;
            R d2 = dot(dir, dir);
            R s2 = l.radius * l.radius / d2;
            R ct = std::sqrt(R(1) - s2);
            pdf = uniform_pdf_cone(ct);
            return l.radiance;
        }
        pdf = R(0);
        return V3<R>(R(0));
    }
    pdf = R(0);
    return V3<R>(R(0));
}
// SampleLight, Light.h:54-76, 118-141, 158-168.  A point light returns
// radiance / distance^2 with pdf 1 (a delta distribution).
template <class R> inline V3<R> sample_light(const Lt<R>& l, const V3<R>& p, R s0, R s1, V3<R>& L, R& dist, R& pdf) {
    if (l.type == RT_LIGHT_QUAD) {
        V3<R> n = normalize(cross(l.u, l.v));
        V3<R> pos = l.position + l.u * s0 + l.v * s1;
        L = pos - p;
        R d2 = dot(L, L);
        dist = std::sqrt(d2);
        L /= dist;
        R ct = dot(L, n);
        if (!l.two_sided && ct < R(0)) {
            pdf = R(0);
            return V3<R>(R(0));
        }
        R area = length(l.u) * length(l.v);
        pdf = R(1) / area;
        pdf *= d2 / std::fabs(ct);
        return l.radiance;
    }
    if (l.type == RT_LIGHT_SPHERE) {
        V3<R> dir = l.position - p;
        R d2 = dot(dir, dir);
        R inv = R(1) / std::sqrt(d2);
        dir *= inv;
        dist = d2 * inv;
        R st = l.radius * inv;
        if (st < R(1)) {
            R ct = std::sqrt(R(1) - st * st);
            V3<R> lL = uniform_sample_cone(s0, s1, ct);
            R ci = lL.z;
            L = to_world(lL, dir);
            pdf = uniform_pdf_cone(ct);
            dist = ci * dist - std::sqrt(dmax(R(0), l.radius * l.radius - (R(1) - ci * ci) * d2));
            return l.radiance;
        }
        pdf = R(0);
        return V3<R>(R(0));
    }
    if (l.type == RT_LIGHT_POINT) {
        V3<R> dir = l.position - p;
        R d2 = dot(dir, dir);
        dist = std::sqrt(d2);
        L = dir / dist;
        pdf = R(1);
        return l.radiance / d2;
    }
    pdf = R(0);
    return V3<R>(R(0));
}

// ---------------------------------------------------------------- media
template <class R> struct Grid;
template <class R> struct Med {
    int type, phase;
    V3<R> g, sigma_s, sigma_a;
    R scale;
    const Grid<R>* grid = nullptr;
    void set(const rt_medium& m) {
        type = m.type;
        phase = m.phase;
        g = from3<R>(m.g);
        sigma_s = from3<R>(m.sigma_s);
        sigma_a = from3<R>(m.sigma_a);
        scale = R(m.scale);
    }
};
// core/cuda/Medium.h:7-79 (isotropic and per-channel Henyey-Greenstein)
template <class R> inline V3<R> hg_terms(const Med<R>& m, R ct, R& pdf) {
    V3<R> att;
    pdf = R(0);
    for (int c = 0; c < 3; ++c) {
        R g = m.g[c];
        R tmp = R(1) + g * g + R(2) * g * ct;
        att[c] = (R(0.25f) * K<R>::INV_PI) * (R(1) - g * g) / (tmp * std::sqrt(tmp));
        pdf += att[c];
    }
    pdf *= (R(1) / R(3));
    return att;
}
// EvaluatePhase, Medium.h:83-94
template <class R> inline V3<R> evaluate_phase(const Med<R>& m, const V3<R>& V, const V3<R>& L, R& pdf) {
    pdf = R(0);
    if (m.phase == RT_PHASE_ISOTROPIC) {
        pdf = R(0.25f) * K<R>::INV_PI;
        return V3<R>(R(0.25f) * K<R>::INV_PI);
    }
    if (m.phase == RT_PHASE_HENYEY_GREENSTEIN) {
        V3<R> a = hg_terms(m, dot(L, V), pdf);
        if (pdf <= R(0)) return V3<R>(R(0));
        return a;
    }
    return V3<R>(R(0));
}
// SamplePhase, Medium.h:96-108 (Medium.h:14-22, 44-79)
template <class R> inline V3<R> sample_phase(const Med<R>& m, Rng& rng, const V3<R>& V, V3<R>& L, R& pdf) {
    pdf = R(0);
    if (m.phase == RT_PHASE_ISOTROPIC) {
        R u0 = rng.next(), u1 = rng.next();
        L = uniform_sample_sphere(u0, u1);
        pdf = R(0.25f) * K<R>::INV_PI;
        return V3<R>(R(0.25f) * K<R>::INV_PI);
    }
    if (m.phase == RT_PHASE_HENYEY_GREENSTEIN) {
        int ch = std::min(static_cast<int>(rng.next() * 3.0f), 2);
        R g = m.g[ch];
        R ct;
        if (std::fabs(g) < K<R>::EPS) {
            ct = R(1) - R(2) * R(rng.next());
        } else {
            R st = (R(1) - g * g) / (R(1) - g + R(2) * g * R(rng.next()));
            ct = (R(1) + g * g - st * st) / (R(2) * g);
        }
        V3<R> att = hg_terms(m, ct, pdf);
        if (pdf <= R(0)) return V3<R>(R(0));
        R sn = std::sqrt(dmax(R(0), R(1) - ct * ct));
        R phi = K<R>::TWO_PI * R(rng.next());
        V3<R> lL = normalize(V3<R>(sn * std::cos(phi), sn * std::sin(phi), ct));
        L = to_world(lL, V);
        return att;
    }
    return V3<R>(R(0));
}
template <class R> inline R homog_weight(const V3<R>& st, const V3<R>& alb) {
    R w = R(0);
    for (int c = 0; c < 3; ++c)
        if (alb[c] > w && st[c] != R(0)) w = alb[c];
    if (w > R(0)) w = dmax(w, R(0.5f));
    return w;
}
// EvaluateMediumDistance, Medium.h:112-158, 222-231
template <class R> inline V3<R> eval_medium_distance(const Med<R>& m, bool scattered, R dist, R& tp) {
    tp = R(0);
    if (m.type != RT_MEDIUM_HOMOGENEOUS) return V3<R>(R(0));
    V3<R> ss = m.sigma_s * m.scale, sa = m.sigma_a * m.scale, st = sa + ss;
    V3<R> alb = ss / st;
    R w = homog_weight(st, alb);
    V3<R> att;
    R pdf = R(0);
    bool valid = false;
    for (int c = 0; c < 3; ++c) {
        att[c] = std::exp(-st[c] * dist);
        if (att[c] > R(0)) valid = true;
    }
    if (scattered) {
        for (int c = 0; c < 3; ++c) pdf += st[c] * att[c];
        pdf *= w * (R(1) / R(3));
        att *= ss;
    } else {
        for (int c = 0; c < 3; ++c) pdf += att[c];
        pdf = w * (R(1) / R(3)) * pdf + (R(1) - w);
    }
    tp = pdf;
    if (!valid) att = V3<R>(R(0));
    return att;
}
// SampleMediumDistance, Medium.h:160-218, 233-244
template <class R> inline bool sample_medium_distance(const Med<R>& m, R maxd, R& dist, R& tp, V3<R>& tr, Rng& rng) {
    tp = R(0);
    tr = V3<R>(R(0));
    if (m.type != RT_MEDIUM_HOMOGENEOUS) return false;
    V3<R> ss = m.sigma_s * m.scale, sa = m.sigma_a * m.scale, st = sa + ss;
    V3<R> alb = ss / st;
    R w = homog_weight(st, alb);
    bool scattered = false;
    R x1 = rng.next();
    if (x1 < w) {
        x1 /= w;
        int ch = std::min(static_cast<int>(rng.next() * 3.0f), 2);
        dist = -std::log(R(1) - x1) / st[ch];
        if (dist < maxd) {
            tp = R(0);
            for (int c = 0; c < 3; ++c) tp += st[c] * std::exp(-st[c] * dist);
            tp *= w * (R(1) / R(3));
            scattered = true;
        }
    }
    if (!scattered) {
        dist = maxd;
        tp = R(0);
        for (int c = 0; c < 3; ++c) tp += std::exp(-st[c] * dist);
        tp = w * (R(1) / R(3)) * tp + (R(1) - w);
    }
    bool valid = false;
    for (int c = 0; c < 3; ++c) {
        tr[c] = std::exp(-st[c] * dist);
        if (tr[c] > R(0)) valid = true;
    }
    if (scattered) tr *= ss;
    if (!valid) tr = V3<R>(R(0));
    return scattered;
}

// ---------------------------------------------------------------- grid media
// Not in the reference (homogeneous only).  Gray extinction
// sigma_t = scale * max_c(sigma_a + sigma_s) times a trilinear density, per
// channel albedo; delta tracking for distances and ratio tracking for
// next-event transmittance against a majorant grid walked by a 3D DDA, with at
// most 4096 tentative collisions per call.  Mirrors the renderer's
// rt_media.cuh in arithmetic and in the order random numbers are drawn.
template <class R> struct Grid {
    V3<R> bmin, bmax, albedo;
    int res[3];
    int mres;
    R sigma_t;
    const float* density;
    const float* majorant;
};
inline void grid_majorants(const float* dens, const int res[3], int mres, std::vector<float>& out) {
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
                        for (int x = lo[0]; x <= hi[0]; x++) m = std::max(m, dens[(size_t(z) * res[1] + y) * res[0] + x]);
                out[(size_t(cz) * mres + cy) * mres + cx] = m;
            }
}
template <class R> inline R grid_density(const Grid<R>& g, const V3<R>& p) {
    V3<R> ext = g.bmax - g.bmin;
    R gx = (p.x - g.bmin.x) / ext.x * R(g.res[0]) - R(0.5f);
    R gy = (p.y - g.bmin.y) / ext.y * R(g.res[1]) - R(0.5f);
    R gz = (p.z - g.bmin.z) / ext.z * R(g.res[2]) - R(0.5f);
    if (!(gx > R(-0.5f) && gy > R(-0.5f) && gz > R(-0.5f) && gx < R(g.res[0]) - R(0.5f) && gy < R(g.res[1]) - R(0.5f) &&
          gz < R(g.res[2]) - R(0.5f)))
        return R(0);
    gx = dmin(dmax(gx, R(0)), R(g.res[0] - 1));
    gy = dmin(dmax(gy, R(0)), R(g.res[1] - 1));
    gz = dmin(dmax(gz, R(0)), R(g.res[2] - 1));
    int x0 = std::min(int(gx), g.res[0] - 1), y0 = std::min(int(gy), g.res[1] - 1), z0 = std::min(int(gz), g.res[2] - 1);
    int x1 = std::min(x0 + 1, g.res[0] - 1), y1 = std::min(y0 + 1, g.res[1] - 1), z1 = std::min(z0 + 1, g.res[2] - 1);
    R fx = gx - R(x0), fy = gy - R(y0), fz = gz - R(z0);
    auto at = [&](int x, int y, int z) { return R(g.density[(size_t(z) * g.res[1] + y) * g.res[0] + x]); };
    R c00 = mixr(at(x0, y0, z0), at(x1, y0, z0), fx), c10 = mixr(at(x0, y1, z0), at(x1, y1, z0), fx);
    R c01 = mixr(at(x0, y0, z1), at(x1, y0, z1), fx), c11 = mixr(at(x0, y1, z1), at(x1, y1, z1), fx);
    return mixr(mixr(c00, c10, fy), mixr(c01, c11, fy), fz);
}
template <class R> inline bool grid_clip(const Grid<R>& g, const V3<R>& o, const V3<R>& d, R tmax, R& t0, R& t1) {
    t0 = R(0);
    t1 = tmax;
    for (int a = 0; a < 3; a++) {
        R inv = R(1) / d[a];
        R ta = (g.bmin[a] - o[a]) * inv, tb = (g.bmax[a] - o[a]) * inv;
        if (ta > tb) std::swap(ta, tb);
        t0 = dmax(t0, ta);
        t1 = dmin(t1, tb);
    }
    return t0 < t1;
}
template <class R, class F> inline void majorant_walk(const Grid<R>& g, const V3<R>& o, const V3<R>& d, R t0, R t1, F&& f) {
    const int M = g.mres;
    V3<R> ext = g.bmax - g.bmin;
    V3<R> p = o + t0 * d;
    int c[3], step[3];
    R tnext[3], tdelta[3];
    for (int a = 0; a < 3; a++) {
        R cell = ext[a] / R(M);
        R rel = (p[a] - g.bmin[a]) / cell;
        int ci = std::min(std::max(int(std::floor(rel)), 0), M - 1);
        c[a] = ci;
        if (d[a] > R(0)) {
            step[a] = 1;
            tnext[a] = t0 + ((g.bmin[a] + R(ci + 1) * cell) - p[a]) / d[a];
            tdelta[a] = cell / d[a];
        } else if (d[a] < R(0)) {
            step[a] = -1;
            tnext[a] = t0 + ((g.bmin[a] + R(ci) * cell) - p[a]) / d[a];
            tdelta[a] = -cell / d[a];
        } else {
            step[a] = 0;
            tnext[a] = R(FLT_MAX);
            tdelta[a] = R(FLT_MAX);
        }
    }
    R t = t0;
    for (int it = 0; it < 3 * M + 3 && t < t1; it++) {
        int a = tnext[0] < tnext[1] ? (tnext[0] < tnext[2] ? 0 : 2) : (tnext[1] < tnext[2] ? 1 : 2);
        R te = dmin(tnext[a], t1);
        R mj = R(g.majorant[(size_t(c[2]) * M + c[1]) * M + c[0]]);
        if (!f(t, te, mj)) return;
        t = te;
        c[a] += step[a];
        if (c[a] < 0 || c[a] >= M) return;
        tnext[a] += tdelta[a];
    }
}
template <class R> inline bool grid_sample_distance(const Grid<R>& g, const V3<R>& o, const V3<R>& d, R maxd, Rng& rng,
                                                    R& dist, V3<R>& weight) {
    weight = V3<R>(R(1));
    R t0, t1;
    if (!grid_clip(g, o, d, maxd, t0, t1) || g.sigma_t <= R(0)) return false;
    bool scattered = false;
    int steps = 0;
    majorant_walk(g, o, d, t0, t1, [&](R ca, R cb, R mj) {
        R smax = mj * g.sigma_t;
        if (smax <= R(0)) return true;
        R t = ca;
        while (true) {
            if (++steps > 4096) {
                weight = V3<R>(R(0));
                return false;
            }
            t -= std::log(R(1) - R(rng.next())) / smax;
            if (t >= cb) return true;
            R sv = grid_density(g, o + t * d) * g.sigma_t;
            if (R(rng.next()) * smax < sv) {
                scattered = true;
                dist = t;
                return false;
            }
        }
    });
    if (scattered) weight = g.albedo;
    return scattered;
}
template <class R> inline R grid_transmittance(const Grid<R>& g, const V3<R>& o, const V3<R>& d, R maxd, Rng& rng) {
    R t0, t1;
    if (!grid_clip(g, o, d, maxd, t0, t1) || g.sigma_t <= R(0)) return R(1);
    R T = R(1);
    int steps = 0;
    majorant_walk(g, o, d, t0, t1, [&](R ca, R cb, R mj) {
        R smax = mj * g.sigma_t;
        if (smax <= R(0)) return true;
        R t = ca;
        while (true) {
            if (++steps > 4096) {
                T = R(0);
                return false;
            }
            t -= std::log(R(1) - R(rng.next())) / smax;
            if (t >= cb) return true;
            R sv = grid_density(g, o + t * d) * g.sigma_t;
            T *= R(1) - sv / smax;
            if (T <= R(0)) return false;
        }
    });
    return T;
}

// ---------------------------------------------------------------- filter
// core/cuda/Filter.h:5-56
template <class R> inline void filter_jitter(int type, R s0, R s1, R& jx, R& jy) {
    if (type == RT_FILTER_BOX) {
        jx = s0 - R(0.5f);
        jy = s1 - R(0.5f);
    } else if (type == RT_FILTER_TENT) {
        R x = s0 * R(2), y = s1 * R(2);
        x = x < R(1) ? std::sqrt(x) - R(1) : R(1) - std::sqrt(R(2) - x);
        y = y < R(1) ? std::sqrt(y) - R(1) : R(1) - std::sqrt(R(2) - y);
        jx = R(0.5f) + x;
        jy = R(0.5f) + y;
    } else if (type == RT_FILTER_TRIANGLE) {
        R u1 = s0, u2 = s1;
        if (u2 > u1) {
            u1 *= R(0.5f);
            u2 -= u1;
        } else {
            u2 *= R(0.5f);
            u1 -= u2;
        }
        jx = R(0.5f) + u1;
        jy = R(0.5f) + u2;
    } else if (type == RT_FILTER_GAUSSIAN) {
        R r1 = dmax(R(FLT_MIN), s0);
        R r = std::sqrt(R(-2) * std::log(r1));
        R th = K<R>::TWO_PI * s1;
        jx = R(0.5f) + R(0.375f) * (r * std::cos(th));
        jy = R(0.5f) + R(0.375f) * (r * std::sin(th));
    } else {
        jx = s0;
        jy = s1;
    }
}

// ---------------------------------------------------------------- environment
// tex2D<float4> with normalized coordinates, wrap addressing and linear
// filtering (core/src/Scene.cpp:340-349), evaluated with float weights.
template <class R> inline void tex_bilinear(const float* img, int w, int h, R u, R v, R out[4]) {
    u = u - std::floor(u);
    v = v - std::floor(v);
    R x = u * R(w) - R(0.5f), y = v * R(h) - R(0.5f);
    R fx = std::floor(x), fy = std::floor(y);
    R a = x - fx, b = y - fy;
    int x0 = int(fx), y0 = int(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = ((x0 % w) + w) % w;
    x1 = ((x1 % w) + w) % w;
    y0 = ((y0 % h) + h) % h;
    y1 = ((y1 % h) + h) % h;
    for (int c = 0; c < 4; ++c) {
        R t00 = R(img[(size_t(y0) * w + x0) * 4 + c]), t10 = R(img[(size_t(y0) * w + x1) * 4 + c]);
        R t01 = R(img[(size_t(y1) * w + x0) * 4 + c]), t11 = R(img[(size_t(y1) * w + x1) * 4 + c]);
        out[c] = mixr(mixr(t00, t10, a), mixr(t01, t11, a), b);
    }
}
// tex2D<float4> of an RGBA8 material texture (core/src/Renderer.cpp:100-143:
// uchar4 texels read as normalized floats, normalized coordinates, wrap
// addressing, linear filtering), evaluated with float weights on texels
// converted as byte * (1/255).
template <class R> inline void tex_rgba8(const uint32_t* img, int w, int h, R u, R v, R out[4]) {
    u = u - std::floor(u);
    v = v - std::floor(v);
    R x = u * R(w) - R(0.5f), y = v * R(h) - R(0.5f);
    R fx = std::floor(x), fy = std::floor(y);
    R a = x - fx, b = y - fy;
    int x0 = int(fx), y0 = int(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = ((x0 % w) + w) % w;
    x1 = ((x1 % w) + w) % w;
    y0 = ((y0 % h) + h) % h;
    y1 = ((y1 % h) + h) % h;
    const uint32_t p00 = img[size_t(y0) * w + x0], p10 = img[size_t(y0) * w + x1];
    const uint32_t p01 = img[size_t(y1) * w + x0], p11 = img[size_t(y1) * w + x1];
    for (int c = 0; c < 4; ++c) {
        auto texel = [c](uint32_t px) { return R(float((px >> (8 * c)) & 0xFFu) * (1.0f / 255.0f)); };
        out[c] = mixr(mixr(texel(p00), texel(p10), a), mixr(texel(p01), texel(p11), a), b);
    }
}

// NormalFromTangentToWorld, core/cuda/Utils.h:85-94.
template <class R> inline V3<R> normal_from_tangent(const V3<R>& n, V3<R> t) {
    t = normalize(t * R(2) - V3<R>(R(1)));
    V3<R> up = std::abs(n.z) < R(0.9f) ? V3<R>(R(0), R(0), R(1)) : V3<R>(R(1), R(0), R(0));
    V3<R> tx = normalize(cross(up, n));
    V3<R> ty = normalize(cross(n, tx));
    return normalize(tx * t.x + ty * t.y + n * t.z);
}

// HdrTexture::CalculateHdrCache, core/src/Scene.cpp:217-313 (float
// arithmetic in the same order; the marginal index is clamped to width-1
// where the reference would read past the table).
inline void env_cache(const float* hdr, int width, int height, float* cache) {
    const int comp = 4;
    float lum_sum = 0.0f;
    std::vector<float> pdf(size_t(width) * height);
    for (int i = 0; i < height; i++)
        for (int j = 0; j < width; j++) {
            const float* p = hdr + comp * (size_t(i) * width + j);
            float lum = 0.299f * p[0] + 0.587f * p[1] + 0.114f * p[2];
            pdf[size_t(i) * width + j] = lum;
            lum_sum += lum;
        }
    for (size_t q = 0; q < pdf.size(); q++) pdf[q] /= lum_sum;
    std::vector<float> px(width, 0.0f);
    for (int j = 0; j < width; j++)
        for (int i = 0; i < height; i++) px[j] += pdf[size_t(i) * width + j];
    std::vector<float> cx = px;
    for (int i = 1; i < width; i++) cx[i] += cx[i - 1];
    std::vector<float> cy(size_t(width) * height);  // [j][i]
    for (int j = 0; j < width; j++) {
        float acc = 0.0f;
        for (int i = 0; i < height; i++) {
            float val = pdf[size_t(i) * width + j] / px[j];
            acc = (i == 0) ? val : acc + val;
            cy[size_t(j) * height + i] = acc;
        }
    }
    for (int j = 0; j < width; j++)
        for (int i = 0; i < height; i++) {
            float xi1 = float(i) / height, xi2 = float(j) / width;
            int x = int(std::lower_bound(cx.begin(), cx.end(), xi1) - cx.begin());
            if (x > width - 1) x = width - 1;
            const float* col = cy.data() + size_t(x) * height;
            int y = int(std::lower_bound(col, col + height, xi2) - col);
            float* c = cache + comp * (size_t(i) * width + j);
            c[0] = float(x) / width;
            c[1] = float(y) / height;
            c[2] = pdf[size_t(i) * width + j];
            c[3] = 0.0f;
        }
}

// ---------------------------------------------------------------- geometry
// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013), evaluated in
// R; returns t and the barycentrics (b1 weights vertex 1, b2 vertex 2, as
// optixGetTriangleBarycentrics).  `margin` reports how close the hit is to an
// edge relative to the magnitude of the edge-function terms.
template <class R> struct RayPre {
    int kx, ky, kz;
    R Sx, Sy, Sz;
    V3<R> o;
    void init(const V3<R>& org, const V3<R>& d) {
        o = org;
        R ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
        kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
        kx = (kz + 1) % 3;
        ky = (kx + 1) % 3;
        if (d[kz] < R(0)) std::swap(kx, ky);
        Sx = d[kx] / d[kz];
        Sy = d[ky] / d[kz];
        Sz = R(1) / d[kz];
    }
};
template <class R> inline bool tri_hit(const RayPre<R>& rp, const V3<R>& p0, const V3<R>& p1, const V3<R>& p2, R tmin, R tmax,
                                       R& t, R& b1, R& b2, R* margin = nullptr) {
    V3<R> A = p0 - rp.o, B = p1 - rp.o, C = p2 - rp.o;
    R Ax = A[rp.kx] - rp.Sx * A[rp.kz], Ay = A[rp.ky] - rp.Sy * A[rp.kz];
    R Bx = B[rp.kx] - rp.Sx * B[rp.kz], By = B[rp.ky] - rp.Sy * B[rp.kz];
    R Cx = C[rp.kx] - rp.Sx * C[rp.kz], Cy = C[rp.ky] - rp.Sy * C[rp.kz];
    R U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if ((U < R(0) || V < R(0) || W < R(0)) && (U > R(0) || V > R(0) || W > R(0))) return false;
    R det = U + V + W;
    if (det == R(0)) return false;
    R Az = rp.Sz * A[rp.kz], Bz = rp.Sz * B[rp.kz], Cz = rp.Sz * C[rp.kz];
    R T = U * Az + V * Bz + W * Cz;
    R inv = R(1) / det;
    t = T * inv;
    if (!(t > tmin && t < tmax)) return false;
    b1 = V * inv;
    b2 = W * inv;
    if (margin) {
        R mu = std::fabs(U) / (std::fabs(Cx * By) + std::fabs(Cy * Bx) + R(1e-300));
        R mv = std::fabs(V) / (std::fabs(Ax * Cy) + std::fabs(Ay * Cx) + R(1e-300));
        R mw = std::fabs(W) / (std::fabs(Bx * Ay) + std::fabs(By * Ax) + R(1e-300));
        *margin = std::min(mu, std::min(mv, mw));
    }
    return true;
}

// A plain binary BVH over the triangles (median split on the longest
// centroid axis) used only to make the oracle's ray queries fast.
struct Bvh2 {
    struct Node {
        double lo[3], hi[3];
        int left, right, first, count;
    };
    std::vector<Node> nodes;
    std::vector<int> prims;
    void build(const float* tv, int64_t ntri) {
        prims.resize(size_t(ntri));
        std::vector<double> cen(size_t(ntri) * 3), blo(size_t(ntri) * 3), bhi(size_t(ntri) * 3);
        for (int64_t i = 0; i < ntri; i++) {
            prims[size_t(i)] = int(i);
            for (int a = 0; a < 3; a++) {
                double x0 = tv[i * 9 + a], x1 = tv[i * 9 + 3 + a], x2 = tv[i * 9 + 6 + a];
                blo[i * 3 + a] = std::min(x0, std::min(x1, x2));
                bhi[i * 3 + a] = std::max(x0, std::max(x1, x2));
                cen[i * 3 + a] = 0.5 * (blo[i * 3 + a] + bhi[i * 3 + a]);
            }
        }
        nodes.clear();
        nodes.reserve(size_t(2 * ntri + 1));
        struct Item { int node, first, count; };
        std::vector<Item> st;
        nodes.push_back(Node());
        st.push_back({0, 0, int(ntri)});
        while (!st.empty()) {
            Item it = st.back();
            st.pop_back();
            Node nd;
            for (int a = 0; a < 3; a++) {
                nd.lo[a] = 1e300;
                nd.hi[a] = -1e300;
            }
            double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
            for (int q = it.first; q < it.first + it.count; q++) {
                int p = prims[size_t(q)];
                for (int a = 0; a < 3; a++) {
                    nd.lo[a] = std::min(nd.lo[a], blo[size_t(p) * 3 + a]);
                    nd.hi[a] = std::max(nd.hi[a], bhi[size_t(p) * 3 + a]);
                    clo[a] = std::min(clo[a], cen[size_t(p) * 3 + a]);
                    chi[a] = std::max(chi[a], cen[size_t(p) * 3 + a]);
                }
            }
            nd.first = it.first;
            nd.count = it.count;
            nd.left = nd.right = -1;
            if (it.count > 4) {
                int ax = 0;
                for (int a = 1; a < 3; a++)
                    if (chi[a] - clo[a] > chi[ax] - clo[ax]) ax = a;
                int mid = it.first + it.count / 2;
                std::nth_element(prims.begin() + it.first, prims.begin() + mid, prims.begin() + it.first + it.count,
                                 [&](int a, int b) { return cen[size_t(a) * 3 + ax] < cen[size_t(b) * 3 + ax]; });
                nd.left = int(nodes.size());
                nodes.push_back(Node());
                nd.right = int(nodes.size());
                nodes.push_back(Node());
                st.push_back({nd.left, it.first, mid - it.first});
                st.push_back({nd.right, mid, it.first + it.count - mid});
                nd.count = 0;
            }
            nodes[size_t(it.node)] = nd;
        }
    }
    // Slab test in double with a small relative widening.
    static bool box_hit(const Node& n, const double o[3], const double id[3], double tmin, double tmax) {
        double t0 = tmin, t1 = tmax;
        for (int a = 0; a < 3; a++) {
            double lo = n.lo[a] - 1e-9 * (1.0 + std::fabs(n.lo[a]));
            double hi = n.hi[a] + 1e-9 * (1.0 + std::fabs(n.hi[a]));
            double ta = (lo - o[a]) * id[a], tb = (hi - o[a]) * id[a];
            if (std::isnan(ta)) ta = -1e300;
            if (std::isnan(tb)) tb = 1e300;
            if (ta > tb) std::swap(ta, tb);
            t0 = std::max(t0, ta);
            t1 = std::min(t1, tb);
            if (t0 > t1) return false;
        }
        return true;
    }
};

// Closest-hit query in R with tie diagnostics (the two nearest distinct hits).
template <class R> struct HitInfo {
    R t, b1, b2, margin, t2;
    int prim, prim2;
};
template <class R> inline void closest_hit(const Bvh2& bvh, const float* tv, const V3<R>& o, const V3<R>& d, R tmin, R tmax,
                                           HitInfo<R>& h) {
    RayPre<R> rp;
    rp.init(o, d);
    h.t = tmax;
    h.t2 = tmax;
    h.prim = -1;
    h.prim2 = -1;
    h.margin = R(1);
    h.b1 = h.b2 = R(0);
    double od[3] = {double(o.x), double(o.y), double(o.z)};
    double id[3];
    for (int a = 0; a < 3; a++) id[a] = 1.0 / double(d[a]);
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Bvh2::Node& n = bvh.nodes[size_t(stack[--sp])];
        if (!Bvh2::box_hit(n, od, id, double(tmin) * 0.999, double(h.t2) * 1.001 + 1e-12)) continue;
        if (n.left < 0) {
            for (int q = n.first; q < n.first + n.count; q++) {
                int p = bvh.prims[size_t(q)];
                const float* f = tv + size_t(p) * 9;
                R t, b1, b2, mg;
                if (tri_hit(rp, from3<R>(f), from3<R>(f + 3), from3<R>(f + 6), tmin, tmax, t, b1, b2, &mg)) {
                    if (t < h.t) {
                        h.t2 = h.t;
                        h.prim2 = h.prim;
                        h.t = t;
                        h.prim = p;
                        h.b1 = b1;
                        h.b2 = b2;
                        h.margin = mg;
                    } else if (t < h.t2) {
                        h.t2 = t;
                        h.prim2 = p;
                    }
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
}
template <class R> inline bool any_hit(const Bvh2& bvh, const float* tv, const V3<R>& o, const V3<R>& d, R tmin, R tmax) {
    RayPre<R> rp;
    rp.init(o, d);
    double od[3] = {double(o.x), double(o.y), double(o.z)};
    double id[3];
    for (int a = 0; a < 3; a++) id[a] = 1.0 / double(d[a]);
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Bvh2::Node& n = bvh.nodes[size_t(stack[--sp])];
        if (!Bvh2::box_hit(n, od, id, double(tmin) * 0.999, double(tmax) * 1.001 + 1e-12)) continue;
        if (n.left < 0) {
            for (int q = n.first; q < n.first + n.count; q++) {
                const float* f = tv + size_t(bvh.prims[size_t(q)]) * 9;
                R t, b1, b2;
                if (tri_hit(rp, from3<R>(f), from3<R>(f + 3), from3<R>(f + 6), tmin, tmax, t, b1, b2)) return true;
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

}  // namespace orc
