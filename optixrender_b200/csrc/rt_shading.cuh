// rt_shading.cuh - device shading: microfacet BSDFs, analytic lights, media,
// environment lookup and pixel filters.  The arithmetic follows the reference
// renderer's shading headers (core/cuda/{Sampling,Microfacet,Material,Light,
// Medium,Environment,Filter,Utils}.h) term for term, in FP32, so that a CPU
// restatement fed the same random numbers traces the same paths.  Random
// numbers are always drawn left to right.
#pragma once

#include "rt_device.cuh"

namespace rtd {

// ------------------------------------------------------------ sampling
RT_D float power_heuristic(float a, float b) {  // Sampling.h:5-10 (beta = 2)
    float p = a * a, q = b * b;
    return p / (p + q);
}
RT_D v3 plane_to_sphere(float u, float v) {  // Sampling.h:12-24
    float phi = kTwoPi * (u - 0.5f);
    float theta = kPi * (v - 0.5f);
    float st, ct, sp, cp;
    sincosf(theta, &st, &ct);
    sincosf(phi, &sp, &cp);
    return normalize(v3(ct * cp, st, ct * sp));
}
RT_D void sphere_to_plane(v3 d, float& u, float& v) {  // Sampling.h:26-33
    u = atan2f(d.z, d.x) / kTwoPi + 0.5f;
    v = asinf(d.y) / kPi + 0.5f;
}
RT_D v3 uniform_sample_cone(float s0, float s1, float cos_angle) {  // Sampling.h:36-48
    float phi = kTwoPi * s0;
    float ct = mixf(cos_angle, 1.0f, s1);
    float st = sqrtf(1.0f - ct * ct);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return normalize(v3(st * cp, st * sp, ct));
}
RT_D float uniform_pdf_cone(float cos_angle) { return 1.0f / (kTwoPi * (1.0f - cos_angle)); }
RT_D v3 uniform_sample_sphere(float s0, float s1) {  // Sampling.h:76-88
    float phi = kTwoPi * s0;
    float ct = 1.0f - 2.0f * s1;
    float st = sqrtf(1.0f - ct * ct);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return normalize(v3(st * cp, st * sp, ct));
}

template <class R>
RT_D vec3t<R> cosine_sample_hemisphere(R s0, R s1) {  // Sampling.h:56-69
    R r = sqrt_r(s0);
    R sp, cp;
    sincos_2pi_r(s1, &sp, &cp);
    vec3t<R> p(r * cp, r * sp, 0.0f);
    p.z = sqrt_r(fmax_r(0.0f, 1.0f - p.x * p.x - p.y * p.y));
    return normalize(p);
}
template <class R>
RT_D R cosine_pdf(R ndotl) { return ndotl * Kc<R>::inv_pi; }
// ------------------------------------------------------------ frames
template <class R>
RT_D vec3t<R> reflect(vec3t<R> v, vec3t<R> n) { return normalize(v - 2.0f * dot(v, n) * n); }  // Utils.h:28-30
template <class R>
RT_D vec3t<R> refract(vec3t<R> v, vec3t<R> n, sc_t<R> eta) {                                       // Utils.h:32-38
    R ct = fmin_r(dot(-v, n), 1.0f);
    vec3t<R> perp = eta * (v + ct * n);
    vec3t<R> par = -sqrt_r(fabs_r(1.0f - dot(perp, perp))) * n;
    return normalize(perp + par);
}
template <class R>
RT_D void frame_axes(vec3t<R> up, vec3t<R>& B, vec3t<R>& C) {  // Utils.h:99-109
    if (fabs_r(up.x) > fabs_r(up.y)) {
        R inv = 1.0f / sqrt_r(up.x * up.x + up.z * up.z);
        C = vec3t<R>(up.z * inv, 0.0f, -up.x * inv);
    } else {
        R inv = 1.0f / sqrt_r(up.y * up.y + up.z * up.z);
        C = vec3t<R>(0.0f, up.z * inv, -up.y * inv);
    }
    B = cross(C, up);
}
template <class R>
RT_D vec3t<R> to_local(vec3t<R> d, vec3t<R> up) {
    vec3t<R> B, C;
    frame_axes(up, B, C);
    return vec3t<R>(dot(d, B), dot(d, C), dot(d, up));
}
template <class R>
RT_D vec3t<R> to_world(vec3t<R> d, vec3t<R> up) {  // Utils.h:117-129
    vec3t<R> B, C;
    frame_axes(up, B, C);
    return normalize(d.x * B + d.y * C + d.z * up);
}

// ------------------------------------------------------------ microfacet
template <class R>
RT_D vec3t<R> fresnel_conductor(vec3t<R> V, vec3t<R> H, vec3t<R> er, vec3t<R> ei) {  // Microfacet.h:22-46
    R c = dot(V, H), c2 = c * c, s2 = 1.0f - c2, s4 = s2 * s2;
    vec3t<R> t1 = er * er - ei * ei - s2;
    vec3t<R> a2 = t1 * t1 + 4.0f * ei * ei * er * er;
    a2 = vec3t<R>(sqrt_r(fmax_r(0.0f, a2.x)), sqrt_r(fmax_r(0.0f, a2.y)), sqrt_r(fmax_r(0.0f, a2.z)));
    vec3t<R> a = 0.5f * (a2 + t1);
    a = vec3t<R>(sqrt_r(fmax_r(0.0f, a.x)), sqrt_r(fmax_r(0.0f, a.y)), sqrt_r(fmax_r(0.0f, a.z)));
    vec3t<R> term1 = a2 + s2, term2 = 2.0f * c * a, term3 = a2 * c2 + s4, term4 = term2 * s2;
    vec3t<R> rs = (term1 - term2) / (term1 + term2);
    vec3t<R> rp = rs * (term3 - term4) / (term3 + term4);
    return 0.5f * (rs + rp);
}
template <class R>
RT_D vec3t<R> average_fresnel_conductor(vec3t<R> eta, vec3t<R> k) {  // Microfacet.h:48-70
    R rr[3], ee[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        R e = eta[i], kk = k[i];
        R r = (sqr(e - 1.0f) + sqr(kk)) / (sqr(e + 1.0f) + sqr(kk));
        R t1 = 1.0f + sqrt_r(r), t2 = 1.0f - sqrt_r(r), t3 = (1.0f - r) / (1.0f + r);
        rr[i] = r;
        ee[i] = (t1 - e * t2) / (t1 - t3 * t2);
    }
    vec3t<R> refl(rr[0], rr[1], rr[2]), edge(ee[0], ee[1], ee[2]);
    return vec3t<R>(0.087237f) + 0.0230685f * edge - 0.0864902f * edge * edge + 0.0774594f * edge * edge * edge +
           0.782654f * refl - 0.136432f * refl * refl + 0.278708f * refl * refl * refl + 0.19744f * edge * refl +
           0.0360605f * edge * edge * refl - 0.2586f * edge * refl * refl;
}
template <class R>
RT_D R fresnel_dielectric(vec3t<R> V, vec3t<R> H, sc_t<R> eta_inv) {  // Microfacet.h:72-85
    R ci = fabs_r(dot(V, H));
    R ct2 = 1.0f - sqr(eta_inv) * (1.0f - sqr(ci));
    if (ct2 <= 0.0f) return 1.0f;
    R ct = sqrt_r(ct2);
    R rs = (eta_inv * ci - ct) / (eta_inv * ci + ct);
    R rp = (ci - eta_inv * ct) / (ci + eta_inv * ct);
    return (rs * rs + rp * rp) / 2.0f;
}
template <class R>
RT_D R average_fresnel_dielectric(R eta) {  // Microfacet.h:87-113
    if (eta < 1.0f) return -1.4399f * (eta * eta) + 0.7099f * eta + 0.6681f + 0.0636f / eta;
    R i1 = 1.0f / eta, i2 = i1 * i1, i3 = i2 * i1, i4 = i3 * i1, i5 = i4 * i1;
    return 0.919317f - 3.4793f * i1 + 6.75335f * i2 - 7.80989f * i3 + 4.98554f * i4 - 1.36881f * i5;
}
template <class R>
RT_D R smith_g1(vec3t<R> V, vec3t<R> H, vec3t<R> N, sc_t<R> au, sc_t<R> av) {  // Microfacet.h:117-142
    R cvn = dot(V, N);
    if (cvn * dot(V, H) <= 0.0f) return 0.0f;
    if (fabs_r(cvn - 1.0f) < R(kEps)) return 1.0f;
    if (au == av) {
        R c2 = sqr(cvn), t2 = (1.0f - c2) / c2;
        return 2.0f / (1.0f + sqrt_r(1.0f + au * au * t2));
    }
    vec3t<R> d = to_local(V, N);
    R t = (sqr(au * d.x) + sqr(av * d.y)) / sqr(d.z);
    return 2.0f / (1.0f + sqrt_r(1.0f + t));
}
template <class R>
RT_D R ggx_d(vec3t<R> H, vec3t<R> N, sc_t<R> au, sc_t<R> av) {  // Microfacet.h:144-160
    R c = dot(H, N);
    if (c <= 0.0f) return 0.0f;
    R c2 = sqr(c), t2 = (1.0f - c2) / c2, a2 = au * av;
    if (au == av) return a2 / (Kc<R>::pi * (c * c) * sqr(a2 + t2));
    vec3t<R> d = to_local(H, N);
    return 1.0f / (Kc<R>::pi * a2 * sqr(sqr(d.x / au) + sqr(d.y / av) + sqr(d.z)));
}
template <class R>
RT_D R ggx_dv(vec3t<R> V, vec3t<R> H, vec3t<R> N, sc_t<R> au, sc_t<R> av) {  // Microfacet.h:162-164
    return smith_g1(V, H, N, au, av) * dot(V, H) * ggx_d(H, N, au, av) / dot(N, V);
}
template <class R>
RT_D vec3t<R> sample_vndf(vec3t<R> N, vec3t<R> Ve, sc_t<R> au, sc_t<R> av, sc_t<R> s0, sc_t<R> s1) {  // Microfacet.h:188-214
    vec3t<R> V = to_local(Ve, N);
    vec3t<R> Vh = normalize(vec3t<R>(au * V.x, av * V.y, V.z));
    R len2 = sqr(Vh.x) + sqr(Vh.y);
    vec3t<R> T1 = len2 > 0.0f ? vec3t<R>(-Vh.y, Vh.x, 0.0f) * sqrt_r(1.0f / len2) : vec3t<R>(1.0f, 0.0f, 0.0f);
    vec3t<R> T2 = cross(Vh, T1);
    R r = sqrt_r(s0);
    R sp, cp;
    sincos_2pi_r(R(s1), &sp, &cp);
    R t1 = r * cp, t2 = r * sp;
    R s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrt_r(1.0f - sqr(t1)) + s * t2;
    vec3t<R> Nh = t1 * T1 + t2 * T2 + sqrt_r(fmax_r(0.0f, 1.0f - sqr(t1) - sqr(t2))) * Vh;
    return normalize(vec3t<R>(au * Nh.x, av * Nh.y, fmax_r(0.0f, Nh.z)));
}
// Kulla-Conty tables, Microfacet.h:293-346
template <class R>
RT_D R lut_bsdf_avg(R cos_theta, R rough, const float* t) {
    const int kN = 64;
    R o1 = sqr(rough) * kN, o2 = cos_theta * kN;
    int i1 = int(o1), i2 = int(o2);
    if (i1 >= kN - 1) {
        if (i2 >= kN - 1) return __ldg(t + (kN - 1) * kN + kN - 1);
        return mix_r<R>(__ldg(t + (kN - 1) * kN + i2), __ldg(t + (kN - 1) * kN + i2 + 1), o2 - i2);
    }
    if (i2 >= kN - 1) return mix_r<R>(__ldg(t + i1 * kN + kN - 1), __ldg(t + (i1 + 1) * kN + kN - 1), o1 - i1);
    return mix_r<R>(mix_r<R>(__ldg(t + i1 * kN + i2), __ldg(t + (i1 + 1) * kN + i2), o1 - i1),
                mix_r<R>(__ldg(t + i1 * kN + i2 + 1), __ldg(t + (i1 + 1) * kN + i2 + 1), o1 - i1), o2 - i2);
}
template <class R>
RT_D R lut_albedo_avg(R rough, const float* t) {
    R o = sqr(rough) * 64;
    int i = int(o);
    if (i >= 63) return __ldg(t + 63);
    return mix_r<R>(__ldg(t + i), __ldg(t + i + 1), o - i);
}
template <class R>
RT_D vec3t<R> multiple_scatter(const SceneView& sc, sc_t<R> NdotL, sc_t<R> NdotV, sc_t<R> rough, vec3t<R> Favg) {
    R bl = lut_bsdf_avg(NdotL, rough, sc.lut), bv = lut_bsdf_avg(NdotV, rough, sc.lut);
    R ea = lut_albedo_avg(rough, sc.lut_avg);
    R fms = (1.0f - bl) * (1.0f - bv) / (Kc<R>::pi * (1.0f - ea));
    vec3t<R> fadd = Favg * Favg * ea / (1.0f - Favg * (1.0f - ea));
    return fms * fadd;
}

// ------------------------------------------------------------ materials
struct Surf {
    v3 sn;                    // shading normal facing the incoming ray
    bool front;
    const DevMaterial* mat;   // nullptr: no material (evaluates to zero)
};

template <class R>
struct MatParamsT {
    vec3t<R> albedo, eta, k, specular;
    R rough, aniso, int_ior, ext_ior, metallic, coat_weight, cru, crv;
    bool nonlinear;
    int type;
};
RT_D MatParamsT<float> load_material(const DevMaterial* m) {
    MatParamsT<float> p;
    // plain loads: `m` may be a path's textured copy written earlier in the same kernel
    const float4* q = reinterpret_cast<const float4*>(m);
    float4 w0 = q[0], w1 = q[1], w2 = q[2], w3 = q[3], w4 = q[4], w5 = q[5];
    p.type = __float_as_int(w0.x);
    p.albedo = v3(w0.y, w0.z, w0.w);
    p.rough = w1.x;
    p.aniso = w1.y;
    p.int_ior = w1.z;
    p.ext_ior = w1.w;
    p.eta = v3(w2.x, w2.y, w2.z);
    p.metallic = w2.w;
    p.k = v3(w3.x, w3.y, w3.z);
    p.coat_weight = w3.w;
    p.specular = v3(w4.x, w4.y, w4.z);
    p.nonlinear = __float_as_int(w4.w) != 0;
    p.cru = w5.x;
    p.crv = w5.y;
    return p;
}

// The material parameters in the sampler's precision.
template <class R>
RT_D MatParamsT<R> mat_cast(const MatParamsT<float>& a) {
    MatParamsT<R> p;
    p.albedo = vec3t<R>(a.albedo.x, a.albedo.y, a.albedo.z);
    p.eta = vec3t<R>(a.eta.x, a.eta.y, a.eta.z);
    p.k = vec3t<R>(a.k.x, a.k.y, a.k.z);
    p.specular = vec3t<R>(a.specular.x, a.specular.y, a.specular.z);
    p.rough = a.rough, p.aniso = a.aniso, p.int_ior = a.int_ior, p.ext_ior = a.ext_ior;
    p.metallic = a.metallic, p.coat_weight = a.coat_weight, p.cru = a.cru, p.crv = a.crv;
    p.nonlinear = a.nonlinear;
    p.type = a.type;
    return p;
}
template <class R>
RT_D vec3t<R> cvt(v3 a) {
    return vec3t<R>(a.x, a.y, a.z);
}
using MatParams = MatParamsT<float>;

// Diffuse, Material.h:7-72
template <class R>
RT_D vec3t<R> diffuse_f(const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, sc_t<R> NdotL, R& pdf) {
    vec3t<R> H = normalize(V + L);
    R NdotV = dot(N, V), VdotH = dot(V, H);
    if (NdotL <= 0.0f || NdotV <= 0.0f) return vec3t<R>(0.0f);
    R a = m.rough * m.rough, s2 = a * a;
    R VdotL = 2.0f * VdotH * VdotH - 1.0f;
    R cosri = VdotL - NdotV * NdotL;
    R C1 = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    R C2 = 0.45f * s2 / (s2 + 0.09f) * cosri * (cosri >= 0.0f ? fmax_r(NdotL, NdotV) : 1.0f);
    pdf = cosine_pdf(NdotL);
    return m.albedo * Kc<R>::inv_pi * (C1 + C2) * (1.0f + m.rough * 0.5f);
}
// Conductor, Material.h:76-146
template <class R>
RT_D vec3t<R> conductor_f(const SceneView& sc, const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, vec3t<R> H, R& pdf) {
    R au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    vec3t<R> Favg = average_fresnel_conductor(m.eta, m.k);
    R Dv = ggx_dv(V, H, N, au, av);
    pdf = Dv * fabs_r(1.0f / (4.0f * dot(V, H)));
    R NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= 0.0f || NdotL <= 0.0f) return vec3t<R>(0.0f);
    vec3t<R> F = fresnel_conductor(V, H, m.eta, m.k);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    return m.albedo * (F * D * G / (4.0f * NdotV * NdotL) + multiple_scatter(sc, NdotL, NdotV, m.rough, Favg));
}
// Dielectric, Material.h:150-269 (shared tail of evaluate and sample)
template <class R>
RT_D vec3t<R> dielectric_f(const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, vec3t<R> H, sc_t<R> e, bool refl, sc_t<R> Dv, sc_t<R> F, sc_t<R> D,
                     sc_t<R> au, sc_t<R> av, R& pdf) {
    R NdotV = fabs_r(dot(N, V)), NdotL = fabs_r(dot(N, L));
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    if (refl) {
        R dwh = fabs_r(1.0f / (4.0f * dot(V, H)));
        pdf = F * Dv * dwh;
        return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
    }
    R HdotV = dot(H, V), HdotL = dot(H, L);
    R sd = e * HdotV + HdotL;
    R factor = fabs_r(HdotL * HdotV / (NdotL * NdotV));
    R dwh = fabs_r(HdotL) / sqr(sd);
    pdf = (1.0f - F) * Dv * dwh;
    vec3t<R> f = m.albedo * (1.0f - F) * D * G * factor / sqr(sd);
    f *= sqr(1.0f / e);
    return f;
}
// Plastic, Material.h:273-403 (shared tail)
template <class R>
RT_D vec3t<R> plastic_f(const SceneView& sc, const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, vec3t<R> H, sc_t<R> Fo, sc_t<R> Fi, sc_t<R> ps,
                  R& pdf) {
    R au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    R eta = m.int_ior / m.ext_ior;
    R Favg = average_fresnel_dielectric(eta);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    R Dv = ggx_dv(V, H, N, au, av);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    R F = fresnel_dielectric(L, H, 1.0f / eta);
    vec3t<R> f = m.nonlinear ? m.albedo / (1.0f - m.albedo * Favg) : m.albedo / (1.0f - Favg);
    f *= (1.0f - Fi) * (1.0f - Fo) * Kc<R>::inv_pi;
    f += m.specular * (vec3t<R>(F) * D * G / (4.0f * NdotL * NdotV) + multiple_scatter(sc, NdotL, NdotV, m.rough, vec3t<R>(Favg)));
    pdf = ps * Dv * fabs_r(1.0f / (4.0f * dot(V, H))) + (1.0f - ps) * cosine_pdf(NdotL);
    return f;
}
template <class R>
RT_D R plastic_weight(const MatParamsT<R>& m) {
    R d = m.albedo.x + m.albedo.y + m.albedo.z, s = m.specular.x + m.specular.y + m.specular.z;
    return s / (s + d);
}
// Metal workflow, Material.h:407-516 (shared tail)
template <class R>
RT_D vec3t<R> metal_f(const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, vec3t<R> H, R& pdf) {
    R au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    R diel = 1.0f - m.metallic, spec = m.metallic + diel, pdiff = diel / (diel + spec);
    R Dv = ggx_dv(V, H, N, au, av);
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    vec3t<R> F0 = vec3t<R>(0.04f) * (1.0f - m.metallic) + m.albedo * m.metallic;
    R vdh = dot(V, H);
    R tmp = 1.0f - fmin_r(1.0f, fmax_r(0.0f, vdh));
    R tmp2 = tmp * tmp, Fc = tmp2 * tmp2 * tmp;
    vec3t<R> F = F0 + (1.0f - F0) * Fc;
    vec3t<R> sb = D * F * G / (4.0f * NdotL * NdotV);
    vec3t<R> db = m.albedo * Kc<R>::inv_pi;
    pdf = (1.0f - pdiff) * Dv * fabs_r(1.0f / (4.0f * vdh)) + pdiff * cosine_pdf(NdotL);
    return pdiff * db + (1.0f - pdiff) * sb;
}
template <class R>
RT_D R thin_fresnel(vec3t<R> V, vec3t<R> H, sc_t<R> eta) {  // Material.h:548-551
    R F = fresnel_dielectric(V, H, 1.0f / eta);
    if (F < 1.0f) F *= 2.0f / (1.0f + F);
    return F;
}
// Clear-coated conductor coat term, Material.h:634-734
template <class R>
RT_D vec3t<R> clearcoat_mix(const SceneView& sc, const MatParamsT<R>& m, vec3t<R> N, vec3t<R> V, vec3t<R> L, vec3t<R> H, vec3t<R> cond, sc_t<R> cpdf,
                      R& pdf) {
    R au = sqr(m.cru), av = sqr(m.crv);
    R NdotV = dot(N, V), NdotL = dot(N, L);
    R Dv = ggx_dv(V, H, N, au, av);
    R F = fresnel_dielectric(V, H, 1.0f / 1.5f);
    R cw = m.coat_weight * F;
    R G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    R D = ggx_d(H, N, au, av);
    R coat_pdf = Dv * fabs_r(1.0f / (4.0f * dot(V, H)));
    vec3t<R> coat(D * G / (4.0f * NdotV * NdotL));
    pdf = cw * coat_pdf + (1.0f - cw) * cpdf;
    return cw * coat + (1.0f - cw) * cond;
}

// EvaluateMaterial, Material.h:783-813
template <class R>
RT_D vec3t<R> eval_material(const SceneView& sc, const Surf& s, vec3t<R> V, vec3t<R> L, R& pdf) {
    pdf = 0.0f;
    if (!s.mat) return vec3t<R>(0.0f);
    const MatParamsT<R> m = mat_cast<R>(load_material(s.mat));
    const vec3t<R> N = cvt<R>(s.sn);
    switch (m.type) {
        case RT_MAT_DIFFUSE: {
            vec3t<R> lL = to_local(L, N);
            return diffuse_f(m, N, V, L, lL.z, pdf);
        }
        case RT_MAT_CONDUCTOR: return conductor_f(sc, m, N, V, L, normalize(V + L), pdf);
        case RT_MAT_DIELECTRIC: {
            R au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
            R eta = m.int_ior / m.ext_ior;
            R e = s.front ? (1.0f / eta) : eta;
            bool refl = dot(N, L) * dot(N, V) > 0.0f;
            vec3t<R> H;
            if (refl) {
                H = normalize(V + L);
            } else {
                H = -normalize(e * V + L);
                if (dot(N, H) < 0.0f) H = -H;
            }
            R Dv = ggx_dv(V, H, N, au, av);
            pdf = Dv * fabs_r(1.0f / (4.0f * dot(V, H)));
            R F = fresnel_dielectric(V, H, e);
            R D = ggx_d(H, N, au, av);
            return dielectric_f(m, N, V, L, H, e, refl, Dv, F, D, au, av, pdf);
        }
        case RT_MAT_PLASTIC: {
            R eta = m.int_ior / m.ext_ior;
            vec3t<R> H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            R Fo = fresnel_dielectric(V, N, 1.0f / eta), Fi = fresnel_dielectric(L, N, 1.0f / eta);
            R w = plastic_weight(m);
            R ps = Fi * w, pd = (1.0f - Fi) * (1.0f - w);
            ps = ps / (ps + pd);
            return plastic_f(sc, m, N, V, L, H, Fo, Fi, ps, pdf);
        }
        case RT_MAT_METAL_WORKFLOW: {
            vec3t<R> H = normalize(L + V);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            return metal_f(m, N, V, L, H, pdf);
        }
        case RT_MAT_THIN_DIELECTRIC: {
            R eta = m.int_ior / m.ext_ior, a = sqr(m.rough);
            bool refl = dot(N, L) * dot(N, V) > 0.0f;
            vec3t<R> H;
            if (refl) {
                H = normalize(V + L);
            } else {
                vec3t<R> Vr = to_world(to_local(V, -N), N);
                H = normalize(Vr + L);
                if (dot(N, H) < 0.0f) H = -H;
            }
            R Dv = ggx_dv(V, H, N, a, a);
            R F = thin_fresnel(V, H, eta);
            R D = ggx_d(H, N, a, a);
            R dwh = fabs_r(1.0f / (4.0f * dot(V, H)));
            R NdotV = fabs_r(dot(N, V)), NdotL = fabs_r(dot(N, L));
            R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
            if (refl) {
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
                pdf = F * Dv * dwh;
                return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
            }
            if (dot(N, L) * dot(N, V) >= 0.0f) return vec3t<R>(0.0f);
            pdf = (1.0f - F) * Dv * dwh;
            return m.albedo * (1.0f - F) * D * G / (4.0f * NdotV * NdotL);
        }
        case RT_MAT_CLEARCOATED_CONDUCTOR: {
            vec3t<R> H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            R cpdf = 0.0f;
            vec3t<R> cond = conductor_f(sc, m, N, V, L, H, cpdf);
            return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
        }
        case RT_MAT_DIFFUSE_TRANSMITTER: {
            vec3t<R> Nn = -N;
            vec3t<R> lL = to_local(L, Nn);
            R NdotL = lL.z, NdotV = dot(Nn, V);
            if (NdotL * NdotV >= 0.0f) return vec3t<R>(0.0f);
            pdf = cosine_pdf(fabs_r(NdotL));
            return m.albedo * Kc<R>::inv_pi;
        }
    }
    return vec3t<R>(0.0f);
}

// SampleMaterial, Material.h:815-845
template <class R, class RNG>
RT_D vec3t<R> sample_material_t(const SceneView& sc, const Surf& s, RNG& rng, vec3t<R> V, vec3t<R>& L, R& pdf) {
    pdf = 0.0f;
    if (!s.mat) return vec3t<R>(0.0f);
    const MatParamsT<R> m = mat_cast<R>(load_material(s.mat));
    const vec3t<R> N = cvt<R>(s.sn);
    R au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    switch (m.type) {
        case RT_MAT_DIFFUSE: {
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> lL = cosine_sample_hemisphere(u0, u1);
            L = to_world(lL, N);
            return diffuse_f(m, N, V, L, lL.z, pdf);
        }
        case RT_MAT_CONDUCTOR: {
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            L = reflect(-V, H);
            return conductor_f(sc, m, N, V, L, H, pdf);
        }
        case RT_MAT_DIELECTRIC: {
            R eta = m.int_ior / m.ext_ior;
            R e = s.front ? (1.0f / eta) : eta;
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            R Dv = ggx_dv(V, H, N, au, av);
            R F = fresnel_dielectric(V, H, e);
            R D = ggx_d(H, N, au, av);
            if (rng.next() < F) {
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
                return dielectric_f(m, N, V, L, H, e, true, Dv, F, D, au, av, pdf);
            }
            L = refract(-V, H, e);
            if (dot(N, L) * dot(N, V) >= 0.0f) return vec3t<R>(0.0f);
            return dielectric_f(m, N, V, L, H, e, false, Dv, F, D, au, av, pdf);
        }
        case RT_MAT_PLASTIC: {
            R eta = m.int_ior / m.ext_ior;
            if (dot(N, V) <= 0.0f) return vec3t<R>(0.0f);
            R Fo = fresnel_dielectric(V, N, 1.0f / eta), Fi = Fo;
            R w = plastic_weight(m);
            R ps = Fi * w, pd = (1.0f - Fi) * (1.0f - w);
            ps = ps / (ps + pd);
            vec3t<R> H;
            if (rng.next() < ps) {
                R u0 = rng.next(), u1 = rng.next();
                H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            } else {
                R u0 = rng.next(), u1 = rng.next();
                L = to_world(cosine_sample_hemisphere(u0, u1), N);
                H = normalize(V + L);
                Fi = fresnel_dielectric(L, N, 1.0f / eta);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            }
            return plastic_f(sc, m, N, V, L, H, Fo, Fi, ps, pdf);
        }
        case RT_MAT_METAL_WORKFLOW: {
            if (dot(N, V) <= 0.0f) return vec3t<R>(0.0f);
            R diel = 1.0f - m.metallic, spec = m.metallic + diel, pdiff = diel / (diel + spec);
            vec3t<R> H;
            if (rng.next() < pdiff) {
                R u0 = rng.next(), u1 = rng.next();
                L = to_world(cosine_sample_hemisphere(u0, u1), N);
                H = normalize(V + L);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            } else {
                R u0 = rng.next(), u1 = rng.next();
                H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            }
            return metal_f(m, N, V, L, H, pdf);
        }
        case RT_MAT_THIN_DIELECTRIC: {
            R eta = m.int_ior / m.ext_ior, a = sqr(m.rough);
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> H = to_world(sample_vndf(N, V, a, a, u0, u1), N);
            R Dv = ggx_dv(V, H, N, a, a);
            R F = thin_fresnel(V, H, eta);
            R D = ggx_d(H, N, a, a);
            R dwh = fabs_r(1.0f / (4.0f * dot(V, H)));
            if (rng.next() < F) {
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
                R NdotV = fabs_r(dot(N, V)), NdotL = fabs_r(dot(N, L));
                R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
                pdf = F * Dv * dwh;
                return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
            }
            L = -V;
            if (dot(N, L) * dot(N, V) >= 0.0f) return vec3t<R>(0.0f);
            R NdotV = fabs_r(dot(N, V)), NdotL = fabs_r(dot(N, L));
            R G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
            pdf = (1.0f - F) * Dv * dwh;
            return m.albedo * (1.0f - F) * D * G / (4.0f * NdotV * NdotL);
        }
        case RT_MAT_CLEARCOATED_CONDUCTOR: {
            R cau = sqr(m.cru), cav = sqr(m.crv);
            R F = fresnel_dielectric(V, N, 1.0f / 1.5f);
            R cw = m.coat_weight * F;
            if (rng.next() < cw) {
                R u0 = rng.next(), u1 = rng.next();
                vec3t<R> H = to_world(sample_vndf(N, V, cau, cav, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
                R cpdf = 0.0f;
                vec3t<R> cond = conductor_f(sc, m, N, V, L, normalize(V + L), cpdf);
                return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
            }
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> Hc = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            L = reflect(-V, Hc);
            R cpdf = 0.0f;
            vec3t<R> cond = conductor_f(sc, m, N, V, L, Hc, cpdf);
            vec3t<R> H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return vec3t<R>(0.0f);
            return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
        }
        case RT_MAT_DIFFUSE_TRANSMITTER: {
            R u0 = rng.next(), u1 = rng.next();
            vec3t<R> lL = cosine_sample_hemisphere(u0, u1);
            vec3t<R> Nn = -N;
            L = to_world(lL, Nn);
            R NdotL = lL.z, NdotV = dot(Nn, V);
            if (NdotL * NdotV >= 0.0f) return vec3t<R>(0.0f);
            pdf = cosine_pdf(fabs_r(NdotL));
            return m.albedo * Kc<R>::inv_pi;
        }
    }
    return vec3t<R>(0.0f);
}


// SampleMaterial in double precision: the sampled direction and the f and
// pdf reported for it come from the double instantiation of the material
// code above, fed the FP32 inputs and the FP32 random numbers, and are
// rounded once at the end.  The visible-normal map and the f / pdf chains
// amplify FP32 rounding well past 1e-5 relative (by 1 / alpha^2 in the
// (1 - cos^2) / cos^2 of a sharp GGX lobe, and near the rim of the
// projected disk), which double arithmetic keeps at the output rounding.
// Random numbers are consumed as by the FP32 code.
template <class RNG>
RT_D v3 sample_material(const SceneView& sc, const Surf& s, RNG& rng, v3 V, v3& L, float& pdf) {
    v3d Ld = to_d(L);
    double pd = 0.0;
    const v3d f = sample_material_t<double>(sc, s, rng, to_d(V), Ld, pd);
    L = to_f(Ld);
    pdf = float(pd);
    return to_f(f);
}

// The isotropic GGX distribution with the cos^4 of its definition (the
// anisotropic branch of ggx_d already has it): the density with which the
// visible-normal sampler draws half vectors is smith_g1 * (V.H) * this / (N.V).
RT_D float ggx_d_exact(v3 H, v3 N, float au, float av) {
    if (au != av) return ggx_d(H, N, au, av);
    const float c = dot(H, N);
    if (c <= 0.0f) return 0.0f;
    const float c2 = sqr(c), t2 = (1.0f - c2) / c2, a2 = au * av;
    return a2 / (kPi * c2 * c2 * sqr(a2 + t2));
}
RT_D float vndf_reflect_pdf(v3 V, v3 H, v3 N, float au, float av) {
    return smith_g1(V, H, N, au, av) * dot(V, H) * ggx_d_exact(H, N, au, av) / dot(N, V) *
           fabsf(1.0f / (4.0f * dot(V, H)));
}

// What plain BSDF sampling integrates, for the one-sample MIS of guided
// sampling.  The reference's sampler draws half vectors from the exact
// visible-normal distribution, but its isotropic DistributionGGX
// (Microfacet.h:144-160) divides by cos^2 where the definition has cos^4, so
// the pdf it reports, like EvaluateMaterial's, is not the density of its
// samples; and plastic and the clear-coated conductor pick their lobe with a
// Fresnel term of V alone (SamplePlastic, Material.h:327; Sample-
// ClearCoatedConductor, :669) where the evaluators use F(L, N), resp. F(V, H)
// (:273, :634).  A BSDF-sampled path is weighted by f / pdf as the sampler
// reports them, so plain BSDF sampling integrates f_dir = p_true * E[f / pdf |
// L].  Outputs: f_dir; p_true, the sampler's real density at L; p_rep, the
// pdf the sampler reports at L (plain sampling's emission MIS weight uses it).
// With these, guided sampling reduces exactly to plain sampling as the
// mixture probability goes to zero.
RT_D void guide_bsdf(const SceneView& sc, const Surf& s, v3 V, v3 L, v3& f_dir, float& p_true, float& p_rep) {
    f_dir = v3(0.0f);
    p_true = p_rep = 0.0f;
    if (!s.mat) return;
    const MatParams m = load_material(s.mat);
    const v3 N = s.sn;
    const float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    switch (m.type) {
        case RT_MAT_CONDUCTOR:
        case RT_MAT_METAL_WORKFLOW:
        case RT_MAT_CLEARCOATED_CONDUCTOR: {
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return;
            float pb = 0.0f;
            const v3 fb = eval_material(sc, s, V, L, pb);
            const v3 H = normalize(V + L);
            const float spec = vndf_reflect_pdf(V, H, N, au, av);
            if (m.type == RT_MAT_CONDUCTOR) {
                p_true = spec;
            } else if (m.type == RT_MAT_METAL_WORKFLOW) {
                const float diel = 1.0f - m.metallic, sp = m.metallic + diel, pdiff = diel / (diel + sp);
                p_true = (1.0f - pdiff) * spec + pdiff * cosine_pdf(dot(N, L));
            } else {
                const float cw = m.coat_weight * fresnel_dielectric(V, N, 1.0f / 1.5f);
                p_true = cw * vndf_reflect_pdf(V, H, N, sqr(m.cru), sqr(m.crv)) + (1.0f - cw) * spec;
            }
            p_rep = pb;
            if (pb > 0.0f) f_dir = fb * (p_true / pb);
            return;
        }
        case RT_MAT_PLASTIC: {
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return;
            const float eta = m.int_ior / m.ext_ior;
            const v3 H = normalize(V + L);
            const float Fo = fresnel_dielectric(V, N, 1.0f / eta), Fi = fresnel_dielectric(L, N, 1.0f / eta);
            const float w = plastic_weight(m);
            float ps = Fo * w, pd = (1.0f - Fo) * (1.0f - w);
            ps = ps / (ps + pd);
            float unused;
            const v3 f_spec = plastic_f(sc, m, N, V, L, H, Fo, Fo, ps, unused);  // SamplePlastic's specular branch
            const v3 f_diff = plastic_f(sc, m, N, V, L, H, Fo, Fi, ps, p_rep);    // its diffuse branch; the reported pdf
            const float pc = cosine_pdf(dot(N, L));
            const float spec_true = vndf_reflect_pdf(V, H, N, au, av);
            p_true = ps * spec_true + (1.0f - ps) * pc;
            if (p_rep > 0.0f) f_dir = (ps * spec_true * f_spec + (1.0f - ps) * pc * f_diff) / p_rep;
            return;
        }
        default: {  // cosine-sampled types: the reported pdf is the density
            f_dir = eval_material(sc, s, V, L, p_true);
            p_rep = p_true;
        }
    }
}

// ------------------------------------------------------------ lights
struct LightParams {
    int type;
    bool two_sided;
    float radius;
    int medium;
    v3 radiance, position, u, v;
};
RT_D LightParams load_light(const DevLight* l) {
    const float4* q = reinterpret_cast<const float4*>(l);
    float4 w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2), w3 = __ldg(q + 3), w4 = __ldg(q + 4);
    LightParams p;
    p.type = __float_as_int(w0.x);
    p.two_sided = __float_as_int(w0.y) != 0;
    p.radius = w0.z;
    p.medium = __float_as_int(w0.w);
    p.radiance = xyz(w1);
    p.position = xyz(w2);
    p.u = xyz(w3);
    p.v = xyz(w4);
    return p;
}
RT_D float intersect_quad(v3 o, v3 d, v3 corner, v3 u_, v3 v_) {  // Light.h:6-26
    v3 n = normalize(cross(u_, v_));
    v3 u = u_ * (1.0f / dot(u_, u_));
    v3 v = v_ * (1.0f / dot(v_, v_));
    float dt = dot(d, n);
    float t = (dot(n, corner) - dot(n, o)) / dt;
    if (t > kEps) {
        v3 p = o + d * t;
        v3 vi = p - corner;
        float a1 = dot(u, vi);
        if (a1 >= 0.0f && a1 <= 1.0f) {
            float a2 = dot(v, vi);
            if (a2 >= 0.0f && a2 <= 1.0f) return t;
        }
    }
    return FLT_MAX;
}
RT_D float intersect_sphere(v3 o, v3 d, v3 c, float radius) {  // Light.h:78-98
    v3 co = c - o;
    float b = dot(co, d);
    float det = b * b - dot(co, co) + radius * radius;
    if (det < 0.0f) return FLT_MAX;
    det = sqrtf(det);
    float t1 = b - det;
    if (t1 > kEps) return t1;
    float t2 = b + det;
    if (t2 > kEps) return t2;
    return FLT_MAX;
}
// EvaluateLight, Light.h:145-156 (quad :28-52, sphere :100-116)
RT_D v3 evaluate_light(const LightParams& l, v3 o, v3 d, float distance, float& pdf, float& ld) {
    if (l.type == RT_LIGHT_QUAD) {
        v3 n = normalize(cross(l.u, l.v));
        float ct = dot(d, n);
        if (!l.two_sided && ct < 0.0f) {
            pdf = 0.0f;
            return v3(0.0f);
        }
        ld = intersect_quad(o, d, l.position, l.u, l.v);
        float area = length(l.u) * length(l.v);
        if (ld < distance) {
            pdf = 1.0f / area;
            pdf *= sqr(ld) / fabsf(ct);
            return l.radiance;
        }
        pdf = 0.0f;
        return v3(0.0f);
    }
    if (l.type == RT_LIGHT_SPHERE) {
        ld = intersect_sphere(o, d, l.position, l.radius);
        if (ld < distance) {
            v3 dir = l.position - o;
            float d2 = dot(dir, dir);
            float s2 = l.radius * l.radius / d2;
            pdf = uniform_pdf_cone(sqrtf(1.0f - s2));
            return l.radiance;
        }
        pdf = 0.0f;
        return v3(0.0f);
    }
    pdf = 0.0f;
    return v3(0.0f);
}
// SampleLight, Light.h:158-168 (quad :54-76, sphere :118-141) + point light.
RT_D v3 sample_light(const LightParams& l, v3 p, float s0, float s1, v3& L, float& dist, float& pdf) {
    if (l.type == RT_LIGHT_QUAD) {
        v3 n = normalize(cross(l.u, l.v));
        v3 pos = l.position + l.u * s0 + l.v * s1;
        L = pos - p;
        float d2 = dot(L, L);
        dist = sqrtf(d2);
        L /= dist;
        float ct = dot(L, n);
        if (!l.two_sided && ct < 0.0f) {
            pdf = 0.0f;
            return v3(0.0f);
        }
        float area = length(l.u) * length(l.v);
        pdf = 1.0f / area;
        pdf *= d2 / fabsf(ct);
        return l.radiance;
    }
    if (l.type == RT_LIGHT_SPHERE) {
        v3 dir = l.position - p;
        float d2 = dot(dir, dir);
        float inv = 1.0f / sqrtf(d2);
        dir *= inv;
        dist = d2 * inv;
        float st = l.radius * inv;
        if (st < 1.0f) {
            float ct = sqrtf(1.0f - st * st);
            v3 lL = uniform_sample_cone(s0, s1, ct);
            float ci = lL.z;
            L = to_world(lL, dir);
            pdf = uniform_pdf_cone(ct);
            dist = ci * dist - sqrtf(fmaxf(0.0f, l.radius * l.radius - (1.0f - ci * ci) * d2));
            return l.radiance;
        }
        pdf = 0.0f;
        return v3(0.0f);
    }
    if (l.type == RT_LIGHT_POINT) {
        v3 dir = l.position - p;
        float d2 = dot(dir, dir);
        dist = sqrtf(d2);
        L = dir / dist;
        pdf = 1.0f;
        return l.radiance / d2;
    }
    pdf = 0.0f;
    return v3(0.0f);
}

// ------------------------------------------------------------ media
struct MedParams {
    int type, phase;
    v3 g, sigma_s, sigma_a;
    float scale;
};
RT_D MedParams load_medium(const DevMedium* m) {
    MedParams p;
    p.type = m->type;
    p.phase = m->phase;
    p.scale = m->scale;
    p.g = ld3(m->g);
    p.sigma_s = ld3(m->sigma_s);
    p.sigma_a = ld3(m->sigma_a);
    return p;
}
RT_D v3 hg_terms(const MedParams& m, float ct, float& pdf) {  // Medium.h:26-42
    float a[3];
    pdf = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float g = m.g[c];
        float tmp = 1.0f + g * g + 2.0f * g * ct;
        a[c] = (0.25f * kInvPi) * (1.0f - g * g) / (tmp * sqrtf(tmp));
        pdf += a[c];
    }
    pdf *= (1.0f / 3.0f);
    return v3(a[0], a[1], a[2]);
}
RT_D v3 evaluate_phase(const MedParams& m, v3 V, v3 L, float& pdf) {  // Medium.h:83-94
    pdf = 0.0f;
    if (m.phase == RT_PHASE_ISOTROPIC) {
        pdf = 0.25f * kInvPi;
        return v3(0.25f * kInvPi);
    }
    if (m.phase == RT_PHASE_HENYEY_GREENSTEIN) {
        v3 a = hg_terms(m, dot(L, V), pdf);
        if (pdf <= 0.0f) return v3(0.0f);
        return a;
    }
    return v3(0.0f);
}
template <class RNG>
RT_D v3 sample_phase(const MedParams& m, RNG& rng, v3 V, v3& L, float& pdf) {  // Medium.h:96-108
    pdf = 0.0f;
    if (m.phase == RT_PHASE_ISOTROPIC) {
        float u0 = rng.next(), u1 = rng.next();
        L = uniform_sample_sphere(u0, u1);
        pdf = 0.25f * kInvPi;
        return v3(0.25f * kInvPi);
    }
    if (m.phase == RT_PHASE_HENYEY_GREENSTEIN) {
        int ch = min(int(rng.next() * 3.0f), 2);
        float g = m.g[ch];
        float ct;
        if (fabsf(g) < kEps) {
            ct = 1.0f - 2.0f * rng.next();
        } else {
            float st = (1.0f - g * g) / (1.0f - g + 2.0f * g * rng.next());
            ct = (1.0f + g * g - st * st) / (2.0f * g);
        }
        v3 att = hg_terms(m, ct, pdf);
        if (pdf <= 0.0f) return v3(0.0f);
        float sn = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float phi = kTwoPi * rng.next();
        float sp, cp;
        sincosf(phi, &sp, &cp);
        L = to_world(normalize(v3(sn * cp, sn * sp, ct)), V);
        return att;
    }
    return v3(0.0f);
}
RT_D float homog_weight(v3 st, v3 alb) {  // Medium.h:119-129
    float w = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (alb[c] > w && st[c] != 0.0f) w = alb[c];
    if (w > 0.0f) w = fmaxf(w, 0.5f);
    return w;
}
// EvaluateMediumDistance (homogeneous), Medium.h:112-158
RT_D v3 eval_medium_distance(const MedParams& m, bool scattered, float dist, float& tp) {
    tp = 0.0f;
    if (m.type != RT_MEDIUM_HOMOGENEOUS) return v3(0.0f);
    v3 ss = m.sigma_s * m.scale, sa = m.sigma_a * m.scale, st = sa + ss;
    float w = homog_weight(st, ss / st);
    float at[3];
    bool valid = false;
    float pdf = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        at[c] = expf(-st[c] * dist);
        if (at[c] > 0.0f) valid = true;
    }
    v3 att(at[0], at[1], at[2]);
    if (scattered) {
        pdf = st.x * at[0] + st.y * at[1] + st.z * at[2];
        pdf *= w * (1.0f / 3.0f);
        att *= ss;
    } else {
        pdf = at[0] + at[1] + at[2];
        pdf = w * (1.0f / 3.0f) * pdf + (1.0f - w);
    }
    tp = pdf;
    if (!valid) att = v3(0.0f);
    return att;
}
// SampleMediumDistance (homogeneous), Medium.h:160-218
template <class RNG>
RT_D bool sample_medium_distance(const MedParams& m, float maxd, float& dist, float& tp, v3& tr, RNG& rng) {
    tp = 0.0f;
    tr = v3(0.0f);
    if (m.type != RT_MEDIUM_HOMOGENEOUS) return false;
    v3 ss = m.sigma_s * m.scale, sa = m.sigma_a * m.scale, st = sa + ss;
    float w = homog_weight(st, ss / st);
    bool scattered = false;
    float x1 = rng.next();
    if (x1 < w) {
        x1 /= w;
        int ch = min(int(rng.next() * 3.0f), 2);
        dist = -logf(1.0f - x1) / st[ch];
        if (dist < maxd) {
            tp = st.x * expf(-st.x * dist);
            tp += st.y * expf(-st.y * dist);
            tp += st.z * expf(-st.z * dist);
            tp *= w * (1.0f / 3.0f);
            scattered = true;
        }
    }
    if (!scattered) {
        dist = maxd;
        tp = expf(-st.x * dist);
        tp += expf(-st.y * dist);
        tp += expf(-st.z * dist);
        tp = w * (1.0f / 3.0f) * tp + (1.0f - w);
    }
    float a[3];
    bool valid = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        a[c] = expf(-st[c] * dist);
        if (a[c] > 0.0f) valid = true;
    }
    tr = v3(a[0], a[1], a[2]);
    if (scattered) tr *= ss;
    if (!valid) tr = v3(0.0f);
    return scattered;
}

// ------------------------------------------------------------ environment
// tex2D<float4> semantics of the reference's environment textures
// (core/src/Scene.cpp:340-349: normalized coordinates, wrap, linear filter),
// evaluated in software with FP32 weights.
RT_D float4 tex_bilinear(const float4* img, int w, int h, float u, float v) {
    u = u - floorf(u);
    v = v - floorf(v);
    float x = u * float(w) - 0.5f, y = v * float(h) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float a = x - fx, b = y - fy;
    int x0 = int(fx), y0 = int(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = x0 < 0 ? x0 + w : (x0 >= w ? x0 - w : x0);
    x1 = x1 < 0 ? x1 + w : (x1 >= w ? x1 - w : x1);
    y0 = y0 < 0 ? y0 + h : (y0 >= h ? y0 - h : y0);
    y1 = y1 < 0 ? y1 + h : (y1 >= h ? y1 - h : y1);
    float4 t00 = __ldg(img + size_t(y0) * w + x0), t10 = __ldg(img + size_t(y0) * w + x1);
    float4 t01 = __ldg(img + size_t(y1) * w + x0), t11 = __ldg(img + size_t(y1) * w + x1);
    float4 r;
    r.x = mixf(mixf(t00.x, t10.x, a), mixf(t01.x, t11.x, a), b);
    r.y = mixf(mixf(t00.y, t10.y, a), mixf(t01.y, t11.y, a), b);
    r.z = mixf(mixf(t00.z, t10.z, a), mixf(t01.z, t11.z, a), b);
    r.w = mixf(mixf(t00.w, t10.w, a), mixf(t01.w, t11.w, a), b);
    return r;
}

// ------------------------------------------------------------ material textures
// tex2D<float4> of an RGBA8 texture with cudaReadModeNormalizedFloat,
// normalized coordinates, wrap addressing and linear filtering
// (core/src/Renderer.cpp:100-143), evaluated in software with FP32 weights on
// texels converted as byte * (1/255).
RT_D float4 texel_rgba8(uint32_t p) {
    const float s = 1.0f / 255.0f;
    return make_float4(float(p & 0xFFu) * s, float((p >> 8) & 0xFFu) * s, float((p >> 16) & 0xFFu) * s,
                       float(p >> 24) * s);
}
RT_D float4 tex_rgba8(const uint32_t* img, int w, int h, float u, float v) {
    u = u - floorf(u);
    v = v - floorf(v);
    float x = u * float(w) - 0.5f, y = v * float(h) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float a = x - fx, b = y - fy;
    int x0 = int(fx), y0 = int(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = x0 < 0 ? x0 + w : (x0 >= w ? x0 - w : x0);
    x1 = x1 < 0 ? x1 + w : (x1 >= w ? x1 - w : x1);
    y0 = y0 < 0 ? y0 + h : (y0 >= h ? y0 - h : y0);
    y1 = y1 < 0 ? y1 + h : (y1 >= h ? y1 - h : y1);
    float4 t00 = texel_rgba8(__ldg(img + size_t(y0) * w + x0)), t10 = texel_rgba8(__ldg(img + size_t(y0) * w + x1));
    float4 t01 = texel_rgba8(__ldg(img + size_t(y1) * w + x0)), t11 = texel_rgba8(__ldg(img + size_t(y1) * w + x1));
    float4 r;
    r.x = mixf(mixf(t00.x, t10.x, a), mixf(t01.x, t11.x, a), b);
    r.y = mixf(mixf(t00.y, t10.y, a), mixf(t01.y, t11.y, a), b);
    r.z = mixf(mixf(t00.z, t10.z, a), mixf(t01.z, t11.z, a), b);
    r.w = mixf(mixf(t00.w, t10.w, a), mixf(t01.w, t11.w, a), b);
    return r;
}
RT_D float4 tex_lookup(const SceneView& sc, int id, float u, float v) {
    int4 info = __ldg(sc.tex_info + id);
    return tex_rgba8(sc.tex + info.x, info.y, info.z, u, v);
}

// NormalFromTangentToWorld, core/cuda/Utils.h:85-94.
RT_D v3 normal_from_tangent(v3 n, v3 t) {
    t = normalize(t * 2.0f - v3(1.0f));
    v3 up = fabsf(n.z) < 0.9f ? v3(0.0f, 0.0f, 1.0f) : v3(1.0f, 0.0f, 0.0f);
    v3 tx = normalize(cross(up, n));
    v3 ty = normalize(cross(n, tx));
    return normalize(tx * t.x + ty * t.y + n * t.z);
}

// ------------------------------------------------------------ filter
RT_D void filter_jitter(int type, float s0, float s1, float& jx, float& jy) {  // Filter.h:5-56
    if (type == RT_FILTER_BOX) {
        jx = s0 - 0.5f;
        jy = s1 - 0.5f;
    } else if (type == RT_FILTER_TENT) {
        float x = s0 * 2.0f, y = s1 * 2.0f;
        x = x < 1.0f ? sqrtf(x) - 1.0f : 1.0f - sqrtf(2.0f - x);
        y = y < 1.0f ? sqrtf(y) - 1.0f : 1.0f - sqrtf(2.0f - y);
        jx = 0.5f + x;
        jy = 0.5f + y;
    } else if (type == RT_FILTER_TRIANGLE) {
        float u1 = s0, u2 = s1;
        if (u2 > u1) {
            u1 *= 0.5f;
            u2 -= u1;
        } else {
            u2 *= 0.5f;
            u1 -= u2;
        }
        jx = 0.5f + u1;
        jy = 0.5f + u2;
    } else if (type == RT_FILTER_GAUSSIAN) {
        float r1 = fmaxf(FLT_MIN, s0);
        float r = sqrtf(-2.0f * logf(r1));
        float st, ct;
        sincosf(kTwoPi * s1, &st, &ct);
        jx = 0.5f + 0.375f * (r * ct);
        jy = 0.5f + 0.375f * (r * st);
    } else {
        jx = s0;
        jy = s1;
    }
}

}  // namespace rtd
