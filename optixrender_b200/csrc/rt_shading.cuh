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
RT_D v3 cosine_sample_hemisphere(float s0, float s1) {  // Sampling.h:56-69
    float r = sqrtf(s0);
    float phi = kTwoPi * s1;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    v3 p(r * cp, r * sp, 0.0f);
    p.z = sqrtf(fmaxf(0.0f, 1.0f - p.x * p.x - p.y * p.y));
    return normalize(p);
}
RT_D float cosine_pdf(float ndotl) { return ndotl * kInvPi; }
RT_D v3 uniform_sample_sphere(float s0, float s1) {  // Sampling.h:76-88
    float phi = kTwoPi * s0;
    float ct = 1.0f - 2.0f * s1;
    float st = sqrtf(1.0f - ct * ct);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return normalize(v3(st * cp, st * sp, ct));
}

// ------------------------------------------------------------ frames
RT_D v3 reflect(v3 v, v3 n) { return normalize(v - 2.0f * dot(v, n) * n); }  // Utils.h:28-30
RT_D v3 refract(v3 v, v3 n, float eta) {                                       // Utils.h:32-38
    float ct = fminf(dot(-v, n), 1.0f);
    v3 perp = eta * (v + ct * n);
    v3 par = -sqrtf(fabsf(1.0f - dot(perp, perp))) * n;
    return normalize(perp + par);
}
RT_D void frame_axes(v3 up, v3& B, v3& C) {  // Utils.h:99-109
    if (fabsf(up.x) > fabsf(up.y)) {
        float inv = 1.0f / sqrtf(up.x * up.x + up.z * up.z);
        C = v3(up.z * inv, 0.0f, -up.x * inv);
    } else {
        float inv = 1.0f / sqrtf(up.y * up.y + up.z * up.z);
        C = v3(0.0f, up.z * inv, -up.y * inv);
    }
    B = cross(C, up);
}
RT_D v3 to_local(v3 d, v3 up) {
    v3 B, C;
    frame_axes(up, B, C);
    return v3(dot(d, B), dot(d, C), dot(d, up));
}
RT_D v3 to_world(v3 d, v3 up) {  // Utils.h:117-129
    v3 B, C;
    frame_axes(up, B, C);
    return normalize(d.x * B + d.y * C + d.z * up);
}

// ------------------------------------------------------------ microfacet
RT_D v3 fresnel_conductor(v3 V, v3 H, v3 er, v3 ei) {  // Microfacet.h:22-46
    float c = dot(V, H), c2 = c * c, s2 = 1.0f - c2, s4 = s2 * s2;
    v3 t1 = er * er - ei * ei - s2;
    v3 a2 = t1 * t1 + 4.0f * ei * ei * er * er;
    a2 = v3(sqrtf(fmaxf(0.0f, a2.x)), sqrtf(fmaxf(0.0f, a2.y)), sqrtf(fmaxf(0.0f, a2.z)));
    v3 a = 0.5f * (a2 + t1);
    a = v3(sqrtf(fmaxf(0.0f, a.x)), sqrtf(fmaxf(0.0f, a.y)), sqrtf(fmaxf(0.0f, a.z)));
    v3 term1 = a2 + s2, term2 = 2.0f * c * a, term3 = a2 * c2 + s4, term4 = term2 * s2;
    v3 rs = (term1 - term2) / (term1 + term2);
    v3 rp = rs * (term3 - term4) / (term3 + term4);
    return 0.5f * (rs + rp);
}
RT_D v3 average_fresnel_conductor(v3 eta, v3 k) {  // Microfacet.h:48-70
    float rr[3], ee[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float e = eta[i], kk = k[i];
        float r = (sqr(e - 1.0f) + sqr(kk)) / (sqr(e + 1.0f) + sqr(kk));
        float t1 = 1.0f + sqrtf(r), t2 = 1.0f - sqrtf(r), t3 = (1.0f - r) / (1.0f + r);
        rr[i] = r;
        ee[i] = (t1 - e * t2) / (t1 - t3 * t2);
    }
    v3 refl(rr[0], rr[1], rr[2]), edge(ee[0], ee[1], ee[2]);
    return v3(0.087237f) + 0.0230685f * edge - 0.0864902f * edge * edge + 0.0774594f * edge * edge * edge +
           0.782654f * refl - 0.136432f * refl * refl + 0.278708f * refl * refl * refl + 0.19744f * edge * refl +
           0.0360605f * edge * edge * refl - 0.2586f * edge * refl * refl;
}
RT_D float fresnel_dielectric(v3 V, v3 H, float eta_inv) {  // Microfacet.h:72-85
    float ci = fabsf(dot(V, H));
    float ct2 = 1.0f - sqr(eta_inv) * (1.0f - sqr(ci));
    if (ct2 <= 0.0f) return 1.0f;
    float ct = sqrtf(ct2);
    float rs = (eta_inv * ci - ct) / (eta_inv * ci + ct);
    float rp = (ci - eta_inv * ct) / (ci + eta_inv * ct);
    return (rs * rs + rp * rp) / 2.0f;
}
RT_D float average_fresnel_dielectric(float eta) {  // Microfacet.h:87-113
    if (eta < 1.0f) return -1.4399f * (eta * eta) + 0.7099f * eta + 0.6681f + 0.0636f / eta;
    float i1 = 1.0f / eta, i2 = i1 * i1, i3 = i2 * i1, i4 = i3 * i1, i5 = i4 * i1;
    return 0.919317f - 3.4793f * i1 + 6.75335f * i2 - 7.80989f * i3 + 4.98554f * i4 - 1.36881f * i5;
}
RT_D float smith_g1(v3 V, v3 H, v3 N, float au, float av) {  // Microfacet.h:117-142
    float cvn = dot(V, N);
    if (cvn * dot(V, H) <= 0.0f) return 0.0f;
    if (fabsf(cvn - 1.0f) < kEps) return 1.0f;
    if (au == av) {
        float c2 = sqr(cvn), t2 = (1.0f - c2) / c2;
        return 2.0f / (1.0f + sqrtf(1.0f + au * au * t2));
    }
    v3 d = to_local(V, N);
    float t = (sqr(au * d.x) + sqr(av * d.y)) / sqr(d.z);
    return 2.0f / (1.0f + sqrtf(1.0f + t));
}
RT_D float ggx_d(v3 H, v3 N, float au, float av) {  // Microfacet.h:144-160
    float c = dot(H, N);
    if (c <= 0.0f) return 0.0f;
    float c2 = sqr(c), t2 = (1.0f - c2) / c2, a2 = au * av;
    if (au == av) return a2 / (kPi * (c * c) * sqr(a2 + t2));
    v3 d = to_local(H, N);
    return 1.0f / (kPi * a2 * sqr(sqr(d.x / au) + sqr(d.y / av) + sqr(d.z)));
}
RT_D float ggx_dv(v3 V, v3 H, v3 N, float au, float av) {  // Microfacet.h:162-164
    return smith_g1(V, H, N, au, av) * dot(V, H) * ggx_d(H, N, au, av) / dot(N, V);
}
RT_D v3 sample_vndf(v3 N, v3 Ve, float au, float av, float s0, float s1) {  // Microfacet.h:188-214
    v3 V = to_local(Ve, N);
    v3 Vh = normalize(v3(au * V.x, av * V.y, V.z));
    float len2 = sqr(Vh.x) + sqr(Vh.y);
    v3 T1 = len2 > 0.0f ? v3(-Vh.y, Vh.x, 0.0f) * sqrtf(1.0f / len2) : v3(1.0f, 0.0f, 0.0f);
    v3 T2 = cross(Vh, T1);
    float r = sqrtf(s0), phi = s1 * kTwoPi;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float t1 = r * cp, t2 = r * sp;
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - sqr(t1)) + s * t2;
    v3 Nh = t1 * T1 + t2 * T2 + sqrtf(fmaxf(0.0f, 1.0f - sqr(t1) - sqr(t2))) * Vh;
    return normalize(v3(au * Nh.x, av * Nh.y, fmaxf(0.0f, Nh.z)));
}
// Kulla-Conty tables, Microfacet.h:293-346
RT_D float lut_bsdf_avg(float cos_theta, float rough, const float* t) {
    const int R = 64;
    float o1 = sqr(rough) * R, o2 = cos_theta * R;
    int i1 = int(o1), i2 = int(o2);
    if (i1 >= R - 1) {
        if (i2 >= R - 1) return __ldg(t + (R - 1) * R + R - 1);
        return mixf(__ldg(t + (R - 1) * R + i2), __ldg(t + (R - 1) * R + i2 + 1), o2 - i2);
    }
    if (i2 >= R - 1) return mixf(__ldg(t + i1 * R + R - 1), __ldg(t + (i1 + 1) * R + R - 1), o1 - i1);
    return mixf(mixf(__ldg(t + i1 * R + i2), __ldg(t + (i1 + 1) * R + i2), o1 - i1),
                mixf(__ldg(t + i1 * R + i2 + 1), __ldg(t + (i1 + 1) * R + i2 + 1), o1 - i1), o2 - i2);
}
RT_D float lut_albedo_avg(float rough, const float* t) {
    float o = sqr(rough) * 64;
    int i = int(o);
    if (i >= 63) return __ldg(t + 63);
    return mixf(__ldg(t + i), __ldg(t + i + 1), o - i);
}
RT_D v3 multiple_scatter(const SceneView& sc, float NdotL, float NdotV, float rough, v3 Favg) {
    float bl = lut_bsdf_avg(NdotL, rough, sc.lut), bv = lut_bsdf_avg(NdotV, rough, sc.lut);
    float ea = lut_albedo_avg(rough, sc.lut_avg);
    float fms = (1.0f - bl) * (1.0f - bv) / (kPi * (1.0f - ea));
    v3 fadd = Favg * Favg * ea / (1.0f - Favg * (1.0f - ea));
    return fms * fadd;
}

// ------------------------------------------------------------ materials
struct Surf {
    v3 sn;                    // shading normal facing the incoming ray
    bool front;
    const DevMaterial* mat;   // nullptr: no material (evaluates to zero)
};

struct MatParams {
    v3 albedo, eta, k, specular;
    float rough, aniso, int_ior, ext_ior, metallic, coat_weight, cru, crv;
    bool nonlinear;
    int type;
};
RT_D MatParams load_material(const DevMaterial* m) {
    MatParams p;
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

// Diffuse, Material.h:7-72
RT_D v3 diffuse_f(const MatParams& m, v3 N, v3 V, v3 L, float NdotL, float& pdf) {
    v3 H = normalize(V + L);
    float NdotV = dot(N, V), VdotH = dot(V, H);
    if (NdotL <= 0.0f || NdotV <= 0.0f) return v3(0.0f);
    float a = m.rough * m.rough, s2 = a * a;
    float VdotL = 2.0f * VdotH * VdotH - 1.0f;
    float cosri = VdotL - NdotV * NdotL;
    float C1 = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    float C2 = 0.45f * s2 / (s2 + 0.09f) * cosri * (cosri >= 0.0f ? fmaxf(NdotL, NdotV) : 1.0f);
    pdf = cosine_pdf(NdotL);
    return m.albedo * kInvPi * (C1 + C2) * (1.0f + m.rough * 0.5f);
}
// Conductor, Material.h:76-146
RT_D v3 conductor_f(const SceneView& sc, const MatParams& m, v3 N, v3 V, v3 L, v3 H, float& pdf) {
    float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    v3 Favg = average_fresnel_conductor(m.eta, m.k);
    float Dv = ggx_dv(V, H, N, au, av);
    pdf = Dv * fabsf(1.0f / (4.0f * dot(V, H)));
    float NdotV = dot(N, V), NdotL = dot(N, L);
    if (NdotV <= 0.0f || NdotL <= 0.0f) return v3(0.0f);
    v3 F = fresnel_conductor(V, H, m.eta, m.k);
    float G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    float D = ggx_d(H, N, au, av);
    return m.albedo * (F * D * G / (4.0f * NdotV * NdotL) + multiple_scatter(sc, NdotL, NdotV, m.rough, Favg));
}
// Dielectric, Material.h:150-269 (shared tail of evaluate and sample)
RT_D v3 dielectric_f(const MatParams& m, v3 N, v3 V, v3 L, v3 H, float e, bool refl, float Dv, float F, float D,
                     float au, float av, float& pdf) {
    float NdotV = fabsf(dot(N, V)), NdotL = fabsf(dot(N, L));
    float G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    if (refl) {
        float dwh = fabsf(1.0f / (4.0f * dot(V, H)));
        pdf = F * Dv * dwh;
        return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
    }
    float HdotV = dot(H, V), HdotL = dot(H, L);
    float sd = e * HdotV + HdotL;
    float factor = fabsf(HdotL * HdotV / (NdotL * NdotV));
    float dwh = fabsf(HdotL) / sqr(sd);
    pdf = (1.0f - F) * Dv * dwh;
    v3 f = m.albedo * (1.0f - F) * D * G * factor / sqr(sd);
    f *= sqr(1.0f / e);
    return f;
}
// Plastic, Material.h:273-403 (shared tail)
RT_D v3 plastic_f(const SceneView& sc, const MatParams& m, v3 N, v3 V, v3 L, v3 H, float Fo, float Fi, float ps,
                  float& pdf) {
    float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    float eta = m.int_ior / m.ext_ior;
    float Favg = average_fresnel_dielectric(eta);
    float NdotV = dot(N, V), NdotL = dot(N, L);
    float Dv = ggx_dv(V, H, N, au, av);
    float G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    float D = ggx_d(H, N, au, av);
    float F = fresnel_dielectric(L, H, 1.0f / eta);
    v3 f = m.nonlinear ? m.albedo / (1.0f - m.albedo * Favg) : m.albedo / (1.0f - Favg);
    f *= (1.0f - Fi) * (1.0f - Fo) * kInvPi;
    f += m.specular * (v3(F) * D * G / (4.0f * NdotL * NdotV) + multiple_scatter(sc, NdotL, NdotV, m.rough, v3(Favg)));
    pdf = ps * Dv * fabsf(1.0f / (4.0f * dot(V, H))) + (1.0f - ps) * cosine_pdf(NdotL);
    return f;
}
RT_D float plastic_weight(const MatParams& m) {
    float d = m.albedo.x + m.albedo.y + m.albedo.z, s = m.specular.x + m.specular.y + m.specular.z;
    return s / (s + d);
}
// Metal workflow, Material.h:407-516 (shared tail)
RT_D v3 metal_f(const MatParams& m, v3 N, v3 V, v3 L, v3 H, float& pdf) {
    float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    float NdotV = dot(N, V), NdotL = dot(N, L);
    float diel = 1.0f - m.metallic, spec = m.metallic + diel, pdiff = diel / (diel + spec);
    float Dv = ggx_dv(V, H, N, au, av);
    float G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    float D = ggx_d(H, N, au, av);
    v3 F0 = v3(0.04f) * (1.0f - m.metallic) + m.albedo * m.metallic;
    float vdh = dot(V, H);
    float tmp = 1.0f - fminf(1.0f, fmaxf(0.0f, vdh));
    float tmp2 = tmp * tmp, Fc = tmp2 * tmp2 * tmp;
    v3 F = F0 + (1.0f - F0) * Fc;
    v3 sb = D * F * G / (4.0f * NdotL * NdotV);
    v3 db = m.albedo * kInvPi;
    pdf = (1.0f - pdiff) * Dv * fabsf(1.0f / (4.0f * vdh)) + pdiff * cosine_pdf(NdotL);
    return pdiff * db + (1.0f - pdiff) * sb;
}
RT_D float thin_fresnel(v3 V, v3 H, float eta) {  // Material.h:548-551
    float F = fresnel_dielectric(V, H, 1.0f / eta);
    if (F < 1.0f) F *= 2.0f / (1.0f + F);
    return F;
}
// Clear-coated conductor coat term, Material.h:634-734
RT_D v3 clearcoat_mix(const SceneView& sc, const MatParams& m, v3 N, v3 V, v3 L, v3 H, v3 cond, float cpdf,
                      float& pdf) {
    float au = sqr(m.cru), av = sqr(m.crv);
    float NdotV = dot(N, V), NdotL = dot(N, L);
    float Dv = ggx_dv(V, H, N, au, av);
    float F = fresnel_dielectric(V, H, 1.0f / 1.5f);
    float cw = m.coat_weight * F;
    float G = smith_g1(V, H, N, au, av) * smith_g1(L, H, N, au, av);
    float D = ggx_d(H, N, au, av);
    float coat_pdf = Dv * fabsf(1.0f / (4.0f * dot(V, H)));
    v3 coat(D * G / (4.0f * NdotV * NdotL));
    pdf = cw * coat_pdf + (1.0f - cw) * cpdf;
    return cw * coat + (1.0f - cw) * cond;
}

// EvaluateMaterial, Material.h:783-813
RT_D v3 eval_material(const SceneView& sc, const Surf& s, v3 V, v3 L, float& pdf) {
    pdf = 0.0f;
    if (!s.mat) return v3(0.0f);
    const MatParams m = load_material(s.mat);
    const v3 N = s.sn;
    switch (m.type) {
        case RT_MAT_DIFFUSE: {
            v3 lL = to_local(L, N);
            return diffuse_f(m, N, V, L, lL.z, pdf);
        }
        case RT_MAT_CONDUCTOR: return conductor_f(sc, m, N, V, L, normalize(V + L), pdf);
        case RT_MAT_DIELECTRIC: {
            float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
            float eta = m.int_ior / m.ext_ior;
            float e = s.front ? (1.0f / eta) : eta;
            bool refl = dot(N, L) * dot(N, V) > 0.0f;
            v3 H;
            if (refl) {
                H = normalize(V + L);
            } else {
                H = -normalize(e * V + L);
                if (dot(N, H) < 0.0f) H = -H;
            }
            float Dv = ggx_dv(V, H, N, au, av);
            pdf = Dv * fabsf(1.0f / (4.0f * dot(V, H)));
            float F = fresnel_dielectric(V, H, e);
            float D = ggx_d(H, N, au, av);
            return dielectric_f(m, N, V, L, H, e, refl, Dv, F, D, au, av, pdf);
        }
        case RT_MAT_PLASTIC: {
            float eta = m.int_ior / m.ext_ior;
            v3 H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return v3(0.0f);
            float Fo = fresnel_dielectric(V, N, 1.0f / eta), Fi = fresnel_dielectric(L, N, 1.0f / eta);
            float w = plastic_weight(m);
            float ps = Fi * w, pd = (1.0f - Fi) * (1.0f - w);
            ps = ps / (ps + pd);
            return plastic_f(sc, m, N, V, L, H, Fo, Fi, ps, pdf);
        }
        case RT_MAT_METAL_WORKFLOW: {
            v3 H = normalize(L + V);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return v3(0.0f);
            return metal_f(m, N, V, L, H, pdf);
        }
        case RT_MAT_THIN_DIELECTRIC: {
            float eta = m.int_ior / m.ext_ior, a = sqr(m.rough);
            bool refl = dot(N, L) * dot(N, V) > 0.0f;
            v3 H;
            if (refl) {
                H = normalize(V + L);
            } else {
                v3 Vr = to_world(to_local(V, -N), N);
                H = normalize(Vr + L);
                if (dot(N, H) < 0.0f) H = -H;
            }
            float Dv = ggx_dv(V, H, N, a, a);
            float F = thin_fresnel(V, H, eta);
            float D = ggx_d(H, N, a, a);
            float dwh = fabsf(1.0f / (4.0f * dot(V, H)));
            float NdotV = fabsf(dot(N, V)), NdotL = fabsf(dot(N, L));
            float G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
            if (refl) {
                if (dot(N, L) <= 0.0f) return v3(0.0f);
                pdf = F * Dv * dwh;
                return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
            }
            if (dot(N, L) * dot(N, V) >= 0.0f) return v3(0.0f);
            pdf = (1.0f - F) * Dv * dwh;
            return m.albedo * (1.0f - F) * D * G / (4.0f * NdotV * NdotL);
        }
        case RT_MAT_CLEARCOATED_CONDUCTOR: {
            v3 H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return v3(0.0f);
            float cpdf = 0.0f;
            v3 cond = conductor_f(sc, m, N, V, L, H, cpdf);
            return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
        }
        case RT_MAT_DIFFUSE_TRANSMITTER: {
            v3 Nn = -N;
            v3 lL = to_local(L, Nn);
            float NdotL = lL.z, NdotV = dot(Nn, V);
            if (NdotL * NdotV >= 0.0f) return v3(0.0f);
            pdf = cosine_pdf(fabsf(NdotL));
            return m.albedo * kInvPi;
        }
    }
    return v3(0.0f);
}

// SampleMaterial, Material.h:815-845
template <class RNG>
RT_D v3 sample_material(const SceneView& sc, const Surf& s, RNG& rng, v3 V, v3& L, float& pdf) {
    pdf = 0.0f;
    if (!s.mat) return v3(0.0f);
    const MatParams m = load_material(s.mat);
    const v3 N = s.sn;
    float au = sqr(m.rough) * (1.0f + m.aniso), av = sqr(m.rough) * (1.0f - m.aniso);
    switch (m.type) {
        case RT_MAT_DIFFUSE: {
            float u0 = rng.next(), u1 = rng.next();
            v3 lL = cosine_sample_hemisphere(u0, u1);
            L = to_world(lL, N);
            return diffuse_f(m, N, V, L, lL.z, pdf);
        }
        case RT_MAT_CONDUCTOR: {
            float u0 = rng.next(), u1 = rng.next();
            v3 H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            L = reflect(-V, H);
            return conductor_f(sc, m, N, V, L, H, pdf);
        }
        case RT_MAT_DIELECTRIC: {
            float eta = m.int_ior / m.ext_ior;
            float e = s.front ? (1.0f / eta) : eta;
            float u0 = rng.next(), u1 = rng.next();
            v3 H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            float Dv = ggx_dv(V, H, N, au, av);
            float F = fresnel_dielectric(V, H, e);
            float D = ggx_d(H, N, au, av);
            if (rng.next() < F) {
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
                return dielectric_f(m, N, V, L, H, e, true, Dv, F, D, au, av, pdf);
            }
            L = refract(-V, H, e);
            if (dot(N, L) * dot(N, V) >= 0.0f) return v3(0.0f);
            return dielectric_f(m, N, V, L, H, e, false, Dv, F, D, au, av, pdf);
        }
        case RT_MAT_PLASTIC: {
            float eta = m.int_ior / m.ext_ior;
            if (dot(N, V) <= 0.0f) return v3(0.0f);
            float Fo = fresnel_dielectric(V, N, 1.0f / eta), Fi = Fo;
            float w = plastic_weight(m);
            float ps = Fi * w, pd = (1.0f - Fi) * (1.0f - w);
            ps = ps / (ps + pd);
            v3 H;
            if (rng.next() < ps) {
                float u0 = rng.next(), u1 = rng.next();
                H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
            } else {
                float u0 = rng.next(), u1 = rng.next();
                L = to_world(cosine_sample_hemisphere(u0, u1), N);
                H = normalize(V + L);
                Fi = fresnel_dielectric(L, N, 1.0f / eta);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
            }
            return plastic_f(sc, m, N, V, L, H, Fo, Fi, ps, pdf);
        }
        case RT_MAT_METAL_WORKFLOW: {
            if (dot(N, V) <= 0.0f) return v3(0.0f);
            float diel = 1.0f - m.metallic, spec = m.metallic + diel, pdiff = diel / (diel + spec);
            v3 H;
            if (rng.next() < pdiff) {
                float u0 = rng.next(), u1 = rng.next();
                L = to_world(cosine_sample_hemisphere(u0, u1), N);
                H = normalize(V + L);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
            } else {
                float u0 = rng.next(), u1 = rng.next();
                H = to_world(sample_vndf(N, V, au, av, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
            }
            return metal_f(m, N, V, L, H, pdf);
        }
        case RT_MAT_THIN_DIELECTRIC: {
            float eta = m.int_ior / m.ext_ior, a = sqr(m.rough);
            float u0 = rng.next(), u1 = rng.next();
            v3 H = to_world(sample_vndf(N, V, a, a, u0, u1), N);
            float Dv = ggx_dv(V, H, N, a, a);
            float F = thin_fresnel(V, H, eta);
            float D = ggx_d(H, N, a, a);
            float dwh = fabsf(1.0f / (4.0f * dot(V, H)));
            if (rng.next() < F) {
                L = reflect(-V, H);
                if (dot(N, L) <= 0.0f) return v3(0.0f);
                float NdotV = fabsf(dot(N, V)), NdotL = fabsf(dot(N, L));
                float G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
                pdf = F * Dv * dwh;
                return m.albedo * F * D * G / (4.0f * NdotV * NdotL);
            }
            L = -V;
            if (dot(N, L) * dot(N, V) >= 0.0f) return v3(0.0f);
            float NdotV = fabsf(dot(N, V)), NdotL = fabsf(dot(N, L));
            float G = smith_g1(V, H, N, a, a) * smith_g1(L, H, N, a, a);
            pdf = (1.0f - F) * Dv * dwh;
            return m.albedo * (1.0f - F) * D * G / (4.0f * NdotV * NdotL);
        }
        case RT_MAT_CLEARCOATED_CONDUCTOR: {
            float cau = sqr(m.cru), cav = sqr(m.crv);
            float F = fresnel_dielectric(V, N, 1.0f / 1.5f);
            float cw = m.coat_weight * F;
            if (rng.next() < cw) {
                float u0 = rng.next(), u1 = rng.next();
                v3 H = to_world(sample_vndf(N, V, cau, cav, u0, u1), N);
                L = reflect(-V, H);
                if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return v3(0.0f);
                float cpdf = 0.0f;
                v3 cond = conductor_f(sc, m, N, V, L, normalize(V + L), cpdf);
                return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
            }
            float u0 = rng.next(), u1 = rng.next();
            v3 Hc = to_world(sample_vndf(N, V, au, av, u0, u1), N);
            L = reflect(-V, Hc);
            float cpdf = 0.0f;
            v3 cond = conductor_f(sc, m, N, V, L, Hc, cpdf);
            v3 H = normalize(V + L);
            if (dot(N, V) <= 0.0f || dot(N, L) <= 0.0f) return v3(0.0f);
            return clearcoat_mix(sc, m, N, V, L, H, cond, cpdf, pdf);
        }
        case RT_MAT_DIFFUSE_TRANSMITTER: {
            float u0 = rng.next(), u1 = rng.next();
            v3 lL = cosine_sample_hemisphere(u0, u1);
            v3 Nn = -N;
            L = to_world(lL, Nn);
            float NdotL = lL.z, NdotV = dot(Nn, V);
            if (NdotL * NdotV >= 0.0f) return v3(0.0f);
            pdf = cosine_pdf(fabsf(NdotL));
            return m.albedo * kInvPi;
        }
    }
    return v3(0.0f);
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
