// ref_driver.cpp - extern "C" access to the reference renderer's own shading
// code, compiled for the host from the reference sources where they lie.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ when
// the reference tree is present; used by the CPU tests to pin the oracle
// restatement (oracle/pt_oracle.hpp) to the reference's functions.  The random
// generator type the reference uses (gdt::LCG<16>, aliased as Random in
// core/cuda/Utils.h:8) is specialised here to read a caller-supplied list, so
// every sampling routine can be fed explicit numbers.  g++ evaluates the two
// arguments of `vec2f(random(), random())` right to left; callers that compare
// against a left-to-right consumer swap each such pair.
#include "gdt/random/random.h"

namespace gdt {
template <>
struct LCG<16> {
    const float* list = nullptr;
    int n = 0;
    int used = 0;
    inline float operator()() {
        used++;
        return (used - 1) < n ? list[used - 1] : 0.5f;
    }
};
}  // namespace gdt

#include "Environment.h"
#include "Filter.h"
#include "Light.h"
#include "Material.h"
#include "Medium.h"

#include "../../include/rt_capi.h"

namespace {

vec3f v3(const float* p) { return vec3f(p[0], p[1], p[2]); }

float g_lut[kLutResolution * kLutResolution];
float g_avg[kLutResolution];
bool g_lut_ready = false;

Material to_ref(const rt_material& m) {
    Material r;
    r.type = MaterialType(m.type);
    r.albedo = v3(m.albedo);
    r.roughness = m.roughness;
    r.anisotropy = m.anisotropy;
    r.eta = v3(m.eta);
    r.k = v3(m.k);
    r.int_ior = m.int_ior;
    r.ext_ior = m.ext_ior;
    r.nonlinear = m.nonlinear != 0;
    r.specular = v3(m.specular);
    r.metallic = m.metallic;
    r.coat_weight = m.coat_weight;
    r.coat_roughness_u = m.coat_roughness_u;
    r.coat_roughness_v = m.coat_roughness_v;
    r.bsdf_avg_buffer = g_lut;
    r.albedo_avg_buffer = g_avg;
    return r;
}

Light to_ref(const rt_light& l) {
    Light r;
    r.type = LightType(l.type);
    r.doubleSide = l.double_side != 0;
    r.radiance = v3(l.radiance);
    r.position = v3(l.position);
    r.u = v3(l.u);
    r.v = v3(l.v);
    r.radius = l.radius;
    r.medium = l.medium;
    return r;
}

Medium to_ref(const rt_medium& m) {
    Medium r;
    r.type = MediumType(m.type);
    r.phase.type = PhaseType(m.phase);
    r.phase.g = v3(m.g);
    r.sigma_s = v3(m.sigma_s);
    r.sigma_a = v3(m.sigma_a);
    r.scale = m.scale;
    return r;
}

}  // namespace

extern "C" {

// ComputeKullaConty, core/cuda/Microfacet.h:231-291.
void ref_kulla_conty(float* bsdf, float* avg) {
    if (!g_lut_ready) {
        ComputeKullaConty(g_lut, g_avg);
        g_lut_ready = true;
    }
    for (int i = 0; i < kLutResolution * kLutResolution; i++) bsdf[i] = g_lut[i];
    for (int i = 0; i < kLutResolution; i++) avg[i] = g_avg[i];
}

// The shading ops of rt_verify_shading (include/rt_capi.h), evaluated by the
// reference's own functions.
int ref_shading(int32_t op, const rt_material* mats, int32_t nmat, const rt_light* lights, int32_t nl,
                const rt_medium* media, int32_t nm, const float* in, int64_t n, float* out) {
    if (!g_lut_ready) {
        ComputeKullaConty(g_lut, g_avg);
        g_lut_ready = true;
    }
    for (int64_t q = 0; q < n; q++) {
        const float* x = in + q * 16;
        float* y = out + q * 8;
        for (int k = 0; k < 8; k++) y[k] = 0.0f;
        Random rng;
        if (op == RT_VERIFY_BSDF_EVAL || op == RT_VERIFY_BSDF_SAMPLE) {
            Interaction it;
            it.shadeNormal = v3(x);
            bool sample = op == RT_VERIFY_BSDF_SAMPLE;
            it.frontFace = (sample ? x[12] : x[9]) != 0.0f;
            int mi = int(sample ? x[13] : x[10]);
            if (mi < 0 || mi >= nmat) return 1;
            it.material = to_ref(mats[mi]);
            vec3f V = v3(x + 3);
            float pdf = 0.0f;
            vec3f f;
            if (!sample) {
                f = EvaluateMaterial(it, V, v3(x + 6), pdf);
            } else {
                rng.list = x + 6;
                rng.n = 6;
                vec3f L(0.0f);
                f = SampleMaterial(it, rng, V, L, pdf);
                y[4] = L.x;
                y[5] = L.y;
                y[6] = L.z;
                y[7] = float(rng.used);
            }
            y[0] = f.x;
            y[1] = f.y;
            y[2] = f.z;
            y[3] = pdf;
        } else if (op == RT_VERIFY_LIGHT_SAMPLE) {
            Light l = to_ref(lights[int(x[5])]);
            vec3f L(0.0f);
            float dist = 0.0f, pdf = 0.0f;
            vec3f Li = SampleLight(l, v3(x), vec2f(x[3], x[4]), L, dist, pdf);
            y[0] = Li.x; y[1] = Li.y; y[2] = Li.z; y[3] = pdf;
            y[4] = L.x; y[5] = L.y; y[6] = L.z; y[7] = dist;
        } else if (op == RT_VERIFY_LIGHT_EVAL) {
            Light l = to_ref(lights[int(x[7])]);
            Ray ray;
            ray.origin = v3(x);
            ray.direction = v3(x + 3);
            float pdf = 0.0f, ld = 0.0f;
            vec3f Li = EvaluateLight(l, ray, x[6], pdf, ld);
            y[0] = Li.x; y[1] = Li.y; y[2] = Li.z; y[3] = pdf; y[4] = ld;
        } else if (op == RT_VERIFY_MEDIUM_SAMPLE) {
            Medium m = to_ref(media[int(x[3])]);
            rng.list = x + 1;
            rng.n = 2;
            float dist = 0.0f, tp = 0.0f;
            vec3f tr(0.0f);
            bool s = SampleMediumDistance(m, x[0], dist, tp, tr, rng);
            y[0] = tr.x; y[1] = tr.y; y[2] = tr.z; y[3] = tp; y[4] = dist; y[5] = s ? 1.0f : 0.0f;
            y[6] = float(rng.used);
        } else if (op == RT_VERIFY_PHASE_SAMPLE) {
            Medium m = to_ref(media[int(x[7])]);
            rng.list = x + 3;
            rng.n = 4;
            Interaction it;
            vec3f L(0.0f);
            float pdf = 0.0f;
            vec3f a = SamplePhase(m, it, rng, v3(x), L, pdf);
            y[0] = a.x; y[1] = a.y; y[2] = a.z; y[3] = pdf;
            y[4] = L.x; y[5] = L.y; y[6] = L.z; y[7] = float(rng.used);
        } else if (op == RT_VERIFY_PHASE_EVAL) {
            Medium m = to_ref(media[int(x[6])]);
            Interaction it;
            float pdf = 0.0f;
            vec3f a = EvaluatePhase(m, it, v3(x), v3(x + 3), pdf);
            y[0] = a.x; y[1] = a.y; y[2] = a.z; y[3] = pdf;
        }
    }
    return 0;
}

// FilterJitter, core/cuda/Filter.h:45-56: n x 2 samples in, n x 2 jitters out.
void ref_filter(int32_t type, const float* in, int64_t n, float* out) {
    for (int64_t i = 0; i < n; i++) {
        vec2f j = FilterJitter(vec2f(in[2 * i], in[2 * i + 1]), FilterType(type));
        out[2 * i] = j.x;
        out[2 * i + 1] = j.y;
    }
}

// SphereToPlane / PlaneToSphere, core/cuda/Sampling.h:12-33.
void ref_sphere_plane(const float* dirs, int64_t n, float* uv, float* back) {
    for (int64_t i = 0; i < n; i++) {
        vec2f p = SphereToPlane(v3(dirs + 3 * i));
        uv[2 * i] = p.x;
        uv[2 * i + 1] = p.y;
        vec3f d = PlaneToSphere(p);
        back[3 * i] = d.x;
        back[3 * i + 1] = d.y;
        back[3 * i + 2] = d.z;
    }
}

// The +-pair evaluation order of this compiler: 1 if `vec2f(random(), random())`
// takes its x from the second call.
int ref_pair_order_reversed(void) {
    Random r;
    float list[2] = {0.25f, 0.75f};
    r.list = list;
    r.n = 2;
    vec2f p(r(), r());
    return p.x == 0.75f ? 1 : 0;
}

}  // extern "C"
