// ref_pt.cpp - the reference renderer's CPU path: its own shading code
// (core/cuda/*.h, common/gdt) compiled for the host, driven by a restatement
// of __raygen__renderFrame (core/cuda/devicePrograms.cu:170-532) in an OpenMP
// per-pixel loop.  optixTrace is replaced by the oracle's FP32 watertight
// intersector over a binary BVH, and tex2D by bilinear filtering of the same
// float images.  Unlike the oracle this keeps the reference's NaN behaviour for
// zero-pdf light samples.
//
// TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py (kind
// "reference") and a statistical cross-check of the oracle.  Built by
// oracle/Makefile into oracle/_ref/ when the reference tree is present.
#include <cstring>
#include <omp.h>

#include "pt_oracle.hpp"  // before the reference headers: they define EPS as a macro

#include "Environment.h"
#include "Filter.h"
#include "Light.h"
#include "Material.h"
#include "Medium.h"

namespace {

struct RefScene {
    std::vector<float> tv, tn;
    std::vector<int> tri_mesh;
    std::vector<Material> mats;
    std::vector<int> mesh_in, mesh_out;
    std::vector<Light> lights;
    std::vector<Medium> media;
    std::vector<float> env, cache;
    int env_w = 0, env_h = 0;
    orc::Bvh2 bvh;
    float lut[kLutResolution * kLutResolution];
    float lut_avg[kLutResolution];
};

vec3f v3(const float* p) { return vec3f(p[0], p[1], p[2]); }

vec4f tex(const std::vector<float>& img, int w, int h, float u, float v) {
    float o[4];
    orc::tex_bilinear<float>(img.data(), w, h, u, v, o);
    return vec4f(o[0], o[1], o[2], o[3]);
}

// optixTrace with DISABLE_ANYHIT: closest hit in [EPS, tmax).
bool trace(const RefScene& s, const vec3f& o, const vec3f& d, float tmax, int& prim, float& u, float& v) {
    orc::HitInfo<float> h;
    orc::closest_hit<float>(s.bvh, s.tv.data(), orc::V3<float>(o.x, o.y, o.z), orc::V3<float>(d.x, d.y, d.z), 1e-4f, tmax,
                            h);
    prim = h.prim;
    u = h.b1;
    v = h.b2;
    return h.prim >= 0;
}
// optixTrace with TERMINATE_ON_FIRST_HIT: true if nothing blocks [EPS, tmax).
bool visible(const RefScene& s, const vec3f& o, const vec3f& d, float tmax) {
    if (!(tmax > 1e-4f)) return true;
    return !orc::any_hit<float>(s.bvh, s.tv.data(), orc::V3<float>(o.x, o.y, o.z), orc::V3<float>(d.x, d.y, d.z), 1e-4f,
                                tmax);
}

struct PRD {
    Random random;
    bool lightVisible;
    Interaction isect;
    vec3f pixelAlbedo;
    vec3f pixelNormal;
    bool firstBounce;
};

void closest_hit_program(const RefScene& s, PRD& prd, int prim, float u, float v, const vec3f& rayDir) {
    // __closesthit__radiance, devicePrograms.cu:71-132 (no textures)
    const float* n = &s.tn[size_t(prim) * 9];
    const float* p = &s.tv[size_t(prim) * 9];
    vec3f Ns = ((1.0f - u - v) * v3(n) + u * v3(n + 3) + v * v3(n + 6));
    Ns = normalize(Ns);
    int mesh = s.tri_mesh[size_t(prim)];
    const Material& material = s.mats[size_t(mesh)];
    const vec3f surfPos = (1.0f - u - v) * v3(p) + u * v3(p + 3) + v * v3(p + 6);
    prd.isect.SetFaceNormal(rayDir, Ns);
    prd.isect.distance = length(surfPos - prd.isect.position);
    prd.isect.position = surfPos;
    prd.isect.material = material;
    prd.isect.mi = MediumInterface(s.mesh_in[size_t(mesh)], s.mesh_out[size_t(mesh)]);
    if (prd.firstBounce) {
        prd.pixelNormal = Ns;
        prd.pixelAlbedo = material.albedo;
        prd.firstBounce = false;
    }
}

void render_pixel(const RefScene& s, const rt_options& opt, const float* cam, int cam_medium, int frame, int ix, int iy,
                  float* out) {
    const int W = opt.width, H = opt.height;
    const vec3f position = v3(cam), direction = v3(cam + 3), horizontal = v3(cam + 6), vertical = v3(cam + 9);
    const int lightSize = int(s.lights.size());
    const int mediumSize = int(s.media.size());
    const bool hasEnv = s.env_w > 0;
    PRD prd;
    prd.random.init(ix + W * iy, frame);
    vec3f pixelColor = 0.0f;
    auto lightTrace = [&](const Ray& ray, Interaction& isect, vec3f& light_radiance, float& light_pdf,
                          float& closest_distance) -> bool {
        bool hitLight = false;
        for (int i = 0; i < lightSize; i++) {
            const Light& light = s.lights[size_t(i)];
            float light_distance = 0.0f;
            vec3f Li = EvaluateLight(light, ray, closest_distance, light_pdf, light_distance);
            if (light_pdf == 0.0f) continue;
            hitLight = true;
            light_radiance = Li;
            closest_distance = light_distance;
            isect.mi = MediumInterface(light.medium);
        }
        return hitLight;
    };
    for (int sampleID = 0; sampleID < opt.spp; sampleID++) {
        float r0 = prd.random(), r1 = prd.random();
        vec2f jitter = FilterJitter(vec2f(r0, r1), FilterType(opt.filter));
        vec2f screen(vec2f(ix + 0.5f + jitter.x, iy + 0.5f + jitter.y) / vec2f(float(W), float(H)));
        vec3f rayDir = normalize(direction + (screen.x - 0.5f) * horizontal + (screen.y - 0.5f) * vertical);
        Ray ray;
        ray.origin = position;
        ray.direction = rayDir;
        vec3f radiance(0.0f), history(1.0f), V = -ray.direction, L = ray.direction;
        float light_pdf = 0.0f, bsdf_pdf = 0.0f, phase_pdf = 0.0f;
        vec3f bsdf = 0.0f, attenuation = 0.0f, light_radiance = 0.0f;
        float closest_distance = FLT_MAX;
        vec3f pre_position = position;
        float pre_pdf = 0.0f, mult_trans_pdf = 1.0f, trans_pdf = 1.0f;
        vec3f transmittance = 0.0f;
        prd.isect.distance = FLT_MAX;
        prd.isect.position = ray.origin;
        prd.firstBounce = true;
        prd.isect.mi = MediumInterface(cam_medium);
        for (int bounce = 0; bounce < opt.max_depth; bounce++) {
            int prim;
            float bu, bv;
            if (trace(s, ray.origin, ray.direction, FLT_MAX, prim, bu, bv)) {
                closest_hit_program(s, prd, prim, bu, bv, ray.direction);
            } else {  // __miss__radiance, devicePrograms.cu:148-159
                prd.isect.distance = FLT_MAX;
                prd.isect.mi = MediumInterface(cam_medium);
                prd.isect.frontFace = true;
                if (prd.firstBounce) prd.firstBounce = false;
            }
            closest_distance = prd.isect.distance;
            bool hitLight = lightTrace(ray, prd.isect, light_radiance, light_pdf, closest_distance);
            bool scattered = false;
            int medium_index = -1;
            if (mediumSize != 0) {
                medium_index = prd.isect.mi.GetMedium(hitLight ? true : prd.isect.frontFace);
                float distance = 0.0f;
                if (medium_index != -1) {
                    const Medium& medium = s.media[size_t(medium_index)];
                    scattered = SampleMediumDistance(medium, closest_distance, distance, trans_pdf, transmittance, prd.random);
                    history *= (transmittance / trans_pdf);
                    mult_trans_pdf *= trans_pdf;
                    if (scattered) {
                        prd.isect.position = pre_position + distance * L;
                        prd.isect.distance = distance;
                        if (lightSize != 0) {
                            int index = clamp(int(lightSize * prd.random()), 0, lightSize - 1);
                            const Light& light = s.lights[size_t(index)];
                            float light_distance = 0.0f;
                            Ray shadowRay;
                            shadowRay.origin = prd.isect.position;
                            float s0 = prd.random(), s1 = prd.random();
                            light_radiance = SampleLight(light, shadowRay.origin, vec2f(s0, s1), shadowRay.direction,
                                                         light_distance, light_pdf);
                            light_pdf *= (1.0f / (float)lightSize);
                            prd.lightVisible = visible(s, shadowRay.origin, shadowRay.direction, light_distance - 1e-4f);
                            vec3f tv;
                            float t;
                            Interaction ti;
                            closest_distance = light_distance - 1e-4f;
                            if (!lightTrace(shadowRay, ti, tv, t, closest_distance) && prd.lightVisible) {
                                transmittance = EvaluateMediumDistance(medium, false, closest_distance, trans_pdf);
                                attenuation = EvaluatePhase(medium, prd.isect, V, shadowRay.direction, phase_pdf);
                                float misWeight = PowerHeuristic(light_pdf, phase_pdf * trans_pdf, 2);
                                radiance += misWeight * (transmittance / trans_pdf) * light_radiance * attenuation * history / light_pdf;
                            }
                        }
                        attenuation = SamplePhase(medium, prd.isect, prd.random, V, L, phase_pdf);
                        history *= (attenuation / phase_pdf);
                        pre_pdf = phase_pdf;
                    }
                }
            }
            if (!scattered) {
                if (hitLight) {
                    float misWeight = 1.0f;
                    if (bounce != 0) {
                        pre_pdf *= mult_trans_pdf;
                        misWeight = PowerHeuristic(pre_pdf, light_pdf, 2);
                    }
                    radiance += misWeight * history * light_radiance;
                    break;
                }
                bool notHit = closest_distance == FLT_MAX;
                if (notHit && medium_index == -1) {
                    if (hasEnv) {
                        vec2f uv = EvaluateEnvironment(s.env_w, s.env_h, light_pdf, ray.direction);
                        light_radiance = vec3f(tex(s.env, s.env_w, s.env_h, uv.x, uv.y));
                        light_pdf *= tex(s.cache, s.env_w, s.env_h, uv.x, uv.y).z;
                        float misWeight = 1.0f;
                        if (bounce != 0) {
                            pre_pdf *= mult_trans_pdf;
                            misWeight = PowerHeuristic(pre_pdf, light_pdf, 2);
                        }
                        radiance += misWeight * history * light_radiance;
                    }
                    break;
                }
                if (hasEnv) {
                    float e0 = prd.random(), e1 = prd.random();
                    vec4f uv_t = tex(s.cache, s.env_w, s.env_h, e0, e1);
                    vec2f uv(uv_t.x, uv_t.y);
                    Ray shadowRay;
                    shadowRay.origin = prd.isect.position;
                    SampleEnvironment(s.env_w, s.env_h, light_pdf, shadowRay.direction, uv);
                    light_pdf *= tex(s.cache, s.env_w, s.env_h, uv.x, uv.y).z;
                    light_radiance = vec3f(tex(s.env, s.env_w, s.env_h, uv.x, uv.y));
                    prd.lightVisible = visible(s, shadowRay.origin, shadowRay.direction, FLT_MAX);
                    vec3f tv;
                    float t;
                    Interaction ti;
                    closest_distance = FLT_MAX;
                    if (!lightTrace(shadowRay, ti, tv, t, closest_distance) && prd.lightVisible) {
                        bsdf = EvaluateMaterial(prd.isect, V, shadowRay.direction, bsdf_pdf);
                        float costheta = abs(dot(prd.isect.shadeNormal, shadowRay.direction));
                        float misWeight = PowerHeuristic(light_pdf, bsdf_pdf, 2);
                        vec3f t_history = 1.0f;
                        if (medium_index != -1) {
                            const Medium& medium = s.media[size_t(medium_index)];
                            transmittance = EvaluateMediumDistance(medium, false, closest_distance, trans_pdf);
                            t_history = (transmittance / trans_pdf);
                            misWeight = PowerHeuristic(light_pdf, bsdf_pdf * trans_pdf, 2);
                        }
                        radiance += misWeight * t_history * light_radiance * bsdf * costheta * history / light_pdf;
                    }
                }
                if (lightSize != 0) {
                    int index = clamp(int(lightSize * prd.random()), 0, lightSize - 1);
                    const Light& light = s.lights[size_t(index)];
                    float light_distance = 0.0f;
                    Ray shadowRay;
                    shadowRay.origin = prd.isect.position;
                    float s0 = prd.random(), s1 = prd.random();
                    light_radiance = SampleLight(light, shadowRay.origin, vec2f(s0, s1), shadowRay.direction, light_distance,
                                                 light_pdf);
                    light_pdf *= (1.0f / (float)lightSize);
                    prd.lightVisible = visible(s, shadowRay.origin, shadowRay.direction, light_distance - 1e-4f);
                    vec3f tv;
                    float t;
                    Interaction ti;
                    closest_distance = light_distance - 1e-4f;
                    if (!lightTrace(shadowRay, ti, tv, t, closest_distance) && prd.lightVisible) {
                        bsdf = EvaluateMaterial(prd.isect, V, shadowRay.direction, bsdf_pdf);
                        float costheta = abs(dot(prd.isect.shadeNormal, shadowRay.direction));
                        float misWeight = PowerHeuristic(light_pdf, bsdf_pdf, 2);
                        vec3f t_history = 1.0f;
                        if (medium_index != -1) {
                            const Medium& medium = s.media[size_t(medium_index)];
                            transmittance = EvaluateMediumDistance(medium, false, closest_distance, trans_pdf);
                            t_history = (transmittance / trans_pdf);
                            misWeight = PowerHeuristic(light_pdf, bsdf_pdf * trans_pdf, 2);
                        }
                        radiance += misWeight * t_history * light_radiance * bsdf * costheta * history / light_pdf;
                    }
                }
                bsdf = SampleMaterial(prd.isect, prd.random, V, L, bsdf_pdf);
                float costheta = abs(dot(prd.isect.shadeNormal, L));
                history *= (bsdf * costheta / bsdf_pdf);
                pre_pdf = bsdf_pdf;
            }
            if (bounce >= opt.rr_depth) {
                float prr = min((history.x + history.y + history.z) / 3.0f, 0.95f);
                if (prd.random() > prr) break;
                history /= prr;
            }
            if (IsNan(history)) break;
            V = -L;
            ray.origin = prd.isect.position;
            ray.direction = L;
            mult_trans_pdf = 1.0f;
            pre_position = prd.isect.position;
        }
        if (IsNan(radiance)) break;
        pixelColor += radiance;
    }
    out[0] = pixelColor.x / opt.spp;
    out[1] = pixelColor.y / opt.spp;
    out[2] = pixelColor.z / opt.spp;
    out[3] = 1.0f;
}

}  // namespace

extern "C" {

void* refpt_scene_new(const float* tri_v, const int32_t* tri_mesh, int64_t ntri, const rt_material* mats,
                      const int32_t* mesh_media, int32_t n_mesh, const rt_light* lights, int32_t nl,
                      const rt_medium* media, int32_t nm, const float* env, int32_t ew, int32_t eh) {
    RefScene* s = new RefScene();
    s->tv.assign(tri_v, tri_v + ntri * 9);
    s->tn.resize(size_t(ntri) * 9);
    for (int64_t i = 0; i < ntri; i++) {  // face normals, Scene.cpp:150-158
        const float* p = tri_v + i * 9;
        vec3f n = normalize(cross(normalize(v3(p + 3) - v3(p)), normalize(v3(p + 6) - v3(p))));
        for (int k = 0; k < 3; k++) {
            s->tn[size_t(i) * 9 + k * 3 + 0] = n.x;
            s->tn[size_t(i) * 9 + k * 3 + 1] = n.y;
            s->tn[size_t(i) * 9 + k * 3 + 2] = n.z;
        }
    }
    s->tri_mesh.assign(tri_mesh, tri_mesh + ntri);
    ComputeKullaConty(s->lut, s->lut_avg);
    for (int i = 0; i < n_mesh; i++) {
        const rt_material& m = mats[i];
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
        r.bsdf_avg_buffer = s->lut;
        r.albedo_avg_buffer = s->lut_avg;
        s->mats.push_back(r);
        s->mesh_out.push_back(mesh_media[2 * i]);
        s->mesh_in.push_back(mesh_media[2 * i + 1]);
    }
    for (int i = 0; i < nl; i++) {
        Light l;
        l.type = LightType(lights[i].type);
        l.doubleSide = lights[i].double_side != 0;
        l.radiance = v3(lights[i].radiance);
        l.position = v3(lights[i].position);
        l.u = v3(lights[i].u);
        l.v = v3(lights[i].v);
        l.radius = lights[i].radius;
        l.medium = lights[i].medium;
        s->lights.push_back(l);
    }
    for (int i = 0; i < nm; i++) {
        Medium m;
        m.type = MediumType(media[i].type);
        m.phase.type = PhaseType(media[i].phase);
        m.phase.g = v3(media[i].g);
        m.sigma_s = v3(media[i].sigma_s);
        m.sigma_a = v3(media[i].sigma_a);
        m.scale = media[i].scale;
        s->media.push_back(m);
    }
    if (env && ew > 0 && eh > 0) {
        s->env.assign(env, env + size_t(ew) * eh * 4);
        s->cache.resize(s->env.size());
        orc::env_cache(s->env.data(), ew, eh, s->cache.data());
        s->env_w = ew;
        s->env_h = eh;
    }
    s->bvh.build(s->tv.data(), ntri);
    return s;
}

void refpt_scene_free(void* p) { delete static_cast<RefScene*>(p); }

// The reference's own default-constructed Material, Light and Medium
// (core/include/Scene.h:48-155) as the C ABI structs, so the benchmark's
// reference arm builds its scene without the product library.
void refpt_material_default(rt_material* out) {
    Material r{};  // value-initialised: fields without an initialiser are zero
    std::memset(out, 0, sizeof(*out));
    out->type = int32_t(r.type);
    for (int a = 0; a < 3; a++) {
        out->albedo[a] = r.albedo[a];
        out->eta[a] = r.eta[a];
        out->k[a] = r.k[a];
        out->specular[a] = r.specular[a];
    }
    out->roughness = r.roughness;
    out->anisotropy = r.anisotropy;
    out->int_ior = r.int_ior;
    out->ext_ior = r.ext_ior;
    out->nonlinear = r.nonlinear ? 1 : 0;
    out->metallic = r.metallic;
    out->coat_weight = r.coat_weight;
    out->coat_roughness_u = r.coat_roughness_u;
    out->coat_roughness_v = r.coat_roughness_v;
    const int ids[8] = {r.albedoTextureID, r.roughnessTextureID, r.anisotropyTextureID, r.specularTextureID,
                        r.metallicTextureID, r.coat_roughness_uTextureID, r.coat_roughness_vTextureID,
                        r.normalTextureID};
    for (int t = 0; t < 8; t++) out->texture_ids[t] = ids[t];
}

void refpt_light_default(rt_light* out) {
    Light r{};
    std::memset(out, 0, sizeof(*out));
    out->type = int32_t(r.type);
    out->double_side = r.doubleSide ? 1 : 0;
    for (int a = 0; a < 3; a++) {
        out->radiance[a] = r.radiance[a];
        out->position[a] = r.position[a];
        out->u[a] = r.u[a];
        out->v[a] = r.v[a];
    }
    out->radius = r.radius;
    out->medium = r.medium;
}

void refpt_medium_default(rt_medium* out) {
    Medium r{};
    std::memset(out, 0, sizeof(*out));
    out->type = int32_t(r.type);
    out->phase = int32_t(r.phase.type);
    for (int a = 0; a < 3; a++) {
        out->g[a] = 0.0f;  // Phase::g is left indeterminate by the reference (vec3f's empty constructor)
        out->sigma_s[a] = r.sigma_s[a];
        out->sigma_a[a] = r.sigma_a[a];
    }
    out->scale = r.scale;
}

// One launch (numPixelSamples = opts->spp) of rows [row0, row1) into color
// (w*h*4 floats); cam = position, direction, horizontal, vertical.
int refpt_render(void* p, const rt_options* opt, const float* cam, int32_t cam_medium, int32_t frame, float* color,
                 int32_t nthreads, int32_t row0, int32_t row1) {
    const RefScene* s = static_cast<const RefScene*>(p);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if (row1 <= row0) {
        row0 = 0;
        row1 = opt->height;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int iy = row0; iy < row1; iy++)
        for (int ix = 0; ix < opt->width; ix++)
            render_pixel(*s, *opt, cam, cam_medium, frame, ix, iy, color + (size_t(iy) * opt->width + ix) * 4);
    return 0;
}

}  // extern "C"
