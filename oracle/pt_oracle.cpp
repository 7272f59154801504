// pt_oracle.cpp - extern "C" entry points of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, by __graft_entry__.smoke() and by
// bench.py's CPU-baseline leg, always as the checker.  The integrator below
// restates __raygen__renderFrame, __closesthit__radiance and the miss programs
// of the reference (core/cuda/devicePrograms.cu:71-165 and :170-532), the
// camera of Renderer::SetCamera (core/src/Renderer.cpp:796-813) and the
// tonemap of core/cuda/PostProcessing.cu:18-48, with an OpenMP loop over
// pixels standing in for optixLaunch.
#include <cstring>
#include <omp.h>

#include <memory>

#include "pt_oracle.hpp"

using namespace orc;

namespace {

template <class R>
struct Scene {
    const float* tv = nullptr;
    const float* tn = nullptr;
    const float* tuv = nullptr;
    const uint32_t* tex = nullptr;      // all textures' texels
    const int32_t* tex_info = nullptr;  // offset, width, height per texture
    const int32_t* tri_mesh = nullptr;
    int64_t ntri = 0;
    std::vector<Mat<R>> mats;
    std::vector<int> mesh_in, mesh_out;
    std::vector<Lt<R>> lights;
    std::vector<Med<R>> media;
    std::vector<Grid<R>> grids;
    const float* env = nullptr;
    const float* cache = nullptr;
    int env_w = 0, env_h = 0;
    const Bvh2* bvh = nullptr;
    const float* lut = nullptr;
    const float* lut_avg = nullptr;
};

struct SceneHandle {
    std::vector<float> tv, tn, tuv;
    std::vector<uint32_t> tex;
    std::vector<int32_t> tex_info;
    std::vector<int32_t> tri_mesh;
    int64_t ntri = 0;
    std::vector<rt_material> mats;
    std::vector<int32_t> mesh_media;
    std::vector<rt_light> lights;
    std::vector<rt_medium> media;
    std::vector<std::vector<float>> dens, maj;
    std::vector<float> env, cache;
    int env_w = 0, env_h = 0;
    Bvh2 bvh;
    float lut[kLut * kLut];
    float lut_avg[kLut];
    std::unique_ptr<Scene<float>> sf;
    std::unique_ptr<Scene<double>> sd;
};

template <class R>
Scene<R>* make_scene(SceneHandle* h) {
    Scene<R>* s = new Scene<R>();
    s->ntri = h->ntri;
    s->mats.resize(h->mats.size());
    for (size_t i = 0; i < h->mats.size(); i++) s->mats[i].set(h->mats[i]);
    for (size_t i = 0; i < h->mats.size(); i++) {
        s->mesh_out.push_back(h->mesh_media[2 * i + 0]);
        s->mesh_in.push_back(h->mesh_media[2 * i + 1]);
    }
    s->lights.resize(h->lights.size());
    for (size_t i = 0; i < h->lights.size(); i++) s->lights[i].set(h->lights[i]);
    s->media.resize(h->media.size());
    s->grids.resize(h->media.size());
    for (size_t i = 0; i < h->media.size(); i++) {
        const rt_medium& m = h->media[i];
        s->media[i].set(m);
        if (m.type != RT_MEDIUM_GRID) continue;
        Grid<R>& g = s->grids[i];
        g.bmin = from3<R>(m.bounds_min);
        g.bmax = from3<R>(m.bounds_max);
        for (int a = 0; a < 3; a++) g.res[a] = m.grid_res[a];
        g.mres = m.majorant_res > 0 ? m.majorant_res : 8;
        R mx = R(0);
        for (int c = 0; c < 3; c++) mx = dmax(mx, R(m.sigma_a[c]) + R(m.sigma_s[c]));
        g.sigma_t = mx * R(m.scale);
        V3<R> ss = from3<R>(m.sigma_s), st = from3<R>(m.sigma_a) + ss;
        for (int c = 0; c < 3; c++) g.albedo[c] = st[c] > R(0) ? ss[c] / st[c] : R(0);
        g.density = h->dens[i].data();
        g.majorant = h->maj[i].data();
        s->media[i].grid = &s->grids[i];
    }
    s->env_w = h->env_w;
    s->env_h = h->env_h;
    s->tv = h->tv.data();
    s->tn = h->tn.data();
    s->tuv = h->tuv.data();
    s->tex = h->tex.empty() ? nullptr : h->tex.data();
    s->tex_info = h->tex_info.empty() ? nullptr : h->tex_info.data();
    s->tri_mesh = h->tri_mesh.data();
    s->env = h->env.empty() ? nullptr : h->env.data();
    s->cache = h->cache.empty() ? nullptr : h->cache.data();
    s->bvh = &h->bvh;
    s->lut = h->lut;
    s->lut_avg = h->lut_avg;
    return s;
}

template <class R>
struct Cam {
    V3<R> pos, dir, hor, ver;
    int medium;
};

// lightTrace lambda, core/cuda/devicePrograms.cu:192-211
template <class R>
bool light_trace(const Scene<R>& sc, const V3<R>& o, const V3<R>& d, int* mi_in, int* mi_out, V3<R>& lrad, R& lpdf,
                 R& closest) {
    bool hit = false;
    for (size_t i = 0; i < sc.lights.size(); i++) {
        const Lt<R>& l = sc.lights[i];
        R ld = R(0);
        V3<R> Li = evaluate_light(l, o, d, closest, lpdf, ld);
        if (lpdf == R(0)) continue;
        hit = true;
        lrad = Li;
        closest = ld;
        if (mi_in) {
            *mi_in = l.medium;
            *mi_out = l.medium;
        }
    }
    return hit;
}

inline bool nee_pdf_ok(double p) { return p > 0.0 && std::isfinite(p); }

template <class R>
bool medium_sample(const Med<R>& m, const V3<R>& o, const V3<R>& d, R maxd, R& dist, R& tp, V3<R>& tr, Rng& rng) {
    if (m.type == RT_MEDIUM_GRID) {
        tp = R(1);
        return grid_sample_distance(*m.grid, o, d, maxd, rng, dist, tr);
    }
    return sample_medium_distance(m, maxd, dist, tp, tr, rng);
}
template <class R>
V3<R> medium_transmittance(const Med<R>& m, const V3<R>& o, const V3<R>& d, R dist, R& tp, Rng& rng) {
    if (m.type == RT_MEDIUM_GRID) {
        tp = R(1);
        return V3<R>(grid_transmittance(*m.grid, o, d, dist, rng));
    }
    return eval_medium_distance(m, false, dist, tp);
}

template <class R>
void trace_sample(const Scene<R>& sc, const float* tv, const float* tn, const Cam<R>& cam, const rt_options& opt,
                  const Lut<R>& lut, Rng& rng, const V3<R>& ray_dir, V3<R>& radiance, V3<R>& p_albedo, V3<R>& p_normal) {
    const R EPS = K<R>::EPS;
    const R FMAX = R(FLT_MAX);
    V3<R> o = cam.pos, d = ray_dir;
    radiance = V3<R>(R(0));
    V3<R> history(R(1));
    V3<R> V = -d, L = d;
    R light_pdf = R(0), bsdf_pdf = R(0), phase_pdf = R(0);
    V3<R> bsdf(R(0)), attenuation(R(0)), light_radiance(R(0));
    R closest = FMAX;
    V3<R> pre_position = cam.pos;
    R pre_pdf = R(0), mult_trans_pdf = R(1), trans_pdf = R(1);
    V3<R> transmittance(R(0));
    Isect<R> it;
    Mat<R> tex_mat;  // the textured copy of the last hit's material
    it.distance = FMAX;
    it.position = o;
    it.sn = V3<R>(R(0));
    it.front = true;
    it.mat = nullptr;
    it.in_medium = it.out_medium = cam.medium;
    bool first = true;
    const int nl = int(sc.lights.size());
    const bool has_env = sc.env_w > 0;
    const int ew = sc.env_w, eh = sc.env_h;
    const float* env = sc.env;
    const float* cache = sc.cache;

    for (int bounce = 0; bounce < opt.max_depth; bounce++) {
        // optixTrace radiance (devicePrograms.cu:258-269) + closest hit (:71-132) / miss (:148-159)
        HitInfo<R> h;
        closest_hit(*sc.bvh, tv, o, d, EPS, FMAX, h);
        if (h.prim >= 0) {
            int p = h.prim;
            R u = h.b1, v = h.b2;
            const float* nn = tn + size_t(p) * 9;
            const float* vv = tv + size_t(p) * 9;
            R w0 = R(1) - u - v;
            V3<R> Ns = normalize(w0 * from3<R>(nn) + u * from3<R>(nn + 3) + v * from3<R>(nn + 6));
            int mesh = sc.tri_mesh[size_t(p)];
            const Mat<R>* mat = &sc.mats[size_t(mesh)];
            if (mat->textured) {  // texture overrides, devicePrograms.cu:89-115
                const float* uv = sc.tuv + size_t(p) * 6;
                R tcx = w0 * R(uv[0]) + u * R(uv[2]) + v * R(uv[4]);
                R tcy = w0 * R(uv[1]) + u * R(uv[3]) + v * R(uv[5]);
                tex_mat = *mat;
                R t4[4];
                auto fetch = [&](int slot) {
                    const int32_t* ti = sc.tex_info + 3 * mat->tex[slot];
                    tex_rgba8(sc.tex + ti[0], ti[1], ti[2], tcx, tcy, t4);
                };
                if (mat->tex[0] >= 0) fetch(0), tex_mat.albedo = V3<R>(t4[0], t4[1], t4[2]);
                if (mat->tex[1] >= 0) fetch(1), tex_mat.roughness = t4[0];
                if (mat->tex[2] >= 0) fetch(2), tex_mat.anisotropy = t4[0];
                if (mat->tex[3] >= 0) fetch(3), tex_mat.specular = V3<R>(t4[0], t4[1], t4[2]);
                if (mat->tex[4] >= 0) fetch(4), tex_mat.metallic = t4[0];
                if (mat->tex[5] >= 0) fetch(5), tex_mat.cru = t4[0];
                if (mat->tex[6] >= 0) fetch(6), tex_mat.crv = t4[0];
                if (mat->tex[7] >= 0) fetch(7), Ns = normal_from_tangent(Ns, V3<R>(t4[0], t4[1], t4[2]));
                mat = &tex_mat;
            }
            V3<R> P = w0 * from3<R>(vv) + u * from3<R>(vv + 3) + v * from3<R>(vv + 6);
            it.set_face_normal(d, Ns);
            it.distance = length(P - it.position);
            it.position = P;
            it.mat = mat;
            it.in_medium = sc.mesh_in[size_t(mesh)];
            it.out_medium = sc.mesh_out[size_t(mesh)];
            if (first) {
                p_normal = Ns;
                p_albedo = it.mat->albedo;
                first = false;
            }
        } else {
            it.distance = FMAX;
            it.in_medium = it.out_medium = cam.medium;
            it.front = true;
            if (first) {
                p_albedo = V3<R>(R(0));
                p_normal = V3<R>(R(0));
                first = false;
            }
        }
        closest = it.distance;
        bool hit_light = light_trace(sc, o, d, &it.in_medium, &it.out_medium, light_radiance, light_pdf, closest);

        bool scattered = false;
        int medium_index = -1;
        if (!sc.media.empty()) {
            medium_index = (hit_light ? true : it.front) ? it.out_medium : it.in_medium;
            R distance = R(0);
            if (medium_index != -1) {
                const Med<R>& med = sc.media[size_t(medium_index)];
                scattered = medium_sample(med, o, d, closest, distance, trans_pdf, transmittance, rng);
                history *= (transmittance / trans_pdf);
                mult_trans_pdf *= trans_pdf;
                if (scattered) {
                    it.position = pre_position + distance * L;
                    it.distance = distance;
                    if (nl != 0) {  // devicePrograms.cu:292-331
                        int idx = std::min(std::max(int(R(nl) * R(rng.next())), 0), nl - 1);
                        const Lt<R>& l = sc.lights[size_t(idx)];
                        R ld = R(0);
                        V3<R> so = it.position, sd;
                        R s0 = rng.next(), s1 = rng.next();
                        light_radiance = sample_light(l, so, s0, s1, sd, ld, light_pdf);
                        light_pdf *= (R(1) / R(nl));
                        bool occ = any_hit(*sc.bvh, tv, so, sd, EPS, ld - EPS);
                        closest = ld - EPS;
                        V3<R> tvv;
                        R tpdf;
                        if (!light_trace(sc, so, sd, nullptr, nullptr, tvv, tpdf, closest) &&
                            nee_pdf_ok(double(light_pdf))) {
                            transmittance = medium_transmittance(med, so, sd, closest, trans_pdf, rng);
                            attenuation = evaluate_phase(med, V, sd, phase_pdf);
                            R w = (l.type == RT_LIGHT_POINT) ? R(1) : power_heuristic(light_pdf, phase_pdf * trans_pdf);
                            if (!occ)
                                radiance += w * (transmittance / trans_pdf) * light_radiance * attenuation * history / light_pdf;
                        }
                    }
                    attenuation = sample_phase(med, rng, V, L, phase_pdf);
                    history *= (attenuation / phase_pdf);
                    pre_pdf = phase_pdf;
                }
            }
        }

        if (!scattered) {
            if (hit_light) {  // devicePrograms.cu:342-351
                R w = R(1);
                if (bounce != 0) {
                    pre_pdf *= mult_trans_pdf;
                    w = power_heuristic(pre_pdf, light_pdf);
                }
                radiance += w * history * light_radiance;
                break;
            }
            bool not_hit = closest == FMAX;
            if (not_hit && medium_index == -1) {  // devicePrograms.cu:354-373
                if (has_env) {
                    R u, v;
                    sphere_to_plane(d, u, v);
                    light_pdf = R(float(ew * eh)) / (R(2) * sqr(K<R>::PI));
                    R e[4], c[4];
                    tex_bilinear(env, ew, eh, u, v, e);
                    tex_bilinear(cache, ew, eh, u, v, c);
                    light_radiance = V3<R>(e[0], e[1], e[2]);
                    light_pdf *= c[2];
                    R w = R(1);
                    if (bounce != 0) {
                        pre_pdf *= mult_trans_pdf;
                        w = power_heuristic(pre_pdf, light_pdf);
                    }
                    radiance += w * history * light_radiance;
                }
                break;
            }
            if (has_env) {  // environment NEE, devicePrograms.cu:376-424
                R r0 = rng.next(), r1 = rng.next();
                R c[4];
                tex_bilinear(cache, ew, eh, r0, r1, c);
                R u = c[0], v = c[1];
                V3<R> so = it.position;
                V3<R> sd = plane_to_sphere(u, v);
                light_pdf = R(float(ew * eh)) / (R(2) * sqr(K<R>::PI));
                R c2[4], e[4];
                tex_bilinear(cache, ew, eh, u, v, c2);
                light_pdf *= c2[2];
                tex_bilinear(env, ew, eh, u, v, e);
                light_radiance = V3<R>(e[0], e[1], e[2]);
                bool occ = any_hit(*sc.bvh, tv, so, sd, EPS, FMAX);
                closest = FMAX;
                V3<R> tvv;
                R tpdf;
                if (!light_trace(sc, so, sd, nullptr, nullptr, tvv, tpdf, closest) && nee_pdf_ok(double(light_pdf))) {
                    bsdf = eval_material(it, lut, V, sd, bsdf_pdf);
                    R ct = std::fabs(dot(it.sn, sd));
                    R w = power_heuristic(light_pdf, bsdf_pdf);
                    V3<R> th(R(1));
                    if (medium_index != -1) {
                        const Med<R>& med = sc.media[size_t(medium_index)];
                        transmittance = medium_transmittance(med, so, sd, closest, trans_pdf, rng);
                        th = transmittance / trans_pdf;
                        w = power_heuristic(light_pdf, bsdf_pdf * trans_pdf);
                    }
                    if (!occ) radiance += w * th * light_radiance * bsdf * ct * history / light_pdf;
                }
            }
            if (nl != 0) {  // light NEE, devicePrograms.cu:426-471
                int idx = std::min(std::max(int(R(nl) * R(rng.next())), 0), nl - 1);
                const Lt<R>& l = sc.lights[size_t(idx)];
                R ld = R(0);
                V3<R> so = it.position, sd;
                R s0 = rng.next(), s1 = rng.next();
                light_radiance = sample_light(l, so, s0, s1, sd, ld, light_pdf);
                light_pdf *= (R(1) / R(nl));
                bool occ = any_hit(*sc.bvh, tv, so, sd, EPS, ld - EPS);
                closest = ld - EPS;
                V3<R> tvv;
                R tpdf;
                if (!light_trace(sc, so, sd, nullptr, nullptr, tvv, tpdf, closest) && nee_pdf_ok(double(light_pdf))) {
                    bsdf = eval_material(it, lut, V, sd, bsdf_pdf);
                    R ct = std::fabs(dot(it.sn, sd));
                    R w = (l.type == RT_LIGHT_POINT) ? R(1) : power_heuristic(light_pdf, bsdf_pdf);
                    V3<R> th(R(1));
                    if (medium_index != -1) {
                        const Med<R>& med = sc.media[size_t(medium_index)];
                        transmittance = medium_transmittance(med, so, sd, closest, trans_pdf, rng);
                        th = transmittance / trans_pdf;
                        if (l.type != RT_LIGHT_POINT) w = power_heuristic(light_pdf, bsdf_pdf * trans_pdf);
                    }
                    if (!occ) radiance += w * th * light_radiance * bsdf * ct * history / light_pdf;
                }
            }
            // BSDF sampling, devicePrograms.cu:474-477
            bsdf = sample_material_device(it, lut, rng, V, L, bsdf_pdf);
            R ct = std::fabs(dot(it.sn, L));
            history *= (bsdf * ct / bsdf_pdf);
            pre_pdf = bsdf_pdf;
        }

        // Russian roulette, devicePrograms.cu:480-489 (from bounce rr_depth)
        if (bounce >= opt.rr_depth) {
            R prr = dmin((history.x + history.y + history.z) / R(3), R(0.95f));
            if (R(rng.next()) > prr) break;
            history /= prr;
        }
        if (is_nan3(history)) break;

        V = -L;
        o = it.position;
        d = L;
        mult_trans_pdf = R(1);
        pre_position = it.position;
    }
}

template <class R>
void camera_setup(const rt_camera& c, int w, int h, Cam<R>& cam) {
    // Renderer::SetCamera, core/src/Renderer.cpp:796-813
    V3<float> from(c.from[0], c.from[1], c.from[2]), at(c.at[0], c.at[1], c.at[2]), up(c.up[0], c.up[1], c.up[2]);
    V3<float> dir = normalize(at - from);
    float cos_fovy = 0.66f;
    if (c.fov_y_deg > 0.0f) cos_fovy = 2.0f * std::tan(0.5f * c.fov_y_deg * 3.14159265358979323846f / 180.0f);
    float aspect = float(w) / float(h);
    V3<float> hor = cos_fovy * aspect * normalize(cross(dir, up));
    V3<float> ver = cos_fovy * normalize(cross(hor, dir));
    cam.pos = V3<R>(R(from.x), R(from.y), R(from.z));
    cam.dir = V3<R>(R(dir.x), R(dir.y), R(dir.z));
    cam.hor = V3<R>(R(hor.x), R(hor.y), R(hor.z));
    cam.ver = V3<R>(R(ver.x), R(ver.y), R(ver.z));
    cam.medium = c.medium;
}

template <class R>
int render_impl(SceneHandle* h, Scene<R>& sc, const rt_options& opt, const rt_camera& rc, int frame, float* color,
                float* albedo, float* normal, int64_t* nan_count, int nthreads, int row0, int row1) {
    Cam<R> cam;
    camera_setup(rc, opt.width, opt.height, cam);
    Lut<R> lut{h->lut, h->lut_avg};
    const int W = opt.width, H = opt.height;
    const int npix = W * H;
    int64_t nans = 0;
    if (row1 <= row0) {
        row0 = 0;
        row1 = H;
    }
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nans)
    for (int iy = row0; iy < row1; iy++) {
        for (int ix = 0; ix < W; ix++) {
            const int pix = ix + W * iy;
            Rng rng;
            if (opt.rng == RT_RNG_LCG) {
                rng.kind = 0;
                rng.lcg.init(uint32_t(pix), uint32_t(frame));
            } else {
                rng.kind = 1;
            }
            V3<R> pc(R(0)), pa(R(0)), pn(R(0));
            for (int s = 0; s < opt.spp; s++) {
                if (opt.rng != RT_RNG_LCG) rng.pcg.seed(pcg_frame_state(opt.seed, frame), uint64_t(s) * uint64_t(npix) + uint64_t(pix));
                R u0 = rng.next(), u1 = rng.next();
                R jx, jy;
                filter_jitter(opt.filter, u0, u1, jx, jy);
                // devicePrograms.cu:220-227
                R sx = (R(float(ix)) + R(0.5f) + jx) / R(float(W));
                R sy = (R(float(iy)) + R(0.5f) + jy) / R(float(H));
                V3<R> dir = normalize(cam.dir + (sx - R(0.5f)) * cam.hor + (sy - R(0.5f)) * cam.ver);
                V3<R> rad, a(R(0)), n(R(0));
                trace_sample(sc, sc.tv, sc.tn, cam, opt, lut, rng, dir, rad, a, n);
                if (is_nan3(rad)) {  // devicePrograms.cu:499-501
                    nans++;
                    if (opt.rng == RT_RNG_LCG) break;
                    continue;
                }
                pc += rad;
                pa += a;
                pn += n;
            }
            // devicePrograms.cu:518-531
            R inv = R(float(opt.spp));
            R c[4] = {pc.x / inv, pc.y / inv, pc.z / inv, R(1)};
            float* out = color + size_t(pix) * 4;
            if (frame > 0) {
                for (int k = 0; k < 4; k++) {
                    c[k] += R(float(frame)) * R(out[k]);
                    c[k] /= (R(float(frame)) + R(1));
                }
            }
            for (int k = 0; k < 4; k++) out[k] = float(c[k]);
            if (albedo) {
                float* a = albedo + size_t(pix) * 4;
                a[0] = float(pa.x / inv);
                a[1] = float(pa.y / inv);
                a[2] = float(pa.z / inv);
                a[3] = 1.0f;
            }
            if (normal) {
                float* n = normal + size_t(pix) * 4;
                n[0] = float(pn.x / inv);
                n[1] = float(pn.y / inv);
                n[2] = float(pn.z / inv);
                n[3] = 1.0f;
            }
        }
    }
    if (nan_count) *nan_count = nans;
    return 0;
}

template <class R>
void shading_impl(SceneHandle* lut_src, int op, const rt_material* mats, int nmat, const rt_light* lights, int nl,
                  const rt_medium* media, int nm, const float* in, int64_t n, float* out) {
    std::vector<Mat<R>> M(size_t(std::max(nmat, 0)));
    for (int i = 0; i < nmat; i++) M[size_t(i)].set(mats[i]);
    std::vector<Lt<R>> Ls(size_t(std::max(nl, 0)));
    for (int i = 0; i < nl; i++) Ls[size_t(i)].set(lights[i]);
    std::vector<Med<R>> Ms(size_t(std::max(nm, 0)));
    for (int i = 0; i < nm; i++) Ms[size_t(i)].set(media[i]);
    Lut<R> lut{lut_src->lut, lut_src->lut_avg};
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const float* x = in + q * 16;
        float* y = out + q * 8;
        for (int k = 0; k < 8; k++) y[k] = 0.0f;
        Rng rng;
        rng.kind = 2;
        if (op == RT_VERIFY_BSDF_EVAL || op == RT_VERIFY_BSDF_SAMPLE) {
            Isect<R> it;
            it.sn = from3<R>(x);
            it.front = (op == RT_VERIFY_BSDF_EVAL ? x[9] : x[12]) != 0.0f;
            int mi = int(op == RT_VERIFY_BSDF_EVAL ? x[10] : x[13]);
            it.mat = &M[size_t(mi)];
            V3<R> V = from3<R>(x + 3);
            R pdf = R(0);
            V3<R> f;
            if (op == RT_VERIFY_BSDF_EVAL) {
                f = eval_material(it, lut, V, from3<R>(x + 6), pdf);
            } else {
                rng.list = x + 6;
                rng.list_n = 6;
                V3<R> L(R(0));
                f = sample_material(it, lut, rng, V, L, pdf);
                y[4] = float(L.x);
                y[5] = float(L.y);
                y[6] = float(L.z);
                y[7] = float(rng.used);
            }
            y[0] = float(f.x);
            y[1] = float(f.y);
            y[2] = float(f.z);
            y[3] = float(pdf);
        } else if (op == RT_VERIFY_LIGHT_SAMPLE) {
            const Lt<R>& l = Ls[size_t(int(x[5]))];
            V3<R> L(R(0));
            R dist = R(0), pdf = R(0);
            V3<R> Li = sample_light(l, from3<R>(x), R(x[3]), R(x[4]), L, dist, pdf);
            y[0] = float(Li.x);
            y[1] = float(Li.y);
            y[2] = float(Li.z);
            y[3] = float(pdf);
            y[4] = float(L.x);
            y[5] = float(L.y);
            y[6] = float(L.z);
            y[7] = float(dist);
        } else if (op == RT_VERIFY_LIGHT_EVAL) {
            const Lt<R>& l = Ls[size_t(int(x[7]))];
            R pdf = R(0), ld = R(0);
            V3<R> Li = evaluate_light(l, from3<R>(x), from3<R>(x + 3), R(x[6]), pdf, ld);
            y[0] = float(Li.x);
            y[1] = float(Li.y);
            y[2] = float(Li.z);
            y[3] = float(pdf);
            y[4] = float(ld);
        } else if (op == RT_VERIFY_MEDIUM_SAMPLE) {
            const Med<R>& m = Ms[size_t(int(x[3]))];
            rng.list = x + 1;
            rng.list_n = 2;
            R dist = R(0), tp = R(0);
            V3<R> tr;
            bool s = sample_medium_distance(m, R(x[0]), dist, tp, tr, rng);
            y[0] = float(tr.x);
            y[1] = float(tr.y);
            y[2] = float(tr.z);
            y[3] = float(tp);
            y[4] = float(dist);
            y[5] = s ? 1.0f : 0.0f;
            y[6] = float(rng.used);
        } else if (op == RT_VERIFY_PHASE_SAMPLE) {
            const Med<R>& m = Ms[size_t(int(x[7]))];
            rng.list = x + 3;
            rng.list_n = 4;
            V3<R> L(R(0));
            R pdf = R(0);
            V3<R> a = sample_phase(m, rng, from3<R>(x), L, pdf);
            y[0] = float(a.x);
            y[1] = float(a.y);
            y[2] = float(a.z);
            y[3] = float(pdf);
            y[4] = float(L.x);
            y[5] = float(L.y);
            y[6] = float(L.z);
            y[7] = float(rng.used);
        } else if (op == RT_VERIFY_PHASE_EVAL) {
            const Med<R>& m = Ms[size_t(int(x[6]))];
            R pdf = R(0);
            V3<R> a = evaluate_phase(m, from3<R>(x), from3<R>(x + 3), pdf);
            y[0] = float(a.x);
            y[1] = float(a.y);
            y[2] = float(a.z);
            y[3] = float(pdf);
        }
    }
}

SceneHandle* lut_holder() {
    static SceneHandle* h = [] {
        SceneHandle* s = new SceneHandle();
        kulla_conty(s->lut, s->lut_avg);
        return s;
    }();
    return h;
}

}  // namespace

extern "C" {

// A scene in the de-indexed form of TriangleMesh (core/src/Scene.cpp:167-174):
// ntri*9 positions, optional ntri*9 normals (NULL: face normals as in
// Scene.cpp:150-158), optional ntri*6 texcoords, a mesh index per triangle,
// one material and (out, in) medium pair per mesh.
// Material textures: `texels` holds every texture's RGBA8 texels (row 0 at
// v = 0), `info` offset / width / height per texture.  Call before the
// first render.
void orc_scene_set_textures(void* hp, const uint32_t* texels, int64_t ntexels, const int32_t* info, int32_t ntex) {
    SceneHandle* h = static_cast<SceneHandle*>(hp);
    h->tex.assign(texels, texels + ntexels);
    h->tex_info.assign(info, info + 3 * ntex);
    h->sf.reset(make_scene<float>(h));
    h->sd.reset(make_scene<double>(h));
}

void* orc_scene_new(const float* tri_v, const float* tri_n, const float* tri_uv, const int32_t* tri_mesh, int64_t ntri,
                    const rt_material* mesh_mats, const int32_t* mesh_media, int32_t n_mesh, const rt_light* lights,
                    int32_t nl, const rt_medium* media, int32_t nm, const float* env_rgba, int32_t env_w, int32_t env_h) {
    SceneHandle* h = new SceneHandle();
    h->ntri = ntri;
    h->tv.assign(tri_v, tri_v + ntri * 9);
    if (tri_n) {
        h->tn.assign(tri_n, tri_n + ntri * 9);
    } else {
        h->tn.resize(size_t(ntri) * 9);
        for (int64_t i = 0; i < ntri; i++) {
            const float* p = tri_v + i * 9;
            V3<float> v0(p[0], p[1], p[2]), v1(p[3], p[4], p[5]), v2(p[6], p[7], p[8]);
            V3<float> n = normalize(cross(normalize(v1 - v0), normalize(v2 - v0)));
            for (int k = 0; k < 3; k++) {
                h->tn[size_t(i) * 9 + k * 3 + 0] = n.x;
                h->tn[size_t(i) * 9 + k * 3 + 1] = n.y;
                h->tn[size_t(i) * 9 + k * 3 + 2] = n.z;
            }
        }
    }
    if (tri_uv) {
        h->tuv.assign(tri_uv, tri_uv + ntri * 6);
    } else {
        h->tuv.resize(size_t(ntri) * 6);
        for (int64_t i = 0; i < ntri; i++) {
            float* t = h->tuv.data() + i * 6;
            t[0] = 0.f; t[1] = 0.f; t[2] = 1.f; t[3] = 0.f; t[4] = 0.f; t[5] = 1.f;
        }
    }
    h->tri_mesh.assign(tri_mesh, tri_mesh + ntri);
    h->mats.assign(mesh_mats, mesh_mats + n_mesh);
    h->mesh_media.assign(mesh_media, mesh_media + 2 * n_mesh);
    if (nl > 0) h->lights.assign(lights, lights + nl);
    if (nm > 0) h->media.assign(media, media + nm);
    h->dens.resize(size_t(std::max(nm, 0)));
    h->maj.resize(size_t(std::max(nm, 0)));
    for (int i = 0; i < nm; i++) {
        if (media[i].type != RT_MEDIUM_GRID || !media[i].density) continue;
        size_t n = size_t(media[i].grid_res[0]) * media[i].grid_res[1] * media[i].grid_res[2];
        h->dens[size_t(i)].assign(media[i].density, media[i].density + n);
        int mres = media[i].majorant_res > 0 ? media[i].majorant_res : 8;
        grid_majorants(h->dens[size_t(i)].data(), media[i].grid_res, mres, h->maj[size_t(i)]);
        h->media[size_t(i)].density = nullptr;
    }
    if (env_rgba && env_w > 0 && env_h > 0) {
        h->env.assign(env_rgba, env_rgba + size_t(env_w) * env_h * 4);
        h->cache.resize(h->env.size());
        env_cache(h->env.data(), env_w, env_h, h->cache.data());
        h->env_w = env_w;
        h->env_h = env_h;
    }
    h->bvh.build(h->tv.data(), ntri);
    kulla_conty(h->lut, h->lut_avg);
    h->sf.reset(make_scene<float>(h));
    h->sd.reset(make_scene<double>(h));
    return h;
}

void orc_scene_free(void* p) { delete static_cast<SceneHandle*>(p); }

// One Renderer::Render() (devicePrograms.cu:170-532 for every pixel of rows
// [row0, row1), or all rows when row1 <= row0).  `color` holds the running
// mean and is updated as in devicePrograms.cu:524-529.
int orc_render(void* p, int32_t precision, const rt_options* opt, const rt_camera* cam, int32_t frame, float* color,
               float* albedo, float* normal, int64_t* nan_count, int32_t nthreads, int32_t row0, int32_t row1) {
    SceneHandle* h = static_cast<SceneHandle*>(p);
    if (!h || !opt || !cam || !color) return 1;
    if (precision == 64) return render_impl(h, *h->sd, *opt, *cam, frame, color, albedo, normal, nan_count, nthreads, row0, row1);
    return render_impl(h, *h->sf, *opt, *cam, frame, color, albedo, normal, nan_count, nthreads, row0, row1);
}

// Camera vectors of Renderer::SetCamera: pos, direction, horizontal, vertical.
void orc_camera(const rt_camera* c, int32_t w, int32_t h, float* out12) {
    Cam<float> cam;
    camera_setup(*c, w, h, cam);
    const V3<float>* v[4] = {&cam.pos, &cam.dir, &cam.hor, &cam.ver};
    for (int i = 0; i < 4; i++) {
        out12[i * 3 + 0] = v[i]->x;
        out12[i * 3 + 1] = v[i]->y;
        out12[i * 3 + 2] = v[i]->z;
    }
}

// Ray queries: rays n x 8 (o, tmin, d, tmax).  Closest: out n x 8 =
// (t, b1, b2, prim, edge margin, second t, second prim, 0).  Any: out[i*8] = 1
// if occluded.
int orc_trace(void* p, int32_t precision, int32_t any, const float* rays, int64_t n, double* out) {
    SceneHandle* h = static_cast<SceneHandle*>(p);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; i++) {
        const float* r = rays + i * 8;
        double* y = out + i * 8;
        if (precision == 64) {
            V3<double> o = from3<double>(r), d = from3<double>(r + 4);
            if (any) {
                y[0] = any_hit(h->bvh, h->tv.data(), o, d, double(r[3]), double(r[7])) ? 1.0 : 0.0;
                continue;
            }
            HitInfo<double> hi;
            closest_hit(h->bvh, h->tv.data(), o, d, double(r[3]), double(r[7]), hi);
            y[0] = hi.t; y[1] = hi.b1; y[2] = hi.b2; y[3] = hi.prim; y[4] = hi.margin; y[5] = hi.t2; y[6] = hi.prim2; y[7] = 0;
        } else {
            V3<float> o = from3<float>(r), d = from3<float>(r + 4);
            if (any) {
                y[0] = any_hit(h->bvh, h->tv.data(), o, d, r[3], r[7]) ? 1.0 : 0.0;
                continue;
            }
            HitInfo<float> hi;
            closest_hit(h->bvh, h->tv.data(), o, d, r[3], r[7], hi);
            y[0] = hi.t; y[1] = hi.b1; y[2] = hi.b2; y[3] = hi.prim; y[4] = hi.margin; y[5] = hi.t2; y[6] = hi.prim2; y[7] = 0;
        }
    }
    return 0;
}

// Same layouts as rt_verify_shading (include/rt_capi.h).
int orc_shading(int32_t precision, int32_t op, const rt_material* mats, int32_t nmat, const rt_light* lights, int32_t nl,
                const rt_medium* media, int32_t nm, const float* in, int64_t n, float* out) {
    if (precision == 64)
        shading_impl<double>(lut_holder(), op, mats, nmat, lights, nl, media, nm, in, n, out);
    else
        shading_impl<float>(lut_holder(), op, mats, nmat, lights, nl, media, nm, in, n, out);
    return 0;
}

void orc_kulla_conty(float* bsdf, float* avg) { kulla_conty(bsdf, avg); }

// The reference's field defaults (core/include/Scene.h:48-55 Medium,
// :70-116 Material, :143-155 Light) restated for the C ABI structs, so the
// oracle builds scenes without the product library.  Phase::g has no
// initialiser there; it is zero here.
void orc_material_default(rt_material* m) {
    std::memset(m, 0, sizeof(*m));
    m->type = RT_MAT_METAL_WORKFLOW;
    const float eta[3] = {0.14282f, 0.37414f, 1.43944f}, k[3] = {3.97472f, 2.38066f, 1.59981f};
    for (int a = 0; a < 3; a++) {
        m->albedo[a] = 1.0f;
        m->eta[a] = eta[a];
        m->k[a] = k[a];
        m->specular[a] = 1.0f;
    }
    m->roughness = 0.1f;
    m->anisotropy = 0.0f;
    m->int_ior = 1.5f;
    m->ext_ior = 1.0f;
    m->nonlinear = 1;
    m->metallic = 0.8f;
    m->coat_weight = 2.0f;
    m->coat_roughness_u = 0.1f;
    m->coat_roughness_v = 0.1f;
    for (int t = 0; t < 8; t++) m->texture_ids[t] = -1;
}

void orc_light_default(rt_light* l) {
    std::memset(l, 0, sizeof(*l));
    l->type = RT_LIGHT_SPHERE;
    for (int a = 0; a < 3; a++) l->radiance[a] = 3.0f;
    l->position[0] = 6.0f;
    l->position[1] = 2.0f;
    l->u[2] = 6.0f;
    l->v[0] = 6.0f;
    l->radius = 3.0f;
    l->medium = -1;
}

void orc_medium_default(rt_medium* m) {
    std::memset(m, 0, sizeof(*m));
    m->type = RT_MEDIUM_HOMOGENEOUS;
    m->phase = RT_PHASE_ISOTROPIC;
    const float ss[3] = {0.74f, 0.88f, 1.01f}, sa[3] = {0.032f, 0.17f, 0.48f};
    for (int a = 0; a < 3; a++) {
        m->sigma_s[a] = ss[a];
        m->sigma_a[a] = sa[a];
    }
    m->scale = 500.0f;
}

void orc_env_cache(const float* rgba, int32_t w, int32_t h, float* cache) { env_cache(rgba, w, h, cache); }

// ComputeFinalPixelColorsKernel, core/cuda/PostProcessing.cu:18-48 (mode 0),
// ACES filmic (Narkowicz 2015 fit) + sRGB encoding (mode 1), clamp (mode 2).
void orc_tonemap(const float* color, int64_t n, int32_t mode, float exposure, uint32_t* out) {
    for (int64_t i = 0; i < n; i++) {
        const float* c = color + i * 4;
        float x = c[0] * exposure, y = c[1] * exposure, z = c[2] * exposure, w = c[3];
        float r, g, b;
        if (mode == RT_TONEMAP_REINHARD) {
            float lum = 0.299f * x + 0.587f * y + 0.114f * z;
            float f = 1.0f / (1.0f + lum / 1.5f);
            float v[4] = {x * f, y * f, z * f, z * f};
            for (int k = 0; k < 4; k++) v[k] = std::pow(v[k], 1.0f / 2.2f);
            for (int k = 0; k < 4; k++) v[k] = std::fmin(1.0f, std::fmax(0.0f, v[k]));
            r = v[0];
            g = v[1];
            b = v[2];
            (void)w;
            uint32_t q = uint32_t(r * 255.9f) | (uint32_t(g * 255.9f) << 8) | (uint32_t(b * 255.9f) << 16) | (255u << 24);
            out[i] = q;
            continue;
        }
        float v[3] = {x, y, z};
        for (int k = 0; k < 3; k++) {
            float t = v[k];
            if (mode == RT_TONEMAP_ACES_SRGB) {
                t = (t * (2.51f * t + 0.03f)) / (t * (2.43f * t + 0.59f) + 0.14f);
                t = std::fmin(1.0f, std::fmax(0.0f, t));
                t = t <= 0.0031308f ? 12.92f * t : 1.055f * std::pow(t, 1.0f / 2.4f) - 0.055f;
            }
            v[k] = std::fmin(1.0f, std::fmax(0.0f, t));
        }
        out[i] = uint32_t(v[0] * 255.0f + 0.5f) | (uint32_t(v[1] * 255.0f + 0.5f) << 8) |
                 (uint32_t(v[2] * 255.0f + 0.5f) << 16) | (255u << 24);
    }
}

}  // extern "C"
