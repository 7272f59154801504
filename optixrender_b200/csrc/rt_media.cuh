// rt_media.cuh - heterogeneous (density grid) media.
//
// The reference has homogeneous media only (core/cuda/Medium.h:112-244).  A
// grid medium scales the extinction sigma_t = scale * max_c(sigma_a + sigma_s)
// by a trilinearly interpolated density; its single-scattering albedo
// sigma_s / (sigma_a + sigma_s) stays per channel.  Free-flight distances are
// sampled by delta tracking (Woodcock) against a coarse majorant grid walked
// with a 3D DDA; transmittance for next-event rays is estimated by ratio
// tracking.  Both estimators are unbiased and keep the reference integrator's
// form `history *= transmittance / trans_pdf` with trans_pdf = 1:
//   scattered:  transmittance = albedo
//   passed:     transmittance = 1
// Loops are bounded (kMaxTrackingSteps): a walk that runs out ends with zero
// weight and adds one to `budget_hits`, which the renderer reports as
// RT_ERR_DEVICE_WATCHDOG.
#pragma once

#include "rt_device.cuh"

namespace rtd {


struct GridParams {
    v3 bmin, bmax;
    int res[3];
    int mres;
    float sigma_t;      // extinction per unit density
    v3 albedo;
    const float* density;
    const float* majorant;  // mres^3 maximum densities
};

RT_HD float grid_sigma_t0(const float* sa, const float* ss, float scale) {
    float m = 0.0f;
    for (int c = 0; c < 3; c++) m = fmaxf(m, sa[c] + ss[c]);
    return m * scale;
}

RT_D GridParams load_grid(const DevMedium* m) {
    GridParams g;
    g.bmin = ld3(m->bmin);
    g.bmax = ld3(m->bmax);
    g.res[0] = m->res[0];
    g.res[1] = m->res[1];
    g.res[2] = m->res[2];
    g.mres = m->majorant_res;
    g.sigma_t = grid_sigma_t0(m->sigma_a, m->sigma_s, m->scale);
    v3 ss = ld3(m->sigma_s), st = ld3(m->sigma_a) + ss;
    g.albedo = v3(st.x > 0.0f ? ss.x / st.x : 0.0f, st.y > 0.0f ? ss.y / st.y : 0.0f, st.z > 0.0f ? ss.z / st.z : 0.0f);
    g.density = m->density;
    g.majorant = m->majorant;
    return g;
}

// Trilinear density at world position p; zero outside the box.
RT_D float grid_density(const GridParams& g, v3 p) {
    v3 ext = g.bmax - g.bmin;
    float gx = (p.x - g.bmin.x) / ext.x * float(g.res[0]) - 0.5f;
    float gy = (p.y - g.bmin.y) / ext.y * float(g.res[1]) - 0.5f;
    float gz = (p.z - g.bmin.z) / ext.z * float(g.res[2]) - 0.5f;
    if (!(gx > -0.5f && gy > -0.5f && gz > -0.5f && gx < float(g.res[0]) - 0.5f && gy < float(g.res[1]) - 0.5f &&
          gz < float(g.res[2]) - 0.5f))
        return 0.0f;
    gx = fminf(fmaxf(gx, 0.0f), float(g.res[0] - 1));
    gy = fminf(fmaxf(gy, 0.0f), float(g.res[1] - 1));
    gz = fminf(fmaxf(gz, 0.0f), float(g.res[2] - 1));
    int x0 = min(int(gx), g.res[0] - 1), y0 = min(int(gy), g.res[1] - 1), z0 = min(int(gz), g.res[2] - 1);
    int x1 = min(x0 + 1, g.res[0] - 1), y1 = min(y0 + 1, g.res[1] - 1), z1 = min(z0 + 1, g.res[2] - 1);
    float fx = gx - float(x0), fy = gy - float(y0), fz = gz - float(z0);
    auto at = [&](int x, int y, int z) { return __ldg(g.density + (size_t(z) * g.res[1] + y) * g.res[0] + x); };
    float c00 = mixf(at(x0, y0, z0), at(x1, y0, z0), fx), c10 = mixf(at(x0, y1, z0), at(x1, y1, z0), fx);
    float c01 = mixf(at(x0, y0, z1), at(x1, y0, z1), fx), c11 = mixf(at(x0, y1, z1), at(x1, y1, z1), fx);
    return mixf(mixf(c00, c10, fy), mixf(c01, c11, fy), fz);
}

// Slab intersection of the ray with the grid box; false if it misses [0, tmax].
RT_D bool grid_clip(const GridParams& g, v3 o, v3 d, float tmax, float& t0, float& t1) {
    t0 = 0.0f;
    t1 = tmax;
    for (int a = 0; a < 3; a++) {
        float inv = 1.0f / d[a];
        float ta = (g.bmin[a] - o[a]) * inv, tb = (g.bmax[a] - o[a]) * inv;
        if (ta > tb) {
            float t = ta;
            ta = tb;
            tb = t;
        }
        t0 = fmaxf(t0, ta);
        t1 = fminf(t1, tb);
    }
    return t0 < t1;
}

// Walks the majorant cells the ray crosses in [t0, t1] and calls
// f(cell_t0, cell_t1, majorant_density); f returns false to stop the walk.
template <class F>
RT_D void majorant_walk(const GridParams& g, v3 o, v3 d, float t0, float t1, F&& f) {
    const int R = g.mres;
    v3 ext = g.bmax - g.bmin;
    v3 p = o + t0 * d;
    int c[3], step[3];
    float tnext[3], tdelta[3];
    for (int a = 0; a < 3; a++) {
        float cell = ext[a] / float(R);
        float rel = (p[a] - g.bmin[a]) / cell;
        int ci = min(max(int(floorf(rel)), 0), R - 1);
        c[a] = ci;
        float da = d[a];
        if (da > 0.0f) {
            step[a] = 1;
            tnext[a] = t0 + ((g.bmin[a] + float(ci + 1) * cell) - p[a]) / da;
            tdelta[a] = cell / da;
        } else if (da < 0.0f) {
            step[a] = -1;
            tnext[a] = t0 + ((g.bmin[a] + float(ci) * cell) - p[a]) / da;
            tdelta[a] = -cell / da;
        } else {
            step[a] = 0;
            tnext[a] = FLT_MAX;
            tdelta[a] = FLT_MAX;
        }
    }
    float t = t0;
    for (int it = 0; it < 3 * R + 3 && t < t1; it++) {
        int a = tnext[0] < tnext[1] ? (tnext[0] < tnext[2] ? 0 : 2) : (tnext[1] < tnext[2] ? 1 : 2);
        float te = fminf(tnext[a], t1);
        float mj = __ldg(g.majorant + (size_t(c[2]) * R + c[1]) * R + c[0]);
        if (!f(t, te, mj)) return;
        t = te;
        c[a] += step[a];
        if (c[a] < 0 || c[a] >= R) return;
        tnext[a] += tdelta[a];
    }
}

// Delta tracking inside [0, maxd): returns true with the collision distance
// when a real collision happens.  `steps` counts tentative collisions.
template <class RNG>
RT_D bool grid_sample_distance(const GridParams& g, v3 o, v3 d, float maxd, RNG& rng, float& dist, v3& weight,
                                int& budget_hits) {
    weight = v3(1.0f);
    float t0, t1;
    if (!grid_clip(g, o, d, maxd, t0, t1) || g.sigma_t <= 0.0f) return false;
    bool scattered = false;
    int steps = 0;
    majorant_walk(g, o, d, t0, t1, [&](float ca, float cb, float mj) {
        float smax = mj * g.sigma_t;
        if (smax <= 0.0f) return true;
        float t = ca;
        while (true) {
            if (++steps > kMaxTrackingSteps) {
                weight = v3(0.0f);
                budget_hits++;
                return false;
            }
            t -= logf(1.0f - rng.next()) / smax;
            if (t >= cb) return true;
            float s = grid_density(g, o + t * d) * g.sigma_t;
            if (rng.next() * smax < s) {
                scattered = true;
                dist = t;
                return false;
            }
        }
    });
    if (scattered) weight = g.albedo;
    return scattered;
}

// Ratio-tracking transmittance along [0, maxd).
template <class RNG>
RT_D float grid_transmittance(const GridParams& g, v3 o, v3 d, float maxd, RNG& rng, int& budget_hits) {
    float t0, t1;
    if (!grid_clip(g, o, d, maxd, t0, t1) || g.sigma_t <= 0.0f) return 1.0f;
    float T = 1.0f;
    int steps = 0;
    majorant_walk(g, o, d, t0, t1, [&](float ca, float cb, float mj) {
        float smax = mj * g.sigma_t;
        if (smax <= 0.0f) return true;
        float t = ca;
        while (true) {
            if (++steps > kMaxTrackingSteps) {
                T = 0.0f;
                budget_hits++;
                return false;
            }
            t -= logf(1.0f - rng.next()) / smax;
            if (t >= cb) return true;
            float s = grid_density(g, o + t * d) * g.sigma_t;
            T *= 1.0f - s / smax;
            if (T <= 0.0f) return false;
        }
    });
    return T;
}

}  // namespace rtd
