// rt_tables.cpp - host-built tables uploaded with a scene.  Both follow the
// reference's float arithmetic operation for operation, so the tables are
// bit-identical to the ones the reference builds on its host (compile without
// FMA contraction).
#include <algorithm>
#include <cmath>
#include <vector>

#include "rt_bvh.h"

namespace rth {
using rtd::v3;

namespace {
v3 nrm(v3 v) { return v / std::sqrt(rtd::dot(v, v)); }
v3 refl(v3 v, v3 n) { return nrm(v - 2.0f * rtd::dot(v, n) * n); }

// SampleGGX, core/cuda/Microfacet.h:166-186 (isotropic branch)
v3 ggx_half(float a, float s0, float s1) {
    float phi = 6.28318530717958647692f * s1;
    float cp = std::cos(phi), sp = std::sin(phi);
    float a2 = a * a;
    float t2 = a2 * s0 / (1.0f - s0);
    float ct = 1.0f / std::sqrt(1.0f + t2);
    float st = std::sqrt(1.0f - ct * ct);
    return nrm(v3(st * cp, st * sp, ct));
}
// GeometrySmith_1, Microfacet.h:117-142 (isotropic branch)
float g1(v3 V, v3 H, v3 N, float a) {
    float c = rtd::dot(V, N);
    if (c * rtd::dot(V, H) <= 0.0f) return 0.0f;
    if (std::fabs(c - 1.0f) < 1e-4f) return 1.0f;
    float c2 = c * c, t2 = (1.0f - c2) / c2, a2 = a * a;
    return 2.0f / (1.0f + std::sqrt(1.0f + a2 * t2));
}
// Hammersley, Microfacet.h:220-229
void hammersley(uint32_t i, uint32_t n, float& x, float& y) {
    uint32_t b = (i << 16u) | (i >> 16u);
    b = ((b & 0x55555555u) << 1u) | ((b & 0xAAAAAAAAu) >> 1u);
    b = ((b & 0x33333333u) << 2u) | ((b & 0xCCCCCCCCu) >> 2u);
    b = ((b & 0x0F0F0F0Fu) << 4u) | ((b & 0xF0F0F0F0u) >> 4u);
    b = ((b & 0x00FF00FFu) << 8u) | ((b & 0xFF00FF00u) >> 8u);
    y = float(b) * 2.3283064365386963e-10f;
    x = float(i) / float(n);
}
}  // namespace

// ComputeKullaConty, Microfacet.h:231-291: E(mu, alpha) over a 64 x 64 grid
// with 128 Hammersley GGX samples per cell, and its cosine-weighted average.
void kulla_conty_tables(float* bsdf, float* avg) {
    const int R = 64;
    const uint32_t n = 128;
    const float inv_n = 1.0f / n;
    const v3 N(0.0f, 0.0f, 1.0f);
    const float step = 1.0f / R;
    for (int i = R - 1; i >= 0; --i) {
        float acc_albedo = 0.0f;
        float a = step * (float(i) + 0.5f);
        for (int j = R - 1; j >= 0; --j) {
            float mu = step * (float(j) + 0.5f);
            v3 V(std::sqrt(1.0f - mu * mu), 0.0f, mu);
            float acc = 0.0f;
            for (uint32_t k = 0; k < n; ++k) {
                float x, y;
                hammersley(k + 1, n + 1, x, y);
                v3 H = ggx_half(a, x, y);
                v3 L = refl(-V, H);
                float G = g1(L, H, N, a) * g1(V, H, N, a);
                float NdotV = rtd::dot(N, V), NdotL = rtd::dot(N, L), NdotH = rtd::dot(N, H), HdotV = rtd::dot(H, V);
                if (NdotL > 0.0f && NdotH > 0.0f && HdotV > 0.0f) acc += (HdotV * G) / (NdotV * NdotH);
            }
            float e = std::min(acc * inv_n, 1.0f);
            bsdf[i * R + j] = e;
            float al = 0.0f;
            for (uint32_t k = 0; k < n; ++k) {
                float x, y;
                hammersley(k + 1, n + 1, x, y);
                v3 H = ggx_half(a, x, y);
                v3 L = refl(-V, H);
                float HdotV = rtd::dot(H, V), NdotL = rtd::dot(N, L), NdotH = rtd::dot(N, H);
                if (NdotL > 0.0f && NdotH > 0.0f && HdotV > 0.0f) al += e * NdotL;
            }
            acc_albedo += al * 2.0f * inv_n;
        }
        avg[i] = acc_albedo * step;
    }
}

// HdrTexture::CalculateHdrCache, core/src/Scene.cpp:217-313: luminance pdf,
// column marginal and per-column conditional CDFs, and a w x h table mapping a
// uniform (u, v) to a texel by inverse-CDF lookups; texel (i, j) stores
// (x / w, y / h, pdf(i, j), 0).  The marginal index is clamped to w - 1.
void env_sampling_cache(const float* img, int w, int h, float* cache) {
    const size_t n = size_t(w) * h;
    std::vector<float> pdf(n);
    float sum = 0.0f;
    for (size_t q = 0; q < n; q++) {
        const float* p = img + q * 4;
        float lum = 0.299f * p[0] + 0.587f * p[1] + 0.114f * p[2];
        pdf[q] = lum;
        sum += lum;
    }
    for (size_t q = 0; q < n; q++) pdf[q] /= sum;
    std::vector<float> col(size_t(w), 0.0f), cdf_col;
    for (int x = 0; x < w; x++)
        for (int y = 0; y < h; y++) col[size_t(x)] += pdf[size_t(y) * w + x];
    cdf_col = col;
    for (int x = 1; x < w; x++) cdf_col[size_t(x)] += cdf_col[size_t(x) - 1];
    std::vector<float> cdf_row(n);  // column-major: [x][y]
    for (int x = 0; x < w; x++) {
        float run = 0.0f;
        for (int y = 0; y < h; y++) {
            float c = pdf[size_t(y) * w + x] / col[size_t(x)];
            run = y == 0 ? c : run + c;
            cdf_row[size_t(x) * h + y] = run;
        }
    }
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            float xi1 = float(y) / h, xi2 = float(x) / w;
            int cx = int(std::lower_bound(cdf_col.begin(), cdf_col.end(), xi1) - cdf_col.begin());
            cx = std::min(cx, w - 1);
            const float* c = cdf_row.data() + size_t(cx) * h;
            int cy = int(std::lower_bound(c, c + h, xi2) - c);
            float* o = cache + (size_t(y) * w + x) * 4;
            o[0] = float(cx) / w;
            o[1] = float(cy) / h;
            o[2] = pdf[size_t(y) * w + x];
            o[3] = 0.0f;
        }
    }
}

}  // namespace rth
