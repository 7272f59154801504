// rt_device.cuh - device-side data layout, vector math and random streams of
// the B200 path tracer.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/rt_capi.h"

#define RT_HD __host__ __device__ __forceinline__
#define RT_D __device__ __forceinline__

namespace rtd {

// ------------------------------------------------------------------ vec3
// A 3-vector of float (v3, the renderer's arithmetic) or double (v3d, the
// BSDF sampler's).  The scalar of a mixed vector-scalar expression converts
// to the vector's type, so float literals keep their float value.
template <class R>
struct vec3t {
    R x, y, z;
    RT_HD vec3t() : x(R(0)), y(R(0)), z(R(0)) {}
    RT_HD explicit vec3t(R s) : x(s), y(s), z(s) {}
    RT_HD vec3t(R a, R b, R c) : x(a), y(b), z(c) {}
    RT_HD R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
using v3 = vec3t<float>;
using v3d = vec3t<double>;
template <class T>
struct same_t {
    using type = T;
};
template <class R> using sc_t = typename same_t<R>::type;  // not deduced: takes the vector's scalar type

template <class R> RT_HD vec3t<R> operator+(vec3t<R> a, vec3t<R> b) { return vec3t<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R> RT_HD vec3t<R> operator-(vec3t<R> a, vec3t<R> b) { return vec3t<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R> RT_HD vec3t<R> operator*(vec3t<R> a, vec3t<R> b) { return vec3t<R>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class R> RT_HD vec3t<R> operator/(vec3t<R> a, vec3t<R> b) { return vec3t<R>(a.x / b.x, a.y / b.y, a.z / b.z); }
template <class R> RT_HD vec3t<R> operator*(vec3t<R> a, sc_t<R> s) { return vec3t<R>(a.x * s, a.y * s, a.z * s); }
template <class R> RT_HD vec3t<R> operator*(sc_t<R> s, vec3t<R> a) { return vec3t<R>(s * a.x, s * a.y, s * a.z); }
template <class R> RT_HD vec3t<R> operator/(vec3t<R> a, sc_t<R> s) { return vec3t<R>(a.x / s, a.y / s, a.z / s); }
template <class R> RT_HD vec3t<R> operator+(vec3t<R> a, sc_t<R> s) { return vec3t<R>(a.x + s, a.y + s, a.z + s); }
template <class R> RT_HD vec3t<R> operator-(sc_t<R> s, vec3t<R> a) { return vec3t<R>(s - a.x, s - a.y, s - a.z); }
template <class R> RT_HD vec3t<R> operator-(vec3t<R> a, sc_t<R> s) { return vec3t<R>(a.x - s, a.y - s, a.z - s); }
template <class R> RT_HD vec3t<R> operator-(vec3t<R> a) { return vec3t<R>(-a.x, -a.y, -a.z); }
template <class R> RT_HD vec3t<R>& operator+=(vec3t<R>& a, vec3t<R> b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
template <class R> RT_HD vec3t<R>& operator*=(vec3t<R>& a, vec3t<R> b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
template <class R> RT_HD vec3t<R>& operator*=(vec3t<R>& a, sc_t<R> s) { a.x *= s; a.y *= s; a.z *= s; return a; }
template <class R> RT_HD vec3t<R>& operator/=(vec3t<R>& a, sc_t<R> s) { a.x /= s; a.y /= s; a.z /= s; return a; }
template <class R> RT_HD R dot(vec3t<R> a, vec3t<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> RT_HD vec3t<R> cross(vec3t<R> a, vec3t<R> b) {
    return vec3t<R>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
// Math of either precision: the float forms are the ones the renderer has
// always used (sqrtf, fabsf, ...); the double forms are CUDA's double ones.
RT_HD float sqrt_r(float x) { return sqrtf(x); }
RT_HD double sqrt_r(double x) { return sqrt(x); }
RT_HD float fabs_r(float x) { return fabsf(x); }
RT_HD double fabs_r(double x) { return fabs(x); }
RT_HD float fmin_r(float a, float b) { return fminf(a, b); }
RT_HD double fmin_r(double a, double b) { return fmin(a, b); }
RT_HD float fmax_r(float a, float b) { return fmaxf(a, b); }
RT_HD double fmax_r(double a, double b) { return fmax(a, b); }
// a float literal beside a double promotes to double
RT_HD double fmin_r(float a, double b) { return fmin(double(a), b); }
RT_HD double fmin_r(double a, float b) { return fmin(a, double(b)); }
RT_HD double fmax_r(float a, double b) { return fmax(double(a), b); }
RT_HD double fmax_r(double a, float b) { return fmax(a, double(b)); }
RT_HD void sincos_r(float a, float* s, float* c) { sincosf(a, s, c); }
RT_HD void sincos_r(double a, double* s, double* c) { sincos(a, s, c); }
// sin and cos of 2 pi u for u in [0, 1): FP32 keeps the reference's
// sincosf(2 pi u); FP64 takes sincospi(2 u), which reduces its argument
// exactly (no wide-range reduction path) and differs from sin(2 pi u)
// evaluated in double only by the rounding of 2 pi u (~1e-16).
RT_HD void sincos_2pi_r(float u, float* s, float* c) { sincosf(6.28318530717958647692f * u, s, c); }
RT_HD void sincos_2pi_r(double u, double* s, double* c) {
#ifdef __CUDA_ARCH__
    sincospi(2.0 * u, s, c);
#else
    sincos_r(6.28318530717958647692 * u, s, c);
#endif
}
template <class R> RT_HD R length(vec3t<R> v) { return sqrt_r(dot(v, v)); }
// Component-wise division by the length, as gdt's normalize (vec.h:306-310).
template <class R> RT_HD vec3t<R> normalize(vec3t<R> v) { return v / sqrt_r(dot(v, v)); }
// Double precision (the BSDF sampler): one reciprocal or reciprocal square
// root and three products instead of three divisions.  That is within 2 ulp
// of double, far below the single-precision rounding the sampler's outputs
// end in; the single-precision forms above keep the reference's divisions.
RT_HD v3d operator/(v3d a, double s) {
    const double r = 1.0 / s;
    return v3d(a.x * r, a.y * r, a.z * r);
}
RT_HD v3d normalize(v3d v) {
#ifdef __CUDA_ARCH__
    const double r = rsqrt(dot(v, v));
#else
    const double r = 1.0 / sqrt(dot(v, v));
#endif
    return v3d(v.x * r, v.y * r, v.z * r);
}
template <class R> RT_HD bool any_nan(vec3t<R> v) { return v.x != v.x || v.y != v.y || v.z != v.z; }
RT_HD float sqr(float x) { return x * x; }
RT_HD double sqr(double x) { return x * x; }
RT_HD float mixf(float x, float y, float t) { return x * (1.0f - t) + y * t; }
template <class R> RT_HD R mix_r(R x, R y, R t) { return x * (R(1) - t) + y * t; }
RT_HD v3d to_d(v3 a) { return v3d(double(a.x), double(a.y), double(a.z)); }
RT_HD v3 to_f(v3d a) { return v3(float(a.x), float(a.y), float(a.z)); }
RT_HD v3 xyz(float4 a) { return v3(a.x, a.y, a.z); }
RT_HD float4 f4(v3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
RT_HD v3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

// Depth limit of the per-thread traversal stack; a BVH deeper than this is
// rejected at upload.
constexpr int kStackSize = 32;
// Tentative collisions one delta- or ratio-tracking walk may take (rt_media.cuh).
constexpr int kMaxTrackingSteps = 4096;

constexpr float kEps = 1e-4f;                                  // core/cuda/Utils.h:10
constexpr float kPi = 3.14159265358979323846f;                 // Utils.h:11
constexpr float kTwoPi = 6.28318530717958647692f;              // Utils.h:14
constexpr float kInvPi = 0.318309886183790671538f;             // Utils.h:13
// The same constants rounded to either precision (float: identical to the above).
template <class R>
struct Kc {
    static constexpr R pi = R(3.14159265358979323846);
    static constexpr R two_pi = R(6.28318530717958647692);
    static constexpr R inv_pi = R(0.318309886183790671538);
};

// ------------------------------------------------------------------ random
// gdt::LCG<16> of the reference (common/gdt/gdt/random/random.h:54-87).
RT_HD uint32_t lcg_seed(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
#pragma unroll
    for (int n = 0; n < 16; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
// PCG32 (pcg-random.org, pcg32_random_r); the increment is derived from the
// path index so only the 64-bit state travels with a path.
RT_HD uint64_t pcg_inc(uint64_t seq) { return (seq << 1u) | 1u; }
RT_HD uint64_t pcg_seed(uint64_t initstate, uint64_t seq) {
    uint64_t inc = pcg_inc(seq);
    uint64_t s = inc;  // 0 * mult + inc
    s += initstate;
    s = s * 6364136223846793005ULL + inc;
    return s;
}
RT_HD uint64_t pcg_frame_state(uint64_t seed, int frame) {
    return seed ^ (uint64_t(uint32_t(frame)) * 0x9E3779B97F4A7C15ULL);
}

// One random stream: the reference LCG (24-bit floats) or PCG32.
struct Rng {
    uint64_t state;
    uint64_t inc;  // 0 selects the LCG
    RT_HD float next() {
        if (inc == 0) {
            uint32_t s = uint32_t(state) * 1664525u + 1013904223u;
            state = s;
            return float(s & 0x00FFFFFFu) / float(0x01000000);
        }
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        uint32_t r = (xs >> rot) | (xs << ((32u - rot) & 31u));
        return float(r >> 8) * (1.0f / 16777216.0f);
    }
};

// ------------------------------------------------------------------ scene
// Device copy of rt_material (core/include/Scene.h:70-116), 128 bytes.
struct __align__(16) DevMaterial {
    int type;
    float albedo[3];
    float roughness, anisotropy, int_ior, ext_ior;
    float eta[3];
    float metallic;
    float k[3];
    float coat_weight;
    float specular[3];
    int nonlinear;
    float coat_roughness_u, coat_roughness_v;
    int textured;  // any tex[] >= 0
    float pad1;
    int tex[8];    // texture ids: albedo, roughness, anisotropy, specular, metallic, coat u, coat v, normal
};
static_assert(sizeof(DevMaterial) == 128, "DevMaterial layout");

// Device copy of rt_light (Scene.h:143-155), 64 bytes.
struct __align__(16) DevLight {
    int type;
    int double_side;
    float radius;
    int medium;
    float radiance[3];
    float pad0;
    float position[3];
    float pad1;
    float u[3];
    float pad2;
    float v[3];
    float pad3;
};

// Device copy of rt_medium (Scene.h:48-55) plus the density grid.
struct __align__(16) DevMedium {
    int type, phase;
    float scale;
    int majorant_res;
    float g[3];
    float pad0;
    float sigma_s[3];
    float pad1;
    float sigma_a[3];
    float pad2;
    float bmin[3];
    float max_density;
    float bmax[3];
    float pad3;
    int res[3];
    int pad4;
    const float* density;
    const float* majorant;
};

// Per mesh: material index and medium interface (TriangleMeshSBTData,
// core/include/LaunchParams.h:16-26).
struct __align__(16) MeshInfo {
    int material;
    int in_medium;
    int out_medium;
    int pad;
};

// Compressed 8-wide BVH node (after Ylitie, Karras, Laine, HPG 2017):
// 80 bytes, read as five 16-byte words.
struct __align__(16) CwNode {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(CwNode) == 80, "CwNode layout");

// Everything a kernel needs about one scene, all device pointers.
struct SceneView {
    const CwNode* nodes;
    const float4* tri_v;   // 3 per triangle: v0 (w = original id bits), v1, v2
    const float4* tri_a;   // 4 per triangle: normals, texcoords, mesh id
    int num_nodes;
    int num_tris;
    int bvh_depth;           // wide levels (<= kStackSize)
    const MeshInfo* meshes;
    const DevMaterial* materials;
    const DevLight* lights;
    int num_lights;
    int num_media;
    const DevMedium* media;
    const float4* env;
    const float4* env_cache;
    int env_w, env_h;
    const float* lut;
    const float* lut_avg;
    const uint32_t* tex;     // RGBA8 texels of every material texture
    const int4* tex_info;    // offset, width, height per texture
    int num_tex;
};

// Camera vectors of Renderer::SetCamera (core/src/Renderer.cpp:796-813).
struct CameraView {
    float pos[3], dir[3], hor[3], ver[3];
    int medium;
};

}  // namespace rtd
