// optixrender.hpp - C++ host API of the B200 path tracer, header-only, over
// the C ABI of rt_capi.h.
//
// Mirrors the reference renderer's host classes so code written against
// GraphicsEnthusiast/OptiXRender ports by renaming the include:
//   Scene     core/include/Scene.h:195-214   AddMesh / AddLight / AddMedium / AddEnv
//   Renderer  core/include/Renderer.h:9-187  Render / Resize / SetCamera / DownloadPixels
//   Material, Light, Medium, Camera          core/include/Scene.h:11-155 field names
// Errors are reported as rt::Error exceptions on the C++ side of the boundary
// (the reference throws std::runtime_error from CUDA_CHECK, common/optix7.h:26-37);
// nothing throws across the C ABI itself.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "rt_capi.h"

namespace rt {

struct Error : std::runtime_error {
    rt_status code;
    Error(rt_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(rt_status s) {
    if (s != RT_OK) throw Error(s, rt_last_error_message());
}

struct vec3f {
    float x, y, z;
};

enum MaterialType {
    Diffuse = RT_MAT_DIFFUSE,
    Conductor = RT_MAT_CONDUCTOR,
    Dielectric = RT_MAT_DIELECTRIC,
    Plastic = RT_MAT_PLASTIC,
    MetalWorkflow = RT_MAT_METAL_WORKFLOW,
    ThinDielectric = RT_MAT_THIN_DIELECTRIC,
    ClearCoatedConductor = RT_MAT_CLEARCOATED_CONDUCTOR,
    DiffuseTransmitter = RT_MAT_DIFFUSE_TRANSMITTER
};
enum LightType { Quad = RT_LIGHT_QUAD, Sphere = RT_LIGHT_SPHERE, Point = RT_LIGHT_POINT };
enum FilterType { Box = RT_FILTER_BOX, Tent = RT_FILTER_TENT, Triangle = RT_FILTER_TRIANGLE, Gaussian = RT_FILTER_GAUSSIAN };

// struct Material (Scene.h:70-116) with the same defaults.
struct Material : rt_material {
    Material() { rt_material_default(this); }
    explicit Material(MaterialType t) {
        rt_material_default(this);
        type = t;
    }
};
// struct Light (Scene.h:143-155).
struct Light : rt_light {
    Light() { rt_light_default(this); }
};
// struct Medium (Scene.h:48-55).
struct Medium : rt_medium {
    Medium() { rt_medium_default(this); }
};
// struct Camera (Scene.h:11-20).
struct Camera : rt_camera {
    Camera() { rt_camera_default(this); }
    Camera(vec3f from_, vec3f at_, vec3f up_, int medium_ = -1) {
        rt_camera_default(this);
        from[0] = from_.x, from[1] = from_.y, from[2] = from_.z;
        at[0] = at_.x, at[1] = at_.y, at[2] = at_.z;
        up[0] = up_.x, up[1] = up_.y, up[2] = up_.z;
        medium = medium_;
    }
};
struct Options : rt_options {
    Options() { rt_options_default(this); }
};

// class Scene, core/include/Scene.h:195-214.
class Scene {
public:
    Scene() { check(rt_scene_create(&h_)); }
    ~Scene() { rt_scene_destroy(h_); }
    Scene(const Scene&) = delete;
    Scene& operator=(const Scene&) = delete;

    // Scene::AddMesh from an OBJ path (Scene.cpp:22-64).
    int AddMesh(const std::string& objFile, const Material& material, int out_med = -1, int in_med = -1) {
        int32_t id = -1;
        check(rt_scene_add_mesh_obj(h_, objFile.c_str(), &material, out_med, in_med, &id));
        return id;
    }
    // Scene::AddMesh from arrays (3 floats per position / normal, 2 per texcoord).
    int AddMesh(const std::vector<float>& positions, const std::vector<int32_t>& indices, const Material& material,
                int out_med = -1, int in_med = -1, const std::vector<float>* normals = nullptr,
                const std::vector<float>* texcoords = nullptr) {
        rt_mesh_desc d{};
        d.positions = positions.data();
        d.num_vertices = int64_t(positions.size() / 3);
        d.indices = indices.empty() ? nullptr : indices.data();
        d.num_triangles = indices.empty() ? d.num_vertices / 3 : int64_t(indices.size() / 3);
        d.normals = normals ? normals->data() : nullptr;
        d.texcoords = texcoords ? texcoords->data() : nullptr;
        int32_t id = -1;
        check(rt_scene_add_mesh(h_, &d, &material, out_med, in_med, &id));
        return id;
    }
    // Scene::AddTexture(fileName) (Scene.cpp:66-69): BMP or binary PGM/PPM.
    int AddTexture(const std::string& fileName) {
        int32_t id = -1;
        check(rt_scene_add_texture_file(h_, fileName.c_str(), &id));
        return id;
    }
    // A decoded RGBA8 image, row 0 at the bottom (v = 0).
    int AddTexture(const std::vector<uint8_t>& rgba, int width, int height) {
        int32_t id = -1;
        check(rt_scene_add_texture(h_, rgba.data(), width, height, &id));
        return id;
    }
    void AddLight(const Light& l) { check(rt_scene_add_light(h_, &l)); }
    void AddMedium(const Medium& m) { check(rt_scene_add_medium(h_, &m)); }
    // Scene::AddEnv with an equirectangular RGBA float image (row 0 at the bottom).
    void AddEnv(const std::vector<float>& rgba, int width, int height, float scale = 1.0f) {
        check(rt_scene_set_env(h_, rgba.data(), width, height, scale));
    }
    // Scene::AddEnv(fileName) (Scene.cpp:79-81): a Radiance .hdr (or LDR) file.
    void AddEnv(const std::string& path, float scale = 1.0f) { check(rt_scene_set_env_file(h_, path.c_str(), scale)); }
    // SceneParser::LoadFromJson (SceneParser.cpp:3-23), returning the settings.
    void LoadFromJson(const std::string& path, Options& opts, Camera& cam) {
        check(rt_scene_load_json(h_, path.c_str(), &opts, &cam));
    }
    void Bounds(vec3f& lo, vec3f& hi) const {
        float l[3], u[3];
        check(rt_scene_get_bounds(h_, l, u));
        lo = {l[0], l[1], l[2]};
        hi = {u[0], u[1], u[2]};
    }
    const rt_scene* handle() const { return h_; }

private:
    rt_scene* h_ = nullptr;
};

// class Renderer, core/include/Renderer.h:9-187.
class Renderer {
public:
    explicit Renderer(const Scene& scene, const Options& opts = Options()) {
        check(rt_renderer_create(scene.handle(), &opts, &h_));
    }
    ~Renderer() { rt_renderer_destroy(h_); }
    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;

    void Render() { check(rt_renderer_render(h_)); }
    void Resize(int w, int h) { check(rt_renderer_resize(h_, w, h)); }
    void SetCamera(const Camera& c) { check(rt_renderer_set_camera(h_, &c)); }
    void DownloadPixels(uint32_t h_pixels[]) { check(rt_renderer_download_rgba8(h_, h_pixels)); }
    void DownloadLinear(float* rgba) { check(rt_renderer_download_linear(h_, rgba)); }
    void DownloadAov(int kind, float* rgba) { check(rt_renderer_download_aov(h_, kind, rgba)); }
    void Synchronize() { check(rt_renderer_synchronize(h_)); }
    Options GetOptions() const {
        Options o;
        check(rt_renderer_get_options(h_, &o));
        return o;
    }
    void SetOptions(const Options& o) { check(rt_renderer_set_options(h_, &o)); }
    rt_render_stats Stats() const {
        rt_render_stats s{};
        check(rt_renderer_get_stats(h_, &s));
        return s;
    }
    // The reference's public fields (Renderer.h:139-143): progressive and
    // launchParams.numPixelSamples / maxBounce, set through the options.
    void SetProgressive(bool on) {
        Options o = GetOptions();
        o.progressive = on ? 1 : 0;
        SetOptions(o);
    }
    void SetSamplesPerPixel(int spp) {
        Options o = GetOptions();
        o.spp = spp;
        SetOptions(o);
    }
    // Renderer::denoiserOn (Renderer.h:139): DownloadPixels shows the denoised colour.
    void SetDenoiser(bool on) {
        Options o = GetOptions();
        o.denoise = on ? 1 : 0;
        SetOptions(o);
    }
    rt_renderer* handle() { return h_; }

private:
    rt_renderer* h_ = nullptr;
};

// The continuous-batching server over resident scenes (rt_server_*; the
// reference renders one frame per Renderer and has no counterpart).
class Server {
public:
    explicit Server(const rt_server_options* o = nullptr) { check(rt_server_create(o, &h_)); }
    ~Server() { rt_server_destroy(h_); }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    int AddScene(const Scene& scene) {
        int32_t id = -1;
        check(rt_server_add_scene(h_, scene.handle(), &id));
        return id;
    }
    int64_t Submit(const rt_job_desc& job) {
        int64_t id = -1;
        check(rt_server_submit(h_, &job, &id));
        return id;
    }
    rt_job_status Wait(int64_t job, double timeout_ms = -1.0) {
        rt_job_status st{};
        check(rt_server_wait(h_, job, timeout_ms, &st));
        return st;
    }
    rt_job_status Poll(int64_t job) {
        rt_job_status st{};
        check(rt_server_poll(h_, job, &st));
        return st;
    }
    void Cancel(int64_t job) { check(rt_server_cancel(h_, job)); }
    void DownloadPixels(int64_t job, uint32_t* pixels) { check(rt_server_download_rgba8(h_, job, pixels)); }
    void DownloadLinear(int64_t job, float* rgba) { check(rt_server_download(h_, job, rgba)); }
    void Release(int64_t job) { check(rt_server_release(h_, job)); }
    rt_server_stats Stats() {
        rt_server_stats st{};
        check(rt_server_get_stats(h_, &st));
        return st;
    }
    rt_server* handle() { return h_; }

private:
    rt_server* h_ = nullptr;
};

}  // namespace rt
