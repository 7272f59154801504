/*
 * rt_capi.h - C ABI of the B200 path tracer (optixrender_b200).
 *
 * This is the drop-in boundary for the reference renderer's host API
 * (GraphicsEnthusiast/OptiXRender).  Each entry point names the reference
 * interface it replaces as `file:line` inside that project.  All functions
 * return an rt_status (0 = RT_OK); nothing throws across the ABI and nothing
 * calls exit().  rt_last_error_message() returns a thread-local description of
 * the last failure on the calling thread.
 *
 * Pointers are plain host pointers unless a parameter says "device".  The
 * library copies everything it needs, so a scene may be destroyed once a
 * renderer has been created from it.
 */
#ifndef RT_CAPI_H
#define RT_CAPI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define RT_API __declspec(dllexport)
#else
#define RT_API __attribute__((visibility("default")))
#endif

typedef int32_t rt_status;

enum {
    RT_OK = 0,
    RT_ERR_INVALID_ARG = 1,
    RT_ERR_CUDA = 2,
    RT_ERR_OUT_OF_MEMORY = 3,
    RT_ERR_IO = 4,
    RT_ERR_PARSE = 5,
    RT_ERR_STATE = 6,
    RT_ERR_TIMEOUT = 7,
    RT_ERR_UNSUPPORTED = 8,
    RT_ERR_DEVICE_WATCHDOG = 9
};

/* ---------------------------------------------------------------------- */
/* Scene description types                                                 */
/* ---------------------------------------------------------------------- */

/* Material types; values match enum MaterialType, core/include/Scene.h:59-68. */
enum {
    RT_MAT_DIFFUSE = 0,
    RT_MAT_CONDUCTOR = 1,
    RT_MAT_DIELECTRIC = 2,
    RT_MAT_PLASTIC = 3,
    RT_MAT_METAL_WORKFLOW = 4,
    RT_MAT_THIN_DIELECTRIC = 5,
    RT_MAT_CLEARCOATED_CONDUCTOR = 6,
    RT_MAT_DIFFUSE_TRANSMITTER = 7
};

/* struct Material, core/include/Scene.h:70-116 (texture objects are replaced
 * by texture ids; the LUT pointers are owned by the renderer).  Call
 * rt_material_default() for the reference's field defaults. */
typedef struct rt_material {
    int32_t type;
    float albedo[3];
    float roughness;          /* reference units: alpha = roughness^2 */
    float anisotropy;
    float eta[3];
    float k[3];
    float int_ior;
    float ext_ior;
    int32_t nonlinear;
    float specular[3];
    float metallic;
    float coat_weight;
    float coat_roughness_u;
    float coat_roughness_v;
    /* texture ids (-1 = constant): albedo, roughness, anisotropy, specular,
     * metallic, coat_roughness_u, coat_roughness_v, normal */
    int32_t texture_ids[8];
} rt_material;

/* Light types: enum LightType, core/include/Scene.h:138-141, plus a point light. */
enum { RT_LIGHT_QUAD = 0, RT_LIGHT_SPHERE = 1, RT_LIGHT_POINT = 2 };

/* struct Light, core/include/Scene.h:143-155.  A quad emits towards
 * -normalize(cross(u, v)) unless double_side is set.  A point light uses
 * `radiance` as radiant intensity (W/sr) at `position`. */
typedef struct rt_light {
    int32_t type;
    int32_t double_side;
    float radiance[3];
    float position[3];
    float u[3];
    float v[3];
    float radius;
    int32_t medium;
} rt_light;

/* Phase types: enum PhaseType, core/include/Scene.h:33-36. */
enum { RT_PHASE_ISOTROPIC = 0, RT_PHASE_HENYEY_GREENSTEIN = 1 };
/* Medium types: enum MediumType, core/include/Scene.h:44-46, plus a density grid. */
enum { RT_MEDIUM_HOMOGENEOUS = 0, RT_MEDIUM_GRID = 1 };

/* struct Medium, core/include/Scene.h:48-55.  For RT_MEDIUM_GRID the
 * coefficients are multiplied by a trilinearly interpolated density read from
 * `density` (grid_res[0]*grid_res[1]*grid_res[2] floats, x fastest) over the
 * box [bounds_min, bounds_max]; outside the box the density is zero.  The grid
 * is tracked with delta tracking against a majorant grid of majorant_res^3
 * cells (0 = 8). */
typedef struct rt_medium {
    int32_t type;
    int32_t phase;
    float g[3];
    float sigma_s[3];
    float sigma_a[3];
    float scale;
    int32_t grid_res[3];
    int32_t majorant_res;
    float bounds_min[3];
    float bounds_max[3];
    const float* density;
} rt_medium;

/* One triangle mesh, the input of Scene::AddMesh (core/src/Scene.cpp:22-64,
 * TriangleMesh::LoadMesh core/src/Scene.cpp:83-179).  If `indices` is NULL the
 * positions are already de-indexed (3 vertices per triangle).  Missing normals
 * become the face normal and missing texcoords become (0,0),(1,0),(0,1), as
 * in Scene.cpp:150-165. */
typedef struct rt_mesh_desc {
    const float* positions;   /* 3 floats per vertex */
    const float* normals;     /* optional, 3 floats per vertex */
    const float* texcoords;   /* optional, 2 floats per vertex */
    const int32_t* indices;   /* optional, 3 per triangle */
    int64_t num_vertices;
    int64_t num_triangles;
} rt_mesh_desc;

/* struct Camera, core/include/Scene.h:11-20.  fov_y_deg <= 0 keeps the
 * reference's fixed screen height of 0.66 (core/src/Renderer.cpp:803). */
typedef struct rt_camera {
    float from[3];
    float at[3];
    float up[3];
    int32_t medium;
    float fov_y_deg;
} rt_camera;

/* enum FilterType, core/include/Scene.h:24-29. */
enum { RT_FILTER_BOX = 0, RT_FILTER_TENT = 1, RT_FILTER_TRIANGLE = 2, RT_FILTER_GAUSSIAN = 3 };
/* Random streams: RT_RNG_LCG is the reference's gdt::LCG<16> seeded per pixel
 * and frame (common/gdt/gdt/random/random.h:29-68), consumed sample after
 * sample; RT_RNG_PCG32 gives every (pixel, sample) path its own PCG32 stream. */
enum { RT_RNG_LCG = 0, RT_RNG_PCG32 = 1 };
/* Output mappings: the reference's luminance Reinhard + gamma 2.2
 * (core/cuda/PostProcessing.cu:18-48), ACES filmic + sRGB, or a plain clamp. */
enum { RT_TONEMAP_REINHARD = 0, RT_TONEMAP_ACES_SRGB = 1, RT_TONEMAP_CLAMP = 2 };

/* Renderer settings.  The reference keeps these in LaunchParams
 * (core/include/LaunchParams.h:28-69) and Renderer's public fields
 * (core/include/Renderer.h:139-143). */
typedef struct rt_options {
    int32_t width;
    int32_t height;
    int32_t spp;              /* numPixelSamples per Render() */
    int32_t max_depth;        /* maxBounce (reference default 25) */
    int32_t filter;           /* RT_FILTER_* (reference default Gaussian) */
    int32_t rng;              /* RT_RNG_* */
    int32_t rr_depth;         /* first bounce with Russian roulette (reference: 0) */
    int32_t progressive;      /* running mean over Render() calls */
    uint64_t seed;            /* PCG32 seed (ignored by RT_RNG_LCG) */
    int32_t tonemap;          /* RT_TONEMAP_* */
    int32_t wave_paths;       /* paths in flight per wave (0 = automatic: up to 2^26, at most a quarter of
                                 free device memory; at most 2^26) */
    int32_t collect_stats;    /* count rays, nodes and triangles */
    float exposure;           /* multiplier before tonemapping (1) */
    /* Learned proposal (PCG32 streams only): the first guide_train_spp samples
     * per pixel (counted over Render() calls) are rendered one sample per pixel
     * per wave, and after each of those waves the guiding network takes
     * guide_steps Adam steps on up to 2^18 radiance samples from it; from then
     * on the trained mixture is sampled with probability guide_prob at every
     * non-dielectric surface vertex and combined with BSDF sampling by
     * one-sample MIS, so the estimate stays unbiased. */
    int32_t guided;           /* 0: plain BSDF + NEE (the reference method) */
    int32_t guide_train_spp;  /* 32 */
    float guide_prob;         /* 0.5 */
    int32_t guide_steps;      /* 4 */
    int32_t bvh_build;        /* RT_BVH_GPU (default): built on the device; RT_BVH_HOST: on the host */
    /* Renderer::denoiserOn (core/include/Renderer.h:139, off by default): the
     * displayed image (RGBA8) is the denoised colour; the accumulated colour
     * stays noisy and RT_AOV_DENOISED downloads the denoised linear colour. */
    int32_t denoise;
} rt_options;

/* Per-render statistics. */
typedef struct rt_render_stats {
    int64_t paths;
    int64_t extend_rays;
    int64_t shadow_rays;
    int64_t nodes_visited;     /* wide nodes fetched, extend + shadow */
    int64_t tris_tested;
    int64_t extend_nodes;
    int64_t extend_tris;
    int64_t nan_samples;       /* samples dropped for a NaN radiance */
    int32_t waves;
    int32_t launches;          /* kernels launched by the last Render() */
    float ms_total;            /* device time of the last Render() */
    float ms_extend;           /* per-kernel device time (collect_stats only) */
    float ms_shade;
    float ms_shadow;
    float ms_other;
    int64_t extend_launches;
    int64_t nan_throughput_paths; /* paths ended by IsNan(history), devicePrograms.cu:487-489 */
    int64_t wave_paths;        /* path slots per wave of the last Render() */
    int64_t h2d_bytes;         /* bytes copied host to device by the last Render() */
    int64_t watchdog_walks;    /* grid-medium walks that hit the device step budget (see rt_renderer_synchronize) */
    int64_t stack_overflows;   /* traversal node groups that found the stack full (0 unless the BVH depth check fails) */
    float ms_sample;           /* per-kernel device time of BSDF sampling (k_sample; collect_stats only) */
    float pad;
} rt_render_stats;

/* AOV kinds for rt_renderer_download_aov. */
enum { RT_AOV_COLOR = 0, RT_AOV_ALBEDO = 1, RT_AOV_NORMAL = 2, RT_AOV_DENOISED = 3 };

typedef struct rt_scene rt_scene;
typedef struct rt_renderer rt_renderer;

/* ---------------------------------------------------------------------- */
/* Library                                                                 */
/* ---------------------------------------------------------------------- */

RT_API const char* rt_last_error_message(void);
RT_API int32_t rt_version(void);

/* Field defaults of Material (Scene.h:70-116), Light (Scene.h:143-155),
 * Medium (Scene.h:48-55), Camera, and LaunchParams (LaunchParams.h:28-69). */
RT_API void rt_material_default(rt_material* m);
RT_API void rt_light_default(rt_light* l);
RT_API void rt_medium_default(rt_medium* m);
RT_API void rt_camera_default(rt_camera* c);
RT_API void rt_options_default(rt_options* o);

/* ---------------------------------------------------------------------- */
/* Scene: replaces class Scene, core/include/Scene.h:195-214               */
/* ---------------------------------------------------------------------- */

/* Scene::Scene() */
RT_API rt_status rt_scene_create(rt_scene** out);
/* Scene::~Scene(), core/src/Scene.cpp:10-20 */
RT_API rt_status rt_scene_destroy(rt_scene* s);
/* Scene::AddMesh, core/src/Scene.cpp:22-64 (the material is copied per mesh
 * as in the reference's hit records, core/src/Renderer.cpp:590). */
RT_API rt_status rt_scene_add_mesh(rt_scene* s, const rt_mesh_desc* mesh, const rt_material* material,
                                   int32_t out_medium, int32_t in_medium, int32_t* out_mesh_id);
/* Scene::AddMesh with an OBJ path (TriangleMesh::LoadMesh, Scene.cpp:83-179). */
RT_API rt_status rt_scene_add_mesh_obj(rt_scene* s, const char* obj_path, const rt_material* material,
                                       int32_t out_medium, int32_t in_medium, int32_t* out_mesh_id);
/* Scene::AddLight, core/src/Scene.cpp:71-73 */
RT_API rt_status rt_scene_add_light(rt_scene* s, const rt_light* light);
/* Scene::AddMedium, core/src/Scene.cpp:75-77 (grid media copy `density`). */
RT_API rt_status rt_scene_add_medium(rt_scene* s, const rt_medium* medium);
/* Scene::AddTexture, core/src/Scene.cpp:66-69 + Texture, Scene.cpp:181-189:
 * an RGBA8 image (w*h*4 bytes, row 0 = bottom, i.e. v = 0, as stbi's
 * vertical flip gives).  Materials refer to it by the returned id in
 * rt_material.texture_ids; it is sampled as the reference's tex2D (normalized
 * coordinates, wrap, bilinear, texels read as byte/255). */
RT_API rt_status rt_scene_add_texture(rt_scene* s, const uint8_t* rgba, int32_t width, int32_t height,
                                      int32_t* texture_id);
/* Scene::AddTexture(fileName), core/src/Scene.cpp:66-69 (stbi_load): PNG
 * (not interlaced; grey, RGB, palette, grey+alpha, RGBA at 1-16 bits),
 * uncompressed BMP (8/24/32-bit) or binary PGM/PPM (P5/P6), flipped so that
 * row 0 is the bottom. */
RT_API rt_status rt_scene_add_texture_file(rt_scene* s, const char* path, int32_t* texture_id);
/* Size of texture `texture_id` and, when `rgba` is not NULL, its texels as stored. */
RT_API rt_status rt_scene_get_texture(const rt_scene* s, int32_t texture_id, int32_t* width, int32_t* height,
                                      uint8_t* rgba);
/* Scene::AddEnv, core/src/Scene.cpp:79-81 + HdrTexture, Scene.cpp:197-313:
 * an equirectangular RGBA float image (w*h*4 floats, row 0 = bottom) scaled
 * by `scale`; the sampling cache is built as in CalculateHdrCache. */
RT_API rt_status rt_scene_set_env(rt_scene* s, const float* rgba, int32_t width, int32_t height, float scale);
/* Scene::AddEnv(const std::string& fileName), core/src/Scene.cpp:79-81 with
 * HdrTexture's loader (Scene.cpp:197-206: stbi_loadf, rows flipped so row 0
 * is the bottom): a Radiance .hdr file as floats, or a PNG / baseline JPEG /
 * BMP / PGM / PPM image converted as stbi_loadf does (colour (v/255)^2.2,
 * alpha v/255), scaled by `scale`.  Unreadable files give RT_ERR_IO (the
 * reference leaves the scene without an environment). */
RT_API rt_status rt_scene_set_env_file(rt_scene* s, const char* path, float scale);
/* The scene's environment image (width*height*4 floats, row 0 = bottom, scale
 * applied); `rgba` may be NULL to query the size (0 x 0: no environment). */
RT_API rt_status rt_scene_get_env(const rt_scene* s, float* rgba, int32_t* width, int32_t* height);
/* Scene::bounds, core/include/Scene.h:213 */
RT_API rt_status rt_scene_get_bounds(const rt_scene* s, float lo[3], float hi[3]);
RT_API rt_status rt_scene_counts(const rt_scene* s, int64_t* triangles, int32_t* meshes, int32_t* lights,
                                 int32_t* media);
enum { RT_BVH_GPU = 0, RT_BVH_HOST = 1 };
/* Deepest wide BVH (levels) the traversal stack holds; deeper trees are
 * rejected with RT_ERR_UNSUPPORTED by the builds below and by renderers and
 * servers when they upload a scene. */
enum { RT_MAX_BVH_DEPTH = 32 };

/* The same acceleration structure built on the current device (binned SAH on
 * all SMs, then the collapse), copied back and validated on the host. */
RT_API rt_status rt_scene_build_bvh_gpu(const rt_scene* s, int64_t* num_nodes, int32_t* depth);
/* Builds the acceleration structure (the work of optixAccelBuild,
 * core/src/Renderer.cpp:146-285) on the host and validates it: every child and
 * triangle index in range, every quantised box containing what it bounds.
 * Needs no device.  `num_nodes` and `depth` are written also when the tree is
 * rejected for being deeper than RT_MAX_BVH_DEPTH. */
RT_API rt_status rt_scene_build_bvh(const rt_scene* s, int64_t* num_nodes, int32_t* depth);
/* SceneParser::LoadFromJson, core/src/SceneParser.cpp:3-23 and the schema of
 * models/test.json.  Fills `opts`/`cam` (may be NULL) from the file. */
RT_API rt_status rt_scene_load_json(rt_scene* s, const char* path, rt_options* opts, rt_camera* cam);
RT_API rt_status rt_scene_load_json_string(rt_scene* s, const char* json, const char* base_dir,
                                           rt_options* opts, rt_camera* cam);

/* ---------------------------------------------------------------------- */
/* Renderer: replaces class Renderer, core/include/Renderer.h:9-187        */
/* ---------------------------------------------------------------------- */

/* Renderer::Renderer(const Scene*), core/src/Renderer.cpp:39-93: builds the
 * acceleration structure on the current CUDA device and uploads the scene. */
RT_API rt_status rt_renderer_create(const rt_scene* s, const rt_options* opts, rt_renderer** out);
RT_API rt_status rt_renderer_destroy(rt_renderer* r);
/* Public LaunchParams fields (numPixelSamples, maxBounce, filterType) and
 * Renderer::progressive; changing them does not reset accumulation. */
RT_API rt_status rt_renderer_set_options(rt_renderer* r, const rt_options* opts);
RT_API rt_status rt_renderer_get_options(const rt_renderer* r, rt_options* opts);
/* Renderer::Resize, core/src/Renderer.cpp:816-875 */
RT_API rt_status rt_renderer_resize(rt_renderer* r, int32_t width, int32_t height);
/* Renderer::SetCamera, core/src/Renderer.cpp:796-813 (resets accumulation) */
RT_API rt_status rt_renderer_set_camera(rt_renderer* r, const rt_camera* cam);
/* Use an external CUDA stream (cudaStream_t) for all work; NULL = own stream. */
RT_API rt_status rt_renderer_set_stream(rt_renderer* r, void* cuda_stream);
/* Renderer::Render, core/src/Renderer.cpp:635-793: one launch of `spp`
 * samples per pixel, running-mean accumulation when progressive, and the
 * tonemap of core/cuda/PostProcessing.cu:50-59.  Asynchronous. */
RT_API rt_status rt_renderer_render(rt_renderer* r);
/* Waits for the renderer's work.  RT_ERR_DEVICE_WATCHDOG: some walk through
 * a grid medium in the last render exhausted the device's step budget (4096
 * tentative collisions) and was ended with zero weight; the image is complete
 * but those samples are missing (the reference's equivalent is a hung or
 * timed-out launch).  The same status reports traversals that found their
 * 32-entry stack full (rt_render_stats.stack_overflows; renderers reject
 * BVHs deeper than RT_MAX_BVH_DEPTH, so this stays zero). */
RT_API rt_status rt_renderer_synchronize(rt_renderer* r);
/* Renderer::DownloadPixels, core/src/Renderer.cpp:878-880 (RGBA8). */
RT_API rt_status rt_renderer_download_rgba8(rt_renderer* r, uint32_t* pixels);
/* Headless replacement of the GL blit: the float4 colour buffer. */
RT_API rt_status rt_renderer_download_linear(rt_renderer* r, float* rgba);
/* The albedo / normal AOVs the reference feeds its denoiser
 * (core/cuda/devicePrograms.cu:518-531). */
RT_API rt_status rt_renderer_download_aov(rt_renderer* r, int32_t kind, float* rgba);
/* The denoiser of rt_options.denoise on caller buffers (host pointers, w*h*4
 * floats each; row 0 = bottom): colour and its first-hit albedo and normal
 * AOVs in, denoised linear colour out.  Replaces optixDenoiserInvoke
 * (core/src/Renderer.cpp:756) with an edge-avoiding a-trous wavelet filter;
 * synchronous; allocates its device buffers. */
/* Writes an RGBA8 frame (DownloadPixels layout, row 0 = bottom) as a PNG
 * file: the screenshot the reference's viewer saves (main.cpp:82-85). */
RT_API rt_status rt_write_png(const char* path, const uint32_t* rgba8, int32_t width, int32_t height);
RT_API rt_status rt_denoise_image(const float* color, const float* albedo, const float* normal, int32_t width,
                                  int32_t height, float* out);
/* Device pointers of the float4 colour buffer and the RGBA8 buffer. */
RT_API rt_status rt_renderer_device_buffers(rt_renderer* r, void** color_f32x4, void** rgba8);
RT_API rt_status rt_renderer_get_stats(const rt_renderer* r, rt_render_stats* stats);
/* Frame counter of progressive accumulation (LaunchParams::frame.frameID). */
RT_API rt_status rt_renderer_frame_index(const rt_renderer* r, int32_t* frame);

/* The renderer's guiding network, created on first use; it stays owned by
 * the renderer.  Positions it takes are normalised to the scene bounds grown
 * by 1% on each side. */
typedef struct rt_guide rt_guide;
RT_API rt_status rt_renderer_guide(rt_renderer* r, rt_guide** guide);
/* Training samples collected by the last training wave: `count` of them, up to
 * `max_samples` copied as 8 floats each (network input position, weight,
 * direction, 1). */
RT_API rt_status rt_renderer_guide_samples(rt_renderer* r, float* out, int64_t max_samples, int64_t* count);

/* Ray queries against the renderer's scene: the equivalent of optixTrace,
 * core/cuda/devicePrograms.cu:258-269 (closest hit) and :303-319 (shadow /
 * any hit, terminate on first hit).  rays: n x 8 floats (ox oy oz tmin dx dy dz
 * tmax).  hits: n x 4 floats (t, u, v, primitive id as float bits; id -1 on a
 * miss).  For any-hit queries hits[i*4+3] holds 1 (occluded) or -1 bits.
 * `device_ptrs` nonzero means both buffers are device memory. */
RT_API rt_status rt_renderer_trace(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n, float* hits,
                                   int32_t device_ptrs);

/* The queries of rt_renderer_trace (host buffers), answered by the path
 * tracer's own persistent traversal kernels instead of a one-thread-per-ray
 * kernel: the batch becomes the extend queue (closest hit) or the shadow
 * queue (any hit) of a one-bounce wave, and the kernels Render() launches for
 * devicePrograms.cu:258-269 and :303-319 run on it with the same launch
 * shape, lane refill and triangle postponing.  Every ray must have tmin =
 * 1e-4 (EPS, core/cuda/Utils.h:10, the offset of every ray the integrator
 * traces) and closest-hit rays tmax = FLT_MAX or +inf (the extend kernel's
 * extent); any-hit rays keep their own tmax.  Other extents give
 * RT_ERR_INVALID_ARG.  hits: as rt_renderer_trace for closest hits; an
 * occluded any-hit ray gives (0, 0, 0, 1 bits), a miss (FLT_MAX, 0, 0, -1
 * bits).  `counters` (NULL, or 3 values) receives rays traced, wide nodes
 * visited and triangles tested, counted by the instrumented build of the same
 * kernel (the one rt_options.collect_stats renders with).  Batches above 2^22
 * rays run as several waves.  Returns after the hits are in `hits`. */
RT_API rt_status rt_renderer_trace_wavefront(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n,
                                             float* hits, int64_t* counters);

/* rt_renderer_trace with host buffers, for callers that must not allocate
 * device memory during the call (no counterpart in the reference).
 * cudaMalloc and cudaFree, which rt_renderer_trace uses for its per-call
 * buffers, can synchronise the whole device, stalling a render or serving
 * loop's other streams, and they fail once the caller has taken the remaining
 * device memory for its own pool.  This call allocates nothing: the rays and
 * hits pass through one fixed device array per device (65,536 rays, 3 MiB),
 * and larger batches are rejected with RT_ERR_INVALID_ARG.  Nothing in the
 * array needs to start at zero.  Every call works on the array of the
 * renderer's own device (the device it was created on), whichever device is
 * current on the calling thread, and looks up the array's address there
 * (cudaGetSymbolAddress, which allocates nothing); the first call on a device
 * may also load the library's kernels onto it, so make that first call
 * outside any stream capture.  Calls on one device share the array: calls
 * that overlap in time (several host threads, or several renderers on one
 * device) race on it and may return each other's hits, so serialise them.
 * Returns after the hits are in `hits` (the renderer's stream is
 * synchronised). */
RT_API rt_status rt_renderer_trace_noalloc(rt_renderer* r, int32_t any_hit, const float* rays, int64_t n,
                                           float* hits);

/* ---------------------------------------------------------------------- */
/* Path-guiding network (no counterpart in the reference): a multiresolution */
/* hash encoding of the position (16 levels x 2 features, 2^19 entries per   */
/* level) feeding a 32-64-64-64-32 MLP (FP16 weights, FP32 accumulation)      */
/* whose outputs are an 8-lobe von Mises-Fisher mixture over directions.     */
/* These calls expose the network on host buffers; the renderer trains and   */
/* queries it on device buffers when rt_options.guided is set.               */
/* ---------------------------------------------------------------------- */

typedef struct rt_guide_options {
    float learning_rate;       /* Adam step size (1e-2) */
    int32_t max_resolution;    /* grid resolution of the finest level (64); the coarsest is min(16, it) */
    uint64_t seed;             /* parameter initialisation */
    float max_log_kappa;       /* log of the highest lobe concentration (4) */
    int32_t pad;
} rt_guide_options;

RT_API void rt_guide_options_default(rt_guide_options* o);
RT_API rt_status rt_guide_create(const rt_guide_options* o, rt_guide** out);
RT_API rt_status rt_guide_destroy(rt_guide* g);
/* Parameter counts: hash table (levels x 2^19 x 2 floats, level-major) and MLP
 * (W0 64x32, W1 64x64, W2 64x64, W3 32x64, each row-major [out][in]). */
RT_API void rt_guide_sizes(int64_t* table_params, int64_t* mlp_params);
RT_API rt_status rt_guide_get_params(const rt_guide* g, float* table, float* mlp);
RT_API rt_status rt_guide_set_params(rt_guide* g, const float* table, const float* mlp);
/* Raw outputs (n x 32) of positions in [0,1]^3 (n x 3). */
RT_API rt_status rt_guide_forward(rt_guide* g, const float* pos, int64_t n, float* raw);
/* Loss (1/n) sum_i -weight_i log q(dir_i | pos_i) and its gradients (the
 * gradients are not applied). */
RT_API rt_status rt_guide_gradients(rt_guide* g, const float* pos, const float* dir, const float* weight, int64_t n,
                                    float* loss, float* grad_table, float* grad_mlp);
/* One Adam step on the loss with the weights normalised to sum 1. */
RT_API rt_status rt_guide_train_step(rt_guide* g, const float* pos, const float* dir, const float* weight, int64_t n,
                                     float* loss);
/* Learning rate, finest grid resolution and highest log-concentration; a
 * value <= 0 (0 for the concentration) keeps the current one.  The hash table
 * is kept, so a new resolution re-indexes the trained features. */
RT_API rt_status rt_guide_set_hyperparameters(rt_guide* g, float learning_rate, int32_t max_resolution,
                                              float max_log_kappa);
/* Loss of the last training step and the number of steps taken. */
RT_API rt_status rt_guide_last_loss(rt_guide* g, float* loss, int64_t* steps);
/* Mixture pdf at (pos, dir) pairs; with `u` (n x 3 uniforms) instead, samples
 * directions into `out_dir` and returns their pdf. */
RT_API rt_status rt_guide_pdf(rt_guide* g, const float* pos, const float* dir, const float* u, int64_t n,
                              float* out_dir, float* pdf);

/* ---------------------------------------------------------------------- */
/* Serving: many render jobs batched into shared wavefront launches         */
/* (no counterpart in the reference, which renders one frame at a time).    */
/* ---------------------------------------------------------------------- */

typedef struct rt_server rt_server;

typedef struct rt_server_options {
    int64_t hbm_budget_bytes;  /* device memory for resident scenes + admitted jobs (0 = 80% of free) */
    int32_t wave_paths;        /* paths per shared wave (0 = 2^23) */
    int32_t max_jobs;          /* jobs resident at once (<= 256; 0 = 256) */
    int32_t max_depth;         /* bounce budget of the shared launches (>= every job's max_depth; 0 = 32) */
    int32_t background;        /* nonzero: a server thread runs the loop; zero: call rt_server_step */
    int32_t waves_in_flight;   /* waves queued ahead on the device (0 = 2) */
    int32_t policy;            /* RT_SERVE_FAIR (default), RT_SERVE_FIFO or RT_SERVE_SRPT */
    /* Guided jobs (rt_job_desc.guided): each resident scene has one guiding
     * network, trained on the scene's first guide_train_waves guided waves
     * (guide_steps Adam steps after each) and then shared by every guided
     * job on that scene. */
    int32_t guide_train_waves; /* 0 = 32 */
    int32_t guide_steps;       /* 0 = 4 */
    float guide_prob;          /* probability of sampling the mixture (0 = 0.5) */
    int32_t pad;
} rt_server_options;

/* How a wave's path slots are split among admitted jobs.  FAIR: up to 16 jobs,
 * taken round-robin, share each wave evenly (latency grows with job size).
 * FIFO: the oldest job takes all it can.  SRPT: the jobs with the fewest paths
 * left go first (shortest remaining work; lowest mean time-to-image).
 * A wave holds either plain jobs (of any scenes) or the guided jobs of one
 * scene; the policy also picks which of these groups the next wave serves. */
enum { RT_SERVE_FAIR = 0, RT_SERVE_FIFO = 1, RT_SERVE_SRPT = 2 };

/* One request: a resident scene, a camera and the renderer settings of one
 * Render() (PCG32 streams seeded by `seed`). */
typedef struct rt_job_desc {
    int32_t scene;
    rt_camera camera;
    int32_t width, height, spp, max_depth, rr_depth, filter, tonemap;
    uint64_t seed;
    float exposure;
    int32_t guided;            /* nonzero: sample with the scene's guiding network (unbiased; the
                                  image then depends on the network's training, not only on seed) */
} rt_job_desc;

enum { RT_JOB_QUEUED = 0, RT_JOB_RUNNING = 1, RT_JOB_DONE = 2, RT_JOB_FAILED = 3, RT_JOB_CANCELLED = 4 };

typedef struct rt_job_status {
    int32_t state;
    int32_t pad;
    double submit_ms;          /* host clock (ms since server creation) */
    double admit_ms;
    double done_ms;            /* time the finished image was observed ready */
    int64_t paths;
    int64_t bytes;             /* device bytes held while admitted */
} rt_job_status;

typedef struct rt_server_stats {
    int64_t jobs_submitted, jobs_done, jobs_queued, jobs_running;
    int64_t waves, paths;
    int64_t bytes_in_use, bytes_budget;
    int32_t max_segments_in_a_wave;
    int32_t device;            /* the CUDA device the server was created on (and works on) */
    double busy_ms;            /* device time of the finished waves (CUDA events) */
    double mean_wave_depth;    /* bounces launched per wave, averaged */
    int64_t guided_waves;      /* waves of guided jobs, training waves included */
    int64_t training_waves;    /* guided waves followed by training steps */
    int32_t worker_device;     /* current device of the background thread (-1: manual mode or not started) */
    int32_t pad;
} rt_server_stats;

RT_API void rt_server_options_default(rt_server_options* o);
RT_API rt_status rt_server_create(const rt_server_options* o, rt_server** out);
RT_API rt_status rt_server_destroy(rt_server* s);
/* Uploads a scene (BVH, triangles, materials, media, environment) and keeps it resident. */
RT_API rt_status rt_server_add_scene(rt_server* s, const rt_scene* scene, int32_t* scene_id);
RT_API rt_status rt_server_submit(rt_server* s, const rt_job_desc* job, int64_t* job_id);
RT_API rt_status rt_server_cancel(rt_server* s, int64_t job_id);
RT_API rt_status rt_server_poll(rt_server* s, int64_t job_id, rt_job_status* st);
/* Waits until the job is done (or timeout_ms passes; < 0 = forever); RT_ERR_TIMEOUT on expiry. */
RT_API rt_status rt_server_wait(rt_server* s, int64_t job_id, double timeout_ms, rt_job_status* st);
/* Float RGBA image of a finished job (width*height*4). */
RT_API rt_status rt_server_download(rt_server* s, int64_t job_id, float* rgba);
/* Tonemapped RGBA8 image of a finished job (width*height words). */
RT_API rt_status rt_server_download_rgba8(rt_server* s, int64_t job_id, uint32_t* pixels);
/* Frees a finished (or queued) job and forgets its id. */
RT_API rt_status rt_server_release(rt_server* s, int64_t job_id);
/* Manual mode: admits, issues one wave and retires finished jobs; *did_work = 0 when idle. */
RT_API rt_status rt_server_step(rt_server* s, int32_t* did_work);
RT_API rt_status rt_server_get_stats(rt_server* s, rt_server_stats* st);

/* ---------------------------------------------------------------------- */
/* Shading verification: runs the renderer's device shading code on         */
/* batches so it can be compared with a CPU oracle.                         */
/* ---------------------------------------------------------------------- */

enum {
    /* EvaluateMaterial, core/cuda/Material.h:783-813.
     * in: 16 floats/query: N[3] V[3] L[3] front_face material_index pad[5]
     * out: 8 floats: f[3] pdf pad[4] */
    RT_VERIFY_BSDF_EVAL = 0,
    /* SampleMaterial, core/cuda/Material.h:815-845, random numbers taken
     * from the query in order.
     * in: 16 floats: N[3] V[3] u[6] front_face material_index pad[2]
     * out: 8 floats: f[3] pdf L[3] used_randoms */
    RT_VERIFY_BSDF_SAMPLE = 1,
    /* SampleLight, core/cuda/Light.h:158-168 (+ point light).
     * in: 16 floats: P[3] u[2] light_index pad[10]
     * out: 8 floats: Li[3] pdf L[3] distance */
    RT_VERIFY_LIGHT_SAMPLE = 2,
    /* EvaluateLight, core/cuda/Light.h:145-156.
     * in: 16 floats: O[3] D[3] max_distance light_index pad[8]
     * out: 8 floats: Li[3] pdf distance pad[3] */
    RT_VERIFY_LIGHT_EVAL = 3,
    /* SampleMediumDistance, core/cuda/Medium.h:233-244 (homogeneous).
     * in: 16 floats: max_distance u[2] medium_index pad[12]
     * out: 8 floats: transmittance[3] trans_pdf distance scattered used pad */
    RT_VERIFY_MEDIUM_SAMPLE = 4,
    /* SamplePhase, core/cuda/Medium.h:96-108.
     * in: 16 floats: V[3] u[4] medium_index pad[8]
     * out: 8 floats: attenuation[3] pdf L[3] used_randoms */
    RT_VERIFY_PHASE_SAMPLE = 5,
    /* EvaluatePhase, core/cuda/Medium.h:83-94.
     * in: 16 floats: V[3] L[3] medium_index pad[9]
     * out: 8 floats: attenuation[3] pdf pad[4] */
    RT_VERIFY_PHASE_EVAL = 6,
    /* What guided sampling mixes with its proposal: the real density of the
     * directions SampleMaterial draws, at L (the reported pdfs use the
     * reference's isotropic GGX D with cos^2 for cos^4, and plastic and the
     * clear-coated conductor select lobes by a Fresnel term of V), the pdf
     * EvaluateMaterial and the sampler report there, and f_dir, what plain
     * BSDF sampling integrates at L.
     * in: 16 floats: N[3] V[3] L[3] front_face material_index pad[5]
     * out: 8 floats: sampling_density evaluate_pdf sampler_reported_pdf f_dir[3] pad[2] */
    RT_VERIFY_BSDF_SAMPLE_PDF = 7
};

/* Runs one verification op over n queries on the device.  `materials`,
 * `lights` and `media` are host arrays indexed by the queries. */
RT_API rt_status rt_verify_shading(int32_t op, const rt_material* materials, int32_t num_materials,
                                   const rt_light* lights, int32_t num_lights, const rt_medium* media,
                                   int32_t num_media, const float* in, int64_t n, float* out);
/* ComputeKullaConty, core/cuda/Microfacet.h:231-291, as the renderer builds
 * it: 64*64 floats of E(mu, alpha) and 64 floats of E_avg. */
RT_API rt_status rt_kulla_conty_lut(float* bsdf_avg, float* albedo_avg);
/* HdrTexture::CalculateHdrCache, core/src/Scene.cpp:217-313, as the renderer
 * builds it: w*h*4 floats (sample x, sample y, pdf, 0). */
RT_API rt_status rt_env_sampling_cache(const float* rgba, int32_t width, int32_t height, float* cache);

#ifdef __cplusplus
}
#endif

#endif /* RT_CAPI_H */
