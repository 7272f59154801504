"""B200 path tracer: Python bindings of the C ABI (include/rt_capi.h).

The classes mirror the reference renderer's host API
(GraphicsEnthusiast/OptiXRender): ``Scene`` follows core/include/Scene.h
(AddMesh, AddLight, AddMedium, AddEnv) and ``Renderer`` follows
core/include/Renderer.h (Render, Resize, SetCamera, DownloadPixels).  All
rendering runs in the in-tree CUDA library ``_lib/liboptixrender_b200.so``;
there is no CPU fallback, and importing the package fails if the library is
missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIBRARY_PATH = _PKG / "_lib" / "liboptixrender_b200.so"

# ---------------------------------------------------------------- constants
RT_OK = 0
(RT_ERR_INVALID_ARG, RT_ERR_CUDA, RT_ERR_OUT_OF_MEMORY, RT_ERR_IO, RT_ERR_PARSE, RT_ERR_STATE, RT_ERR_TIMEOUT,
 RT_ERR_UNSUPPORTED, RT_ERR_DEVICE_WATCHDOG) = range(1, 10)
MAT_DIFFUSE, MAT_CONDUCTOR, MAT_DIELECTRIC, MAT_PLASTIC = 0, 1, 2, 3
MAT_METAL_WORKFLOW, MAT_THIN_DIELECTRIC, MAT_CLEARCOATED_CONDUCTOR, MAT_DIFFUSE_TRANSMITTER = 4, 5, 6, 7
LIGHT_QUAD, LIGHT_SPHERE, LIGHT_POINT = 0, 1, 2
PHASE_ISOTROPIC, PHASE_HG = 0, 1
MEDIUM_HOMOGENEOUS, MEDIUM_GRID = 0, 1
FILTER_BOX, FILTER_TENT, FILTER_TRIANGLE, FILTER_GAUSSIAN = 0, 1, 2, 3
RNG_LCG, RNG_PCG32 = 0, 1
BVH_GPU, BVH_HOST = 0, 1
TONEMAP_REINHARD, TONEMAP_ACES_SRGB, TONEMAP_CLAMP = 0, 1, 2
AOV_COLOR, AOV_ALBEDO, AOV_NORMAL, AOV_DENOISED = 0, 1, 2, 3
VERIFY_BSDF_EVAL, VERIFY_BSDF_SAMPLE, VERIFY_LIGHT_SAMPLE, VERIFY_LIGHT_EVAL = 0, 1, 2, 3
VERIFY_MEDIUM_SAMPLE, VERIFY_PHASE_SAMPLE, VERIFY_PHASE_EVAL, VERIFY_BSDF_SAMPLE_PDF = 4, 5, 6, 7

F3 = C.c_float * 3


class Material(C.Structure):
    """struct Material, core/include/Scene.h:70-116 (rt_material)."""
    _fields_ = [("type", C.c_int32), ("albedo", F3), ("roughness", C.c_float), ("anisotropy", C.c_float),
                ("eta", F3), ("k", F3), ("int_ior", C.c_float), ("ext_ior", C.c_float), ("nonlinear", C.c_int32),
                ("specular", F3), ("metallic", C.c_float), ("coat_weight", C.c_float),
                ("coat_roughness_u", C.c_float), ("coat_roughness_v", C.c_float), ("texture_ids", C.c_int32 * 8)]


class Light(C.Structure):
    """struct Light, core/include/Scene.h:143-155 (rt_light)."""
    _fields_ = [("type", C.c_int32), ("double_side", C.c_int32), ("radiance", F3), ("position", F3), ("u", F3),
                ("v", F3), ("radius", C.c_float), ("medium", C.c_int32)]


class Medium(C.Structure):
    """struct Medium, core/include/Scene.h:48-55 (rt_medium) plus the density grid."""
    _fields_ = [("type", C.c_int32), ("phase", C.c_int32), ("g", F3), ("sigma_s", F3), ("sigma_a", F3),
                ("scale", C.c_float), ("grid_res", C.c_int32 * 3), ("majorant_res", C.c_int32),
                ("bounds_min", F3), ("bounds_max", F3), ("density", C.POINTER(C.c_float))]


class MeshDesc(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("texcoords", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_int32)),
                ("num_vertices", C.c_int64), ("num_triangles", C.c_int64)]


class Camera(C.Structure):
    """struct Camera, core/include/Scene.h:11-20 (rt_camera)."""
    _fields_ = [("from_", F3), ("at", F3), ("up", F3), ("medium", C.c_int32), ("fov_y_deg", C.c_float)]


class Options(C.Structure):
    """LaunchParams settings, core/include/LaunchParams.h:28-69 (rt_options)."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("filter", C.c_int32), ("rng", C.c_int32), ("rr_depth", C.c_int32), ("progressive", C.c_int32),
                ("seed", C.c_uint64), ("tonemap", C.c_int32), ("wave_paths", C.c_int32),
                ("collect_stats", C.c_int32), ("exposure", C.c_float), ("guided", C.c_int32),
                ("guide_train_spp", C.c_int32), ("guide_prob", C.c_float), ("guide_steps", C.c_int32),
                ("bvh_build", C.c_int32), ("denoise", C.c_int32)]


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_int64), ("extend_rays", C.c_int64), ("shadow_rays", C.c_int64),
                ("nodes_visited", C.c_int64), ("tris_tested", C.c_int64), ("extend_nodes", C.c_int64),
                ("extend_tris", C.c_int64), ("nan_samples", C.c_int64), ("waves", C.c_int32),
                ("launches", C.c_int32), ("ms_total", C.c_float), ("ms_extend", C.c_float),
                ("ms_shade", C.c_float), ("ms_shadow", C.c_float), ("ms_other", C.c_float),
                ("extend_launches", C.c_int64), ("nan_throughput_paths", C.c_int64), ("wave_paths", C.c_int64),
                ("h2d_bytes", C.c_int64), ("watchdog_walks", C.c_int64), ("stack_overflows", C.c_int64),
                ("ms_sample", C.c_float), ("pad", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("wave_paths", C.c_int32), ("max_jobs", C.c_int32),
                ("max_depth", C.c_int32), ("background", C.c_int32), ("waves_in_flight", C.c_int32),
                ("policy", C.c_int32), ("guide_train_waves", C.c_int32), ("guide_steps", C.c_int32),
                ("guide_prob", C.c_float), ("pad", C.c_int32)]


class JobDesc(C.Structure):
    _fields_ = [("scene", C.c_int32), ("camera", Camera), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("max_depth", C.c_int32), ("rr_depth", C.c_int32), ("filter", C.c_int32),
                ("tonemap", C.c_int32), ("seed", C.c_uint64), ("exposure", C.c_float), ("guided", C.c_int32)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4
SERVE_FAIR, SERVE_FIFO, SERVE_SRPT = 0, 1, 2


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("pad", C.c_int32), ("submit_ms", C.c_double), ("admit_ms", C.c_double),
                ("done_ms", C.c_double), ("paths", C.c_int64), ("bytes", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_int64), ("jobs_done", C.c_int64), ("jobs_queued", C.c_int64),
                ("jobs_running", C.c_int64), ("waves", C.c_int64), ("paths", C.c_int64),
                ("bytes_in_use", C.c_int64), ("bytes_budget", C.c_int64), ("max_segments_in_a_wave", C.c_int32),
                ("device", C.c_int32), ("busy_ms", C.c_double), ("mean_wave_depth", C.c_double),
                ("guided_waves", C.c_int64), ("training_waves", C.c_int64), ("worker_device", C.c_int32),
                ("pad", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class GuideOptions(C.Structure):
    _fields_ = [("learning_rate", C.c_float), ("max_resolution", C.c_int32), ("seed", C.c_uint64),
                ("max_log_kappa", C.c_float), ("pad", C.c_int32)]


class RTError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rt error {code}: {msg}")
        self.code = code


_lib = None


def load_library():
    """Loads the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise ImportError(f"{LIBRARY_PATH} is missing: run `python -m optixrender_b200.build` (no CPU fallback)")
    lib = C.CDLL(str(LIBRARY_PATH))
    P, I32, I64, F, VP = C.POINTER, C.c_int32, C.c_int64, C.c_float, C.c_void_p
    sig = {
        "rt_last_error_message": (C.c_char_p, []),
        "rt_version": (I32, []),
        "rt_material_default": (None, [P(Material)]),
        "rt_light_default": (None, [P(Light)]),
        "rt_medium_default": (None, [P(Medium)]),
        "rt_camera_default": (None, [P(Camera)]),
        "rt_options_default": (None, [P(Options)]),
        "rt_scene_create": (I32, [P(VP)]),
        "rt_scene_destroy": (I32, [VP]),
        "rt_scene_add_mesh": (I32, [VP, P(MeshDesc), P(Material), I32, I32, P(I32)]),
        "rt_scene_add_mesh_obj": (I32, [VP, C.c_char_p, P(Material), I32, I32, P(I32)]),
        "rt_scene_add_light": (I32, [VP, P(Light)]),
        "rt_scene_add_medium": (I32, [VP, P(Medium)]),
        "rt_scene_set_env": (I32, [VP, P(F), I32, I32, F]),
        "rt_scene_set_env_file": (I32, [VP, C.c_char_p, F]),
        "rt_scene_get_env": (I32, [VP, P(F), P(I32), P(I32)]),
        "rt_scene_add_texture": (I32, [VP, P(C.c_uint8), I32, I32, P(I32)]),
        "rt_scene_add_texture_file": (I32, [VP, C.c_char_p, P(I32)]),
        "rt_scene_get_texture": (I32, [VP, I32, P(I32), P(I32), P(C.c_uint8)]),
        "rt_scene_get_bounds": (I32, [VP, P(F), P(F)]),
        "rt_scene_counts": (I32, [VP, P(I64), P(I32), P(I32), P(I32)]),
        "rt_scene_load_json": (I32, [VP, C.c_char_p, P(Options), P(Camera)]),
        "rt_scene_build_bvh": (I32, [VP, P(I64), P(I32)]),
        "rt_scene_build_bvh_gpu": (I32, [VP, P(I64), P(I32)]),
        "rt_scene_load_json_string": (I32, [VP, C.c_char_p, C.c_char_p, P(Options), P(Camera)]),
        "rt_renderer_create": (I32, [VP, P(Options), P(VP)]),
        "rt_renderer_destroy": (I32, [VP]),
        "rt_renderer_set_options": (I32, [VP, P(Options)]),
        "rt_renderer_get_options": (I32, [VP, P(Options)]),
        "rt_renderer_resize": (I32, [VP, I32, I32]),
        "rt_renderer_set_camera": (I32, [VP, P(Camera)]),
        "rt_renderer_set_stream": (I32, [VP, VP]),
        "rt_renderer_render": (I32, [VP]),
        "rt_renderer_synchronize": (I32, [VP]),
        "rt_renderer_download_rgba8": (I32, [VP, P(C.c_uint32)]),
        "rt_renderer_download_linear": (I32, [VP, P(F)]),
        "rt_renderer_download_aov": (I32, [VP, I32, P(F)]),
        "rt_renderer_device_buffers": (I32, [VP, P(VP), P(VP)]),
        "rt_renderer_get_stats": (I32, [VP, P(RenderStats)]),
        "rt_renderer_frame_index": (I32, [VP, P(I32)]),
        "rt_renderer_trace": (I32, [VP, I32, VP, I64, VP, I32]),
        "rt_renderer_trace_wavefront": (I32, [VP, I32, VP, I64, VP, P(I64)]),
        "rt_denoise_image": (I32, [P(F), P(F), P(F), I32, I32, P(F)]),
        "rt_write_png": (I32, [C.c_char_p, P(C.c_uint32), I32, I32]),
        "rt_verify_shading": (I32, [I32, P(Material), I32, P(Light), I32, P(Medium), I32, P(F), I64, P(F)]),
        "rt_kulla_conty_lut": (I32, [P(F), P(F)]),
        "rt_guide_options_default": (None, [P(GuideOptions)]),
        "rt_guide_create": (I32, [P(GuideOptions), P(VP)]),
        "rt_guide_destroy": (I32, [VP]),
        "rt_guide_sizes": (None, [P(I64), P(I64)]),
        "rt_guide_get_params": (I32, [VP, P(F), P(F)]),
        "rt_guide_set_params": (I32, [VP, P(F), P(F)]),
        "rt_guide_forward": (I32, [VP, P(F), I64, P(F)]),
        "rt_guide_gradients": (I32, [VP, P(F), P(F), P(F), I64, P(F), P(F), P(F)]),
        "rt_guide_train_step": (I32, [VP, P(F), P(F), P(F), I64, P(F)]),
        "rt_guide_pdf": (I32, [VP, P(F), P(F), P(F), I64, P(F), P(F)]),
        "rt_guide_last_loss": (I32, [VP, P(F), P(I64)]),
        "rt_guide_set_hyperparameters": (I32, [VP, F, I32, F]),
        "rt_renderer_guide": (I32, [VP, P(VP)]),
        "rt_renderer_guide_samples": (I32, [VP, P(F), I64, P(I64)]),
        "rt_server_options_default": (None, [P(ServerOptions)]),
        "rt_server_create": (I32, [P(ServerOptions), P(VP)]),
        "rt_server_destroy": (I32, [VP]),
        "rt_server_add_scene": (I32, [VP, VP, P(I32)]),
        "rt_server_submit": (I32, [VP, P(JobDesc), P(I64)]),
        "rt_server_cancel": (I32, [VP, I64]),
        "rt_server_poll": (I32, [VP, I64, P(JobStatus)]),
        "rt_server_wait": (I32, [VP, I64, C.c_double, P(JobStatus)]),
        "rt_server_download": (I32, [VP, I64, P(F)]),
        "rt_server_download_rgba8": (I32, [VP, I64, P(C.c_uint32)]),
        "rt_server_release": (I32, [VP, I64]),
        "rt_server_step": (I32, [VP, P(I32)]),
        "rt_server_get_stats": (I32, [VP, P(ServerStats)]),
        "rt_env_sampling_cache": (I32, [P(F), I32, I32, P(F)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(code):
    if code != RT_OK:
        msg = _lib.rt_last_error_message().decode(errors="replace")
        raise RTError(code, msg)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f3(v):
    return F3(*[float(x) for x in v])


def material(type=MAT_DIFFUSE, **kw):
    """A Material with the reference defaults (Scene.h:70-116) and overrides."""
    lib = load_library()
    m = Material()
    lib.rt_material_default(C.byref(m))
    m.type = type
    for k, v in kw.items():
        if k == "texture_ids":
            ids = list(v) + [-1] * (8 - len(v))
            m.texture_ids = (C.c_int32 * 8)(*ids)
        else:
            setattr(m, k, _f3(v) if k in ("albedo", "eta", "k", "specular") else v)
    return m


def light(type=LIGHT_QUAD, **kw):
    lib = load_library()
    l = Light()
    lib.rt_light_default(C.byref(l))
    l.type = type
    for k, v in kw.items():
        setattr(l, k, _f3(v) if k in ("radiance", "position", "u", "v") else v)
    return l


def medium(type=MEDIUM_HOMOGENEOUS, density=None, **kw):
    lib = load_library()
    m = Medium()
    lib.rt_medium_default(C.byref(m))
    m.type = type
    for k, v in kw.items():
        if k in ("g", "sigma_s", "sigma_a", "bounds_min", "bounds_max"):
            setattr(m, k, _f3(v))
        elif k == "grid_res":
            m.grid_res = (C.c_int32 * 3)(*v)
        else:
            setattr(m, k, v)
    if density is not None:
        d = np.ascontiguousarray(density, dtype=np.float32)
        m._density_keepalive = d
        m.density = _fptr(d)
        if type == MEDIUM_GRID and "grid_res" not in kw:
            m.grid_res = (C.c_int32 * 3)(d.shape[2], d.shape[1], d.shape[0])
    return m


def camera(from_, at, up=(0, 1, 0), medium=-1, fov_y_deg=0.0):
    c = Camera()
    c.from_ = _f3(from_)
    c.at = _f3(at)
    c.up = _f3(up)
    c.medium = medium
    c.fov_y_deg = fov_y_deg
    return c


def options(**kw):
    lib = load_library()
    o = Options()
    lib.rt_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Scene:
    """class Scene, core/include/Scene.h:195-214."""

    def __init__(self):
        self._lib = load_library()
        self._h = C.c_void_p()
        _check(self._lib.rt_scene_create(C.byref(self._h)))

    def close(self):
        if self._h:
            self._lib.rt_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def add_mesh(self, positions, mat, indices=None, normals=None, texcoords=None, out_medium=-1, in_medium=-1):
        """Scene::AddMesh (core/src/Scene.cpp:22-64); returns the mesh id."""
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        d = MeshDesc()
        d.positions = _fptr(pos)
        d.num_vertices = pos.shape[0]
        keep = [pos]
        if indices is not None:
            idx = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1, 3)
            keep.append(idx)
            d.indices = idx.ctypes.data_as(C.POINTER(C.c_int32))
            d.num_triangles = idx.shape[0]
        else:
            d.num_triangles = pos.shape[0] // 3
        if normals is not None:
            n = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
            keep.append(n)
            d.normals = _fptr(n)
        if texcoords is not None:
            t = np.ascontiguousarray(texcoords, dtype=np.float32).reshape(-1, 2)
            keep.append(t)
            d.texcoords = _fptr(t)
        mid = C.c_int32()
        _check(self._lib.rt_scene_add_mesh(self._h, C.byref(d), C.byref(mat), out_medium, in_medium, C.byref(mid)))
        return mid.value

    def add_texture(self, rgba):
        """Scene::AddTexture: (h, w, 4) uint8, row 0 at the bottom (v = 0); returns the texture id."""
        a = np.ascontiguousarray(rgba, dtype=np.uint8)
        if a.ndim != 3 or a.shape[2] != 4:
            raise ValueError("texture must be (h, w, 4) uint8")
        tid = C.c_int32()
        _check(self._lib.rt_scene_add_texture(self._h, a.ctypes.data_as(C.POINTER(C.c_uint8)), a.shape[1],
                                              a.shape[0], C.byref(tid)))
        return tid.value

    def set_env_file(self, path, scale=1.0):
        """Scene::AddEnv(fileName) (core/src/Scene.cpp:79-81): a Radiance .hdr or LDR image file."""
        _check(self._lib.rt_scene_set_env_file(self._h, os.fsencode(str(path)), float(scale)))

    def get_env(self):
        """The environment image, (H, W, 4) float32 with row 0 at the bottom (None: no environment)."""
        w, h = C.c_int32(), C.c_int32()
        _check(self._lib.rt_scene_get_env(self._h, None, C.byref(w), C.byref(h)))
        if w.value <= 0:
            return None
        out = np.empty((h.value, w.value, 4), np.float32)
        _check(self._lib.rt_scene_get_env(self._h, _fptr(out), C.byref(w), C.byref(h)))
        return out

    def add_texture_file(self, path):
        tid = C.c_int32()
        _check(self._lib.rt_scene_add_texture_file(self._h, str(path).encode(), C.byref(tid)))
        return tid.value

    def get_texture(self, tid):
        w, h = C.c_int32(), C.c_int32()
        _check(self._lib.rt_scene_get_texture(self._h, int(tid), C.byref(w), C.byref(h), None))
        out = np.empty((h.value, w.value, 4), np.uint8)
        _check(self._lib.rt_scene_get_texture(self._h, int(tid), None, None, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def add_mesh_obj(self, path, mat, out_medium=-1, in_medium=-1):
        mid = C.c_int32()
        _check(self._lib.rt_scene_add_mesh_obj(self._h, str(path).encode(), C.byref(mat), out_medium, in_medium,
                                               C.byref(mid)))
        return mid.value

    def add_light(self, l):
        """Scene::AddLight."""
        _check(self._lib.rt_scene_add_light(self._h, C.byref(l)))

    def add_medium(self, m):
        """Scene::AddMedium."""
        _check(self._lib.rt_scene_add_medium(self._h, C.byref(m)))

    def add_env(self, rgba, scale=1.0):
        """Scene::AddEnv with an in-memory equirectangular RGBA float image."""
        img = np.ascontiguousarray(rgba, dtype=np.float32)
        h, w = img.shape[:2]
        _check(self._lib.rt_scene_set_env(self._h, _fptr(img), w, h, float(scale)))

    def load_json(self, path):
        """SceneParser::LoadFromJson; returns (Options, Camera)."""
        o = options()
        c = Camera()
        self._lib.rt_camera_default(C.byref(c))
        _check(self._lib.rt_scene_load_json(self._h, str(path).encode(), C.byref(o), C.byref(c)))
        return o, c

    def load_json_string(self, text, base_dir="."):
        o = options()
        c = Camera()
        self._lib.rt_camera_default(C.byref(c))
        _check(self._lib.rt_scene_load_json_string(self._h, text.encode(), str(base_dir).encode(), C.byref(o),
                                                   C.byref(c)))
        return o, c

    def build_bvh(self):
        """Host build and validation of the acceleration structure: (nodes, depth)."""
        n, d = C.c_int64(), C.c_int32()
        _check(self._lib.rt_scene_build_bvh(self._h, C.byref(n), C.byref(d)))
        return n.value, d.value

    def build_bvh_gpu(self):
        """Builds the wide BVH on the device and validates it on the host: (nodes, depth)."""
        n, d = C.c_int64(), C.c_int32()
        _check(self._lib.rt_scene_build_bvh_gpu(self._h, C.byref(n), C.byref(d)))
        return n.value, d.value

    def bounds(self):
        lo = (C.c_float * 3)()
        hi = (C.c_float * 3)()
        _check(self._lib.rt_scene_get_bounds(self._h, lo, hi))
        return np.array(lo[:]), np.array(hi[:])

    def counts(self):
        t = C.c_int64()
        m, l, md = C.c_int32(), C.c_int32(), C.c_int32()
        _check(self._lib.rt_scene_counts(self._h, C.byref(t), C.byref(m), C.byref(l), C.byref(md)))
        return {"triangles": t.value, "meshes": m.value, "lights": l.value, "media": md.value}


class Renderer:
    """class Renderer, core/include/Renderer.h:9-187."""

    def __init__(self, scene: Scene, opts: Options | None = None):
        self._lib = load_library()
        self._h = C.c_void_p()
        _check(self._lib.rt_renderer_create(scene.handle, C.byref(opts) if opts is not None else None,
                                            C.byref(self._h)))

    def close(self):
        if self._h:
            self._lib.rt_renderer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def options(self) -> Options:
        o = Options()
        _check(self._lib.rt_renderer_get_options(self._h, C.byref(o)))
        return o

    def set_options(self, o: Options):
        _check(self._lib.rt_renderer_set_options(self._h, C.byref(o)))

    def resize(self, w, h):
        """Renderer::Resize."""
        _check(self._lib.rt_renderer_resize(self._h, int(w), int(h)))

    def set_camera(self, cam: Camera):
        """Renderer::SetCamera (resets accumulation)."""
        _check(self._lib.rt_renderer_set_camera(self._h, C.byref(cam)))

    def set_stream(self, stream_ptr: int | None):
        _check(self._lib.rt_renderer_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def render(self):
        """Renderer::Render (asynchronous)."""
        _check(self._lib.rt_renderer_render(self._h))

    def synchronize(self):
        _check(self._lib.rt_renderer_synchronize(self._h))

    def _wh(self):
        o = self.options
        return o.width, o.height

    def download_pixels(self, out=None):
        """Renderer::DownloadPixels: RGBA8 as uint32 (h, w)."""
        w, h = self._wh()
        if out is None:
            out = np.empty((h, w), dtype=np.uint32)
        _check(self._lib.rt_renderer_download_rgba8(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def download_linear(self, out=None):
        w, h = self._wh()
        if out is None:
            out = np.empty((h, w, 4), dtype=np.float32)
        _check(self._lib.rt_renderer_download_linear(self._h, _fptr(out)))
        return out

    def download_aov(self, kind):
        w, h = self._wh()
        out = np.empty((h, w, 4), dtype=np.float32)
        _check(self._lib.rt_renderer_download_aov(self._h, kind, _fptr(out)))
        return out

    def device_buffers(self):
        c, r = C.c_void_p(), C.c_void_p()
        _check(self._lib.rt_renderer_device_buffers(self._h, C.byref(c), C.byref(r)))
        return c.value, r.value

    def stats(self) -> dict:
        s = RenderStats()
        _check(self._lib.rt_renderer_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def frame_index(self):
        f = C.c_int32()
        _check(self._lib.rt_renderer_frame_index(self._h, C.byref(f)))
        return f.value

    def trace(self, rays, any_hit=False):
        """optixTrace-equivalent ray queries: rays (n, 8) float32 -> hits (n, 4)."""
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), dtype=np.float32)
        _check(self._lib.rt_renderer_trace(self._h, 1 if any_hit else 0, r.ctypes.data, r.shape[0],
                                           out.ctypes.data, 0))
        return out

    def trace_wavefront(self, rays, any_hit=False, counters=False):
        """The same queries answered by the path tracer's persistent extend (closest hit) or shadow
        (any hit) kernel; rays need tmin = 1e-4 (and tmax = FLT_MAX for closest hits).  With
        `counters`, also returns (rays, wide nodes visited, triangles tested)."""
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), dtype=np.float32)
        cnt = (C.c_int64 * 3)()
        _check(self._lib.rt_renderer_trace_wavefront(self._h, 1 if any_hit else 0, r.ctypes.data, r.shape[0],
                                                     out.ctypes.data, cnt if counters else None))
        return (out, tuple(int(v) for v in cnt)) if counters else out

    def guide_samples(self, max_samples=1 << 22):
        """The last training wave's samples: (n, 8) = input position, weight, direction, 1."""
        n = C.c_int64()
        _check(self._lib.rt_renderer_guide_samples(self._h, None, 0, C.byref(n)))
        k = min(n.value, max_samples)
        out = np.empty((k, 8), np.float32)
        _check(self._lib.rt_renderer_guide_samples(self._h, _fptr(out), k, C.byref(n)))
        return out

    def guide(self):
        """The renderer's guiding network (borrowed; created on first use)."""
        h = C.c_void_p()
        _check(self._lib.rt_renderer_guide(self._h, C.byref(h)))
        return Guide(handle=h.value, owner=self)

    def trace_device(self, rays_ptr, n, hits_ptr, any_hit=False):
        _check(self._lib.rt_renderer_trace(self._h, 1 if any_hit else 0, rays_ptr, n, hits_ptr, 1))


def server_options(**kw):
    load_library()
    o = ServerOptions()
    _lib.rt_server_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def job(scene, cam, width, height, spp, max_depth=25, rr_depth=0, filter=FILTER_GAUSSIAN, tonemap=TONEMAP_REINHARD,
        seed=1, exposure=1.0, guided=0):
    """One render request: the settings of a Renderer::Render() on a resident scene (PCG32 streams);
    `guided` samples with the scene's guiding network."""
    return JobDesc(scene=int(scene), camera=cam, width=int(width), height=int(height), spp=int(spp),
                   max_depth=int(max_depth), rr_depth=int(rr_depth), filter=int(filter), tonemap=int(tonemap),
                   seed=int(seed), exposure=float(exposure), guided=int(guided))


class Server:
    """Continuous-batching render server: resident scenes, queued jobs packed into shared waves."""

    def __init__(self, opts: ServerOptions | None = None):
        self._lib = load_library()
        self._h = C.c_void_p()
        self._sizes = {}
        _check(self._lib.rt_server_create(C.byref(opts) if opts is not None else None, C.byref(self._h)))

    def close(self):
        if self._h:
            self._lib.rt_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene: Scene) -> int:
        i = C.c_int32()
        _check(self._lib.rt_server_add_scene(self._h, scene.handle, C.byref(i)))
        return i.value

    def submit(self, desc: JobDesc) -> int:
        i = C.c_int64()
        _check(self._lib.rt_server_submit(self._h, C.byref(desc), C.byref(i)))
        self._sizes[i.value] = (desc.height, desc.width)
        return i.value

    def cancel(self, job_id):
        _check(self._lib.rt_server_cancel(self._h, int(job_id)))

    def poll(self, job_id) -> dict:
        st = JobStatus()
        _check(self._lib.rt_server_poll(self._h, int(job_id), C.byref(st)))
        return st.as_dict()

    def wait(self, job_id, timeout_ms=-1.0) -> dict:
        st = JobStatus()
        _check(self._lib.rt_server_wait(self._h, int(job_id), float(timeout_ms), C.byref(st)))
        return st.as_dict()

    def download(self, job_id):
        h, w = self._sizes[job_id]
        out = np.empty((h, w, 4), dtype=np.float32)
        _check(self._lib.rt_server_download(self._h, int(job_id), _fptr(out)))
        return out

    def download_pixels(self, job_id):
        h, w = self._sizes[job_id]
        out = np.empty((h, w), dtype=np.uint32)
        _check(self._lib.rt_server_download_rgba8(self._h, int(job_id), out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def release(self, job_id):
        _check(self._lib.rt_server_release(self._h, int(job_id)))
        self._sizes.pop(job_id, None)

    def step(self) -> bool:
        w = C.c_int32()
        _check(self._lib.rt_server_step(self._h, C.byref(w)))
        return bool(w.value)

    def stats(self) -> dict:
        st = ServerStats()
        _check(self._lib.rt_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()


class Guide:
    """The path-guiding network on host buffers: hash grid + MLP + 8-lobe vMF mixture."""

    def __init__(self, learning_rate=1e-2, seed=1, handle=None, owner=None, max_resolution=None,
                 max_log_kappa=None):
        self._lib = load_library()
        self._owned = handle is None
        self._owner = owner  # keeps a borrowed handle's renderer alive
        if handle is None:
            o = GuideOptions()
            self._lib.rt_guide_options_default(C.byref(o))
            o.learning_rate, o.seed = learning_rate, seed
            if max_resolution is not None:
                o.max_resolution = max_resolution
            if max_log_kappa is not None:
                o.max_log_kappa = max_log_kappa
            self._h = C.c_void_p()
            _check(self._lib.rt_guide_create(C.byref(o), C.byref(self._h)))
        else:
            self._h = C.c_void_p(handle)
        t, m = C.c_int64(), C.c_int64()
        self._lib.rt_guide_sizes(C.byref(t), C.byref(m))
        self.table_size, self.mlp_size = t.value, m.value

    def close(self):
        if self._h and self._owned:
            self._lib.rt_guide_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_hyperparameters(self, learning_rate=0.0, max_resolution=0, max_log_kappa=0.0):
        _check(self._lib.rt_guide_set_hyperparameters(self._h, float(learning_rate), int(max_resolution),
                                                      float(max_log_kappa)))

    def last_loss(self):
        loss, steps = C.c_float(), C.c_int64()
        _check(self._lib.rt_guide_last_loss(self._h, C.byref(loss), C.byref(steps)))
        return loss.value, steps.value

    @staticmethod
    def _f32(a, cols=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        return a if cols is None else a.reshape(-1, cols)

    def get_params(self):
        t = np.empty(self.table_size, np.float32)
        m = np.empty(self.mlp_size, np.float32)
        _check(self._lib.rt_guide_get_params(self._h, _fptr(t), _fptr(m)))
        return t, m

    def set_params(self, table=None, mlp=None):
        t = None if table is None else self._f32(table).reshape(-1)
        m = None if mlp is None else self._f32(mlp).reshape(-1)
        _check(self._lib.rt_guide_set_params(self._h, None if t is None else _fptr(t), None if m is None else _fptr(m)))

    def forward(self, pos):
        p = self._f32(pos, 3)
        out = np.empty((p.shape[0], 32), np.float32)
        _check(self._lib.rt_guide_forward(self._h, _fptr(p), p.shape[0], _fptr(out)))
        return out

    def gradients(self, pos, dirs, weights):
        p, d, w = self._f32(pos, 3), self._f32(dirs, 3), self._f32(weights).reshape(-1)
        loss = np.zeros(1, np.float32)
        gt = np.empty(self.table_size, np.float32)
        gm = np.empty(self.mlp_size, np.float32)
        _check(self._lib.rt_guide_gradients(self._h, _fptr(p), _fptr(d), _fptr(w), p.shape[0], _fptr(loss),
                                            _fptr(gt), _fptr(gm)))
        return float(loss[0]), gt, gm

    def train_step(self, pos, dirs, weights):
        p, d, w = self._f32(pos, 3), self._f32(dirs, 3), self._f32(weights).reshape(-1)
        loss = np.zeros(1, np.float32)
        _check(self._lib.rt_guide_train_step(self._h, _fptr(p), _fptr(d), _fptr(w), p.shape[0], _fptr(loss)))
        return float(loss[0])

    def pdf(self, pos, dirs):
        p, d = self._f32(pos, 3), self._f32(dirs, 3)
        out = np.empty(p.shape[0], np.float32)
        _check(self._lib.rt_guide_pdf(self._h, _fptr(p), _fptr(d), None, p.shape[0], None, _fptr(out)))
        return out

    def sample(self, pos, u):
        p, uu = self._f32(pos, 3), self._f32(u, 3)
        d = np.empty((p.shape[0], 3), np.float32)
        out = np.empty(p.shape[0], np.float32)
        _check(self._lib.rt_guide_pdf(self._h, _fptr(p), None, _fptr(uu), p.shape[0], _fptr(d), _fptr(out)))
        return d, out


def write_png(path, pixels):
    """Writes an (H, W) uint32 RGBA8 frame (row 0 = bottom, as download_pixels) as a PNG file."""
    lib = load_library()
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    if px.ndim != 2:
        raise ValueError("pixels must be an (H, W) uint32 array")
    h, w = px.shape
    _check(lib.rt_write_png(os.fsencode(str(path)), px.ctypes.data_as(C.POINTER(C.c_uint32)), w, h))


def denoise_image(color, albedo, normal):
    """The denoiser of Options.denoise on (H, W, 4) float32 colour, albedo and
    normal images (row 0 = bottom); returns the denoised colour."""
    lib = load_library()
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (color, albedo, normal)]
    if any(a.ndim != 3 or a.shape[2] != 4 or a.shape != arrs[0].shape for a in arrs):
        raise ValueError("color, albedo and normal must be (H, W, 4) images of one size")
    h, w = arrs[0].shape[:2]
    out = np.empty((h, w, 4), np.float32)
    fp = C.POINTER(C.c_float)
    _check(lib.rt_denoise_image(*(a.ctypes.data_as(fp) for a in arrs), w, h, out.ctypes.data_as(fp)))
    return out


def verify_shading(op, inputs, materials=(), lights=(), media=()):
    lib = load_library()
    x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, 16)
    out = np.zeros((x.shape[0], 8), dtype=np.float32)
    M = (Material * max(1, len(materials)))(*materials)
    L = (Light * max(1, len(lights)))(*lights)
    D = (Medium * max(1, len(media)))(*media)
    _check(lib.rt_verify_shading(op, M, len(materials), L, len(lights), D, len(media), _fptr(x), x.shape[0],
                                 _fptr(out)))
    return out


def kulla_conty_lut():
    lib = load_library()
    a = np.zeros(64 * 64, np.float32)
    b = np.zeros(64, np.float32)
    _check(lib.rt_kulla_conty_lut(_fptr(a), _fptr(b)))
    return a.reshape(64, 64), b


def env_sampling_cache(rgba):
    lib = load_library()
    img = np.ascontiguousarray(rgba, dtype=np.float32)
    h, w = img.shape[:2]
    out = np.zeros_like(img)
    _check(lib.rt_env_sampling_cache(_fptr(img), w, h, _fptr(out)))
    return out
