"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker of the CUDA library.  It
also loads the host build of the reference's own shading code
(oracle/_ref/*.so) when that was built, for pinning the oracle.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_DIR = HERE / "_ref"

_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise ImportError(f"{LIB} missing: run `make -C oracle`")
        _lib = C.CDLL(str(LIB))
        P, VP, I32, I64, F = C.POINTER, C.c_void_p, C.c_int32, C.c_int64, C.c_float
        _lib.orc_scene_new.restype = VP
        _lib.orc_scene_new.argtypes = [P(F), P(F), P(F), P(I32), I64, VP, P(I32), I32, VP, I32, VP, I32, P(F), I32,
                                       I32]
        _lib.orc_scene_free.argtypes = [VP]
        _lib.orc_scene_set_textures.argtypes = [VP, P(C.c_uint32), I64, P(I32), I32]
        _lib.orc_render.restype = I32
        _lib.orc_render.argtypes = [VP, I32, VP, VP, I32, P(F), P(F), P(F), P(I64), I32, I32, I32]
        _lib.orc_camera.argtypes = [VP, I32, I32, P(F)]
        _lib.orc_trace.restype = I32
        _lib.orc_trace.argtypes = [VP, I32, I32, P(F), I64, P(C.c_double)]
        _lib.orc_shading.restype = I32
        _lib.orc_shading.argtypes = [I32, I32, VP, I32, VP, I32, VP, I32, P(F), I64, P(F)]
        _lib.orc_kulla_conty.argtypes = [P(F), P(F)]
        _lib.orc_env_cache.argtypes = [P(F), I32, I32, P(F)]
        _lib.orc_tonemap.argtypes = [P(F), I64, I32, F, P(C.c_uint32)]
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


# ------------------------------------------------------------ scene structs
# The C ABI's struct layouts come from the optixrender_b200 package (plain
# ctypes classes; importing them loads no library).  Their default values come
# from a CPU library: the oracle's restatement of the reference's defaults
# (prefix "orc") or the reference's own default-constructed structs in its
# host build (prefix "refpt", oracle/refpt.py), so the oracle and the
# benchmark's reference arm never load the product library.
_VEC3 = {"albedo", "eta", "k", "specular", "radiance", "position", "u", "v", "g", "sigma_s", "sigma_a",
         "bounds_min", "bounds_max"}


def _fill(obj, kw):
    for k, v in kw.items():
        if k in _VEC3:
            setattr(obj, k, (C.c_float * 3)(*[float(x) for x in v]))
        elif k == "texture_ids":
            ids = list(v) + [-1] * (8 - len(v))
            obj.texture_ids = (C.c_int32 * 8)(*ids)
        elif k == "grid_res":
            obj.grid_res = (C.c_int32 * 3)(*v)
        else:
            setattr(obj, k, v)
    return obj


class StructDefaults:
    """Material / Light / Medium constructors with defaults from `lib`'s
    <prefix>_material_default, <prefix>_light_default, <prefix>_medium_default."""

    def __init__(self, lib, prefix):
        import optixrender_b200 as rt
        self.rt = rt
        self.fns = {}
        for name, cls in (("material", rt.Material), ("light", rt.Light), ("medium", rt.Medium)):
            fn = getattr(lib, f"{prefix}_{name}_default")
            fn.restype = None
            fn.argtypes = [C.POINTER(cls)]
            self.fns[name] = (fn, cls)

    def _make(self, name, type_, kw):
        fn, cls = self.fns[name]
        o = cls()
        fn(C.byref(o))
        o.type = type_
        return _fill(o, kw)

    def material(self, type=0, **kw):
        return self._make("material", type, kw)

    def light(self, type=0, **kw):
        return self._make("light", type, kw)

    def medium(self, type=0, density=None, **kw):
        m = self._make("medium", type, kw)
        if density is not None:
            d = np.ascontiguousarray(density, dtype=np.float32)
            m._density_keepalive = d
            m.density = d.ctypes.data_as(C.POINTER(C.c_float))
            if type == self.rt.MEDIUM_GRID and "grid_res" not in kw:  # x fastest: (z, y, x) array
                m.grid_res = (C.c_int32 * 3)(d.shape[2], d.shape[1], d.shape[0])
        return m


def oracle_structs():
    return StructDefaults(load(), "orc")


def options(**kw):
    """rt_options with the reference's launch defaults (LaunchParams.h:29-30 and
    :66: one sample, 25 bounces, Gaussian filter; the reference's LCG stream),
    built without the product library."""
    import optixrender_b200 as rt
    o = rt.Options()
    o.spp, o.max_depth, o.filter, o.rng, o.seed, o.exposure = 1, 25, rt.FILTER_GAUSSIAN, rt.RNG_LCG, 1, 1.0
    o.guide_train_spp, o.guide_prob, o.guide_steps = 32, 0.5, 4
    return _fill(o, kw)


def _normalize(v):
    """float32 normalize with the library's operation order: v / sqrt((x*x + y*y) + z*z)."""
    v = v.astype(np.float32)
    x, y, z = v[..., 0], v[..., 1], v[..., 2]
    ln = np.sqrt((x * x + y * y) + z * z)
    return v / ln[..., None]


def _face_normals(tris):
    """Per-vertex face normals of de-indexed triangles (m, 9), as rt_scene_add_mesh computes them."""
    t = tris.reshape(-1, 3, 3).astype(np.float32)
    e1, e2 = _normalize(t[:, 1] - t[:, 0]), _normalize(t[:, 2] - t[:, 0])
    c = np.stack([e1[:, 1] * e2[:, 2] - e2[:, 1] * e1[:, 2], e1[:, 2] * e2[:, 0] - e2[:, 2] * e1[:, 0],
                  e1[:, 0] * e2[:, 1] - e2[:, 0] * e1[:, 1]], -1)
    n = _normalize(c)
    return np.repeat(n, 3, axis=0).reshape(-1, 9)


class OracleScene:
    """The oracle's copy of a SceneSpec (optixrender_b200.scenes)."""

    def __init__(self, spec):
        import optixrender_b200 as rt
        lib = load()
        st = oracle_structs()
        tris, tmesh = [], []
        tnorm, tuv = [], []
        mats = []
        media_pairs = []
        for i, m in enumerate(spec.meshes):
            t = m.triangles()
            tris.append(t)
            tn = m.tri_normals()
            tnorm.append(None if tn is None else _normalize(tn.reshape(-1, 3)).reshape(-1, 9))
            tuv.append(m.tri_texcoords())
            tmesh.append(np.full(t.shape[0], i, np.int32))
            mats.append(st.material(**m.material))
            media_pairs += [m.out_medium, m.in_medium]
        self.tv = np.ascontiguousarray(np.concatenate(tris), np.float32)
        self.tn = self.tuv = None
        if any(n is not None for n in tnorm):
            self.tn = np.ascontiguousarray(np.concatenate(
                [n if n is not None else _face_normals(t) for n, t in zip(tnorm, tris)]), np.float32)
        if any(u is not None for u in tuv):
            self.tuv = np.ascontiguousarray(np.concatenate(
                [u if u is not None else np.tile(np.float32([0, 0, 1, 0, 0, 1]), (t.shape[0], 1))
                 for u, t in zip(tuv, tris)]), np.float32)
        self.tmesh = np.ascontiguousarray(np.concatenate(tmesh), np.int32)
        self.mats = (rt.Material * len(mats))(*mats)
        self.mm = np.asarray(media_pairs, np.int32)
        self.lights = (rt.Light * max(1, len(spec.lights)))(*[st.light(**l) for l in spec.lights])
        self.media = (rt.Medium * max(1, len(spec.media)))(*[st.medium(**m) for m in spec.media])
        env = spec.env
        self.env = None if env is None else np.ascontiguousarray(env, np.float32)
        eh, ew = (0, 0) if env is None else env.shape[:2]
        self.h = lib.orc_scene_new(_f(self.tv), None if self.tn is None else _f(self.tn),
                                   None if self.tuv is None else _f(self.tuv),
                                   self.tmesh.ctypes.data_as(C.POINTER(C.c_int32)),
                                   self.tv.shape[0], C.cast(self.mats, C.c_void_p),
                                   self.mm.ctypes.data_as(C.POINTER(C.c_int32)), len(mats),
                                   C.cast(self.lights, C.c_void_p), len(spec.lights), C.cast(self.media, C.c_void_p),
                                   len(spec.media), None if env is None else _f(self.env), ew, eh)
        if spec.textures:
            texels, info, off = [], [], 0
            for t in spec.textures:
                a = np.ascontiguousarray(t, np.uint8)
                texels.append(a.view(np.uint32).reshape(-1))
                info += [off, a.shape[1], a.shape[0]]
                off += a.shape[0] * a.shape[1]
            self.texels = np.ascontiguousarray(np.concatenate(texels))
            self.tex_info = np.asarray(info, np.int32)
            lib.orc_scene_set_textures(self.h, self.texels.ctypes.data_as(C.POINTER(C.c_uint32)), self.texels.size,
                                       self.tex_info.ctypes.data_as(C.POINTER(C.c_int32)), len(spec.textures))
        self.spec = spec

    def close(self):
        if self.h:
            load().orc_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, opts, cam, frame=0, color=None, precision=32, threads=0, rows=None, want_aov=True):
        """One Renderer::Render of the reference integrator on the CPU.
        Returns (color, albedo, normal, nan_count) as (h, w, 4) arrays."""
        lib = load()
        w, h = opts.width, opts.height
        if color is None:
            color = np.zeros((h, w, 4), np.float32)
        alb = np.zeros((h, w, 4), np.float32) if want_aov else None
        nrm = np.zeros((h, w, 4), np.float32) if want_aov else None
        nan = C.c_int64()
        r0, r1 = rows if rows is not None else (0, 0)
        rc = lib.orc_render(self.h, precision, C.byref(opts), C.byref(cam), frame, _f(color),
                            None if alb is None else _f(alb), None if nrm is None else _f(nrm), C.byref(nan),
                            threads, r0, r1)
        if rc:
            raise RuntimeError("orc_render failed")
        return color, alb, nrm, nan.value

    def trace(self, rays, any_hit=False, precision=64):
        lib = load()
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros((r.shape[0], 8), np.float64)
        lib.orc_trace(self.h, precision, 1 if any_hit else 0, _f(r), r.shape[0],
                      out.ctypes.data_as(C.POINTER(C.c_double)))
        return out


def shading(op, inputs, materials=(), lights=(), media=(), precision=64):
    import optixrender_b200 as rt
    lib = load()
    x = np.ascontiguousarray(inputs, np.float32).reshape(-1, 16)
    out = np.zeros((x.shape[0], 8), np.float32)
    M = (rt.Material * max(1, len(materials)))(*materials)
    L = (rt.Light * max(1, len(lights)))(*lights)
    D = (rt.Medium * max(1, len(media)))(*media)
    lib.orc_shading(precision, op, C.cast(M, C.c_void_p), len(materials), C.cast(L, C.c_void_p), len(lights),
                    C.cast(D, C.c_void_p), len(media), _f(x), x.shape[0], _f(out))
    return out


def kulla_conty():
    lib = load()
    a = np.zeros(4096, np.float32)
    b = np.zeros(64, np.float32)
    lib.orc_kulla_conty(_f(a), _f(b))
    return a.reshape(64, 64), b


def env_cache(rgba):
    lib = load()
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    out = np.zeros_like(img)
    lib.orc_env_cache(_f(img), w, h, _f(out))
    return out


def tonemap(color, mode=0, exposure=1.0):
    lib = load()
    c = np.ascontiguousarray(color, np.float32).reshape(-1, 4)
    out = np.zeros(c.shape[0], np.uint32)
    lib.orc_tonemap(_f(c), c.shape[0], mode, exposure, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out.reshape(color.shape[:-1])


def camera_vectors(cam, w, h):
    lib = load()
    out = np.zeros(12, np.float32)
    lib.orc_camera(C.byref(cam), w, h, _f(out))
    return out.reshape(4, 3)


# ---------------------------------------------------------------- reference host build
def ref_libs():
    """(shading, scene, rng) libraries built from the reference sources, or None."""
    paths = [REF_DIR / n for n in ("libref_shading.so", "libref_scene.so", "libref_rng.so")]
    if not all(p.exists() for p in paths):
        return None
    return tuple(C.CDLL(str(p)) for p in paths)
