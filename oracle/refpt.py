"""ctypes wrapper of oracle/_ref/libref_pt.so: the reference renderer's own
shading code compiled for the host, in an OpenMP per-pixel loop.

TEST INFRASTRUCTURE ONLY: bench.py's CPU baseline (kind "reference") and a
statistical cross-check of the oracle in tests/.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libref_pt.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise ImportError(f"{LIB} missing (needs the reference tree at build time)")
        _lib = C.CDLL(str(LIB))
        VP, I32, I64, P, F = C.c_void_p, C.c_int32, C.c_int64, C.POINTER, C.c_float
        _lib.refpt_scene_new.restype = VP
        _lib.refpt_scene_new.argtypes = [P(F), P(I32), I64, VP, P(I32), I32, VP, I32, VP, I32, P(F), I32, I32]
        _lib.refpt_scene_free.argtypes = [VP]
        _lib.refpt_render.restype = I32
        _lib.refpt_render.argtypes = [VP, VP, P(F), I32, I32, P(F), I32, I32, I32]
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def ref_structs():
    """Material / Light / Medium constructors whose defaults are the reference's
    own default-constructed structs (core/include/Scene.h:48-155)."""
    import pyoracle
    return pyoracle.StructDefaults(load(), "refpt")


class RefScene:
    def __init__(self, spec):
        import optixrender_b200 as rt
        import pyoracle
        lib = load()
        st = ref_structs()
        tris, tmesh, mats, mm = [], [], [], []
        for i, m in enumerate(spec.meshes):
            t = m.triangles()
            tris.append(t)
            tmesh.append(np.full(t.shape[0], i, np.int32))
            mats.append(st.material(**m.material))
            mm += [m.out_medium, m.in_medium]
        self.tv = np.ascontiguousarray(np.concatenate(tris), np.float32)
        self.tmesh = np.ascontiguousarray(np.concatenate(tmesh), np.int32)
        self.mats = (rt.Material * len(mats))(*mats)
        self.mm = np.asarray(mm, np.int32)
        self.lights = (rt.Light * max(1, len(spec.lights)))(*[st.light(**l) for l in spec.lights])
        self.media = (rt.Medium * max(1, len(spec.media)))(*[st.medium(**m) for m in spec.media])
        self.env = None if spec.env is None else np.ascontiguousarray(spec.env, np.float32)
        eh, ew = (0, 0) if spec.env is None else spec.env.shape[:2]
        self.h = lib.refpt_scene_new(_f(self.tv), self.tmesh.ctypes.data_as(C.POINTER(C.c_int32)), self.tv.shape[0],
                                     C.cast(self.mats, C.c_void_p), self.mm.ctypes.data_as(C.POINTER(C.c_int32)),
                                     len(mats), C.cast(self.lights, C.c_void_p), len(spec.lights),
                                     C.cast(self.media, C.c_void_p), len(spec.media),
                                     None if self.env is None else _f(self.env), ew, eh)
        self.spec = spec
        self._pyoracle = pyoracle

    def close(self):
        if self.h:
            load().refpt_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, opts, cam, frame=0, rows=None, threads=0):
        lib = load()
        w, h = opts.width, opts.height
        out = np.zeros((h, w, 4), np.float32)
        cv = np.ascontiguousarray(self._pyoracle.camera_vectors(cam, w, h).ravel(), np.float32)
        r0, r1 = rows if rows is not None else (0, 0)
        lib.refpt_render(self.h, C.byref(opts), _f(cv), cam.medium, frame, _f(out), threads, r0, r1)
        return out
