"""Pins the CPU oracle (oracle/pt_oracle.hpp) to the reference renderer.

The golden vectors in tests/golden/reference_shading.npz are outputs of the
reference's own shading code compiled for the host (tests/golden/make_golden.py).
The FP32 oracle must reproduce them to float rounding; the FP64 oracle within
the reference's FP32 error.  Where the reference tree has been built into
oracle/_ref the same checks also run live against it.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import optixrender_b200 as rt
import pyoracle

GOLD = np.load(Path(__file__).parent / "golden" / "reference_shading.npz")


def _structs(cls, key):
    raw = GOLD[key].tobytes()
    n = len(raw) // C.sizeof(cls)
    return list((cls * n).from_buffer_copy(raw))


MATS = _structs(rt.Material, "materials")
LIGHTS = _structs(rt.Light, "lights")
MEDIA = _structs(rt.Medium, "media")


def close(a, b, rel, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    err = np.abs(a - b)
    tol = rel * np.maximum(np.abs(a), np.abs(b)) + floor
    ok = (err <= tol) | both_nan | ((a == b) & np.isfinite(a))
    return ok


def test_kulla_conty_lut_bitwise():
    lut, avg = pyoracle.kulla_conty()
    assert np.array_equal(lut.view(np.uint32), GOLD["kc_lut"].view(np.uint32))
    assert np.array_equal(avg.view(np.uint32), GOLD["kc_avg"].view(np.uint32))
    assert GOLD["kc_avg"][0] > 1.0  # the reference table's first entry exceeds one (1.0020117)


def test_env_cache_bitwise():
    cache = pyoracle.env_cache(GOLD["env_in"])
    assert np.array_equal(cache[..., :3], GOLD["env_cache"][..., :3])


def test_lcg_sequences():
    import sys
    sys.path.insert(0, str(Path(__file__).parents[1] / "optixrender_b200"))
    for (a, b), seq in zip(GOLD["lcg_seeds"], GOLD["lcg_seq"]):
        # restated TEA-16 + LCG in numpy (random.h:54-87)
        v0, v1, s0 = np.uint32(a), np.uint32(b), np.uint32(0)
        with np.errstate(over="ignore"):
            for _ in range(16):
                s0 = np.uint32(s0 + np.uint32(0x9E3779B9))
                v0 = np.uint32(v0 + (np.uint32((v1 << np.uint32(4)) + np.uint32(0xA341316C)) ^ np.uint32(v1 + s0) ^
                                     np.uint32((v1 >> np.uint32(5)) + np.uint32(0xC8013EA4))))
                v1 = np.uint32(v1 + (np.uint32((v0 << np.uint32(4)) + np.uint32(0xAD90777D)) ^ np.uint32(v0 + s0) ^
                                     np.uint32((v0 >> np.uint32(5)) + np.uint32(0x7E95761E))))
            st = v0
            out = []
            for _ in range(16):
                st = np.uint32(np.uint32(1664525) * st + np.uint32(1013904223))
                out.append(np.float32(int(st) & 0xFFFFFF) / np.float32(16777216))
        assert np.array_equal(np.array(out, np.float32), seq)


@pytest.mark.parametrize("op,key", [(rt.VERIFY_BSDF_EVAL, "bsdf_eval"), (rt.VERIFY_BSDF_SAMPLE, "bsdf_sample"),
                                    (rt.VERIFY_LIGHT_SAMPLE, "light_sample"), (rt.VERIFY_LIGHT_EVAL, "light_eval"),
                                    (rt.VERIFY_MEDIUM_SAMPLE, "medium_sample"),
                                    (rt.VERIFY_PHASE_SAMPLE, "phase_sample"), (rt.VERIFY_PHASE_EVAL, "phase_eval")])
def test_shading_matches_reference(op, key):
    x = GOLD[key + "_in"]
    ref = GOLD[key + "_out"]
    y32 = pyoracle.shading(op, x, MATS, LIGHTS, MEDIA, precision=32)
    y64 = pyoracle.shading(op, x, MATS, LIGHTS, MEDIA, precision=64)
    # FP32 restatement: bit-identical to the reference's own FP32 code
    exact = np.all((y32 == ref) | (np.isnan(y32) & np.isnan(ref)), axis=1).mean()
    assert exact >= 0.999, f"{key}: FP32 oracle is bit-identical on {exact:.4f} of queries"
    # FP64 oracle against the reference's FP32 result
    ok64 = close(y64, ref, 1e-3, 1e-5)
    frac64 = ok64.all(axis=1).mean()
    assert frac64 >= 0.99, f"{key}: FP64 oracle matches {frac64:.4f} of queries"


def test_filters_and_sphere_mapping():
    lib = pyoracle.load()  # noqa: F841  (oracle loaded)
    # the oracle's filter code is exercised through shading-free restatements
    fj = GOLD["filter_in"].astype(np.float64)
    for t in range(4):
        out = GOLD[f"filter_out_{t}"]
        if t == rt.FILTER_BOX:
            mine = fj - 0.5
        elif t == rt.FILTER_TENT:
            j = fj * 2
            mine = 0.5 + np.where(j < 1, np.sqrt(j) - 1, 1 - np.sqrt(2 - j))
        elif t == rt.FILTER_TRIANGLE:
            u1, u2 = fj[:, 0].copy(), fj[:, 1].copy()
            m = u2 > u1
            u1h = np.where(m, u1 * 0.5, u1 - u2 * 0.5)
            u2h = np.where(m, u2 - u1 * 0.5, u2 * 0.5)
            mine = 0.5 + np.stack([u1h, u2h], 1)
        else:
            r = np.sqrt(-2 * np.log(np.maximum(fj[:, 0], 1.1754944e-38)))
            th = 2 * np.pi * fj[:, 1]
            mine = 0.5 + 0.375 * np.stack([r * np.cos(th), r * np.sin(th)], 1)
        assert np.allclose(mine, out, rtol=1e-5, atol=2e-6), t
    d = GOLD["sphere_in"].astype(np.float64)
    u = np.arctan2(d[:, 2], d[:, 0]) / (2 * np.pi) + 0.5
    v = np.arcsin(d[:, 1]) / np.pi + 0.5
    assert np.allclose(np.stack([u, v], 1), GOLD["sphere_uv"], atol=3e-6)
    assert np.allclose(GOLD["sphere_back"], d, atol=1e-5)


def test_live_reference_build_when_present():
    libs = pyoracle.ref_libs()
    if libs is None:
        pytest.skip("reference host build not present (oracle/_ref)")
    shading, scene, _ = libs
    F = C.POINTER(C.c_float)
    lut = np.zeros(4096, np.float32)
    avg = np.zeros(64, np.float32)
    shading.ref_kulla_conty(lut.ctypes.data_as(F), avg.ctypes.data_as(F))
    assert np.array_equal(lut, GOLD["kc_lut"].ravel())
    assert bool(shading.ref_pair_order_reversed()) == bool(GOLD["pair_order_reversed"])


def test_struct_defaults_agree_with_the_reference():
    """Scene struct defaults (core/include/Scene.h:48-155): the oracle's
    restatement, the reference's own default-constructed structs (when its
    host build is present) and the product's rt_*_default give the same
    fields."""
    import refpt

    def fields(o):
        return {k: (list(getattr(o, k)) if hasattr(getattr(o, k), "__len__") else getattr(o, k))
                for k, _ in o._fields_ if k not in ("density", "majorant_res", "grid_res", "bounds_min", "bounds_max")}

    srcs = [pyoracle.oracle_structs()]
    if refpt.available():
        srcs.append(refpt.ref_structs())
    for kind in ("material", "light", "medium"):
        prod = fields(getattr(rt, kind)(type=0))
        for src in srcs:
            assert fields(getattr(src, kind)(type=0)) == prod, kind


def test_point_light_is_the_small_sphere_limit_of_the_reference():
    """Point lights have no reference counterpart; their nearest analogue is
    the reference's sphere light (SampleSphere, core/cuda/Light.h:118-141) as
    its radius goes to zero.  A uniformly emitting sphere of radius r and
    radiance I / (pi r^2) that lies wholly above a surface's horizon gives that
    surface exactly the irradiance of a point of intensity I, I cos / d^2, for
    any r; so the reference's own sphere sampling (a 16 x 16 stratified grid of
    its two random numbers, r / d <= 0.05) must reproduce the oracle's point
    light within the FP32 rounding of its cone (1 - cos theta_max)."""
    libs = pyoracle.ref_libs()
    if libs is None:
        pytest.skip("reference host build not present (oracle/_ref)")
    shading = libs[0]
    F = C.POINTER(C.c_float)
    rng = np.random.default_rng(17)
    c, I, radius = np.array([0.2, 1.1, -0.3]), np.array([2.0, 3.0, 4.0]), 0.04
    point = rt.light(rt.LIGHT_POINT, position=tuple(c), radiance=tuple(I))
    sphere = rt.light(rt.LIGHT_SPHERE, position=tuple(c), radius=radius,
                      radiance=tuple(I / (np.pi * radius * radius)))
    p = c + rng.normal(size=(400, 3)) * 0.8
    p = p[np.linalg.norm(p - c, axis=1) > 0.8]
    to_c = (c - p) / np.linalg.norm(c - p, axis=1, keepdims=True)
    nrm = to_c + rng.normal(size=p.shape) * 0.5
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    keep = (nrm * to_c).sum(1) > 0.3  # the whole sphere above the horizon
    p, nrm = p[keep], nrm[keep]
    n_pts, k = len(p), 256
    g = (np.arange(16) + 0.5) / 16
    u = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    x = np.zeros((n_pts * k, 16), np.float32)
    x[:, 0:3] = np.repeat(p, k, 0)
    x[:, 3:5] = np.tile(u, (n_pts, 1))
    Ls = (rt.Light * 1)(sphere)
    M = (rt.Material * 1)(rt.material(rt.MAT_DIFFUSE))
    D = (rt.Medium * 1)(rt.medium())
    y = np.zeros((n_pts * k, 8), np.float32)
    shading.ref_shading(rt.VERIFY_LIGHT_SAMPLE, C.cast(M, C.c_void_p), 1, C.cast(Ls, C.c_void_p), 1,
                        C.cast(D, C.c_void_p), 0, x.ctypes.data_as(F), x.shape[0], y.ctypes.data_as(F))
    cos = np.maximum(0.0, (y[:, 4:7].astype(np.float64) * np.repeat(nrm, k, 0)).sum(1))
    e_sphere = (y[:, 0:3] * (cos / y[:, 3])[:, None]).reshape(n_pts, k, 3).mean(1)
    xp = np.zeros((n_pts, 16), np.float32)
    xp[:, 0:3] = p
    yp = pyoracle.shading(rt.VERIFY_LIGHT_SAMPLE, xp, [rt.material(rt.MAT_DIFFUSE)], [point], [], precision=64)
    assert np.all(yp[:, 3] == 1.0)  # a delta light: its sample carries weight 1
    np.testing.assert_allclose(yp[:, 7], np.linalg.norm(p - c, axis=1), rtol=1e-6)
    np.testing.assert_allclose(yp[:, 4:7], to_c[keep], rtol=0, atol=1e-6)
    e_point = yp[:, 0:3] * np.maximum(0.0, (yp[:, 4:7] * nrm).sum(1))[:, None]
    assert n_pts > 100
    rel = np.abs(e_sphere - e_point) / e_point
    print(f"point vs sphere: max rel {rel.max():.2e}, mean {rel.mean():.2e} over {n_pts} points")
    assert rel.max() < 2e-3


@pytest.mark.parametrize("name", ["cornell", "media", "textured", "portal"])
def test_oracle_scene_structs_equal_the_products(name):
    """The oracle builds its scenes without the product library; every
    material, light and medium it makes from a scene spec must be the one the
    product's constructors make (field for field, grid resolution included)."""
    from optixrender_b200 import scenes
    spec = {"cornell": lambda: scenes.cornell(8, 8, 1), "media": lambda: scenes.media(8, 8, 1, grid_res=16, env_size=(16, 8)),
            "textured": lambda: scenes.textured(8, 8, 1), "portal": lambda: scenes.portal(8, 8, 1)}[name]()
    st = pyoracle.oracle_structs()

    def raw(o):
        b = bytearray(bytes(o))
        if isinstance(o, rt.Medium):  # the density pointer and the library's majorant default (0 means 8)
            off = rt.Medium.density.offset
            b[off:off + 8] = bytes(8)
            mo = rt.Medium.majorant_res.offset
            if int.from_bytes(b[mo:mo + 4], "little") == 8:
                b[mo:mo + 4] = bytes(4)
        return bytes(b)

    for m in spec.meshes:
        assert raw(st.material(**m.material)) == raw(rt.material(**m.material))
    for l in spec.lights:
        assert raw(st.light(**l)) == raw(rt.light(**l))
    for md in spec.media:
        a, b = st.medium(**md), rt.medium(**md)
        assert raw(a) == raw(b)
        assert list(a.grid_res) == list(b.grid_res)
