"""Host-side checks of the C ABI (include/rt_capi.h); no GPU needed.

* the library exports every function the header declares;
* defaults equal the reference's struct initialisers (Scene.h, LaunchParams.h);
* errors come back as status codes with a message, never as crashes;
* the host-built tables (Kulla-Conty LUT, environment cache) are bit-identical
  to the reference's (golden vectors);
* the scene formats (JSON of models/test.json, OBJ, Radiance HDR) load;
* the wide BVH of every benchmark scene builds and validates on the host.
"""
import ctypes as C
import re
import struct
from pathlib import Path

import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes

ROOT = Path(__file__).resolve().parents[1]
GOLD = np.load(Path(__file__).parent / "golden" / "reference_shading.npz")


def declared_functions():
    names = []
    for hdr in (ROOT / "include").glob("*.h"):
        text = hdr.read_text()
        names += re.findall(r"RT_API\s+[\w\s\*]+?\b(rt_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(rt.LIBRARY_PATH))
    names = declared_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_struct_sizes_match_header_layout():
    assert C.sizeof(rt.Material) == 120
    assert C.sizeof(rt.Light) == 64
    assert C.sizeof(rt.Medium) == 96
    assert C.sizeof(rt.Options) == 80
    assert C.sizeof(rt.Camera) == 44
    assert C.sizeof(rt.MeshDesc) == 48


def test_reference_defaults():
    m = rt.material(rt.MAT_METAL_WORKFLOW)  # Scene.h:70-116
    assert list(m.albedo) == [1.0, 1.0, 1.0] and m.roughness == pytest.approx(0.1)
    assert list(m.eta) == pytest.approx([0.14282, 0.37414, 1.43944])
    assert list(m.k) == pytest.approx([3.97472, 2.38066, 1.59981])
    assert m.int_ior == pytest.approx(1.5) and m.ext_ior == 1.0 and m.nonlinear == 1
    assert m.metallic == pytest.approx(0.8) and m.coat_weight == 2.0
    assert list(m.texture_ids) == [-1] * 8
    lib = rt.load_library()
    l = rt.Light()
    lib.rt_light_default(C.byref(l))  # Scene.h:143-155
    assert l.type == rt.LIGHT_SPHERE and list(l.radiance) == [3.0] * 3 and l.radius == 3.0 and l.medium == -1
    assert list(l.position) == [6.0, 2.0, 0.0] and list(l.u) == [0, 0, 6.0] and list(l.v) == [6.0, 0, 0]
    md = rt.Medium()
    lib.rt_medium_default(C.byref(md))  # Scene.h:48-55
    assert md.scale == 500.0 and list(md.sigma_s) == pytest.approx([0.74, 0.88, 1.01])
    o = rt.options()  # LaunchParams.h:28-69
    assert o.spp == 1 and o.max_depth == 25 and o.filter == rt.FILTER_GAUSSIAN and o.rng == rt.RNG_LCG


def test_errors_are_status_codes():
    s = rt.Scene()
    with pytest.raises(rt.RTError) as e:
        s.add_mesh(np.zeros((3, 3)), rt.material(rt.MAT_DIFFUSE), indices=np.array([[0, 1, 5]]))
    assert e.value.code == 1 and "index out of range" in str(e.value)
    with pytest.raises(rt.RTError):
        s.add_mesh(np.zeros((3, 3)), rt.material(99))
    with pytest.raises(rt.RTError) as e:
        s.load_json("/nonexistent/scene.json")
    assert e.value.code == 4
    with pytest.raises(rt.RTError) as e:
        s.load_json_string("{ not json")
    assert e.value.code == 5
    lib = rt.load_library()
    assert lib.rt_scene_add_light(None, None) == 1
    assert lib.rt_renderer_render(None) == 1


def test_host_tables_bit_identical_to_reference():
    lut, avg = rt.kulla_conty_lut()
    assert np.array_equal(lut.view(np.uint32), GOLD["kc_lut"].view(np.uint32))
    assert np.array_equal(avg.view(np.uint32), GOLD["kc_avg"].view(np.uint32))
    cache = rt.env_sampling_cache(GOLD["env_in"])
    assert np.array_equal(cache[..., :3], GOLD["env_cache"][..., :3])


def test_scene_counts_bounds_and_deindexing():
    spec = scenes.cornell()
    s = scenes.build_scene(spec)
    c = s.counts()
    assert c == {"triangles": 34, "meshes": 7, "lights": 1, "media": 0}
    lo, hi = s.bounds()
    assert np.allclose(lo, [0, 0, 0]) and np.allclose(hi, [1, 1, 1])


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_wide_bvh_builds_and_validates(name):
    spec = scenes.SCENES[name]()
    s = scenes.build_scene(spec)
    nodes, depth = s.build_bvh()
    assert nodes >= 1 and 1 <= depth <= 32
    if name == "spheres":
        assert s.counts()["triangles"] == 2590720


def _chain_scene(lo, hi, step):
    """Triangles at positions 2^e for e in [lo, hi): each binned SAH split
    peels off the largest few, so the tree is a chain, and the small end has
    centroid extents for which 32 / extent overflows."""
    x = 2.0 ** np.arange(lo, hi, step)
    z = np.zeros_like(x)
    tris = np.stack([np.stack([x, z, z], 1), np.stack([1.25 * x, 0.25 * x, z], 1), np.stack([x, z, 0.25 * x], 1)], 1)
    s = rt.Scene()
    s.add_mesh(tris.astype(np.float32).reshape(-1, 3), rt.material(rt.MAT_DIFFUSE))
    return s


def test_bvh_deeper_than_the_traversal_stack_is_rejected():
    """The traversal keeps node groups on a 32-entry stack, so a tree deeper
    than RT_MAX_BVH_DEPTH levels could skip subtrees: the build reports the
    depth and refuses the tree (renderers and servers share the check)."""
    lib = rt.load_library()
    s = _chain_scene(-149, 127, 0.2)
    nodes, depth = C.c_int64(), C.c_int32()
    st = lib.rt_scene_build_bvh(s.handle, C.byref(nodes), C.byref(depth))
    assert depth.value > 32 and nodes.value > 0
    assert st == rt.RT_ERR_UNSUPPORTED
    assert "too deep" in lib.rt_last_error_message().decode()


def test_bvh_build_of_vanishing_centroid_extents():
    """Nodes whose centroid extent is so small that the bin scale overflows
    to infinity: every centroid must still land in one of the 32 bins."""
    s = _chain_scene(-120, 120, 0.5)
    nodes, depth = s.build_bvh()
    assert nodes >= 1 and 1 <= depth <= 32


def test_obj_loader(tmp_path):
    obj = tmp_path / "q.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nvn 0 0 1\n"
                   "f 1/1/1 2/2/1 3/3/1 4/4/1\nf -4 -2 -1\n")
    s = rt.Scene()
    mid = s.add_mesh_obj(obj, rt.material(rt.MAT_DIFFUSE))
    assert mid == 0 and s.counts()["triangles"] == 3  # quad fan-triangulated + one triangle
    with pytest.raises(rt.RTError):
        bad = tmp_path / "bad.obj"
        bad.write_text("v 0 0 0\nf 1 2 3\n")
        s.add_mesh_obj(bad, rt.material(rt.MAT_DIFFUSE))


def _write_hdr(path, img):
    """Writes a flat (non-RLE) Radiance RGBE file, top row first."""
    h, w = img.shape[:2]
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h - 1, -1, -1):
        for x in range(w):
            r, g, b = img[y, x, :3]
            m = max(r, g, b)
            if m < 1e-32:
                out += b"\0\0\0\0"
                continue
            mant, e = np.frexp(m)
            sc = mant * 256.0 / m
            out += bytes([int(r * sc), int(g * sc), int(b * sc), int(e + 128)])
    path.write_bytes(bytes(out))


def test_json_scene_loads_reference_schema(tmp_path):
    # models/test.json schema: width/height/depth/filter/camera/light/shape/material/medium
    (tmp_path / "box.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    env = np.ones((4, 8, 4), np.float32)
    env[1, 2, :3] = 5.0
    _write_hdr(tmp_path / "sky.hdr", env)
    text = """{
      "width": 80, "height": 60, "depth": 5, "spp": 3,
      "filter": {"type": "tent"},
      "camera": {"look_from": [0, 0, -3], "up": [0, 1, 0]},
      "light": [{"type": "infinite", "hdr_path": "sky.hdr", "scale": 2},
                {"type": "point", "position": [0, 2, 0], "radiance": [5, 5, 5]}],
      "shape": [{"type": "mesh", "mesh_path": "box.obj", "translate": [1, 0, 0], "rotate": [0, 90, 0],
                 "scale": [2, 2, 2], "material": "die1", "medium_int": "fog"}],
      "material": [{"type": "rough_dielectric", "name": "die1", "albedo_texture_type": "constant",
                    "albedo": [1, 1, 1], "roughness": 0.05, "int_ior": 1.5, "ext_ior": 1.0}],
      "medium": [{"type": "homogeneous", "name": "fog", "phase": "isotropic",
                  "sigma_a": [0.1, 0.2, 0.3], "sigma_s": [0, 0, 0], "scale": 0.6}],
      "tonemap": {"type": "aces", "exposure": 1.5}
    }"""
    (tmp_path / "scene.json").write_text(text)
    s = rt.Scene()
    o, cam = s.load_json(tmp_path / "scene.json")
    assert (o.width, o.height, o.max_depth, o.spp, o.filter) == (80, 60, 5, 3, rt.FILTER_TENT)
    assert o.tonemap == rt.TONEMAP_ACES_SRGB and o.exposure == pytest.approx(1.5)
    assert list(cam.from_) == [0, 0, -3]
    c = s.counts()
    assert c == {"triangles": 1, "meshes": 1, "lights": 1, "media": 1}
    lo, hi = s.bounds()
    # rotate 90 degrees about y, scale 2, translate x by 1: (1,0,0) -> (1, 0, -2)
    assert np.allclose(lo, [1, 0, -2], atol=1e-5) and np.allclose(hi, [1, 2, 0], atol=1e-5)
    # look_at defaults to the scene bounds centre (main.cpp:221)
    assert np.allclose(list(cam.at), (lo + hi) / 2, atol=1e-5)


def test_env_from_file_as_scene_add_env(tmp_path):
    """Scene::AddEnv(fileName) (core/src/Scene.cpp:79-81, 197-206): a Radiance
    file keeps its floats with row 0 at the bottom; an LDR image is converted
    as stbi_loadf converts it, (v/255)^2.2 for colour and v/255 for alpha."""
    rng = np.random.default_rng(3)
    env = rng.uniform(0.01, 20.0, (6, 10, 4)).astype(np.float32)
    env[..., 3] = 1.0
    _write_hdr(tmp_path / "sky.hdr", env)
    s = rt.Scene()
    assert s.get_env() is None
    s.set_env_file(tmp_path / "sky.hdr", scale=2.0)
    got = s.get_env()
    assert got.shape == (6, 10, 4)
    # RGBE: 8-bit mantissas under one shared exponent per pixel
    tol = 2.0 * env[..., :3].max(-1, keepdims=True) / 128
    assert np.all(np.abs(got[..., :3] - 2.0 * env[..., :3]) <= tol)
    # the same file through the JSON "infinite" light gives the same image
    s2 = rt.Scene()
    s2.load_json_string('{"light": [{"type": "infinite", "hdr_path": "sky.hdr", "scale": 2}]}', str(tmp_path))
    assert np.array_equal(s2.get_env(), got)
    px = rng.integers(0, 2 ** 32, (5, 7), dtype=np.uint64).astype(np.uint32)
    rt.write_png(tmp_path / "sky.png", px)
    s.set_env_file(tmp_path / "sky.png")
    ldr = s.get_env()
    b = px.view(np.uint8).reshape(5, 7, 4).astype(np.float64)
    np.testing.assert_allclose(ldr[..., :3], (b[..., :3] / 255.0) ** 2.2, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(ldr[..., 3], b[..., 3] / 255.0, rtol=1e-6)
    with pytest.raises(rt.RTError) as e:
        s.set_env_file(tmp_path / "missing.hdr")
    assert e.value.code == rt.RT_ERR_IO


def test_json_rejects_unknown_material_and_medium():
    s = rt.Scene()
    with pytest.raises(rt.RTError):
        s.load_json_string('{"material": [{"type": "velvet", "name": "x"}]}')
    with pytest.raises(rt.RTError):
        s.load_json_string('{"light": [{"type": "laser"}]}')
