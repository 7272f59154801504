"""Material textures: Scene::AddTexture (core/src/Scene.cpp:66-69, 181-189),
the texture overrides and normal map of __closesthit__radiance
(core/cuda/devicePrograms.cu:84-115) and the JSON "image" texture keys
(models/test.json:67-74).

Host tests check the image readers (BMP 8/24/32-bit, binary PGM/PPM) against
pixels written here, with stbi's vertical flip (row 0 = bottom); GPU tests
check a textured scene against the oracle on the same random streams.
"""
import os
import struct

import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes
import pyoracle


def _bmp(path, rgba, bpp, top_down=False):
    h, w = rgba.shape[:2]
    stride = (w * bpp // 8 + 3) & ~3
    rows = []
    order = range(h) if top_down else range(h)  # file row y = picture row y from the bottom (or top when top-down)
    for y in order:
        src = rgba[h - 1 - y] if top_down else rgba[y]
        if bpp == 24:
            row = src[:, [2, 1, 0]].tobytes()
        elif bpp == 32:
            row = src[:, [2, 1, 0, 3]].tobytes()
        else:
            row = bytes(src[:, 0])  # palette index = red value, grey palette
        rows.append(row + b"\0" * (stride - len(row)))
    pal = b"".join(bytes([i, i, i, 0]) for i in range(256)) if bpp == 8 else b""
    off = 14 + 40 + len(pal)
    data = b"".join(rows)
    hdr = struct.pack("<2sIHHI", b"BM", off + len(data), 0, 0, off)
    info = struct.pack("<IiiHHIIiiII", 40, w, -h if top_down else h, 1, bpp, 0, len(data), 2835, 2835,
                       256 if bpp == 8 else 0, 0)
    path.write_bytes(hdr + info + pal + data)


def _ppm(path, rgba, grey=False):
    h, w = rgba.shape[:2]
    top_first = rgba[::-1]  # PNM rows run top-down
    body = top_first[..., 0].tobytes() if grey else top_first[..., :3].tobytes()
    path.write_bytes((b"P5" if grey else b"P6") + f"\n# test\n{w} {h}\n255\n".encode() + body)


@pytest.fixture
def img():
    rng = np.random.default_rng(3)
    a = rng.integers(0, 256, (5, 7, 4), dtype=np.uint8)
    a[..., 3] = 255
    return a


@pytest.mark.parametrize("bpp,top_down", [(24, False), (32, False), (24, True), (8, False)])
def test_bmp_reader(tmp_path, img, bpp, top_down):
    a = img.copy()
    if bpp == 8:
        a[..., 1] = a[..., 2] = a[..., 0]
    p = tmp_path / "t.bmp"
    _bmp(p, a, bpp, top_down)
    s = rt.Scene()
    tid = s.add_texture_file(p)
    assert np.array_equal(s.get_texture(tid), a)


@pytest.mark.parametrize("grey", [False, True])
def test_pnm_reader(tmp_path, img, grey):
    a = img.copy()
    if grey:
        a[..., 1] = a[..., 2] = a[..., 0]
    p = tmp_path / ("t.pgm" if grey else "t.ppm")
    _ppm(p, a, grey)
    s = rt.Scene()
    assert np.array_equal(s.get_texture(s.add_texture_file(p)), a)


def test_texture_errors(tmp_path):
    s = rt.Scene()
    bad = tmp_path / "x.png"
    bad.write_bytes(b"\x89PNG....")
    with pytest.raises(rt.RTError):
        s.add_texture_file(bad)
    with pytest.raises(rt.RTError):
        s.add_texture(np.zeros((0, 4, 4), np.uint8))
    with pytest.raises(rt.RTError):
        s.get_texture(0)


def test_json_image_textures(tmp_path, img):
    _bmp(tmp_path / "alb.bmp", img, 24)
    _ppm(tmp_path / "nrm.ppm", img)
    (tmp_path / "q.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nf 1/1 2/2 3/3\n")
    js = """{"width": 8, "height": 8, "shape": [{"type": "mesh", "mesh_path": "q.obj", "material": 0}],
             "material": [{"type": "metal_workflow", "albedo_texture_type": "image", "albedo_path": "alb.bmp",
                           "normal_texture_type": "image", "normal_path": "nrm.ppm",
                           "roughness_texture_type": "constant", "roughness": 0.3}]}"""
    s = rt.Scene()
    s.load_json_string(js, str(tmp_path))
    assert np.array_equal(s.get_texture(0), img)
    assert np.array_equal(s.get_texture(1), img)
    missing = js.replace('"normal_path": "nrm.ppm",', "")
    with pytest.raises(rt.RTError):
        rt.Scene().load_json_string(missing, str(tmp_path))


def _agreement(a, b, rel=1e-3):
    d = np.abs(a[..., :3].astype(np.float64) - b[..., :3]).max(-1)
    m = np.maximum(np.abs(a[..., :3]), np.abs(b[..., :3])).max(-1)
    return (d <= rel * m + rel * 1e-3).mean()


@pytest.mark.gpu
def test_textured_scene_same_streams():
    spec = scenes.textured(64, 64, 16)
    s, r = scenes.build_renderer(spec)
    r.render()
    gpu = r.download_linear()
    o = rt.options(**spec.settings)
    cpu, alb, nrm, _ = pyoracle.OracleScene(spec).render(o, rt.camera(**spec.camera))
    ga, gn = r.download_aov(rt.AOV_ALBEDO), r.download_aov(rt.AOV_NORMAL)
    agree = _agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    aa, an = _agreement(ga, alb, 1e-4), _agreement(gn, nrm, 1e-4)
    print(f"textured: agreeing {agree:.4f} means {mg:.6f} / {mc:.6f}; albedo AOV {aa:.4f} normal AOV {an:.4f}")
    if os.environ.get("RT_DUMP_DIR"):
        np.savez(os.path.join(os.environ["RT_DUMP_DIR"], "textured.npz"), gpu=gpu, cpu=cpu, ga=ga, alb=alb, gn=gn,
                 nrm=nrm)
    assert aa >= 0.99  # checker and texture albedos in the first-hit AOV
    assert an >= 0.99  # the normal-mapped wall
    assert agree >= 0.97
    assert abs(mg - mc) <= 2e-3 * abs(mc)


@pytest.mark.gpu
def test_textures_change_the_image():
    spec = scenes.textured(48, 48, 8)
    plain = scenes.textured(48, 48, 8)
    for m in plain.meshes:
        m.material.pop("texture_ids", None)
    plain.textures = []
    imgs = []
    for sp in (spec, plain):
        s, r = scenes.build_renderer(sp)
        r.render()
        imgs.append(r.download_aov(rt.AOV_ALBEDO))
    assert np.abs(imgs[0] - imgs[1]).max() > 0.1
