"""Baseline JPEG textures (Scene::AddTexture reads JPEG through stb_image,
core/src/Scene.cpp:181-189).  Files are written by Pillow and the decoder's
pixels compared with Pillow's own decode of the same file: within rounding
for 4:4:4 and grey (different inverse DCTs); with subsampled chroma both
interpolate between chroma sample centres, so a few levels at most."""
import io

import numpy as np
import pytest

import optixrender_b200 as rt

Image = pytest.importorskip("PIL.Image")


def _picture(h=45, w=67):
    y, x = np.mgrid[0:h, 0:w]
    img = np.zeros((h, w, 3), np.float64)
    img[..., 0] = 128 + 100 * np.sin(x / 9.0)
    img[..., 1] = 128 + 90 * np.cos(y / 7.0)
    img[..., 2] = 60 + 2.5 * (x + y)
    img[15:30, 20:40] = (200, 40, 90)  # a flat block with edges
    return np.clip(img, 0, 255).astype(np.uint8)


def _decode(tmp_path, data, name="t.jpg"):
    p = tmp_path / name
    p.write_bytes(data)
    s = rt.Scene()
    return s.get_texture(s.add_texture_file(p))


def _save(img, mode="RGB", **kw):
    b = io.BytesIO()
    Image.fromarray(img, mode).save(b, "JPEG", **kw)
    return b.getvalue()


def _pillow(data):
    return np.asarray(Image.open(io.BytesIO(data)).convert("RGB"))


@pytest.mark.parametrize("quality", [50, 95])
def test_444_matches_pillow(tmp_path, quality):
    data = _save(_picture(), quality=quality, subsampling=0)
    got = _decode(tmp_path, data)[::-1]  # row 0 is the bottom
    want = _pillow(data)
    d = np.abs(got[..., :3].astype(int) - want.astype(int))
    print("4:4:4 max", d.max(), "mean", d.mean())
    assert d.max() <= 3 and d.mean() < 0.6 and (got[..., 3] == 255).all()


@pytest.mark.parametrize("subsampling", [1, 2])  # 4:2:2, 4:2:0
def test_subsampled_chroma(tmp_path, subsampling):
    data = _save(_picture(), quality=90, subsampling=subsampling)
    got = _decode(tmp_path, data)[::-1]
    d = np.abs(got[..., :3].astype(int) - _pillow(data).astype(int))
    print("subsampled max", d.max(), "mean", d.mean())
    assert d.max() <= 4 and d.mean() < 0.6


def test_grey_and_odd_sizes(tmp_path):
    g = _picture(13, 29)[..., 1]
    data = _save(g, "L", quality=90)
    got = _decode(tmp_path, data)[::-1]
    want = np.asarray(Image.open(io.BytesIO(data)))
    assert np.abs(got[..., 0].astype(int) - want.astype(int)).max() <= 3
    assert np.array_equal(got[..., 0], got[..., 1]) and np.array_equal(got[..., 0], got[..., 2])


def test_restart_intervals(tmp_path):
    try:
        data = _save(_picture(), quality=90, subsampling=0, restart_marker_blocks=3)
    except TypeError:
        pytest.skip("this Pillow cannot write restart markers")
    if b"\xff\xdd" not in data:
        pytest.skip("this Pillow ignored the restart interval")
    got = _decode(tmp_path, data)[::-1]
    assert np.abs(got[..., :3].astype(int) - _pillow(data).astype(int)).max() <= 3


def test_progressive_is_rejected(tmp_path):
    data = _save(_picture(), quality=90, progressive=True)
    with pytest.raises(rt.RTError) as e:
        _decode(tmp_path, data)
    assert e.value.code == rt.RT_ERR_IO
