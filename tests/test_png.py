"""PNG textures (Scene::AddTexture, core/src/Scene.cpp:66-69, which uses
stb_image: RGBA, row 0 = bottom) and PNG frame output (rt_write_png).

The decoder is checked against PNG files written here with Python's zlib at
full compression (dynamic Huffman blocks), every row filter, every colour type
and bit depth, and against files written by Pillow when it is installed.
"""
import struct
import zlib

import numpy as np
import pytest

import optixrender_b200 as rt


def _chunk(t, data):
    return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xFFFFFFFF)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def _filter(rows, bpp):
    """Each row gets filter type y % 5 (None, Sub, Up, Average, Paeth)."""
    out = []
    prev = np.zeros_like(rows[0], dtype=np.int32)
    for y, row in enumerate(rows):
        r = row.astype(np.int32)
        a = np.concatenate([np.zeros(bpp, np.int32), r[:-bpp]])
        c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        f = y % 5
        pred = [0, a, prev, (a + prev) // 2, _paeth(a, prev, c)][f]
        out.append(bytes([f]) + ((r - pred) % 256).astype(np.uint8).tobytes())
        prev = r
    return b"".join(out)


def _png(rows_bytes, w, h, depth, ctype, bpp, extra=b"", interlace=0, level=9):
    raw = _filter([np.frombuffer(r, np.uint8) for r in rows_bytes], bpp)
    ihdr = struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, interlace)
    z = zlib.compress(raw, level)
    return b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", ihdr) + extra + _chunk(b"IDAT", z[:7]) + \
        _chunk(b"IDAT", z[7:]) + _chunk(b"IEND", b"")


def _load(tmp_path, data, name="t.png"):
    p = tmp_path / name
    p.write_bytes(data)
    s = rt.Scene()
    return s.get_texture(s.add_texture_file(p))


@pytest.fixture
def img():
    rng = np.random.default_rng(7)
    a = rng.integers(0, 256, (13, 17, 4), dtype=np.uint8)
    a[3:7, 4:9] = a[3, 4]  # runs that the compressor turns into back-references
    return a


def _top_first(rgba):
    return rgba[::-1]  # PNG rows run top-down; the texture's row 0 is the bottom


@pytest.mark.parametrize("ctype", [6, 2, 4, 0])
def test_8bit_colour_types(tmp_path, img, ctype):
    h, w = img.shape[:2]
    ch = {6: [0, 1, 2, 3], 2: [0, 1, 2], 4: [0, 3], 0: [0]}[ctype]
    rows = [r[:, ch].tobytes() for r in _top_first(img)]
    got = _load(tmp_path, _png(rows, w, h, 8, ctype, len(ch)))
    want = img.copy()
    if ctype in (0, 4):
        want[..., 1] = want[..., 2] = want[..., 0]
    if ctype in (0, 2):
        want[..., 3] = 255
    assert np.array_equal(got, want)


def test_16bit_rgba_takes_the_high_byte(tmp_path, img):
    h, w = img.shape[:2]
    lo = np.random.default_rng(1).integers(0, 256, img.shape, dtype=np.uint8)
    px16 = (img.astype(np.uint16) << 8) | lo
    rows = [r.astype(">u2").tobytes() for r in _top_first(px16)]
    assert np.array_equal(_load(tmp_path, _png(rows, w, h, 16, 6, 8)), img)


@pytest.mark.parametrize("depth", [1, 2, 4, 8])
def test_palette_with_transparency(tmp_path, depth):
    h, w = 9, 11
    n = 1 << depth
    rng = np.random.default_rng(depth)
    pal = rng.integers(0, 256, (n, 3), dtype=np.uint8)
    alpha = rng.integers(0, 256, n // 2 + 1, dtype=np.uint8)  # tRNS may be shorter than the palette
    idx = rng.integers(0, n, (h, w))
    rows = []
    for r in idx[::-1]:
        bits = "".join(format(int(v), f"0{depth}b") for v in r)
        bits += "0" * (-len(bits) % 8)
        rows.append(int(bits, 2).to_bytes(len(bits) // 8, "big"))
    extra = _chunk(b"PLTE", pal.tobytes()) + _chunk(b"tRNS", alpha.tobytes())
    got = _load(tmp_path, _png(rows, w, h, depth, 3, 1, extra))
    want = np.zeros((h, w, 4), np.uint8)
    want[..., :3] = pal[idx]
    full_alpha = np.full(n, 255, np.uint8)
    full_alpha[: len(alpha)] = alpha
    want[..., 3] = full_alpha[idx]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("depth", [1, 2, 4])
def test_low_bit_grey_scales_to_8_bits(tmp_path, depth):
    h, w = 5, 9
    v = np.random.default_rng(3).integers(0, 1 << depth, (h, w))
    rows = []
    for r in v[::-1]:
        bits = "".join(format(int(x), f"0{depth}b") for x in r)
        bits += "0" * (-len(bits) % 8)
        rows.append(int(bits, 2).to_bytes(len(bits) // 8, "big"))
    got = _load(tmp_path, _png(rows, w, h, depth, 0, 1))
    g = (v * 255 // ((1 << depth) - 1)).astype(np.uint8)
    assert np.array_equal(got[..., 0], g) and np.array_equal(got[..., 2], g) and (got[..., 3] == 255).all()


def test_stored_and_fixed_blocks(tmp_path, img):
    h, w = img.shape[:2]
    rows = [r.tobytes() for r in _top_first(img)]
    for level in (0, 1):  # level 0: stored blocks; level 1: usually fixed Huffman
        assert np.array_equal(_load(tmp_path, _png(rows, w, h, 8, 6, 4, level=level)), img)


def test_write_png_round_trip(tmp_path, img):
    px = img.view(np.uint32).reshape(img.shape[:2])
    p = tmp_path / "frame.png"
    rt.write_png(p, px)
    s = rt.Scene()
    assert np.array_equal(s.get_texture(s.add_texture_file(p)), img)


def test_pillow_files(tmp_path, img):
    Image = pytest.importorskip("PIL.Image")
    p = tmp_path / "pil.png"
    Image.fromarray(_top_first(img), "RGBA").save(p, optimize=True)
    s = rt.Scene()
    assert np.array_equal(s.get_texture(s.add_texture_file(p)), img)
    q = tmp_path / "pil_frame.png"
    rt.write_png(q, img.view(np.uint32).reshape(img.shape[:2]))
    assert np.array_equal(np.asarray(Image.open(q).convert("RGBA")), _top_first(img))


def test_png_errors(tmp_path, img):
    h, w = img.shape[:2]
    rows = [r.tobytes() for r in _top_first(img)]
    good = _png(rows, w, h, 8, 6, 4)
    bad_crc = bytearray(good)
    bad_crc[40] ^= 0xFF  # inside the first IDAT chunk
    for data in (bytes(bad_crc), good[:60], _png(rows, w, h, 8, 6, 4, interlace=1)):
        with pytest.raises(rt.RTError):
            _load(tmp_path, data)


def test_corrupted_files_fail_cleanly(tmp_path, img):
    """Random byte flips in the compressed data of PNG and JPEG files (CRCs
    recomputed so the PNG damage reaches the inflater) end in an error or a
    decoded image, never in a crash."""
    h, w = img.shape[:2]
    rows = [r.tobytes() for r in _top_first(img)]
    png = bytearray(_png(rows, w, h, 8, 6, 4))
    rng = np.random.default_rng(11)
    start = png.index(b"IDAT") + 4
    for k in range(200):
        bad = bytearray(png)
        for _ in range(int(rng.integers(1, 6))):
            bad[int(rng.integers(start, len(bad) - 12))] = int(rng.integers(0, 256))
        # recompute the CRC of every chunk
        pos = 8
        while pos + 12 <= len(bad):
            n = struct.unpack(">I", bad[pos:pos + 4])[0]
            if pos + 12 + n > len(bad):
                break
            bad[pos + 8 + n:pos + 12 + n] = struct.pack(">I", zlib.crc32(bytes(bad[pos + 4:pos + 8 + n])) & 0xFFFFFFFF)
            pos += 12 + n
        try:
            _load(tmp_path, bytes(bad), f"f{k}.png")
        except rt.RTError:
            pass
    try:
        from PIL import Image
    except ImportError:
        return
    import io
    b = io.BytesIO()
    Image.fromarray(img[..., :3]).save(b, "JPEG", quality=80)
    jpg = bytearray(b.getvalue())
    for k in range(200):
        bad = bytearray(jpg)
        for _ in range(int(rng.integers(1, 6))):
            bad[int(rng.integers(2, len(bad)))] = int(rng.integers(0, 256))
        try:
            _load(tmp_path, bytes(bad), f"f{k}.jpg")
        except rt.RTError:
            pass
