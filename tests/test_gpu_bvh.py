"""The acceleration structure built on the device (rt_scene_build_bvh_gpu and
the default scene upload) against the host build of the same rules: the wide
BVH validates on the host (every index in range, the triangle order a
permutation, every quantised box containing what it stands for), its size and
depth are close to the host build's, and renders and ray queries through
either BVH agree.
"""
import time

import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cornell", "spheres_small", "spheres", "media"])
def test_gpu_build_validates_and_matches_host_size(name):
    if name == "cornell":
        spec = scenes.cornell(8, 8, 1)
    elif name == "spheres_small":
        spec = scenes.spheres(8, 8, 1, ico_level=4, env_size=(16, 8))
    elif name == "spheres":
        spec = scenes.spheres(8, 8, 1, env_size=(16, 8))
    else:
        spec = scenes.media(8, 8, 1, grid_res=8, env_size=(16, 8))
    s = scenes.build_scene(spec)
    t0 = time.perf_counter()
    gn, gd = s.build_bvh_gpu()
    tg = time.perf_counter() - t0
    t0 = time.perf_counter()
    hn, hd = s.build_bvh()
    th = time.perf_counter() - t0
    print(f"{name}: GPU {gn} nodes depth {gd} ({tg * 1e3:.0f} ms incl. copies and host validation), "
          f"host {hn} nodes depth {hd} ({th * 1e3:.0f} ms)")
    assert gd <= 32
    assert abs(gn - hn) <= max(2, 0.1 * hn)
    assert abs(gd - hd) <= 3


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cornell", "spheres_small"])
def test_renders_through_gpu_and_host_bvh_agree(name):
    spec = scenes.cornell(48, 48, 4) if name == "cornell" else \
        scenes.spheres(64, 36, 2, ico_level=5, env_size=(256, 128))
    imgs = []
    for b in (rt.BVH_GPU, rt.BVH_HOST):
        s, r = scenes.build_renderer(spec, bvh_build=b)
        r.render()
        imgs.append(r.download_linear())
    same = np.all(np.abs(imgs[0] - imgs[1]) <= 1e-6 * np.maximum(1.0, np.abs(imgs[1])), axis=-1).mean()
    print(f"{name}: pixels equal {same:.4f}")
    assert same >= 0.999


@pytest.mark.gpu
def test_closest_hits_through_gpu_bvh_match_host_bvh():
    spec = scenes.spheres(16, 16, 1, ico_level=6, env_size=(16, 8))
    rng = np.random.default_rng(3)
    n = 1 << 16
    o = rng.uniform(-3, 3, (n, 3))
    d = rng.uniform(-1, 1, (n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3], rays[:, 3], rays[:, 4:7], rays[:, 7] = o, 1e-4, d, 3.0e38
    hits = []
    for b in (rt.BVH_GPU, rt.BVH_HOST):
        s, r = scenes.build_renderer(spec, bvh_build=b)
        hits.append(r.trace(rays))
    ids = [h[:, 3].view(np.int32) for h in hits]
    agree = (ids[0] == ids[1]).mean()
    print("closest-hit ids equal", agree)
    assert agree >= 0.9999
    hit = ids[1] >= 0
    assert np.allclose(hits[0][hit, 0], hits[1][hit, 0], rtol=1e-6)


@pytest.mark.gpu
def test_gpu_build_of_degenerate_chains():
    """Triangles at positions 2^e: binned SAH peels off a few per split, so
    the tree is a chain, and at the small end 32 / extent overflows (the
    device's saturating bin index keeps every centroid in a bin).  The chain
    that fits the traversal stack builds and validates on the device like on
    the host; the one deeper than RT_MAX_BVH_DEPTH is refused by both."""
    from test_capi import _chain_scene
    import ctypes as C
    lib = rt.load_library()
    s = _chain_scene(-120, 120, 0.5)
    gn, gd = s.build_bvh_gpu()
    hn, hd = s.build_bvh()
    assert gd <= 32 and abs(gd - hd) <= 3
    deep = _chain_scene(-149, 127, 0.2)
    nodes, depth = C.c_int64(), C.c_int32()
    st = lib.rt_scene_build_bvh_gpu(deep.handle, C.byref(nodes), C.byref(depth))
    # refused: deeper than the stack, or a tree the host validation rejects
    # (its wide levels exceed the validator's recursion bound), or a build error
    msg = lib.rt_last_error_message().decode()
    print(f"deep chain on the device: status {st}, depth {depth.value}: {msg}")
    assert st in (rt.RT_ERR_UNSUPPORTED, rt.RT_ERR_CUDA)
    assert depth.value > 32 or "BVH" in msg
    # a renderer refuses the scene too: its device-built tree is validated and,
    # when invalid, built again on the host, which finds it too deep
    with pytest.raises(rt.RTError) as e:
        rt.Renderer(deep, rt.options(width=4, height=4))
    assert "too deep" in str(e.value) or "BVH" in str(e.value)
