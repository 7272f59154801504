"""Closest-hit and any-hit parity of the CUDA traversal against the FP64
watertight oracle (replaces optixTrace, core/cuda/devicePrograms.cu:258-269 and
:303-319).

A ray is a near-tie, and is excluded, when the FP64 hit lies within 1e-4 of an
edge relative to the magnitude of its edge-function terms, when the second
nearest FP64 hit is within 1e-5 (relative) of the nearest, or when the hit
distance is within 1e-5 of tmin.  Every other ray must report the same
triangle id bit-exactly, and the hit distance within 1e-5 of max(t, 1).
"""
import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes
import pyoracle

FMAX = np.float32(3.4028235e38)


def random_rays(rng, n, lo, hi, tmin=1e-4):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = o, tmin, d, FMAX
    return r


def camera_rays(spec, w, h, rng):
    cv = pyoracle.camera_vectors(rt.camera(**spec.camera), w, h).astype(np.float64)
    pos, dr, hor, ver = cv
    sx = (np.arange(w)[None, :] + rng.random((h, w))) / w
    sy = (np.arange(h)[:, None] + rng.random((h, w))) / h
    d = dr + (sx[..., None] - 0.5) * hor + (sy[..., None] - 0.5) * ver
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    r = np.zeros((h * w, 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = pos, 1e-4, d.reshape(-1, 3), FMAX
    return r


def compare(gpu, ref, rays):
    gid = gpu[:, 3].view(np.int32)
    rid = ref[:, 3].astype(np.int64)
    t, t2, margin = ref[:, 0], ref[:, 5], ref[:, 4]
    hit = rid >= 0
    tie = hit & ((margin < 1e-4) | ((t2 - t) <= 1e-5 * np.abs(t)) | (np.abs(t - rays[:, 3]) <= 1e-5 * np.abs(t)))
    keep = ~tie
    same = gid[keep] == rid[keep]
    bad = np.flatnonzero(keep)[~same]
    # FP32 error of the watertight distance scales with the ray length and
    # the origin's distance from the triangle, so it is measured against
    # max(t, 1) in scene units
    dt = np.abs(gpu[keep & hit, 0] - t[keep & hit]) / np.maximum(np.abs(t[keep & hit]), 1.0)
    return same.mean(), len(bad), tie.mean(), dt.max() if dt.size else 0.0, hit.mean()


def _check(spec, rays):
    s = scenes.build_scene(spec)
    r = rt.Renderer(s, rt.options(width=4, height=4))
    gpu = r.trace(rays)
    ref = pyoracle.OracleScene(spec).trace(rays, precision=64)
    frac, nbad, tie, dtmax, hitfrac = compare(gpu, ref, rays)
    print(f"{spec.name}: rays={len(rays)} hit={hitfrac:.3f} ties={tie:.5f} match={frac:.6f} bad={nbad} dt={dtmax:.2e}")
    assert nbad == 0, f"{nbad} non-tie rays disagree on the closest triangle"
    assert dtmax <= 1e-5
    assert tie < 0.01
    return r, s


@pytest.mark.gpu
def test_closest_hit_cornell():
    rng = np.random.default_rng(7)
    spec = scenes.cornell()
    rays = np.concatenate([random_rays(rng, 20000, 0.01, 0.99), camera_rays(spec, 64, 64, rng)])
    _check(spec, rays)


@pytest.mark.gpu
def test_closest_hit_full_size_spheres():
    """The 2.59M-triangle scene of the 1080p benchmark."""
    rng = np.random.default_rng(11)
    spec = scenes.spheres()
    assert spec.num_triangles == 1310720 + 64 * 20000
    rays = np.concatenate([random_rays(rng, 30000, -2.5, 2.5), camera_rays(spec, 192, 108, rng)])
    _check(spec, rays)


@pytest.mark.gpu
def test_any_hit_matches_closest_hit():
    rng = np.random.default_rng(5)
    spec = scenes.cornell()
    rays = random_rays(rng, 20000, 0.01, 0.99)
    rays[:, 7] = rng.uniform(0.05, 1.5, len(rays)).astype(np.float32)  # finite tmax
    s = scenes.build_scene(spec)
    r = rt.Renderer(s, rt.options(width=4, height=4))
    occ = r.trace(rays, any_hit=True)[:, 3].view(np.int32) == 1
    ref = pyoracle.OracleScene(spec).trace(rays, precision=64)
    ref_occ = ref[:, 3] >= 0
    t = ref[:, 0]
    near = np.abs(t - rays[:, 7]) <= 1e-5 * rays[:, 7]
    tie = (ref[:, 4] < 1e-4) | near
    assert np.array_equal(occ[~tie], ref_occ[~tie])


@pytest.mark.gpu
def test_empty_scene_and_device_pointers():
    torch = pytest.importorskip("torch")
    s = rt.Scene()
    r = rt.Renderer(s, rt.options(width=4, height=4))
    rays = random_rays(np.random.default_rng(1), 100, -1, 1)
    h = r.trace(rays)
    assert (h[:, 3].view(np.int32) == -1).all()
    # device-pointer path on a real scene
    spec = scenes.cornell()
    r2 = rt.Renderer(scenes.build_scene(spec), rt.options(width=4, height=4))
    rr = random_rays(np.random.default_rng(2), 4096, 0.01, 0.99)
    dr = torch.from_numpy(rr).cuda()
    dh = torch.empty((4096, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    r2.trace_device(dr.data_ptr(), 4096, dh.data_ptr())
    assert np.array_equal(dh.cpu().numpy().view(np.int32), r2.trace(rr).view(np.int32))
