"""Closest-hit and any-hit parity of the CUDA traversal against the FP64
watertight oracle (replaces optixTrace, core/cuda/devicePrograms.cu:258-269 and
:303-319).

Two device paths are checked: rt_renderer_trace (one thread per ray) and
rt_renderer_trace_wavefront, which runs the batch through the path tracer's
own persistent k_extend / k_shadow kernels (lane refill, triangle postponing)
with the launch shape Render() uses, so the traversal loop the benchmark times
is compared ray by ray with the oracle.

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


def tie_mask(ref, rays):
    t, t2, margin = ref[:, 0], ref[:, 5], ref[:, 4]
    hit = ref[:, 3] >= 0
    return hit & ((margin < 1e-4) | ((t2 - t) <= 1e-5 * np.abs(t)) | (np.abs(t - rays[:, 3]) <= 1e-5 * np.abs(t)))


def compare(gpu, ref, rays):
    gid = gpu[:, 3].view(np.int32)
    rid = ref[:, 3].astype(np.int64)
    t = ref[:, 0]
    hit = rid >= 0
    tie = tie_mask(ref, rays)
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


def surface_rays(spec, oracle, rng, n_cam=(192, 108)):
    """Secondary rays as the integrator traces them: from the FP64 hit point of
    a camera ray (rounded to FP32) into a random direction, tmin = 1e-4."""
    cam = camera_rays(spec, n_cam[0], n_cam[1], rng)
    ref = oracle.trace(cam, precision=64)
    hit = ref[:, 3] >= 0
    p = cam[hit, 0:3].astype(np.float64) + ref[hit, 0:1] * cam[hit, 4:7].astype(np.float64)
    d = rng.normal(size=(len(p), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((len(p), 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = p, 1e-4, d, FMAX
    return r


@pytest.fixture(scope="module")
def spheres_full():
    """The 2.59M-triangle scene of the 1080p benchmark, its renderer and its FP64 oracle."""
    spec = scenes.spheres()
    assert spec.num_triangles == 1310720 + 64 * 20000
    s = scenes.build_scene(spec)
    r = rt.Renderer(s, rt.options(width=4, height=4))
    return spec, s, r, pyoracle.OracleScene(spec)


def _occlusion_check(gpu_occ, ref, rays):
    """Any-hit parity: occluded iff the FP64 closest hit in [tmin, tmax) exists,
    excluding edge ties and hits within 1e-5 (relative) of tmax."""
    ref_occ = ref[:, 3] >= 0
    t = ref[:, 0]
    tmax = rays[:, 7].astype(np.float64)
    near = ref_occ & (np.abs(t - tmax) <= 1e-5 * np.abs(tmax))
    tie = (ref_occ & (ref[:, 4] < 1e-4)) | near
    bad = np.flatnonzero(~tie & (gpu_occ != ref_occ))
    return bad, tie.mean(), ref_occ.mean()


@pytest.mark.gpu
def test_wavefront_closest_hit_full_size_spheres(spheres_full):
    """k_extend, the benchmark's closest-hit kernel, on camera rays, rays from
    random points and rays leaving surfaces, against the FP64 oracle; and the
    same ids as the one-thread-per-ray path."""
    spec, s, r, orc = spheres_full
    rng = np.random.default_rng(21)
    rays = np.concatenate([random_rays(rng, 30000, -2.5, 2.5), camera_rays(spec, 192, 108, rng),
                           surface_rays(spec, orc, rng)])
    assert len(rays) >= 50000
    gpu, cnt = r.trace_wavefront(rays, counters=True)
    ref = orc.trace(rays, precision=64)
    frac, nbad, tie, dtmax, hitfrac = compare(gpu, ref, rays)
    print(f"wavefront closest: rays={len(rays)} hit={hitfrac:.3f} ties={tie:.5f} bad={nbad} dt={dtmax:.2e} "
          f"nodes/ray={cnt[1] / cnt[0]:.2f} tris/ray={cnt[2] / cnt[0]:.2f}")
    assert nbad == 0, f"{nbad} non-tie rays disagree on the closest triangle"
    assert dtmax <= 1e-5
    assert tie < 0.01
    assert cnt[0] == len(rays) and cnt[1] > 0 and cnt[2] > 0
    # the per-thread loop gives the same ids; only exactly equal FP32 distances
    # (near-ties) could resolve differently, since the loops test in different orders
    per_thread = r.trace(rays)
    differ = gpu[:, 3].view(np.int32) != per_thread[:, 3].view(np.int32)
    assert not (differ & ~tie_mask(ref, rays)).any(), f"{differ.sum()} rays differ between the two device loops"


@pytest.mark.gpu
@pytest.mark.parametrize("extent", ["finite", "infinite"])
def test_wavefront_any_hit_full_size_spheres(spheres_full, extent):
    """k_shadow, the benchmark's any-hit kernel: shadow rays towards points
    (finite tmax) and towards the environment (tmax = FLT_MAX), from surfaces
    and from free space, against the FP64 oracle."""
    spec, s, r, orc = spheres_full
    rng = np.random.default_rng(31 if extent == "finite" else 37)
    rays = np.concatenate([random_rays(rng, 35000, -2.5, 2.5), surface_rays(spec, orc, rng, n_cam=(320, 180))])
    if extent == "finite":
        rays[:, 7] = rng.uniform(0.02, 3.0, len(rays)).astype(np.float32)
    assert len(rays) >= 50000
    gpu, cnt = r.trace_wavefront(rays, any_hit=True, counters=True)
    occ = gpu[:, 3].view(np.int32) == 1
    ref = orc.trace(rays, precision=64)
    bad, tie, occ_frac = _occlusion_check(occ, ref, rays)
    print(f"wavefront any-hit ({extent}): rays={len(rays)} occluded={occ_frac:.3f} ties={tie:.5f} bad={len(bad)} "
          f"nodes/ray={cnt[1] / cnt[0]:.2f} tris/ray={cnt[2] / cnt[0]:.2f}")
    assert len(bad) == 0, f"{len(bad)} non-tie rays disagree on occlusion"
    assert 0.05 < occ_frac < 0.95  # both outcomes well represented
    assert tie < 0.01
    # the per-thread any-hit path agrees on every non-tie ray too
    occ_pt = r.trace(rays, any_hit=True)[:, 3].view(np.int32) == 1
    bad_pt, _, _ = _occlusion_check(occ_pt, ref, rays)
    assert len(bad_pt) == 0


@pytest.mark.gpu
def test_wavefront_cornell_and_chunking():
    """Cornell box through both wavefront kernels, with a batch above one
    wave (2^22 rays) so the chunked path runs; extents the kernels do not
    trace are refused."""
    rng = np.random.default_rng(41)
    spec = scenes.cornell()
    s = scenes.build_scene(spec)
    r = rt.Renderer(s, rt.options(width=4, height=4))
    orc = pyoracle.OracleScene(spec)
    rays = np.concatenate([random_rays(rng, 20000, 0.01, 0.99), camera_rays(spec, 64, 64, rng)])
    gpu = r.trace_wavefront(rays)
    ref = orc.trace(rays, precision=64)
    _, nbad, tie, dtmax, _ = compare(gpu, ref, rays)
    assert nbad == 0 and dtmax <= 1e-5 and tie < 0.01
    sh = rays.copy()
    sh[:, 7] = rng.uniform(0.05, 1.5, len(sh)).astype(np.float32)
    occ = r.trace_wavefront(sh, any_hit=True)[:, 3].view(np.int32) == 1
    bad, _, _ = _occlusion_check(occ, orc.trace(sh, precision=64), sh)
    assert len(bad) == 0
    big = np.tile(rays, ((1 << 22) // len(rays) + 2, 1))
    assert len(big) > 1 << 22
    hb = r.trace_wavefront(big)
    assert np.array_equal(hb[:, 3].view(np.int32), np.tile(gpu[:, 3].view(np.int32), len(big) // len(rays)))
    bad_tmin = rays[:10].copy()
    bad_tmin[:, 3] = 0.0
    with pytest.raises(rt.RTError):
        r.trace_wavefront(bad_tmin)
    bad_tmax = rays[:10].copy()
    bad_tmax[:, 7] = 2.0
    with pytest.raises(rt.RTError):
        r.trace_wavefront(bad_tmax)
    assert r.trace_wavefront(np.zeros((0, 8), np.float32)).shape == (0, 4)
