"""Rendered-image parity of the wavefront CUDA renderer against the CPU
restatement of the reference integrator (core/cuda/devicePrograms.cu:170-532).

1. Same random streams: the GPU and the FP32 oracle draw identical numbers for
   each path, so they trace the same paths; pixels may only diverge where FP32
   rounding (FMA contraction, CUDA math-library ulps) flips a branch.
   At least 97% of pixels agree within 1e-3 relative and the image means agree
   within 1e-3 relative.
2. Independent streams: image means agree within 3 standard errors.
3. Renderer semantics: progressive running mean (devicePrograms.cu:524-529),
   AOVs (devicePrograms.cu:127-131, 514-531) and the tonemap
   (PostProcessing.cu:18-48).
"""
import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes
import pyoracle


def render_both(spec, frame_opts=None, **over):
    st = dict(spec.settings)
    st.update(over)
    s, r = scenes.build_renderer(spec, **over)
    r.render()
    gpu = r.download_linear()
    o = rt.options(**st)
    cam = rt.camera(**spec.camera)
    cpu, alb, nrm, nan = pyoracle.OracleScene(spec).render(o, cam)
    return r, gpu, cpu, alb, nrm


def pixel_agreement(a, b, rel=1e-3, floor=1e-3):
    d = np.abs(a[..., :3].astype(np.float64) - b[..., :3]).max(-1)
    m = np.maximum(np.abs(a[..., :3]), np.abs(b[..., :3])).max(-1)
    return (d <= rel * m + floor * rel).mean()


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", [rt.RNG_PCG32, rt.RNG_LCG])
def test_cornell_same_streams(rng_mode):
    spec = scenes.cornell(64, 64, 16)
    r, gpu, cpu, alb, nrm = render_both(spec, rng=rng_mode)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"rng {rng_mode}: pixels agreeing {agree:.4f}, means {mg:.6f} / {mc:.6f}")
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)
    assert np.allclose(gpu[..., 3], 1.0)
    ga, gn = r.download_aov(rt.AOV_ALBEDO), r.download_aov(rt.AOV_NORMAL)
    assert pixel_agreement(ga, alb, 1e-4) >= 0.97
    assert pixel_agreement(gn, nrm, 1e-4) >= 0.97


@pytest.mark.gpu
def test_cornell_independent_streams_mean_within_3se():
    spec = scenes.cornell(64, 64, 64)
    s, r = scenes.build_renderer(spec, seed=101)
    r.render()
    gpu = r.download_linear()[..., :3].astype(np.float64)
    o = rt.options(**dict(spec.settings, seed=202))
    cpu = pyoracle.OracleScene(spec).render(o, rt.camera(**spec.camera))[0][..., :3].astype(np.float64)
    # standard error of the mean difference, from the per-pixel difference image
    diff = (gpu - cpu).mean(-1)
    se = diff.std() / np.sqrt(diff.size)
    print(f"mean gpu {gpu.mean():.6f} cpu {cpu.mean():.6f} se {se:.2e}")
    assert abs(diff.mean()) <= 3 * se


@pytest.mark.gpu
def test_progressive_running_mean():
    spec = scenes.cornell(32, 32, 4)
    s, r = scenes.build_renderer(spec, progressive=1)
    frames = []
    for f in range(3):
        r.render()
        frames.append(r.download_linear().copy())
    assert r.frame_index() == 3
    sc = pyoracle.OracleScene(spec)
    o = rt.options(**dict(spec.settings, progressive=1))
    cam = rt.camera(**spec.camera)
    color = None
    for f in range(3):
        color = sc.render(o, cam, frame=f, color=color)[0]
    assert pixel_agreement(frames[-1], color) >= 0.97
    # SetCamera resets accumulation (Renderer.cpp:799)
    r.set_camera(cam)
    assert r.frame_index() == 0
    r.render()
    assert pixel_agreement(r.download_linear(), frames[0]) >= 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [rt.TONEMAP_REINHARD, rt.TONEMAP_ACES_SRGB])
def test_tonemap_matches_oracle(mode):
    spec = scenes.cornell(64, 64, 4)
    s, r = scenes.build_renderer(spec, tonemap=mode)
    r.render()
    lin = r.download_linear()
    px = r.download_pixels()
    ref = pyoracle.tonemap(lin, mode)
    a = px.view(np.uint8).reshape(px.shape + (4,)).astype(int)
    b = ref.view(np.uint8).reshape(ref.shape + (4,)).astype(int)
    assert np.abs(a - b).max() <= 1
    assert (a != b).any(axis=-1).mean() < 1e-3


@pytest.mark.gpu
def test_spheres_same_streams_small():
    """The 2.59M-triangle benchmark scene at 96x54, 4 spp."""
    spec = scenes.spheres(96, 54, 4, env_size=(512, 256))
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"spheres: agreeing {agree:.4f} means {mg:.5f} / {mc:.5f}")
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)


@pytest.mark.gpu
def test_c1_full_resolution_same_streams():
    """The benchmark configuration itself at 4 spp: 1920x1080, depth 16, the
    2.59M-triangle scene with its 2048x1024 sky (the spp is what the
    oracle's time bounds: about 5 s on 8 host threads)."""
    spec = scenes.spheres(1920, 1080, 4)
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"C1 full resolution: agreeing {agree:.5f} means {mg:.5f} / {mc:.5f}")
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)


@pytest.mark.gpu
def test_stats_and_resize():
    spec = scenes.cornell(32, 32, 2)
    s, r = scenes.build_renderer(spec, collect_stats=1)
    r.render()
    st = r.stats()
    assert st["paths"] == 32 * 32 * 2
    assert st["extend_rays"] >= st["paths"]
    assert st["nodes_visited"] > 0 and st["ms_total"] > 0
    r.resize(48, 16)
    r.render()
    assert r.download_linear().shape == (16, 48, 4)


@pytest.mark.gpu
def test_media_scene_same_streams():
    """Homogeneous fog, a density grid tracked against its majorant grid, a
    dielectric sphere, an area light and the sky (the media configuration at
    160x90, 16 spp, a 64^3 grid)."""
    spec = scenes.media(160, 90, 16, grid_res=64, env_size=(512, 256))
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"media: agreeing {agree:.4f} means {mg:.5f} / {mc:.5f}")
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)


@pytest.mark.gpu
def test_media_independent_streams_mean_within_3se():
    spec = scenes.media(96, 54, 64, grid_res=64, env_size=(512, 256))
    s, r = scenes.build_renderer(spec, seed=7)
    r.render()
    gpu = r.download_linear()[..., :3].astype(np.float64).mean(-1)
    o = rt.options(**dict(spec.settings, seed=8))
    cpu = pyoracle.OracleScene(spec).render(o, rt.camera(**spec.camera))[0][..., :3].astype(np.float64).mean(-1)
    d = gpu - cpu
    se = d.std() / np.sqrt(d.size)
    print(f"media mean gpu {gpu.mean():.5f} cpu {cpu.mean():.5f} se {se:.2e}")
    assert abs(d.mean()) <= 3 * se


@pytest.mark.gpu
def test_medium_step_budget_is_reported_as_a_watchdog_error():
    """A 128^3 grid whose 8^3 majorant cells each hold one dense voxel in
    empty space: the majorant is that voxel's density everywhere, so a walk
    through the medium takes ~10^5 tentative collisions (ratio tracking never
    stops early).  The device's 4096-step budget ends those walks with zero
    weight, and the host hears of it as RT_ERR_DEVICE_WATCHDOG from
    synchronize (no hang, no fault); the next ordinary render reports
    nothing."""
    spec = scenes.media(32, 24, 2, grid_res=128, env_size=(64, 32))
    grid = [md for md in spec.media if md["type"] == rt.MEDIUM_GRID][0]
    dens = np.zeros((128, 128, 128), np.float32)
    dens[8::16, 8::16, 8::16] = 1.0  # one voxel in each 16^3 block
    grid["density"] = dens
    grid["scale"] = 1e5
    s, r = scenes.build_renderer(spec)
    r.render()
    with pytest.raises(rt.RTError) as e:
        r.synchronize()
    assert e.value.code == rt.RT_ERR_DEVICE_WATCHDOG
    assert r.stats()["watchdog_walks"] > 0
    assert np.isfinite(r.download_linear()).all()
    s2, r2 = scenes.build_renderer(scenes.media(32, 24, 2, grid_res=16, env_size=(64, 32)))
    r2.render()
    r2.synchronize()
    assert r2.stats()["watchdog_walks"] == 0


@pytest.mark.gpu
def test_c0_cornell_exact_configuration():
    """C0 exactly: Cornell box, 34 triangles, 256x256, 16 spp, max depth 8,
    Russian roulette from depth 3, PCG32 seed 1, linear FP32 output; same
    streams as the FP32 oracle, then an independent stream within 3 SE."""
    spec = scenes.cornell(256, 256, 16, seed=1)
    st = spec.settings
    assert (st["width"], st["height"], st["spp"], st["max_depth"], st["rr_depth"], st["rng"], st["seed"]) == \
        (256, 256, 16, 8, 3, rt.RNG_PCG32, 1)
    assert sum(len(m.triangles()) for m in spec.meshes) == 34
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"C0: pixels agreeing {agree:.5f}, means {mg:.6f} / {mc:.6f}")
    assert agree >= 0.99
    assert abs(mg - mc) <= 1e-3 * abs(mc)
    o = rt.options(**dict(st, seed=2))
    ind = pyoracle.OracleScene(spec).render(o, rt.camera(**spec.camera))[0][..., :3].astype(np.float64).mean(-1)
    d = gpu[..., :3].astype(np.float64).mean(-1) - ind
    se = d.std() / np.sqrt(d.size)
    assert abs(d.mean()) <= 3 * se


@pytest.mark.gpu
def test_c2_media_full_grid_same_streams():
    """C2's medium at full size: the 128^3 fBm density grid (sigma_t 0-5,
    albedo 0.9, HG g = 0.6) with its 8^3 majorant grid inside the IOR-1.33
    sphere, the fog, the area light and the sky, depth 32, at 160x90 and
    16 spp (the oracle's time bounds the resolution)."""
    spec = scenes.media(160, 90, 16, grid_res=128, env_size=(512, 256))
    grid = [m for m in spec.media if m["type"] == rt.MEDIUM_GRID][0]
    assert grid["density"].shape == (128, 128, 128) and grid["majorant_res"] == 8
    assert 0.0 <= grid["density"].min() and grid["density"].max() <= 5.0
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"C2 full grid: agreeing {agree:.4f} means {mg:.5f} / {mc:.5f}")
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)
    r.synchronize()  # no walk ran out of its step budget


def _point_light_cornell(w, h, spp, seed=1):
    """The Cornell box lit by a point light (radiant intensity 1.2 W/sr) in
    place of the ceiling quad."""
    spec = scenes.cornell(w, h, spp, seed=seed)
    spec.lights[:] = [dict(type=rt.LIGHT_POINT, position=(0.5, 0.8, 0.4), radiance=(1.2, 1.0, 0.8))]
    return spec


@pytest.mark.gpu
def test_point_light_scene_same_and_independent_streams():
    """Point lights (no reference counterpart; NEE only, MIS weight 1):
    same-stream parity with the oracle and an independent stream within 3 SE."""
    spec = _point_light_cornell(96, 96, 16)
    r, gpu, cpu, alb, nrm = render_both(spec)
    agree = pixel_agreement(gpu, cpu)
    mg, mc = gpu[..., :3].mean(), cpu[..., :3].mean()
    print(f"point light: agreeing {agree:.4f} means {mg:.6f} / {mc:.6f}")
    assert mg > 0.01
    assert agree >= 0.97
    assert abs(mg - mc) <= 1e-3 * abs(mc)
    o = rt.options(**dict(spec.settings, seed=9))
    ind = pyoracle.OracleScene(spec).render(o, rt.camera(**spec.camera))[0][..., :3].astype(np.float64).mean(-1)
    d = gpu[..., :3].astype(np.float64).mean(-1) - ind
    assert abs(d.mean()) <= 3 * d.std() / np.sqrt(d.size)
