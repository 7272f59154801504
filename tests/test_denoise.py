"""The denoiser behind Options.denoise (the reference's denoiserOn,
core/src/Renderer.cpp:660-785, whose OptiX AI denoiser is a closed library):
an edge-avoiding a-trous wavelet filter on irradiance, guided by the first-hit
albedo and normal AOVs.

The CUDA kernels are checked against the plain FP32 numpy restatement below
(tolerance 1e-4 relative: the kernel uses the fast exponential), and the
filter's purpose against a high-spp render: at 4 spp the denoised Cornell box
is several times closer to the reference than the noisy image.
"""
import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes

PASSES, SIGMA_C, SIGMA_N, SIGMA_A, ALBEDO_MIN, FIREFLY = 5, 1.0, 0.3, 0.1, 1e-3, 4.0
HK = np.array([1 / 16, 1 / 4, 3 / 8, 1 / 4, 1 / 16], np.float32)


def denoise_ref(color, albedo, normal):
    """FP32 numpy restatement of k_dn_demod, k_dn_clamp, 5 x k_dn_atrous, k_dn_remod."""
    c3, a3, n3 = (x[..., :3].astype(np.float32) for x in (color, albedo, normal))
    f = np.where(a3 > ALBEDO_MIN, a3, np.float32(1.0))
    irr = c3 / f
    h, w = irr.shape[:2]
    lum = 0.2126 * irr[..., 0] + 0.7152 * irr[..., 1] + 0.0722 * irr[..., 2]
    pad = np.pad(lum, 1, constant_values=0.0)
    nb = np.stack([pad[1 + j:1 + j + h, 1 + i:1 + i + w] for j in (-1, 0, 1) for i in (-1, 0, 1) if (i, j) != (0, 0)])
    bound = np.float32(FIREFLY) * nb.max(0)
    scale = np.where((lum > bound) & (lum > 0), bound / np.where(lum > 0, lum, 1), 1.0).astype(np.float32)
    irr = irr * scale[..., None]
    inv_sc2 = np.float32(1.0 / (SIGMA_C * SIGMA_C))
    inv_sn2, inv_sa2 = np.float32(1.0 / SIGMA_N ** 2), np.float32(1.0 / SIGMA_A ** 2)
    ys, xs = np.mgrid[0:h, 0:w]
    for it in range(PASSES):
        step = 1 << it
        lp = 0.2126 * irr[..., 0] + 0.7152 * irr[..., 1] + 0.0722 * irr[..., 2]
        cs = inv_sc2 / (lp * lp + np.float32(1e-4))
        acc = np.zeros_like(irr)
        ws = np.zeros((h, w), np.float32)
        for j in range(-2, 3):
            for i in range(-2, 3):
                yy, xx = ys + j * step, xs + i * step
                ok = (yy >= 0) & (yy < h) & (xx >= 0) & (xx < w)
                yc, xc = np.clip(yy, 0, h - 1), np.clip(xx, 0, w - 1)
                cq, nq, aq = irr[yc, xc], n3[yc, xc], a3[yc, xc]
                dc = ((cq - irr) ** 2).sum(-1)
                dn = ((nq - n3) ** 2).sum(-1)
                da = ((aq - a3) ** 2).sum(-1)
                wq = HK[i + 2] * HK[j + 2] * np.exp(-(dc * cs + dn * inv_sn2 + da * inv_sa2)) * ok
                acc += wq[..., None] * cq
                ws += wq
        irr = acc / ws[..., None]
        inv_sc2 = inv_sc2 * 4
    out = np.ones(color.shape, np.float32)
    out[..., :3] = irr * f
    return out


def _random_case(h=37, w=53, seed=3):
    rng = np.random.default_rng(seed)
    color = np.ones((h, w, 4), np.float32)
    albedo = np.ones((h, w, 4), np.float32)
    normal = np.ones((h, w, 4), np.float32)
    color[..., :3] = rng.gamma(1.0, 0.5, (h, w, 3))
    albedo[..., :3] = np.where(rng.random((h, w, 1)) < 0.1, 0.0, rng.uniform(0.2, 0.9, (h, w, 3)))
    albedo[: h // 2, :, :3] = 0.7  # a flat region and an edge
    n = rng.normal(size=(h, w, 3))
    n[:, : w // 2] = (0.0, 1.0, 0.0)
    normal[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    return color, albedo, normal


def test_reference_filter_properties():
    """The numpy restatement: a constant image stays constant, and the filter
    does not mix across a normal edge."""
    h, w = 24, 24
    c = np.ones((h, w, 4), np.float32) * 0.5
    a = np.ones((h, w, 4), np.float32) * 0.5
    n = np.zeros((h, w, 4), np.float32)
    n[..., 1] = 1.0
    assert np.allclose(denoise_ref(c, a, n)[..., :3], c[..., :3], rtol=1e-6)
    c2 = c.copy()
    c2[:, w // 2:, :3] = 2.0
    n2 = n.copy()
    n2[:, w // 2:, 1] = 0.0
    n2[:, w // 2:, 0] = 1.0
    out = denoise_ref(c2, a, n2)
    assert np.allclose(out[:, : w // 2, :3], 0.5, rtol=1e-3) and np.allclose(out[:, w // 2:, :3], 2.0, rtol=1e-3)


@pytest.mark.gpu
def test_kernels_match_the_fp32_restatement():
    color, albedo, normal = _random_case()
    got = rt.denoise_image(color, albedo, normal)
    ref = denoise_ref(color, albedo, normal)
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-6)
    print("max rel diff", rel.max())
    assert rel.max() < 1e-4


@pytest.mark.gpu
def test_denoised_render_is_closer_to_the_reference():
    spec = scenes.cornell(128, 128, 1024)
    _, r_ref = scenes.build_renderer(spec, seed=5)
    r_ref.render()
    ref = r_ref.download_linear()

    def relmse(img):
        a, b = img[..., :3].astype(np.float64), ref[..., :3].astype(np.float64)
        return float(np.mean((a - b) ** 2 / (b * b + 1e-2)))

    _, r = scenes.build_renderer(spec, spp=4, seed=6, denoise=1)
    r.render()
    noisy, den = r.download_linear(), r.download_aov(rt.AOV_DENOISED)
    px = r.download_pixels()
    e_noisy, e_den = relmse(noisy), relmse(den)
    print(f"relMSE noisy {e_noisy:.4e} denoised {e_den:.4e} ratio {e_noisy / e_den:.1f}")
    assert e_den < e_noisy / 3
    # the displayed image is the denoised colour, as with the reference's denoiser
    _, r2 = scenes.build_renderer(spec, spp=4, seed=6)
    r2.render()
    assert np.array_equal(r2.download_linear(), noisy)
    assert not np.array_equal(r2.download_pixels(), px)
    with pytest.raises(rt.RTError) as e:
        r2.download_aov(rt.AOV_DENOISED)
    assert e.value.code == rt.RT_ERR_STATE
