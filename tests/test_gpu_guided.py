"""Guided rendering with the learned proposal (rt_options.guided).

The guided estimator samples the trained vMF mixture with probability
guide_prob and the BSDF otherwise, weighting by the combined density (one-sample
MIS), and uses the combined density in the NEE weights: its expectation is the
plain estimator's.  Tests: the guided image agrees with a plain render within 3
standard errors; on the portal scene (light reaching the camera's half of a
room through an opening) the guided image has a lower relative MSE than the
plain one at equal samples per pixel.
"""
import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes


def relmse(img, ref):
    """mean over pixels and channels of (I - I_ref)^2 / (I_ref^2 + 1e-2)."""
    a, b = img[..., :3].astype(np.float64), ref[..., :3].astype(np.float64)
    return float(np.mean((a - b) ** 2 / (b * b + 1e-2)))


def render(spec, **over):
    s, r = scenes.build_renderer(spec, **over)
    r.render()
    return s, r, r.download_linear()


def assert_same_mean(a, b, label):
    d = (a[..., :3].astype(np.float64) - b[..., :3]).mean(-1)
    se = d.std() / np.sqrt(d.size)
    print(f"{label}: mean diff {d.mean():.3e} se {se:.3e}")
    assert abs(d.mean()) <= 3 * se


def _coated_cornell(w, h, spp):
    """The Cornell box with plastic walls and a rough clear-coated conductor
    box: the two materials whose BSDF sampler density differs from the
    evaluator's pdf."""
    spec = scenes.cornell(w, h, spp)
    for m in spec.meshes:
        if m.material["type"] == rt.MAT_DIFFUSE:
            m.material = dict(type=rt.MAT_PLASTIC, albedo=m.material["albedo"], roughness=0.4, int_ior=1.5,
                              ext_ior=1.0)
        else:
            m.material = dict(type=rt.MAT_CLEARCOATED_CONDUCTOR, albedo=(1.0, 1.0, 1.0), roughness=0.5,
                              coat_weight=1.0, coat_roughness_u=0.4, coat_roughness_v=0.4)
    return spec


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["portal", "cornell", "coated"])
def test_guided_agrees_with_plain_within_3se(name):
    spec = {"portal": scenes.portal, "cornell": scenes.cornell, "coated": _coated_cornell}[name](48, 48, 256)
    _, _, plain = render(spec, seed=101)
    _, _, guided = render(spec, seed=202, guided=1, guide_train_spp=32)
    assert np.isfinite(guided).all()
    assert_same_mean(guided, plain, name)


@pytest.mark.gpu
def test_guiding_lowers_relmse_at_equal_spp():
    """What the trained network gains: at 256 spp (the first 64 of them
    training it) the guided image is closer to a 4096-spp plain reference
    than the plain image is (measured about 1.2x lower relMSE), and the
    trained mixture explains the incident light much better than the
    untrained one (cross-entropy on its own training samples)."""
    spec = scenes.portal(256, 256, 4096)
    _, _, ref = render(spec, seed=9)
    eq = dict(spp=256)
    _, _, plain = render(spec, seed=10, **eq)
    s, r, _ = render(spec, seed=11, guided=1, guide_train_spp=0, **eq)  # guided by the untrained network
    assert len(r.guide_samples()) == 0  # no training wave ran
    untrained = r.guide()
    s2, r2, guided = render(spec, seed=11, guided=1, guide_train_spp=64, **eq)
    ep, eg = relmse(plain, ref), relmse(guided, ref)
    print(f"portal 256 spp: relMSE plain {ep:.4e} guided {eg:.4e} ratio {ep / eg:.2f}")
    assert eg < ep
    tr = r2.guide_samples()
    w = tr[:, 3] / tr[:, 3].sum()
    ce_trained = float(-(w * np.log(r2.guide().pdf(tr[:, :3], tr[:, 4:7]))).sum())
    ce_untrained = float(-(w * np.log(untrained.pdf(tr[:, :3], tr[:, 4:7]))).sum())
    print(f"cross-entropy of the last training wave: untrained {ce_untrained:.3f} trained {ce_trained:.3f}")
    assert ce_trained < ce_untrained - 0.5


@pytest.mark.gpu
def test_guided_training_spans_progressive_renders():
    spec = scenes.portal(32, 32, 16)
    s, r = scenes.build_renderer(spec, guided=1, guide_train_spp=32, progressive=1)
    for _ in range(4):
        r.render()
    img = r.download_linear()
    st = r.stats()
    assert np.isfinite(img).all() and st["paths"] == 32 * 32 * 16
    assert r.frame_index() == 4
    assert r.guide().last_loss()[1] == 32 * 4  # 32 training waves of 4 steps


@pytest.mark.gpu
def test_guided_options_are_checked():
    spec = scenes.cornell(8, 8, 1)
    with pytest.raises(rt.RTError):
        scenes.build_renderer(spec, guided=1, rng=rt.RNG_LCG)
    with pytest.raises(rt.RTError):
        scenes.build_renderer(spec, guided=1, guide_prob=0.0)
