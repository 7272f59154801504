"""The reference's own shading code on the CPU (oracle/_ref/libref_pt.so)
against the oracle's restatement: independent RNG streams, so the image means
must agree within 3 standard errors.  The scene keeps every surface in front
of the one-sided light, where the reference and the oracle do the same thing
(the oracle drops zero-pdf light samples, the reference turns them into NaN)."""
import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes
import pyoracle
import refpt


@pytest.mark.skipif(not refpt.available(), reason="reference host build not present")
def test_reference_cpu_path_matches_oracle_statistics():
    spec = scenes.cornell(48, 48, 64)
    spec.lights[0]["double_side"] = 1   # no surface behind the light: both methods are identical here
    o = rt.options(**dict(spec.settings, rng=rt.RNG_LCG))
    cam = rt.camera(**spec.camera)
    ref = refpt.RefScene(spec).render(o, cam)[..., :3].astype(np.float64).mean(-1)
    o2 = rt.options(**dict(spec.settings, rng=rt.RNG_PCG32, seed=5))  # an independent stream
    orc = pyoracle.OracleScene(spec).render(o2, cam)[0][..., :3].astype(np.float64).mean(-1)
    d = ref - orc
    se = d.std() / np.sqrt(d.size)
    print(f"reference {ref.mean():.5f} oracle {orc.mean():.5f} se {se:.2e}")
    assert abs(d.mean()) <= 3 * se
