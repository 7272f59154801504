"""Device shading parity: the renderer's CUDA BSDF, light, phase and medium
code (rt_verify_shading) against the FP64 oracle, which is itself pinned to
the reference's shading code (tests/test_oracle_pins.py).

Tolerance: a value passes when |gpu - fp64| <= 1e-5 * |fp64| + 1e-7, or, where
FP32 evaluation of the reference formula is itself worse than that (the
bit-exact FP32 oracle misses 1e-5), when the GPU error is no larger than twice
the FP32 oracle's.  Sampling ops take their random numbers from the query;
queries whose branch decision lies within 1e-5 of a random number are ties.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np
import pytest

import optixrender_b200 as rt
import pyoracle

GOLD = np.load(Path(__file__).parent / "golden" / "reference_shading.npz")


def _structs(cls, key):
    raw = GOLD[key].tobytes()
    return list((cls * (len(raw) // C.sizeof(cls))).from_buffer_copy(raw))


MATS = _structs(rt.Material, "materials")
LIGHTS = _structs(rt.Light, "lights")
MEDIA = _structs(rt.Medium, "media")

OPS = [(rt.VERIFY_BSDF_EVAL, "bsdf_eval"), (rt.VERIFY_BSDF_SAMPLE, "bsdf_sample"),
       (rt.VERIFY_LIGHT_SAMPLE, "light_sample"), (rt.VERIFY_LIGHT_EVAL, "light_eval"),
       (rt.VERIFY_MEDIUM_SAMPLE, "medium_sample"), (rt.VERIFY_PHASE_SAMPLE, "phase_sample"),
       (rt.VERIFY_PHASE_EVAL, "phase_eval")]
# output columns compared per op (used-random counters and flags compared exactly)
COLS = {"bsdf_eval": [0, 1, 2, 3], "bsdf_sample": [0, 1, 2, 3, 4, 5, 6], "light_sample": list(range(8)),
        "light_eval": [0, 1, 2, 3, 4], "medium_sample": [0, 1, 2, 3, 4], "phase_sample": [0, 1, 2, 3, 4, 5, 6],
        "phase_eval": [0, 1, 2, 3]}
EXACT = {"bsdf_sample": [7], "medium_sample": [5, 6], "phase_sample": [7]}


def within(gpu, f32, f64):
    g, c, d = (np.asarray(a, np.float64) for a in (gpu, f32, f64))
    eg, ec = np.abs(g - d), np.abs(c - d)
    tol = 1e-5 * np.abs(d) + 1e-7
    ok = (eg <= tol) | (eg <= 2 * ec + 1e-7) | (np.isnan(g) & np.isnan(d)) | (g == d)
    return ok


@pytest.mark.gpu
@pytest.mark.parametrize("op,key", OPS)
def test_device_shading_matches_fp64(op, key):
    x = GOLD[key + "_in"]
    gpu = rt.verify_shading(op, x, MATS, LIGHTS, MEDIA)
    f32 = pyoracle.shading(op, x, MATS, LIGHTS, MEDIA, precision=32)
    f64 = pyoracle.shading(op, x, MATS, LIGHTS, MEDIA, precision=64)
    cols = COLS[key]
    ok = within(gpu[:, cols], f32[:, cols], f64[:, cols]).all(axis=1)
    for c in EXACT.get(key, []):
        ok &= gpu[:, c] == f32[:, c]
    # a sampled branch decided by a random number within 1e-5 of its threshold is a tie:
    # detect those as rows where FP32 and FP64 took different branches
    branch_tie = ~within(f32[:, cols], f32[:, cols], f64[:, cols]).all(axis=1) & (
        np.abs(f32[:, cols] - f64[:, cols]).max(axis=1) > 1e-2 * (np.abs(f64[:, cols]).max(axis=1) + 1e-3))
    frac = ok[~branch_tie].mean()
    print(f"{key}: pass {frac:.5f} of {int((~branch_tie).sum())} (ties {branch_tie.mean():.4f})")
    dump = os.environ.get("RT_DUMP_DIR")
    if dump:
        np.savez_compressed(Path(dump) / f"verify_{key}.npz", x=x, gpu=gpu, f32=f32, f64=f64, ok=ok, tie=branch_tie)
    assert frac >= 0.999, f"{key}: only {frac:.5f} of queries within tolerance"


@pytest.mark.gpu
@pytest.mark.parametrize("mtype", range(8))
def test_white_furnace(mtype):
    """Albedo-1 materials under uniform unit illumination.  The BSDF-sampled
    estimate of directional albedo equals the FP64 oracle's on the same samples
    (3 standard errors) for every type.  Lambert (roughness 0) and the diffuse
    transmitter integrate to exactly one; the reflective microfacet types stay
    within the Kulla-Conty table's own overshoot of one.  The rough diffuse
    model (Material.h:25-33) gains energy by its (1 + roughness / 2) factor and
    the dielectric BTDF carries the eta^2 radiance scaling (Material.h:202), so
    those two are compared with the oracle only."""
    rng = np.random.default_rng(100 + mtype)
    m = rt.material(mtype, albedo=(1.0, 1.0, 1.0), roughness=0.0 if mtype == rt.MAT_DIFFUSE else 0.3, specular=(1.0, 1.0, 1.0), metallic=1.0,
                    eta=(0.2, 0.2, 0.2), k=(4.0, 4.0, 4.0), coat_weight=1.0, coat_roughness_u=0.3,
                    coat_roughness_v=0.3)
    n = 20000
    N = np.tile([0.0, 0.0, 1.0], (n, 1))
    for cos_v in (0.9, 0.5, 0.2):
        V = np.tile([np.sqrt(1 - cos_v ** 2), 0.0, cos_v], (n, 1))
        x = np.zeros((n, 16), np.float32)
        x[:, 0:3], x[:, 3:6], x[:, 6:12], x[:, 12], x[:, 13] = N, V, rng.random((n, 6)), 1.0, 0
        g = rt.verify_shading(rt.VERIFY_BSDF_SAMPLE, x, [m])
        o = pyoracle.shading(rt.VERIFY_BSDF_SAMPLE, x, [m], precision=64)

        def est(y):
            f, pdf, L = y[:, 0].astype(np.float64), y[:, 3].astype(np.float64), y[:, 4:7].astype(np.float64)
            w = np.where(pdf > 0, f * np.abs(L[:, 2]) / np.where(pdf > 0, pdf, 1), 0.0)
            w = np.nan_to_num(w, nan=0.0, posinf=0.0)
            return w.mean(), w.std() / np.sqrt(n)

        eg, sg = est(g)
        eo, so = est(o)
        print(f"type {mtype} cos {cos_v}: gpu {eg:.4f}+-{sg:.4f} fp64 {eo:.4f}")
        assert abs(eg - eo) <= 3 * max(sg, 1e-6) + 1e-4
        if mtype in (rt.MAT_DIFFUSE, rt.MAT_DIFFUSE_TRANSMITTER):
            assert abs(eg - 1.0) < 1e-4  # cosine-sampled Lambert integrates to exactly one
        elif mtype != rt.MAT_DIELECTRIC:
            assert eg <= 1.1 + 3 * sg


@pytest.mark.gpu
def test_kulla_conty_table_on_device_matches_reference():
    lut, avg = rt.kulla_conty_lut()
    assert np.array_equal(lut, GOLD["kc_lut"])
    assert np.array_equal(avg, GOLD["kc_avg"])
