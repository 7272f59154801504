"""Generates the golden vectors that pin the oracle to the reference renderer.

Runs the reference's own shading code, compiled for the host from the
reference sources by oracle/Makefile into oracle/_ref/, on seeded inputs and
writes tests/golden/reference_shading.npz.  The reference itself has no tests
or fixtures; these vectors are its outputs on:
  * ComputeKullaConty (core/cuda/Microfacet.h:231-291)
  * HdrTexture::CalculateHdrCache (core/src/Scene.cpp:217-313) on a seeded image
  * gdt::LCG<16> (common/gdt/gdt/random/random.h:54-87) sequences
  * EvaluateMaterial / SampleMaterial for all eight material types
  * SampleLight / EvaluateLight, SamplePhase / EvaluatePhase, SampleMediumDistance
  * FilterJitter and SphereToPlane / PlaneToSphere

Sampling routines read their random numbers from a list; g++ evaluates the two
arguments of `vec2f(random(), random())` right to left, so each such pair is
stored swapped and the recorded `u` column is the left-to-right order.

Usage: python tests/golden/make_golden.py   (needs `make -C oracle` with the
reference tree present)
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import optixrender_b200 as rt  # noqa: E402
import pyoracle  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_shading.npz"

# positions of `vec2f(random(), random())` pairs in the left-to-right stream
PAIRS_BSDF = {
    rt.MAT_DIFFUSE: [(0, 1)], rt.MAT_CONDUCTOR: [(0, 1)], rt.MAT_DIELECTRIC: [(0, 1)], rt.MAT_PLASTIC: [(1, 2)],
    rt.MAT_METAL_WORKFLOW: [(1, 2)], rt.MAT_THIN_DIELECTRIC: [(0, 1)], rt.MAT_CLEARCOATED_CONDUCTOR: [(1, 2)],
    rt.MAT_DIFFUSE_TRANSMITTER: [(0, 1)],
}


def materials():
    ms = []
    for t in range(8):
        for rough, aniso in ((0.2, 0.0), (0.55, 0.0), (0.35, 0.4)):
            ms.append(rt.material(t, albedo=(0.8, 0.6, 0.4), roughness=rough, anisotropy=aniso,
                                  specular=(0.9, 0.9, 0.9), metallic=0.6, coat_roughness_u=0.2,
                                  coat_roughness_v=0.3 if aniso else 0.2, coat_weight=0.8))
    return ms


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def bsdf_queries(rng, n, nmat):
    N = unit(rng, n)
    V = unit(rng, n)
    flip = np.sum(N * V, 1) < 0
    V[flip] *= -1  # mostly outside
    V[rng.random(n) < 0.15] *= -1  # some from below
    L = unit(rng, n)
    u = rng.random((n, 6)).astype(np.float32)
    front = (rng.random(n) < 0.7).astype(np.float32)
    mi = rng.integers(0, nmat, n).astype(np.float32)
    ev = np.zeros((n, 16), np.float32)
    ev[:, 0:3], ev[:, 3:6], ev[:, 6:9], ev[:, 9], ev[:, 10] = N, V, L, front, mi
    sm = np.zeros((n, 16), np.float32)
    sm[:, 0:3], sm[:, 3:6], sm[:, 6:12], sm[:, 12], sm[:, 13] = N, V, u, front, mi
    return ev, sm


def swap_pairs(x, col0, pairs_of_row):
    y = x.copy()
    for i in range(x.shape[0]):
        for a, b in pairs_of_row(i):
            y[i, col0 + a], y[i, col0 + b] = x[i, col0 + b], x[i, col0 + a]
    return y


def main():
    libs = pyoracle.ref_libs()
    if libs is None:
        raise SystemExit("oracle/_ref not built: run `make -C oracle` with the reference tree present")
    shading, scene, rngl = libs
    F = C.POINTER(C.c_float)
    reversed_pairs = bool(shading.ref_pair_order_reversed())
    out = {"pair_order_reversed": np.array(reversed_pairs)}
    rng = np.random.default_rng(20240611)

    lut = np.zeros(4096, np.float32)
    avg = np.zeros(64, np.float32)
    shading.ref_kulla_conty(lut.ctypes.data_as(F), avg.ctypes.data_as(F))
    out["kc_lut"], out["kc_avg"] = lut.reshape(64, 64), avg

    env = np.concatenate([rng.gamma(2.0, 1.0, (32, 64, 3)), np.ones((32, 64, 1))], -1).astype(np.float32)
    env[10, 20, :3] = 300.0
    cache = np.zeros_like(env)
    scene.ref_env_cache(env.ctypes.data_as(F), 64, 32, cache.ctypes.data_as(F))
    out["env_in"], out["env_cache"] = env, cache

    seeds = np.array([[0, 0], [1, 0], [12345, 7], [65535, 3], [4000000, 99]], np.uint32)
    seq = np.zeros((len(seeds), 16), np.float32)
    for i, (a, b) in enumerate(seeds):
        rngl.ref_lcg(C.c_uint32(int(a)), C.c_uint32(int(b)), 16, seq[i].ctypes.data_as(F))
    out["lcg_seeds"], out["lcg_seq"] = seeds, seq

    mats = materials()
    M = (rt.Material * len(mats))(*mats)
    out["materials"] = np.frombuffer(bytes(M), np.uint8)
    lights = [rt.light(rt.LIGHT_QUAD, position=(-1, 2, -1), u=(2, 0, 0), v=(0, 0, 2), radiance=(5, 4, 3)),
              rt.light(rt.LIGHT_QUAD, position=(-1, -2, -1), u=(0, 0, 2), v=(2, 0, 0), radiance=(1, 2, 3),
                       double_side=1),
              rt.light(rt.LIGHT_SPHERE, position=(0.5, 1.5, 0.2), radius=0.4, radiance=(7, 7, 7))]
    Ls = (rt.Light * len(lights))(*lights)
    out["lights"] = np.frombuffer(bytes(Ls), np.uint8)
    media = [rt.medium(rt.MEDIUM_HOMOGENEOUS, sigma_s=(0.7, 0.9, 1.0), sigma_a=(0.03, 0.2, 0.5), scale=2.0),
             rt.medium(rt.MEDIUM_HOMOGENEOUS, phase=rt.PHASE_HG, g=(0.6, 0.3, -0.2), sigma_s=(0.5, 0.5, 0.5),
                       sigma_a=(0.1, 0.1, 0.1), scale=1.0),
             rt.medium(rt.MEDIUM_HOMOGENEOUS, phase=rt.PHASE_HG, g=(0.0, 0.0, 0.0), sigma_s=(1.0, 0.0, 0.2),
                       sigma_a=(0.0, 0.3, 0.2), scale=3.0)]
    Ds = (rt.Medium * len(media))(*media)
    out["media"] = np.frombuffer(bytes(Ds), np.uint8)

    def run(op, x):
        y = np.zeros((x.shape[0], 8), np.float32)
        shading.ref_shading(op, C.cast(M, C.c_void_p), len(mats), C.cast(Ls, C.c_void_p), len(lights),
                            C.cast(Ds, C.c_void_p), len(media), np.ascontiguousarray(x).ctypes.data_as(F),
                            x.shape[0], y.ctypes.data_as(F))
        return y

    ev, sm = bsdf_queries(rng, 4000, len(mats))
    out["bsdf_eval_in"], out["bsdf_eval_out"] = ev, run(rt.VERIFY_BSDF_EVAL, ev)
    mtype = [mats[int(i)].type for i in sm[:, 13]]
    ref_in = swap_pairs(sm, 6, lambda i: PAIRS_BSDF[mtype[i]]) if reversed_pairs else sm
    out["bsdf_sample_in"], out["bsdf_sample_out"] = sm, run(rt.VERIFY_BSDF_SAMPLE, ref_in)

    n = 1500
    ls = np.zeros((n, 16), np.float32)
    ls[:, 0:3] = rng.uniform(-1.5, 1.5, (n, 3))
    ls[:, 3:5] = rng.random((n, 2))
    ls[:, 5] = rng.integers(0, len(lights), n)
    out["light_sample_in"], out["light_sample_out"] = ls, run(rt.VERIFY_LIGHT_SAMPLE, ls)
    le = np.zeros((n, 16), np.float32)
    le[:, 0:3] = rng.uniform(-1.0, 1.0, (n, 3))
    le[:, 3:6] = unit(rng, n)
    le[:, 6] = np.where(rng.random(n) < 0.8, 3.0e38, rng.uniform(0.1, 3.0, n))
    le[:, 7] = rng.integers(0, len(lights), n)
    out["light_eval_in"], out["light_eval_out"] = le, run(rt.VERIFY_LIGHT_EVAL, le)

    ms_ = np.zeros((n, 16), np.float32)
    ms_[:, 0] = np.where(rng.random(n) < 0.2, 3.0e38, rng.uniform(0.01, 5.0, n))
    ms_[:, 1:3] = rng.random((n, 2))
    ms_[:, 3] = rng.integers(0, len(media), n)
    out["medium_sample_in"], out["medium_sample_out"] = ms_, run(rt.VERIFY_MEDIUM_SAMPLE, ms_)
    ps = np.zeros((n, 16), np.float32)
    ps[:, 0:3] = unit(rng, n)
    ps[:, 3:7] = rng.random((n, 4))
    ps[:, 7] = rng.integers(0, len(media), n)
    iso = np.array([media[int(i)].phase == rt.PHASE_ISOTROPIC for i in ps[:, 7]])
    ref_ps = swap_pairs(ps, 3, lambda i: [(0, 1)] if iso[i] else []) if reversed_pairs else ps
    out["phase_sample_in"], out["phase_sample_out"] = ps, run(rt.VERIFY_PHASE_SAMPLE, ref_ps)
    pe = np.zeros((n, 16), np.float32)
    pe[:, 0:3] = unit(rng, n)
    pe[:, 3:6] = unit(rng, n)
    pe[:, 6] = rng.integers(0, len(media), n)
    out["phase_eval_in"], out["phase_eval_out"] = pe, run(rt.VERIFY_PHASE_EVAL, pe)

    fj = rng.random((1000, 2)).astype(np.float32)
    out["filter_in"] = fj
    for t in range(4):
        y = np.zeros_like(fj)
        shading.ref_filter(t, fj.ctypes.data_as(F), fj.shape[0], y.ctypes.data_as(F))
        out[f"filter_out_{t}"] = y
    d = unit(rng, 1000).astype(np.float32)
    uv = np.zeros((1000, 2), np.float32)
    back = np.zeros((1000, 3), np.float32)
    shading.ref_sphere_plane(d.ctypes.data_as(F), 1000, uv.ctypes.data_as(F), back.ctypes.data_as(F))
    out["sphere_in"], out["sphere_uv"], out["sphere_back"] = d, uv, back

    np.savez_compressed(OUT, **out)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
