"""Throughput and image error of one configuration, side by side.

Mpaths/s of the plain tracer on a configuration (device time of `--steps`
Render() calls with CUDA events on the renderer's stream, after `--warmup`),
and the relMSE of the rendered frame against a plain render of `--ref-spp`
samples per pixel with independent seeds, accumulated in FP64 on the host
(relMSE = mean over pixels and channels of (I - I_ref)^2 / (I_ref^2 + 1e-2)).

    python -m optixrender_b200.config_bench --config c0     # Cornell 256^2, 16 spp, depth 8
    python -m optixrender_b200.config_bench --config c2     # media 1280x720, 256 spp, depth 32, 128^3 grid
    python -m optixrender_b200.config_bench --config c1     # spheres 1920x1080, 64 spp, depth 16
"""
import argparse
import json

import numpy as np

from optixrender_b200 import scenes
from optixrender_b200.guide_bench import reference, relmse

CONFIGS = {
    "c0": lambda: scenes.cornell(256, 256, 16, seed=1),
    "c1": lambda: scenes.spheres(1920, 1080, 64, seed=1),
    "c2": lambda: scenes.media(1280, 720, 256, seed=1),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c0", choices=sorted(CONFIGS))
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--ref-spp", type=int, default=65536)
    a = ap.parse_args(argv)
    import torch
    spec = CONFIGS[a.config]()
    st = spec.settings
    s, r = scenes.build_renderer(spec)
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)
    for _ in range(a.warmup):
        r.render()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        r.render()
    e1.record(stream)
    torch.cuda.synchronize()
    r.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    paths = st["width"] * st["height"] * st["spp"]
    frame = r.download_linear()
    r.close()
    s.close()
    ref, ref_spp, ref_ms = reference(spec, a.ref_spp, frame_spp=min(256, st["spp"] * 16))
    line = {"config": a.config, "scene": spec.name, "width": st["width"], "height": st["height"], "spp": st["spp"],
            "max_depth": st["max_depth"], "ms_per_frame": ms, "Mpaths_s": paths / ms / 1e3,
            "relmse": relmse(frame, ref), "reference_spp": ref_spp, "reference_device_ms": ref_ms,
            "reference": "plain render, independent seeds, FP64-accumulated", "data": "synthetic"}
    print(json.dumps(line))
    return line


if __name__ == "__main__":
    main()
