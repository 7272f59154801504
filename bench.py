#!/usr/bin/env python
"""Benchmark: Mpaths/s of the plain path tracer on the 1080p spheres scene.

Workload (one step = one Renderer::Render of the full frame): 1920x1080,
64 samples per pixel, max depth 16, a 1.31M-triangle fBm-displaced icosphere
plus 64 spheres of 20k triangles (2.59M triangles), conductor / dielectric /
plastic materials, a 2048x1024 sky with a 5e3 sun.  The scene, BVH and frame
buffers stay resident on the device; the scene and BVH (~0.3 GB) exceed the
126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders its own replica (a different seed); `value`
is all ranks' paths over the slowest rank's time ("replicas only": the path
has no exchange step).  `--impl reference` times the reference's CPU path
(the reference shading code compiled for the host, in an OpenMP per-pixel
loop; the restated oracle when that build is absent) on a bounded sample of
the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

WORKLOAD = dict(width=1920, height=1080, spp=64, max_depth=16)
NODE_BYTES, TRI_BYTES, RAY_BYTES = 80, 48, 52  # wide node, triangle record, ray in + hit out + queue entry
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_extend
# launch of this workload, recorded from an ncu capture (the summary and its
# command are in profiles/); this run does not measure it.  Keyed by the wave
# size the capture used: a figure for another wave size is not reported.
RECORDED_EXTEND_DRAM_BYTES = {67108864: 1354235264}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--spp", type=int, default=WORKLOAD["spp"])
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--wave-paths", type=int, default=0, help="path slots per wave (0 = the library's choice)")
    p.add_argument("--ref-spp", type=int, default=None,
                   help="samples per pixel of the FP64-accumulated plain reference the frame's relMSE is measured "
                        "against (0: no relMSE; default 65536 on one GPU, none on more, where every rank renders "
                        "the same workload and the reference would hold all GPUs for two minutes)")
    return p.parse_args()


def dist_init(n):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL
    on GPUs, gloo where there is none (the CPU tests of this plumbing)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return rank, world, local


def reduce_max(x: float, world: int) -> float:
    """The maximum of x over all ranks (the slowest rank's time)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mpaths(paths_per_rank: int, world: int, ms: float) -> float:
    """Whole-job Mpaths/s: every rank's paths over the slowest rank's time."""
    return paths_per_rank * world / (ms / 1e3) / 1e6


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    every 10 ms from a thread (reads only), nvidia-smi when NVML is absent."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x for x in vis.split(",") if x.strip()]
        self.gpu = int(ids[gpu]) if gpu < len(ids) and ids[gpu].strip().isdigit() else gpu
        self.proc = None
        self.lines = []
        self.sm, self.mask, self.max_mhz = [], 0, None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.reason_fn = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                getattr(pynvml, "nvmlDeviceGetCurrentClocksThrottleReasons")
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _poll(self):
        while not self.stop.is_set():
            try:
                self.sm.append(float(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM)))
                self.mask |= int(self.reason_fn(self.h))
            except Exception:
                pass
            self.stop.wait(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.t.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.nvml is not None:
            reasons = sorted(k for k, bit in self.REASONS.items() if self.mask & bit)
            return {"sm_mhz": float(np.median(self.sm)) if self.sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.sm), "source": "nvml"}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class CpuRunner:
    """The CPU implementation of the path: the reference's shading code built
    for the host (oracle/_ref/libref_pt.so) when present, else the oracle port."""

    def __init__(self, spec):
        import pyoracle
        self.spec = spec
        self.kind = "port"
        self.impl = None
        if (ROOT / "oracle" / "_ref" / "libref_pt.so").exists():
            try:
                import refpt
                self.impl = refpt.RefScene(spec)
                self.kind = "reference"
            except Exception:
                self.impl = None
        if self.impl is None:
            self.impl = pyoracle.OracleScene(spec)

    def sample(self, spp, seconds, threads=0):
        """Times a band of rows (then more samples) sized to about `seconds`."""
        from optixrender_b200 import camera  # a plain ctypes struct: no library is loaded
        from pyoracle import options
        spec = self.spec
        cam = camera(**spec.camera)
        H, W = spec.settings["height"], spec.settings["width"]
        rows, spp_s = 8, 1
        while True:
            o = options(**dict(spec.settings, spp=spp_s))
            band = (max(0, H // 2 - rows // 2), min(H, H // 2 - rows // 2 + rows))
            t = time.perf_counter()
            if self.kind == "reference":
                self.impl.render(o, cam, rows=band, threads=threads)
            else:
                self.impl.render(o, cam, rows=band, threads=threads, want_aov=False)
            dt = time.perf_counter() - t
            if dt * 2 >= seconds or (rows >= H and spp_s >= spp):
                break
            grow = max(2.0, seconds / max(dt, 1e-3) * 0.6)
            if rows < H:
                rows = min(H, int(rows * grow))
            else:
                spp_s = min(spp, int(spp_s * grow))
        paths = rows * W * spp_s
        nthreads = threads or os.cpu_count()
        return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": nthreads, "kind": self.kind,
                "sample": f"{rows} centre rows x {W} px x {spp_s} spp of the {W}x{H} frame ({paths} paths, "
                          f"{dt:.1f} s); the full step is {spp} spp"}


def bench_config(spp, triangles, world):
    """The workload as both arms report it."""
    return {"workload": "spheres-1080p", **dict(WORKLOAD, spp=spp), "triangles": triangles,
            "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (scene + BVH ~0.3 GB)"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path on the host cores.  It loads
    the reference's host build (or the oracle), never the product library."""
    from optixrender_b200 import scenes
    if rank != 0:
        return 0
    spec = scenes.spheres(spp=args.spp)
    runner = CpuRunner(spec)
    vals = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = runner.sample(args.spp, args.cpu_seconds / 3)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(np.median(vals))
    cb["value"] = v
    line = {"impl": "reference", "metric": "Mpaths/s", "value": v, "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args.spp, spec.num_triangles, world),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank, world, local = dist_init(args.gpus)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    import torch
    import optixrender_b200 as rt
    from optixrender_b200 import scenes
    torch.cuda.set_device(local)
    spec = scenes.spheres(spp=args.spp, seed=1 + rank)
    s, r = scenes.build_renderer(spec, collect_stats=0, wave_paths=args.wave_paths)
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)
    W, H = spec.settings["width"], spec.settings["height"]
    paths_per_step = W * H * args.spp
    for _ in range(args.warmup):
        r.render()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # timed region A: the production path (one captured graph per wave)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            r.render()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    st0 = r.stats()
    launches_per_step, wave_paths = st0["launches"], st0["wave_paths"]
    ms = reduce_max(ms, world)
    ms_step = ms / args.steps
    value = job_mpaths(paths_per_step, world, ms_step)

    # timed region B: the same steps with a CUDA event pair around every kernel
    # and device counters of nodes / triangles / rays, for the roofline
    o = r.options
    o.collect_stats = 1
    r.set_options(o)
    kern = {"extend": 0.0, "shade": 0.0, "sample": 0.0, "shadow": 0.0, "other": 0.0}
    counters = {"extend_rays": 0, "extend_nodes": 0, "extend_tris": 0, "shadow_rays": 0, "nodes": 0, "tris": 0,
                "extend_launches": 0, "nan": 0, "nan_history": 0, "ms": 0.0}
    r.render()  # warm the per-kernel path once
    torch.cuda.synchronize()
    for _ in range(args.steps):
        r.render()
        st = r.stats()
        for k in kern:
            kern[k] += st["ms_" + k]
        counters["ms"] += st["ms_total"]
        counters["extend_rays"] += st["extend_rays"]
        counters["extend_nodes"] += st["extend_nodes"]
        counters["extend_tris"] += st["extend_tris"]
        counters["shadow_rays"] += st["shadow_rays"]
        counters["nodes"] += st["nodes_visited"]
        counters["tris"] += st["tris_tested"]
        counters["extend_launches"] += st["extend_launches"]
        counters["nan"] += st["nan_samples"]
        counters["nan_history"] += st["nan_throughput_paths"]
    o.collect_stats = 0
    r.set_options(o)

    # end to end through the C ABI: render + RGBA8 download to pinned host memory
    host = torch.empty((H, W), dtype=torch.int32, pin_memory=True)
    out = host.numpy().view(np.uint32)
    e2e_t = []
    for i in range(args.steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r.render()
        r.download_pixels(out)
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_t.append(dt)
    e2e_ms = float(np.median(e2e_t)) * 1e3  # host clock: a single stall of the shared host would swing a mean
    e2e_ms = reduce_max(e2e_ms, world)
    e2e_value = job_mpaths(paths_per_step, world, e2e_ms)
    h2d = int(r.stats()["h2d_bytes"])  # launch parameters + wave table uploaded by each Render()

    # image error of the benchmarked frame (after every timed region): relMSE
    # against a plain render of ref_spp samples per pixel with independent
    # seeds, accumulated in FP64; the reference's own noise adds about
    # spp / ref_spp of the value (0.1% at 64 / 65536)
    quality = None
    ref_spp_arg = args.ref_spp if args.ref_spp is not None else (65536 if world == 1 else 0)
    if ref_spp_arg > 0 and rank == 0:
        from optixrender_b200.guide_bench import reference, relmse
        frame = r.download_linear()
        ref_img, ref_spp, ref_ms = reference(spec, ref_spp_arg)
        quality = {"relmse": relmse(frame, ref_img), "reference_spp": ref_spp,
                   "reference": "plain render, frames of 256 spp with independent seeds accumulated in FP64",
                   "reference_device_ms": ref_ms}
        del ref_img
    peak, peak_kind = measured_peak()
    ext_bytes = (counters["extend_nodes"] * NODE_BYTES + counters["extend_tris"] * TRI_BYTES +
                 counters["extend_rays"] * RAY_BYTES)
    ext_ms = kern["extend"]
    achieved = ext_bytes / (ext_ms / 1e3) / 1e9 if ext_ms > 0 else 0.0
    traffic = RECORDED_EXTEND_DRAM_BYTES.get(wave_paths)
    line = {
        "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args.spp, spec.num_triangles, world),
        "wave_paths": wave_paths,
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": W * H * 4},
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"bound": "hbm", "kernel": "k_extend (closest-hit traversal)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak if peak else None,
                     "traffic": traffic, "peak_source": peak_kind,
                     "traffic_source": "recorded ncu capture of one k_extend launch of this workload (profiles/), "
                                       "not measured by this run" if traffic is not None else None,
                     "algorithmic_bytes_per_launch": ext_bytes / max(1, counters["extend_launches"]),
                     "ms_extend_per_launch": ext_ms / max(1, counters["extend_launches"])},
        "kernel_ms_per_step": {k: v / args.steps for k, v in kern.items()},
        "instrumented_ms_per_step": counters["ms"] / args.steps,
        "rays_per_step": {"extend": counters["extend_rays"] / args.steps,
                          "shadow": counters["shadow_rays"] / args.steps},
        "per_ray": {"extend_nodes": counters["extend_nodes"] / max(1, counters["extend_rays"]),
                    "extend_tris": counters["extend_tris"] / max(1, counters["extend_rays"]),
                    "shadow_nodes": (counters["nodes"] - counters["extend_nodes"]) / max(1, counters["shadow_rays"]),
                    "shadow_tris": (counters["tris"] - counters["extend_tris"]) / max(1, counters["shadow_rays"])},
        "nan_samples_per_step": counters["nan"] / args.steps,
        "paths_ended_by_nan_throughput_per_step": counters["nan_history"] / args.steps,
        "launches_per_step": launches_per_step,
        "clocks": clk.summary(),
        "image": quality,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = CpuRunner(spec).sample(args.spp, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    r.close()
    s.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
