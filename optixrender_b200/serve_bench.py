"""Serving benchmark: seeded render requests with Poisson arrivals through the
continuous-batching server, reporting time-to-image p50/p99 and aggregate
Mpaths/s.

Requests: resolution uniform from {256^2, 512^2, 1024^2, 1920x1080}, spp
uniform from {4, 16, 64, 256}, scene uniform from the Cornell box (34
triangles), the displaced icosphere with 64 spheres (2,590,720 triangles) and
the media scene (128^3 grid), a random camera orbiting the scene's own, guided
or plain drawn 50/50 (guided jobs sample their scene's guiding network, trained
on the scene's first guided waves).

First every request is submitted at once (saturation): aggregate Mpaths/s and
the saturation job rate.  Then the same requests arrive as a Poisson stream at
`load` x that rate, and time-to-image (submit -> final image in device memory,
as the server's host clock observes it) is reported as p50/p99, both raw and
as slowdown = time-to-image / (job paths / saturation Mpaths/s), and per
quartile of job size.

    python -m optixrender_b200.serve_bench --requests 1000 --load 0.8
    python -m optixrender_b200.serve_bench --requests 1000 --loads 0.25,0.5,0.8,1.0   # latency against load
    python -m optixrender_b200.serve_bench --mix plain-spheres --loads ""            # saturation only

`--mix plain-spheres` draws every request from the 1080p spheres scene without
guiding, the mix whose saturation throughput compares with a single
Renderer's on the benchmark frame.
"""
import argparse
import json
import math
import threading
import time

import numpy as np

import optixrender_b200 as rt
from optixrender_b200 import scenes

RESOLUTIONS = [(256, 256), (512, 512), (1024, 1024), (1920, 1080)]
SPPS = [4, 16, 64, 256]


def build_scenes(small=False):
    """The three scene families; `small` shrinks geometry and grids for tests."""
    if small:
        specs = [scenes.cornell(64, 64, 4), scenes.spheres(64, 64, 4, ico_level=4, env_size=(256, 128)),
                 scenes.media(64, 64, 4, grid_res=16, env_size=(256, 128))]
    else:
        specs = [scenes.cornell(), scenes.spheres(), scenes.media()]
    return specs, [scenes.build_scene(s) for s in specs]


def orbit_camera(cam, rng):
    """The spec camera turned about its target by +-30 deg yaw, +-10 deg pitch, distance x U[0.8, 1.2]."""
    f, a = np.array(cam["from_"], np.float64), np.array(cam["at"], np.float64)
    d = f - a
    r = np.linalg.norm(d)
    yaw = math.atan2(d[0], d[2]) + rng.uniform(-math.pi / 6, math.pi / 6)
    pitch = math.asin(np.clip(d[1] / r, -0.99, 0.99)) + rng.uniform(-math.pi / 18, math.pi / 18)
    r *= rng.uniform(0.8, 1.2)
    nf = a + r * np.array([math.cos(pitch) * math.sin(yaw), math.sin(pitch), math.cos(pitch) * math.cos(yaw)])
    out = dict(cam)
    out["from_"] = tuple(float(x) for x in nf)
    return out


def make_requests(n, specs, seed=1, resolutions=RESOLUTIONS, spps=SPPS, scene_choices=None, guided=None):
    rng = np.random.default_rng(seed)
    reqs = []
    choices = list(range(len(specs))) if scene_choices is None else list(scene_choices)
    for i in range(n):
        si = choices[int(rng.integers(len(choices)))]
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        spp = spps[int(rng.integers(len(spps)))]
        spec = specs[si]
        reqs.append(dict(scene=si, width=w, height=h, spp=spp, max_depth=spec.settings["max_depth"],
                         rr_depth=spec.settings["rr_depth"], camera=orbit_camera(spec.camera, rng),
                         guided=bool(rng.integers(2)) if guided is None else bool(guided),
                         seed=int(rng.integers(1 << 62))))
    return reqs


def _desc(req, scene_ids):
    return rt.job(scene_ids[req["scene"]], rt.camera(**req["camera"]), req["width"], req["height"], req["spp"],
                  max_depth=req["max_depth"], rr_depth=req["rr_depth"], filter=rt.FILTER_BOX,
                  tonemap=rt.TONEMAP_ACES_SRGB, seed=req["seed"], guided=int(req["guided"]))


def run_stream(srv, reqs, scene_ids, arrivals_s):
    """Submits reqs[i] at arrivals_s[i] (seconds from now); returns per-job status dicts."""
    submitted = [None] * len(reqs)
    done = {}
    lock = threading.Lock()
    t0 = time.perf_counter()

    def submitter():
        for i, req in enumerate(reqs):
            delay = t0 + arrivals_s[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            jid = srv.submit(_desc(req, scene_ids))
            with lock:
                submitted[i] = jid

    th = threading.Thread(target=submitter)
    th.start()
    outstanding = set()
    while len(done) < len(reqs):
        with lock:
            for i, jid in enumerate(submitted):
                if jid is not None and i not in done:
                    outstanding.add(i)
        for i in list(outstanding):
            st = srv.poll(submitted[i])
            if st["state"] in (rt.JOB_DONE, rt.JOB_FAILED, rt.JOB_CANCELLED):
                if st["state"] != rt.JOB_DONE:
                    raise RuntimeError(f"job {i} ended in state {st['state']}")
                done[i] = st
                outstanding.discard(i)
                srv.release(submitted[i])
        time.sleep(0.0005)
    th.join()
    return [done[i] for i in range(len(reqs))]


def summarize(sts, reqs, sat_mpaths=None):
    lat = np.array([s["done_ms"] - s["submit_ms"] for s in sts])
    paths = np.array([r["width"] * r["height"] * r["spp"] for r in reqs], np.float64)
    span_ms = max(s["done_ms"] for s in sts) - min(s["submit_ms"] for s in sts)
    out = {"requests": len(reqs), "paths": int(paths.sum()), "makespan_s": span_ms / 1e3,
           "aggregate_Mpaths_s": paths.sum() / (span_ms * 1e3),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean())}
    out["p99_over_p50"] = out["p99_ms"] / out["p50_ms"]
    if sat_mpaths:
        service_ms = paths / (sat_mpaths * 1e3)
        slow = lat / service_ms
        out.update(slowdown_p50=float(np.percentile(slow, 50)), slowdown_p99=float(np.percentile(slow, 99)))
        out["slowdown_p99_over_p50"] = out["slowdown_p99"] / out["slowdown_p50"]
    # latency within classes of similar job size (quartiles of paths per job)
    edges = np.quantile(paths, [0.25, 0.5, 0.75])
    cls = np.searchsorted(edges, paths, side="right")
    out["by_size_quartile"] = [
        {"paths_max": int(paths[cls == k].max()), "jobs": int((cls == k).sum()),
         "p50_ms": float(np.percentile(lat[cls == k], 50)), "p99_ms": float(np.percentile(lat[cls == k], 99))}
        for k in range(4) if (cls == k).any()]
    return out


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--requests", type=int, default=1000)
    p.add_argument("--load", type=float, default=0.8)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--policy", default="fair", choices=["fair", "fifo", "srpt"])
    p.add_argument("--wave-paths", type=int, default=1 << 23)
    p.add_argument("--max-jobs", type=int, default=256)
    p.add_argument("--loads", default=None,
                   help="comma-separated loads (fractions of the saturation job rate) to sweep; overrides --load")
    p.add_argument("--mix", default="c4", choices=["c4", "plain-spheres"])
    p.add_argument("--small", action="store_true", help="small scenes and resolutions (tests)")
    a = p.parse_args(argv)
    specs, keep = build_scenes(a.small)
    res = [(32, 32), (64, 48), (96, 64), (128, 72)] if a.small else RESOLUTIONS
    spps = [1, 2, 4, 8] if a.small else SPPS
    if a.mix == "plain-spheres":
        reqs = make_requests(a.requests, specs, a.seed, res, spps, scene_choices=[1], guided=False)
    else:
        reqs = make_requests(a.requests, specs, a.seed, res, spps)
    loads = [a.load] if a.loads is None else [float(x) for x in a.loads.split(",") if x.strip()]
    srv = rt.Server(rt.server_options(wave_paths=a.wave_paths, max_jobs=a.max_jobs, max_depth=32,
                                      policy={"fair": rt.SERVE_FAIR, "fifo": rt.SERVE_FIFO,
                                              "srpt": rt.SERVE_SRPT}[a.policy]))
    ids = [srv.add_scene(s) for s in keep]
    warm = make_requests(4, specs, a.seed + 1, res[:1], spps[:1])
    run_stream(srv, warm, ids, [0.0] * len(warm))  # graphs captured, scenes touched
    def phase(arrivals, sat_mpaths=None):
        before = srv.stats()
        out = summarize(run_stream(srv, reqs, ids, arrivals), reqs, sat_mpaths)
        after = srv.stats()
        waves = after["waves"] - before["waves"]
        # device time of the phase's waves over its makespan: how busy the GPU was
        out["device_busy_fraction"] = (after["busy_ms"] - before["busy_ms"]) / (out["makespan_s"] * 1e3)
        out["waves"] = waves
        out["mean_paths_per_wave"] = (after["paths"] - before["paths"]) / max(1, waves)
        return out

    sat = phase([0.0] * len(reqs))
    curve = []
    for load in loads:
        rate = load * len(reqs) / sat["makespan_s"]
        gaps = np.random.default_rng(a.seed + 2).exponential(1.0 / rate, len(reqs))
        arrivals = np.cumsum(gaps) - gaps[0]
        pt = phase(arrivals, sat["aggregate_Mpaths_s"])
        pt["load"], pt["rate_jobs_s"] = load, rate
        curve.append(pt)
    stats = srv.stats()
    srv.close()
    line = {"metric": "serving time-to-image", "unit": "ms", "higher_is_better": False, "mix": a.mix,
            "policy": a.policy, "wave_paths": a.wave_paths, "saturation": sat, "curve": curve,
            "guided_requests": int(sum(r["guided"] for r in reqs)),
            "server": stats, "data": "synthetic", "small": a.small}
    for pt in curve:  # the headline point: the load closest to 0.8
        if abs(pt["load"] - 0.8) <= min(abs(q["load"] - 0.8) for q in curve):
            line.update(p50_ms=pt["p50_ms"], p99_ms=pt["p99_ms"], p99_over_p50=pt["p99_over_p50"],
                        slowdown_p50=pt["slowdown_p50"], slowdown_p99=pt["slowdown_p99"],
                        slowdown_p99_over_p50=pt["slowdown_p99_over_p50"],
                        aggregate_Mpaths_s=pt["aggregate_Mpaths_s"], load=pt["load"], rate_jobs_s=pt["rate_jobs_s"],
                        loaded=pt)
            break
    print(json.dumps(line))
    return line


if __name__ == "__main__":
    main()
