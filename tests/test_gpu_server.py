"""The continuous-batching render server (rt_server_*).

Each job draws PCG32 streams keyed by (seed, path index) and sums every
pixel's samples in sample order, so a job's image must be bit-identical to a
Renderer::Render() with the same settings, whichever jobs shared its waves and
however its paths were split across waves.
"""
import time

import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes


def _specs():
    return [
        scenes.cornell(64, 48, 6, seed=7),
        scenes.spheres(80, 45, 3, seed=3, ico_level=5, env_size=(256, 128)),
        scenes.media(48, 40, 4, seed=5, grid_res=16, env_size=(256, 128)),
    ]


def _job_for(spec, scene_id, **over):
    st = dict(spec.settings)
    st.update(over)
    return rt.job(scene_id, rt.camera(**spec.camera), st["width"], st["height"], st["spp"],
                  max_depth=st["max_depth"], rr_depth=st["rr_depth"], filter=st.get("filter", rt.FILTER_BOX),
                  tonemap=st.get("tonemap", rt.TONEMAP_REINHARD), seed=st["seed"], guided=st.get("guided", 0))


def _alone(spec, **over):
    st = dict(spec.settings)
    st.update(over)
    st.setdefault("filter", rt.FILTER_BOX)
    s, r = scenes.build_renderer(spec, **st)
    r.render()
    return r.download_linear(), r.download_pixels()


@pytest.mark.gpu
@pytest.mark.parametrize("wave_paths,policy", [(4096, rt.SERVE_FAIR), (1 << 16, rt.SERVE_FAIR),
                                               (4096, rt.SERVE_FIFO), (4096, rt.SERVE_SRPT)])
def test_jobs_in_a_mix_match_renders_alone_bitwise(wave_paths, policy):
    specs = _specs()
    srv = rt.Server(rt.server_options(wave_paths=wave_paths, max_jobs=8, max_depth=32, policy=policy))
    keep = [scenes.build_scene(sp) for sp in specs]
    ids = [srv.add_scene(s) for s in keep]
    jobs = []
    for rep in range(2):  # each scene twice, second time with another seed
        for sp, sid in zip(specs, ids):
            jobs.append((sp, rep, srv.submit(_job_for(sp, sid, seed=sp.settings["seed"] + rep))))
    for sp, rep, jid in jobs:
        st = srv.wait(jid, 120000.0)
        assert st["state"] == rt.JOB_DONE
        assert st["done_ms"] >= st["admit_ms"] >= st["submit_ms"]
    stats = srv.stats()
    print(stats)
    assert stats["jobs_done"] == len(jobs)
    assert stats["paths"] == sum(sp.settings["width"] * sp.settings["height"] * sp.settings["spp"]
                                 for sp, _, _ in jobs)
    assert stats["max_segments_in_a_wave"] >= 2  # jobs really shared waves
    for sp, rep, jid in jobs:
        lin, px = _alone(sp, seed=sp.settings["seed"] + rep)
        got = srv.download(jid)
        assert np.array_equal(got.view(np.uint32), lin.view(np.uint32)), sp.name
        assert np.array_equal(srv.download_pixels(jid), px)
        srv.release(jid)
    srv.close()


@pytest.mark.gpu
def test_manual_mode_admits_within_the_memory_budget():
    """With room for one job's buffers, jobs run one at a time; a finished job
    holds its memory until it is released."""
    spec = scenes.cornell(100, 100, 2, seed=11)
    job_bytes = 100 * 100 * 104
    srv = rt.Server(rt.server_options(background=0, hbm_budget_bytes=int(1.5 * job_bytes),
                                      wave_paths=1 << 14, max_depth=8))
    scene = scenes.build_scene(spec)
    sid = srv.add_scene(scene)
    ids = [srv.submit(_job_for(spec, sid, seed=20 + i)) for i in range(4)]
    most_running = 0
    images = {}
    while srv.step():
        st = srv.stats()
        most_running = max(most_running, st["jobs_running"])
        assert st["bytes_in_use"] <= st["bytes_budget"]
        for i, jid in enumerate(ids):
            if i not in images and srv.poll(jid)["state"] == rt.JOB_DONE:
                images[i] = srv.download(jid)
                srv.release(jid)
    assert most_running == 1 and len(images) == 4
    for i in range(4):
        lin, _ = _alone(spec, seed=20 + i)
        assert np.array_equal(images[i].view(np.uint32), lin.view(np.uint32))
    srv.close()

    # an unreleased finished job blocks the next one: waiting on it reports why
    srv = rt.Server(rt.server_options(background=0, hbm_budget_bytes=int(1.5 * job_bytes),
                                      wave_paths=1 << 14, max_depth=8))
    sid = srv.add_scene(scene)
    a, b = srv.submit(_job_for(spec, sid)), srv.submit(_job_for(spec, sid))
    assert srv.wait(a)["state"] == rt.JOB_DONE
    with pytest.raises(rt.RTError) as e:
        srv.wait(b)
    assert e.value.code == rt.RT_ERR_STATE
    srv.release(a)
    assert srv.wait(b)["state"] == rt.JOB_DONE
    srv.close()


@pytest.mark.gpu
def test_submit_errors_cancel_and_timeout():
    spec = scenes.cornell(32, 32, 1)
    srv = rt.Server(rt.server_options(background=0, hbm_budget_bytes=8 << 20, max_depth=8))
    sid = srv.add_scene(scenes.build_scene(spec))
    with pytest.raises(rt.RTError) as e:
        srv.submit(_job_for(spec, sid, width=4096, height=4096))  # over the budget alone
    assert e.value.code == rt.RT_ERR_OUT_OF_MEMORY
    with pytest.raises(rt.RTError):
        srv.submit(_job_for(spec, sid, max_depth=9))  # deeper than the server's launches
    with pytest.raises(rt.RTError):
        srv.submit(_job_for(spec, sid + 1))
    a = srv.submit(_job_for(spec, sid))
    b = srv.submit(_job_for(spec, sid))
    srv.cancel(b)
    assert srv.poll(b)["state"] == rt.JOB_CANCELLED
    with pytest.raises(rt.RTError):
        srv.download(a)  # not run yet
    assert srv.wait(a)["state"] == rt.JOB_DONE
    srv.release(a)
    srv.release(b)
    srv.close()

    bg = rt.Server(rt.server_options(max_depth=8))
    sid = bg.add_scene(scenes.build_scene(scenes.cornell(32, 32, 1)))
    big = bg.submit(_job_for(spec, sid, width=512, height=512, spp=64))
    t = time.perf_counter()
    with pytest.raises(rt.RTError) as e:
        bg.wait(big, 0.0)
    assert e.value.code == rt.RT_ERR_TIMEOUT and time.perf_counter() - t < 1.0
    assert bg.wait(big, 120000.0)["state"] == rt.JOB_DONE
    bg.close()


@pytest.mark.gpu
@pytest.mark.parametrize("policy", ["fair", "srpt"])
def test_serve_bench_small(policy):
    """The serving benchmark end to end on small scenes: every request
    finishes, and the device-busy fraction from the server's wave events is a
    fraction of the phase's wall time."""
    from optixrender_b200 import serve_bench
    line = serve_bench.main(["--small", "--requests", "24", "--policy", policy, "--wave-paths", str(1 << 15),
                             "--loads", "0.5,0.8"])
    for ph in [line["saturation"]] + line["curve"]:
        assert ph["requests"] == 24
        assert 0.0 < ph["device_busy_fraction"] <= 1.05
    assert [pt["load"] for pt in line["curve"]] == [0.5, 0.8] and line["load"] == 0.8
    assert line["server"]["jobs_done"] == 24 * 3 + 4
    assert line["p99_ms"] >= line["p50_ms"] > 0.0


def _mean_diff_se(a, b):
    d = (a[..., :3].astype(np.float64) - b[..., :3]).mean(-1)
    return d.mean(), d.std() / np.sqrt(d.size)


@pytest.mark.gpu
@pytest.mark.parametrize("policy", [rt.SERVE_FAIR, rt.SERVE_SRPT])
def test_guided_jobs_share_the_scene_network(policy):
    """Guided jobs sample their scene's network: it trains on the scene's
    first guide_train_waves guided waves only, later guided jobs reuse it, each
    guided image agrees with a plain render within 3 standard errors, and a
    plain job served beside them is still bit-identical to its render alone."""
    spec = scenes.portal(48, 48, 256)
    srv = rt.Server(rt.server_options(wave_paths=1 << 14, max_depth=8, guide_train_waves=8, policy=policy))
    keep = scenes.build_scene(spec)
    sid = srv.add_scene(keep)
    plain = srv.submit(_job_for(spec, sid, seed=101))
    first = srv.submit(_job_for(spec, sid, seed=202, guided=1))
    for jid in (plain, first):
        assert srv.wait(jid, 120000.0)["state"] == rt.JOB_DONE
    st = srv.stats()
    assert st["training_waves"] == 8 and st["guided_waves"] > 8
    second = srv.submit(_job_for(spec, sid, seed=303, guided=1))
    assert srv.wait(second, 120000.0)["state"] == rt.JOB_DONE
    st2 = srv.stats()
    assert st2["training_waves"] == 8 and st2["guided_waves"] > st["guided_waves"]
    ref = srv.download(plain)
    lin, _ = _alone(spec, seed=101)
    assert np.array_equal(ref.view(np.uint32), lin.view(np.uint32))
    for jid in (first, second):
        img = srv.download(jid)
        assert np.isfinite(img).all()
        m, se = _mean_diff_se(img, ref)
        print(f"guided job {jid}: mean diff {m:.3e} se {se:.3e}")
        assert abs(m) <= 3 * se
        srv.release(jid)
    srv.release(plain)
    srv.close()


@pytest.mark.gpu
def test_background_worker_works_on_the_servers_device():
    """The background thread makes the server's device current before it
    records events, captures graphs or launches waves (a new thread starts on
    device 0); the stats report both.  Jobs submitted, awaited and downloaded
    from another host thread come out the same as from the creating thread."""
    import threading
    torch = pytest.importorskip("torch")
    spec = scenes.cornell(32, 32, 2, seed=9)
    srv = rt.Server(rt.server_options(wave_paths=4096, max_jobs=4, max_depth=8))
    keep = scenes.build_scene(spec)
    sid = srv.add_scene(keep)
    jid = srv.submit(_job_for(spec, sid))
    assert srv.wait(jid, 60000.0)["state"] == rt.JOB_DONE
    st = srv.stats()
    assert st["device"] == torch.cuda.current_device()
    assert st["worker_device"] == st["device"]
    out = {}

    def other_thread():
        j2 = srv.submit(_job_for(spec, sid))
        out["state"] = srv.wait(j2, 60000.0)["state"]
        out["img"] = srv.download(j2)
        srv.release(j2)

    t = threading.Thread(target=other_thread)
    t.start()
    t.join(120.0)
    assert out["state"] == rt.JOB_DONE
    assert np.array_equal(out["img"].view(np.uint32), srv.download(jid).view(np.uint32))
    srv.release(jid)
    srv.close()
