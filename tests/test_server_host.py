"""Host side of the render server: C layouts of its structures and clean
errors where no device is present."""
import ctypes as C
import subprocess

import pytest

import optixrender_b200 as rt
from conftest import ROOT

PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "rt_capi.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(rt_server_options), sizeof(rt_job_desc), sizeof(rt_job_status),
           sizeof(rt_server_stats), offsetof(rt_job_desc, seed), offsetof(rt_job_desc, width),
           sizeof(rt_render_stats), sizeof(rt_guide_options));
    return 0;
}
"""


def test_server_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(rt.ServerOptions), C.sizeof(rt.JobDesc), C.sizeof(rt.JobStatus), C.sizeof(rt.ServerStats),
            rt.JobDesc.seed.offset, rt.JobDesc.width.offset, C.sizeof(rt.RenderStats), C.sizeof(rt.GuideOptions)]
    assert got == want


def test_server_defaults():
    o = rt.server_options()
    assert (o.wave_paths, o.max_jobs, o.max_depth, o.background, o.waves_in_flight) == (1 << 23, 256, 32, 1, 2)
    assert (o.guide_train_waves, o.guide_steps, o.guide_prob) == (32, 4, 0.5)
    j = rt.job(0, rt.camera((0, 0, 1), (0, 0, 0)), 8, 8, 1)
    assert (j.max_depth, j.rr_depth, j.filter, j.seed) == (25, 0, rt.FILTER_GAUSSIAN, 1)


def test_server_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(rt.RTError) as e:
        rt.Server(rt.server_options(background=0))
    assert e.value.code == rt.RT_ERR_CUDA
    lib = rt.load_library()
    assert lib.rt_server_submit(None, None, None) == rt.RT_ERR_INVALID_ARG
    assert lib.rt_server_destroy(None) == rt.RT_OK
