"""rt_renderer_trace_noalloc: the ray queries of rt_renderer_trace (host
buffers) staged in the library's fixed device array instead of buffers
allocated per call.  It serves callers that cannot allocate device memory
during a query: a render or serving loop whose other streams must not be
stalled by the device-wide synchronisation of cudaMalloc/cudaFree, and a
process whose own memory pool already holds the rest of the GPU's memory.

Tolerance: the same traversal code runs on the same wide BVH, so primitive ids
must be identical and t, u, v equal within 1e-6 relative (they are expected to
be bit-identical).  Named to be collected last, so that it also runs after
every other GPU test in one process.
"""
import ctypes as C

import numpy as np
import pytest

import optixrender_b200 as rt
from optixrender_b200 import scenes

SCRATCH_RAYS = 65536


def _noalloc():
    lib = rt.load_library()
    f = lib.rt_renderer_trace_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p]
    return lib, f


def _rays(n, seed):
    """Rays from points around the scene towards points near its centre."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-2.5, 2.5, (n, 3))
    d = rng.uniform(-0.8, 0.8, (n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 3], r[:, 4:7], r[:, 7] = o, 1e-4, d, 3.0e38
    return r


def _same(got, want):
    assert np.array_equal(got[:, 3].view(np.int32), want[:, 3].view(np.int32))
    hit = want[:, 3].view(np.int32) >= 0
    np.testing.assert_allclose(got[hit, :3], want[hit, :3], rtol=1e-6, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("any_hit", [0, 1])
def test_noalloc_trace_matches_trace_on_two_calls_in_a_row(any_hit):
    spec = scenes.spheres(64, 64, 1, ico_level=5, env_size=(64, 32))
    s, r = scenes.build_renderer(spec)
    lib, f = _noalloc()
    for n in (SCRATCH_RAYS, 1000):
        rays = _rays(n, 7 * n + any_hit)
        want = r.trace(rays, any_hit=bool(any_hit))
        assert (want[:, 3].view(np.int32) >= 0).mean() > 0.2  # the batch hits the scene
        for _ in range(2):
            got = np.full((n, 4), np.nan, np.float32)
            assert f(r.handle, any_hit, rays.ctypes.data, n, got.ctypes.data) == rt.RT_OK
            _same(got, want)


@pytest.mark.gpu
def test_noalloc_trace_rejects_batches_beyond_the_scratch():
    spec = scenes.cornell(8, 8, 1)
    s, r = scenes.build_renderer(spec)
    lib, f = _noalloc()
    n = SCRATCH_RAYS + 1
    rays = _rays(n, 3)
    out = np.zeros((n, 4), np.float32)
    assert f(r.handle, 0, rays.ctypes.data, n, out.ctypes.data) == rt.RT_ERR_INVALID_ARG
    assert str(SCRATCH_RAYS) in lib.rt_last_error_message().decode()
    assert f(r.handle, 0, rays.ctypes.data, 0, out.ctypes.data) == rt.RT_OK
    assert f(r.handle, 0, None, 5, out.ctypes.data) == rt.RT_ERR_INVALID_ARG
