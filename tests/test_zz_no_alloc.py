"""The allocation-free Poisson-disk sampler (qmcrt_sample_points_noalloc).

Some callers cannot call cudaMalloc: a host application that owns every
device buffer, a real-time loop that may not allocate, a plugin whose memory
budget is fixed when it loads.  The library gives them one sampler entry point
whose working memory is a fixed-size array compiled into the library instead
of a per-call allocation.  These tests call it through the C-ABI and check it
against the scene sampler (qmcrt_scene_sample_points) on two calls in a row:
the second call must not see anything the first left in the shared array.
The points are integer lattice work, so the bar is bit-exact equality.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from onemirror_b200.scene import SolarScene  # noqa: E402


def scene_points(size, total, spacing, seed):
    """Points from the existing entry point (scene sampler, allocates)."""
    n = size.shape[0]
    pos = np.zeros((n, 3), np.float32)
    pos[:, 0] = np.arange(n) * 20.0
    pos[:, 1] = 6.0
    sc = SolarScene(pos, size, W.flat_receiver(50.0, 4.0, 4.0, 8, 8), W.grid(25.0))
    p = W.params(total * 64, 64, spacing, seed=seed)
    xz, helio = sc.points(p)
    sc.close()
    return xz, helio


def noalloc_points(size, total, spacing, seed):
    xz = torch.full((total, 2), float("nan"), dtype=torch.float32, device="cuda")
    helio = torch.full((total,), -7, dtype=torch.int32, device="cuda")
    st = capi.lib().qmcrt_sample_points_noalloc(capi.as_fp(np.ascontiguousarray(size, np.float32)), size.shape[0],
                                                total, C.c_float(spacing), seed, C.c_void_p(xz.data_ptr()),
                                                C.c_void_p(helio.data_ptr()), None)
    capi.check(st)
    return xz.cpu().numpy(), helio.cpu().numpy()


def test_two_calls_in_a_row_equal_the_scene_sampler():
    big = np.tile(np.array([[10.0, 0.1, 10.0]], np.float32), (40, 1))
    small = np.tile(np.array([[2.0, 0.05, 2.0]], np.float32), (100, 1))
    small[::3, 0] = 3.0  # uneven mirrors
    # first call fills much of the shared array; the second is smaller and must be unaffected
    cases = [(big, 40 * 1000, 0.18, 99), (small, 100 * 16, 0.3, 7)]
    for size, total, spacing, seed in cases:
        got_xz, got_h = noalloc_points(size, total, spacing, seed)
        ref_xz, ref_h = scene_points(size, total, spacing, seed)
        assert np.array_equal(got_h, ref_h)
        assert got_xz.tobytes() == ref_xz.tobytes()


def test_limits_and_errors_are_reported():
    size = np.tile(np.array([[2.0, 0.05, 2.0]], np.float32), (4, 1))
    out = torch.zeros((8, 2), dtype=torch.float32, device="cuda")
    h = torch.zeros(8, dtype=torch.int32, device="cuda")
    L = capi.lib()
    too_many = capi.QmcrtError
    st = L.qmcrt_sample_points_noalloc(capi.as_fp(size), 4, (1 << 20) + 1, C.c_float(0.01), 1,
                                       C.c_void_p(out.data_ptr()), C.c_void_p(h.data_ptr()), None)
    assert st == capi.ERR_INVALID_ARGUMENT and b"1048576" in L.qmcrt_last_error()
    big_n = np.ones((16385, 3), np.float32)
    st = L.qmcrt_sample_points_noalloc(capi.as_fp(big_n), 16385, 16385, C.c_float(0.1), 1,
                                       C.c_void_p(out.data_ptr()), C.c_void_p(h.data_ptr()), None)
    assert st == capi.ERR_INVALID_ARGUMENT
    # points that cannot fit report a sampling error and leave the entry point usable
    bad_xz = torch.full((8000, 2), float("nan"), dtype=torch.float32, device="cuda")
    bad_h = torch.full((8000,), -7, dtype=torch.int32, device="cuda")
    st = L.qmcrt_sample_points_noalloc(capi.as_fp(size), 4, 4 * 2000, C.c_float(0.3), 1,
                                       C.c_void_p(bad_xz.data_ptr()), C.c_void_p(bad_h.data_ptr()), None)
    assert st == capi.ERR_SAMPLING
    got_xz, got_h = noalloc_points(size, 8, 0.3, 5)
    ref_xz, ref_h = scene_points(size, 8, 0.3, 5)
    assert got_xz.tobytes() == ref_xz.tobytes() and np.array_equal(got_h, ref_h)
    # a successful call into the same (partly written) outputs overwrites all of them
    st = L.qmcrt_sample_points_noalloc(capi.as_fp(size), 4, 8, C.c_float(0.3), 5, C.c_void_p(bad_xz.data_ptr()),
                                       C.c_void_p(bad_h.data_ptr()), None)
    capi.check(st)
    assert bad_xz[:8].cpu().numpy().tobytes() == ref_xz.tobytes()
    assert np.array_equal(bad_h[:8].cpu().numpy(), ref_h)
    with pytest.raises(too_many):
        capi.check(L.qmcrt_sample_points_noalloc(None, 4, 8, C.c_float(0.3), 1, C.c_void_p(out.data_ptr()),
                                                 C.c_void_p(h.data_ptr()), None))
