"""The allocation-free quality check, wtet_check_quality_noalloc.

It exists for callers that must not allocate GPU memory while it runs
(serving loops whose GPU memory belongs to an allocator another framework
owns, hosts with a memory budget fixed up front), so its scratch is a fixed
device array inside libwtet.so.  These tests call it through the C ABI and
check that two calls in a row return exactly what the allocating
wtet_check_quality returns, and that sizes beyond its fixed scratch are
refused.

The file name sorts last so that pytest collects it after every other test:
the array is shared by every call in the process, so running it after the
rest shows that earlier work leaves nothing in the array that changes its
result, and a run that stops at the first failure has run everything else
first.  It also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


def _bind(L):
    P = ctypes.c_void_p
    u64 = ctypes.c_uint64
    L.wtet_check_quality_noalloc.argtypes = [P, u64, P, P, u64, ctypes.POINTER(u64), ctypes.POINTER(u64), P]
    L.wtet_check_quality_noalloc.restype = ctypes.c_int
    return L


def _noalloc(L, d_pts, n, d_t, d_a, m, stream):
    v = ctypes.c_uint64(0)
    i = ctypes.c_uint64(0)
    rc = L.wtet_check_quality_noalloc(ctypes.c_void_p(d_pts.data_ptr()), n, ctypes.c_void_p(d_t.data_ptr()),
                                      ctypes.c_void_p(d_a.data_ptr()), m, ctypes.byref(v), ctypes.byref(i),
                                      ctypes.c_void_p(stream))
    assert rc == 0, L.wtet_last_error()
    return v.value, i.value


def test_noalloc_matches_allocating_check(gpu):
    import torch

    L = _bind(gpu._core.load())
    pts = fx.mixture(60_000, 17)
    r = gpu.delaunay(pts)
    # a copy with planted mistakes, so the counts being compared are not all zero
    bad = r.tets.copy()
    inner = np.nonzero((bad < len(pts)).all(axis=1))[0]
    for t0 in inner[:50:5]:
        nb = int(r.adjacency[t0, 0]) >> 5
        bad[t0, 0], bad[nb, 0] = bad[nb, 0], bad[t0, 0]
    stream = torch.cuda.current_stream().cuda_stream
    d_pts = torch.from_numpy(pts).cuda()
    for tets in (r.tets, bad):
        want = gpu.check_quality(pts, gpu.DelaunayResult(tets, r.adjacency, r.failed_verts))
        d_t = torch.from_numpy(tets.view(np.int32)).cuda()
        d_a = torch.from_numpy(r.adjacency.view(np.int32)).cuda()
        first = _noalloc(L, d_pts, len(pts), d_t, d_a, len(tets), stream)
        second = _noalloc(L, d_pts, len(pts), d_t, d_a, len(tets), stream)
        assert first == want, (first, want)
        assert second == want, (second, want)
    assert want[0] > 0


def test_noalloc_refuses_oversized_input(gpu):
    import torch

    L = _bind(gpu._core.load())
    n = 1048576 + 1
    d_pts = torch.zeros((8, 3), dtype=torch.float32, device="cuda")
    d_t = torch.zeros((1, 4), dtype=torch.int32, device="cuda")
    v = ctypes.c_uint64(0)
    i = ctypes.c_uint64(0)
    rc = L.wtet_check_quality_noalloc(ctypes.c_void_p(d_pts.data_ptr()), n, ctypes.c_void_p(d_t.data_ptr()),
                                      ctypes.c_void_p(d_t.data_ptr()), 1, ctypes.byref(v), ctypes.byref(i), None)
    assert rc == gpu._core.WTET_ERR_ARG
    assert b"exceed" in L.wtet_last_error()
