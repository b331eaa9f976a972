"""The allocation-free ray sort (ray_sort_rays_noalloc) against the
allocating one (ray_sort_rays), through the C ABI.

ray_sort_rays_noalloc is for callers that cannot call cudaMalloc: hosts whose
GPU memory belongs to their own allocator and budget, and frame loops that
must not stall on cudaMalloc's implicit device-wide synchronisation. Its
scratch is one static array shared by every call, so two calls in a row on
different inputs must each give exactly the allocating entry point's keys,
permutation and reordered rays (integer results: bit for bit). This file is
collected last so that, if it fails, a run that stops at the first failure
has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from raydemo_b200 import capi, scenes
from raydemo_b200.api import Renderer

pytestmark = pytest.mark.gpu


def _buffers(torch, n):
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    return keys, perm, out


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(cuda_device):
    import torch

    L = capi.lib()
    r = Renderer(16, 16)
    root_min = (C.c_float * 3)(0.0, 0.0, 0.0)
    cell = (C.c_float * 3)(1 / 255, 1 / 255, 1 / 255)
    # two calls in a row on different inputs; the second is smaller, so stale
    # scratch contents from the first call would show up as wrong results
    for n, seed in ((1 << 20, 71), (300001, 72)):
        rays = scenes.incoherent_rays(n, seed=seed)
        rays[:, 0:3] = rays[:, 0:3] * 3.0 - 1.0
        rd = torch.from_numpy(rays).cuda()
        ka, pa, oa = _buffers(torch, n)
        kb, pb, ob = _buffers(torch, n)
        capi.check(L.ray_sort_rays(r.handle, rd.data_ptr(), n, root_min, cell, ka.data_ptr(), pa.data_ptr(), oa.data_ptr(), None))
        torch.cuda.synchronize()
        capi.check(L.ray_sort_rays_noalloc(rd.data_ptr(), n, root_min, cell, kb.data_ptr(), pb.data_ptr(), ob.data_ptr(), None))
        torch.cuda.synchronize()
        assert np.array_equal(_host(kb), _host(ka))
        assert np.array_equal(_host(pb), _host(pa))
        assert np.array_equal(_host(ob), _host(oa))


def test_noalloc_sort_rejects_more_than_its_scratch_holds(cuda_device):
    import torch

    L = capi.lib()
    root_min = (C.c_float * 3)(0.0, 0.0, 0.0)
    cell = (C.c_float * 3)(1.0, 1.0, 1.0)
    n = (1 << 20) + 1
    rd = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = L.ray_sort_rays_noalloc(rd.data_ptr(), n, root_min, cell, None, perm.data_ptr(), None, None)
    assert rc == capi.RAY_ERR_INVALID_ARG
    assert b"RAY_SORT_NOALLOC_MAX_RAYS" in L.ray_last_error()


def test_noalloc_sort_allocates_nothing_on_a_side_stream(cuda_device):
    """A warmed call leaves the device's free memory unchanged (nothing is
    allocated), and a call on a caller's stream with keys_out and rays_out
    NULL gives the allocating sort's permutation."""
    import torch

    L = capi.lib()
    r = Renderer(16, 16)
    root_min = (C.c_float * 3)(0.0, 0.0, 0.0)
    cell = (C.c_float * 3)(1 / 255, 1 / 255, 1 / 255)
    n = 200003
    rays = scenes.incoherent_rays(n, seed=73)
    rd = torch.from_numpy(rays).cuda()
    ka, pa, oa = _buffers(torch, n)
    pb = torch.zeros(n, dtype=torch.int32, device="cuda")
    capi.check(L.ray_sort_rays(r.handle, rd.data_ptr(), n, root_min, cell, ka.data_ptr(), pa.data_ptr(), oa.data_ptr(), None))
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    capi.check(L.ray_sort_rays_noalloc(rd.data_ptr(), n, root_min, cell, None, pb.data_ptr(), None, s.cuda_stream))  # warm
    s.synchronize()
    pb.zero_()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    capi.check(L.ray_sort_rays_noalloc(rd.data_ptr(), n, root_min, cell, None, pb.data_ptr(), None, s.cuda_stream))
    s.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    assert np.array_equal(_host(pb), _host(pa))
