"""Failure detection through the C ABI, with every failure made on the host:
a corrupt BVH written into the scene's device arrays (the traversal's index
checks and step bounds end every ray and report it), device allocations that
fail on purpose (the calls return RAY_ERR_OUT_OF_MEMORY and free what they
made), host waits whose bound runs out (RAY_ERR_TIMEOUT, the GPU work itself
finishing normally), and destroyed or unknown handles. Nothing here faults,
traps or hangs the GPU: every access the kernels make stays in bounds."""
import ctypes as C

import numpy as np
import pytest

from raydemo_b200 import capi, scenes
from raydemo_b200.api import Renderer

pytestmark = pytest.mark.gpu


def _raw_scene(L, r):
    """An empty scene through the raw C ABI (no Python wrapper that would
    destroy it again)."""
    s = C.c_void_p()
    capi.check(L.ray_create_scene(r.handle, C.byref(s)))
    return s


def _scene(r, tris):
    sc = r.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(tris)
    m = sc.AddMaterial()
    sc.AddMeshInstance(sc.AddMesh(attrs, idx, [(m, 0, len(idx))]))
    return sc


@pytest.fixture(scope="module")
def renderer(cuda_device):
    return Renderer(16, 16)


def test_destroyed_and_unknown_handles_are_rejected(renderer):
    L = capi.lib()
    s = _raw_scene(L, renderer)
    capi.check(L.ray_scene_commit(s))
    capi.check(L.ray_destroy_scene(s))
    assert L.ray_scene_commit(s) == capi.RAY_ERR_INVALID_ARG
    assert b"destroyed" in L.ray_last_error()
    assert L.ray_destroy_scene(s) == capi.RAY_ERR_INVALID_ARG  # a second destroy
    bogus = C.c_void_p(0x1234560)
    assert L.ray_scene_commit(bogus) == capi.RAY_ERR_INVALID_ARG
    assert L.ray_render(bogus, bogus, None) == capi.RAY_ERR_INVALID_ARG
    info = capi.TraceInfo()
    assert L.ray_scene_last_trace_info(bogus, C.byref(info)) == capi.RAY_ERR_INVALID_ARG
    # the live renderer still works
    capi.check(L.ray_resize(renderer.handle, 16, 16))


def _corrupt_root(sc, child_base=None, cycle=False):
    """Rewrites the root wide node (20 words: origin xyz; per-axis quantum
    exponents with the internal-child mask in the top byte; child base,
    triangle base, leaf metadata; lo x/y/z and hi x/y/z quantised planes).
    Origin -1000 and quantum 2^3 (biased exponent 130) on every axis with lo
    planes 0 and hi planes 255: every child box spans [-1000, 1040]^3, so
    every ray enters all eight, all internal. cycle: child base 0, so slot s
    is node s, the root among them, and the walk pushes a group per step
    without end; else the given child base (outside the node array)."""
    node = np.zeros(20, np.uint32)
    node[0:3] = np.float32(-1000.0).view(np.uint32)
    node[3] = 130 | (130 << 8) | (130 << 16) | (0xFF << 24)
    node[4] = 0 if cycle else child_base
    node[14:20] = 0xFFFFFFFF
    sc.debug_write(0, 0, node.tobytes())


@pytest.mark.parametrize("kind", ["bounds", "cycle"])
def test_corrupt_bvh_is_reported(renderer, kind):
    tris = scenes.random_triangles(20000, seed=91, mean_edge=0.01)
    rays = scenes.incoherent_rays(5000, seed=92)
    sc = _scene(renderer, tris)
    good = sc.trace_closest(rays)
    assert sc.last_trace_info().error_flags == 0
    if kind == "bounds":
        _corrupt_root(sc, child_base=0xFFFFFF00)
        expect = capi.RAY_ERR_CUDA
    else:
        _corrupt_root(sc, cycle=True)
        expect = capi.RAY_ERR_STACK_OVERFLOW
    with pytest.raises(capi.RayError) as e:
        sc.trace_closest(rays)
    assert e.value.code == expect, e.value
    assert sc.last_trace_info().error_flags != 0
    assert (good["prim"] >= 0).any()


def test_device_allocation_failures_return_out_of_memory(renderer):
    """Fail the k-th device allocation of building and tracing a scene, for
    every k until the work needs no more: each failing call returns
    RAY_ERR_OUT_OF_MEMORY; destroying the scene gives the device memory
    back; the scene built without a failure traces as before."""
    import torch

    L = capi.lib()
    tris = scenes.random_triangles(30000, seed=93, mean_edge=0.01)
    rays = scenes.incoherent_rays(20000, seed=94)
    ref = _scene(renderer, tris).trace_closest(rays)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    try:
        for k in range(200):
            sc = _scene(renderer, tris)
            L.ray_debug_fail_device_alloc(k)
            try:
                hits = sc.trace_closest(rays)
            except capi.RayError as e:
                assert e.code == capi.RAY_ERR_OUT_OF_MEMORY, e
                failures += 1
                L.ray_debug_fail_device_alloc(-1)
                del sc
                continue
            L.ray_debug_fail_device_alloc(-1)
            assert np.array_equal(hits.view(np.uint32), ref.view(np.uint32))
            break
        else:
            pytest.fail("a scene still needed allocations after 200 of them")
    finally:
        L.ray_debug_fail_device_alloc(-1)
    assert failures >= 3
    del sc
    import gc

    gc.collect()
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) <= 64 << 20


def test_host_wait_bound_returns_timeout(renderer):
    """A 1 ms bound on the library's host waits: a host-buffer trace that
    takes longer returns RAY_ERR_TIMEOUT while its GPU work goes on; after
    the work ends, the same call with the default bound returns the hits."""
    import torch

    L = capi.lib()
    tris = scenes.random_triangles(200000, seed=95)
    n = 1 << 22
    rays = scenes.incoherent_rays(n, seed=96)
    sc = _scene(renderer, tris)
    sc.Commit()
    rays_h = torch.from_numpy(rays).pin_memory()
    hits_h = torch.zeros((n, 4), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    try:
        L.ray_set_wait_timeout_ms(1)
        rc = L.ray_scene_trace_closest(sc.handle, rays_h.data_ptr(), n, hits_h.data_ptr(), None, capi.RAY_MEM_HOST, None)
    finally:
        L.ray_set_wait_timeout_ms(0)
    assert rc == capi.RAY_ERR_TIMEOUT, L.ray_last_error()
    torch.cuda.synchronize()
    capi.check(L.ray_scene_trace_closest(sc.handle, rays_h.data_ptr(), n, hits_h.data_ptr(), None, capi.RAY_MEM_HOST, None))
    dev = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    rd = torch.from_numpy(rays).cuda()
    sc.trace_closest_device(rd.data_ptr(), n, dev.data_ptr(), 0, 0)
    torch.cuda.synchronize()
    assert np.array_equal(hits_h.numpy().view(np.uint32), dev.cpu().numpy().view(np.uint32))
