"""Concurrent calls from several host threads, as the reference's demo makes
them (GSRayTest.cpp: a thread pool renders 64-pixel buckets of one renderer
and scene, each bucket with its own RegionContext): every C-ABI call holds
one process-wide lock while it enqueues its work, so the calls serialise onto
the renderer's stream and the image equals the one-thread render."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu

pytestmark = pytest.mark.gpu


def _buckets(w, h, size):
    return [(x, y, min(size, w - x), min(size, h - y)) for y in range(0, h, size) for x in range(0, w, size)]


def _render(spec, iterations, threads):
    w, h = spec["size"]
    r = api.Renderer(w, h)
    sc = build_gpu(r, spec)
    r.Clear()
    regions = [api.RegionContext(*b) for b in _buckets(w, h, 32)]
    if threads == 1:
        for _ in range(iterations):
            for reg in regions:
                r.RenderScene(sc, reg)
    else:
        with ThreadPoolExecutor(threads) as pool:
            for _ in range(iterations):
                list(pool.map(lambda reg: r.RenderScene(sc, reg), regions))
    return r.get_pixels_ref()


def test_bucket_render_from_a_thread_pool(cuda_device):
    spec = scenes.cornell_box(0, 160, 96)
    one = _render(spec, 3, 1)
    many = _render(spec, 3, 8)
    assert np.array_equal(one.view(np.uint32), many.view(np.uint32))
    assert one[..., :3].mean() > 0.01


def test_concurrent_traces_of_one_scene(cuda_device):
    tris = scenes.random_triangles(50000, seed=81, mean_edge=0.01)
    r = api.Renderer(8, 8)
    sc = r.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(tris)
    m = sc.AddMaterial()
    sc.AddMeshInstance(sc.AddMesh(attrs, idx, [(m, 0, len(idx))]))
    sets = [scenes.incoherent_rays(20000 + 997 * k, seed=90 + k) for k in range(12)]
    alone = [sc.trace_closest(rs) for rs in sets]
    with ThreadPoolExecutor(6) as pool:
        together = list(pool.map(sc.trace_closest, sets))
    for a, b in zip(alone, together):
        assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def _soup_scene(r, n_tris, seed):
    sc = r.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(scenes.random_triangles(n_tris, seed=seed, mean_edge=0.01))
    m = sc.AddMaterial()
    sc.AddMeshInstance(sc.AddMesh(attrs, idx, [(m, 0, len(idx))]))
    return sc


def test_host_trace_waits_without_the_api_lock(cuda_device):
    """A host-buffer trace holds the process-wide lock only while it enqueues
    its work: while one thread waits for a long trace, another thread's calls
    go through (the longest pause between them stays far below the trace's
    duration), and both threads' results equal the one-thread results."""
    import threading
    import time

    import torch

    from raydemo_b200 import capi

    r = api.Renderer(8, 8)
    big, small = _soup_scene(r, 400000, 61), _soup_scene(r, 20000, 62)
    n = 8 * 1024 * 1024
    rays = torch.from_numpy(scenes.incoherent_rays(n, seed=63)).pin_memory()
    hits = torch.empty((n, 4), dtype=torch.float32).pin_memory()
    L = capi.lib()

    def trace_big():
        capi.check(L.ray_scene_trace_closest(big.handle, rays.data_ptr(), n, hits.data_ptr(), None, capi.RAY_MEM_HOST, None))

    trace_big()
    expect = hits.clone()
    t0 = time.perf_counter()
    trace_big()
    t_one = time.perf_counter() - t0
    small_rays = scenes.incoherent_rays(2000, seed=64)
    small_expect = np.asarray(small.trace_closest(small_rays)).view(np.uint32).copy()

    done = threading.Event()

    def worker():
        for _ in range(6):
            trace_big()
        done.set()

    th = threading.Thread(target=worker)
    stamps, small_results = [], []
    th.start()
    while not done.is_set():
        small.get_trace_tuning()
        stamps.append(time.perf_counter())
        if len(small_results) < 20:
            small_results.append(np.asarray(small.trace_closest(small_rays)).view(np.uint32).copy())
    th.join()
    gaps = np.diff(np.asarray(stamps))
    print(f"one trace {t_one * 1e3:.2f} ms; {len(stamps)} calls from the other thread meanwhile, longest pause {gaps.max() * 1e3:.2f} ms")
    assert len(stamps) > 50
    assert gaps.max() < 0.5 * t_one, (gaps.max(), t_one)
    assert torch.equal(hits.view(torch.int32), expect.view(torch.int32))
    for s in small_results:
        assert np.array_equal(s, small_expect)


def test_pixel_read_back_waits_without_the_api_lock(cuda_device):
    """ray_get_pixels waits for the renderer's frames with the process-wide
    lock let go: while one thread is inside a read-back whose frames are still
    rendering, another thread's calls keep going through (several of them
    complete in the first half of every such read-back), and the read-back
    images equal the one-thread one."""
    import threading
    import time

    spec = scenes.cornell_box(0, 1024, 1024, max_bounces=6)
    w, h = spec["size"]
    r = api.Renderer(w, h)
    sc = build_gpu(r, spec)
    r.set_kernel(1)  # fixed settings: no timed tuning frames
    r.set_ray_sort(0)
    r.set_trace_variant(0)
    other = _soup_scene(api.Renderer(8, 8), 20000, 65)

    def frames(spans=None):
        r.Clear()
        reg = api.RegionContext()
        for _ in range(4):
            r.RenderScene(sc, reg)
        t0 = time.perf_counter()
        img = r.get_pixels_ref().copy()
        if spans is not None:
            spans.append((t0, time.perf_counter()))
        return img

    expect = frames()
    frames()
    done = threading.Event()
    got, spans = [], []

    def worker():
        for _ in range(4):
            got.append(frames(spans))
        done.set()

    th = threading.Thread(target=worker)
    stamps = []
    th.start()
    while not done.is_set():
        other.get_trace_tuning()
        stamps.append(time.perf_counter())
    th.join()
    stamps = np.asarray(stamps)
    inside = [int(np.sum((stamps > a0) & (stamps < 0.5 * (a0 + a1)))) for a0, a1 in spans]
    print("read-backs (ms):", [round((a1 - a0) * 1e3, 2) for a0, a1 in spans], "calls in their first halves:", inside)
    for (a0, a1), k in zip(spans, inside):
        if a1 - a0 > 2e-3:  # a read-back that waited for its frames
            assert k >= 3, (a1 - a0, k)
    assert any(a1 - a0 > 2e-3 for a0, a1 in spans)
    for img in got:
        assert np.array_equal(img.view(np.uint32), expect.view(np.uint32))
