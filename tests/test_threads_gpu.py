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
