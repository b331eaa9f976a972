"""Dynamic instances: SetMeshInstanceTransform / AddMeshInstance /
RemoveMeshInstance between traces and frames (the reference rebuilds its
instance tree, SceneRef.cpp:370-414, 492-516). Here the instance level is a
list of instance records that the traversal tests box by box, so an edit
re-uploads the records and rebuilds nothing; the upload waits for the traces
and frames already enqueued that read the old records."""
import time

import numpy as np
import pytest

from raydemo_b200 import api, scenes

from render_scenes import build_gpu, render_gpu

pytestmark = pytest.mark.gpu


def _xform(rng):
    a = rng.random() * 6.28
    s = 0.5 + rng.random()
    m = np.eye(4, dtype=np.float32)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a) * s, -np.sin(a) * s, np.sin(a) * s, np.cos(a) * s
    m[1, 1] = s
    m[3, 0:3] = rng.random(3) * 2 - 1
    return m.reshape(-1)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_edited_instances_match_fresh_scene_and_reference(cuda_device, reflib):
    from oracle.oracle import RefScene

    rng = np.random.default_rng(61)
    tris = scenes.random_triangles(60000, seed=62, mean_edge=0.01)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    pos, faces = scenes.icosphere(3, 0.3)
    sattrs = np.concatenate([pos, pos / np.linalg.norm(pos, axis=1, keepdims=True), np.zeros((len(pos), 2))], 1).astype(np.float32)
    r = api.Renderer(16, 16)
    sc = r.CreateScene()
    m = sc.AddMaterial()
    meshes = [sc.AddMesh(attrs, idx, [(m, 0, len(idx))]), sc.AddMesh(sattrs, faces.reshape(-1), [(m, 0, faces.size)])]
    inst = [(meshes[k % 2], _xform(rng)) for k in range(6)]
    for mesh, x in inst:
        sc.AddMeshInstance(mesh, x)
    rays = scenes.incoherent_rays(40000, seed=63)
    rays[:, 0:3] = rays[:, 0:3] * 3 - 1.5
    before, _ = sc.trace_closest(rays, with_obj=True)
    # move three, remove one, add one
    t0 = time.perf_counter()
    for k in (0, 3, 4):
        x = _xform(rng)
        inst[k] = (inst[k][0], x)
        sc.SetMeshInstanceTransform(k, x)
    sc.RemoveMeshInstance(2)
    del inst[2]
    x = _xform(rng)
    sc.AddMeshInstance(meshes[1], x)
    inst.append((meshes[1], x))
    sc.Commit()
    dt = time.perf_counter() - t0
    print(f"instance edits + commit: {dt * 1e3:.3f} ms")
    hits, obj = sc.trace_closest(rays, with_obj=True)
    assert sc.last_trace_info().error_flags == 0
    assert not _same(hits, before)
    fresh = r.CreateScene()
    fm = fresh.AddMaterial()
    fmeshes = [fresh.AddMesh(attrs, idx, [(fm, 0, len(idx))]), fresh.AddMesh(sattrs, faces.reshape(-1), [(fm, 0, faces.size)])]
    for mesh, x in inst:
        fresh.AddMeshInstance(fmeshes[mesh], x)
    fh, fo = fresh.trace_closest(rays, with_obj=True)
    assert _same(hits, fh) and np.array_equal(obj, fo)
    rsc = RefScene(reflib, True)
    rmat = rsc.add_material(0)
    rmeshes = [rsc.add_mesh(attrs, idx, [(rmat, 0xFFFFFFFF, 0, len(idx))]),
               rsc.add_mesh(sattrs, faces.reshape(-1), [(rmat, 0xFFFFFFFF, 0, faces.size)])]
    for mesh, x in inst:
        rsc.add_instance(rmeshes[mesh], x)
    ref_hits, ref_obj = rsc.trace_closest(rays)
    assert np.array_equal(hits["prim"], ref_hits["prim"]) and np.array_equal(obj, ref_obj)
    assert _same(hits["t"], ref_hits["t"])


def test_instance_moves_between_frames_in_flight(cuda_device):
    """Frames enqueued and the sphere moved right after each, without waiting:
    the image equals the same sequence with the host waiting for every frame."""
    spec = scenes.cornell_box(0, 96, 96)
    rng = np.random.default_rng(64)
    moves = []
    for _ in range(6):
        xf = np.eye(4, dtype=np.float32)
        xf[3, 0:3] = (0.3 + 0.4 * rng.random(), 0.3 + 0.4 * rng.random(), 0.2 + 0.3 * rng.random())
        moves.append(xf.reshape(-1))

    def run(wait):
        import torch

        w, h = spec["size"]
        r = api.Renderer(w, h)
        r.set_kernel(1)
        sc = build_gpu(r, spec)
        r.Clear()
        reg = api.RegionContext()
        for xf in moves:
            r.RenderScene(sc, reg)
            if wait:
                torch.cuda.synchronize()
            sc.SetMeshInstanceTransform(1, xf)
        r.RenderScene(sc, reg)
        return r.get_pixels_ref()

    a, b = run(False), run(True)
    assert _same(a, b)
    still, _, _ = render_gpu(spec, 7, kernel=1)
    assert not _same(a, still)  # the moves show


def test_instance_edits_render_as_the_ref_renderer(reflib, cuda_device):
    """The same instance edits through both libraries (add, move, remove; the
    reference rebuilds its instance tree, SceneRef.cpp:370-420): the images agree."""
    from oracle.oracle import RefRenderer

    from render_scenes import build_ref, image_diff

    spec = scenes.cornell_box(4, 96, 96)
    w, h = spec["size"]
    moved = np.eye(4, dtype=np.float32)
    moved[3, 0:3] = (0.35, 0.3, 0.55)
    extra = np.eye(4, dtype=np.float32)
    extra[3, 0:3] = (0.7, 0.75, 0.6)
    r = api.Renderer(w, h)
    r.set_kernel(1)
    sc = build_gpu(r, spec)
    rs = build_ref(reflib, spec)
    for edit in (lambda s: s.AddMeshInstance(1, extra.reshape(-1)), lambda s: s.SetMeshInstanceTransform(1, moved.reshape(-1)),
                 lambda s: s.RemoveMeshInstance(2)):
        edit(sc)
    rs.add_instance(1, extra.reshape(-1))
    rs.set_instance_xform(1, moved.reshape(-1))
    rs.remove_instance(2)
    r.Clear()
    reg = api.RegionContext()
    for _ in range(4):
        r.RenderScene(sc, reg)
    gpu = r.get_pixels_ref()
    rr = RefRenderer(reflib, w, h, RefRenderer.REF, True)
    rr.render(rs, 4, reset=True, nthreads=1)
    d = image_diff(gpu, rr.pixels())
    print("instance edits", d)
    assert d["identical_px"] >= 0.95 and d["rmse"] <= 1e-3, d
    still, _, _ = render_gpu(spec, 4, kernel=1)
    assert not _same(gpu, still)
