"""The instance tree: a BVH over the instances' world boxes built on the GPU
at commit (the reference's macro tree, SceneRef.cpp:492-516, traversed first
by Traverse_MacroTree_WithStack_ClosestHit, CoreRef.cpp:1133-1222), refitted
when only instance transforms changed. Hits with the tree equal the hits of
the instance-by-instance walk and of the compiled reference bit for bit;
trace time grows sublinearly with the instance count; a move of many
instances commits as a refit in well under a millisecond."""
import time

import numpy as np
import pytest

from raydemo_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _xforms(n, seed, spread):
    """n random transforms: rotation about y, scale U[0.5, 2], translation
    uniform in [0, spread)^3 (column-major 4x4, translation at 12..14)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 16), np.float32)
    for i in range(n):
        a = rng.random() * 6.283185
        s = 0.5 + 1.5 * rng.random()
        m = np.eye(4, dtype=np.float32)
        m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a) * s, -np.sin(a) * s, np.sin(a) * s, np.cos(a) * s
        m[1, 1] = s
        m[3, 0:3] = rng.random(3) * spread
        out[i] = m.reshape(-1)
    return out


def _rays(n, seed, spread):
    rays = scenes.incoherent_rays(n, seed=seed)
    rays[:, 0:3] = rays[:, 0:3] * spread
    return rays


def _mesh():
    tris = scenes.random_triangles(300, seed=41, mean_edge=0.08)
    return scenes.triangle_soup_mesh(tris)


def _scene(r, xf, tree):
    attrs, idx = _mesh()
    sc = r.CreateScene()
    m = sc.AddMaterial()
    mesh = sc.AddMesh(attrs, idx, [(m, 0, len(idx))])
    for x in xf:
        sc.AddMeshInstance(mesh, x)
    sc.set_trace_tuning(instance_tree=tree)
    return sc


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.fixture(scope="module")
def renderer(cuda_device):
    return api.Renderer(16, 16)


@pytest.mark.parametrize("n_inst", [2, 33, 4096])
def test_tree_equals_instance_walk_and_reference(renderer, reflib, n_inst):
    from oracle.oracle import RefScene

    spread = 2.0 * round(n_inst ** (1 / 3) + 1)
    xf = _xforms(n_inst, 42 + n_inst, spread)
    rays = _rays(60000, 43, spread)
    tree = _scene(renderer, xf, 1)
    flat = _scene(renderer, xf, -1)
    ht, ot = tree.trace_closest(rays, with_obj=True)
    assert tree.last_trace_info().error_flags == 0
    assert tree.instance_tree_info().instances == n_inst
    assert flat.instance_tree_info().instances == 0
    hf, of = flat.trace_closest(rays, with_obj=True)
    assert (ht["prim"] >= 0).mean() > 0.01
    assert _same(ht, hf) and np.array_equal(ot, of)
    # the compiled reference (its own macro tree over the same instances)
    attrs, idx = _mesh()
    rs = RefScene(reflib, True)
    m = rs.add_material(0)
    me = rs.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))])
    for x in xf:
        rs.add_instance(me, x)
    sub = rays[:20000]
    rh, ro = rs.trace_closest(sub)
    assert np.array_equal(ht["prim"][:20000], rh["prim"])
    hit = rh["prim"] >= 0
    assert _same(ht[:20000][hit], rh[hit])
    assert np.array_equal(ot[:20000][hit], ro[hit])


def test_trace_time_grows_sublinearly_with_instances(renderer):
    """The same rays in scenes of 256 and 4096 instances spread over the
    same volume: walking the instance tree, 16x the instances costs less
    than half of 16x the time (the denser scene also gives each ray more
    geometry to meet); testing the instances in turn costs far more."""
    import torch

    spread = 40.0
    n = 1 << 20
    rays = _rays(n, 44, spread)
    rd = torch.from_numpy(rays).cuda()
    hd = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()

    def ms(sc):
        for _ in range(2):
            sc.trace_closest_device(rd.data_ptr(), n, hd.data_ptr(), 0, s.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(3):
            sc.trace_closest_device(rd.data_ptr(), n, hd.data_ptr(), 0, s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        assert sc.last_trace_info().error_flags == 0
        return e0.elapsed_time(e1) / 3

    t = {}
    for k in (256, 4096):
        xf = _xforms(k, 45, spread)
        t[("tree", k)] = ms(_scene(renderer, xf, 1))
        t[("flat", k)] = ms(_scene(renderer, xf, -1))
    print("trace ms", {f"{a}{b}": round(v, 3) for (a, b), v in t.items()})
    assert t[("tree", 4096)] < 8.0 * t[("tree", 256)]  # 16x the instances (and the geometry a ray meets)
    assert t[("flat", 4096)] > 4.0 * t[("tree", 4096)]


def test_moves_refit_the_tree(renderer):
    """1000 of 4096 instances moved, then one commit: a refit (same
    topology, new boxes) measured in well under a millisecond of host time;
    the hits equal those of a scene built fresh with the new transforms and
    of the instance-by-instance walk."""
    spread = 36.0
    xf = _xforms(4096, 46, spread)
    rays = _rays(60000, 47, spread)
    sc = _scene(renderer, xf, 1)
    sc.trace_closest(rays[:10])  # built
    assert sc.instance_tree_info().refit == 0
    moved = _xforms(1000, 48, spread)
    pick = np.random.default_rng(49).choice(4096, 1000, replace=False)
    best = 1e9
    for rep in range(3):
        for i, x in zip(pick, moved if rep % 2 == 0 else xf[pick]):
            sc.SetMeshInstanceTransform(int(i), x)
        t0 = time.perf_counter()
        sc.Commit()
        best = min(best, (time.perf_counter() - t0) * 1e3)
        info = sc.instance_tree_info()
        assert info.refit == 1 and info.instances == 4096
    # the moves applied last (rep 2: the moved transforms)
    xf2 = xf.copy()
    xf2[pick] = moved
    print("refit commit ms", round(best, 3), "tree ms", round(info.ms, 3))
    assert best < 1.0
    hits = sc.trace_closest(rays)
    assert sc.last_trace_info().error_flags == 0
    fresh = _scene(renderer, xf2, 1).trace_closest(rays)
    walk = _scene(renderer, xf2, -1).trace_closest(rays)
    assert _same(hits, fresh) and _same(hits, walk)


def test_render_loop_with_the_tree_equals_the_walk(cuda_device):
    """A frame of the Cornell box's scene with the instance tree forced on
    (its few instances would otherwise be walked in turn) renders the same
    image."""
    from render_scenes import build_gpu

    spec = scenes.cornell_box(0, 64, 48)
    imgs = []
    for tree in (-1, 1):
        r = api.Renderer(*spec["size"])
        sc = build_gpu(r, spec)
        sc.set_trace_tuning(instance_tree=tree)
        r.set_kernel(1)
        reg = api.RegionContext()
        for _ in range(2):
            r.RenderScene(sc, reg)
        assert r.frame_info().error_flags == 0
        imgs.append(r.get_pixels_ref())
    assert _same(imgs[0], imgs[1])
