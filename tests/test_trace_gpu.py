"""Closest hits on the GPU against the oracle and the reference: prim id, t,
u and v bit for bit."""
import numpy as np
import pytest

from raydemo_b200 import scenes
from raydemo_b200.api import Renderer

pytestmark = pytest.mark.gpu


def _scene(tris, renderer, xform=None, instances=1):
    sc = renderer.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(tris)
    sc.AddTexture(np.full((1, 1, 4), 255, np.uint8))
    m = sc.AddMaterial()
    mesh = sc.AddMesh(attrs, idx, [(m, 0, len(idx))])
    for _ in range(instances):
        sc.AddMeshInstance(mesh, xform)
    return sc


def _same(a, b):
    return np.array_equal(a.view(np.uint32).reshape(len(a), -1), b.view(np.uint32).reshape(len(b), -1))


@pytest.fixture(scope="module")
def renderer(cuda_device):
    return Renderer(64, 64)


def test_golden_hits(renderer, ref_outputs):
    sc = _scene(ref_outputs["hits_tris"], renderer)
    hits = sc.trace_closest(ref_outputs["hits_rays"])
    assert np.array_equal(hits["prim"], ref_outputs["hits_prim"])
    hit = hits["prim"] >= 0
    for k in ("t", "u", "v"):
        assert np.array_equal(hits[k][hit].view(np.uint32), ref_outputs[f"hits_{k}"][hit].view(np.uint32))


@pytest.mark.parametrize("n_tris,n_rays,seed", [(1, 1000, 1), (2, 1000, 2), (7, 2000, 3), (1000, 5000, 4), (200000, 50000, 5)])
def test_random_scenes_vs_oracle(renderer, oracle, n_tris, n_rays, seed):
    tris = scenes.random_triangles(n_tris, seed=seed, mean_edge=0.05 if n_tris < 1000 else 0.005)
    rays = scenes.incoherent_rays(n_rays, seed=seed + 100)
    sc = _scene(tris, renderer)
    hits = sc.trace_closest(rays)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    exp = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays) if n_tris > 5000 else oracle.closest_hit_brute(acc, rays)
    assert (exp["prim"] >= 0).any() or n_tris < 10
    miss = exp["prim"] < 0
    assert np.array_equal(hits["prim"], exp["prim"])
    assert _same(hits[~miss], exp[~miss])


def test_live_reference(renderer, reflib):
    from oracle.oracle import RefScene

    tris = scenes.random_triangles(100000, seed=31)
    rays = scenes.incoherent_rays(40000, seed=32)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    sc = RefScene(reflib, True)
    m = sc.add_material(0)
    sc.add_instance(sc.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))]))
    ref_hits, ref_obj = sc.trace_closest(rays)
    hits, obj = _scene(tris, renderer).trace_closest(rays, with_obj=True)
    assert np.array_equal(hits["prim"], ref_hits["prim"])
    assert np.array_equal(obj, ref_obj)
    hit = hits["prim"] >= 0
    assert _same(hits[hit], ref_hits[hit])


def test_tmax_and_coherent(renderer, oracle):
    tris = scenes.random_triangles(50000, seed=41)
    rays = scenes.coherent_rays(128, 128)
    rays[::3, 3] = 1.7  # short rays
    sc = _scene(tris, renderer)
    hits = sc.trace_closest(rays)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    exp = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays)
    assert np.array_equal(hits["prim"], exp["prim"])
    assert _same(hits[exp["prim"] >= 0], exp[exp["prim"] >= 0])
    assert np.all(hits["t"][::3][hits["prim"][::3] >= 0] < 1.7)


def test_axis_aligned_geometry_and_rays(renderer, oracle):
    # a grid of axis-aligned quads hit by axis-aligned rays (zero direction
    # components, origins on box planes)
    quads = []
    for k in range(8):
        z = 0.1 * k
        quads += [[[0, 0, z], [1, 0, z], [1, 1, z]], [[0, 0, z], [1, 1, z], [0, 1, z]]]
    tris = np.asarray(quads, np.float32)
    g = np.linspace(0.0, 1.0, 33, dtype=np.float32)
    X, Y = np.meshgrid(g, g)
    n = X.size
    rays = np.zeros((2 * n, 8), np.float32)
    rays[:n, 0], rays[:n, 1], rays[:n, 2], rays[:n, 6] = X.ravel(), Y.ravel(), -1.0, 1.0
    rays[n:, 0], rays[n:, 1], rays[n:, 2], rays[n:, 6] = X.ravel(), Y.ravel(), 0.35, -1.0
    rays[:, 3] = 1e30
    hits = _scene(tris, renderer).trace_closest(rays)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    exp = oracle.closest_hit_brute(oracle.preprocess_tris(attrs[:, :3].copy(), idx), rays)
    assert np.array_equal(hits["prim"], exp["prim"])
    assert _same(hits[exp["prim"] >= 0], exp[exp["prim"] >= 0])


def test_instances_with_transforms(renderer, reflib):
    from oracle.oracle import RefScene

    tris = scenes.random_triangles(20000, seed=51, mean_edge=0.01)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    rng = np.random.default_rng(52)
    xforms = []
    for k in range(5):
        a = rng.random() * 6.28
        s = 0.5 + rng.random()
        m = np.eye(4, dtype=np.float32)
        m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a) * s, -np.sin(a) * s, np.sin(a) * s, np.cos(a) * s
        m[1, 1] = s
        m[3, 0:3] = rng.random(3) * 2 - 1  # translation in elements 12..14 (column-major)
        xforms.append(m.reshape(-1))
    rsc = RefScene(reflib, True)
    mat = rsc.add_material(0)
    rm = rsc.add_mesh(attrs, idx, [(mat, 0xFFFFFFFF, 0, len(idx))])
    gsc = renderer.CreateScene()
    gm_mat = gsc.AddMaterial()
    gm = gsc.AddMesh(attrs, idx, [(gm_mat, 0, len(idx))])
    for x in xforms:
        rsc.add_instance(rm, x)
        gsc.AddMeshInstance(gm, x)
    rays = scenes.incoherent_rays(30000, seed=53)
    rays[:, 0:3] = rays[:, 0:3] * 3 - 1.5
    ref_hits, ref_obj = rsc.trace_closest(rays)
    hits, obj = gsc.trace_closest(rays, with_obj=True)
    assert np.array_equal(hits["prim"], ref_hits["prim"])
    assert np.array_equal(obj, ref_obj)
    hit = hits["prim"] >= 0
    assert _same(hits[hit], ref_hits[hit])


def test_empty_and_degenerate(renderer, oracle):
    sc = renderer.CreateScene()
    hits = sc.trace_closest(scenes.incoherent_rays(100, seed=1))
    assert np.all(hits["prim"] == -1)
    tris = scenes.random_triangles(500, seed=61, mean_edge=0.05)
    tris[::7, 1] = tris[::7, 0]  # zero-area triangles never hit (InvalidTriangle)
    rays = scenes.incoherent_rays(3000, seed=62)
    hits = _scene(tris, renderer).trace_closest(rays)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    exp = oracle.closest_hit_brute(oracle.preprocess_tris(attrs[:, :3].copy(), idx), rays)
    assert np.array_equal(hits["prim"], exp["prim"])
    assert not np.any(np.isin(hits["prim"], np.arange(0, 500, 7)))
    assert len(sc.trace_closest(np.zeros((0, 8), np.float32))) == 0


def test_full_size_microbench_subset(renderer, oracle):
    """The 2,097,152-triangle scene: all 4,194,304 rays traced on the GPU,
    a seeded subset checked against the oracle, plus size-independent
    properties on the full set."""
    tris = scenes.random_triangles(2097152, seed=0)
    rays = scenes.incoherent_rays(4194304, seed=1)
    sc = _scene(tris, renderer)
    hits = sc.trace_closest(rays)
    info = sc.last_trace_info()
    assert info.error_flags == 0
    hit = hits["prim"] >= 0
    assert 0.85 < hit.mean() < 0.99
    assert np.all(hits["t"][hit] > 0) and np.all(hits["prim"][hit] < len(tris))
    sub = np.random.default_rng(7).choice(len(rays), 65536, replace=False)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    exp = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays[sub])
    assert np.array_equal(hits["prim"][sub], exp["prim"])
    assert _same(hits[sub][exp["prim"] >= 0], exp[exp["prim"] >= 0])
    # tracing twice gives the same bytes
    assert _same(sc.trace_closest(rays[:100000]), hits[:100000])
