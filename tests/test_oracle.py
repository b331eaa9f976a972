"""The CPU oracle against the reference's own golden vectors and against the
compiled reference library (CPU only)."""
import os

import numpy as np
import pytest

from raydemo_b200 import scenes


def test_primary_ray_gen_golden(oracle, ref_tests):
    # test_primary_ray_gen.cpp:19-65: camera at (0,0,4) looking -z, fov 53.13,
    # Box filter, iteration 0, 4x4 rect, all-zero sample table, eps 1e-3
    cam = oracle.construct_camera((0, 0, 4), (0, 0, -1), (0, 0, 0), 53.13, filter=0, gamma=2.2)
    rays = oracle.generate_primary_rays(cam, 0, (0, 0, 4, 4), 4, 4, np.zeros(512, np.float32))
    g = ref_tests["prim_ray_gen"]
    assert np.array_equal(rays["xy"], g[:, 0].astype(np.int32))
    got = np.concatenate([rays["o"], rays["d"], rays["c"], rays["ior"][:, None], rays["do_dx"], rays["dd_dx"], rays["do_dy"],
                          rays["dd_dy"]], axis=1)
    np.testing.assert_allclose(got, g[:, 1:], atol=1e-3)


def test_halton_matches_reference(oracle, ref_outputs):
    assert np.array_equal(oracle.halton_perms(), ref_outputs["halton_perms"])
    for it in (1, 300):
        assert np.array_equal(oracle.halton_table(it).view(np.uint32), ref_outputs[f"halton_it{it}"].view(np.uint32))


def test_closest_hit_matches_reference(oracle, ref_outputs):
    tris = ref_outputs["hits_tris"]
    rays = ref_outputs["hits_rays"]
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    for hits in (oracle.closest_hit_brute(acc, rays), oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays)):
        assert np.array_equal(hits["prim"], ref_outputs["hits_prim"])
        for k in ("t", "u", "v"):
            hit = hits["prim"] >= 0
            assert np.array_equal(hits[k][hit].view(np.uint32), ref_outputs[f"hits_{k}"][hit].view(np.uint32))


def test_sort_matches_reference(oracle, ref_outputs):
    keys = oracle.ray_hash(ref_outputs["sort_rays"], ref_outputs["sort_root_min"], ref_outputs["sort_cell"])
    assert np.array_equal(keys, ref_outputs["sort_keys"])
    assert np.array_equal(oracle.sort_perm(keys), ref_outputs["sort_perm"])


def test_raygen_matches_reference(oracle, ref_outputs):
    p = ref_outputs["cam_params"]
    cam = oracle.construct_camera(p[0:3], p[3:6], p[6:9], float(p[9]), filter=1, focus_distance=float(p[10]),
                                  focus_factor=float(p[11]))
    rays = oracle.generate_primary_rays(cam, 5, (3, 2, 9, 7), 32, 24, ref_outputs["halton_it1"] * 0 + oracle.halton_table(5))
    assert np.array_equal(rays.view(np.float32).reshape(len(rays), -1).view(np.uint32), ref_outputs["cam_rays"].view(np.uint32))


def test_brute_force_equals_bvh_oracle(oracle):
    tris = scenes.random_triangles(20000, seed=5)
    rays = scenes.incoherent_rays(3000, seed=6)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    a = oracle.closest_hit_brute(acc, rays)
    b = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_live_reference_large(oracle, reflib):
    """Against the reference library itself, when it is built here."""
    from oracle.oracle import RefScene

    tris = scenes.random_triangles(60000, seed=21)
    rays = scenes.incoherent_rays(20000, seed=22)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    sc = RefScene(reflib, True)
    m = sc.add_material(0)
    sc.add_instance(sc.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))]))
    ref_hits, _ = sc.trace_closest(rays)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    hits = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays)
    assert np.array_equal(hits["prim"], ref_hits["prim"])


def test_oracle_matches_reference_at_full_size(oracle):
    """The oracle's closest hits on the whole headline workload (2,097,152
    triangles, 4,194,304 incoherent rays) against the compiled reference's
    Ref traversal, through the committed per-chunk digests; the fixture's
    recorded reference deviations (exact-t ties kept in traversal order) are
    where the two answers may differ, and there the oracle must give the
    recorded closest hit."""
    import bench

    tris, rays = bench.make_workload(0)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    acc = oracle.preprocess_tris(attrs[:, :3].copy(), idx)
    box = np.concatenate([tris.reshape(-1, 3).min(axis=0), tris.reshape(-1, 3).max(axis=0)])
    threads = len(os.sched_getaffinity(0))
    hits = oracle.closest_hit_bvh(acc, scenes.tri_aabbs(tris), rays, nthreads=threads, world_box=box)
    par = bench.parity_vs_reference("inc", tris, rays, hits.view(np.uint32).reshape(-1, 4))
    assert par["mismatch"] == 0 and par["unexplained_deviation_rays"] == 0, par
    assert par["hits"] == par["ref_hits"]
