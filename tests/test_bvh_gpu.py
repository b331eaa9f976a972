"""Structure of the GPU-built wide BVH, read back and checked on the host:
every triangle sits in exactly one leaf, and its box lies inside the decoded
box of every slot on its path from the root (so no box test can reject a ray
that reaches the triangle)."""
import ctypes as C

import numpy as np
import pytest

from raydemo_b200 import capi, scenes
from raydemo_b200.api import Renderer

pytestmark = pytest.mark.gpu

NODE = np.dtype([("p", "<f4", 3), ("e", "u1", 3), ("imask", "u1"), ("child_base", "<u4"), ("tri_base", "<u4"), ("meta", "u1", 8),
                 ("qlo", "u1", (3, 8)), ("qhi", "u1", (3, 8))])
TRI = np.dtype([("f", "<f4", 10), ("mi", "<u4"), ("back_mi", "<u4")])
assert NODE.itemsize == 80 and TRI.itemsize == 48


def _read(sc, what, dtype):
    n = C.c_uint64()
    capi.check(capi.lib().ray_scene_debug_read(sc.handle, what, None, 0, C.byref(n)))
    buf = np.zeros(n.value // dtype.itemsize, dtype)
    capi.check(capi.lib().ray_scene_debug_read(sc.handle, what, buf.ctypes.data, n.value, C.byref(n)))
    return buf


def _check(tris):
    r = Renderer(16, 16)
    sc = r.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(tris)
    m = sc.AddMaterial()
    sc.AddMeshInstance(sc.AddMesh(attrs, idx, [(m, 0, len(idx))]))
    sc.Commit()
    nodes = _read(sc, 0, NODE)
    leaf = _read(sc, 1, TRI)
    info = sc.mesh_bvh_info(0)
    assert len(nodes) == info.nodes and len(leaf) == len(tris)
    lo_t, hi_t = tris.min(axis=1), tris.max(axis=1)
    seen = np.zeros(len(tris), np.int32)
    depth_max = 0
    stack = [(0, np.full(3, -np.inf, np.float32), np.full(3, np.inf, np.float32), 1)]
    while stack:
        ni, elo, ehi, depth = stack.pop()
        depth_max = max(depth_max, depth)
        nd = nodes[ni]
        scale = np.ldexp(np.float32(1.0), nd["e"].astype(np.int32) - 127).astype(np.float32)
        rank = 0
        toff_seen = []
        for s in range(8):
            meta = int(nd["meta"][s])
            if meta == 0:
                continue
            # exact decode: p + q * 2^e is representable, so float32 == float64 here
            clo = (nd["p"].astype(np.float64) + nd["qlo"][:, s] * scale.astype(np.float64))
            chi = (nd["p"].astype(np.float64) + nd["qhi"][:, s] * scale.astype(np.float64))
            assert np.array_equal(clo.astype(np.float32).astype(np.float64), clo)
            assert np.array_equal(chi.astype(np.float32).astype(np.float64), chi)
            slo, shi = np.maximum(elo, clo), np.minimum(ehi, chi)
            if (meta & 31) >= 24:
                assert (meta & 31) == 24 + s and (nd["imask"] >> s) & 1
                stack.append((int(nd["child_base"]) + rank, slo, shi, depth + 1))
                rank += 1
            else:
                cnt = bin(meta >> 5).count("1")
                assert (meta >> 5) == (1 << cnt) - 1 and 1 <= cnt <= 3
                for k in range(cnt):
                    li = int(nd["tri_base"]) + (meta & 31) + k
                    toff_seen.append((meta & 31) + k)
                    t = int(leaf[li]["mi"])
                    seen[t] += 1
                    assert np.all(lo_t[t] >= slo) and np.all(hi_t[t] <= shi), (ni, s, t)
        assert len(set(toff_seen)) == len(toff_seen)
    assert np.all(seen == 1)
    assert depth_max == info.depth
    return info


@pytest.mark.parametrize("n,seed,edge", [(1, 1, 0.1), (2, 2, 0.1), (3, 3, 0.1), (4, 4, 0.1), (100, 5, 0.05), (20000, 6, 0.01)])
def test_bvh_structure(cuda_device, n, seed, edge):
    _check(scenes.random_triangles(n, seed=seed, mean_edge=edge))


def test_bvh_structure_far_from_origin(cuda_device):
    # large coordinates with small extents: the quantisation frame must still decode exactly
    tris = scenes.random_triangles(5000, seed=7, mean_edge=1e-4) * np.float32(1e-2) + np.float32(3000.0)
    _check(tris)


def test_bvh_structure_duplicates(cuda_device):
    # many identical centroids (equal Morton keys) and flat geometry
    base = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    tris = np.repeat(base, 3000, axis=0)
    _check(tris)
