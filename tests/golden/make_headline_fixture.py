"""Generates headline_ref.npz: the compiled reference's closest hits on the
full closest-hit microbench (2,097,152 random triangles; 4,194,304
incoherent rays and the 4,194,304 coherent 2048x2048 pinhole rays), stored as
per-chunk digests so that the fixture stays small.

The reference run is Ray::Ref::Traverse_MacroTree_WithStack_ClosestHit
(src/Ray/internal/CoreRef.cpp:1133-1222) over the reference's own SAH wide BVH,
through oracle/_ref (built from the reference sources by oracle/Makefile with
-ffp-contract=off), on all host threads.

Where the reference's answer differs from the order-independent one (the
closest hit, exact ties in t going to the lower triangle index) the ray is
recorded explicitly with both answers, classified by a brute-force test of all
triangles with the reference's triangle arithmetic (the oracle):
  kind 0  exact-t tie: the reference kept another triangle at the same t
          (its traversal keeps the first one it meets, CoreRef.cpp:34);
  kind 1  reference box false negative: a closer hit exists that the
          reference's traversal culled.
Any other difference stops the script.

Usage: python tests/golden/make_headline_fixture.py   (needs oracle/_ref built;
takes a few minutes: the reference's SAH build of 2M triangles is ~30 s, its
scalar traversal of 8M rays ~2 min on 8 threads)
"""
from __future__ import annotations

import hashlib
import os
import platform
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "headline_ref.npz")


def _records(hits) -> np.ndarray:
    """(n, 4) uint32 records prim, t, u, v from a HIT_DTYPE array."""
    r = np.zeros((len(hits), 4), np.uint32)
    r[:, 0] = hits["prim"].view(np.uint32)
    r[:, 1] = hits["t"].view(np.uint32)
    r[:, 2] = hits["u"].view(np.uint32)
    r[:, 3] = hits["v"].view(np.uint32)
    return r


def _one(name, tris, rays, ref_scene, orc, acc, aabbs, box, threads) -> dict:
    import bench

    t0 = time.perf_counter()
    ref_hits, _ = ref_scene.trace_closest(rays, nthreads=threads, backend=0)
    t_ref = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc_hits = orc.closest_hit_bvh(acc, aabbs, rays, nthreads=threads, world_box=box)
    t_orc = time.perf_counter() - t0
    R = _records(ref_hits)
    O = _records(orc_hits)
    miss = orc_hits["prim"] < 0
    # a miss carries no t/u/v worth comparing: the records keep tmax and zeros
    diff = np.nonzero(np.any(R != O, axis=1))[0]
    kinds = []
    for i in diff:
        b = orc.closest_hit_brute(acc, rays[i:i + 1], nthreads=1, world_box=box)[0]
        bo = _records(np.array([b], dtype=orc_hits.dtype))[0]
        if not np.array_equal(bo, O[i]):
            raise SystemExit(f"{name} ray {i}: oracle BVH {O[i]} differs from brute force {bo}")
        rp = int(ref_hits["prim"][i])
        if rp >= 0 and b["prim"] >= 0 and ref_hits["t"][i] == b["t"]:
            # the reference's triangle must hit at exactly the same t
            one = orc.closest_hit_brute(acc[rp:rp + 1], rays[i:i + 1], nthreads=1)[0]
            if one["prim"] != 0 or one["t"] != b["t"]:
                raise SystemExit(f"{name} ray {i}: reference triangle {rp} does not hit at t={b['t']}")
            kinds.append(0)
        elif b["prim"] >= 0 and (rp < 0 or ref_hits["t"][i] > b["t"]):
            kinds.append(1)
        else:
            raise SystemExit(f"{name} ray {i}: reference {R[i]} is closer than brute force {bo}")
    dig = bench.chunk_digests(R)
    print(f"{name}: reference {t_ref:.1f} s, oracle {t_orc:.1f} s, hits {int((ref_hits['prim'] >= 0).sum())}, "
          f"deviations {len(diff)} (ties {kinds.count(0)}, box false negatives {kinds.count(1)})", flush=True)
    return {f"{name}_digests": dig, f"{name}_hits": np.int64((ref_hits["prim"] >= 0).sum()),
            f"{name}_sha256": np.bytes_(hashlib.sha256(R.tobytes()).hexdigest()),
            f"{name}_inputs_sha256": np.bytes_(bench.inputs_sha256(tris, rays)),
            f"{name}_dev_idx": diff.astype(np.int64), f"{name}_dev_ref": R[diff], f"{name}_dev_ours": O[diff],
            f"{name}_dev_kind": np.asarray(kinds, np.int8), f"{name}_misses": np.int64(miss.sum())}


def main() -> None:
    import bench
    from oracle.oracle import Oracle, RefLib, RefScene
    from raydemo_b200 import scenes

    threads = len(os.sched_getaffinity(0))
    tris, rays = bench.make_workload(0)
    coh = scenes.coherent_rays(2048, 2048)
    ref = RefLib()
    t0 = time.perf_counter()
    sc = RefScene(ref, True)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    m = sc.add_material(0)
    sc.add_instance(sc.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))]))
    print(f"reference SAH build {time.perf_counter() - t0:.1f} s", flush=True)
    orc = Oracle()
    acc = orc.preprocess_tris(attrs[:, :3].copy(), idx)
    aabbs = scenes.tri_aabbs(tris)
    box = np.concatenate([tris.reshape(-1, 3).min(axis=0), tris.reshape(-1, 3).max(axis=0)])
    out = {}
    out.update(_one("inc", tris, rays, sc, orc, acc, aabbs, box, threads))
    out.update(_one("coh", tris, coh, sc, orc, acc, aabbs, box, threads))
    gxx = subprocess.run(["g++", "--version"], capture_output=True, text=True).stdout.splitlines()[0]
    out["chunk"] = np.int64(bench.PARITY_CHUNK)
    out["made_with"] = np.bytes_(f"{gxx}; -ffp-contract=off; Ref wide BVH; {platform.machine()}")
    np.savez_compressed(OUT, **out)
    print("written", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
