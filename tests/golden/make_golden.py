"""Generates the golden fixtures in this directory. Runs only where the
reference tree is present (it reads it as text and runs the reference library
built by oracle/Makefile); the tests read the committed .npz files.

  ref_tests.npz  -- data read from the reference's own tests (src/Ray/tests):
      prim_ray_gen   (16, 23) float32  g_primary_ray_gen_test_data, test_data.cpp:1-18
      scene1_attrs / scene1_indices / scene1_groups       test_scene1.h
      img1           (64, 64, 4) uint8  golden image of test_mesh_lights, test_img1.h
      scene2_attrs / scene2_indices / scene2_groups       test_scene2.h
  ref_outputs.npz -- outputs of the reference library on seeded inputs:
      halton_perms (1002,) uint16; halton_it1, halton_it300 (6144,) float32
      hits_*: closest hits of a 3,000-triangle random scene (Ref traversal)
      sort_*: keys and permutation of Ref::SortRays_CPU
      cam_*:  primary rays of Ref::GeneratePrimaryRays (tent filter, DOF)

Usage: python tests/golden/make_golden.py [/path/to/reference]   (default: $RAY_REFERENCE_SRC, or the
tree oracle/_ref was built from)
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)


def _array(src: str, name: str, conv):
    m = re.search(r"\b" + re.escape(name) + r"\s*\[\]\s*=\s*\{(.*?)\};", src, flags=re.S)
    if not m:
        raise ValueError(f"array {name} not found")
    body = m.group(1)
    toks = [t.strip() for t in body.replace("\n", " ").split(",")]
    return [conv(t) for t in toks if t]


def _float(t: str) -> float:
    return float(t.rstrip("fF"))


def _int(t: str) -> int:
    return int(t, 0)


def ref_tests(ref: str) -> dict:
    tdir = os.path.join(ref, "src", "Ray", "tests")
    out = {}
    src = open(os.path.join(tdir, "test_data.cpp")).read()
    out["prim_ray_gen"] = np.asarray(_array(src, "g_primary_ray_gen_test_data", _float), np.float32).reshape(16, 23)
    for k in ("1", "2"):
        src = open(os.path.join(tdir, f"test_scene{k}.h")).read()
        out[f"scene{k}_attrs"] = np.asarray(_array(src, "attrs", _float), np.float32)
        out[f"scene{k}_indices"] = np.asarray(_array(src, "indices", _int), np.uint32)
        out[f"scene{k}_groups"] = np.asarray(_array(src, "groups", _int), np.uint32)
    src = open(os.path.join(tdir, "test_img1.h")).read()
    out["img1"] = np.asarray(_array(src, "img_data", _int), np.uint8).reshape(64, 64, 4)
    return out


def ref_outputs() -> dict:
    from oracle.oracle import RbCameraDesc, RefLib, RefScene
    from raydemo_b200 import scenes

    ref = RefLib()
    out = {"halton_perms": ref.halton_perms(), "halton_it1": ref.halton_table(1), "halton_it300": ref.halton_table(300)}
    tris = scenes.random_triangles(3000, seed=11, mean_edge=0.05)
    rays = scenes.incoherent_rays(4000, seed=12)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    sc = RefScene(ref, True)
    m = sc.add_material(0)
    me = sc.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))])
    sc.add_instance(me)
    hits, obj = sc.trace_closest(rays)
    out.update(hits_tris=tris, hits_rays=rays, hits_prim=hits["prim"], hits_t=hits["t"], hits_u=hits["u"], hits_v=hits["v"])
    srays = scenes.incoherent_rays(5000, seed=13)
    srays[:, 0:3] = srays[:, 0:3] * 4.0 - 1.0  # some origins outside the root box
    root_min = np.array([0.0, 0.0, 0.0], np.float32)
    cell = np.array([2.0 / 255, 2.0 / 255, 2.0 / 255], np.float32)
    keys, perm = ref.sort_rays(srays, root_min, cell)
    out.update(sort_rays=srays, sort_root_min=root_min, sort_cell=cell, sort_keys=keys, sort_perm=perm)
    cam = RbCameraDesc()
    cam.type, cam.filter, cam.dtype = 0, 1, 0
    cam.origin[:] = [0.5, 1.0, 3.0]
    cam.fwd[:] = [0.0, -0.2, -0.9797959]
    cam.up[:] = [0.0, 1.0, 0.0]
    cam.fov, cam.gamma, cam.focus_distance, cam.focus_factor = 60.0, 1.0, 2.5, 0.1
    halton = ref.halton_table(5)
    rays_c = ref.generate_primary_rays(cam, 5, (3, 2, 9, 7), 32, 24, halton)
    out.update(cam_params=np.array([0.5, 1.0, 3.0, 0.0, -0.2, -0.9797959, 0.0, 1.0, 0.0, 60.0, 2.5, 0.1], np.float32),
               cam_rays=rays_c.view(np.float32).reshape(len(rays_c), -1))
    return out


def main() -> None:
    from oracle.oracle import reference_src

    src = sys.argv[1] if len(sys.argv) > 1 else reference_src()
    if not src:
        raise SystemExit("give the reference tree as the argument or in RAY_REFERENCE_SRC")
    ref = os.path.dirname(src) if os.path.basename(os.path.normpath(src)) == "src" else src
    np.savez_compressed(os.path.join(HERE, "ref_tests.npz"), **ref_tests(ref))
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), **ref_outputs())
    print("written", os.listdir(HERE))


if __name__ == "__main__":
    main()
