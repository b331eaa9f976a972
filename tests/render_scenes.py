"""Builds one scene spec (raydemo_b200.scenes) twice -- through this library's
API and through the reference library -- and renders both, for the image
parity tests."""
from __future__ import annotations

import numpy as np

from raydemo_b200 import api


def build_gpu(renderer: api.Renderer, spec: dict) -> api.Scene:
    sc = renderer.CreateScene()
    if "env" in spec:
        sc.SetEnvironment(**spec["env"])
    for rgba, srgb, mips in spec.get("textures", []):
        sc.AddTexture(rgba, is_srgb=srgb, generate_mipmaps=mips)
    for m in spec.get("materials", []):
        sc.AddMaterial(**m)
    for attrs, idx, shapes, layout in spec.get("meshes", []):
        sc.AddMesh(attrs, idx, shapes, layout=layout)
    for mesh, xf in spec.get("instances", []):
        sc.AddMeshInstance(mesh, xf)
    for l in spec.get("lights", []):
        sc.AddLight(**l)
    cam = sc.AddCamera(api.CameraDesc(**spec["camera"]))
    sc.set_current_cam(cam)
    return sc


def build_ref(ref, spec: dict):
    from oracle.oracle import RbCameraDesc, RefScene

    sc = RefScene(ref, True)
    if "env" in spec:
        e = spec["env"]
        sc.set_environment(e.get("env_col", (0, 0, 0)), e.get("env_clamp", 0.0), e.get("env_map", 0xFFFFFFFF))
    for rgba, srgb, mips in spec.get("textures", []):
        sc.add_texture(rgba, srgb, mips)
    for m in spec.get("materials", []):
        sc.add_material(**m)
    for attrs, idx, shapes, layout in spec.get("meshes", []):
        sc.add_mesh(attrs, idx, [tuple(s) if len(s) == 4 else (s[0], 0xFFFFFFFF, s[1], s[2]) for s in shapes], layout=layout)
    for mesh, xf in spec.get("instances", []):
        sc.add_instance(mesh, xf)
    for l in spec.get("lights", []):
        sc.add_light(**l)
    c = api.CameraDesc(**spec["camera"]).to_c()
    d = RbCameraDesc()
    for f, _ in RbCameraDesc._fields_:
        setattr(d, f, getattr(c, f))
    sc.add_camera(d)
    return sc


def render_gpu(spec: dict, iterations: int, rect=(0, 0, 0, 0), kernel: int = 0):
    w, h = spec["size"]
    r = api.Renderer(w, h)
    r.set_kernel(kernel)
    sc = build_gpu(r, spec)
    r.Clear()
    reg = api.RegionContext(*rect)
    for _ in range(iterations):
        r.RenderScene(sc, reg)
    return r.get_pixels_ref(), r, sc


def render_ref(ref, spec: dict, iterations: int, rect=(0, 0, 0, 0)):
    from oracle.oracle import RefRenderer

    w, h = spec["size"]
    rr = RefRenderer(ref, w, h, RefRenderer.REF, True)
    sc = build_ref(ref, spec)
    rr.render(sc, iterations, rect=rect, reset=True, nthreads=1)
    return rr.pixels()


def image_diff(a: np.ndarray, b: np.ndarray) -> dict:
    d = a.astype(np.float64) - b.astype(np.float64)
    same = np.all(a == b, axis=-1)
    return {"rmse": float(np.sqrt(np.mean(d[..., :3] ** 2))), "max": float(np.max(np.abs(d[..., :3]))),
            "identical_px": float(np.mean(same))}
