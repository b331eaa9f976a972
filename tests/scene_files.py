"""Writers of the demo's scene file formats for the loader tests: TGA
(uncompressed and run-length), Radiance HDR (run-length and flat), OBJ, BIN
and a JSON scene description over them, all made from seeded synthetic data."""
from __future__ import annotations

import json
import os
import struct

import numpy as np

from raydemo_b200 import scenes


def write_tga(path: str, rgba: np.ndarray, rle: bool = False, top_left: bool = False, channels: int = 4) -> None:
    """rgba: (h, w, 4) top-down. channels: 4 (BGRA), 3 (BGR) or 1 (grey from red)."""
    h, w, _ = rgba.shape
    img_type = (3 if channels == 1 else 2) + (8 if rle else 0)
    desc = (0x20 if top_left else 0) | (8 if channels == 4 else 0)
    hdr = struct.pack("<BBB5sHHHHBB", 0, 0, img_type, b"\0" * 5, 0, 0, w, h, 8 * channels, desc)
    rows = rgba if top_left else rgba[::-1]
    if channels == 1:
        px = rows[..., 0:1]
    elif channels == 3:
        px = rows[..., [2, 1, 0]]
    else:
        px = rows[..., [2, 1, 0, 3]]
    flat = [bytes(p) for p in px.reshape(-1, channels)]
    if not rle:
        body = b"".join(flat)
    else:
        out, k = [], 0
        while k < len(flat):
            run = 1
            while k + run < len(flat) and run < 128 and flat[k + run] == flat[k]:
                run += 1
            if run >= 2:
                out.append(bytes([0x80 | (run - 1)]) + flat[k])
                k += run
                continue
            raw = 1
            while k + raw < len(flat) and raw < 128 and flat[k + raw] != flat[k + raw - 1]:
                raw += 1
            out.append(bytes([raw - 1]) + b"".join(flat[k:k + raw]))
            k += raw
        body = b"".join(out)
    with open(path, "wb") as f:
        f.write(hdr + body)


def write_hdr(path: str, rgbe: np.ndarray, rle: bool = True) -> None:
    """rgbe: (h, w, 4) uint8 in file order."""
    h, w, _ = rgbe.shape
    out = [b"#?RADIANCE\n", b"FORMAT=32-bit_rle_rgbe\n", b"EXPOSURE=1.0\n", b"\n", f"-Y {h} +X {w}\n".encode()]
    if not rle:
        out.append(rgbe.tobytes())
    else:
        for y in range(h):
            out.append(bytes([2, 2, w >> 8, w & 255]))
            for ch in range(4):
                vals = rgbe[y, :, ch].tolist()
                k = 0
                while k < w:
                    run = 1
                    while k + run < w and run < 127 and vals[k + run] == vals[k]:
                        run += 1
                    if run >= 3:
                        out.append(bytes([128 + run, vals[k]]))
                        k += run
                        continue
                    raw = 1
                    while k + raw < w and raw < 128 and not (k + raw + 2 < w and vals[k + raw] == vals[k + raw + 1] == vals[k + raw + 2]):
                        raw += 1
                    out.append(bytes([raw]) + bytes(vals[k:k + raw]))
                    k += raw
    with open(path, "wb") as f:
        f.write(b"".join(out))


def _g(x) -> str:
    return "%.9g" % float(x)


def write_obj(path: str, attrs: np.ndarray, idx: np.ndarray, groups, crlf: bool = False) -> None:
    """attrs (n, 8) PxyzNxyzTuv; groups: [(name, start, count)] over idx; every
    face corner written as v/vt/vn of its own vertex."""
    nl = "\r\n" if crlf else "\n"
    lines = ["# synthetic mesh"]
    for a in attrs:
        lines.append("v " + " ".join(_g(x) for x in a[0:3]))
        lines.append("vt " + " ".join(_g(x) for x in a[6:8]))
        lines.append("vn " + " ".join(_g(x) for x in a[3:6]))
    for name, start, count in groups:
        lines.append(f"g {name}")
        for t in range(start, start + count, 3):
            lines.append("f " + " ".join(f"{i + 1}/{i + 1}/{i + 1}" for i in idx[t:t + 3]))
    with open(path, "w", newline="") as f:
        f.write(nl.join(lines) + nl)


def write_bin(path: str, attrs: np.ndarray, idx: np.ndarray, groups) -> None:
    a = np.ascontiguousarray(attrs, np.float32).reshape(-1)
    i = np.ascontiguousarray(idx, np.uint32)
    g = np.array([x for s in groups for x in s[1:3]], np.uint32)
    with open(path, "wb") as f:
        f.write(struct.pack("<III", a.size, i.size, g.size) + a.tobytes() + i.tobytes() + g.tobytes())


def make_scene_dir(root: str, seed: int = 0, env_map: bool = False) -> dict:
    """A Cornell-style scene as demo files under root: the room and boxes as an
    OBJ (one group per part), the icosphere as a BIN, TGA textures of every
    kind, every material type, a sun, instances placed with pos and rot, and a
    targeted camera. Returns the JSON dict (paths relative to root)."""
    rng = np.random.default_rng(seed)
    os.makedirs(os.path.join(root, "assets"), exist_ok=True)
    spec = scenes.cornell_box(seed)
    attrs, idx, shapes, _ = spec["meshes"][0]
    write_obj(os.path.join(root, "assets/room.obj"), attrs, idx, [(f"part{k}", s[2], s[3]) for k, s in enumerate(shapes)], crlf=True)
    sattrs, sidx, sshapes, _ = spec["meshes"][1]
    write_bin(os.path.join(root, "assets/sphere.bin"), sattrs, sidx, [("s", 0, len(sidx))])
    white = np.full((4, 4, 4), 255, np.uint8)
    write_tga(os.path.join(root, "assets/white.tga"), white, channels=3)
    noise = rng.integers(0, 256, (16, 16, 4)).astype(np.uint8)
    write_tga(os.path.join(root, "assets/noise_rle.tga"), noise, rle=True, top_left=True)
    blocks = np.repeat(np.repeat(rng.integers(0, 256, (4, 4, 4)).astype(np.uint8), 8, 0), 8, 1)
    write_tga(os.path.join(root, "assets/blocks.tga"), blocks, rle=True, channels=3)
    grey = rng.integers(0, 256, (8, 8, 4)).astype(np.uint8)
    write_tga(os.path.join(root, "assets/grey.tga"), grey, channels=1)
    nrm = np.zeros((8, 8, 4), np.uint8)
    nrm[..., 0], nrm[..., 1], nrm[..., 2], nrm[..., 3] = 128, 128, 255, 255
    nrm[::2, :, 0] = 150
    write_tga(os.path.join(root, "assets/normals.tga"), nrm, top_left=True)

    def col():
        return [float(x) for x in rng.uniform(0.2, 0.8, 3)]

    mats = {
        "floor": {"type": "diffuse", "main_texture": "assets/blocks.tga", "main_color": col(), "roughness": 0.4},
        "ceiling": {"type": "diffuse", "main_texture": "assets/white.tga", "main_color": col()},
        "back_diff": {"type": "diffuse", "main_texture": "assets/noise_rle.tga"},
        "back_gloss": {"type": "glossy", "main_texture": "assets/white.tga", "roughness": 0.2},
        "back": {"type": "mix", "main_texture": "assets/grey.tga", "strength": 0.5, "int_ior": 1.5,
                 "materials": ["back_diff", "back_gloss", "not_defined"]},
        "left": {"type": "diffuse", "main_texture": "assets/white.tga", "main_color": [0.7, 0.2, 0.2],
                 "normal_map": "assets/normals.tga"},
        "right": {"type": "glossy", "main_texture": "assets/white.tga", "main_color": [0.2, 0.7, 0.2], "roughness": 0.05},
        "tall": {"type": "refractive", "main_texture": "assets/white.tga", "roughness": 0.0, "int_ior": 1.45, "ext_ior": 1.0},
        "short": {"type": "transparent", "main_texture": "assets/white.tga", "main_color": [0.9, 0.9, 0.6]},
        "light": {"type": "emissive", "main_texture": "assets/white.tga", "strength": 15.0},
        "sphere": {"type": "diffuse", "main_texture": "assets/noise_rle.tga", "main_color": col()},
    }
    names = ["floor", "ceiling", "back", "left", "right", "tall", "short", "light"]
    env = {"sun_dir": [0.3, -1.0, 0.2], "sun_col": [1.5, 1.4, 1.2], "sun_softness": 3.0, "env_col": [0.05, 0.06, 0.08]}
    if env_map:
        rgbe = rng.integers(100, 140, (8, 16, 4)).astype(np.uint8)
        write_hdr(os.path.join(root, "assets/sky.hdr"), rgbe, rle=False)
        env["env_map"] = "assets/sky.hdr"
        env["env_clamp"] = 4.0
    js = {
        "environment": env,
        "camera": {"view_origin": [0.5, 0.55, -1.2], "view_target": [0.5, 0.45, 0.5], "fov": 42.0, "filter": "box", "srgb": False},
        "materials": mats,
        "meshes": {"room": {"vertex_data": "assets/room.obj", "materials": names},
                   "ball": {"vertex_data": "assets/sphere.bin", "materials": ["sphere"], "use_fast_bvh_build": True}},
        "mesh_instances": [{"mesh": "room"},
                           {"mesh": "ball", "pos": [0.62, 0.7, 0.3]},
                           {"mesh": "ball", "pos": [0.25, 0.45, 0.45], "rot": [30.0, 45.0, -60.0]}],
    }
    with open(os.path.join(root, "scene.json"), "w") as f:
        json.dump(js, f, indent=1)
    return js
