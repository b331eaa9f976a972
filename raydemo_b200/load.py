"""Scene files of the Ray demo: the JSON scene description and the files it
names (OBJ and BIN meshes; TGA, PNG, JPEG and Radiance HDR images), read into
a Scene of this library through the reference-named API.

`load_scene(renderer, js)` is LoadScene (src/DemoLib/load/Load.cpp:22-417):
the same keys, defaults, order of texture / material / mesh / instance /
camera creation and the same error behaviour -- None where the reference
returns null (its std::runtime_error cases: an unreadable texture, an unknown
filter, material or mesh type), an exception where the reference's lookup of
a missing key or name throws out of LoadScene (std::out_of_range; KeyError
here). `parse_scene` does the reading alone and returns the scene as a spec
(the dict form of raydemo_b200.scenes), so that the same scene can be handed
to any builder.

The readers restate the demo's: LoadOBJ (Load.cpp:515-634) with its vertex
merging, LoadBIN (Load.cpp:636-658), LoadHDR (Load.cpp:679-811, including its
handling of files without run-length scanlines) and Load_stb_image
(Load.cpp:813-831): stb_image with rows flipped, so the first row handed to
AddTexture is the image's bottom row. TGA (uncompressed and run-length, 8-,
24- and 32-bit, either origin) is decoded here; other formats through Pillow,
which decodes PNG exactly as stb_image does and JPEG with its own IDCT and
chroma upsampling (texel values can differ by a few units from stb_image's).

Paths in the JSON are taken as the reference takes them, relative to the
working directory, or to `base_dir` when given.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import json
import os
import struct

import numpy as np

from . import api

_F = np.float32
_TEX_BASE = 2  # a new scene holds two textures (default normal map and environment): the first added gets index 2


class LoadError(RuntimeError):
    """What LoadScene reports by returning null (its std::runtime_error cases)."""


# ---- float arithmetic as the reference's float code does it

_libm = None


def _m():
    global _libm
    if _libm is None:
        _libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
        for f in ("sinf", "cosf"):
            getattr(_libm, f).restype = ctypes.c_float
            getattr(_libm, f).argtypes = [ctypes.c_float]
        _libm.strtof.restype = ctypes.c_float
        _libm.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return _libm


def _strtof(tok: str) -> np.float32:
    """istream >> float: the decimal rounded once to float (strtof)."""
    return _F(_m().strtof(tok.encode(), None))


def _num(v) -> np.float32:
    """(float)JsNumber::val: the JSON number read as a double, then rounded to float."""
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise LoadError("expected a number")
    return _F(float(v))


def _vec3(a) -> list:
    if not isinstance(a, list):
        raise LoadError("expected an array")
    if len(a) < 3:
        raise KeyError("Index out of range!")
    return [_num(a[0]), _num(a[1]), _num(a[2])]


def _normalize(v):
    """Ren::Normalize (MVec.h:200-203): v / sqrt(Dot(v, v)), Dot summed from element 0."""
    d = v[0] * v[0]
    d = d + v[1] * v[1]
    d = d + v[2] * v[2]
    n = _F(np.sqrt(d))
    return [v[0] / n, v[1] / n, v[2] / n]


def _translate(m, v):
    """Ren::Translate (MMat.h:403-407); m: 4 columns of 4 floats."""
    c = [m[0][k] * v[0] + m[1][k] * v[1] + m[2][k] * v[2] for k in range(4)]
    res = [list(col) for col in m]
    res[3] = [m[3][k] + c[k] for k in range(4)]
    return res


def _rotate(m, angle, axis):
    """Ren::Rotate (MMat.h:409-438), cos / sin of the float angle by libm's cosf / sinf."""
    c = _F(_m().cosf(float(angle)))
    s = _F(_m().sinf(float(angle)))
    ax = _normalize([_F(x) for x in axis])
    one_c = _F(1.0) - c
    t = [one_c * ax[0], one_c * ax[1], one_c * ax[2]]
    z = _F(0.0)
    rot = [[c + t[0] * ax[0], z + t[0] * ax[1] + s * ax[2], z + t[0] * ax[2] - s * ax[1]],
           [z + t[1] * ax[0] - s * ax[2], c + t[1] * ax[1], z + t[1] * ax[2] + s * ax[0]],
           [z + t[2] * ax[0] + s * ax[1], z + t[2] * ax[1] - s * ax[0], c + t[2] * ax[2]]]
    res = []
    for j in range(3):
        res.append([m[0][k] * rot[j][0] + m[1][k] * rot[j][1] + m[2][k] * rot[j][2] for k in range(4)])
    res.append(list(m[3]))
    return res


# ---- images

def _flip(rgba: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(rgba[::-1])


def _load_tga(data: bytes) -> np.ndarray:
    """Top-down RGBA8 of a TGA file as stb_image decodes it (image types 2, 3,
    10, 11; 8-bit grey, 24-bit BGR, 32-bit BGRA; bit 5 of the descriptor
    marks a top-left origin)."""
    if len(data) < 18:
        raise LoadError("truncated TGA")
    id_len, cmap_type, img_type = data[0], data[1], data[2]
    w, h = struct.unpack_from("<HH", data, 12)
    bpp, desc = data[16], data[17]
    if cmap_type != 0 or img_type not in (2, 3, 10, 11) or w == 0 or h == 0:
        raise LoadError("unsupported TGA")
    grey = img_type in (3, 11)
    if (grey and bpp != 8) or (not grey and bpp not in (24, 32)):
        raise LoadError("unsupported TGA depth")
    comp = bpp // 8
    n = w * h
    pos = 18 + id_len
    if img_type in (2, 3):
        raw = np.frombuffer(data, np.uint8, n * comp, pos)
    else:
        out = bytearray(n * comp)
        k = 0
        while k < n:
            if pos >= len(data):
                raise LoadError("truncated TGA")
            hdr = data[pos]
            pos += 1
            cnt = (hdr & 0x7F) + 1
            if hdr & 0x80:
                px = data[pos:pos + comp]
                pos += comp
                for _ in range(min(cnt, n - k)):
                    out[k * comp:(k + 1) * comp] = px
                    k += 1
            else:
                m = min(cnt, n - k)
                out[k * comp:(k + m) * comp] = data[pos:pos + m * comp]
                pos += cnt * comp
                k += m
        raw = np.frombuffer(bytes(out), np.uint8)
    if raw.size < n * comp:
        raise LoadError("truncated TGA")
    px = raw.reshape(h, w, comp)
    rgba = np.empty((h, w, 4), np.uint8)
    if grey:
        rgba[..., 0] = rgba[..., 1] = rgba[..., 2] = px[..., 0]
        rgba[..., 3] = 255
    else:
        rgba[..., 0], rgba[..., 1], rgba[..., 2] = px[..., 2], px[..., 1], px[..., 0]
        rgba[..., 3] = px[..., 3] if comp == 4 else 255
    if not (desc >> 5) & 1:  # bottom-left origin: rows stored bottom-up
        rgba = rgba[::-1]
    return np.ascontiguousarray(rgba)


def load_image(path: str) -> np.ndarray:
    """Load_stb_image (Load.cpp:813-831): (h, w, 4) RGBA8 with the rows flipped
    (row 0 is the image's bottom row), as AddTexture receives it."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise LoadError(f"Cannot load image! {e}") from None
    if path.lower().endswith(".tga"):
        return _flip(_load_tga(data))
    try:
        from PIL import Image
    except ImportError:
        raise LoadError("Cannot load image! (Pillow is needed for formats other than TGA)") from None
    import io

    try:
        img = Image.open(io.BytesIO(data))
        img.load()
    except Exception as e:
        raise LoadError(f"Cannot load image! {e}") from None
    return _flip(np.asarray(img.convert("RGBA"), np.uint8))


def load_hdr(path: str) -> np.ndarray:
    """LoadHDR (Load.cpp:679-811): (h, w, 4) RGBE8 texels in file order. A file
    whose first unread scanline is not run-length encoded is read the
    reference's way: that pixel into texel 0, the rest of the file from texel 4
    on (texels 1-3 stay as they were)."""
    try:
        f = open(path, "rb")
    except OSError:
        raise LoadError("Is not HDR file!") from None
    with f:
        def getline():
            b = f.readline()
            return None if not b else b.decode("latin-1").rstrip("\n")

        if getline() != "#?RADIANCE":
            raise LoadError("Is not HDR file!")
        fmt = ""
        while True:
            line = getline()
            if line is None or line == "":
                break
            if line.startswith("FORMAT"):
                fmt = line[7:]
        if fmt != "32-bit_rle_rgbe":
            raise LoadError("Wrong format!")
        res = getline()
        if res is None:
            raise LoadError("Cannot read resolution!")
        tok = res.split()
        if len(tok) < 4 or tok[0] != "-Y" or tok[2] != "+X":
            raise LoadError("Unsupported format!")
        h_, w_ = _atoi(tok[1]), _atoi(tok[3])
        if not w_ or not h_:
            raise LoadError("Unsupported format!")
        data = np.zeros((w_ * h_ * 4, 4), np.uint8)
        off = 0
        left = h_
        while left:
            rgbe = f.read(4)
            if len(rgbe) < 4:
                raise LoadError("Cannot read file!")
            if rgbe[0] != 2 or rgbe[1] != 2 or (rgbe[2] & 0x80):
                data[0] = np.frombuffer(rgbe, np.uint8)
                cnt = w_ * left - 1
                rest = f.read(cnt * 4)
                if len(rest) < cnt * 4:
                    raise LoadError("Cannot read file!")
                data[4:4 + cnt] = np.frombuffer(rest, np.uint8).reshape(cnt, 4)
                return data[:w_ * h_].reshape(h_, w_, 4).copy()
            if ((rgbe[2] << 8) | rgbe[3]) != w_:
                raise LoadError("Wrong scanline width!")
            line = bytearray(w_ * 4)
            idx = 0
            for ch in range(4):
                end = (ch + 1) * w_
                while idx < end:
                    b = f.read(2)
                    if len(b) < 2:
                        raise LoadError("Cannot read file!")
                    if b[0] > 128:
                        cnt = b[0] - 128
                        if cnt == 0 or cnt > end - idx:
                            raise LoadError("Wrong data!")
                        line[idx:idx + cnt] = bytes([b[1]]) * cnt
                        idx += cnt
                    else:
                        cnt = b[0]
                        if cnt == 0 or cnt > end - idx:
                            raise LoadError("Wrong data!")
                        line[idx] = b[1]
                        idx += 1
                        cnt -= 1
                        if cnt > 0:
                            more = f.read(cnt)
                            if len(more) < cnt:
                                raise LoadError("Cannot read file!")
                            line[idx:idx + cnt] = more
                            idx += cnt
            sl = np.frombuffer(bytes(line), np.uint8).reshape(4, w_)
            data[off:off + w_] = sl.T
            off += w_
            left -= 1
        return data[:w_ * h_].reshape(h_, w_, 4).copy()


def _atoi(s: str) -> int:
    """atoi: optional sign and leading digits, 0 where there are none."""
    s = s.lstrip()
    k = 1 if s[:1] in "+-" else 0
    while k < len(s) and s[k].isdigit():
        k += 1
    try:
        return int(s[:k])
    except ValueError:
        return 0


# ---- meshes

def load_obj(path: str):
    """LoadOBJ (Load.cpp:515-634): PxyzNxyzTuv attributes (n, 8) float32,
    uint32 indices and groups (start, count pairs). Each face corner reuses
    an earlier vertex among the last 1000 whose eight values all lie within
    1e-7 of its own (the latest such), else appends one; triangles only."""
    try:
        f = open(path, "rb")
    except OSError:
        raise LoadError("File can not be opened!") from None
    v, vn, vt = [], [], []
    attrs = np.zeros((1024, 8), np.float32)
    n_attr = 0
    indices, groups = [], []
    eps = _F(0.0000001)
    with f:
        for raw in f:
            tok = raw.decode("latin-1").split()
            if not tok:
                continue
            t0 = tok[0]
            if t0 == "v" or t0 == "vn":
                vals = [_strtof(x) for x in tok[1:4]] + [_F(0.0)] * (3 - len(tok[1:4]))
                (v if t0 == "v" else vn).extend(vals)
            elif t0 == "vt":
                vals = [_strtof(x) for x in tok[1:3]] + [_F(0.0)] * (2 - len(tok[1:3]))
                vt.extend(vals)
            elif t0 == "f":
                for j in range(3):
                    parts = (tok[1 + j] if 1 + j < len(tok) else tok[-1]).split("/") + ["", ""]
                    i1, i2, i3 = _atoi(parts[0]) - 1, _atoi(parts[1]) - 1, _atoi(parts[2]) - 1
                    cand = np.array([v[i1 * 3], v[i1 * 3 + 1], v[i1 * 3 + 2], vn[i3 * 3], vn[i3 * 3 + 1], vn[i3 * 3 + 2],
                                     vt[i2 * 2], vt[i2 * 2 + 1]], np.float32)
                    found = -1
                    if n_attr:
                        lo = max(0, n_attr - 1000)
                        win = attrs[lo:n_attr]
                        ok = np.all(np.abs(win - cand) < eps, axis=1)
                        hit = np.nonzero(ok)[0]
                        if hit.size:
                            found = lo + int(hit[-1])
                    if found >= 0:
                        indices.append(found)
                    else:
                        if n_attr == attrs.shape[0]:
                            attrs = np.concatenate([attrs, np.zeros_like(attrs)])
                        attrs[n_attr] = cand
                        indices.append(n_attr)
                        n_attr += 1
            elif t0 == "g":
                if groups:
                    groups.append(len(indices) - groups[-1])
                groups.append(len(indices))
    if not groups:
        groups.append(0)
    groups.append(len(indices) - groups[-1])
    return (np.ascontiguousarray(attrs[:n_attr]), np.array(indices, np.uint32), np.array(groups, np.uint32))


def load_bin(path: str):
    """LoadBIN (Load.cpp:636-658): three uint32 counts, then the attribute
    floats, indices and groups."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError:
        raise LoadError("File can not be opened!") from None
    if len(data) < 12:
        raise LoadError("truncated mesh file")
    na, ni, ng = struct.unpack_from("<III", data, 0)
    if len(data) < 12 + 4 * (na + ni + ng):
        raise LoadError("truncated mesh file")
    attrs = np.frombuffer(data, np.float32, na, 12).reshape(-1, 8).copy()
    idx = np.frombuffer(data, np.uint32, ni, 12 + 4 * na).copy()
    grp = np.frombuffer(data, np.uint32, ng, 12 + 4 * (na + ni)).copy()
    return attrs, idx, grp


# ---- the scene description

def _path(base_dir, name: str) -> str:
    return name if base_dir is None or os.path.isabs(name) else os.path.join(base_dir, name)


def _flag(obj: dict, key: str) -> bool:
    return obj.get(key) is True


def parse_scene(js, base_dir: str | None = None) -> dict | None:
    """LoadScene's reading of a scene description (a dict, JSON text or a
    path): the scene as a spec -- textures [(rgba, srgb, mips)], materials
    (AddMaterial keywords), meshes [(attrs, indices, shapes, layout)],
    instances [(mesh, xform)], lights, env, camera (CameraDesc keywords) --
    in the reference's creation order, texture indices counted from the
    scene's two default textures. None where LoadScene returns null."""
    if isinstance(js, str) and js.lstrip().startswith("{"):
        js = json.loads(js)
    elif not isinstance(js, dict):
        with open(js, "rb") as f:
            js = json.load(f)
    spec = {"textures": [], "materials": [], "meshes": [], "instances": [], "lights": []}
    textures, materials, meshes = {}, {}, {}
    z = _F(0.0)
    view_origin, view_dir, view_up, view_target = [z, z, z], [z, z, _F(-1.0)], [z, z, z], [z, z, z]
    view_targeted = False
    fov = _F(45.0)
    filt = api.Tent
    srgb = True

    def get_texture(name: str, is_srgb: bool, mips: bool) -> int:
        if not isinstance(name, str):
            raise LoadError("expected a string")
        if name not in textures:
            if len(name) >= 3 and name[-3:].lower() == "hdr":
                data = load_hdr(_path(base_dir, name))
            else:
                data = load_image(_path(base_dir, name))
            spec["textures"].append((data, is_srgb, mips))
            textures[name] = _TEX_BASE + len(spec["textures"]) - 1
        return textures[name]

    try:
        cam = js.get("camera")
        if cam is not None:
            if "view_origin" in cam:
                view_origin = _vec3(cam["view_origin"])
            if "view_dir" in cam:
                view_dir = _vec3(cam["view_dir"])
            if "view_up" in cam:
                view_up = _vec3(cam["view_up"])
            if "view_target" in cam:
                view_target = _vec3(cam["view_target"])
                view_targeted = True
            if "fov" in cam:
                fov = _num(cam["fov"])
            if "filter" in cam:
                if cam["filter"] == "box":
                    filt = api.Box
                elif cam["filter"] == "tent":
                    filt = api.Tent
                else:
                    raise LoadError("Unknown filter parameter!")
            if "srgb" in cam:
                srgb = cam["srgb"] is True
        env = js.get("environment")
        if env is not None:
            sun_dir, sun_col = env["sun_dir"], env["sun_col"]
            e = {"env_col": (0.0, 0.0, 0.0), "env_clamp": 0.0, "env_map": 0xFFFFFFFF}
            if "env_col" in env:
                e["env_col"] = tuple(float(x) for x in _vec3(env["env_col"]))
            if "env_clamp" in env:
                e["env_clamp"] = float(_num(env["env_clamp"]))
            if "env_map" in env:
                e["env_map"] = get_texture(env["env_map"], False, False)
            spec["env"] = e
            spec["lights"].append({"type": api.DirectionalLight, "position": (0.0, 0.0, 0.0), "radius": 0.0,
                                   "direction": tuple(float(x) for x in _vec3(sun_dir)),
                                   "color": tuple(float(x) for x in _vec3(sun_col)),
                                   "angle": float(_num(env["sun_softness"])) if "sun_softness" in env else 0.0})
        for name, m in js["materials"].items():
            t = m["type"]
            d = {"main_color": (1.0, 1.0, 1.0), "normal_map": 0xFFFFFFFF, "mix_materials": [0xFFFFFFFF, 0], "roughness": 0.0,
                 "strength": 1.0, "fresnel": 1.0, "int_ior": 1.0, "ext_ior": 1.0}
            d["main_texture"] = get_texture(m["main_texture"], t != "mix", t != "mix")
            if "main_color" in m:
                d["main_color"] = tuple(float(x) for x in _vec3(m["main_color"]))
            if "normal_map" in m:
                d["normal_map"] = get_texture(m["normal_map"], False, False)
            if "roughness" in m:
                d["roughness"] = float(_num(m["roughness"]))
            elif "strength" in m:
                d["strength"] = float(_num(m["strength"]))
            for k in ("fresnel", "int_ior", "ext_ior"):
                if k in m:
                    d[k] = float(_num(m[k]))
            kinds = {"diffuse": api.DiffuseMaterial, "glossy": api.GlossyMaterial, "refractive": api.RefractiveMaterial,
                     "emissive": api.EmissiveMaterial, "mix": api.MixMaterial, "transparent": api.TransparentMaterial}
            if t not in kinds:
                raise LoadError("unknown material type")
            d["type"] = kinds[t]
            if t == "mix":
                for other in m["materials"]:
                    if other in materials:
                        if d["mix_materials"][0] == 0xFFFFFFFF:
                            d["mix_materials"][0] = materials[other]
                        else:
                            d["mix_materials"][1] = materials[other]
            d["mix_materials"] = tuple(d["mix_materials"])
            spec["materials"].append(d)
            materials[name] = len(spec["materials"]) - 1
        for name, mesh in js["meshes"].items():
            vd = mesh["vertex_data"]
            if ".obj" in vd:
                attrs, idx, groups = load_obj(_path(base_dir, vd))
            elif ".bin" in vd:
                attrs, idx, groups = load_bin(_path(base_dir, vd))
            else:
                raise LoadError("unknown mesh type")
            mats = mesh["materials"]
            shapes = []
            for i in range(0, len(groups) - 1, 2):
                if i // 2 >= len(mats):
                    raise KeyError("Index out of range!")
                mi = materials[mats[i // 2]]
                shapes.append((mi, mi, int(groups[i]), int(groups[i + 1])))
            spec["meshes"].append((attrs, idx, shapes, 0))
            meshes[name] = len(spec["meshes"]) - 1
        deg = _F(np.float32(np.pi)) / _F(180.0)
        for inst in js["mesh_instances"]:
            name = inst["mesh"]
            m = [[_F(1.0) if r == c else z for r in range(4)] for c in range(4)]
            if "pos" in inst:
                m = _translate(m, _vec3(inst["pos"]))
            if "rot" in inst:
                rx, ry, rz = (a * deg for a in _vec3(inst["rot"]))
                m = _rotate(m, rz, (0.0, 0.0, 1.0))
                m = _rotate(m, rx, (1.0, 0.0, 0.0))
                m = _rotate(m, ry, (0.0, 1.0, 0.0))
            spec["instances"].append((meshes[name], np.array(m, np.float32).reshape(-1)))
    except LoadError:
        return None
    if view_targeted:
        d = [view_origin[k] - view_target[k] for k in range(3)]
        view_dir = _normalize([-d[0], -d[1], -d[2]])
    spec["camera"] = {"type": api.Persp, "filter": filt, "dtype": api.SRGB if srgb else api.NoDevice,
                      "origin": tuple(float(x) for x in view_origin), "fwd": tuple(float(x) for x in view_dir),
                      "up": tuple(float(x) for x in view_up), "fov": float(fov), "gamma": 1.0, "focus_distance": 1.0,
                      "focus_factor": 0.0, "clamp": True}
    return spec


def build_scene(renderer: api.Renderer, spec: dict) -> api.Scene:
    """A new scene of `renderer` holding `spec`, created in its order."""
    sc = renderer.CreateScene()
    # the textures first (their indices are the ones the spec counted), then
    # the rest in the reference's order: environment and sun, materials,
    # meshes, instances, camera
    for k, (rgba, is_srgb, mips) in enumerate(spec.get("textures", [])):
        got = sc.AddTexture(rgba, is_srgb=is_srgb, generate_mipmaps=mips)
        if got != _TEX_BASE + k:
            raise RuntimeError(f"texture {k} took index {got}, not {_TEX_BASE + k}")
    if "env" in spec:
        sc.SetEnvironment(**spec["env"])
    for light in spec.get("lights", []):
        sc.AddLight(**light)
    for m in spec.get("materials", []):
        sc.AddMaterial(**m)
    for attrs, idx, shapes, layout in spec.get("meshes", []):
        sc.AddMesh(attrs, idx, shapes, layout=layout)
    for mesh, xf in spec.get("instances", []):
        sc.AddMeshInstance(mesh, xf)
    sc.set_current_cam(sc.AddCamera(api.CameraDesc(**spec["camera"])))
    return sc


def load_scene(renderer: api.Renderer, js, base_dir: str | None = None) -> api.Scene | None:
    """LoadScene (Load.cpp:22-417): a new scene of `renderer` from a scene
    description (dict, JSON text or path); None where the reference returns null."""
    spec = parse_scene(js, base_dir)
    return None if spec is None else build_scene(renderer, spec)
