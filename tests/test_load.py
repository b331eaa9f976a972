"""The scene loader (raydemo_b200.load) against the reference's own loader
(src/DemoLib/load/Load.cpp, compiled into the reference library with the JSON
and TGA readers it calls): the image and mesh readers bit for bit, and whole
scene descriptions -- the camera, environment, triangle count and instance
transforms LoadScene makes, and the Ref renderer's image of our spec against
its image of LoadScene's scene. CPU only."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import reference_src

from raydemo_b200 import load

from render_scenes import build_ref
from scene_files import make_scene_dir, write_bin, write_hdr, write_obj, write_tga

# the reference's source tree (its scene files are read by one test, on CPU only)
REF_SRC_DIR = reference_src() or ""


@pytest.fixture
def loader_ref(reflib):
    if not reflib.has_loader:
        pytest.skip("the reference library was built without the demo's loader")
    return reflib


def test_tga_readers_match_stb(loader_ref, tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (13, 21, 4)).astype(np.uint8)
    img[2:6, 3:15] = img[2, 3]  # runs for the run-length packets
    for rle in (False, True):
        for top_left in (False, True):
            for ch in (1, 3, 4):
                p = str(tmp_path / f"t_{rle}_{top_left}_{ch}.tga")
                write_tga(p, img, rle=rle, top_left=top_left, channels=ch)
                ours = load.load_image(p)
                ref = loader_ref.load_image(p)
                assert ref is not None
                np.testing.assert_array_equal(ours, ref, err_msg=p)
    # the first row handed to AddTexture is the image's bottom row
    np.testing.assert_array_equal(load.load_image(str(tmp_path / "t_False_True_4.tga"))[0], img[-1])


def test_png_reader_matches_stb(loader_ref, tmp_path):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(4)
    for mode in ("RGBA", "RGB", "L"):
        arr = rng.integers(0, 256, (9, 14, 4)).astype(np.uint8)
        im = Image.fromarray(arr if mode == "RGBA" else arr[..., :3]).convert(mode)
        p = str(tmp_path / f"p_{mode}.png")
        im.save(p)
        np.testing.assert_array_equal(load.load_image(p), loader_ref.load_image(p), err_msg=mode)


def test_hdr_reader_matches_reference(loader_ref, tmp_path):
    rng = np.random.default_rng(5)
    rgbe = rng.integers(0, 256, (6, 40, 4)).astype(np.uint8)
    rgbe[:, 5:20, 3] = 130
    rgbe[:, :, 0] = np.where(rgbe[:, :, 0] == 2, 3, rgbe[:, :, 0])
    for rle in (True, False):
        p = str(tmp_path / f"h_{rle}.hdr")
        write_hdr(p, rgbe, rle=rle)
        ours = load.load_hdr(p)
        ref = loader_ref.load_image(p, hdr=True)
        np.testing.assert_array_equal(ours, ref)
        if rle:
            np.testing.assert_array_equal(ours, rgbe)
        else:  # the reference's flat read: texel 0, then the file from texel 4 on
            assert np.all(ours.reshape(-1, 4)[1:4] == 0)
    bad = str(tmp_path / "bad.hdr")
    with open(bad, "wb") as f:
        f.write(b"#?RGBE\n")
    with pytest.raises(load.LoadError):
        load.load_hdr(bad)
    assert loader_ref.load_image(bad, hdr=True) is None


def test_mesh_readers_match_reference(loader_ref, tmp_path):
    from raydemo_b200 import scenes

    spec = scenes.cornell_box(1)
    attrs, idx, shapes, _ = spec["meshes"][0]
    groups = [(f"g{k}", s[2], s[3]) for k, s in enumerate(shapes)]
    for crlf in (False, True):
        p = str(tmp_path / f"m_{crlf}.obj")
        write_obj(p, attrs, idx, groups, crlf=crlf)
        a, i, g = load.load_obj(p)
        ra, ri, rg = loader_ref.load_mesh(p)
        np.testing.assert_array_equal(a, ra)
        np.testing.assert_array_equal(i, ri)
        np.testing.assert_array_equal(g, rg)
        assert len(a) < len(idx)  # corners merged with equal earlier vertices
    # a face list without groups: one group over everything
    p = str(tmp_path / "nogroups.obj")
    write_obj(p, attrs, idx, [("x", 0, len(idx))])
    with open(p) as f:
        text = f.read().replace("g x\n", "")
    with open(p, "w") as f:
        f.write(text)
    np.testing.assert_array_equal(load.load_obj(p)[2], loader_ref.load_mesh(p)[2])
    b = str(tmp_path / "m.bin")
    write_bin(b, attrs, idx, [("a", 0, 12), ("b", 12, len(idx) - 12)])
    for x, y in zip(load.load_bin(b), loader_ref.load_mesh(b, bin=True)):
        np.testing.assert_array_equal(x, y)


def _render_both(ref, js, root, w=64, h=48, spp=2):
    from oracle.oracle import RefLoadedScene, RefRenderer

    spec = load.parse_scene(js, base_dir=root)
    assert spec is not None
    spec["size"] = (w, h)
    mine = RefRenderer(ref, w, h, RefRenderer.REF, True)
    mine.render(build_ref(ref, spec), spp, reset=True, nthreads=1)
    theirs = RefRenderer(ref, w, h, RefRenderer.REF, True)
    cwd = os.getcwd()
    os.chdir(root)
    try:
        loaded = RefLoadedScene(theirs, json.dumps(js))
    finally:
        os.chdir(cwd)
    assert loaded.ok
    theirs.render_loaded(loaded, spp)
    return spec, loaded, mine.pixels(), theirs.pixels()


@pytest.mark.parametrize("env_map", [False, True], ids=["env_col", "env_map"])
def test_scene_matches_reference_loadscene(loader_ref, tmp_path, env_map):
    root = str(tmp_path)
    js = make_scene_dir(root, 0, env_map=env_map)
    spec, loaded, a, b = _render_both(loader_ref, js, root)
    cam = loaded.camera()
    c = spec["camera"]
    assert cam.type == c["type"] and cam.filter == c["filter"] and cam.dtype == c["dtype"] and cam.clamp == 1
    for k in ("origin", "fwd"):
        np.testing.assert_array_equal(np.float32(getattr(cam, k)[:]), np.float32(c[k]), err_msg=k)
    # GetCamera reports the constructed (orthonormalised) up
    from oracle.oracle import Oracle

    built = Oracle().construct_camera(c["origin"], c["fwd"], c["up"], c["fov"])
    np.testing.assert_array_equal(np.float32(cam.up[:]), np.float32(built.up[:]))
    assert np.float32(cam.fov) == np.float32(c["fov"])
    col, clamp, env_idx = loaded.environment()
    np.testing.assert_array_equal(col, np.float32(spec["env"]["env_col"]))
    assert np.float32(clamp) == np.float32(spec["env"]["env_clamp"])
    # SetEnvironment stores the scene's default environment texture (its first texture) for "none"
    assert env_idx == (spec["env"]["env_map"] if spec["env"]["env_map"] != 0xFFFFFFFF else 0)
    assert loaded.triangle_count() == sum(len(m[1]) // 3 for m in spec["meshes"])
    xf = loaded.instance_xforms()
    assert len(xf) == len(spec["instances"])
    for (_, ours), theirs in zip(spec["instances"], xf):
        np.testing.assert_array_equal(ours, theirs)  # pos and rot, bit for bit
    assert a.mean() > 0.01
    np.testing.assert_array_equal(a, b)  # the same scene, so the same image


def test_loader_errors_as_reference(loader_ref, tmp_path):
    from oracle.oracle import RefLoadedScene, RefRenderer

    root = str(tmp_path)
    base = make_scene_dir(root, 1)
    rr = RefRenderer(loader_ref, 16, 16, RefRenderer.REF, True)
    cwd = os.getcwd()

    def theirs(js):
        os.chdir(root)
        try:
            return RefLoadedScene(rr, json.dumps(js)).ok
        finally:
            os.chdir(cwd)

    # null where LoadScene returns null: unknown material type, unreadable texture, unknown mesh type, unknown filter
    cases = []
    j = json.loads(json.dumps(base))
    j["materials"]["floor"]["type"] = "velvet"
    cases.append(j)
    j = json.loads(json.dumps(base))
    j["materials"]["floor"]["main_texture"] = "assets/missing.tga"
    cases.append(j)
    j = json.loads(json.dumps(base))
    j["meshes"]["ball"]["vertex_data"] = "assets/sphere.ply"
    cases.append(j)
    j = json.loads(json.dumps(base))
    j["camera"]["filter"] = "gauss"
    cases.append(j)
    for j in cases:
        assert load.parse_scene(j, base_dir=root) is None
        assert not theirs(j)
    # a missing required key or name throws out of LoadScene (std::out_of_range)
    j = json.loads(json.dumps(base))
    del j["mesh_instances"]
    with pytest.raises(KeyError):
        load.parse_scene(j, base_dir=root)
    j = json.loads(json.dumps(base))
    j["mesh_instances"][1]["mesh"] = "nothing"
    with pytest.raises(KeyError):
        load.parse_scene(j, base_dir=root)
    assert theirs(base)


def test_reference_scene_file(loader_ref):
    """The reference's own scene description assets/scenes/sponza_simple.json
    (its BIN mesh and JPEG textures), read here and by LoadScene: the same
    camera, triangle count and instance transforms; the JPEG texels (Pillow's
    decoder, not stb_image's) within 3 units of the reference's, so the Ref
    renderer's images of the two scenes agree to the texture differences."""
    import time

    from oracle.oracle import RefLoadedScene, RefRenderer

    root = os.path.join(os.path.dirname(REF_SRC_DIR), "assets")
    path = os.path.join(root, "scenes", "sponza_simple.json")
    if not os.path.exists(path):
        pytest.skip("the reference's assets are not present")
    base = os.path.dirname(root)
    with open(path) as f:
        js = json.load(f)
    spec = load.parse_scene(js, base_dir=base)
    assert spec is not None
    for m in js["materials"].values():
        name = m["main_texture"]
        ours = load.load_image(os.path.join(base, name))
        theirs = loader_ref.load_image(os.path.join(base, name))
        d = np.abs(ours.astype(int) - theirs.astype(int))
        assert d.max() <= 3 and (d > 0).mean() < 0.05, name
    w, h = 48, 36
    spec["size"] = (w, h)
    mine = RefRenderer(loader_ref, w, h, RefRenderer.REF, True)
    mine.render(build_ref(loader_ref, spec), 1, nthreads=8)
    theirs = RefRenderer(loader_ref, w, h, RefRenderer.REF, True)
    cwd = os.getcwd()
    os.chdir(base)
    try:
        loaded = RefLoadedScene(theirs, json.dumps(js))
    finally:
        os.chdir(cwd)
    assert loaded.ok
    assert loaded.triangle_count() == sum(len(m[1]) // 3 for m in spec["meshes"])
    for (_, x), y in zip(spec["instances"], loaded.instance_xforms()):
        np.testing.assert_array_equal(x, y)
    cam = loaded.camera()
    np.testing.assert_array_equal(np.float32(cam.origin[:]), np.float32(spec["camera"]["origin"]))
    np.testing.assert_array_equal(np.float32(cam.fwd[:]), np.float32(spec["camera"]["fwd"]))
    theirs.render_loaded(loaded, 1, 8)
    a, b = mine.pixels()[..., :3].astype(np.float64), theirs.pixels()[..., :3]
    assert a.mean() > 0.05
    assert np.sqrt(np.mean((a - b) ** 2)) <= 0.02
