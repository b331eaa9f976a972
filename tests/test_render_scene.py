"""The headless scene renderer (python -m raydemo_b200.render_scene): a JSON
scene file in, an image file out, with the same pixels as the scene loaded
and rendered through the API directly."""
import json
import os

import numpy as np
import pytest

from raydemo_b200 import render_scene


def _read_ppm(path):
    with open(path, "rb") as f:
        parts = f.read().split(b"\n", 3)
    assert parts[0] == b"P6" and parts[2] == b"255"
    w, h = (int(x) for x in parts[1].split())
    return np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


def test_ppm_writer(tmp_path):
    img = np.zeros((3, 5, 4), np.float32)
    img[0, 0, :3] = (1.0, 0.5, 0.0)
    img[2, 4, :3] = (2.0, -1.0, 0.25)  # clamped to [0, 1]
    p = str(tmp_path / "a.ppm")
    render_scene.write_ppm(p, img)
    px = _read_ppm(p)
    assert px.shape == (3, 5, 3)
    assert tuple(px[0, 0]) == (255, 128, 0)
    assert tuple(px[2, 4]) == (255, 0, 64)
    assert px[1].sum() == 0


@pytest.mark.parametrize("args", [dict(width=0, height=4, samples=1), dict(width=4, height=4, samples=0),
                                  dict(width=4, height=4, samples=1, kernel="fastest")])
def test_bad_arguments_are_rejected_before_rendering(tmp_path, args):
    with pytest.raises(ValueError):
        render_scene.render_file(str(tmp_path / "missing.json"), **args)


@pytest.mark.gpu
def test_rendered_file_equals_the_api_render(cuda_device, tmp_path):
    from raydemo_b200 import api, load

    from scene_files import make_scene_dir

    root = str(tmp_path)
    js = make_scene_dir(root, 3)
    path = os.path.join(root, "scene.json")
    with open(path, "w") as f:
        json.dump(js, f)
    w, h, spp = 80, 48, 3
    out, raw = os.path.join(root, "img.ppm"), os.path.join(root, "img.npy")
    assert render_scene.main([path, "--width", str(w), "--height", str(h), "--samples", str(spp), "--out", out,
                              "--raw", raw, "--kernel", "wavefront"]) == 0
    r = api.Renderer(w, h)
    sc = load.load_scene(r, js, base_dir=root)
    r.set_kernel(1)
    r.Clear()
    reg = api.RegionContext()
    for _ in range(spp):
        r.RenderScene(sc, reg)
    expect = r.get_pixels_ref()
    got = np.load(raw)
    assert np.array_equal(got.view(np.uint32), expect.view(np.uint32))
    assert expect[..., :3].mean() > 0.01
    px = _read_ppm(out)
    assert np.array_equal(px, np.floor(np.clip(expect[..., :3], 0, 1) * 255.0 + 0.5).astype(np.uint8))
