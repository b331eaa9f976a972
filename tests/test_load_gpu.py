"""Scenes read by raydemo_b200.load and rendered on the GPU against the
reference's own LoadScene (src/DemoLib/load/Load.cpp) rendered by its Ref
renderer: the same JSON scene description and files (seeded synthetic TGA,
HDR, OBJ and BIN files covering every material type, a sun, an environment
map and rotated instances) give the same image."""
import json
import os

import numpy as np
import pytest

from raydemo_b200 import api, load

from render_scenes import image_diff
from scene_files import make_scene_dir

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("env_map", [False, True], ids=["env_col", "env_map"])
def test_loaded_scene_matches_ref_renderer(reflib, cuda_device, tmp_path, env_map):
    from oracle.oracle import RefLoadedScene, RefRenderer

    if not reflib.has_loader:
        pytest.skip("the reference library was built without the demo's loader")
    root = str(tmp_path)
    js = make_scene_dir(root, 2, env_map=env_map)
    w, h, spp = 96, 72, 4
    r = api.Renderer(w, h)
    sc = load.load_scene(r, js, base_dir=root)
    assert sc is not None
    r.Clear()
    reg = api.RegionContext()
    for _ in range(spp):
        r.RenderScene(sc, reg)
    gpu = r.get_pixels_ref()
    rr = RefRenderer(reflib, w, h, RefRenderer.REF, True)
    cwd = os.getcwd()
    os.chdir(root)
    try:
        loaded = RefLoadedScene(rr, json.dumps(js))
    finally:
        os.chdir(cwd)
    assert loaded.ok
    rr.render_loaded(loaded, spp)
    d = image_diff(gpu, rr.pixels())
    print("loaded scene", d)
    assert gpu[..., :3].mean() > 0.01
    assert d["identical_px"] >= 0.9, d
    assert d["rmse"] <= 1e-3, d
    # the scene as the reference's GetCamera / GetEnvironment report it
    cam, ref_cam = sc.GetCamera(sc.current_cam()), loaded.camera()
    for k in ("origin", "fwd", "up"):
        np.testing.assert_array_equal(np.float32(getattr(cam, k)), np.float32(getattr(ref_cam, k)[:]), err_msg=k)
    assert sc.GetEnvironment()["env_map"] == loaded.environment()[2]
