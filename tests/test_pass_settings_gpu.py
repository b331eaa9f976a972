"""The camera's pass settings (pass_settings_t, Types.h:39-57; SceneBase.cpp:69-83)
against the reference's Ref renderer on the scene with punctual lights and
every Ref material: lighting only, direct or indirect light skipped, no
background, and the per-kind bounce limits with early Russian roulette
(ShadeSurface's depth checks, CoreRef.cpp:2055-2391)."""
import numpy as np
import pytest

from render_scenes import image_diff, render_gpu, render_ref
from test_render_gpu import _lights_spec

pytestmark = pytest.mark.gpu

CASES = {
    "lighting_only": {"lighting_only": True},
    "skip_direct": {"skip_direct_lighting": True},
    "no_background": {"no_background": True},
    "depth_limits": {"max_diff_depth": 2, "max_glossy_depth": 1, "max_refr_depth": 2, "max_transp_depth": 1, "max_total_depth": 5,
                     "termination_start_depth": 1},
}


@pytest.mark.parametrize("case", list(CASES))
def test_pass_settings_match_ref_renderer(reflib, cuda_device, case):
    spec = _lights_spec()
    spec["camera"].update(CASES[case])
    gpu, r, _ = render_gpu(spec, 4, kernel=1)
    cpu = render_ref(reflib, spec, 4)
    d = image_diff(gpu, cpu)
    print(case, d)
    assert r.frame_info().error_flags == 0
    assert d["identical_px"] >= 0.9, d
    assert d["rmse"] <= 1e-3, d
    # the setting changes the image
    plain, _, _ = render_gpu(_lights_spec(), 4, kernel=1)
    assert not np.array_equal(plain.view(np.uint32), gpu.view(np.uint32))
