"""The C++ adapter (include/raygpu_ray.hpp): this library behind the Ray
library's RendererBase / SceneBase. On CPU: the header compiles against the
reference's own headers (every override matches a virtual of theirs). On the
GPU: oracle/_ref/adapter_check builds one scene through SceneBase calls for
the reference's Ref renderer and for this library and compares the images."""
import json
import os
import shutil
import subprocess

import pytest

from oracle.oracle import reference_src

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = reference_src() or ""
CHECK = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


def test_adapter_compiles_against_the_reference_headers(tmp_path):
    if not os.path.exists(os.path.join(REF_SRC, "Ray", "RendererBase.h")):
        pytest.skip("reference headers not present")
    cxx = os.environ.get("CXX") or shutil.which("g++")
    src = tmp_path / "use.cpp"
    src.write_text('#include "raygpu_ray.hpp"\n'
                   "std::shared_ptr<Ray::RendererBase> make(const Ray::settings_t &s) { return Ray::Gpu::CreateRenderer(s); }\n"
                   "static_assert(sizeof(ray_pixel) == sizeof(Ray::pixel_color_t), \"pixel layout\");\n"
                   "static_assert(sizeof(ray_shl1) == sizeof(Ray::shl1_data_t), \"SH layout\");\n")
    for std in ("c++11", "c++17"):
        out = subprocess.run([cxx, f"-std={std}", "-fsyntax-only", "-DDISABLE_OCL", f"-I{REF_SRC}", f"-I{ROOT}/include", str(src)],
                             capture_output=True, text=True)
        assert out.returncode == 0, out.stderr[-3000:]


def _run(w, h, iterations, mode, json_path=None, cwd=None):
    args = [CHECK, str(w), str(h), str(iterations), str(int(mode))] + ([json_path] if json_path else [])
    out = subprocess.run(args, capture_output=True, text=True, timeout=600, cwd=cwd)
    assert out.returncode == 0, out.stdout + out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


@pytest.mark.gpu
@pytest.mark.parametrize("geo", [False, True], ids=["perspective", "lightmap"])
def test_adapter_renders_as_the_ref_renderer(cuda_device, geo):
    if not os.path.exists(CHECK):
        pytest.skip("oracle/_ref/adapter_check not built")
    d = _run(96, 80, 4, geo)
    print("adapter", d)
    assert d["type"] == 64 and (d["w"], d["h"]) == (96, 80)
    assert d["tris_gpu"] == d["tris_ref"] > 0
    assert d["mean"] > 0.005
    assert d["identical_px"] >= 0.95, d
    assert d["rmse"] <= 1e-3, d
    assert d["sh"] == int(geo)


@pytest.mark.gpu
def test_demo_loader_runs_unchanged_on_the_adapter(cuda_device, tmp_path):
    """The demo's own LoadScene (src/DemoLib/load/Load.cpp, compiled from the
    reference's sources) given the GPU renderer through the adapter: its scene
    renders as the same description loaded for the Ref renderer."""
    from scene_files import make_scene_dir

    if not os.path.exists(CHECK):
        pytest.skip("oracle/_ref/adapter_check not built")
    make_scene_dir(str(tmp_path), 3, env_map=True)
    d = _run(96, 72, 3, 2, "scene.json", cwd=str(tmp_path))
    print("adapter loader", d)
    assert d["tris_gpu"] == d["tris_ref"] > 0
    assert d["mean"] > 0.005
    assert d["identical_px"] >= 0.9, d
    assert d["rmse"] <= 1e-3, d


REF_TESTS = os.path.join(ROOT, "oracle", "_ref", "ref_tests_gpu")


@pytest.mark.gpu
def test_reference_image_tests_pass_unchanged_on_the_gpu(cuda_device, tmp_path):
    """The reference's own test_mesh_lights (64x64, 2048 samples, mean 8-bit
    error <= 1.0 against its golden image, with and without SH output) and
    test_texture (256x256, 256 samples, mean |p - 0.5| <= 0.0015), compiled
    unchanged from its tree and linked with the replacement factory
    (include/raygpu_factory.cpp): every backend they loop over is the GPU
    renderer. They exit non-zero on a failed check and print OK at the end."""
    if not os.path.exists(REF_TESTS):
        pytest.skip("oracle/_ref/ref_tests_gpu not built")
    p = subprocess.run([REF_TESTS], capture_output=True, text=True, timeout=900, cwd=str(tmp_path))
    print(p.stdout[-3000:])
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert p.stdout.strip().endswith("OK")
    assert "CUDA sm_100a renderer" in p.stdout
