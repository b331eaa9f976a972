"""Headless rendering of a scene description: the demo's JSON scene files,
read as its LoadScene reads them (raydemo_b200.load; src/DemoLib/load/
Load.cpp:22-417), rendered on the GPU through the RenderScene loop with no
window, the image written to a file.

    python -m raydemo_b200.render_scene scene.json --width 1280 --height 720 \\
        --samples 64 --out image.ppm [--raw image.npy] [--kernel wavefront]

The demo shows the renderer's tone-mapped framebuffer (get_pixels_ref) in a
window; here that framebuffer goes to a binary PPM (8 bits per channel, the
first framebuffer row first) and, with --raw, to a .npy array of its float
RGBA values. Relative file names in the scene resolve against the scene
file's directory (--base-dir overrides it), as the demo resolves them against
its working directory.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from . import api, load

KERNELS = {"auto": 0, "wavefront": 1, "path": 2}


def write_ppm(path: str, rgba: np.ndarray) -> None:
    """Binary PPM (P6) of the RGB channels of an (h, w, 4) float image in
    [0, 1], rounded to 8 bits; values outside [0, 1] are clamped."""
    h, w = rgba.shape[:2]
    rgb = np.clip(np.asarray(rgba, np.float32)[..., :3], 0.0, 1.0)
    data = np.floor(rgb * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(data).tobytes())


def render_file(scene: str, width: int, height: int, samples: int, out: str | None = None, raw: str | None = None,
                kernel: str = "auto", base_dir: str | None = None) -> tuple[np.ndarray, float]:
    """Loads `scene`, renders `samples` samples of its current camera at
    width x height, writes the requested files and returns the framebuffer
    (h, w, 4) with the rendering time in seconds (the RenderScene calls and
    the read-back)."""
    if width <= 0 or height <= 0 or samples <= 0:
        raise ValueError("width, height and samples must be positive")
    if kernel not in KERNELS:
        raise ValueError(f"kernel is one of {sorted(KERNELS)}")
    if base_dir is None:
        base_dir = os.path.dirname(os.path.abspath(scene))
    r = api.Renderer(width, height)
    sc = load.load_scene(r, scene, base_dir=base_dir)
    if sc is None:
        raise RuntimeError(f"{scene}: the scene loader rejected the description")
    r.set_kernel(KERNELS[kernel])
    r.Clear()
    reg = api.RegionContext()
    t0 = time.perf_counter()
    for _ in range(samples):
        r.RenderScene(sc, reg)
    pixels = r.get_pixels_ref()
    seconds = time.perf_counter() - t0
    if out:
        write_ppm(out, pixels)
    if raw:
        np.save(raw, pixels)
    return pixels, seconds


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description="Render a JSON scene description to an image file, without a window.")
    ap.add_argument("scene", help="the scene description (JSON)")
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--samples", type=int, default=16, help="samples per pixel (RenderScene calls)")
    ap.add_argument("--out", default="render.ppm", help="binary PPM of the tone-mapped image")
    ap.add_argument("--raw", default=None, help="also save the float RGBA framebuffer as .npy")
    ap.add_argument("--kernel", default="auto", choices=sorted(KERNELS), help="wavefront, path kernel or the faster of the two")
    ap.add_argument("--base-dir", default=None, help="directory relative file names resolve against (default: the scene's)")
    a = ap.parse_args(argv)
    _, seconds = render_file(a.scene, a.width, a.height, a.samples, a.out, a.raw, a.kernel, a.base_dir)
    print(f"{a.out}: {a.width}x{a.height}, {a.samples} samples in {seconds * 1e3:.1f} ms")
    return 0


if __name__ == "__main__":
    sys.exit(main())
