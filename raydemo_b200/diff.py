"""Differentiable rendering from PyTorch (RAY_MAT_PRINCIPLED albedo texture
and roughness; the reference's RAY_MAT_DIFFUSE main colour and Oren-Nayar
roughness).

`render` is a thin torch.autograd.Function over the C ABI: its forward is
`ray_render_diff` (the render loop with the parameters read from the given
tensors), its backward is the path-replay adjoint `ray_render_adjoint`. Both
run on the renderer's device, ordered on torch's current stream. torch is the
harness only (tensors, the optimiser); every pixel and gradient comes from
the library's kernels.
"""
from __future__ import annotations

import torch

from . import api

_SIDE = {}


def _enter(dev):
    """The stream the library's work goes on, ordered after torch's current
    stream: that stream itself, or (torch's legacy default stream does not
    order the library's non-blocking streams) a side stream made to wait for
    it. Returns (stream, the stream that must wait for it afterwards)."""
    cur = torch.cuda.current_stream(dev)
    if cur.cuda_stream != 0:
        return cur, None
    side = _SIDE.get(dev.index)
    if side is None:
        side = _SIDE[dev.index] = torch.cuda.Stream(dev)
    side.wait_stream(cur)
    return side, cur


def _leave(side, cur):
    if cur is not None:
        cur.wait_stream(side)


def _bind(scene, albedo, roughness, slots, rs, color):
    ah, aw = (albedo.shape[0], albedo.shape[1]) if albedo is not None else (0, 0)
    scene.set_diff_params(albedo.data_ptr() if albedo is not None else 0, aw, ah, roughness.data_ptr(), roughness.numel(), slots,
                          rs.data_ptr() if rs is not None else 0, color.data_ptr() if color is not None else 0)


class _DiffRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, roughness, color, renderer, scene, material_slot, first_iteration, samples, roughness_sampling):
        if not roughness.is_cuda or (albedo is not None and not albedo.is_cuda) or (color is not None and not color.is_cuda):
            raise ValueError("parameters must be CUDA tensors")
        albedo = albedo.detach().contiguous().float() if albedo is not None else None
        roughness = roughness.detach().contiguous().float()
        color = color.detach().contiguous().float() if color is not None else None
        if albedo is not None and (albedo.dim() != 3 or albedo.shape[2] != 3):
            raise ValueError("albedo must be (h, w, 3)")
        if color is not None and color.shape != (roughness.numel(), 3):
            raise ValueError("color must be (n_roughness, 3)")
        rs = roughness_sampling.detach().contiguous().float() if roughness_sampling is not None else None
        _bind(scene, albedo, roughness, material_slot, rs, color)
        w, h = renderer.size()
        dev = roughness.device
        image = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
        per_sample = torch.empty((samples, h, w, 3), dtype=torch.float32, device=dev)
        side, cur = _enter(dev)
        renderer.set_stream(side.cuda_stream)
        renderer.render_diff(scene, first_iteration, samples, image.data_ptr(), per_sample.data_ptr())
        _leave(side, cur)
        ctx.save_for_backward(roughness, per_sample)
        ctx.albedo, ctx.color = albedo, color
        ctx.rough_sampling = rs
        ctx.renderer, ctx.scene, ctx.slots = renderer, scene, material_slot
        ctx.first_iteration, ctx.samples = first_iteration, samples
        return image

    @staticmethod
    def backward(ctx, d_image):
        roughness, per_sample = ctx.saved_tensors
        albedo, color = ctx.albedo, ctx.color
        r, sc = ctx.renderer, ctx.scene
        # the parameters the forward pass read (the caller may have rebound them since)
        _bind(sc, albedo, roughness, ctx.slots, ctx.rough_sampling, color)
        d = d_image.detach().contiguous().float()
        g_albedo = torch.zeros_like(albedo) if albedo is not None else None
        g_rough = torch.zeros_like(roughness)
        g_color = torch.zeros_like(color) if color is not None else None
        side, cur = _enter(roughness.device)
        r.set_stream(side.cuda_stream)
        r.render_adjoint(sc, ctx.first_iteration, ctx.samples, per_sample.data_ptr(), d.data_ptr(),
                         g_albedo.data_ptr() if g_albedo is not None else 0, g_rough.data_ptr(),
                         g_color.data_ptr() if g_color is not None else 0)
        _leave(side, cur)
        return g_albedo, g_rough, g_color, None, None, None, None, None, None


def render(albedo: torch.Tensor | None, roughness: torch.Tensor, renderer: api.Renderer, scene: api.Scene, material_slot,
           first_iteration: int = 1, samples: int = 8, roughness_sampling: torch.Tensor | None = None,
           color: torch.Tensor | None = None) -> torch.Tensor:
    """The (h, w, 3) mean of `samples` samples (iterations first_iteration ..)
    of scene's current camera with the differentiable parameters albedo
    (ah, aw, 3; None when no RAY_MAT_PRINCIPLED material has a slot),
    roughness (n,) and color (n, 3: the RAY_MAT_DIFFUSE slots' main colours;
    None: the materials' own); differentiable with respect to all three.
    roughness_sampling: frozen roughness for direction sampling and pdfs."""
    return _DiffRender.apply(albedo, roughness, color, renderer, scene, material_slot, first_iteration, samples, roughness_sampling)
