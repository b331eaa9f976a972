"""raydemo_b200 -- B200-native wavefront path tracer behind the Ray library's
renderer/scene interface (SerhiiY-94/RayDemo, src/Ray).

`Renderer` and `Scene` mirror Ray::RendererBase and Ray::SceneBase
(src/Ray/RendererBase.h:55-103, src/Ray/SceneBase.h:157-285) over the C ABI
in include/raygpu.h; the compute runs in libraygpu.so (sm_100a).
"""
from .api import (CameraDesc, Renderer, Scene, create_renderer, DiffuseMaterial, GlossyMaterial, RefractiveMaterial,
                  EmissiveMaterial, MixMaterial, TransparentMaterial, PointLight, SpotLight, DirectionalLight)
from .capi import RayError

__all__ = ["Renderer", "Scene", "CameraDesc", "create_renderer", "RayError", "DiffuseMaterial", "GlossyMaterial",
           "RefractiveMaterial", "EmissiveMaterial", "MixMaterial", "TransparentMaterial", "PointLight", "SpotLight",
           "DirectionalLight"]
