"""torch_psdr_b200: B200-native differentiable path tracer with torch_psdr's Python API.

    import torch_psdr_b200 as dr
    scene = dr.Scene([dr.PerspectiveCamera(...)], [dr.Mesh(...)], [dr.AreaLight(...)])
    img = dr.PathIntegrator(spp_interior=16).renderD(scene)[0]

The renderer is the native library libpsdr_b200.so (include/psdr.h): an LBVH and
wavefront path-tracing kernels for sm_100a with a path-replay adjoint.
"""
from .api import (AreaLight, BaseCamera, BatchRender, Camera, DiffuseBsdfMaterial, DiffuseMaterial, EnvLight, Light, Material,
                  Mesh, OrthographicCamera, PathIntegrator, PerspectiveCamera, PrincipledMaterial, Scene, SH9Light,
                  Texture, VarContex)

__all__ = ["AreaLight", "BaseCamera", "BatchRender", "Camera", "DiffuseBsdfMaterial", "DiffuseMaterial", "EnvLight", "Light",
           "Material", "Mesh", "OrthographicCamera", "PathIntegrator", "PerspectiveCamera", "PrincipledMaterial",
           "Scene", "SH9Light", "Texture", "VarContex"]
