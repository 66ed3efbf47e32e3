"""PyTorch API of the B200 path tracer: a drop-in for torch_psdr's Python surface.

Mirrors src/python/torch_psdr.py (class names, constructor arguments, asserts and
the renderC / renderD contract). Tensors are borrowed as CUDA buffers and handed to
the native library through the C ABI; the only PyTorch machinery is the
torch.autograd.Function below, whose forward calls psdr_render_fwd and whose backward
calls psdr_render_bwd (the path-replay adjoint).
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import List, Optional, Union

import torch
from torch import Tensor

from . import _lib as L
from . import synth


def _dev_tensor(t: Tensor, dtype) -> Tensor:
    if not isinstance(t, Tensor):
        t = torch.as_tensor(t)
    if not t.is_cuda:
        raise ValueError("torch_psdr_b200 renders on the GPU: tensors must be CUDA tensors")
    return t.detach().to(dtype).contiguous().clone()


def check_indices(idx: Tensor, n: int, what: str) -> None:
    """Every entry of the index buffer idx must lie in [0, n): the native kernels gather
    vertices and uvs through these buffers without bounds checks (as the reference's
    gathers do), so an out-of-range index would read outside the buffer. One device
    reduction and one host read; empty buffers are left to the library's own check."""
    if idx.numel() == 0:
        return
    lo, hi = torch.stack([idx.min(), idx.max()]).tolist()
    if lo < 0 or hi >= n:
        raise ValueError(f"{what} must lie in [0, {n}): found values in [{lo}, {hi}]")


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _host3(t: Tensor):
    v = t.detach().reshape(-1).float().cpu().tolist()
    return (C.c_float * 3)(*v[:3])


class VarContex:
    """Collects the tensors that require grad, in the order torch_psdr.py:84-103 does."""

    def __init__(self):
        self.torch_vars: List[Tensor] = []

    def append_variable(self, torch_var: Tensor):
        if isinstance(torch_var, Tensor) and torch_var.requires_grad:
            self.torch_vars.append(torch_var)

    def merge_variables(self, torch_vars):
        for t in torch_vars:
            if t.requires_grad:
                self.torch_vars.append(t)

    def get_variables(self):
        return self.torch_vars


class BaseCamera(VarContex):
    """Base class of PerspectiveCamera and OrthographicCamera (torch_psdr.py:106-110)."""


class PerspectiveCamera(BaseCamera):
    def __init__(self, look_from: Tensor, look_at: Tensor, up: Tensor, vfov: Tensor, height: int, width: int):
        """Pinhole camera (torch_psdr.py:113-158; camera.h:208-277).

        Args:
            look_from: (3,) camera position.  look_at: (3,) target.  up: (3,) up vector.
            vfov: (1,) vertical field of view in radians.  height, width: image size.
        """
        super().__init__()
        assert look_from.size() == (3,)
        assert look_at.size() == (3,)
        assert up.size() == (3,)
        assert vfov.size() == (1,)
        assert height > 0 and width > 0
        self.look_from, self.look_at, self.up, self.vfov = look_from, look_at, up, vfov
        for t in (look_from, look_at, up, vfov):
            self.append_variable(t)
        self.height = int(height)
        self.width = int(width)

    def _desc(self):
        d = L.CameraDesc()
        d.type = L.CAM_PERSPECTIVE
        d.look_from = _host3(self.look_from)
        d.look_at = _host3(self.look_at)
        d.up = _host3(self.up)
        d.fov = float(self.vfov.detach().reshape(-1)[0].item())
        d.height, d.width = self.height, self.width
        return d


Camera = PerspectiveCamera  # example/optimize_texture.py:76 uses dr.Camera


class OrthographicCamera(BaseCamera):
    def __init__(self, look_from, look_at, up, view_width, height: int, width: int):
        """Orthographic camera (torch_psdr.py:161-206; camera.h:279-353): parallel rays
        along the view direction from a view box view_width wide and view_width * height /
        width high."""
        super().__init__()
        assert look_from.size() == (3,)
        assert look_at.size() == (3,)
        assert up.size() == (3,)
        assert view_width.size() == (1,)
        assert height > 0 and width > 0
        self.look_from, self.look_at, self.up, self.view_width = look_from, look_at, up, view_width
        self.vfov = view_width  # the lens parameter slot shared with PerspectiveCamera
        for t in (look_from, look_at, up, view_width):
            self.append_variable(t)
        self.height = int(height)
        self.width = int(width)

    def _desc(self):
        d = L.CameraDesc()
        d.type = L.CAM_ORTHOGRAPHIC
        d.look_from = _host3(self.look_from)
        d.look_at = _host3(self.look_at)
        d.up = _host3(self.up)
        d.fov = float(self.view_width.detach().reshape(-1)[0].item())
        d.height, d.width = self.height, self.width
        return d


class Texture(VarContex):
    def __init__(self, tex: Tensor):
        """Constant (1,)/(3,) or image (H,W,1)/(H,W,3) texture (torch_psdr.py:209-269).

        The image keeps the caller's row order; the library applies the row flip of
        torch_psdr.py:250 when it indexes (nearest texel, texture.h:65-74).
        """
        super().__init__()
        tex_type = None
        size = tuple(tex.size())
        if tex.dim() == 1:
            if size == (1,):
                tex_type = "Constant1f"
            elif size == (3,):
                tex_type = "Constant3f"
        elif tex.dim() == 2:
            # torch_psdr.py:232-234 tests `tex_type == "UV1f"` (a comparison, not an
            # assignment), so a (H, W) texture fails its assert; kept as is.
            pass
        elif tex.dim() == 3:
            if size[-1] == 1:
                tex_type = "UV1f"
            elif size[-1] == 3:
                tex_type = "UV3f"
        assert tex_type is not None
        self.tex_type = tex_type
        self.tensor = tex
        self.append_variable(tex)
        self.data = _dev_tensor(tex, torch.float32)

    def _desc(self):
        d = L.TextureDesc()
        if self.tex_type.startswith("Constant"):
            d.kind = L.TEX_CONSTANT
            d.channels = 1 if self.tex_type == "Constant1f" else 3
            d.height = d.width = 1
        else:
            d.kind = L.TEX_UV
            d.height, d.width = int(self.data.shape[0]), int(self.data.shape[1])
            d.channels = int(self.data.shape[2])
        d.data = self.data.data_ptr()
        return d


class Material(VarContex):
    """Base class of the materials (torch_psdr.py:272-277)."""


class DiffuseMaterial(Material):
    def __init__(self, tex: Union[Tensor, Texture]):
        """Lambertian reflectance (torch_psdr.py:280-295; diffuse_material.cc:3-45)."""
        super().__init__()
        if isinstance(tex, Tensor):
            tex = Texture(tex)
        assert tex.tex_type == "Constant3f" or tex.tex_type == "UV3f"
        self.texture = tex
        self.roughness = None
        self.normal = None
        self.merge_variables(tex.get_variables())
        self.mat_type = L.MAT_DIFFUSE


class DiffuseBsdfMaterial(Material):
    def __init__(self, color, roughness, normal=None):
        """Lambertian / Oren-Nayar diffuse reflection (torch_psdr.py:298-335;
        diffuse_bsdf.cc:3-88): color (3,) or (H,W,3), roughness (1,) or (H,W,1) (0 is
        Lambertian), normal (3,) or (H,W,3) shading normals in the (tangent,
        normal x tangent, normal) frame, 0.5 + n/2 per channel; None = geometric normal."""
        super().__init__()
        if isinstance(color, Tensor):
            color = Texture(color)
        if isinstance(roughness, Tensor):
            roughness = Texture(roughness)
        if isinstance(normal, Tensor):
            normal = Texture(normal)
        assert color.tex_type == "Constant3f" or color.tex_type == "UV3f"
        assert roughness.tex_type == "Constant1f" or roughness.tex_type == "UV1f"
        assert normal is None or normal.tex_type == "Constant3f" or normal.tex_type == "UV3f"
        self.texture = color
        self.roughness = roughness
        self.normal = normal
        self.merge_variables(color.get_variables())
        self.merge_variables(roughness.get_variables())
        if normal is not None:
            self.merge_variables(normal.get_variables())
        self.mat_type = L.MAT_DIFFUSE_BSDF


class PrincipledMaterial(Material):
    pass


class Mesh(VarContex):
    def __init__(self, vertices: Tensor, uvs, face_indices: Tensor, uv_indices, material: Material):
        """Triangle mesh with its material (torch_psdr.py:343-379; mesh.cc:5-95)."""
        super().__init__()
        assert vertices.dim() == 2 and vertices.size(-1) == 3
        assert uvs is None or (uvs.dim() == 2 and uvs.size(-1) == 2)
        assert face_indices.dim() == 2 and face_indices.size(-1) == 3
        assert uv_indices is None or (uv_indices.dim() == 2 and uv_indices.size(-1) == 3)
        assert uvs is None or uv_indices is None or uv_indices.size(0) == face_indices.size(0)
        self.vertices = vertices
        self.v = _dev_tensor(vertices, torch.float32)
        self.f = _dev_tensor(face_indices, torch.int32)
        check_indices(self.f, self.v.shape[0], "face_indices")
        no_uvs = uvs is None or uv_indices is None
        self.uv = None if no_uvs else _dev_tensor(uvs, torch.float32)
        self.uvi = None if no_uvs else _dev_tensor(uv_indices, torch.int32)
        if self.uvi is not None:
            check_indices(self.uvi, self.uv.shape[0], "uv_indices")
        self.material = material
        self.append_variable(vertices)
        self.merge_variables(material.get_variables())

    def set_vertices(self, vertices: Tensor):
        """Copy new vertex positions (same count) into the buffer the native scene reads
        when it rebuilds (psdr_scene_update, or the forward graph of a BatchRender); the
        given tensor becomes the one that receives the vertex gradient."""
        assert tuple(vertices.shape) == tuple(self.v.shape)
        self.v.copy_(vertices.detach())
        self.vertices = vertices

    def get_variables(self):
        out = [self.vertices] if self.vertices.requires_grad else []
        return out + self.material.get_variables()

    def _desc(self):
        d = L.MeshDesc()
        d.vertices, d.num_vertices = self.v.data_ptr(), int(self.v.shape[0])
        d.faces, d.num_faces = self.f.data_ptr(), int(self.f.shape[0])
        if self.uv is not None:
            d.uvs, d.num_uvs, d.uv_indices = self.uv.data_ptr(), int(self.uv.shape[0]), self.uvi.data_ptr()
        d.material = self.material.mat_type
        d.color = self.material.texture._desc()
        none = L.TextureDesc(L.TEX_NONE, 0, 0, 0, None)
        d.roughness = self.material.roughness._desc() if self.material.roughness is not None else none
        d.normal = self.material.normal._desc() if self.material.normal is not None else none
        return d


class Light(VarContex):
    """Base class of the lights (torch_psdr.py:382-385)."""


class AreaLight(Light):
    def __init__(self, vertices: Tensor, face_indices: Tensor, emit: Tensor):
        """Triangle-mesh emitter with constant radiance (torch_psdr.py:388-414; emitter.cc:4-92)."""
        super().__init__()
        assert vertices.dim() == 2 and vertices.size(-1) == 3
        assert face_indices.dim() == 2 and face_indices.size(-1) == 3
        assert emit.dim() == 1 and emit.size(0) == 3
        self.vertices, self.emit = vertices, emit
        self.v = _dev_tensor(vertices, torch.float32)
        self.f = _dev_tensor(face_indices, torch.int32)
        check_indices(self.f, self.v.shape[0], "face_indices")
        self.append_variable(vertices)
        self.append_variable(emit)

    def _desc(self):
        d = L.AreaLightDesc()
        d.vertices, d.num_vertices = self.v.data_ptr(), int(self.v.shape[0])
        d.faces, d.num_faces = self.f.data_ptr(), int(self.f.shape[0])
        d.emit = _host3(self.emit)
        return d


class EnvLight(Light):
    def __init__(self, cube_map: Texture):
        """Cube-map environment light (torch_psdr.py:417-430; emitter.cc:94-141): an
        emissive box around the scene, 1000 times its size (scene.cc:31-49), showing the
        cube map laid out as a 4 x 3 cross."""
        super().__init__()
        assert cube_map.tex_type == "UV3f"
        self.cube_map = cube_map
        self.merge_variables(cube_map.get_variables())
        self.vertices = self.v = self.emit = None
        self.params, self.params_data = cube_map.tensor, cube_map.data

    def _desc(self, box):
        d = L.AreaLightDesc()
        d.type = L.LIGHT_ENV
        d.cube_map = self.cube_map._desc()
        d.box_min, d.box_max = (C.c_float * 3)(*map(float, box[0])), (C.c_float * 3)(*map(float, box[1]))
        return d


class SH9Light(Light):
    def __init__(self, sh9_coeff: Tensor):
        """Second-order spherical-harmonics light (torch_psdr.py:433-447;
        emitter.cc:206-283): the same box as EnvLight, emitting sum_k c_k Y_k(wi) of the
        incoming direction wi at its hit point. sh9_coeff: (9, 3)."""
        super().__init__()
        assert sh9_coeff.size() == (9, 3)
        self.sh9_coeff = sh9_coeff
        self.append_variable(sh9_coeff)
        self.vertices = self.v = self.emit = None
        self.params = sh9_coeff
        self.params_data = torch.zeros((9, 3), dtype=torch.float32, device="cuda")

    def _desc(self, box):
        d = L.AreaLightDesc()
        d.type = L.LIGHT_SH9
        d.sh9 = (C.c_float * 27)(*self.sh9_coeff.detach().reshape(-1).cpu().tolist())
        d.box_min, d.box_max = (C.c_float * 3)(*map(float, box[0])), (C.c_float * 3)(*map(float, box[1]))
        return d


def _is_env(light):
    return isinstance(light, (EnvLight, SH9Light))


class Scene(VarContex):
    def __init__(self, cameras: List[BaseCamera], meshes: List[Mesh], lights: List[Light]):
        """Cameras, meshes and lights (torch_psdr.py:450-474). Builds the native scene
        (triangle records, edge list, sampling CDFs, LBVH) on the current stream."""
        super().__init__()
        self.cameras = list(cameras)
        self.meshes = list(meshes)
        # scene.cc:15-53: one environment light, appended after the other lights around the
        # box of the camera positions and mesh vertices (self.lights keeps that order)
        env = [lt for lt in lights if _is_env(lt)]
        assert len(env) <= 1, "only support no more than one env_light"
        self.lights = [lt for lt in lights if not _is_env(lt)] + env
        box = None
        if env:
            box = synth.env_box([c.look_from.detach().cpu().numpy() for c in self.cameras],
                                [m.v.detach().cpu().numpy() for m in self.meshes])
        lib = L.load()
        md = (L.MeshDesc * max(1, len(self.meshes)))(*[m._desc() for m in self.meshes])
        ld = (L.AreaLightDesc * max(1, len(self.lights)))(*[lt._desc(box) if _is_env(lt) else lt._desc()
                                                            for lt in self.lights])
        desc = L.SceneDesc(md, len(self.meshes), ld, len(self.lights))
        handle = C.c_void_p()
        L.check(lib.psdr_scene_create(C.byref(desc), _stream(), C.byref(handle)), "psdr_scene_create")
        self._handle = handle
        self._lib = lib

    @property
    def handle(self):
        return self._handle

    def get_variables(self):
        """Tensors requiring grad, cameras then meshes then lights (torch_psdr.py:469-471)."""
        out = []
        for part in self.cameras + self.meshes + self.lights:
            out += [t for t in part.get_variables() if t.requires_grad]
        return out

    def info(self):
        out = (C.c_int64 * 6)()
        L.check(self._lib.psdr_scene_info(self._handle, out), "psdr_scene_info")
        return dict(zip(["triangles", "vertices", "edges", "bvh_nodes", "lights", "objects"], list(out)))

    def update(self, refit: bool = False):
        """Rebuild triangle records, edges, CDFs and the BVH after Mesh.set_vertices.
        refit=True keeps the BVH's tree and recomputes only its boxes (same hits; for small
        vertex moves between full rebuilds)."""
        if refit:
            L.check(self._lib.psdr_scene_refit(self._handle, _stream()), "psdr_scene_refit")
        else:
            L.check(self._lib.psdr_scene_update(self._handle, _stream()), "psdr_scene_update")

    def _camera_descs(self):
        return (L.CameraDesc * len(self.cameras))(*[c._desc() for c in self.cameras])

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                self._lib.psdr_scene_destroy(h)
            except Exception:
                pass
            self._handle = None


class _RenderD(torch.autograd.Function):
    """Replaces Wrap2torch (torch_psdr.py:29-72): forward renders, backward runs the
    path-replay adjoint and returns the gradient of every input tensor."""

    @staticmethod
    def forward(ctx, integrator, scene, *torch_vars):
        imgs = integrator._render(scene)
        ctx.integrator = integrator
        ctx.scene = scene
        ctx.n_vars = len(torch_vars)
        ctx.vars = torch_vars
        return tuple(imgs)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, *grads):
        grads = [g if g is not None else None for g in grads]
        out = ctx.integrator._backward(ctx.scene, grads, ctx.vars)
        return (None, None) + tuple(out)


def _grad_buf(param, internal):
    """Zeroed gradient buffer shaped like `internal`, or None when `param` does not
    require grad."""
    if isinstance(param, Tensor) and param.requires_grad:
        return torch.zeros_like(internal)
    return None


def _tex_grad(tex):
    """Gradient buffer of an optional Texture (None when absent or not requiring grad)."""
    return None if tex is None else _grad_buf(tex.tensor, tex.data)


def _ptrs(bufs):
    """ctypes pointer array of optional tensors (at least one entry)."""
    P = C.c_void_p
    return (P * max(1, len(bufs)))(*[None if t is None else t.data_ptr() for t in bufs])


def _wants(t) -> bool:
    return isinstance(t, Tensor) and t.requires_grad


def _lens_buf(cam, unbiased: bool):
    """(10,) camera-lens gradient buffer (look_from through the basis, look_at, up, fov), or
    None when no camera parameter that enters the basis or the projection requires grad.
    With the unbiased estimator look_from needs it too: moving look_from with look_at fixed
    turns the camera. Orthographic cameras have no lens gradient: their look_at, up and
    view_width gradients are refused rather than returned as zeros."""
    lens_params = (cam.look_at, cam.up, cam.vfov)
    if isinstance(cam, OrthographicCamera):
        if any(_wants(t) for t in lens_params):
            raise NotImplementedError("gradients of an OrthographicCamera's look_at, up and view_width are not "
                                      "implemented; only look_from (with the camera's basis held fixed)")
        return None
    if any(_wants(t) for t in lens_params) or (unbiased and _wants(cam.look_from)):
        return torch.zeros(10, dtype=torch.float32, device="cuda")
    return None


def _add_camera_grads(add, cam, origin_g, lens_g):
    """Map a camera's origin gradient (basis fixed) and its lens gradient onto its tensors."""
    if lens_g is None:
        add(cam.look_from, origin_g)
        return
    add(cam.look_from, origin_g + lens_g[0:3])
    add(cam.look_at, lens_g[3:6])
    add(cam.up, lens_g[6:9])
    add(cam.vfov, lens_g[9:10])


class PathIntegrator:
    def __init__(self, enable_light_visable: bool = False, n_pass: int = 1, spp_interior: int = 1,
                 max_bounce: int = 3, mis_light_samples: int = 1, mis_bsdf_samples: int = 1,
                 spp_primary_edge: int = 1, spp_secondary_edge: int = 1, primary_edge_preprocess_rounds: int = 1,
                 secondary_edge_preprocess_rounds: int = 1, primary_edge_hypercube_resolution: int = 10000,
                 secondary_edge_hypercube_resolution: List[int] = [10000, 6, 6], estimator: str = "reference",
                 seed: int = 0, tile_paths: int = 0, gradient_terms: int = 0,
                 spp_pixel_boundary: Optional[int] = None, trace_queue: int = 0, batch_lanes: int = 0,
                 batch_records: int = 0):
        """Path-space differentiable integrator (torch_psdr.py:477-536; path_integrator.h:8-21).

        B200 extensions: estimator ("reference" reproduces renderD exactly; "unbiased"
        is the derivative of the rendered image: material-form interior term plus
        pixel-border, silhouette and shadow-boundary terms), seed (0 = the reference's
        sample streams), tile_paths (wavefront tile, 0 = automatic), gradient_terms
        (bitmask: 1 interior, 2 primary edges, 4 direct edges, 8 pixel borders, 16
        DiffuseBsdfMaterial BRDF jumps, 32 interpenetration creases, 64 indirect shadow
        boundaries; 0 = all that apply: bits 8-64 with the unbiased estimator only, bit 16
        when a DiffuseBsdfMaterial mesh is in the scene),
        spp_pixel_boundary (unbiased: samples per unit pixel-border segment; default
        spp_primary_edge), trace_queue (rays each SM traverses concurrently, in units of
        128; 0 = 8, the autotuner picks it), batch_lanes (BatchRender only: concurrent
        streams, each with its own workspace, over which a batch spreads its forward tiles
        and its backward's interior tiles and per-view boundary terms; 1..8, 0 = 4; the
        gradients do not depend on it), batch_records (BatchRender only: the forward keeps
        every interior path's replay record and the backward runs the adjoint from them
        instead of re-tracing; 0 = when they fit in a quarter of the free device memory,
        1 = always, -1 = never; the gradients do not depend on it).
        """
        assert n_pass > 0
        assert spp_interior > 0
        assert spp_primary_edge > 0
        assert spp_secondary_edge > 0
        assert max_bounce > 0
        assert mis_light_samples >= 0
        assert mis_bsdf_samples >= 0
        assert primary_edge_preprocess_rounds > 0
        assert secondary_edge_preprocess_rounds > 0
        assert primary_edge_hypercube_resolution > 0
        assert len(secondary_edge_hypercube_resolution) == 3
        for reso in secondary_edge_hypercube_resolution:
            assert reso > 0
        assert estimator in ("reference", "unbiased")
        cfg = L.Config()
        cfg.n_pass = n_pass
        cfg.spp_interior = spp_interior
        cfg.enable_light_visable = int(bool(enable_light_visable))
        cfg.spp_primary_edge = spp_primary_edge
        cfg.spp_secondary_edge = spp_secondary_edge
        cfg.max_bounce = max_bounce
        cfg.mis_light_samples = mis_light_samples
        cfg.mis_bsdf_samples = mis_bsdf_samples
        cfg.primary_edge_preprocess_rounds = primary_edge_preprocess_rounds
        cfg.secondary_edge_preprocess_rounds = secondary_edge_preprocess_rounds
        cfg.primary_edge_hypercube_resolution = primary_edge_hypercube_resolution
        cfg.secondary_edge_hypercube_resolution = (C.c_int32 * 3)(*secondary_edge_hypercube_resolution)
        cfg.estimator = L.EST_REFERENCE if estimator == "reference" else L.EST_UNBIASED
        cfg.tile_paths = tile_paths
        cfg.terms = gradient_terms
        cfg.spp_pixel_boundary = spp_primary_edge if spp_pixel_boundary is None else spp_pixel_boundary
        assert cfg.spp_pixel_boundary >= 0
        cfg.seed = seed
        assert 0 <= trace_queue <= 8
        cfg.trace_queue = trace_queue
        assert 0 <= batch_lanes <= 8
        cfg.batch_lanes = batch_lanes
        assert batch_records in (-1, 0, 1)
        cfg.batch_records = batch_records
        self.cfg = cfg
        self._lib = L.load()
        self._ws = None

    def _workspace(self):
        if self._ws is None:
            h = C.c_void_p()
            L.check(self._lib.psdr_workspace_create(C.byref(h)), "psdr_workspace_create")
            self._ws = h
        return self._ws

    def __del__(self):
        if getattr(self, "_ws", None) is not None:
            try:
                self._lib.psdr_workspace_destroy(self._ws)
            except Exception:
                pass

    def _render(self, scene: Scene) -> List[Tensor]:
        imgs = [torch.empty((c.height, c.width, 3), dtype=torch.float32, device="cuda") for c in scene.cameras]
        ptrs = (C.c_void_p * len(imgs))(*[i.data_ptr() for i in imgs])
        cams = scene._camera_descs()
        L.check(self._lib.psdr_render_fwd(scene.handle, self._workspace(), cams, len(imgs), C.byref(self.cfg),
                                          ptrs, _stream()), "psdr_render_fwd")
        return imgs

    def autotune(self, scene: Scene, cache: Optional[str] = None) -> dict:
        """Pick the wavefront tile size and the scene's BVH leaf size by timing forward
        renders of the scene's cameras (psdr_autotune); the integrator keeps the tile
        size, the scene keeps the leaf size. Extension: the reference has no tuner.

        cache: path of a JSON file of earlier results, keyed by the GPU (name, SM count)
        and the job's shape (triangles, view sizes, spp, depth, light and BSDF samples,
        estimator). A hit applies the stored sizes without timing (and returns them with
        "cached": True); a miss tunes and adds its result to the file."""
        key = self._tune_key(scene) if cache else None
        if key is not None and os.path.exists(cache):
            with open(cache) as f:
                entry = json.load(f).get(key)
            if entry is not None:
                self._apply_tuning(scene, entry)
                return dict(entry, cached=True)
        entry = self._autotune_native(scene)
        if key is not None:
            table = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    table = json.load(f)
            table[key] = entry
            tmp = cache + ".tmp"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        return entry

    def _autotune_native(self, scene: Scene) -> dict:
        leaf = C.c_int32()
        ms = C.c_float()
        cams = scene._camera_descs()
        L.check(self._lib.psdr_autotune(scene.handle, self._workspace(), cams, len(cams), C.byref(self.cfg),
                                        C.byref(leaf), C.byref(ms), _stream()), "psdr_autotune")
        return {"tile_paths": int(self.cfg.tile_paths), "leaf_size": int(leaf.value),
                "trace_queue": int(self.cfg.trace_queue), "forward_ms": float(ms.value)}

    def _apply_tuning(self, scene: Scene, entry: dict) -> None:
        self.cfg.tile_paths = int(entry["tile_paths"])
        self.cfg.trace_queue = int(entry.get("trace_queue", 0))
        L.check(self._lib.psdr_scene_set_leaf_size(scene.handle, int(entry["leaf_size"]), _stream()),
                "psdr_scene_set_leaf_size")

    @staticmethod
    def _gpu_id() -> dict:
        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        return {"gpu": p.name, "sms": int(p.multi_processor_count)}

    def _tune_key(self, scene: Scene) -> str:
        c = self.cfg
        tris = sum(int(m.f.shape[0]) for m in scene.meshes) + sum(
            int(lt.f.shape[0]) for lt in scene.lights if getattr(lt, "f", None) is not None)
        shape = dict(self._gpu_id(), tris=tris, views=[[int(v.height), int(v.width)] for v in scene.cameras],
                     spp=int(c.spp_interior), depth=int(c.max_bounce), nl=int(c.mis_light_samples),
                     nb=int(c.mis_bsdf_samples), estimator=int(c.estimator))
        return json.dumps(shape, sort_keys=True)

    def render_samples(self, scene: Scene, camera_index: int = 0) -> Tensor:
        """Per-sample interior radiance (H*W*spp, 3) of one camera (the values the film averages)."""
        c = scene.cameras[camera_index]
        out = torch.empty((c.height * c.width * self.cfg.spp_interior, 3), dtype=torch.float32, device="cuda")
        cams = scene._camera_descs()
        L.check(self._lib.psdr_render_samples(scene.handle, self._workspace(), C.byref(cams[camera_index]),
                                              C.byref(self.cfg), out.data_ptr(), _stream()), "psdr_render_samples")
        return out

    def _backward(self, scene: Scene, grads, torch_vars):
        dev = "cuda"
        dimgs = []
        for g, c in zip(grads, scene.cameras):
            if g is None:
                g = torch.zeros((c.height, c.width, 3), dtype=torch.float32, device=dev)
            dimgs.append(g.detach().float().contiguous())
        nm, nl = len(scene.meshes), len(scene.lights)
        # vertex gradients only for the meshes/lights whose vertices require grad (the
        # library then skips the others' scatters)
        vert_g = [_grad_buf(m.vertices, m.v) for m in scene.meshes] + [_grad_buf(lt.vertices, lt.v)
                                                                        for lt in scene.lights]
        tex_g = [_grad_buf(m.material.texture.tensor, m.material.texture.data) for m in scene.meshes]
        rough_g = [_tex_grad(m.material.roughness) for m in scene.meshes]
        nrm_g = [_tex_grad(m.material.normal) for m in scene.meshes]
        emit_g = [torch.zeros(3, dtype=torch.float32, device=dev) for _ in scene.lights]
        light_g = [_grad_buf(lt.params, lt.params_data) if _is_env(lt) else None for lt in scene.lights]
        cam_g = [torch.zeros(3, dtype=torch.float32, device=dev) for _ in scene.cameras]
        unb = self.cfg.estimator == L.EST_UNBIASED
        lens_g = [_lens_buf(c, unb) for c in scene.cameras]
        P = C.c_void_p
        vp = (P * (nm + nl))(*[None if t is None else t.data_ptr() for t in vert_g])
        tp = (P * max(1, nm))(*[None if t is None else t.data_ptr() for t in tex_g])
        ep = (P * max(1, nl))(*[t.data_ptr() for t in emit_g])
        cp = (P * len(cam_g))(*[t.data_ptr() for t in cam_g])
        tg = L.GradTargets(vp, tp, ep, cp, 0, _ptrs(rough_g), _ptrs(nrm_g), _ptrs(light_g), _ptrs(lens_g))
        dp = (P * len(dimgs))(*[d.data_ptr() for d in dimgs])
        cams = scene._camera_descs()
        L.check(self._lib.psdr_render_bwd(scene.handle, self._workspace(), cams, len(dimgs), C.byref(self.cfg), dp,
                                          C.byref(tg), _stream()), "psdr_render_bwd")
        # map the accumulators onto the input tensors (a tensor may play several roles)
        acc = {}

        def add(t, g):
            if t is None or not isinstance(t, Tensor) or not t.requires_grad:
                return
            g = g.reshape(t.shape).to(t.dtype)
            key = id(t)
            acc[key] = g if key not in acc else acc[key] + g

        for i, m in enumerate(scene.meshes):
            add(m.vertices, vert_g[i])
            add(m.material.texture.tensor, tex_g[i])
            if rough_g[i] is not None:
                add(m.material.roughness.tensor, rough_g[i])
            if nrm_g[i] is not None:
                add(m.material.normal.tensor, nrm_g[i])
        for j, lt in enumerate(scene.lights):
            add(lt.vertices, vert_g[nm + j])
            add(lt.emit, emit_g[j])
            if light_g[j] is not None:
                add(lt.params, light_g[j])
        for k, c in enumerate(scene.cameras):
            _add_camera_grads(add, c, cam_g[k], lens_g[k])
        return [acc.get(id(t), torch.zeros_like(t)) for t in torch_vars]

    def renderC(self, scene: Scene) -> List[Tensor]:
        """Plain render (path_integrator.cc:408-410): one (H, W, 3) image per camera."""
        with torch.no_grad():
            return self._render(scene)

    def renderD(self, scene: Scene) -> List[Tensor]:
        """Differentiable render (torch_psdr.py:547-556): images requiring grad; their
        backward runs the path-replay adjoint with both edge-sampling terms."""
        torch_vars = scene.get_variables()
        if not torch_vars:
            return self._render(scene)
        for c in scene.cameras:  # refuse unsupported camera gradients before rendering
            _lens_buf(c, self.cfg.estimator == L.EST_UNBIASED)
        imgs = _RenderD.apply(self, scene, *torch_vars)
        return list(imgs)


class BatchRender:
    """All cameras of one or more scenes rendered as one work list from CUDA graphs.

    The forward graph rebuilds every scene's geometry from its meshes' vertex buffers
    (update them in place with `Mesh.set_vertices`) and renders every camera; the
    backward graph runs the path-replay adjoint and every boundary term of the
    integrator's estimator for all views. Images, image gradients and gradient buffers
    are allocated once and bound to the graphs; vertex gradients are kept for the
    meshes and lights whose vertices require grad when the batch is created (keep
    that when swapping buffers with `Mesh.set_vertices`). Extension: the reference has
    no batching.

    Inside each graph the job's independent parts (the forward's tiles; the backward's
    interior tiles and every boundary term of every view) run on the integrator's
    `batch_lanes` concurrent streams, each with its own workspace, and with
    `batch_records` the forward keeps every interior path's replay record so that the
    backward runs the adjoint without re-tracing. Neither changes a bit of the images or
    gradients. Against `PathIntegrator.renderD` of each scene alone the images are equal
    and the gradients agree to float rounding (the batch packs all scenes' paths into
    shared tiles, which changes the per-thread sums of the light and camera gradients).
    The memory cost is one workspace per lane plus, with kept records,
    16 B x (1 + D R + 2 D) + 8 B per path (D = max_bounce, R = light + BSDF samples + 1).
    """

    def __init__(self, integrator: PathIntegrator, scenes: List[Scene], differentiable: bool = True):
        self.integrator = integrator
        self.scenes = list(scenes)
        self.lib = L.load()
        self.stream = torch.cuda.Stream()
        dev = "cuda"
        cams, cam_scene = [], []
        for si, sc in enumerate(self.scenes):
            for c in sc.cameras:
                cams.append(c)
                cam_scene.append(si)
        self.cams = cams
        self.images = [torch.zeros((c.height, c.width, 3), dtype=torch.float32, device=dev) for c in cams]
        self.d_images = [torch.zeros_like(i) for i in self.images] if differentiable else None
        P = C.c_void_p
        self._keep = []
        targets = []
        self.grads = []
        cam_g = [torch.zeros(3, dtype=torch.float32, device=dev) for _ in cams]
        cp = (P * len(cam_g))(*[t.data_ptr() for t in cam_g])
        self.cam_grads = cam_g
        unb = integrator.cfg.estimator == L.EST_UNBIASED
        self.lens_grads = [_lens_buf(c, unb) for c in cams] if differentiable else [None] * len(cams)
        lp_cam = _ptrs(self.lens_grads)
        for sc in self.scenes:
            vg = [_grad_buf(m.vertices, m.v) for m in sc.meshes] + [_grad_buf(lt.vertices, lt.v)
                                                                    for lt in sc.lights]
            tg = [_grad_buf(m.material.texture.tensor, m.material.texture.data) for m in sc.meshes]
            eg = [torch.zeros(3, dtype=torch.float32, device=dev) for _ in sc.lights]
            rg = [_tex_grad(m.material.roughness) for m in sc.meshes]
            ng = [_tex_grad(m.material.normal) for m in sc.meshes]
            lg = [_grad_buf(lt.params, lt.params_data) if _is_env(lt) else None for lt in sc.lights]
            self.grads.append((vg, tg, eg, rg, ng, lg))
            vp, tp, ep, rp, npp, lp = _ptrs(vg), _ptrs(tg), _ptrs(eg), _ptrs(rg), _ptrs(ng), _ptrs(lg)
            self._keep += [vp, tp, ep, rp, npp, lp]
            targets.append(L.GradTargets(vp, tp, ep, cp, 0, rp, npp, lp, lp_cam))
        self._keep += [cp, lp_cam]
        tgt = (L.GradTargets * len(targets))(*targets)
        sh = (P * len(self.scenes))(*[s.handle for s in self.scenes])
        cd = (L.CameraDesc * len(cams))(*[c._desc() for c in cams])
        csc = (C.c_int32 * len(cams))(*cam_scene)
        ip = (P * len(cams))(*[t.data_ptr() for t in self.images])
        dp = (P * len(cams))(*[t.data_ptr() for t in self.d_images]) if differentiable else None
        self._keep += [tgt, sh, cd, csc, ip, dp]
        h = C.c_void_p()
        torch.cuda.synchronize()
        L.check(self.lib.psdr_batch_create(sh, len(self.scenes), cd, csc, len(cams), C.byref(integrator.cfg), ip, dp,
                                           tgt, C.byref(h)), "psdr_batch_create")
        self._handle = h

    def forward(self) -> List[Tensor]:
        """Rebuild geometry and render every camera (returns the bound image buffers)."""
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        L.check(self.lib.psdr_batch_forward(self._handle, C.c_void_p(self.stream.cuda_stream)), "psdr_batch_forward")
        cur.wait_stream(self.stream)
        return self.images

    def backward(self, d_images: List[Tensor]):
        """Run the adjoint for dLoss/dImage of every camera; fills the bound gradient buffers."""
        for dst, g in zip(self.d_images, d_images):
            if g is None:
                dst.zero_()
            else:
                dst.copy_(g)
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        L.check(self.lib.psdr_batch_backward(self._handle, C.c_void_p(self.stream.cuda_stream)),
                "psdr_batch_backward")
        cur.wait_stream(self.stream)

    def renderD(self) -> List[Tensor]:
        """Differentiable batched render: images whose backward fills .grad of the
        scenes' input tensors, like PathIntegrator.renderD."""
        torch_vars = []
        for sc in self.scenes:
            torch_vars += sc.get_variables()
        return list(_BatchRenderD.apply(self, *torch_vars))

    def _map_grads(self, torch_vars):
        acc = {}

        def add(t, g):
            if t is None or not isinstance(t, Tensor) or not t.requires_grad:
                return
            g = g.reshape(t.shape).to(t.dtype)
            acc[id(t)] = g if id(t) not in acc else acc[id(t)] + g

        k = 0
        for sc, (vg, tg, eg, rg, ng, lg) in zip(self.scenes, self.grads):
            nm = len(sc.meshes)
            for i, m in enumerate(sc.meshes):
                add(m.vertices, vg[i])
                add(m.material.texture.tensor, tg[i])
                if rg[i] is not None:
                    add(m.material.roughness.tensor, rg[i])
                if ng[i] is not None:
                    add(m.material.normal.tensor, ng[i])
            for j, lt in enumerate(sc.lights):
                add(lt.vertices, vg[nm + j])
                add(lt.emit, eg[j])
                if lg[j] is not None:
                    add(lt.params, lg[j])
            for c in sc.cameras:
                _add_camera_grads(add, c, self.cam_grads[k], self.lens_grads[k])
                k += 1
        return [acc.get(id(t), torch.zeros_like(t)) for t in torch_vars]

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                self.lib.psdr_batch_destroy(h)
            except Exception:
                pass
            self._handle = None


class _BatchRenderD(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, *torch_vars):
        imgs = batch.forward()
        ctx.batch = batch
        ctx.vars = torch_vars
        return tuple(i.clone() for i in imgs)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, *grads):
        ctx.batch.backward(list(grads))
        return (None,) + tuple(ctx.batch._map_grads(ctx.vars))
