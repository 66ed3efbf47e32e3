"""Test helpers: synthetic scene specs -> torch_psdr_b200 objects, and tolerances."""
import math

import numpy as np
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth


def to_torch_scene(spec, requires_grad=(), device="cuda"):
    """Build a dr.Scene from a synth.SceneSpec. requires_grad: subset of
    {"verts", "tex", "rough", "normal", "light_verts", "emit", "env", "cam"}; returns
    (scene, dict of tensors). Meshes with a roughness get a DiffuseBsdfMaterial; lights of
    kind 1 / 2 become EnvLight / SH9Light (their parameters under "env{j}").

    "cam" makes T["cam{k}"] a translation of camera k: a perspective camera's look_at is
    look_from plus a constant, so the gradient of T["cam{k}"] is the derivative with the
    camera's basis held fixed (the oracle's camera derivative). An orthographic camera's
    look_at stays constant (its look_from gradient is already the translation)."""
    T = {}
    meshes = []
    for i, m in enumerate(spec.meshes):
        v = torch.tensor(m.vertices, dtype=torch.float32, device=device, requires_grad="verts" in requires_grad)
        f = torch.tensor(m.faces, dtype=torch.int32, device=device)
        uv = None if m.uvs is None else torch.tensor(m.uvs, dtype=torch.float32, device=device)
        uvi = None if m.uv_indices is None else torch.tensor(m.uv_indices, dtype=torch.int32, device=device)
        tex = torch.tensor(m.texture, dtype=torch.float32, device=device, requires_grad="tex" in requires_grad)
        T[f"verts{i}"] = v
        T[f"tex{i}"] = tex
        if getattr(m, "roughness", None) is None:
            mat = dr.DiffuseMaterial(tex)
        else:
            r = np.asarray(m.roughness, np.float32)
            r = r if r.ndim == 1 else r.reshape(r.shape[0], r.shape[1], 1)
            rough = torch.tensor(r, device=device, requires_grad="rough" in requires_grad)
            nrm = None
            if m.normal is not None:
                nrm = torch.tensor(m.normal, dtype=torch.float32, device=device,
                                   requires_grad="normal" in requires_grad)
            T[f"rough{i}"] = rough
            T[f"normal{i}"] = nrm
            mat = dr.DiffuseBsdfMaterial(tex, rough, nrm)
        meshes.append(dr.Mesh(v, uv, f, uvi, mat))
    lights = []
    for j, l in enumerate(spec.lights):
        kind = getattr(l, "kind", 0)
        if kind == 1:
            cube = torch.tensor(l.cube_map, dtype=torch.float32, device=device, requires_grad="env" in requires_grad)
            T[f"env{j}"] = cube
            lights.append(dr.EnvLight(dr.Texture(cube)))
            continue
        if kind == 2:
            sh = torch.tensor(l.sh9, dtype=torch.float32, device=device, requires_grad="env" in requires_grad)
            T[f"env{j}"] = sh
            lights.append(dr.SH9Light(sh))
            continue
        v = torch.tensor(l.vertices, dtype=torch.float32, device=device, requires_grad="light_verts" in requires_grad)
        f = torch.tensor(l.faces, dtype=torch.int32, device=device)
        e = torch.tensor(l.emit, dtype=torch.float32, device=device, requires_grad="emit" in requires_grad)
        T[f"lverts{j}"] = v
        T[f"emit{j}"] = e
        lights.append(dr.AreaLight(v, f, e))
    cams = []
    for k, c in enumerate(spec.cameras):
        lf = torch.tensor(c.look_from, dtype=torch.float32, device=device, requires_grad="cam" in requires_grad)
        T[f"cam{k}"] = lf
        ortho = getattr(c, "kind", 0) == 1
        cls = dr.OrthographicCamera if ortho else dr.PerspectiveCamera
        at = torch.tensor(c.look_at, dtype=torch.float32, device=device)
        if "cam" in requires_grad and not ortho:
            at = lf + (at - lf.detach())
        cams.append(cls(lf, at, torch.tensor(c.up, dtype=torch.float32, device=device),
                        torch.tensor([c.vfov], dtype=torch.float32, device=device), c.height, c.width))
    return dr.Scene(cams, meshes, lights), T


def rel_mse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.mean((a - b) ** 2) / max(np.mean(b ** 2), 1e-30))


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# ---------------------------------------------------------------- gradient-check scenes
def wall_mesh(tex_hw=15, z=0.0, half=8.0, seed=5):
    """Square facing +z at depth z (two triangles); textured (tex_hw^2) or constant grey."""
    V = np.array([[-half, -half, z], [half, -half, z], [half, half, z], [-half, half, z]], np.float32)
    F = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    if not tex_hw:
        return synth.MeshSpec(V, F, None, None, np.array([0.5, 0.5, 0.5], np.float32))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    return synth.MeshSpec(V, F, uv, F.copy(), synth.uniform_texture(tex_hw, tex_hw, seed))


def front_light():
    """1x1 light at z = 3, y in [1.5, 2.5], facing -z, radiance 20."""
    V = np.array([[-0.5, 1.5, 3.0], [0.5, 1.5, 3.0], [0.5, 2.5, 3.0], [-0.5, 2.5, 3.0]], np.float32)
    F = np.array([[0, 2, 1], [0, 3, 2]], np.int32)
    return synth.LightSpec(V, F, np.array([20, 20, 20], np.float32))


def ball(level=2, textured=True, noise=0.02, scale=1.0, center=(0, 0, 0)):
    V, F = synth.icosphere(level)
    if noise:
        V = synth.radial_noise(V, noise, 2)
    V = (V * scale + np.asarray(center)).astype(np.float32)
    if textured:
        uvs, uvi = synth.spherical_uv(V, F)
        return synth.MeshSpec(V, F, uvs, uvi, synth.uniform_texture(32, 32, 0))
    return synth.MeshSpec(V, F, None, None, np.array([0.6, 0.4, 0.3], np.float32))


def front_camera(h, w):
    return synth.CameraSpec(np.array([0, 0.5, 4], np.float32), np.zeros(3, np.float32),
                            np.array([0, 1, 0], np.float32), math.pi / 4, h, w)


def gradient_case(name, h, w):
    """(spec, index of the moving mesh) of the named translation-gradient case:
    'ball'   - textured noisy ball before a textured wall (all four terms),
    'shadow' - an occluder outside the view casting a shadow on a grey wall (direct term),
    'wall'   - a textured wall filling the view (pixel borders).
    Wall textures have an odd texel count: with an even one a texel edge lies on the
    camera's centre line and so exactly on a pixel border, where the radiance that
    crosses the border is that of the texel edge itself (a measure-zero alignment at
    which the image is not differentiable and point samples on the border pick one
    side)."""
    cam = front_camera(h, w)
    if name == "ball":
        # off-centre for the same reason: the ball's uv seam texel edge faces the camera
        return synth.SceneSpec([ball(center=(0.05, 0.02, 0.0)), wall_mesh(15, z=-2)], [front_light()], [cam]), 0
    if name == "shadow":
        occ = ball(textured=False, noise=0.0, scale=0.25, center=(0, 1.8, 2.2))
        return synth.SceneSpec([occ, wall_mesh(0)], [front_light()], [cam]), 0
    if name == "wall":
        return synth.SceneSpec([wall_mesh(15)], [front_light()], [cam]), 0
    if name == "sunk":
        # a smooth textured ball sunk 0.3 into a textured ground, seen from above: the curve
        # where the two meshes cross is in view (interpenetration-crease term)
        sph = ball(level=3, textured=True, noise=0.0, center=(0.0, -0.7, 0.0))
        gV, gF = synth.quad((0.0, 0.0), 10.0, -1.0, facing_down=False)
        uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
        ground = synth.MeshSpec(gV, gF, uv, gF.copy(), synth.uniform_texture(15, 15, 7))
        # the light in front of the ball, so that both sides of the front crease are lit
        lV, lF = synth.quad((0.0, 2.5), 1.0, 3.0, facing_down=True)
        light = synth.LightSpec(lV, lF, np.array([20.0, 20.0, 20.0], np.float32))
        top = synth.CameraSpec(np.array([0.3, 2.0, 3.0], np.float32), np.array([0.0, -0.8, 0.0], np.float32),
                               np.array([0, 1, 0], np.float32), 0.8, h, w)
        return synth.SceneSpec([sph, ground], [light], [top]), 0
    if name == "creased":
        # a textured wall tilted 45 degrees, cut by a textured ground along a straight
        # crease (texel edges kept off the crease), the light in front (interpenetration
        # crease term; the planar case, where the crease velocity is exact)
        x0 = 0.3
        WV = np.array([[x0 - 1.0, -2, -3], [x0 - 1.0, -2, 3], [x0 + 2.0, 1, 3], [x0 + 2.0, 1, -3]], np.float32)
        WF = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
        uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
        wall = synth.MeshSpec(WV, WF, uv * np.float32(0.93) + np.float32(0.031), WF.copy(),
                              synth.uniform_texture(9, 9, 3))
        gV, gF = synth.quad((0.0, 0.0), 10.0, -1.0, facing_down=False)
        ground = synth.MeshSpec(gV, gF, uv, gF.copy(), synth.uniform_texture(15, 15, 7))
        lV, lF = synth.quad((-1.0, 0.0), 1.0, 3.0, facing_down=True)
        light = synth.LightSpec(lV, lF, np.array([20.0, 20.0, 20.0], np.float32))
        side = synth.CameraSpec(np.array([-1.5, 1.0, 2.5], np.float32), np.array([0.3, -1.0, 0.0], np.float32),
                                np.array([0, 1, 0], np.float32), 0.9, h, w)
        return synth.SceneSpec([wall, ground], [light], [side]), 0
    raise ValueError(name)


def smooth_weights(h, w):
    """Smooth image-space loss gradient (keeps the loss nearly linear over the FD step)."""
    yy, xx = np.meshgrid(np.arange(h) + 0.5, np.arange(w) + 0.5, indexing="ij")
    return np.stack([np.sin(2 * np.pi * xx / w * 1.3 + c) * np.cos(2 * np.pi * yy / h * 0.7) + 0.3
                     for c in range(3)], -1)


def translation_seeds(spec, mesh):
    """Directional seeds (V_total, 3, 8): directions 0..2 translate mesh `mesh` along x, y, z."""
    # an environment light's box has 8 vertices in the scene's vertex list
    nvt = sum(m.vertices.shape[0] for m in spec.meshes) + sum(
        l.vertices.shape[0] if getattr(l, "kind", 0) == 0 else 8 for l in spec.lights)
    seeds = np.zeros((nvt, 3, 8))
    off = sum(m.vertices.shape[0] for m in spec.meshes[:mesh])
    n = spec.meshes[mesh].vertices.shape[0]
    for k in range(3):
        seeds[off:off + n, k, k] = 1.0
    return seeds


def fd_translation(render, spec, mesh, g, h):
    """Central differences of sum(g * image) for translations of mesh `mesh` by +-h along
    x, y, z; render(spec) -> image (H, W, 3) with fixed sample seeds (common random numbers)."""
    V0 = spec.meshes[mesh].vertices.copy()
    out = []
    for k in range(3):
        phi = []
        for sgn in (1.0, -1.0):
            spec.meshes[mesh].vertices = (V0 + np.float32(sgn * h) * np.eye(3, dtype=np.float32)[k]).astype(np.float32)
            phi.append(float((g * render(spec)).sum()))
        out.append((phi[0] - phi[1]) / (2 * h))
    spec.meshes[mesh].vertices = V0
    return np.array(out)
