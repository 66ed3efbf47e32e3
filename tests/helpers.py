"""Test helpers: synthetic scene specs -> torch_psdr_b200 objects, and tolerances."""
import math

import numpy as np
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth


def to_torch_scene(spec, requires_grad=(), device="cuda"):
    """Build a dr.Scene from a synth.SceneSpec. requires_grad: subset of
    {"verts", "tex", "light_verts", "emit", "cam"}; returns (scene, dict of tensors)."""
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
        meshes.append(dr.Mesh(v, uv, f, uvi, dr.DiffuseMaterial(tex)))
    lights = []
    for j, l in enumerate(spec.lights):
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
        cams.append(dr.PerspectiveCamera(lf, torch.tensor(c.look_at, dtype=torch.float32, device=device),
                                         torch.tensor(c.up, dtype=torch.float32, device=device),
                                         torch.tensor([c.vfov], dtype=torch.float32, device=device),
                                         c.height, c.width))
    return dr.Scene(cams, meshes, lights), T


def rel_mse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.mean((a - b) ** 2) / max(np.mean(b ** 2), 1e-30))


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
