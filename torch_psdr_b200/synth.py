"""Seeded synthetic scenes for the path tracer (numpy only).

The reference measures nothing on a public dataset; its examples load OBJ assets
that are not part of the repository. These generators build the synthetic
workloads used by the tests and the benchmark: geodesic icospheres (frequency-n
subdivision of an icosahedron, 20*n^2 triangles) with a spherical uv mapping,
optional radial vertex noise, a ground quad, an area-light quad and uniform
random textures. Every array is float32 / int32 so it can be handed to the
renderer, the oracle, or torch without conversion.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0

_ICO_V = np.array([
    [-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
    [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
    [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1],
], dtype=np.float64)

_ICO_F = np.array([
    [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
    [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
    [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
    [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
], dtype=np.int64)


def geodesic_sphere(freq: int, radius: float = 1.0):
    """Icosahedron with every face split into freq^2 triangles, projected to a sphere.

    Returns (vertices (V,3) float64 on the unit sphere * radius, faces (F,3) int32).
    Vertices shared between faces are deduplicated exactly through integer lattice
    keys, so the mesh is closed (every edge has two faces).
    """
    n = int(freq)
    assert n >= 1
    key_to_idx: dict = {}
    verts = []
    faces = []

    def vid(fa, i, j):
        # point = a*(n-i-j) + b*i + c*j on face fa; key by the multiset of
        # (corner vertex, weight) so points on shared edges/corners coincide.
        a, b, c = _ICO_F[fa]
        w = {}
        for v, k in ((a, n - i - j), (b, i), (c, j)):
            if k:
                w[int(v)] = w.get(int(v), 0) + k
        key = tuple(sorted(w.items()))
        idx = key_to_idx.get(key)
        if idx is None:
            p = sum(_ICO_V[v] * k for v, k in key) / n
            p = p / np.linalg.norm(p)
            idx = len(verts)
            verts.append(p)
            key_to_idx[key] = idx
        return idx

    for fa in range(20):
        for i in range(n):
            for j in range(n - i):
                v0 = vid(fa, i, j)
                v1 = vid(fa, i + 1, j)
                v2 = vid(fa, i, j + 1)
                faces.append((v0, v1, v2))
                if i + j + 2 <= n:
                    v3 = vid(fa, i + 1, j + 1)
                    faces.append((v1, v3, v2))
    V = np.asarray(verts, dtype=np.float64) * radius
    F = np.asarray(faces, dtype=np.int32)
    return V, F


def icosphere(level: int, radius: float = 1.0):
    """Level-L icosphere (20*4^L triangles), i.e. geodesic frequency 2^L."""
    return geodesic_sphere(2 ** int(level), radius)


def spherical_uv(V: np.ndarray, F: np.ndarray):
    """Per-corner spherical uv with the seam split per face.

    Returns (uvs (3F,2) float32, uv_indices (F,3) int32). u = 0.5 + atan2(z,x)/2pi,
    v = 0.5 + asin(y/r)/pi. A face straddling the u seam gets u+1 on its small
    corners so its uv triangle is not flipped across the texture.
    """
    r = np.linalg.norm(V, axis=1)
    u = 0.5 + np.arctan2(V[:, 2], V[:, 0]) / (2 * math.pi)
    v = 0.5 + np.arcsin(np.clip(V[:, 1] / np.maximum(r, 1e-12), -1, 1)) / math.pi
    fu = u[F]
    fv = v[F]
    span = fu.max(axis=1) - fu.min(axis=1)
    wrap = span > 0.5
    fu = np.where(wrap[:, None] & (fu < 0.5), fu + 1.0, fu)
    uvs = np.stack([fu.reshape(-1), fv.reshape(-1)], axis=1).astype(np.float32)
    uv_idx = np.arange(3 * F.shape[0], dtype=np.int32).reshape(-1, 3)
    return uvs, uv_idx


def radial_noise(V: np.ndarray, sigma: float, seed: int):
    rng = np.random.default_rng(seed)
    r = np.linalg.norm(V, axis=1, keepdims=True)
    n = V / r
    return V + n * rng.normal(0.0, sigma, size=(V.shape[0], 1))


def quad(center, size, y, facing_down: bool):
    """Axis-aligned square in the plane y=const (2 triangles)."""
    cx, cz = center
    h = size / 2.0
    V = np.array([[cx - h, y, cz - h], [cx + h, y, cz - h],
                  [cx + h, y, cz + h], [cx - h, y, cz + h]], dtype=np.float32)
    if facing_down:
        F = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)
    else:
        F = np.array([[0, 2, 1], [0, 3, 2]], dtype=np.int32)
    return V, F


def uniform_texture(h, w, seed, lo=0.2, hi=0.8):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(h, w, 3)).astype(np.float32)


@dataclass
class MeshSpec:
    vertices: np.ndarray            # (V,3) float32
    faces: np.ndarray               # (F,3) int32
    uvs: np.ndarray | None = None   # (T,2) float32
    uv_indices: np.ndarray | None = None  # (F,3) int32
    texture: np.ndarray = None      # (3,) constant or (H,W,3)
    roughness: np.ndarray | None = None  # DiffuseBsdfMaterial: (1,) or (H,W)
    normal: np.ndarray | None = None     # DiffuseBsdfMaterial normal map: (3,) or (H,W,3)


@dataclass
class LightSpec:
    vertices: np.ndarray | None     # AreaLight mesh (environment lights: None)
    faces: np.ndarray | None
    emit: np.ndarray                # AreaLight radiance (environment lights: unused)
    kind: int = 0                   # 0 AreaLight, 1 EnvLight, 2 SH9Light
    cube_map: np.ndarray | None = None  # EnvLight: (H, W, 3) cube-map cross (4 x 3 faces)
    sh9: np.ndarray | None = None       # SH9Light: (9, 3) coefficients


@dataclass
class CameraSpec:
    look_from: np.ndarray
    look_at: np.ndarray
    up: np.ndarray
    vfov: float                     # perspective: vertical fov (radians); orthographic: view width
    height: int
    width: int
    kind: int = 0                   # 0 perspective, 1 orthographic


@dataclass
class SceneSpec:
    meshes: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    cameras: list = field(default_factory=list)


def default_camera(h, w):
    return CameraSpec(np.array([0, 0.5, 4], np.float32), np.array([0, 0, 0], np.float32),
                      np.array([0, 1, 0], np.float32), math.pi / 4, h, w)


def ground_and_light():
    gV, gF = quad((0.0, 0.0), 10.0, -1.0, facing_down=False)
    ground = MeshSpec(gV, gF, None, None, np.array([0.5, 0.5, 0.5], np.float32))
    lV, lF = quad((0.0, 0.0), 1.0, 3.0, facing_down=True)
    light = LightSpec(lV, lF, np.array([20.0, 20.0, 20.0], np.float32))
    return ground, light


def sphere_scene(level=3, tex_hw=256, tex_seed=0, noise_sigma=0.0, noise_seed=2,
                 height=128, width=128, freq=None) -> SceneSpec:
    """Textured icosphere on a ground quad under a 1x1 area light (radiance 20).

    level=3, tex_hw=256, 128x128 is the plain forward workload; level=5 with noise
    0.02 (seed 2) at 512x512 is the geometry-gradient workload.
    """
    if freq is None:
        V, F = icosphere(level)
    else:
        V, F = geodesic_sphere(freq)
    if noise_sigma > 0:
        V = radial_noise(V, noise_sigma, noise_seed)
    uvs, uvi = spherical_uv(V, F)
    tex = uniform_texture(tex_hw, tex_hw, tex_seed)
    sphere = MeshSpec(V.astype(np.float32), F, uvs, uvi, tex)
    ground, light = ground_and_light()
    return SceneSpec([sphere, ground], [light], [default_camera(height, width)])


def large_scene(n_spheres=16, level=6, tex_hw=512, seed=4, noise_sigma=0.02, height=1024,
                width=1024) -> SceneSpec:
    """Many-object workload: n_spheres noisy level-`level` icospheres (radius 1, radial
    noise N(0, noise_sigma) seeded per sphere) centred uniformly in the box [-5, 5]^3
    (seed `seed`), each with its own tex_hw^2 texture (seeds seed*100 + i); a 40x40
    ground quad at y = -6.5 (albedo 0.5) and a 4x4 area light at y = 7 facing down
    (radiance 20); the camera at (0, 4, 20) looks at the origin with a 45 degree field
    of view, which frames the whole box. 16 level-6 spheres are 1,310,720 triangles."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-5.0, 5.0, size=(n_spheres, 3))
    V0, F = icosphere(level)
    uvs, uvi = spherical_uv(V0, F)
    meshes = []
    for i in range(n_spheres):
        V = radial_noise(V0, noise_sigma, seed * 100 + i) if noise_sigma > 0 else V0
        meshes.append(MeshSpec((V + centres[i]).astype(np.float32), F, uvs, uvi,
                               uniform_texture(tex_hw, tex_hw, seed * 100 + i)))
    gV, gF = quad((0.0, 0.0), 40.0, -6.5, facing_down=False)
    meshes.append(MeshSpec(gV, gF, None, None, np.array([0.5, 0.5, 0.5], np.float32)))
    lV, lF = quad((0.0, 0.0), 4.0, 7.0, facing_down=True)
    light = LightSpec(lV, lF, np.array([20.0, 20.0, 20.0], np.float32))
    cam = CameraSpec(np.array([0, 4, 20], np.float32), np.array([0, 0, 0], np.float32),
                     np.array([0, 1, 0], np.float32), math.pi / 4, height, width)
    return SceneSpec(meshes, [light], [cam])


def orbit_cameras(n, radius, seed, size_lo=128, size_hi=512):
    """n cameras uniform on a sphere of the given radius looking at the origin,
    image sizes uniform in [size_lo, size_hi] (independently for H and W)."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        hw = rng.integers(size_lo, size_hi + 1, size=2)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        up = np.array([0, 1, 0], np.float32)
        if abs(d[1]) > 0.99:
            up = np.array([1, 0, 0], np.float32)
        cams.append(CameraSpec((d * radius).astype(np.float32), np.zeros(3, np.float32), up,
                               math.pi / 4, int(hw[0]), int(hw[1])))
    return cams


def env_box(cam_positions, mesh_vertices):
    """Bounding box of the environment lights (scene.cc:31-49), in float32 like the
    reference: the box of the camera positions and mesh vertices, its centre c and
    d = 1000 * its largest extent; returns (c - d, c + d)."""
    pmin = np.asarray(cam_positions[0], np.float32).copy()
    pmax = pmin.copy()
    for p in cam_positions:
        p = np.asarray(p, np.float32)
        pmin = np.minimum(pmin, p)
        pmax = np.maximum(pmax, p)
    for v in mesh_vertices:
        v = np.asarray(v, np.float32).reshape(-1, 3)
        pmin = np.minimum(pmin, v.min(0))
        pmax = np.maximum(pmax, v.max(0))
    d = np.float32(1000) * np.max(pmax - pmin)
    c = (pmin + pmax) * np.float32(0.5)
    return (c - d).astype(np.float32), (c + d).astype(np.float32)
