"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Marshals a torch_psdr_b200.synth.SceneSpec into the oracle's C structs and exposes
render / directional-derivative / intersection / edge queries. Parity unpinned: the
reference has no golden vectors; see psdr_oracle.hpp.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build as _build  # noqa: E402

_lib = None


class OrcTexture(C.Structure):
    _fields_ = [("kind", C.c_int), ("h", C.c_int), ("w", C.c_int), ("c", C.c_int), ("data", C.c_void_p)]


class OrcMesh(C.Structure):
    _fields_ = [("V", C.c_void_p), ("nV", C.c_int), ("F", C.c_void_p), ("nF", C.c_int),
                ("uv", C.c_void_p), ("nUV", C.c_int), ("uvi", C.c_void_p), ("mat", C.c_int),
                ("color", OrcTexture), ("rough", OrcTexture), ("normal", OrcTexture)]


class OrcLight(C.Structure):
    _fields_ = [("V", C.c_void_p), ("nV", C.c_int), ("F", C.c_void_p), ("nF", C.c_int),
                ("emit", C.c_float * 3), ("type", C.c_int), ("cube_map", OrcTexture), ("sh9", C.c_float * 27),
                ("box_min", C.c_float * 3), ("box_max", C.c_float * 3)]


class OrcCamera(C.Structure):
    _fields_ = [("look_from", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("fov", C.c_float), ("h", C.c_int), ("w", C.c_int), ("type", C.c_int)]


class OrcConfig(C.Structure):
    _fields_ = [("n_pass", C.c_int), ("spp_interior", C.c_int), ("enable_light_visable", C.c_int),
                ("spp_primary_edge", C.c_int), ("spp_secondary_edge", C.c_int), ("max_bounce", C.c_int),
                ("mis_light_samples", C.c_int), ("mis_bsdf_samples", C.c_int), ("pe_rounds", C.c_int),
                ("se_rounds", C.c_int), ("pe_res", C.c_int), ("se_res", C.c_int * 3), ("mode", C.c_int),
                ("spp_pixel_boundary", C.c_int), ("seed", C.c_uint64)]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = C.CDLL(path)
        P = C.c_void_p
        _lib.orc_render.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_int, P, P]
        _lib.orc_grad_dir.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_int, P, P, P, P, P, P]
        _lib.orc_intersect.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, P, P, P]
        _lib.orc_edges.argtypes = [P, C.c_int, P, C.c_int, C.c_int, P, P]
        _lib.orc_set_threads.argtypes = [C.c_int]
        _lib.orc_pcg32.argtypes = [C.c_uint64, C.c_uint64, C.c_int, P]
        _lib.orc_sampler_floats.argtypes = [C.c_uint64, C.c_int, P]
        _lib.orc_discrete_sample.argtypes = [P, C.c_int, P, C.c_int, P, P, P]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Marshal:
    """Keeps the numpy buffers alive while the C structs point at them."""

    def __init__(self, spec):
        self.keep = []
        self.meshes = (OrcMesh * max(1, len(spec.meshes)))()
        for i, m in enumerate(spec.meshes):
            V = np.ascontiguousarray(m.vertices, np.float32)
            F = np.ascontiguousarray(m.faces, np.int32)
            uv = None if m.uvs is None else np.ascontiguousarray(m.uvs, np.float32)
            uvi = None if m.uv_indices is None else np.ascontiguousarray(m.uv_indices, np.int32)
            t = self._tex(m.texture)
            self.keep += [V, F, uv, uvi]
            rough = getattr(m, "roughness", None)
            normal = getattr(m, "normal", None)
            mat = 0 if rough is None else 1
            self.meshes[i] = OrcMesh(_ptr(V), V.shape[0], _ptr(F), F.shape[0], _ptr(uv),
                                     0 if uv is None else uv.shape[0], _ptr(uvi), mat, t, self._tex(rough),
                                     self._tex(normal))
        self.lights = (OrcLight * max(1, len(spec.lights)))()
        box = None
        if any(getattr(l, "kind", 0) != 0 for l in spec.lights):
            from torch_psdr_b200.synth import env_box
            box = env_box([c.look_from for c in spec.cameras], [m.vertices for m in spec.meshes])
        for i, l in enumerate(spec.lights):
            kind = int(getattr(l, "kind", 0))
            if kind == 0:
                V = np.ascontiguousarray(l.vertices, np.float32)
                F = np.ascontiguousarray(l.faces, np.int32)
            else:
                V = np.zeros((0, 3), np.float32)
                F = np.zeros((0, 3), np.int32)
            self.keep += [V, F]
            sh = np.zeros(27, np.float32) if kind != 2 else np.asarray(l.sh9, np.float32).reshape(27)
            bmin, bmax = box if kind != 0 else (np.zeros(3, np.float32), np.zeros(3, np.float32))
            self.lights[i] = OrcLight(_ptr(V), V.shape[0], _ptr(F), F.shape[0],
                                      (C.c_float * 3)(*[float(x) for x in l.emit]), kind,
                                      self._tex(l.cube_map if kind == 1 else None), (C.c_float * 27)(*map(float, sh)),
                                      (C.c_float * 3)(*map(float, bmin)), (C.c_float * 3)(*map(float, bmax)))
        self.cams = (OrcCamera * max(1, len(spec.cameras)))()
        for i, c in enumerate(spec.cameras):
            self.cams[i] = OrcCamera((C.c_float * 3)(*map(float, c.look_from)), (C.c_float * 3)(*map(float, c.look_at)),
                                     (C.c_float * 3)(*map(float, c.up)), float(c.vfov), int(c.height), int(c.width),
                                     int(getattr(c, "kind", 0)))
        self.nm, self.nl, self.nc = len(spec.meshes), len(spec.lights), len(spec.cameras)

    def _tex(self, a):
        """OrcTexture of a constant (1-D) or uv map ((H, W) or (H, W, C)); None -> absent."""
        if a is None:
            return OrcTexture(-1, 0, 0, 0, None)
        a = np.ascontiguousarray(a, np.float32)
        self.keep.append(a)
        if a.ndim == 1:
            return OrcTexture(0, 1, 1, a.shape[0], _ptr(a))
        c = 1 if a.ndim == 2 else a.shape[2]
        return OrcTexture(1, a.shape[0], a.shape[1], c, _ptr(a))

    def args(self):
        return (C.byref(self.meshes), self.nm, C.byref(self.lights), self.nl, C.byref(self.cams), self.nc)


def make_config(n_pass=1, spp_interior=1, enable_light_visable=False, spp_primary_edge=1, spp_secondary_edge=1,
                max_bounce=3, mis_light_samples=1, mis_bsdf_samples=1, primary_edge_preprocess_rounds=1,
                secondary_edge_preprocess_rounds=1, primary_edge_hypercube_resolution=10000,
                secondary_edge_hypercube_resolution=(10000, 6, 6), mode=0, spp_pixel_boundary=0, seed=0, **_):
    return OrcConfig(n_pass, spp_interior, int(enable_light_visable), spp_primary_edge, spp_secondary_edge,
                     max_bounce, mis_light_samples, mis_bsdf_samples, primary_edge_preprocess_rounds,
                     secondary_edge_preprocess_rounds, primary_edge_hypercube_resolution,
                     (C.c_int * 3)(*secondary_edge_hypercube_resolution), mode, spp_pixel_boundary, int(seed))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def render(spec, precision=1, per_sample=False, **cfg):
    """Interior image(s) of every camera, (H, W, 3) float64 each."""
    L = lib()
    m = Marshal(spec)
    c = make_config(**cfg)
    sizes = [(cam.height, cam.width) for cam in spec.cameras]
    total = sum(h * w for h, w in sizes)
    out = np.zeros(total * 3, np.float64)
    ps = np.zeros(total * 3 * c.spp_interior, np.float64) if per_sample else None
    rc = L.orc_render(*m.args(), C.byref(c), int(precision), _ptr(out), _ptr(ps))
    if rc != 0:
        raise ValueError(f"oracle render failed (code {rc})")
    imgs, off = [], 0
    for h, w in sizes:
        imgs.append(out[off * 3:(off + h * w) * 3].reshape(h, w, 3))
        off += h * w
    if per_sample:
        return imgs, ps.reshape(-1, 3)
    return imgs


def grad_dir(spec, dLdI, which=1, seed_verts=None, seed_tex=None, seed_emit=None, seed_cam=None, **cfg):
    """dPhi/dtheta . seed_k for k < 8 with Phi = sum(dLdI * renderD(scene)).

    Seeds have a trailing axis of 8 (directions): verts (V_total,3,8), tex (elements,8),
    emit (n_lights,3,8), cam (n_cams,3,8)."""
    L = lib()
    m = Marshal(spec)
    c = make_config(**cfg)
    g = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64).reshape(-1) for x in dLdI]))
    sv = None if seed_verts is None else np.ascontiguousarray(seed_verts, np.float64)
    st = None if seed_tex is None else np.ascontiguousarray(seed_tex, np.float64)
    se = None if seed_emit is None else np.ascontiguousarray(seed_emit, np.float64)
    sc = None if seed_cam is None else np.ascontiguousarray(seed_cam, np.float64)
    out = np.zeros(8, np.float64)
    rc = L.orc_grad_dir(*m.args(), C.byref(c), int(which), _ptr(g), _ptr(sv), _ptr(st), _ptr(se), _ptr(sc),
                        _ptr(out))
    if rc != 0:
        raise ValueError(f"oracle gradient failed (code {rc})")
    return out


def intersect(spec, rays, use_bvh=True):
    """rays (n,6) float32 -> (tri (n,), bary (n,2), t (n,)) from the float brute force / BVH."""
    L = lib()
    m = Marshal(spec)
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    tri = np.zeros(n, np.int32)
    bary = np.zeros((n, 2), np.float32)
    t = np.zeros(n, np.float32)
    L.orc_intersect(*m.args()[:4], _ptr(rays), n, int(use_bvh), _ptr(tri), _ptr(bary), _ptr(t))
    return tri, bary, t


def edges(spec, cap=None):
    L = lib()
    m = Marshal(spec)
    if cap is None:
        cap = 3 * sum(int(x.faces.shape[0]) for x in spec.meshes + spec.lights)
    v01 = np.zeros((cap, 2), np.int32)
    geo = np.zeros((cap, 16), np.float32)
    n = L.orc_edges(*m.args()[:4], cap, _ptr(v01), _ptr(geo))
    return v01[:n], geo[:n]


def pcg32(initstate, initseq, n):
    out = np.zeros(n, np.uint32)
    lib().orc_pcg32(initstate, initseq, n, _ptr(out))
    return out


def discrete_sample(weights, u):
    """DiscreteSampler::sample_reuse (float instance) of the uniforms u over the weights:
    (indices, rescaled uniforms, pmf of each index)."""
    w = np.ascontiguousarray(weights, np.float64)
    uu = np.ascontiguousarray(u, np.float32)
    idx = np.zeros(uu.shape[0], np.int32)
    uo = np.zeros(uu.shape[0], np.float32)
    pm = np.zeros(uu.shape[0], np.float32)
    lib().orc_discrete_sample(_ptr(w), w.shape[0], _ptr(uu), uu.shape[0], _ptr(idx), _ptr(uo), _ptr(pm))
    return idx, uo, pm


def sampler_floats(i, n):
    out = np.zeros(n, np.float32)
    lib().orc_sampler_floats(i, n, _ptr(out))
    return out
