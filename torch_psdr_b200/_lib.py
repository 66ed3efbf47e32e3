"""ctypes binding of libpsdr_b200.so (the C ABI in include/psdr.h).

The library is built in-tree (torch_psdr_b200/_lib/libpsdr_b200.so). Loading fails
loudly when it is missing: there is no CPU or Python fallback for the renderer.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PSDR_B200_LIB overrides the library location (e.g. a build installed elsewhere).
LIB_PATH = os.environ.get("PSDR_B200_LIB", os.path.join(HERE, "_lib", "libpsdr_b200.so"))

PSDR_OK = 0
PSDR_ERR_INVALID_ARG = 1
PSDR_ERR_UNSUPPORTED = 6
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "NUMERIC", 6: "UNSUPPORTED"}

TEX_NONE, TEX_CONSTANT, TEX_UV = -1, 0, 1
MAT_DIFFUSE, MAT_DIFFUSE_BSDF = 0, 1
CAM_PERSPECTIVE, CAM_ORTHOGRAPHIC = 0, 1
LIGHT_AREA, LIGHT_ENV, LIGHT_SH9 = 0, 1, 2
EST_REFERENCE, EST_UNBIASED = 0, 1


class TextureDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("channels", C.c_int32), ("height", C.c_int32), ("width", C.c_int32),
                ("data", C.c_void_p)]


class MeshDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("num_vertices", C.c_int32), ("faces", C.c_void_p),
                ("num_faces", C.c_int32), ("uvs", C.c_void_p), ("num_uvs", C.c_int32), ("uv_indices", C.c_void_p),
                ("material", C.c_int32), ("color", TextureDesc), ("roughness", TextureDesc),
                ("normal", TextureDesc)]


class AreaLightDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("num_vertices", C.c_int32), ("faces", C.c_void_p),
                ("num_faces", C.c_int32), ("emit", C.c_float * 3), ("type", C.c_int32),
                ("cube_map", TextureDesc), ("sh9", C.c_float * 27), ("box_min", C.c_float * 3),
                ("box_max", C.c_float * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(MeshDesc)), ("num_meshes", C.c_int32), ("lights", C.POINTER(AreaLightDesc)),
                ("num_lights", C.c_int32)]


class CameraDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("look_from", C.c_float * 3), ("look_at", C.c_float * 3),
                ("up", C.c_float * 3), ("fov", C.c_float), ("height", C.c_int32), ("width", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("n_pass", C.c_int32), ("spp_interior", C.c_int32), ("enable_light_visable", C.c_int32),
                ("spp_primary_edge", C.c_int32), ("spp_secondary_edge", C.c_int32), ("max_bounce", C.c_int32),
                ("mis_light_samples", C.c_int32), ("mis_bsdf_samples", C.c_int32),
                ("primary_edge_preprocess_rounds", C.c_int32), ("secondary_edge_preprocess_rounds", C.c_int32),
                ("primary_edge_hypercube_resolution", C.c_int32),
                ("secondary_edge_hypercube_resolution", C.c_int32 * 3), ("estimator", C.c_int32),
                ("tile_paths", C.c_int32), ("leaf_size", C.c_int32), ("terms", C.c_int32),
                ("spp_pixel_boundary", C.c_int32), ("seed", C.c_uint64), ("trace_queue", C.c_int32),
                ("batch_lanes", C.c_int32), ("batch_records", C.c_int32)]


class GradTargets(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_void_p)), ("textures", C.POINTER(C.c_void_p)),
                ("emit", C.POINTER(C.c_void_p)), ("camera_origin", C.POINTER(C.c_void_p)),
                ("accumulate", C.c_int32), ("roughness", C.POINTER(C.c_void_p)),
                ("normal", C.POINTER(C.c_void_p)), ("light_params", C.POINTER(C.c_void_p)),
                ("camera_lens", C.POINTER(C.c_void_p))]


# Every symbol include/psdr.h declares, with its ctypes signature.
P = C.c_void_p
SIGNATURES = {
    "psdr_last_error": ([], C.c_char_p),
    "psdr_version": ([], C.c_char_p),
    "psdr_abi_version": ([], C.c_int32),
    "psdr_scene_create": ([C.POINTER(SceneDesc), P, C.POINTER(P)], C.c_int),
    "psdr_scene_validate": ([C.POINTER(SceneDesc), P], C.c_int),
    "psdr_scene_destroy": ([P], C.c_int),
    "psdr_scene_update": ([P, P], C.c_int),
    "psdr_scene_refit": ([P, P], C.c_int),
    "psdr_scene_set_leaf_size": ([P, C.c_int32, P], C.c_int),
    "psdr_scene_info": ([P, C.POINTER(C.c_int64)], C.c_int),
    "psdr_scene_edges": ([P, P, P, C.c_int64, C.POINTER(C.c_int64), P], C.c_int),
    "psdr_intersect": ([P, P, C.c_int64, P, P, P, C.c_int32, P], C.c_int),
    "psdr_camera_lens_jacobian": ([P, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "psdr_workspace_create": ([C.POINTER(P)], C.c_int),
    "psdr_workspace_destroy": ([P], C.c_int),
    "psdr_render_fwd": ([P, P, C.POINTER(CameraDesc), C.c_int32, C.POINTER(Config), C.POINTER(P), P], C.c_int),
    "psdr_render_samples": ([P, P, C.POINTER(CameraDesc), C.POINTER(Config), P, P], C.c_int),
    "psdr_autotune": ([P, P, C.POINTER(CameraDesc), C.c_int32, C.POINTER(Config), C.POINTER(C.c_int32),
                       C.POINTER(C.c_float), P], C.c_int),
    "psdr_render_fwd_noalloc": ([P, C.POINTER(CameraDesc), C.POINTER(Config), P, P], C.c_int),
    "psdr_render_bwd": ([P, P, C.POINTER(CameraDesc), C.c_int32, C.POINTER(Config), C.POINTER(P),
                         C.POINTER(GradTargets), P], C.c_int),
    "psdr_batch_create": ([C.POINTER(P), C.c_int32, C.POINTER(CameraDesc), C.POINTER(C.c_int32), C.c_int32,
                           C.POINTER(Config), C.POINTER(P), C.POINTER(P), C.POINTER(GradTargets), C.POINTER(P)],
                          C.c_int),
    "psdr_batch_forward": ([P, P], C.c_int),
    "psdr_batch_backward": ([P, P], C.c_int),
    "psdr_batch_destroy": ([P], C.c_int),
    "psdr_profile_enable": ([C.c_int32], C.c_int),
    "psdr_profile_reset": ([], C.c_int),
    "psdr_profile_read": ([C.POINTER(C.c_int64), C.POINTER(C.c_double)], C.c_int),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the native library (no compilation, no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libpsdr_b200.so not found at {path}; build it with `python -m torch_psdr_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class PsdrError(RuntimeError):
    pass


def check(status: int, what: str = ""):
    if status == PSDR_OK:
        return
    msg = _lib.psdr_last_error().decode(errors="replace") if _lib is not None else ""
    text = f"{what}: {STATUS_NAMES.get(status, status)}: {msg}"
    if status == PSDR_ERR_INVALID_ARG:
        raise ValueError(text)
    raise PsdrError(text)
