"""The C-ABI library builds, loads and exports every symbol include/psdr.h declares;
host-side argument checks and the Python API asserts (no GPU needed)."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import _lib as L
from torch_psdr_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return L.load()


def header_symbols():
    text = open(os.path.join(ROOT, "include", "psdr.h")).read()
    return sorted(set(re.findall(r"\b(psdr_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(lib):
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(L.SIGNATURES)


def test_version_and_errors(lib):
    assert b"sm_100a" in lib.psdr_version()
    assert lib.psdr_abi_version() == 6
    out = C.c_void_p()
    st = lib.psdr_scene_create(None, None, C.byref(out))
    assert st == L.PSDR_ERR_INVALID_ARG
    assert b"null" in lib.psdr_last_error()
    desc = L.SceneDesc(None, 0, None, 0)
    assert lib.psdr_scene_create(C.byref(desc), None, C.byref(out)) == L.PSDR_ERR_INVALID_ARG
    assert b"no geometry" in lib.psdr_last_error()
    with pytest.raises(ValueError):
        L.check(L.PSDR_ERR_INVALID_ARG, "x")


def test_render_rejects_bad_config(lib):
    ws = C.c_void_p()
    assert lib.psdr_workspace_create(C.byref(ws)) == 0
    cfg = L.Config()
    cfg.n_pass = 0
    cam = L.CameraDesc()
    img = (C.c_void_p * 1)(None)
    # a non-null fake scene handle is never dereferenced: the config check fails first
    st = lib.psdr_render_fwd(C.c_void_p(1), ws, C.byref(cam), 1, C.byref(cfg), img, None)
    assert st == L.PSDR_ERR_INVALID_ARG and b"n_pass" in lib.psdr_last_error()
    assert lib.psdr_workspace_destroy(ws) == 0


def test_batch_options_are_checked(lib):
    """batch_lanes (0..8) and batch_records (-1, 0, 1) are range-checked by the C ABI and
    the Python constructor, before any device work."""
    ws = C.c_void_p()
    assert lib.psdr_workspace_create(C.byref(ws)) == 0
    cam = L.CameraDesc()
    img = (C.c_void_p * 1)(None)
    for field, bad in (("batch_lanes", 9), ("batch_lanes", -1), ("batch_records", 2), ("batch_records", -2)):
        cfg = dr.PathIntegrator().cfg
        setattr(cfg, field, bad)
        st = lib.psdr_render_fwd(C.c_void_p(1), ws, C.byref(cam), 1, C.byref(cfg), img, None)
        assert st == L.PSDR_ERR_INVALID_ARG and field.encode() in lib.psdr_last_error()
    assert lib.psdr_workspace_destroy(ws) == 0
    with pytest.raises(AssertionError):
        dr.PathIntegrator(batch_lanes=9)
    with pytest.raises(AssertionError):
        dr.PathIntegrator(batch_records=2)
    cfg = dr.PathIntegrator(batch_lanes=8, batch_records=-1).cfg
    assert (cfg.batch_lanes, cfg.batch_records) == (8, -1)


def test_api_asserts_mirror_reference():
    t3 = torch.zeros(3)
    with pytest.raises(AssertionError):
        dr.PerspectiveCamera(torch.zeros(2), t3, t3, torch.zeros(1), 4, 4)
    with pytest.raises(AssertionError):
        dr.PerspectiveCamera(t3, t3, t3, torch.zeros(1), 0, 4)
    with pytest.raises(AssertionError):
        dr.Texture(torch.zeros(4, 4))  # the reference's (H, W) branch never sets tex_type
    with pytest.raises(AssertionError):
        dr.PathIntegrator(spp_interior=0)
    with pytest.raises(AssertionError):
        dr.PathIntegrator(secondary_edge_hypercube_resolution=[1, 2])
    with pytest.raises(AssertionError):
        dr.AreaLight(torch.zeros(4, 3), torch.zeros(2, 3, dtype=torch.int32), torch.zeros(4))
    with pytest.raises(AssertionError):
        dr.SH9Light(torch.zeros(8, 3))  # torch_psdr.py:445 (9, 3) coefficients
    with pytest.raises(AssertionError):
        dr.OrthographicCamera(t3, t3, t3, torch.zeros(2), 4, 4)  # view_width (1,)
    with pytest.raises(AssertionError):
        dr.OrthographicCamera(t3, t3, t3, torch.zeros(1), 4, 0)
    cam = dr.OrthographicCamera(torch.tensor([0.0, 0.5, 4.0]), torch.zeros(3), torch.tensor([0.0, 1.0, 0.0]),
                                torch.tensor([3.0]), 23, 25)
    d = cam._desc()
    assert (d.type, d.fov, d.height, d.width) == (L.CAM_ORTHOGRAPHIC, 3.0, 23, 25)
    assert dr.Camera is dr.PerspectiveCamera


def test_cpu_tensors_are_rejected():
    with pytest.raises(ValueError):
        dr.Texture(torch.zeros(3))


def test_index_buffers_are_range_checked():
    """Mesh and AreaLight check face and uv indices against their vertex and uv counts
    (the native gathers do not), on CPU tensors here."""
    from torch_psdr_b200.api import check_indices
    f = torch.tensor([[0, 1, 2], [0, 2, 3]], dtype=torch.int32)
    check_indices(f, 4, "face_indices")
    check_indices(torch.zeros((0, 3), dtype=torch.int32), 0, "face_indices")
    with pytest.raises(ValueError, match=r"\[0, 3\): found values in \[0, 3\]"):
        check_indices(f, 3, "face_indices")
    with pytest.raises(ValueError, match="uv_indices"):
        check_indices(f - 1, 4, "uv_indices")
    with pytest.raises(AssertionError):  # one uv triangle per face
        dr.Mesh(torch.zeros(4, 3), torch.zeros(4, 2), f, f[:1], None)


# ctypes mirror -> C struct of include/psdr.h, and the C field names where they differ
_STRUCTS = {
    "TextureDesc": ("psdr_texture_desc", {}),
    "MeshDesc": ("psdr_mesh_desc", {}),
    "AreaLightDesc": ("psdr_area_light_desc", {}),
    "SceneDesc": ("psdr_scene_desc", {}),
    "CameraDesc": ("psdr_camera_desc", {}),
    "Config": ("psdr_config", {}),
    "GradTargets": ("psdr_grad_targets", {}),
}


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror in torch_psdr_b200/_lib.py has the size and field offsets of
    its C struct (compiled here against include/psdr.h with gcc)."""
    import os
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "psdr.h"', "int main(void) {"]
    for py, (cname, rename) in _STRUCTS.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(L, py)._fields_:
            lines.append(f'  printf("{py} {field} %zu\\n", offsetof({cname}, {rename.get(field, field)}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        py, what, value = line.split()
        cls = getattr(L, py)
        want = C.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert int(value) == want, (py, what, int(value), want)
        seen += 1
    assert seen > 40


def test_environment_light_arguments_are_checked(lib):
    """psdr_scene_create refuses malformed environment lights before any device work:
    a bad light type, an environment light that is not the last light, an empty box,
    a scene without meshes, a cube map that is not UV3f."""
    V = (C.c_float * 9)(0, 0, 0, 1, 0, 0, 0, 1, 0)
    F = (C.c_int32 * 3)(0, 1, 2)
    mesh = L.MeshDesc()
    mesh.vertices, mesh.num_vertices, mesh.faces, mesh.num_faces = C.cast(V, C.c_void_p), 3, C.cast(F, C.c_void_p), 1
    mesh.color = L.TextureDesc(L.TEX_CONSTANT, 3, 1, 1, C.cast((C.c_float * 3)(0.5, 0.5, 0.5), C.c_void_p))
    area = L.AreaLightDesc()
    area.vertices, area.num_vertices, area.faces, area.num_faces = C.cast(V, C.c_void_p), 3, C.cast(F, C.c_void_p), 1

    def sh9(lo=-1.0, hi=1.0):
        d = L.AreaLightDesc()
        d.type = L.LIGHT_SH9
        d.box_min = (C.c_float * 3)(lo, lo, lo)
        d.box_max = (C.c_float * 3)(hi, hi, hi)
        return d

    def create(meshes, lights):
        md = (L.MeshDesc * max(1, len(meshes)))(*meshes)
        ld = (L.AreaLightDesc * max(1, len(lights)))(*lights)
        desc = L.SceneDesc(md, len(meshes), ld, len(lights))
        out = C.c_void_p()
        return lib.psdr_scene_create(C.byref(desc), None, C.byref(out)), lib.psdr_last_error()

    bad = sh9()
    bad.type = 7
    assert create([mesh], [bad]) == (L.PSDR_ERR_INVALID_ARG, b"bad light type")
    st, msg = create([mesh], [sh9(), area])
    assert st == L.PSDR_ERR_INVALID_ARG and b"last light" in msg
    st, msg = create([mesh], [area, sh9(1.0, 1.0)])
    assert st == L.PSDR_ERR_INVALID_ARG and b"empty environment light box" in msg
    st, msg = create([], [sh9()])
    assert st == L.PSDR_ERR_INVALID_ARG and b"needs a mesh" in msg
    env = sh9()
    env.type = L.LIGHT_ENV
    env.cube_map = L.TextureDesc(L.TEX_CONSTANT, 3, 1, 1, C.cast((C.c_float * 3)(1, 1, 1), C.c_void_p))
    st, msg = create([mesh], [env])
    assert st == L.PSDR_ERR_INVALID_ARG and b"UV3f" in msg


def test_material_and_camera_arguments_are_checked(lib):
    """A DiffuseBsdfMaterial roughness of 3 channels and a camera with a non-positive
    fov / view width are refused before device work."""
    V = (C.c_float * 9)(0, 0, 0, 1, 0, 0, 0, 1, 0)
    F = (C.c_int32 * 3)(0, 1, 2)
    mesh = L.MeshDesc()
    mesh.vertices, mesh.num_vertices, mesh.faces, mesh.num_faces = C.cast(V, C.c_void_p), 3, C.cast(F, C.c_void_p), 1
    c3 = C.cast((C.c_float * 3)(0.5, 0.5, 0.5), C.c_void_p)
    mesh.color = L.TextureDesc(L.TEX_CONSTANT, 3, 1, 1, c3)
    mesh.material = L.MAT_DIFFUSE_BSDF
    mesh.roughness = L.TextureDesc(L.TEX_CONSTANT, 3, 1, 1, c3)
    mesh.normal = L.TextureDesc(L.TEX_NONE, 0, 0, 0, None)
    md = (L.MeshDesc * 1)(mesh)
    desc = L.SceneDesc(md, 1, None, 0)
    out = C.c_void_p()
    assert lib.psdr_scene_create(C.byref(desc), None, C.byref(out)) == L.PSDR_ERR_INVALID_ARG
    assert b"roughness texture must have 1 channel" in lib.psdr_last_error()
    ws = C.c_void_p()
    assert lib.psdr_workspace_create(C.byref(ws)) == 0
    cfg = L.Config()
    for k, v in dict(n_pass=1, spp_interior=1, spp_primary_edge=1, spp_secondary_edge=1, max_bounce=1,
                     mis_light_samples=1, mis_bsdf_samples=1, primary_edge_preprocess_rounds=1,
                     secondary_edge_preprocess_rounds=1, primary_edge_hypercube_resolution=10).items():
        setattr(cfg, k, v)
    cfg.secondary_edge_hypercube_resolution[:] = [10, 1, 1]
    cam = L.CameraDesc()
    cam.type, cam.fov, cam.height, cam.width = L.CAM_ORTHOGRAPHIC, 0.0, 4, 4
    img = (C.c_void_p * 1)(None)
    st = lib.psdr_render_fwd(C.c_void_p(1), ws, C.byref(cam), 1, C.byref(cfg), img, None)
    assert st == L.PSDR_ERR_INVALID_ARG and b"view width" in lib.psdr_last_error()
    assert lib.psdr_workspace_destroy(ws) == 0


def test_autotune_cache_keys_and_reuse(tmp_path, monkeypatch):
    """PathIntegrator.autotune(scene, cache=path): a miss tunes (the native call, faked
    here) and records the result under a key of the GPU and the job's shape; a hit
    applies the stored sizes without tuning; another shape or GPU misses."""
    from types import SimpleNamespace as NS
    integ = dr.PathIntegrator(spp_interior=8, max_bounce=3)
    calls, applied = [], []
    monkeypatch.setattr(integ, "_autotune_native",
                        lambda scene: calls.append(scene) or {"tile_paths": 1 << 19, "leaf_size": 2, "forward_ms": 1.5})
    monkeypatch.setattr(integ, "_apply_tuning", lambda scene, entry: applied.append(dict(entry)))
    gpu = {"gpu": "B200", "sms": 148}
    monkeypatch.setattr(dr.PathIntegrator, "_gpu_id", staticmethod(lambda: dict(gpu)))
    mesh = NS(f=torch.zeros((20, 3), dtype=torch.int32))
    light = NS(f=torch.zeros((2, 3), dtype=torch.int32))
    scene = NS(meshes=[mesh], lights=[light], cameras=[NS(height=64, width=48)])
    path = str(tmp_path / "tune.json")
    first = integ.autotune(scene, cache=path)
    assert len(calls) == 1 and "cached" not in first
    again = integ.autotune(scene, cache=path)
    assert len(calls) == 1 and again["cached"] and applied == [first]
    key = json.loads(next(iter(json.load(open(path)))))
    assert key == {"gpu": "B200", "sms": 148, "tris": 22, "views": [[64, 48]], "spp": 8, "depth": 3, "nl": 1,
                   "nb": 1, "estimator": int(integ.cfg.estimator)}
    scene.cameras[0].width = 49          # another view size misses
    integ.autotune(scene, cache=path)
    gpu["sms"] = 132                      # another GPU misses
    integ.autotune(scene, cache=path)
    assert len(calls) == 3 and len(json.load(open(path))) == 3
    integ.autotune(scene)                 # no cache: always tunes
    assert len(calls) == 4


def test_scene_validate_argument_checks(lib):
    """psdr_scene_validate (the opt-in index-range check before psdr_scene_create): its
    host-side argument checks, which return before any device work."""
    assert lib.psdr_scene_validate(None, None) == L.PSDR_ERR_INVALID_ARG
    assert b"null" in lib.psdr_last_error()
    desc = L.SceneDesc(None, 1, None, 0)
    assert lib.psdr_scene_validate(C.byref(desc), None) == L.PSDR_ERR_INVALID_ARG
    assert b"null mesh array" in lib.psdr_last_error()
    m = L.MeshDesc()
    m.num_vertices, m.num_faces = 3, -1
    meshes = (L.MeshDesc * 1)(m)
    desc = L.SceneDesc(meshes, 1, None, 0)
    assert lib.psdr_scene_validate(C.byref(desc), None) == L.PSDR_ERR_INVALID_ARG
    assert b"negative counts" in lib.psdr_last_error()
    meshes[0].num_faces = 1  # faces null
    assert lib.psdr_scene_validate(C.byref(desc), None) == L.PSDR_ERR_INVALID_ARG
    assert b"null face buffer" in lib.psdr_last_error()
    empty = L.SceneDesc(None, 0, None, 0)
    assert lib.psdr_scene_validate(C.byref(empty), None) == L.PSDR_OK  # nothing to check


def test_header_is_strict_c99_and_cxx17(tmp_path):
    """include/psdr.h compiles warning-free as ISO C99 and as C++17 (the bindings a C,
    C++ or FFI host writes against it)."""
    import shutil
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "hdr.c"
    src.write_text('#include "psdr.h"\nint main(void) { return (int)sizeof(psdr_config) == 0; }\n')
    for cc, flags in (("gcc", ["-std=c99"]), ("g++", ["-std=c++17", "-x", "c++"])):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not available")
        subprocess.run([cc, *flags, "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(root, "include"),
                        str(src), "-o", str(tmp_path / f"hdr_{cc}")], check=True)


def _lens_map(p):
    """The raster-to-direction map of a perspective camera from (look_from, look_at, up,
    fov) = p[0:3], p[3:6], p[6:9], p[9], restated from camera.h:7-64 (numpy, float64):
    M = C diag(2 tan(fov/2) / W, -2 tan(fov/2) / H, -1), C = (right, up', dir)."""
    W, H = 40.0, 30.0
    frm, at, up, fov = p[0:3], p[3:6], p[6:9], p[9]
    d = (frm - at) / np.linalg.norm(frm - at)
    r = np.cross(up / np.linalg.norm(up), d)
    u2 = np.cross(d, r)
    t = np.tan(fov / 2)
    return np.stack([r * 2 * t / W, u2 * -2 * t / H, -d], axis=1)


def test_camera_lens_jacobian_matches_finite_differences():
    """psdr_camera_lens_jacobian (host code behind the camera_lens gradient): M equals the
    restated map and P_j = M^-1 dM/dtheta_j equals central differences of it."""
    lib = L.load()
    p = np.array([0.3, 0.5, 4.0, 0.1, -0.2, 0.05, 0.1, 1.0, 0.2, 0.8])
    d = L.CameraDesc()
    d.type = L.CAM_PERSPECTIVE
    d.look_from = (C.c_float * 3)(*p[0:3])
    d.look_at = (C.c_float * 3)(*p[3:6])
    d.up = (C.c_float * 3)(*p[6:9])
    d.fov = float(p[9])
    d.height, d.width = 30, 40
    pf = np.array(list(d.look_from) + list(d.look_at) + list(d.up) + [d.fov], np.float64)  # the float inputs
    m = (C.c_double * 9)()
    P = (C.c_double * 90)()
    assert lib.psdr_camera_lens_jacobian(C.byref(d), m, P) == L.PSDR_OK
    M = _lens_map(pf)
    np.testing.assert_allclose(np.array(m).reshape(3, 3), M, rtol=1e-12, atol=1e-14)
    Minv = np.linalg.inv(M)
    for j in range(10):
        e = np.zeros(10)
        e[j] = 1e-6
        dM = (_lens_map(pf + e) - _lens_map(pf - e)) / 2e-6
        np.testing.assert_allclose(np.array(P[9 * j:9 * j + 9]).reshape(3, 3), Minv @ dM, rtol=1e-6, atol=1e-8)
    d.type = L.CAM_ORTHOGRAPHIC
    assert lib.psdr_camera_lens_jacobian(C.byref(d), m, P) == L.PSDR_ERR_INVALID_ARG
