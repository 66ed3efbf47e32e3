"""OrthographicCamera (camera.h:279-353; torch_psdr.py:161-206), CPU only.

* the oracle's orthographic image matches a far-away perspective camera whose field of
  view spans the same width at the target (rays nearly parallel);
* the oracle's unbiased estimator with an orthographic camera (camera Jacobian |n.look|,
  rays from the camera plane, silhouette velocities without the depth ratio, camera
  connections along the view direction) matches central differences;
* the library's unbiased gradients still refuse orthographic cameras through the C ABI
  (status PSDR_ERR_UNSUPPORTED before any device work).
"""
import ctypes as C
import math

import numpy as np
import pytest

import orc
from torch_psdr_b200 import synth
from torch_psdr_b200 import _lib as L
from helpers import rel_mse


def ortho_spec(view_width=3.0, height=23, width=25, level=2, tex_hw=16):
    spec = synth.sphere_scene(level=level, tex_hw=tex_hw, height=height, width=width)
    c = spec.cameras[0]
    spec.cameras[0] = synth.CameraSpec(c.look_from, c.look_at, c.up, float(view_width), height, width, 1)
    return spec


def test_orthographic_matches_telephoto_perspective():
    spec = ortho_spec(height=32, width=32, level=3, tex_hw=32)
    c = spec.cameras[0]
    a = orc.render(spec, precision=1, spp_interior=64)[0]
    la = np.asarray(c.look_at, np.float64)
    d = np.asarray(c.look_from, np.float64) - la
    d /= np.linalg.norm(d)
    dist = 300.0
    spec.cameras[0] = synth.CameraSpec((la + d * dist).astype(np.float32), c.look_at, c.up,
                                       float(2 * math.atan(c.vfov / 2 / dist)), 32, 32, 0)
    b = orc.render(spec, precision=1, spp_interior=64)[0]
    print("orthographic vs telephoto: means", a.mean(), b.mean(), "rel MSE", rel_mse(a, b))
    assert a.mean() > 0
    assert abs(a.mean() - b.mean()) < 0.06 * b.mean()
    assert rel_mse(a, b) < 2e-2


@pytest.mark.parametrize("name", ["ball", "wall"])
def test_oracle_unbiased_orthographic_matches_fd(name):
    from helpers import fd_translation, gradient_case, rel_l2, smooth_weights, translation_seeds
    spec, mesh = gradient_case(name, 48, 48)
    c = spec.cameras[0]
    spec.cameras[0] = synth.CameraSpec(c.look_from, c.look_at, c.up, 2.6, c.height, c.width, 1)
    spp = 1024
    cfg = dict(max_bounce=2, primary_edge_hypercube_resolution=2000, mode=1, spp_interior=spp, spp_primary_edge=spp,
               spp_secondary_edge=spp, spp_pixel_boundary=spp, secondary_edge_hypercube_resolution=(2000, 6, 6))
    g = smooth_weights(48, 48)
    ad = orc.grad_dir(spec, [g], which=15, seed_verts=translation_seeds(spec, mesh), **cfg)[:3]
    fd = fd_translation(lambda s: orc.render(s, precision=1, **cfg)[0], spec, mesh, g, 1e-2)
    assert rel_l2(ad, fd) < 0.05, (ad, fd)


def test_unbiased_gradients_refuse_orthographic():
    lib = L.load()
    ws = C.c_void_p()
    assert lib.psdr_workspace_create(C.byref(ws)) == 0
    cfg = L.Config()
    for k, v in dict(n_pass=1, spp_interior=1, spp_primary_edge=1, spp_secondary_edge=1, max_bounce=1,
                     mis_light_samples=1, mis_bsdf_samples=1, primary_edge_preprocess_rounds=1,
                     secondary_edge_preprocess_rounds=1, primary_edge_hypercube_resolution=10,
                     estimator=L.EST_UNBIASED, spp_pixel_boundary=1).items():
        setattr(cfg, k, v)
    cfg.secondary_edge_hypercube_resolution[:] = [10, 1, 1]
    cam = L.CameraDesc()
    cam.type, cam.fov, cam.height, cam.width = L.CAM_ORTHOGRAPHIC, 2.0, 4, 4
    d_img = (C.c_void_p * 1)(None)
    grads = L.GradTargets()
    # a non-null fake scene handle is never dereferenced: the camera check fails first
    st = lib.psdr_render_bwd(C.c_void_p(1), ws, C.byref(cam), 1, C.byref(cfg), d_img, C.byref(grads), None)
    assert st == L.PSDR_ERR_UNSUPPORTED and b"perspective" in lib.psdr_last_error()
    assert lib.psdr_workspace_destroy(ws) == 0
