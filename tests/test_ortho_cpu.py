"""OrthographicCamera (camera.h:279-353; torch_psdr.py:161-206), CPU only.

* the oracle's orthographic image matches a far-away perspective camera whose field of
  view spans the same width at the target (rays nearly parallel);
* the oracle's unbiased estimator with an orthographic camera (camera Jacobian |n.look|,
  rays from the camera plane, silhouette velocities without the depth ratio, camera
  connections along the view direction) matches central differences;
"""
import math

import numpy as np
import pytest

import orc
from torch_psdr_b200 import synth
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
