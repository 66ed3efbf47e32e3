"""Camera gradients beyond the origin: look_at, up, vfov, and look_from through the camera's
basis (torch_psdr.py:145-152 makes all four differentiable; camera.h:7-64 builds the basis).

Unbiased estimator: the derivative of the image, checked against central differences of
renders with common random numbers. Reference estimator: zeros, as the reference's tape
has no path from these inputs to the image. Orthographic cameras refuse them."""
import math

import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from helpers import gradient_case, rel_l2, smooth_weights, to_torch_scene

pytestmark = pytest.mark.gpu


def _camera_tensors(c, dev="cuda"):
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    return t(c.look_from), t(c.look_at), t(c.up), t([c.vfov])


def _scene_with_camera(spec, cam_params):
    scene, _ = to_torch_scene(spec)
    c = spec.cameras[0]
    scene.cameras = [dr.PerspectiveCamera(*cam_params, c.height, c.width)]
    return scene


def _phi_fd(spec, integ, g, base, h):
    """Central differences of sum(g * image) in each of the ten camera scalars."""
    flat = torch.cat([p.detach().reshape(-1) for p in base])
    out = []
    for j in range(10):
        vals = []
        for sgn in (1.0, -1.0):
            f = flat.clone()
            f[j] += sgn * h[j]
            params = (f[0:3], f[3:6], f[6:9], f[9:10])
            with torch.no_grad():
                img = integ.renderC(_scene_with_camera(spec, params))[0]
            vals.append(float((img.double() * g).sum()))
        out.append((vals[0] - vals[1]) / (2 * h[j]))
    return np.array(out)


def _lens_ad(spec, integ, g):
    params = [p.clone().requires_grad_(True) for p in _camera_tensors(spec.cameras[0])]
    img = integ.renderD(_scene_with_camera(spec, params))[0]
    img.backward(g.float())
    return np.concatenate([p.grad.double().cpu().numpy().reshape(-1) for p in params])


@pytest.mark.parametrize("name", ["ball", "wall"])
def test_camera_lens_gradient_vs_finite_differences(cuda, name):
    size = 64
    spec, _ = gradient_case(name, size, size)
    # look slightly off-axis with a tilted up vector, so every parameter moves the image
    c = spec.cameras[0]
    c.look_at = np.array([0.1, -0.05, 0.0], np.float32)
    c.up = np.array([0.1, 1.0, 0.05], np.float32)
    g = torch.tensor(smooth_weights(size, size), dtype=torch.float64, device="cuda")
    kw = dict(spp_interior=256, spp_primary_edge=64, spp_secondary_edge=4096, spp_pixel_boundary=64,
              max_bounce=2, estimator="unbiased")
    ad = np.mean([_lens_ad(spec, dr.PathIntegrator(seed=s, **kw), g) for s in (1, 2)], axis=0)
    h = [2e-3] * 9 + [1e-3]
    fd = _phi_fd(spec, dr.PathIntegrator(**dict(kw, spp_interior=1024, seed=1)), g,
                 _camera_tensors(spec.cameras[0]), h)
    e = rel_l2(ad, fd)
    print(f"{name}: AD {np.round(ad, 3)}\nFD {np.round(fd, 3)}\nrel L2 {e:.4f}")
    assert e < 0.05
    # the part that does not move the image: up along the view direction, and look_at
    # along the view direction, have (near) zero derivative on both sides
    d = (c.look_from - c.look_at) / np.linalg.norm(c.look_from - c.look_at)
    assert abs(float(ad[3:6] @ d)) < 0.05 * np.linalg.norm(ad[3:6]) + 1e-9


def test_camera_translation_of_from_and_at_is_the_origin_gradient(cuda):
    """Moving look_from and look_at together translates the camera: the sum of their
    gradients is the basis-fixed origin gradient, and that equals minus the sum of every
    vertex gradient (moving the scene the other way)."""
    spec, _ = gradient_case("ball", 32, 32)
    scene, T = to_torch_scene(spec, requires_grad={"verts", "light_verts"})
    params = [p.clone().requires_grad_(True) for p in _camera_tensors(spec.cameras[0])]
    c = spec.cameras[0]
    scene.cameras = [dr.PerspectiveCamera(*params, c.height, c.width)]
    integ = dr.PathIntegrator(spp_interior=16, spp_primary_edge=16, spp_secondary_edge=64, spp_pixel_boundary=8,
                              max_bounce=2, estimator="unbiased")
    img = integ.renderD(scene)[0]
    img.backward(torch.tensor(np.random.default_rng(5).normal(size=tuple(img.shape)), dtype=torch.float32,
                              device="cuda"))
    cam = (params[0].grad + params[1].grad).double().cpu().numpy()
    tot = sum(v.grad.double().sum(0).cpu().numpy() for k, v in T.items()
              if (k.startswith("verts") or k.startswith("lverts")) and v.grad is not None)
    scale = np.abs(tot).max()
    print(f"camera {cam} -sum(vertices) {-tot}")
    np.testing.assert_allclose(cam, -tot, rtol=0, atol=2e-3 * scale)


def test_reference_estimator_lens_gradients_are_zero(cuda):
    """The reference's renderD never uses the camera ray's direction after the hit, so its
    look_at, up and vfov gradients are zero and look_from's is the origin's."""
    spec, _ = gradient_case("ball", 24, 24)
    params = [p.clone().requires_grad_(True) for p in _camera_tensors(spec.cameras[0])]
    integ = dr.PathIntegrator(spp_interior=4, spp_primary_edge=4, spp_secondary_edge=4, max_bounce=2)
    img = integ.renderD(_scene_with_camera(spec, params))[0]
    img.sum().backward()
    for p in params[1:]:
        assert torch.count_nonzero(p.grad) == 0
    assert torch.count_nonzero(params[0].grad) > 0


def test_orthographic_lens_gradients_are_refused(cuda):
    spec, _ = gradient_case("wall", 16, 16)
    scene, _ = to_torch_scene(spec)
    c = spec.cameras[0]
    lf, at, up, _ = _camera_tensors(c)
    width = torch.tensor([2.0], device="cuda", requires_grad=True)
    scene.cameras = [dr.OrthographicCamera(lf, at, up, width, c.height, c.width)]
    with pytest.raises(NotImplementedError):
        dr.PathIntegrator(estimator="unbiased").renderD(scene)


def test_batched_lens_gradients_match_plain(cuda):
    spec, _ = gradient_case("ball", 32, 32)
    kw = dict(spp_interior=8, spp_primary_edge=8, spp_secondary_edge=16, spp_pixel_boundary=8, max_bounce=2,
              estimator="unbiased")
    g = torch.tensor(np.random.default_rng(2).normal(size=(32, 32, 3)), dtype=torch.float32, device="cuda")
    params = [p.clone().requires_grad_(True) for p in _camera_tensors(spec.cameras[0])]
    integ = dr.PathIntegrator(**kw)
    integ.renderD(_scene_with_camera(spec, params))[0].backward(g)
    plain = [p.grad.clone() for p in params]
    for p in params:
        p.grad = None
    batch = dr.BatchRender(integ, [_scene_with_camera(spec, params)])
    batch.renderD()[0].backward(g)
    torch.cuda.synchronize()
    for a, b in zip(plain, params):
        torch.testing.assert_close(b.grad, a, rtol=1e-4, atol=1e-5 * float(a.abs().max()) + 1e-7)
