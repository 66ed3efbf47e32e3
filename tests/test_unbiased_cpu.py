"""The oracle's unbiased estimator against central finite differences of its own image.

The unbiased estimator is the material-form derivative of the path integral: interior
term with area and camera Jacobians, plus the pixel-border, silhouette and shadow-boundary
terms. Loss weights are smooth in image space so that the loss stays nearly linear over
the FD step; the renders of the FD share sample seeds (common random numbers)."""
import numpy as np
import pytest

import orc
from helpers import fd_translation, gradient_case, rel_l2, smooth_weights, translation_seeds

CFG = dict(max_bounce=2, primary_edge_hypercube_resolution=2000, mode=1)


@pytest.mark.parametrize("name,size,spp,se_res,tol", [
    ("ball", 48, 1024, 2000, 0.03),
    ("shadow", 48, 4096, 20000, 0.06),
    ("wall", 48, 1024, 2000, 0.03),
])
def test_unbiased_translation_matches_fd(name, size, spp, se_res, tol):
    spec, mesh = gradient_case(name, size, size)
    cfg = dict(CFG, spp_interior=spp, spp_primary_edge=spp, spp_secondary_edge=spp, spp_pixel_boundary=spp,
               secondary_edge_hypercube_resolution=(se_res, 6, 6))
    g = smooth_weights(size, size)
    ad = orc.grad_dir(spec, [g], which=15, seed_verts=translation_seeds(spec, mesh), **cfg)[:3]
    fd = fd_translation(lambda s: orc.render(s, precision=1, **cfg)[0], spec, mesh, g, 1e-2)
    assert rel_l2(ad, fd) < tol, (ad, fd)


def test_reference_estimator_is_not_fd_consistent():
    """The reference's own boundary formulas (world-space edge measure, no raster Jacobian,
    sample count per pixel only) are far from FD; the unbiased mode exists for this reason."""
    spec, mesh = gradient_case("ball", 32, 32)
    cfg = dict(CFG, mode=0, spp_interior=64, spp_primary_edge=16, spp_secondary_edge=16,
               secondary_edge_hypercube_resolution=(2000, 6, 6))
    g = smooth_weights(32, 32)
    ad = orc.grad_dir(spec, [g], which=7, seed_verts=translation_seeds(spec, mesh), **cfg)[:3]
    fd = fd_translation(lambda s: orc.render(s, precision=1, **cfg)[0], spec, mesh, g, 1e-2)
    assert rel_l2(ad, fd) > 1.0


@pytest.mark.parametrize("kind", [2, 1])
def test_unbiased_translation_matches_fd_under_environment_light(kind):
    """The ball case with an SH9 light (direction-dependent radiance) or a cube-map
    environment added to its area light."""
    from torch_psdr_b200 import synth
    spec, mesh = gradient_case("ball", 48, 48)
    rng = np.random.default_rng(1)
    if kind == 2:
        sh = rng.normal(scale=0.2, size=(9, 3)).astype(np.float32)
        sh[0] = [1.0, 0.8, 0.6]
        spec.lights.append(synth.LightSpec(None, None, np.zeros(3, np.float32), 2, sh9=sh))
    else:
        spec.lights.append(synth.LightSpec(None, None, np.zeros(3, np.float32), 1,
                                           cube_map=rng.uniform(0.3, 0.8, size=(6, 8, 3)).astype(np.float32)))
    spp = 1024
    cfg = dict(CFG, spp_interior=spp, spp_primary_edge=spp, spp_secondary_edge=spp, spp_pixel_boundary=spp,
               secondary_edge_hypercube_resolution=(2000, 6, 6))
    g = smooth_weights(48, 48)
    # the shadow-boundary term's samples are heavy-tailed here (one run moves its share by
    # tens of percent, about 3 % of the whole gradient), so the gradient is the mean of eight
    # independent runs and the finite differences the mean of two
    ad = np.mean([orc.grad_dir(spec, [g], which=15, seed_verts=translation_seeds(spec, mesh), seed=s, **cfg)[:3]
                  for s in range(8)], axis=0)
    fd = np.mean([fd_translation(lambda sp: orc.render(sp, precision=1, seed=s, **cfg)[0], spec, mesh, g, 1e-2)
                  for s in range(2)], axis=0)
    assert rel_l2(ad, fd) < 0.06, (ad, fd)
