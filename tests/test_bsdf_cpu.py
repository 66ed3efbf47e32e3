"""The oracle's DiffuseBsdfMaterial (diffuse_bsdf.cc:3-88), CPU only.

* roughness 0 without a normal map is the Lambertian DiffuseMaterial, bit for bit;
* the roughness derivative of the interior term (forward-mode duals) against central
  finite differences with common random numbers (the roughness does not move the
  sampled directions, so the estimate is smooth in it);
* a normal map moves the image;
* the unbiased estimator's BRDF-jump term (translation gradients against central
  differences: a wall at roughness 0.6, depth 2; a ball before a wall at 0.9, depth 3).
"""
import numpy as np
import pytest

import orc
from torch_psdr_b200 import synth
from helpers import rel_mse


def _spec(rough, normal=None, hw=24):
    spec = synth.sphere_scene(level=2, tex_hw=16, height=hw, width=hw)
    spec.meshes[0].roughness = rough
    spec.meshes[0].normal = normal
    spec.meshes[1].roughness = np.array([0.0], np.float32)
    return spec


KW = dict(spp_interior=4, max_bounce=3)


def test_zero_roughness_is_lambertian():
    a = orc.render(_spec(np.zeros((5, 5), np.float32)), precision=1, **KW)[0]
    b = orc.render(synth.sphere_scene(level=2, tex_hw=16, height=24, width=24), precision=1, **KW)[0]
    np.testing.assert_array_equal(a, b)


def test_roughness_derivative_vs_finite_differences():
    rng = np.random.default_rng(1)
    rough = rng.uniform(0.2, 0.9, size=(5, 5)).astype(np.float32)
    spec = _spec(rough)
    g = rng.normal(size=(24, 24, 3))
    ncol = sum(m.texture.size for m in spec.meshes)
    st = np.zeros((ncol + rough.size + 1, 8))
    st[ncol:ncol + rough.size, 0] = rng.normal(size=rough.size)
    ad = orc.grad_dir(spec, [g], which=1, seed_tex=st, **KW)[0]
    d = st[ncol:ncol + rough.size, 0].reshape(rough.shape)
    h = 1e-3
    ph = []
    for sgn in (1, -1):
        spec.meshes[0].roughness = (rough + sgn * h * d).astype(np.float32)
        ph.append(float((g * orc.render(spec, precision=1, **KW)[0]).sum()))
    fd = (ph[0] - ph[1]) / (2 * h)
    print("roughness derivative AD", ad, "FD", fd)
    assert abs(ad) > 0
    assert abs(ad - fd) <= 2e-2 * abs(fd)


def test_normal_map_changes_the_image():
    rough = np.full((5, 5), 0.5, np.float32)
    flat = np.concatenate([np.full((4, 4, 2), 0.5), np.ones((4, 4, 1))], -1).astype(np.float32)
    tilt = flat.copy()
    tilt[..., 0] = 0.7
    a = orc.render(_spec(rough), precision=1, **KW)[0]
    b = orc.render(_spec(rough, flat), precision=1, **KW)[0]
    c = orc.render(_spec(rough, tilt), precision=1, **KW)[0]
    # (0.5, 0.5, 1) maps to the geometric normal: the same sampled directions and values
    assert rel_mse(b, a) < 1e-10
    assert rel_mse(c, a) > 1e-4


def test_zero_roughness_derivatives_are_lambertian():
    """With roughness 0 the rough-diffuse BRDF is color / pi (b = 0, no jump), so both
    estimators' derivatives equal DiffuseMaterial's (the unbiased one with its BRDF-jump term, which
    vanishes)."""
    from helpers import translation_seeds
    rng = np.random.default_rng(2)
    g = rng.normal(size=(24, 24, 3))
    for mode in (0, 1):
        kw = dict(KW, mode=mode, spp_primary_edge=2, spp_secondary_edge=2, spp_pixel_boundary=2,
                  primary_edge_hypercube_resolution=200, secondary_edge_hypercube_resolution=(200, 3, 3))
        a = orc.grad_dir(_spec(np.zeros((5, 5), np.float32)), [g], which=31 if mode else 7,
                         seed_verts=translation_seeds(_spec(np.zeros((5, 5), np.float32)), 0), **kw)
        lam = synth.sphere_scene(level=2, tex_hw=16, height=24, width=24)
        b = orc.grad_dir(lam, [g], which=31 if mode else 7, seed_verts=translation_seeds(lam, 0), **kw)
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())


@pytest.mark.parametrize("name,rough,depth", [("wall", 0.6, 2), ("ball", 0.9, 3)])
def test_unbiased_bsdf_jump_term_matches_fd(name, rough, depth):
    """The rough-diffuse BRDF jumps across t = V.L - (N.L)(N.V) = 0. Without the jump term
    (terms 1, 2, 4, 8) the unbiased estimator misses that boundary's motion (15-31 %
    against central differences here); with it (term 16) it matches."""
    from helpers import fd_translation, gradient_case, rel_l2, smooth_weights, translation_seeds
    spec, mesh = gradient_case(name, 48, 48)
    for m in spec.meshes:
        m.roughness = np.array([rough], np.float32)
    spp = 1024
    cfg = dict(max_bounce=depth, primary_edge_hypercube_resolution=2000, mode=1, spp_interior=spp,
               spp_primary_edge=spp, spp_secondary_edge=spp, spp_pixel_boundary=spp,
               secondary_edge_hypercube_resolution=(2000, 6, 6))
    g = smooth_weights(48, 48)
    seeds = translation_seeds(spec, mesh)
    without = orc.grad_dir(spec, [g], which=15, seed_verts=seeds, **cfg)[:3]
    ad = orc.grad_dir(spec, [g], which=31, seed_verts=seeds, **cfg)[:3]
    fd = fd_translation(lambda s: orc.render(s, precision=1, **cfg)[0], spec, mesh, g, 1e-2)
    print(f"{name} roughness {rough} depth {depth}: without the jump term {rel_l2(without, fd):.3f}, "
          f"with it {rel_l2(ad, fd):.4f} rel L2 against FD")
    assert rel_l2(without, fd) > 0.1
    assert rel_l2(ad, fd) < 0.03, (ad, fd)
