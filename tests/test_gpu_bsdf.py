"""GPU parity of DiffuseBsdfMaterial (diffuse_bsdf.cc:3-88; torch_psdr.py:298-335).

A sphere with a roughness map and a normal map on a ground whose DiffuseBsdfMaterial has
a constant roughness and no normal map: per-sample radiance and images against the oracle
(same sampler streams), and every gradient term of both estimators against the oracle's
forward-mode derivatives along random directions, for the vertices, the color,
roughness and normal-map textures and the camera origin (the incoming direction of the
primary vertex depends on it).
"""
import numpy as np
import pytest
import torch

import orc
import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from helpers import rel_mse, to_torch_scene

pytestmark = pytest.mark.gpu


def bsdf_spec(height=23, width=25, tex_hw=16, level=2, normal=True, seed=4):
    """Odd image sizes: the scene's symmetry plane (x = 0, where mesh edges lie) then
    does not project onto a pixel border, where the pixel of an edge sample would hang
    on the last bit of its projection."""
    spec = synth.sphere_scene(level=level, tex_hw=tex_hw, height=height, width=width)
    rng = np.random.default_rng(seed)
    sph, ground = spec.meshes
    sph.roughness = rng.uniform(0.2, 0.9, size=(9, 7)).astype(np.float32)
    if normal:
        sph.normal = np.stack([rng.uniform(0.35, 0.65, (5, 11)), rng.uniform(0.35, 0.65, (5, 11)),
                               np.ones((5, 11))], -1).astype(np.float32)
    ground.roughness = np.array([0.6], np.float32)
    return spec


def _cfg(**kw):
    base = dict(spp_interior=4, max_bounce=3)
    base.update(kw)
    return base


@pytest.mark.parametrize("nl,nb,lv", [(1, 1, False), (2, 0, False), (0, 2, True)])
def test_bsdf_per_sample_radiance_matches_oracle(cuda, nl, nb, lv):
    spec = bsdf_spec(height=32, width=32)
    kw = _cfg(mis_light_samples=nl, mis_bsdf_samples=nb, enable_light_visable=lv)
    scene, _ = to_torch_scene(spec)
    gpu = dr.PathIntegrator(**kw).render_samples(scene).cpu().numpy().astype(np.float64)
    _, ref = orc.render(spec, precision=0, per_sample=True, **kw)
    close = np.abs(gpu - ref) <= 1e-3 * (1.0 + np.abs(ref))
    frac = close.all(axis=1).mean()
    print(f"per-sample agreement {frac:.5f}, mean |diff| {np.abs(gpu - ref).mean():.3e}")
    assert frac > 0.995
    assert rel_mse(gpu, ref) < 1e-3


def test_bsdf_image_matches_fp64_oracle(cuda):
    spec = bsdf_spec(height=48, width=48, tex_hw=64, level=3)
    kw = _cfg(spp_interior=32)
    scene, _ = to_torch_scene(spec)
    img = dr.PathIntegrator(**kw).renderC(scene)[0].cpu().numpy()
    ref = orc.render(spec, precision=1, **kw)[0]
    e = rel_mse(img, ref)
    print("image rel MSE vs FP64 oracle", e)
    assert e < 1e-4
    # roughness 0 without a normal map is the Lambertian material
    lam = bsdf_spec(height=48, width=48, tex_hw=64, level=3, normal=False)
    lam.meshes[0].roughness = np.zeros((9, 7), np.float32)
    lam.meshes[1].roughness = np.zeros(1, np.float32)
    a = dr.PathIntegrator(**kw).renderC(to_torch_scene(lam)[0])[0]
    plain = synth.sphere_scene(level=3, tex_hw=64, height=48, width=48)
    b = dr.PathIntegrator(**kw).renderC(to_torch_scene(plain)[0])[0]
    assert rel_mse(a.cpu().numpy(), b.cpu().numpy()) < 1e-8


def _seeds(spec, kinds, rng):
    """Random directions (8) over the parameters: GPU tensors by name, oracle seeds."""
    nv = [m.vertices.shape[0] for m in spec.meshes] + [l.vertices.shape[0] for l in spec.lights]
    gpu = {}
    sv = rng.normal(size=(sum(nv), 3, 8)) if "verts" in kinds else None
    if sv is not None:
        off = 0
        for i in range(len(spec.meshes)):
            gpu[f"verts{i}"] = sv[off:off + nv[i]]
            off += nv[i]
        for j in range(len(spec.lights)):
            gpu[f"lverts{j}"] = sv[off:off + nv[len(spec.meshes) + j]]
            off += nv[len(spec.meshes) + j]
    # texture elements: every color texture, then per mesh its roughness and normal map
    blocks = [(f"tex{i}", m.texture.size, "tex") for i, m in enumerate(spec.meshes)]
    for i, m in enumerate(spec.meshes):
        if m.roughness is not None:
            blocks.append((f"rough{i}", m.roughness.size, "rough"))
            if m.normal is not None:
                blocks.append((f"normal{i}", m.normal.size, "normal"))
    st = np.zeros((sum(b[1] for b in blocks), 8))
    off = 0
    for name, n, kind in blocks:
        if kind in kinds:
            st[off:off + n] = rng.normal(size=(n, 8))
            gpu[name] = st[off:off + n]
        off += n
    sc = rng.normal(size=(len(spec.cameras), 3, 8)) if "cam" in kinds else None
    if sc is not None:
        for k in range(len(spec.cameras)):
            gpu[f"cam{k}"] = sc[k]
    return gpu, dict(seed_verts=sv, seed_tex=st, seed_cam=sc)


BSDF_GRAD_CASES = [
    # (estimator, terms bitmask, parameters)
    ("reference", 1, ("tex", "rough", "normal")),
    ("reference", 1, ("verts",)),
    ("reference", 1, ("cam",)),
    ("reference", 2, ("verts",)),
    ("reference", 4, ("verts",)),
    ("unbiased", 1, ("verts",)),
    ("unbiased", 1, ("rough", "normal", "cam")),
    ("unbiased", 2, ("verts",)),
    ("unbiased", 4, ("verts",)),
    ("unbiased", 8, ("verts",)),
    # the BRDF-jump term (gradient_terms bit 16; in the unbiased default for these scenes)
    ("unbiased", 16, ("verts",)),
    ("unbiased", 16, ("normal", "cam")),
]


@pytest.mark.parametrize("estimator,terms,kinds", BSDF_GRAD_CASES)
def test_bsdf_gradient_terms_match_oracle(cuda, estimator, terms, kinds):
    spec = bsdf_spec()
    kw = _cfg(spp_interior=4, spp_primary_edge=4, spp_secondary_edge=4, primary_edge_hypercube_resolution=500,
              secondary_edge_hypercube_resolution=[500, 3, 3])
    unb = estimator == "unbiased"
    if unb:
        kw.update(spp_pixel_boundary=4)
    rng = np.random.default_rng(3)
    gseeds, oseeds = _seeds(spec, kinds, rng)
    params = set()
    for k in kinds:
        params |= {"verts": {"verts", "light_verts"}, "tex": {"tex"}, "rough": {"rough"}, "normal": {"normal"},
                   "cam": {"cam"}}[k]
    scene, T = to_torch_scene(spec, requires_grad=params)
    integ = dr.PathIntegrator(gradient_terms=terms, estimator=estimator, **kw)
    img = integ.renderD(scene)[0]
    dLdI = np.random.default_rng(5).normal(size=tuple(img.shape))
    img.backward(torch.tensor(dLdI, dtype=torch.float32, device="cuda"))
    got = np.zeros(8)
    for name, seed in gseeds.items():
        g = T[name].grad.detach().cpu().numpy().astype(np.float64).reshape(-1)
        got += g @ seed.reshape(g.shape[0], 8)
    ref = orc.grad_dir(spec, [dLdI], which=terms, mode=1 if unb else 0, **oseeds, **kw)
    err = np.abs(got - ref) / (np.abs(ref).max() + 1e-30)
    print(f"{estimator} terms={terms} {kinds}: gpu {got[:4]} oracle {ref[:4]} max rel {err.max():.2e}")
    assert np.abs(ref).max() > 0
    # the direct (shadow-boundary) term samples its guiding cells in fp64 and traces
    # bounce chains: small differences in a few samples move it more than the others
    # the BRDF-jump arc rays start on the surface, like the shadow-boundary rays
    assert err.max() < (1e-2 if terms in (4, 16) else 2e-3)


def test_unbiased_default_terms_include_brdf_jumps(cuda):
    """With a DiffuseBsdfMaterial mesh in the scene, the unbiased estimator's default
    gradient terms (gradient_terms=0) are the six terms plus the BRDF jumps (bit 16)."""
    spec = bsdf_spec()
    kw = _cfg(spp_interior=4, spp_primary_edge=2, spp_secondary_edge=2, primary_edge_hypercube_resolution=500,
              secondary_edge_hypercube_resolution=[500, 3, 3], spp_pixel_boundary=2)
    dLdI = None
    grads = {}
    for terms in (0, 111 | 16, 111):
        scene, T = to_torch_scene(spec, requires_grad={"verts"})
        img = dr.PathIntegrator(gradient_terms=terms, estimator="unbiased", **kw).renderD(scene)[0]
        if dLdI is None:
            dLdI = torch.tensor(np.random.default_rng(7).normal(size=tuple(img.shape)), dtype=torch.float32,
                                device="cuda")
        img.backward(dLdI)
        grads[terms] = T["verts0"].grad.clone()
    assert torch.equal(grads[0], grads[111 | 16])
    assert not torch.equal(grads[0], grads[111])
