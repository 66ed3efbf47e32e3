"""GPU parity of OrthographicCamera (camera.h:279-353; torch_psdr.py:161-206).

Per-sample radiance and images against the oracle (same sampler streams), and the
reference estimator's gradient terms against the oracle's forward-mode derivatives: the
interior term, the primary-edge term (whose ray origin, the edge point's foot on the
camera plane, moves with the edge point and the camera) and the direct-edge term (whose
visibility ray runs along the view direction), for the vertices and the camera origin;
also with a DiffuseBsdfMaterial, whose value depends on the incoming direction; and the
unbiased estimator's four terms (orthographic camera Jacobian, camera-plane border and
silhouette rays, camera connections along the view direction).
"""
import numpy as np
import pytest
import torch

import orc
import torch_psdr_b200 as dr
from helpers import rel_mse, to_torch_scene
from test_gpu_bsdf import _seeds, bsdf_spec
from test_ortho_cpu import ortho_spec

pytestmark = pytest.mark.gpu


def _to_ortho(spec, view_width=3.0):
    c = spec.cameras[0]
    spec.cameras[0] = type(c)(c.look_from, c.look_at, c.up, float(view_width), c.height, c.width, 1)
    return spec


def test_ortho_per_sample_radiance_matches_oracle(cuda):
    spec = ortho_spec(height=32, width=32, level=3, tex_hw=64)
    kw = dict(spp_interior=4, max_bounce=3)
    scene, _ = to_torch_scene(spec)
    gpu = dr.PathIntegrator(**kw).render_samples(scene).cpu().numpy().astype(np.float64)
    _, ref = orc.render(spec, precision=0, per_sample=True, **kw)
    close = np.abs(gpu - ref) <= 1e-3 * (1.0 + np.abs(ref))
    frac = close.all(axis=1).mean()
    print(f"per-sample agreement {frac:.5f}, mean |diff| {np.abs(gpu - ref).mean():.3e}")
    assert frac > 0.995
    assert rel_mse(gpu, ref) < 1e-3


def test_ortho_image_matches_fp64_oracle(cuda):
    spec = ortho_spec(height=48, width=40, level=3, tex_hw=64)
    kw = dict(spp_interior=32, max_bounce=3)
    scene, _ = to_torch_scene(spec)
    img = dr.PathIntegrator(**kw).renderC(scene)[0].cpu().numpy()
    ref = orc.render(spec, precision=1, **kw)[0]
    e = rel_mse(img, ref)
    print("image rel MSE vs FP64 oracle", e)
    assert img.mean() > 0 and e < 1e-4


ORTHO_GRAD_CASES = [
    # (material, estimator, terms bitmask, parameters)
    ("diffuse", "reference", 1, ("verts",)),
    ("diffuse", "reference", 2, ("verts",)),
    ("diffuse", "reference", 2, ("cam",)),
    ("diffuse", "reference", 4, ("verts",)),
    ("bsdf", "reference", 1, ("verts", "cam")),
    ("bsdf", "reference", 2, ("verts",)),
    ("diffuse", "unbiased", 1, ("verts", "cam")),
    ("diffuse", "unbiased", 2, ("verts", "cam")),
    ("diffuse", "unbiased", 4, ("verts",)),
    ("diffuse", "unbiased", 8, ("verts", "cam")),
    ("bsdf", "unbiased", 1, ("verts",)),
]


@pytest.mark.parametrize("material,estimator,terms,kinds", ORTHO_GRAD_CASES)
def test_ortho_gradient_terms_match_oracle(cuda, material, estimator, terms, kinds):
    spec = ortho_spec() if material == "diffuse" else _to_ortho(bsdf_spec())
    kw = dict(spp_interior=4, max_bounce=3, spp_primary_edge=4, spp_secondary_edge=4,
              primary_edge_hypercube_resolution=500, secondary_edge_hypercube_resolution=[500, 3, 3])
    unb = estimator == "unbiased"
    if unb:
        kw.update(spp_pixel_boundary=4)
    gseeds, oseeds = _seeds(spec, kinds, np.random.default_rng(3))
    params = set()
    for k in kinds:
        params |= {"verts": {"verts", "light_verts"}, "cam": {"cam"}}[k]
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
    print(f"ortho {material} {estimator} terms={terms} {kinds}: gpu {got[:4]} oracle {ref[:4]} max rel {err.max():.2e}")
    assert np.abs(ref).max() > 0
    assert err.max() < (1e-2 if terms == 4 else 2e-3)
