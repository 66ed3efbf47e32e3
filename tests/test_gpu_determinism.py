"""Gradient accumulation is exact and order-independent (fixed-point sums in integer limbs):
backward passes are bitwise reproducible across runs. Across wavefront tile sizes, which
change which thread adds which contribution and in what order, the scattered mesh vertex and
texture gradients stay bitwise equal; the light-vertex, emission and camera gradients, which
each thread first sums over its paths in registers, agree to float rounding. The reference
accumulates with order-dependent float scatter_add (camera.h:81-85; enoki's reverse sweep)."""
import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from helpers import to_torch_scene

pytestmark = pytest.mark.gpu


def _grads(spec, **kw):
    scene, T = to_torch_scene(spec, requires_grad={"verts", "tex", "light_verts", "emit", "cam"})
    img = dr.PathIntegrator(**kw).renderD(scene)[0]
    g = torch.tensor(np.random.default_rng(7).normal(size=tuple(img.shape)), dtype=torch.float32, device="cuda")
    img.backward(g)
    torch.cuda.synchronize()
    return {k: v.grad.detach().cpu().numpy().copy() for k, v in T.items() if v.grad is not None}


@pytest.mark.parametrize("estimator", ["reference", "unbiased"])
def test_backward_is_bitwise_reproducible(cuda, estimator):
    spec = synth.sphere_scene(level=4, tex_hw=64, noise_sigma=0.02, height=96, width=96)
    kw = dict(spp_interior=16, spp_primary_edge=4, spp_secondary_edge=4, max_bounce=3, estimator=estimator,
              primary_edge_hypercube_resolution=500, secondary_edge_hypercube_resolution=[500, 3, 3])
    a = _grads(spec, **kw)
    b = _grads(spec, **kw)
    # tiles of 2^15 paths split the 147k camera paths into five tiles (the default tile holds them all)
    c = _grads(spec, tile_paths=1 << 15, **kw)
    assert set(a) == set(b) == set(c) and len(a) >= 4
    for k in a:
        assert np.abs(a[k]).max() > 0, k
        assert np.array_equal(a[k], b[k]), f"{k}: runs differ"
        if k.startswith("verts") or k.startswith("tex"):
            assert np.array_equal(a[k], c[k]), f"{k}: tile sizes differ"
        else:
            np.testing.assert_allclose(c[k], a[k], rtol=1e-5, atol=1e-6 * np.abs(a[k]).max())
