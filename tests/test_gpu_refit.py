"""BVH refit (psdr_scene_refit): after vertex moves the refit tree gives the closest hits
of a brute-force intersector bit for bit, so renders equal those of a freshly built
scene, over consecutive refits."""
import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from helpers import to_torch_scene
from test_gpu_parity import gpu_intersect
from test_oracle_cpu import _random_rays

pytestmark = pytest.mark.gpu


def _deform(V, k):
    r = np.linalg.norm(V, axis=1, keepdims=True)
    wobble = 1.0 + 0.08 * np.sin(3.0 * V[:, :1] + k) * np.cos(2.0 * V[:, 1:2] - k)
    return (V / r * r * wobble + np.array([0.05 * k, -0.03 * k, 0.02], np.float32)).astype(np.float32)


def test_refit_matches_fresh_build(cuda):
    spec = synth.sphere_scene(level=4, noise_sigma=0.02, tex_hw=32, height=40, width=48)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(spp_interior=8, max_bounce=3)
    base = spec.meshes[0].vertices.copy()
    for k in (1, 2):
        moved = _deform(base, k)
        scene.meshes[0].set_vertices(torch.tensor(moved, device="cuda"))
        scene.update(refit=True)
        spec.meshes[0].vertices = moved
        rays = _random_rays(spec, 20000, 10 + k)
        t_bvh, b_bvh, tt_bvh = gpu_intersect(scene, rays, False)
        t_bf, b_bf, tt_bf = gpu_intersect(scene, rays, True)
        assert (t_bf >= 0).mean() > 0.3
        np.testing.assert_array_equal(t_bvh, t_bf)
        np.testing.assert_array_equal(b_bvh, b_bf)
        np.testing.assert_array_equal(tt_bvh, tt_bf)
        fresh, _ = to_torch_scene(spec)
        a = integ.renderC(scene)[0]
        b = integ.renderC(fresh)[0]
        assert torch.equal(a, b), k
