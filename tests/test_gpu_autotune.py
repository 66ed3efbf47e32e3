"""BVH leaf sizes and the autotuner: every leaf size gives the brute-force hits bit for
bit, and tuning changes no image (hits and films do not depend on tile or leaf size)."""
import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from torch_psdr_b200 import _lib as L
from helpers import to_torch_scene
from test_gpu_parity import _stream, gpu_intersect
from test_oracle_cpu import _random_rays

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("leaf", [1, 2, 4, 8])
def test_leaf_sizes_match_brute_force(cuda, leaf):
    spec = synth.sphere_scene(level=5, noise_sigma=0.02, height=8, width=8)
    scene, _ = to_torch_scene(spec)
    L.check(L.load().psdr_scene_set_leaf_size(scene.handle, leaf, _stream()), "leaf")
    rays = _random_rays(spec, 20000, 13)
    t_bf, b_bf, tt_bf = gpu_intersect(scene, rays, 1)
    assert (t_bf >= 0).mean() > 0.3
    for mode in (0, 2):  # one-shot traversal, the wavefront kernel's resumable traversal
        t_bvh, b_bvh, tt_bvh = gpu_intersect(scene, rays, mode)
        np.testing.assert_array_equal(t_bvh, t_bf)
        np.testing.assert_array_equal(b_bvh, b_bf)
        np.testing.assert_array_equal(tt_bvh, tt_bf)


def test_tiny_scene_with_large_leaves(cuda):
    """Fewer triangles than the leaf size: the root stays an internal node."""
    _, light = synth.ground_and_light()
    spec = synth.SceneSpec([synth.MeshSpec(*synth.quad((0.3, 0.2), 2.0, 0.1, False), None, None,
                                           np.array([0.5, 0.5, 0.5], np.float32))], [light],
                           [synth.default_camera(8, 8)])
    scene, _ = to_torch_scene(spec)
    L.check(L.load().psdr_scene_set_leaf_size(scene.handle, 8, _stream()), "leaf")
    rays = _random_rays(spec, 4000, 17)
    b = gpu_intersect(scene, rays, 1)
    for mode in (0, 2):
        a = gpu_intersect(scene, rays, mode)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_autotune_keeps_images(cuda):
    spec = synth.sphere_scene(level=4, tex_hw=64, height=96, width=80)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(spp_interior=8, max_bounce=3)
    before = integ.renderC(scene)[0].clone()
    info = integ.autotune(scene)
    print("autotune", info)
    assert info["tile_paths"] in (1 << 18, 1 << 19, 1 << 20, 1 << 21)
    assert info["leaf_size"] in (1, 2, 4)
    assert info["trace_queue"] in (4, 6, 8)
    assert info["forward_ms"] > 0
    after = integ.renderC(scene)[0]
    torch.cuda.synchronize()
    assert torch.equal(before, after)
