"""The seeded synthetic workloads (torch_psdr_b200.synth) have the sizes of the
benchmark configurations they stand in for (the reference's OBJ assets are absent):
the forward scene (level-3 icosphere, 1,284 triangles with ground and light), the
geometry-gradient scene (level-5 icosphere, 10,242 vertices, 20,484 triangles), the
multi-view scenes (geodesic spheres of 20 n^2 = 5,120 / 50,000 / 200,000 triangles,
64 orbit cameras of 128..512 pixels a side) and the large scene (16 level-6
icospheres, 1,310,724 triangles with ground and light). Also checked: the camera,
light and ground that the configurations share, and the seeded inputs' determinism."""
import math

import numpy as np

from torch_psdr_b200 import synth


def _tris(spec):
    return sum(len(m.faces) for m in spec.meshes) + sum(len(l.faces) for l in spec.lights if l.faces is not None)


def test_forward_and_gradient_scenes():
    fwd = synth.sphere_scene(level=3, tex_hw=256, height=128, width=128)
    assert _tris(fwd) == 1284
    assert fwd.meshes[0].texture.shape == (256, 256, 3)
    tex = fwd.meshes[0].texture
    assert 0.2 <= tex.min() and tex.max() <= 0.8
    cam = fwd.cameras[0]
    np.testing.assert_array_equal(cam.look_from, [0, 0.5, 4])
    assert cam.vfov == math.pi / 4 and (cam.height, cam.width) == (128, 128)
    np.testing.assert_array_equal(fwd.lights[0].emit, [20, 20, 20])
    np.testing.assert_array_equal(fwd.meshes[1].texture, [0.5, 0.5, 0.5])
    geo = synth.sphere_scene(level=5, tex_hw=256, noise_sigma=0.02, noise_seed=2, height=512, width=512)
    assert _tris(geo) == 20484 and len(geo.meshes[0].vertices) == 10242
    r = np.linalg.norm(geo.meshes[0].vertices, axis=1)
    assert abs(r.mean() - 1) < 0.01 and 0.015 < r.std() < 0.025   # radial noise N(0, 0.02)
    again = synth.sphere_scene(level=5, tex_hw=256, noise_sigma=0.02, noise_seed=2, height=512, width=512)
    np.testing.assert_array_equal(geo.meshes[0].vertices, again.meshes[0].vertices)
    np.testing.assert_array_equal(geo.meshes[0].texture, again.meshes[0].texture)


def test_multiview_scenes_and_cameras():
    for n, tris in ((16, 5120), (50, 50000), (100, 200000)):
        assert len(synth.sphere_scene(freq=n, tex_hw=8).meshes[0].faces) == tris
    cams = synth.orbit_cameras(64, 4.0, seed=3, size_lo=128, size_hi=512)
    assert len(cams) == 64
    assert all(128 <= c.height <= 512 and 128 <= c.width <= 512 for c in cams)
    assert all(abs(np.linalg.norm(c.look_from) - 4.0) < 1e-5 for c in cams)


def test_large_scene():
    spec = synth.large_scene(height=8, width=8)
    assert _tris(spec) == 1310724 and len(spec.meshes) == 17
    assert all(m.texture.shape == (512, 512, 3) for m in spec.meshes[:16])
    centres = np.stack([m.vertices.mean(0) for m in spec.meshes[:16]])
    assert (np.abs(centres) < 5.2).all()
