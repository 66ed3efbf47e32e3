"""EnvLight and SH9Light (emitter.cc:94-352; scene.cc:15-53), CPU only.

Both are a 12-triangle box 1000 times the size of the scene (cameras and meshes) around
its centre, sampled by area and emitting a cube-map texel (EnvLight) or second-order
spherical harmonics of the incoming direction (SH9Light). Known answers of the oracle,
with BSDF sampling only (the reference's light samples do not mask directions below the
surface, so with them the box's lower half adds negative terms, as in the reference):
a Lambertian ground of albedo rho under a constant environment of radiance E reflects
exactly rho E per sample; under an SH9 light with only the constant coefficient c,
rho c / sqrt(4 pi); with only the Y(1,-1) = sqrt(3 / 4 pi) y coefficient k (y up, the
direction taken from the box toward the ground), -(2/3) rho k sqrt(3 / 4 pi).
"""
import math

import numpy as np

import orc
from torch_psdr_b200 import synth


def env_spec(kind, value, hw=16, cube=(6, 8)):
    gV, gF = synth.quad((0.0, 0.0), 10.0, -1.0, facing_down=False)
    ground = synth.MeshSpec(gV, gF, None, None, np.array([0.5, 0.4, 0.3], np.float32))
    cam = synth.CameraSpec(np.array([0, 2, 3], np.float32), np.array([0, -1, 0], np.float32),
                           np.array([0, 1, 0], np.float32), math.pi / 6, hw, hw)
    if kind == 1:
        light = synth.LightSpec(None, None, np.zeros(3, np.float32), 1,
                                cube_map=np.broadcast_to(np.asarray(value, np.float32), cube + (3,)).copy())
    else:
        sh = np.zeros((9, 3), np.float32)
        sh[0] = value
        light = synth.LightSpec(None, None, np.zeros(3, np.float32), 2, sh9=sh)
    return synth.SceneSpec([ground], [light], [cam])


BSDF_ONLY = dict(mis_light_samples=0, mis_bsdf_samples=1, max_bounce=2)
RHO = np.array([0.5, 0.4, 0.3])


def test_constant_environment_reflects_albedo_times_radiance():
    E = np.array([2.0, 1.0, 0.5])
    img = orc.render(env_spec(1, E), precision=1, spp_interior=4, **BSDF_ONLY)[0]
    np.testing.assert_allclose(img.reshape(-1, 3), np.broadcast_to(RHO * E, (img.size // 3, 3)), rtol=1e-6)


def test_constant_sh9_reflects_albedo_times_y00():
    c = np.array([3.0, 2.0, 1.0])
    img = orc.render(env_spec(2, c), precision=1, spp_interior=4, **BSDF_ONLY)[0]
    want = RHO * c / math.sqrt(4 * math.pi)
    np.testing.assert_allclose(img.reshape(-1, 3), np.broadcast_to(want, (img.size // 3, 3)), rtol=1e-6)


def test_sh9_linear_term_direction_convention():
    spec = env_spec(2, np.zeros(3))
    k = np.array([1.0, 2.0, 3.0])
    spec.lights[0].sh9[1] = k
    img = orc.render(spec, precision=1, spp_interior=64, **BSDF_ONLY)[0]
    want = -(2.0 / 3.0) * RHO * k * math.sqrt(0.75 / math.pi)
    got = img.reshape(-1, 3).mean(0)
    print("sh9 y term: got", got, "want", want)
    np.testing.assert_allclose(got, want, rtol=0.03)


def test_env_box_matches_scene_bounds_rule():
    lo, hi = synth.env_box([np.array([0, 2, 3], np.float32)], [np.array([[-10, -1, -10], [10, -1, 10]], np.float32)])
    # box of the camera and the mesh: (-10, -1, -10) .. (10, 2, 10); centre (0, 0.5, 0),
    # largest extent 20 -> half size 20000
    np.testing.assert_allclose(lo, [-20000.0, -19999.5, -20000.0])
    np.testing.assert_allclose(hi, [20000.0, 20000.5, 20000.0])


def _fd_check(spec, attr, seed_slice_of, shape, kw, h=1e-2):
    """Directional derivative of sum(g * image) along a random direction of a light
    parameter (the tail of the oracle's texture seeds) against central differences."""
    rng = np.random.default_rng(11)
    H, W = spec.cameras[0].height, spec.cameras[0].width
    g = rng.normal(size=(H, W, 3))
    base = getattr(spec.lights[-1], attr).copy()
    d = rng.normal(size=shape)
    ntex = sum(m.texture.size for m in spec.meshes)
    st = np.zeros((ntex + d.size, 8))
    st[ntex:, 0] = d.reshape(-1)
    ad = orc.grad_dir(spec, [g], which=1, seed_tex=st, **kw)[0]
    ph = []
    for sgn in (1, -1):
        setattr(spec.lights[-1], attr, (base + sgn * h * d).astype(np.float32))
        ph.append(float((g * orc.render(spec, precision=1, **kw)[0]).sum()))
    setattr(spec.lights[-1], attr, base)
    fd = (ph[0] - ph[1]) / (2 * h)
    print(attr, "AD", ad, "FD", fd)
    assert abs(ad) > 0
    # the radiance is linear in the parameters; what remains is the float32 rounding of
    # the perturbed parameters (about 1e-7 / h relative)
    assert abs(ad - fd) <= 1e-4 * abs(fd)


def test_cube_map_derivative_vs_finite_differences():
    spec = env_spec(1, np.array([1.0, 0.8, 0.6]))
    spec.lights[0].cube_map = np.random.default_rng(3).uniform(0.5, 1.5, size=(6, 8, 3)).astype(np.float32)
    _fd_check(spec, "cube_map", None, (6, 8, 3), dict(spp_interior=4, max_bounce=2))


def test_sh9_coefficient_derivative_vs_finite_differences():
    spec = env_spec(2, np.array([2.0, 1.0, 0.5]))
    spec.lights[0].sh9 = (np.random.default_rng(4).normal(scale=0.3, size=(9, 3)) +
                          np.array([[2.0, 1.0, 0.5]] + [[0, 0, 0]] * 8)).astype(np.float32)
    _fd_check(spec, "sh9", None, (9, 3), dict(spp_interior=4, max_bounce=2))
