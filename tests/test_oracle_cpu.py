"""CPU tests of the oracle against the known-answer vectors and its own invariants."""
import json
import os

import numpy as np
import pytest

import orc
from torch_psdr_b200 import synth
from helpers import rel_mse

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_pcg32_published_vector():
    with open(os.path.join(GOLDEN, "pcg32_demo.json")) as f:
        g = json.load(f)
    assert [int(x) for x in orc.pcg32(g["initstate"], g["initseq"], len(g["outputs"]))] == g["outputs"]


def test_sampler_streams_golden():
    g = np.load(os.path.join(GOLDEN, "sampler_streams.npz"))
    for i, row in zip(g["index"], g["draws"]):
        np.testing.assert_array_equal(orc.sampler_floats(int(i), row.shape[0]), row)
    d = g["draws"]
    assert np.all((d >= 0) & (d < 1))
    assert len({tuple(r) for r in d}) == d.shape[0]


def test_oracle_tiny_golden():
    spec = synth.sphere_scene(level=1, tex_hw=8, tex_seed=0, height=16, width=16)
    img = orc.render(spec, precision=1, spp_interior=4, max_bounce=3)[0]
    np.testing.assert_allclose(img, np.load(os.path.join(GOLDEN, "oracle_tiny.npz"))["image"], rtol=0, atol=1e-12)


def test_oracle_ext_golden():
    """DiffuseBsdfMaterial, orthographic camera, EnvLight and SH9Light renders of the
    oracle against their fixtures (tests/golden/make_golden.py)."""
    import importlib.util
    spec_path = os.path.join(GOLDEN, "make_golden.py")
    mod_spec = importlib.util.spec_from_file_location("make_golden", spec_path)
    mg = importlib.util.module_from_spec(mod_spec)
    mod_spec.loader.exec_module(mg)
    want = np.load(os.path.join(GOLDEN, "oracle_ext.npz"))
    for name, s in mg.ext_specs().items():
        img = orc.render(s, precision=1, spp_interior=4, max_bounce=3)[0]
        assert img.mean() > 0, name
        np.testing.assert_allclose(img, want[name], rtol=0, atol=1e-12, err_msg=name)


def test_oracle_gradient_golden():
    """Every gradient term of both estimators (the unbiased one's BRDF jumps included) on
    the tiny scenes, as directional derivatives, against their fixtures
    (tests/golden/make_golden.py grad). Per-sample contributions are summed in sample
    order, so the values do not depend on the thread count."""
    import importlib.util
    spec_path = os.path.join(GOLDEN, "make_golden.py")
    mod_spec = importlib.util.spec_from_file_location("make_golden", spec_path)
    mg = importlib.util.module_from_spec(mod_spec)
    mod_spec.loader.exec_module(mg)
    want = np.load(os.path.join(GOLDEN, "oracle_grad.npz"))
    got = mg.grad_pins()
    assert sorted(got) == sorted(want.files)
    for name in want.files:
        assert np.abs(want[name]).max() > 0, name
        np.testing.assert_allclose(got[name], want[name], rtol=1e-12, atol=1e-12 * np.abs(want[name]).max(),
                                   err_msg=name)


def _random_rays(spec, n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-3, 3, size=(n, 3))
    tgt = rng.uniform(-1.2, 1.2, size=(n, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # rays aimed exactly at vertices and edge midpoints (ties and watertightness)
    V = spec.meshes[0].vertices.astype(np.float64)
    F = spec.meshes[0].faces
    k = n // 4
    pick = rng.integers(0, V.shape[0], size=k)
    o[:k] = V[pick] * 3.0 + rng.normal(size=(k, 3)) * 0.01
    d[:k] = V[pick] - o[:k]
    fe = rng.integers(0, F.shape[0], size=k)
    mid = 0.5 * (V[F[fe, 0]] + V[F[fe, 1]])
    o[k:2 * k] = mid * 2.5
    d[k:2 * k] = mid - o[k:2 * k]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], axis=1).astype(np.float32)


@pytest.mark.parametrize("level", [1, 3])
def test_oracle_bvh_equals_bruteforce(level):
    spec = synth.sphere_scene(level=level, height=8, width=8, noise_sigma=0.02)
    rays = _random_rays(spec, 4000, 7)
    t0, b0, tt0 = orc.intersect(spec, rays, use_bvh=False)
    t1, b1, tt1 = orc.intersect(spec, rays, use_bvh=True)
    np.testing.assert_array_equal(t0, t1)
    np.testing.assert_array_equal(b0, b1)
    np.testing.assert_array_equal(tt0, tt1)
    assert (t0 >= 0).mean() > 0.3


def test_edges_topology():
    spec = synth.sphere_scene(level=2, height=8, width=8)
    v01, geo = orc.edges(spec)
    nf_sphere = spec.meshes[0].faces.shape[0]
    # closed sphere: 3F/2 edges; each quad (ground, light): 4 boundary + 1 diagonal
    assert v01.shape[0] == 3 * nf_sphere // 2 + 5 + 5
    assert np.all(v01[:, 0] < v01[:, 1])
    # sorted (min, max) order
    key = v01[:, 0].astype(np.int64) * 10**7 + v01[:, 1]
    assert np.all(np.diff(key) > 0)
    lens = geo[:, 15]
    np.testing.assert_allclose(lens, np.linalg.norm(geo[:, 0:3] - geo[:, 3:6], axis=1), rtol=1e-6)
    # unit normals
    np.testing.assert_allclose(np.linalg.norm(geo[:, 9:12], axis=1), 1.0, rtol=1e-5)


def test_float_and_double_instances_agree():
    spec = synth.sphere_scene(level=2, tex_hw=32, height=24, width=24)
    a = orc.render(spec, precision=0, spp_interior=4)[0]
    b = orc.render(spec, precision=1, spp_interior=4)[0]
    assert rel_mse(a, b) < 1e-6


def test_n_pass_identical_passes():
    spec = synth.sphere_scene(level=1, tex_hw=8, height=12, width=12)
    a = orc.render(spec, precision=1, spp_interior=2)[0]
    b = orc.render(spec, precision=1, spp_interior=2, n_pass=3)[0]
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


def test_dual_texture_derivative_matches_fd():
    spec = synth.sphere_scene(level=2, tex_hw=8, height=16, width=16)
    rng = np.random.default_rng(0)
    dLdI = [rng.normal(size=(16, 16, 3))]
    ntex = 8 * 8 * 3 + 3  # sphere uv texture + ground constant
    seeds = np.zeros((ntex, 8))
    seeds[:, 0] = rng.normal(size=ntex)
    d = orc.grad_dir(spec, dLdI, which=1, seed_tex=seeds, spp_interior=4)[0]
    h = 1e-4
    tex0 = spec.meshes[0].texture.copy()
    g0 = spec.meshes[1].texture.copy()
    def phi(eps):
        spec.meshes[0].texture = (tex0 + eps * seeds[:192, 0].reshape(8, 8, 3)).astype(np.float32)
        spec.meshes[1].texture = (g0 + eps * seeds[192:, 0]).astype(np.float32)
        return float(np.sum(dLdI[0] * orc.render(spec, precision=1, spp_interior=4)[0]))
    fd = (phi(h) - phi(-h)) / (2 * h)
    spec.meshes[0].texture, spec.meshes[1].texture = tex0, g0
    assert abs(d - fd) <= 2e-3 * max(abs(fd), 1e-6), (d, fd)


def test_dual_light_emission_derivative_is_linear():
    # the image is linear in the emitted radiance (NEE + MIS, no light visibility)
    spec = synth.sphere_scene(level=1, tex_hw=8, height=12, width=12)
    rng = np.random.default_rng(1)
    dLdI = [rng.normal(size=(12, 12, 3))]
    seeds = np.zeros((1, 3, 8))
    seeds[0, :, 0] = 1.0
    d = orc.grad_dir(spec, dLdI, which=1, seed_emit=seeds, spp_interior=2)[0]
    phi = float(np.sum(dLdI[0] * orc.render(spec, precision=1, spp_interior=2)[0]))
    assert abs(d * 20.0 - phi) <= 1e-9 * max(1.0, abs(phi))
