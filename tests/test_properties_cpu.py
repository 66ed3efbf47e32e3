"""Property tests (hypothesis) of the oracle's building blocks, CPU only.

* closest hits through the oracle's BVH equal brute force, bit for bit, on random
  triangle soups with rays aimed at random points of random triangles (including their
  vertices and edges), so ties and shared edges are exercised;
* watertightness: rays from inside a closed, noisy icosphere always hit it;
* DiscreteSampler::sample_reuse (sampler.h:86-117): indices are monotone in the uniform,
  land on positive weights, carry pmf = w / sum(w), and the rescaled uniform stays in
  [0, 1] up to float rounding;
* every sampler stream draws floats in [0, 1).
"""
import numpy as np
from hypothesis import given, settings, strategies as st

import orc
from torch_psdr_b200 import synth

GREY = np.array([0.5, 0.5, 0.5], np.float32)


def _soup(seed, ntri):
    rng = np.random.default_rng(seed)
    V = rng.uniform(-1, 1, (3 * ntri, 3)).astype(np.float32)
    # share some vertices between triangles, so edges are shared too
    F = np.arange(3 * ntri, dtype=np.int32).reshape(ntri, 3)
    if ntri > 1:
        F[1:, 0] = F[:-1, 1]
    return synth.SceneSpec([synth.MeshSpec(V, F, None, None, GREY)], [], []), V, F, rng


@settings(max_examples=40, deadline=None)
@given(seed=st.integers(0, 2**31 - 1), ntri=st.integers(1, 60))
def test_bvh_closest_hit_equals_bruteforce(seed, ntri):
    spec, V, F, rng = _soup(seed, ntri)
    n = 256
    tri = rng.integers(0, ntri, n)
    b = rng.dirichlet(np.ones(3), n)
    # a quarter of the targets are exact vertices, a quarter exact edge midpoints
    b[: n // 4] = np.eye(3)[rng.integers(0, 3, n // 4)]
    b[n // 4: n // 2] = np.array([0.5, 0.5, 0.0])
    P = V[F[tri]].astype(np.float64)
    target = np.einsum("nk,nkj->nj", b, P)
    o = rng.uniform(-3, 3, (n, 3))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    got = orc.intersect(spec, rays, use_bvh=True)
    ref = orc.intersect(spec, rays, use_bvh=False)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)
    assert (got[0] >= 0).mean() > 0.5


@settings(max_examples=10, deadline=None)
@given(seed=st.integers(0, 2**31 - 1), level=st.integers(1, 3))
def test_rays_from_inside_a_closed_mesh_always_hit(seed, level):
    V, F = synth.icosphere(level)
    V = synth.radial_noise(V, 0.05, seed).astype(np.float32)
    spec = synth.SceneSpec([synth.MeshSpec(V, F, None, None, GREY)], [], [])
    rng = np.random.default_rng(seed)
    n = 2048
    o = rng.uniform(-0.3, 0.3, (n, 3))
    # directions through vertices and edge midpoints, where a leaky test would slip through
    k = n // 2
    tgt = V[rng.integers(0, V.shape[0], k)].astype(np.float64)
    fe = F[rng.integers(0, F.shape[0], n - k)]
    tgt = np.concatenate([tgt, 0.5 * (V[fe[:, 0]] + V[fe[:, 1]])])
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tri, _, _ = orc.intersect(spec, np.concatenate([o, d], 1).astype(np.float32), use_bvh=True)
    assert (tri >= 0).all(), int((tri < 0).sum())


@settings(max_examples=60, deadline=None)
@given(w=st.lists(st.floats(0.0, 100.0), min_size=1, max_size=40).filter(lambda x: sum(x) > 1e-3),
       seed=st.integers(0, 2**31 - 1))
def test_discrete_sample_reuse_invariants(w, seed):
    w = np.asarray(w, np.float64)
    u = np.sort(np.random.default_rng(seed).uniform(1e-6, 1.0, 200).astype(np.float32))
    idx, ur, pmf = orc.discrete_sample(w, u)
    assert (np.diff(idx) >= 0).all()                      # monotone in u
    assert (w[idx] > 0).all()                             # never a zero weight
    np.testing.assert_allclose(pmf, (w / w.sum())[idx].astype(np.float32), rtol=1e-6)
    assert (ur >= -1e-6).all() and (ur <= 1 + 1e-4).all()  # rescaled uniform for reuse


@settings(max_examples=30, deadline=None)
@given(i=st.integers(0, 2**32 - 1))
def test_sampler_stream_floats_in_unit_interval(i):
    f = orc.sampler_floats(i, 64)
    assert (f >= 0).all() and (f < 1).all()
