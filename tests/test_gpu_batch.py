"""Batched multi-view / multi-scene rendering from CUDA graphs (psdr_batch_*) against the
plain per-scene entry points: same images, same gradients, geometry updates picked up."""
import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from helpers import to_torch_scene

pytestmark = pytest.mark.gpu

KW = dict(spp_interior=4, spp_primary_edge=2, spp_secondary_edge=2, max_bounce=3,
          primary_edge_hypercube_resolution=500, secondary_edge_hypercube_resolution=[500, 3, 3])


def make_specs():
    specs = []
    for i, (freq, n_cam) in enumerate([(4, 2), (6, 1), (3, 2)]):
        s = synth.sphere_scene(freq=freq, tex_hw=16, tex_seed=i, noise_sigma=0.02, noise_seed=10 + i)
        s.cameras = synth.orbit_cameras(n_cam, 4.0, seed=20 + i, size_lo=16, size_hi=40)
        specs.append(s)
    return specs


def test_batch_forward_matches_plain(cuda):
    specs = make_specs()
    scenes = [to_torch_scene(s)[0] for s in specs]
    integ = dr.PathIntegrator(**KW)
    plain = [img.clone() for sc in scenes for img in integ.renderC(sc)]
    batch = dr.BatchRender(integ, scenes, differentiable=False)
    for _ in range(2):  # capture, then replay
        imgs = batch.forward()
        torch.cuda.synchronize()
        for a, b in zip(imgs, plain):
            assert torch.equal(a, b)


def test_batch_backward_matches_plain(cuda):
    specs = make_specs()
    integ = dr.PathIntegrator(**KW)
    rng = np.random.default_rng(0)
    # plain: one renderD + backward per scene
    plain_grads, dLdIs = [], []
    for s in specs:
        sc, T = to_torch_scene(s, requires_grad={"verts", "tex", "emit", "cam", "light_verts"})
        imgs = integ.renderD(sc)
        gs = [torch.tensor(rng.normal(size=tuple(i.shape)), dtype=torch.float32, device="cuda") for i in imgs]
        dLdIs.append(gs)
        torch.autograd.backward(imgs, gs)
        plain_grads.append({k: v.grad.clone() for k, v in T.items() if v.grad is not None})
    # batched: all scenes, all views, one graph each way
    scenes, Ts = zip(*[to_torch_scene(s, requires_grad={"verts", "tex", "emit", "cam", "light_verts"}) for s in specs])
    batch = dr.BatchRender(integ, list(scenes))
    for rep in range(2):
        for T in Ts:
            for v in T.values():
                v.grad = None
        imgs = batch.renderD()
        torch.autograd.backward(imgs, [g for gs in dLdIs for g in gs])
        torch.cuda.synchronize()
        for pg, T in zip(plain_grads, Ts):
            for k, g in pg.items():
                got = T[k].grad
                scale = g.abs().max().item() + 1e-30
                err = (got - g).abs().max().item() / scale
                assert err < 1e-5, (rep, k, err)


def test_batch_picks_up_vertex_updates(cuda):
    spec = synth.sphere_scene(level=2, tex_hw=16, height=32, width=32)
    integ = dr.PathIntegrator(spp_interior=4, max_bounce=2)
    scene, T = to_torch_scene(spec)
    batch = dr.BatchRender(integ, [scene], differentiable=False)
    first = batch.forward()[0].clone()
    moved = spec.meshes[0].vertices + np.array([0.2, 0.1, 0.0], np.float32)
    scene.meshes[0].set_vertices(torch.tensor(moved, device="cuda"))
    second = batch.forward()[0].clone()
    spec.meshes[0].vertices = moved
    fresh, _ = to_torch_scene(spec)
    ref = integ.renderC(fresh)[0]
    torch.cuda.synchronize()
    assert not torch.equal(first, second)
    assert torch.equal(second, ref)


def test_batch_extended_features_match_plain(cuda):
    """DiffuseBsdfMaterial, SH9 / cube-map environment lights and an orthographic view
    through the batched graphs: the same images and gradients as the plain path."""
    from test_gpu_envlight import compact_env_spec
    specs = []
    for kind in (2, 1):
        s = compact_env_spec(kind, height=20, width=22)
        rng = np.random.default_rng(kind)
        s.meshes[0].roughness = rng.uniform(0.2, 0.9, size=(5, 7)).astype(np.float32)
        c = s.cameras[0]
        s.cameras.append(synth.CameraSpec(c.look_from, c.look_at, c.up, 3.0, 18, 21, 1))
        specs.append(s)
    kinds = {"verts", "tex", "rough", "env", "cam"}
    integ = dr.PathIntegrator(**KW)
    rng = np.random.default_rng(0)
    plain_imgs, plain_grads, dLdIs = [], [], []
    for s in specs:
        sc, T = to_torch_scene(s, requires_grad=kinds)
        imgs = integ.renderD(sc)
        plain_imgs += [i.detach().clone() for i in imgs]
        gs = [torch.tensor(rng.normal(size=tuple(i.shape)), dtype=torch.float32, device="cuda") for i in imgs]
        dLdIs.append(gs)
        torch.autograd.backward(imgs, gs)
        plain_grads.append({k: v.grad.clone() for k, v in T.items() if v is not None and v.grad is not None})
    scenes, Ts = zip(*[to_torch_scene(s, requires_grad=kinds) for s in specs])
    batch = dr.BatchRender(integ, list(scenes))
    imgs = batch.renderD()
    for a, b in zip(imgs, plain_imgs):
        assert torch.equal(a.detach(), b)
    torch.autograd.backward(imgs, [g for gs in dLdIs for g in gs])
    torch.cuda.synchronize()
    assert any("env" in k for pg in plain_grads for k in pg)
    for pg, T in zip(plain_grads, Ts):
        for k, g in pg.items():
            got = T[k].grad
            err = (got - g).abs().max().item() / (g.abs().max().item() + 1e-30)
            assert err < 1e-5, (k, err)


@pytest.mark.parametrize("estimator", ["unbiased", "reference"])
def test_batch_lanes_give_bitwise_equal_results(cuda, estimator):
    """The batch's concurrent lanes (forward tiles, backward interior tiles and per-view
    boundary terms on forked streams with their own workspaces) and its kept replay
    records (the backward's adjoint reads the forward's records instead of re-tracing)
    change neither the images nor any gradient: the integer gradient sums do not depend on
    the order of additions, and the kept records are the ones a replay writes."""
    specs = make_specs()
    kinds = {"verts", "tex", "emit", "cam", "light_verts"}
    rng = np.random.default_rng(1)
    results, gs = [], None
    # small tiles: several interior tiles for the lanes to share
    kw = dict(KW, tile_paths=4096)
    for lanes, records in ((1, -1), (3, -1), (8, 0), (1, 1), (4, 1)):
        integ = dr.PathIntegrator(estimator=estimator, batch_lanes=lanes, batch_records=records, **kw)
        scenes, Ts = zip(*[to_torch_scene(s, requires_grad=kinds) for s in specs])
        batch = dr.BatchRender(integ, list(scenes))
        for rep in range(2):  # capture, then replay
            for T in Ts:
                for v in T.values():
                    if v is not None:
                        v.grad = None
            imgs = batch.renderD()
            if gs is None:
                gs = [torch.tensor(rng.normal(size=tuple(i.shape)), dtype=torch.float32, device="cuda")
                      for i in imgs]
            torch.autograd.backward(imgs, gs)
            torch.cuda.synchronize()
        results.append(([i.detach().clone() for i in imgs],
                        [{k: v.grad.clone() for k, v in T.items() if v is not None and v.grad is not None}
                         for T in Ts]))
    imgs0, grads0 = results[0]
    assert sum(len(g) for g in grads0) >= 10
    for imgs, grads in results[1:]:
        for a, b in zip(imgs, imgs0):
            assert torch.equal(a, b)
        for g, g0 in zip(grads, grads0):
            assert g.keys() == g0.keys()
            for k in g0:
                assert torch.equal(g[k], g0[k]), k
