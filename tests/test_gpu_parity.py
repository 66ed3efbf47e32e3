"""GPU parity: the native sm_100a path against the oracle, through the C ABI.

* intersection KAT: LBVH closest hit == GPU brute force == oracle float brute force,
  bit-exact (triangle id, barycentrics, t), including rays aimed at vertices/edges;
* edge list == oracle edge list;
* per-sample radiance and images against the oracle (same sampler streams);
* every gradient term (interior / primary edges / direct edges) against the oracle's
  forward-mode derivatives along random directions;
* texture gradient against central finite differences (common random numbers).
"""
import ctypes as C

import numpy as np
import pytest
import torch

import orc
import torch_psdr_b200 as dr
from torch_psdr_b200 import synth
from torch_psdr_b200 import _lib as L
from helpers import rel_l2, rel_mse, to_torch_scene
from test_oracle_cpu import _random_rays

pytestmark = pytest.mark.gpu


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def gpu_intersect(scene, rays6, brute):
    n = rays6.shape[0]
    r8 = np.zeros((n, 8), np.float32)
    r8[:, 0:3] = rays6[:, 0:3]
    r8[:, 3] = 1e-3
    r8[:, 4:7] = rays6[:, 3:6]
    r8[:, 7] = np.inf
    rays = torch.tensor(r8, device="cuda")
    tri = torch.empty(n, dtype=torch.int32, device="cuda")
    bary = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    lib = L.load()
    L.check(lib.psdr_intersect(scene.handle, rays.data_ptr(), n, tri.data_ptr(), bary.data_ptr(), t.data_ptr(),
                               int(brute), _stream()), "intersect")
    torch.cuda.synchronize()
    return tri.cpu().numpy(), bary.cpu().numpy(), t.cpu().numpy()


@pytest.mark.parametrize("level,noise", [(3, 0.0), (5, 0.02)])
def test_intersect_kat_bit_exact(cuda, level, noise):
    spec = synth.sphere_scene(level=level, noise_sigma=noise, height=8, width=8)
    scene, _ = to_torch_scene(spec)
    rays = _random_rays(spec, 20000, 11)
    t_bvh, b_bvh, tt_bvh = gpu_intersect(scene, rays, 0)
    t_bf, b_bf, tt_bf = gpu_intersect(scene, rays, 1)
    t_wf, b_wf, tt_wf = gpu_intersect(scene, rays, 2)  # the wavefront kernel's traversal
    t_or, b_or, tt_or = orc.intersect(spec, rays, use_bvh=False)
    assert (t_bf >= 0).mean() > 0.3
    np.testing.assert_array_equal(t_bvh, t_bf)
    np.testing.assert_array_equal(b_bvh, b_bf)
    np.testing.assert_array_equal(tt_bvh, tt_bf)
    np.testing.assert_array_equal(t_wf, t_bf)
    np.testing.assert_array_equal(b_wf, b_bf)
    np.testing.assert_array_equal(tt_wf, tt_bf)
    np.testing.assert_array_equal(t_bf, t_or)
    np.testing.assert_array_equal(b_bf, b_or)
    np.testing.assert_array_equal(tt_bf, tt_or)


def test_intersect_single_triangle_and_misses(cuda):
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    F = np.array([[0, 1, 2]], np.int32)
    spec = synth.SceneSpec([synth.MeshSpec(V, F, None, None, np.array([0.5, 0.5, 0.5], np.float32))], [],
                           [synth.default_camera(4, 4)])
    scene, _ = to_torch_scene(spec)
    rays = np.array([[0.2, 0.2, 1, 0, 0, -1], [2, 2, 1, 0, 0, -1], [0.2, 0.2, -1, 0, 0, -1]], np.float32)
    for mode in (0, 2):
        t, b, tt = gpu_intersect(scene, rays, mode)
        assert list(t) == [0, -1, -1]
        np.testing.assert_allclose(b[0], [0.2, 0.2], atol=1e-6)
        np.testing.assert_allclose(tt[0], 1.0, atol=1e-6)


def test_edges_match_oracle(cuda):
    spec = synth.sphere_scene(level=3, noise_sigma=0.02, height=8, width=8)
    scene, _ = to_torch_scene(spec)
    v_or, g_or = orc.edges(spec)
    cap = 3 * sum(m.faces.shape[0] for m in spec.meshes + spec.lights)
    v01 = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    geo = torch.empty((cap, 16), dtype=torch.float32, device="cuda")
    n = C.c_int64()
    lib = L.load()
    L.check(lib.psdr_scene_edges(scene.handle, v01.data_ptr(), geo.data_ptr(), cap, C.byref(n), _stream()), "edges")
    n = n.value
    assert n == v_or.shape[0]
    np.testing.assert_array_equal(v01[:n].cpu().numpy(), v_or)
    np.testing.assert_allclose(geo[:n].cpu().numpy(), g_or, rtol=1e-4, atol=2e-5)
    info = scene.info()
    assert info["edges"] == n and info["triangles"] == sum(m.faces.shape[0] for m in spec.meshes + spec.lights)


def _cfg(**kw):
    base = dict(spp_interior=4, max_bounce=3)
    base.update(kw)
    return base


@pytest.mark.parametrize("nl,nb,lv", [(1, 1, False), (2, 0, False), (0, 2, True), (3, 3, False)])
def test_per_sample_radiance_matches_oracle(cuda, nl, nb, lv):
    spec = synth.sphere_scene(level=3, tex_hw=64, height=32, width=32)
    kw = _cfg(mis_light_samples=nl, mis_bsdf_samples=nb, enable_light_visable=lv)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(**kw)
    gpu = integ.render_samples(scene).cpu().numpy().astype(np.float64)
    _, ref = orc.render(spec, precision=0, per_sample=True, **kw)
    close = np.abs(gpu - ref) <= 1e-3 * (1.0 + np.abs(ref))
    frac = close.all(axis=1).mean()
    print(f"per-sample agreement {frac:.5f}, mean |diff| {np.abs(gpu - ref).mean():.3e}")
    assert frac > 0.995
    assert rel_mse(gpu, ref) < 1e-3


def test_image_matches_fp64_oracle(cuda):
    spec = synth.sphere_scene(level=3, tex_hw=256, height=64, width=64)
    kw = _cfg(spp_interior=64)
    scene, _ = to_torch_scene(spec)
    img = dr.PathIntegrator(**kw).renderC(scene)[0].cpu().numpy()
    ref = orc.render(spec, precision=1, **kw)[0]
    e = rel_mse(img, ref)
    print("image rel MSE vs FP64 oracle", e)
    assert e < 1e-4
    # n_pass averages identical passes
    img3 = dr.PathIntegrator(n_pass=3, **kw).renderC(scene)[0].cpu().numpy()
    np.testing.assert_allclose(img3, img, rtol=1e-6, atol=1e-7)


def test_render_is_deterministic(cuda):
    spec = synth.sphere_scene(level=3, tex_hw=64, height=48, width=40)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(spp_interior=8, tile_paths=4096)
    a = integ.renderC(scene)[0]
    b = integ.renderC(scene)[0]
    c = dr.PathIntegrator(spp_interior=8).renderC(scene)[0]
    assert torch.equal(a, b) and torch.equal(a, c)


def _gpu_dir_derivs(spec, which_terms, seeds, kw, params):
    """Directional derivatives of Phi = sum(dLdI * renderD) from the GPU adjoint."""
    scene, T = to_torch_scene(spec, requires_grad=params)
    integ = dr.PathIntegrator(gradient_terms=which_terms, **kw)
    img = integ.renderD(scene)[0]
    rng = np.random.default_rng(5)
    dLdI = rng.normal(size=tuple(img.shape))
    img.backward(torch.tensor(dLdI, dtype=torch.float32, device="cuda"))
    out = np.zeros(8)
    for name, seed in seeds.items():
        g = T[name].grad.detach().cpu().numpy().astype(np.float64).reshape(-1)
        out += g @ seed.reshape(g.shape[0], 8)
    return out, dLdI


def _seeds_for(spec, kinds, rng):
    """Random seed directions: returns (gpu seed dict, oracle seed kwargs)."""
    nv = [m.vertices.shape[0] for m in spec.meshes] + [l.vertices.shape[0] for l in spec.lights]
    sv = rng.normal(size=(sum(nv), 3, 8)) if "verts" in kinds else None
    ntex = [m.texture.size for m in spec.meshes]
    st = rng.normal(size=(sum(ntex), 8)) if "tex" in kinds else None
    se = rng.normal(size=(len(spec.lights), 3, 8)) if "emit" in kinds else None
    sc = rng.normal(size=(len(spec.cameras), 3, 8)) if "cam" in kinds else None
    gpu = {}
    off = 0
    for i, m in enumerate(spec.meshes):
        if sv is not None:
            gpu[f"verts{i}"] = sv[off:off + nv[i]]
        off += nv[i]
    for j, l in enumerate(spec.lights):
        if sv is not None:
            gpu[f"lverts{j}"] = sv[off:off + nv[len(spec.meshes) + j]]
        off += nv[len(spec.meshes) + j]
    toff = 0
    for i, m in enumerate(spec.meshes):
        if st is not None:
            gpu[f"tex{i}"] = st[toff:toff + ntex[i]]
        toff += ntex[i]
    if se is not None:
        for j in range(len(spec.lights)):
            gpu[f"emit{j}"] = se[j]
    if sc is not None:
        for k in range(len(spec.cameras)):
            gpu[f"cam{k}"] = sc[k]
    return gpu, dict(seed_verts=sv, seed_tex=st, seed_emit=se, seed_cam=sc)


GRAD_CASES = [
    # (terms bitmask, parameters)
    (1, ("tex",)),
    (1, ("verts",)),
    (1, ("emit",)),
    (2, ("verts",)),
    (2, ("cam",)),
    (4, ("verts",)),
]


@pytest.mark.parametrize("terms,kinds", GRAD_CASES)
def test_gradient_terms_match_oracle(cuda, terms, kinds):
    spec = synth.sphere_scene(level=2, tex_hw=16, height=24, width=24)
    kw = _cfg(spp_interior=4, spp_primary_edge=4, spp_secondary_edge=4, primary_edge_hypercube_resolution=500,
              secondary_edge_hypercube_resolution=[500, 3, 3])
    rng = np.random.default_rng(3)
    gseeds, oseeds = _seeds_for(spec, kinds, rng)
    params = set()
    for k in kinds:
        params |= {"verts": {"verts", "light_verts"}, "tex": {"tex"}, "emit": {"emit"}, "cam": {"cam"}}[k]
    got, dLdI = _gpu_dir_derivs(spec, terms, gseeds, kw, params)
    ref = orc.grad_dir(spec, [dLdI], which=terms, **oseeds, **kw)
    err = np.abs(got - ref) / (np.abs(ref).max() + 1e-30)
    print(f"terms={terms} {kinds}: gpu {got[:4]} oracle {ref[:4]} max rel {err.max():.2e}")
    assert np.abs(ref).max() > 0
    assert err.max() < 2e-3


def test_texture_gradient_vs_finite_differences(cuda):
    spec = synth.sphere_scene(level=3, tex_hw=32, height=48, width=48)
    kw = dict(spp_interior=16, max_bounce=3)
    scene, T = to_torch_scene(spec, requires_grad={"tex"})
    integ = dr.PathIntegrator(gradient_terms=1, **kw)
    tgt_spec = synth.sphere_scene(level=3, tex_hw=32, tex_seed=1, height=48, width=48)
    tgt_scene, _ = to_torch_scene(tgt_spec)
    target = integ.renderC(tgt_scene)[0]
    img = integ.renderD(scene)[0]
    loss = ((img - target) ** 2).sum()
    loss.backward()
    grad = T["tex0"].grad.detach().cpu().numpy().reshape(-1)
    rng = np.random.default_rng(0)
    cand = np.nonzero(np.abs(grad) > 1e-3 * np.abs(grad).max())[0]
    pick = rng.choice(cand, size=min(64, cand.size), replace=False)
    tex0 = spec.meshes[0].texture.copy()
    h = 1e-3

    def loss_at(tex):
        spec.meshes[0].texture = tex
        sc, _ = to_torch_scene(spec)
        return float(((integ.renderC(sc)[0].double() - target.double()) ** 2).sum())

    fd = []
    for k in pick:
        tp = tex0.copy().reshape(-1)
        tm = tex0.copy().reshape(-1)
        tp[k] += h
        tm[k] -= h
        fd.append((loss_at(tp.reshape(tex0.shape)) - loss_at(tm.reshape(tex0.shape))) / (2 * h))
    spec.meshes[0].texture = tex0
    e = rel_l2(grad[pick], np.array(fd))
    print("texture grad rel L2 vs FD", e)
    assert e < 0.05


def test_scene_validate_accepts_valid_and_names_bad_index(cuda):
    """psdr_scene_validate, and psdr_scene_create, which runs the same check: a valid
    description passes; one face index out of range is refused and named."""
    spec = synth.sphere_scene(level=2, tex_hw=16, height=16, width=16)
    scene, _ = to_torch_scene(spec)
    lib = L.load()
    sphere = scene.meshes[0]
    md = (L.MeshDesc * 2)(*[m._desc() for m in scene.meshes])
    ld = (L.AreaLightDesc * 1)(*[lt._desc() for lt in scene.lights])
    desc = L.SceneDesc(md, 2, ld, 1)
    assert lib.psdr_scene_validate(C.byref(desc), _stream()) == L.PSDR_OK
    bad_faces = sphere.f.clone()
    bad_faces.view(-1)[17] = sphere.v.shape[0]  # one past the last vertex
    md[0].faces = bad_faces.data_ptr()
    assert lib.psdr_scene_validate(C.byref(desc), _stream()) == L.PSDR_ERR_INVALID_ARG
    assert b"mesh 0 face" in lib.psdr_last_error()
    out = C.c_void_p()
    assert lib.psdr_scene_create(C.byref(desc), _stream(), C.byref(out)) == L.PSDR_ERR_INVALID_ARG
    assert b"mesh 0 face" in lib.psdr_last_error()
    bad_faces.view(-1)[17] = -1
    assert lib.psdr_scene_validate(C.byref(desc), _stream()) == L.PSDR_ERR_INVALID_ARG
    torch.cuda.synchronize()
