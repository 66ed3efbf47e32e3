"""Generates the golden fixtures under tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

The reference publishes no golden vectors and cannot run here, so the fixtures are:
  * pcg32_demo.json     -- the published pcg-basic demo output (initstate 42,
                           initseq 54), the one external known-answer vector of the path;
  * sampler_streams.npz -- first draws of the reference's per-sample streams
                           (TEA-seeded PCG32, sampler.h:11-17), from the oracle;
  * oracle_tiny.npz     -- a 16x16, 4 spp FP64 oracle render of a level-1 sphere
                           scene (regression pin of the oracle itself);
  * oracle_ext.npz      -- the same kind of pin for DiffuseBsdfMaterial (roughness and
                           normal maps), an orthographic camera, and EnvLight / SH9Light
                           (`python tests/golden/make_golden.py ext` writes only this one);
  * oracle_grad.npz     -- regression pins of the oracle's gradient terms: directional
                           derivatives (8 random directions over vertices, texels, light
                           parameters, emission and camera origin) of every term of both
                           estimators on the same tiny scenes
                           (`python tests/golden/make_golden.py grad` writes only this one).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402
from torch_psdr_b200 import synth  # noqa: E402


def tiny_spec():
    return synth.sphere_scene(level=1, tex_hw=8, tex_seed=0, height=16, width=16)


def ext_specs():
    """Tiny scenes of the DiffuseBsdfMaterial, orthographic and environment-light pins."""
    rng = np.random.default_rng(0)
    bsdf = tiny_spec()
    bsdf.meshes[0].roughness = rng.uniform(0.2, 0.9, size=(3, 5)).astype(np.float32)
    bsdf.meshes[0].normal = np.stack([rng.uniform(0.4, 0.6, (4, 3)), rng.uniform(0.4, 0.6, (4, 3)),
                                      np.ones((4, 3))], -1).astype(np.float32)
    bsdf.meshes[1].roughness = np.array([0.5], np.float32)
    ortho = tiny_spec()
    c = ortho.cameras[0]
    ortho.cameras[0] = synth.CameraSpec(c.look_from, c.look_at, c.up, 3.0, 16, 16, 1)
    env = tiny_spec()
    env.meshes[1].vertices = (env.meshes[1].vertices * np.array([0.2, 1.0, 0.2], np.float32)).astype(np.float32)
    env.lights.append(synth.LightSpec(None, None, np.zeros(3, np.float32), 1,
                                      cube_map=rng.uniform(0.5, 1.5, size=(3, 4, 3)).astype(np.float32)))
    sh = tiny_spec()
    sh.meshes[1].vertices = env.meshes[1].vertices.copy()
    coeff = rng.normal(scale=0.3, size=(9, 3)).astype(np.float32)
    coeff[0] = [2.0, 1.5, 1.0]
    sh.lights.append(synth.LightSpec(None, None, np.zeros(3, np.float32), 2, sh9=coeff))
    return {"bsdf": bsdf, "ortho": ortho, "env": env, "sh9": sh}


GRAD_CFG = dict(spp_interior=4, max_bounce=3, spp_primary_edge=2, spp_secondary_edge=2, spp_pixel_boundary=2,
                primary_edge_hypercube_resolution=100, secondary_edge_hypercube_resolution=(100, 3, 3))


def grad_cases():
    """(name, scene, estimator mode, terms) of the gradient pins: every term of both
    estimators on the DiffuseBsdfMaterial scene (the unbiased one's BRDF jumps included),
    and all unbiased terms together on the other scenes."""
    out = [(f"bsdf_m{mode}_t{terms}", "bsdf", mode, terms)
           for mode, terms in ((0, 1), (0, 2), (0, 4), (1, 1), (1, 2), (1, 4), (1, 8), (1, 16))]
    out += [(f"{key}_m1_t15", key, 1, 15) for key in ("tiny", "ortho", "env", "sh9")]
    return out


def grad_seeds(spec, seed=7):
    """Random directions over every parameter: vertices (an environment light's box counts
    8), texture elements in the oracle's order (color, roughness, normal map per mesh,
    then cube maps and SH coefficients), emission and camera origin."""
    rng = np.random.default_rng(seed)
    nvt = sum(m.vertices.shape[0] for m in spec.meshes) + sum(
        l.vertices.shape[0] if getattr(l, "kind", 0) == 0 else 8 for l in spec.lights)
    ntex = sum(np.size(a) for m in spec.meshes for a in (m.texture, m.roughness, m.normal) if a is not None)
    ntex += sum(np.size(l.cube_map) if l.kind == 1 else 27 if l.kind == 2 else 0 for l in spec.lights)
    return dict(seed_verts=rng.normal(size=(nvt, 3, 8)), seed_tex=rng.normal(size=(ntex, 8)),
                seed_emit=rng.normal(size=(len(spec.lights), 3, 8)), seed_cam=rng.normal(size=(len(spec.cameras), 3, 8)))


def grad_pins():
    specs = dict(ext_specs(), tiny=tiny_spec())
    out = {}
    for name, key, mode, terms in grad_cases():
        s = specs[key]
        g = np.random.default_rng(5).normal(size=(s.cameras[0].height, s.cameras[0].width, 3))
        out[name] = orc.grad_dir(s, [g], which=terms, mode=mode, **grad_seeds(s), **GRAD_CFG)
    return out


def write_grad():
    np.savez(os.path.join(HERE, "oracle_grad.npz"), **grad_pins())


def write_ext():
    imgs = {k: orc.render(s, precision=1, spp_interior=4, max_bounce=3)[0] for k, s in ext_specs().items()}
    np.savez(os.path.join(HERE, "oracle_ext.npz"), **imgs)


def main():
    demo = [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]
    got = [int(x) for x in orc.pcg32(42, 54, 6)]
    assert got == demo, (got, demo)
    with open(os.path.join(HERE, "pcg32_demo.json"), "w") as f:
        json.dump({"initstate": 42, "initseq": 54, "outputs": demo,
                   "source": "pcg-basic pcg32-demo, first block of printed outputs (published PCG reference output)"}, f, indent=1)
    idx = np.array([0, 1, 2, 3, 1000, 123456, 262143, 4194303], np.uint64)
    draws = np.stack([orc.sampler_floats(int(i), 8) for i in idx])
    np.savez(os.path.join(HERE, "sampler_streams.npz"), index=idx, draws=draws)
    img = orc.render(tiny_spec(), precision=1, spp_interior=4, max_bounce=3)[0]
    np.savez(os.path.join(HERE, "oracle_tiny.npz"), image=img)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if sys.argv[1:] == ["ext"]:
        write_ext()
    elif sys.argv[1:] == ["grad"]:
        write_grad()
    else:
        main()
        write_ext()
        write_grad()
