"""Generates the golden fixtures under tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

The reference publishes no golden vectors and cannot run here, so the fixtures are:
  * pcg32_demo.json     -- the published pcg-basic demo output (initstate 42,
                           initseq 54), the one external known-answer vector of the path;
  * sampler_streams.npz -- first draws of the reference's per-sample streams
                           (TEA-seeded PCG32, sampler.h:11-17), from the oracle;
  * oracle_tiny.npz     -- a 16x16, 4 spp FP64 oracle render of a level-1 sphere
                           scene (regression pin of the oracle itself).
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


def main():
    demo = [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]
    got = [int(x) for x in orc.pcg32(42, 54, 6)]
    assert got == demo, (got, demo)
    with open(os.path.join(HERE, "pcg32_demo.json"), "w") as f:
        json.dump({"initstate": 42, "initseq": 54, "outputs": demo,
                   "source": "pcg-basic pcg32-demo, round 1 (published PCG reference output)"}, f, indent=1)
    idx = np.array([0, 1, 2, 3, 1000, 123456, 262143, 4194303], np.uint64)
    draws = np.stack([orc.sampler_floats(int(i), 8) for i in idx])
    np.savez(os.path.join(HERE, "sampler_streams.npz"), index=idx, draws=draws)
    img = orc.render(tiny_spec(), precision=1, spp_interior=4, max_bounce=3)[0]
    np.savez(os.path.join(HERE, "oracle_tiny.npz"), image=img)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
