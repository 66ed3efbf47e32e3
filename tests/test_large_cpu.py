"""The many-object workload (torch_psdr_b200.synth.large_scene: 16 noisy level-6
icospheres, 1,310,724 triangles with ground and light) in the oracle, CPU only: the
float restatement, which the GPU image matches per sample (tests/test_gpu_large.py),
against the FP64 restatement at 64x64, 64 spp, depth 5. Float and double resolve some
of the small triangles' hits differently, so a few paths diverge; the image error
stays well inside the 1e-3 relative-MSE gate."""
import numpy as np

import orc
from torch_psdr_b200 import synth
from helpers import rel_mse


def test_large_scene_float_matches_fp64_oracle():
    spec = synth.large_scene(height=64, width=64)
    assert sum(len(m.faces) for m in spec.meshes) + sum(len(l.faces) for l in spec.lights) == 1310724
    kw = dict(spp_interior=64, max_bounce=5)
    a = orc.render(spec, precision=0, **kw)[0]
    b = orc.render(spec, precision=1, **kw)[0]
    e = rel_mse(a, b)
    print("large scene: float vs FP64 oracle rel MSE", e)
    assert b.mean() > 0
    assert e < 1e-3
