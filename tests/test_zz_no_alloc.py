"""The allocation-free forward entry point (psdr_render_fwd_noalloc).

Some callers cannot allocate device memory when they render: a host that hands the
library a fixed memory budget up front, or a loop that cannot pay for cudaMalloc's
implicit device synchronisation. For them the library renders one camera out of a
fixed 32 MiB scratch array compiled into the library. These tests call that entry
point through the C ABI twice in a row, compare each image with the regular
psdr_render_fwd output, and check that the second call changes neither torch's
allocator counters nor the device's free memory. This file is collected last on
purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import torch_psdr_b200 as dr
from torch_psdr_b200 import _lib as L
from torch_psdr_b200 import synth
from helpers import to_torch_scene

pytestmark = pytest.mark.gpu


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("h,w,spp,nl,nb", [(64, 48, 8, 1, 1), (37, 91, 16, 2, 0)])
def test_noalloc_matches_render_fwd_twice(cuda, h, w, spp, nl, nb):
    spec = synth.sphere_scene(level=3, tex_hw=64, height=h, width=w)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(spp_interior=spp, mis_light_samples=nl, mis_bsdf_samples=nb)
    ref = integ.renderC(scene)[0]
    lib = L.load()
    cams = scene._camera_descs()
    outs = [torch.full_like(ref, float("nan")) for _ in range(2)]
    torch.cuda.synchronize()
    for k, out in enumerate(outs):
        if k == 1:  # the first call resolved the scratch address; the second must allocate nothing
            stats0 = _alloc_counters()
            free0 = torch.cuda.mem_get_info()[0]
        L.check(lib.psdr_render_fwd_noalloc(scene.handle, C.byref(cams[0]), C.byref(integ.cfg), out.data_ptr(),
                                            _stream()), "psdr_render_fwd_noalloc")
        torch.cuda.synchronize()
        if k == 1:
            assert torch.cuda.mem_get_info()[0] == free0
            assert _alloc_counters() == stats0
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-6, atol=1e-7)


def _alloc_counters():
    s = torch.cuda.memory_stats()
    return {k: s.get(k) for k in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current")}


def test_noalloc_rejects_oversized_tiles(cuda):
    spec = synth.sphere_scene(level=1, tex_hw=8, height=4, width=4)
    scene, _ = to_torch_scene(spec)
    integ = dr.PathIntegrator(spp_interior=1 << 20)
    lib = L.load()
    cams = scene._camera_descs()
    out = torch.empty((4, 4, 3), device="cuda")
    st = lib.psdr_render_fwd_noalloc(scene.handle, C.byref(cams[0]), C.byref(integ.cfg), out.data_ptr(), _stream())
    assert st == L.PSDR_ERR_INVALID_ARG
    assert b"exceeds the allocation-free tile" in lib.psdr_last_error()
