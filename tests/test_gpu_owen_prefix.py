"""Owen prefix tables: the first scrambling rounds of the draw blocks come from a per-seed table
(built by k_owen_prefix) in the wavefront entry points, and must give exactly the words of the
fully computed Owen loop.  The allocation-free entry point draws without the table, so the two
entry points' lanes are compared bit for bit (every field), on the Cornell box and on the mixed
material scene (conductor and dielectric lobes draw from the same blocks), with two seeds.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, native, renderer, scenes

pytestmark = pytest.mark.gpu


def _untabulated(scene_handle, request, torch):
    q = request.to_c()
    lanes = q.pixel_count * q.sample_count
    out = torch.full((lanes * 80,), 0xFF, dtype=torch.uint8, device="cuda")
    diag = C.create_string_buffer(512)
    st = native.lib().rp_cuda_sample_device_static(scene_handle, C.byref(q), C.c_void_p(out.data_ptr()), lanes, None,
                                                    diag, 512)
    torch.cuda.synchronize()
    assert st == abi.RP_SUCCESS, diag.value.decode()
    return out.cpu().numpy().view(abi.packet_dtype())


@pytest.mark.parametrize("which", ["cornell", "mixed"])
def test_tabulated_owen_rounds_give_identical_lanes(which):
    torch = pytest.importorskip("torch")
    if which == "cornell":
        scene = scenes.cornell_box(64, 64, 4, 8)
        width, height = 64, 64
    else:
        scene = scenes.mixed_scene(96, 64, 2, 16, subdivisions=3)
        width, height = 96, 64
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    for seed, begin in ((1, 0), (12345, 5)):
        req = renderer.RenderRequest(width, height, seed=seed, sample_begin=begin, sample_count=2,
                                     sampler=abi.SAMPLER_SOBOL, randomization=abi.RANDOMIZE_OWEN)
        tab = built.scene.sample(req)
        assert tab.status == abi.RP_SUCCESS, tab.diagnostic
        ref = _untabulated(built.scene.handle, req, torch)
        for f in ref.dtype.names:
            np.testing.assert_array_equal(tab.packet_samples[f], ref[f], err_msg=f)
    built.scene.close()
