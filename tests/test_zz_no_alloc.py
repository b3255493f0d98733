"""The allocation-free sampling entry point, rp_cuda_sample_device_static.

Some callers cannot allocate device memory at render time: a host application that owns the
whole device memory budget and lends the GPU to the renderer between its own phases, or code
that runs where the allocator must not be touched.  For them the library keeps the
wavefront's scratch in one file-scope device array and this entry point allocates nothing.
These tests check, through the C ABI, that it returns what the allocating entry point
(rp_cuda_sample) returns for the same requests, on two different calls in a row (the shared
scratch keeps the previous call's contents, which must not leak into the next), and that a
request larger than the scratch is refused with a clear message.

The allocation-free entry point runs the same kernels in the same order as the allocating
one, so their packets are compared byte for byte: a value left over in the shared scratch from
an earlier call would show as a difference.  The checks also run on the scene's own stream
(stream NULL), and the device's free memory is the same before and after a call on a scene
that has never sampled (so it owns no wavefront pool yet).

This file is named so pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, native, renderer, scenes

pytestmark = pytest.mark.gpu

RP_STATIC_MAX_LANES = 118976  # include/rypath_cuda.h
REQUESTS = [renderer.RenderRequest(32, 32, sample_begin=0, sample_count=4),
            renderer.RenderRequest(32, 32, pixel_begin=100, pixel_count=600, sample_begin=9, sample_count=3,
                                   sampler=abi.SAMPLER_INDEPENDENT)]


def _static_sample(scene_handle, request, torch, own_stream=True):
    """One call of the allocation-free entry point into a buffer poisoned with 0xff; on a
    stream of the caller's (own_stream) or on the scene's own stream (NULL)."""
    q = request.to_c()
    lanes = q.pixel_count * q.sample_count
    stream = torch.cuda.Stream() if own_stream else None
    out = torch.full((lanes * 80,), 0xFF, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    diag = C.create_string_buffer(512)
    st = native.lib().rp_cuda_sample_device_static(scene_handle, C.byref(q), C.c_void_p(out.data_ptr()), lanes,
                                                    C.c_void_p(stream.cuda_stream if stream else None), diag, 512)
    torch.cuda.synchronize()
    return st, diag.value.decode(), out.cpu().numpy().view(abi.packet_dtype())


@pytest.mark.parametrize("own_stream", [True, False])
def test_static_entry_point_matches_allocating_one_twice(own_stream):
    torch = pytest.importorskip("torch")
    built = renderer.build_renderer(scenes.cornell_box(32, 32, 4))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    for req in REQUESTS:
        st, diag, static = _static_sample(built.scene.handle, req, torch, own_stream)
        assert st == abi.RP_SUCCESS, diag
        ref = built.scene.sample(req)
        assert ref.status == abi.RP_SUCCESS, ref.diagnostic
        assert static.tobytes() == ref.packet_samples.tobytes()
    built.scene.close()


def test_static_entry_point_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    # load the kernels first (lazy module loading places their code in device memory)
    warm = renderer.build_renderer(scenes.cornell_box(32, 32, 4))
    assert warm.status == abi.RP_SUCCESS, warm.diagnostic
    st, diag, _ = _static_sample(warm.scene.handle, REQUESTS[0], torch)
    assert st == abi.RP_SUCCESS, diag
    warm.scene.close()
    built = renderer.build_renderer(scenes.cornell_box(32, 32, 4))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    q = REQUESTS[0].to_c()
    lanes = q.pixel_count * q.sample_count
    out = torch.empty(lanes * 80, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    diag = C.create_string_buffer(512)
    for _ in range(2):
        st = native.lib().rp_cuda_sample_device_static(built.scene.handle, C.byref(q), C.c_void_p(out.data_ptr()),
                                                        lanes, None, diag, 512)
        assert st == abi.RP_SUCCESS, diag.value.decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    static = out.cpu().numpy().view(abi.packet_dtype())
    ref = built.scene.sample(REQUESTS[0])
    assert static.tobytes() == ref.packet_samples.tobytes()
    built.scene.close()


def test_static_entry_point_refuses_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    scene = scenes.cornell_box(1024, 1024, 1)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    q = renderer.RenderRequest(1024, 1024, pixel_count=RP_STATIC_MAX_LANES + 1, sample_count=1).to_c()
    out = torch.empty(80, dtype=torch.uint8, device="cuda")
    diag = C.create_string_buffer(512)
    st = native.lib().rp_cuda_sample_device_static(built.scene.handle, C.byref(q), C.c_void_p(out.data_ptr()),
                                                    RP_STATIC_MAX_LANES + 1, None, diag, 512)
    assert st == abi.RP_INVALID_ARGUMENT
    assert str(RP_STATIC_MAX_LANES) in diag.value.decode()
    built.scene.close()
