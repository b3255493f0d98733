"""The allocation-free sampling entry point, rp_cuda_sample_device_static.

Some callers cannot allocate device memory at render time: a host application that owns the
whole device memory budget and lends the GPU to the renderer between its own phases, or code
that runs where the allocator must not be touched.  For them the library keeps the
wavefront's scratch in one file-scope device array and this entry point allocates nothing.
These tests check, through the C ABI, that it returns what the allocating entry point
(rp_cuda_sample) returns for the same requests, on two different calls in a row (the shared
scratch keeps the previous call's contents, which must not leak into the next), and that a
request larger than the scratch is refused with a clear message.

This file is named so pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, native, renderer, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-3  # the per-lane tolerance of tests/test_gpu_parity.py
RP_STATIC_MAX_LANES = 178464  # include/rypath_cuda.h


def _static_sample(scene_handle, request, torch):
    q = request.to_c()
    lanes = q.pixel_count * q.sample_count
    stream = torch.cuda.Stream()  # an explicit stream: a NULL stream means the scene's own stream
    with torch.cuda.stream(stream):
        out = torch.full((lanes * 80,), 0xFF, dtype=torch.uint8, device="cuda")
    diag = C.create_string_buffer(512)
    st = native.lib().rp_cuda_sample_device_static(scene_handle, C.byref(q), C.c_void_p(out.data_ptr()), lanes,
                                                    C.c_void_p(stream.cuda_stream), diag, 512)
    stream.synchronize()
    torch.cuda.synchronize()
    return st, diag.value.decode(), out.cpu().numpy().view(abi.packet_dtype())


def _same(static, reference):
    for f in ("status", "pixel", "sample_low", "sample_high", "splat_count"):
        np.testing.assert_array_equal(static[f], reference[f])
    for f in ("wavelengths", "wavelength_pdfs", "radiance", "filter_weight"):
        np.testing.assert_allclose(static[f], reference[f], rtol=RTOL, atol=1e-7)


def test_static_entry_point_matches_allocating_one_twice():
    torch = pytest.importorskip("torch")
    scene = scenes.cornell_box(32, 32, 4)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    requests = [renderer.RenderRequest(32, 32, sample_begin=0, sample_count=4),
                renderer.RenderRequest(32, 32, pixel_begin=100, pixel_count=600, sample_begin=9, sample_count=3,
                                       sampler=abi.SAMPLER_INDEPENDENT)]
    for req in requests:
        st, diag, static = _static_sample(built.scene.handle, req, torch)
        assert st == abi.RP_SUCCESS, diag
        ref = built.scene.sample(req)
        assert ref.status == abi.RP_SUCCESS, ref.diagnostic
        _same(static, ref.packet_samples)
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
