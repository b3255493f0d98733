"""The C ABI library loads without a GPU, exports every entry point include/rypath_cuda.h
declares, agrees with the ctypes layouts, and builds the same light tables as the oracle and
as rypath's own build_light_sampling (src/light_sampling.cpp:384-572)."""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, native
from tests.oracle_lib import oracle, reference
from tests.test_oracle_pins import light_rows


def test_library_exports_every_declared_entry_point():
    L = native.lib()
    names = native.header_entry_points()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_library():
    L = native.lib()
    for name, (cls, size) in abi.EXPECTED_SIZES.items():
        assert C.sizeof(cls) == L.rp_cuda_abi_size(name.encode()), name
    assert C.sizeof(abi.SceneDesc) == L.rp_cuda_abi_size(b"rp_scene_desc")
    assert C.sizeof(abi.Timing) == L.rp_cuda_abi_size(b"rp_timing")
    assert C.sizeof(abi.DeviceInfo) == L.rp_cuda_abi_size(b"rp_device_info")
    assert L.rp_cuda_abi_size(b"rp_packet_result") == 80


def _tables(fn, rows):
    n = rows.shape[0]
    alias = np.zeros((n, 4), np.uint32)
    rec = np.zeros((n, 4), np.uint32)
    nodes = np.zeros((2 * n, 16), np.uint32)
    inf = np.zeros(n, np.uint32)
    cnt = C.c_uint32(0)
    k = fn(rows.ctypes.data, n, alias.ctypes.data, rec.ctypes.data, nodes.ctypes.data, inf.ctypes.data, C.byref(cnt))
    return k, alias, rec, nodes[:max(k, 0)], inf[:cnt.value]


@pytest.mark.parametrize("n", [1, 3, 17, 128, 400])
def test_light_tables_match_oracle_and_reference(n):
    rows = light_rows(n, np.random.default_rng(100 + n))
    ours = _tables(native.lib().rp_cuda_build_light_tables, rows)
    theirs = _tables(oracle().or_build_light_tables, rows)
    assert ours[0] == theirs[0]
    for a, b in zip(ours[1:], theirs[1:]):
        np.testing.assert_array_equal(a, b)
    ref = reference()
    if ref is not None:
        r = _tables(ref.ref_build_light_tables, rows)
        for a, b in zip(ours[1:], r[1:]):
            np.testing.assert_array_equal(a, b)


def test_no_device_reports_status_not_exception():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    diag = C.create_string_buffer(256)
    info = abi.DeviceInfo()
    st = native.lib().rp_cuda_device_info(0, C.byref(info), diag, 256)
    assert st == abi.RP_NO_DEVICE
