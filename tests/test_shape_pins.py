"""The oracle's procedural primitive tests pinned to rypath's own shaders compiled for the
host (oracle/_ref/libref_shapes.so from shaders/bilinear.h and shaders/analytic.h, built by
oracle/ref.mk): bilinear patch hits bit for bit, analytic shape hits and parameterisations bit
for bit, on seeded queries that reach every branch (planar and warped patches, edges and
corners, slivers, far-off patches; clipped spheres, holed disks, partial sweeps, inside and
grazing rays).  CPU only."""

import ctypes as C
import os

import numpy as np
import pytest

from oracle_lib import oracle
from shape_queries import analytic_queries, bilinear_queries

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref_shapes.so")


def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/libref_shapes.so not built (needs a rypath checkout: oracle/ref.mk)")
    lib = C.CDLL(REF)
    lib.ref_bilinear.argtypes = lib.ref_analytic.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    return lib


def run(fn, q, width):
    out = np.zeros((q.shape[0], width), np.float32)
    fn(q.ctypes.data, q.shape[0], out.ctypes.data)
    return out


def test_bilinear_oracle_equals_rypath_shader():
    lib = ref()
    o = oracle()
    o.or_probe_bilinear.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    q = bilinear_queries()
    a, b = run(lib.ref_bilinear, q, 4), run(o.or_probe_bilinear, q, 4)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    hits = a[:, 0] == 1
    assert 0.3 < hits.mean() < 0.95, hits.mean()
    assert np.all((a[hits, 2:] >= 0) & (a[hits, 2:] <= 1))


def test_analytic_oracle_equals_rypath_shader():
    lib = ref()
    o = oracle()
    o.or_probe_analytic.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    q = analytic_queries()
    a, b = run(lib.ref_analytic, q, 16), run(o.or_probe_analytic, q, 16)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    hits = a[:, 0] == 1
    assert 0.3 < hits.mean() < 0.95, hits.mean()
    sub = q[:, 1].view(np.uint32)
    for k in (1, 2, 3):
        assert hits[sub == k].mean() > 0.2


def test_bilinear_hits_lie_on_the_patch():
    """Independent of both: the reported (t, u, v) of a hit names the same point twice, on the
    ray and on the patch, to float accuracy."""
    lib = ref()
    q = bilinear_queries(4000, seed=5)
    r = run(lib.ref_bilinear, q, 4)
    hit = r[:, 0] == 1
    p = q[hit, :12].reshape(-1, 4, 3).astype(np.float64)
    u, v = r[hit, 2:3].astype(np.float64), r[hit, 3:4].astype(np.float64)
    on_patch = (1 - u) * (1 - v) * p[:, 0] + u * (1 - v) * p[:, 1] + (1 - u) * v * p[:, 2] + u * v * p[:, 3]
    on_ray = q[hit, 12:15].astype(np.float64) + r[hit, 1:2].astype(np.float64) * q[hit, 15:18]
    scale = np.abs(p).max(axis=(1, 2)) + np.abs(q[hit, 12:15]).max(axis=1)
    err = np.abs(on_patch - on_ray).max(axis=1) / scale
    assert np.quantile(err, 0.999) < 1e-4, np.quantile(err, 0.999)
