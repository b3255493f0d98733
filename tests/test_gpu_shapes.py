"""Bilinear patches and analytic shapes on the device against the oracle.

* The intersection kernels: bilinear patch hits bit for bit (plain float arithmetic); analytic
  hits and parameterisations within 1e-4 (the device's acos / atan2 / sin / cos round
  differently from the host's), hit decisions equal for all but a sliver of boundary rays.
* Closest hits through the device tree (procedural leaves beside the triangles) equal the
  oracle's on the shapes box.
* Lanes of the shapes box (hero: Sobol and independent; scalar: Sobol): identity and status
  bit for bit, radiance within 1e-3 for at least 97% of lanes.
* The device films of the white furnaces return the shapes' reflectance where they cover a
  pixel and the environment elsewhere (six standard errors), in both transports.
* Scene validation: invalid shapes are refused, emission from shapes is not built.
"""

import math

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, native, renderer, scenes
from shape_queries import analytic_queries, bilinear_queries
from test_shapes import covered_pixels

pytestmark = pytest.mark.gpu


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def device_probe(name, q, width):
    import ctypes as C

    out = np.zeros((q.shape[0], width), np.float32)
    diag = C.create_string_buffer(512)
    st = getattr(native.lib(), name)(q.ctypes.data, q.shape[0], out.ctypes.data, diag, 512)
    native.check(st, diag, name)
    return out


def oracle_probe(name, q, width):
    import ctypes as C

    fn = getattr(oracle(), name)
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    out = np.zeros((q.shape[0], width), np.float32)
    fn(q.ctypes.data, q.shape[0], out.ctypes.data)
    return out


def test_bilinear_kernel_is_bit_exact():
    q = bilinear_queries()
    g, c = device_probe("rp_cuda_probe_bilinear", q, 4), oracle_probe("or_probe_bilinear", q, 4)
    np.testing.assert_array_equal(g.view(np.uint32), c.view(np.uint32))


def test_analytic_kernel_matches_the_oracle():
    q = analytic_queries()
    g, c = device_probe("rp_cuda_probe_analytic", q, 16), oracle_probe("or_probe_analytic", q, 16)
    same = g[:, 0] == c[:, 0]
    assert same.mean() > 0.999, same.mean()
    both = same & (g[:, 0] == 1)
    np.testing.assert_allclose(g[both, 1], c[both, 1], rtol=1e-4, atol=1e-6)
    close = np.all(np.abs(g[both, 2:] - c[both, 2:]) <= 1e-4 * (1 + np.abs(c[both, 2:])), axis=1)
    assert close.mean() > 0.999, close.mean()


def test_device_closest_hits_equal_the_oracle():
    scene = scenes.cornell_shapes(8, 8, 1)
    rng = np.random.default_rng(3)
    rays = np.zeros((50000, 7), np.float32)
    rays[:, 0:3] = rng.uniform([-0.9, 0.1, -0.9], [0.9, 1.9, 0.9], (50000, 3))
    d = rng.normal(size=(50000, 3))
    rays[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 6] = np.inf
    rs = build(scene)
    g = rs.trace(rays)
    rs.close()
    c = np.zeros((rays.shape[0], 4), np.float32)
    orc = OracleScene(scene)  # held: the oracle scene must outlive the call
    oracle().or_trace_rays(orc.handle, rays.ctypes.data, rays.shape[0], 0, 0, c.ctypes.data)
    gp, cp = g[:, 3].view(np.uint32), c[:, 3].view(np.uint32)
    same = gp == cp
    assert same.mean() > 0.999, same.mean()
    tri = sum(int(i.triangle_count) for i in scene.instances)
    triangles = same & (cp < tri)
    np.testing.assert_array_equal(g[triangles].view(np.uint32), c[triangles].view(np.uint32))
    shapes = same & (cp >= tri) & (cp != abi.RP_NONE)
    assert shapes.sum() > 2000
    np.testing.assert_allclose(g[shapes, 0], c[shapes, 0], rtol=1e-4)


@pytest.mark.parametrize("transport,sampler", [(abi.TRANSPORT_HERO, abi.SAMPLER_SOBOL),
                                               (abi.TRANSPORT_HERO, abi.SAMPLER_INDEPENDENT),
                                               (abi.TRANSPORT_SCALAR, abi.SAMPLER_SOBOL)])
def test_shape_lanes_match_the_oracle(transport, sampler):
    scene = scenes.cornell_shapes(32, 32, 4, transport=transport)
    q = request(32, 32, 4, sampler=sampler)
    rs = build(scene)
    req = renderer.RenderRequest(32, 32, seed=q.seed, sample_count=4, sampler=sampler)
    if transport == abi.TRANSPORT_SCALAR:
        res = rs.sample_scalar(req)
        ref = OracleScene(scene).sample_scalar(q)
    else:
        res = rs.sample(req)
        ref = OracleScene(scene).sample(q)
    rs.close()
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    got = res.samples if transport == abi.TRANSPORT_SCALAR else res.packet_samples
    for f in ("status", "pixel", "sample_low", "sample_high"):
        np.testing.assert_array_equal(got[f], ref[f])
    close = np.isclose(got["radiance"], ref["radiance"], rtol=1e-3, atol=1e-7)
    if close.ndim > 1:
        close = close.all(axis=1)
    assert close.mean() >= 0.97, close.mean()
    assert np.all(ref["status"] == abi.SAMPLE_SUCCESS)


@pytest.mark.parametrize("transport", [abi.TRANSPORT_HERO, abi.TRANSPORT_SCALAR])
@pytest.mark.parametrize("kind", ["sphere", "disk", "cylinder", "patch"])
def test_white_furnace_on_the_device(kind, transport):
    scene = scenes.shape_furnace(kind, 16, 16, 1, transport=transport)
    inside, outside = covered_pixels(scene)
    rs = build(scene)
    st, diag, film = rs.render_film(renderer.RenderSettings(16, 16, samples=2048, batch_size=512, seed=9,
                                                            sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert st == abi.RP_SUCCESS, diag
    n = film["count"][:, None].astype(np.float64)
    mean = (film["sum"] + film["correction"]) / n
    var = np.maximum(film["square"] / n - mean ** 2, 0) / n
    empty = scenes.shape_furnace(kind, 16, 16, 1, transport=transport)  # the environment alone
    empty.instances = []
    rs = build(empty)
    st, diag, sky = rs.render_film(renderer.RenderSettings(16, 16, samples=2048, batch_size=512, seed=10,
                                                           sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert st == abi.RP_SUCCESS, diag
    sky_mean = ((sky["sum"] + sky["correction"]) / sky["count"][:, None]).mean(axis=0)
    for mask, expected in ((inside, 0.5), (outside, 1.0)):
        m, v = mean[mask].mean(axis=0), var[mask].sum(axis=0) / mask.sum() ** 2
        assert np.all(np.abs(m - expected * sky_mean) <= 6 * np.sqrt(v) + 1e-3 * sky_mean), (m, expected * sky_mean)


def test_shape_validation():
    bad = scenes.shape_furnace("sphere")
    bad.analytics[0].radius = -1.0
    built = renderer.build_renderer(bad)
    assert built.status == abi.RP_INVALID_ARGUMENT and "radius" in built.diagnostic
    glowing = scenes.shape_furnace("disk")
    glowing.emissions = [(np.ones(471, np.float32), False)]
    glowing.instances[0].emission = 0
    built = renderer.build_renderer(glowing)
    assert built.status == abi.RP_NOT_BUILT
    wide = scenes.shape_furnace("patch")
    wide.instances[0].patch_count = 5
    assert renderer.build_renderer(wide).status == abi.RP_INVALID_ARGUMENT


@pytest.mark.parametrize("transport", [abi.TRANSPORT_HERO, abi.TRANSPORT_SCALAR])
def test_shape_film_statistics_agree_with_the_oracle(transport):
    """Per-pixel XYZ of the device film of the shapes box within 3 sigma of the oracle's film on
    independent seeds."""
    from oracle_lib import oracle_film

    scene = scenes.cornell_shapes(16, 16, 64, transport=transport)
    rs = build(scene)
    st, diag, film = rs.render_film(renderer.RenderSettings(16, 16, samples=512, batch_size=128, seed=5,
                                                            sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert st == abi.RP_SUCCESS, diag
    host = oracle_film(scene, 16, 16, 512, seed=6, sampler=abi.SAMPLER_INDEPENDENT,
                       scalar=transport == abi.TRANSPORT_SCALAR, chunk=128)

    def moments(f):
        n = f["count"][:, None].astype(np.float64)
        mean = (f["sum"] + f["correction"]) / n
        return mean, np.maximum(f["square"] / n - mean ** 2, 0) / n

    m1, v1 = moments(film)
    m2, v2 = moments(host)
    z = np.abs(m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(z < 3) > 0.97, np.mean(z < 3)
    assert abs(m1.sum() / m2.sum() - 1) < 0.03
