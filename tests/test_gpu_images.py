"""GPU parity of the image path: device texture lookups, RGB reconstruction and environment
queries against the oracle (itself pinned bit for bit to rypath's image shader headers and host
sources by test_image_pins.py), and renders of the environment-image Cornell box against the
oracle lane by lane and statistically.

Tolerances: everything that uses only IEEE arithmetic (texel decoding, the bilinear and
trilinear blends, the sRGB reconstruction, the pinned octahedral map of the radiance lookup) is
bit exact; the mip level of a lookup takes a logarithm (CUDA's logf against the host libm,
within an ulp), so a lookup whose level sits on an integer boundary may blend another pair of
levels -- at least 99% of lookups are bit exact and 99.5% within 1e-4; the sampling density's
cell takes an arctangent and a sampled direction a sine and cosine (last-bit differences), so
at least 99.8% of densities are bit exact and sampled directions agree within 1e-5.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, images, native, renderer, scenes
from tests.oracle_lib import oracle
from tests.test_gpu_mixed import statistics_gates
from tests.test_image_pins import environment_queries, environment_set, lookup, lookup_queries, rgb_queries, \
    tables, texture_set, wire

pytestmark = pytest.mark.gpu


def test_image_lookup_probe_matches_oracle():
    rng = np.random.default_rng(50)
    s = texture_set(rng)
    w = wire(s)
    keep = []
    im = s.to_c(keep)
    q = lookup_queries(rng, 8000)
    for index in range(len(s.textures)):
        cpu = lookup(oracle(), "or_", w, index, q)
        gpu = np.zeros_like(cpu)
        native.check(native.lib().rp_cuda_probe_image_lookup(C.byref(im), index, q.ctypes.data, q.shape[0],
                                                              gpu.ctypes.data, None, 0))
        exact = np.all(gpu.view(np.uint32) == cpu.view(np.uint32), axis=1)
        close = np.all(np.isclose(gpu, cpu, rtol=1e-4, atol=1e-7, equal_nan=True), axis=1)
        assert exact.mean() >= 0.99 and close.mean() >= 0.995, (index, exact.mean(), close.mean())


def test_rgb_spectrum_probe_bit_exact():
    rng = np.random.default_rng(51)
    q = rgb_queries(rng, 40000)
    table = images.rgb_table()
    cpu = np.zeros((q.shape[0], 2), np.float32)
    gpu = np.zeros_like(cpu)
    oracle().or_rgb_spectrum(table.ctypes.data, q.ctypes.data, q.shape[0], cpu.ctypes.data)
    s = images.ImageSet()
    s.add_image(np.zeros((1, 1, 3), np.float32))
    keep = []
    im = s.to_c(keep)
    native.check(native.lib().rp_cuda_probe_rgb_spectrum(C.byref(im), q.ctypes.data, q.shape[0], gpu.ctypes.data,
                                                          None, 0))
    np.testing.assert_array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("width,seed,fmt", [(1, 1, abi.TEXELS_FLOAT), (7, 3, abi.TEXELS_HALF),
                                            (32, 4, abi.TEXELS_FLOAT), (16, 5, abi.TEXELS_SRGB8)])
def test_environment_probe_matches_oracle(width, seed, fmt):
    rng = np.random.default_rng(52 + width)
    s = environment_set(width, seed, fmt)
    c, sn = np.cos(0.7), np.sin(0.7)
    s.environment_from_world = (c, 0, sn, 0, 1, 0, -sn, 0, c)
    s.environment_scale = 1.25
    cdf, w, off, _ = tables(oracle(), "or_", s)
    tex, nt, levels, nl, texels, nw, transfer, ntr = wire(s)
    frame = np.array(s.environment_from_world, np.float32)
    q = environment_queries(rng, 20000)
    cpu = np.zeros((q.shape[0], 12), np.float32)
    oracle().or_environment_queries(C.cast(tex, C.c_void_p), nt, s.environment_image, levels.ctypes.data, nl,
                                    texels.ctypes.data, nw, transfer.ctypes.data, ntr, images.rgb_table().ctypes.data,
                                    images.d65().ctypes.data, cdf.ctypes.data, cdf.size, w, off, 1.25,
                                    frame.ctypes.data, q.ctypes.data, q.shape[0], cpu.ctypes.data)
    keep = []
    im = s.to_c(keep)
    gpu = np.zeros_like(cpu)
    native.check(native.lib().rp_cuda_probe_environment(C.byref(im), q.ctypes.data, q.shape[0], gpu.ctypes.data,
                                                         None, 0))
    g32, c32 = gpu.view(np.uint32), cpu.view(np.uint32)
    np.testing.assert_array_equal(g32[:, 0], c32[:, 0])  # radiance: the pinned map
    assert (g32[:, 1:3] == c32[:, 1:3]).all(axis=1).mean() >= 0.998
    same = (gpu[:, 3] == cpu[:, 3]) & (gpu[:, 8] == cpu[:, 8])
    assert same.mean() >= 0.999
    ok = same & (cpu[:, 3] == 1)
    assert ok.mean() > 0.99
    assert np.abs(gpu[ok, 4:7] - cpu[ok, 4:7]).max() <= 1e-5
    assert (g32[ok, 7] == c32[ok, 7]).mean() >= 0.998
    ok2 = same & (cpu[:, 8] == 1)
    assert np.abs(gpu[ok2, 9:12] - cpu[ok2, 9:12]).max() <= 1e-5


def test_environment_image_statistics():
    """The environment-image Cornell box at 48 spp: within 3 combined standard errors per pixel
    of an independent oracle render, relative RMSE against a 4096-spp FP64 oracle render below
    0.2 and within 30% of an oracle render of the same spp."""
    scene = scenes.cornell_features("env_image", 24, 24, 48)
    device, other = statistics_gates(scene, 48, 0.2)
    assert device > 0


def test_environment_image_counts_and_escape():
    """Escaped paths read the image: a render with the sun's texels zeroed is darker, and the
    environment light is sampled (shadow rays on most lanes)."""
    scene = scenes.cornell_features("env_image", 32, 32, 4)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    built.scene.set_counting(True)
    res = built.scene.sample(renderer.RenderRequest(32, 32, sample_count=4))
    built.scene.close()
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    g = res.packet_samples
    assert (g["reserved"][:, 1] > 0).mean() > 0.5
    dark = scenes.cornell_features("env_image", 32, 32, 4)
    dark.images.environment_scale = 0.0
    built = renderer.build_renderer(dark)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    res2 = built.scene.sample(renderer.RenderRequest(32, 32, sample_count=4))
    built.scene.close()
    assert res2.status == abi.RP_SUCCESS
    assert res2.packet_samples["radiance"].sum() == 0 and g["radiance"].sum() > 0


def test_texture_footprint_probe_bit_exact():
    """The device footprint functions (primary and approximate ray differentials, the uv
    derivatives' least squares) against the oracle: IEEE arithmetic only, bit exact."""
    from tests.test_image_pins import footprint_queries

    q = footprint_queries(np.random.default_rng(60), 20000)
    cpu = np.zeros((q.shape[0], 24), np.float32)
    gpu = np.zeros_like(cpu)
    oracle().or_texture_footprint(q.ctypes.data, q.shape[0], cpu.ctypes.data)
    native.check(native.lib().rp_cuda_probe_texture_footprint(q.ctypes.data, q.shape[0], gpu.ctypes.data, None, 0))
    np.testing.assert_array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


def test_texture_statistics():
    """The textured Cornell box (sRGB trilinear back wall, float EWA floor, half point box)
    at 48 spp against oracle renders: 3 combined standard errors per pixel, relative RMSE below
    0.2 against a 4096-spp FP64 render and within 30% of an oracle render of the same spp."""
    scene = scenes.cornell_features("texture", 24, 24, 48)
    statistics_gates(scene, 48, 0.2)


def test_texture_refusals():
    """Image reflectance needs a fixed sample budget; an EWA-filtered image needs the EWA
    table."""
    scene = scenes.cornell_features("texture", 16, 16, 1)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    req = renderer.RenderRequest(16, 16, sample_count=1)
    c = req.to_c()
    c.total_samples = 0
    out = np.zeros(256, abi.packet_dtype())
    diag = C.create_string_buffer(256)
    st = native.lib().rp_cuda_sample(built.scene.handle, C.byref(c), out.ctypes.data, 256, diag, 256)
    assert st == abi.RP_INVALID_ARGUMENT and b"fixed total sample budget" in diag.value
    built.scene.close()
    ewa = scenes.cornell_features("texture", 16, 16, 1)
    keep = []
    desc = ewa.desc()
    desc.images.contents.ewa_weights = None
    out_scene = C.c_void_p()
    st = native.lib().rp_cuda_scene_create(C.byref(desc), 0, C.byref(out_scene), diag, 256)
    assert st == abi.RP_INVALID_ARGUMENT and b"EWA" in diag.value
