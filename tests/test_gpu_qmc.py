"""Halton and ZSobol samplers on the device (src/qmc_shared.h, shaders/render.metal:113-198).

Raygen words (camera, wavelength, roulette and lens words, indices) and primary rays are
bit-exact against the oracle (itself pinned to rypath's 28 PBRT known answers and to the
reference header); transport lanes of the hero and scalar paths agree per lane as the Sobol
ones do.  The sampler-range rules of validate_sampler_range (src/sampling.cpp:51-113) are
enforced on requests.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes
from tests.oracle_lib import OracleScene, oracle, request

pytestmark = pytest.mark.gpu

RTOL = 1e-3
MATCH_FRACTION = 0.97


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


@pytest.mark.parametrize("sampler,mode", [(abi.SAMPLER_HALTON, abi.RANDOMIZE_NONE),
                                          (abi.SAMPLER_HALTON, abi.RANDOMIZE_PERMUTEDIGITS),
                                          (abi.SAMPLER_HALTON, abi.RANDOMIZE_OWEN),
                                          (abi.SAMPLER_ZSOBOL, abi.RANDOMIZE_NONE),
                                          (abi.SAMPLER_ZSOBOL, abi.RANDOMIZE_FASTOWEN),
                                          (abi.SAMPLER_ZSOBOL, abi.RANDOMIZE_OWEN)])
@pytest.mark.parametrize("lens", [False, True])
def test_raygen_words_and_rays_bit_exact(sampler, mode, lens):
    scene = scenes.cornell_box(24, 20, 1)
    if lens:
        eye = (0.0, 1.0, 3.94)
        scene.lens = scenes.thin_lens(eye, (0, 1, 0), (0, 1, 0), 0.2)
    req = renderer.RenderRequest(24, 20, pixel_begin=5, pixel_count=300, sample_begin=3, sample_count=5,
                                 sampler=sampler, randomization=mode, seed=19317, total_samples=16)
    words, rays = build(scene).raygen(req)
    q = req.to_c()
    lanes = words.shape[0]
    cw = np.zeros((lanes, 11), np.uint32)
    cr = np.zeros((lanes, 6), np.float32)
    orc = OracleScene(scene)  # held: the oracle scene must outlive the call
    assert oracle().or_probe_raygen(orc.handle, C.byref(q), cw.ctypes.data, cr.ctypes.data, lanes) == 0
    np.testing.assert_array_equal(words, cw)
    if lens:
        np.testing.assert_allclose(rays, cr, rtol=0, atol=2e-6)
    else:
        np.testing.assert_array_equal(rays.view(np.uint32), cr.view(np.uint32))


@pytest.mark.parametrize("sampler,mode", [(abi.SAMPLER_HALTON, abi.RANDOMIZE_OWEN),
                                          (abi.SAMPLER_ZSOBOL, abi.RANDOMIZE_FASTOWEN)])
def test_hero_lanes_match_oracle(sampler, mode):
    scene = scenes.cornell_box(32, 32, 4)
    req = renderer.RenderRequest(32, 32, sample_count=4, sampler=sampler, randomization=mode)
    res = build(scene).sample(req)
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    g = res.packet_samples
    c = OracleScene(scene).sample(req.to_c())
    np.testing.assert_array_equal(c["status"], 0)
    for f in ("pixel", "sample_low", "sample_high"):
        np.testing.assert_array_equal(g[f], c[f])
    gr, cr = g["radiance"].astype(np.float64), c["radiance"].astype(np.float64)
    close = np.all(np.abs(gr - cr) <= RTOL * np.maximum(np.abs(cr), 1e-6) + 1e-7, axis=1)
    assert close.mean() >= MATCH_FRACTION, close.mean()


def test_scalar_fog_lanes_match_oracle_with_halton():
    scene = scenes.cornell_fog(24, 24, 4)
    req = renderer.RenderRequest(24, 24, sample_count=4, sampler=abi.SAMPLER_HALTON,
                                 randomization=abi.RANDOMIZE_PERMUTEDIGITS)
    res = build(scene).sample_scalar(req)
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    ref = OracleScene(scene).sample_scalar(req.to_c())
    np.testing.assert_array_equal(res.samples["wavelength"].view(np.uint32), ref["wavelength"].view(np.uint32))
    close = (res.samples["scatterings"] == ref["scatterings"]) & np.isclose(res.samples["radiance"], ref["radiance"],
                                                                            rtol=RTOL, atol=1e-7)
    assert close.mean() >= MATCH_FRACTION, close.mean()


def test_sampler_range_rules():
    rs = build(scenes.cornell_box(8, 8, 1))
    bad = [
        renderer.RenderRequest(8, 8, sampler=abi.SAMPLER_HALTON, randomization=abi.RANDOMIZE_FASTOWEN),
        renderer.RenderRequest(8, 8, sampler=abi.SAMPLER_ZSOBOL, sample_count=3, total_samples=3),
        renderer.RenderRequest(8, 8, sampler=abi.SAMPLER_ZSOBOL, sample_begin=14, sample_count=4, total_samples=16),
        renderer.RenderRequest(8, 8, sampler=abi.SAMPLER_SOBOL, seed=1 << 40),
    ]
    for req in bad:
        assert rs.sample(req).status == abi.RP_INVALID_ARGUMENT
    ok = renderer.RenderRequest(8, 8, sampler=abi.SAMPLER_ZSOBOL, sample_begin=12, sample_count=4, total_samples=16)
    assert rs.sample(ok).status == abi.RP_SUCCESS
