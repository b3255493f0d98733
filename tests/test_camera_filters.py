"""Thin-lens camera and Gaussian pixel filter (shaders/render.metal:200-236, :366-432).

CPU (oracle): the lens words are the reference's (Sobol dimensions 1022/1023, Philox block
0xc0000000; tests/lens_render_tests.cpp:226-330 checks the same streams), every lens ray passes
through the point where its pinhole ray meets the plane of focus, the lens words leave the
camera and wavelength words unchanged, and Gaussian filter offsets stay inside the radii.
GPU: raygen words (lens words included) bit-exact, rays bit-exact for the Gaussian filter and
within 2e-6 for the lens (its concentric-disk sin/cos), and the hero film with a Gaussian
filter equals the oracle's `PacketFilmBatch` reduction of the same lanes, filter weight (the
table's integral) included.
"""

import ctypes as C

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle
from rypath_b200 import abi, renderer, scenes


def lens_scene(radius=0.25, focus=None):
    s = scenes.cornell_box(16, 12, 1)
    eye, target, up = (0.3, 1.1, 3.94), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0)
    s.camera = scenes.pinhole_camera(eye, target, up, 40.0, 16, 12)
    s.lens = scenes.thin_lens(eye, target, up, radius, focus)
    return s


def gaussian_scene(rx=1.5, ry=1.5, sigma=0.5):
    s = scenes.cornell_box(16, 12, 1)
    s.filter_kind = abi.FILTER_GAUSSIAN
    s.filter_radius = (rx, ry)
    s.filter_sigma = sigma
    return s


def probe(scene, sampler, lanes_req=None):
    orc = OracleScene(scene)
    req = lanes_req or renderer.RenderRequest(16, 12, pixel_begin=3, pixel_count=150, sample_begin=17, sample_count=5,
                                              sampler=sampler, seed=19317)
    q = req.to_c()
    lanes = q.pixel_count * q.sample_count
    words = np.zeros((lanes, 11), np.uint32)
    rays = np.zeros((lanes, 6), np.float32)
    assert oracle().or_probe_raygen(orc.handle, C.byref(q), words.ctypes.data, rays.ctypes.data, lanes) == 0
    return req, words, rays


@pytest.mark.parametrize("sampler", [abi.SAMPLER_SOBOL, abi.SAMPLER_INDEPENDENT])
def test_lens_words_leave_camera_words_and_focus(sampler):
    _, pin_words, pin_rays = probe(lens_scene(0.0), sampler)
    _, words, rays = probe(lens_scene(0.25), sampler)
    np.testing.assert_array_equal(words[:, :9], pin_words[:, :9])
    assert np.all(pin_words[:, 9:] == 0) and np.any(words[:, 9:] != 0)
    # every lens ray meets its pinhole ray in the plane of focus (focus distance along the
    # camera axis): closest approach of the two lines, in units of the scene
    scene = lens_scene(0.25)
    origin = np.array(scenes.pinhole_camera((0.3, 1.1, 3.94), (0, 1, 0), (0, 1, 0), 40.0, 16, 12)[0], np.float64)
    axis = np.array((0.0, 1.0, 0.0)) - np.array((0.3, 1.1, 3.94))
    axis /= np.linalg.norm(axis)
    focus = scene.lens[1]
    p = pin_rays[:, 3:].astype(np.float64)
    t = focus / (p @ axis)
    focus_points = origin + p * t[:, None]
    o, d = rays[:, :3].astype(np.float64), rays[:, 3:].astype(np.float64)
    assert np.all(np.abs(np.linalg.norm(o - origin, axis=1)) <= 0.25 * (1 + 1e-5))
    w = focus_points - o
    miss = np.linalg.norm(w - (np.sum(w * d, axis=1))[:, None] * d, axis=1)
    assert miss.max() < 2e-5, miss.max()


def test_gaussian_offsets_stay_in_the_filter_support():
    for sampler in (abi.SAMPLER_SOBOL, abi.SAMPLER_INDEPENDENT):
        _, box_words, box_rays = probe(scenes.cornell_box(16, 12, 1), sampler)
        _, words, rays = probe(gaussian_scene(1.5, 0.75, 0.5), sampler)
        np.testing.assert_array_equal(words, box_words)
        assert np.all(np.isfinite(rays))
        assert not np.array_equal(rays, box_rays)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["lens", "gaussian"])
@pytest.mark.parametrize("sampler", [abi.SAMPLER_SOBOL, abi.SAMPLER_INDEPENDENT])
def test_device_raygen_matches_oracle(kind, sampler):
    scene = lens_scene(0.25) if kind == "lens" else gaussian_scene(1.5, 0.75, 0.5)
    req, words, rays = probe(scene, sampler)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    gw, gr = built.scene.raygen(req)
    np.testing.assert_array_equal(gw, words)
    if kind == "gaussian":
        np.testing.assert_array_equal(gr.view(np.uint32), rays.view(np.uint32))
    else:
        np.testing.assert_allclose(gr, rays, rtol=0, atol=2e-6)


@pytest.mark.gpu
def test_device_gaussian_film_matches_oracle_film():
    scene = gaussian_scene(1.5, 1.5, 0.5)
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    res = built.scene.sample(renderer.RenderRequest(16, 12, sample_count=4))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    lanes = res.packet_samples
    assert np.all(lanes["filter_weight"] == lanes["filter_weight"][0]) and lanes["filter_weight"][0] > 0
    settings = renderer.RenderSettings(width=16, height=12, samples=4, batch_size=4, seed=1)
    st, diag, film = built.scene.render_film(settings)
    assert st == abi.RP_SUCCESS, diag
    ref = np.zeros(16 * 12, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    lanes = np.ascontiguousarray(lanes)
    assert oracle().or_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, 16 * 12, ref.ctypes.data) == 0
    assert film.tobytes() == ref.tobytes()
