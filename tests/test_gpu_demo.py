"""GPU parity of the demo model (`rypath --render-demo`, scalar transport).

* the unit sky and the unobstructed Lambertian floor against rypath's analytic moments
  (tests/render_reference.cpp analytic_xyz), 32768 paths of one pixel, within rypath's own six
  standard errors (tests/render_tests.cpp:525-549);
* the demo scene's lanes against the oracle: identity and status bit-exact, wavelengths bit
  exact, radiance within 1e-3 for at least 97% of lanes (sin / cos of the sky sample and the
  hemisphere direction differ in the last bits between CUDA and the host), the same
  scattering counts for at least 99%;
* the device film equals the host reduction (FilmBatch's demo arithmetic, pinned by
  test_demo.py) of the same device samples;
* the device's demo image against rypath's CPU estimator within five combined standard errors
  over replicates (tests/render_tests.cpp:570-603).
"""

import json
import os

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes
from tests.oracle_lib import OracleScene, oracle, request

pytestmark = pytest.mark.gpu

# rypath's analytic moments and CPU estimator, recorded by tests/golden/make_demo_golden.py
GOLDEN = json.loads(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                      "demo_reference.json")).read())


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def film_xyz(film):
    return (film["sum"] + film["correction"]) / film["count"][:, None]


@pytest.mark.parametrize("case", ["sky", "floor", "grey"])
def test_demo_device_meets_analytic_moments(case):
    reflectance = GOLDEN["analytic"][case]["reflectance"]
    mean, var = np.array(GOLDEN["analytic"][case]["mean"]), np.array(GOLDEN["analytic"][case]["variance"])
    paths = 32768
    rs = build(scenes.demo_floor(reflectance))
    st, diag, film = rs.render_film(renderer.RenderSettings(1, 1, samples=paths, batch_size=paths, seed=0x9E314FD9,
                                                            sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert st == abi.RP_SUCCESS, diag
    xyz = film_xyz(film)[0]
    se = np.sqrt(var / paths)
    assert np.all(np.abs(xyz - mean) <= 6 * se + 2e-5 * np.maximum(1, np.abs(mean))), (xyz, mean, se)


@pytest.mark.parametrize("sampler", [abi.SAMPLER_INDEPENDENT])  # QMC samplers need the PBRT model
def test_demo_lanes_match_oracle(sampler):
    scene = scenes.demo_scene(64, 48, 8)
    rs = build(scene)
    g = rs.sample_scalar(renderer.RenderRequest(64, 48, sample_count=8, sampler=sampler))
    rs.close()
    assert g.status == abi.RP_SUCCESS, g.diagnostic
    g = g.samples
    c = OracleScene(scene).sample_scalar(request(64, 48, 8, sampler=sampler))
    for f in ("status", "pixel", "sample_low", "sample_high"):
        np.testing.assert_array_equal(g[f], c[f])
    np.testing.assert_array_equal(g["wavelength"].view(np.uint32), c["wavelength"].view(np.uint32))
    close = np.abs(g["radiance"].astype(np.float64) - c["radiance"]) <= 1e-3 * np.maximum(np.abs(c["radiance"]), 1e-6)
    assert close.mean() >= 0.97, close.mean()
    assert (g["scatterings"] == c["scatterings"]).mean() >= 0.99
    assert c["scatterings"].max() >= 4 and (c["radiance"] > 0).mean() > 0.9


def test_demo_device_film_equals_host_reduction():
    scene = scenes.demo_scene(16, 12, 8)
    rs = build(scene)
    st, diag, film = rs.render_film(renderer.RenderSettings(16, 12, samples=8, batch_size=4, seed=3,
                                                            sampler=abi.SAMPLER_INDEPENDENT))
    assert st == abi.RP_SUCCESS, diag
    res = rs.sample_scalar(renderer.RenderRequest(16, 12, seed=3, sample_count=8, sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    host = np.zeros(16 * 12, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    samples = np.ascontiguousarray(res.samples)
    assert oracle().or_scalar_film_add(samples.ctypes.data, samples.size, cie.ctypes.data, 16 * 12,
                                       host.ctypes.data, 1) == 0
    np.testing.assert_array_equal(film["count"], host["count"])
    np.testing.assert_array_equal(film["sum"], host["sum"])
    np.testing.assert_array_equal(film["correction"], host["correction"])


def test_demo_device_matches_rypath_estimator():
    est = GOLDEN["estimator"]
    w, h, spp = est["width"], est["height"], est["samples"]
    assert est["max_scatterings"] >= 4
    ref, dev = est["means"], []
    rs = build(scenes.demo_scene(w, h, spp))
    for k in range(est["replicates"]):
        st, diag, film = rs.render_film(renderer.RenderSettings(w, h, samples=spp, batch_size=spp, seed=0x71AC6A05 + k,
                                                                sampler=abi.SAMPLER_INDEPENDENT))
        assert st == abi.RP_SUCCESS, diag
        dev.append(film_xyz(film).mean(axis=0))
    rs.close()
    ref, dev = np.array(ref), np.array(dev)
    se = np.sqrt(ref.var(axis=0, ddof=1) / len(ref) + dev.var(axis=0, ddof=1) / len(dev))
    assert np.all(np.abs(ref.mean(0) - dev.mean(0)) <= 5 * se + 2e-5), (ref.mean(0), dev.mean(0), se)
