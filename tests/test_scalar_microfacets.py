"""Conductor and dielectric surfaces in the oracle's scalar transport (rypath_render_paths,
shaders/scalar_transport.h:589-900).  CPU only.

* The scalar and hero transports estimate the same pixel integral: on the Cornell-style box with
  a rough anisotropic conductor, rough glass and a Dirac mirror, and on the box with smooth
  dispersive glass, the scalar oracle's image agrees with the hero oracle's (whose BSDF
  proposals are pinned to rypath's shader headers) per pixel and over the image.
* The demo model's analytic floors under the unit sky: a smooth conductor seen head on reflects
  F(1) of the sky on every path; a smooth dielectric reflects F and transmits (1 - F) / eta^2,
  both reaching the sky (rypath's six-standard-error gate, tests/render_tests.cpp:525-549).
"""

import math

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle_film, request
from rypath_b200 import abi, scenes


def hero_and_scalar(name):
    if name == "microfacets":
        return (scenes.cornell_microfacets(16, 16, 1, transport=abi.TRANSPORT_HERO),
                scenes.cornell_microfacets(16, 16, 1, transport=abi.TRANSPORT_SCALAR))
    hero, scalar = scenes.cornell_features("cauchy", 16, 16, 1), scenes.cornell_features("cauchy", 16, 16, 1)
    scalar.transport = abi.TRANSPORT_SCALAR
    return hero, scalar


@pytest.mark.parametrize("name", ["microfacets", "cauchy"])
def test_scalar_and_hero_transports_agree_with_microfacets(name):
    hero, scalar = hero_and_scalar(name)
    spp = 2048
    s = OracleScene(scalar).sample_scalar(request(16, 16, spp, seed=3, sampler=abi.SAMPLER_INDEPENDENT))
    h = OracleScene(hero).sample(request(16, 16, spp, seed=4, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(s["status"] == abi.SAMPLE_SUCCESS) and np.all(h["status"] == abi.SAMPLE_SUCCESS)
    assert s["scatterings"].mean() > 2
    sv = (s["radiance"].astype(np.float64) * 470.0).reshape(spp, 256)  # uniform wavelength pdf 1/470
    hv = (np.sum(h["radiance"] / h["wavelength_pdfs"], axis=1) / 4.0).reshape(spp, 256)
    se = math.sqrt(sv.var() / sv.size + hv.var() / hv.size)
    assert abs(sv.mean() - hv.mean()) < 4 * se, (sv.mean(), hv.mean(), se)
    z = np.abs(sv.mean(0) - hv.mean(0)) / np.sqrt(sv.var(0) / spp + hv.var(0) / spp + 1e-30)
    assert np.mean(z < 3) > 0.97, np.mean(z < 3)


def conductor_fresnel(eta, k):
    return ((eta - 1) ** 2 + k ** 2) / ((eta + 1) ** 2 + k ** 2)


def demo_film(scene, paths=16384, seed=0x9E314FD9):
    film = oracle_film(scene, 1, 1, paths, seed=seed, sampler=abi.SAMPLER_INDEPENDENT, scalar=True, chunk=paths)
    return (film["sum"] + film["correction"])[0] / film["count"][0]


def test_demo_mirror_floor_reflects_the_sky():
    sky = demo_film(scenes.demo_floor(None))
    scene = scenes.demo_floor((0.5,) * 8)
    scene.materials[0] = scenes.conductor_material(scene, 0.3, 2.5, 0.0, 0.0)
    mirror = demo_film(scene)
    np.testing.assert_allclose(mirror, conductor_fresnel(0.3, 2.5) * sky, rtol=1e-4)


@pytest.mark.parametrize("eta", [1.5, 2.2])
def test_demo_glass_floor_reflects_and_transmits_the_sky(eta):
    paths = 32768
    scene = scenes.demo_floor((0.5,) * 8)
    scene.materials[0] = scenes.dielectric_material(scene, eta, 0.0)
    out = OracleScene(scene).sample_scalar(request(1, 1, paths, seed=19317, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(out["status"] == abi.SAMPLE_SUCCESS) and np.all(out["scatterings"] == 1)
    F = ((eta - 1) / (eta + 1)) ** 2
    expected = F + (1 - F) / eta ** 2
    r = out["radiance"].astype(np.float64)
    e = np.float32(eta)
    assert set(np.unique(out["radiance"]).tolist()) <= {1.0, float(np.float32(1) / (e * e))}
    assert abs(r.mean() - expected) <= 6 * r.std(ddof=1) / math.sqrt(paths) + 2e-5, (r.mean(), expected)


def test_rough_conductor_floor_keeps_energy_below_one():
    """A rough conductor under the unit sky returns at most the sky (and well above zero)."""
    scene = scenes.demo_floor((0.5,) * 8)
    scene.materials[0] = scenes.conductor_material(scene, 0.2, 3.4, 0.3, 0.3)
    out = OracleScene(scene).sample_scalar(request(1, 1, 32768, seed=5, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(out["status"] == abi.SAMPLE_SUCCESS)
    mean = out["radiance"].astype(np.float64).mean()
    assert 0.6 < mean < conductor_fresnel(0.2, 3.4) + 0.02, mean
