"""Conductor and dielectric surfaces in the CUDA scalar transport against the oracle.

* Lanes (rp_cuda_sample_scalar): identity, status and wavelength bit for bit; radiance within
  1e-3 and the same scattering count for at least 97% of lanes (sin / cos / sqrt round
  differently on the device, so a few paths take another branch) on the Cornell-style box
  with a rough anisotropic conductor, rough glass and a mirror (Sobol, Halton, independent),
  the box with smooth dispersive glass, the fog-filled box with a rough glass box, the demo
  scene with metal and glass boxes, and, under an environment image (light samples from its
  importance table, MIS on escape), the Cornell-style box and the fog-filled box, and the
  textured box (image reflectance at the hit's footprint).
* The device film's per-pixel XYZ within 3 sigma of the oracle's on independent seeds.
* The demo model's mirror floor reflects F(1) of the sky on every path.
* The QMC samplers' depth limits of rypath (sampler_max_depth, src/sampling.cpp:129-135):
  a dielectric lowers them, and QMC needs the PBRT model.
"""

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu

MATCH_FRACTION = 0.97


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def fog_glass(width, height, spp):
    scene = scenes.cornell_fog(width, height, spp, max_depth=16)
    base = len(scene.materials)
    scene.materials.append(scenes.dielectric_material(scene, 1.5, 0.05))
    scene.instances[6].material = base
    return scene


def cauchy(width, height, spp):
    scene = scenes.cornell_features("cauchy", width, height, spp)
    scene.transport = abi.TRANSPORT_SCALAR
    return scene


CASES = [("microfacets", abi.SAMPLER_SOBOL), ("microfacets", abi.SAMPLER_HALTON),
         ("microfacets", abi.SAMPLER_INDEPENDENT), ("cauchy", abi.SAMPLER_SOBOL), ("fog_glass", abi.SAMPLER_SOBOL),
         ("demo", abi.SAMPLER_INDEPENDENT), ("env_image", abi.SAMPLER_SOBOL), ("fog_env", abi.SAMPLER_SOBOL),
         ("texture", abi.SAMPLER_SOBOL)]


def make(name, width, height, spp):
    if name == "microfacets":
        return scenes.cornell_microfacets(width, height, spp)
    if name == "cauchy":
        return cauchy(width, height, spp)
    if name == "fog_glass":
        return fog_glass(width, height, spp)
    if name in ("env_image", "texture"):
        scene = scenes.cornell_features(name, width, height, spp)
        scene.transport = abi.TRANSPORT_SCALAR
        return scene
    if name == "fog_env":
        from test_scalar_environment import fog_under_sky

        return fog_under_sky(width, height, spp)
    return scenes.demo_microfacets(width, height, spp)


@pytest.mark.parametrize("name,sampler", CASES)
def test_microfacet_lanes_match_the_oracle(name, sampler):
    scene = make(name, 32, 32, 4)
    rand = abi.RANDOMIZE_NONE if sampler == abi.SAMPLER_HALTON else abi.RANDOMIZE_OWEN
    q = request(32, 32, 4, sampler=sampler, randomization=rand)
    ref = OracleScene(scene).sample_scalar(q)
    res = build(scene).sample_scalar(renderer.RenderRequest(32, 32, seed=q.seed, sample_count=4, sampler=sampler,
                                                            randomization=rand))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    got = res.samples
    for f in ("status", "pixel", "sample_low", "sample_high", "random_words"):
        np.testing.assert_array_equal(got[f], ref[f])
    np.testing.assert_array_equal(got["wavelength"].view(np.uint32), ref["wavelength"].view(np.uint32))
    same = (got["scatterings"] == ref["scatterings"]) & np.isclose(got["radiance"], ref["radiance"], rtol=1e-3,
                                                                   atol=1e-7)
    assert np.mean(same) >= MATCH_FRACTION, np.mean(same)
    assert np.all(ref["status"] == abi.SAMPLE_SUCCESS) and ref["scatterings"].mean() > 1.5


def test_microfacet_film_statistics_agree_with_the_oracle():
    scene = scenes.cornell_microfacets(16, 16, 64)
    rs = build(scene)
    st, diag, film = rs.render_film(renderer.RenderSettings(16, 16, samples=512, batch_size=128, seed=5,
                                                            sampler=abi.SAMPLER_INDEPENDENT))
    rs.close()
    assert st == abi.RP_SUCCESS, diag
    ref = OracleScene(scene).sample_scalar(request(16, 16, 512, seed=6, sampler=abi.SAMPLER_INDEPENDENT))
    host = np.zeros(256, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_scalar_film_add(ref.ctypes.data, ref.size, cie.ctypes.data, 256, host.ctypes.data, 0) == 0

    def moments(f):
        n = f["count"][:, None].astype(np.float64)
        mean = (f["sum"] + f["correction"]) / n
        return mean, np.maximum(f["square"] / n - mean ** 2, 0) / n

    m1, v1 = moments(film)
    m2, v2 = moments(host)
    z = np.abs(m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(z < 3) > 0.97, np.mean(z < 3)
    assert abs(m1.sum() / m2.sum() - 1) < 0.03


def test_demo_mirror_floor_on_the_device():
    def film_of(scene):
        rs = build(scene)
        st, diag, film = rs.render_film(renderer.RenderSettings(1, 1, samples=16384, batch_size=16384,
                                                                seed=0x9E314FD9, sampler=abi.SAMPLER_INDEPENDENT))
        rs.close()
        assert st == abi.RP_SUCCESS, diag
        return (film["sum"] + film["correction"])[0] / film["count"][0]

    sky = film_of(scenes.demo_floor(None))
    scene = scenes.demo_floor((0.5,) * 8)
    scene.materials[0] = scenes.conductor_material(scene, 0.3, 2.5, 0.0, 0.0)
    F = ((0.3 - 1) ** 2 + 2.5 ** 2) / ((0.3 + 1) ** 2 + 2.5 ** 2)
    np.testing.assert_allclose(film_of(scene), F * sky, rtol=1e-4)


def sample_status(scene, sampler, randomization=abi.RANDOMIZE_OWEN):
    rs = build(scene)
    res = rs.sample_scalar(renderer.RenderRequest(4, 4, sample_count=1, sampler=sampler, randomization=randomization))
    rs.close()
    return res.status, res.diagnostic


@pytest.mark.parametrize("sampler,plain,glass", [(abi.SAMPLER_SOBOL, 127, 113), (abi.SAMPLER_ZSOBOL, 127, 113),
                                                 (abi.SAMPLER_HALTON, 124, 110)])
def test_qmc_depth_limits(sampler, plain, glass):
    rand = abi.RANDOMIZE_NONE if sampler == abi.SAMPLER_HALTON else abi.RANDOMIZE_OWEN
    for depth, dielectric, ok in [(plain, False, True), (plain + 1, False, False), (glass, True, True),
                                  (glass + 1, True, False)]:
        scene = scenes.cornell_microfacets(4, 4, 1, max_depth=depth)
        if not dielectric:  # every material counts (scene_has_dielectrics, src/render.cpp:927-932)
            scene.materials[-2] = scenes.conductor_material(scene, 0.2, 3.4, 0.3, 0.08)
        st, diag = sample_status(scene, sampler, rand)
        assert (st == abi.RP_SUCCESS) == ok, (depth, dielectric, diag)
        if not ok:
            assert st == abi.RP_INVALID_ARGUMENT and f"maxdepth at most {glass if dielectric else plain}" in diag
    st, _ = sample_status(scenes.cornell_microfacets(4, 4, 1, max_depth=10000), abi.SAMPLER_INDEPENDENT)
    assert st == abi.RP_SUCCESS


def test_qmc_samplers_need_the_pbrt_model():
    st, diag = sample_status(scenes.demo_scene(4, 4, 1), abi.SAMPLER_SOBOL)
    assert st == abi.RP_INVALID_ARGUMENT and "PBRT" in diag
    assert sample_status(scenes.demo_scene(4, 4, 1), abi.SAMPLER_INDEPENDENT)[0] == abi.RP_SUCCESS
