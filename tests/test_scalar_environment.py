"""The environment image in the oracle's scalar transport (shaders/scalar_lighting.h:14-23,
:102-113; shaders/scalar_transport.h:219-224, :431-443): light samples from its compensated
importance table, radiance on escape with MIS against them.  The scalar and hero transports
estimate the same pixel integral under the sky image of the Cornell-style box (per pixel and
over the image), and a fog-filled box under the same sky renders without failures.  CPU only."""

import math

import numpy as np

from oracle_lib import OracleScene, request
from rypath_b200 import abi, images, scenes


def test_scalar_and_hero_transports_agree_under_the_environment_image():
    hero = scenes.cornell_features("env_image", 16, 16, 1)
    scalar = scenes.cornell_features("env_image", 16, 16, 1)
    scalar.transport = abi.TRANSPORT_SCALAR
    spp = 2048
    s = OracleScene(scalar).sample_scalar(request(16, 16, spp, seed=3, sampler=abi.SAMPLER_INDEPENDENT))
    h = OracleScene(hero).sample(request(16, 16, spp, seed=4, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(s["status"] == abi.SAMPLE_SUCCESS) and np.all(h["status"] == abi.SAMPLE_SUCCESS)
    sv = (s["radiance"].astype(np.float64) * 470.0).reshape(spp, 256)
    hv = (np.sum(h["radiance"] / h["wavelength_pdfs"], axis=1) / 4.0).reshape(spp, 256)
    se = math.sqrt(sv.var() / sv.size + hv.var() / hv.size)
    assert abs(sv.mean() - hv.mean()) < 4 * se, (sv.mean(), hv.mean(), se)
    z = np.abs(sv.mean(0) - hv.mean(0)) / np.sqrt(sv.var(0) / spp + hv.var(0) / spp + 1e-30)
    assert np.mean(z < 3) > 0.97, np.mean(z < 3)


def fog_under_sky(width=16, height=16, spp=4):
    scene = scenes.cornell_fog(width, height, spp, max_depth=16)
    scene.instances[-2].emission = abi.RP_NONE  # the area light off: the sky alone
    scene.emissions = []
    scene.images = images.ImageSet()
    scene.images.environment_image = scene.images.add_image(images.sky_image(32, seed=3), wrap=abi.WRAP_CLAMP)
    scene.images.environment_scale = 1.5
    return scene


def test_fog_box_under_the_environment_image():
    out = OracleScene(fog_under_sky()).sample_scalar(request(16, 16, 64, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(out["status"] == abi.SAMPLE_SUCCESS)
    assert (out["radiance"] > 0).mean() > 0.5 and out["scatterings"].mean() > 1


def test_scalar_and_hero_transports_agree_on_image_reflectance():
    """The textured Cornell-style box (sRGB trilinear, float EWA, half point, RGB sigmoid) in
    both transports: image reflectance at the hit's footprint, per wavelength."""
    hero = scenes.cornell_features("texture", 16, 16, 1)
    scalar = scenes.cornell_features("texture", 16, 16, 1)
    scalar.transport = abi.TRANSPORT_SCALAR
    spp = 2048
    s = OracleScene(scalar).sample_scalar(request(16, 16, spp, seed=3, sampler=abi.SAMPLER_INDEPENDENT))
    h = OracleScene(hero).sample(request(16, 16, spp, seed=4, sampler=abi.SAMPLER_INDEPENDENT))
    assert np.all(s["status"] == abi.SAMPLE_SUCCESS) and np.all(h["status"] == abi.SAMPLE_SUCCESS)
    sv = (s["radiance"].astype(np.float64) * 470.0).reshape(spp, 256)
    hv = (np.sum(h["radiance"] / h["wavelength_pdfs"], axis=1) / 4.0).reshape(spp, 256)
    se = math.sqrt(sv.var() / sv.size + hv.var() / hv.size)
    assert abs(sv.mean() - hv.mean()) < 4 * se, (sv.mean(), hv.mean(), se)
    z = np.abs(sv.mean(0) - hv.mean(0)) / np.sqrt(sv.var(0) / spp + hv.var(0) / spp + 1e-30)
    assert np.mean(z < 3) > 0.97, np.mean(z < 3)
