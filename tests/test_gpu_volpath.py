"""CUDA scalar transport with homogeneous media (rp_cuda_sample_scalar) against the oracle.

Per lane on the fog-filled Cornell box: identity, status and wavelength bit for bit; scattering
counts and radiance within the per-lane tolerance of the hero parity tests (the device's
exp/log/sin/cos round differently from the host's, so a small fraction of paths may take a
different branch and are allowed to differ).  Whole transport: the analytic answers of
rypath's medium tests (tests/medium_render_tests.cpp), the six-standard-error gate.  The device
film equals the host reduction of the same samples, and any split of a request into pixel or
sample ranges returns the same lanes.
"""

import math

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-3
MATCH_FRACTION = 0.97
NONE = abi.RP_NONE


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def to_request(q):
    return renderer.RenderRequest(q.width, q.height, seed=q.seed, pixel_begin=q.pixel_begin, pixel_count=q.pixel_count,
                                  sample_begin=q.sample_begin, sample_count=q.sample_count, sampler=q.sampler_kind,
                                  randomization=q.randomization, boundary_limit=q.boundary_limit)


@pytest.mark.parametrize("sampler", [abi.SAMPLER_SOBOL, abi.SAMPLER_INDEPENDENT])
def test_fog_box_lanes_match_the_oracle(sampler):
    scene = scenes.cornell_fog(32, 32, 4)
    q = request(32, 32, 4, sampler=sampler)
    ref = OracleScene(scene).sample_scalar(q)
    res = build(scene).sample_scalar(to_request(q))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    got = res.samples
    for f in ("status", "pixel", "sample_low", "sample_high", "random_words"):
        np.testing.assert_array_equal(got[f], ref[f])
    np.testing.assert_array_equal(got["wavelength"].view(np.uint32), ref["wavelength"].view(np.uint32))
    same_path = got["scatterings"] == ref["scatterings"]
    close = np.isclose(got["radiance"], ref["radiance"], rtol=RTOL, atol=1e-7)
    assert np.mean(same_path & close) >= MATCH_FRACTION, np.mean(same_path & close)
    assert ref["scatterings"].mean() > 1.5  # the medium scatters


def medium(a, s, emission=0.0, g=0.0):
    return dict(sigma_a=a, sigma_s=s, emission=emission, g=g)


def plane(z, positive, media=(NONE, NONE), **kw):
    return dict(z=z, positive=positive, media=media, **kw)


def gpu_paths(scene, count=32768):
    res = build(scene).sample_scalar(renderer.RenderRequest(1, 1, seed=19317, sample_count=count,
                                                             sampler=abi.SAMPLER_INDEPENDENT))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    return res.samples


def mean_gate(out, expected, numerical=2e-5):
    residual = out["radiance"].astype(np.float64) - expected
    n = residual.size
    mean = residual.mean()
    var = max(0.0, (np.sum(residual ** 2) - residual.sum() * mean) / (n - 1))
    assert abs(mean) <= 6 * math.sqrt(var / n) + numerical, (mean, math.sqrt(var / n))


def test_slab_beer_and_emission_on_the_device():
    planes = [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))]
    mean_gate(gpu_paths(scenes.slab_scene([medium(.6, 0, 2)], planes)), 2 - math.exp(-.6))
    mean_gate(gpu_paths(scenes.slab_scene([medium(.6, 0, 2)], planes, max_depth=0)), math.exp(-.6))


def test_infinite_emitting_medium_on_the_device():
    for depth in (0, 1, 2, 3):
        scene = scenes.slab_scene([medium(.4, .6, 2, .65)], [plane(-100000, True)], camera_medium=0,
                                  environment=0.0, max_depth=depth)
        mean_gate(gpu_paths(scene, 4096), 2 * (1 - .6 ** depth))


def test_geometry_free_camera_medium_on_the_device():
    """scalar_sky_step: no geometry at all, an all-space emitting medium."""
    scene = scenes.slab_scene([medium(.4, .6, 2, .65)], [], camera_medium=0, environment=0.0, max_depth=2)
    mean_gate(gpu_paths(scene, 4096), 2 * (1 - .6 ** 2))


def test_nested_media_and_split_interfaces_on_the_device():
    media = [medium(.2, 0), medium(.8, 0)]
    planes = [plane(1, False, (0, NONE)), plane(1.5, False, (1, 0)), plane(2.5, True, (1, 0)),
              plane(3, True, (0, NONE))]
    mean_gate(gpu_paths(scenes.slab_scene(media, planes)), math.exp(-1.))
    split = [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))] + [plane(1 + i / 8, True) for i in range(1, 8)]
    mean_gate(gpu_paths(scenes.slab_scene([medium(1, 0)], split, max_depth=0)), math.exp(-1.))


def test_single_scatter_slab_on_the_device():
    from test_volpath_oracle import single_scatter_slab

    for g in (0.0, .65, -.55):
        scene = scenes.slab_scene([medium(.3, .7, 0, g)], [plane(-1, False, (0, NONE)), plane(1, True, (0, NONE))],
                                  camera_medium=0)
        mean_gate(gpu_paths(scene), single_scatter_slab(g), numerical=4e-5)


def test_point_light_through_media_on_the_device():
    diffuse = abi.Material()
    diffuse.scattering, diffuse.kind, diffuse.scalar_value = abi.DIFFUSE, abi.REFLECTANCE_CONSTANT, .5
    light = dict(position=(0.0, 0.0, 0.0), intensity=np.full(471, 2.0, np.float32), kind=abi.POINT_LIGHT)
    planes = [plane(1, False, material=1), plane(.25, False, (0, NONE)), plane(.5, True, (0, NONE)),
              plane(-5e-6, True, material=1)]
    scene = scenes.slab_scene([medium(.4, 0)], planes, environment=0.0, materials=[diffuse], positional=[light])
    mean_gate(gpu_paths(scene), math.exp(-.4 * .5) / math.pi)


def test_partitions_return_the_same_lanes():
    """tests/medium_render_tests.cpp:401-440: pixel and sample ranges of one request."""
    scene = scenes.slab_scene([medium(.2, .8, .4, .6)], [plane(1, False, (0, NONE)), plane(2, True, (0, NONE)),
                                                          plane(1.5, True)], max_depth=3)
    rs = build(scene)
    for sampler, randomization in ((abi.SAMPLER_INDEPENDENT, 0), (abi.SAMPLER_SOBOL, abi.RANDOMIZE_NONE),
                                   (abi.SAMPLER_SOBOL, abi.RANDOMIZE_OWEN)):
        whole = rs.sample_scalar(renderer.RenderRequest(2, 2, seed=19317, sample_count=73, sampler=sampler,
                                                        randomization=randomization))
        assert whole.status == abi.RP_SUCCESS, whole.diagnostic
        key = {(int(r["pixel"]), int(r["sample_low"])): r for r in whole.samples}
        for pixel in (0, 2):
            for begin, count in ((0, 31), (31, 42)):
                part = rs.sample_scalar(renderer.RenderRequest(2, 2, seed=19317, pixel_begin=pixel, pixel_count=2,
                                                               sample_begin=begin, sample_count=count, sampler=sampler,
                                                               randomization=randomization))
                assert part.status == abi.RP_SUCCESS, part.diagnostic
                for r in part.samples:
                    w = key[(int(r["pixel"]), int(r["sample_low"]))]
                    assert r.tobytes() == w.tobytes()


def test_device_film_equals_host_reduction_of_the_same_samples():
    scene = scenes.cornell_fog(16, 16, 8)
    rs = build(scene)
    settings = renderer.RenderSettings(width=16, height=16, samples=8, batch_size=4, seed=1)
    st, diag, film = rs.render_film(settings)
    assert st == abi.RP_SUCCESS, diag
    res = rs.sample_scalar(renderer.RenderRequest(16, 16, seed=1, sample_count=8))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    host = np.zeros(256, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    samples = np.ascontiguousarray(res.samples)
    assert oracle().or_scalar_film_add(samples.ctypes.data, samples.size, cie.ctypes.data, 256, host.ctypes.data, 0) == 0
    np.testing.assert_array_equal(film["count"], host["count"])
    np.testing.assert_allclose(film["sum"] + film["correction"], host["sum"] + host["correction"], rtol=1e-12,
                               atol=1e-300)


def test_fog_film_statistics_agree_with_the_oracle():
    """Per-pixel XYZ of the device film within 3 sigma of the oracle's, on independent seeds."""
    scene = scenes.cornell_fog(16, 16, 64)
    rs = build(scene)
    settings = renderer.RenderSettings(width=16, height=16, samples=256, batch_size=64, seed=5,
                                       sampler=abi.SAMPLER_INDEPENDENT)
    st, diag, film = rs.render_film(settings)
    assert st == abi.RP_SUCCESS, diag
    ref = OracleScene(scene).sample_scalar(request(16, 16, 256, seed=6, sampler=abi.SAMPLER_INDEPENDENT))
    host = np.zeros(256, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_scalar_film_add(ref.ctypes.data, ref.size, cie.ctypes.data, 256, host.ctypes.data, 0) == 0

    def moments(f):
        n = f["count"][:, None].astype(np.float64)
        mean = (f["sum"] + f["correction"]) / n
        var = np.maximum(f["square"] / n - mean ** 2, 0) / n
        return mean, var

    m1, v1 = moments(film)
    m2, v2 = moments(host)
    z = np.abs(m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(z < 3) > 0.98, np.mean(z < 3)
    assert abs(m1.sum() / m2.sum() - 1) < 0.03


def test_scene_validation_for_the_two_transports():
    fog = scenes.cornell_fog(8, 8, 1)
    fog.transport = abi.TRANSPORT_HERO
    built = renderer.build_renderer(fog)
    assert built.status == abi.RP_INVALID_ARGUMENT and "vacuum" in built.diagnostic
    layered = scenes.cornell_box(8, 8, 1)
    layered.materials[0].scattering = 5  # rypath's coated diffuse: not built for either transport
    layered.transport = abi.TRANSPORT_SCALAR
    built = renderer.build_renderer(layered)
    assert built.status == abi.RP_NOT_BUILT
    rs = build(scenes.cornell_fog(8, 8, 1))
    res = rs.sample(renderer.RenderRequest(8, 8))
    assert res.status == abi.RP_INVALID_ARGUMENT
