"""The oracle's scalar transport with homogeneous media (rypath_render_paths), pinned.

* The medium equations (shaders/medium.h: segment, flight, phase, phase_sample) against the
  reference's own header compiled for the host (oracle/_ref/libref.so), bit for bit.
* Whole-transport estimates against the analytic answers of rypath's medium tests
  (tests/medium_render_tests.cpp): Beer transmission with slab emission, depth-zero Beer,
  wavelength-dependent Beer, an infinite emitting medium at finite depth, nested and reversed
  interfaces, split null interfaces, and the single-scatter slab quadrature that checks the
  phase/light MIS.  Each gate is rypath's: the mean residual within six standard errors plus
  a stated numerical allowance, on independent (Philox) paths with seed 19317.
* The scalar and hero transports agree on the vacuum Cornell box (both estimate the same
  pixel integral).
"""

import ctypes as C
import math

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, reference, request
from rypath_b200 import abi, scenes

NONE = abi.RP_NONE


def medium(a, s, emission=0.0, g=0.0):
    return dict(sigma_a=a, sigma_s=s, emission=emission, g=g)


def plane(z, positive, media=(NONE, NONE), **kw):
    return dict(z=z, positive=positive, media=media, **kw)


def paths(scene, count=32768, threads=0):
    q = request(1, 1, count, seed=19317, sampler=abi.SAMPLER_INDEPENDENT)
    out = OracleScene(scene).sample_scalar(q, threads)
    assert np.all(out["status"] == abi.SAMPLE_SUCCESS)
    assert np.all(np.isfinite(out["radiance"])) and np.all(out["radiance"] >= 0)
    return out


def mean_gate(out, expected, numerical=2e-5):
    """tests/medium_render_tests.cpp:86-101: six standard errors plus a numerical allowance."""
    residual = out["radiance"].astype(np.float64) - expected
    n = residual.size
    mean = residual.mean()
    var = max(0.0, (np.sum(residual ** 2) - residual.sum() * mean) / (n - 1))
    assert abs(mean) <= 6 * math.sqrt(var / n) + numerical, (mean, math.sqrt(var / n))


def medium_queries(rng, n):
    q = np.zeros((n, 15), np.float32)
    q[:, 0] = rng.choice([0.0, 0.01, 0.3, 1.0, 7.0], n) * rng.random(n)
    q[:, 1] = rng.choice([0.0, 0.05, 0.5, 3.0], n) * rng.random(n)
    q[:, 2] = rng.choice([0.0, 1.0, 4.0], n) * rng.random(n)
    q[:, 3] = rng.choice([0.0, 1e-4, 0.1, 1.0, 20.0, np.inf], n) * rng.random(n)
    q[:, 4] = rng.choice([0.0, 0.2, 1.0, 5.0], n) * rng.random(n)
    q[:, 5] = np.where(rng.random(n) < 0.3, rng.random(n) * 0.125, rng.random(n))
    wo = rng.normal(size=(n, 3))
    wi = rng.normal(size=(n, 3))
    q[:, 6:9] = wo / np.linalg.norm(wo, axis=1, keepdims=True)
    q[:, 9:12] = wi / np.linalg.norm(wi, axis=1, keepdims=True)
    q[:, 12] = rng.choice([-0.995, -0.55, 0.0, 1e-5, 0.3, 0.65, 0.99, 1.2], n)
    q[:, 13] = rng.random(n)
    q[:, 14] = rng.random(n)
    return np.ascontiguousarray(q)


def test_medium_equations_match_the_reference_header_bitwise():
    ref = reference()
    if ref is None:
        pytest.skip("oracle/_ref/libref.so not built (needs a rypath checkout)")
    q = medium_queries(np.random.default_rng(7), 20000)
    a = np.zeros((q.shape[0], 8), np.float32)
    b = np.zeros_like(a)
    oracle().or_probe_medium(q.ctypes.data, q.shape[0], a.ctypes.data)
    ref.ref_probe_medium(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_medium_equations_against_closed_forms():
    """tests/medium_reference.hpp: HG density and emission integral in high precision."""
    q = medium_queries(np.random.default_rng(3), 4000)
    out = np.zeros((q.shape[0], 8), np.float32)
    oracle().or_probe_medium(q.ctypes.data, q.shape[0], out.ctypes.data)
    a, s, le, d = (q[:, i].astype(np.float64) for i in range(4))
    ok = out[:, 2] == 1
    assert ok.all()  # every query above is valid
    with np.errstate(invalid="ignore"):
        expect_t = np.where((a + s == 0) | (d == 0), 1.0, np.exp(-(a + s) * d))
        expect_e = np.where((a == 0) | (le == 0) | (d == 0), 0.0, le * a / (a + s) * -np.expm1(-(a + s) * d))
    # binary32 rounding of the optical depth sigma_t * d scales with the depth itself
    depth = np.where(np.isfinite(d), (a + s) * np.where(np.isfinite(d), d, 0), 0)
    tol = 2e-6 + 1.2e-7 * depth
    assert np.all(np.abs(out[:, 0] - expect_t) <= tol * np.abs(expect_t) + 1e-30)
    assert np.all(np.abs(out[:, 1] - expect_e) <= (tol + 2e-6) * np.abs(expect_e) + 1e-30)
    g = np.clip(q[:, 12].astype(np.float64), -0.99, 0.99)
    # the cosine as binary32 forms it: the narrow HG peak amplifies any error in it
    wo, wi = q[:, 6:9], q[:, 9:12]
    cos32 = (wo[:, 0] * wi[:, 0] + wo[:, 1] * wi[:, 1]) + wo[:, 2] * wi[:, 2]
    cos = np.clip(cos32.astype(np.float64), -1, 1)
    denom = 1 + g * g + 2 * g * cos
    hg = (1 - g * g) / (4 * math.pi * denom * np.sqrt(denom))
    np.testing.assert_allclose(out[:, 4], hg, rtol=2e-5)
    # sampled directions are unit vectors; flight inverts the exponential CDF
    np.testing.assert_allclose(np.linalg.norm(out[:, 5:8], axis=1), 1.0, rtol=1e-6)
    st, u = q[:, 4].astype(np.float64), q[:, 5].astype(np.float64)
    finite = st > 0
    np.testing.assert_allclose(out[finite, 3], -np.log1p(-u[finite]) / st[finite], rtol=4e-6)
    assert np.all(np.isinf(out[~finite, 3]))


def test_beer_plus_analytic_slab_emission():
    scene = scenes.slab_scene([medium(.6, 0, 2)], [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))])
    mean_gate(paths(scene), 2 - math.exp(-.6))


def test_depth_zero_beer_transmission():
    scene = scenes.slab_scene([medium(.6, 0, 2)], [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))],
                              max_depth=0)
    mean_gate(paths(scene), math.exp(-.6))


def test_wavelength_dependent_beer_transmission():
    sigma = (.1 + .8 * np.arange(471) / 470).astype(np.float32)
    scene = scenes.slab_scene([medium(sigma, 0)], [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))])
    out = paths(scene)
    idx = np.clip(np.floor(out["wavelength"].astype(np.float64) + 0.5).astype(int) - 360, 0, 470)
    mean_gate(out, np.exp(-sigma[idx].astype(np.float64)))


@pytest.mark.parametrize("empty", [False, True])
def test_infinite_emitting_medium_at_finite_depth(empty):
    planes = [] if empty else [plane(-100000, True)]
    for depth in (0, 1, 2, 3):
        scene = scenes.slab_scene([medium(.4, .6, 2, .65)], planes, camera_medium=0, environment=0.0,
                                  max_depth=depth)
        mean_gate(paths(scene, 4096), 2 * (1 - .6 ** depth))
    scene = scenes.slab_scene([medium(0, .7, 4)], planes, camera_medium=0, environment=0.0, max_depth=2)
    assert np.all(paths(scene, 256)["radiance"] == 0)  # Le alone does not emit without absorption
    scene = scenes.slab_scene([medium(.7, 0)], planes, camera_medium=0, environment=3.0, max_depth=2)
    assert np.all(paths(scene, 256)["radiance"] == 0)  # positive extinction never escapes
    scene = scenes.slab_scene([medium(0, 0, 4)], planes, camera_medium=0, environment=3.0, max_depth=2)
    assert np.all(paths(scene, 256)["radiance"] == 3)  # zero extinction is transparent


def test_nested_and_reversed_medium_sides():
    media = [medium(.2, 0), medium(.8, 0)]
    planes = [plane(1, False, (0, NONE)), plane(1.5, False, (1, 0)), plane(2.5, True, (1, 0)),
              plane(3, True, (0, NONE))]
    mean_gate(paths(scenes.slab_scene(media, planes)), math.exp(-1.))
    # reversing orientation and swapping the authored sides keeps the physical regions
    swapped = [dict(p, reverse=True, media=(p["media"][1], p["media"][0])) for p in planes]
    mean_gate(paths(scenes.slab_scene(media, swapped)), math.exp(-1.))
    # a mirrored placement flips the winding; with the swapped sides the slab is the same
    mirror = (-1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)
    mirrored = [dict(p, media=(p["media"][1], p["media"][0]), matrix=mirror) for p in planes]
    mean_gate(paths(scenes.slab_scene(media, mirrored)), math.exp(-1.))


def test_split_null_interfaces_use_fresh_flight_draws():
    planes = [plane(1, False, (0, NONE)), plane(2, True, (0, NONE))]
    planes += [plane(1 + i / 8, True) for i in range(1, 8)]
    scene = scenes.slab_scene([medium(1, 0)], planes, max_depth=0)
    mean_gate(paths(scene), math.exp(-1.))


def single_scatter_slab(g):
    """tests/medium_render_tests.cpp:329-349: deterministic quadrature of one scattering in
    the slab z in [-1, 1] seen from its centre along +z."""
    n = 800
    t = (np.arange(n) + .5) / n
    mu = -1 + 2 * (np.arange(n) + .5) / n
    T, M = np.meshgrid(t, mu, indexing="ij")
    distance = np.where(M > 0, (1 - T) / M, (-1 - T) / M)
    denom = 1 + g * g - 2 * g * M
    phase_2pi = .5 * (1 - g * g) / denom ** 1.5
    angular = np.sum(phase_2pi * np.exp(-distance) * 2 / n, axis=1)
    return math.exp(-1.) + float(np.sum(.7 * np.exp(-t) * angular / n))


@pytest.mark.parametrize("g", [0.0, .65, -.55])
def test_phase_light_mis_against_single_scatter_quadrature(g):
    scene = scenes.slab_scene([medium(.3, .7, 0, g)], [plane(-1, False, (0, NONE)), plane(1, True, (0, NONE))],
                              camera_medium=0)
    mean_gate(paths(scene), single_scatter_slab(g), numerical=4e-5)


def test_finite_point_light_through_two_beer_segments():
    """tests/medium_render_tests.cpp:176-208: camera and shadow legs each cross .25 of absorber."""
    diffuse = abi.Material()
    diffuse.scattering, diffuse.kind, diffuse.scalar_value = abi.DIFFUSE, abi.REFLECTANCE_CONSTANT, .5
    light = dict(position=(0.0, 0.0, 0.0), intensity=np.full(471, 2.0, np.float32), kind=abi.POINT_LIGHT)
    planes = [plane(1, False, material=1), plane(.25, False, (0, NONE)), plane(.5, True, (0, NONE)),
              plane(-5e-6, True, material=1)]  # opaque, just behind the light and the camera
    scene = scenes.slab_scene([medium(.4, 0)], planes, environment=0.0, materials=[diffuse], positional=[light])
    mean_gate(paths(scene), math.exp(-.4 * .5) / math.pi)


@pytest.mark.parametrize("reverse", [False, True])
@pytest.mark.parametrize("transformed", [False, True])
def test_grazing_shared_edge_beer_chord(reverse, transformed):
    """tests/medium_render_tests.cpp:150-181: a grazing view along the quads' shared diagonal."""
    zs, shift = (2.0, .25) if transformed else (1.0, 0.0)
    m = (2.0 if transformed else 1.0, 0, 0, 0, 0, 2.0 if transformed else 1.0, 0, 0, 0, 0, zs, shift)
    planes = [plane(.001, False, (0, NONE), matrix=m), plane(.002, True, (0, NONE), matrix=m)]
    scene = scenes.slab_scene([medium(.6, 0)], planes, max_depth=0)
    low = np.float32(shift) + np.float32(zs) * np.float32(.001)
    high = np.float32(shift) + np.float32(zs) * np.float32(.002)
    origin_z = float(high + np.float32(zs) * np.float32(.001)) if reverse else shift
    scene.camera = ((0.0, 0.0, origin_z), (1.0, 1.0, -.001 if reverse else .001), (1e-10, 0.0, 0.0), (0.0, 1e-10, 0.0))
    chord = float(high - low) * math.sqrt(2. + .001 * .001) / .001
    mean_gate(paths(scene, 16384), math.exp(-.6 * chord))


def test_scalar_and_hero_transports_agree_on_the_vacuum_cornell_box():
    hero = scenes.cornell_box(16, 16, 1)
    scalar = scenes.cornell_box(16, 16, 1)
    scalar.transport = abi.TRANSPORT_SCALAR
    q = request(16, 16, 64, sampler=abi.SAMPLER_INDEPENDENT)
    s = OracleScene(scalar).sample_scalar(q)
    h = OracleScene(hero).sample(q)
    assert np.all(s["status"] == 0) and np.all(h["status"] == 0)
    sv = s["radiance"].astype(np.float64) * 470.0  # scalar: uniform wavelength pdf 1/470
    hv = np.sum(h["radiance"] / h["wavelength_pdfs"], axis=1) / 4.0
    diff = sv.mean() - hv.mean()
    se = math.sqrt(sv.var() / sv.size + hv.var() / hv.size)
    assert abs(diff) < 4 * se, (sv.mean(), hv.mean(), se)


def test_scalar_film_reduction_matches_host_accumulation():
    scene = scenes.cornell_fog(8, 8, 1)
    out = OracleScene(scene).sample_scalar(request(8, 8, 4))
    film = np.zeros(64, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_scalar_film_add(out.ctypes.data, out.size, cie.ctypes.data, 64, film.ctypes.data, 0) == 0
    assert np.all(film["count"] == 4)
    expected = np.zeros((64, 3))
    for r in out:
        row = int(round(float(r["wavelength"]))) - 360
        expected[r["pixel"]] += cie[row] * (470.0 * float(r["radiance"]))
    np.testing.assert_allclose(film["sum"] + film["correction"], expected, rtol=1e-12, atol=1e-300)


def test_oracle_rejects_scalar_requests_on_hero_scenes():
    q = request(4, 4, 1)
    o = OracleScene(scenes.cornell_box(4, 4, 1))
    with pytest.raises(RuntimeError):
        o.sample_scalar(q)
