"""The demo model (`rypath --render-demo`): the oracle against rypath's own demo code.

rypath's src/render.cpp (make_demo_scene, FilmBatch, wavelength_xyz) and its CPU demo reference
tests/render_reference.cpp (analytic sky and floor moments, its own path estimator) are compiled
from the checkout into oracle/_ref/libref_demo.so by oracle/ref.mk.  The checks: the demo
fixture of rypath_b200.scenes equals make_demo_scene; the oracle's demo film reduction equals
FilmBatch bit for bit; the oracle's sky and floor estimates meet the analytic moments within
rypath's own six-standard-error gate; the oracle's image of the demo scene agrees with
rypath's CPU estimator within five combined standard errors over replicates.  CPU only.
"""

import ctypes as C
import os

import numpy as np
import pytest

from rypath_b200 import abi, scenes
from tests.oracle_lib import OracleScene, oracle, oracle_film, request

REF_DEMO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libref_demo.so")


def need_ref():
    if not os.path.exists(REF_DEMO):
        pytest.skip("oracle/_ref/libref_demo.so not built (needs a rypath checkout: oracle/ref.mk)")
    lib = C.CDLL(REF_DEMO)
    vp = C.c_void_p
    lib.ref_demo_scene.argtypes = [vp] * 10 + [C.c_uint32]
    lib.ref_demo_film.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp]
    lib.ref_demo_analytic.argtypes = [vp, vp]
    lib.ref_demo_reference_image.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, vp]
    return lib


def test_demo_scene_matches_rypath():
    """Geometry, placements, reflectances, camera and depth of make_demo_scene."""
    lib = need_ref()
    counts, mb = np.zeros(4, np.uint32), np.zeros(64, np.uint32)
    pos, tri = np.zeros(3000, np.float32), np.zeros(3000, np.uint32)
    im, it, imat = np.zeros(64, np.uint32), np.zeros(64 * 12, np.float32), np.zeros(64, np.uint32)
    refl, cam, depth = np.zeros(64 * 8, np.float32), np.zeros(10, np.float32), np.zeros(1, np.uint32)
    assert lib.ref_demo_scene(*(a.ctypes.data for a in (counts, mb, pos, tri, im, it, imat, refl, cam, depth)),
                              1000) == 0
    s = scenes.demo_scene()
    assert len(s.instances) == counts[3] and len(s.materials) == 6 and s.max_depth == depth[0]
    for i, inst in enumerate(s.instances):
        mesh = im[i]
        v0, t0 = mb[2 * mesh], mb[2 * mesh + 1]
        nt = inst.triangle_count
        np.testing.assert_array_equal(s.triangles[inst.triangle_begin:inst.triangle_begin + nt],
                                      tri[3 * t0:3 * (t0 + nt)].reshape(-1, 3))
        nv = int(s.triangles[inst.triangle_begin:inst.triangle_begin + nt].max()) + 1
        np.testing.assert_array_equal(s.positions[inst.vertex_begin:inst.vertex_begin + nv],
                                      pos[3 * v0:3 * (v0 + nv)].reshape(-1, 3))
        np.testing.assert_array_equal(np.array(inst.matrix[:], np.float32), it[12 * i:12 * i + 12])
        assert inst.material == imat[i]
        np.testing.assert_array_equal(np.array(s.materials[inst.material].reflectance[:], np.float32),
                                      refl[8 * imat[i]:8 * imat[i] + 8])
    (o, f, r, u), scale = scenes.demo_camera(tuple(cam[0:3]), tuple(cam[3:6]), tuple(cam[6:9]), float(cam[9]))
    assert s.camera == (o, f, r, u) and s.film_scale == scale


def test_demo_film_matches_rypath():
    """The oracle's demo film reduction (wavelength_xyz, unweighted radiance) equals
    FilmBatch's bit for bit, edges of the wavelength range included."""
    lib = need_ref()
    rng = np.random.default_rng(70)
    w, h, spp = 8, 4, 6
    n = w * h * spp
    rows = np.zeros((n, 4), np.float32)
    pixel = np.tile(np.arange(w * h, dtype=np.uint32), spp)
    sample = np.repeat(np.arange(spp, dtype=np.uint32), w * h)
    rows[:, 0] = pixel.view(np.float32)
    rows[:, 1] = sample.view(np.float32)
    rows[:, 2] = rng.uniform(360, 830, n).astype(np.float32)
    rows[:5, 2] = [360.0, 830.0, 829.99994, 360.00003, 555.0]
    rows[:, 3] = np.exp(rng.uniform(-5, 2, n)).astype(np.float32)
    ref = np.zeros((w * h, 7))
    assert lib.ref_demo_film(rows.ctypes.data, n, w, h, spp, ref.ctypes.data) == 0
    res = np.zeros(n, abi.scalar_dtype())
    res["pixel"], res["status"] = pixel, 0
    res["sample_low"] = sample
    res["wavelength"], res["radiance"] = rows[:, 2], rows[:, 3]
    film = np.zeros(w * h, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_scalar_film_add(res.ctypes.data, n, cie.ctypes.data, w * h, film.ctypes.data, 1) == 0
    np.testing.assert_array_equal(film["sum"], ref[:, 0:3])
    np.testing.assert_array_equal(film["correction"], ref[:, 3:6])
    np.testing.assert_array_equal(film["count"], ref[:, 6])


def analytic(lib, reflectance):
    out = np.zeros(6)
    r = None if reflectance is None else np.asarray(reflectance, np.float32)
    lib.ref_demo_analytic(None if r is None else r.ctypes.data, out.ctypes.data)
    return out[:3], out[3:]


FLOOR = (0.54, 0.54, 0.55, 0.58, 0.61, 0.63, 0.65, 0.65)


@pytest.mark.parametrize("reflectance", [None, FLOOR, (0.5,) * 8])
def test_demo_oracle_meets_analytic_moments(reflectance):
    """The unit sky and the unobstructed Lambertian floor (rypath's native_analytic fixtures,
    tests/render_tests.cpp:525-549): 32768 paths of one pixel within 6 standard errors."""
    lib = need_ref()
    mean, var = analytic(lib, reflectance)
    paths = 32768
    scene = scenes.demo_floor(reflectance)
    film = oracle_film(scene, 1, 1, paths, seed=0x9E314FD9, sampler=abi.SAMPLER_INDEPENDENT, scalar=True,
                       chunk=paths)
    xyz = (film["sum"] + film["correction"])[0] / film["count"][0]
    se = np.sqrt(var / paths)
    assert np.all(np.abs(xyz - mean) <= 6 * se + 2e-5 * np.maximum(1, np.abs(mean))), (xyz, mean, se)


def test_demo_oracle_matches_rypath_estimator():
    """The demo scene's image mean from the oracle against rypath's CPU estimator
    (tests/render_reference.cpp reference_image), 8 replicates each of 8x6 pixels at 64 spp:
    within 5 combined standard errors, both reaching the fourth bounce."""
    lib = need_ref()
    w, h, spp = 8, 6, 64
    ref, orc = [], []
    for k in range(8):
        out = np.zeros(4)
        lib.ref_demo_reference_image(w, h, spp, 0x56DA2309 + k, out.ctypes.data)
        ref.append(out[:3])
        assert out[3] >= 4
        scene = scenes.demo_scene(w, h, spp)
        film = oracle_film(scene, w, h, spp, seed=0x71AC6A05 + k, sampler=abi.SAMPLER_INDEPENDENT, scalar=True)
        orc.append(((film["sum"] + film["correction"]) / film["count"][:, None]).mean(axis=0))
    ref, orc = np.array(ref), np.array(orc)
    se = np.sqrt(ref.var(axis=0, ddof=1) / len(ref) + orc.var(axis=0, ddof=1) / len(orc))
    assert np.all(np.abs(ref.mean(0) - orc.mean(0)) <= 5 * se + 2e-5), (ref.mean(0), orc.mean(0), se)


def test_golden_demo_answers_are_rypaths():
    """tests/golden/demo_reference.json (read by the GPU tests) holds what rypath's code gives."""
    import json

    lib = need_ref()
    golden = json.loads(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                          "demo_reference.json")).read())
    for case in golden["analytic"].values():
        mean, var = analytic(lib, case["reflectance"])
        assert mean.tolist() == case["mean"] and var.tolist() == case["variance"]
    est = golden["estimator"]
    out = np.zeros(4)
    lib.ref_demo_reference_image(est["width"], est["height"], est["samples"], est["seed"], out.ctypes.data)
    assert out[:3].tolist() == est["means"][0]
