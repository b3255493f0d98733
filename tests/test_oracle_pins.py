"""Pin the oracle: rypath's own known-answer vectors, and bit-for-bit agreement with rypath's
host-compilable sources compiled where they lie (oracle/_ref, built by oracle/ref.mk).

References: Sobol KATs tests/sampling_tests.cpp:26-142; Philox KATs tests/replay_tests.cpp:22-36;
visible wavelength checks tests/packet_spectrum_tests.cpp:9-56; light tables
src/light_sampling.cpp:384-572; packet film src/packet_film.cpp:198-265; Gaussian filter
digests tests/gaussian_filter_tests.cpp:89-127; roulette known answers
tests/packet_roulette_tests.cpp:18-139; hero BSDF proposals shaders/hero_scattering.h:67-231;
hero roulette and MIS weight shaders/hero_pt_helpers.h:56-138.
"""

import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from rypath_b200 import abi, scenes
from tests.oracle_lib import ROULETTE_KNOWN_ANSWERS, oracle, reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TABLES = scenes.sobol_tables()
TABLE_BUF = C.create_string_buffer(TABLES, len(TABLES))


def need_ref():
    lib = reference()
    if lib is None:
        pytest.skip("oracle/_ref/libref.so not built (needs a rypath checkout)")
    return lib


def sobol_query(answer, mode=3):
    seed = answer["seed"] & 0xFFFFFFFF
    s = answer["sample"]
    return [answer["m"], answer["x"], answer["y"], s & 0xFFFFFFFF, s >> 32, answer["dimension"], mode, seed]


def test_table_identity_with_reference():
    lib = need_ref()
    ref = C.string_at(lib.ref_sobol_tables(), abi.RP_SOBOL_TABLE_BYTES)
    assert ref == TABLES


def test_sobol_known_answers():
    answers = json.load(open(os.path.join(GOLDEN, "sobol_known_answers.json")))
    assert len(answers) == 8
    for a in answers:
        for mode in range(4):
            q = np.array(sobol_query(a, mode), np.uint32)
            out = np.zeros(6, np.uint32)
            oracle().or_probe_sobol(TABLE_BUF, q.ctypes.data, 1, out.ctypes.data)
            index = int(out[0]) | (int(out[1]) << 32)
            assert index == a["index"]
            assert out[3] == a["hash"]
            assert out[2] == a["words"][mode], (a, mode)
        # binary32 pixel remap of the unscrambled camera dimensions (sobol::camera_uniform)
        for dim, pix in ((0, a["x"]), (1, a["y"])):
            q = np.array(sobol_query(dict(a, dimension=dim), 0), np.uint32)
            out = np.zeros(6, np.uint32)
            oracle().or_probe_sobol(TABLE_BUF, q.ctypes.data, 1, out.ctypes.data)
            assert float(camera_uniform(int(out[2]), a["m"], pix)) == float.fromhex(a["camera"][dim])


ONE_MINUS = np.float32(float.fromhex("0x1.fffffep-1"))


def sobol_uniform(word):
    return min(np.float32(np.float32(word) * np.float32(2.0 ** -32)), ONE_MINUS)


def camera_uniform(word, m, pixel):
    local = np.float32(np.float32(sobol_uniform(word) * np.float32(1 << m)) - np.float32(pixel))
    return np.float32(0) if local < 0 else min(local, ONE_MINUS)


def test_sobol_uniform_special_values():
    # tests/sampling_tests.cpp:136-141
    assert sobol_uniform(0xFFFFFFFF) == ONE_MINUS
    assert sobol_uniform(0) == 0
    assert float(sobol_uniform(0x80000081)) == float.fromhex("0x1.000002p-1")
    assert camera_uniform(0x7FFFFFFF, 1, 0) == ONE_MINUS


def test_philox_known_answers():
    kats = json.load(open(os.path.join(GOLDEN, "philox_known_answers.json")))
    assert len(kats) == 3
    q = np.array([k["counter"] + k["key"] for k in kats], np.uint32)
    out = np.zeros((len(kats), 4), np.uint32)
    oracle().or_probe_philox(q.ctypes.data, len(kats), out.ctypes.data)
    for k, row in zip(kats, out):
        assert list(map(int, row)) == k["expected"]


def test_sobol_matches_reference_random():
    lib = need_ref()
    rng = np.random.default_rng(7)
    n = 4000
    m = rng.integers(0, 26, n)
    x = (rng.integers(0, 2**31, n) % np.maximum(1, 1 << m)).astype(np.uint64)
    y = (rng.integers(0, 2**31, n) % np.maximum(1, 1 << m)).astype(np.uint64)
    sample = rng.integers(0, 2**40, n).astype(np.uint64) >> (2 * m).astype(np.uint64)
    q = np.stack([m, x, y, sample & 0xFFFFFFFF, sample >> 32, rng.integers(0, 1024, n),
                  rng.integers(0, 4, n), rng.integers(0, 2**32, n)], 1).astype(np.uint32)
    a = np.zeros((n, 6), np.uint32)
    b = np.zeros((n, 6), np.uint32)
    oracle().or_probe_sobol(TABLE_BUF, q.ctypes.data, n, a.ctypes.data)
    lib.ref_probe_sobol(q.ctypes.data, n, b.ctypes.data)
    np.testing.assert_array_equal(a, b)


def test_philox_matches_reference_random():
    lib = need_ref()
    q = np.random.default_rng(3).integers(0, 2**32, (5000, 6)).astype(np.uint32)
    a = np.zeros((5000, 4), np.uint32)
    b = np.zeros((5000, 4), np.uint32)
    oracle().or_probe_philox(q.ctypes.data, 5000, a.ctypes.data)
    lib.ref_probe_philox(q.ctypes.data, 5000, b.ctypes.data)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("mode", [abi.HERO_UNIFORM, abi.HERO_VISIBLE])
def test_hero_wavelengths_match_reference(mode):
    lib = need_ref()
    u = np.concatenate([(np.arange(4096) + 0.5) / 4096, np.arange(4096) / 4096,
                        [np.nextafter(np.float32(1), np.float32(0))]]).astype(np.float32)
    a = np.zeros((u.size, 8), np.float32)
    b = np.zeros((u.size, 8), np.float32)
    oracle().or_probe_wavelengths(u.ctypes.data, u.size, mode, a.ctypes.data)
    lib.ref_probe_wavelengths(u.ctypes.data, u.size, mode, b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_visible_wavelengths_properties():
    # tests/packet_spectrum_tests.cpp restated for the hero lattice shift
    u = np.concatenate([(np.arange(4096) + 0.5) / 4096, np.arange(4096) / 4096]).astype(np.float32)
    out = np.zeros((u.size, 8), np.float32)
    oracle().or_probe_wavelengths(u.ctypes.data, u.size, abi.HERO_VISIBLE, out.ctypes.data)
    lam, pdf = out[:, :4].astype(np.float64), out[:, 4:].astype(np.float64)
    coord = np.floor(u.astype(np.float64) * 16777216.0).astype(np.int64)
    for k in range(4):
        shifted = ((coord + k * 4194304) & 0xFFFFFF) * 2.0 ** -24
        expect = np.clip(538 - 138.888889 * np.arctanh(.85691062 - 1.82750197 * shifted), 360, 830)
        assert np.all(np.abs(lam[:, k] - expect) <= 1e-3)
        c = np.cosh(.0072 * (lam[:, k] - 538))
        assert np.all(np.abs(pdf[:, k] - .0039398042 / (c * c)) <= 1e-8)
    bad = np.array([-1, -1e-45, 1, 2, np.inf, np.nan], np.float32)
    out = np.zeros((bad.size, 8), np.float32)
    oracle().or_probe_wavelengths(bad.ctypes.data, bad.size, abi.HERO_VISIBLE, out.ctypes.data)
    assert np.all(~np.isfinite(out))


def _advance_queries(n, rng):
    q = np.zeros((n, 20), np.float32)
    q[:, 0:4] = rng.uniform(0.5, 1.0, (n, 4))
    q[:, 4:8] = rng.integers(-160, 60, (n, 4))
    zero = rng.uniform(size=(n, 4)) < 0.1
    q[:, 0:4][zero] = 0
    q[:, 4:8][zero] = 0
    q[:, 8:12] = np.exp(rng.uniform(-80, 40, (n, 4)))
    q[:, 12:16] = np.exp(rng.uniform(-60, 20, (n, 4))) * (rng.uniform(size=(n, 4)) > 0.1)
    q[:, 16:20] = np.exp(rng.uniform(-60, 20, (n, 4))) * (rng.uniform(size=(n, 4)) > 0.1)
    return q


def test_hero_advance_matches_reference():
    lib = need_ref()
    q = _advance_queries(20000, np.random.default_rng(11))
    a = np.zeros((q.shape[0], 13), np.float32)
    b = np.zeros((q.shape[0], 13), np.float32)
    oracle().or_probe_advance(q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_probe_advance(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert a[:, 12].mean() > 0.3  # the generator exercises valid updates


def bsdf_queries(n, rng):
    q = np.zeros((n, 16), np.float32)
    kind = rng.integers(1, 3, n)
    q[:, 0] = kind
    q[:, 1] = np.where(kind == 1, rng.uniform(0.1, 3, n), rng.uniform(1.0, 2.4, n))
    q[:, 2] = rng.uniform(0, 5, n)
    rough = rng.uniform(0, 0.6, n) * (rng.uniform(size=n) > 0.15)
    q[:, 3] = rough
    q[:, 4] = rough * rng.uniform(0.5, 1.5, n)
    q[:, 5] = rng.integers(0, 2, n)
    for s in (6, 9):
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        q[:, s:s + 3] = v
    q[:, 12:15] = rng.uniform(0, 1, (n, 3))
    return q


def test_bsdf_match_reference():
    lib = need_ref()
    q = bsdf_queries(20000, np.random.default_rng(5))
    a = np.zeros((q.shape[0], 12), np.float32)
    b = np.zeros((q.shape[0], 12), np.float32)
    oracle().or_probe_bsdf(q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_probe_bsdf(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a[:, :10].view(np.uint32), b[:, :10].view(np.uint32))


def light_rows(n, rng):
    rows = np.zeros((n, 16))
    rows[:, 0] = rng.uniform(0, 10, n) * (rng.uniform(size=n) > 0.05)
    rows[:, 1] = np.where(rng.uniform(size=n) < 0.5, -1, rng.uniform(0, 20, n))
    lo = rng.uniform(-5, 5, (n, 3))
    rows[:, 2:5] = lo
    rows[:, 5:8] = lo + rng.uniform(0, 1, (n, 3)) * (rng.uniform(size=(n, 1)) > 0.3)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rows[:, 8:11] = d
    rows[:, 11] = np.where(rng.uniform(size=n) < 0.5, np.nextafter(np.float32(1), np.float32(0)),
                           rng.uniform(-1, 1, n))
    rows[:, 12] = rng.uniform(-1, 1, n) * (rng.uniform(size=n) < 0.3)
    rows[:, 13] = rng.integers(0, 2, n)
    rows[:, 14] = rng.uniform(size=n) < 0.05
    # float32-representable values as the C structs hold them
    rows[:, 2:13] = rows[:, 2:13].astype(np.float32)
    return rows


@pytest.mark.parametrize("n", [1, 2, 7, 64, 300])
def test_light_tables_match_reference(n):
    lib = need_ref()
    rows = light_rows(n, np.random.default_rng(n))
    outs = []
    for fn in (oracle().or_build_light_tables, lib.ref_build_light_tables):
        alias = np.zeros((n, 4), np.uint32)
        rec = np.zeros((n, 4), np.uint32)
        nodes = np.zeros((2 * n, 16), np.uint32)
        inf = np.zeros(n, np.uint32)
        cnt = C.c_uint32(0)
        k = fn(rows.ctypes.data, n, alias.ctypes.data, rec.ctypes.data, nodes.ctypes.data, inf.ctypes.data,
               C.byref(cnt))
        outs.append((k, alias, rec, nodes[:max(k, 0)], inf[:cnt.value]))
    (ka, *a), (kb, *b) = outs
    assert ka == kb
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_film_reduction_matches_packet_film_batch():
    lib = need_ref()
    cie = scenes.cie_xyz()
    lib.ref_set_cie(np.ascontiguousarray(cie).ctypes.data)
    rng = np.random.default_rng(2)
    w, h, spp = 8, 5, 6
    res = np.zeros(w * h * spp, abi.packet_dtype())
    lane = np.arange(res.size)
    res["pixel"] = lane % (w * h)
    res["sample_low"] = lane // (w * h)
    res["wavelengths"] = rng.uniform(360, 830, (res.size, 4))
    res["wavelength_pdfs"] = rng.uniform(0.001, 0.004, (res.size, 4))
    res["radiance"] = rng.exponential(1.0, (res.size, 4)) * (rng.uniform(size=(res.size, 4)) > 0.3)
    res["filter_weight"] = 1.0
    ref_out = np.zeros((w * h, 9))
    assert lib.ref_film_add(res.ctypes.data, res.size, w, h, ref_out.ctypes.data) == 0
    film = np.zeros(w * h, abi.film_dtype())
    assert oracle().or_film_add(res.ctypes.data, res.size, np.ascontiguousarray(cie).ctypes.data, w * h,
                                film.ctypes.data) == 0
    np.testing.assert_array_equal(film["sum"], ref_out[:, 0:3])
    np.testing.assert_array_equal(film["correction"], ref_out[:, 3:6])
    np.testing.assert_array_equal(film["weight_sum"], ref_out[:, 6])
    np.testing.assert_array_equal(film["count"], ref_out[:, 8])


@pytest.mark.parametrize("exposure, clamp", [(1.0, 0.35), (2.5, 1.2), (0.7, 0.05)])
def test_clamped_film_matches_packet_film_batch(exposure, clamp):
    """The compatibility planes of a finite film clamp (clamp_sensor, src/packet_film.cpp:39-47)
    bit for bit against rypath's own PacketFilmBatch with the same exposure and clamp."""
    lib = need_ref()
    cie = scenes.cie_xyz()
    lib.ref_set_cie(np.ascontiguousarray(cie).ctypes.data)
    rng = np.random.default_rng(3)
    w, h, spp = 7, 6, 5
    res = np.zeros(w * h * spp, abi.packet_dtype())
    lane = np.arange(res.size)
    res["pixel"] = lane % (w * h)
    res["sample_low"] = lane // (w * h)
    res["wavelengths"] = rng.uniform(360, 830, (res.size, 4))
    res["wavelength_pdfs"] = rng.uniform(0.001, 0.004, (res.size, 4))
    res["radiance"] = rng.exponential(1.0, (res.size, 4)) * (rng.uniform(size=(res.size, 4)) > 0.3)
    res["filter_weight"] = rng.uniform(0.5, 1.0, res.size).astype(np.float32)
    ref_out = np.zeros((w * h, 15))
    assert lib.ref_film_add_clamped(res.ctypes.data, res.size, w, h, exposure, clamp, ref_out.ctypes.data) == 0
    film = np.zeros(w * h, abi.film_dtype())
    assert oracle().or_film_add_clamped(res.ctypes.data, res.size, np.ascontiguousarray(cie).ctypes.data, w * h,
                                        exposure, clamp, film.ctypes.data) == 0
    np.testing.assert_array_equal(film["sum"], ref_out[:, 0:3])
    np.testing.assert_array_equal(film["weight_sum"], ref_out[:, 6])
    np.testing.assert_array_equal(film["compatibility_sum"], ref_out[:, 9:12])
    np.testing.assert_array_equal(film["compatibility_correction"], ref_out[:, 12:15])
    assert (film["compatibility_sum"] < film["sum"] * exposure - 1e-12).any()  # the clamp bites


def _fnv_floats(values, h=14695981039346656037):
    for b in np.asarray(values, np.float32).tobytes():
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_gaussian_filter_table_and_samples_match_rypath_known_answers():
    """tests/gaussian_filter_tests.cpp:89-127: FNV-1a digests of every CDF entry and of 33x33
    samples (u, v = k / 32 clamped below 1) for three configurations, pinned by rypath against
    PBRT v4 b0bdf461."""
    import ctypes as C

    known = json.load(open(os.path.join(GOLDEN, "gaussian_filter_known_answers.json")))
    grid = np.array([[min(x / 32, float.fromhex("0x1.fffffep-1")), min(y / 32, float.fromhex("0x1.fffffep-1"))]
                     for y in range(33) for x in range(33)], np.float32)
    for k in known:
        cdf = np.zeros(1 << 20, np.float32)
        size = np.zeros(2, np.uint32)
        integral = C.c_float()
        out = np.zeros((grid.shape[0], 2), np.float32)
        n = oracle().or_gaussian_filter(k["x_radius"], k["y_radius"], k["sigma"], cdf.ctypes.data, cdf.size,
                                        size.ctypes.data, C.byref(integral), grid.ctypes.data, grid.shape[0],
                                        out.ctypes.data)
        assert n > 0
        assert _fnv_floats(cdf[:n]) == k["cdf_hash"]
        assert _fnv_floats(out.reshape(-1)) == k["sample_hash"]
        assert integral.value > 0


def _qmc_queries(rng, n):
    q = []
    for _ in range(n):
        kind = int(rng.choice([2, 3]))
        w, h = int(rng.integers(1, 400)), int(rng.integers(1, 300))
        spp = int(2 ** rng.integers(0, 11))
        sample = int(rng.integers(0, spp if kind == 3 else 1 << 20))
        mode = int(rng.choice([0, 1, 3] if kind == 2 else [0, 1, 2, 3]))
        d = int(rng.integers(2, 997)) if kind == 2 else int(rng.integers(0, 1023))
        seed = int(rng.integers(-(2 ** 31), 2 ** 31))
        q.append([kind, w, h, int(rng.integers(0, w)), int(rng.integers(0, h)), sample, d, mode, seed, spp])
    return np.ascontiguousarray(q, np.int64)


def test_qmc_halton_and_zsobol_match_rypath_known_answers():
    """tests/qmc_sampling_tests.cpp:21-77: 28 PBRT v4 known answers (12 Halton, 16 ZSobol)."""
    known = json.load(open(os.path.join(GOLDEN, "qmc_known_answers.json")))
    q = np.ascontiguousarray([k["q"] for k in known], np.int64)
    out = np.zeros((len(known), 6), np.uint64)
    oracle().or_probe_qmc(C.cast(TABLE_BUF, C.c_void_p), q.ctypes.data, len(known), out.ctypes.data)
    np.testing.assert_array_equal(out, np.array([k["a"] for k in known], np.uint64))


def test_qmc_matches_reference_header():
    ref = need_ref()
    q = _qmc_queries(np.random.default_rng(11), 3000)
    a = np.zeros((q.shape[0], 6), np.uint64)
    b = np.zeros_like(a)
    oracle().or_probe_qmc(C.cast(TABLE_BUF, C.c_void_p), q.ctypes.data, q.shape[0], a.ctypes.data)
    ref.ref_probe_qmc(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a, b)


def test_roulette_known_answers_of_rypath_against_the_oracle():
    """rypath's own roulette test program (tests/packet_roulette_tests.cpp: dyadic Bernoulli
    means, eta accounting and its unsafe-value fallbacks, tiny-probability fallbacks, lane
    permutation symmetry), compiled by oracle/ref.mk with the roulette header replaced by the
    oracle's restatement, passes."""
    import subprocess

    if not os.path.exists(ROULETTE_KNOWN_ANSWERS):
        pytest.skip("oracle/_ref/roulette_known_answers not built (needs a rypath checkout)")
    run = subprocess.run([ROULETTE_KNOWN_ANSWERS], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def hero_queries(n, rng):
    """Hero BSDF queries (layout of or_probe_hero): diffuse, conductor and dielectric packets
    with per-lane parameters (dispersive eta, smooth and rough lanes, matched indices), random
    masks; evaluation directions random, mirrored or refracted (so Dirac lanes see their own
    direction)."""
    q = np.zeros((n, 32), np.float32)
    kind = rng.integers(0, 3, n)
    q[:, 0] = kind
    mask = rng.integers(0, 16, n) | 1
    q[:, 1] = np.where(rng.uniform(size=n) < 0.5, 15, mask)
    q[:, 2] = rng.integers(0, 2, n)
    base_eta = np.where(kind == 1, rng.uniform(0.1, 3, n), rng.uniform(1.0, 2.4, n))
    base_eta = np.where((kind == 2) & (rng.uniform(size=n) < 0.05), 1.0, base_eta)
    dispersion = rng.uniform(0, 0.05, n) * (rng.uniform(size=n) < 0.6)
    rough = rng.uniform(0, 0.6, n) * (rng.uniform(size=n) > 0.35)
    for k in range(4):
        lane = 4 + 4 * k
        q[:, lane] = np.where(kind == 0, rng.uniform(0, 1, n), base_eta * (1 + dispersion * (k - 1.5)))
        q[:, lane + 1] = rng.uniform(0, 5, n)
        q[:, lane + 2] = rough
        q[:, lane + 3] = rough * rng.uniform(0.5, 1.5, n)
    wo = _unit(rng, n)
    q[:, 20:23] = wo
    wi = _unit(rng, n)
    mirror = wo * np.array([-1, -1, 1])
    eta = np.where(wo[:, 2] > 0, q[:, 4], 1 / q[:, 4]).astype(np.float64)
    cos_t2 = 1 - (1 - wo[:, 2] ** 2) / eta ** 2
    refract = np.concatenate([-wo[:, :2] / eta[:, None],
                              (-np.sign(wo[:, 2]) * np.sqrt(np.maximum(cos_t2, 0)))[:, None]], 1)
    choice = rng.integers(0, 3, n)
    q[:, 23:26] = np.where(choice[:, None] == 0, wi, np.where(choice[:, None] == 1, mirror, refract))
    q[:, 26:29] = rng.uniform(0, 1, (n, 3))
    return q


def test_hero_bsdf_matches_reference():
    """The oracle's hero proposals (companion densities on the hero direction, Dirac masses,
    dispersive companion support, event eta) equal rypath_hero_scattering's, compiled from
    shaders/hero_scattering.h, bit for bit."""
    lib = need_ref()
    q = hero_queries(30000, np.random.default_rng(21))
    a = np.zeros((q.shape[0], 32), np.float32)
    b = np.zeros((q.shape[0], 32), np.float32)
    oracle().or_probe_hero(q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_probe_hero(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    flags = a[:, 15].astype(np.int64)
    # the generator reaches every branch: accepted continuous and Dirac samples, transmissions,
    # dispersive Dirac companions with zero support, valid evaluations and Dirac lane masses
    assert ((flags & 5) == 5).mean() > 0.05 and ((flags & 5) == 4).mean() > 0.2
    assert ((flags & 2) != 0).mean() > 0.05
    dirac = (flags & 1) == 1
    assert ((a[:, 7:11] == 0) & (q[:, 1:2].astype(np.int64) == 15))[dirac].any()
    assert (a[:, 24] == 1).mean() > 0.5 and (a[:, 25] > 0).mean() > 0.02


def test_hero_roulette_matches_reference():
    """hero_continue and hero_account_eta (shaders/hero_pt_helpers.h:56-98), compiled from
    rypath's header, against the oracle's restatement on random tracks and edge values."""
    lib = need_ref()
    rng = np.random.default_rng(22)
    n = 30000
    q = np.zeros((n, 16), np.float32)
    q[:, 0:4] = np.exp(rng.uniform(-12, 1, (n, 4))) * (rng.uniform(size=(n, 4)) > 0.2)
    special = rng.uniform(size=(n, 4))
    q[:, 0:4] = np.where(special < 0.01, np.float32(1e-40), q[:, 0:4])
    q[:, 0:4] = np.where((special > 0.01) & (special < 0.015), np.inf, q[:, 0:4])
    q[:, 4:8] = np.exp(rng.uniform(-3, 3, (n, 4)))
    q[:, 4:8] = np.where(rng.uniform(size=(n, 4)) < 0.01, np.float32(2.0 ** 120), q[:, 4:8])
    q[:, 8] = rng.uniform(size=n) > 0.1
    q[:, 9] = rng.integers(0, 5, n)
    q[:, 10] = rng.uniform(0, 1, n)
    q[:, 11] = rng.integers(0, 2, n)
    q[:, 12:16] = rng.uniform(0.3, 2.5, (n, 4))
    q[:, 12:16] = np.where(rng.uniform(size=(n, 4)) < 0.01, 0.0, q[:, 12:16])
    a = np.zeros((n, 12), np.float32)
    b = np.zeros((n, 12), np.float32)
    oracle().or_probe_roulette(q.ctypes.data, n, a.ctypes.data)
    lib.ref_probe_roulette(q.ctypes.data, n, b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert 0.05 < (a[:, 0] == 0).mean() < 0.8  # paths are terminated and survive
    assert ((a[:, 1:5] != q[:, 0:4]).any(1) & (a[:, 0] == 1)).mean() > 0.05  # survivors are rescaled
    assert (a[:, 9] == 0).mean() > (q[:, 8] == 0).mean()  # unsafe eta disables roulette


def test_hero_weight_matches_reference():
    """The MIS weight of hero contributions (hero_weight, shaders/hero_pt_helpers.h:122-138)."""
    lib = need_ref()
    q = _advance_queries(30000, np.random.default_rng(23))
    rng = np.random.default_rng(24)
    q[:, 16:20] = np.where(rng.uniform(size=(q.shape[0], 1)) < 0.1, 0, q[:, 16:20])
    a = np.zeros((q.shape[0], 5), np.float32)
    b = np.zeros((q.shape[0], 5), np.float32)
    oracle().or_probe_hero_weight(q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_probe_hero_weight(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (a[:, 4] == 0).mean() > 0.3
