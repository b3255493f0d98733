"""Mix materials and pass-through surfaces: the host-side scene rules (no GPU needed: they are
checked before any device is looked for) and the oracle's transport semantics.

Rules follow src/render.cpp:302-315 (finite mix amounts), :1955-1995 (children in range, no
cycle, at most 64 nested levels, no null-interface child) and :1537-1590 (hero transport needs
inactive media).  Semantics: a per-hit stochastic mix of two diffuse materials estimates the
diffuse material with the mixed reflectance, and a null interface in vacuum scatters nothing.
"""

import ctypes as C

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, native, scenes


def create(scene):
    """rp_cuda_scene_create's status and diagnostic (RP_NO_DEVICE once the scene passed)."""
    desc = scene.desc()
    handle = C.c_void_p()
    diag = C.create_string_buffer(512)
    st = native.lib().rp_cuda_scene_create(C.byref(desc), 0, C.byref(handle), diag, 512)
    if st == abi.RP_SUCCESS:
        native.lib().rp_cuda_scene_destroy(handle)
    return st, diag.value.decode()


def passes(st):
    return st in (abi.RP_SUCCESS, abi.RP_NO_DEVICE)


def box_with(materials, short_box, tall_box=None):
    scene = scenes.cornell_box(8, 8, 1, 4)
    scene.materials += materials
    scene.instances[5].material = short_box
    if tall_box is not None:
        scene.instances[6].material = tall_box
    return scene


def test_mix_graph_rules():
    n = 4  # cornell_box has four materials
    ok, diag = create(box_with([scenes.mix_material(0, 1, 0.3), scenes.mix_material(n, 2, 0.5)], n + 1))
    assert passes(ok), diag
    st, diag = create(box_with([scenes.mix_material(n + 1, 0, 0.3), scenes.mix_material(n, 1, 0.5)], n))
    assert st == abi.RP_INVALID_ARGUMENT and "Cyclic" in diag
    st, diag = create(box_with([scenes.mix_material(0, 99, 0.3)], n))
    assert st == abi.RP_INVALID_ARGUMENT and "invalid child" in diag
    st, diag = create(box_with([scenes.mix_material(0, 1, float("nan"))], n))
    assert st == abi.RP_INVALID_ARGUMENT and "finite amount" in diag
    interface = abi.Material()
    interface.scattering = abi.INTERFACE
    st, diag = create(box_with([interface, scenes.mix_material(0, n, 0.5)], n + 1))
    assert st == abi.RP_INVALID_ARGUMENT and "null boundaries" in diag
    # an unused cyclic mix fails too (rypath's preflight checks every material)
    st, diag = create(box_with([scenes.mix_material(n, n, 0.5)], 0))
    assert st == abi.RP_INVALID_ARGUMENT and "Cyclic" in diag


@pytest.mark.parametrize("levels, ok", [(64, True), (65, False)])
def test_mix_nesting_limit(levels, ok):
    n = 4
    chain = [scenes.mix_material(0, 1, 0.5)] + [scenes.mix_material(n + i, 2, 0.5) for i in range(levels - 1)]
    st, diag = create(box_with(chain, n + levels - 1))
    assert passes(st) == ok, diag
    if not ok:
        assert "64 levels" in diag


def test_hero_vacuum_rule_counts_only_active_media():
    scene = scenes.cornell_pass_through(8, 8, 1, 4)
    scene.media = [dict(sigma_a=0.0, sigma_s=0.0, emission=0.0, g=0.3)]
    scene.camera_medium = 0  # cleared for the vacuum transport, as rypath's transport selection does
    st, diag = create(scene)
    assert passes(st), diag
    scene.media = [dict(sigma_a=0.0, sigma_s=0.5, emission=0.0, g=0.3)]
    st, diag = create(scene)
    assert st == abi.RP_INVALID_ARGUMENT and "vacuum" in diag


def oracle_film(scene, width, height, spp, seed):
    lanes = OracleScene(scene).sample(request(width, height, spp, seed=seed, sampler=abi.SAMPLER_INDEPENDENT))
    assert (lanes["status"] == 0).all()
    film = np.zeros(width * height, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, width * height, film.ctypes.data) == 0
    n = film["count"][:, None].astype(np.float64)
    mean = (film["sum"] + film["correction"]) / n
    return mean, np.maximum(film["square"] / n - mean ** 2, 0) / n


def constant_diffuse(value):
    m = abi.Material()
    m.scattering, m.kind, m.scalar_value = abi.DIFFUSE, abi.REFLECTANCE_CONSTANT, value
    return m


def test_diffuse_mix_estimates_the_mixed_reflectance():
    """mix(0.8, 0.2, amount 0.25) on every wall and box against a constant 0.65 diffuse."""
    def scene(mixed):
        s = scenes.cornell_box(8, 8, 1, 5)
        s.materials += [constant_diffuse(0.8), constant_diffuse(0.2), scenes.mix_material(4, 5, 0.25),
                        constant_diffuse(0.75 * 0.8 + 0.25 * 0.2)]
        for i in range(7):
            s.instances[i].material = 6 if mixed else 7
        return s

    m1, v1 = oracle_film(scene(True), 8, 8, 1024, 11)
    m2, v2 = oracle_film(scene(False), 8, 8, 1024, 12)
    z = (m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(np.abs(z) < 4) > 0.98
    assert abs(m1.sum() - m2.sum()) < 4 * np.sqrt(v1.sum() + v2.sum())


def test_null_pane_in_vacuum_scatters_nothing():
    def scene(pane):
        return scenes.cornell_pass_through(8, 8, 1, 5, pane=pane, invisible_light=False, mixes=False)

    m1, v1 = oracle_film(scene(True), 8, 8, 512, 21)
    m2, v2 = oracle_film(scene(False), 8, 8, 512, 22)
    z = (m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(np.abs(z) < 4) > 0.98
    assert abs(m1.sum() - m2.sum()) < 4 * np.sqrt(v1.sum() + v2.sum())
