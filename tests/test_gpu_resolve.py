"""Pass-through surfaces and mix materials on the device against the oracle.

Hero transport (shaders/packet_pt_event_body.inc:100-205, shaders/packet_transport.h:377-446):
a null-interface pane and an invisible area light that camera, bounce and shadow rays cross,
and nested mix materials resolved per hit by the PBRT alpha hash.  Scalar transport
(shaders/scalar_transport.h:541-587): mix materials in the fog-filled box.  Per lane: identity
and status bit for bit, radiance within the per-lane tolerance of the hero parity tests.  A mix
at amount 0 or 1 renders its first or second child bit for bit (rypath's mix endpoint test,
tests/surface_material_render_tests.cpp:77-110).
"""

import numpy as np
import pytest

from oracle_lib import OracleScene, request
from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-3
MATCH_FRACTION = 0.97


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def to_request(q):
    return renderer.RenderRequest(q.width, q.height, seed=q.seed, pixel_begin=q.pixel_begin, pixel_count=q.pixel_count,
                                  sample_begin=q.sample_begin, sample_count=q.sample_count, sampler=q.sampler_kind,
                                  randomization=q.randomization, boundary_limit=q.boundary_limit)


def assert_lanes_match(g, c):
    for f in ("status", "pixel", "sample_low", "sample_high"):
        np.testing.assert_array_equal(g[f], c[f])
    gr, cr = g["radiance"].astype(np.float64), c["radiance"].astype(np.float64)
    close = np.all(np.abs(gr - cr) <= RTOL * np.maximum(np.abs(cr), 1e-6) + 1e-7, axis=1)
    assert close.mean() >= MATCH_FRACTION, close.mean()
    return gr


@pytest.mark.parametrize("sampler", [abi.SAMPLER_SOBOL, abi.SAMPLER_INDEPENDENT])
def test_pass_through_and_mix_lanes_match_the_oracle(sampler):
    scene = scenes.cornell_pass_through(32, 32, 4, 8)
    q = request(32, 32, 4, sampler=sampler)
    c = OracleScene(scene).sample(q)
    res = build(scene).sample(to_request(q))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    gr = assert_lanes_match(res.packet_samples, c)
    np.testing.assert_array_equal(c["status"], 0)
    assert (gr.sum(1) > 0).mean() > 0.2


def test_boundary_limit_is_the_oracles():
    """Two panes in a row and a limit of one crossing: every camera ray through both fails with
    boundary exhaustion, as in the oracle."""
    scene = scenes.cornell_pass_through(16, 16, 2, 8, invisible_light=False, mixes=False)
    pane = scene.instances[-1]
    second = scenes.identity_instance(scene.positions.shape[0], scene.triangles.shape[0], 2, pane.material)
    scene.positions = np.concatenate([scene.positions, scene.positions[-4:] + np.float32([0, 0, 0.1])])
    scene.triangles = np.concatenate([scene.triangles, scene.triangles[-2:]])
    scene.instances.append(second)
    q = request(16, 16, 2)
    q.boundary_limit = 1
    c = OracleScene(scene).sample(q)
    res = build(scene).sample(to_request(q))
    assert res.status != abi.RP_SUCCESS  # failed lanes fail the call
    assert_lanes_match(res.packet_samples, c)
    assert (c["status"] == abi.BOUNDARY_EXHAUSTION).mean() > 0.3


def test_pane_and_invisible_light_leave_the_image_statistically_unchanged():
    """A null interface in vacuum scatters nothing: the film with the pane equals the film without
    it within 4 combined standard errors per pixel."""
    def film(pane):
        rs = build(scenes.cornell_pass_through(16, 16, 64, 6, pane=pane, invisible_light=False, mixes=False))
        st, diag, f = rs.render_film(renderer.RenderSettings(16, 16, samples=256, batch_size=64, seed=3,
                                                             sampler=abi.SAMPLER_INDEPENDENT))
        assert st == abi.RP_SUCCESS, diag
        n = f["count"][:, None].astype(np.float64)
        mean = (f["sum"] + f["correction"]) / n
        return mean, np.maximum(f["square"] / n - mean ** 2, 0) / n

    m1, v1 = film(True)
    m2, v2 = film(False)
    z = np.abs(m1 - m2) / np.sqrt(v1 + v2 + 1e-30)
    assert np.mean(z < 4) > 0.99, np.mean(z < 4)


@pytest.mark.parametrize("amount, child", [(0.0, 0), (1.0, 1)])
def test_mix_endpoints_render_the_child_bit_for_bit(amount, child):
    mixed = scenes.cornell_box(24, 24, 2, 6)
    direct = scenes.cornell_box(24, 24, 2, 6)
    children = (0, 1)  # white, red
    mixed.materials.append(scenes.mix_material(children[0], children[1], amount))
    mixed.instances[5].material = mixed.instances[6].material = len(mixed.materials) - 1
    direct.instances[5].material = direct.instances[6].material = children[child]
    req = renderer.RenderRequest(24, 24, sample_count=2)
    a = build(mixed).sample(req)
    b = build(direct).sample(req)
    assert a.status == b.status == abi.RP_SUCCESS
    assert a.packet_samples.tobytes() == b.packet_samples.tobytes()


def test_scalar_mix_lanes_match_the_oracle():
    """In an absorbing (non-scattering) medium: the alpha hash of a mix depends on every bit of
    the hit point, and free-flight distances drawn through the device's logf and the host's
    would move scattering vertices by an ulp now and then, flipping the mix's choice there."""
    scene = scenes.cornell_fog(24, 24, 4, 8)
    scene.media[0]["sigma_s"] = np.zeros(471, np.float32)
    scene.media[0]["sigma_a"] = np.full(471, 0.3, np.float32)
    scene.materials.append(scenes.mix_material(0, 1, 0.4))
    scene.materials.append(scenes.mix_material(len(scene.materials) - 1, 2, 0.6))
    scene.instances[5].material = len(scene.materials) - 2
    scene.instances[6].material = len(scene.materials) - 1
    q = request(24, 24, 4, sampler=abi.SAMPLER_INDEPENDENT)
    ref = OracleScene(scene).sample_scalar(q)
    res = build(scene).sample_scalar(to_request(q))
    assert res.status == abi.RP_SUCCESS, res.diagnostic
    got = res.samples
    for f in ("status", "pixel", "sample_low", "sample_high", "random_words"):
        np.testing.assert_array_equal(got[f], ref[f])
    same = got["scatterings"] == ref["scatterings"]
    close = np.isclose(got["radiance"], ref["radiance"], rtol=RTOL, atol=1e-7)
    assert np.mean(same & close) >= MATCH_FRACTION


def test_the_allocation_free_entry_point_refuses_resolve_scenes():
    """Its static scratch has no room for resolved materials and shadow targets; the refusal
    comes before any device work."""
    import ctypes as C

    from rypath_b200 import native

    torch = pytest.importorskip("torch")
    rs = build(scenes.cornell_pass_through(8, 8, 1, 4))
    out = torch.zeros(64 * 80, dtype=torch.uint8, device="cuda")
    diag = C.create_string_buffer(256)
    req = renderer.RenderRequest(8, 8, sample_count=1).to_c()
    st = native.lib().rp_cuda_sample_device_static(rs.handle, C.byref(req), C.c_void_p(out.data_ptr()), 64, None,
                                                   diag, 256)
    assert st == abi.RP_INVALID_ARGUMENT and b"pass-through, mix" in diag.value
