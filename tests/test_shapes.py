"""Bilinear patches and analytic shapes in the oracle's transports (rypath's procedural
primitives: GeometryMesh::patches / ::analytics, shaders/bilinear.h, shaders/analytic.h,
shaders/render.metal:970-1132).  CPU only.

* The oracle's closest hits on the shapes box equal a brute-force scan.
* A planar patch gives the hits of the two triangles of the same quad.
* The white furnace: convex diffuse shapes (sphere, holed disk, open cylinder, flat patch) of
  reflectance 0.5 under a constant unit environment return 0.5 at every pixel they cover and 1
  elsewhere, in both transports (six standard errors).
* The scalar and hero transports agree on the shapes box per pixel and over the image.
"""

import ctypes as C
import math

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, scenes


def trace(scene, rays, brute=False):
    o = OracleScene(scene)
    out = np.zeros((rays.shape[0], 4), np.float32)
    oracle().or_trace_rays(o.handle, rays.ctypes.data, rays.shape[0], 0, int(brute), out.ctypes.data)
    return out


def test_oracle_closest_hits_equal_a_brute_force_scan():
    scene = scenes.cornell_shapes(8, 8, 1)
    rng = np.random.default_rng(3)
    rays = np.zeros((20000, 7), np.float32)
    rays[:, 0:3] = rng.uniform([-0.9, 0.1, -0.9], [0.9, 1.9, 0.9], (20000, 3))
    d = rng.normal(size=(20000, 3))
    rays[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 6] = np.inf
    a, b = trace(scene, rays), trace(scene, rays, brute=True)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    prim = a[:, 3].view(np.uint32)
    triangle_prims = sum(int(i.triangle_count) for i in scene.instances)
    hit = prim != abi.RP_NONE
    assert hit.mean() > 0.7  # the box is open at the front
    assert np.mean(hit & (prim >= triangle_prims)) > 0.05  # patches and shapes are hit


def planar_scenes():
    quad = [(-0.5, -0.4, 0.0), (0.6, -0.5, 0.1), (-0.4, 0.5, -0.1), (0.7, 0.4, 0.0)]
    quad[3] = tuple(np.add(np.subtract(quad[1], quad[0]), quad[2]))  # a parallelogram
    m = scenes.diffuse_material(0)
    tri = scenes.Scene("tri", 4, 4, 1, np.array([quad[0], quad[1], quad[3], quad[2]], np.float32),
                       np.array([(0, 1, 2), (0, 2, 3)], np.uint32), [scenes.identity_instance(0, 0, 2, 0)], [m],
                       scenes.knots_from_curve(0.5))
    pat = scenes.Scene("patch", 4, 4, 1, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), [], [m],
                       scenes.knots_from_curve(0.5))
    scenes.add_patches(pat, [quad], 0)
    return tri, pat


def test_planar_patch_hits_equal_its_triangles():
    tri, pat = planar_scenes()
    rng = np.random.default_rng(4)
    rays = np.zeros((5000, 7), np.float32)
    rays[:, 0:3] = rng.uniform(-1, 1, (5000, 3)) + np.array([0, 0, 3])
    target = rng.uniform(-0.8, 0.8, (5000, 3)) * np.array([1, 1, 0])
    rays[:, 3:6] = target - rays[:, 0:3]
    rays[:, 6] = np.inf
    a, b = trace(tri, rays), trace(pat, rays)
    ha, hb = a[:, 3].view(np.uint32) != abi.RP_NONE, b[:, 3].view(np.uint32) != abi.RP_NONE
    assert 0.3 < ha.mean() < 0.9
    # rays within float rounding of the boundary may go either way
    assert np.mean(ha == hb) > 0.999
    both = ha & hb
    np.testing.assert_allclose(a[both, 0], b[both, 0], rtol=2e-5)


def pixel_corner_rays(scene):
    o, corner, dx, dy = (np.asarray(v, np.float64) for v in scene.camera)
    w, h = scene.width, scene.height
    xs, ys = np.meshgrid(np.arange(w + 1) / w, np.arange(h + 1) / h)
    d = corner + xs[..., None] * dx + ys[..., None] * dy
    rays = np.zeros(((h + 1) * (w + 1), 7), np.float32)
    rays[:, 0:3] = o
    rays[:, 3:6] = d.reshape(-1, 3)
    rays[:, 6] = np.inf
    return rays


def covered_pixels(scene):
    """Pixels whose four corner rays hit the (convex) object, and pixels none of whose corner
    rays do and whose neighbours' corners miss too."""
    hit = trace(scene, pixel_corner_rays(scene))[:, 3].view(np.uint32) != abi.RP_NONE
    hit = hit.reshape(scene.height + 1, scene.width + 1)
    inside = hit[:-1, :-1] & hit[1:, :-1] & hit[:-1, 1:] & hit[1:, 1:]
    any_corner = hit[:-1, :-1] | hit[1:, :-1] | hit[:-1, 1:] | hit[1:, 1:]
    return inside.reshape(-1), ~any_corner.reshape(-1)


def furnace_values(scene, spp, seed):
    w, h = scene.width, scene.height
    q = request(w, h, spp, seed=seed, sampler=abi.SAMPLER_INDEPENDENT)
    if scene.transport == abi.TRANSPORT_SCALAR:
        r = OracleScene(scene).sample_scalar(q)
        assert np.all(r["status"] == abi.SAMPLE_SUCCESS)
        return r["radiance"].astype(np.float64).reshape(spp, w * h)  # radiance of a unit-sky path
    r = OracleScene(scene).sample(q)
    assert np.all(r["status"] == abi.SAMPLE_SUCCESS)
    return (np.sum(r["radiance"] / r["wavelength_pdfs"], axis=1) / (4.0 * 470.0)).reshape(spp, w * h)


def furnace_gate(values, inside, outside, rho=0.5):
    for mask, expected in ((inside, rho), (outside, 1.0)):
        v = values[:, mask]
        se = v.std(ddof=1) / math.sqrt(v.size)
        assert abs(v.mean() - expected) <= 6 * se + 1e-4, (v.mean(), expected, se)


@pytest.mark.parametrize("transport", [abi.TRANSPORT_HERO, abi.TRANSPORT_SCALAR])
@pytest.mark.parametrize("kind", ["sphere", "disk", "cylinder", "patch"])
def test_white_furnace_of_convex_shapes(kind, transport):
    scene = scenes.shape_furnace(kind, 16, 16, 1, transport=transport)
    inside, outside = covered_pixels(scene)
    assert inside.sum() >= 8 and outside.sum() >= 40
    furnace_gate(furnace_values(scene, 512, 7), inside, outside)


def test_scalar_and_hero_transports_agree_on_the_shapes_box():
    hero = scenes.cornell_shapes(16, 16, 1, transport=abi.TRANSPORT_HERO)
    scalar = scenes.cornell_shapes(16, 16, 1, transport=abi.TRANSPORT_SCALAR)
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
