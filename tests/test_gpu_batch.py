"""Batched views (rp_cuda_render_views_device): many views of uneven size and sample count in
one wavefront must give every view the film a plain render of that view gives, bit for bit,
with waves that split views, with and without CUDA-graph replay, and with the configuration
the autotuner picks.
"""

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def batch_film(rs, views, request, torch):
    total = renderer.pack_views(views)
    film = torch.zeros(total * abi.FILM_PIXEL_BYTES, dtype=torch.uint8, device="cuda")
    used = rs.render_views_device(views, request, film.data_ptr())
    torch.cuda.synchronize()
    return film.cpu().numpy().view(abi.film_dtype()), used


def plain_film(rs, view, seed=1):
    settings = renderer.RenderSettings(width=view.width, height=view.height, samples=view.sample_count,
                                       batch_size=view.sample_count, seed=seed)
    st, diag, film = rs.render_film(settings, sample_begin=view.sample_begin)
    assert st == abi.RP_SUCCESS, diag
    return film


def per_view_plain(scene, views):
    films = []
    for v in views:
        one = scenes.Scene(**{k: getattr(scene, k) for k in scene.__dataclass_fields__ if k != "_keep"})
        one.camera = v.camera
        rs = build(one)
        films.append(plain_film(rs, v))
        rs.close()
    return films


def cornell_views():
    base = scenes.cornell_box(8, 8, 1)
    views = []
    for (w, h, spp, begin) in ((16, 16, 3, 0), (40, 24, 5, 0), (7, 9, 2, 3), (33, 17, 1, 5), (64, 64, 4, 0)):
        cam = scenes.pinhole_camera((0.2 * w / 64, 1.0, 3.94), (0, 1, 0), (0, 1, 0), 40.0, w, h)
        views.append(renderer.View(cam, w, h, begin, spp))
    return base, views


def assert_same(batch, plains, views):
    for v, plain in zip(views, plains):
        got = batch[v.film_offset:v.film_offset + v.width * v.height]
        assert got.tobytes() == plain.tobytes()


@pytest.mark.parametrize("use_graph", [1, 2])
def test_batched_views_equal_plain_renders_bit_for_bit(use_graph):
    torch = pytest.importorskip("torch")
    scene, views = cornell_views()
    rs = build(scene)
    request = renderer.BatchRequest(wave_lanes=1000, trace_block=64, shade_block=256, blocks_per_sm=8,
                                    use_graph=use_graph)
    film, used = batch_film(rs, views, request, torch)
    assert used.wave_lanes == 1000 and used.use_graph == use_graph
    assert_same(film, per_view_plain(scene, views), views)
    t = rs.timing()
    assert t.samples == sum(v.width * v.height * v.sample_count for v in views)


def test_autotuned_batch_equals_plain_renders():
    torch = pytest.importorskip("torch")
    scene, views = cornell_views()
    rs = build(scene)
    renderer.pack_views(views)
    chosen = rs.tune_views(views, renderer.BatchRequest())
    assert chosen.trace_block in (64, 128) and chosen.shade_block in (128, 256)
    assert 1 <= chosen.blocks_per_sm <= 32 and 0 < chosen.wave_lanes <= 1 << 23
    assert chosen.probe_ms_per_mlane > 0
    film, used = batch_film(rs, views, renderer.BatchRequest(), torch)
    assert used.wave_lanes > 0
    assert_same(film, per_view_plain(scene, views), views)


def test_batched_mixed_scene_views_equal_plain_renders():
    torch = pytest.importorskip("torch")
    scene = scenes.mixed_scene(8, 8, 1, 6, subdivisions=4)
    views = scenes.view_batch(scene, count=3, seed=3, min_size=(24, 16), max_size=(48, 40), spp=(1, 2, 3))
    rs = build(scene)
    film, _ = batch_film(rs, views, renderer.BatchRequest(wave_lanes=4096, trace_block=128, shade_block=128,
                                                          blocks_per_sm=12), torch)
    assert_same(film, per_view_plain(scene, views), views)


def test_batch_validation():
    torch = pytest.importorskip("torch")
    scene, views = cornell_views()
    rs = build(scene)
    total = renderer.pack_views(views)
    film = torch.zeros(total * abi.FILM_PIXEL_BYTES, dtype=torch.uint8, device="cuda")  # a valid film: rejection precedes launches
    views[2].film_offset = 0  # overlaps view 0
    with pytest.raises(RuntimeError, match="overlap"):
        rs.render_views_device(views, renderer.BatchRequest(wave_lanes=1000, trace_block=64, shade_block=128,
                                                            blocks_per_sm=8), film.data_ptr())
    renderer.pack_views(views)
    with pytest.raises(RuntimeError, match="trace block"):
        rs.render_views_device(views, renderer.BatchRequest(wave_lanes=1000, trace_block=96, shade_block=128,
                                                            blocks_per_sm=8), film.data_ptr())
