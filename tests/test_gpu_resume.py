"""Failure handling and resume of the progressive film, through the C ABI, with host-made
failures only.

rypath's driver commits a film batch by batch; a batch with a failed lane fails the render
and leaves the committed film as it was (src/render_driver.cpp:201-214), and a render resumes
from a committed film at its next absolute sample (src/render_driver.cpp:67-111,
src/render_job.cpp:120-170).  Because the device film reduces every batch in canonical
(absolute sample, pixel) order onto the committed sums, a resumed render equals the one
uninterrupted render bit for bit, and so does any batch size (rypath's progressive
bit-exactness across batch sizes, docs/rendering.md:179-192).  The failure is made on the host:
an emergency depth limit of one vertex, which the Cornell box's second bounces exceed.
"""

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu

W = H = 32


@pytest.fixture(scope="module")
def cornell():
    built = renderer.build_renderer(scenes.cornell_box(W, H, 8))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    yield built.scene
    built.scene.close()


@pytest.fixture(scope="module")
def fog():
    built = renderer.build_renderer(scenes.crop(scenes.cornell_fog(256, 256), 96, 96, W, H))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    yield built.scene
    built.scene.close()


def settings(spp, batch, **kw):
    return renderer.RenderSettings(W, H, samples=spp, batch_size=batch, seed=1, **kw)


def test_failed_batch_keeps_the_committed_host_film(cornell):
    st, diag, committed = cornell.render_film(settings(4, 4))
    assert st == abi.RP_SUCCESS, diag
    before = committed.copy()
    st, diag, film = cornell.render_film(settings(4, 2, emergency_limit=1), committed, sample_begin=4)
    assert st == abi.RP_FAILURE
    assert "batch failed" in diag
    assert film.tobytes() == before.tobytes()
    # the failed call leaves the scene usable: the resumed render still completes
    st, diag, film = cornell.render_film(settings(4, 4), film, sample_begin=4)
    assert st == abi.RP_SUCCESS, diag
    assert film["count"].min() == 8


def test_failed_batch_keeps_the_committed_device_film(cornell):
    torch = pytest.importorskip("torch")
    st, diag, committed = cornell.render_film(settings(4, 4))
    assert st == abi.RP_SUCCESS, diag
    device = torch.from_numpy(committed.view(np.uint8).copy()).cuda()
    st, diag = cornell.render_film_device(settings(4, 4, emergency_limit=1), device.data_ptr(), sample_begin=4,
                                          check=False)
    assert st == abi.RP_FAILURE and "batch failed" in diag
    assert device.cpu().numpy().tobytes() == committed.tobytes()


@pytest.mark.parametrize("transport", ["hero", "scalar"])
def test_resumed_render_equals_one_render(cornell, fog, transport):
    scene = cornell if transport == "hero" else fog
    st, diag, whole = scene.render_film(settings(8, 8))
    assert st == abi.RP_SUCCESS, diag
    st, diag, first = scene.render_film(settings(4, 4))
    assert st == abi.RP_SUCCESS, diag
    st, diag, resumed = scene.render_film(settings(4, 4), first.copy(), sample_begin=4)
    assert st == abi.RP_SUCCESS, diag
    assert resumed.tobytes() == whole.tobytes()
    assert whole["count"].min() == 8


@pytest.mark.parametrize("batch", [1, 3, 7])
def test_batch_size_does_not_change_the_film(cornell, batch):
    st, diag, reference = cornell.render_film(settings(8, 8))
    assert st == abi.RP_SUCCESS, diag
    st, diag, film = cornell.render_film(settings(8, batch))
    assert st == abi.RP_SUCCESS, diag
    assert film.tobytes() == reference.tobytes()


def test_device_film_resume_equals_host_film(cornell):
    torch = pytest.importorskip("torch")
    st, diag, whole = cornell.render_film(settings(8, 8))
    assert st == abi.RP_SUCCESS, diag
    device = torch.zeros(W * H * abi.film_dtype().itemsize, dtype=torch.uint8, device="cuda")
    cornell.render_film_device(settings(4, 2), device.data_ptr(), fresh=True)
    cornell.render_film_device(settings(4, 4), device.data_ptr(), sample_begin=4)
    assert device.cpu().numpy().tobytes() == whole.tobytes()
