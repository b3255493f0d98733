"""Frame sessions (FrameSession, src/frame_session.hpp:182-212) through the C ABI.

A frame renders one absolute sample of every pixel into raw XYZ on the device
(shaders/frame_sensor.h): the packet sensor value without the filter weight, in binary32.  It
therefore equals the film mean of a one-sample film render at the same absolute sample (FP64,
box filter) to binary32 rounding.  Frames are asynchronous and hold one of two slots until
released; a camera in the request replaces the session's camera; the scalar transport's
frames use its own sensor (matching functions x 470 x radiance).
"""

import numpy as np
import pytest

from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu

W = H = 32


@pytest.fixture(scope="module")
def cornell():
    built = renderer.build_renderer(scenes.cornell_box(W, H, 1))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    yield built.scene
    built.scene.close()


def film_frame(scene, sample_index, sampler=abi.SAMPLER_INDEPENDENT):
    st, diag, film = scene.render_film(renderer.RenderSettings(W, H, samples=1, batch_size=1, seed=1, sampler=sampler),
                                       sample_begin=sample_index, fresh=True)
    assert st == abi.RP_SUCCESS, diag
    return renderer.film_mean(film).reshape(H, W, 3)


@pytest.mark.parametrize("sampler", [abi.SAMPLER_INDEPENDENT, abi.SAMPLER_SOBOL])
def test_frame_equals_one_sample_film(cornell, sampler):
    fs = renderer.FrameSession(cornell, renderer.FrameConfig(W, H, seed=1, sampler=sampler))
    for k in (0, 5):
        st, frame, busy, diag = fs.submit(k, epoch=k)
        assert st == abi.RP_SUCCESS and not busy, diag
        info = fs.wait(frame)
        assert info.status == abi.FRAME_COMPLETE and info.sample_index == k and info.epoch == k
        assert info.completed_samples == W * H and info.gpu_ms > 0
        st, diag, xyz = fs.capture(frame)
        assert st == abi.RP_SUCCESS, diag
        np.testing.assert_allclose(xyz, film_frame(cornell, k, sampler), rtol=2e-6, atol=1e-12)
        fs.release(frame)
    fs.close()


def test_frames_are_asynchronous_and_hold_two_slots(cornell):
    fs = renderer.FrameSession(cornell, renderer.FrameConfig(W, H))
    st, a, _, diag = fs.submit(1)
    assert st == abi.RP_SUCCESS, diag
    st, b, _, diag = fs.submit(2)
    assert st == abi.RP_SUCCESS and a != b, diag
    st, c, busy, diag = fs.submit(3)
    assert st == abi.RP_FAILURE and busy and c is None
    assert fs.poll(a).status in (abi.FRAME_PENDING, abi.FRAME_COMPLETE)
    fs.wait(b)
    _, _, xb = fs.capture(b)
    _, _, xa = fs.capture(a)
    assert not np.array_equal(xa, xb)  # another absolute sample
    fs.release(a)
    st, c, busy, diag = fs.submit(1)
    assert st == abi.RP_SUCCESS and c == a, diag
    _, _, xc = fs.capture(c)
    assert xc.tobytes() == xa.tobytes()  # the same sample again: the same frame
    fs.release(b)
    fs.release(c)
    fs.close()


def test_frame_camera_replaces_the_scene_camera(cornell):
    moved = scenes.pinhole_camera((0.4, 1.1, 3.6), (0.0, 0.9, 0.0), (0, 1, 0), 44.0, W, H)
    fs = renderer.FrameSession(cornell, renderer.FrameConfig(W, H))
    st, frame, _, diag = fs.submit(3, camera=moved)
    assert st == abi.RP_SUCCESS, diag
    _, _, xyz = fs.capture(frame)
    fs.release(frame)
    st, frame, _, diag = fs.submit(3)  # the session keeps the new camera
    _, _, again = fs.capture(frame)
    fs.release(frame)
    fs.close()
    other = scenes.cornell_box(W, H, 1)
    other.camera = moved
    built = renderer.build_renderer(other)
    fs2 = renderer.FrameSession(built.scene, renderer.FrameConfig(W, H))
    st, frame, _, diag = fs2.submit(3)
    _, _, reference = fs2.capture(frame)
    fs2.release(frame)
    fs2.close()
    built.scene.close()
    assert xyz.tobytes() == reference.tobytes() == again.tobytes()
    # and the scene's own camera is untouched by the session
    assert not np.array_equal(film_frame(cornell, 3), reference)


def test_scalar_frame_equals_one_sample_film():
    built = renderer.build_renderer(scenes.crop(scenes.cornell_fog(256, 256), 96, 96, W, H))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    fs = renderer.FrameSession(built.scene, renderer.FrameConfig(W, H, sampler=abi.SAMPLER_INDEPENDENT))
    st, frame, _, diag = fs.submit(7)
    assert st == abi.RP_SUCCESS, diag
    st, diag, xyz = fs.capture(frame)
    assert st == abi.RP_SUCCESS, diag
    fs.release(frame)
    fs.close()
    np.testing.assert_allclose(xyz, film_frame(built.scene, 7), rtol=2e-6, atol=1e-12)
    built.scene.close()
