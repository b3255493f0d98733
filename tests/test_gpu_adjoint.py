"""Path-replay adjoint of the hero film render (rp_cuda_adjoint_device).

* Against the FP64 host adjoint of the oracle on the same lanes (same contributions, float
  device accumulation against double host accumulation).
* Against central finite differences of the device forward render with common random
  numbers, at depth 1 where no Russian roulette runs (with roulette the survival test is a
  step in the parameters, which finite differences see and the adjoint, by design, does not).
* Through the test-only torch.autograd.Function: autograd's gradient is the adjoint's, and
  Adam steps on reflectance knots lower an L2 image loss.
"""

import numpy as np
import pytest

from oracle_lib import oracle_adjoint
from rypath_b200 import abi, renderer, scenes

pytestmark = pytest.mark.gpu


def build(scene):
    built = renderer.build_renderer(scene)
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    return built.scene


def device_mean(rs, settings, torch):
    from torch_adjoint import film_mean_device

    pixels = settings.width * settings.height
    film = torch.zeros(pixels * abi.FILM_PIXEL_BYTES, dtype=torch.uint8, device="cuda")
    rs.render_film_device(settings, film.data_ptr())
    torch.cuda.synchronize()
    return film_mean_device(film, pixels)


def device_adjoint(rs, settings, materials, g, params, torch):
    grad = torch.zeros(params, dtype=torch.float32, device="cuda")
    rs.adjoint_device(settings, materials, g.contiguous().data_ptr(), grad.data_ptr())
    torch.cuda.synchronize()
    return grad.cpu().numpy().astype(np.float64)


def test_device_adjoint_matches_the_fp64_host_adjoint():
    torch = pytest.importorskip("torch")
    w = h = 16
    scene = scenes.cornell_box(w, h, 4, max_depth=6)
    rs = build(scene)
    settings = renderer.RenderSettings(width=w, height=h, samples=4, batch_size=4, seed=1)
    mean = device_mean(rs, settings, torch)
    target = 0.6 * mean
    g = 2 * (mean - target)
    materials = [0, 1, 2]
    got = device_adjoint(rs, settings, materials, g, 96, torch)
    ref = oracle_adjoint(scene, w, h, 4, materials, g.cpu().numpy())
    assert np.linalg.norm(ref) > 0
    assert np.linalg.norm(got - ref) <= 5e-3 * np.linalg.norm(ref), (np.linalg.norm(got - ref), np.linalg.norm(ref))
    big = np.abs(ref) > 1e-2 * np.abs(ref).max()
    np.testing.assert_allclose(got[big], ref[big], rtol=2e-2)


def test_device_adjoint_matches_central_differences_without_roulette():
    torch = pytest.importorskip("torch")
    w = h = 32
    scene = scenes.cornell_box(w, h, 8, max_depth=1)
    rs = build(scene)
    settings = renderer.RenderSettings(width=w, height=h, samples=8, batch_size=8, seed=1)
    mean = device_mean(rs, settings, torch)
    target = 0.5 * mean
    materials = [0, 1, 2]
    grad = device_adjoint(rs, settings, materials, 2 * (mean - target), 96, torch)

    def loss():
        return float(((device_mean(rs, settings, torch) - target) ** 2).sum())

    step = 1e-3
    for m, j in ((0, 5), (0, 20), (1, 25), (2, 12), (2, 3)):
        k = int(scene.materials[m].knot_begin) + j
        v0 = float(scene.knots[k, 1])
        rs.set_knot_values(k, [v0 + step])
        up = loss()
        rs.set_knot_values(k, [v0 - step])
        down = loss()
        rs.set_knot_values(k, [v0])
        fd = (up - down) / (2 * step)
        assert abs(fd - grad[m * 32 + j]) <= 2e-3 * abs(fd) + 1e-6 * np.abs(grad).max(), (m, j, fd, grad[m * 32 + j])


def test_autograd_function_and_adam_lower_the_loss():
    torch = pytest.importorskip("torch")
    from torch_adjoint import SpectralFilm, knot_parameters

    w = h = 16
    truth = scenes.cornell_box(w, h, 8, max_depth=4)
    settings = renderer.RenderSettings(width=w, height=h, samples=8, batch_size=8, seed=1)
    target = device_mean(build(truth), settings, torch).detach()
    scene = scenes.cornell_box(w, h, 8, max_depth=4)
    materials = [0, 1, 2]
    for m in materials:  # start from constant 0.5 reflectance
        kb = scene.materials[m].knot_begin
        scene.knots[kb:kb + 32, 1] = 0.5
    rs = build(scene)
    theta = torch.tensor(knot_parameters(scene, materials), requires_grad=True)
    out = SpectralFilm.apply(theta, rs, scene, settings, materials)
    loss = ((out - target) ** 2).sum()
    loss.backward()
    direct = device_adjoint(rs, settings, materials, 2 * (out.detach() - target), 96, torch)
    np.testing.assert_allclose(theta.grad.numpy(), direct, rtol=1e-5, atol=1e-12)
    opt = torch.optim.Adam([theta], lr=0.03)
    losses = []
    for _ in range(8):
        opt.zero_grad()
        loss = ((SpectralFilm.apply(theta, rs, scene, settings, materials) - target) ** 2).sum()
        loss.backward()
        opt.step()
        with torch.no_grad():
            theta.clamp_(0.01, 1.0)
        losses.append(float(loss.detach()))
    assert losses[-1] < 0.5 * losses[0], losses


def test_adjoint_validation():
    torch = pytest.importorskip("torch")
    scene = scenes.cornell_box(8, 8, 1, max_depth=16)
    rs = build(scene)
    settings = renderer.RenderSettings(width=8, height=8, samples=1, batch_size=1)
    g = torch.zeros(64 * 3, dtype=torch.float64, device="cuda")
    grad = torch.zeros(32, dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError, match="depth"):
        rs.adjoint_device(settings, [0], g.data_ptr(), grad.data_ptr())
    ok = build(scenes.cornell_box(8, 8, 1, max_depth=4))
    with pytest.raises(RuntimeError, match="twice"):
        ok.adjoint_device(settings, [0, 0], g.data_ptr(), grad.data_ptr())
