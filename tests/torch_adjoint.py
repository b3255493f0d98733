"""A thin torch.autograd.Function over the forward film render and the path-replay adjoint
(rp_cuda_render_film_device / rp_cuda_adjoint_device).  Test infrastructure only: the
differentiable renderer itself is the C ABI; this wrapper lets tests drive it with torch
losses and optimisers.
"""

import numpy as np
import torch

from rypath_b200 import abi


def film_mean_device(film_bytes, pixels):
    """Film-mean XYZ (pixels x 3, float64) of a device rp_film_pixel buffer."""
    f = film_bytes.view(torch.float64).reshape(pixels, abi.FILM_PIXEL_BYTES // 8)
    return (f[:, 0:3] + f[:, 3:6]) / (f[:, 6:7] + f[:, 7:8])


class SpectralFilm(torch.autograd.Function):
    """theta (the knot values of `materials`, concatenated) -> film-mean XYZ of the render."""

    @staticmethod
    def forward(ctx, theta, rs, scene, settings, materials):
        values = theta.detach().cpu().numpy().astype(np.float32)
        offset = 0
        for m in materials:
            mat = scene.materials[m]
            rs.set_knot_values(int(mat.knot_begin), values[offset:offset + mat.knot_count])
            offset += mat.knot_count
        pixels = settings.width * settings.height
        film = torch.zeros(pixels * abi.FILM_PIXEL_BYTES, dtype=torch.uint8, device="cuda")
        rs.render_film_device(settings, film.data_ptr())
        ctx.rs, ctx.settings, ctx.materials, ctx.params = rs, settings, list(materials), offset
        ctx.theta_device, ctx.theta_dtype = theta.device, theta.dtype
        return film_mean_device(film, pixels)

    @staticmethod
    def backward(ctx, grad_xyz):
        g = grad_xyz.detach().to(device="cuda", dtype=torch.float64).contiguous()
        grad = torch.zeros(ctx.params, dtype=torch.float32, device="cuda")
        ctx.rs.adjoint_device(ctx.settings, ctx.materials, g.data_ptr(), grad.data_ptr())
        torch.cuda.synchronize()
        return grad.to(device=ctx.theta_device, dtype=ctx.theta_dtype), None, None, None, None


def knot_parameters(scene, materials):
    return np.concatenate([scene.knots[scene.materials[m].knot_begin:
                                       scene.materials[m].knot_begin + scene.materials[m].knot_count, 1]
                           for m in materials]).astype(np.float32)
