"""Image pins: the oracle's image restatement against rypath's own image code.

rypath's image shader headers (shaders/image_texture.h, shaders/image_lighting.h) and its host
image sources (src/image_texture.cpp, src/environment_sampling.cpp, src/rgb_spectrum.cpp,
src/light_sampling.cpp) are compiled from the checkout into oracle/_ref/libref_image.so by
oracle/ref.mk.  The oracle's texture lookups, RGB reconstruction, environment tables and
environment queries must equal them bit for bit on seeded inputs covering every texel format,
wrap mode and filter the oracle restates, the octahedral seams and poles, and degenerate
images; the library's own host-built environment tables (rp_cuda_environment_tables, no GPU)
must equal the oracle's.  CPU only.
"""

import ctypes as C

import numpy as np
import pytest

from rypath_b200 import abi, images, native
from tests.oracle_lib import oracle, reference_image


def need_ref():
    lib = reference_image()
    if lib is None:
        pytest.skip("oracle/_ref/libref_image.so not built (needs a rypath checkout: oracle/ref.mk)")
    return lib


def wire(imset):
    """The wire arrays of an ImageSet: textures, texture count, levels, level count, texels,
    word count, transfer, transfer count (numpy / ctypes objects kept alive by the caller)."""
    tex = (abi.ImageTexture * len(imset.textures))(*imset.textures)
    levels = np.array(imset.levels, np.uint32).reshape(-1, 3)
    texels = np.concatenate(imset.texels).astype(np.uint32)
    transfer = (np.concatenate(imset.transfer) if imset.transfer else np.zeros(1)).astype(np.float32)
    return tex, len(imset.textures), levels, levels.shape[0], texels, texels.size, transfer, 256 * len(imset.transfer)


def lookup(lib, prefix, w, index, q):
    out = np.zeros((q.shape[0], 4), np.float32)
    tex, nt, levels, nl, texels, nw, transfer, ntr = w
    extra = [images.ewa_weights().ctypes.data] if prefix == "or_" else []
    getattr(lib, prefix + "image_lookup")(C.cast(tex, C.c_void_p), nt, index, levels.ctypes.data, nl,
                                          texels.ctypes.data, nw, transfer.ctypes.data, ntr, q.ctypes.data,
                                          q.shape[0], out.ctypes.data, *extra)
    return out


def texture_set(rng):
    """Textures of every texel format, wrap and filter over seeded mip chains."""
    s = images.ImageSet()
    base = rng.uniform(0, 1, (16, 16, 3)).astype(np.float32)
    base[3, 5] = [1, 1, 1]
    base[7, 2] = [0.2, 0.2, 0.2]
    chain = images.box_pyramid(base)
    code = np.round(base * 255).astype(np.uint8)
    code_chain = [np.round(np.clip(c, 0, 1) * 255).astype(np.uint8) for c in chain]
    odd = rng.uniform(0, 2, (5, 7, 3)).astype(np.float32)  # one level, not a power of two
    for wrap in (abi.WRAP_REPEAT, abi.WRAP_CLAMP, abi.WRAP_BLACK):
        for filt in (abi.TEXTURE_POINT, abi.TEXTURE_BILINEAR, abi.TEXTURE_TRILINEAR):
            s.add_image([c.astype(np.float32) for c in chain], abi.TEXELS_FLOAT, wrap, filt,
                        uvscale=(1.5, 0.75), uvdelta=(0.1, -0.2))
            s.add_image([c.astype(np.float32) for c in chain], abi.TEXELS_HALF, wrap, filt)
            s.add_image(code_chain, abi.TEXELS_SRGB8, wrap, filt, uvscale=(2.0, 2.0))
        s.add_image([odd], abi.TEXELS_FLOAT, wrap, abi.TEXTURE_BILINEAR)
        s.add_image([code], abi.TEXELS_LINEAR8, wrap, abi.TEXTURE_POINT)
        # EWA over power-of-two chains, anisotropy caps from none to PBRT's largest
        for cap in (1.0, 8.0, 16.0):
            s.add_image([c.astype(np.float32) for c in chain], abi.TEXELS_FLOAT, wrap, abi.TEXTURE_EWA,
                        uvscale=(1.25, 3.0), uvdelta=(0.3, 0.1), max_anisotropy=cap)
        s.add_image(code_chain, abi.TEXELS_SRGB8, wrap, abi.TEXTURE_EWA, uvscale=(40.0, 70.0))
    return s


def lookup_queries(rng, n):
    q = np.zeros((n, 6), np.float32)
    q[:, 0:2] = rng.uniform(-2, 3, (n, 2))
    # texel-centre ties and exact edges
    q[: n // 8, 0:2] = (rng.integers(0, 16, (n // 8, 2)) + 0.5) / 16
    q[n // 8: n // 4, 0:2] = rng.choice([0.0, 1.0, -1.0, 2.0, 0.5], (n // 4 - n // 8, 2))
    scale = np.exp(rng.uniform(np.log(1e-5), np.log(2.0), (n, 1)))
    q[:, 2:6] = rng.normal(0, 1, (n, 4)) * scale
    q[n // 2: n // 2 + n // 16, 2:6] = 0
    return q


def test_image_lookup_matches_reference():
    """rypath_image::lookup / lookup_scalar (point, bilinear, trilinear, EWA) over float, half,
    sRGB and linear 8-bit texels with repeat, clamp and black wrap."""
    lib = need_ref()
    rng = np.random.default_rng(40)
    s = texture_set(rng)
    w = wire(s)
    q = lookup_queries(rng, 4000)
    for index in range(len(s.textures)):
        a = lookup(oracle(), "or_", w, index, q)
        b = lookup(lib, "ref_", w, index, q)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32), err_msg=f"texture {index}")


def test_host_image_lookup_agrees_with_shader():
    """rypath's host lookup (image_linear_rgb) and its shader lookup read the same texels the
    same way: the shader header, which the oracle restates, agrees with rypath's host code."""
    lib = need_ref()
    rng = np.random.default_rng(41)
    s = texture_set(rng)
    w = wire(s)
    tex, nt, levels, nl, texels, nw, transfer, ntr = w
    q = lookup_queries(rng, 2000)
    f = np.float32
    for index in range(len(s.textures)):
        t = s.textures[index]
        # the host lookup takes mapped coordinates in image row order (s, 1 - t)
        hq = np.empty_like(q)
        hq[:, 0] = (q[:, 0] * f(t.uscale)).astype(f) + f(t.udelta)
        hq[:, 1] = f(1) - ((q[:, 1] * f(t.vscale)).astype(f) + f(t.vdelta))
        hq[:, 2], hq[:, 3] = q[:, 2] * f(t.uscale), q[:, 3] * f(t.vscale)
        hq[:, 4], hq[:, 5] = q[:, 4] * f(t.uscale), q[:, 5] * f(t.vscale)
        host = np.zeros((q.shape[0], 4), np.float32)
        lib.ref_host_image_lookup(C.cast(tex, C.c_void_p), index, levels.ctypes.data, texels.ctypes.data, nw,
                                  transfer.ctypes.data, hq.ctypes.data, q.shape[0], host.ctypes.data)
        shader = lookup(lib, "ref_", w, index, q)
        valid = host[:, 3] == 1
        assert valid.mean() > 0.9
        close = np.isclose(host[valid, :3], shader[valid, :3], rtol=1e-5, atol=1e-6).all(axis=1)
        assert close.mean() >= 0.99, (index, close.mean())


def rgb_queries(rng, n):
    q = np.zeros((n, 4), np.float32)
    q[:, :3] = rng.uniform(0, 1, (n, 3))
    q[: n // 10, :3] = rng.uniform(-0.2, 1.3, (n // 10, 3))            # clamped inputs
    q[n // 10: n // 5, :3] = q[n // 10: n // 5, :1]                   # grey
    q[n // 5: n // 4, :3] = rng.choice([0.0, 1.0, 0.5], (n // 4 - n // 5, 3))
    q[n // 4: n // 4 + 50, :3] = rng.uniform(0, 1e-30, (50, 3))        # tiny channels
    q[:, 3] = rng.uniform(360, 830, n)
    q[: n // 20, 3] = rng.choice([360.0, 830.0, 555.0], n // 20)
    return q


def test_rgb_spectrum_matches_reference():
    """The bounded and unbounded sRGB reconstructions: oracle, rypath's shader and rypath's host
    code (for the inputs the host accepts) agree bit for bit."""
    lib = need_ref()
    rng = np.random.default_rng(42)
    q = rgb_queries(rng, 20000)
    table = images.rgb_table()
    a = np.zeros((q.shape[0], 2), np.float32)
    b = np.zeros_like(a)
    h = np.zeros_like(a)
    oracle().or_rgb_spectrum(table.ctypes.data, q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_rgb_spectrum(table.ctypes.data, q.ctypes.data, q.shape[0], b.ctypes.data)
    lib.ref_host_rgb_spectrum(q.ctypes.data, q.shape[0], h.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    accepted = np.all((q[:, :3] >= 0) & (q[:, :3] <= 1), axis=1)
    assert accepted.mean() > 0.8
    np.testing.assert_array_equal(h[accepted, 0].view(np.uint32), b[accepted, 0].view(np.uint32))
    unbounded = np.all(q[:, :3] >= 0, axis=1)
    np.testing.assert_array_equal(h[unbounded, 1].view(np.uint32), b[unbounded, 1].view(np.uint32))
    assert ((a[:, 0] > 0) & (a[:, 0] < 1)).mean() > 0.5


def environment_set(width, seed, fmt=abi.TEXELS_FLOAT):
    s = images.ImageSet()
    if width == 0:  # a black map: uniform tables
        rgb = np.zeros((4, 4, 3), np.float32)
    else:
        rgb = images.sky_image(width, seed=seed, fmt=fmt)
    s.environment_image = s.add_image(rgb, fmt, abi.WRAP_CLAMP)
    return s


def tables(lib, prefix, s):
    tex, nt, levels, nl, texels, nw, transfer, ntr = wire(s)
    width = levels[0, 0]
    cdf = np.zeros(2 * (width + 1) ** 2, np.float32)
    w, off, power = C.c_uint32(), C.c_uint32(), C.c_double()
    extra = [images.rgb_table().ctypes.data, images.d65().ctypes.data] if prefix == "or_" else []
    rc = getattr(lib, prefix + "environment_tables")(C.cast(tex, C.c_void_p), s.environment_image,
                                                     levels.ctypes.data, texels.ctypes.data, nw,
                                                     transfer.ctypes.data, *extra, cdf.ctypes.data, cdf.size,
                                                     C.byref(w), C.byref(off), C.byref(power))
    assert rc == 0
    return cdf, w.value, off.value, power.value


ENV_CASES = [(1, 1, abi.TEXELS_FLOAT), (2, 2, abi.TEXELS_FLOAT), (7, 3, abi.TEXELS_HALF), (32, 4, abi.TEXELS_FLOAT),
             (16, 5, abi.TEXELS_SRGB8), (0, 0, abi.TEXELS_FLOAT)]


@pytest.mark.parametrize("width,seed,fmt", ENV_CASES)
def test_environment_tables_match_reference(width, seed, fmt):
    """build_environment_sampling's full and compensated tables and light_image_power's mean
    power, from rypath's host sources, against the oracle's and the library's host build."""
    lib = need_ref()
    s = environment_set(width, seed, fmt)
    a = tables(oracle(), "or_", s)
    b = tables(lib, "ref_", s)
    np.testing.assert_array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
    assert a[1:3] == b[1:3]
    assert a[3] == b[3]
    # the library's scene-build tables (host code, no GPU)
    keep = []
    im = s.to_c(keep)
    cdf = np.zeros_like(a[0])
    w, off, power = C.c_uint32(), C.c_uint32(), C.c_double()
    native.check(native.lib().rp_cuda_environment_tables(C.byref(im), cdf.ctypes.data, cdf.size, C.byref(w),
                                                         C.byref(off), C.byref(power), None, 0))
    np.testing.assert_array_equal(cdf.view(np.uint32), a[0].view(np.uint32))
    assert (w.value, off.value) == a[1:3] and power.value == a[3]


def environment_queries(rng, n):
    q = np.zeros((n, 8), np.float32)
    d = rng.normal(size=(n, 3))
    d[: n // 10] = rng.choice([-1.0, 0.0, 1.0], (n // 10, 3))        # axes, poles and seams
    d[n // 10: n // 5, 2] = 0                                      # the equator
    d[n // 5: n // 4, 0] = 0
    d[np.all(d == 0, axis=1)] = [0, 0, 1]
    q[:, :3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 3] = rng.uniform(360, 830, n)
    q[:, 4:6] = rng.uniform(0, 1, (n, 2))
    q[: n // 20, 4:6] = rng.choice([0.0, 1.0, 0.0625, 0.5], (n // 20, 2))
    return q


@pytest.mark.parametrize("width,seed,fmt", ENV_CASES[:5])
def test_environment_queries_match_reference(width, seed, fmt):
    """environment_radiance, environment_pdf and sample_environment (shaders/image_lighting.h),
    compensated and full, through rypath's shader header against the oracle, with a rotated
    environment frame."""
    lib = need_ref()
    rng = np.random.default_rng(43 + width)
    s = environment_set(width, seed, fmt)
    cdf, w, off, _ = tables(oracle(), "or_", s)
    tex, nt, levels, nl, texels, nw, transfer, ntr = wire(s)
    c, sn = np.cos(0.7), np.sin(0.7)
    frame = np.array([c, 0, sn, 0, 1, 0, -sn, 0, c], np.float32)
    q = environment_queries(rng, 6000)
    out = {}
    for prefix, l in (("or_", oracle()), ("ref_", lib)):
        o = np.zeros((q.shape[0], 12), np.float32)
        getattr(l, prefix + "environment_queries")(
            C.cast(tex, C.c_void_p), nt, s.environment_image, levels.ctypes.data, nl, texels.ctypes.data, nw,
            transfer.ctypes.data, ntr, images.rgb_table().ctypes.data, images.d65().ctypes.data, cdf.ctypes.data,
            cdf.size, w, off, 1.25, frame.ctypes.data, q.ctypes.data, q.shape[0], o.ctypes.data)
        out[prefix] = o
    np.testing.assert_array_equal(out["or_"].view(np.uint32), out["ref_"].view(np.uint32))
    o = out["or_"]
    assert (o[:, 3] == 1).mean() > 0.99 and (o[:, 0] > 0).mean() > 0.5


def footprint_queries(rng, n):
    """Texture footprint inputs: camera-relative points on random planes seen along random
    rays, one-pixel ray offsets, texture tangents and camera frames (some degenerate)."""
    q = np.zeros((n, 48), np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.exp(rng.uniform(-2, 4, (n, 1)))
    q[:, 0:3] = d * t
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    q[:, 3:6] = nrm
    q[:, 6:9] = d
    eps = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), (n, 1)))
    q[:, 9:12] = d + eps * rng.normal(size=(n, 3))
    q[:, 12:15] = d + eps * rng.normal(size=(n, 3))
    q[:, 15] = rng.choice([0.125, 0.25, 1.0], n)
    for k in range(n):
        a = rng.normal(size=(3, 3))
        qm, _ = np.linalg.qr(a)
        q[k, 16:25] = qm.reshape(-1)
        q[k, 25:34] = qm.T.reshape(-1)
    q[:, 34:37] = rng.normal(0, 1e-3, (n, 3))
    q[:, 37:40] = rng.normal(0, 1e-3, (n, 3))
    q[:, 40:43] = rng.normal(size=(n, 3))
    q[:, 43:46] = rng.normal(size=(n, 3))
    q[: n // 20, 43:46] = q[: n // 20, 40:43] * 2   # parallel tangents: a singular system
    q[n // 20: n // 10, 3:6] = 0                   # a zero normal: no primary footprint
    return q


def test_texture_footprint_matches_reference():
    """rypath_texture_primary_dp / approximate_dp / uv_derivatives / direction
    (shaders/texture_footprint.h) against the oracle, bit for bit."""
    lib = need_ref()
    rng = np.random.default_rng(44)
    q = footprint_queries(rng, 5000)
    a = np.zeros((q.shape[0], 24), np.float32)
    b = np.zeros_like(a)
    oracle().or_texture_footprint(q.ctypes.data, q.shape[0], a.ctypes.data)
    lib.ref_texture_footprint(q.ctypes.data, q.shape[0], b.ctypes.data)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (a[:, 0] == 1).mean() > 0.8 and (a[:, 13] == 1).mean() > 0.99


@pytest.mark.parametrize("size", [(32, 32), (1920, 1080), (7, 3)])
def test_texture_camera_differentials_match_reference(size):
    """prepare_texture_camera_differentials (src/texture_footprint.cpp:199-232) of pinhole
    cameras of several poses and films against the oracle's restatement, bit for bit."""
    from rypath_b200 import scenes

    lib = need_ref()
    rng = np.random.default_rng(45)
    for k in range(6):
        origin = rng.normal(size=3) * 3
        target = origin + rng.normal(size=3)
        up = rng.normal(size=3)
        _, corner, dx, dy = scenes.pinhole_camera(tuple(origin), tuple(target), tuple(up), float(rng.uniform(20, 90)),
                                                  *size)
        c, x, y = (np.asarray(v, np.float32) for v in (corner, dx, dy))
        out = {}
        for prefix, l in (("or_", oracle()), ("ref_", lib)):
            o = np.zeros(6, np.float32)
            assert getattr(l, prefix + "texture_camera_differentials")(c.ctypes.data, x.ctypes.data, y.ctypes.data,
                                                                       size[0], size[1], o.ctypes.data) == 0
            out[prefix] = o
        np.testing.assert_array_equal(out["or_"].view(np.uint32), out["ref_"].view(np.uint32))


def test_library_texture_camera_differentials_match_oracle():
    """The library's host search for the texture camera's minimum differentials (scene renders
    use it per film size) equals the oracle's, bit for bit; the oracle's equals rypath's own."""
    from rypath_b200 import scenes

    rng = np.random.default_rng(46)
    for size in ((32, 32), (1920, 1080), (640, 480)):
        origin = rng.normal(size=3) * 3
        cam = scenes.pinhole_camera(tuple(origin), tuple(origin + rng.normal(size=3)), (0, 1, 0), 45.0, *size)
        c = abi.Camera()
        c.origin[:], c.corner[:], c.dx[:], c.dy[:] = cam[0], cam[1], cam[2], cam[3]
        mx, my = np.zeros(3, np.float32), np.zeros(3, np.float32)
        native.check(native.lib().rp_cuda_texture_camera_differentials(C.byref(c), size[0], size[1], mx.ctypes.data,
                                                                        my.ctypes.data, None, 0))
        o = np.zeros(6, np.float32)
        corner, dx, dy = (np.asarray(v, np.float32) for v in cam[1:])
        assert oracle().or_texture_camera_differentials(corner.ctypes.data, dx.ctypes.data, dy.ctypes.data, size[0],
                                                        size[1], o.ctypes.data) == 0
        np.testing.assert_array_equal(np.concatenate([mx, my]).view(np.uint32), o.view(np.uint32))
