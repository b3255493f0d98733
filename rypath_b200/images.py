"""Image inputs of a scene: image textures and the environment image, in rypath's wire layout.

A RenderScene carries its images already decoded into mip chains of texel words
(``ImagePyramid``, src/image_texture.hpp:66-77); ``ImageSet`` is that form for the seeded
synthetic scenes here.  Texel storage is float (4 words: r, g, b, a), half (2 words: r | g << 16,
b | a << 16) or 8-bit (1 word: r | g << 8 | b << 16 | a << 24 through a 256-entry transfer
table).  The sRGB reconstruction table and the dense D65 illuminant are rypath's
(``srgb_reconstruction_table``, ``pbrt_d65``; src/rgb_spectrum.hpp), extracted by
``data/make_tables.py``.
"""

from __future__ import annotations

import ctypes as C
import functools
import hashlib
import lzma
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import abi

DATA = Path(__file__).resolve().parent / "data"
SRGB_SHA256 = "6adffc41eefcf064b6524606cb8734941aa69ac962ac268fd9276f440cef61d5"
RGB_TABLE_FLOATS = 64 + 3 * 64 ** 3 * 3


@functools.lru_cache(maxsize=1)
def rgb_table() -> np.ndarray:
    """PBRT's sRGB-to-spectrum table (64 z nodes, then 3 x 64^3 x 3 coefficients), checked
    against the SHA-256 rypath pins."""
    planes = lzma.decompress((DATA / "srgb_spectrum.xz").read_bytes())
    n = len(planes) // 4
    blob = np.frombuffer(planes, np.uint8).reshape(4, n).T.copy().tobytes()
    if hashlib.sha256(blob).hexdigest() != SRGB_SHA256:
        raise RuntimeError("srgb_spectrum.xz does not restore the pinned sRGB table")
    table = np.frombuffer(blob, "<f4").copy()
    assert table.size == RGB_TABLE_FLOATS
    return table


@functools.lru_cache(maxsize=1)
def d65() -> np.ndarray:
    """PBRT's luminance-normalised D65 at 360..830 nm in 1 nm steps."""
    return np.frombuffer((DATA / "d65_dense.bin").read_bytes(), "<f4").copy()


@functools.lru_cache(maxsize=1)
def ewa_weights() -> np.ndarray:
    """PBRT's 128-entry EWA Gaussian filter table (rypath_ewa::weights, src/ewa_weights.h)."""
    return np.frombuffer((DATA / "ewa_weights.bin").read_bytes(), "<f4").copy()


def srgb_transfer() -> np.ndarray:
    """8-bit sRGB code values to linear (IEC 61966-2-1), as 256 binary32."""
    c = np.arange(256, dtype=np.float64) / 255.0
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4).astype(np.float32)


def linear_transfer() -> np.ndarray:
    return (np.arange(256, dtype=np.float64) / 255.0).astype(np.float32)


def _texel_words(rgb: np.ndarray, fmt: int) -> np.ndarray:
    """Pack an (H, W, 3) image (float for float/half storage, uint8 code values otherwise)."""
    h, w, _ = rgb.shape
    if fmt == abi.TEXELS_FLOAT:
        rgba = np.concatenate([rgb.astype(np.float32), np.ones((h, w, 1), np.float32)], axis=2)
        return rgba.reshape(-1).view(np.uint32).copy()
    if fmt == abi.TEXELS_HALF:
        hbits = np.concatenate([rgb.astype(np.float16), np.ones((h, w, 1), np.float16)], axis=2).view(np.uint16)
        hbits = hbits.reshape(-1, 4).astype(np.uint32)
        return np.stack([hbits[:, 0] | (hbits[:, 1] << 16), hbits[:, 2] | (hbits[:, 3] << 16)], axis=1).reshape(-1)
    code = np.asarray(rgb, np.uint8).reshape(-1, 3).astype(np.uint32)
    return code[:, 0] | (code[:, 1] << 8) | (code[:, 2] << 16) | (np.uint32(255) << 24)


def box_pyramid(rgb: np.ndarray) -> list:
    """Mip chain of a power-of-two image by 2x2 box averaging (float), down to 1x1."""
    levels = [np.asarray(rgb, np.float64)]
    while levels[-1].shape[0] > 1 or levels[-1].shape[1] > 1:
        a = levels[-1]
        h, w = max(1, a.shape[0] // 2), max(1, a.shape[1] // 2)
        a = a[: 2 * h if a.shape[0] > 1 else 1, : 2 * w if a.shape[1] > 1 else 1]
        if a.shape[0] > 1:
            a = 0.5 * (a[0::2] + a[1::2])
        if a.shape[1] > 1:
            a = 0.5 * (a[:, 0::2] + a[:, 1::2])
        levels.append(a)
    return levels


@dataclass
class ImageSet:
    textures: list = field(default_factory=list)   # abi.ImageTexture
    levels: list = field(default_factory=list)     # (width, height, offset)
    texels: list = field(default_factory=list)     # uint32 arrays
    words: int = 0
    transfer: list = field(default_factory=list)   # 256-float tables
    environment_image: int = abi.RP_NONE
    environment_scale: float = 1.0
    environment_from_world: tuple = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    uvs: np.ndarray | None = None                  # (N, 2) f32
    instance_uv_begin: list | None = None
    frames: np.ndarray | None = None               # (M, 6) f32
    instance_frame_begin: list | None = None
    world_from_camera: tuple = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    camera_from_world: tuple = (1, 0, 0, 0, 1, 0, 0, 0, 1)

    def add_image(self, chain, fmt=abi.TEXELS_FLOAT, wrap=abi.WRAP_REPEAT, filt=abi.TEXTURE_BILINEAR,
                  scale=1.0, invert=False, uvscale=(1.0, 1.0), uvdelta=(0.0, 0.0), max_anisotropy=8.0,
                  transfer=None) -> int:
        """Append a texture over the given mip chain ((H, W, 3) arrays, finest first); returns
        its index."""
        if isinstance(chain, np.ndarray):
            chain = [chain]
        t = abi.ImageTexture()
        t.level_begin, t.level_count = len(self.levels), len(chain)
        for level in chain:
            h, w = level.shape[:2]
            words = _texel_words(level, fmt)
            self.levels.append((w, h, self.words))
            self.texels.append(words)
            self.words += int(words.size)
        t.wrap, t.texel_format, t.filter = wrap, fmt, filt
        t.uscale, t.vscale = uvscale
        t.udelta, t.vdelta = uvdelta
        t.scale, t.invert, t.max_anisotropy = scale, int(invert), max_anisotropy
        t.channels = 3
        t.transfer_offset = 0
        if fmt in (abi.TEXELS_SRGB8, abi.TEXELS_LINEAR8):
            table = transfer if transfer is not None else (srgb_transfer() if fmt == abi.TEXELS_SRGB8
                                                           else linear_transfer())
            t.transfer_offset = 256 * len(self.transfer)
            self.transfer.append(np.asarray(table, np.float32))
        t.gltf, t.wrap_t, t.min_filter, t.mag_filter = 0, 10497, 9987, 9729
        self.textures.append(t)
        return len(self.textures) - 1

    def to_c(self, keep: list) -> abi.Images:
        def arr(a, ctype):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        im = abi.Images()
        tex = (abi.ImageTexture * max(1, len(self.textures)))(*self.textures)
        keep.append(tex)
        im.texture_count, im.textures = len(self.textures), C.cast(tex, C.POINTER(abi.ImageTexture))
        lv = (abi.TextureLevel * max(1, len(self.levels)))()
        for i, (w, h, off) in enumerate(self.levels):
            lv[i].width, lv[i].height, lv[i].offset = w, h, off
        keep.append(lv)
        im.level_count, im.levels = len(self.levels), C.cast(lv, C.POINTER(abi.TextureLevel))
        words = np.concatenate(self.texels).astype(np.uint32) if self.texels else np.zeros(1, np.uint32)
        im.texel_word_count, im.texels = self.words, arr(words, C.c_uint32)
        tr = np.concatenate(self.transfer).astype(np.float32) if self.transfer else np.zeros(1, np.float32)
        im.transfer_count, im.transfer = 256 * len(self.transfer), arr(tr, C.c_float)
        im.rgb_table = arr(rgb_table(), C.c_float)
        im.illuminant = arr(d65(), C.c_float)
        im.environment_image = self.environment_image
        im.environment_scale = self.environment_scale
        im.environment_from_world[:] = list(self.environment_from_world)
        if self.uvs is not None:
            im.uv_count, im.uvs = int(self.uvs.shape[0]), arr(np.asarray(self.uvs, np.float32), C.c_float)
        if self.instance_uv_begin is not None:
            im.instance_uv_begin = arr(np.asarray(self.instance_uv_begin, np.uint32), C.c_uint32)
        if self.frames is not None:
            im.frame_count, im.frames = int(self.frames.shape[0]), arr(np.asarray(self.frames, np.float32), C.c_float)
        if self.instance_frame_begin is not None:
            im.instance_frame_begin = arr(np.asarray(self.instance_frame_begin, np.uint32), C.c_uint32)
        im.world_from_camera[:] = list(self.world_from_camera)
        im.camera_from_world[:] = list(self.camera_from_world)
        im.ewa_weights = arr(ewa_weights(), C.c_float)
        return im


def sky_image(width=64, seed=1, sun=(0.3, 0.5, 0.81), sun_radiance=40.0, fmt=abi.TEXELS_FLOAT) -> np.ndarray:
    """A seeded equal-area octahedral sky: a blue-to-white gradient over +z, a warm ground below,
    a small bright sun and low-amplitude noise, as linear RGB of shape (width, width, 3) in the
    octahedral square's row order (row y, column x)."""
    rng = np.random.default_rng(seed)
    u = (np.arange(width) + 0.5) / width
    uu, vv = np.meshgrid(u, u)
    su, sv = 2 * uu - 1, 2 * vv - 1
    qu, qv = np.abs(su), np.abs(sv)
    diagonal = 1 - (qu + qv)
    radius = 1 - np.abs(diagonal)
    phi = np.where(radius == 0, 1.0, (qv - qu) / np.where(radius == 0, 1, radius) + 1) * (np.pi / 4)
    z = np.copysign(1 - radius ** 2, diagonal)
    radial = radius * np.sqrt(np.maximum(0, 2 - radius ** 2))
    x, y = np.copysign(np.cos(phi), su) * radial, np.copysign(np.sin(phi), sv) * radial
    up = np.clip(z, 0, 1)[..., None]
    sky = (1 - up) * np.array([1.0, 0.95, 0.9]) + up * np.array([0.25, 0.45, 1.0])
    ground = np.array([0.35, 0.25, 0.15])
    rgb = np.where((z >= 0)[..., None], sky, ground * (0.6 + 0.4 * (1 + z))[..., None])
    s = np.asarray(sun, np.float64)
    s = s / np.linalg.norm(s)
    cosang = x * s[0] + y * s[1] + z * s[2]
    rgb = rgb + (cosang > 0.995)[..., None] * sun_radiance * np.array([1.0, 0.85, 0.6])
    rgb = rgb * (1 + 0.05 * rng.standard_normal((width, width, 1)))
    rgb = np.maximum(rgb, 0)
    if fmt in (abi.TEXELS_SRGB8, abi.TEXELS_LINEAR8):
        return np.clip(np.round(rgb / rgb.max() * 255), 0, 255).astype(np.uint8)
    return rgb.astype(np.float32)
