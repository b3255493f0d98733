"""Host-side mirror of rypath's renderer interface over the C ABI.

Names and meanings follow the reference (src/metal_render.hpp:14-95, src/render_driver.hpp):

* ``build_renderer(scene)`` ~ ``build_metal_renderer(RenderScene, ...)`` -> ``RenderBuildResult``
  with ``status``, ``diagnostic`` and ``scene`` (a ``CudaRenderScene``).
* ``CudaRenderScene.sample(request)`` ~ ``MetalRenderScene::sample(RenderRequest)`` ->
  ``RenderSamplesResult`` whose ``packet_samples`` are the 80-byte packet results in lane order;
  ``sample_scalar(request)`` the same for scalar-transport (media) scenes, whose ``samples``
  are RenderSample rows (src/metal_render.mm:2136-2166).
* ``render_progressive(scene, settings)`` ~ the driver loop of src/render_driver.cpp:166-275 with
  the packet film reduction performed on the device.

Errors follow the reference: failures are statuses plus diagnostics, never exceptions from
the native layer (a Python exception is raised only for misuse of this binding).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi, native, scenes


@dataclass
class RenderRequest:
    width: int
    height: int
    seed: int = 1
    material_seed: int = 0
    pixel_begin: int = 0
    pixel_count: int = 0
    sample_begin: int = 0
    sample_count: int = 1
    emergency_limit: int = 1024
    sampler: int = abi.SAMPLER_SOBOL
    randomization: int = abi.RANDOMIZE_OWEN
    boundary_limit: int = 4096
    total_samples: int = 0  # the render's sample budget (ZSobol); 0: sample_begin + sample_count

    def to_c(self) -> abi.Request:
        r = abi.Request()
        r.width, r.height, r.seed, r.material_seed = self.width, self.height, self.seed, self.material_seed
        r.pixel_begin = self.pixel_begin
        r.pixel_count = self.pixel_count or self.width * self.height
        r.sample_begin, r.sample_count = self.sample_begin, self.sample_count
        r.emergency_limit, r.sampler_kind = self.emergency_limit, self.sampler
        r.randomization, r.boundary_limit = self.randomization, self.boundary_limit
        r.total_samples = self.total_samples or (self.sample_begin + self.sample_count)
        return r


@dataclass
class RenderSamplesResult:
    status: int = abi.RP_FAILURE
    diagnostic: str = ""
    packet_samples: np.ndarray | None = None
    samples: np.ndarray | None = None  # scalar transport: RenderSample rows (abi.scalar_dtype)


@dataclass
class RenderBuildResult:
    status: int = abi.RP_FAILURE
    diagnostic: str = ""
    scene: "CudaRenderScene | None" = None
    device: abi.DeviceInfo | None = None


@dataclass
class RenderSettings:
    width: int = 256
    height: int = 192
    samples: int = 128
    batch_size: int = 8
    seed: int = 1
    sampler: int = abi.SAMPLER_SOBOL
    randomization: int = abi.RANDOMIZE_OWEN
    exposure: float = 1.0             # Film::exposure (compatibility planes only)
    max_component_value: float = 0.0  # Film::max_component_value; 0 or inf: no clamp
    emergency_limit: int = 1024       # render_emergency_limit (src/render.hpp:22-26)


@dataclass
class View:
    """One camera view of a batch (rp_view): camera as (origin, corner, dx, dy), film size,
    absolute sample range and the first film pixel of the view in the batch film."""
    camera: tuple
    width: int
    height: int
    sample_begin: int = 0
    sample_count: int = 1
    film_offset: int = 0

    def to_c(self) -> abi.View:
        v = abi.View()
        o, corner, dx, dy = self.camera
        v.camera.origin[:] = list(o)
        v.camera.corner[:] = list(corner)
        v.camera.dx[:] = list(dx)
        v.camera.dy[:] = list(dy)
        v.width, v.height = self.width, self.height
        v.sample_begin, v.sample_count, v.film_offset = self.sample_begin, self.sample_count, self.film_offset
        return v


@dataclass
class BatchRequest:
    seed: int = 1
    sampler: int = abi.SAMPLER_SOBOL
    randomization: int = abi.RANDOMIZE_OWEN
    emergency_limit: int = 1024
    wave_lanes: int = 0     # 0: tuned
    trace_block: int = 0    # 0: tuned
    shade_block: int = 0    # 0: tuned
    blocks_per_sm: int = 0  # 0: tuned
    use_graph: int = 1      # 1: CUDA graph replay per wave, 2: direct launches
    exposure: float = 1.0
    max_component_value: float = 0.0  # 0 or inf: no film clamp

    def to_c(self) -> abi.BatchRequest:
        r = abi.BatchRequest()
        r.seed, r.sampler_kind, r.randomization, r.emergency_limit = (self.seed, self.sampler, self.randomization,
                                                                      self.emergency_limit)
        c = r.config
        c.wave_lanes, c.trace_block, c.shade_block = self.wave_lanes, self.trace_block, self.shade_block
        c.blocks_per_sm, c.use_graph = self.blocks_per_sm, self.use_graph
        r.exposure, r.max_component_value = self.exposure, self.max_component_value
        return r


def pack_views(views):
    """Assign consecutive film offsets; returns the total film pixels."""
    offset = 0
    for v in views:
        v.film_offset = offset
        offset += v.width * v.height
    return offset


class CudaRenderScene:
    """A scene resident on one GPU.  Synchronous calls need external serialisation."""

    def __init__(self, handle):
        self._handle = C.c_void_p(handle)
        self._cie_set = False

    def close(self):
        if self._handle and native is not None:
            native.lib().rp_cuda_scene_destroy(self._handle)
            self._handle = C.c_void_p()

    __del__ = close

    @property
    def handle(self):
        return self._handle

    def sample(self, request: RenderRequest) -> RenderSamplesResult:
        q = request.to_c()
        lanes = q.pixel_count * q.sample_count
        out = np.zeros(lanes, abi.packet_dtype())
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_sample(self._handle, C.byref(q), out.ctypes.data, lanes, diag, 512)
        return RenderSamplesResult(st, diag.value.decode(errors="replace"), out)

    def sample_scalar(self, request: RenderRequest) -> RenderSamplesResult:
        """Scalar-transport lanes (``samples``): scenes built with ``transport=TRANSPORT_SCALAR``."""
        q = request.to_c()
        lanes = q.pixel_count * q.sample_count
        out = np.zeros(lanes, abi.scalar_dtype())
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_sample_scalar(self._handle, C.byref(q), out.ctypes.data, lanes, diag, 512)
        return RenderSamplesResult(st, diag.value.decode(errors="replace"), None, out)

    def sample_device(self, request: RenderRequest, device_ptr: int, capacity: int, stream: int = 0) -> int:
        q = request.to_c()
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_sample_device(self._handle, C.byref(q), C.c_void_p(device_ptr), capacity,
                                                C.c_void_p(stream), diag, 512)
        native.check(st, diag, "rp_cuda_sample_device")
        return st

    def _ensure_cie(self):
        if not self._cie_set:
            cie = np.ascontiguousarray(scenes.cie_xyz())
            native.check(native.lib().rp_cuda_set_cie(self._handle, cie.ctypes.data), None, "rp_cuda_set_cie")
            self._cie_set = True

    def render_film(self, settings: RenderSettings, film: np.ndarray | None = None, sample_begin: int = 0,
                    fresh: bool = False):
        """Progressive render into a host film (structured rp_film_pixel array).

        The render accumulates onto ``film``'s committed state; with ``fresh`` (or no film given)
        it starts from an empty film without reading or uploading ``film``."""
        self._ensure_cie()
        pixels = settings.width * settings.height
        if film is None:
            film = np.empty(pixels, abi.film_dtype())
            fresh = True
        r = abi.FilmRequest(width=settings.width, height=settings.height, seed=settings.seed,
                            sample_begin=sample_begin, sample_count=settings.samples, batch_size=settings.batch_size,
                            sampler_kind=settings.sampler, randomization=settings.randomization,
                            emergency_limit=settings.emergency_limit,
                            flags=abi.FILM_FRESH if fresh else 0, exposure=settings.exposure,
                            max_component_value=settings.max_component_value)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_render_film(self._handle, C.byref(r), film.ctypes.data, diag, 512)
        return st, diag.value.decode(errors="replace"), film

    def render_film_device(self, settings: RenderSettings, device_film_ptr: int, sample_begin: int = 0,
                           fresh: bool = False, check: bool = True):
        """Progressive render into a device film (rp_film_pixel rows at ``device_film_ptr``), onto
        its committed state (``fresh``: from an empty film).  Returns (status, diagnostic); with
        ``check`` a failed call raises instead."""
        self._ensure_cie()
        r = abi.FilmRequest(width=settings.width, height=settings.height, seed=settings.seed,
                            sample_begin=sample_begin, sample_count=settings.samples, batch_size=settings.batch_size,
                            sampler_kind=settings.sampler, randomization=settings.randomization,
                            emergency_limit=settings.emergency_limit, flags=abi.FILM_FRESH if fresh else 0,
                            exposure=settings.exposure, max_component_value=settings.max_component_value)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_render_film_device(self._handle, C.byref(r), C.c_void_p(device_film_ptr), diag, 512)
        if check:
            native.check(st, diag, "rp_cuda_render_film_device")
        return st, diag.value.decode(errors="replace")

    def render_views_device(self, views, request: "BatchRequest", device_film_ptr: int) -> abi.BatchConfig:
        """All ``views`` (a list of ``View``) into one device film, sharing one wavefront.

        Returns the batch configuration that ran (the autotuner fills fields left at zero)."""
        self._ensure_cie()
        arr = (abi.View * len(views))(*[v.to_c() for v in views])
        used = abi.BatchConfig()
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_render_views_device(self._handle, arr, len(views), C.byref(request.to_c()),
                                                       C.c_void_p(device_film_ptr), C.byref(used), diag, 512)
        native.check(st, diag, "rp_cuda_render_views_device")
        return used

    def tune_views(self, views, request: "BatchRequest") -> abi.BatchConfig:
        self._ensure_cie()
        arr = (abi.View * len(views))(*[v.to_c() for v in views])
        chosen = abi.BatchConfig()
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_tune_views(self._handle, arr, len(views), C.byref(request.to_c()), C.byref(chosen),
                                              diag, 512)
        native.check(st, diag, "rp_cuda_tune_views")
        return chosen

    def set_knot_values(self, first: int, values):
        """Overwrite knot values [first, first + len(values)) of the scene's spectral knots."""
        v = np.ascontiguousarray(values, np.float32)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_set_knot_values(self._handle, first, v.size, v.ctypes.data, diag, 512)
        native.check(st, diag, "rp_cuda_set_knot_values")

    def adjoint_device(self, settings: RenderSettings, materials, d_loss_d_xyz_ptr: int, gradient_ptr: int,
                       sample_begin: int = 0):
        """Backward pass of ``render_film`` with these settings: d loss / d knot values of
        ``materials`` (device float gradient) from d loss / d film-mean XYZ (device doubles)."""
        self._ensure_cie()
        mats = np.ascontiguousarray(materials, np.uint32)
        r = abi.AdjointRequest()
        r.film = abi.FilmRequest(width=settings.width, height=settings.height, seed=settings.seed,
                                 sample_begin=sample_begin, sample_count=settings.samples,
                                 batch_size=settings.batch_size, sampler_kind=settings.sampler,
                                 randomization=settings.randomization, emergency_limit=1024)
        r.material_count = mats.size
        r.materials = mats.ctypes.data_as(C.POINTER(C.c_uint32))
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_adjoint_device(self._handle, C.byref(r), C.c_void_p(d_loss_d_xyz_ptr),
                                                  C.c_void_p(gradient_ptr), diag, 512)
        native.check(st, diag, "rp_cuda_adjoint_device")

    def timing(self) -> abi.Timing:
        t = abi.Timing()
        native.lib().rp_cuda_last_timing(self._handle, C.byref(t))
        return t

    def set_counting(self, enabled: bool):
        native.lib().rp_cuda_set_counting(self._handle, int(enabled))

    def export_bvh(self, n: int):
        nodes = np.zeros((max(n - 1, 1), 3), np.uint32)
        order = np.zeros(n, np.uint32)
        keys = np.zeros(n, np.uint64)
        bounds = np.zeros((2 * n - 1 if n else 1, 6), np.float32)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_scene_export_bvh(self._handle, nodes.ctypes.data, order.ctypes.data,
                                                    keys.ctypes.data, bounds.ctypes.data, n, diag, 512)
        native.check(st, diag, "rp_cuda_scene_export_bvh")
        return nodes, order, keys, bounds

    def export_wide(self, n: int):
        """The compressed 8-wide traversal tree: (80-byte node records as a uint8 array of shape
        (nodes, 80), wide leaves as float32 (n, 3, 4))."""
        count = C.c_uint32()
        diag = C.create_string_buffer(512)
        tris = np.zeros((max(n, 1), 3, 4), np.float32)
        st = native.lib().rp_cuda_scene_export_wide(self._handle, None, 0, tris.ctypes.data, n, C.byref(count), diag,
                                                     512)
        nodes = np.zeros((max(count.value, 1), 80), np.uint8)
        st = native.lib().rp_cuda_scene_export_wide(self._handle, nodes.ctypes.data, count.value, tris.ctypes.data, n,
                                                     C.byref(count), diag, 512)
        native.check(st, diag, "rp_cuda_scene_export_wide")
        return nodes[:count.value], tris[:n]

    def trace(self, rays: np.ndarray, any_hit: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 4), np.float32)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_trace_rays(self._handle, rays.ctypes.data, rays.shape[0], int(any_hit),
                                              hits.ctypes.data, diag, 512)
        native.check(st, diag, "rp_cuda_trace_rays")
        return hits

    def raygen(self, request: RenderRequest):
        q = request.to_c()
        lanes = q.pixel_count * q.sample_count
        words = np.zeros((lanes, 11), np.uint32)
        rays = np.zeros((lanes, 6), np.float32)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_probe_raygen(self._handle, C.byref(q), words.ctypes.data, rays.ctypes.data, lanes,
                                                diag, 512)
        native.check(st, diag, "rp_cuda_probe_raygen")
        return words, rays


@dataclass
class FrameConfig:
    """FrameConfig (src/frame_session.hpp:58-100): film size, sampler and its seed."""
    width: int
    height: int
    seed: int = 1
    sampler: int = abi.SAMPLER_SOBOL
    randomization: int = abi.RANDOMIZE_OWEN
    footprint_samples: int = 0  # the fixed budget ZSobol needs; 0: none

    def to_c(self) -> abi.FrameConfig:
        return abi.FrameConfig(self.width, self.height, self.seed, self.sampler, self.randomization,
                               self.footprint_samples)


class FrameSession:
    """FrameSession (src/frame_session.hpp:182-212) over the C ABI: each submitted frame renders
    one absolute sample of every pixel into raw XYZ on the device, asynchronously; two frame
    slots, each held by its frame until ``release``."""

    def __init__(self, scene: "CudaRenderScene", config: FrameConfig):
        scene._ensure_cie()
        self.scene = scene  # the scene outlives the session
        self.config = config
        handle = C.c_void_p()
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_frame_session_create(scene.handle, C.byref(config.to_c()), C.byref(handle), diag, 512)
        native.check(st, diag, "rp_cuda_frame_session_create")
        self._handle = handle

    def close(self):
        if getattr(self, "_handle", None) and self._handle.value and native is not None:
            native.lib().rp_cuda_frame_session_destroy(self._handle)
            self._handle = C.c_void_p()

    __del__ = close

    def submit(self, sample_index: int, epoch: int = 0, camera=None):
        """Returns (status, frame slot or None, busy, diagnostic); ``camera`` (origin, corner, dx, dy)
        replaces the session's camera from this frame on."""
        cam = None
        if camera is not None:
            cam = abi.Camera()
            o, corner, dx, dy = camera
            cam.origin[:], cam.corner[:], cam.dx[:], cam.dy[:] = list(o), list(corner), list(dx), list(dy)
        req = abi.FrameRequest(sample_index, epoch, C.pointer(cam) if cam is not None else None)
        frame, busy = C.c_uint32(), C.c_int()
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_frame_submit(self._handle, C.byref(req), C.byref(frame), C.byref(busy), diag, 512)
        return st, (frame.value if st == abi.RP_SUCCESS else None), bool(busy.value), diag.value.decode()

    def poll(self, frame: int) -> abi.FrameInfo:
        info = abi.FrameInfo()
        native.check(native.lib().rp_cuda_frame_poll(self._handle, frame, C.byref(info)), None, "rp_cuda_frame_poll")
        return info

    def wait(self, frame: int) -> abi.FrameInfo:
        info = abi.FrameInfo()
        native.check(native.lib().rp_cuda_frame_wait(self._handle, frame, C.byref(info)), None, "rp_cuda_frame_wait")
        return info

    def capture(self, frame: int):
        """(status, diagnostic, raw XYZ as float32 (height, width, 3))."""
        xyz = np.zeros((self.config.height, self.config.width, 3), np.float32)
        diag = C.create_string_buffer(512)
        st = native.lib().rp_cuda_frame_capture(self._handle, frame, xyz.ctypes.data, xyz.shape[0] * xyz.shape[1],
                                                diag, 512)
        return st, diag.value.decode(), xyz

    def device_xyz(self, frame: int) -> int:
        ptr = C.c_void_p()
        native.check(native.lib().rp_cuda_frame_device_xyz(self._handle, frame, C.byref(ptr)), None,
                     "rp_cuda_frame_device_xyz")
        return ptr.value

    def release(self, frame: int):
        native.check(native.lib().rp_cuda_frame_release(self._handle, frame), None, "rp_cuda_frame_release")


def build_renderer(scene: scenes.Scene, device: int = 0) -> RenderBuildResult:
    """build_metal_renderer (src/metal_render.hpp:84-95) for the CUDA backend."""
    L = native.lib()
    diag = C.create_string_buffer(1024)
    info = abi.DeviceInfo()
    st = L.rp_cuda_device_info(device, C.byref(info), diag, 1024)
    if st != abi.RP_SUCCESS:
        return RenderBuildResult(st, diag.value.decode(errors="replace"))
    desc = scene.desc()
    handle = C.c_void_p()
    st = L.rp_cuda_scene_create(C.byref(desc), device, C.byref(handle), diag, 1024)
    if st != abi.RP_SUCCESS:
        return RenderBuildResult(st, diag.value.decode(errors="replace"), None, info)
    return RenderBuildResult(st, "", CudaRenderScene(handle.value), info)


def film_mean(film: np.ndarray, compatibility: bool = False) -> np.ndarray:
    """Per-pixel XYZ mean, film_mean (src/packet_film.cpp:116-135) without splats; with
    ``compatibility``, of the clamped compatibility planes."""
    weight = film["weight_sum"] + film["weight_correction"]
    if compatibility:
        xyz = film["compatibility_sum"] + film["compatibility_correction"]
    else:
        xyz = film["sum"] + film["correction"]
    return np.where(weight[:, None] > 0, xyz / np.where(weight > 0, weight, 1)[:, None], 0.0)


def render_progressive(scene: scenes.Scene, settings: RenderSettings, device: int = 0,
                       film: np.ndarray | None = None, fresh: bool = False):
    """render_progressive (src/render_driver.cpp:287-316): build, then render every batch into
    ``film`` (a host rp_film_pixel array holding the committed state; ``fresh`` starts a new
    render without reading it)."""
    built = build_renderer(scene, device)
    if built.status != abi.RP_SUCCESS:
        return built.status, built.diagnostic, None
    st, diag, film = built.scene.render_film(settings, film, fresh=fresh)
    built.scene.close()
    return st, diag, film
