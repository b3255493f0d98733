"""ctypes binding of librypath_cuda.so (include/rypath_cuda.h).

Loading fails loudly: there is no CPU fallback for the render path.  Build the library with
``python -m rypath_b200.build`` (or ``__graft_entry__.build()``).
"""

import ctypes as C
import os
import re

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librypath_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "rypath_cuda.h")
_lib = None


class NativeLibraryMissing(RuntimeError):
    pass


def header_entry_points():
    """Names of every entry point declared in include/rypath_cuda.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(rp_cuda_\w+)\s*\(", text)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryMissing(f"{LIB_PATH} is not built; run python -m rypath_b200.build")
    L = C.CDLL(LIB_PATH)
    vp, u32, sz, cp = C.c_void_p, C.c_uint32, C.c_size_t, C.c_char_p
    st = C.c_int
    sig = {
        "rp_cuda_device_info": (st, [C.c_int, C.POINTER(abi.DeviceInfo), cp, sz]),
        "rp_cuda_scene_create": (st, [C.POINTER(abi.SceneDesc), C.c_int, C.POINTER(vp), cp, sz]),
        "rp_cuda_scene_destroy": (None, [vp]),
        "rp_cuda_sample": (st, [vp, C.POINTER(abi.Request), vp, sz, cp, sz]),
        "rp_cuda_sample_device": (st, [vp, C.POINTER(abi.Request), vp, sz, vp, cp, sz]),
        "rp_cuda_sample_scalar": (st, [vp, C.POINTER(abi.Request), vp, sz, cp, sz]),
        "rp_cuda_render_film": (st, [vp, C.POINTER(abi.FilmRequest), vp, cp, sz]),
        "rp_cuda_render_film_device": (st, [vp, C.POINTER(abi.FilmRequest), vp, cp, sz]),
        "rp_cuda_set_cie": (st, [vp, vp]),
        "rp_cuda_last_timing": (st, [vp, C.POINTER(abi.Timing)]),
        "rp_cuda_set_counting": (st, [vp, C.c_int]),
        "rp_cuda_probe_sobol": (st, [vp, vp, u32, vp, cp, sz]),
        "rp_cuda_probe_philox": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_probe_wavelengths": (st, [vp, u32, u32, vp, cp, sz]),
        "rp_cuda_probe_raygen": (st, [vp, C.POINTER(abi.Request), vp, vp, sz, cp, sz]),
        "rp_cuda_probe_bsdf": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_probe_hero": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_probe_bilinear": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_probe_analytic": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_probe_texture_footprint": (st, [vp, u32, vp, cp, sz]),
        "rp_cuda_texture_camera_differentials": (st, [C.POINTER(abi.Camera), u32, u32, vp, vp, cp, sz]),
        "rp_cuda_probe_image_lookup": (st, [vp, u32, vp, u32, vp, cp, sz]),
        "rp_cuda_probe_rgb_spectrum": (st, [vp, vp, u32, vp, cp, sz]),
        "rp_cuda_probe_environment": (st, [vp, vp, u32, vp, cp, sz]),
        "rp_cuda_environment_tables": (st, [vp, vp, sz, C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_double), cp, sz]),
        "rp_cuda_scene_export_bvh": (st, [vp, vp, vp, vp, vp, sz, cp, sz]),
        "rp_cuda_scene_export_wide": (st, [vp, vp, sz, vp, sz, C.POINTER(u32), cp, sz]),
        "rp_cuda_trace_rays": (st, [vp, vp, u32, C.c_int, vp, cp, sz]),
        "rp_cuda_abi_size": (u32, [cp]),
        "rp_cuda_sample_device_static": (st, [vp, C.POINTER(abi.Request), vp, sz, vp, cp, sz]),
        "rp_cuda_build_light_tables": (C.c_int, [vp, u32, vp, vp, vp, vp, vp]),
        "rp_cuda_render_views_device": (st, [vp, C.POINTER(abi.View), u32, C.POINTER(abi.BatchRequest), vp,
                                             C.POINTER(abi.BatchConfig), cp, sz]),
        "rp_cuda_set_knot_values": (st, [vp, u32, u32, vp, cp, sz]),
        "rp_cuda_adjoint_device": (st, [vp, C.POINTER(abi.AdjointRequest), vp, vp, cp, sz]),
        "rp_cuda_tune_views": (st, [vp, C.POINTER(abi.View), u32, C.POINTER(abi.BatchRequest),
                                    C.POINTER(abi.BatchConfig), cp, sz]),
        "rp_cuda_frame_session_create": (st, [vp, C.POINTER(abi.FrameConfig), C.POINTER(vp), cp, sz]),
        "rp_cuda_frame_session_destroy": (None, [vp]),
        "rp_cuda_frame_submit": (st, [vp, C.POINTER(abi.FrameRequest), C.POINTER(u32), C.POINTER(C.c_int), cp, sz]),
        "rp_cuda_frame_poll": (st, [vp, u32, C.POINTER(abi.FrameInfo)]),
        "rp_cuda_frame_wait": (st, [vp, u32, C.POINTER(abi.FrameInfo)]),
        "rp_cuda_frame_capture": (st, [vp, u32, vp, sz, cp, sz]),
        "rp_cuda_frame_device_xyz": (st, [vp, u32, C.POINTER(vp)]),
        "rp_cuda_frame_release": (st, [vp, u32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status, diag=None, what="call"):
    if status != abi.RP_SUCCESS:
        msg = diag.value.decode(errors="replace") if diag is not None else ""
        raise RuntimeError(f"{what} failed: {abi.STATUS_NAMES.get(status, status)}: {msg}")
