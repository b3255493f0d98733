"""ctypes access to the oracle (the CPU checker) and to the reference-compiled pin library.

Test infrastructure only.  ``oracle()`` builds oracle/_build/liboracle.so with make when it
is missing; ``reference()`` returns None when oracle/_ref/libref.so was not built (it is built
from a rypath checkout by oracle/ref.mk).
"""

import ctypes as C
import os
import subprocess

from rypath_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libref.so")
REF_IMAGE = os.path.join(ROOT, "oracle", "_ref", "libref_image.so")
ROULETTE_KNOWN_ANSWERS = os.path.join(ROOT, "oracle", "_ref", "roulette_known_answers")
_oracle = None
_ref = None
_ref_image = None


def _image_args(lib, prefix):
    vp, u32, sz, fp = C.c_void_p, C.c_uint32, C.c_size_t, C.c_float
    getattr(lib, prefix + "image_lookup").argtypes = [vp, u32, u32, vp, u32, vp, u32, vp, u32, vp, u32, vp] + \
        ([vp] if prefix == "or_" else [])
    getattr(lib, prefix + "rgb_spectrum").argtypes = [vp, vp, u32, vp]
    getattr(lib, prefix + "environment_queries").argtypes = [vp, u32, u32, vp, u32, vp, u32, vp, u32, vp, vp, vp,
                                                               u32, u32, u32, fp, vp, vp, u32, vp]
    getattr(lib, prefix + "texture_footprint").argtypes = [vp, u32, vp]
    getattr(lib, prefix + "texture_camera_differentials").argtypes = [vp, vp, vp, u32, u32, vp]


def oracle():
    global _oracle
    if _oracle is None:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        lib = C.CDLL(ORACLE)
        vp, u32, sz = C.c_void_p, C.c_uint32, C.c_size_t
        lib.or_scene_create.restype = vp
        lib.or_scene_create.argtypes = [C.POINTER(abi.SceneDesc), C.c_char_p, sz]
        lib.or_scene_destroy.argtypes = [vp]
        _image_args(lib, "or_")
        lib.or_environment_tables.argtypes = [vp, u32, vp, vp, u32, vp, vp, vp, vp, sz, C.POINTER(u32),
                                              C.POINTER(u32), C.POINTER(C.c_double)]
        lib.or_scene_light_count.argtypes = [vp]
        lib.or_scene_light_count.restype = u32
        lib.or_sample.argtypes = [vp, C.POINTER(abi.Request), vp, sz, C.c_int]
        lib.or_probe_sobol.argtypes = [vp, vp, u32, vp]
        lib.or_probe_philox.argtypes = [vp, u32, vp]
        lib.or_probe_wavelengths.argtypes = [vp, u32, u32, vp]
        lib.or_probe_raygen.argtypes = [vp, C.POINTER(abi.Request), vp, vp, sz]
        lib.or_probe_bsdf.argtypes = [vp, u32, vp]
        lib.or_export_bvh.argtypes = [vp, vp, vp, vp, vp, sz]
        lib.or_trace_rays.argtypes = [vp, vp, u32, C.c_int, C.c_int, vp]
        lib.or_probe_advance.argtypes = [vp, u32, vp]
        lib.or_build_light_tables.argtypes = [vp, u32, vp, vp, vp, vp, vp]
        lib.or_probe_light_select.argtypes = [vp, vp, u32, vp]
        lib.or_film_add.argtypes = [vp, sz, vp, u32, vp]
        lib.or_film_add_clamped.argtypes = [vp, sz, vp, u32, C.c_double, C.c_double, vp]
        lib.or_sample_scalar.argtypes = [vp, C.POINTER(abi.Request), vp, sz, C.c_int]
        lib.or_probe_medium.argtypes = [vp, u32, vp]
        lib.or_scalar_film_add.argtypes = [vp, sz, vp, u32, vp, C.c_int]
        lib.or_adjoint.argtypes = [vp, C.POINTER(abi.FilmRequest), vp, u32, vp, vp, vp, C.c_int]
        lib.or_probe_qmc.argtypes = [vp, vp, u32, vp]
        lib.or_gaussian_filter.argtypes = [C.c_float, C.c_float, C.c_float, vp, sz, vp, vp, vp, u32, vp]
        lib.or_probe_hero.argtypes = [vp, u32, vp]
        lib.or_probe_roulette.argtypes = [vp, u32, vp]
        lib.or_probe_hero_weight.argtypes = [vp, u32, vp]
        _oracle = lib
    return _oracle


def reference():
    global _ref
    if _ref is None:
        if not os.path.exists(REF):
            return None
        lib = C.CDLL(REF)
        vp, u32, sz = C.c_void_p, C.c_uint32, C.c_size_t
        lib.ref_sobol_tables.restype = vp
        lib.ref_probe_sobol.argtypes = [vp, u32, vp]
        lib.ref_probe_philox.argtypes = [vp, u32, vp]
        lib.ref_probe_wavelengths.argtypes = [vp, u32, u32, vp]
        lib.ref_probe_advance.argtypes = [vp, u32, vp]
        lib.ref_probe_bsdf.argtypes = [vp, u32, vp]
        lib.ref_build_light_tables.argtypes = [vp, u32, vp, vp, vp, vp, vp]
        lib.ref_light_spectrum_power.argtypes = [vp]
        lib.ref_light_spectrum_power.restype = C.c_double
        lib.ref_outward.argtypes = [u32, C.c_int, C.POINTER(C.c_int)]
        lib.ref_outward.restype = u32
        lib.ref_set_cie.argtypes = [vp]
        lib.ref_film_add.argtypes = [vp, sz, u32, u32, vp]
        lib.ref_film_add_clamped.argtypes = [vp, sz, u32, u32, C.c_double, C.c_double, vp]
        lib.ref_probe_medium.argtypes = [vp, u32, vp]
        lib.ref_probe_qmc.argtypes = [vp, u32, vp]
        lib.ref_probe_hero.argtypes = [vp, u32, vp]
        lib.ref_probe_roulette.argtypes = [vp, u32, vp]
        lib.ref_probe_hero_weight.argtypes = [vp, u32, vp]
        _ref = lib
    return _ref


def reference_image():
    """rypath's image shader headers and host image sources (oracle/_ref/libref_image.so), or
    None when oracle/ref.mk has not built them."""
    global _ref_image
    if _ref_image is None:
        if not os.path.exists(REF_IMAGE):
            return None
        lib = C.CDLL(REF_IMAGE)
        vp, u32, sz = C.c_void_p, C.c_uint32, C.c_size_t
        _image_args(lib, "ref_")
        lib.ref_host_image_lookup.argtypes = [vp, u32, vp, vp, u32, vp, vp, u32, vp]
        lib.ref_host_rgb_spectrum.argtypes = [vp, u32, vp]
        lib.ref_environment_tables.argtypes = [vp, u32, vp, vp, u32, vp, vp, sz, C.POINTER(u32), C.POINTER(u32),
                                               C.POINTER(C.c_double)]
        _ref_image = lib
    return _ref_image


class OracleScene:
    def __init__(self, scene):
        self.scene = scene
        self.desc = scene.desc()
        diag = C.create_string_buffer(512)
        self.handle = oracle().or_scene_create(C.byref(self.desc), diag, 512)
        self.handle = C.c_void_p(self.handle) if self.handle else None
        if not self.handle:
            raise RuntimeError(diag.value.decode())

    def __del__(self):
        if getattr(self, "handle", None):
            oracle().or_scene_destroy(self.handle)
            self.handle = None

    def sample(self, request, threads=0):
        import numpy as np

        lanes = request.pixel_count * request.sample_count
        out = np.zeros(lanes, abi.packet_dtype())
        rc = oracle().or_sample(self.handle, C.byref(request), out.ctypes.data, lanes, threads)
        if rc < 0:
            raise RuntimeError("oracle sample rejected the request")
        return out

    def sample_scalar(self, request, threads=0):
        import numpy as np

        lanes = request.pixel_count * request.sample_count
        out = np.zeros(lanes, abi.scalar_dtype())
        rc = oracle().or_sample_scalar(self.handle, C.byref(request), out.ctypes.data, lanes, threads)
        if rc < 0:
            raise RuntimeError("oracle scalar sample rejected the request")
        return out


def request(width, height, spp=1, sample_begin=0, pixel_begin=0, pixel_count=None, seed=1,
            sampler=abi.SAMPLER_SOBOL, randomization=abi.RANDOMIZE_OWEN):
    r = abi.Request()
    r.width, r.height, r.seed = width, height, seed
    r.pixel_begin = pixel_begin
    r.pixel_count = width * height if pixel_count is None else pixel_count
    r.sample_begin, r.sample_count = sample_begin, spp
    r.emergency_limit, r.sampler_kind, r.randomization, r.boundary_limit = 1024, sampler, randomization, 4096
    r.total_samples = sample_begin + spp
    return r


def film_request(width, height, spp, seed=1, sample_begin=0, sampler=abi.SAMPLER_SOBOL,
                 randomization=abi.RANDOMIZE_OWEN, batch_size=None):
    return abi.FilmRequest(width=width, height=height, seed=seed, sample_begin=sample_begin, sample_count=spp,
                           batch_size=batch_size or spp, sampler_kind=sampler, randomization=randomization,
                           emergency_limit=1024)


def oracle_film_mean(scene, width, height, spp, seed=1, sampler=abi.SAMPLER_SOBOL, threads=0):
    """Film-mean XYZ (pixels x 3) of the oracle's hero render."""
    import numpy as np

    from rypath_b200 import renderer, scenes

    lanes = OracleScene(scene).sample(request(width, height, spp, seed=seed, sampler=sampler), threads)
    film = np.zeros(width * height, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, width * height, film.ctypes.data) == 0
    return renderer.film_mean(film)


def oracle_adjoint(scene, width, height, spp, materials, d_loss_d_xyz, seed=1, sampler=abi.SAMPLER_SOBOL, threads=0):
    import numpy as np

    from rypath_b200 import scenes

    o = OracleScene(scene)
    mats = np.ascontiguousarray(materials, np.uint32)
    params = sum(int(scene.materials[m].knot_count) for m in materials)
    grad = np.zeros(params, np.float64)
    g = np.ascontiguousarray(d_loss_d_xyz, np.float64)
    cie = np.ascontiguousarray(scenes.cie_xyz())
    fr = film_request(width, height, spp, seed=seed, sampler=sampler)
    rc = oracle().or_adjoint(o.handle, C.byref(fr), mats.ctypes.data, len(materials), g.ctypes.data, cie.ctypes.data,
                             grad.ctypes.data, threads)
    assert rc == 0, rc
    return grad


def oracle_film(scene, width, height, spp, seed=1, sampler=abi.SAMPLER_SOBOL, scalar=False, chunk=256, threads=0):
    """The oracle's FP64 film (rp_film_pixel rows) of samples [0, spp) of every pixel, rendered
    and reduced in chunks of `chunk` samples (canonical order: absolute sample, then pixel)."""
    import numpy as np

    from rypath_b200 import scenes

    o = OracleScene(scene)
    film = np.zeros(width * height, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    for begin in range(0, spp, chunk):
        count = min(chunk, spp - begin)
        r = request(width, height, count, sample_begin=begin, seed=seed, sampler=sampler)
        r.total_samples = spp
        if scalar:
            lanes = o.sample_scalar(r, threads)
            rc = oracle().or_scalar_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, width * height,
                                             film.ctypes.data, int(scene.model == abi.MODEL_DEMO))
        else:
            lanes = o.sample(r, threads)
            rc = oracle().or_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, width * height,
                                      film.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle film reduction rejected a lane")
    return film


def film_mean_variance(film):
    """Per-pixel mean XYZ and the variance of that mean (second moments over the count)."""
    import numpy as np

    n = film["count"].astype(np.float64)[:, None]
    m = (film["sum"] + film["correction"]) / n
    var = np.maximum(film["square"] / n - m * m, 0) / n
    return m, var
