"""ctypes mirror of include/rypath_cuda.h (the C ABI of the CUDA backend).

The structures below must match the C declarations byte for byte; tests/test_abi.py checks
their sizes against the values the library itself reports.
"""

import ctypes as C

RP_ABI_VERSION = 3
RP_NONE = 0xFFFFFFFF
RP_SPECTRUM_BINS = 471
RP_SOBOL_TABLE_BYTES = 234208

RP_SUCCESS, RP_NOT_BUILT, RP_NO_DEVICE, RP_NO_RAY_TRACING, RP_FAILURE, RP_INVALID_ARGUMENT = range(6)
STATUS_NAMES = {0: "success", 1: "not_built", 2: "no_device", 3: "no_ray_tracing", 4: "failure",
                5: "invalid_argument"}

SAMPLE_SUCCESS, EMERGENCY_DEPTH, INVALID_ARITHMETIC, INVALID_HIT, BOUNDARY_EXHAUSTION = range(5)

SAMPLER_INDEPENDENT, SAMPLER_SOBOL, SAMPLER_HALTON, SAMPLER_ZSOBOL = 0, 1, 2, 3
RANDOMIZE_NONE, RANDOMIZE_PERMUTEDIGITS, RANDOMIZE_FASTOWEN, RANDOMIZE_OWEN = range(4)
FILTER_BOX, FILTER_TRIANGLE, FILTER_GAUSSIAN = 0, 1, 2
DIFFUSE, CONDUCTOR, DIELECTRIC = 0, 1, 2
MODEL_PBRT, MODEL_DEMO = 0, 1
INTERFACE = 10  # null interface: medium change (scalar transport), pass-through (hero transport)
MIX = 9  # stochastic mix of two materials
REFLECTANCE_KNOTS, REFLECTANCE_CONSTANT, REFLECTANCE_RGB, REFLECTANCE_IMAGE, REFLECTANCE_BLACKBODY = 0, 1, 2, 3, 4
WRAP_REPEAT, WRAP_CLAMP, WRAP_BLACK = 0, 1, 2
TEXTURE_BILINEAR, TEXTURE_TRILINEAR, TEXTURE_POINT, TEXTURE_EWA = 0, 1, 2, 3
TEXELS_SRGB8, TEXELS_LINEAR8, TEXELS_HALF, TEXELS_FLOAT = 0, 1, 2, 3
POINT_LIGHT, SPOT_LIGHT = 0, 1
LIGHTS_BVH, LIGHTS_POWER, LIGHTS_UNIFORM = 0, 1, 2
TRANSPORT_SCALAR, TRANSPORT_HERO = 0, 2
HERO_UNIFORM, HERO_VISIBLE = 0, 1

u32, u64, i32, f32, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_float, C.c_double
P = C.POINTER


class Knot(C.Structure):
    _fields_ = [("wavelength", f32), ("value", f32)]


class Instance(C.Structure):
    _fields_ = [("matrix", f32 * 12), ("vertex_begin", u32), ("triangle_begin", u32),
                ("triangle_count", u32), ("material", u32), ("reverse_orientation", u32),
                ("emission", u32), ("normal_begin", u32), ("inside_medium", u32),
                ("outside_medium", u32), ("invisible_emitter", u32), ("patch_begin", u32),
                ("patch_count", u32), ("analytic_begin", u32), ("analytic_count", u32)]


PRIMITIVE_TRIANGLE, PRIMITIVE_PATCH, PRIMITIVE_ANALYTIC = 1, 2, 4
ANALYTIC_SPHERE, ANALYTIC_DISK, ANALYTIC_CYLINDER = 1, 2, 3


class Analytic(C.Structure):
    _fields_ = [("kind", u32), ("subtype", u32), ("radius", f32), ("z_min", f32), ("z_max", f32),
                ("phi_max", f32), ("inner_radius", f32), ("height", f32)]


class Material(C.Structure):
    _fields_ = [("scattering", u32), ("kind", u32), ("knot_begin", u32), ("knot_count", u32),
                ("scalar_value", f32), ("eta_begin", u32), ("eta_count", u32), ("k_begin", u32),
                ("k_count", u32), ("optical_extensions", u32), ("u_roughness", f32),
                ("v_roughness", f32), ("remap_roughness", u32), ("first_material", u32),
                ("second_material", u32), ("mix_amount", f32), ("image_texture", u32),
                ("coefficients", f32 * 3), ("reflectance", f32 * 8)]


class ImageTexture(C.Structure):
    _fields_ = [("level_begin", u32), ("level_count", u32), ("wrap", u32), ("texel_format", u32),
                ("uscale", f32), ("vscale", f32), ("udelta", f32), ("vdelta", f32), ("scale", f32),
                ("invert", u32), ("filter", u32), ("max_anisotropy", f32), ("transfer_offset", u32),
                ("channels", u32), ("gltf", u32), ("wrap_t", u32), ("min_filter", u32),
                ("mag_filter", u32)]


class TextureLevel(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("offset", u32)]


class Images(C.Structure):
    _fields_ = [
        ("texture_count", u32), ("textures", P(ImageTexture)),
        ("level_count", u32), ("levels", P(TextureLevel)),
        ("texel_word_count", u32), ("texels", P(u32)),
        ("transfer_count", u32), ("transfer", P(f32)),
        ("rgb_table", P(f32)), ("illuminant", P(f32)),
        ("environment_image", u32), ("environment_scale", f32),
        ("environment_from_world", f32 * 9),
        ("uv_count", u32), ("uvs", P(f32)), ("instance_uv_begin", P(u32)),
        ("frame_count", u32), ("frames", P(f32)), ("instance_frame_begin", P(u32)),
        ("world_from_camera", f32 * 9), ("camera_from_world", f32 * 9),
        ("ewa_weights", P(f32)),
    ]


class AreaEmission(C.Structure):
    _fields_ = [("radiance", f32 * RP_SPECTRUM_BINS), ("two_sided", u32)]


class PositionalLight(C.Structure):
    _fields_ = [("position", f32 * 3), ("intensity", f32 * RP_SPECTRUM_BINS), ("kind", u32),
                ("light_from_world", f32 * 9), ("cos_falloff_start", f32),
                ("cos_falloff_end", f32)]


class Medium(C.Structure):
    _fields_ = [("sigma_a", f32 * RP_SPECTRUM_BINS), ("sigma_s", f32 * RP_SPECTRUM_BINS),
                ("emission", f32 * RP_SPECTRUM_BINS), ("g", f32)]


class Camera(C.Structure):
    _fields_ = [("origin", f32 * 3), ("corner", f32 * 3), ("dx", f32 * 3), ("dy", f32 * 3)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("abi_version", u32),
        ("vertex_count", u32), ("positions", P(f32)),
        ("normal_count", u32), ("normals", P(f32)),
        ("triangle_count", u32), ("triangles", P(u32)),
        ("instance_count", u32), ("instances", P(Instance)),
        ("material_count", u32), ("materials", P(Material)),
        ("knot_count", u32), ("knots", P(Knot)),
        ("emission_count", u32), ("emissions", P(AreaEmission)),
        ("positional_count", u32), ("positional", P(PositionalLight)),
        ("medium_count", u32), ("media", P(Medium)),
        ("camera_medium", u32),
        ("environment", P(f32)),
        ("camera", Camera),
        ("filter_kind", u32), ("filter_x_radius", f32), ("filter_y_radius", f32),
        ("max_depth", u32),
        ("light_sampler", u32),
        ("transport", u32),
        ("hero_wavelengths", u32),
        ("sobol_tables", C.c_void_p),
        ("lens_radius", f32), ("focal_distance", f32), ("lens_x", f32 * 3), ("lens_y", f32 * 3),
        ("filter_sigma", f32),
        ("images", P(Images)),
        ("model", u32), ("film_scale", f32),
        ("patch_count", u32), ("patches", P(u32)),
        ("analytic_count", u32), ("analytics", P(Analytic)),
    ]


class Request(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("seed", u64), ("material_seed", i32),
                ("pixel_begin", u32), ("pixel_count", u32), ("sample_begin", u64),
                ("sample_count", u32), ("emergency_limit", u32), ("sampler_kind", u32),
                ("randomization", u32), ("boundary_limit", u32), ("total_samples", u64)]


class PacketResult(C.Structure):
    _fields_ = [("status", u32), ("pixel", u32), ("sample_low", u32), ("sample_high", u32),
                ("splat_count", u32), ("wavelengths", f32 * 4), ("wavelength_pdfs", f32 * 4),
                ("radiance", f32 * 4), ("filter_weight", f32), ("reserved", u32 * 2)]


class ScalarResult(C.Structure):
    _fields_ = [("status", u32), ("pixel", u32), ("sample_low", u32), ("sample_high", u32),
                ("wavelength", f32), ("radiance", f32), ("scatterings", u32),
                ("random_words", u32 * 4)]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 128), ("device", C.c_int), ("sm_count", C.c_int),
                ("major", C.c_int), ("minor", C.c_int), ("total_memory", u64)]


class FilmPixel(C.Structure):
    _fields_ = [("sum", f64 * 3), ("correction", f64 * 3), ("weight_sum", f64),
                ("weight_correction", f64), ("square", f64 * 3), ("count", u64),
                ("compatibility_sum", f64 * 3), ("compatibility_correction", f64 * 3)]


class FilmRequest(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("seed", u64), ("sample_begin", u64),
                ("sample_count", u64), ("batch_size", u64), ("sampler_kind", u32),
                ("randomization", u32), ("emergency_limit", u32), ("total_samples", u64), ("flags", u32),
                ("exposure", C.c_double), ("max_component_value", C.c_double)]


FILM_FRESH = 1


class View(C.Structure):
    _fields_ = [("camera", Camera), ("width", u32), ("height", u32), ("sample_begin", u64),
                ("sample_count", u64), ("film_offset", u64)]


class BatchConfig(C.Structure):
    _fields_ = [("wave_lanes", u32), ("trace_block", u32), ("shade_block", u32), ("blocks_per_sm", u32),
                ("use_graph", u32), ("probe_ms_per_mlane", f32)]


class BatchRequest(C.Structure):
    _fields_ = [("seed", u64), ("sampler_kind", u32), ("randomization", u32), ("emergency_limit", u32),
                ("config", BatchConfig), ("exposure", C.c_double), ("max_component_value", C.c_double)]


class AdjointRequest(C.Structure):
    _fields_ = [("film", FilmRequest), ("material_count", u32), ("materials", P(u32))]


class Timing(C.Structure):
    _fields_ = [("total_ms", f64), ("trace_ms", f64), ("shadow_ms", f64), ("shade_ms", f64),
                ("other_ms", f64), ("closest_rays", u64), ("shadow_rays", u64),
                ("kernel_launches", u64), ("samples", u64), ("nodes_visited", u64),
                ("triangles_tested", u64), ("trace_launches", u64), ("shadow_launches", u64),
                ("shade_launches", u64), ("other_launches", u64), ("shadow_nodes_visited", u64),
                ("shadow_triangles_tested", u64), ("build_ms", f64), ("build_host_ms", f64),
                ("build_bvh_ms", f64), ("shade_family_ms", f64 * 4)]


# numpy dtypes with the same layouts, for bulk views of result buffers
def packet_dtype():
    import numpy as np

    return np.dtype([("status", "<u4"), ("pixel", "<u4"), ("sample_low", "<u4"),
                     ("sample_high", "<u4"), ("splat_count", "<u4"), ("wavelengths", "<f4", 4),
                     ("wavelength_pdfs", "<f4", 4), ("radiance", "<f4", 4),
                     ("filter_weight", "<f4"), ("reserved", "<u4", 2)])


def scalar_dtype():
    import numpy as np

    return np.dtype([("status", "<u4"), ("pixel", "<u4"), ("sample_low", "<u4"),
                     ("sample_high", "<u4"), ("wavelength", "<f4"), ("radiance", "<f4"),
                     ("scatterings", "<u4"), ("random_words", "<u4", 4)])


def film_dtype():
    import numpy as np

    return np.dtype([("sum", "<f8", 3), ("correction", "<f8", 3), ("weight_sum", "<f8"),
                     ("weight_correction", "<f8"), ("square", "<f8", 3), ("count", "<u8"),
                     ("compatibility_sum", "<f8", 3), ("compatibility_correction", "<f8", 3)])


FILM_PIXEL_BYTES = 144  # sizeof(rp_film_pixel)


class FrameConfig(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("seed", u64), ("sampler_kind", u32), ("randomization", u32),
                ("footprint_samples", u64)]


class FrameRequest(C.Structure):
    _fields_ = [("sample_index", u64), ("epoch", u64), ("camera", C.POINTER(Camera))]


class FrameInfo(C.Structure):
    _fields_ = [("status", u32), ("width", u32), ("height", u32), ("sample_index", u64), ("epoch", u64),
                ("gpu_ms", f64), ("completed_samples", u64), ("failed_pixels", u32)]


FRAME_PENDING, FRAME_COMPLETE, FRAME_FAILED = 0, 1, 2

EXPECTED_SIZES = {
    "rp_instance": (Instance, 104), "rp_analytic": (Analytic, 32), "rp_material": (Material, 112), "rp_knot": (Knot, 8),
    "rp_area_emission": (AreaEmission, 1888), "rp_positional_light": (PositionalLight, 1948),
    "rp_medium": (Medium, 5656), "rp_camera": (Camera, 48), "rp_request": (Request, 64),
    "rp_packet_result": (PacketResult, 80), "rp_scalar_result": (ScalarResult, 44),
    "rp_film_pixel": (FilmPixel, 144), "rp_film_request": (FilmRequest, 88),
    "rp_view": (View, 80), "rp_batch_config": (BatchConfig, 24), "rp_batch_request": (BatchRequest, 64),
    "rp_adjoint_request": (AdjointRequest, 104),
    "rp_image_texture": (ImageTexture, 72), "rp_texture_level": (TextureLevel, 12),
    "rp_images": (Images, 248),
    "rp_frame_config": (FrameConfig, 32), "rp_frame_request": (FrameRequest, 24), "rp_frame_info": (FrameInfo, 56),
}
