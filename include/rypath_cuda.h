/*
 * rypath_cuda.h -- C ABI of the B200 spectral path-tracing backend.
 *
 * This is the boundary that replaces rypath's Metal render adapter.  The reference
 * binds its renderer through C++ (`build_metal_renderer` / `MetalRenderScene::sample`,
 * src/metal_render.hpp:14-95) behind the progressive driver's sample-source seam
 * (`detail::RenderSampleSource`, src/render_driver.hpp:6-14).  Every entry point below is
 * what a C++ adapter in the reference's tree calls instead of Objective-C++/Metal.
 *
 * Conventions (the reference's, src/metal_render.hpp:47-52 and src/render_driver.cpp:280-283):
 *   - No exceptions cross the boundary: every call returns an rp_status and writes a
 *     NUL-terminated diagnostic into (diag, diag_capacity) when one is supplied.
 *   - A scene deep-copies everything it is given and retains no caller storage.
 *   - Synchronous operations on one scene require external serialisation.
 *   - Plain pointers and sizes only.  "host" pointers are CPU memory; "device" pointers
 *     are CUDA global memory on the scene's device.
 */
#ifndef RYPATH_CUDA_H
#define RYPATH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RP_ABI_VERSION 3u
#define RP_NONE 0xffffffffu
#define RP_SPECTRUM_BINS 471u /* 360..830 nm at 1 nm, src/render.hpp:29-36 */
#define RP_SOBOL_TABLE_BYTES 234208u /* sizeof(sobol::Tables), src/sobol_shared.h:42 */
#define RP_MAX_DEPTH 64u        /* packet_wire::max_depth, src/packet_wire.h:12 */
#define RP_MAX_POSITIONAL 64u   /* max_positional_lights, src/render.hpp:173 */

/* Build / call status; mirrors GeometryStatus (src/metal_geometry.hpp:16). */
typedef enum rp_status {
    RP_SUCCESS = 0,
    RP_NOT_BUILT = 1,
    RP_NO_DEVICE = 2,
    RP_NO_RAY_TRACING = 3,
    RP_FAILURE = 4,
    RP_INVALID_ARGUMENT = 5
} rp_status;

/* Per-lane sample status; render_wire status codes (src/render_wire.h:20-26). */
enum {
    RP_SAMPLE_SUCCESS = 0,
    RP_SAMPLE_EMERGENCY_DEPTH = 1,
    RP_SAMPLE_INVALID_ARITHMETIC = 2,
    RP_SAMPLE_INVALID_HIT = 3,
    RP_SAMPLE_BOUNDARY_EXHAUSTION = 4
};

/* Sampler kinds and Sobol randomisations (src/render_wire.h:40, src/sobol_shared.h:26-34). */
enum { RP_SAMPLER_INDEPENDENT = 0, RP_SAMPLER_SOBOL = 1, RP_SAMPLER_HALTON = 2, RP_SAMPLER_ZSOBOL = 3 };
enum { RP_RANDOMIZE_NONE = 0, RP_RANDOMIZE_PERMUTEDIGITS = 1, RP_RANDOMIZE_FASTOWEN = 2,
       RP_RANDOMIZE_OWEN = 3 };
/* Pixel filters (src/render_wire.h:29). */
enum { RP_FILTER_BOX = 0, RP_FILTER_TRIANGLE = 1, RP_FILTER_GAUSSIAN = 2 };
/* Scattering families (wire::Material::scattering, src/render_wire.h:121). */
enum { RP_DIFFUSE = 0, RP_CONDUCTOR = 1, RP_DIELECTRIC = 2 };
/* Null medium interface (ScatteringKind::null_interface, wire scattering 10): scatters
 * nothing.  The scalar transport changes the ray's medium there
 * (shaders/scalar_transport.h:450-472); the hero transport, in vacuum, passes through it
 * (shaders/packet_pt_event_body.inc:130-145, 193-205), and so do shadow rays
 * (shaders/packet_transport.h:377-446). */
enum { RP_INTERFACE = 10 };
/* Mix of two materials (ScatteringKind::mix, wire scattering 9): each hit resolves to
 * second_material where the PBRT alpha hash of (point, -direction, material index) is below
 * mix_amount, else first_material (shaders/packet_pt_event_body.inc:165-190,
 * shaders/scalar_transport.h:566-587); nesting is acyclic, at most 64 levels, and reaches no
 * null interface (src/render.cpp:1955-1995). */
enum { RP_MIX = 9 };
/* Reflectance sources (src/render_wire.h:41-48).  RP_REFLECTANCE_IMAGE (wire::image_material)
 * reads images->textures[image_texture] at the hit's texture coordinates and reconstructs a
 * bounded spectrum from the filtered linear RGB (shaders/packet_walk.h:22-57). */
enum {
    RP_REFLECTANCE_KNOTS = 0,
    RP_REFLECTANCE_CONSTANT = 1,
    RP_REFLECTANCE_RGB = 2, /* wire::rgb_sigmoid_material: PBRT RGBAlbedoSpectrum coefficients */
    RP_REFLECTANCE_IMAGE = 3,
    RP_REFLECTANCE_BLACKBODY = 4
};
/* Image wrap, filter and texel storage (ImageWrap / ImageFilter, src/image_texture.hpp:14-15;
 * texel formats src/render_wire.h:35-40). */
enum { RP_WRAP_REPEAT = 0, RP_WRAP_CLAMP = 1, RP_WRAP_BLACK = 2 };
enum { RP_TEXTURE_BILINEAR = 0, RP_TEXTURE_TRILINEAR = 1, RP_TEXTURE_POINT = 2, RP_TEXTURE_EWA = 3 };
enum { RP_TEXELS_SRGB8 = 0, RP_TEXELS_LINEAR8 = 1, RP_TEXELS_HALF = 2, RP_TEXELS_FLOAT = 3 };
/* Floats of rypath's sRGB reconstruction table (srgb_reconstruction_table,
 * src/rgb_spectrum.hpp:31): 64 z nodes, then 3 x 64^3 cells of 3 quadratic coefficients. */
#define RP_RGB_TABLE_FLOATS (64u + 3u * 64u * 64u * 64u * 3u)
/* Positional light kinds (src/render_wire.h:200). */
enum { RP_POINT_LIGHT = 0, RP_SPOT_LIGHT = 1 };
/* Light selection (LightSamplerKind, src/render.hpp:217; wire word src/render_wire.h:304). */
enum { RP_LIGHTS_BVH = 0, RP_LIGHTS_POWER = 1, RP_LIGHTS_UNIFORM = 2 };
/* Scene model (RenderModel, src/render.hpp:135): PBRT scenes (raster camera, knot spectra, the
 * PBRT film) or rypath's demo model (`--render-demo`: a look-at camera, 8-knot reflectances,
 * a unit equal-energy sky sampled by the light sample, the demo film). */
enum { RP_MODEL_PBRT = 0, RP_MODEL_DEMO = 1 };
/* Spectral transport (SpectralTransport, src/render.hpp:218). */
enum { RP_TRANSPORT_SCALAR = 0, RP_TRANSPORT_HERO = 2 };
/* Hero wavelength sampling (HeroWavelengthSampling, src/render.hpp:220). */
enum { RP_HERO_UNIFORM = 0, RP_HERO_VISIBLE = 1 };

typedef struct rp_knot { float wavelength, value; } rp_knot; /* wire::SpectralKnot */

/* PBRT analytic shapes in object space (GeometryAnalytic, src/geometry.hpp:25-37, as the wire
 * record geometry_wire::Analytic, src/geometry_wire.h:31-40): angles in radians; a sphere of
 * `radius` clipped to z in [z_min, z_max] and phi in [0, phi_max]; a disk of `radius` and
 * `inner_radius` in the plane z = height; a cylinder of `radius` over z in [z_min, z_max]
 * without end caps.  `kind` is the wire tag RP_PRIMITIVE_ANALYTIC. */
enum { RP_PRIMITIVE_TRIANGLE = 1, RP_PRIMITIVE_PATCH = 2, RP_PRIMITIVE_ANALYTIC = 4 };
enum { RP_ANALYTIC_SPHERE = 1, RP_ANALYTIC_DISK = 2, RP_ANALYTIC_CYLINDER = 3 };
typedef struct rp_analytic {
    uint32_t kind, subtype;
    float radius, z_min, z_max, phi_max, inner_radius, height;
} rp_analytic;

/* One mesh placement; the subset of wire::Instance (src/render_wire.h:168-188) the hot
 * path reads.  matrix is row-major 3x4 object-to-world. */
typedef struct rp_instance {
    float matrix[12];
    uint32_t vertex_begin, triangle_begin, triangle_count;
    uint32_t material;
    uint32_t reverse_orientation;
    uint32_t emission;     /* index into emissions or RP_NONE */
    uint32_t normal_begin; /* index into normals or RP_NONE */
    uint32_t inside_medium, outside_medium; /* RP_NONE = vacuum */
    uint32_t invisible_emitter; /* nonzero: rays pass through it (RenderScene::instance_invisible_emitters) */
    /* the placement's bilinear patches (GeometryMesh::patches) and analytic shapes
     * (GeometryMesh::analytics): ranges of rp_scene_desc.patches / .analytics (wire::Instance
     * patch_begin / patch_count / analytic_begin / analytic_count, src/render_wire.h:168-188);
     * patch corners index the instance's vertices like its triangles */
    uint32_t patch_begin, patch_count;
    uint32_t analytic_begin, analytic_count;
} rp_instance;

/* The subset of wire::Material (src/render_wire.h:107-130) used by diffuse, conductor and
 * dielectric scattering with sampled / constant / blackbody reflectance. */
typedef struct rp_material {
    uint32_t scattering;   /* RP_DIFFUSE / RP_CONDUCTOR / RP_DIELECTRIC */
    uint32_t kind;         /* RP_REFLECTANCE_* */
    uint32_t knot_begin, knot_count; /* reflectance knots */
    float scalar_value;    /* constant reflectance or blackbody C2/T factor */
    uint32_t eta_begin, eta_count, k_begin, k_count;
    uint32_t optical_extensions; /* bit 0: extend eta endpoints, bit 1: extend k */
    float u_roughness, v_roughness;
    uint32_t remap_roughness;
    uint32_t first_material, second_material; /* RP_MIX children (MaterialAuxiliary, src/render_wire.h:159) */
    float mix_amount;                         /* RP_MIX constant amount (src/render_wire.h:160) */
    uint32_t image_texture; /* RP_REFLECTANCE_IMAGE: index into images->textures */
    float coefficients[3];  /* RP_REFLECTANCE_RGB: the sigmoid polynomial's c0 l^2 + c1 l + c2 */
    float reflectance[8];   /* RP_MODEL_DEMO sampled reflectance at the 8 demo knots (360 420 470 520 570 620 700 830 nm) */
} rp_material;

/* wire::ImageTexture (src/render_wire.h:68-87), field for field.  level_begin/level_count
 * select a mip chain in images->levels (level 0 the finest); the glTF fields are carried
 * for layout only (glTF images are refused). */
typedef struct rp_image_texture {
    uint32_t level_begin, level_count;
    uint32_t wrap;          /* RP_WRAP_* */
    uint32_t texel_format;  /* RP_TEXELS_* */
    float uscale, vscale, udelta, vdelta;
    float scale;            /* RGB multiplier after the lookup */
    uint32_t invert;        /* nonzero: 1 - rgb after scaling */
    uint32_t filter;        /* RP_TEXTURE_* */
    float max_anisotropy;   /* EWA cap, 1..16 */
    uint32_t transfer_offset; /* 8-bit formats: first of 256 floats in images->transfer */
    uint32_t channels;      /* 1, 3 or 4 */
    uint32_t gltf, wrap_t, min_filter, mag_filter;
} rp_image_texture;

/* wire::TextureLevel (src/render_wire.h:63-67): a level of width x height texels starting
 * at texel word `offset` (4 words a texel for float storage, 2 for half, 1 for 8-bit). */
typedef struct rp_texture_level {
    uint32_t width, height, offset;
} rp_texture_level;

/* The image inputs of a RenderScene (image_textures, texture_camera, instance_texture_frames,
 * environment_image, src/render.hpp:251-261) in rypath's wire layout.  rgb_table and
 * illuminant are rypath's srgb_reconstruction_table() and pbrt_d65() (src/rgb_spectrum.hpp).
 * An environment image (RP_NONE: none) is a square equal-area octahedral map with one level;
 * it replaces the constant environment, and its importance tables are built from its
 * texels when the scene is created (src/environment_sampling.cpp).  Image reflectance needs
 * texture coordinates: per instance the first of its vertices' uvs (instance_uv_begin[i],
 * RP_NONE: the triangle's default (0,0), (1,0), (1,1)), per textured triangle its tangents
 * dpdu, dpdv (6 floats, TextureTriangleFrame, from instance_frame_begin[i] on), and the
 * texture camera (TextureCamera, src/texture_footprint.hpp:9-12; row-major). */
typedef struct rp_images {
    uint32_t texture_count;    const rp_image_texture *textures;
    uint32_t level_count;      const rp_texture_level *levels;
    uint32_t texel_word_count; const uint32_t *texels;
    uint32_t transfer_count;   const float *transfer;
    const float *rgb_table;    /* RP_RGB_TABLE_FLOATS */
    const float *illuminant;   /* RP_SPECTRUM_BINS */
    uint32_t environment_image;
    float environment_scale;
    float environment_from_world[9]; /* environment_texture_from_world, linear part */
    uint32_t uv_count;         const float *uvs; /* 2 floats per uv */
    const uint32_t *instance_uv_begin;    /* instance_count entries */
    uint32_t frame_count;      const float *frames;
    const uint32_t *instance_frame_begin; /* instance_count entries (RP_NONE: untextured) */
    float world_from_camera[9], camera_from_world[9];
    const float *ewa_weights; /* 128 floats: rypath_ewa::weights (src/ewa_weights.h), for EWA filters */
} rp_images;

typedef struct rp_area_emission { /* wire::AreaEmission subset, src/render_wire.h:219 */
    float radiance[RP_SPECTRUM_BINS];
    uint32_t two_sided;
} rp_area_emission;

typedef struct rp_positional_light { /* PointLight / SpotLight, src/render.hpp:178-191 */
    float position[3];
    float intensity[RP_SPECTRUM_BINS];
    uint32_t kind; /* RP_POINT_LIGHT / RP_SPOT_LIGHT */
    float light_from_world[9]; /* row-major; spot axis is +z after this map */
    float cos_falloff_start, cos_falloff_end;
} rp_positional_light;

typedef struct rp_medium { /* HomogeneousMedium, src/render.hpp:29-36 */
    float sigma_a[RP_SPECTRUM_BINS];
    float sigma_s[RP_SPECTRUM_BINS];
    float emission[RP_SPECTRUM_BINS];
    float g;
} rp_medium;

/* PBRT raster camera (RasterCamera, src/render.hpp:152-157): a primary direction is
 * corner + x*dx + y*dy at normalised raster (x, y). */
typedef struct rp_camera {
    float origin[3], corner[3], dx[3], dy[3];
} rp_camera;

/* Everything build_metal_renderer reads from a RenderScene on the PT/hero path
 * (src/metal_render.mm:147-290, :505-700).  Arrays are host memory. */
typedef struct rp_scene_desc {
    uint32_t abi_version; /* RP_ABI_VERSION */
    uint32_t vertex_count;   const float *positions;   /* xyz per vertex (object space) */
    uint32_t normal_count;   const float *normals;     /* xyz per normal, may be 0 */
    uint32_t triangle_count; const uint32_t *triangles; /* 3 vertex indices per triangle */
    uint32_t instance_count; const rp_instance *instances;
    uint32_t material_count; const rp_material *materials;
    uint32_t knot_count;     const rp_knot *knots;
    uint32_t emission_count; const rp_area_emission *emissions;
    uint32_t positional_count; const rp_positional_light *positional;
    uint32_t medium_count;   const rp_medium *media;
    uint32_t camera_medium;  /* RP_NONE = vacuum camera */
    const float *environment; /* RP_SPECTRUM_BINS constant environment radiance, or NULL */
    rp_camera camera;
    uint32_t filter_kind; float filter_x_radius, filter_y_radius;
    uint32_t max_depth;
    uint32_t light_sampler;    /* RP_LIGHTS_* */
    uint32_t transport;        /* RP_TRANSPORT_HERO (scalar volpath: RP_TRANSPORT_SCALAR) */
    uint32_t hero_wavelengths; /* RP_HERO_* */
    const void *sobol_tables;  /* RP_SOBOL_TABLE_BYTES, sobol::Tables layout */
    /* PerspectiveLens (src/render.hpp:159-164): aperture radius (0 = pinhole), focal
     * distance, and the camera's x / y axes in world space.  Batched views are pinhole. */
    float lens_radius, focal_distance;
    float lens_x[3], lens_y[3];
    /* RP_FILTER_GAUSSIAN: PBRT sigma; the radii are filter_x_radius / filter_y_radius. */
    float filter_sigma;
    const rp_images *images; /* NULL: no image textures and no environment image */
    /* RP_MODEL_DEMO: the camera is RenderCamera's look-at basis -- camera.origin, camera.corner =
     * forward, camera.dx = right, camera.dy = up (unit vectors, src/metal_render.mm:194-204) --
     * and film_scale = tan(vertical fov / 2). */
    uint32_t model;
    float film_scale;
    /* Bilinear patches: 4 vertex indices each in tensor-product order p00, p10, p01, p11
     * (src/geometry.hpp:44-45); analytic shapes (rp_analytic). */
    uint32_t patch_count;    const uint32_t *patches;
    uint32_t analytic_count; const rp_analytic *analytics;
} rp_scene_desc;

/* RenderRequest (src/metal_render.hpp:14-32). */
typedef struct rp_request {
    uint32_t width, height;
    uint64_t seed;
    int32_t material_seed;
    uint32_t pixel_begin, pixel_count;
    uint64_t sample_begin;
    uint32_t sample_count;
    uint32_t emergency_limit;  /* render_emergency_limit = 1024 */
    uint32_t sampler_kind;     /* RP_SAMPLER_* */
    uint32_t randomization;    /* RP_RANDOMIZE_* */
    uint32_t boundary_limit;   /* medium_boundary_limit = 4096 */
    uint64_t total_samples;    /* the render's sample budget (RenderRequest::total_samples); ZSobol needs it */
} rp_request;

/* packet_wire::Result, 80 bytes (src/packet_wire.h:13-18). */
typedef struct rp_packet_result {
    uint32_t status, pixel, sample_low, sample_high, splat_count;
    float wavelengths[4], wavelength_pdfs[4], radiance[4];
    float filter_weight;
    uint32_t reserved[2];
} rp_packet_result;

/* render_wire::Sample-derived scalar output (RenderSample, src/render.hpp:285-294). */
typedef struct rp_scalar_result {
    uint32_t status, pixel, sample_low, sample_high;
    float wavelength, radiance;
    uint32_t scatterings;
    uint32_t random_words[4];
} rp_scalar_result;

/* MetalDeviceInfo analogue. */
typedef struct rp_device_info {
    char name[128];
    int device, sm_count, major, minor;
    uint64_t total_memory;
} rp_device_info;

/* Device film: per-pixel FP64 Neumaier sums in canonical (absolute sample, pixel) order,
 * the reduction PacketFilmBatch::add performs on the host (src/packet_film.cpp:198-265),
 * plus per-pixel second moments of the XYZ estimate for the 3-sigma statistics and, under a
 * finite film clamp, the compatibility planes: the sums of the exposed XYZ scaled down to
 * the maximum component (clamp_sensor, src/packet_film.cpp:39-47; FilmPixel,
 * src/render.hpp:317-326). */
typedef struct rp_film_pixel {
    double sum[3], correction[3];
    double weight_sum, weight_correction;
    double square[3];
    uint64_t count;
    double compatibility_sum[3], compatibility_correction[3];
} rp_film_pixel;

/* Film request: render samples [sample_begin, sample_begin + sample_count) for every pixel,
 * batch_size absolute samples per launch (RenderSettings, src/render.hpp:240-248). */
typedef struct rp_film_request {
    uint32_t width, height;
    uint64_t seed;
    uint64_t sample_begin, sample_count, batch_size;
    uint32_t sampler_kind, randomization;
    uint32_t emergency_limit;
    uint64_t total_samples; /* the render's sample budget; 0 = sample_begin + sample_count */
    uint32_t flags;         /* RP_FILM_FRESH: the film starts from zero, its contents are not read */
    double exposure;        /* Film::exposure, applied to the compatibility planes only */
    double max_component_value; /* Film::max_component_value; 0 or infinity: no clamp, no compatibility planes */
} rp_film_request;
enum { RP_FILM_FRESH = 1 };

/* Kernel-level timing of the last call on a scene (CUDA events on the scene stream). */
typedef struct rp_timing {
    double total_ms;          /* whole call, device time */
    double trace_ms;          /* closest-hit traversal kernels */
    double shadow_ms;         /* any-hit traversal kernels */
    double shade_ms;          /* shading kernels */
    double other_ms;          /* raygen, queue resets, film */
    uint64_t closest_rays, shadow_rays, kernel_launches, samples;
    uint64_t nodes_visited, triangles_tested; /* closest-hit rays; only when counting */
    uint64_t trace_launches, shadow_launches, shade_launches, other_launches;
    uint64_t shadow_nodes_visited, shadow_triangles_tested; /* any-hit rays; only when counting */
    double build_ms, build_host_ms, build_bvh_ms; /* scene creation: total, host preparation, LBVH */
    /* hero shade kernels by BSDF family (0 diffuse, 1 conductor, 2 dielectric, 3 escape), each
     * kernel's own launch time summed over the call; only when counting, whose family kernels
     * run one after another (otherwise they run side by side) */
    double shade_family_ms[4];
} rp_timing;

/* ---- device and lifetime ------------------------------------------------------------ */

/* Device probe; MetalDeviceInfo in build_metal_renderer (src/metal_render.hpp:76-77). */
rp_status rp_cuda_device_info(int device, rp_device_info *info, char *diag, size_t diag_capacity);

/* build_metal_renderer(const RenderScene&, library, RenderBuildOptions, RenderTimings*)
 * (src/metal_render.hpp:84-95; stub src/metal_render_stub.cpp:14-50).  Uploads the scene,
 * builds the LBVH on the device and the light-selection tables on the host.  On failure
 * *scene is NULL and diag says why. */
rp_status rp_cuda_scene_create(const rp_scene_desc *desc, int device, struct rp_scene **scene,
                               char *diag, size_t diag_capacity);
/* ~MetalRenderScene (src/metal_render.hpp:56). */
void rp_cuda_scene_destroy(struct rp_scene *scene);

/* ---- sampling (driver-compatible) ----------------------------------------------------- */

/* MetalRenderScene::sample(const RenderRequest&) for the packet/hero transport
 * (src/metal_render.hpp:56-57; body src/metal_render.mm:1940-2170).  Host output: one
 * 80-byte packet result per lane, lane order, pixel = pixel_begin + lane % pixel_count,
 * sample = sample_begin + lane / pixel_count.  capacity is in results.  A nonzero per-lane
 * status is reported as RP_FAILURE with a diagnostic, as the reference does
 * (src/metal_render.mm:2058-2064); the results are still written. */
rp_status rp_cuda_sample(struct rp_scene *scene, const rp_request *request,
                         rp_packet_result *host_results, size_t capacity, char *diag,
                         size_t diag_capacity);
/* Same, device output, asynchronous on `stream` (a cudaStream_t, NULL = the scene stream);
 * results are complete when the stream is. */
rp_status rp_cuda_sample_device(struct rp_scene *scene, const rp_request *request,
                                rp_packet_result *device_results, size_t capacity,
                                void *stream, char *diag, size_t diag_capacity);
/* Scalar (one-wavelength) PT / volpath lanes: rypath_render_paths
 * (shaders/render.metal:2299-2371), RenderSample output (src/metal_render.mm:2136-2166). */
rp_status rp_cuda_sample_scalar(struct rp_scene *scene, const rp_request *request,
                                rp_scalar_result *host_results, size_t capacity, char *diag,
                                size_t diag_capacity);

/* ---- device film ---------------------------------------------------------------------- */

/* Progressive render into a device film: the loop of drive_progressive
 * (src/render_driver.cpp:166-275) with the packet film reduction of PacketFilmBatch
 * (src/packet_film.cpp:198-265) done on the device.  film (host, width*height pixels) is
 * read as the committed state and overwritten with the new one; a failed batch leaves it
 * unchanged (src/render_driver.cpp:201-214). */
rp_status rp_cuda_render_film(struct rp_scene *scene, const rp_film_request *request,
                              rp_film_pixel *host_film, char *diag, size_t diag_capacity);
/* Same with the film resident on the device (no host copies). */
rp_status rp_cuda_render_film_device(struct rp_scene *scene, const rp_film_request *request,
                                     rp_film_pixel *device_film, char *diag,
                                     size_t diag_capacity);

/* CIE 1931 2-degree colour matching functions at 1 nm, 360..830 (471 rows of x, y, z as
 * doubles): the sensor response of packet_sensor_xyz (src/packet_film.cpp:102-114, table of
 * src/render.cpp:2147-2152).  Required before the film entry points. */
rp_status rp_cuda_set_cie(struct rp_scene *scene, const double *cie_xyz);

/* ---- batched views ------------------------------------------------------------------- */

/* One camera view of a batch: a PBRT raster camera, its film size, its absolute sample range
 * and where its pixels start in the batch film.  Views share the scene (and its filter,
 * depth, lights and materials). */
typedef struct rp_view {
    rp_camera camera;
    uint32_t width, height;
    uint64_t sample_begin, sample_count;
    uint64_t film_offset; /* first rp_film_pixel of this view in the batch film */
} rp_view;

/* Batch execution: lanes per wave, block shapes and grid size of the wavefront kernels, and
 * whether each wave replays a CUDA graph.  A zero field is picked by the autotuner. */
typedef struct rp_batch_config {
    uint32_t wave_lanes;    /* up to 2^23 */
    uint32_t trace_block;   /* 64 or 128 threads (closest-hit and any-hit kernels) */
    uint32_t shade_block;   /* 128 or 256 threads (shading kernels) */
    uint32_t blocks_per_sm; /* resident blocks per SM the grids are sized for */
    uint32_t use_graph;     /* 1: one CUDA graph replayed per wave; 2: direct launches */
    float probe_ms_per_mlane; /* tuning: measured cost of the chosen configuration */
} rp_batch_config;

typedef struct rp_batch_request {
    uint64_t seed;
    uint32_t sampler_kind, randomization, emergency_limit;
    rp_batch_config config;
    double exposure, max_component_value; /* the film clamp, as in rp_film_request */
} rp_batch_request;

/* Renders every view's samples into one device film (the views' pixels, in rp_film_pixel
 * rows, accumulating onto what it holds), all views' lanes sharing one wavefront: the
 * batched form of rp_cuda_render_film_device.  Each view's film equals a plain render of
 * that view (same camera, size and samples) bit for bit.  `used` (optional) receives the
 * configuration that ran.  A failed lane fails the call (the film is then partial).  No
 * counterpart in rypath, which renders one view per job (src/render_driver.cpp:166-275). */
rp_status rp_cuda_render_views_device(struct rp_scene *scene, const rp_view *views, uint32_t view_count,
                                      const rp_batch_request *request, rp_film_pixel *device_film,
                                      rp_batch_config *used, char *diag, size_t diag_capacity);
/* The autotuner alone: times one probe wave of the batch per candidate configuration (wave
 * size, then trace block, shade block and grid size, each with the others fixed) and
 * returns the fastest.  Nonzero fields of request->config are kept as given. */
rp_status rp_cuda_tune_views(struct rp_scene *scene, const rp_view *views, uint32_t view_count,
                             const rp_batch_request *request, rp_batch_config *chosen, char *diag,
                             size_t diag_capacity);

/* ---- differentiation ------------------------------------------------------------------- */

/* Overwrites knot values [first, first + count) of the scene's spectral knots (the
 * reflectance spectra of materials with RP_REFLECTANCE_KNOTS); wavelengths are kept.  The
 * forward render of new parameters is then an ordinary rp_cuda_render_film(_device).  No
 * counterpart in rypath. */
rp_status rp_cuda_set_knot_values(struct rp_scene *scene, uint32_t first, uint32_t count, const float *values,
                                  char *diag, size_t diag_capacity);

/* The backward pass of a film render: the film request's lanes (samples [sample_begin,
 * sample_begin + sample_count) of every pixel) are traced again with the same random numbers
 * and, given d loss / d XYZ of every pixel's film mean (device, 3 doubles per pixel), the
 * gradient of the loss with respect to the knot values of the listed materials (diffuse,
 * RP_REFLECTANCE_KNOTS) is accumulated into device_gradient (zeroed first; the listed
 * materials' knot_count entries each, in list order).  Depth at most 15; at most 2048
 * gradient entries.  No counterpart in rypath. */
typedef struct rp_adjoint_request {
    rp_film_request film;
    uint32_t material_count;
    const uint32_t *materials; /* host array of scene material indices */
} rp_adjoint_request;
rp_status rp_cuda_adjoint_device(struct rp_scene *scene, const rp_adjoint_request *request,
                                 const double *device_d_loss_d_xyz, float *device_gradient, char *diag,
                                 size_t diag_capacity);

/* ---- frame sessions ------------------------------------------------------------------- */

/* An interactive frame session (FrameSession, src/frame_session.hpp:182-212, with the
 * independent estimator and the path tracer): each frame renders one fresh absolute sample of
 * every pixel into raw XYZ that stays on the device until it is captured, asynchronously on
 * the session's stream.  A session has two frame slots; a submitted frame holds its slot until
 * it is released, also after completion.  The session renders its scene on that scene's
 * device; the scene must outlive the session.  Calls on one session need external
 * serialisation, and a session shares its scene's stream and wavefront with the scene's other
 * calls (serialise them too). */
typedef struct rp_frame_config { /* FrameConfig subset, src/frame_session.hpp:58-100 */
    uint32_t width, height;
    uint64_t seed;
    uint32_t sampler_kind, randomization;
    uint64_t footprint_samples; /* the fixed sample budget ZSobol needs (FrameConfig::footprint_samples) */
} rp_frame_config;
typedef struct rp_frame_request { /* FrameRequest, src/frame_session.hpp:113-116 */
    uint64_t sample_index, epoch;
    const rp_camera *camera; /* NULL: the scene's camera; else this raster camera from now on */
} rp_frame_request;
enum { RP_FRAME_PENDING = 0, RP_FRAME_COMPLETE = 1, RP_FRAME_FAILED = 2 }; /* FrameStatus */
typedef struct rp_frame_info { /* FrameInfo subset, src/frame_session.hpp:118-150 */
    uint32_t status;           /* RP_FRAME_* */
    uint32_t width, height;
    uint64_t sample_index, epoch;
    double gpu_ms;             /* device time of the frame's work, when complete */
    uint64_t completed_samples;
    uint32_t failed_pixels;    /* pixels whose sample failed (a failed frame has at least one) */
} rp_frame_info;

rp_status rp_cuda_frame_session_create(struct rp_scene *scene, const rp_frame_config *config,
                                       struct rp_frame_session **session, char *diag, size_t diag_capacity);
/* Waits for the session's frames and frees them. */
void rp_cuda_frame_session_destroy(struct rp_frame_session *session);
/* FrameSession::submit.  On success *frame is the frame's slot (0 or 1).  When both slots are
 * held the call returns RP_FAILURE with *busy set (FrameSubmitResult::busy). */
rp_status rp_cuda_frame_submit(struct rp_frame_session *session, const rp_frame_request *request, uint32_t *frame,
                               int *busy, char *diag, size_t diag_capacity);
/* Frame::poll (no wait) and Frame::wait. */
rp_status rp_cuda_frame_poll(struct rp_frame_session *session, uint32_t frame, rp_frame_info *info);
rp_status rp_cuda_frame_wait(struct rp_frame_session *session, uint32_t frame, rp_frame_info *info);
/* Frame::capture: waits, then copies the frame's raw XYZ (3 floats per pixel, row major) into
 * host memory of capacity_pixels pixels.  The sensor value of a pixel is packet_sensor_xyz of
 * its sample without the filter weight, which cancels (shaders/frame_sensor.h:33-52); the
 * scalar transport's is its wavelength's matching-function value times 470 times radiance
 * (:22-31). */
rp_status rp_cuda_frame_capture(struct rp_frame_session *session, uint32_t frame, float *host_xyz,
                                size_t capacity_pixels, char *diag, size_t diag_capacity);
/* The frame's device raw XYZ (valid until the frame is released). */
rp_status rp_cuda_frame_device_xyz(struct rp_frame_session *session, uint32_t frame, const float **device_xyz);
/* Releases the frame's slot (the Frame's destructor); waits for its work first. */
rp_status rp_cuda_frame_release(struct rp_frame_session *session, uint32_t frame);

/* ---- instrumentation ------------------------------------------------------------------ */

/* Timing of the last sample/film call on this scene. */
rp_status rp_cuda_last_timing(struct rp_scene *scene, rp_timing *timing);
/* Enable (1) or disable (0) exact node/triangle visit counting in traversal. */
rp_status rp_cuda_set_counting(struct rp_scene *scene, int enabled);

/* ---- fixed-input probes (the reference's rypath_*_probe kernels) ------------------------ */

/* rypath_sobol_probe (shaders/render.metal:74-93): per query {m, x, y, sample_lo,
 * sample_hi, dimension, mode, seed} -> {index_lo, index_hi, word, hash, uniform bits,
 * camera uniform bits}.  8 words in, 6 words out per query; tables from the scene. */
rp_status rp_cuda_probe_sobol(const void *sobol_tables, const uint32_t *queries, uint32_t count,
                              uint32_t *results, char *diag, size_t diag_capacity);
/* Philox4x32-10 (shaders/render.metal:97-109): 6 words in {counter[4], key[2]}, 4 out. */
rp_status rp_cuda_probe_philox(const uint32_t *queries, uint32_t count, uint32_t *results,
                               char *diag, size_t diag_capacity);
/* Hero wavelengths (src/hero_spectrum_shared.h:199-244): u -> lambda[4], pdf[4]. */
rp_status rp_cuda_probe_wavelengths(const float *u, uint32_t count, uint32_t mode,
                                    float *results, char *diag, size_t diag_capacity);
/* Begin-sample words (shaders/render.metal:238-311) for a request: per lane
 * {pixel, sample_lo, sample_hi, index_lo, index_hi, words[4], lens[2]} (11 words) and the
 * primary ray {origin[3], direction[3]} (6 floats). */
rp_status rp_cuda_probe_raygen(struct rp_scene *scene, const rp_request *request,
                               uint32_t *words, float *rays, size_t capacity, char *diag,
                               size_t diag_capacity);
/* BSDF probes (shaders/conductor.h, dielectric.h, transmission.h): per query 16 floats
 * {kind, p0..p4, wo[3], wi[3], uc, u[2], pad} -> 12 floats {f, pdf, valid, sample wi[3],
 * weight, sample pdf, flags, eta, pad, pad}. */
rp_status rp_cuda_probe_bsdf(const float *queries, uint32_t count, float *results, char *diag,
                             size_t diag_capacity);
/* Image probes over a description's images (uploaded as scene creation uploads them, the
 * environment tables included): texture lookups of texture `index` through the point /
 * bilinear / trilinear filters (shaders/image_texture.h:403-456; 6 floats {u, v, dudx, dvdx,
 * dudy, dvdy} -> 4 {rgb[3], scalar}); the sRGB reconstruction (shaders/image_texture.h:458-507;
 * 4 {r, g, b, wavelength} -> 2 {bounded, unbounded}); environment queries
 * (shaders/image_lighting.h:170-325; 8 {direction[3], wavelength, u[2], unused[2]} -> 12
 * {radiance, compensated pdf, full pdf, sample ok, direction[3], pdf, full-table sample ok,
 * direction[3]}). */
rp_status rp_cuda_probe_image_lookup(const rp_images *images, uint32_t index, const float *queries,
                                     uint32_t count, float *results, char *diag,
                                     size_t diag_capacity);
rp_status rp_cuda_probe_rgb_spectrum(const rp_images *images, const float *queries, uint32_t count,
                                     float *results, char *diag, size_t diag_capacity);
rp_status rp_cuda_probe_environment(const rp_images *images, const float *queries, uint32_t count,
                                    float *results, char *diag, size_t diag_capacity);
/* Texture footprint probe (shaders/texture_footprint.h): per query 48 floats {camera-relative
 * point[3], geometric normal[3], ray direction[3], one-pixel x and y camera rays[3 + 3], spp
 * scale, world_from_camera[9], camera_from_world[9] (row-major), minimum dx[3], dy[3], dpdu[3],
 * dpdv[3], unused[2]} -> 24 floats {primary ok, primary dpdx[3], dpdy[3], approximate dpdx[3],
 * dpdy[3], derivatives ok, dstdx[2], dstdy[2] (of the primary footprint where it exists),
 * texture direction of the x ray[3], unused[3]}. */
rp_status rp_cuda_probe_texture_footprint(const float *queries, uint32_t count, float *results,
                                          char *diag, size_t diag_capacity);
/* Bilinear patch intersection (intersect_bilinear, shaders/bilinear.h: PBRT's ruled-surface
 * solve in float pairs): per query 20 floats {p00[3], p10[3], p01[3], p11[3], origin[3],
 * direction[3], t_min, t_max} -> 4 floats {hit, t, u, v}. */
rp_status rp_cuda_probe_bilinear(const float *queries, uint32_t count, float *results, char *diag,
                                 size_t diag_capacity);
/* Analytic shape intersection and evaluation (intersect_analytic / evaluate_analytic,
 * shaders/analytic.h): per query 16 words {rp_analytic (8 words), origin[3], direction[3],
 * t_min, t_max} -> 16 floats {hit, t, u, v, then at the hit (u, v) the object-space
 * position[3], normal[3], dpdu[3], dpdv[3]}. */
rp_status rp_cuda_probe_analytic(const float *queries, uint32_t count, float *results, char *diag,
                                 size_t diag_capacity);
/* The minimum one-pixel camera-ray differentials a film of width x height gives the texture
 * footprints of a scene with image reflectance (prepare_texture_camera_differentials,
 * src/texture_footprint.cpp:199-232), on the host. */
rp_status rp_cuda_texture_camera_differentials(const rp_camera *camera, uint32_t width,
                                               uint32_t height, float *minimum_dx,
                                               float *minimum_dy, char *diag,
                                               size_t diag_capacity);
/* The environment image's importance tables as scene creation builds them, on the host (no
 * device is used): the full then the compensated table (each a marginal CDF and one
 * conditional CDF per row, width + 1 floats apiece; build_environment_sampling,
 * src/environment_sampling.cpp:20-115) into cdf (2 (width + 1)^2 floats), and the image's mean
 * RGB illuminant power (light_image_power, src/light_sampling.cpp:78-95). */
rp_status rp_cuda_environment_tables(const rp_images *images, float *cdf, size_t capacity,
                                     uint32_t *width, uint32_t *compensated_offset,
                                     double *mean_power, char *diag, size_t diag_capacity);
/* Hero BSDF probe (shaders/hero_current_bsdf.h:121-203, hero_frozen_bsdf.h:167-250,
 * hero_scattering.h:100-138): per query 32 floats {kind, active mask, remap, unused, per
 * wavelength {eta or reflectance, k, roughness u, roughness v}, wo[3], wi[3], uc, ux, uy,
 * unused[3]} -> 32 floats {sampled wi[3], numerator[4], pdf[4], eta[4], flags (delta 1 |
 * transmission 2 | accepted 4 | valid 8), evaluated f[4], pdf[4], valid, wavelength 0's Dirac
 * mass, pdf, eta, Dirac ok, connectible, prepared, unused}.  The wavelengths share wavelength
 * 0's roughness. */
rp_status rp_cuda_probe_hero(const float *queries, uint32_t count, float *results, char *diag,
                             size_t diag_capacity);
/* Export the scene's binary LBVH over its n triangles: per internal node {left, right,
 * parent} (n-1 nodes; a child with bit 31 set is leaf slot child & 0x7fffffff, the root's
 * parent is RP_NONE), the leaf order (triangle id of each leaf slot), the sorted 63-bit
 * Morton keys, and bounds {lo[3], hi[3]}: internal node i at row i, leaf slot j at row n-1+j.
 * capacity is in triangles. */
rp_status rp_cuda_scene_export_bvh(struct rp_scene *scene, uint32_t *nodes, uint32_t *leaf_order,
                                   uint64_t *keys, float *bounds, size_t capacity, char *diag,
                                   size_t diag_capacity);
/* Export the compressed 8-wide traversal tree the walks use: *node_count 80-byte nodes into
 * `nodes` (when node_capacity suffices) and the n wide leaves (3 x 4 floats each: v0 with the
 * triangle id's bits in w, v1, v2) into `triangles`.  Node layout (little endian): p[3] floats,
 * then bytes e.x, e.y, e.z (biased exponents of the plane steps) and the internal-child mask;
 * child_base, tri_base, leaf mask, unused (u32 each); then the 8 child slots' bytes of lo.x,
 * lo.y, lo.z, hi.x, hi.y, hi.z.  Child k's box lies within the planes p + q 2^(e - 127) of
 * its bytes; internal children are nodes child_base + (internal children before slot k),
 * leaves are tri_base + (leaves before slot k).  No counterpart in rypath (Metal's
 * acceleration structure is opaque). */
rp_status rp_cuda_scene_export_wide(struct rp_scene *scene, void *nodes, size_t node_capacity, float *triangles,
                                    size_t triangle_capacity, uint32_t *node_count, char *diag,
                                    size_t diag_capacity);
/* Closest-hit (any_hit == 0) or occlusion (any_hit == 1) queries for host rays
 * {origin[3], direction[3], tmax} (7 floats each) -> {t, b1, b2, primitive bits} (4 floats;
 * primitive RP_NONE bits = miss).  For occlusion only field 0 (1 = occluded) is used. */
rp_status rp_cuda_trace_rays(struct rp_scene *scene, const float *rays, uint32_t count,
                             int any_hit, float *hits, char *diag, size_t diag_capacity);

/* ---- allocation-free sampling -------------------------------------------------------------- */

/* Size of the library's file-scope device scratch array used by rp_cuda_sample_device_static.
 * Every GPU that loads this library holds this much device memory until the process exits. */
#define RP_STATIC_SCRATCH_BYTES (64u << 20)
/* Largest request, in lanes (pixel_count * sample_count), that fits that scratch. */
#define RP_STATIC_MAX_LANES 118976u

/* No counterpart in rypath.  Same work and results as rp_cuda_sample_device, for callers that
 * must not allocate device memory during a render call -- for example a host that hands the
 * GPU to us between its own allocation-free phases, or code running where the allocator is
 * unavailable or forbidden (inside a memory budget owned by someone else).  The wavefront's
 * per-lane scratch (path state, queues, family bins, counters) lives in one file-scope
 * __device__ array of RP_STATIC_SCRATCH_BYTES instead of memory from the scene's pool; the
 * caller still passes the scene (created earlier) and a device output buffer.  Nothing is
 * allocated: no cudaMalloc / cudaMallocAsync / cudaFree and no allocating library call.
 *   - Limit: request lanes (pixel_count * sample_count) <= RP_STATIC_MAX_LANES;
 *     larger requests return RP_INVALID_ARGUMENT with a diagnostic naming the maximum.
 *   - The first call on a scene looks up the array's device address once, with the scene's
 *     device current, and keeps it with the scene; make that first call before any stream
 *     capture.
 *   - Work runs on `stream` (a cudaStream_t; NULL = the scene's stream) and is complete when
 *     the stream is.  Every call shares the one array: calls whose GPU work overlaps (two
 *     streams, two scenes, two threads) race and corrupt each other; serialise them. */
rp_status rp_cuda_sample_device_static(struct rp_scene *scene, const rp_request *request,
                                       rp_packet_result *device_results, size_t capacity,
                                       void *stream, char *diag, size_t diag_capacity);

/* ---- host helpers ----------------------------------------------------------------------- */

/* sizeof() of an ABI struct by name ("rp_request", ...), 0 if unknown; lets bindings check
 * their layouts against this library. */
uint32_t rp_cuda_abi_size(const char *type_name);
/* The light-selection tables rp_cuda_scene_create builds, for inspection: build_light_sampling
 * (src/light_sampling.cpp:384-572).  Rows of 16 doubles {power, bounds_power, low[3],
 * high[3], direction[3], cos_outer, cos_emission, two_sided, infinite, unused}; outputs are
 * LightAlias (4 words each), LightRecord (4 words each), LightBounds (16 words each) and the
 * infinite-light ids.  Returns the node count, or -1 on invalid input. */
int rp_cuda_build_light_tables(const double *rows, uint32_t count, uint32_t *alias, uint32_t *records,
                               uint32_t *nodes, uint32_t *infinite, uint32_t *infinite_count);

#ifdef __cplusplus
}
#endif

#endif /* RYPATH_CUDA_H */
