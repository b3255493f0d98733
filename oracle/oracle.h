/* ORACLE -- test infrastructure only.  C ABI of the CPU restatement of rypath's spectral
 * path-tracing hot path.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load this library, and only as the checker / CPU baseline. */
#ifndef RYPATH_ORACLE_H
#define RYPATH_ORACLE_H

#include "../include/rypath_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_scene or_scene;

/* Deep copy of a scene description; builds the light tables and the CPU LBVH. */
or_scene *or_scene_create(const rp_scene_desc *desc, char *diag, size_t diag_capacity);
void or_scene_destroy(or_scene *scene);
uint32_t or_scene_light_count(const or_scene *scene);

/* Hero packet lanes of a request (rypath_render_packets), threads <= 0: all cores. */
int or_sample(const or_scene *scene, const rp_request *request, rp_packet_result *results,
              size_t capacity, int threads);

/* Probes mirroring rp_cuda_probe_* (same layouts). */
void or_probe_sobol(const void *tables, const uint32_t *queries, uint32_t count, uint32_t *results);
void or_probe_philox(const uint32_t *queries, uint32_t count, uint32_t *results);
void or_probe_wavelengths(const float *u, uint32_t count, uint32_t mode, float *results);
int or_probe_raygen(const or_scene *scene, const rp_request *request, uint32_t *words, float *rays,
                    size_t capacity);
void or_probe_bsdf(const float *queries, uint32_t count, float *results);

/* LBVH export in the rp_cuda_scene_export_bvh layout. */
int or_export_bvh(const or_scene *scene, uint32_t *nodes, uint32_t *leaf_order, uint64_t *keys,
                  float *bounds, size_t capacity);
/* Ray queries in the rp_cuda_trace_rays layout; brute != 0 scans every triangle. */
void or_trace_rays(const or_scene *scene, const float *rays, uint32_t count, int any_hit, int brute,
                   float *hits);

/* Hero likelihood arithmetic probes (src/hero_spectrum_shared.h): per query 12 floats
 * {prefix frac[4] as floats, prefix exponent[4] as floats, beta[4]} plus 8 more
 * {numerator[4], pdf[4]} -> {beta'[4], density frac[4], density exp[4], valid}. */
void or_probe_advance(const float *queries, uint32_t count, float *results);

/* Light selection tables: lights as LightInput rows of 16 doubles
 * {power, bounds_power, low[3], high[3], direction[3], cos_outer, cos_emission, two_sided,
 * infinite, pad} -> alias (4 words each), records (4 words each), nodes (16 words each),
 * infinite ids.  Returns the node count, or -1. */
int or_build_light_tables(const double *rows, uint32_t count, uint32_t *alias, uint32_t *records,
                          uint32_t *nodes, uint32_t *infinite, uint32_t *infinite_count);

/* Light selection probe: queries {px,py,pz,nx,ny,nz,u,id} -> {light bits, pmf, pmf(id)}. */
void or_probe_light_select(const or_scene *scene, const float *queries, uint32_t count, float *results);

/* Film reduction of packet results in canonical order (PacketFilmBatch::add). */
int or_film_add(const rp_packet_result *results, size_t count, const double *cie_xyz,
                uint32_t pixel_count, rp_film_pixel *film);
/* The same with a finite film clamp: the compatibility planes of clamp_sensor
 * (src/packet_film.cpp:39-47); max_component_value 0 or infinity: none. */
int or_film_add_clamped(const rp_packet_result *results, size_t count, const double *cie_xyz,
                        uint32_t pixel_count, double exposure, double max_component_value, rp_film_pixel *film);

/* Gaussian pixel filter: the table of compile_gaussian_filter (src/gaussian_filter.cpp) and the
 * device inverse of shaders/render.metal:200-236 on count (u, v) pairs.  Returns the table
 * size in floats (conditional rows then marginal), or -1. */
int or_gaussian_filter(float x_radius, float y_radius, float sigma, float *cdf, size_t capacity, uint32_t *size,
                       float *integral, const float *uv, uint32_t count, float *samples);

/* Halton / ZSobol probe (rypath's QMC known-answer layout): 10 int64 per query -> 6 uint64. */
void or_probe_qmc(const void *sobol_tables, const int64_t *queries, uint32_t count, uint64_t *results);

/* FP64 path-replay adjoint of a film render (the rp_cuda_adjoint_device contract): gradient of
 * the loss with respect to the knot values of `materials`, given d loss / d film-mean XYZ per
 * pixel and the CIE table.  0, 1 when a lane failed, -1 on a bad material list. */
int or_adjoint(const or_scene *scene, const rp_film_request *film, const uint32_t *materials, uint32_t count,
               const double *d_loss_d_xyz, const double *cie_xyz, double *gradient, int threads);

/* Scalar (one-wavelength) PT / volpath lanes of a request (rypath_render_paths); the scene
 * must be built with RP_TRANSPORT_SCALAR.  threads <= 0: all cores.  0, 1 on a failed
 * lane, -1 on a bad request. */
int or_sample_scalar(const or_scene *scene, const rp_request *request, rp_scalar_result *results,
                     size_t capacity, int threads);
/* Homogeneous-medium equations (shaders/medium.h): per query 15 floats {sigma_a, sigma_s,
 * Le, distance, sigma_t, u, wo[3], wi[3], g, ux, uy} -> 8 floats {transmission, emission,
 * valid, flight, phase, sampled direction[3]}. */
void or_probe_medium(const float *queries, uint32_t count, float *results);
/* Film reduction of scalar samples in the given order (FilmBatch::add); demo: the demo
 * model's film (wavelength_xyz, unweighted radiance). */
int or_scalar_film_add(const rp_scalar_result *results, size_t count, const double *cie_xyz,
                       uint32_t pixel_count, rp_film_pixel *film, int demo);

/* Image probes, in the layouts of oracle/_ref's ref_image_lookup, ref_rgb_spectrum,
 * ref_environment_tables and ref_environment_queries: texture lookups of texture `index`
 * (6 floats {u, v, dudx, dvdx, dudy, dvdy} -> 4 {rgb[3], scalar}); RGB reconstruction
 * (4 {r, g, b, wavelength} -> 2 {bounded, unbounded}); the environment tables of a square
 * image (the EWA filter reads the 128 weights given); environment queries (8 {direction[3],
 * wavelength, u[2], unused[2]} -> 12 {radiance,
 * compensated pdf, full pdf, sample ok, direction[3], pdf, full-table sample ok,
 * direction[3]}). */
void or_image_lookup(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                     uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                     uint32_t transfer_count, const float *queries, uint32_t count, float *results,
                     const float *ewa_weights);
void or_rgb_spectrum(const float *table, const float *queries, uint32_t count, float *results);
/* Bilinear patch and analytic shape queries in the layouts of rp_cuda_probe_bilinear and
 * rp_cuda_probe_analytic (oracle_shapes.hpp). */
void or_probe_bilinear(const float *queries, uint32_t count, float *results);
void or_probe_analytic(const float *queries, uint32_t count, float *results);
int or_environment_tables(const void *textures, uint32_t index, const void *levels, const uint32_t *texels,
                          uint32_t words, const float *transfer, const float *table, const float *illuminant,
                          float *cdf, size_t capacity, uint32_t *width, uint32_t *compensated_offset,
                          double *power);
void or_environment_queries(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                            uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                            uint32_t transfer_count, const float *table, const float *illuminant,
                            const float *cdf, uint32_t cdf_count, uint32_t width, uint32_t compensated_offset,
                            float scale, const float *env_from_world, const float *queries, uint32_t count,
                            float *results);

/* Texture footprints (shaders/texture_footprint.h) in the layout of oracle/_ref's
 * ref_texture_footprint (48 floats -> 24), and the texture camera's minimum differentials
 * (src/texture_footprint.cpp:199-232; 0, or -1 when refused). */
void or_texture_footprint(const float *queries, uint32_t count, float *results);
int or_texture_camera_differentials(const float *corner, const float *dx, const float *dy, uint32_t width,
                                    uint32_t height, float *out);

#ifdef __cplusplus
}
#endif
#endif
