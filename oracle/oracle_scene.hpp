// ORACLE -- test infrastructure only (see oracle_math.hpp).  Scene tables, light selection,
// light geometry sampling, surface reconstruction and the binary LBVH with watertight
// triangle tests, restated on the CPU.
#pragma once

#include "oracle_math.hpp"
#include "oracle_image.hpp"
#include "oracle_shapes.hpp"
#include "../include/rypath_cuda.h"

#include <functional>
#include <string>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- light selection tables
// Wire records, src/render_wire.h:227-244.
struct LightAlias {
    float threshold, pmf;
    u32 alias, padding;
};
struct LightBounds {
    float low[3], high[3], direction[3];
    float power, cos_outer, cos_emission;
    u32 child, parent, light, flags;
};
struct LightRecord {
    u32 leaf, flags, padding0, padding1;
};
static_assert(sizeof(LightBounds) == 64 && sizeof(LightAlias) == 16);
// src/light_sampling.hpp:11-17
struct LightInput {
    double power = 0, bounds_power = -1;
    float low[3] = {0, 0, 0}, high[3] = {0, 0, 0}, direction[3] = {0, 0, 1};
    float cos_outer = -1, cos_emission = 0;
    bool two_sided = true, infinite = false;
};
struct LightTables {
    std::vector<LightAlias> alias;
    std::vector<LightRecord> records;
    std::vector<LightBounds> nodes;
    std::vector<u32> infinite;
};
bool build_light_tables(const std::vector<LightInput> &in, LightTables &out, std::string &error);
// src/packet_spectrum_shared.h:33-59 (the non-hero four-wavelength sampler)
Wavelengths packet_sample_visible(float u);
// src/light_sampling.cpp:17-27
double light_spectrum_power(const float *spectrum);

// ---------------------------------------------------------------- scene
struct Instance {
    float m[12];
    u32 vertex_begin, triangle_begin, triangle_count, material, reverse, emission, normal_begin;
    u32 emitter_begin;
    u32 inside_medium = RP_NONE, outside_medium = RP_NONE;
    u32 invisible = 0; // RenderScene::instance_invisible_emitters
    u32 patch_begin = 0, patch_count = 0, analytic_begin = 0, analytic_count = 0;
    float inverse[12] = {}; // world-to-object 3x4 of instances with procedural primitives
};
// HomogeneousMedium (src/render.hpp:29-36)
struct Medium {
    std::array<float, 471> sigma_a, sigma_s, emission;
    float g;
};
struct Material {
    u32 scattering, kind, knot_begin, knot_count;
    float scalar_value;
    u32 eta_begin, eta_count, k_begin, k_count, optical_extensions;
    float u_roughness, v_roughness;
    u32 remap;
    u32 first = RP_NONE, second = RP_NONE; // mix children (MaterialAuxiliary, src/render_wire.h:159-161)
    float mix_amount = 0;
    u32 image_texture = RP_NONE; // RP_REFLECTANCE_IMAGE
    float coefficients[3] = {0, 0, 0}; // RP_REFLECTANCE_RGB
    float reflectance[8] = {0, 0, 0, 0, 0, 0, 0, 0}; // demo model
};
struct Positional {
    F3 position;
    float intensity[471];
    u32 kind;
    float light_from_world[9];
    float cos_falloff_start, cos_falloff_end;
};
struct Emitter {
    u32 instance, primitive;
};
struct Scene {
    std::vector<F3> positions, normals;
    std::vector<std::array<u32, 3>> triangles;
    std::vector<Instance> instances;
    std::vector<Material> materials;
    std::vector<Knot> knots;
    std::vector<std::array<float, 471>> emission;
    std::vector<u32> emission_two_sided;
    std::vector<Positional> positional;
    std::vector<Emitter> emitters;
    std::array<float, 471> environment{};
    bool has_environment = false;
    Images images; // image textures and the environment image (env_image RP_NONE: none)
    bool textured = false; // a diffuse material reads an image
    u32 model = RP_MODEL_PBRT; // RP_MODEL_DEMO: look-at camera, 8-knot reflectance, unit sky
    float film_scale = 1;
    // media (scalar transport)
    std::vector<Medium> media;
    u32 camera_medium = RP_NONE, transport = RP_TRANSPORT_HERO;
    bool media_enabled = false;
    // camera (wire::Parameters slots for the PBRT model, src/metal_render.mm:158-191)
    F3 origin, forward, right, up, camera_normal;
    u32 filter_kind = 0;
    float filter_x = .5f, filter_y = .5f;
    // Gaussian filter table (conditional rows of gauss_w + 1, then the marginal) and the
    // packet film weight; thin lens
    std::vector<float> gauss_cdf;
    u32 gauss_w = 0, gauss_h = 0;
    float filter_weight = 1;
    float lens_radius = 0, focal_distance = 1e6f;
    F3 lens_x{1, 0, 0}, lens_y{0, 1, 0};
    u32 max_depth = 5, light_sampler = 0, hero_mode = 1;
    float scene_radius = 1;
    F3 scene_center{};
    // light tables
    LightTables lights;
    u32 light_count = 0, environment_light = RP_NONE;
    const SobolTables *sobol = nullptr;
    std::vector<unsigned char> sobol_storage;
    // world-space triangles and their owning instance (flattened), then the procedural
    // primitives: every instance's patches, then every instance's analytic shapes
    std::vector<std::array<F3, 3>> world;
    std::vector<u32> tri_instance, tri_local;
    std::vector<std::array<u32, 4>> patches;
    std::vector<Analytic> analytics;
    u32 tri_prims = 0, patch_prims = 0, procedural_prims = 0;
};
bool load_scene(const rp_scene_desc &d, Scene &s, std::string &error);
// compile_gaussian_filter (src/gaussian_filter.cpp:84-137); empty string on success
std::string gaussian_filter_table(float x_radius, float y_radius, float sigma, std::vector<float> &cdf, u32 &width,
                                  u32 &height, float &integral);

// ---------------------------------------------------------------- binary LBVH
struct Box {
    float lo[3], hi[3];
};
struct Bvh {
    u32 n = 0;
    std::vector<u64> keys;       // sorted Morton keys
    std::vector<u32> order;      // sorted triangle ids
    std::vector<u32> left, right, parent; // internal nodes; child >= 0x80000000 is a leaf slot
    std::vector<u32> leaf_parent;
    std::vector<Box> node_box;   // internal node bounds
    std::vector<Box> leaf_box;   // leaf slot bounds
};
void build_lbvh(const std::vector<std::array<F3, 3>> &tris, Bvh &bvh);

struct Hit {
    float t = INFINITY, b1 = 0, b2 = 0;
    u32 prim = RP_NONE;
};
// Watertight ray/triangle test; returns true when t in (0, tmax) is found.
bool intersect_triangle(F3 o, F3 d, const std::array<F3, 3> &v, float tmax, float &t, float &b1,
                        float &b2);
// The closest triangle hit alone (the binary tree holds the triangles).
Hit trace_triangles(const Scene &s, const Bvh &b, F3 o, F3 d, float tmax);
Hit trace_closest(const Scene &s, const Bvh &bvh, F3 o, F3 d, float tmax);
bool trace_any(const Scene &s, const Bvh &bvh, F3 o, F3 d, float tmax);
Hit trace_closest_brute(const Scene &s, F3 o, F3 d, float tmax);

// ---------------------------------------------------------------- surface points
// SurfacePoint subset, shaders/render.metal:870-881
struct SurfacePoint {
    F3 position, error, geometric_normal, shading_normal;
    float inverse_area_pdf = 0;
    float world_extent = 0;
    bool curved = false; // a patch or analytic point
};
// The reflectance of a material at one wavelength (shaders/packet_walk.h:22-57); `image` is the
// hit's filtered, scaled linear RGB for image reflectance
bool reflectance(const Scene &s, const Material &m, float w, const Rgb *image, float &rho);
// surface_point (shaders/render.metal:1120-1132) of flattened primitive `prim` at a native hit
bool hit_surface_point(const Scene &s, u32 prim, u32 instance, u32 local, float b1, float b2, SurfacePoint &p);
// The ray's point at t and its rounding bound (shaders/render.metal:1913-1929)
void ray_point(F3 o, F3 d, float t, bool curved, F3 &position, F3 &error);
bool triangle_surface_point(const Scene &s, u32 instance, u32 local, float u, float v,
                            bool native_hit, SurfacePoint &p);

// ---------------------------------------------------------------- pass-through and mix surfaces
// PBRT's alpha hash as a uniform (shaders/alpha_hash.h:10-36); t is the bit pattern of the
// material index the event passes as a float.
float alpha_uniform(F3 origin, F3 direction, u32 t_bits);
// The material a hit on mix root `material` resolves to (shaders/packet_pt_event_body.inc:
// 165-190); returns the sample status (0, RP_SAMPLE_INVALID_ARITHMETIC or _INVALID_HIT).
u32 resolve_mix(const Scene &s, F3 position, F3 toward_origin, u32 &material);
// A hero pass-through instance: an invisible emitter or a null-interface root material
// (shaders/packet_pt_event_body.inc:130-145).
bool pass_through(const Scene &s, const Instance &in);
// shaders/render.metal:1939-1977: the origin past a pass-through surface hit at t
bool spawn_boundary(F3 o, F3 d, float t, const SurfacePoint &pt, F3 direction, F3 &origin);

// ---------------------------------------------------------------- light selection / geometry
struct Selected {
    u32 light;
    float pmf;
};
Selected light_sample(const Scene &s, F3 position, F3 normal, float u);
float light_pmf(const Scene &s, F3 position, F3 normal, u32 id);
bool light_geometry_sample(const Scene &s, u32 emitter, F3 reference, F3 normal, float ux, float uy,
                           float &b1, float &b2, SurfacePoint &point, float &pdf);
float light_geometry_pdf(const Scene &s, u32 emitter, F3 reference, F3 normal,
                         const SurfacePoint &point);

} // namespace oracle

// The opaque scene handle of the oracle's C ABI (oracle.h).
struct or_scene {
    oracle::Scene scene;
    oracle::Bvh bvh;
};
