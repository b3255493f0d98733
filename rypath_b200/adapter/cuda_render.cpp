// SPDX-License-Identifier: GPL-3.0-only
// rypath's GPU backend boundary (src/metal_render.hpp) implemented over the B200 backend's C ABI
// (include/rypath_cuda.h).  This translation unit takes the place of src/metal_render_stub.cpp
// in rypath_metal_backend (CMakeLists.txt:190-236): the progressive driver, job, checkpoint,
// CLI and output code are unchanged and reach the B200 kernels through build_metal_renderer
// and MetalRenderScene::sample, exactly as they reach Metal on Apple hardware; interactive
// callers reach them through build_frame_session / FrameSession (src/frame_session.hpp).
//
// Beyond that boundary, cuda_backend::FilmRenderer (cuda_render.hpp) renders whole batches into
// rypath's Film on the device (the PacketFilmBatch reduction done there, film_fold.hpp).
#include "cuda_render.hpp"
#include "ewa_weights.h"
#include "film_fold.hpp"
#include "frame_session.hpp"
#include "image_texture.hpp"
#include "metal_render.hpp"
#include "rgb_spectrum.hpp"
#include "sampling.hpp"
#include "texture_footprint.hpp"

#include <rypath_cuda.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <numbers>
#include <memory>
#include <string>
#include <vector>

namespace rypath {

struct MetalRenderScene::Impl {
    rp_scene *scene = nullptr;
    bool scalar = false; // RenderScene::spectral_transport == scalar (the volpath lanes)
    ~Impl() { rp_cuda_scene_destroy(scene); }
};
MetalRenderScene::MetalRenderScene(std::unique_ptr<Impl> impl) : impl_(std::move(impl)) {}
MetalRenderScene::~MetalRenderScene() = default;
MetalRenderScene::MetalRenderScene(MetalRenderScene &&) noexcept = default;
MetalRenderScene &MetalRenderScene::operator=(MetalRenderScene &&) noexcept = default;

namespace cuda_backend {
namespace {

GeometryStatus status_of(rp_status s) {
    switch (s) {
    case RP_SUCCESS:
        return GeometryStatus::success;
    case RP_NOT_BUILT:
        return GeometryStatus::not_built;
    case RP_NO_DEVICE:
        return GeometryStatus::no_device;
    case RP_NO_RAY_TRACING:
        return GeometryStatus::no_ray_tracing;
    default:
        return GeometryStatus::failure;
    }
}

template <class Array> void copy_spectrum(const Array &from, float (&to)[RP_SPECTRUM_BINS]) {
    std::copy(from.begin(), from.end(), to);
}

// The arrays an rp_scene_desc points into; they live until the scene is created (the backend
// deep-copies everything).
struct Arena {
    std::vector<float> positions, normals, environment;
    // images in the wire layout (src/render_wire.h:35-95)
    std::vector<rp_image_texture> textures;
    std::vector<rp_texture_level> levels;
    std::vector<std::uint32_t> texels, uv_begin, frame_begin;
    std::vector<float> transfer, uvs, frames;
    rp_images images{};
    std::vector<std::uint32_t> triangles, patches;
    std::vector<rp_analytic> analytics;
    std::vector<rp_instance> instances;
    std::vector<rp_material> materials;
    std::vector<rp_knot> knots;
    std::vector<rp_area_emission> emissions;
    std::vector<rp_positional_light> positional;
    std::vector<rp_medium> media;
};

std::uint32_t append_knots(const std::vector<SpectralKnot> &from, Arena &a) {
    const auto begin = std::uint32_t(a.knots.size());
    for (const auto &k : from)
        a.knots.push_back({k.wavelength, k.value});
    return begin;
}

// The scene's images as the backend reads them (RenderScene::image_textures, texture_camera,
// instance_texture_frames and environment_image, src/render.hpp:251-261): each distinct
// pyramid's levels once, rypath's sRGB and linear transfer tables (then any custom ones), the
// uvs of the meshes of textured instances and each instance's triangle frames.  The sRGB
// reconstruction table, D65 and the EWA weights are rypath's own.
std::string describe_images(const RenderScene &s, Arena &a) {
    if (s.image_textures.empty() && s.environment_image == UINT32_MAX)
        return {};
    a.transfer.resize(512);
    std::ranges::copy(image_transfer_table(ImageEncoding::srgb), a.transfer.begin());
    std::ranges::copy(image_transfer_table(ImageEncoding::linear), a.transfer.begin() + 256);
    std::map<const std::array<float, 256> *, std::uint32_t> custom;
    std::map<const ImagePyramid *, std::uint32_t> chains;
    for (const ImageTexture &texture : s.image_textures) {
        if (!texture.image)
            return "image texture without a pyramid";
        if (texture.gltf_sampler)
            return "the CUDA backend does not render glTF image textures";
        const ImagePyramid &image = *texture.image;
        rp_image_texture t{};
        t.filter = texture.filter == ImageFilter::point       ? RP_TEXTURE_POINT
                   : texture.filter == ImageFilter::trilinear ? RP_TEXTURE_TRILINEAR
                   : texture.filter == ImageFilter::ewa       ? RP_TEXTURE_EWA
                                                              : RP_TEXTURE_BILINEAR;
        t.texel_format = image.storage == ImageStorage::linear_float  ? RP_TEXELS_FLOAT
                         : image.storage == ImageStorage::linear_half ? RP_TEXELS_HALF
                         : image.encoding != ImageEncoding::srgb      ? RP_TEXELS_LINEAR8
                                                                      : RP_TEXELS_SRGB8;
        t.transfer_offset = image.encoding == ImageEncoding::srgb ? 0 : 256;
        if (image.custom_transfer) {
            const auto [it, fresh] = custom.try_emplace(image.custom_transfer.get(), std::uint32_t(a.transfer.size()));
            t.transfer_offset = it->second;
            if (fresh)
                a.transfer.insert(a.transfer.end(), image.custom_transfer->begin(), image.custom_transfer->end());
        }
        const auto [chain, added] = chains.try_emplace(&image, std::uint32_t(a.levels.size()));
        if (added) {
            const auto base = std::uint32_t(a.texels.size());
            for (const ImageMipLevel &l : image.levels)
                a.levels.push_back({l.width, l.height, base + l.offset});
            a.texels.insert(a.texels.end(), image.texels.begin(), image.texels.end());
        }
        t.level_begin = chain->second;
        t.level_count = std::uint32_t(image.levels.size());
        t.wrap = std::uint32_t(image.wrap);
        t.uscale = texture.uscale;
        t.vscale = texture.vscale;
        t.udelta = texture.udelta;
        t.vdelta = texture.vdelta;
        t.scale = texture.scale;
        t.invert = texture.invert ? 1u : 0u;
        t.max_anisotropy = texture.max_anisotropy;
        t.channels = image.source_channels;
        t.wrap_t = 10497;
        t.min_filter = 9987;
        t.mag_filter = 9729;
        a.textures.push_back(t);
    }
    // texture coordinates of the instances whose shading reads a texture context
    std::map<std::uint32_t, std::uint32_t> mesh_uvs;
    const bool framed = !s.instance_texture_frames.empty();
    for (std::size_t i = 0; i < s.geometry.instances.size(); ++i) {
        std::uint32_t uv = RP_NONE, frame = RP_NONE;
        const std::uint32_t mesh_index = s.geometry.instances[i].mesh_index;
        const GeometryMesh &mesh = s.geometry.meshes[mesh_index];
        if (framed && !s.instance_texture_frames[i].empty()) {
            frame = std::uint32_t(a.frames.size() / 6);
            for (const TextureTriangleFrame &f : s.instance_texture_frames[i])
                a.frames.insert(a.frames.end(), {f.dpdu.x, f.dpdu.y, f.dpdu.z, f.dpdv.x, f.dpdv.y, f.dpdv.z});
            if (!mesh.uvs.empty()) {
                const auto [it, fresh] = mesh_uvs.try_emplace(mesh_index, std::uint32_t(a.uvs.size() / 2));
                uv = it->second;
                if (fresh)
                    for (const auto &c : mesh.uvs)
                        a.uvs.insert(a.uvs.end(), {c[0], c[1]});
            }
        }
        a.uv_begin.push_back(uv);
        a.frame_begin.push_back(frame);
    }
    rp_images &im = a.images;
    im = {};
    im.texture_count = std::uint32_t(a.textures.size());
    im.textures = a.textures.data();
    im.level_count = std::uint32_t(a.levels.size());
    im.levels = a.levels.data();
    im.texel_word_count = std::uint32_t(a.texels.size());
    im.texels = a.texels.data();
    im.transfer_count = std::uint32_t(a.transfer.size());
    im.transfer = a.transfer.data();
    im.rgb_table = srgb_reconstruction_table().data();
    im.illuminant = pbrt_d65().data();
    im.ewa_weights = rypath_ewa::weights;
    im.environment_image = s.environment_image;
    im.environment_scale = s.environment_image_scale;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            im.environment_from_world[3 * r + c] = float(s.environment_texture_from_world.values[4 * r + c]);
    im.uv_count = std::uint32_t(a.uvs.size() / 2);
    im.uvs = a.uvs.data();
    im.instance_uv_begin = a.uv_begin.data();
    im.frame_count = std::uint32_t(a.frames.size() / 6);
    im.frames = a.frames.data();
    im.instance_frame_begin = a.frame_begin.data();
    std::copy(s.texture_camera.world_from_camera.begin(), s.texture_camera.world_from_camera.end(), im.world_from_camera);
    std::copy(s.texture_camera.camera_from_world.begin(), s.texture_camera.camera_from_world.end(), im.camera_from_world);
    return {};
}

// RenderScene -> rp_scene_desc: what build_metal_renderer reads on the PT / hero path and for
// the demo model (src/metal_render.mm:147-290, :505-700).  Returns a diagnostic for what the
// backend does not build (texture graphs and surface detail, some light kinds).  Bilinear
// patches (GeometryMesh::patches, corner order p00 p10 p01 p11) and analytic shapes
// (GeometryMesh::analytics, packed as pack_analytic does, src/analytic.hpp:51-60) go with their
// mesh.
std::string describe(const RenderScene &s, Arena &a, rp_scene_desc &d) {
    const bool demo = s.model == RenderModel::demo;
    if (!demo && !s.raster_camera)
        return "a PBRT-model scene needs its raster camera";
    std::vector<std::uint32_t> mesh_vertex(s.geometry.meshes.size()), mesh_triangle(s.geometry.meshes.size()),
        mesh_normal(s.geometry.meshes.size(), RP_NONE), mesh_patch(s.geometry.meshes.size()),
        mesh_analytic(s.geometry.meshes.size());
    for (std::size_t m = 0; m < s.geometry.meshes.size(); ++m) {
        const GeometryMesh &mesh = s.geometry.meshes[m];
        mesh_patch[m] = std::uint32_t(a.patches.size() / 4);
        for (const auto &q : mesh.patches)
            a.patches.insert(a.patches.end(), q.begin(), q.end());
        mesh_analytic[m] = std::uint32_t(a.analytics.size());
        for (const GeometryAnalytic &g : mesh.analytics)
            a.analytics.push_back({RP_PRIMITIVE_ANALYTIC, std::uint32_t(g.kind), g.radius, g.z_min, g.z_max, g.phi_max,
                                   g.inner_radius, g.height});
        mesh_vertex[m] = std::uint32_t(a.positions.size() / 3);
        mesh_triangle[m] = std::uint32_t(a.triangles.size() / 3);
        for (const auto &p : mesh.positions)
            a.positions.insert(a.positions.end(), {p.x, p.y, p.z});
        for (const auto &t : mesh.triangles)
            a.triangles.insert(a.triangles.end(), t.begin(), t.end());
        if (!mesh.normals.empty() && mesh.normals.size() == mesh.positions.size()) {
            mesh_normal[m] = std::uint32_t(a.normals.size() / 3);
            for (const auto &n : mesh.normals)
                a.normals.insert(a.normals.end(), {n.x, n.y, n.z});
        }
    }
    if (const std::string images = describe_images(s, a); !images.empty())
        return images;
    for (std::size_t i = 0; i < s.geometry.instances.size(); ++i) {
        const GeometryInstance &g = s.geometry.instances[i];
        rp_instance in{};
        std::copy(g.transform.values.begin(), g.transform.values.end(), in.matrix);
        in.vertex_begin = mesh_vertex[g.mesh_index];
        in.triangle_begin = mesh_triangle[g.mesh_index];
        in.triangle_count = std::uint32_t(s.geometry.meshes[g.mesh_index].triangles.size());
        in.patch_begin = mesh_patch[g.mesh_index];
        in.patch_count = std::uint32_t(s.geometry.meshes[g.mesh_index].patches.size());
        in.analytic_begin = mesh_analytic[g.mesh_index];
        in.analytic_count = std::uint32_t(s.geometry.meshes[g.mesh_index].analytics.size());
        in.material = s.instance_materials[i];
        in.reverse_orientation = s.instance_reverse_orientation.empty() ? 0 : s.instance_reverse_orientation[i];
        in.emission = s.instance_emissions.empty() ? RP_NONE : s.instance_emissions[i];
        in.normal_begin = mesh_normal[g.mesh_index];
        in.inside_medium = s.instance_media.empty() ? RP_NONE : s.instance_media[i].inside;
        in.outside_medium = s.instance_media.empty() ? RP_NONE : s.instance_media[i].outside;
        in.invisible_emitter = s.instance_invisible_emitters.empty() ? 0 : s.instance_invisible_emitters[i];
        a.instances.push_back(in);
    }
    for (const SpectralMaterial &m : s.materials) {
        rp_material w{};
        w.scattering = std::uint32_t(m.scattering); // ScatteringKind: diffuse 0 ... mix 9, null interface 10
        w.kind = std::uint32_t(m.kind);             // SpectralMaterialKind: sampled 0, constant 1, blackbody 4
        w.knot_begin = append_knots(m.knots, a);
        w.knot_count = std::uint32_t(m.knots.size());
        w.scalar_value = m.kind == SpectralMaterialKind::blackbody ? blackbody_exponent_factor(m.temperature_kelvin)
                                                                    : m.constant;
        w.eta_begin = append_knots(m.eta.knots, a);
        w.eta_count = std::uint32_t(m.eta.knots.size());
        w.k_begin = append_knots(m.k.knots, a);
        w.k_count = std::uint32_t(m.k.knots.size());
        w.optical_extensions = (m.eta.extend_endpoints ? 1u : 0u) | (m.k.extend_endpoints ? 2u : 0u);
        w.u_roughness = m.u_roughness;
        w.v_roughness = m.v_roughness;
        w.remap_roughness = m.remap_roughness ? 1u : 0u;
        w.first_material = m.surface.first_material;
        w.second_material = m.surface.second_material;
        w.mix_amount = m.surface.mix_amount;
        w.image_texture = m.image_texture;
        std::copy(m.reflectance.begin(), m.reflectance.end(), w.reflectance);
        std::copy(m.coefficients.begin(), m.coefficients.end(), w.coefficients);
        if (m.kind == SpectralMaterialKind::texture_graph ||
            m.bump_root != UINT32_MAX || m.normal_map != UINT32_MAX || m.table || m.texture_root != UINT32_MAX)
            return "the CUDA backend renders sampled, constant, RGB, blackbody and image reflectance without surface detail";
        a.materials.push_back(w);
    }
    for (const AreaEmission &e : s.area_emissions) {
        rp_area_emission w{};
        copy_spectrum(e.radiance, w.radiance);
        w.two_sided = e.two_sided ? 1u : 0u;
        a.emissions.push_back(w);
    }
    for (const PointLight &l : s.point_lights) {
        rp_positional_light w{};
        w.position[0] = l.position.x;
        w.position[1] = l.position.y;
        w.position[2] = l.position.z;
        copy_spectrum(l.intensity, w.intensity);
        w.kind = RP_POINT_LIGHT;
        w.light_from_world[0] = w.light_from_world[4] = w.light_from_world[8] = 1;
        w.cos_falloff_start = 1;
        a.positional.push_back(w);
    }
    for (const SpotLight &l : s.spot_lights) {
        rp_positional_light w{};
        w.position[0] = l.position.x;
        w.position[1] = l.position.y;
        w.position[2] = l.position.z;
        copy_spectrum(l.intensity, w.intensity);
        w.kind = RP_SPOT_LIGHT;
        std::copy(l.light_from_world.begin(), l.light_from_world.end(), w.light_from_world);
        w.cos_falloff_start = l.cos_falloff_start;
        w.cos_falloff_end = l.cos_falloff_end;
        a.positional.push_back(w);
    }
    if (!s.goniometric_lights.empty() || !s.projection_lights.empty() || !s.distant_lights.empty())
        return "the CUDA backend samples area, point and spot lights and a constant environment";
    for (const HomogeneousMedium &m : s.media) {
        rp_medium w{};
        copy_spectrum(m.sigma_a, w.sigma_a);
        copy_spectrum(m.sigma_s, w.sigma_s);
        copy_spectrum(m.emission, w.emission);
        w.g = m.g;
        a.media.push_back(w);
    }
    a.environment.assign(s.environment.begin(), s.environment.end());
    d = {};
    d.abi_version = RP_ABI_VERSION;
    d.vertex_count = std::uint32_t(a.positions.size() / 3);
    d.positions = a.positions.data();
    d.normal_count = std::uint32_t(a.normals.size() / 3);
    d.normals = a.normals.empty() ? nullptr : a.normals.data();
    d.triangle_count = std::uint32_t(a.triangles.size() / 3);
    d.triangles = a.triangles.data();
    d.patch_count = std::uint32_t(a.patches.size() / 4);
    d.patches = a.patches.empty() ? nullptr : a.patches.data();
    d.analytic_count = std::uint32_t(a.analytics.size());
    d.analytics = a.analytics.empty() ? nullptr : a.analytics.data();
    d.instance_count = std::uint32_t(a.instances.size());
    d.instances = a.instances.data();
    d.material_count = std::uint32_t(a.materials.size());
    d.materials = a.materials.data();
    d.knot_count = std::uint32_t(a.knots.size());
    d.knots = a.knots.data();
    d.emission_count = std::uint32_t(a.emissions.size());
    d.emissions = a.emissions.data();
    d.positional_count = std::uint32_t(a.positional.size());
    d.positional = a.positional.data();
    d.medium_count = std::uint32_t(a.media.size());
    d.media = a.media.data();
    d.camera_medium = s.camera_medium; // no_medium == RP_NONE
    d.environment = a.environment.data();
    d.images = a.textures.empty() && s.environment_image == UINT32_MAX ? nullptr : &a.images;
    if (demo) {
        // the demo camera slots (src/metal_render.mm:194-206): the look-at basis in double,
        // rounded to binary32, and tan(fov / 2)
        const RenderCamera &c = s.camera;
        const std::array<double, 3> o{c.origin.x, c.origin.y, c.origin.z};
        std::array<double, 3> f{double{c.target.x} - o[0], double{c.target.y} - o[1], double{c.target.z} - o[2]};
        const auto unit = [](std::array<double, 3> v) {
            const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            return std::array<double, 3>{v[0] / n, v[1] / n, v[2] / n};
        };
        const auto cross = [](const std::array<double, 3> &a, const std::array<double, 3> &b) {
            return std::array<double, 3>{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        };
        f = unit(f);
        const auto r = unit(cross(f, {c.up.x, c.up.y, c.up.z}));
        const auto u = cross(r, f);
        for (int k = 0; k < 3; ++k) {
            d.camera.origin[k] = float(o[k]);
            d.camera.corner[k] = float(f[k]);
            d.camera.dx[k] = float(r[k]);
            d.camera.dy[k] = float(u[k]);
        }
        d.model = RP_MODEL_DEMO;
        d.film_scale = float(std::tan(c.vertical_fov_degrees * (std::numbers::pi_v<double> / 360.0)));
    } else {
        const RasterCamera &c = *s.raster_camera;
        const GeometryPoint *points[4] = {&c.origin, &c.corner, &c.dx, &c.dy};
        float *dst[4] = {d.camera.origin, d.camera.corner, d.camera.dx, d.camera.dy};
        for (int k = 0; k < 4; ++k) {
            dst[k][0] = points[k]->x;
            dst[k][1] = points[k]->y;
            dst[k][2] = points[k]->z;
        }
        d.model = RP_MODEL_PBRT;
    }
    d.filter_kind = std::uint32_t(s.filter.kind);
    d.filter_x_radius = s.filter.x_radius;
    d.filter_y_radius = s.filter.y_radius;
    d.filter_sigma = s.filter.sigma;
    if (s.perspective_lens) {
        const PerspectiveLens &l = *s.perspective_lens;
        d.lens_radius = l.radius;
        d.focal_distance = l.focal_distance;
        d.lens_x[0] = l.camera_x.x;
        d.lens_x[1] = l.camera_x.y;
        d.lens_x[2] = l.camera_x.z;
        d.lens_y[0] = l.camera_y.x;
        d.lens_y[1] = l.camera_y.y;
        d.lens_y[2] = l.camera_y.z;
    } else {
        d.focal_distance = 1e6f;
        d.lens_x[0] = d.lens_y[1] = 1;
    }
    d.max_depth = s.max_depth;
    d.light_sampler = std::uint32_t(s.light_sampler);
    d.transport = std::uint32_t(s.spectral_transport); // scalar 0 (volpath), hero 2
    d.hero_wavelengths = std::uint32_t(s.hero_wavelengths);
    d.sobol_tables = &sobol_tables();
    return {};
}

// Builds the device scene of a RenderScene on device 0; on failure returns the status and
// fills diag.
rp_status create(const RenderScene &scene, rp_scene **out, std::string &diag) {
    Arena arena;
    rp_scene_desc desc;
    diag = describe(scene, arena, desc);
    if (!diag.empty())
        return RP_NOT_BUILT;
    char text[1024] = {};
    const rp_status st = rp_cuda_scene_create(&desc, 0, out, text, sizeof text);
    diag = text;
    return st;
}

rp_request request_of(const RenderRequest &r) {
    rp_request q{};
    q.width = r.width;
    q.height = r.height;
    q.seed = r.seed;
    q.material_seed = r.material_seed;
    q.pixel_begin = r.pixel_begin;
    q.pixel_count = r.pixel_count;
    q.sample_begin = r.sample_begin;
    q.sample_count = r.sample_count;
    q.emergency_limit = r.emergency_limit;
    q.sampler_kind = std::uint32_t(r.sampler.kind);
    q.randomization = std::uint32_t(r.sampler.randomization);
    q.boundary_limit = r.boundary_limit;
    q.total_samples = r.total_samples;
    return q;
}

std::vector<double> cie_rows() {
    // CIE 1931 2-degree matching functions at 1 nm from 360 nm (the table of packet_sensor_xyz,
    // src/render.cpp:2147-2152), read through rypath's own lookup
    std::vector<double> rows(3 * RP_SPECTRUM_BINS);
    for (std::uint32_t i = 0; i < RP_SPECTRUM_BINS; ++i) {
        const auto xyz = pbrt_cie_xyz(float(360 + i));
        for (int c = 0; c < 3; ++c)
            rows[3 * i + c] = xyz[c];
    }
    return rows;
}

} // namespace

std::unique_ptr<FilmRenderer> FilmRenderer::build(const RenderScene &scene, std::string &diag) {
    rp_scene *handle = nullptr;
    if (create(scene, &handle, diag) != RP_SUCCESS)
        return nullptr;
    const std::vector<double> cie = cie_rows();
    if (rp_cuda_set_cie(handle, cie.data()) != RP_SUCCESS) {
        rp_cuda_scene_destroy(handle);
        diag = "rp_cuda_set_cie failed";
        return nullptr;
    }
    return std::unique_ptr<FilmRenderer>(new FilmRenderer(handle));
}

FilmRenderer::~FilmRenderer() { rp_cuda_scene_destroy(scene_); }

std::string FilmRenderer::render(const RenderSettings &settings, std::uint64_t sample_begin, std::uint64_t count,
                                 Film &film) {
    const std::size_t pixels = std::size_t(settings.width) * settings.height;
    if (film.pixels.size() != pixels)
        return "Film size differs from the render settings";
    std::vector<rp_film_pixel> rows(pixels);
    if (sample_begin != 0) {
        const std::string e = unfold_film(film, rows);
        if (!e.empty())
            return e;
    }
    rp_film_request q{};
    q.width = settings.width;
    q.height = settings.height;
    q.seed = settings.seed;
    q.sample_begin = sample_begin;
    q.sample_count = count;
    q.batch_size = settings.batch_size;
    q.sampler_kind = std::uint32_t(settings.sampler.kind);
    q.randomization = std::uint32_t(settings.sampler.randomization);
    q.emergency_limit = render_emergency_limit;
    q.total_samples = settings.samples;
    q.flags = sample_begin == 0 ? std::uint32_t(RP_FILM_FRESH) : 0u;
    q.exposure = film.exposure;
    q.max_component_value = film.max_component_value;
    char diag[1024] = {};
    const rp_status st = rp_cuda_render_film(scene_, &q, rows.data(), diag, sizeof diag);
    // the returned rows hold the committed state, also when a later batch failed
    const std::string e = fold_film(rows, film);
    if (st != RP_SUCCESS)
        return diag[0] ? std::string(diag) : std::string("CUDA film render failed");
    return e;
}

} // namespace cuda_backend

RenderBuildResult build_metal_renderer(const RenderScene &scene, const std::filesystem::path &) {
    RenderBuildResult r;
    char text[1024] = {};
    rp_device_info info{};
    rp_status st = rp_cuda_device_info(0, &info, text, sizeof text);
    r.diagnostic = text;
    if (st == RP_SUCCESS) {
        auto impl = std::make_unique<MetalRenderScene::Impl>();
        impl->scalar = scene.spectral_transport == SpectralTransport::scalar;
        st = cuda_backend::create(scene, &impl->scene, r.diagnostic);
        if (st == RP_SUCCESS)
            r.scene.reset(new MetalRenderScene(std::move(impl)));
    }
    r.status = cuda_backend::status_of(st);
    r.device.name = info.name;
    r.device.architecture = "sm_" + std::to_string(info.major * 10 + info.minor);
    r.device.compute_ray_tracing = st == RP_SUCCESS;
    return r;
}

RenderBuildResult build_metal_renderer(const RenderScene &scene, const std::filesystem::path &library,
                                       RenderTimings *) {
    return build_metal_renderer(scene, library);
}

RenderBuildResult build_metal_renderer(const RenderScene &scene, const std::filesystem::path &library,
                                       RenderBuildOptions options, RenderTimings *) {
    RenderBuildResult result = build_metal_renderer(scene, library);
    result.shadow_traversal.requested = options.shadow_traversal;
    result.acceleration_build.requested = options.acceleration_build_policy;
    result.acceleration_build.diagnostic = result.diagnostic;
    return result;
}

RenderSamplesResult MetalRenderScene::sample(const RenderRequest &request) {
    RenderSamplesResult out;
    const rp_request q = cuda_backend::request_of(request);
    const std::size_t lanes = std::size_t(q.pixel_count) * q.sample_count;
    char diag[1024] = {};
    if (impl_->scalar) { // RenderSample rows of rypath_render_paths (src/metal_render.mm:2136-2166)
        std::vector<rp_scalar_result> paths(lanes);
        const rp_status st = rp_cuda_sample_scalar(impl_->scene, &q, paths.data(), paths.size(), diag, sizeof diag);
        out.status = cuda_backend::status_of(st);
        out.diagnostic = diag;
        out.samples.reserve(lanes);
        for (const rp_scalar_result &l : paths)
            out.samples.push_back({l.pixel, (std::uint64_t(l.sample_high) << 32) | l.sample_low, l.wavelength,
                                   l.radiance, l.scatterings,
                                   {l.random_words[0], l.random_words[1], l.random_words[2], l.random_words[3]}});
        return out;
    }
    std::vector<rp_packet_result> results(lanes);
    const rp_status st = rp_cuda_sample(impl_->scene, &q, results.data(), results.size(), diag, sizeof diag);
    out.status = cuda_backend::status_of(st);
    out.diagnostic = diag;
    out.packet_samples.reserve(lanes);
    for (const rp_packet_result &l : results) { // decoded as src/metal_render.mm:2052-2100 does
        PacketSample p;
        p.pixel = l.pixel;
        p.sample = (std::uint64_t(l.sample_high) << 32) | l.sample_low;
        std::copy(l.wavelengths, l.wavelengths + 4, p.wavelengths.begin());
        std::copy(l.wavelength_pdfs, l.wavelength_pdfs + 4, p.wavelength_pdfs.begin());
        std::copy(l.radiance, l.radiance + 4, p.radiance.begin());
        p.filter_weight = l.filter_weight;
        p.splat_count = l.splat_count;
        out.packet_samples.push_back(p);
    }
    return out;
}

RenderSamplesResult MetalRenderScene::sample(const RenderRequest &request, RenderTimings &) {
    return sample(request);
}

ShadingNormalProbeResult probe_shading_normal(const std::vector<shading_normal_probe::Query> &,
                                              const std::filesystem::path &) {
    return {.status = MetalStatus::not_built,
            .diagnostic = "the CUDA backend has no shading-normal probe",
            .values = {},
            .guard_count = 0};
}

// ---- frame sessions (src/frame_session.hpp) over rp_cuda_frame_*: the independent estimator
// and the path tracer, rypath's FrameSession sampler (the independent sampler,
// src/metal_render.mm:4035).  A session and the frames it returns share one handle, so a Frame
// stays valid after its FrameSession is destroyed (src/frame_session.hpp:176-181).
namespace cuda_backend {
struct FrameHandle {
    rp_scene *scene = nullptr;
    rp_frame_session *session = nullptr;
    std::uint32_t width = 0, height = 0;
    ~FrameHandle() {
        rp_cuda_frame_session_destroy(session);
        rp_cuda_scene_destroy(scene);
    }
};
} // namespace cuda_backend

struct Frame::Impl {
    std::shared_ptr<cuda_backend::FrameHandle> handle;
    std::uint32_t slot = 0;
    ~Impl() { rp_cuda_frame_release(handle->session, slot); }
};
struct FrameSession::Impl {
    std::shared_ptr<cuda_backend::FrameHandle> handle;
};

namespace {
FrameInfo frame_info(const rp_frame_info &f) {
    FrameInfo info;
    info.width = f.width;
    info.height = f.height;
    info.sample_index = f.sample_index;
    info.epoch = f.epoch;
    info.status = f.status == RP_FRAME_PENDING    ? FrameStatus::pending
                  : f.status == RP_FRAME_COMPLETE ? FrameStatus::complete
                                                  : FrameStatus::failed;
    info.gpu_seconds = f.gpu_ms / 1e3;
    info.gpu_time_valid = f.status != RP_FRAME_PENDING;
    info.completed_samples = f.completed_samples;
    info.command_count = 1;
    if (f.status == RP_FRAME_FAILED)
        info.diagnostic = std::to_string(f.failed_pixels) + " pixel samples failed";
    return info;
}
} // namespace

Frame::Frame(std::shared_ptr<Impl> impl) : impl_(std::move(impl)) {}
Frame::~Frame() = default;
Frame::Frame(Frame &&) noexcept = default;
Frame &Frame::operator=(Frame &&) noexcept = default;
FrameInfo Frame::poll() const {
    rp_frame_info f{};
    if (rp_cuda_frame_poll(impl_->handle->session, impl_->slot, &f) != RP_SUCCESS)
        return {.status = FrameStatus::failed, .diagnostic = "CUDA frame poll failed"};
    return frame_info(f);
}
FrameInfo Frame::wait() const {
    rp_frame_info f{};
    if (rp_cuda_frame_wait(impl_->handle->session, impl_->slot, &f) != RP_SUCCESS)
        return {.status = FrameStatus::failed, .diagnostic = "CUDA frame wait failed"};
    return frame_info(f);
}
FrameCapture Frame::capture() const {
    FrameCapture out;
    const auto &h = *impl_->handle;
    out.width = h.width;
    out.height = h.height;
    out.raw_xyz.resize(std::size_t(h.width) * h.height);
    char diag[1024] = {};
    const rp_status st = rp_cuda_frame_capture(h.session, impl_->slot, out.raw_xyz.front().data(), out.raw_xyz.size(),
                                               diag, sizeof diag);
    out.status = cuda_backend::status_of(st);
    out.diagnostic = diag;
    return out;
}
FrameSession::FrameSession(std::unique_ptr<Impl> impl) : impl_(std::move(impl)) {}
FrameSession::~FrameSession() = default;
FrameSession::FrameSession(FrameSession &&) noexcept = default;
FrameSession &FrameSession::operator=(FrameSession &&) noexcept = default;
FrameSubmitResult FrameSession::submit(const FrameRequest &request) {
    FrameSubmitResult out;
    rp_camera camera{};
    rp_frame_request q{request.sample_index, request.epoch, nullptr};
    if (request.camera) {
        if (!request.camera->raster_camera) {
            out.status = GeometryStatus::not_built;
            out.diagnostic = "CUDA frame sessions take PBRT raster cameras";
            return out;
        }
        const RasterCamera &c = *request.camera->raster_camera;
        const GeometryPoint *points[4] = {&c.origin, &c.corner, &c.dx, &c.dy};
        float *dst[4] = {camera.origin, camera.corner, camera.dx, camera.dy};
        for (int k = 0; k < 4; ++k) {
            dst[k][0] = points[k]->x;
            dst[k][1] = points[k]->y;
            dst[k][2] = points[k]->z;
        }
        q.camera = &camera;
    }
    std::uint32_t slot = 0;
    int busy = 0;
    char diag[1024] = {};
    const rp_status st = rp_cuda_frame_submit(impl_->handle->session, &q, &slot, &busy, diag, sizeof diag);
    out.status = cuda_backend::status_of(st);
    out.busy = busy != 0;
    out.diagnostic = diag;
    if (st == RP_SUCCESS) {
        auto frame = std::make_shared<Frame::Impl>();
        frame->handle = impl_->handle;
        frame->slot = slot;
        out.frame.reset(new Frame(std::move(frame)));
    }
    return out;
}
FrameSessionBuildResult build_frame_session(const RenderScene &scene, const FrameConfig &config,
                                            const std::filesystem::path &) {
    FrameSessionBuildResult result;
    result.shadow_traversal.requested = config.shadow_traversal;
    result.acceleration_build.requested = config.acceleration_build_policy;
    auto handle = std::make_shared<cuda_backend::FrameHandle>();
    handle->width = config.width;
    handle->height = config.height;
    rp_status st = cuda_backend::create(scene, &handle->scene, result.diagnostic);
    if (st == RP_SUCCESS) {
        const std::vector<double> cie = cuda_backend::cie_rows();
        st = rp_cuda_set_cie(handle->scene, cie.data());
    }
    if (st == RP_SUCCESS) {
        rp_frame_config c{};
        c.width = config.width;
        c.height = config.height;
        c.seed = config.seed;
        c.sampler_kind = RP_SAMPLER_INDEPENDENT;
        c.footprint_samples = config.footprint_samples;
        char diag[1024] = {};
        st = rp_cuda_frame_session_create(handle->scene, &c, &handle->session, diag, sizeof diag);
        result.diagnostic = diag;
    }
    result.status = cuda_backend::status_of(st);
    result.acceleration_build.diagnostic = result.diagnostic;
    if (st == RP_SUCCESS) {
        auto impl = std::make_unique<FrameSession::Impl>();
        impl->handle = std::move(handle);
        result.session.reset(new FrameSession(std::move(impl)));
    }
    return result;
}

} // namespace rypath
