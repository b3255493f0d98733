// Test infrastructure only: rypath's demo model (`--render-demo`) compiled from the checkout
// (oracle/ref.mk) as a C ABI that pins the oracle and the backend: the demo scene itself
// (make_demo_scene, src/render.cpp:2060-2106), the demo film (FilmBatch with wavelength_xyz,
// src/render.cpp:2131-2145, :2355-2385), and rypath's CPU demo reference
// (tests/render_reference.cpp: analytic sky / floor moments and its own path estimator).
// src/render.cpp names two functions of rypath's PBRT translator for meshes with authored
// shading normals; the demo path never calls them, and this unit defines them as refusals so
// that the library links without the translator.
#include "render.hpp"
#include "render_reference.hpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <span>
#include <string>
#include <vector>

namespace rypath {
std::string prepare_shading_normals(const GeometryMesh &, const GeometryTransform &, bool,
                                    std::vector<GeometryPoint> &) {
    return "shading normals are not part of the demo pin";
}
std::string validate_normal_emission(const GeometryMesh &, const GeometryTransform &, bool, bool,
                                     std::span<const GeometryPoint>) {
    return "shading normals are not part of the demo pin";
}
} // namespace rypath

extern "C" {

// make_demo_scene's data: counts[0..3] = meshes, total vertices, total triangles, instances.
// Per mesh its first vertex and triangle (mesh_begin, 2 words each); positions (3 floats per
// vertex), triangles (3 words, mesh-local), per instance its mesh and 12 transform floats,
// per instance its material, per material 8 reflectances; camera = origin, target, up, fov;
// max depth.  Returns 0, or -1 when a capacity is too small.
int ref_demo_scene(uint32_t *counts, uint32_t *mesh_begin, float *positions, uint32_t *triangles,
                   uint32_t *instance_mesh, float *instance_transform, uint32_t *instance_material,
                   float *reflectance, float *camera, uint32_t *max_depth, uint32_t capacity) {
    const rypath::RenderScene s = rypath::make_demo_scene();
    uint32_t v = 0, t = 0;
    for (std::size_t m = 0; m < s.geometry.meshes.size(); ++m) {
        const auto &mesh = s.geometry.meshes[m];
        if (v + mesh.positions.size() > capacity || t + mesh.triangles.size() > capacity)
            return -1;
        mesh_begin[2 * m] = v;
        mesh_begin[2 * m + 1] = t;
        for (const auto &p : mesh.positions) {
            positions[3 * v] = p.x;
            positions[3 * v + 1] = p.y;
            positions[3 * v + 2] = p.z;
            ++v;
        }
        for (const auto &tri : mesh.triangles) {
            std::copy(tri.begin(), tri.end(), triangles + 3 * t);
            ++t;
        }
    }
    for (std::size_t i = 0; i < s.geometry.instances.size(); ++i) {
        instance_mesh[i] = s.geometry.instances[i].mesh_index;
        std::copy(s.geometry.instances[i].transform.values.begin(), s.geometry.instances[i].transform.values.end(),
                  instance_transform + 12 * i);
        instance_material[i] = s.instance_materials[i];
    }
    for (std::size_t m = 0; m < s.materials.size(); ++m)
        std::copy(s.materials[m].reflectance.begin(), s.materials[m].reflectance.end(), reflectance + 8 * m);
    const rypath::RenderCamera &c = s.camera;
    const float cam[10] = {c.origin.x, c.origin.y, c.origin.z, c.target.x, c.target.y,
                           c.target.z, c.up.x,     c.up.y,     c.up.z,     c.vertical_fov_degrees};
    std::memcpy(camera, cam, sizeof(cam));
    counts[0] = uint32_t(s.geometry.meshes.size());
    counts[1] = v;
    counts[2] = t;
    counts[3] = uint32_t(s.geometry.instances.size());
    *max_depth = s.max_depth;
    return 0;
}

// The demo film of scalar samples (pixel, sample, wavelength, radiance per row; 4 words), one
// FilmBatch of `samples` samples per pixel; per pixel out: sum[3], correction[3], count.
// Returns 0, or 1 when rypath's FilmBatch refuses the samples.
int ref_demo_film(const float *rows, uint32_t count, uint32_t width, uint32_t height, uint32_t samples,
                  double *out) {
    rypath::Film film = rypath::make_film(width, height);
    rypath::FilmBatch batch(film, samples);
    std::vector<rypath::RenderSample> v(count);
    for (uint32_t i = 0; i < count; ++i) {
        uint32_t pixel, sample;
        std::memcpy(&pixel, rows + 4 * i, 4);
        std::memcpy(&sample, rows + 4 * i + 1, 4);
        v[i].pixel = pixel;
        v[i].sample = sample;
        v[i].wavelength = rows[4 * i + 2];
        v[i].radiance = rows[4 * i + 3];
    }
    if (!batch.add(v).empty() || !batch.commit(film).empty())
        return 1;
    for (std::size_t p = 0; p < film.pixels.size(); ++p) {
        const auto &f = film.pixels[p];
        for (int c = 0; c < 3; ++c) {
            out[7 * p + c] = f.sum[c];
            out[7 * p + 3 + c] = f.correction[c];
        }
        out[7 * p + 6] = double(f.count);
    }
    return 0;
}

// analytic_xyz (tests/render_reference.cpp): mean[3] and variance[3] of the demo sky
// (reflectance null) or of the unobstructed Lambertian floor with the 8 given reflectances.
void ref_demo_analytic(const float *reflectance, double *out) {
    rypath::SpectralMaterial m{};
    if (reflectance)
        std::copy(reflectance, reflectance + 8, m.reflectance.begin());
    const auto moments = rypath::test::analytic_xyz(reflectance ? &m : nullptr);
    for (int c = 0; c < 3; ++c) {
        out[c] = moments.mean[c];
        out[3 + c] = moments.variance[c];
    }
}

// rypath's CPU demo estimator (reference_image) on make_demo_scene: mean XYZ over the image
// and the largest scattering count.
void ref_demo_reference_image(uint32_t width, uint32_t height, uint64_t samples, uint64_t seed, double *out) {
    rypath::RenderSettings settings;
    settings.width = width;
    settings.height = height;
    settings.samples = samples;
    settings.batch_size = samples;
    settings.seed = seed;
    const auto image = rypath::test::reference_image(rypath::make_demo_scene(), settings);
    for (int c = 0; c < 3; ++c)
        out[c] = image.mean[c];
    out[3] = double(image.max_scatterings);
}

} // extern "C"
