// Test infrastructure only: rypath's image shader headers (shaders/image_texture.h,
// shaders/image_lighting.h, shaders/texture_footprint.h) compiled from the checkout (oracle/ref.mk), behind the host
// stand-in for <metal_stdlib>, as a C ABI that pins the oracle's restatement.  The code of this file is
// only the marshalling: wire records in, results out.  rypath's host image sources are bound in
// ref_image_host.cpp (a separate unit: the stand-in's address-space macros would rewrite
// their identifiers).
#include <metal_stdlib>
// Metal's read-only constant address space, in C++ terms (oracle/ref.mk gives this unit a
// copy of image_lighting.h whose `const constant` reads `const`)
#undef constant
#define constant const
#include "render_wire.h"
#include "image_lighting.h"
#include "texture_footprint.h"

#include <cstdint>

namespace {
namespace wire = rypath::render_wire;
static_assert(sizeof(wire::ImageTexture) == 72 && sizeof(wire::TextureLevel) == 12);

wire::TextureParameters texture_parameters(uint32_t textures, uint32_t levels, uint32_t words, uint32_t transfer) {
    wire::TextureParameters p{};
    p.texture_count = textures;
    p.level_count = levels;
    p.texel_word_count = words;
    p.transfer_count = transfer;
    return p;
}
} // namespace

extern "C" {

// Texture lookups of texture `index` of the wire arrays through rypath_image::lookup and
// lookup_scalar (shaders/image_texture.h:556-575): per query 6 floats {u, v, dudx, dvdx, dudy,
// dvdy} -> 4 floats {rgb[3], scalar}.
void ref_image_lookup(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                      uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                      uint32_t transfer_count, const float *q, uint32_t count, float *out) {
    const auto *t = static_cast<const wire::ImageTexture *>(textures);
    const auto *l = static_cast<const wire::TextureLevel *>(levels);
    const wire::TextureParameters p = texture_parameters(texture_count, level_count, words, transfer_count);
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 6 * i;
        float *o = out + 4 * i;
        const float2 uv(a[0], a[1]), dx(a[2], a[3]), dy(a[4], a[5]);
        const float3 rgb = rypath_image::lookup(t[index], l, texels, transfer, p, uv, dx, dy);
        o[0] = rgb.x;
        o[1] = rgb.y;
        o[2] = rgb.z;
        o[3] = rypath_image::lookup_scalar(t[index], l, texels, transfer, p, uv, dx, dy);
    }
}

// RGB reconstruction through rypath_image::spectrum and unbounded_spectrum
// (shaders/image_texture.h:458-507): per query 4 floats {r, g, b, wavelength} -> 2 floats
// {bounded, unbounded}.
void ref_rgb_spectrum(const float *table, const float *q, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 4 * i;
        const float3 rgb(a[0], a[1], a[2]);
        out[2 * i] = rypath_image::spectrum(rgb, a[3], table);
        out[2 * i + 1] = rypath_image::unbounded_spectrum(rgb, a[3], table);
    }
}

// Environment queries through shaders/image_lighting.h with the given tables: per query 8
// floats {direction[3], wavelength, u[2], unused[2]} -> 12 floats {radiance, pdf (compensated),
// pdf (full), sample ok, sampled direction[3], sample pdf, full-table sample ok, direction[3]}.
void ref_environment_queries(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                             uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                             uint32_t transfer_count, const float *table, const float *illuminant, const float *cdf,
                             uint32_t cdf_count, uint32_t width, uint32_t compensated_offset, float scale,
                             const float *env_from_world, const float *q, uint32_t count, float *out) {
    const wire::TextureParameters tp = texture_parameters(texture_count, level_count, words, transfer_count);
    const rypath_image_light::Images images{static_cast<const wire::ImageTexture *>(textures),
                                            static_cast<const wire::TextureLevel *>(levels),
                                            texels,
                                            transfer,
                                            table,
                                            illuminant,
                                            &tp};
    wire::TextureGraphParameters gp{};
    gp.environment_image = index;
    gp.environment_scale = scale;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            gp.environment_from_world[3 * r + c] = env_from_world[3 * r + c];
            gp.world_from_environment[3 * c + r] = env_from_world[3 * r + c];
        }
    gp.environment_width = width;
    gp.environment_cdf_count = cdf_count;
    gp.environment_compensated_offset = compensated_offset;
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 8 * i;
        float *o = out + 12 * i;
        const float3 d(a[0], a[1], a[2]);
        o[0] = rypath_image_light::environment_radiance(images, gp, d, a[3]);
        o[1] = rypath_image_light::environment_pdf(gp, cdf, d, true);
        o[2] = rypath_image_light::environment_pdf(gp, cdf, d, false);
        float3 w(0);
        float pdf = 0;
        const bool ok = rypath_image_light::sample_environment(gp, cdf, float2(a[4], a[5]), w, pdf, true);
        o[3] = ok ? 1.f : 0.f;
        o[4] = w.x;
        o[5] = w.y;
        o[6] = w.z;
        o[7] = pdf;
        float3 w2(0);
        float pdf2 = 0;
        o[8] = rypath_image_light::sample_environment(gp, cdf, float2(a[4], a[5]), w2, pdf2, false) ? 1.f : 0.f;
        o[9] = w2.x;
        o[10] = w2.y;
        o[11] = w2.z;
    }
}

// Texture footprints through shaders/texture_footprint.h: per query 48 floats {relative p[3],
// n[3], ray direction[3], x ray[3], y ray[3], spp scale, world_from_camera[9] (row-major),
// camera_from_world[9], minimum dx[3], minimum dy[3], dpdu[3], dpdv[3], unused[2]} -> 24
// floats {primary ok, primary dpdx[3], dpdy[3], approximate dpdx[3], dpdy[3], derivatives ok,
// dstdx[2], dstdy[2] (of the primary footprint when it exists, else the approximate one),
// texture direction of the x ray[3], unused[3]}.
void ref_texture_footprint(const float *q, uint32_t count, float *out) {
    const auto matrix = [](const float *m) {
        return float3x3(float3(m[0], m[3], m[6]), float3(m[1], m[4], m[7]), float3(m[2], m[5], m[8]));
    };
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 48 * i;
        float *o = out + 24 * i;
        const float3 rp(a[0], a[1], a[2]), n(a[3], a[4], a[5]), d(a[6], a[7], a[8]);
        const float3 rx(a[9], a[10], a[11]), ry(a[12], a[13], a[14]);
        float3 pdx(0), pdy(0), adx(0), ady(0);
        const bool primary = rypath_texture_primary_dp(rp, n, d, rx, ry, a[15], pdx, pdy);
        rypath_texture_approximate_dp(rp, n, matrix(a + 16), matrix(a + 25), float3(a[34], a[35], a[36]),
                                      float3(a[37], a[38], a[39]), a[15], adx, ady);
        float2 sx(0), sy(0);
        const bool ok = rypath_texture_uv_derivatives(float3(a[40], a[41], a[42]), float3(a[43], a[44], a[45]),
                                                      primary ? pdx : adx, primary ? pdy : ady, sx, sy);
        const float3 td = rypath_texture_direction(rx);
        const float v[24] = {primary ? 1.f : 0.f, pdx.x, pdx.y, pdx.z, pdy.x, pdy.y, pdy.z, adx.x, adx.y, adx.z,
                             ady.x, ady.y, ady.z, ok ? 1.f : 0.f, sx.x, sx.y, sy.x, sy.y, td.x, td.y, td.z, 0, 0, 0};
        for (int k = 0; k < 24; ++k)
            o[k] = v[k];
    }
}

} // extern "C"
