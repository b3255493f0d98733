// Test infrastructure only: rypath's host image sources (src/image_texture.cpp,
// src/environment_sampling.cpp, src/rgb_spectrum.cpp, src/light_sampling.cpp) compiled where
// they lie (oracle/ref.mk) as a C ABI that pins the oracle's restatement.  The code of this
// file is only the marshalling.  rgb_spectrum.cpp reads its table through
// rypath::detail::srgb_table_bytes, which rypath's build generates from
// third_party/pbrt/srgb.bin; here it returns the bytes of that file, read once.
#include "environment_sampling.hpp"
#include "image_texture.hpp"
#include "light_sampling.hpp"
#include "render_wire.h"
#include "rgb_spectrum.hpp"
#include "texture_footprint.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#ifndef RYPATH_SRGB_BIN
#error "RYPATH_SRGB_BIN must name third_party/pbrt/srgb.bin of the rypath checkout"
#endif

namespace rypath::detail {
const char *srgb_table_bytes(std::size_t offset) {
    static const std::vector<char> bytes = [] {
        std::vector<char> b;
        if (FILE *f = std::fopen(RYPATH_SRGB_BIN, "rb")) {
            char chunk[65536];
            std::size_t n;
            while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0)
                b.insert(b.end(), chunk, chunk + n);
            std::fclose(f);
        }
        return b;
    }();
    return bytes.data() + offset;
}
} // namespace rypath::detail

namespace {
namespace wire = rypath::render_wire;

// An ImagePyramid over one texture's wire levels (src/image_texture.hpp:66-77)
std::shared_ptr<rypath::ImagePyramid> pyramid(const wire::ImageTexture &t, const wire::TextureLevel *levels,
                                              const uint32_t *texels, uint32_t words, const float *transfer,
                                              bool native) {
    auto p = std::make_shared<rypath::ImagePyramid>();
    p->encoding = t.texel_format == wire::srgb8_texel_format ? rypath::ImageEncoding::srgb
                                                              : rypath::ImageEncoding::linear;
    p->wrap = t.wrap == 0 ? rypath::ImageWrap::repeat : t.wrap == 1 ? rypath::ImageWrap::clamp : rypath::ImageWrap::black;
    const uint32_t per = t.texel_format == wire::linear_float_texel_format  ? 4u
                         : t.texel_format == wire::linear_half_texel_format ? 2u
                                                                            : 1u;
    uint32_t base = levels[t.level_begin].offset, end = base;
    for (uint32_t k = 0; k < t.level_count; ++k) {
        const auto &l = levels[t.level_begin + k];
        p->levels.push_back({l.width, l.height, l.offset - base});
        end = std::max(end, l.offset + l.width * l.height * per);
    }
    p->texels.assign(texels + base, texels + std::min(end, words));
    p->storage = t.texel_format == wire::linear_float_texel_format  ? rypath::ImageStorage::linear_float
                 : t.texel_format == wire::linear_half_texel_format ? rypath::ImageStorage::linear_half
                                                                    : rypath::ImageStorage::encoded8;
    p->source_channels = t.channels;
    if (p->storage == rypath::ImageStorage::encoded8) {
        auto table = std::make_shared<std::array<float, 256>>();
        std::memcpy(table->data(), transfer + t.transfer_offset, 256 * sizeof(float));
        p->custom_transfer = table;
    }
    p->native_base = native;
    return p;
}
rypath::ImageFilter host_filter(uint32_t f) {
    return f == 1 ? rypath::ImageFilter::trilinear
           : f == 2 ? rypath::ImageFilter::point
           : f == 3 ? rypath::ImageFilter::ewa
                    : rypath::ImageFilter::bilinear;
}
} // namespace

extern "C" {

// Host texture lookups (image_linear_rgb, src/image_texture.cpp:1301-1310) of texture `index`:
// per query 6 floats {u, v, dudx, dvdx, dudy, dvdy} -> 4 floats {rgb[3], valid}.
void ref_host_image_lookup(const void *textures, uint32_t index, const void *levels, const uint32_t *texels,
                           uint32_t words, const float *transfer, const float *q, uint32_t count, float *out) {
    const auto *t = static_cast<const wire::ImageTexture *>(textures);
    const auto image = pyramid(t[index], static_cast<const wire::TextureLevel *>(levels), texels, words, transfer, false);
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 6 * i;
        float *o = out + 4 * i;
        const auto host = rypath::image_linear_rgb(*image, a[0], a[1], a[2], a[3], a[4], a[5],
                                                   host_filter(t[index].filter), t[index].max_anisotropy);
        o[0] = host ? (*host)[0] : 0;
        o[1] = host ? (*host)[1] : 0;
        o[2] = host ? (*host)[2] : 0;
        o[3] = host ? 1.f : 0.f;
    }
}

// Host RGB reconstruction (reconstruct_srgb + evaluate_srgb, evaluate_unbounded_srgb;
// src/rgb_spectrum.cpp:62-145): per query {r, g, b, wavelength} -> {bounded, unbounded}, NaN
// where rypath refuses the input.
void ref_host_rgb_spectrum(const float *q, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 4 * i;
        const auto r = rypath::reconstruct_srgb({a[0], a[1], a[2]});
        out[2 * i] = r ? rypath::evaluate_srgb(*r, a[3]) : NAN;
        const auto u = rypath::evaluate_unbounded_srgb({a[0], a[1], a[2]}, a[3]);
        out[2 * i + 1] = u ? *u : NAN;
    }
}

// The environment tables of a square one-level image (texture `index`):
// build_environment_sampling (src/environment_sampling.cpp:20-115) into cdf (2 (w+1)^2
// floats) and light_image_power (src/light_sampling.cpp:78-95); returns 0, or -1 without tables.
int ref_environment_tables(const void *textures, uint32_t index, const void *levels, const uint32_t *texels,
                           uint32_t words, const float *transfer, float *cdf, size_t capacity, uint32_t *width,
                           uint32_t *compensated_offset, double *power) {
    const auto *t = static_cast<const wire::ImageTexture *>(textures);
    const auto image = pyramid(t[index], static_cast<const wire::TextureLevel *>(levels), texels, words, transfer, true);
    std::string diagnostic;
    const auto tables = rypath::build_environment_sampling(*image, SIZE_MAX, diagnostic);
    if (!tables || tables->cdf.size() > capacity)
        return -1;
    std::copy(tables->cdf.begin(), tables->cdf.end(), cdf);
    *width = tables->width;
    *compensated_offset = tables->compensated_offset;
    const auto p = rypath::light_image_power(*image);
    *power = p ? *p : -1;
    return 0;
}

// prepare_texture_camera_differentials (src/texture_footprint.cpp:199-232): the raster corner
// and full-extent steps of a PBRT camera and the film size -> minimum dx[3], dy[3]; 0, or -1
// with rypath's diagnostic refused.
int ref_texture_camera_differentials(const float *corner, const float *dx, const float *dy, uint32_t width,
                                     uint32_t height, float *out) {
    rypath::TextureCameraDifferentials d;
    const std::string err = rypath::prepare_texture_camera_differentials(
        {corner[0], corner[1], corner[2]}, {dx[0], dx[1], dx[2]}, {dy[0], dy[1], dy[2]}, width, height, d);
    if (!err.empty())
        return -1;
    const float v[6] = {d.minimum_dx.x, d.minimum_dx.y, d.minimum_dx.z, d.minimum_dy.x, d.minimum_dy.y, d.minimum_dy.z};
    std::memcpy(out, v, sizeof(v));
    return 0;
}

} // extern "C"
