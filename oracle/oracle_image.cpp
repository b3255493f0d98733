// ORACLE -- test infrastructure only (see oracle_math.hpp).  Scene-build side of the images:
// copying a description's images, the environment importance tables and the environment's
// light power.
#include "oracle_image.hpp"
#include "oracle_scene.hpp"
#include "oracle.h"

namespace oracle {
namespace {

// src/image_texture.cpp:1324-1332 (image_base_texel_linear_rgb): the decoded texel, or
// nothing when a channel is not finite
bool base_texel(const Images &im, const rp_image_texture &t, u32 x, u32 y, Rgb &out) {
    out = image_texel(im, im.levels[t.level_begin], int(x), int(y), RP_WRAP_CLAMP, t.texel_format, t.transfer_offset);
    return finite_rgb(out);
}
// src/rgb_spectrum.cpp:62-107 (reconstruct_srgb) and :109-127 (evaluate_srgb)
bool reconstruct_evaluate(const float *table, const float rgb[3], float wavelength, float &value) {
    for (int c = 0; c < 3; ++c)
        if (!std::isfinite(rgb[c]) || rgb[c] < 0 || rgb[c] > 1)
            return false;
    if (rgb[0] == rgb[1] && rgb[1] == rgb[2]) {
        value = rgb[0];
        return true;
    }
    int maxc = 0;
    for (int c = 1; c < 3; ++c)
        if (rgb[c] >= rgb[maxc])
            maxc = c;
    const float z = rgb[maxc];
    const float x = rgb[(maxc + 1) % 3] * 63 / z;
    const float y = rgb[(maxc + 2) % 3] * 63 / z;
    const int xi = std::min(int(x), 62), yi = std::min(int(y), 62);
    const int zi = int(std::lower_bound(table + 1, table + 63, z) - table) - 1;
    const float dx = x - float(xi), dy = y - float(yi);
    const float dz = (z - table[zi]) / (table[zi + 1] - table[zi]);
    const auto lerp = [](float t, float a, float b) { return (1.0f - t) * a + t * b; };
    float co[3];
    for (int i = 0; i < 3; ++i) {
        const auto at = [&](int ox, int oy, int oz) {
            const int plane = maxc * 64 + zi + oz, row = plane * 64 + yi + oy, cell = row * 64 + xi + ox;
            return table[64 + 3 * cell + i];
        };
        co[i] = lerp(dz, lerp(dy, lerp(dx, at(0, 0, 0), at(1, 0, 0)), lerp(dx, at(0, 1, 0), at(1, 1, 0))),
                     lerp(dy, lerp(dx, at(0, 0, 1), at(1, 0, 1)), lerp(dx, at(0, 1, 1), at(1, 1, 1))));
    }
    const float p = std::fma(wavelength, std::fma(wavelength, co[0], co[1]), co[2]);
    if (!std::isfinite(p)) {
        value = NAN;
        return true;
    }
    if (std::abs(p) <= 1.0f) {
        value = 0.5f + 0.5f * (p / std::sqrt(1.0f + p * p));
    } else {
        const float r = 1.0f / p;
        value = 0.5f + 0.5f * std::copysign(1.0f / std::sqrt(1.0f + r * r), p);
    }
    return true;
}
// src/light_sampling.cpp:28-44 (light_rgb_power)
bool rgb_power(const Images &im, Rgb c, double &value) {
    const float amplitude = 2 * std::max({c.r, c.g, c.b});
    value = 0;
    if (amplitude == 0)
        return true;
    if (!std::isfinite(amplitude))
        return false;
    const float n[3] = {c.r / amplitude, c.g / amplitude, c.b / amplitude};
    for (float v : n)
        if (!(v >= 0 && v <= 1))
            return false;
    const Wavelengths l = packet_sample_visible(.5f);
    for (int i = 0; i < 4; ++i) {
        const unsigned w = unsigned(std::round(l.lambda[i]) - 360);
        float s = 0;
        reconstruct_evaluate(im.rgb_table.data(), n, float(w + 360), s);
        value += double(amplitude) * s * im.illuminant[w] / l.pdf[i] / 4;
    }
    return true;
}

} // namespace

std::string build_environment_tables(Images &im) {
    const rp_image_texture &t = im.textures[im.env_image];
    const rp_texture_level &l = im.levels[t.level_begin];
    if (t.level_count != 1 || l.width != l.height)
        return "Environment sampling requires a square native image base";
    const u32 width = l.width;
    const size_t side = size_t(width) + 1;
    im.env_width = width;
    im.env_comp_offset = u32(side * side);
    im.env_cdf.assign(2 * side * side, 0.f);
    const auto mass = [&](u32 x, u32 y, double &out) {
        Rgb c;
        if (!base_texel(im, t, x, y, c))
            return false;
        out = (double(std::max(c.r, 0.f)) + double(std::max(c.g, 0.f)) + double(std::max(c.b, 0.f))) / 3;
        return true;
    };
    std::vector<double> full_rows(width), comp_rows(width), full_prefix(side), comp_prefix(side);
    double total = 0, power = 0;
    for (u32 y = 0; y < width; ++y) {
        double row = 0;
        for (u32 x = 0; x < width; ++x) {
            double v;
            if (!mass(x, y, v))
                return "Environment sampling texel is invalid";
            row += v;
            Rgb c;
            base_texel(im, t, x, y, c);
            double p;
            if (!rgb_power(im, c, p))
                return "Invalid environment light sampling image";
            power += p;
        }
        full_rows[y] = row;
        total += row;
    }
    im.env_power = power / (double(width) * width);
    const double average = total / (double(width) * width);
    const auto write_prefix = [&](size_t offset, const std::vector<double> &prefix, double sum) {
        for (u32 x = 1; x <= width; ++x)
            im.env_cdf[offset + x] = sum > 0 ? float(prefix[x] / sum) : float(x) / float(width);
        im.env_cdf[offset + width] = 1.f;
    };
    double comp_total = 0;
    for (u32 y = 0; y < width; ++y) {
        full_prefix[0] = comp_prefix[0] = 0;
        for (u32 x = 0; x < width; ++x) {
            double v = 0;
            mass(x, y, v);
            full_prefix[x + 1] = full_prefix[x] + v;
            comp_prefix[x + 1] = comp_prefix[x] + std::max(v - average, 0.);
        }
        comp_rows[y] = comp_prefix.back();
        comp_total += comp_rows[y];
        write_prefix(side * (y + 1), full_prefix, full_rows[y]);
        write_prefix(im.env_comp_offset + side * (y + 1), comp_prefix, comp_rows[y]);
    }
    double full_sum = 0, comp_sum = 0;
    for (u32 y = 0; y < width; ++y) {
        full_sum += full_rows[y];
        comp_sum += comp_rows[y];
        im.env_cdf[y + 1] = total > 0 ? float(full_sum / total) : float(y + 1) / float(width);
        im.env_cdf[im.env_comp_offset + y + 1] =
            comp_total > 0 ? float(comp_sum / comp_total) : float(y + 1) / float(width);
    }
    im.env_cdf[width] = im.env_cdf[im.env_comp_offset + width] = 1.f;
    return {};
}

std::string load_images(const rp_images *in, Images &out) {
    out = Images{};
    if (!in)
        return {};
    out.textures.assign(in->textures, in->textures + in->texture_count);
    out.levels.assign(in->levels, in->levels + in->level_count);
    out.texels.assign(in->texels, in->texels + in->texel_word_count);
    out.transfer.assign(in->transfer, in->transfer + in->transfer_count);
    if (in->texture_count) {
        if (!in->rgb_table || !in->illuminant)
            return "images need the sRGB reconstruction table and the D65 illuminant";
        out.rgb_table.assign(in->rgb_table, in->rgb_table + RP_RGB_TABLE_FLOATS);
        out.illuminant.assign(in->illuminant, in->illuminant + 471);
    }
    if (in->environment_image != RP_NONE) {
        if (in->environment_image >= in->texture_count)
            return "environment image out of range";
        out.env_image = in->environment_image;
        out.env_scale = in->environment_scale;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                out.env_from_world[3 * r + c] = in->environment_from_world[3 * r + c];
                out.world_from_env[3 * c + r] = in->environment_from_world[3 * r + c];
            }
        const std::string err = build_environment_tables(out);
        if (!err.empty())
            return err;
    }
    return {};
}

} // namespace oracle

namespace {
oracle::Images probe_images(const void *textures, uint32_t texture_count, const void *levels, uint32_t level_count,
                            const uint32_t *texels, uint32_t words, const float *transfer, uint32_t transfer_count) {
    oracle::Images im;
    const auto *t = static_cast<const rp_image_texture *>(textures);
    const auto *l = static_cast<const rp_texture_level *>(levels);
    im.textures.assign(t, t + texture_count);
    im.levels.assign(l, l + level_count);
    im.texels.assign(texels, texels + words);
    im.transfer.assign(transfer, transfer + transfer_count);
    return im;
}
} // namespace

extern "C" {

void or_image_lookup(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                     uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                     uint32_t transfer_count, const float *q, uint32_t count, float *out) {
    const oracle::Images im =
        probe_images(textures, texture_count, levels, level_count, texels, words, transfer, transfer_count);
    const rp_image_texture &t = im.textures[index];
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 6 * i;
        float *o = out + 4 * i;
        const oracle::F2 uv{a[0], a[1]}, dx{a[2], a[3]}, dy{a[4], a[5]};
        const oracle::Rgb c = oracle::image_lookup_standard(im, t, uv, dx, dy, false, false);
        o[0] = c.r;
        o[1] = c.g;
        o[2] = c.b;
        o[3] = oracle::image_lookup_standard(im, t, uv, dx, dy, true, false).r;
    }
}

void or_rgb_spectrum(const float *table, const float *q, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 4 * i;
        const oracle::Rgb c{a[0], a[1], a[2]};
        out[2 * i] = oracle::srgb_spectrum(table, c, a[3]);
        out[2 * i + 1] = oracle::srgb_spectrum_unbounded(table, c, a[3]);
    }
}

int or_environment_tables(const void *textures, uint32_t index, const void *levels, const uint32_t *texels,
                          uint32_t words, const float *transfer, const float *table, const float *illuminant,
                          float *cdf, size_t capacity, uint32_t *width, uint32_t *compensated_offset,
                          double *power) {
    const auto *t = static_cast<const rp_image_texture *>(textures);
    oracle::Images im = probe_images(textures, index + 1, levels, t[index].level_begin + t[index].level_count, texels,
                                     words, transfer, transfer ? t[index].transfer_offset + 256 : 0);
    im.rgb_table.assign(table, table + RP_RGB_TABLE_FLOATS);
    im.illuminant.assign(illuminant, illuminant + 471);
    im.env_image = index;
    if (!oracle::build_environment_tables(im).empty() || im.env_cdf.size() > capacity)
        return -1;
    std::copy(im.env_cdf.begin(), im.env_cdf.end(), cdf);
    *width = im.env_width;
    *compensated_offset = im.env_comp_offset;
    *power = im.env_power;
    return 0;
}

void or_environment_queries(const void *textures, uint32_t texture_count, uint32_t index, const void *levels,
                            uint32_t level_count, const uint32_t *texels, uint32_t words, const float *transfer,
                            uint32_t transfer_count, const float *table, const float *illuminant, const float *cdf,
                            uint32_t cdf_count, uint32_t width, uint32_t compensated_offset, float scale,
                            const float *env_from_world, const float *q, uint32_t count, float *out) {
    oracle::Images im =
        probe_images(textures, texture_count, levels, level_count, texels, words, transfer, transfer_count);
    im.rgb_table.assign(table, table + RP_RGB_TABLE_FLOATS);
    im.illuminant.assign(illuminant, illuminant + 471);
    im.env_image = index;
    im.env_scale = scale;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            im.env_from_world[3 * r + c] = env_from_world[3 * r + c];
            im.world_from_env[3 * c + r] = env_from_world[3 * r + c];
        }
    im.env_cdf.assign(cdf, cdf + cdf_count);
    im.env_width = width;
    im.env_comp_offset = compensated_offset;
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 8 * i;
        float *o = out + 12 * i;
        const oracle::F3 d{a[0], a[1], a[2]};
        o[0] = oracle::env_image_radiance(im, d, a[3]);
        o[1] = oracle::env_image_pdf(im, d, true);
        o[2] = oracle::env_image_pdf(im, d, false);
        oracle::F3 w;
        float pdf = 0;
        o[3] = oracle::env_image_sample(im, a[4], a[5], true, w, pdf) ? 1.f : 0.f;
        o[4] = w.x;
        o[5] = w.y;
        o[6] = w.z;
        o[7] = pdf;
        oracle::F3 w2;
        float pdf2 = 0;
        o[8] = oracle::env_image_sample(im, a[4], a[5], false, w2, pdf2) ? 1.f : 0.f;
        o[9] = w2.x;
        o[10] = w2.y;
        o[11] = w2.z;
    }
}

} // extern "C"
