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

std::string texture_camera_differentials(F3 corner, F3 dx, F3 dy, u32 width, u32 height, F3 &min_dx, F3 &min_dy) {
    if (width == 0 || height == 0)
        return "Texture camera raster extent must be positive";
    using V = std::array<double, 3>;
    const V c{corner.x, corner.y, corner.z}, u{dx.x, dx.y, dx.z}, v{dy.x, dy.y, dy.z};
    const auto dotd = [](const V &a, const V &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const auto unit = [](V a, V &out) {
        const double len = std::hypot(a[0], a[1], a[2]);
        if (!(len > 0 && std::isfinite(len)))
            return false;
        for (auto &x : a)
            x /= len;
        out = a;
        return true;
    };
    const auto direction = [&](double x, double y, V &out) {
        V d;
        for (int i = 0; i < 3; ++i) {
            d[i] = std::fma(y, v[i], std::fma(x, u[i], c[i]));
            if (!(std::abs(d[i]) <= double(FLT_MAX)))
                return false;
        }
        return unit(d, out);
    };
    const double px = 1. / width, py = 1. / height;
    V best_x{}, best_y{};
    double len_x = INFINITY, len_y = INFINITY;
    for (unsigned i = 0; i < 512; ++i) {
        const double t = double(i) / 511;
        V d, xr, yr;
        if (!direction(t, t, d) || !direction(t + px, t, xr) || !direction(t, t + py, yr))
            return "Texture camera differential ray is unrepresentable or zero";
        // PBRT's CoordinateSystem of the ray direction (Duff et al. 2017)
        const double sign = std::copysign(1., d[2]);
        const double a = -1 / (sign + d[2]);
        const double b = d[0] * d[1] * a;
        const V b0{1 + sign * d[0] * d[0] * a, sign * b, -sign * d[0]}, b1{b, sign + d[1] * d[1] * a, -d[1]};
        const auto local = [&](const V &r) { return V{dotd(b0, r), dotd(b1, r), dotd(d, r)}; };
        const V base = local(d);
        V lx, ly;
        if (!unit(local(xr), lx) || !unit(local(yr), ly))
            return "Texture camera differential ray collapses in its local frame";
        const V ex{lx[0] - base[0], lx[1] - base[1], lx[2] - base[2]}, ey{ly[0] - base[0], ly[1] - base[1], ly[2] - base[2]};
        if (dotd(ex, ex) < len_x) {
            len_x = dotd(ex, ex);
            best_x = ex;
        }
        if (dotd(ey, ey) < len_y) {
            len_y = dotd(ey, ey);
            best_y = ey;
        }
    }
    min_dx = {float(best_x[0]), float(best_x[1]), float(best_x[2])};
    min_dy = {float(best_y[0]), float(best_y[1]), float(best_y[2])};
    return {};
}

std::string load_images(const rp_images *in, u32 instance_count, Images &out) {
    out = Images{};
    if (!in)
        return {};
    for (u32 i = 0; i < in->uv_count; ++i)
        out.uvs.push_back({in->uvs[2 * i], in->uvs[2 * i + 1]});
    for (u32 i = 0; i < in->frame_count; ++i) {
        const float *f = in->frames + 6 * i;
        out.frames.push_back({F3{f[0], f[1], f[2]}, F3{f[3], f[4], f[5]}});
    }
    out.inst_uv_begin.assign(instance_count, RP_NONE);
    out.inst_frame_begin.assign(instance_count, RP_NONE);
    if (in->instance_uv_begin)
        out.inst_uv_begin.assign(in->instance_uv_begin, in->instance_uv_begin + instance_count);
    if (in->instance_frame_begin)
        out.inst_frame_begin.assign(in->instance_frame_begin, in->instance_frame_begin + instance_count);
    std::copy(in->world_from_camera, in->world_from_camera + 9, out.world_from_camera);
    std::copy(in->camera_from_world, in->camera_from_world + 9, out.camera_from_world);
    if (in->ewa_weights)
        out.ewa_weights.assign(in->ewa_weights, in->ewa_weights + 128);
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
                     uint32_t transfer_count, const float *q, uint32_t count, float *out, const float *ewa_weights) {
    oracle::Images im =
        probe_images(textures, texture_count, levels, level_count, texels, words, transfer, transfer_count);
    if (ewa_weights)
        im.ewa_weights.assign(ewa_weights, ewa_weights + 128);
    const rp_image_texture &t = im.textures[index];
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 6 * i;
        float *o = out + 4 * i;
        const oracle::F2 uv{a[0], a[1]}, dx{a[2], a[3]}, dy{a[4], a[5]};
        const oracle::Rgb c = oracle::image_lookup(im, t, uv, dx, dy, false, false);
        o[0] = c.r;
        o[1] = c.g;
        o[2] = c.b;
        o[3] = oracle::image_lookup(im, t, uv, dx, dy, true, false).r;
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

void or_texture_footprint(const float *q, uint32_t count, float *out) {
    using oracle::F3;
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 48 * i;
        float *o = out + 24 * i;
        const F3 rp{a[0], a[1], a[2]}, n{a[3], a[4], a[5]}, d{a[6], a[7], a[8]}, rx{a[9], a[10], a[11]},
            ry{a[12], a[13], a[14]};
        F3 pdx, pdy, adx, ady;
        const bool primary = oracle::texture_primary_dp(rp, n, d, rx, ry, a[15], pdx, pdy);
        oracle::texture_approximate_dp(rp, n, a + 16, a + 25, F3{a[34], a[35], a[36]}, F3{a[37], a[38], a[39]}, a[15],
                                       adx, ady);
        oracle::F2 sx, sy;
        const bool ok = oracle::texture_uv_derivatives(F3{a[40], a[41], a[42]}, F3{a[43], a[44], a[45]},
                                                       primary ? pdx : adx, primary ? pdy : ady, sx, sy);
        const F3 td = oracle::texture_direction(rx);
        const float v[24] = {primary ? 1.f : 0.f, pdx.x, pdx.y, pdx.z, pdy.x, pdy.y, pdy.z, adx.x, adx.y, adx.z,
                             ady.x, ady.y, ady.z, ok ? 1.f : 0.f, sx.x, sx.y, sy.x, sy.y, td.x, td.y, td.z, 0, 0, 0};
        std::copy(v, v + 24, o);
    }
}

int or_texture_camera_differentials(const float *corner, const float *dx, const float *dy, uint32_t width,
                                    uint32_t height, float *out) {
    oracle::F3 mx, my;
    if (!oracle::texture_camera_differentials({corner[0], corner[1], corner[2]}, {dx[0], dx[1], dx[2]},
                                              {dy[0], dy[1], dy[2]}, width, height, mx, my)
             .empty())
        return -1;
    const float v[6] = {mx.x, mx.y, mx.z, my.x, my.y, my.z};
    std::copy(v, v + 6, out);
    return 0;
}

} // extern "C"
