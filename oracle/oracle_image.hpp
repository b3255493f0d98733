// ORACLE -- test infrastructure only (see oracle_math.hpp).  Image textures, the sRGB
// spectrum reconstruction and the equal-area environment image, restated on the CPU from
// rypath's shaders/image_texture.h, shaders/image_lighting.h, src/rgb_spectrum.cpp and
// src/environment_sampling.cpp.
#pragma once

#include "oracle_math.hpp"
#include "../include/rypath_cuda.h"

#include <string>
#include <vector>

namespace oracle {

struct F2 {
    float x = 0, y = 0;
};
struct Rgb {
    float r = 0, g = 0, b = 0;
};
inline Rgb rgb_nan() { return {NAN, NAN, NAN}; }
inline bool finite_rgb(Rgb c) { return std::isfinite(c.r) && std::isfinite(c.g) && std::isfinite(c.b); }

// The scene's images (src/render.hpp:251-261) and the environment tables built from them.
struct Images {
    std::vector<rp_image_texture> textures;
    std::vector<rp_texture_level> levels;
    std::vector<u32> texels;
    std::vector<float> transfer;
    std::vector<float> rgb_table, illuminant;
    u32 env_image = RP_NONE;
    float env_scale = 1;
    float env_from_world[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, world_from_env[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::vector<float> env_cdf;
    u32 env_width = 0, env_comp_offset = 0;
    double env_power = 0; // mean RGB illuminant power of the environment texels
    // texture coordinates: per-vertex uvs, per-triangle tangents (dpdu, dpdv), per-instance
    // first uv and first frame (RP_NONE: default uvs / no frames), the texture camera
    std::vector<F2> uvs;
    std::vector<std::array<F3, 2>> frames;
    std::vector<u32> inst_uv_begin, inst_frame_begin;
    float world_from_camera[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, camera_from_world[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::vector<float> ewa_weights; // PBRT's 128-entry EWA Gaussian table (rypath_ewa::weights)
};

// shaders/image_texture.h:14-27
inline float half_bits(u32 bits) {
    const u32 sign = (bits & 0x8000u) << 16, e = (bits >> 10) & 31u, m = bits & 1023u;
    if (e == 0) {
        if (m == 0)
            return std::bit_cast<float>(sign);
        const u32 lead = 31u - u32(std::countl_zero(m));
        return std::bit_cast<float>(sign | ((103u + lead) << 23) | ((m << (23u - lead)) & 0x7fffffu));
    }
    return std::bit_cast<float>(sign | ((e == 31u ? 255u : e + 112u) << 23) | (m << 13));
}
// shaders/image_texture.h:29-62
inline Rgb image_texel(const Images &im, const rp_texture_level &l, int x, int y, u32 wrap, u32 format,
                       u32 transfer_offset, bool alpha = false) {
    const int w = int(l.width), h = int(l.height);
    if (wrap == RP_WRAP_REPEAT) {
        x = (x % w + w) % w;
        y = (y % h + h) % h;
    } else if (wrap == RP_WRAP_CLAMP) {
        x = std::clamp(x, 0, w - 1);
        y = std::clamp(y, 0, h - 1);
    } else if (x < 0 || x >= w || y < 0 || y >= h) {
        return {};
    }
    const u32 index = u32(y) * l.width + u32(x);
    if (format == RP_TEXELS_FLOAT) {
        const u32 word = l.offset + 4u * index;
        if (alpha)
            return {std::bit_cast<float>(im.texels[word + 3]), 0, 0};
        return {std::bit_cast<float>(im.texels[word]), std::bit_cast<float>(im.texels[word + 1]),
                std::bit_cast<float>(im.texels[word + 2])};
    }
    if (format == RP_TEXELS_HALF) {
        const u32 word = l.offset + 2u * index;
        const u32 rg = im.texels[word], b = im.texels[word + 1];
        if (alpha)
            return {half_bits(b >> 16), 0, 0};
        return {half_bits(rg & 0xffffu), half_bits(rg >> 16), half_bits(b & 0xffffu)};
    }
    const u32 v = im.texels[l.offset + index];
    const float *t = im.transfer.data() + transfer_offset;
    if (alpha)
        return {t[v >> 24], 0, 0};
    return {t[v & 255u], t[(v >> 8) & 255u], t[(v >> 16) & 255u]};
}
// shaders/image_texture.h:64-73
inline bool image_level_valid(const Images &im, const rp_texture_level &l, u32 format) {
    const u32 per = format == RP_TEXELS_FLOAT ? 4u : format == RP_TEXELS_HALF ? 2u : 1u;
    const u32 words = u32(im.texels.size());
    return l.width > 0 && l.height > 0 && l.width <= 8192 && l.height <= 8192 && l.offset <= words &&
           l.width * l.height * per <= words - l.offset;
}
// shaders/image_texture.h:75-95
inline Rgb image_bilinear_texels(const Images &im, const rp_image_texture &t, const rp_texture_level &l, F2 xy,
                                 bool scalar) {
    const float fx = std::floor(xy.x), fy = std::floor(xy.y);
    const int bx = int(fx), by = int(fy);
    const float dx = xy.x - fx, dy = xy.y - fy;
    const bool alpha = scalar && t.channels == 4u;
    const Rgb a = image_texel(im, l, bx, by, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const Rgb b = image_texel(im, l, bx + 1, by, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const Rgb c = image_texel(im, l, bx, by + 1, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const Rgb e = image_texel(im, l, bx + 1, by + 1, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const float w00 = (1.0f - dx) * (1.0f - dy), w10 = dx * (1.0f - dy), w01 = (1.0f - dx) * dy, w11 = dx * dy;
    Rgb out{w00 * a.r + w10 * b.r + w01 * c.r + w11 * e.r, w00 * a.g + w10 * b.g + w01 * c.g + w11 * e.g,
            w00 * a.b + w10 * b.b + w01 * c.b + w11 * e.b};
    if (scalar && t.channels == 3u)
        out.r = (out.r + out.g + out.b) / 3.0f;
    return out;
}
// shaders/image_texture.h:97-109
inline Rgb image_bilinear(const Images &im, const rp_image_texture &t, const rp_texture_level &l, F2 st,
                          bool scalar) {
    if (t.wrap == RP_WRAP_REPEAT) {
        st.x -= std::floor(st.x);
        st.y -= std::floor(st.y);
    } else if (t.wrap == RP_WRAP_CLAMP) {
        st.x = std::clamp(st.x, 0.0f, 1.0f);
        st.y = std::clamp(st.y, 0.0f, 1.0f);
    } else if (st.x < -1.0f || st.y < -1.0f || st.x > 2.0f || st.y > 2.0f) {
        return {};
    }
    return image_bilinear_texels(im, t, l, {st.x * float(l.width) - 0.5f, st.y * float(l.height) - 0.5f}, scalar);
}
// shaders/image_texture.h:127-139
inline int image_point_coordinate(float st, float dimension, u32 wrap) {
    if (wrap == RP_WRAP_CLAMP)
        st = std::clamp(st, 0.0f, 1.0f);
    else if (wrap == RP_WRAP_BLACK)
        st = std::clamp(st, -1.0f, 2.0f);
    const float index = std::round(st * dimension - 0.5f);
    if (wrap == RP_WRAP_REPEAT)
        return std::isfinite(index) ? int(std::fmod(index, dimension)) : 0;
    return int(index);
}
// shaders/image_texture.h:390-401
inline bool image_lookup_valid(const Images &im, const rp_image_texture &t, F2 uv, F2 dx, F2 dy) {
    const u32 levels = u32(im.levels.size()), transfer = u32(im.transfer.size());
    return std::isfinite(uv.x) && std::isfinite(uv.y) && std::isfinite(dx.x) && std::isfinite(dx.y) &&
           std::isfinite(dy.x) && std::isfinite(dy.y) && t.wrap <= 2u &&
           (t.channels == 1u || t.channels == 3u || t.channels == 4u) && t.texel_format <= RP_TEXELS_FLOAT &&
           (t.texel_format >= RP_TEXELS_HALF || (t.transfer_offset <= transfer && transfer - t.transfer_offset >= 256u)) &&
           t.level_count != 0 && t.level_begin <= levels && t.level_count <= levels - t.level_begin;
}
// shaders/image_texture.h:403-456 (point, bilinear, trilinear)
inline Rgb image_lookup_standard(const Images &im, const rp_image_texture &t, F2 uv, F2 dx, F2 dy, bool scalar,
                                 bool mapped) {
    const bool point = t.filter == RP_TEXTURE_POINT;
    if (!image_lookup_valid(im, t, uv, dx, dy) ||
        (!point && t.filter != RP_TEXTURE_BILINEAR && t.filter != RP_TEXTURE_TRILINEAR))
        return rgb_nan();
    if (!mapped) {
        dx = {dx.x * t.uscale, dx.y * t.vscale};
        dy = {dy.x * t.uscale, dy.y * t.vscale};
    }
    const float extent = std::max(std::max(std::fabs(dx.x), std::fabs(dx.y)), std::max(std::fabs(dy.x), std::fabs(dy.y)));
    const float coarsest = float(t.level_count - 1u);
    float lod = coarsest;
    if (!(extent >= 0.5f)) {
        const float width = std::max(2.0f * extent, 1e-8f);
        const float log_width = std::log(width) * 1.4426950408889634f;
        lod = coarsest + log_width;
    }
    const bool wide = lod >= coarsest;
    const u32 index = wide ? t.level_count - 1u : u32(std::max(0.0f, std::floor(lod)));
    const rp_texture_level &level = im.levels[t.level_begin + index];
    if (!image_level_valid(im, level, t.texel_format))
        return rgb_nan();
    if (wide)
        return image_texel(im, level, 0, 0, t.wrap, t.texel_format, t.transfer_offset);
    const bool interpolate = t.filter == RP_TEXTURE_TRILINEAR && index > 0;
    if (interpolate && !image_level_valid(im, im.levels[t.level_begin + index + 1u], t.texel_format))
        return rgb_nan();
    F2 st = uv;
    if (!mapped) {
        const float su = uv.x * t.uscale, sv = uv.y * t.vscale;
        st = {su + t.udelta, sv + t.vdelta};
    }
    st.y = 1.0f - st.y;
    if (!std::isfinite(st.x) || !std::isfinite(st.y))
        return rgb_nan();
    if (point) {
        const int x = image_point_coordinate(st.x, float(level.width), t.wrap);
        const int y = image_point_coordinate(st.y, float(level.height), t.wrap);
        return image_texel(im, level, x, y, t.wrap, t.texel_format, t.transfer_offset);
    }
    const Rgb lower = image_bilinear(im, t, level, st, scalar);
    if (!interpolate)
        return lower;
    const Rgb upper = image_bilinear(im, t, im.levels[t.level_begin + index + 1u], st, scalar);
    const float delta = lod - float(index);
    return {(1.0f - delta) * lower.r + delta * upper.r, (1.0f - delta) * lower.g + delta * upper.g,
            (1.0f - delta) * lower.b + delta * upper.b};
}

// ---------------------------------------------------------------- EWA (PBRT's elliptically
// weighted average over the two mip levels around the footprint's minor axis)
inline u32 ewa_magnitude(float v) { return std::bit_cast<u32>(v) & 0x7fffffffu; }
inline bool ewa_subnormal(u32 m) { return m != 0u && m < 0x00800000u; }
// shaders/image_texture.h:168-204: value * scale rounded to nearest even with gradual underflow,
// reconstructed from the significands where an operand or the product is subnormal
inline float ewa_product(float value, float scale) {
    const float mapped = value * scale;
    const u32 a = ewa_magnitude(value), b = ewa_magnitude(scale);
    if (a == 0u || b == 0u || (ewa_magnitude(mapped) != 0u && !ewa_subnormal(a) && !ewa_subnormal(b)))
        return mapped;
    const int a_exp = int(a >> 23), b_exp = int(b >> 23);
    const u32 a_sig = (a & 0x007fffffu) | (a_exp == 0 ? 0u : 0x00800000u);
    const u32 b_sig = (b & 0x007fffffu) | (b_exp == 0 ? 0u : 0x00800000u);
    const uint64_t product = uint64_t(a_sig) * b_sig;
    const int exponent = std::max(1, a_exp) + std::max(1, b_exp) - 300;
    const int leading = 63 - int(std::countl_zero(product));
    const u32 sign = (std::bit_cast<u32>(value) ^ std::bit_cast<u32>(scale)) & 0x80000000u;
    if (exponent + leading > 127)
        return std::bit_cast<float>(sign | 0x7f800000u);
    const int shift = std::max(leading - 23, -149 - exponent);
    if (shift > 48)
        return std::bit_cast<float>(sign);
    u32 rounded;
    if (shift <= 0) {
        rounded = u32(product << -shift);
    } else {
        const uint64_t halfway = uint64_t(1) << (shift - 1);
        const uint64_t truncated = product >> shift;
        rounded = u32((product + halfway - 1u + (truncated & 1u)) >> shift);
    }
    return std::bit_cast<float>(sign | ((u32(exponent + shift + 149) << 23) + rounded));
}
// shaders/image_texture.h:206-211
inline float ewa_lift(float v) {
    const u32 m = ewa_magnitude(v);
    if (ewa_subnormal(m))
        return std::copysign(float(m) * 0x1p-125f, v);
    return v * 0x1p24f;
}
// shaders/image_texture.h:141-152
inline float ewa_center(float st, float dimension, u32 wrap) {
    if (std::fabs(st) <= 64.0f || wrap == RP_WRAP_BLACK)
        return st * dimension - 0.5f;
    const float phase = std::fmod(st, 1.0f) * dimension;
    if (wrap == RP_WRAP_REPEAT)
        return phase - 0.5f;
    return ((st < 0.0f ? -64.0f : dimension + 64.0f) + phase) - 0.5f;
}
// shaders/image_texture.h:154-159
inline bool ewa_black_disjoint(F2 st, F2 dims, F2 radius) {
    const auto axis = [](float s, float d, float r) {
        return std::fabs(s) > 64.0f && (s < (0.5f - r) / d || s > ((d - 0.5f) + r) / d);
    };
    return axis(st.x, dims.x, radius.x) || axis(st.y, dims.y, radius.y);
}
// shaders/image_texture.h:134-139
inline bool ewa_level_valid(const Images &im, const rp_texture_level &l, u32 format, u32 levels_above) {
    return image_level_valid(im, l, format) && (l.width & (l.width - 1u)) == 0u && (l.height & (l.height - 1u)) == 0u &&
           std::max(l.width, l.height) == (1u << levels_above);
}
// shaders/image_texture.h:213-256
inline Rgb ewa_level(const Images &im, const rp_image_texture &t, const rp_texture_level &l, F2 st, F2 dx, F2 dy) {
    const F2 dims{float(l.width), float(l.height)};
    const F2 u{dx.x * dims.x, dx.y * dims.y}, v{dy.x * dims.x, dy.y * dims.y};
    const float area = u.x * v.y - u.y * v.x;
    const float determinant = ((1.0f + (u.x * u.x + u.y * u.y)) + (v.x * v.x + v.y * v.y)) + area * area;
    const F2 radius{std::sqrt((1.0f + u.x * u.x) + v.x * v.x), std::sqrt((1.0f + u.y * u.y) + v.y * v.y)};
    if (t.wrap == RP_WRAP_BLACK && ewa_black_disjoint(st, dims, radius))
        return {};
    const F2 center{ewa_center(st.x, dims.x, t.wrap), ewa_center(st.y, dims.y, t.wrap)};
    const F2 begin{std::ceil(center.x - radius.x), std::ceil(center.y - radius.y)};
    const F2 end{std::floor(center.x + radius.x), std::floor(center.y + radius.y)};
    const F2 count{(end.x - begin.x) + 1.0f, (end.y - begin.y) + 1.0f};
    if (!std::isfinite(begin.x) || !std::isfinite(begin.y) || !std::isfinite(end.x) || !std::isfinite(end.y) ||
        std::fabs(begin.x) > 0x1p19f || std::fabs(begin.y) > 0x1p19f || std::fabs(end.x) > 0x1p19f ||
        std::fabs(end.y) > 0x1p19f || count.x <= 0.0f || count.y <= 0.0f || count.x * count.y > 4096.0f)
        return rgb_nan();
    if (t.wrap == RP_WRAP_BLACK && (end.x < 0.0f || end.y < 0.0f || begin.x >= dims.x || begin.y >= dims.y))
        return {};
    const int x0 = int(begin.x), y0 = int(begin.y), x1 = int(end.x), y1 = int(end.y);
    Rgb sum{};
    float weight_sum = 0;
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const F2 d{float(x) - center.x, float(y) - center.y};
            const float a = u.x * d.y - u.y * d.x, b = v.x * d.y - v.y * d.x;
            const float r2 = (((d.x * d.x + d.y * d.y) + a * a) + b * b) / determinant;
            if (r2 < 1.0f) {
                const float w = im.ewa_weights[std::min(u32(128.0f * r2), 127u)];
                const Rgb c = image_texel(im, l, x, y, t.wrap, t.texel_format, t.transfer_offset);
                sum = {sum.r + w * c.r, sum.g + w * c.g, sum.b + w * c.b};
                weight_sum += w;
            }
        }
    if (!(std::isfinite(weight_sum) && weight_sum > 0.0f))
        return rgb_nan();
    return {sum.r / weight_sum, sum.g / weight_sum, sum.b / weight_sum};
}
// shaders/image_texture.h:258-388
inline Rgb image_lookup_ewa(const Images &im, const rp_image_texture &t, F2 uv, F2 dx, F2 dy, bool scalar, bool mapped) {
    const float cap = t.max_anisotropy;
    if (t.level_count > 14u || !(cap >= 1.0f && cap <= 16.0f) || !std::isfinite(t.uscale) || !std::isfinite(t.vscale) ||
        !std::isfinite(t.udelta) || !std::isfinite(t.vdelta) || im.ewa_weights.size() < 128)
        return rgb_nan();
    if (!mapped) {
        dx = {ewa_product(dx.x, t.uscale), ewa_product(dx.y, t.vscale)};
        dy = {ewa_product(dy.x, t.uscale), ewa_product(dy.y, t.vscale)};
    }
    if (!std::isfinite(dx.x) || !std::isfinite(dx.y) || !std::isfinite(dy.x) || !std::isfinite(dy.y))
        return rgb_nan();
    const u32 top = t.level_count - 1u;
    const rp_texture_level *mips = im.levels.data() + t.level_begin;
    const u32 x_bits = std::max(ewa_magnitude(dx.x), ewa_magnitude(dx.y));
    const u32 y_bits = std::max(ewa_magnitude(dy.x), ewa_magnitude(dy.y));
    const bool zero = x_bits == 0u || y_bits == 0u;
    float minor = 0.0f;
    if (!zero) {
        if (std::max(x_bits, y_bits) >= std::bit_cast<u32>(32.0f)) {
            minor = 2.0f;
        } else {
            const bool lifted = ewa_subnormal(ewa_magnitude(dx.x)) || ewa_subnormal(ewa_magnitude(dx.y)) ||
                                ewa_subnormal(ewa_magnitude(dy.x)) || ewa_subnormal(ewa_magnitude(dy.y));
            const F2 a = lifted ? F2{ewa_lift(dx.x), ewa_lift(dx.y)} : dx;
            const F2 b = lifted ? F2{ewa_lift(dy.x), ewa_lift(dy.y)} : dy;
            const float x_scale = std::max(std::fabs(a.x), std::fabs(a.y));
            const float y_scale = std::max(std::fabs(b.x), std::fabs(b.y));
            const F2 x{a.x / x_scale, a.y / x_scale}, y{b.x / y_scale, b.y / y_scale};
            const float x_norm = std::sqrt(x.x * x.x + x.y * x.y), y_norm = std::sqrt(y.x * y.x + y.y * y.y);
            const float x_length = x_scale * x_norm, y_length = y_scale * y_norm;
            const bool x_major = x_length >= y_length;
            const float major = x_major ? x_length : y_length;
            minor = x_major ? y_length : x_length;
            const float capped = major / cap;
            if (minor < capped) {
                const float actual = lifted ? capped * 0x1p-24f : capped;
                if (x_major)
                    dy = {(y.x / y_norm) * actual, (y.y / y_norm) * actual};
                else
                    dx = {(x.x / x_norm) * actual, (x.y / x_norm) * actual};
                minor = capped;
            }
            if (lifted)
                minor *= 0x1p-24f;
        }
        if (minor >= 2.0f) {
            if (!ewa_level_valid(im, mips[top], t.texel_format, 0))
                return rgb_nan();
            return image_texel(im, mips[top], 0, 0, t.wrap, t.texel_format, t.transfer_offset);
        }
    }
    F2 st = uv;
    if (!mapped)
        st = {ewa_product(uv.x, t.uscale) + t.udelta, ewa_product(uv.y, t.vscale) + t.vdelta};
    st.y = 1.0f - st.y;
    if (!std::isfinite(st.x) || !std::isfinite(st.y))
        return rgb_nan();
    if (zero) {
        if (!ewa_level_valid(im, mips[0], t.texel_format, top))
            return rgb_nan();
        const F2 dims{float(mips[0].width), float(mips[0].height)};
        if (t.wrap == RP_WRAP_BLACK && ewa_black_disjoint(st, dims, {1.0f, 1.0f}))
            return {};
        const F2 center{ewa_center(st.x, dims.x, t.wrap), ewa_center(st.y, dims.y, t.wrap)};
        return image_bilinear_texels(im, t, mips[0], center, scalar);
    }
    const float lod = std::max(0.0f, float(top) + std::log2(minor));
    const u32 lower = std::min(u32(std::floor(lod)), top);
    if (!ewa_level_valid(im, mips[lower], t.texel_format, top - lower))
        return rgb_nan();
    if (lower < top && (!ewa_level_valid(im, mips[lower + 1u], t.texel_format, top - lower - 1u) ||
                        mips[lower + 1u].width != std::max(1u, mips[lower].width / 2u) ||
                        mips[lower + 1u].height != std::max(1u, mips[lower].height / 2u)))
        return rgb_nan();
    const Rgb a = ewa_level(im, t, mips[lower], st, dx, dy);
    const Rgb b = lower == top ? image_texel(im, mips[top], 0, 0, t.wrap, t.texel_format, t.transfer_offset)
                               : ewa_level(im, t, mips[lower + 1u], st, dx, dy);
    const float delta = lod - float(lower);
    return {(1.0f - delta) * a.r + delta * b.r, (1.0f - delta) * a.g + delta * b.g, (1.0f - delta) * a.b + delta * b.b};
}
// shaders/image_texture.h:541-554 (lookup_filtered): EWA or the standard filters
inline Rgb image_lookup(const Images &im, const rp_image_texture &t, F2 uv, F2 dx, F2 dy, bool scalar, bool mapped) {
    if (t.filter != RP_TEXTURE_EWA)
        return image_lookup_standard(im, t, uv, dx, dy, scalar, mapped);
    if (!image_lookup_valid(im, t, uv, dx, dy))
        return rgb_nan();
    return image_lookup_ewa(im, t, uv, dx, dy, scalar, mapped);
}

// shaders/image_texture.h:458-499 (rypath_image::spectrum)
inline float srgb_spectrum(const float *table, Rgb c, float wavelength) {
    if (!finite_rgb(c))
        return NAN;
    const float ch0[3] = {std::clamp(c.r, 0.0f, 1.0f), std::clamp(c.g, 0.0f, 1.0f), std::clamp(c.b, 0.0f, 1.0f)};
    if (ch0[0] == ch0[1] && ch0[1] == ch0[2])
        return ch0[0];
    u32 channel = 0;
    if (ch0[1] >= ch0[0])
        channel = 1;
    if (ch0[2] >= ch0[channel])
        channel = 2;
    const float z = ch0[channel];
    const float x = ch0[(channel + 1u) % 3u] * 63.0f / z;
    const float y = ch0[(channel + 2u) % 3u] * 63.0f / z;
    const u32 xi = std::min(u32(x), 62u), yi = std::min(u32(y), 62u);
    u32 lower = 1, upper = 63;
    while (lower < upper) {
        const u32 mid = (lower + upper) / 2u;
        if (table[mid] < z)
            lower = mid + 1u;
        else
            upper = mid;
    }
    const u32 zi = lower - 1u;
    const float dx = x - float(xi), dy = y - float(yi);
    const float dz = (z - table[zi]) / (table[zi + 1u] - table[zi]);
    const auto blend = [](float t, float a, float b) { return (1.0f - t) * a + t * b; };
    float co[3];
    for (u32 i = 0; i < 3; ++i) {
        const u32 cell = 64u + 3u * (((channel * 64u + zi) * 64u + yi) * 64u + xi) + i;
        const u32 row = 3u * 64u, plane = row * 64u;
        co[i] = blend(dz,
                      blend(dy, blend(dx, table[cell], table[cell + 3u]),
                            blend(dx, table[cell + row], table[cell + row + 3u])),
                      blend(dy, blend(dx, table[cell + plane], table[cell + plane + 3u]),
                            blend(dx, table[cell + plane + row], table[cell + plane + row + 3u])));
    }
    const float poly = std::fma(std::fma(co[0], wavelength, co[1]), wavelength, co[2]);
    if (!std::isfinite(poly))
        return NAN;
    if (std::fabs(poly) <= 1.0f)
        return 0.5f + 0.5f * poly / std::sqrt(1.0f + poly * poly);
    const float inverse = 1.0f / poly;
    return 0.5f + 0.5f * std::copysign(1.0f / std::sqrt(1.0f + inverse * inverse), poly);
}
// shaders/image_texture.h:500-507
inline float srgb_spectrum_unbounded(const float *table, Rgb c, float wavelength) {
    if (!finite_rgb(c) || c.r < 0 || c.g < 0 || c.b < 0)
        return NAN;
    const float scale = 2 * std::max(std::max(c.r, c.g), c.b);
    if (!std::isfinite(scale))
        return NAN;
    return scale == 0 ? 0.0f : scale * srgb_spectrum(table, {c.r / scale, c.g / scale, c.b / scale}, wavelength);
}

// ---------------------------------------------------------------- environment image
inline F3 env_unit(F3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline F3 env_apply(const float *m, F3 d) {
    return {dot(F3{m[0], m[1], m[2]}, d), dot(F3{m[3], m[4], m[5]}, d), dot(F3{m[6], m[7], m[8]}, d)};
}
// shaders/image_lighting.h:28-40
inline float illuminant_spectrum(const Images &im, Rgb c, float wavelength) {
    if (!finite_rgb(c) || !std::isfinite(wavelength))
        return NAN;
    c = {std::max(0.0f, c.r), std::max(0.0f, c.g), std::max(0.0f, c.b)};
    const float amplitude = 2.0f * std::max(std::max(c.r, c.g), c.b);
    if (amplitude == 0)
        return 0;
    const float nearest = std::round(wavelength);
    if (nearest < 360.0f || nearest > 830.0f)
        return 0;
    return amplitude * srgb_spectrum(im.rgb_table.data(), {c.r / amplitude, c.g / amplitude, c.b / amplitude}, wavelength) *
           im.illuminant[u32(nearest) - 360u];
}
// shaders/image_lighting.h:82-93
inline F3 env_square_to_sphere(F2 uv) {
    const float su = 2.0f * uv.x - 1.0f, sv = 2.0f * uv.y - 1.0f;
    const float qu = std::fabs(su), qv = std::fabs(sv);
    const float diagonal = 1.0f - (qu + qv);
    const float radius = 1.0f - std::fabs(diagonal);
    const float pi = 3.14159265358979323846f;
    const float phi = (radius == 0 ? 1.0f : (qv - qu) / radius + 1.0f) * (pi / 4.0f);
    const float height = std::copysign(1.0f - radius * radius, diagonal);
    const float radial = radius * std::sqrt(std::max(0.0f, 2.0f - radius * radius));
    return {std::copysign(std::cos(phi), su) * radial, std::copysign(std::sin(phi), sv) * radial, height};
}
// shaders/image_lighting.h:95-124
inline F2 env_sphere_to_square(F3 d, bool pinned) {
    const F3 m{std::fabs(d.x), std::fabs(d.y), std::fabs(d.z)};
    float radius, phi;
    if (pinned) {
        radius = std::sqrt(std::max(0.0f, 1.0f - m.z));
        const float larger = std::max(m.x, m.y);
        const float ratio = larger == 0 ? 0.0f : std::min(m.x, m.y) / larger;
        phi = std::fma(ratio, -0.02513909723434835f, 0.041903881802916574f);
        phi = std::fma(ratio, phi, 0.08817706647753163f);
        phi = std::fma(ratio, phi, -0.24733373328126894f);
        phi = std::fma(ratio, phi, 0.006157201789828021f);
        phi = std::fma(ratio, phi, 0.6362265452740161f);
        phi = std::fma(ratio, phi, 0.000004067585662467885f);
        if (m.x < m.y)
            phi = 1.0f - phi;
    } else {
        const float horizontal = std::sqrt(d.x * d.x + d.y * d.y);
        radius = horizontal / std::sqrt(1.0f + m.z);
        phi = horizontal == 0 ? 0.0f : std::atan2(m.y, m.x) * (2.0f / 3.14159265358979323846f);
    }
    F2 uv{radius - phi * radius, phi * radius};
    if (d.z < 0)
        uv = {1.0f - uv.y, 1.0f - uv.x};
    uv = {std::copysign(uv.x, d.x), std::copysign(uv.y, d.y)};
    return {std::clamp(0.5f * (uv.x + 1.0f), 0.0f, 1.0f), std::clamp(0.5f * (uv.y + 1.0f), 0.0f, 1.0f)};
}
// shaders/image_lighting.h:170-208
inline float env_image_radiance(const Images &im, F3 world_direction, float wavelength) {
    if (im.env_image >= im.textures.size())
        return NAN;
    const rp_image_texture &t = im.textures[im.env_image];
    const F3 d = env_unit(env_apply(im.env_from_world, world_direction));
    if (!finite3(d) || !image_lookup_valid(im, t, {}, {}, {}) || t.level_count != 1u)
        return NAN;
    const rp_texture_level &level = im.levels[t.level_begin];
    if (!image_level_valid(im, level, t.texel_format) || level.width != level.height)
        return NAN;
    const int size = int(level.width);
    const F2 uv = env_sphere_to_square(d, true);
    int px = int(uv.x * float(size)), py = int(uv.y * float(size));
    if (px == size) {
        px = size - 1;
        py = size - 1 - py;
    }
    if (py < 0) {
        px = size - 1 - px;
        py = -py;
    } else if (py == size) {
        px = size - 1 - px;
        py = size - 1;
    }
    if (size == 1)
        px = py = 0;
    const Rgb c = image_texel(im, level, px, py, RP_WRAP_CLAMP, t.texel_format, t.transfer_offset);
    return im.env_scale * illuminant_spectrum(im, c, wavelength);
}
// shaders/image_lighting.h:210-219
inline bool env_tables_valid(const Images &im, bool compensated) {
    const u32 w = im.env_width;
    if (w == 0 || w > 8192)
        return false;
    const u32 count = (w + 1u) * (w + 1u), total = u32(im.env_cdf.size());
    const u32 offset = compensated ? im.env_comp_offset : 0u;
    return (!compensated || offset >= count) && offset <= total && count <= total - offset;
}
// shaders/image_lighting.h:221-231
inline bool env_cell(const Images &im, F3 world_direction, u32 &cx, u32 &cy) {
    const F3 d = env_unit(env_apply(im.env_from_world, world_direction));
    if (!finite3(d))
        return false;
    const F2 uv = env_sphere_to_square(d, false);
    cx = std::min(u32(uv.x * float(im.env_width)), im.env_width - 1u);
    cy = std::min(u32(uv.y * float(im.env_width)), im.env_width - 1u);
    return true;
}
// shaders/image_lighting.h:233-246
inline float env_cell_density(const Images &im, u32 cx, u32 cy, bool compensated) {
    const float *cdf = im.env_cdf.data() + (compensated ? im.env_comp_offset : 0u);
    const u32 w = im.env_width;
    const float *row = cdf + (cy + 1u) * (w + 1u);
    const float marginal = cdf[cy + 1u] - cdf[cy];
    const float conditional = row[cx + 1u] - row[cx];
    if (!(marginal >= 0.0f && marginal <= 1.0f && conditional >= 0.0f && conditional <= 1.0f))
        return NAN;
    const float density = (float(w) * marginal) * (float(w) * conditional);
    const float sphere = 0.25f / 3.14159265358979323846f;
    return sphere * (compensated ? density : 0.0625f + (1.0f - 0.0625f) * density);
}
// shaders/image_lighting.h:248-255
inline float env_image_pdf(const Images &im, F3 world_direction, bool compensated) {
    u32 cx, cy;
    if (!env_tables_valid(im, compensated) || !env_cell(im, world_direction, cx, cy))
        return NAN;
    return env_cell_density(im, cx, cy, compensated);
}
// shaders/image_lighting.h:257-273
inline float env_sample_row(const float *cdf, u32 width, float u, u32 &cell) {
    u32 lower = 0, upper = width;
    while (upper - lower > 1u) {
        const u32 middle = lower + (upper - lower) / 2u;
        if (u < cdf[middle])
            upper = middle;
        else
            lower = middle;
    }
    const float mass = cdf[upper] - cdf[lower];
    if (!(mass > 0.0f && mass <= 1.0f))
        return NAN;
    cell = lower;
    const float fraction = std::clamp((u - cdf[lower]) / mass, 0.0f, 0x1.fffffep-1f);
    return (float(lower) + fraction) / float(width);
}
// shaders/image_lighting.h:275-325
inline bool env_image_sample(const Images &im, float ux, float uy, bool compensated, F3 &world_direction, float &pdf) {
    if (!env_tables_valid(im, compensated) || !std::isfinite(ux) || !std::isfinite(uy) || ux < 0.0f || uy < 0.0f ||
        ux > 1.0f || uy > 1.0f)
        return false;
    const float *cdf = im.env_cdf.data() + (compensated ? im.env_comp_offset : 0u);
    const bool importance = compensated || ux >= 0.0625f;
    const u32 w = im.env_width;
    u32 row = 0, column = 0;
    F2 uv;
    if (!importance) {
        uv = {ux / 0.0625f, uy};
    } else {
        uv.y = env_sample_row(cdf, w, std::min(uy, 0x1.fffffep-1f), row);
        const float uc = compensated ? ux : (ux - 0.0625f) / (1.0f - 0.0625f);
        uv.x = env_sample_row(cdf + (row + 1u) * (w + 1u), w, std::min(uc, 0x1.fffffep-1f), column);
    }
    if (!std::isfinite(uv.x) || !std::isfinite(uv.y))
        return false;
    world_direction = env_unit(env_apply(im.world_from_env, env_square_to_sphere(uv)));
    u32 cx, cy;
    if (!env_cell(im, world_direction, cx, cy))
        return false;
    if (importance && (cx != column || cy != row)) {
        const F2 center{(float(column) + 0.5f) / float(w), (float(row) + 0.5f) / float(w)};
        for (float weight = 0x1p-16f; weight <= 1.0f; weight *= 2.0f) {
            const F2 inward{uv.x + (center.x - uv.x) * weight, uv.y + (center.y - uv.y) * weight};
            world_direction = env_unit(env_apply(im.world_from_env, env_square_to_sphere(inward)));
            if (!env_cell(im, world_direction, cx, cy))
                return false;
            if (cx == column && cy == row)
                break;
        }
        if (cx != column || cy != row)
            return false;
    }
    pdf = env_cell_density(im, cx, cy, compensated);
    return std::isfinite(pdf) && pdf > 0;
}

// ---------------------------------------------------------------- texture footprints
// src/metal_render.mm:1962-1963 (spp_scale; shaders/texture_footprint.h:10-12 in binary32)
inline float texture_differential_scale(uint64_t total_spp) {
    return float(std::max(0.125, 1.0 / std::sqrt(double(total_spp))));
}
// shaders/texture_footprint.h:14-20
inline F3 texture_direction(F3 d) {
    const float scale = std::max(std::fabs(d.x), std::max(std::fabs(d.y), std::fabs(d.z)));
    if (!(scale > 0.0f) || !finite3(d))
        return {NAN, NAN, NAN};
    return env_unit(F3{d.x / scale, d.y / scale, d.z / scale});
}
// shaders/texture_footprint.h:22-38
inline bool texture_primary_dp(F3 rel, F3 n, F3 dir, F3 xr, F3 yr, float spp_scale, F3 &dpdx, F3 &dpdy) {
    const F3 rx = dir + spp_scale * (texture_direction(xr) - dir);
    const F3 ry = dir + spp_scale * (texture_direction(yr) - dir);
    const float nx = dot(n, rx), ny = dot(n, ry);
    if (nx == 0.0f || ny == 0.0f || !std::isfinite(nx) || !std::isfinite(ny))
        return false;
    const float plane = dot(n, rel);
    dpdx = (plane / nx) * rx - rel;
    dpdy = (plane / ny) * ry - rel;
    return true;
}
// shaders/texture_footprint.h:40-43
inline F3 texture_reflect(F3 x, F3 normal) { return x - ((2.0f * dot(normal, x)) / dot(normal, normal)) * normal; }
// row-major matrix times vector, summing columns in order (Metal's float3x3 product)
inline F3 texture_apply(const float *m, F3 v) {
    const F3 c0{m[0], m[3], m[6]}, c1{m[1], m[4], m[7]}, c2{m[2], m[5], m[8]};
    return (c0 * v.x + c1 * v.y) + c2 * v.z;
}
inline F3 texture_apply_transposed(const float *m, F3 v) {
    const F3 c0{m[0], m[1], m[2]}, c1{m[3], m[4], m[5]}, c2{m[6], m[7], m[8]};
    return (c0 * v.x + c1 * v.y) + c2 * v.z;
}
// shaders/texture_footprint.h:45-58
inline F3 texture_approximate_axis(F3 p_down_z, F3 n_down_z, F3 delta, F3 u, F3 v, const float *world_from_camera,
                                   float spp_scale) {
    const F3 ray = F3{0, 0, 1} + delta;
    const float denom = dot(n_down_z, ray);
    if (denom == 0.0f)
        return {};
    const F3 offset = ((n_down_z.z * p_down_z.z) / denom) * ray - p_down_z;
    const F3 dp = spp_scale * texture_apply(world_from_camera, texture_reflect(texture_reflect(offset, v), u));
    return finite3(dp) ? dp : F3{};
}
// shaders/texture_footprint.h:60-86 (PBRT's Camera::Approximate_dp_dxy)
inline void texture_approximate_dp(F3 rel, F3 n, const float *world_from_camera, const float *camera_from_world,
                                   F3 min_dx, F3 min_dy, float spp_scale, F3 &dpdx, F3 &dpdy) {
    const F3 p_camera = texture_apply(camera_from_world, rel);
    const F3 direction = texture_direction(p_camera);
    if (!finite3(direction)) {
        dpdx = dpdy = F3{};
        return;
    }
    const F3 z{0, 0, 1};
    const F3 ref = std::fabs(direction.x) < 0.72f ? F3{1, 0, 0} : F3{0, 1, 0};
    const F3 u = ref - direction, v = ref - z;
    const F3 p_down_z = texture_reflect(texture_reflect(p_camera, u), v);
    const F3 n_camera = texture_apply_transposed(world_from_camera, n);
    const F3 n_down_z = texture_reflect(texture_reflect(n_camera, u), v);
    dpdx = texture_approximate_axis(p_down_z, n_down_z, min_dx, u, v, world_from_camera, spp_scale);
    dpdy = texture_approximate_axis(p_down_z, n_down_z, min_dy, u, v, world_from_camera, spp_scale);
}
// shaders/texture_footprint.h:139-142
inline float texture_difference_of_products(float a, float b, float c, float d) {
    const float cd = c * d;
    return std::fma(a, b, -cd) + std::fma(-c, d, cd);
}
// shaders/texture_footprint.h:144-159
inline float texture_sanitize(float d) { return std::isfinite(d) ? std::clamp(d, -1e8f, 1e8f) : 0.0f; }
inline F2 texture_solve_axis(F3 dpdu, F3 dpdv, F3 dp, float aa, float ab, float bb, float inv_det) {
    const float u = dot(dpdu, dp), v = dot(dpdv, dp);
    return {texture_sanitize(inv_det * texture_difference_of_products(bb, u, ab, v)),
            texture_sanitize(inv_det * texture_difference_of_products(aa, v, ab, u))};
}
// shaders/texture_footprint.h:161-185
inline bool texture_uv_derivatives(F3 dpdu, F3 dpdv, F3 dpdx, F3 dpdy, F2 &dstdx, F2 &dstdy) {
    if (!finite3(dpdu) || !finite3(dpdv))
        return false;
    const float aa = dot(dpdu, dpdu), ab = dot(dpdu, dpdv), bb = dot(dpdv, dpdv);
    const float det = texture_difference_of_products(aa, bb, ab, ab);
    const float inv_det = 1.0f / det;
    if (!std::isfinite(inv_det)) {
        dstdx = dstdy = F2{};
        return true;
    }
    dstdx = texture_solve_axis(dpdu, dpdv, dpdx, aa, ab, bb, inv_det);
    dstdy = texture_solve_axis(dpdu, dpdv, dpdy, aa, ab, bb, inv_det);
    return true;
}
// The smallest one-pixel change of a camera ray's direction, over 512 rays along the film's
// diagonal, in each ray's local frame (src/texture_footprint.cpp:199-232, PBRT's
// Camera::FindMinimumDifferentials); empty on success.
std::string texture_camera_differentials(F3 corner, F3 dx, F3 dy, u32 width, u32 height, F3 &min_dx, F3 &min_dy);

// The environment importance tables and the image's mean illuminant power
// (src/environment_sampling.cpp:20-115, src/light_sampling.cpp:28-95); empty on success.
std::string build_environment_tables(Images &im);
// Copy and check a scene description's images; empty on success.
std::string load_images(const rp_images *in, u32 instance_count, Images &out);

} // namespace oracle
