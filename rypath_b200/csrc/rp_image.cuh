// Image textures and the image environment: texel decoding, point / bilinear / trilinear /
// EWA lookups over a mip chain, the sRGB-to-spectrum reconstruction, and the equal-area
// octahedral environment with its importance tables.  The arithmetic follows rypath's
// shaders/image_texture.h and shaders/image_lighting.h; the data layout is rypath's wire
// layout (src/render_wire.h:35-95) so a RenderScene's images upload without conversion.
#pragma once

#include "rp_math.cuh"

namespace rp {

// wire::ImageTexture (src/render_wire.h:68-87)
struct DImageTexture {
    u32 level_begin, level_count, wrap, texel_format;
    float uscale, vscale, udelta, vdelta, scale;
    u32 invert, filter;
    float max_anisotropy;
    u32 transfer_offset, channels, gltf, wrap_t, min_filter, mag_filter;
};
// wire::TextureLevel (src/render_wire.h:63-67)
struct DLevel {
    u32 width, height, offset;
};
constexpr u32 kWrapRepeat = 0, kWrapClamp = 1, kWrapBlack = 2;
constexpr u32 kFilterBilinear = 0, kFilterTrilinear = 1, kFilterPoint = 2, kFilterEwa = 3;
constexpr u32 kTexelsSrgb8 = 0, kTexelsLinear8 = 1, kTexelsHalf = 2, kTexelsFloat = 3;

// The images of a scene on the device.  env_cdf holds the full and the compensated
// importance tables of the environment image (src/environment_sampling.hpp:9-16): a marginal
// CDF then env_width conditional row CDFs, each of env_width + 1 entries.
struct DImages {
    const DImageTexture *textures;
    const DLevel *levels;
    const u32 *texels;
    const float *transfer;
    const float *rgb_table;  // 64 z nodes, then 3 x 64^3 cells of 3 coefficients
    const float *illuminant; // D65 at 360..830 nm
    u32 texture_count, level_count, texel_word_count, transfer_count;
    u32 env_image; // kNone: no environment image
    float env_scale;
    float env_from_world[9], world_from_env[9];
    const float *env_cdf;
    u32 env_width, env_comp_offset, env_cdf_count;
    // texture coordinates of image reflectance
    const float2 *uvs;
    const u32 *inst_uv_begin;    // per instance; 0xffffffff: default triangle uvs
    const float *frames;         // 6 floats (dpdu, dpdv) per textured triangle
    const u32 *inst_frame_begin; // per instance
    u32 uv_count, frame_count;
    float world_from_camera[9], camera_from_world[9];
    // the request's footprint scale and the camera's minimum one-pixel differentials, set by
    // the host before each render of a scene with image reflectance (textured != 0)
    u32 textured;
    float tex_spp_scale;
    float tex_min_dx[3], tex_min_dy[3];
    const float *ewa_weights; // PBRT's 128-entry EWA Gaussian table
};

// The quiet NaN of C's NAN, so that failed lookups read like the host's
RP_DEV float image_nan() { return __int_as_float(0x7fc00000); }

struct F2 {
    float x, y;
};
RP_DEV F2 f2(float x, float y) { return {x, y}; }
struct RGB {
    float r, g, b;
};
RP_DEV RGB rgb3(float r, float g, float b) { return {r, g, b}; }
RP_DEV RGB rgb_nan() { return {image_nan(), image_nan(), image_nan()}; }
RP_DEV bool finite_rgb(RGB c) { return isfinite(c.r) && isfinite(c.g) && isfinite(c.b); }

// binary16 bits to binary32 without half arithmetic, so subnormal halves widen exactly
// (shaders/image_texture.h:14-27)
RP_DEV float half_bits_to_float(u32 bits) {
    const u32 sign = (bits & 0x8000u) << 16;
    const u32 e = (bits >> 10) & 31u, m = bits & 1023u;
    if (e == 0) {
        if (m == 0)
            return __uint_as_float(sign);
        const u32 top = 31u - __clz(m); // highest set bit of the mantissa
        return __uint_as_float(sign | ((103u + top) << 23) | ((m << (23u - top)) & 0x7fffffu));
    }
    return __uint_as_float(sign | ((e == 31u ? 255u : e + 112u) << 23) | (m << 13));
}

// One texel of a level with the texture's wrap applied; black wrap outside is zero.  alpha
// selects the fourth channel (shaders/image_texture.h:29-62).
RP_DEV RGB texel(const DImages &im, const DLevel &level, int x, int y, u32 wrap, u32 format, u32 transfer_offset,
                 bool alpha = false) {
    const int w = int(level.width), h = int(level.height);
    if (wrap == kWrapRepeat) {
        x = (x % w + w) % w;
        y = (y % h + h) % h;
    } else if (wrap == kWrapClamp) {
        x = min(max(x, 0), w - 1);
        y = min(max(y, 0), h - 1);
    } else if (x < 0 || x >= w || y < 0 || y >= h) {
        return rgb3(0, 0, 0);
    }
    const u32 index = u32(y) * level.width + u32(x);
    if (format == kTexelsFloat) {
        const u32 *t = im.texels + level.offset + 4u * index;
        if (alpha)
            return rgb3(__uint_as_float(__ldg(t + 3)), 0, 0);
        return rgb3(__uint_as_float(__ldg(t)), __uint_as_float(__ldg(t + 1)), __uint_as_float(__ldg(t + 2)));
    }
    if (format == kTexelsHalf) {
        const u32 *t = im.texels + level.offset + 2u * index;
        const u32 rg = __ldg(t), b = __ldg(t + 1);
        if (alpha)
            return rgb3(half_bits_to_float(b >> 16), 0, 0);
        return rgb3(half_bits_to_float(rg & 0xffffu), half_bits_to_float(rg >> 16), half_bits_to_float(b & 0xffffu));
    }
    const u32 v = __ldg(im.texels + level.offset + index);
    const float *lut = im.transfer + transfer_offset;
    if (alpha)
        return rgb3(__ldg(lut + (v >> 24)), 0, 0);
    return rgb3(__ldg(lut + (v & 255u)), __ldg(lut + ((v >> 8) & 255u)), __ldg(lut + ((v >> 16) & 255u)));
}

// shaders/image_texture.h:64-73
RP_DEV bool valid_level(const DLevel &level, u32 texel_words, u32 format) {
    const u32 per = format == kTexelsFloat ? 4u : (format == kTexelsHalf ? 2u : 1u);
    return level.width > 0 && level.height > 0 && level.width <= 8192 && level.height <= 8192 &&
           level.offset <= texel_words && level.width * level.height * per <= texel_words - level.offset;
}

// Bilinear weights over the four texels around xy (texel space); a scalar lookup of a
// 3-channel image averages the channels, of a 4-channel image reads alpha
// (shaders/image_texture.h:75-95).
RP_DEV RGB bilinear_texels(const DImages &im, const DImageTexture &t, const DLevel &level, F2 xy, bool scalar) {
    const float fx = floorf(xy.x), fy = floorf(xy.y);
    const int bx = int(fx), by = int(fy);
    const float dx = xy.x - fx, dy = xy.y - fy;
    const bool alpha = scalar && t.channels == 4u;
    const RGB a = texel(im, level, bx, by, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const RGB b = texel(im, level, bx + 1, by, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const RGB c = texel(im, level, bx, by + 1, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const RGB e = texel(im, level, bx + 1, by + 1, t.wrap, t.texel_format, t.transfer_offset, alpha);
    const float w00 = (1.0f - dx) * (1.0f - dy), w10 = dx * (1.0f - dy), w01 = (1.0f - dx) * dy, w11 = dx * dy;
    RGB out = rgb3(w00 * a.r + w10 * b.r + w01 * c.r + w11 * e.r, w00 * a.g + w10 * b.g + w01 * c.g + w11 * e.g,
                   w00 * a.b + w10 * b.b + w01 * c.b + w11 * e.b);
    if (scalar && t.channels == 3u)
        out.r = (out.r + out.g + out.b) / 3.0f;
    return out;
}

// Wrap-aware bilinear lookup at texture coordinates st (shaders/image_texture.h:97-109).
RP_DEV RGB bilinear(const DImages &im, const DImageTexture &t, const DLevel &level, F2 st, bool scalar) {
    if (t.wrap == kWrapRepeat) {
        st.x -= floorf(st.x);
        st.y -= floorf(st.y);
    } else if (t.wrap == kWrapClamp) {
        st.x = fminf(fmaxf(st.x, 0.0f), 1.0f);
        st.y = fminf(fmaxf(st.y, 0.0f), 1.0f);
    } else if (st.x < -1.0f || st.y < -1.0f || st.x > 2.0f || st.y > 2.0f) {
        return rgb3(0, 0, 0);
    }
    return bilinear_texels(im, t, level, f2(st.x * float(level.width) - 0.5f, st.y * float(level.height) - 0.5f),
                           scalar);
}

// Nearest texel index along one axis (shaders/image_texture.h:127-139).
RP_DEV int point_coordinate(float st, float dimension, u32 wrap) {
    if (wrap == kWrapClamp)
        st = fminf(fmaxf(st, 0.0f), 1.0f);
    else if (wrap == kWrapBlack)
        st = fminf(fmaxf(st, -1.0f), 2.0f);
    const float index = roundf(st * dimension - 0.5f);
    if (wrap == kWrapRepeat)
        return isfinite(index) ? int(fmodf(index, dimension)) : 0;
    return int(index);
}

// shaders/image_texture.h:390-401
RP_DEV bool valid_lookup(const DImages &im, const DImageTexture &t, F2 uv, F2 dx, F2 dy) {
    return isfinite(uv.x) && isfinite(uv.y) && isfinite(dx.x) && isfinite(dx.y) && isfinite(dy.x) &&
           isfinite(dy.y) && t.wrap <= 2u && (t.channels == 1u || t.channels == 3u || t.channels == 4u) &&
           t.texel_format <= kTexelsFloat &&
           (t.texel_format >= kTexelsHalf ||
            (t.transfer_offset <= im.transfer_count && im.transfer_count - t.transfer_offset >= 256u)) &&
           t.level_count != 0 && t.level_begin <= im.level_count && t.level_count <= im.level_count - t.level_begin;
}

// PBRT's point, bilinear and trilinear lookups of a mip chain (shaders/image_texture.h:403-456).
// dx, dy are the texture-coordinate derivatives; mapped: uv and derivatives already carry
// the texture's scale and offset.
RP_DEV RGB lookup_standard(const DImages &im, const DImageTexture &t, F2 uv, F2 dx, F2 dy, bool scalar, bool mapped) {
    const bool point = t.filter == kFilterPoint;
    if (!valid_lookup(im, t, uv, dx, dy) || (!point && t.filter != kFilterBilinear && t.filter != kFilterTrilinear))
        return rgb_nan();
    if (!mapped) {
        dx = f2(dx.x * t.uscale, dx.y * t.vscale);
        dy = f2(dy.x * t.uscale, dy.y * t.vscale);
    }
    // a wide footprint selects the coordinate-independent coarsest level before anything
    // that could overflow
    const float extent = fmaxf(fmaxf(fabsf(dx.x), fabsf(dx.y)), fmaxf(fabsf(dy.x), fabsf(dy.y)));
    const float coarsest = float(t.level_count - 1u);
    float lod = coarsest;
    if (!(extent >= 0.5f)) {
        const float width = fmaxf(2.0f * extent, 1e-8f);
        const float log_width = logf(width) * 1.4426950408889634f;
        lod = coarsest + log_width;
    }
    const bool wide = lod >= coarsest;
    const u32 index = wide ? t.level_count - 1u : u32(fmaxf(0.0f, floorf(lod)));
    const DLevel level = im.levels[t.level_begin + index];
    if (!valid_level(level, im.texel_word_count, t.texel_format))
        return rgb_nan();
    if (wide)
        return texel(im, level, 0, 0, t.wrap, t.texel_format, t.transfer_offset);
    // the base level stays unblended for 0 <= lod < 1
    const bool interpolate = t.filter == kFilterTrilinear && index > 0;
    if (interpolate && !valid_level(im.levels[t.level_begin + index + 1u], im.texel_word_count, t.texel_format))
        return rgb_nan();
    F2 st = uv;
    if (!mapped) {
        const float su = uv.x * t.uscale, sv = uv.y * t.vscale;
        st = f2(su + t.udelta, sv + t.vdelta);
    }
    st.y = 1.0f - st.y;
    if (!isfinite(st.x) || !isfinite(st.y))
        return rgb_nan();
    if (point) {
        const int x = point_coordinate(st.x, float(level.width), t.wrap);
        const int y = point_coordinate(st.y, float(level.height), t.wrap);
        return texel(im, level, x, y, t.wrap, t.texel_format, t.transfer_offset);
    }
    const RGB lower = bilinear(im, t, level, st, scalar);
    if (!interpolate)
        return lower;
    const RGB upper = bilinear(im, t, im.levels[t.level_begin + index + 1u], st, scalar);
    const float delta = lod - float(index);
    return rgb3((1.0f - delta) * lower.r + delta * upper.r, (1.0f - delta) * lower.g + delta * upper.g,
                (1.0f - delta) * lower.b + delta * upper.b);
}

// ------------------------------------------------------------------ EWA
// PBRT's elliptically weighted average (shaders/image_texture.h:134-388): the footprint's
// ellipse, its minor axis capped by the anisotropy limit, filtered with a Gaussian on the two
// power-of-two mip levels around the minor axis and blended between them.
RP_DEV u32 ewa_magnitude(float v) { return __float_as_uint(v) & 0x7fffffffu; }
RP_DEV bool ewa_subnormal(u32 m) { return m != 0u && m < 0x00800000u; }
// value * scale, correctly rounded with gradual underflow, reconstructed from the
// significands when an operand or the product is subnormal (shaders/image_texture.h:168-204)
RP_DEV float ewa_product(float value, float scale) {
    const float mapped = value * scale;
    const u32 a = ewa_magnitude(value), b = ewa_magnitude(scale);
    if (a == 0u || b == 0u || (ewa_magnitude(mapped) != 0u && !ewa_subnormal(a) && !ewa_subnormal(b)))
        return mapped;
    const int a_exp = int(a >> 23), b_exp = int(b >> 23);
    const u32 a_sig = (a & 0x007fffffu) | (a_exp == 0 ? 0u : 0x00800000u);
    const u32 b_sig = (b & 0x007fffffu) | (b_exp == 0 ? 0u : 0x00800000u);
    const u64 product = u64(a_sig) * b_sig;
    const int exponent = max(1, a_exp) + max(1, b_exp) - 300;
    const int leading = 63 - __clzll((long long)product);
    const u32 sign = (__float_as_uint(value) ^ __float_as_uint(scale)) & 0x80000000u;
    if (exponent + leading > 127)
        return __uint_as_float(sign | 0x7f800000u);
    const int shift = max(leading - 23, -149 - exponent);
    if (shift > 48)
        return __uint_as_float(sign);
    u32 rounded;
    if (shift <= 0) {
        rounded = u32(product << -shift);
    } else {
        const u64 halfway = u64(1) << (shift - 1);
        const u64 truncated = product >> shift;
        rounded = u32((product + halfway - 1u + (truncated & 1u)) >> shift);
    }
    return __uint_as_float(sign | ((u32(exponent + shift + 149) << 23) + rounded));
}
// shaders/image_texture.h:206-211
RP_DEV float ewa_lift(float v) {
    const u32 m = ewa_magnitude(v);
    if (ewa_subnormal(m))
        return copysignf(float(m) * 0x1p-125f, v);
    return v * 0x1p24f;
}
// shaders/image_texture.h:141-152: the filter centre in texel space, keeping the sub-texel phase
// of large coordinates
RP_DEV float ewa_center(float st, float dimension, u32 wrap) {
    if (fabsf(st) <= 64.0f || wrap == kWrapBlack)
        return st * dimension - 0.5f;
    const float phase = fmodf(st, 1.0f) * dimension;
    if (wrap == kWrapRepeat)
        return phase - 0.5f;
    return ((st < 0.0f ? -64.0f : dimension + 64.0f) + phase) - 0.5f;
}
// shaders/image_texture.h:154-159
RP_DEV bool ewa_black_axis(float s, float d, float r) {
    return fabsf(s) > 64.0f && (s < (0.5f - r) / d || s > ((d - 0.5f) + r) / d);
}
// shaders/image_texture.h:134-139
RP_DEV bool ewa_level_valid(const DImages &im, const DLevel &l, u32 format, u32 levels_above) {
    return valid_level(l, im.texel_word_count, format) && (l.width & (l.width - 1u)) == 0u &&
           (l.height & (l.height - 1u)) == 0u && max(l.width, l.height) == (1u << levels_above);
}
// shaders/image_texture.h:213-256
RP_DEV RGB ewa_level(const DImages &im, const DImageTexture &t, const DLevel &l, F2 st, F2 dx, F2 dy) {
    const F2 dims = f2(float(l.width), float(l.height));
    const F2 u = f2(dx.x * dims.x, dx.y * dims.y), v = f2(dy.x * dims.x, dy.y * dims.y);
    const float area = u.x * v.y - u.y * v.x;
    const float determinant = ((1.0f + (u.x * u.x + u.y * u.y)) + (v.x * v.x + v.y * v.y)) + area * area;
    const F2 radius = f2(sqrtf((1.0f + u.x * u.x) + v.x * v.x), sqrtf((1.0f + u.y * u.y) + v.y * v.y));
    if (t.wrap == kWrapBlack && (ewa_black_axis(st.x, dims.x, radius.x) || ewa_black_axis(st.y, dims.y, radius.y)))
        return rgb3(0, 0, 0);
    const F2 center = f2(ewa_center(st.x, dims.x, t.wrap), ewa_center(st.y, dims.y, t.wrap));
    const float bx = ceilf(center.x - radius.x), by = ceilf(center.y - radius.y);
    const float ex = floorf(center.x + radius.x), ey = floorf(center.y + radius.y);
    const float cx = (ex - bx) + 1.0f, cy = (ey - by) + 1.0f;
    if (!isfinite(bx) || !isfinite(by) || !isfinite(ex) || !isfinite(ey) || fabsf(bx) > 0x1p19f || fabsf(by) > 0x1p19f ||
        fabsf(ex) > 0x1p19f || fabsf(ey) > 0x1p19f || cx <= 0.0f || cy <= 0.0f || cx * cy > 4096.0f)
        return rgb_nan();
    if (t.wrap == kWrapBlack && (ex < 0.0f || ey < 0.0f || bx >= dims.x || by >= dims.y))
        return rgb3(0, 0, 0);
    const int x0 = int(bx), y0 = int(by), x1 = int(ex), y1 = int(ey);
    RGB sum = rgb3(0, 0, 0);
    float weight_sum = 0;
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const float ddx = float(x) - center.x, ddy = float(y) - center.y;
            const float a = u.x * ddy - u.y * ddx, b = v.x * ddy - v.y * ddx;
            const float r2 = (((ddx * ddx + ddy * ddy) + a * a) + b * b) / determinant;
            if (r2 < 1.0f) {
                const float w = __ldg(im.ewa_weights + min(u32(128.0f * r2), 127u));
                const RGB c = texel(im, l, x, y, t.wrap, t.texel_format, t.transfer_offset);
                sum = rgb3(sum.r + w * c.r, sum.g + w * c.g, sum.b + w * c.b);
                weight_sum += w;
            }
        }
    if (!(isfinite(weight_sum) && weight_sum > 0.0f))
        return rgb_nan();
    return rgb3(sum.r / weight_sum, sum.g / weight_sum, sum.b / weight_sum);
}
// shaders/image_texture.h:258-388
RP_DEV RGB lookup_ewa(const DImages &im, const DImageTexture &t, F2 uv, F2 dx, F2 dy, bool scalar, bool mapped) {
    const float cap = t.max_anisotropy;
    if (t.level_count > 14u || !(cap >= 1.0f && cap <= 16.0f) || !isfinite(t.uscale) || !isfinite(t.vscale) ||
        !isfinite(t.udelta) || !isfinite(t.vdelta) || !im.ewa_weights)
        return rgb_nan();
    if (!mapped) {
        dx = f2(ewa_product(dx.x, t.uscale), ewa_product(dx.y, t.vscale));
        dy = f2(ewa_product(dy.x, t.uscale), ewa_product(dy.y, t.vscale));
    }
    if (!isfinite(dx.x) || !isfinite(dx.y) || !isfinite(dy.x) || !isfinite(dy.y))
        return rgb_nan();
    const u32 top = t.level_count - 1u;
    const DLevel *mips = im.levels + t.level_begin;
    const u32 x_bits = max(ewa_magnitude(dx.x), ewa_magnitude(dx.y));
    const u32 y_bits = max(ewa_magnitude(dy.x), ewa_magnitude(dy.y));
    const bool zero = x_bits == 0u || y_bits == 0u;
    float minor = 0.0f;
    if (!zero) {
        if (max(x_bits, y_bits) >= __float_as_uint(32.0f)) {
            minor = 2.0f;
        } else {
            const bool lifted = ewa_subnormal(ewa_magnitude(dx.x)) || ewa_subnormal(ewa_magnitude(dx.y)) ||
                                ewa_subnormal(ewa_magnitude(dy.x)) || ewa_subnormal(ewa_magnitude(dy.y));
            const F2 a = lifted ? f2(ewa_lift(dx.x), ewa_lift(dx.y)) : dx;
            const F2 b = lifted ? f2(ewa_lift(dy.x), ewa_lift(dy.y)) : dy;
            const float x_scale = fmaxf(fabsf(a.x), fabsf(a.y)), y_scale = fmaxf(fabsf(b.x), fabsf(b.y));
            const F2 x = f2(a.x / x_scale, a.y / x_scale), y = f2(b.x / y_scale, b.y / y_scale);
            const float x_norm = sqrtf(x.x * x.x + x.y * x.y), y_norm = sqrtf(y.x * y.x + y.y * y.y);
            const float x_length = x_scale * x_norm, y_length = y_scale * y_norm;
            const bool x_major = x_length >= y_length;
            const float major = x_major ? x_length : y_length;
            minor = x_major ? y_length : x_length;
            const float capped = major / cap;
            if (minor < capped) {
                const float actual = lifted ? capped * 0x1p-24f : capped;
                if (x_major)
                    dy = f2((y.x / y_norm) * actual, (y.y / y_norm) * actual);
                else
                    dx = f2((x.x / x_norm) * actual, (x.y / x_norm) * actual);
                minor = capped;
            }
            if (lifted)
                minor *= 0x1p-24f;
        }
        if (minor >= 2.0f) {
            if (!ewa_level_valid(im, mips[top], t.texel_format, 0))
                return rgb_nan();
            return texel(im, mips[top], 0, 0, t.wrap, t.texel_format, t.transfer_offset);
        }
    }
    F2 st = uv;
    if (!mapped)
        st = f2(ewa_product(uv.x, t.uscale) + t.udelta, ewa_product(uv.y, t.vscale) + t.vdelta);
    st.y = 1.0f - st.y;
    if (!isfinite(st.x) || !isfinite(st.y))
        return rgb_nan();
    if (zero) {
        if (!ewa_level_valid(im, mips[0], t.texel_format, top))
            return rgb_nan();
        const F2 dims = f2(float(mips[0].width), float(mips[0].height));
        if (t.wrap == kWrapBlack && (ewa_black_axis(st.x, dims.x, 1.0f) || ewa_black_axis(st.y, dims.y, 1.0f)))
            return rgb3(0, 0, 0);
        return bilinear_texels(im, t, mips[0], f2(ewa_center(st.x, dims.x, t.wrap), ewa_center(st.y, dims.y, t.wrap)),
                               scalar);
    }
    const float lod = fmaxf(0.0f, float(top) + log2f(minor));
    const u32 lower = min(u32(floorf(lod)), top);
    if (!ewa_level_valid(im, mips[lower], t.texel_format, top - lower))
        return rgb_nan();
    if (lower < top && (!ewa_level_valid(im, mips[lower + 1u], t.texel_format, top - lower - 1u) ||
                        mips[lower + 1u].width != max(1u, mips[lower].width / 2u) ||
                        mips[lower + 1u].height != max(1u, mips[lower].height / 2u)))
        return rgb_nan();
    const RGB a = ewa_level(im, t, mips[lower], st, dx, dy);
    const RGB b = lower == top ? texel(im, mips[top], 0, 0, t.wrap, t.texel_format, t.transfer_offset)
                               : ewa_level(im, t, mips[lower + 1u], st, dx, dy);
    const float delta = lod - float(lower);
    return rgb3((1.0f - delta) * a.r + delta * b.r, (1.0f - delta) * a.g + delta * b.g,
                (1.0f - delta) * a.b + delta * b.b);
}
// shaders/image_texture.h:541-554 (lookup_filtered)
RP_DEV RGB lookup_filtered(const DImages &im, const DImageTexture &t, F2 uv, F2 dx, F2 dy, bool scalar, bool mapped) {
    if (t.filter != kFilterEwa)
        return lookup_standard(im, t, uv, dx, dy, scalar, mapped);
    if (!valid_lookup(im, t, uv, dx, dy))
        return rgb_nan();
    return lookup_ewa(im, t, uv, dx, dy, scalar, mapped);
}

// ------------------------------------------------------------------ RGB -> spectrum
RP_DEV float blend1(float t, float a, float b) { return (1.0f - t) * a + t * b; }
// PBRT's sigmoid-polynomial reconstruction of a bounded reflectance from linear sRGB in
// [0, 1] (Jakob & Hanika 2019 tables; shaders/image_texture.h:458-499): the largest channel
// z picks a cell of the 64^3 grid, whose trilinearly blended coefficients give a quadratic
// in the wavelength, squashed by s(x) = 1/2 + x / (2 sqrt(1 + x^2)).  The coefficients do not
// depend on the wavelength, so they are blended once (rgb_polynomial) and the squashed
// quadratic evaluated per wavelength (rgb_polynomial_at); rgb_spectrum does both.
struct RgbPolynomial {
    float c0, c1, c2;
    float value; // the constant result of a grey or invalid input
    bool constant;
};
RP_DEV RgbPolynomial rgb_polynomial(const float *table, RGB c) {
    RgbPolynomial out{0, 0, 0, image_nan(), true};
    if (!finite_rgb(c))
        return out;
    c.r = fminf(fmaxf(c.r, 0.0f), 1.0f);
    c.g = fminf(fmaxf(c.g, 0.0f), 1.0f);
    c.b = fminf(fmaxf(c.b, 0.0f), 1.0f);
    if (c.r == c.g && c.g == c.b) {
        out.value = c.r;
        return out;
    }
    const float ch[3] = {c.r, c.g, c.b};
    u32 channel = 0;
    if (c.g >= c.r)
        channel = 1;
    if (c.b >= ch[channel])
        channel = 2;
    const float z = ch[channel];
    const float x = ch[(channel + 1u) % 3u] * 63.0f / z;
    const float y = ch[(channel + 2u) % 3u] * 63.0f / z;
    const u32 xi = min(u32(x), 62u), yi = min(u32(y), 62u);
    u32 lo = 1, hi = 63; // first interior node >= z
    while (lo < hi) {
        const u32 mid = (lo + hi) / 2u;
        if (__ldg(table + mid) < z)
            lo = mid + 1u;
        else
            hi = mid;
    }
    const u32 zi = lo - 1u;
    const float dx = x - float(xi), dy = y - float(yi);
    const float z0 = __ldg(table + zi), z1 = __ldg(table + zi + 1u);
    const float dz = (z - z0) / (z1 - z0);
    float coefficient[3];
    const u32 row = 3u * 64u, plane = row * 64u;
#pragma unroll
    for (u32 i = 0; i < 3; ++i) {
        const float *cell = table + 64u + 3u * (((channel * 64u + zi) * 64u + yi) * 64u + xi) + i;
        coefficient[i] = blend1(dz,
                                blend1(dy, blend1(dx, __ldg(cell), __ldg(cell + 3)),
                                       blend1(dx, __ldg(cell + row), __ldg(cell + row + 3))),
                                blend1(dy, blend1(dx, __ldg(cell + plane), __ldg(cell + plane + 3)),
                                       blend1(dx, __ldg(cell + plane + row), __ldg(cell + plane + row + 3))));
    }
    out.c0 = coefficient[0];
    out.c1 = coefficient[1];
    out.c2 = coefficient[2];
    out.constant = false;
    return out;
}
RP_DEV float rgb_polynomial_at(const RgbPolynomial &q, float wavelength) {
    if (q.constant)
        return q.value;
    const float poly = fmaf(fmaf(q.c0, wavelength, q.c1), wavelength, q.c2);
    if (!isfinite(poly))
        return image_nan();
    if (fabsf(poly) <= 1.0f)
        return 0.5f + 0.5f * poly / sqrtf(1.0f + poly * poly);
    const float inv = 1.0f / poly;
    return 0.5f + 0.5f * copysignf(1.0f / sqrtf(1.0f + inv * inv), poly);
}
RP_DEV float rgb_spectrum(const float *table, RGB c, float wavelength) {
    return rgb_polynomial_at(rgb_polynomial(table, c), wavelength);
}
// PBRT RGBUnboundedSpectrum: the reconstruction of rgb / (2 max) scaled back
// (shaders/image_texture.h:500-507).
RP_DEV float rgb_spectrum_unbounded(const float *table, RGB c, float wavelength) {
    if (!finite_rgb(c) || c.r < 0 || c.g < 0 || c.b < 0)
        return image_nan();
    const float scale = 2 * fmaxf(fmaxf(c.r, c.g), c.b);
    if (!isfinite(scale))
        return image_nan();
    return scale == 0 ? 0.0f : scale * rgb_spectrum(table, rgb3(c.r / scale, c.g / scale, c.b / scale), wavelength);
}

// ------------------------------------------------------------------ image environment
// The arithmetic of these helpers is mirrored by the oracle: vectors are normalised as
// v * (1 / |v|).
RP_DEV V3 unit_scaled(V3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
RP_DEV V3 mat3_apply(const float *m, V3 d) {
    return v3(dot(v3(m[0], m[1], m[2]), d), dot(v3(m[3], m[4], m[5]), d), dot(v3(m[6], m[7], m[8]), d));
}
constexpr float kSphereDensity = 0.25f / kPi;
constexpr float kUniformProbability = 0.0625f;

// An emitter's linear RGB as radiance: PBRT's RGBIlluminantSpectrum, the unbounded
// reconstruction of rgb times D65 at the nearest nanometre (shaders/image_lighting.h:28-40).
RP_DEV float illuminant_spectrum(const DImages &im, RGB c, float wavelength) {
    if (!finite_rgb(c) || !isfinite(wavelength))
        return image_nan();
    c = rgb3(fmaxf(0.0f, c.r), fmaxf(0.0f, c.g), fmaxf(0.0f, c.b));
    const float amplitude = 2.0f * fmaxf(fmaxf(c.r, c.g), c.b);
    if (amplitude == 0)
        return 0;
    const float nearest = roundf(wavelength);
    if (nearest < 360.0f || nearest > 830.0f)
        return 0;
    return amplitude * rgb_spectrum(im.rgb_table, rgb3(c.r / amplitude, c.g / amplitude, c.b / amplitude), wavelength) *
           __ldg(im.illuminant + (u32(nearest) - 360u));
}

// Clarberg's equal-area square-to-sphere map (PBRT EqualAreaSquareToSphere;
// shaders/image_lighting.h:82-93).
RP_DEV V3 square_to_sphere(F2 uv) {
    const float su = 2.0f * uv.x - 1.0f, sv = 2.0f * uv.y - 1.0f;
    const float qu = fabsf(su), qv = fabsf(sv);
    const float diagonal = 1.0f - (qu + qv);
    const float radius = 1.0f - fabsf(diagonal);
    const float phi = (radius == 0 ? 1.0f : (qv - qu) / radius + 1.0f) * (kPi / 4.0f);
    const float height = copysignf(1.0f - radius * radius, diagonal);
    const float radial = radius * sqrtf(fmaxf(0.0f, 2.0f - radius * radius));
    return v3(copysignf(cosf(phi), su) * radial, copysignf(sinf(phi), sv) * radial, height);
}
// The inverse map.  pinned: PBRT's polynomial arctangent, used for radiance lookups so a
// direction finds the texel PBRT reads; otherwise the analytic inverse, used for the
// sampling density (shaders/image_lighting.h:95-124).
RP_DEV F2 sphere_to_square(V3 d, bool pinned) {
    const V3 m = vabs(d);
    float radius, phi;
    if (pinned) {
        radius = sqrtf(fmaxf(0.0f, 1.0f - m.z));
        const float larger = fmaxf(m.x, m.y);
        const float ratio = larger == 0 ? 0.0f : fminf(m.x, m.y) / larger;
        phi = fmaf(ratio, -0.02513909723434835f, 0.041903881802916574f);
        phi = fmaf(ratio, phi, 0.08817706647753163f);
        phi = fmaf(ratio, phi, -0.24733373328126894f);
        phi = fmaf(ratio, phi, 0.006157201789828021f);
        phi = fmaf(ratio, phi, 0.6362265452740161f);
        phi = fmaf(ratio, phi, 0.000004067585662467885f);
        if (m.x < m.y)
            phi = 1.0f - phi;
    } else {
        const float horizontal = sqrtf(d.x * d.x + d.y * d.y);
        radius = horizontal / sqrtf(1.0f + m.z);
        phi = horizontal == 0 ? 0.0f : atan2f(m.y, m.x) * (2.0f / kPi);
    }
    F2 uv = f2(radius - phi * radius, phi * radius);
    if (d.z < 0)
        uv = f2(1.0f - uv.y, 1.0f - uv.x);
    uv = f2(copysignf(uv.x, d.x), copysignf(uv.y, d.y));
    return f2(fminf(fmaxf(0.5f * (uv.x + 1.0f), 0.0f), 1.0f), fminf(fmaxf(0.5f * (uv.y + 1.0f), 0.0f), 1.0f));
}

// Radiance of the environment image seen along a world direction: the nearest texel of the
// octahedral map, with the map's seams reflected as PBRT does (shaders/image_lighting.h:170-208).
RP_DEV float environment_image_radiance(const DImages &im, V3 world_direction, float wavelength) {
    if (im.env_image >= im.texture_count)
        return image_nan();
    const DImageTexture t = im.textures[im.env_image];
    const V3 d = unit_scaled(mat3_apply(im.env_from_world, world_direction));
    if (!finite3(d) || !valid_lookup(im, t, f2(0, 0), f2(0, 0), f2(0, 0)) || t.level_count != 1u)
        return image_nan();
    const DLevel level = im.levels[t.level_begin];
    if (!valid_level(level, im.texel_word_count, t.texel_format) || level.width != level.height)
        return image_nan();
    const int size = int(level.width);
    const F2 uv = sphere_to_square(d, true);
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
    const RGB c = texel(im, level, px, py, kWrapClamp, t.texel_format, t.transfer_offset);
    return im.env_scale * illuminant_spectrum(im, c, wavelength);
}

// environment_image_radiance at four wavelengths: the direction, the texel and the RGB's
// reconstruction coefficients are found once (they do not depend on the wavelength)
RP_DEV V4 environment_image_radiance4(const DImages &im, V3 world_direction, V4 lambda) {
    V4 out = v4(image_nan());
    if (im.env_image >= im.texture_count)
        return out;
    const DImageTexture t = im.textures[im.env_image];
    const V3 d = unit_scaled(mat3_apply(im.env_from_world, world_direction));
    if (!finite3(d) || !valid_lookup(im, t, f2(0, 0), f2(0, 0), f2(0, 0)) || t.level_count != 1u)
        return out;
    const DLevel level = im.levels[t.level_begin];
    if (!valid_level(level, im.texel_word_count, t.texel_format) || level.width != level.height)
        return out;
    const int size = int(level.width);
    const F2 uv = sphere_to_square(d, true);
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
    RGB c = texel(im, level, px, py, kWrapClamp, t.texel_format, t.transfer_offset);
    // illuminant_spectrum (shaders/image_lighting.h:28-40) with the coefficients shared
    const bool finite = finite_rgb(c);
    c = rgb3(fmaxf(0.0f, c.r), fmaxf(0.0f, c.g), fmaxf(0.0f, c.b));
    const float amplitude = 2.0f * fmaxf(fmaxf(c.r, c.g), c.b);
    RgbPolynomial q{0, 0, 0, 0, true};
    if (finite && amplitude != 0)
        q = rgb_polynomial(im.rgb_table, rgb3(c.r / amplitude, c.g / amplitude, c.b / amplitude));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float w = lambda.v[k];
        float value;
        if (!finite || !isfinite(w)) {
            value = image_nan();
        } else if (amplitude == 0) {
            value = 0;
        } else {
            const float nearest = roundf(w);
            value = nearest < 360.0f || nearest > 830.0f
                        ? 0.0f
                        : amplitude * rgb_polynomial_at(q, w) * __ldg(im.illuminant + (u32(nearest) - 360u));
        }
        out.v[k] = im.env_scale * value;
    }
    return out;
}
// shaders/image_lighting.h:210-219
RP_DEV bool environment_tables_valid(const DImages &im, bool compensated) {
    const u32 w = im.env_width;
    if (w == 0 || w > 8192)
        return false;
    const u32 count = (w + 1u) * (w + 1u);
    const u32 offset = compensated ? im.env_comp_offset : 0u;
    return (!compensated || offset >= count) && offset <= im.env_cdf_count && count <= im.env_cdf_count - offset;
}
// The importance cell of a world direction (shaders/image_lighting.h:221-231).
RP_DEV bool environment_cell(const DImages &im, V3 world_direction, u32 &cx, u32 &cy) {
    const V3 d = unit_scaled(mat3_apply(im.env_from_world, world_direction));
    if (!finite3(d))
        return false;
    const F2 uv = sphere_to_square(d, false);
    cx = min(u32(uv.x * float(im.env_width)), im.env_width - 1u);
    cy = min(u32(uv.y * float(im.env_width)), im.env_width - 1u);
    return true;
}
// Solid-angle density of a cell: the tables' piecewise-constant density over the equal-area
// square, mixed with 1/16 uniform unless compensated (shaders/image_lighting.h:233-246).
RP_DEV float environment_cell_density(const DImages &im, u32 cx, u32 cy, bool compensated) {
    const float *cdf = im.env_cdf + (compensated ? im.env_comp_offset : 0u);
    const u32 w = im.env_width;
    const float *row = cdf + (cy + 1u) * (w + 1u);
    const float marginal = __ldg(cdf + cy + 1u) - __ldg(cdf + cy);
    const float conditional = __ldg(row + cx + 1u) - __ldg(row + cx);
    if (!(marginal >= 0.0f && marginal <= 1.0f && conditional >= 0.0f && conditional <= 1.0f))
        return image_nan();
    const float density = (float(w) * marginal) * (float(w) * conditional);
    return kSphereDensity * (compensated ? density : kUniformProbability + (1.0f - kUniformProbability) * density);
}
// shaders/image_lighting.h:248-255
RP_DEV float environment_image_pdf(const DImages &im, V3 world_direction, bool compensated) {
    u32 cx, cy;
    if (!environment_tables_valid(im, compensated) || !environment_cell(im, world_direction, cx, cy))
        return image_nan();
    return environment_cell_density(im, cx, cy, compensated);
}
// Inverse-CDF sample of one table row (shaders/image_lighting.h:257-273).
RP_DEV float sample_table(const float *cdf, u32 width, float u, u32 &cell) {
    u32 lo = 0, hi = width;
    while (hi - lo > 1u) {
        const u32 mid = lo + (hi - lo) / 2u;
        if (u < __ldg(cdf + mid))
            hi = mid;
        else
            lo = mid;
    }
    const float c0 = __ldg(cdf + lo);
    const float mass = __ldg(cdf + hi) - c0;
    if (!(mass > 0.0f && mass <= 1.0f))
        return image_nan();
    cell = lo;
    const float fraction = fminf(fmaxf((u - c0) / mass, 0.0f), kOneMinusEps);
    return (float(lo) + fraction) / float(width);
}
// Sample a world direction from the environment image's tables; a sample whose inverse map
// lands in a neighbouring cell is walked toward the selected cell's centre in doubling
// steps (shaders/image_lighting.h:275-325).
RP_DEV bool sample_environment_image(const DImages &im, float ux, float uy, bool compensated, V3 &world_direction,
                                     float &pdf) {
    if (!environment_tables_valid(im, compensated) || !isfinite(ux) || !isfinite(uy) || ux < 0.0f || uy < 0.0f ||
        ux > 1.0f || uy > 1.0f)
        return false;
    const float *cdf = im.env_cdf + (compensated ? im.env_comp_offset : 0u);
    const bool importance = compensated || ux >= kUniformProbability;
    const u32 w = im.env_width;
    u32 row = 0, column = 0;
    F2 uv;
    if (!importance) {
        uv = f2(ux / kUniformProbability, uy);
    } else {
        uv.y = sample_table(cdf, w, fminf(uy, kOneMinusEps), row);
        const float uc = compensated ? ux : (ux - kUniformProbability) / (1.0f - kUniformProbability);
        uv.x = sample_table(cdf + (row + 1u) * (w + 1u), w, fminf(uc, kOneMinusEps), column);
    }
    if (!isfinite(uv.x) || !isfinite(uv.y))
        return false;
    world_direction = unit_scaled(mat3_apply(im.world_from_env, square_to_sphere(uv)));
    u32 cx, cy;
    if (!environment_cell(im, world_direction, cx, cy))
        return false;
    if (importance && (cx != column || cy != row)) {
        const F2 center = f2((float(column) + 0.5f) / float(w), (float(row) + 0.5f) / float(w));
        for (float weight = 0x1p-16f; weight <= 1.0f; weight *= 2.0f) {
            const F2 inward = f2(uv.x + (center.x - uv.x) * weight, uv.y + (center.y - uv.y) * weight);
            world_direction = unit_scaled(mat3_apply(im.world_from_env, square_to_sphere(inward)));
            if (!environment_cell(im, world_direction, cx, cy))
                return false;
            if (cx == column && cy == row)
                break;
        }
        if (cx != column || cy != row)
            return false;
    }
    pdf = environment_cell_density(im, cx, cy, compensated);
    return isfinite(pdf) && pdf > 0;
}

// ------------------------------------------------------------------ texture footprints
// PBRT ray differentials as rypath's shaders/texture_footprint.h computes them: at the primary
// hit from the camera rays one pixel over, elsewhere from the camera's minimum differentials
// (PBRT's Camera::Approximate_dp_dxy); then the texture-coordinate derivatives by least
// squares against the triangle's tangents.
// shaders/texture_footprint.h:14-20
RP_DEV V3 texture_direction(V3 d) {
    const float scale = fmaxf(fabsf(d.x), fmaxf(fabsf(d.y), fabsf(d.z)));
    if (!(scale > 0.0f) || !finite3(d))
        return v3(image_nan(), image_nan(), image_nan());
    return unit_scaled(v3(d.x / scale, d.y / scale, d.z / scale));
}
// shaders/texture_footprint.h:22-38
RP_DEV bool texture_primary_dp(V3 rel, V3 n, V3 dir, V3 xr, V3 yr, float spp_scale, V3 &dpdx, V3 &dpdy) {
    const V3 rx = dir + spp_scale * (texture_direction(xr) - dir);
    const V3 ry = dir + spp_scale * (texture_direction(yr) - dir);
    const float nx = dot(n, rx), ny = dot(n, ry);
    if (nx == 0.0f || ny == 0.0f || !isfinite(nx) || !isfinite(ny))
        return false;
    const float plane = dot(n, rel);
    dpdx = (plane / nx) * rx - rel;
    dpdy = (plane / ny) * ry - rel;
    return true;
}
// shaders/texture_footprint.h:40-43
RP_DEV V3 texture_reflect(V3 x, V3 normal) { return x - ((2.0f * dot(normal, x)) / dot(normal, normal)) * normal; }
// a row-major 3x3 matrix times a vector, summing the columns in order
RP_DEV V3 texture_apply(const float *m, V3 v) {
    return (v3(m[0], m[3], m[6]) * v.x + v3(m[1], m[4], m[7]) * v.y) + v3(m[2], m[5], m[8]) * v.z;
}
RP_DEV V3 texture_apply_transposed(const float *m, V3 v) {
    return (v3(m[0], m[1], m[2]) * v.x + v3(m[3], m[4], m[5]) * v.y) + v3(m[6], m[7], m[8]) * v.z;
}
// shaders/texture_footprint.h:45-58
RP_DEV V3 texture_approximate_axis(V3 pz, V3 nz, V3 delta, V3 u, V3 v, const float *world_from_camera,
                                   float spp_scale) {
    const V3 ray = v3(0, 0, 1) + delta;
    const float denom = dot(nz, ray);
    if (denom == 0.0f)
        return v3(0, 0, 0);
    const V3 offset = ((nz.z * pz.z) / denom) * ray - pz;
    const V3 dp = spp_scale * texture_apply(world_from_camera, texture_reflect(texture_reflect(offset, v), u));
    return finite3(dp) ? dp : v3(0, 0, 0);
}
// shaders/texture_footprint.h:60-86
RP_DEV void texture_approximate_dp(const DImages &im, V3 rel, V3 n, V3 &dpdx, V3 &dpdy) {
    const V3 pc = texture_apply(im.camera_from_world, rel);
    const V3 direction = texture_direction(pc);
    if (!finite3(direction)) {
        dpdx = dpdy = v3(0, 0, 0);
        return;
    }
    // RotateFromTo(direction, +z) as two reflections
    const V3 ref = fabsf(direction.x) < 0.72f ? v3(1, 0, 0) : v3(0, 1, 0);
    const V3 u = ref - direction, v = ref - v3(0, 0, 1);
    const V3 pz = texture_reflect(texture_reflect(pc, u), v);
    const V3 nz = texture_reflect(texture_reflect(texture_apply_transposed(im.world_from_camera, n), u), v);
    const V3 mdx = v3(im.tex_min_dx[0], im.tex_min_dx[1], im.tex_min_dx[2]);
    const V3 mdy = v3(im.tex_min_dy[0], im.tex_min_dy[1], im.tex_min_dy[2]);
    dpdx = texture_approximate_axis(pz, nz, mdx, u, v, im.world_from_camera, im.tex_spp_scale);
    dpdy = texture_approximate_axis(pz, nz, mdy, u, v, im.world_from_camera, im.tex_spp_scale);
}
// Kahan's difference of products (shaders/texture_footprint.h:139-142)
RP_DEV float texture_difference_of_products(float a, float b, float c, float d) {
    const float cd = c * d;
    return fmaf(a, b, -cd) + fmaf(-c, d, cd);
}
// shaders/texture_footprint.h:144-159
RP_DEV float texture_sanitize(float d) { return isfinite(d) ? fminf(fmaxf(d, -1e8f), 1e8f) : 0.0f; }
RP_DEV F2 texture_solve_axis(V3 dpdu, V3 dpdv, V3 dp, float aa, float ab, float bb, float inv_det) {
    const float u = dot(dpdu, dp), v = dot(dpdv, dp);
    return f2(texture_sanitize(inv_det * texture_difference_of_products(bb, u, ab, v)),
              texture_sanitize(inv_det * texture_difference_of_products(aa, v, ab, u)));
}
// shaders/texture_footprint.h:161-185
RP_DEV bool texture_uv_derivatives(V3 dpdu, V3 dpdv, V3 dpdx, V3 dpdy, F2 &dstdx, F2 &dstdy) {
    if (!finite3(dpdu) || !finite3(dpdv))
        return false;
    const float aa = dot(dpdu, dpdu), ab = dot(dpdu, dpdv), bb = dot(dpdv, dpdv);
    const float det = texture_difference_of_products(aa, bb, ab, ab);
    const float inv_det = 1.0f / det;
    if (!isfinite(inv_det)) {
        dstdx = dstdy = f2(0, 0);
        return true;
    }
    dstdx = texture_solve_axis(dpdu, dpdv, dpdx, aa, ab, bb, inv_det);
    dstdy = texture_solve_axis(dpdu, dpdv, dpdy, aa, ab, bb, inv_det);
    return true;
}

} // namespace rp
