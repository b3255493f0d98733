// ORACLE -- test infrastructure only (see oracle_math.hpp).  Sample identity, draw words,
// camera rays and positional-light intensity shared by the hero and scalar transports.
#pragma once

#include "oracle_scene.hpp"

#include <cfloat>

namespace oracle {

struct Params {
    u32 width, height, pixel_begin, pixel_count, sample_low, sample_high;
    u32 seed_low, seed_high, sampler, randomization, m, emergency_limit, max_depth;
};

struct Sample {
    u32 status = 0, pixel = 0, sample_low = 0, sample_high = 0;
    u32 words[4] = {0, 0, 0, 0};
};

// shaders/render.metal:113-118 (sobol and independent samplers)
inline float sample_uniform(const Params &p, u32 w) {
    return p.sampler == RP_SAMPLER_INDEPENDENT ? u01(w) : sobol_uniform(w);
}
// shaders/render.metal:154-179 (draw_words)
inline U4 draw_words(const Scene &s, const Params &p, const Sample &smp, u64 index, u32 block) {
    if (p.sampler == RP_SAMPLER_INDEPENDENT)
        return philox(U4{smp.pixel, smp.sample_low, smp.sample_high, block}, p.seed_low, p.seed_high);
    const u32 d = 4 * block;
    const SobolTables &t = *s.sobol;
    return U4{sobol_word(t, index, d, p.randomization, p.seed_low),
              sobol_word(t, index, d + 1, p.randomization, p.seed_low),
              sobol_word(t, index, d + 2, p.randomization, p.seed_low),
              sobol_word(t, index, d + 3, p.randomization, p.seed_low)};
}
// shaders/render.metal:238-311 (begin_sample; pinhole, box/triangle filter)
inline Sample begin_sample(const Scene &s, const Params &p, u32 lane, u64 &index) {
    Sample r;
    r.pixel = p.pixel_begin + lane % p.pixel_count;
    r.sample_low = p.sample_low + lane / p.pixel_count;
    r.sample_high = p.sample_high + u32(r.sample_low < p.sample_low);
    const u64 sample = (u64(r.sample_high) << 32) | r.sample_low;
    if (p.sampler == RP_SAMPLER_SOBOL) {
        const SobolTables &t = *s.sobol;
        index = sobol_index(t, p.m, r.pixel % p.width, r.pixel / p.width, sample);
        r.words[0] = sobol_word(t, index, 0, 0, 0);
        r.words[1] = sobol_word(t, index, 1, 0, 0);
        r.words[2] = sobol_word(t, index, 2, p.randomization, p.seed_low);
        r.words[3] = sobol_word(t, index, 3, p.randomization, p.seed_low);
    } else {
        index = 0;
        const U4 w = philox(U4{r.pixel, r.sample_low, r.sample_high, 0}, p.seed_low, p.seed_high);
        r.words[0] = w.x;
        r.words[1] = w.y;
        r.words[2] = w.z;
        r.words[3] = w.w;
    }
    return r;
}
// shaders/render.metal:352-357
inline float triangle_offset(float u, float radius) {
    const float s = 2.0f * u - 1.0f;
    return radius * (s / (1.0f + std::sqrt(1.0f - std::fabs(s))));
}
// shaders/render.metal:341-350, :400-476 (primary_ray, PBRT model, no lens)
inline void primary_ray(const Scene &s, const Params &p, const Sample &smp, F3 &o, F3 &d) {
    float ux, uy;
    if (p.sampler == RP_SAMPLER_SOBOL) {
        ux = sobol_camera_uniform(smp.words[0], p.m, smp.pixel % p.width);
        uy = sobol_camera_uniform(smp.words[1], p.m, smp.pixel / p.width);
    } else {
        ux = sample_uniform(p, smp.words[0]);
        uy = sample_uniform(p, smp.words[1]);
    }
    o = s.origin;
    const bool centered = s.filter_kind != RP_FILTER_BOX || s.filter_x != 0.5f || s.filter_y != 0.5f;
    if (centered) {
        const float ox = s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(ux, s.filter_x)
                                                             : (2.0f * ux - 1.0f) * s.filter_x;
        const float oy = s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(uy, s.filter_y)
                                                             : (2.0f * uy - 1.0f) * s.filter_y;
        const float x = ((float(smp.pixel % p.width) + 0.5f) + ox) / float(p.width);
        const float y = ((float(smp.pixel / p.width) + 0.5f) + oy) / float(p.height);
        const F3 dd = fma3(F3{y, y, y}, s.up, fma3(F3{x, x, x}, s.right, s.forward));
        const float scale = std::max(std::fabs(dd.x), std::max(std::fabs(dd.y), std::fabs(dd.z)));
        if (!finite3(dd) || !(scale > 0.0f)) {
            d = F3{NAN, NAN, NAN};
            return;
        }
        const F3 scaled = dd / scale;
        if (!finite3(scaled) || zero3(scaled)) {
            d = F3{NAN, NAN, NAN};
            return;
        }
        d = normalize3(scaled);
        return;
    }
    const float x = (float(smp.pixel % p.width) + ux) / float(p.width);
    const float y = (float(smp.pixel / p.width) + uy) / float(p.height);
    const F3 dd = s.forward + x * s.right + y * s.up;
    const float scale = std::max(std::fabs(dd.x), std::max(std::fabs(dd.y), std::fabs(dd.z)));
    d = normalize3(dd / scale);
}

// ---------------------------------------------------------------- positional lights
// shaders/render.metal:654-657, :682-697
inline bool normal_or_zero(float v) {
    const u32 m = fbits(v) & 0x7fffffffu;
    return m == 0 || (m >= 0x00800000u && m < 0x7f800000u);
}
inline bool spot_product(float a, float b, float &r) {
    if (a != 0 && b != 0 && std::fabs(a) < FLT_MIN / std::fabs(b))
        return false;
    r = a * b;
    return normal_or_zero(r) && (r != 0 || a == 0 || b == 0);
}
inline bool spot_sum(float a, float b, float &r) {
    r = a + b;
    return normal_or_zero(r) && (r != 0 || a == -b);
}
inline bool spot_divide(float a, float b, float &r) {
    r = a / b;
    return normal_or_zero(r) && (r != 0 || a == 0);
}
// shaders/render.metal:699-811 (positional_intensity, point and spot)
inline bool positional_intensity(const Positional &L, F3 wi, float &intensity) {
    if (L.kind == RP_POINT_LIGHT)
        return true;
    if (L.kind != RP_SPOT_LIGHT)
        return false;
    F3 w;
    for (int row = 0; row < 3; ++row) {
        float terms[3];
        for (int col = 0; col < 3; ++col)
            if (!spot_product(L.light_from_world[row * 3 + col], -wi[col], terms[col]))
                return false;
        float sum, comp;
        if (!spot_sum(terms[0], terms[1], sum) || !spot_sum(sum, terms[2], comp))
            return false;
        w[row] = comp;
    }
    const float scale = std::max(std::max(std::fabs(w.x), std::fabs(w.y)), std::fabs(w.z));
    if (!(scale >= FLT_MIN) || !std::isfinite(scale))
        return false;
    for (int i = 0; i < 3; ++i) {
        float c;
        if (!spot_divide(w[i], scale, c))
            return false;
        w[i] = c;
    }
    float cosine;
    if (!spot_divide(w.z, std::sqrt(dot(w, w)), cosine))
        return false;
    const float end = L.cos_falloff_end, start = L.cos_falloff_start;
    const float t = start == end ? (cosine < end ? 0.0f : 1.0f)
                                 : std::clamp((cosine - end) / (start - end), 0.0f, 1.0f);
    const float falloff = start == end ? t : t * t * (3.0f - 2.0f * t);
    intensity *= falloff;
    return std::isfinite(intensity) && intensity >= 0;
}

inline Params make_params(const Scene &s, const rp_request &r) {
    Params p{};
    p.width = r.width;
    p.height = r.height;
    p.pixel_begin = r.pixel_begin;
    p.pixel_count = r.pixel_count;
    p.sample_low = u32(r.sample_begin);
    p.sample_high = u32(r.sample_begin >> 32);
    p.seed_low = u32(r.seed);
    p.seed_high = u32(r.seed >> 32);
    p.sampler = r.sampler_kind;
    p.randomization = r.randomization;
    p.m = r.sampler_kind == RP_SAMPLER_SOBOL ? sobol_scale_exponent(r.width, r.height) : 0;
    p.emergency_limit = r.emergency_limit ? r.emergency_limit : 1024;
    p.max_depth = s.max_depth;
    return p;
}

} // namespace oracle
