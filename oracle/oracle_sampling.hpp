// ORACLE -- test infrastructure only (see oracle_math.hpp).  Sample identity, draw words,
// camera rays and positional-light intensity shared by the hero and scalar transports.
#pragma once

#include "oracle_scene.hpp"

#include <cfloat>

namespace oracle {

struct Params {
    u32 width, height, pixel_begin, pixel_count, sample_low, sample_high;
    u32 seed_low, seed_high, sampler, randomization, m, emergency_limit, max_depth;
    u32 log_spp;        // ZSobol: floor(log2(total samples))
    u32 boundary_limit; // pass-through crossings allowed between two vertices
    // texture footprints (scenes with image reflectance): the request's differential scale and
    // the camera's minimum one-pixel differentials (src/metal_render.mm:1940-1963)
    float tex_spp_scale = 1;
    F3 tex_min_dx{}, tex_min_dy{};
};

struct Sample {
    u32 status = 0, pixel = 0, sample_low = 0, sample_high = 0;
    u32 words[4] = {0, 0, 0, 0};
    u32 lens_words[2] = {0, 0};
    float filter_offsets[2] = {0, 0};
    u32 closest_walks = 0, shadow_walks = 0; // traversal queries of the lane (closest hit / occlusion)
};
// shaders/render.metal:200-236 (gaussian_filter_offsets)
inline void gaussian_filter_offsets(const Scene &s, float ux, float uy, float &x, float &y) {
    const float *cdf = s.gauss_cdf.data();
    const float *marginal = cdf + size_t(s.gauss_h) * (s.gauss_w + 1);
    u32 low = 0, high = s.gauss_h;
    while (low + 1 < high) {
        const u32 mid = (low + high) / 2;
        if (marginal[mid] <= uy)
            low = mid;
        else
            high = mid;
    }
    const u32 row = low;
    const float ty = (float(row) + (uy - marginal[row]) / (marginal[row + 1] - marginal[row])) / float(s.gauss_h);
    const float *conditional = cdf + size_t(row) * (s.gauss_w + 1);
    low = 0;
    high = s.gauss_w;
    while (low + 1 < high) {
        const u32 mid = (low + high) / 2;
        if (conditional[mid] <= ux)
            low = mid;
        else
            high = mid;
    }
    const float tx = (float(low) + (ux - conditional[low]) / (conditional[low + 1] - conditional[low])) / float(s.gauss_w);
    x = (1 - tx) * (-s.filter_x) + tx * s.filter_x;
    y = (1 - ty) * (-s.filter_y) + ty * s.filter_y;
}

// shaders/render.metal:113-122
inline float sample_uniform(const Params &p, u32 w) {
    if (p.sampler == RP_SAMPLER_HALTON)
        return ffrom(w);
    return p.sampler == RP_SAMPLER_INDEPENDENT ? u01(w) : sobol_uniform(w);
}
inline u32 decision_word(const Params &p, u32 w) {
    return p.sampler == RP_SAMPLER_HALTON ? u32(ffrom(w) * 0x1p32f) : w;
}
// shaders/render.metal:123-127
inline u32 zdraw(const Scene &s, const Params &p, u64 index, u32 dimension, u32 axis = 0, bool pair = false) {
    return zsobol_word(*s.sobol, index, dimension, axis, pair, p.m, p.log_spp, p.randomization, p.seed_low);
}
// shaders/render.metal:154-179 (draw_words)
inline U4 draw_words(const Scene &s, const Params &p, const Sample &smp, u64 index, u32 block) {
    if (p.sampler == RP_SAMPLER_INDEPENDENT)
        return philox(U4{smp.pixel, smp.sample_low, smp.sample_high, block}, p.seed_low, p.seed_high);
    const u32 d = 4 * block;
    if (p.sampler == RP_SAMPLER_HALTON)
        return U4{fbits(qmc_radical(d, index, p.randomization, p.seed_low)),
                  fbits(qmc_radical(d + 1, index, p.randomization, p.seed_low)),
                  fbits(qmc_radical(d + 2, index, p.randomization, p.seed_low)),
                  fbits(qmc_radical(d + 3, index, p.randomization, p.seed_low))};
    if (p.sampler == RP_SAMPLER_ZSOBOL) {
        const bool even = (block & 1) == 0;
        return U4{zdraw(s, p, index, d, 0, true), zdraw(s, p, index, d, 1, true), zdraw(s, p, index, d + 2, 0, even),
                  zdraw(s, p, index, even ? d + 2 : d + 3, even ? 1 : 0, even)};
    }
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
    } else if (p.sampler == RP_SAMPLER_HALTON) {
        index = halton_index(p.width, p.height, r.pixel % p.width, r.pixel / p.width, sample);
        r.words[0] = fbits(halton_camera(0, p.width, index));
        r.words[1] = fbits(halton_camera(1, p.height, index));
        r.words[2] = fbits(qmc_radical(2, index, p.randomization, p.seed_low));
        r.words[3] = fbits(qmc_radical(3, index, p.randomization, p.seed_low));
    } else if (p.sampler == RP_SAMPLER_ZSOBOL) {
        index = zsobol_morton(r.pixel % p.width, r.pixel / p.width, p.log_spp, sample);
        r.words[0] = zdraw(s, p, index, 1, 0, true);
        r.words[1] = zdraw(s, p, index, 1, 1, true);
        r.words[2] = zdraw(s, p, index, 0);
        r.words[3] = zdraw(s, p, index, 3);
    } else {
        index = 0;
        const U4 w = philox(U4{r.pixel, r.sample_low, r.sample_high, 0}, p.seed_low, p.seed_high);
        r.words[0] = w.x;
        r.words[1] = w.y;
        r.words[2] = w.z;
        r.words[3] = w.w;
    }
    if (s.lens_radius > 0) {
        if (p.sampler == RP_SAMPLER_SOBOL) {
            const SobolTables &t = *s.sobol;
            r.lens_words[0] = sobol_word(t, index, 1022, p.randomization, p.seed_low); // lens_x_dimension
            r.lens_words[1] = sobol_word(t, index, 1023, p.randomization, p.seed_low);
        } else if (p.sampler == RP_SAMPLER_HALTON) {
            r.lens_words[0] = fbits(qmc_radical(998, index, p.randomization, p.seed_low));
            r.lens_words[1] = fbits(qmc_radical(999, index, p.randomization, p.seed_low));
        } else if (p.sampler == RP_SAMPLER_ZSOBOL) {
            r.lens_words[0] = zdraw(s, p, index, 1022, 0, true);
            r.lens_words[1] = zdraw(s, p, index, 1022, 1, true);
        } else {
            const U4 w = philox(U4{r.pixel, r.sample_low, r.sample_high, 0xc0000000u}, p.seed_low, p.seed_high);
            r.lens_words[0] = w.x;
            r.lens_words[1] = w.y;
        }
    }
    if (s.filter_kind == RP_FILTER_GAUSSIAN) {
        const float ux = p.sampler == RP_SAMPLER_SOBOL ? sobol_camera_uniform(r.words[0], p.m, r.pixel % p.width)
                                                       : sample_uniform(p, r.words[0]);
        const float uy = p.sampler == RP_SAMPLER_SOBOL ? sobol_camera_uniform(r.words[1], p.m, r.pixel / p.width)
                                                       : sample_uniform(p, r.words[1]);
        gaussian_filter_offsets(s, ux, uy, r.filter_offsets[0], r.filter_offsets[1]);
    }
    return r;
}
// shaders/render.metal:352-357
inline float triangle_offset(float u, float radius) {
    const float s = 2.0f * u - 1.0f;
    return radius * (s / (1.0f + std::sqrt(1.0f - std::fabs(s))));
}
// shaders/render.metal:341-476 (primary_ray: pinhole or thin lens; box, triangle or Gaussian filter)
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
    F3 dd;
    if (centered) {
        const float ox = s.filter_kind == RP_FILTER_GAUSSIAN   ? smp.filter_offsets[0]
                         : s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(ux, s.filter_x)
                                                               : (2.0f * ux - 1.0f) * s.filter_x;
        const float oy = s.filter_kind == RP_FILTER_GAUSSIAN   ? smp.filter_offsets[1]
                         : s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(uy, s.filter_y)
                                                               : (2.0f * uy - 1.0f) * s.filter_y;
        const float x = ((float(smp.pixel % p.width) + 0.5f) + ox) / float(p.width);
        const float y = ((float(smp.pixel / p.width) + 0.5f) + oy) / float(p.height);
        dd = fma3(F3{y, y, y}, s.up, fma3(F3{x, x, x}, s.right, s.forward));
    } else {
        const float x = (float(smp.pixel % p.width) + ux) / float(p.width);
        const float y = (float(smp.pixel / p.width) + uy) / float(p.height);
        dd = s.forward + x * s.right + y * s.up;
    }
    if (s.lens_radius > 0) {
        // lens_point (shaders/render.metal:366-387): concentric disk, PBRT perspective lens
        const float lx = 2.0f * sample_uniform(p, smp.lens_words[0]) - 1.0f;
        const float ly = 2.0f * sample_uniform(p, smp.lens_words[1]) - 1.0f;
        F3 offset{0, 0, 0};
        if (!(lx == 0 && ly == 0)) {
            const float pi = 3.14159265358979323846f;
            float radius, theta;
            if (std::fabs(lx) > std::fabs(ly)) {
                radius = lx;
                theta = (pi / 4.0f) * (ly / lx);
            } else {
                radius = ly;
                theta = pi / 2.0f - (pi / 4.0f) * (lx / ly);
            }
            const float r = s.lens_radius * radius;
            const F3 ideal = (r * std::cos(theta)) * s.lens_x + (r * std::sin(theta)) * s.lens_y;
            o = s.origin + ideal;
            offset = o - s.origin;
        }
        // lens_primary_ray (:413-432) and rypath_texture_direction (shaders/texture_footprint.h:14-20)
        dd = dd - offset / s.focal_distance;
        const float scale = std::max(std::fabs(dd.x), std::max(std::fabs(dd.y), std::fabs(dd.z)));
        d = (!(scale > 0.0f) || !finite3(dd)) ? F3{NAN, NAN, NAN} : normalize3(dd / scale);
        return;
    }
    const float scale = std::max(std::fabs(dd.x), std::max(std::fabs(dd.y), std::fabs(dd.z)));
    if (centered) {
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
    if (s.model == RP_MODEL_DEMO) {
        // the demo camera (shaders/render.metal:470-475): a look-at basis and tan(fov / 2)
        const float x = (float(smp.pixel % p.width) + ux) / float(p.width);
        const float y = (float(smp.pixel / p.width) + uy) / float(p.height);
        const float aspect = float(p.width) / float(p.height);
        d = normalize3((s.forward + (((2.0f * x - 1.0f) * aspect) * s.film_scale) * s.right) +
                       ((1.0f - 2.0f * y) * s.film_scale) * s.up);
        return;
    }
    d = normalize3(dd / scale);
}

// shaders/render.metal:479-501 (texture_camera_rays): the camera directions one pixel right and
// one pixel down of the sample's film position, through the lens sample's focus shift; and the
// lens sample's aperture offset (lens_offset, :390-392)
inline void texture_camera_rays(const Scene &s, const Params &p, const Sample &smp, F3 &rx, F3 &ry, F3 &lens) {
    float ux, uy;
    if (p.sampler == RP_SAMPLER_SOBOL) {
        ux = sobol_camera_uniform(smp.words[0], p.m, smp.pixel % p.width);
        uy = sobol_camera_uniform(smp.words[1], p.m, smp.pixel / p.width);
    } else {
        ux = sample_uniform(p, smp.words[0]);
        uy = sample_uniform(p, smp.words[1]);
    }
    const bool centered = s.filter_kind != RP_FILTER_BOX || s.filter_x != 0.5f || s.filter_y != 0.5f;
    F3 dd;
    if (centered) {
        const float ox = s.filter_kind == RP_FILTER_GAUSSIAN   ? smp.filter_offsets[0]
                         : s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(ux, s.filter_x)
                                                               : (2.0f * ux - 1.0f) * s.filter_x;
        const float oy = s.filter_kind == RP_FILTER_GAUSSIAN   ? smp.filter_offsets[1]
                         : s.filter_kind == RP_FILTER_TRIANGLE ? triangle_offset(uy, s.filter_y)
                                                               : (2.0f * uy - 1.0f) * s.filter_y;
        const float x = ((float(smp.pixel % p.width) + 0.5f) + ox) / float(p.width);
        const float y = ((float(smp.pixel / p.width) + 0.5f) + oy) / float(p.height);
        dd = fma3(F3{y, y, y}, s.up, fma3(F3{x, x, x}, s.right, s.forward));
    } else {
        const float x = (float(smp.pixel % p.width) + ux) / float(p.width);
        const float y = (float(smp.pixel / p.width) + uy) / float(p.height);
        dd = s.forward + x * s.right + y * s.up;
    }
    rx = dd + s.right / float(p.width);
    ry = dd + s.up / float(p.height);
    lens = F3{0, 0, 0};
    if (s.lens_radius > 0) {
        const float lx = 2.0f * sample_uniform(p, smp.lens_words[0]) - 1.0f;
        const float ly = 2.0f * sample_uniform(p, smp.lens_words[1]) - 1.0f;
        if (!(lx == 0 && ly == 0)) {
            const float pi = 3.14159265358979323846f;
            float radius, theta;
            if (std::fabs(lx) > std::fabs(ly)) {
                radius = lx;
                theta = (pi / 4.0f) * (ly / lx);
            } else {
                radius = ly;
                theta = pi / 2.0f - (pi / 4.0f) * (lx / ly);
            }
            const float r = s.lens_radius * radius;
            const F3 ideal = (r * std::cos(theta)) * s.lens_x + (r * std::sin(theta)) * s.lens_y;
            lens = (s.origin + ideal) - s.origin;
        }
        const F3 shift = lens / s.focal_distance;
        rx = rx - shift;
        ry = ry - shift;
    }
}

// shaders/render.metal:1312-1408 (surface_texture_context) for a triangle hit (b1, b2) of
// instance `inst`, local triangle `local`: the texture coordinates and their screen-space
// derivatives.  scatterings: the path's scattering events so far (0 at the primary hit, which
// uses the camera's ray differentials).  False when the inputs are invalid.
inline bool texture_context(const Scene &s, const Params &p, const Sample &smp, u32 inst, u32 local, float b1,
                            float b2, F3 geometric_normal, F3 primary_direction, u32 scatterings, F2 &st, F2 &dstdx,
                            F2 &dstdy) {
    const Instance &in = s.instances[inst];
    const Images &im = s.images;
    const auto &tri = s.triangles[in.triangle_begin + local];
    const F3 p0 = s.positions[in.vertex_begin + tri[0]], p1 = s.positions[in.vertex_begin + tri[1]],
             p2 = s.positions[in.vertex_begin + tri[2]];
    const F3 local_p = fma3(F3{b2, b2, b2}, p2 - p0, fma3(F3{b1, b1, b1}, p1 - p0, p0));
    F2 uv[3] = {{0, 0}, {1, 0}, {1, 1}};
    const u32 uv_begin = im.inst_uv_begin.empty() ? RP_NONE : im.inst_uv_begin[inst];
    if (uv_begin != RP_NONE) {
        const u32 count = u32(im.uvs.size());
        for (int k = 0; k < 3; ++k) {
            if (uv_begin >= count || tri[k] >= count - uv_begin)
                return false;
            uv[k] = im.uvs[uv_begin + tri[k]];
            if (!std::isfinite(uv[k].x) || !std::isfinite(uv[k].y))
                return false;
        }
    }
    const float w0 = 1.0f - (b1 + b2);
    st = {(w0 * uv[0].x + b1 * uv[1].x) + b2 * uv[2].x, (w0 * uv[0].y + b1 * uv[1].y) + b2 * uv[2].y};
    const u32 frame_begin = im.inst_frame_begin.empty() ? RP_NONE : im.inst_frame_begin[inst];
    const u32 frame_count = u32(im.frames.size());
    if (!std::isfinite(st.x) || !std::isfinite(st.y) || frame_begin >= frame_count || local >= frame_count - frame_begin)
        return false;
    const F3 dpdu = im.frames[frame_begin + local][0], dpdv = im.frames[frame_begin + local][1];
    // texture_world_vector (:1139-1143) of the local point, plus the translation less the camera
    const auto world_vector = [&](F3 v) {
        return F3{dot(F3{in.m[0], in.m[1], in.m[2]}, v), dot(F3{in.m[4], in.m[5], in.m[6]}, v),
                  dot(F3{in.m[8], in.m[9], in.m[10]}, v)};
    };
    const F3 relative_p = world_vector(local_p) + (F3{in.m[3], in.m[7], in.m[11]} - s.origin);
    if (!finite3(relative_p))
        return false;
    F3 dpdx{}, dpdy{};
    bool primary = false;
    if (scatterings == 0) {
        F3 rx, ry, lens;
        texture_camera_rays(s, p, smp, rx, ry, lens);
        if (!finite3(rx) || !finite3(ry))
            return false;
        const F3 lens_relative = s.lens_radius > 0 ? relative_p - lens : relative_p;
        primary = texture_primary_dp(lens_relative, geometric_normal, primary_direction, rx, ry, p.tex_spp_scale,
                                     dpdx, dpdy);
    }
    if (!primary)
        texture_approximate_dp(relative_p, geometric_normal, im.world_from_camera, im.camera_from_world, p.tex_min_dx,
                               p.tex_min_dy, p.tex_spp_scale, dpdx, dpdy);
    return texture_uv_derivatives(dpdu, dpdv, dpdx, dpdy, dstdx, dstdy);
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
    p.m = r.sampler_kind == RP_SAMPLER_SOBOL || r.sampler_kind == RP_SAMPLER_ZSOBOL
              ? sobol_scale_exponent(r.width, r.height)
              : 0;
    p.log_spp = r.sampler_kind == RP_SAMPLER_ZSOBOL && r.total_samples ? 63 - __builtin_clzll(r.total_samples) : 0;
    p.emergency_limit = r.emergency_limit ? r.emergency_limit : 1024;
    p.max_depth = s.max_depth;
    p.boundary_limit = r.boundary_limit ? r.boundary_limit : 4096; // medium_boundary_limit, src/render.hpp:26
    if (s.textured) {
        p.tex_spp_scale = texture_differential_scale(r.total_samples);
        texture_camera_differentials(s.forward, s.right, s.up, r.width, r.height, p.tex_min_dx, p.tex_min_dy);
    }
    return p;
}

} // namespace oracle
