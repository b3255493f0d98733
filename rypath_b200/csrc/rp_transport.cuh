// Wavefront hero-wavelength path tracing: one event of shaders/packet_pt_event_body.inc split
// at its two traversal points.  The closest-hit query runs in its own kernel, the event body
// (emission MIS, light sample, BSDF continuation, roulette) in the shade kernel, and the
// light sample's visibility in the shadow kernel, with SoA path state in HBM in between.
#pragma once

#include "rp_scene.cuh"

namespace rp {

enum : u32 { kCamera = 0, kSurface = 1, kLight = 2, kEnvironment = 3 };

// Path flags word (ident.w)
enum : u32 {
    F_MASK = 0xfu,            // hero active wavelength mask
    F_ROULETTE = 1u << 4,     // roulette enabled
    F_COMPLETE = 1u << 5,
    F_STATUS_SHIFT = 6,       // 3 bits
    F_LTYPE_SHIFT = 9,        // latest vertex type, 2 bits
    F_PTYPE_SHIFT = 11,       // preceding vertex type, 2 bits
    F_LDELTA = 1u << 13,      // latest vertex sampled a Dirac lobe
    F_LKIND_SHIFT = 14,       // latest BSDF family, 2 bits
    F_LMASK_SHIFT = 16,       // latest BSDF active mask, 4 bits
    F_LSMOOTH = 1u << 20,     // latest BSDF roughness is smooth
};
RP_DEV u32 get_status(u32 f) { return (f >> F_STATUS_SHIFT) & 7u; }
RP_DEV u32 set_status(u32 f, u32 s) { return (f & ~(7u << F_STATUS_SHIFT)) | (s << F_STATUS_SHIFT); }

// Structure-of-arrays path pool: one slot per lane of the wave.
struct PathPool {
    uint4 *ident;      // pixel, sample_low, sample_high, flags
    uint4 *cursor;     // sobol index lo, hi, vertex count, lane
    float4 *lambda, *lambda_pdf, *beta, *radiance;
    float4 *dens_f, *prev_f; // hero density fractions (arrival / previous)
    int4 *dens_e, *prev_e;   // and exponents
    float4 *eta_scale;
    float4 *ray_o, *ray_d;
    float4 *latest_p;      // latest vertex position, alpha_x
    float4 *latest_n;      // latest shading normal, alpha_y
    float4 *latest_param;  // per-wavelength reflectance or eta
    float4 *latest_k;      // per-wavelength conductor k
    float4 *preceding;     // position of the vertex before latest
    float4 *hit;           // t, b1, b2, primitive bits
    // queues
    u32 *queue[2];
    u32 *counters; // [0] queue0, [1] queue1, [2] shadow, [3] failures, [4..7] family bins
    u32 *bins;     // 4 family bins of bin_capacity path ids each
    u32 bin_capacity;
    float4 *sh_o;  // shadow origin, tmax
    float4 *sh_d;  // shadow direction, path id bits
    float4 *sh_c;  // weighted contribution (NaN x: invalid if visible)
    float4 *sh_t;  // shadow target (pass-through walks restart toward it), or nullptr
    u32 *material; // material a mix-root hit resolved to (written by the closest-hit kernel)
    // statistics (optional)
    unsigned long long *stats; // closest [0] nodes, [1] triangles, [2] rays; shadow [3] rays, [4] nodes, [5] triangles
    // light-sample requests, one per path (written by the shade kernel, read by k_nee): the
    // vertex (position + vertex count, shading normal + BSDF bits, geometric normal + alpha_x,
    // error + alpha_y), the outgoing direction, the previous vertex, the throughput and hero
    // density before this event's continuation, and the BSDF's per-wavelength parameters
    float4 *nee_p, *nee_n, *nee_g, *nee_e, *nee_wo, *nee_prev, *nee_beta, *nee_df, *nee_param, *nee_k;
    int4 *nee_de;
    u32 *nee_queue; // three family queues of bin_capacity path ids; counts in counters[8..10]
    // per-lane walk counts of counting runs (pool slot = request lane), or nullptr: closest-hit
    // walks (written by the closest-hit kernel) and any-hit walks (by the shadow kernel, which
    // runs beside the next closest-hit walk, hence two arrays)
    u32 *lane_closest, *lane_shadow;
    // path-replay adjoint (hist == nullptr: off)
    uint4 *hist;            // parameter materials of the diffuse vertices so far, a byte each, 0xff = none
    float4 *adj_w;          // d loss / d radiance of each wavelength lane
    const u32 *adj_slot;    // per scene material: its first gradient entry, kNone if not a parameter
    float *adj_grad;        // gradient of the loss, one entry per parameter knot
    const double *adj_g;    // d loss / d film-mean XYZ, 3 per pixel
    const double *adj_cie;  // CIE 1931 table, 3 per nm from 360 nm
    double adj_inv_weight;  // 1 / film weight of a pixel (its sample count)
    u32 adj_params;         // gradient entries
};

// sampler: 0 independent, 1 Sobol, 2 Halton, 3 ZSobol (src/render_wire.h:41)
struct WaveParams {
    u32 width, height, pixel_begin, pixel_count, sample_low, sample_high;
    u32 seed_low, seed_high, sampler, randomization, m, emergency_limit;
    u32 lanes;
    u32 log_spp;        // ZSobol: log2 of the total sample budget
    u32 boundary_limit; // pass-through crossings allowed between two vertices
    // Sobol sampler with Owen randomisation: the first kOwenPrefixBits scrambling rounds of the
    // draw blocks [4, 4 + owen_blocks) and [133, 133 + owen_blocks), tabulated (null: none)
    const unsigned short *owen_prefix;
    u32 owen_blocks;
};
// Table of one draw block's four dimensions in the Owen prefix table (null if not tabulated).
RP_DEV const unsigned short *owen_prefix_table(const WaveParams &p, u32 block) {
    if (!p.owen_prefix || p.randomization != 3)
        return nullptr;
    if (block - 4u < p.owen_blocks)
        return p.owen_prefix + size_t(block - 4u) * 4 * kOwenPrefixEntries;
    if (block - 133u < p.owen_blocks)
        return p.owen_prefix + size_t(p.owen_blocks + block - 133u) * 4 * kOwenPrefixEntries;
    return nullptr;
}

// shaders/render.metal:113-122
RP_DEV float sample_uniform(const WaveParams &p, u32 w) {
    if (p.sampler == 2)
        return bits_float(w);
    return p.sampler == 0 ? u01(w) : sobol_uniform(w);
}
// Integer decisions quantise the Halton uniform, not its binary32 representation.
RP_DEV u32 decision_word(const WaveParams &p, u32 w) { return p.sampler == 2 ? u32(bits_float(w) * 0x1p32f) : w; }
// shaders/render.metal:123-127
RP_DEV u32 zdraw(const DeviceScene &s, const WaveParams &p, u64 index, u32 dimension, u32 axis = 0, bool pair = false) {
    return zsobol_word(s.sobol, index, dimension, axis, pair, p.m, p.log_spp, p.randomization, p.seed_low);
}

// shaders/render.metal:154-179 (independent and Sobol samplers); out of line, one copy per kernel
__device__ __noinline__ uint4 draw_words(const DeviceScene &s, const WaveParams &p, u32 pixel, u32 slo, u32 shi,
                                         u64 index, u32 block) {
    if (p.sampler == 0)
        return philox(make_uint4(pixel, slo, shi, block), p.seed_low, p.seed_high);
    const u32 d = 4 * block;
    if (p.sampler == 2)
        return make_uint4(float_bits(qmc_radical(s.primes, d, index, p.randomization, p.seed_low)),
                          float_bits(qmc_radical(s.primes, d + 1, index, p.randomization, p.seed_low)),
                          float_bits(qmc_radical(s.primes, d + 2, index, p.randomization, p.seed_low)),
                          float_bits(qmc_radical(s.primes, d + 3, index, p.randomization, p.seed_low)));
    if (p.sampler == 3) {
        const bool even = (block & 1) == 0;
        return make_uint4(zdraw(s, p, index, d, 0, true), zdraw(s, p, index, d, 1, true),
                          zdraw(s, p, index, d + 2, 0, even), zdraw(s, p, index, even ? d + 2 : d + 3, even ? 1 : 0, even));
    }
    return sobol_words4(s.sobol, index, 4 * block, p.randomization, p.seed_low, owen_prefix_table(p, block));
}

// The first word of draw_words (the block's first dimension) alone.
__device__ __noinline__ u32 draw_word0(const DeviceScene &s, const WaveParams &p, u32 pixel, u32 slo, u32 shi,
                                       u64 index, u32 block) {
    if (p.sampler == 1)
        return sobol_word_prefixed(s.sobol, index, 4 * block, p.randomization, p.seed_low, owen_prefix_table(p, block));
    return draw_words(s, p, pixel, slo, shi, index, block).x;
}

struct BeginSample {
    u32 pixel, sample_low, sample_high;
    u64 index;
    uint4 words;
    uint2 lens_words;
    float filter_x, filter_y; // Gaussian filter offsets
};
constexpr u32 kLensBlock = 0xc0000000u;   // src/sampling_contract.h:24
constexpr u32 kLensDimensionX = 1022u;
// shaders/render.metal:200-236 (gaussian_filter_offsets): inverse of the tabulated marginal,
// then of the selected row's conditional
RP_DEV void gaussian_filter_offsets(const DeviceScene &s, float ux, float uy, float &x, float &y) {
    const float *cdf = s.gauss_cdf;
    const float *marginal = cdf + size_t(s.gauss_h) * (s.gauss_w + 1);
    u32 low = 0, high = s.gauss_h;
    while (low + 1 < high) {
        const u32 mid = (low + high) / 2;
        if (__ldg(marginal + mid) <= uy)
            low = mid;
        else
            high = mid;
    }
    const u32 row = low;
    const float m0 = __ldg(marginal + row), m1 = __ldg(marginal + row + 1);
    const float ty = (float(row) + (uy - m0) / (m1 - m0)) / float(s.gauss_h);
    const float *conditional = cdf + size_t(row) * (s.gauss_w + 1);
    low = 0;
    high = s.gauss_w;
    while (low + 1 < high) {
        const u32 mid = (low + high) / 2;
        if (__ldg(conditional + mid) <= ux)
            low = mid;
        else
            high = mid;
    }
    const float c0 = __ldg(conditional + low), c1 = __ldg(conditional + low + 1);
    const float tx = (float(low) + (ux - c0) / (c1 - c0)) / float(s.gauss_w);
    x = (1 - tx) * (-s.filter_x) + tx * s.filter_x;
    y = (1 - ty) * (-s.filter_y) + ty * s.filter_y;
}
// shaders/render.metal:238-311 (begin_sample)
// The sample of (pixel, absolute sample index): its index, camera and lens words and filter
// offsets (the part of begin_sample that does not depend on the lane).
RP_DEV BeginSample begin_sample_at(const DeviceScene &s, const WaveParams &p, u32 pixel, u32 sample_low,
                                   u32 sample_high) {
    BeginSample r;
    r.pixel = pixel;
    r.sample_low = sample_low;
    r.sample_high = sample_high;
    if (p.sampler == 1) {
        const u64 sample = (u64(r.sample_high) << 32) | r.sample_low;
        r.index = sobol_index(s.sobol, p.m, r.pixel % p.width, r.pixel / p.width, sample);
        r.words = make_uint4(sobol_word(s.sobol, r.index, 0, 0, 0), sobol_word(s.sobol, r.index, 1, 0, 0),
                             sobol_word(s.sobol, r.index, 2, p.randomization, p.seed_low),
                             sobol_word(s.sobol, r.index, 3, p.randomization, p.seed_low));
    } else if (p.sampler == 2) {
        const u64 sample = (u64(r.sample_high) << 32) | r.sample_low;
        r.index = halton_index(p.width, p.height, r.pixel % p.width, r.pixel / p.width, sample);
        r.words = make_uint4(float_bits(halton_camera(s.primes, 0, p.width, r.index)),
                             float_bits(halton_camera(s.primes, 1, p.height, r.index)),
                             float_bits(qmc_radical(s.primes, 2, r.index, p.randomization, p.seed_low)),
                             float_bits(qmc_radical(s.primes, 3, r.index, p.randomization, p.seed_low)));
    } else if (p.sampler == 3) {
        const u64 sample = (u64(r.sample_high) << 32) | r.sample_low;
        r.index = zsobol_morton(r.pixel % p.width, r.pixel / p.width, p.log_spp, sample);
        r.words = make_uint4(zdraw(s, p, r.index, 1, 0, true), zdraw(s, p, r.index, 1, 1, true),
                             zdraw(s, p, r.index, 0), zdraw(s, p, r.index, 3));
    } else {
        r.index = 0;
        r.words = philox(make_uint4(r.pixel, r.sample_low, r.sample_high, 0), p.seed_low, p.seed_high);
    }
    r.lens_words = make_uint2(0, 0);
    if (s.lens_radius > 0) {
        if (p.sampler == 1) {
            r.lens_words = make_uint2(sobol_word(s.sobol, r.index, kLensDimensionX, p.randomization, p.seed_low),
                                      sobol_word(s.sobol, r.index, kLensDimensionX + 1, p.randomization, p.seed_low));
        } else if (p.sampler == 2) {
            r.lens_words = make_uint2(float_bits(qmc_radical(s.primes, 998, r.index, p.randomization, p.seed_low)),
                                      float_bits(qmc_radical(s.primes, 999, r.index, p.randomization, p.seed_low)));
        } else if (p.sampler == 3) {
            r.lens_words = make_uint2(zdraw(s, p, r.index, kLensDimensionX, 0, true),
                                      zdraw(s, p, r.index, kLensDimensionX, 1, true));
        } else {
            const uint4 w = philox(make_uint4(r.pixel, r.sample_low, r.sample_high, kLensBlock), p.seed_low, p.seed_high);
            r.lens_words = make_uint2(w.x, w.y);
        }
    }
    r.filter_x = r.filter_y = 0;
    if (s.filter_kind == 2) {
        const float ux =
            p.sampler == 1 ? sobol_camera_uniform(r.words.x, p.m, r.pixel % p.width) : sample_uniform(p, r.words.x);
        const float uy =
            p.sampler == 1 ? sobol_camera_uniform(r.words.y, p.m, r.pixel / p.width) : sample_uniform(p, r.words.y);
        gaussian_filter_offsets(s, ux, uy, r.filter_x, r.filter_y);
    }
    return r;
}
RP_DEV BeginSample begin_sample(const DeviceScene &s, const WaveParams &p, u32 lane) {
    const u32 sample_low = p.sample_low + lane / p.pixel_count;
    return begin_sample_at(s, p, p.pixel_begin + lane % p.pixel_count, sample_low,
                           p.sample_high + u32(sample_low < p.sample_low));
}
// shaders/render.metal:352-357
RP_DEV float triangle_offset(float u, float radius) {
    const float sv = 2.0f * u - 1.0f;
    return radius * (sv / (1.0f + sqrtf(1.0f - fabsf(sv))));
}
// A PBRT raster camera (RasterCamera, src/render.hpp:152-157)
struct RasterCam {
    V3 origin, forward, right, up;
};
// shaders/render.metal:341-476 (primary_ray: pinhole, box / triangle filter) for camera `cam`
RP_DEV void primary_ray_from(const DeviceScene &s, const RasterCam &cam, const WaveParams &p, const BeginSample &b,
                             V3 &o, V3 &d) {
    float ux, uy;
    // camera_uniforms (shaders/render.metal:341-350)
    if (p.sampler == 1) {
        ux = sobol_camera_uniform(b.words.x, p.m, b.pixel % p.width);
        uy = sobol_camera_uniform(b.words.y, p.m, b.pixel / p.width);
    } else {
        ux = sample_uniform(p, b.words.x);
        uy = sample_uniform(p, b.words.y);
    }
    o = cam.origin;
    const float nan = __int_as_float(0x7fffffff);
    // centered_filter / filter_offset (shaders/render.metal:395-411)
    const bool centered = s.filter_kind != 0 || s.filter_x != 0.5f || s.filter_y != 0.5f;
    V3 dd;
    if (centered) {
        const float ox = s.filter_kind == 2   ? b.filter_x
                         : s.filter_kind == 1 ? triangle_offset(ux, s.filter_x)
                                              : (2.0f * ux - 1.0f) * s.filter_x;
        const float oy = s.filter_kind == 2   ? b.filter_y
                         : s.filter_kind == 1 ? triangle_offset(uy, s.filter_y)
                                              : (2.0f * uy - 1.0f) * s.filter_y;
        const float x = ((float(b.pixel % p.width) + 0.5f) + ox) / float(p.width);
        const float y = ((float(b.pixel / p.width) + 0.5f) + oy) / float(p.height);
        dd = fma3(v3(y, y, y), cam.up, fma3(v3(x, x, x), cam.right, cam.forward));
    } else {
        const float x = (float(b.pixel % p.width) + ux) / float(p.width);
        const float y = (float(b.pixel / p.width) + uy) / float(p.height);
        dd = cam.forward + x * cam.right + y * cam.up;
    }
    if (s.lens_radius > 0) {
        // lens_primary_ray / lens_point (shaders/render.metal:366-432): concentric disk sample
        // on the aperture, direction through the focus plane
        const float lx = 2.0f * sample_uniform(p, b.lens_words.x) - 1.0f;
        const float ly = 2.0f * sample_uniform(p, b.lens_words.y) - 1.0f;
        V3 offset = v3(0, 0, 0);
        if (!(lx == 0 && ly == 0)) {
            float radius, theta;
            if (fabsf(lx) > fabsf(ly)) {
                radius = lx;
                theta = (kPi / 4.0f) * (ly / lx);
            } else {
                radius = ly;
                theta = kPi / 2.0f - (kPi / 4.0f) * (lx / ly);
            }
            const float r = s.lens_radius * radius;
            const float disk_x = r * cosf(theta), disk_y = r * sinf(theta);
            const V3 ideal = disk_x * s.lens_x + disk_y * s.lens_y;
            o = cam.origin + ideal;
            offset = o - cam.origin;
        }
        dd = dd - offset / s.focal_distance;
        // rypath_texture_direction (shaders/texture_footprint.h:14-20)
        const float scale = fmaxf(fabsf(dd.x), fmaxf(fabsf(dd.y), fabsf(dd.z)));
        d = (!(scale > 0.0f) || !finite3(dd)) ? v3(nan, nan, nan) : normalize3(dd / scale);
        return;
    }
    if (centered) {
        const float scale = fmaxf(fabsf(dd.x), fmaxf(fabsf(dd.y), fabsf(dd.z)));
        if (!finite3(dd) || !(scale > 0.0f)) {
            d = v3(nan, nan, nan);
            return;
        }
        const V3 scaled = dd / scale;
        if (!finite3(scaled) || zero3(scaled)) {
            d = v3(nan, nan, nan);
            return;
        }
        d = normalize3(scaled);
        return;
    }
    if (s.model == kModelDemo) {
        // the demo camera (shaders/render.metal:470-475): forward, right and up are the look-at
        // basis and film_scale = tan(fov / 2)
        const float x = (float(b.pixel % p.width) + ux) / float(p.width);
        const float y = (float(b.pixel / p.width) + uy) / float(p.height);
        const float aspect = float(p.width) / float(p.height);
        d = normalize3((cam.forward + (((2.0f * x - 1.0f) * aspect) * s.film_scale) * cam.right) +
                       ((1.0f - 2.0f * y) * s.film_scale) * cam.up);
        return;
    }
    const float scale = fmaxf(fabsf(dd.x), fmaxf(fabsf(dd.y), fabsf(dd.z)));
    d = normalize3(dd / scale);
}
RP_DEV void primary_ray(const DeviceScene &s, const WaveParams &p, const BeginSample &b, V3 &o, V3 &d) {
    primary_ray_from(s, RasterCam{s.origin, s.forward, s.right, s.up}, p, b, o, d);
}

// shaders/render.metal:479-501 (texture_camera_rays): the camera directions one pixel right and
// one pixel down of the sample's film position, shifted by the lens sample; and the lens
// sample's aperture offset (lens_offset, :390-392)
RP_DEV void texture_camera_rays(const DeviceScene &s, const WaveParams &p, const BeginSample &b, V3 &rx, V3 &ry,
                                V3 &lens) {
    float ux, uy;
    if (p.sampler == 1) {
        ux = sobol_camera_uniform(b.words.x, p.m, b.pixel % p.width);
        uy = sobol_camera_uniform(b.words.y, p.m, b.pixel / p.width);
    } else {
        ux = sample_uniform(p, b.words.x);
        uy = sample_uniform(p, b.words.y);
    }
    const bool centered = s.filter_kind != 0 || s.filter_x != 0.5f || s.filter_y != 0.5f;
    V3 dd;
    if (centered) {
        const float ox = s.filter_kind == 2   ? b.filter_x
                         : s.filter_kind == 1 ? triangle_offset(ux, s.filter_x)
                                              : (2.0f * ux - 1.0f) * s.filter_x;
        const float oy = s.filter_kind == 2   ? b.filter_y
                         : s.filter_kind == 1 ? triangle_offset(uy, s.filter_y)
                                              : (2.0f * uy - 1.0f) * s.filter_y;
        const float x = ((float(b.pixel % p.width) + 0.5f) + ox) / float(p.width);
        const float y = ((float(b.pixel / p.width) + 0.5f) + oy) / float(p.height);
        dd = fma3(v3(y, y, y), s.up, fma3(v3(x, x, x), s.right, s.forward));
    } else {
        const float x = (float(b.pixel % p.width) + ux) / float(p.width);
        const float y = (float(b.pixel / p.width) + uy) / float(p.height);
        dd = s.forward + x * s.right + y * s.up;
    }
    rx = dd + s.right / float(p.width);
    ry = dd + s.up / float(p.height);
    lens = v3(0, 0, 0);
    if (s.lens_radius > 0) {
        const float lx = 2.0f * sample_uniform(p, b.lens_words.x) - 1.0f;
        const float ly = 2.0f * sample_uniform(p, b.lens_words.y) - 1.0f;
        if (!(lx == 0 && ly == 0)) {
            float radius, theta;
            if (fabsf(lx) > fabsf(ly)) {
                radius = lx;
                theta = (kPi / 4.0f) * (ly / lx);
            } else {
                radius = ly;
                theta = kPi / 2.0f - (kPi / 4.0f) * (lx / ly);
            }
            const float r = s.lens_radius * radius;
            const V3 ideal = (r * cosf(theta)) * s.lens_x + (r * sinf(theta)) * s.lens_y;
            lens = (s.origin + ideal) - s.origin;
        }
        const V3 shift = v3(lens.x / s.focal_distance, lens.y / s.focal_distance, lens.z / s.focal_distance);
        rx = rx - shift;
        ry = ry - shift;
    }
}

// shaders/render.metal:1312-1408 (surface_texture_context) at a triangle hit (b1, b2) of
// instance `instance`, local triangle `local`: the texture coordinates and their screen-space
// derivatives.  scatterings: the path's scattering events so far (0 at the primary hit, whose
// footprint comes from the camera rays of the sample (pixel, sample_low, sample_high)).
RP_DEV bool texture_context(const DeviceScene &s, const WaveParams &p, u32 pixel, u32 sample_low, u32 sample_high,
                            u32 instance, u32 local, float b1, float b2, V3 geometric_normal, V3 primary_direction,
                            u32 scatterings, F2 &st, F2 &dstdx, F2 &dstdy) {
    const DInstance &in = s.instances[instance];
    const DImages &im = s.img;
    const u32 *tri = s.triangles + 3 * (in.triangle_begin + local);
    const u32 i0 = __ldg(tri), i1 = __ldg(tri + 1), i2 = __ldg(tri + 2);
    const V3 p0 = load3(s.positions + 3 * (in.vertex_begin + i0));
    const V3 p1 = load3(s.positions + 3 * (in.vertex_begin + i1));
    const V3 p2 = load3(s.positions + 3 * (in.vertex_begin + i2));
    const V3 local_p = fma3(v3(b2, b2, b2), p2 - p0, fma3(v3(b1, b1, b1), p1 - p0, p0));
    F2 uv0 = f2(0, 0), uv1 = f2(1, 0), uv2 = f2(1, 1);
    const u32 uv_begin = im.inst_uv_begin ? __ldg(im.inst_uv_begin + instance) : kNone;
    if (uv_begin != kNone) {
        if (uv_begin >= im.uv_count || i0 >= im.uv_count - uv_begin || i1 >= im.uv_count - uv_begin ||
            i2 >= im.uv_count - uv_begin)
            return false;
        const float2 a = im.uvs[uv_begin + i0], b = im.uvs[uv_begin + i1], c = im.uvs[uv_begin + i2];
        uv0 = f2(a.x, a.y);
        uv1 = f2(b.x, b.y);
        uv2 = f2(c.x, c.y);
        if (!isfinite(uv0.x) || !isfinite(uv0.y) || !isfinite(uv1.x) || !isfinite(uv1.y) || !isfinite(uv2.x) ||
            !isfinite(uv2.y))
            return false;
    }
    const float w0 = 1.0f - (b1 + b2);
    st = f2((w0 * uv0.x + b1 * uv1.x) + b2 * uv2.x, (w0 * uv0.y + b1 * uv1.y) + b2 * uv2.y);
    const u32 frame_begin = im.inst_frame_begin ? __ldg(im.inst_frame_begin + instance) : kNone;
    if (!isfinite(st.x) || !isfinite(st.y) || frame_begin >= im.frame_count || local >= im.frame_count - frame_begin)
        return false;
    const float *fr = im.frames + 6 * size_t(frame_begin + local);
    const V3 dpdu = load3(fr), dpdv = load3(fr + 3);
    const V3 world = v3(dot(v3(in.m[0], in.m[1], in.m[2]), local_p), dot(v3(in.m[4], in.m[5], in.m[6]), local_p),
                        dot(v3(in.m[8], in.m[9], in.m[10]), local_p));
    const V3 rel = world + (v3(in.m[3], in.m[7], in.m[11]) - s.origin);
    if (!finite3(rel))
        return false;
    V3 dpdx = v3(0, 0, 0), dpdy = v3(0, 0, 0);
    bool primary = false;
    if (scatterings == 0) {
        V3 rx, ry, lens;
        texture_camera_rays(s, p, begin_sample_at(s, p, pixel, sample_low, sample_high), rx, ry, lens);
        if (!finite3(rx) || !finite3(ry))
            return false;
        primary = texture_primary_dp(s.lens_radius > 0 ? rel - lens : rel, geometric_normal, primary_direction, rx,
                                     ry, im.tex_spp_scale, dpdx, dpdy);
    }
    if (!primary)
        texture_approximate_dp(im, rel, geometric_normal, dpdx, dpdy);
    return texture_uv_derivatives(dpdu, dpdv, dpdx, dpdy, dstdx, dstdy);
}
// The filtered, scaled (and inverted) linear RGB of an image reflectance at a footprint
// (shaders/packet_walk.h:39-49)
RP_DEV RGB image_reflectance_rgb(const DImages &im, u32 texture, F2 st, F2 dstdx, F2 dstdy) {
    const DImageTexture t = im.textures[texture];
    RGB c = lookup_filtered(im, t, st, dstdx, dstdy, false, false);
    c = rgb3(c.r * t.scale, c.g * t.scale, c.b * t.scale);
    if (t.invert)
        c = rgb3(1 - c.r, 1 - c.g, 1 - c.b);
    return c;
}

// PBRT's RGBAlbedoSpectrum of a material's sigmoid coefficients (shaders/render.metal:576-588)
RP_DEV float sigmoid_reflectance(const float *c, float w) {
    const float p = fmaf(fmaf(c[0], w, c[1]), w, c[2]);
    if (!isfinite(p))
        return image_nan();
    if (fabsf(p) <= 1.0f)
        return 0.5f + 0.5f * (p / sqrtf(1.0f + p * p));
    const float inverse = 1.0f / p;
    return 0.5f + 0.5f * copysignf(1.0f / sqrtf(1.0f + inverse * inverse), p);
}
// shaders/packet_walk.h:22-57 (sampled / constant / blackbody / RGB / image reflectance; image:
// the reconstruction of the hit's filtered RGB)
RP_DEV bool material_reflectance(const DeviceScene &s, const DMaterial &m, float w, const RgbPolynomial *image,
                                 float &rho) {
    if (m.scattering != 0) {
        rho = 1;
    } else if (m.kind == 3 && image && m.image_texture < s.img.texture_count) {
        rho = rgb_polynomial_at(*image, w);
    } else if (m.kind == 0 && m.knot_count >= 2 && m.knot_begin <= s.knot_count &&
               m.knot_count <= s.knot_count - m.knot_begin) {
        rho = pbrt_reflectance(s.knots + m.knot_begin, m.knot_count, w);
    } else if (m.kind == 1) {
        rho = m.scalar_value;
    } else if (m.kind == 4) {
        rho = blackbody_reflectance(m.scalar_value, w);
    } else if (m.kind == 2) {
        rho = sigmoid_reflectance(m.coefficients, w);
    } else
        return false;
    return isfinite(rho) && rho >= 0 && rho <= 1;
}
// shaders/hero_current_bsdf.h:72-101 with prepare_scattering (shaders/render.metal:2079-2160)
template <int K>
RP_DEV bool prepare_bsdf(const DeviceScene &s, const DMaterial &m, V4 lambda, u32 mask, HeroBsdf &out,
                         const RgbPolynomial *image = nullptr) {
    if (m.scattering != u32(K))
        return false;
    out.kind = m.scattering;
    out.active_mask = mask;
    out.g = {0, 0, true};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        out.param[k] = 0;
        out.k[k] = 0;
    }
    if (m.scattering > 2)
        return false;
    if (m.scattering != 0) {
        const float u = m.u_roughness, v = m.v_roughness;
        if (!isfinite(u) || !isfinite(v) || u < 0 || v < 0)
            return false;
        prepare_roughness(u, v, m.remap != 0, false, out.g);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!(mask & (1u << k)))
            continue;
        float rho;
        if (!material_reflectance(s, m, lambda.v[k], image, rho))
            return false;
        if constexpr (K == 0) {
            out.param[k] = rho;
            continue;
        }
        const float eta = optical_value(s.knots, m.eta_begin, m.eta_count, s.knot_count, (m.optical_extensions & 1u) != 0,
                                        lambda.v[k]);
        const float kk = optical_value(s.knots, m.k_begin, m.k_count, s.knot_count, (m.optical_extensions & 2u) != 0,
                                       lambda.v[k]);
        if constexpr (K == 1) {
            // shaders/conductor.h:22-25
            if (!isfinite(eta) || !isfinite(kk) || eta < 0 || kk < 0 || (eta == 0 && kk == 0))
                return false;
            out.param[k] = eta;
            out.k[k] = kk;
        } else {
            // shaders/dielectric.h:15-18
            if (!isfinite(eta) || eta < 0)
                return false;
            out.param[k] = eta == 0 ? 1 : eta;
        }
    }
    return true;
}

// Compact record of the latest vertex for emission MIS (HeroPrevious, shaders/hero_pt_state.h:6-15).
struct Latest {
    u32 type, kind, mask;
    bool delta, smooth;
    V3 position, shading_normal;
    float alpha_x, alpha_y;
    V4 param, k;
};
RP_DEV HeroBsdf latest_bsdf(const Latest &l) {
    HeroBsdf b;
    b.kind = l.kind;
    b.active_mask = l.mask;
    b.g = {l.alpha_x, l.alpha_y, l.smooth};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        b.param[k] = l.param.v[k];
        b.k[k] = l.k.v[k];
    }
    return b;
}
// shaders/hero_pt_helpers.h:122-132 (hero_represented_pdf) for a surface vertex v with
// finite neighbours (the neighbour after v may be at infinity: pass its direction).
// K selects the BSDF family at compile time; -1 dispatches on the stored family.
template <int K>
RP_DEV V4 represented_pdf(const HeroBsdf &b, V3 shading_normal, V3 position, V3 before, bool after_infinite,
                          V3 after_point, bool &ok) {
    ok = true;
    const V3 wb = before - position;
    const V3 wa = after_infinite ? after_point : after_point - position;
    if (zero3(wb) || zero3(wa))
        return v4(0);
    Frame f;
    if (!shading_frame(shading_normal, f)) {
        ok = false;
        return v4(0);
    }
    HeroEval e;
    if constexpr (K < 0)
        e = hero_evaluate(b, to_local(f, normalize3(wb)), to_local(f, normalize3(wa)));
    else
        e = hero_evaluate_k<K>(b, to_local(f, normalize3(wb)), to_local(f, normalize3(wa)));
    if (!e.valid) {
        ok = false;
        return v4(0);
    }
    return e.pdf;
}
// shaders/hero_pt_helpers.h:133-148 (hero_weight); returns false for invalid arithmetic
RP_DEV bool hero_weight(const Density &prefix, V4 value, V4 sampled, V4 other, V4 &out) {
    if (!finite_nonnegative4(value) || !finite_nonnegative4(sampled) || !finite_nonnegative4(other)) {
        out = v4(0);
        return false;
    }
    if (mixture(prefix, other).fraction == 0) {
        out = value;
        return true;
    }
    const Contribution r = balance_contribution(prefix, value, sampled, other);
    out = r.value;
    return r.valid;
}

RP_DEV Density load_density(float4 f, int4 e) {
    Density d;
    d.lane[0] = {f.x, e.x};
    d.lane[1] = {f.y, e.y};
    d.lane[2] = {f.z, e.z};
    d.lane[3] = {f.w, e.w};
    return d;
}
RP_DEV void store_density(const Density &d, float4 &f, int4 &e) {
    f = make_float4(d.lane[0].fraction, d.lane[1].fraction, d.lane[2].fraction, d.lane[3].fraction);
    e = make_int4(d.lane[0].exponent, d.lane[1].exponent, d.lane[2].exponent, d.lane[3].exponent);
}

// The light-sample request of a path's event (PathPool::nee_*).
RP_DEV void write_nee_request(const PathPool &pool, u32 path, u32 cnt, const SurfacePoint &cp, const HeroBsdf &b,
                              V3 wo, V3 previous, V4 beta, const Density &density) {
    const u32 bits = (b.kind & 3u) | ((b.active_mask & 15u) << 2) | (b.g.smooth ? 64u : 0u);
    pool.nee_p[path] = make_float4(cp.position.x, cp.position.y, cp.position.z, __uint_as_float(cnt));
    pool.nee_n[path] = make_float4(cp.shading_normal.x, cp.shading_normal.y, cp.shading_normal.z, __uint_as_float(bits));
    pool.nee_g[path] = make_float4(cp.geometric_normal.x, cp.geometric_normal.y, cp.geometric_normal.z, b.g.alpha_x);
    pool.nee_e[path] = make_float4(cp.error.x, cp.error.y, cp.error.z, b.g.alpha_y);
    pool.nee_wo[path] = make_float4(wo.x, wo.y, wo.z, 0);
    pool.nee_prev[path] = make_float4(previous.x, previous.y, previous.z, 0);
    pool.nee_beta[path] = to_float4(beta);
    float4 f;
    int4 e;
    store_density(density, f, e);
    pool.nee_df[path] = f;
    pool.nee_de[path] = e;
    pool.nee_param[path] = make_float4(b.param[0], b.param[1], b.param[2], b.param[3]);
    pool.nee_k[path] = make_float4(b.k[0], b.k[1], b.k[2], b.k[3]);
}
RP_DEV void read_nee_request(const PathPool &pool, u32 path, u32 &cnt, SurfacePoint &cp, HeroBsdf &b, V3 &wo,
                             V3 &previous, V4 &beta, Density &density) {
    const float4 pp = pool.nee_p[path], n = pool.nee_n[path], g = pool.nee_g[path], e = pool.nee_e[path];
    const float4 w = pool.nee_wo[path], v = pool.nee_prev[path], pa = pool.nee_param[path], k = pool.nee_k[path];
    cnt = __float_as_uint(pp.w);
    const u32 bits = __float_as_uint(n.w);
    cp.position = v3(pp.x, pp.y, pp.z);
    cp.shading_normal = v3(n.x, n.y, n.z);
    cp.geometric_normal = v3(g.x, g.y, g.z);
    cp.error = v3(e.x, e.y, e.z);
    cp.inverse_area_pdf = 0;
    cp.world_extent = 0;
    b.kind = bits & 3u;
    b.active_mask = (bits >> 2) & 15u;
    b.g = {g.w, e.w, (bits & 64u) != 0};
    b.param[0] = pa.x;
    b.param[1] = pa.y;
    b.param[2] = pa.z;
    b.param[3] = pa.w;
    b.k[0] = k.x;
    b.k[1] = k.y;
    b.k[2] = k.z;
    b.k[3] = k.w;
    wo = v3(w.x, w.y, w.z);
    previous = v3(v.x, v.y, v.z);
    beta = from_float4(pool.nee_beta[path]);
    density = load_density(pool.nee_df[path], pool.nee_de[path]);
}

// shaders/packet_transport.h:77-83
RP_DEV V3 offset_point(V3 position, V3 error, V3 ng, V3 direction) {
    if (!nonzero3(ng))
        return position;
    const V3 n = dot(direction, ng) < 0 ? -ng : ng;
    return round_out(position + dot(vabs(n), error) * n, n);
}
// shaders/render.metal:1939-1977: null-interface crossing anchored at the ray hit, with
// certified separation
RP_DEV bool spawn_boundary(V3 o, V3 d, float t, const SurfacePoint &pt, V3 direction, V3 &origin) {
    if (!(t >= 0) || !isfinite(t))
        return false;
    const V3 ng = pt.geometric_normal;
    const V3 n = dot(ng, direction) < 0 ? -ng : ng;
    const float facing = dot(n, direction);
    if (!(facing > gamma_bound(5) * dot(vabs(n), vabs(direction))))
        return false;
    V3 position, ray_error;
    ray_point(o, d, t, pt.curved, position, ray_error);
    const V3 error = (pt.error + vabs(pt.position - position)) + ray_error;
    const float norm_lower = dot(n, n) * (1 - gamma_bound(4));
    const float height = dot(vabs(n), error) * (1 + gamma_bound(8)) / norm_lower;
    origin = round_out(fma3(v3(height, height, height), n, position), n);
    if (!(norm_lower > 0) || !isfinite(height) || !finite3(origin) || eq3(origin, o))
        return false;
    const V3 departure = origin - pt.position;
    const float separation = dot(n, departure);
    const float rounding = gamma_bound(5) * dot(vabs(n), vabs(departure));
    const float uncertainty = dot(vabs(n), pt.error) * (1 + gamma_bound(4));
    return isfinite(separation) && isfinite(rounding) && isfinite(uncertainty) && separation - rounding > uncertainty;
}

// ------------------------------------------------------------------ path-replay adjoint
// A lane's radiance is a sum of contributions, each a product in which every diffuse vertex
// before it (and, for a light sample, the vertex it leaves from) enters once through its
// reflectance rho(lambda); the selection probabilities, wavelength and light MIS weights
// depend on densities only.  So d contribution / d rho_m(lambda) = contribution * n_m / rho_m,
// and rho is piecewise linear in the knot values (pbrt_reflectance).  Russian roulette is held
// fixed (its survival test only picks which paths are traced).

// d loss / d radiance of each lane: the packet film weight (packet_sensor_xyz,
// src/packet_film.cpp:102-114) against d loss / d XYZ of the lane's pixel.
RP_DEV float4 adjoint_lane_weight(const PathPool &pool, u32 pixel, V4 lambda, V4 pdf) {
    float w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        w[k] = 0;
        if (pdf.v[k] == 0 || !(lambda.v[k] >= 360 && lambda.v[k] <= 830))
            continue;
        const u32 row = u32(round(double(lambda.v[k])) - 360.0);
        const double scale = pool.adj_inv_weight / (double(pdf.v[k]) * 4.0);
        double g = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            g += pool.adj_g[3 * size_t(pixel) + c] * pool.adj_cie[3 * row + c];
        w[k] = float(g * scale);
    }
    return make_float4(w[0], w[1], w[2], w[3]);
}
RP_DEV uint4 empty_history() { return make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu); }
RP_DEV u32 history_byte(uint4 h, u32 j) {
    const u32 word = j < 4 ? h.x : j < 8 ? h.y : j < 12 ? h.z : h.w;
    return (word >> (8 * (j & 3))) & 0xffu;
}
// appends material m; a full history (16 vertices) is refused by the adjoint's depth limit
RP_DEV uint4 history_push(uint4 h, u32 m) {
    for (u32 j = 0; j < 16; ++j)
        if (history_byte(h, j) == 0xffu) {
            const u32 shift = 8 * (j & 3), mask = ~(0xffu << shift), v = (m & 0xffu) << shift;
            if (j < 4)
                h.x = (h.x & mask) | v;
            else if (j < 8)
                h.y = (h.y & mask) | v;
            else if (j < 12)
                h.z = (h.z & mask) | v;
            else
                h.w = (h.w & mask) | v;
            break;
        }
    return h;
}
// d loss / d knots of one contribution, accumulated into the block's shared gradient
__device__ __noinline__ void adjoint_accumulate(const DeviceScene &s, const PathPool &pool, float *sgrad, uint4 hist,
                                                V4 lambda, V4 contribution, float4 w4) {
    const float w[4] = {w4.x, w4.y, w4.z, w4.w};
    for (u32 j = 0; j < 16; ++j) {
        const u32 m = history_byte(hist, j);
        if (m == 0xffu)
            break;
        const u32 slot = __ldg(pool.adj_slot + m);
        const DMaterial M = s.materials[m];
        const float2 *kn = s.knots + M.knot_begin;
        for (int k = 0; k < 4; ++k) {
            const float g0 = w[k] * contribution.v[k];
            const float x = lambda.v[k];
            if (g0 == 0 || !(x >= kn[0].x && x <= kn[M.knot_count - 1].x))
                continue;
            u32 lo = 0, hi = M.knot_count - 1;
            while (hi - lo > 1) {
                const u32 mid = lo + (hi - lo) / 2;
                if (x < kn[mid].x)
                    hi = mid;
                else
                    lo = mid;
            }
            const float t = lo == hi ? 0.0f : (x - kn[lo].x) / (kn[hi].x - kn[lo].x);
            const float rho = kn[lo].y + (kn[hi].y - kn[lo].y) * t;
            if (!(rho > 0))
                continue;
            const float g = g0 / rho;
            atomicAdd(sgrad + slot + lo, g * (1.0f - t));
            if (hi != lo)
                atomicAdd(sgrad + slot + hi, g * t);
        }
    }
}
RP_DEV void adjoint_begin(const PathPool &pool, float *sgrad) {
    if (!pool.hist)
        return;
    for (u32 i = threadIdx.x; i < pool.adj_params; i += blockDim.x)
        sgrad[i] = 0;
    __syncthreads();
}
RP_DEV void adjoint_end(const PathPool &pool, const float *sgrad) {
    if (!pool.hist)
        return;
    __syncthreads();
    for (u32 i = threadIdx.x; i < pool.adj_params; i += blockDim.x)
        if (sgrad[i] != 0)
            atomicAdd(pool.adj_grad + i, sgrad[i]);
}

} // namespace rp
