// Scalar (one-wavelength) path tracing with homogeneous media: the estimator of
// rypath_render_paths (shaders/render.metal:2299-2371), which runs scalar_init / scalar_trace /
// scalar_shade (shaders/scalar_transport.h) until each lane finishes.  The reference renders
// participating media with this transport only (hero transport requires vacuum,
// src/render.cpp:1579-1580).
//
// B200 form: a wavefront over 262,144 resident path slots.  A trip of every slot is one
// closest-hit query (k_scalar_walk: the path's ray or the current leg of its light
// connection, at the walk's own occupancy) and the medium / surface event or connection step
// that consumes it (k_scalar_step); a slot whose path finished takes the next lane from a
// global counter (one atomic per warp), so the slots stay full until the wave's lanes run
// out.  Results leave as one 16-byte record per lane; the film reduction reads them in
// canonical order.
//
// Surfaces: diffuse reflectance and null interfaces (material scattering 10).  Lights: area
// triangles, point and spot lights, constant environment.  Media: homogeneous, 471-bin
// sigma_a / sigma_s / emission with a Henyey-Greenstein phase function.
#pragma once

#include "rp_kernels.cuh"

namespace rp {

constexpr u32 kMediumStride = 1416; // sigma_a[471], sigma_s[471], emission[471], g, 2 pad
constexpr u32 kMediumBlockLimit = 0x20000000u;   // src/sampling_contract.h:45
constexpr u32 kMediumStream = 0x6d656431u;       // medium_stream_v1
enum : u32 {
    S_SUCCESS = 0,
    S_EMERGENCY = 1,
    S_ARITHMETIC = 2,
    S_HIT = 3,
    S_BOUNDARY = 4,
};

RP_DEV float fnan() { return __int_as_float(0x7fffffff); }
RP_DEV float finf() { return __int_as_float(0x7f800000); }
RP_DEV V3 nan3() { return v3(fnan(), fnan(), fnan()); }

// ------------------------------------------------------------------ shaders/medium.h
// :11-17 three positive factors over a fourth without an intermediate range loss
RP_DEV float product_ratio(float a, float b, float c, float d) {
    if (a == 0 || b == 0 || c == 0)
        return 0;
    int ea, eb, ec, ed;
    const float ma = frexpf(a, &ea), mb = frexpf(b, &eb), mc = frexpf(c, &ec), md = frexpf(d, &ed);
    return ldexpf(((ma * mb) * mc) / md, ea + eb + ec - ed);
}
// :19-31 (1 - exp(-x)) / x, series near zero
RP_DEV float attenuation_integral_ratio(float x) {
    if (x <= 0.125f) {
        float v = 1.0f / 40320.0f;
        v = fmaf(v, -x, 1.0f / 5040.0f);
        v = fmaf(v, -x, 1.0f / 720.0f);
        v = fmaf(v, -x, 1.0f / 120.0f);
        v = fmaf(v, -x, 1.0f / 24.0f);
        v = fmaf(v, -x, 1.0f / 6.0f);
        v = fmaf(v, -x, 0.5f);
        return fmaf(v, -x, 1.0f);
    }
    return (1.0f - expf(-x)) / x;
}
struct Segment {
    float transmission, emission;
    bool valid;
};
// :32-57 Beer transmission and the absorbed-emission integral of one segment
RP_DEV Segment medium_segment(float sa, float ss, float le, float distance) {
    if (!isfinite(sa) || !isfinite(ss) || !isfinite(le) || sa < 0 || ss < 0 || le < 0 || isnan(distance) ||
        distance < 0)
        return {0, 0, false};
    const float st = sa + ss;
    if (!isfinite(st))
        return {0, 0, false};
    if (distance == 0 || st == 0)
        return {1, 0, true};
    const float depth = st * distance;
    const float transmission = expf(-depth);
    float emission = 0;
    if (le > 0 && sa > 0) {
        if (depth <= 0.125f) {
            emission = product_ratio(le, sa, distance, 1.0f / attenuation_integral_ratio(depth));
        } else {
            const float loss = isinf(depth) ? 1.0f : 1.0f - transmission;
            emission = product_ratio(le, sa, loss, st);
        }
    }
    return {transmission, emission, isfinite(emission) && emission >= 0};
}
// :58-76 free-flight distance for extinction sigma_t
RP_DEV float medium_flight(float st, float u) {
    if (!isfinite(st) || st < 0 || !isfinite(u) || u < 0 || u > 1)
        return fnan();
    if (st == 0 || u == 1)
        return finf();
    if (u == 0)
        return 0;
    float depth;
    if (u <= 0.125f) {
        float v = 1.0f / 10.0f;
#pragma unroll
        for (int n = 9; n >= 2; --n)
            v = fmaf(v, u, 1.0f / float(n));
        depth = u * fmaf(v, u, 1.0f);
    } else {
        depth = -logf(1.0f - u);
    }
    return depth / st;
}
// :77-87 Henyey-Greenstein, both directions pointing away from the scattering point
RP_DEV float hg_phase(V3 wo, V3 wi, float g) {
    if (!finite3(wo) || !finite3(wi) || !isfinite(g) || fabsf(dot(wo, wo) - 1.0f) > 2e-5f ||
        fabsf(dot(wi, wi) - 1.0f) > 2e-5f)
        return fnan();
    g = fminf(fmaxf(g, -0.99f), 0.99f);
    const float cosine = fminf(fmaxf(dot(wo, wi), -1.0f), 1.0f);
    const float base = 1.0f - fabsf(g);
    const float denominator = fmaf(2.0f * fabsf(g), 1.0f + (g >= 0 ? cosine : -cosine), base * base);
    return (1.0f / (4.0f * kPi)) * ((1.0f - g) * (1.0f + g)) / (denominator * sqrtf(denominator));
}
// :88-112 exact inverse CDF of HG about wo
RP_DEV V3 hg_sample(V3 wo, float g, float ux, float uy) {
    if (!finite3(wo) || !isfinite(g) || !isfinite(ux) || !isfinite(uy) || ux < 0 || uy < 0 || ux > 1 || uy > 1 ||
        fabsf(dot(wo, wo) - 1.0f) > 2e-5f)
        return nan3();
    g = fminf(fmaxf(g, -0.99f), 0.99f);
    const float h = fabsf(g), v = g < 0 ? 1.0f - ux : ux;
    const float d = fmaf(h, 1.0f - 2.0f * v, 1.0f);
    const float ratio = (1.0f - h) / d;
    const float c = fminf(fmaxf(fmaf(2.0f * v * ratio * ratio, fmaf(h, 1.0f - v, 1.0f), -1.0f), -1.0f), 1.0f);
    const float cosine = g < 0 ? -c : c;
    const float sine = sqrtf(fmaxf(0.0f, (1.0f - cosine) * (1.0f + cosine)));
    V3 x;
    if (!unit(cross(fabsf(wo.z) < 0.9f ? v3(0, 0, 1) : v3(0, 1, 0), wo), x))
        return nan3();
    const V3 y = cross(wo, x);
    const float phi = 2.0f * kPi * uy;
    V3 r;
    if (!unit(cosine * wo + sine * (cosf(phi) * x + sinf(phi) * y), r))
        return nan3();
    return r;
}

// ------------------------------------------------------------------ scalar helpers (shaders/render.metal)
// :1901-1909 power heuristic with exponent two, scale-invariant
RP_DEV float power_weight(float a, float b) {
    const float scale = fmaxf(a, b);
    if (!(scale > 0) || !isfinite(scale))
        return fnan();
    a /= scale;
    b /= scale;
    return a * a / (a * a + b * b);
}
// :843-847
RP_DEV float bsdf_weight(float cosine) {
    const float relative = 4.0f * cosine;
    const float square = relative * relative;
    return square / (1.0f + square);
}
// :828-835 cosine-weighted direction about n
RP_DEV V3 cosine_hemisphere(V3 n, float u, float v) {
    const float r = sqrtf(u);
    const float phi = 2.0f * kPi * v;
    const V3 axis = fabsf(n.z) < 0.999f ? v3(0, 0, 1) : v3(0, 1, 0);
    const V3 t = normalize3(cross(axis, n));
    const V3 b = cross(n, t);
    return normalize3((r * cosf(phi)) * t + (r * sinf(phi)) * b + sqrtf(1.0f - u) * n);
}
// :1912-1929: conservative offset of a hit along n, rounded outward
RP_DEV V3 spawn_origin(V3 o, V3 d, float t, const SurfacePoint &pt, V3 n) {
    V3 ray_position, ray_error;
    ray_point(o, d, t, pt.curved, ray_position, ray_error);
    const V3 error = (pt.error + vabs(pt.position - ray_position)) + ray_error;
    return round_out(pt.position + dot(vabs(n), error) * n, n);
}
// :1931-1934
RP_DEV V3 spawn_toward(V3 o, V3 d, float t, const SurfacePoint &pt, V3 direction) {
    const V3 ng = pt.geometric_normal;
    return spawn_origin(o, d, t, pt, dot(ng, direction) < 0.0f ? -ng : ng);
}
// :2221-2232 connection to a sampled area point, ending on its near side
RP_DEV V3 shadow_segment_direction(V3 origin, V3 delta, const SurfacePoint &target, float signed_cosine) {
    const V3 n = signed_cosine > 0.0f ? target.geometric_normal : -target.geometric_normal;
    const float g7 = gamma_bound(7.0f) * target.world_extent;
    const V3 error = (target.error + gamma_bound(2.0f) * (vabs(origin) + vabs(delta))) + v3(g7, g7, g7);
    const V3 endpoint = round_out(target.position + dot(vabs(n), error) * n, n);
    return endpoint - origin;
}
// :659-677
RP_DEV bool point_direction(V3 from, V3 to, V3 &direction, float &distance_squared, bool spot) {
    if (spot) {
        if (!normal_or_zero(from.x) || !normal_or_zero(from.y) || !normal_or_zero(from.z) || !normal_or_zero(to.x) ||
            !normal_or_zero(to.y) || !normal_or_zero(to.z))
            return false;
    }
    const V3 delta = to - from;
    distance_squared = dot(delta, delta);
    if (!(distance_squared >= kFltMin) || !isfinite(distance_squared))
        return false;
    direction = delta / sqrtf(distance_squared);
    if (spot) {
        const float f[3] = {from.x, from.y, from.z}, tt[3] = {to.x, to.y, to.z}, dl[3] = {delta.x, delta.y, delta.z},
                    dr[3] = {direction.x, direction.y, direction.z};
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if ((f[i] != tt[i] && dl[i] == 0) || (dl[i] != 0 && dr[i] == 0) || !normal_or_zero(dr[i]))
                return false;
    }
    return finite3(direction);
}
// :145-150
RP_DEV u32 outgoing_medium(const DInstance &in, u32 current, V3 normal, V3 direction) {
    return in.inside_medium == in.outside_medium ? current
           : dot(normal, direction) > 0          ? in.outside_medium
                                                 : in.inside_medium;
}
// :128-136 Philox stream of medium draws
RP_DEV uint4 medium_words(const WaveParams &p, u32 pixel, u32 slo, u32 shi, u32 &draw) {
    return philox(make_uint4(pixel, slo, shi, kMediumBlockLimit | draw++), p.seed_low, p.seed_high ^ kMediumStream);
}
RP_DEV const float *medium_record(const DeviceScene &s, u32 id) { return s.media + size_t(id) * kMediumStride; }

// ------------------------------------------------------------------ scalar lights (shaders/scalar_lighting.h)
enum : u32 { kIncidentArea = 0, kIncidentPositional = 1, kIncidentDistant = 2, kIncidentEnvironment = 3 };
struct Incident {
    V3 direction, endpoint;
    SurfacePoint target;
    float radiance, pdf;
    u32 kind;
    bool valid;
};
// :23-121 (area, point and spot lights, the environment image; a constant environment offers
// no light sample)
__device__ __noinline__ Incident scalar_light_sample(const DeviceScene &s, float wavelength, V3 position, V3 normal,
                                                     float selection, float ux, float uy) {
    Incident r;
    r.direction = r.endpoint = v3(0, 0, 0);
    r.target.position = r.target.error = r.target.geometric_normal = r.target.shading_normal = v3(0, 0, 0);
    r.target.inverse_area_pdf = r.target.world_extent = 0;
    r.radiance = r.pdf = 0;
    r.kind = kIncidentEnvironment;
    r.valid = true;
    const Selected chosen = light_sample(s, position, normal, selection);
    if (!(chosen.pmf > 0))
        return r;
    const u32 id = chosen.light;
    if (id < s.emitter_count) {
        r.kind = kIncidentArea;
        float conditional = 0;
        if (!light_geometry_sample(s, id, position, normal, ux, uy, r.target, conditional)) {
            r.valid = false;
            return r;
        }
        if (!(conditional > 0))
            return r;
        const V3 d = r.target.position - position;
        const float d2 = dot(d, d);
        if (!(d2 > 0))
            return r;
        r.direction = d / sqrtf(d2);
        r.endpoint = r.target.position;
        r.pdf = chosen.pmf * conditional;
        const DInstance &in = s.instances[s.emitter_instance[id]];
        const float cosine = dot(r.target.geometric_normal, -r.direction);
        if (cosine == 0 || (!s.emission_two_sided[in.emission] && cosine < 0))
            return r;
        // area_radiance (shaders/render.metal:1811-1819)
        r.radiance = r.target.inverse_area_pdf == 0 ? 0.0f : spectrum(s, in.emission * 471u, wavelength);
    } else if (id < s.emitter_count + s.positional_count) {
        r.kind = kIncidentPositional;
        const DPositional &L = s.positional[id - s.emitter_count];
        float intensity = spectrum(s, L.spectrum, wavelength);
        if (intensity == 0)
            return r;
        r.endpoint = v3(L.position[0], L.position[1], L.position[2]);
        float d2 = 0;
        r.valid = point_direction(position, r.endpoint, r.direction, d2, L.kind != 0);
        if (!r.valid)
            return r;
        r.valid = positional_intensity(L, r.direction, intensity);
        r.radiance = intensity / d2;
        r.pdf = chosen.pmf;
    } else if (id == s.environment_light) {
        if (s.img.env_image == kNone)
            return r;
        float conditional = 0;
        r.valid = sample_environment_image(s.img, ux, uy, true, r.direction, conditional);
        if (!r.valid)
            return r;
        r.pdf = chosen.pmf * conditional;
        r.radiance = environment_image_radiance(s.img, r.direction, wavelength);
    } else {
        r.valid = false;
    }
    r.valid = r.valid && isfinite(r.radiance) && r.radiance >= 0 && isfinite(r.pdf) && r.pdf >= 0;
    return r;
}
// environment_pdf (shaders/scalar_lighting.h:14-23): the light sampler's density of an escaped
// direction, zero for a constant environment (continuation alone reaches it)
RP_DEV float scalar_environment_pdf(const DeviceScene &s, V3 position, V3 normal, V3 direction) {
    if (s.img.env_image == kNone || s.environment_light == kNone)
        return 0.0f;
    return light_pmf(s, position, normal, s.environment_light) * environment_image_pdf(s.img, direction, true);
}
RP_DEV bool incident_delta(const Incident &l) { return l.kind == kIncidentPositional || l.kind == kIncidentDistant; }


// ------------------------------------------------------------------ path state
// ScalarState (shaders/scalar_transport.h:38-52), kept in a wavefront slot between trips.
struct ScalarPath {
    u32 lane, pixel, slo, shi, status, scatterings;
    u64 index;
    float wavelength, radiance;
    V3 o, d;
    float throughput, escape_weight, previous_bsdf_pdf;
    bool previous_delta;
    V3 prev_p, prev_n; // previous light-sampling context
    u32 current_medium, medium_draw, boundary_crossings;
};

// What a path does once its pending light connection resolves.
enum : u32 { kAfterContinue = 0, kAfterFinish = 1, kAfterFail = 2 /* + status << 8 */ };

// A light connection in flight: medium_connection (shaders/render.metal:1588-1677) one leg per
// trace, or visible_shadow (:1570-1576) in scenes without media.  It carries the contribution
// it adds when it resolves with transmittance T: a surface sample adds a * T, a medium sample
// checks value = a * T and adds b * value (shaders/render.metal:2237-2260).
struct Connection {
    V3 o, d;         // current leg; d is a unit vector except for the vacuum query
    float remaining; // leg length (world), or the parametric limit of the vacuum query
    V3 end;
    float T;
    u32 medium, crossings, after;
    bool finite_end, vacuum, medium_sample;
    float a, b;
};

struct ScalarParams {
    u32 boundary_limit;
    uint4 *out;               // per lane: status, wavelength bits, radiance bits, scatterings
    const float4 *fresh_ray;  // per lane: primary direction, wavelength
    const uint2 *fresh_index; // per lane: Sobol index
    u32 *next_lane;           // regeneration counter
    unsigned long long *stats; // closest [0] nodes, [1] triangles, [2] rays; connection [3] rays, [4] nodes, [5] triangles
};

// begin_sample + primary_ray + the wavelength of scalar_init (shaders/scalar_transport.h:64-77)
// for every lane of a wave, written once so the step kernel starts paths with loads.
__global__ void k_scalar_raygen(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams p,
                                float4 *ray, uint2 *index) {
    for (u32 lane = blockIdx.x * blockDim.x + threadIdx.x; lane < p.lanes; lane += gridDim.x * blockDim.x) {
        const BeginSample b = begin_sample(s, p, lane);
        V3 o, d;
        primary_ray(s, p, b, o, d);
        ray[lane] = make_float4(d.x, d.y, d.z, 360.0f + 470.0f * sample_uniform(p, b.words.z));
        index[lane] = make_uint2(u32(b.index), u32(b.index >> 32));
    }
}

// scalar_init (shaders/scalar_transport.h:64-77) from the raygen records
RP_DEV void scalar_start(const DeviceScene &s, const WaveParams &p, const ScalarParams &q, u32 lane, ScalarPath &path) {
    path.lane = lane;
    path.pixel = p.pixel_begin + lane % p.pixel_count;
    path.slo = p.sample_low + lane / p.pixel_count;
    path.shi = p.sample_high + u32(path.slo < p.sample_low);
    const float4 r = q.fresh_ray[lane];
    const uint2 ix = q.fresh_index[lane];
    path.index = (u64(ix.y) << 32) | ix.x;
    path.status = S_SUCCESS;
    path.scatterings = 0;
    path.wavelength = r.w;
    path.radiance = 0;
    path.o = s.origin;
    path.d = v3(r.x, r.y, r.z);
    path.throughput = 1;
    path.escape_weight = 1;
    path.previous_bsdf_pdf = 0;
    path.previous_delta = false;
    path.prev_p = path.o;
    path.prev_n = v3(0, 0, 0);
    path.current_medium = s.camera_medium;
    path.medium_draw = 0;
    path.boundary_crossings = 0;
}
// sky_radiance (shaders/render.metal:813-819): the demo model's sky is a unit equal-energy
// spectrum
RP_DEV float environment_radiance(const DeviceScene &s, float wavelength) {
    if (s.model == kModelDemo)
        return 1.0f;
    return s.environment == kNone ? 0.0f : spectrum(s, s.environment, wavelength);
}
// demo_reflectance (shaders/render.metal:537-546) at the demo knots 360 420 470 520 570 620 700 830
RP_DEV float demo_reflectance(const float *r, float w) {
    const float knots[8] = {360, 420, 470, 520, 570, 620, 700, 830};
#pragma unroll
    for (int i = 1; i < 8; ++i)
        if (w <= knots[i]) {
            const float t = (w - knots[i - 1]) / (knots[i] - knots[i - 1]);
            return r[i - 1] + (r[i] - r[i - 1]) * t;
        }
    return r[7];
}

// scalar_sky_step (shaders/scalar_transport.h:88-210): scenes without geometry.  Light
// selection shares the flight draw and phase sampling takes the next medium block.
// Returns true when the path finished.
__device__ __noinline__ bool scalar_sky_step(const DeviceScene &s, const WaveParams &p, ScalarPath &path) {
    if (s.model == kModelPbrt && (!finite3(path.o) || !finite3(path.d))) {
        path.status = S_ARITHMETIC;
        return true;
    }
    if (s.camera_medium != kNone) {
        const float *m = medium_record(s, s.camera_medium);
        const u32 wi = dense_index(path.wavelength);
        const float a = __ldg(m + wi), sc = __ldg(m + 471 + wi), total = a + sc;
        if (total > 0) {
            const Segment seg = medium_segment(a, sc, __ldg(m + 942 + wi), finf());
            if (!seg.valid) {
                path.status = S_ARITHMETIC;
                return true;
            }
            if (path.scatterings < s.max_depth)
                path.radiance += path.throughput * seg.emission;
            if (path.scatterings >= s.max_depth || sc == 0)
                return true;
            if (path.scatterings >= p.emergency_limit) {
                path.status = S_EMERGENCY;
                return true;
            }
            const uint4 flight_words = medium_words(p, path.pixel, path.slo, path.shi, path.medium_draw);
            const float distance = medium_flight(total, u01(flight_words.x));
            const V3 point = fma3(v3(distance, distance, distance), path.d, path.o);
            if (!isfinite(distance) || !finite3(point)) {
                path.status = S_ARITHMETIC;
                return true;
            }
            path.throughput *= sc / total;
            const float g = __ldg(m + 1413);
            const Selected chosen = light_sample(s, point, v3(0, 0, 0), u01(flight_words.y));
            if (chosen.pmf > 0) {
                V3 direction = v3(0, 0, 0);
                float radiance = 0, distance_to_light = 0;
                if (chosen.light >= s.emitter_count && chosen.light < s.emitter_count + s.positional_count) {
                    const DPositional &L = s.positional[chosen.light - s.emitter_count];
                    float d2 = 0, intensity = spectrum(s, L.spectrum, path.wavelength);
                    if (intensity != 0) {
                        if (!point_direction(point, v3(L.position[0], L.position[1], L.position[2]), direction, d2,
                                             L.kind != 0) ||
                            !positional_intensity(L, direction, intensity)) {
                            path.status = S_ARITHMETIC;
                            return true;
                        }
                        radiance = intensity / d2;
                        distance_to_light = sqrtf(d2);
                    }
                }
                if (radiance > 0) {
                    const float tr = expf(-total * distance_to_light);
                    path.radiance += path.throughput * hg_phase(-path.d, direction, g) * (radiance / chosen.pmf) * tr;
                }
                if (!isfinite(path.radiance) || path.radiance < 0) {
                    path.status = S_ARITHMETIC;
                    return true;
                }
            }
            const uint4 phase_words = medium_words(p, path.pixel, path.slo, path.shi, path.medium_draw);
            const V3 wi = hg_sample(-path.d, g, u01(phase_words.x), u01(phase_words.y));
            ++path.scatterings;
            if (path.scatterings >= 3) {
                if (phase_words.z >= 0xc0000000u)
                    return true;
                path.throughput /= .75f;
            }
            if (!finite3(wi) || !isfinite(path.throughput)) {
                path.status = S_ARITHMETIC;
                return true;
            }
            path.o = point;
            path.d = wi;
            return false;
        }
    }
    path.radiance = s.img.env_image != kNone ? environment_image_radiance(s.img, path.d, path.wavelength)
                                             : environment_radiance(s, path.wavelength);
    return true;
}

// The prologue of medium_connection (shaders/render.metal:1593-1606): false on an invalid
// connection, which fails the sample with invalid arithmetic.
RP_DEV bool connection_begin(V3 o, V3 d, float tmax, u32 medium, Connection &c) {
    const float length = length3(d);
    if (!(length > 0) || !isfinite(length))
        return false;
    c.d = d / length;
    c.remaining = tmax * length;
    c.finite_end = isfinite(tmax);
    c.end = c.finite_end ? fma3(v3(tmax, tmax, tmax), d, o) : v3(0, 0, 0);
    if (!(c.remaining > 0) || (c.finite_end && (!isfinite(c.remaining) || !finite3(c.end) || eq3(c.end, o))))
        return false;
    c.o = o;
    c.T = 1;
    c.medium = medium;
    c.crossings = 0;
    c.vacuum = false;
    return true;
}

enum : int { kEventPath = 0, kEventFinished = 1, kEventConnect = 2 };

// Apply what the path does after its connection (or directly, when it made none).
RP_DEV int apply_after(ScalarPath &path, u32 after) {
    if (after == kAfterContinue)
        return kEventPath;
    if (after != kAfterFinish)
        path.status = after >> 8;
    return kEventFinished;
}

// One connection leg after its closest hit.  Returns kEventConnect while legs remain.
RP_DEV int connection_step(const DeviceScene &s, const ScalarParams &q, ScalarPath &path, Connection &c, bool ok,
                           const Hit &h) {
    float T;
    if (c.vacuum) {
        // visible_shadow: any hit occludes; a failed query is invalid arithmetic
        if (!ok) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        T = h.prim == kNone ? 1.0f : 0.0f;
    } else {
        if (!ok) {
            path.status = S_HIT;
            return kEventFinished;
        }
        const bool miss = h.prim == kNone;
        const float distance = miss ? c.remaining : h.t;
        if (c.medium != kNone) {
            const float *m = medium_record(s, c.medium);
            const u32 wi = dense_index(path.wavelength);
            const Segment seg = medium_segment(__ldg(m + wi), __ldg(m + 471 + wi), 0, distance);
            if (!seg.valid) {
                path.status = S_ARITHMETIC;
                return kEventFinished;
            }
            c.T *= seg.transmission;
        }
        T = c.T;
        if (!(miss || T == 0)) {
            if (!isfinite(h.t) || h.prim >= s.prim_count) {
                path.status = S_HIT;
                return kEventFinished;
            }
            const u32 inst = s.tri_instance[h.prim];
            const DInstance &in = s.instances[inst];
            if (in.material >= s.material_count) {
                path.status = S_HIT;
                return kEventFinished;
            }
            if (s.materials[in.material].scattering != kInterfaceScattering) {
                T = 0;
            } else {
                // cross the null interface and continue towards the endpoint
                if (c.crossings++ >= q.boundary_limit) {
                    path.status = S_BOUNDARY;
                    return kEventFinished;
                }
                SurfacePoint pt;
                V3 next;
                if (!hit_surface_point(s, h.prim, inst, s.tri_local[h.prim], h.b1, h.b2, pt) ||
                    !spawn_boundary(c.o, c.d, h.t, pt, c.d, next)) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
                const V3 outgoing_normal =
                    dot(pt.geometric_normal, c.d) < 0 ? -pt.geometric_normal : pt.geometric_normal;
                if (c.finite_end) {
                    const V3 delta = c.end - next;
                    c.remaining = length3(delta);
                    if (!(c.remaining > 0) || !isfinite(c.remaining)) {
                        path.status = S_ARITHMETIC;
                        return kEventFinished;
                    }
                    c.d = delta / c.remaining;
                    const float facing = dot(outgoing_normal, c.d);
                    const float facing_error = gamma_bound(5) * dot(vabs(outgoing_normal), vabs(c.d));
                    if (!(facing > facing_error)) {
                        path.status = S_ARITHMETIC;
                        return kEventFinished;
                    }
                }
                c.medium = outgoing_medium(in, c.medium, pt.geometric_normal, c.d);
                c.o = next;
                return kEventConnect;
            }
        }
    }
    // resolved with transmittance T
    if (c.medium_sample) {
        const float value = c.a * T;
        if (!isfinite(value) || !(value >= 0)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        path.radiance += c.b * value;
    } else if (isnan(c.a)) {
        // a light sample whose weight failed: invalid where the light is seen
        if (T > 0) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
    } else {
        path.radiance += c.a * T;
    }
    return apply_after(path, c.after);
}

// One wavelength of a conductor (kind 1) or dielectric (kind 2) surface: prepare_scattering
// (shaders/render.metal:2079-2160) for constant roughness and tabulated optical constants, with
// rypath_conductor::prepare (shaders/conductor.h:22-34) and rypath_dielectric::prepare
// (shaders/dielectric.h:15-27; eta 1 is smooth).
struct ScalarBsdf {
    u32 kind;
    float eta, k;
    Ggx g;
};
// Out of line: the step kernel's diffuse and medium events do not carry their registers.
__device__ __noinline__ bool prepare_scalar_bsdf(const DeviceScene &s, const DMaterial &m, float w, ScalarBsdf &b) {
    b.kind = m.scattering;
    const float u = m.u_roughness, v = m.v_roughness;
    if (!isfinite(u) || !isfinite(v) || u < 0 || v < 0)
        return false;
    float eta = optical_value(s.knots, m.eta_begin, m.eta_count, s.knot_count, (m.optical_extensions & 1u) != 0, w);
    b.k = 0;
    if (m.scattering == 1) {
        b.k = optical_value(s.knots, m.k_begin, m.k_count, s.knot_count, (m.optical_extensions & 2u) != 0, w);
        if (!isfinite(eta) || !isfinite(b.k) || eta < 0 || b.k < 0 || (eta == 0 && b.k == 0))
            return false;
    } else {
        if (!isfinite(eta) || eta < 0)
            return false;
        eta = eta == 0 ? 1 : eta;
    }
    b.eta = eta;
    return prepare_roughness(u, v, m.remap != 0, m.scattering == 2 && eta == 1, b.g);
}
__device__ __noinline__ Eval scalar_bsdf_evaluate(const ScalarBsdf &b, V3 wo, V3 wi) {
    return b.kind == 2 ? dielectric_evaluate(b.eta, b.g, wo, wi) : conductor_evaluate(b.eta, b.k, b.g, wo, wi);
}
__device__ __noinline__ BSample scalar_bsdf_sample(const ScalarBsdf &b, V3 wo, float lobe, float ux, float uy) {
    float sampled_eta;
    return b.kind == 2 ? dielectric_sample(b.eta, b.g, wo, lobe, ux, uy, sampled_eta)
                       : conductor_sample(b.eta, b.k, b.g, wo, ux, uy);
}
// scattering_direct (shaders/render.metal:2212-2219)
RP_DEV float scattering_direct(float f_cos, float bsdf_pdf, float light_pdf, bool invisible) {
    if (!(f_cos >= 0) || !(bsdf_pdf >= 0) || !(light_pdf > 0) || !isfinite(f_cos) || !isfinite(bsdf_pdf) ||
        !isfinite(light_pdf))
        return fnan();
    if (f_cos == 0)
        return 0;
    return (f_cos / light_pdf) * (invisible ? 1.0f : power_weight(light_pdf, bsdf_pdf));
}
// The dielectric lobe choice of one bounce (shaders/render.metal:180-198): Halton dimension
// 884 + bounce, (Z)Sobol dimension 908 + bounce, else Philox block 0x80000000 | bounce.
RP_DEV u32 dielectric_lobe_word(const DeviceScene &s, const WaveParams &p, u32 pixel, u32 slo, u32 shi, u64 index,
                                u32 bounce) {
    if (p.sampler == 2)
        return float_bits(qmc_radical(s.primes, 884u + bounce, index, p.randomization, p.seed_low));
    if (p.sampler == 3)
        return zdraw(s, p, index, 908u + bounce);
    if (p.sampler == 1)
        return sobol_word(s.sobol, index, 908u + bounce, p.randomization, p.seed_low);
    return philox(make_uint4(pixel, slo, shi, 0x80000000u | bounce), p.seed_low, p.seed_high).x;
}

// One event after the path ray's closest hit: scalar_shade (shaders/scalar_transport.h:286-900)
// for diffuse, conductor and dielectric surfaces and null interfaces.  A light sample that needs a connection leaves it in
// `c` (returning kEventConnect) after the continuation has been sampled: the two use disjoint
// draws, and the connection's contribution and status are applied before the continuation's.
// The surface point of a path hit: any primitive kind, or triangles alone in the plain kernel.
template <bool Full>
RP_DEV bool scalar_surface_point(const DeviceScene &s, u32 prim, u32 inst, u32 local, float b1, float b2,
                                 SurfacePoint &point) {
    if (Full)
        return hit_surface_point(s, prim, inst, local, b1, b2, point);
    return triangle_surface_point(s, inst, local, b1, b2, true, point);
}
// Full: the scene has conductor or dielectric surfaces, procedural primitives or image
// reflectance (their code is compiled out of the plain step kernel).
template <bool Full>
RP_DEV int shade_event(const DeviceScene &s, const WaveParams &p, const ScalarParams &q, ScalarPath &path, bool ok,
                       const Hit &hit, Connection &c) {
    if (!ok) {
        path.status = S_HIT;
        return kEventFinished;
    }
    const bool miss = hit.prim == kNone;
    // medium interaction (:354-420)
    if (path.current_medium != kNone) {
        if (path.current_medium >= s.medium_count) {
            path.status = S_HIT;
            return kEventFinished;
        }
        if (path.medium_draw >= kMediumBlockLimit - 3) {
            path.status = S_BOUNDARY;
            return kEventFinished;
        }
        const float *m = medium_record(s, path.current_medium);
        const u32 wi = dense_index(path.wavelength);
        const float a = __ldg(m + wi), sc = __ldg(m + 471 + wi), total = a + sc;
        const float ray_length = length3(path.d);
        const float distance = miss ? finf() : hit.t * ray_length;
        const Segment seg =
            medium_segment(a, sc, path.scatterings < s.max_depth ? __ldg(m + 942 + wi) : 0.0f, distance);
        if (!seg.valid || !(ray_length > 0) || !isfinite(ray_length)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        path.radiance += path.throughput * seg.emission;
        if (total > 0) {
            const uint4 flight_words = medium_words(p, path.pixel, path.slo, path.shi, path.medium_draw);
            const float flight = medium_flight(total, u01(flight_words.x));
            if (flight < distance || isinf(distance)) {
                if (!isfinite(flight)) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
                if (path.scatterings >= s.max_depth || sc == 0)
                    return kEventFinished;
                if (path.scatterings >= p.emergency_limit) {
                    path.status = S_EMERGENCY;
                    return kEventFinished;
                }
                const V3 direction = path.d / ray_length;
                const V3 position = fma3(v3(flight, flight, flight), direction, path.o);
                if (!finite3(position)) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
                path.throughput *= sc / total;
                const uint4 light_words = medium_words(p, path.pixel, path.slo, path.shi, path.medium_draw);
                const uint4 phase_words = medium_words(p, path.pixel, path.slo, path.shi, path.medium_draw);
                const float g = __ldg(m + 1413);
                // medium_direct (shaders/render.metal:2237-2260)
                const Incident light = scalar_light_sample(s, path.wavelength, position, v3(0, 0, 0),
                                                           u01(light_words.x), u01(light_words.y), u01(light_words.z));
                if (!light.valid) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
                bool connect = false;
                if (light.pdf > 0 && light.radiance != 0) {
                    V3 cd;
                    // connection (shaders/scalar_lighting.h:121-133): the environment's is unbounded
                    const bool unbounded = light.kind == kIncidentEnvironment;
                    if (light.kind == kIncidentArea) {
                        const V3 delta = light.target.position - position;
                        cd = shadow_segment_direction(position, delta, light.target,
                                                      dot(light.target.geometric_normal, -delta));
                    } else {
                        cd = unbounded ? light.direction : light.endpoint - position;
                    }
                    if (!connection_begin(position, cd, unbounded ? finf() : kOneMinusEps, path.current_medium, c)) {
                        path.status = S_ARITHMETIC;
                        return kEventFinished;
                    }
                    const float phase = hg_phase(-direction, light.direction, g);
                    const float weight = incident_delta(light) ? 1.f : power_weight(light.pdf, phase);
                    c.medium_sample = true;
                    c.a = ((phase / light.pdf) * weight) * light.radiance;
                    c.b = path.throughput;
                    connect = true;
                }
                // phase continuation and roulette
                u32 after = kAfterContinue;
                const V3 wi_dir = hg_sample(-direction, g, u01(phase_words.x), u01(phase_words.y));
                const float pdf = hg_phase(-direction, wi_dir, g);
                if (!finite3(wi_dir) || !(pdf > 0) || !isfinite(pdf)) {
                    after = kAfterFail | (S_ARITHMETIC << 8);
                } else {
                    path.previous_bsdf_pdf = pdf;
                    ++path.scatterings;
                    if (path.scatterings >= 3 && phase_words.z >= 0xc0000000u) {
                        after = kAfterFinish;
                    } else {
                        if (path.scatterings >= 3)
                            path.throughput /= .75f;
                        path.previous_delta = false;
                        path.prev_p = position;
                        path.prev_n = v3(0, 0, 0);
                        path.escape_weight = 1;
                        path.o = position;
                        path.d = wi_dir;
                        path.boundary_crossings = 0;
                    }
                }
                if (connect) {
                    c.after = after;
                    return kEventConnect;
                }
                return apply_after(path, after);
            }
        }
    }
    if (miss) {
        // escape (:421-433): MIS against the environment image's light samples (a constant
        // environment has no light-sampling density)
        const float Le = s.img.env_image != kNone ? environment_image_radiance(s.img, path.d, path.wavelength)
                                                  : environment_radiance(s, path.wavelength);
        if (s.model == kModelPbrt && path.scatterings != 0u && !path.previous_delta)
            path.escape_weight = power_weight(path.previous_bsdf_pdf,
                                              scalar_environment_pdf(s, path.prev_p, path.prev_n, path.d));
        path.radiance += path.throughput * path.escape_weight * Le;
        return kEventFinished;
    }
    const u32 bounce = path.scatterings;
    if (!isfinite(hit.t) || hit.prim >= s.prim_count) {
        path.status = S_HIT;
        return kEventFinished;
    }
    const u32 inst = s.tri_instance[hit.prim], local = s.tri_local[hit.prim];
    const DInstance &instance = s.instances[inst];
    if (instance.material >= s.material_count || !isfinite(hit.b1) || !isfinite(hit.b2)) {
        path.status = S_HIT;
        return kEventFinished;
    }
    const DMaterial material = s.materials[instance.material];
    SurfacePoint point;
    if (material.scattering == kInterfaceScattering) {
        // null interface (:450-472): change media, no scattering event
        if (path.boundary_crossings++ >= q.boundary_limit) {
            path.status = S_BOUNDARY;
            return kEventFinished;
        }
        if (!scalar_surface_point<Full>(s, hit.prim, inst, local, hit.b1, hit.b2, point)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        path.current_medium = outgoing_medium(instance, path.current_medium, point.geometric_normal, path.d);
        V3 origin;
        if (!spawn_boundary(path.o, path.d, hit.t, point, path.d, origin)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        path.o = origin;
        return kEventPath;
    }
    const bool emissive = instance.emission != kNone;
    if (emissive) {
        // area emission with MIS against the light sampler (:473-520)
        if (!scalar_surface_point<Full>(s, hit.prim, inst, local, hit.b1, hit.b2, point)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        const float Le = point.inverse_area_pdf == 0 ? 0.0f : spectrum(s, instance.emission * 471u, path.wavelength);
        if (Le > 0.0f && (s.emission_two_sided[instance.emission] || dot(point.geometric_normal, -path.d) >= 0.0f)) {
            float weight = 1.0f;
            if (bounce != 0u && !path.previous_delta) {
                const u32 light_id = instance.emitter_begin + local;
                if (light_id >= s.emitter_count) {
                    path.status = S_HIT;
                    return kEventFinished;
                }
                const float pdf = light_pmf(s, path.prev_p, path.prev_n, light_id) *
                                  light_geometry_pdf(s, light_id, path.prev_p, path.prev_n, point);
                weight = power_weight(path.previous_bsdf_pdf, pdf);
            }
            if (!isfinite(weight)) {
                path.status = S_ARITHMETIC;
                return kEventFinished;
            }
            path.radiance += path.throughput * (weight * Le);
        }
    }
    if (bounce >= s.max_depth)
        return kEventFinished;
    // mix materials resolve at the hit's point (:541-587)
    bool point_ready = emissive;
    u32 material_index = instance.material;
    if (material.scattering == kMixScattering) {
        if (!emissive && !scalar_surface_point<Full>(s, hit.prim, inst, local, hit.b1, hit.b2, point)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        point_ready = true;
        const u32 mix_status = resolve_mix(s, point.position, -path.d, material_index);
        if (mix_status != 0) {
            path.status = mix_status == 2 ? S_ARITHMETIC : S_HIT;
            return kEventFinished;
        }
    }
    const DMaterial surface = s.materials[material_index];
    // conductors and dielectrics carry their spectrum in the BSDF: rho = 1 (:591-598)
    const bool microfacet = Full && surface.scattering != 0;
    float rho = 0;
    if (!Full && surface.scattering != 0) {
        path.status = S_HIT;
        return kEventFinished;
    }
    if (microfacet) {
        if (surface.scattering > 2) {
            path.status = S_HIT;
            return kEventFinished;
        }
        rho = 1.0f;
    } else if (s.model == kModelDemo) {
        if (surface.kind != 0) {
            path.status = S_HIT;
            return kEventFinished;
        }
        rho = demo_reflectance(surface.reflectance, path.wavelength);
    } else if (surface.kind == 0 && surface.knot_count >= 2 && surface.knot_begin <= s.knot_count &&
               surface.knot_count <= s.knot_count - surface.knot_begin) {
        rho = pbrt_reflectance(s.knots + surface.knot_begin, surface.knot_count, path.wavelength);
    } else if (surface.kind == 1) {
        rho = surface.scalar_value;
    } else if (surface.kind == 4) {
        rho = blackbody_reflectance(surface.scalar_value, path.wavelength);
    } else if (surface.kind == 2) {
        rho = sigmoid_reflectance(surface.coefficients, path.wavelength);
    } else if (Full && surface.kind == 3 && s.img.textured && surface.image_texture < s.img.texture_count) {
        // image_reflectance (shaders/render.metal:1154-1240) at the hit's footprint
        if (!point_ready && !scalar_surface_point<Full>(s, hit.prim, inst, local, hit.b1, hit.b2, point)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        point_ready = true;
        F2 st, dstdx, dstdy;
        if (!texture_context(s, p, path.pixel, path.slo, path.shi, inst, local, hit.b1, hit.b2, point.geometric_normal,
                             path.d, path.scatterings, st, dstdx, dstdy)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        rho = rgb_spectrum(s.img.rgb_table, image_reflectance_rgb(s.img, surface.image_texture, st, dstdx, dstdy),
                           path.wavelength);
    } else {
        path.status = S_HIT;
        return kEventFinished;
    }
    if (!isfinite(rho) || !(rho >= 0.0f && rho <= 1.0f)) {
        path.status = S_ARITHMETIC;
        return kEventFinished;
    }
    if (rho == 0.0f)
        return kEventFinished;
    const bool authored_normals = instance.normal_begin != kNone || microfacet;
    if (!authored_normals && bounce >= p.emergency_limit) {
        path.status = S_EMERGENCY;
        return kEventFinished;
    }
    if (!point_ready && !scalar_surface_point<Full>(s, hit.prim, inst, local, hit.b1, hit.b2, point)) {
        path.status = S_ARITHMETIC;
        return kEventFinished;
    }
    const float incident_cosine = dot(point.shading_normal, path.d);
    if (authored_normals && !microfacet && incident_cosine == 0.0f)
        return kEventFinished;
    if (bounce >= p.emergency_limit) {
        path.status = S_EMERGENCY;
        return kEventFinished;
    }
    const V3 n = incident_cosine > 0.0f ? -point.shading_normal : point.shading_normal;
    // the BSDF in the shading frame of the normal (:677-694)
    ScalarBsdf bsdf{};
    Frame frame{};
    V3 wo = v3(0, 0, 0);
    if (microfacet) {
        if (!prepare_scalar_bsdf(s, surface, path.wavelength, bsdf) || !shading_frame(point.shading_normal, frame)) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        wo = to_local(frame, -path.d);
        if (wo.z == 0)
            return kEventFinished;
    }
    const bool dirac = microfacet && bsdf.g.smooth; // delta_only (shaders/scattering.h:25-28)
    const bool both_hemispheres = microfacet && bsdf.kind == 2;
    const V3 context_normal = microfacet ? frame.z : point.shading_normal;
    const bool directional_offset = authored_normals;
    const V3 area_reference = directional_offset ? point.position : spawn_origin(path.o, path.d, hit.t, point, n);
    if (!finite3(area_reference)) {
        path.status = S_ARITHMETIC;
        return kEventFinished;
    }
    const uint4 light_words = draw_words(s, p, path.pixel, path.slo, path.shi, path.index, 2 + 2 * bounce);
    const uint4 bsdf_words = draw_words(s, p, path.pixel, path.slo, path.shi, path.index, 1 + 2 * bounce);
    // light sample: the demo model's sky sampled uniformly over the sphere with the
    // cosine-ratio weight (:709-781); PBRT scenes' lights with power-heuristic MIS (:783-835).
    // Dirac surfaces take no light sample.
    bool connect = false;
    if (s.model == kModelDemo) {
        const float E = 1.0f; // sky_radiance of the demo model
        const float uz = sample_uniform(p, light_words.x), uv = sample_uniform(p, light_words.y);
        const float z = 1.0f - 2.0f * uz;
        const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        const float phi = 2.0f * kPi * uv;
        const V3 direction = v3(r * cosf(phi), r * sinf(phi), z);
        const V3 local_light = microfacet ? to_local(frame, direction) : v3(0, 0, 0);
        const float cosine = both_hemispheres ? fabsf(local_light.z)
                             : microfacet     ? (wo.z > 0 ? local_light.z : -local_light.z)
                                              : dot(n, direction);
        if (!dirac && cosine > 0.0f) {
            const V3 origin = directional_offset ? spawn_toward(path.o, path.d, hit.t, point, direction) : area_reference;
            if (!finite3(origin)) {
                path.status = S_ARITHMETIC;
                return kEventFinished;
            }
            float factor;
            if (microfacet) {
                const Eval e = scalar_bsdf_evaluate(bsdf, wo, local_light);
                factor = e.valid ? scattering_direct(e.f * cosine, e.pdf, 1.0f / (4.0f * kPi), false) : fnan();
            } else {
                const float relative = 4.0f * cosine;
                factor = relative * (1.0f / (1.0f + relative * relative)); // (4 cos) * light_weight(cos)
            }
            const u32 medium = outgoing_medium(instance, path.current_medium, point.geometric_normal, direction);
            if (s.media_enabled) {
                if (!connection_begin(origin, direction, finf(), medium, c)) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
            } else {
                c.o = origin;
                c.d = direction;
                c.remaining = finf();
                c.vacuum = true;
            }
            c.medium_sample = false;
            // a factor that is not finite fails the sample only where the sky is seen (:747-767):
            // the connection carries it as NaN
            c.a = isfinite(factor) ? ((path.throughput * rho) * factor) * E : fnan();
            connect = true;
        }
    } else if (!dirac) {
        const Incident light = scalar_light_sample(s, path.wavelength, point.position, context_normal,
                                                   sample_uniform(p, light_words.x), sample_uniform(p, light_words.y),
                                                   sample_uniform(p, light_words.z));
        if (!light.valid) {
            path.status = S_ARITHMETIC;
            return kEventFinished;
        }
        if (light.pdf > 0 && light.radiance > 0) {
            const V3 local_light = microfacet ? to_local(frame, light.direction) : v3(0, 0, 0);
            const float cosine = both_hemispheres ? fabsf(local_light.z)
                                 : microfacet     ? (wo.z > 0 ? local_light.z : -local_light.z)
                                                  : dot(n, light.direction);
            if (cosine > 0) {
                float f_cos = rho * cosine / kPi;
                float bsdf_pdf = cosine / kPi;
                if (microfacet) {
                    const Eval e = scalar_bsdf_evaluate(bsdf, wo, local_light);
                    if (!e.valid) {
                        path.status = S_ARITHMETIC;
                        return kEventFinished;
                    }
                    f_cos = e.f * cosine;
                    bsdf_pdf = e.pdf;
                }
                const float factor = scattering_direct(f_cos, bsdf_pdf, light.pdf, incident_delta(light));
                const V3 origin = directional_offset ? spawn_toward(path.o, path.d, hit.t, point, light.direction)
                                                     : area_reference;
                V3 cd;
                const bool unbounded = light.kind == kIncidentEnvironment;
                if (light.kind == kIncidentArea) {
                    const V3 delta = light.target.position - origin;
                    cd = shadow_segment_direction(origin, delta, light.target, dot(light.target.geometric_normal, -delta));
                } else {
                    cd = unbounded ? light.direction : light.endpoint - origin;
                }
                if (!isfinite(factor) || !finite3(cd) || !(dot(cd, light.direction) > 0)) {
                    path.status = S_ARITHMETIC;
                    return kEventFinished;
                }
                const u32 medium = outgoing_medium(instance, path.current_medium, point.geometric_normal, light.direction);
                if (s.media_enabled) {
                    if (!connection_begin(origin, cd, unbounded ? finf() : kOneMinusEps, medium, c)) {
                        path.status = S_ARITHMETIC;
                        return kEventFinished;
                    }
                } else {
                    c.o = origin;
                    c.d = cd;
                    c.remaining = unbounded ? finf() : kOneMinusEps;
                    c.vacuum = true;
                }
                c.medium_sample = false;
                c.a = (path.throughput * factor) * light.radiance;
                connect = true;
            }
        }
    }
    // continuation (:837-900); a microfacet sample is resolved in world space by
    // resolve_scattering_continuation (shaders/render.metal:2006-2019)
    u32 after = kAfterContinue;
    V3 wi = v3(0, 0, 0);
    float continuation_pdf = 0, continuation_cosine = 0;
    bool continuation_delta = false;
    if (microfacet) {
        const float ux = sample_uniform(p, bsdf_words.x), uy = sample_uniform(p, bsdf_words.y);
        const float lobe = bsdf.kind == 2 ? sample_uniform(p, dielectric_lobe_word(s, p, path.pixel, path.slo, path.shi,
                                                                                path.index, bounce))
                                          : 0.0f; // the conductor draws no lobe
        BSample sampled = scalar_bsdf_sample(bsdf, wo, lobe, ux, uy);
        if (sampled.valid && sampled.accepted && !unit_vector(to_world(frame, sampled.wi), wi))
            sampled.valid = false;
        if (!sampled.valid) {
            after = kAfterFail | (S_ARITHMETIC << 8);
        } else if (!sampled.accepted) {
            after = kAfterFinish;
        } else {
            path.throughput *= sampled.weight;
            continuation_pdf = sampled.pdf;
            continuation_cosine = fabsf(sampled.wi.z);
            continuation_delta = sampled.delta;
        }
    } else {
        wi = cosine_hemisphere(n, sample_uniform(p, bsdf_words.x), sample_uniform(p, bsdf_words.y));
        path.throughput *= rho;
    }
    if (after != kAfterContinue) {
    } else if (!isfinite(path.throughput) || path.throughput < 0.0f) {
        after = kAfterFail | (S_ARITHMETIC << 8);
    } else {
        ++path.scatterings;
        if (path.scatterings >= 3 && decision_word(p, bsdf_words.z) >= 0xc0000000u) {
            after = kAfterFinish;
        } else {
            if (path.scatterings >= 3)
                path.throughput /= 0.75f;
            const float cosine = microfacet ? continuation_cosine : dot(n, wi);
            if (!isfinite(path.throughput) || !(cosine > 0.0f)) {
                after = kAfterFail | (S_ARITHMETIC << 8);
            } else {
                path.previous_bsdf_pdf = microfacet ? continuation_pdf : cosine / kPi;
                path.previous_delta = continuation_delta;
                path.prev_p = point.position;
                path.prev_n = context_normal;
                path.escape_weight = continuation_delta ? 1.0f
                                     : microfacet       ? power_weight(path.previous_bsdf_pdf, 1.0f / (4.0f * kPi))
                                                        : bsdf_weight(cosine);
                const V3 origin = directional_offset ? spawn_toward(path.o, path.d, hit.t, point, wi) : area_reference;
                if (!finite3(origin)) {
                    after = kAfterFail | (S_ARITHMETIC << 8);
                } else {
                    path.o = origin;
                    path.d = wi;
                    path.current_medium = outgoing_medium(instance, path.current_medium, point.geometric_normal, wi);
                    path.boundary_crossings = 0;
                }
            }
        }
    }
    if (connect) {
        c.after = after;
        return kEventConnect;
    }
    return apply_after(path, after);
}

// scalar_finish (shaders/scalar_transport.h:79-84)
RP_DEV uint4 scalar_record(const ScalarPath &path) {
    u32 status = path.status;
    if (status == S_SUCCESS && (!isfinite(path.radiance) || path.radiance < 0.0f))
        status = S_ARITHMETIC;
    return make_uint4(status, __float_as_uint(path.wavelength), __float_as_uint(path.radiance), path.scatterings);
}

// Wavefront form of the scalar transport (rypath_render_paths, shaders/scalar_transport.h):
// each trip of a path is one closest-hit query -- the path's ray or the current leg of its
// light connection -- and the event or connection step that consumes it.  Each path and its
// connection in flight stay in a slot in global memory between the two kernels:
// k_scalar_walk runs the query of every slot at the walk's own occupancy, k_scalar_step the
// event or connection step and hands finished slots the wave's next lanes.  Each lane's path
// depends only on its own indices, so its record does not depend on the slot or trip that
// ran it.
struct ScalarSlots {
    ScalarPath *path;
    Connection *conn;
    u32 *mode;      // kEvent* in the low byte; bit 8: the walk of this trip succeeded
    Hit *hit;       // the walk's hit
    u32 count;      // slots
    u32 *remaining; // lanes of the wave whose record is not written yet
    // the active slots of a trip sorted by what their step runs, so that a step warp runs one
    // kind: [parity] connection steps, path events that scatter in their medium, path events
    // at a null interface, other path events, counted in qcount[4 parity + 0 / 1 / 2 / 3]
    u32 *queue_connect[2], *queue_medium[2], *queue_interface[2], *queue_path[2];
    u32 *qcount;
};
constexpr u32 kWalkOk = 1u << 8;

RP_DEV bool scalar_ray_valid(const ScalarPath &path) {
    return finite3(path.o) && finite3(path.d) && isfinite(path.throughput) && isfinite(path.radiance);
}

// Warp-aggregated append of `slot` to `queue` (counter `count`) for the lanes with `want`.
RP_DEV void slot_append(u32 *queue, u32 *count, bool want, u32 slot) {
    const u32 ballot = __ballot_sync(0xffffffffu, want);
    const int lane = threadIdx.x & 31;
    u32 base = 0;
    if (lane == 0 && ballot)
        base = atomicAdd(count, __popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (want)
        queue[base + __popc(ballot & ((1u << lane) - 1))] = slot;
}

// Whether shade_event will take its medium-scattering branch for this hit: the same medium
// lookup and free-flight draw, without consuming the draw.  Only groups the step warps; the
// step itself decides.
RP_DEV bool predicts_medium_scatter(const DeviceScene &s, const WaveParams &p, const ScalarPath &path, const Hit &hit) {
    if (path.current_medium == kNone || path.current_medium >= s.medium_count ||
        path.medium_draw >= kMediumBlockLimit - 3)
        return false;
    const float *m = medium_record(s, path.current_medium);
    const u32 wi = dense_index(path.wavelength);
    const float total = __ldg(m + wi) + __ldg(m + 471 + wi);
    if (!(total > 0))
        return false;
    const float distance = hit.prim == kNone ? finf() : hit.t * length3(path.d);
    u32 draw = path.medium_draw;
    const float flight = medium_flight(total, u01(medium_words(p, path.pixel, path.slo, path.shi, draw).x));
    return flight < distance || isinf(distance);
}
// Whether the hit of a path event that does not scatter in its medium is a null interface.
RP_DEV bool hits_interface(const DeviceScene &s, const Hit &hit) {
    if (hit.prim == kNone || hit.prim >= s.prim_count)
        return false;
    const u32 material = s.instances[s.tri_instance[hit.prim]].material;
    return material < s.material_count && s.materials[material].scattering == kInterfaceScattering;
}

// Proc: the scene has procedural primitives.
template <bool Count, int Stack = kStackDepth, bool Proc = false>
__global__ void __launch_bounds__(kTraceBlock, Stack <= kShortStack ? 1024 / kTraceBlock : 1)
    k_scalar_walk(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams p, ScalarSlots w,
                  int parity, unsigned long long *stats) {
    __shared__ uint2 stack[Stack * kTraceBlock];
    u32 counts[6] = {0, 0, 0, 0, 0, 0};
    const u32 stride = gridDim.x * blockDim.x;
    const u32 trips = (w.count + stride - 1) / stride;
    for (u32 trip = 0; trip < trips; ++trip) {
        const u32 i = trip * stride + blockIdx.x * blockDim.x + threadIdx.x;
        u32 mode = kEventFinished;
        bool scatter = false, interface = false;
        if (i < w.count) {
            mode = w.mode[i] & 0xffu;
            if (mode != kEventFinished) {
                V3 ro, rd;
                float tmax;
                bool walk = true;
                const ScalarPath &path = w.path[i];
                if (mode == kEventPath) {
                    ro = path.o;
                    rd = path.d;
                    walk = scalar_ray_valid(path); // else the step kernel records the failure
                    tmax = finf();
                } else {
                    const Connection &c = w.conn[i];
                    ro = c.o;
                    rd = c.d;
                    tmax = c.remaining;
                }
                if (walk) {
                    Hit hit;
                    u32 nodes = 0, tris = 0;
                    const bool ok =
                        walk_closest<Count, Stack, Proc>(s, ro, rd, tmax, hit, stack + threadIdx.x, kTraceBlock, nodes, tris);
                    w.hit[i] = hit;
                    w.mode[i] = mode | (ok ? kWalkOk : 0u);
                    scatter = ok && mode == kEventPath && predicts_medium_scatter(s, p, path, hit);
                    interface = ok && mode == kEventPath && !scatter && hits_interface(s, hit);
                    if (Count && mode == kEventPath) {
                        counts[0] += nodes;
                        counts[1] += tris;
                        counts[2] += 1;
                    } else if (Count) {
                        counts[3] += 1;
                        counts[4] += nodes;
                        counts[5] += tris;
                    }
                }
            }
        }
        slot_append(w.queue_connect[parity], w.qcount + 4 * parity, mode == kEventConnect, i);
        slot_append(w.queue_medium[parity], w.qcount + 4 * parity + 1, mode == kEventPath && scatter, i);
        slot_append(w.queue_interface[parity], w.qcount + 4 * parity + 2, mode == kEventPath && interface, i);
        slot_append(w.queue_path[parity], w.qcount + 4 * parity + 3, mode == kEventPath && !scatter && !interface, i);
    }
    if (Count) {
        atomicAdd(stats + 0, (unsigned long long)counts[0]);
        atomicAdd(stats + 1, (unsigned long long)counts[1]);
        atomicAdd(stats + 2, (unsigned long long)counts[2]);
        atomicAdd(stats + 3, (unsigned long long)counts[3]);
        atomicAdd(stats + 4, (unsigned long long)counts[4]);
        atomicAdd(stats + 5, (unsigned long long)counts[5]);
    }
}

__global__ void k_scalar_slots_init(u32 *mode, u32 count) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        mode[i] = kEventFinished;
}

// The event (or connection step, or geometry-free sky step) of the active slots, then new
// lanes for the finished ones (one atomic per warp).  parity >= 0: the slots the walk of this
// trip queued, connection steps first, then medium-scattering path events, null-interface
// events and the other path events; parity < 0: every slot (the wave's first fill, and geometry-free scenes, which
// take no walk).  Four blocks of 128 per SM (128 registers, a few spilled) hide more of the
// slot loads' latency than three at 154 registers: 133 against 143 ms on the fog box.
template <bool Full>
__global__ void __launch_bounds__(kTraceBlock, 4) k_scalar_step(const __grid_constant__ DeviceScene s,
                                                             const __grid_constant__ WaveParams p, ScalarParams q,
                                                             ScalarSlots w, int parity) {
    const int lane_in_warp = threadIdx.x & 31;
    u32 n_connect = 0, n_medium = 0, n_interface = 0, total = w.count;
    if (parity >= 0) {
        n_connect = w.qcount[4 * parity];
        n_medium = n_connect + w.qcount[4 * parity + 1];
        n_interface = n_medium + w.qcount[4 * parity + 2];
        total = n_interface + w.qcount[4 * parity + 3];
        if (blockIdx.x == 0 && threadIdx.x < 4)
            w.qcount[4 * (parity ^ 1) + threadIdx.x] = 0; // the next trip's walk appends there
    }
    const u32 stride = gridDim.x * blockDim.x;
    const u32 trips = (total + stride - 1) / stride;
    for (u32 trip = 0; trip < trips; ++trip) {
        const u32 k = trip * stride + blockIdx.x * blockDim.x + threadIdx.x;
        u32 i = k;
        if (parity >= 0 && k < total)
            i = k < n_connect     ? w.queue_connect[parity][k]
                : k < n_medium    ? w.queue_medium[parity][k - n_connect]
                : k < n_interface ? w.queue_interface[parity][k - n_medium]
                                  : w.queue_path[parity][k - n_interface];
        u32 mode = kEventFinished;
        bool finished_now = false;
        if (k < total) {
            const u32 m = w.mode[i];
            mode = m & 0xffu;
            if (mode != kEventFinished) {
                ScalarPath path = w.path[i];
                // a connection in flight is read only by its steps, and a path event that
                // begins one sets it up whole (connection_begin and the event's weights)
                Connection c;
                if (mode == kEventConnect)
                    c = w.conn[i];
                if (s.instance_count == 0) {
                    if (scalar_sky_step(s, p, path))
                        mode = kEventFinished;
                } else if (mode == kEventPath && !scalar_ray_valid(path)) {
                    path.status = S_ARITHMETIC;
                    mode = kEventFinished;
                } else {
                    const Hit hit = w.hit[i];
                    const bool ok = (m & kWalkOk) != 0;
                    mode = mode == kEventPath ? shade_event<Full>(s, p, q, path, ok, hit, c)
                                              : connection_step(s, q, path, c, ok, hit);
                }
                if (mode == kEventFinished) {
                    q.out[path.lane] = scalar_record(path);
                    finished_now = true;
                } else {
                    w.path[i] = path;
                    if (mode == kEventConnect)
                        w.conn[i] = c;
                }
                w.mode[i] = mode;
            }
        }
        // records written this trip
        const u32 done = __ballot_sync(0xffffffffu, finished_now);
        if (lane_in_warp == 0 && done)
            atomicSub(w.remaining, __popc(done));
        // refill (the counter stops growing once the wave's lanes are all taken)
        const u32 want = __ballot_sync(0xffffffffu, k < total && mode == kEventFinished);
        u32 base = p.lanes;
        if (lane_in_warp == 0 && want && *reinterpret_cast<volatile u32 *>(q.next_lane) < p.lanes)
            base = atomicAdd(q.next_lane, __popc(want));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (k < total && mode == kEventFinished) {
            const u32 lane = base + __popc(want & ((1u << lane_in_warp) - 1));
            if (lane < p.lanes) {
                ScalarPath path;
                scalar_start(s, p, q, lane, path);
                w.path[i] = path;
                w.mode[i] = kEventPath;
            }
        }
    }
}

// RenderSample rows for the driver-compatible scalar entry point (src/metal_render.mm:2136-2166).
struct ScalarResult {
    u32 status, pixel, sample_low, sample_high;
    float wavelength, radiance;
    u32 scatterings;
    u32 random_words[4];
};
__global__ void k_scalar_results(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams p,
                                 const uint4 *records, ScalarResult *out) {
    for (u32 lane = blockIdx.x * blockDim.x + threadIdx.x; lane < p.lanes; lane += gridDim.x * blockDim.x) {
        const BeginSample b = begin_sample(s, p, lane);
        const uint4 r = records[lane];
        ScalarResult o;
        o.status = r.x;
        o.pixel = b.pixel;
        o.sample_low = b.sample_low;
        o.sample_high = b.sample_high;
        o.wavelength = __uint_as_float(r.y);
        o.radiance = __uint_as_float(r.z);
        o.scatterings = r.w;
        o.random_words[0] = b.words.x;
        o.random_words[1] = b.words.y;
        o.random_words[2] = b.words.z;
        o.random_words[3] = b.words.w;
        out[lane] = o;
    }
}

// FilmBatch::add for scalar samples (src/render.cpp:2355-2385): PBRT scenes XYZ =
// CIE(round(lambda)) * 470 * L, the demo model wavelength_xyz(lambda) * L; FP64 Neumaier sums
// per pixel in canonical (absolute sample, pixel) order.
// The demo film (wavelength_xyz, src/render.cpp:2131-2145): the CIE table linearly interpolated
// at the wavelength (libstdc++'s std::lerp) times 470 / (the trapezoidal integral of y), and
// the radiance unweighted.
RP_DEV double film_lerp(double a, double b, double t) {
    if ((a <= 0 && b >= 0) || (a >= 0 && b <= 0))
        return __dadd_rn(__dmul_rn(t, b), __dmul_rn(__dadd_rn(1.0, -t), a));
    if (t == 1)
        return b;
    const double x = __dadd_rn(a, __dmul_rn(t, __dadd_rn(b, -a)));
    return (t > 1) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}
__global__ void k_scalar_film(const uint4 *records, u32 pixel_count, u32 samples, const double *cie, FilmPixel *film,
                              u32 *failures, u32 demo, double demo_scale) {
    for (u32 px = blockIdx.x * blockDim.x + threadIdx.x; px < pixel_count; px += gridDim.x * blockDim.x) {
        FilmPixel f = film[px];
        for (u32 si = 0; si < samples; ++si) {
            const uint4 r = records[size_t(si) * pixel_count + px];
            const float w = __uint_as_float(r.y), L = __uint_as_float(r.z);
            if (r.x != 0 || !(w >= 360 && w <= 830) || !isfinite(L) || L < 0) {
                atomicAdd(failures, 1u);
                continue;
            }
            double xyz[3], weighted;
            if (demo) {
                const double offset = __dadd_rn(double(w), -360.0);
                const u32 lower = u32(offset), upper = min(lower + 1u, 470u);
                const double t = __dadd_rn(offset, -double(lower));
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    xyz[c] = __dmul_rn(film_lerp(__ldg(cie + 3 * lower + c), __ldg(cie + 3 * upper + c), t), demo_scale);
                weighted = double(L);
            } else {
                const u32 row = u32(round(double(w)) - 360.0);
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    xyz[c] = __ldg(cie + 3 * row + c);
                weighted = __dmul_rn(470.0, double(L));
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double v = __dmul_rn(xyz[c], weighted);
                add_compensated(v, f.sum[c], f.correction[c]);
                f.square[c] = __dadd_rn(f.square[c], __dmul_rn(v, v));
            }
            add_compensated(1.0, f.weight_sum, f.weight_correction);
            ++f.count;
        }
        film[px] = f;
    }
}

// The frame sensor of a scalar lane (shaders/frame_sensor.h:22-31, PBRT model): the matching
// functions at the nearest nanometre times 470 times radiance, in binary32; a failed lane
// writes zero and counts a failure.
__global__ void k_frame_scalar(const uint4 *records, u32 pixel_count, const double *cie, float *xyz, u32 *failures) {
    for (u32 px = blockIdx.x * blockDim.x + threadIdx.x; px < pixel_count; px += gridDim.x * blockDim.x) {
        const uint4 r = records[px];
        const float w = __uint_as_float(r.y), L = __uint_as_float(r.z);
        bool valid = r.x == 0 && w >= 360 && w <= 830 && isfinite(L) && L >= 0;
        float v[3] = {0, 0, 0};
        if (valid) {
            const u32 row = u32(floorf(w + .5f) - 360.f);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                v[c] = float(__ldg(cie + 3 * row + c)) * L * 470.f;
            valid = isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]);
        }
        if (!valid) {
            v[0] = v[1] = v[2] = 0;
            atomicAdd(failures, 1u);
        }
        xyz[3 * size_t(px)] = v[0];
        xyz[3 * size_t(px) + 1] = v[1];
        xyz[3 * size_t(px) + 2] = v[2];
    }
}

} // namespace rp
