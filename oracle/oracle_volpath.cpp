// ORACLE -- test infrastructure only (see oracle_math.hpp).  The scalar (one-wavelength)
// path tracer with homogeneous media of rypath_render_paths (shaders/render.metal:2299-2371):
// scalar_init, scalar_trace and scalar_shade of shaders/scalar_transport.h run one lane at a
// time, with the medium equations of shaders/medium.h and the light connections of
// shaders/scalar_lighting.h and shaders/render.metal.  Diffuse surfaces and null interfaces.
#include "oracle.h"
#include "oracle_sampling.hpp"

#include <atomic>
#include <memory>
#include <thread>

namespace oracle {

namespace {

constexpr u32 medium_block_limit = 0x20000000u; // src/sampling_contract.h:45-46
constexpr u32 medium_stream = 0x6d656431u;
constexpr float pi_f = 3.14159265358979323846f;

// ---------------------------------------------------------------- shaders/medium.h
// :11-17
float product_ratio(float a, float b, float c, float d) {
    if (a == 0 || b == 0 || c == 0)
        return 0;
    int ea, eb, ec, ed;
    const float ma = std::frexp(a, &ea), mb = std::frexp(b, &eb), mc = std::frexp(c, &ec),
                md = std::frexp(d, &ed);
    return std::ldexp(((ma * mb) * mc) / md, ea + eb + ec - ed);
}
// :19-31
float attenuation_integral_ratio(float x) {
    if (x <= 0.125f) {
        float v = 1.0f / 40320.0f;
        v = std::fma(v, -x, 1.0f / 5040.0f);
        v = std::fma(v, -x, 1.0f / 720.0f);
        v = std::fma(v, -x, 1.0f / 120.0f);
        v = std::fma(v, -x, 1.0f / 24.0f);
        v = std::fma(v, -x, 1.0f / 6.0f);
        v = std::fma(v, -x, 0.5f);
        return std::fma(v, -x, 1.0f);
    }
    return (1.0f - std::exp(-x)) / x;
}
struct Segment {
    float transmission, emission;
    bool valid;
};
// :32-57
Segment segment(float sa, float ss, float le, float distance) {
    if (!std::isfinite(sa) || !std::isfinite(ss) || !std::isfinite(le) || sa < 0 || ss < 0 || le < 0 ||
        std::isnan(distance) || distance < 0)
        return {0, 0, false};
    const float st = sa + ss;
    if (!std::isfinite(st))
        return {0, 0, false};
    if (distance == 0 || st == 0)
        return {1, 0, true};
    const float depth = st * distance;
    const float transmission = std::exp(-depth);
    float emission = 0;
    if (le > 0 && sa > 0) {
        if (depth <= 0.125f) {
            emission = product_ratio(le, sa, distance, 1.0f / attenuation_integral_ratio(depth));
        } else {
            const float loss = std::isinf(depth) ? 1.0f : 1.0f - transmission;
            emission = product_ratio(le, sa, loss, st);
        }
    }
    return {transmission, emission, std::isfinite(emission) && emission >= 0};
}
// :58-76
float flight(float st, float u) {
    if (!std::isfinite(st) || st < 0 || !std::isfinite(u) || u < 0 || u > 1)
        return NAN;
    if (st == 0 || u == 1)
        return INFINITY;
    if (u == 0)
        return 0;
    float depth;
    if (u <= 0.125f) {
        float v = 1.0f / 10.0f;
        for (int n = 9; n >= 2; --n)
            v = std::fma(v, u, 1.0f / float(n));
        depth = u * std::fma(v, u, 1.0f);
    } else {
        depth = -std::log(1.0f - u);
    }
    return depth / st;
}
float clampf(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }
// :77-87
float phase(F3 wo, F3 wi, float g) {
    if (!finite3(wo) || !finite3(wi) || !std::isfinite(g) || std::fabs(dot(wo, wo) - 1.0f) > 2e-5f ||
        std::fabs(dot(wi, wi) - 1.0f) > 2e-5f)
        return NAN;
    g = clampf(g, -0.99f, 0.99f);
    const float cosine = clampf(dot(wo, wi), -1.0f, 1.0f);
    const float base = 1.0f - std::fabs(g);
    const float denominator = std::fma(2.0f * std::fabs(g), 1.0f + (g >= 0 ? cosine : -cosine), base * base);
    return (1.0f / (4.0f * pi_f)) * ((1.0f - g) * (1.0f + g)) / (denominator * std::sqrt(denominator));
}
// :88-112
F3 phase_sample(F3 wo, float g, float ux, float uy) {
    const F3 nan3{NAN, NAN, NAN};
    if (!finite3(wo) || !std::isfinite(g) || !std::isfinite(ux) || !std::isfinite(uy) || ux < 0 || uy < 0 ||
        ux > 1 || uy > 1 || std::fabs(dot(wo, wo) - 1.0f) > 2e-5f)
        return nan3;
    g = clampf(g, -0.99f, 0.99f);
    const float h = std::fabs(g), v = g < 0 ? 1.0f - ux : ux;
    const float d = std::fma(h, 1.0f - 2.0f * v, 1.0f);
    const float ratio = (1.0f - h) / d;
    const float c = clampf(std::fma(2.0f * v * ratio * ratio, std::fma(h, 1.0f - v, 1.0f), -1.0f), -1.0f, 1.0f);
    const float cosine = g < 0 ? -c : c;
    const float sine = std::sqrt(std::fmax(0.0f, (1.0f - cosine) * (1.0f + cosine)));
    F3 x;
    if (!unit(cross(std::fabs(wo.z) < 0.9f ? F3{0, 0, 1} : F3{0, 1, 0}, wo), x))
        return nan3;
    const F3 y = cross(wo, x);
    const float phi = 2.0f * pi_f * uy;
    F3 r;
    if (!unit(cosine * wo + sine * (std::cos(phi) * x + std::sin(phi) * y), r))
        return nan3;
    return r;
}

// ---------------------------------------------------------------- shaders/render.metal helpers
// :1901-1909
float power_weight(float a, float b) {
    const float scale = std::fmax(a, b);
    if (!(scale > 0) || !std::isfinite(scale))
        return NAN;
    a /= scale;
    b /= scale;
    return a * a / (a * a + b * b);
}
// :2212-2219
float scattering_direct(float f_cos, float bsdf_pdf, float light_pdf, bool invisible) {
    if (!(f_cos >= 0) || !(bsdf_pdf >= 0) || !(light_pdf > 0) || !std::isfinite(f_cos) || !std::isfinite(bsdf_pdf) ||
        !std::isfinite(light_pdf))
        return NAN;
    if (f_cos == 0)
        return 0;
    return (f_cos / light_pdf) * (invisible ? 1.0f : power_weight(light_pdf, bsdf_pdf));
}
// :180-198 with src/sampling_contract.h:17-42: Halton dimension 884 + bounce, (Z)Sobol
// dimension 908 + bounce, else Philox block 0x80000000 | bounce
u32 dielectric_lobe_word(const Scene &s, const Params &p, const Sample &smp, u64 index, u32 bounce) {
    if (p.sampler == RP_SAMPLER_HALTON)
        return fbits(qmc_radical(884u + bounce, index, p.randomization, p.seed_low));
    if (p.sampler == RP_SAMPLER_ZSOBOL)
        return zdraw(s, p, index, 908u + bounce);
    if (p.sampler == RP_SAMPLER_SOBOL)
        return sobol_word(*s.sobol, index, 908u + bounce, p.randomization, p.seed_low);
    return philox(U4{smp.pixel, smp.sample_low, smp.sample_high, 0x80000000u | bounce}, p.seed_low, p.seed_high).x;
}
// :843-847
float bsdf_weight(float cosine) {
    const float relative = 4.0f * cosine;
    const float square = relative * relative;
    return square / (1.0f + square);
}
// :828-835
F3 hemisphere(F3 n, float u, float v) {
    const float r = std::sqrt(u);
    const float phi = 2.0f * pi_f * v;
    const F3 axis = std::fabs(n.z) < 0.999f ? F3{0, 0, 1} : F3{0, 1, 0};
    const F3 t = normalize3(cross(axis, n));
    const F3 b = cross(n, t);
    return normalize3((r * std::cos(phi)) * t + (r * std::sin(phi)) * b + std::sqrt(1.0f - u) * n);
}
// :1912-1929
F3 spawn_origin(F3 o, F3 d, float t, const SurfacePoint &pt, F3 n) {
    F3 ray_position, ray_error;
    ray_point(o, d, t, pt.curved, ray_position, ray_error);
    const F3 error = (pt.error + fabs3(pt.position - ray_position)) + ray_error;
    return round_out(pt.position + dot(fabs3(n), error) * n, n);
}
// :1931-1934
F3 spawn_toward(F3 o, F3 d, float t, const SurfacePoint &pt, F3 direction) {
    const F3 ng = pt.geometric_normal;
    return spawn_origin(o, d, t, pt, dot(ng, direction) < 0.0f ? -ng : ng);
}
// :2221-2232
F3 shadow_segment_direction(F3 origin, F3 delta, const SurfacePoint &target, float signed_cosine) {
    const F3 n = signed_cosine > 0.0f ? target.geometric_normal : -target.geometric_normal;
    const float g7 = gamma_bound(7.0f) * target.world_extent;
    const F3 error = (target.error + gamma_bound(2.0f) * (fabs3(origin) + fabs3(delta))) + F3{g7, g7, g7};
    const F3 endpoint = round_out(target.position + dot(fabs3(n), error) * n, n);
    return endpoint - origin;
}
// :659-677
bool point_direction(F3 from, F3 to, F3 &direction, float &distance_squared, bool spot) {
    if (spot)
        for (int i = 0; i < 3; ++i)
            if (!normal_or_zero(from[i]) || !normal_or_zero(to[i]))
                return false;
    const F3 delta = to - from;
    distance_squared = dot(delta, delta);
    if (!(distance_squared >= FLT_MIN) || !std::isfinite(distance_squared))
        return false;
    direction = delta / std::sqrt(distance_squared);
    if (spot)
        for (int i = 0; i < 3; ++i)
            if ((from[i] != to[i] && delta[i] == 0) || (delta[i] != 0 && direction[i] == 0) ||
                !normal_or_zero(direction[i]))
                return false;
    return finite3(direction);
}
// :145-150
u32 outgoing_medium(const Instance &in, u32 current, F3 normal, F3 direction) {
    return in.inside_medium == in.outside_medium ? current
           : dot(normal, direction) > 0          ? in.outside_medium
                                                 : in.inside_medium;
}

// ---------------------------------------------------------------- shaders/scalar_lighting.h
enum : u32 { area_light = 0, positional_light = 1, distant_light = 2, environment_light = 3 };
struct Incident {
    F3 direction{}, endpoint{};
    SurfacePoint target{};
    float radiance = 0, pdf = 0;
    u32 kind = environment_light;
    bool valid = true;
};
// :23-121 (area, point and spot; a constant environment has no light sample)
Incident light_sample_scalar(const Scene &s, float wavelength, F3 position, F3 normal, float selection, float ux,
                             float uy) {
    Incident r;
    const Selected chosen = light_sample(s, position, normal, selection);
    if (!(chosen.pmf > 0))
        return r;
    const u32 id = chosen.light;
    const u32 emitters = u32(s.emitters.size());
    if (id < emitters) {
        r.kind = area_light;
        float conditional = 0, b1 = 0, b2 = 0;
        if (!light_geometry_sample(s, id, position, normal, ux, uy, b1, b2, r.target, conditional)) {
            r.valid = false;
            return r;
        }
        if (!(conditional > 0))
            return r;
        const F3 d = r.target.position - position;
        const float d2 = dot(d, d);
        if (!(d2 > 0))
            return r;
        r.direction = d / std::sqrt(d2);
        r.endpoint = r.target.position;
        r.pdf = chosen.pmf * conditional;
        const Instance &in = s.instances[s.emitters[id].instance];
        const float cosine = dot(r.target.geometric_normal, -r.direction);
        if (cosine == 0 || (!s.emission_two_sided[in.emission] && cosine < 0))
            return r;
        // area_radiance, shaders/render.metal:1811-1819
        r.radiance = r.target.inverse_area_pdf == 0 ? 0.0f : s.emission[in.emission][dense_index(wavelength)];
    } else if (id < emitters + s.positional.size()) {
        r.kind = positional_light;
        const Positional &L = s.positional[id - emitters];
        float intensity = L.intensity[dense_index(wavelength)];
        if (intensity == 0)
            return r;
        r.endpoint = L.position;
        float d2 = 0;
        r.valid = point_direction(position, r.endpoint, r.direction, d2, L.kind != RP_POINT_LIGHT);
        if (!r.valid)
            return r;
        r.valid = positional_intensity(L, r.direction, intensity);
        r.radiance = intensity / d2;
        r.pdf = chosen.pmf;
    } else if (id == s.environment_light) {
        // shaders/scalar_lighting.h:102-113: the environment image's compensated table
        if (s.images.env_image == RP_NONE)
            return r;
        float conditional = 0;
        r.valid = env_image_sample(s.images, ux, uy, true, r.direction, conditional);
        if (!r.valid)
            return r;
        r.pdf = chosen.pmf * conditional;
        r.radiance = env_image_radiance(s.images, r.direction, wavelength);
    } else {
        r.valid = false;
    }
    r.valid = r.valid && std::isfinite(r.radiance) && r.radiance >= 0 && std::isfinite(r.pdf) && r.pdf >= 0;
    return r;
}
// shaders/scalar_lighting.h:14-23 (environment_pdf)
float environment_pdf(const Scene &s, F3 position, F3 normal, F3 direction) {
    if (s.images.env_image == RP_NONE || s.environment_light == RP_NONE)
        return 0.0f;
    return light_pmf(s, position, normal, s.environment_light) * env_image_pdf(s.images, direction, true);
}
// the sky's radiance along a direction: the environment image, else the lane's constant
float sky(const Scene &s, float E, F3 direction, float wavelength) {
    return s.images.env_image != RP_NONE ? env_image_radiance(s.images, direction, wavelength) : E;
}
bool delta_light(const Incident &l) { return l.kind == positional_light || l.kind == distant_light; }

struct Transmission {
    float value;
    u32 status;
};
struct Ctx {
    const Scene &s;
    const Bvh &bvh;
    const Params &p;
    u32 boundary_limit;
};
// shaders/render.metal:1588-1677 (medium_connection)
Transmission medium_connection(const Ctx &c, float wavelength, F3 o, F3 d, float tmax, u32 medium) {
    const Scene &s = c.s;
    const float length = std::sqrt(dot(d, d));
    if (!(length > 0) || !std::isfinite(length))
        return {0, RP_SAMPLE_INVALID_ARITHMETIC};
    F3 direction = d / length;
    float remaining = tmax * length;
    const bool finite_connection = std::isfinite(tmax);
    const F3 endpoint = finite_connection ? fma3(F3{tmax, tmax, tmax}, d, o) : F3{0, 0, 0};
    if (!(remaining > 0) ||
        (finite_connection && (!std::isfinite(remaining) || !finite3(endpoint) ||
                               (endpoint.x == o.x && endpoint.y == o.y && endpoint.z == o.z))))
        return {0, RP_SAMPLE_INVALID_ARITHMETIC};
    float transmission = 1;
    const u32 wi = dense_index(wavelength);
    for (u32 crossings = 0;;) {
        const Hit h = trace_closest(s, c.bvh, o, direction, remaining);
        const bool miss = h.prim == RP_NONE;
        const float distance = miss ? remaining : h.t;
        if (medium != RP_NONE) {
            const Medium &m = s.media[medium];
            const Segment seg = segment(m.sigma_a[wi], m.sigma_s[wi], 0, distance);
            if (!seg.valid)
                return {0, RP_SAMPLE_INVALID_ARITHMETIC};
            transmission *= seg.transmission;
        }
        if (miss || transmission == 0)
            return {transmission, RP_SAMPLE_SUCCESS};
        const u32 inst = s.tri_instance[h.prim];
        const Instance &in = s.instances[inst];
        if (s.materials[in.material].scattering != RP_INTERFACE)
            return {0, RP_SAMPLE_SUCCESS};
        if (crossings++ >= c.boundary_limit)
            return {0, RP_SAMPLE_BOUNDARY_EXHAUSTION};
        SurfacePoint pt;
        if (!hit_surface_point(s, h.prim, inst, s.tri_local[h.prim], h.b1, h.b2, pt))
            return {0, RP_SAMPLE_INVALID_ARITHMETIC};
        F3 next;
        if (!spawn_boundary(o, direction, h.t, pt, direction, next))
            return {0, RP_SAMPLE_INVALID_ARITHMETIC};
        const F3 outgoing_normal = dot(pt.geometric_normal, direction) < 0 ? -pt.geometric_normal : pt.geometric_normal;
        if (finite_connection) {
            const F3 delta = endpoint - next;
            remaining = std::sqrt(dot(delta, delta));
            if (!(remaining > 0) || !std::isfinite(remaining))
                return {0, RP_SAMPLE_INVALID_ARITHMETIC};
            direction = delta / remaining;
            const float facing = dot(outgoing_normal, direction);
            const float facing_error = gamma_bound(5) * dot(fabs3(outgoing_normal), fabs3(direction));
            if (!(facing > facing_error))
                return {0, RP_SAMPLE_INVALID_ARITHMETIC};
        }
        medium = outgoing_medium(in, medium, pt.geometric_normal, direction);
        o = next;
    }
}
// shaders/render.metal:1680-1690 (connection_transmission)
Transmission connection_transmission(const Ctx &c, float wavelength, F3 o, F3 d, float tmax, u32 medium) {
    if (c.s.media_enabled)
        return medium_connection(c, wavelength, o, d, tmax, medium);
    const bool occluded = trace_any(c.s, c.bvh, o, d, tmax);
    return {occluded ? 0.0f : 1.0f, RP_SAMPLE_SUCCESS};
}
// shaders/scalar_lighting.h:123-134 (connection)
F3 connection_direction(const Incident &light, F3 origin) {
    if (light.kind == environment_light)
        return light.direction;
    if (light.kind == area_light) {
        const F3 delta = light.target.position - origin;
        return shadow_segment_direction(origin, delta, light.target, dot(light.target.geometric_normal, -delta));
    }
    return light.endpoint - origin;
}

// ---------------------------------------------------------------- scalar lane
struct Lane {
    Sample sample;
    u64 index = 0;
    float wavelength = 0, radiance = 0;
    u32 scatterings = 0;
    F3 o{}, d{};
    float throughput = 1, escape_weight = 1, previous_bsdf_pdf = 0;
    bool previous_delta = false;
    F3 prev_p{}, prev_n{};
    float E = 0;
    u32 current_medium = RP_NONE, medium_draw = 0, boundary_crossings = 0;
};
U4 medium_words(const Params &p, const Lane &l, u32 &draw) {
    return philox(U4{l.sample.pixel, l.sample.sample_low, l.sample.sample_high, medium_block_limit | draw++},
                  p.seed_low, p.seed_high ^ medium_stream);
}
// shaders/scalar_transport.h:64-77 (scalar_init)
Lane scalar_init(const Scene &s, const Params &p, u32 lane) {
    Lane l;
    l.sample = begin_sample(s, p, lane, l.index);
    l.wavelength = 360.0f + 470.0f * sample_uniform(p, l.sample.words[2]);
    primary_ray(s, p, l.sample, l.o, l.d);
    l.prev_p = l.o;
    // sky_radiance (shaders/render.metal:813-819): the demo sky is unit equal-energy
    l.E = s.model == RP_MODEL_DEMO ? 1.0f : s.environment[dense_index(l.wavelength)];
    l.current_medium = s.camera_medium;
    return l;
}

// shaders/scalar_transport.h:88-210 (scalar_sky_step); true when the lane finished
bool sky_step(const Ctx &c, Lane &l) {
    const Scene &s = c.s;
    if (!finite3(l.o) || !finite3(l.d)) {
        l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return true;
    }
    if (s.camera_medium != RP_NONE) {
        const Medium &m = s.media[s.camera_medium];
        const u32 wi = dense_index(l.wavelength);
        const float a = m.sigma_a[wi], sc = m.sigma_s[wi], total = a + sc;
        if (total > 0) {
            const Segment seg = segment(a, sc, m.emission[wi], INFINITY);
            if (!seg.valid) {
                l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
                return true;
            }
            if (l.scatterings < s.max_depth)
                l.radiance += l.throughput * seg.emission;
            if (l.scatterings >= s.max_depth || sc == 0)
                return true;
            if (l.scatterings >= c.p.emergency_limit) {
                l.sample.status = RP_SAMPLE_EMERGENCY_DEPTH;
                return true;
            }
            const U4 flight_words = medium_words(c.p, l, l.medium_draw);
            const float distance = flight(total, u01(flight_words.x));
            const F3 point = fma3(F3{distance, distance, distance}, l.d, l.o);
            if (!std::isfinite(distance) || !finite3(point)) {
                l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
                return true;
            }
            l.throughput *= sc / total;
            const Selected chosen = light_sample(s, point, F3{0, 0, 0}, u01(flight_words.y));
            if (chosen.pmf > 0) {
                F3 direction{0, 0, 0};
                float radiance = 0, distance_to_light = 0;
                const u32 emitters = u32(s.emitters.size());
                if (chosen.light >= emitters && chosen.light < emitters + s.positional.size()) {
                    const Positional &L = s.positional[chosen.light - emitters];
                    float d2 = 0, intensity = L.intensity[wi];
                    if (intensity != 0) {
                        if (!point_direction(point, L.position, direction, d2, L.kind != RP_POINT_LIGHT) ||
                            !positional_intensity(L, direction, intensity)) {
                            l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
                            return true;
                        }
                        radiance = intensity / d2;
                        distance_to_light = std::sqrt(d2);
                    }
                }
                if (radiance > 0) {
                    const float tr = std::exp(-total * distance_to_light);
                    l.radiance += l.throughput * phase(-l.d, direction, m.g) * (radiance / chosen.pmf) * tr;
                }
                if (!std::isfinite(l.radiance) || l.radiance < 0) {
                    l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
                    return true;
                }
            }
            const U4 phase_words = medium_words(c.p, l, l.medium_draw);
            const F3 wi_dir = phase_sample(-l.d, m.g, u01(phase_words.x), u01(phase_words.y));
            ++l.scatterings;
            if (l.scatterings >= 3) {
                if (phase_words.z >= 0xc0000000u)
                    return true;
                l.throughput /= .75f;
            }
            if (!finite3(wi_dir) || !std::isfinite(l.throughput)) {
                l.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
                return true;
            }
            l.o = point;
            l.d = wi_dir;
            return false;
        }
    }
    l.radiance = sky(s, l.E, l.d, l.wavelength);
    return true;
}

// one scalar_trace + scalar_shade (shaders/scalar_transport.h:213-900); true when finished
bool scalar_event(const Ctx &c, Lane &l) {
    const Scene &s = c.s;
    const Params &p = c.p;
    if (s.instances.empty())
        return sky_step(c, l);
    auto fail = [&](u32 status) {
        l.sample.status = status;
        return true;
    };
    if (!finite3(l.o) || !finite3(l.d) || !std::isfinite(l.throughput) || !std::isfinite(l.radiance))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    const Hit hit = trace_closest(s, c.bvh, l.o, l.d, INFINITY);
    const bool miss = hit.prim == RP_NONE;
    // medium interaction, shaders/scalar_transport.h:354-420
    if (l.current_medium != RP_NONE) {
        if (l.current_medium >= s.media.size())
            return fail(RP_SAMPLE_INVALID_HIT);
        if (l.medium_draw >= medium_block_limit - 3)
            return fail(RP_SAMPLE_BOUNDARY_EXHAUSTION);
        const Medium &m = s.media[l.current_medium];
        const u32 wi = dense_index(l.wavelength);
        const float a = m.sigma_a[wi], sc = m.sigma_s[wi], total = a + sc;
        const float ray_length = std::sqrt(dot(l.d, l.d));
        const float distance = miss ? INFINITY : hit.t * ray_length;
        const Segment seg = segment(a, sc, l.scatterings < s.max_depth ? m.emission[wi] : 0.0f, distance);
        if (!seg.valid || !(ray_length > 0) || !std::isfinite(ray_length))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        l.radiance += l.throughput * seg.emission;
        if (total > 0) {
            const U4 flight_words = medium_words(p, l, l.medium_draw);
            const float f = flight(total, u01(flight_words.x));
            if (f < distance || std::isinf(distance)) {
                if (!std::isfinite(f))
                    return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                if (l.scatterings >= s.max_depth || sc == 0)
                    return true;
                if (l.scatterings >= p.emergency_limit)
                    return fail(RP_SAMPLE_EMERGENCY_DEPTH);
                const F3 direction = l.d / ray_length;
                const F3 position = fma3(F3{f, f, f}, direction, l.o);
                if (!finite3(position))
                    return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                l.throughput *= sc / total;
                const U4 light_words = medium_words(p, l, l.medium_draw);
                const U4 phase_words = medium_words(p, l, l.medium_draw);
                // medium_direct, shaders/render.metal:2237-2260
                {
                    const Incident light = light_sample_scalar(s, l.wavelength, position, F3{0, 0, 0},
                                                               u01(light_words.x), u01(light_words.y),
                                                               u01(light_words.z));
                    if (!light.valid)
                        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                    if (light.pdf > 0 && light.radiance != 0) {
                        const Transmission tr = medium_connection(c, l.wavelength, position,
                                                                  connection_direction(light, position),
                                                                  light.kind == environment_light ? INFINITY : 0x1.fffffep-1f,
                                                                  l.current_medium);
                        if (tr.status != RP_SAMPLE_SUCCESS)
                            return fail(tr.status);
                        const float ph = phase(-direction, light.direction, m.g);
                        const float weight = delta_light(light) ? 1.f : power_weight(light.pdf, ph);
                        const float value = (ph / light.pdf) * weight * light.radiance * tr.value;
                        if (!std::isfinite(value) || !(value >= 0))
                            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                        l.radiance += l.throughput * value;
                    }
                }
                const F3 wi_dir = phase_sample(-direction, m.g, u01(phase_words.x), u01(phase_words.y));
                l.previous_bsdf_pdf = phase(-direction, wi_dir, m.g);
                if (!finite3(wi_dir) || !(l.previous_bsdf_pdf > 0) || !std::isfinite(l.previous_bsdf_pdf))
                    return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                ++l.scatterings;
                if (l.scatterings >= 3) {
                    if (phase_words.z >= 0xc0000000u)
                        return true;
                    l.throughput /= .75f;
                }
                l.previous_delta = false;
                l.prev_p = position;
                l.prev_n = F3{0, 0, 0};
                l.escape_weight = 1;
                l.o = position;
                l.d = wi_dir;
                l.boundary_crossings = 0;
                return false;
            }
        }
    }
    if (miss) {
        // shaders/scalar_transport.h:421-433; MIS against the environment image's light samples
        if (s.model == RP_MODEL_PBRT && l.scatterings != 0u && !l.previous_delta)
            l.escape_weight = power_weight(l.previous_bsdf_pdf, environment_pdf(s, l.prev_p, l.prev_n, l.d));
        l.radiance += l.throughput * l.escape_weight * sky(s, l.E, l.d, l.wavelength);
        return true;
    }
    const u32 bounce = l.scatterings;
    const u32 inst = s.tri_instance[hit.prim], local = s.tri_local[hit.prim];
    const Instance &instance = s.instances[inst];
    if (!std::isfinite(hit.t) || !std::isfinite(hit.b1) || !std::isfinite(hit.b2))
        return fail(RP_SAMPLE_INVALID_HIT);
    const Material &material = s.materials[instance.material];
    SurfacePoint point;
    if (material.scattering == RP_INTERFACE) {
        // shaders/scalar_transport.h:450-472
        if (l.boundary_crossings++ >= c.boundary_limit)
            return fail(RP_SAMPLE_BOUNDARY_EXHAUSTION);
        if (!hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, point))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        l.current_medium = outgoing_medium(instance, l.current_medium, point.geometric_normal, l.d);
        F3 origin;
        if (!spawn_boundary(l.o, l.d, hit.t, point, l.d, origin))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        l.o = origin;
        return false;
    }
    const bool emissive = instance.emission != RP_NONE;
    if (emissive) {
        // shaders/scalar_transport.h:473-520
        if (!hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, point))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        const float Le = point.inverse_area_pdf == 0 ? 0.0f : s.emission[instance.emission][dense_index(l.wavelength)];
        if (Le > 0.0f && (s.emission_two_sided[instance.emission] || dot(point.geometric_normal, -l.d) >= 0.0f)) {
            float weight = 1.0f;
            if (bounce != 0u && !l.previous_delta) {
                const u32 light_id = instance.emitter_begin + local;
                const float pdf = light_pmf(s, l.prev_p, l.prev_n, light_id) *
                                  light_geometry_pdf(s, light_id, l.prev_p, l.prev_n, point);
                weight = power_weight(l.previous_bsdf_pdf, pdf);
            }
            if (!std::isfinite(weight))
                return fail(RP_SAMPLE_INVALID_ARITHMETIC);
            l.radiance += l.throughput * (weight * Le);
        }
    }
    if (bounce >= s.max_depth)
        return true;
    // mix materials resolve at the hit's point (shaders/scalar_transport.h:541-587)
    bool point_ready = emissive;
    u32 material_index = instance.material;
    if (material.scattering == 9) {
        if (!emissive && !hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, point))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        point_ready = true;
        if (const u32 mix_status = resolve_mix(s, point.position, -l.d, material_index))
            return fail(mix_status);
    }
    const Material &surface = s.materials[material_index];
    // reflectance, shaders/scalar_transport.h:580-625; conductors and dielectrics carry their
    // spectrum in the BSDF (rho = 1)
    const bool microfacet = surface.scattering != RP_DIFFUSE;
    float rho = 0;
    if (microfacet) {
        if (surface.scattering != RP_CONDUCTOR && surface.scattering != RP_DIELECTRIC)
            return fail(RP_SAMPLE_INVALID_HIT);
        rho = 1.0f;
    } else if (s.model == RP_MODEL_DEMO) {
        // demo_reflectance (shaders/render.metal:537-546)
        if (surface.kind != RP_REFLECTANCE_KNOTS)
            return fail(RP_SAMPLE_INVALID_HIT);
        static const float knots[8] = {360, 420, 470, 520, 570, 620, 700, 830};
        rho = surface.reflectance[7];
        for (int i = 1; i < 8; ++i)
            if (l.wavelength <= knots[i]) {
                const float t = (l.wavelength - knots[i - 1]) / (knots[i] - knots[i - 1]);
                rho = surface.reflectance[i - 1] + (surface.reflectance[i] - surface.reflectance[i - 1]) * t;
                break;
            }
    } else if (surface.kind == RP_REFLECTANCE_KNOTS && surface.knot_count >= 2 && surface.knot_begin <= s.knots.size() &&
               surface.knot_count <= s.knots.size() - surface.knot_begin) {
        rho = pbrt_reflectance(s.knots.data() + surface.knot_begin, surface.knot_count, l.wavelength);
    } else if (surface.kind == RP_REFLECTANCE_CONSTANT) {
        rho = surface.scalar_value;
    } else if (surface.kind == RP_REFLECTANCE_BLACKBODY) {
        rho = blackbody_reflectance(surface.scalar_value, l.wavelength);
    } else if (surface.kind == RP_REFLECTANCE_RGB) {
        reflectance(s, surface, l.wavelength, nullptr, rho); // sigmoid_reflectance; range checked below
    } else if (surface.kind == RP_REFLECTANCE_IMAGE && surface.image_texture < s.images.textures.size()) {
        // image_reflectance (shaders/render.metal:1154-1240) at the hit's footprint
        if (!point_ready && !hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, point))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        point_ready = true;
        F2 uvst, dstdx, dstdy;
        if (!texture_context(s, c.p, l.sample, inst, local, hit.b1, hit.b2, point.geometric_normal, l.d, l.scatterings,
                             uvst, dstdx, dstdy))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        const rp_image_texture &t = s.images.textures[surface.image_texture];
        Rgb rgb = image_lookup(s.images, t, uvst, dstdx, dstdy, false, false);
        rgb = {rgb.r * t.scale, rgb.g * t.scale, rgb.b * t.scale};
        if (t.invert)
            rgb = {1 - rgb.r, 1 - rgb.g, 1 - rgb.b};
        rho = srgb_spectrum(s.images.rgb_table.data(), rgb, l.wavelength);
    } else {
        return fail(RP_SAMPLE_INVALID_HIT);
    }
    if (!std::isfinite(rho) || !(rho >= 0.0f && rho <= 1.0f))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    if (rho == 0.0f)
        return true;
    const bool authored_normals = instance.normal_begin != RP_NONE || microfacet;
    if (!authored_normals && bounce >= p.emergency_limit)
        return fail(RP_SAMPLE_EMERGENCY_DEPTH);
    if (!point_ready && !hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, point))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    const float incident_cosine = dot(point.shading_normal, l.d);
    if (authored_normals && !microfacet && incident_cosine == 0.0f)
        return true;
    if (bounce >= p.emergency_limit)
        return fail(RP_SAMPLE_EMERGENCY_DEPTH);
    const F3 n = incident_cosine > 0.0f ? -point.shading_normal : point.shading_normal;
    // the BSDF in the shading frame of the normal (shaders/scalar_transport.h:677-694;
    // prepare_scattering, shaders/render.metal:2079-2160)
    LaneBsdf bsdf{};
    Frame frame{};
    F3 wo{0, 0, 0};
    if (microfacet) {
        const u32 total = u32(s.knots.size());
        const float eta = optical_value(s.knots.data(), surface.eta_begin, surface.eta_count, total,
                                        (surface.optical_extensions & 1u) != 0, l.wavelength);
        const float kk = optical_value(s.knots.data(), surface.k_begin, surface.k_count, total,
                                       (surface.optical_extensions & 2u) != 0, l.wavelength);
        bsdf.kind = surface.scattering;
        const bool prepared =
            surface.scattering == RP_CONDUCTOR
                ? conductor_prepare(eta, kk, surface.u_roughness, surface.v_roughness, surface.remap != 0, bsdf.conductor)
                : dielectric_prepare(eta, surface.u_roughness, surface.v_roughness, surface.remap != 0, bsdf.dielectric);
        F3 dpdu, dpdv;
        coordinate_system(point.shading_normal, dpdu, dpdv);
        if (!prepared || !scattering_frame(point.shading_normal, dpdu, frame))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        wo = frame.local(-l.d);
        if (wo.z == 0)
            return true;
    }
    const bool dirac = microfacet && delta_only(bsdf);
    const bool both_hemispheres = microfacet && bsdf.kind == RP_DIELECTRIC;
    const F3 context_normal = microfacet ? frame.z : point.shading_normal;
    const bool directional_offset = authored_normals;
    const F3 area_reference = directional_offset ? point.position : spawn_origin(l.o, l.d, hit.t, point, n);
    if (!finite3(area_reference))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    const U4 light_words = draw_words(s, p, l.sample, l.index, 2 + 2 * bounce);
    const U4 bsdf_words = draw_words(s, p, l.sample, l.index, 1 + 2 * bounce);
    // light sample: the demo sky, uniform on the sphere with the cosine-ratio weight
    // (shaders/scalar_transport.h:709-781); PBRT lights, :783-835; none at Dirac surfaces
    if (s.model == RP_MODEL_DEMO) {
        const float E = l.E;
        const float uz = sample_uniform(p, light_words.x), uv = sample_uniform(p, light_words.y);
        // sphere (shaders/render.metal:821-826)
        const float z = 1.0f - 2.0f * uz;
        const float r = std::sqrt(std::max(0.0f, 1.0f - z * z));
        const float phi = 2.0f * pi_f * uv;
        const F3 direction{r * std::cos(phi), r * std::sin(phi), z};
        const F3 local_light = microfacet ? frame.local(direction) : F3{0, 0, 0};
        const float cosine = both_hemispheres ? std::fabs(local_light.z)
                             : microfacet     ? (wo.z > 0 ? local_light.z : -local_light.z)
                                              : dot(n, direction);
        if (!dirac && E > 0.0f && cosine > 0.0f) {
            const F3 origin = directional_offset ? spawn_toward(l.o, l.d, hit.t, point, direction) : area_reference;
            if (!finite3(origin))
                return fail(RP_SAMPLE_INVALID_ARITHMETIC);
            const Transmission vis = connection_transmission(
                c, l.wavelength, origin, direction, INFINITY,
                outgoing_medium(instance, l.current_medium, point.geometric_normal, direction));
            if (vis.status != RP_SAMPLE_SUCCESS)
                return fail(vis.status);
            if (vis.value > 0) {
                float factor;
                if (microfacet) {
                    const Eval e = scalar_evaluate(bsdf, wo, local_light);
                    factor = e.valid ? scattering_direct(e.f * cosine, e.pdf, 1.0f / (4.0f * pi_f), false) : NAN;
                } else {
                    // (4 cos) * light_weight(cos) (shaders/render.metal:838-841)
                    const float relative = 4.0f * cosine;
                    factor = relative * (1.0f / (1.0f + relative * relative));
                }
                if (!std::isfinite(factor))
                    return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                l.radiance += l.throughput * rho * factor * E * vis.value;
            }
        }
    } else if (!dirac) {
        const Incident light = light_sample_scalar(s, l.wavelength, point.position, context_normal,
                                                   sample_uniform(p, light_words.x), sample_uniform(p, light_words.y),
                                                   sample_uniform(p, light_words.z));
        if (!light.valid)
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        if (light.pdf > 0 && light.radiance > 0) {
            const F3 local_light = microfacet ? frame.local(light.direction) : F3{0, 0, 0};
            const float cosine = both_hemispheres ? std::fabs(local_light.z)
                                 : microfacet     ? (wo.z > 0 ? local_light.z : -local_light.z)
                                                  : dot(n, light.direction);
            if (cosine > 0) {
                float f_cos = rho * cosine / pi_f;
                float bsdf_pdf = cosine / pi_f;
                if (microfacet) {
                    const Eval e = scalar_evaluate(bsdf, wo, local_light);
                    if (!e.valid)
                        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                    f_cos = e.f * cosine;
                    bsdf_pdf = e.pdf;
                }
                const float factor = scattering_direct(f_cos, bsdf_pdf, light.pdf, delta_light(light));
                const F3 origin =
                    directional_offset ? spawn_toward(l.o, l.d, hit.t, point, light.direction) : area_reference;
                const F3 cd = connection_direction(light, origin);
                if (!std::isfinite(factor) || !finite3(cd) || !(dot(cd, light.direction) > 0))
                    return fail(RP_SAMPLE_INVALID_ARITHMETIC);
                const Transmission vis = connection_transmission(
                    c, l.wavelength, origin, cd, light.kind == environment_light ? INFINITY : 0x1.fffffep-1f,
                    outgoing_medium(instance, l.current_medium, point.geometric_normal, light.direction));
                if (vis.status != RP_SAMPLE_SUCCESS)
                    return fail(vis.status);
                l.radiance += l.throughput * factor * light.radiance * vis.value;
            }
        }
    }
    // continuation, shaders/scalar_transport.h:837-900; a microfacet sample is resolved in world
    // space by resolve_scattering_continuation (shaders/render.metal:2006-2019)
    F3 wi{0, 0, 0};
    float continuation_pdf = 0, continuation_cosine = 0;
    bool continuation_delta = false;
    if (microfacet) {
        const float lobe = bsdf.kind == RP_DIELECTRIC
                               ? sample_uniform(p, dielectric_lobe_word(s, p, l.sample, l.index, bounce))
                               : 0.0f; // the conductor draws no lobe
        float sampled_eta;
        BSample sampled = scalar_sample(bsdf, wo, lobe, sample_uniform(p, bsdf_words.x),
                                        sample_uniform(p, bsdf_words.y), sampled_eta);
        if (sampled.valid && sampled.accepted && !unit_vector(frame.world(sampled.wi), wi))
            sampled.valid = false;
        if (!sampled.valid)
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
        if (!sampled.accepted)
            return true;
        l.throughput *= sampled.weight;
        continuation_pdf = sampled.pdf;
        continuation_cosine = std::fabs(sampled.wi.z);
        continuation_delta = sampled.delta;
    } else {
        wi = hemisphere(n, sample_uniform(p, bsdf_words.x), sample_uniform(p, bsdf_words.y));
        l.throughput *= rho;
    }
    if (!std::isfinite(l.throughput) || l.throughput < 0.0f)
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    ++l.scatterings;
    if (l.scatterings >= 3) {
        if (decision_word(p, bsdf_words.z) >= 0xc0000000u)
            return true;
        l.throughput /= 0.75f;
        if (!std::isfinite(l.throughput))
            return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    }
    const float cosine = microfacet ? continuation_cosine : dot(n, wi);
    if (!(cosine > 0.0f))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    l.previous_bsdf_pdf = microfacet ? continuation_pdf : cosine / pi_f;
    l.previous_delta = continuation_delta;
    l.prev_p = point.position;
    l.prev_n = context_normal;
    l.escape_weight = continuation_delta ? 1.0f
                      : microfacet       ? power_weight(l.previous_bsdf_pdf, 1.0f / (4.0f * pi_f))
                                         : bsdf_weight(cosine);
    const F3 origin = directional_offset ? spawn_toward(l.o, l.d, hit.t, point, wi) : area_reference;
    if (!finite3(origin))
        return fail(RP_SAMPLE_INVALID_ARITHMETIC);
    l.o = origin;
    l.d = wi;
    l.current_medium = outgoing_medium(instance, l.current_medium, point.geometric_normal, wi);
    l.boundary_crossings = 0;
    return false;
}

rp_scalar_result render_scalar_lane(const Ctx &c, u32 lane) {
    Lane l = scalar_init(c.s, c.p, lane);
    while (!scalar_event(c, l)) {
    }
    rp_scalar_result r{};
    r.status = l.sample.status;
    // scalar_finish, shaders/scalar_transport.h:79-84
    if (r.status == RP_SAMPLE_SUCCESS && (!std::isfinite(l.radiance) || l.radiance < 0.0f))
        r.status = RP_SAMPLE_INVALID_ARITHMETIC;
    r.pixel = l.sample.pixel;
    r.sample_low = l.sample.sample_low;
    r.sample_high = l.sample.sample_high;
    r.wavelength = l.wavelength;
    r.radiance = l.radiance;
    r.scatterings = l.scatterings;
    for (int k = 0; k < 4; ++k)
        r.random_words[k] = l.sample.words[k];
    return r;
}

} // namespace

} // namespace oracle

using namespace oracle;


extern "C" {

int or_sample_scalar(const or_scene *scene, const rp_request *request, rp_scalar_result *results, size_t capacity,
                     int threads) {
    const u64 lanes = u64(request->pixel_count) * request->sample_count;
    if (lanes > capacity || request->pixel_count == 0 || scene->scene.transport != RP_TRANSPORT_SCALAR)
        return -1;
    const Params p = make_params(scene->scene, *request);
    const Ctx c{scene->scene, scene->bvh, p, request->boundary_limit ? request->boundary_limit : 4096u};
    unsigned n = threads > 0 ? unsigned(threads) : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<u64> next{0};
    auto work = [&]() {
        for (;;) {
            const u64 begin = next.fetch_add(64);
            if (begin >= lanes)
                return;
            const u64 end = std::min(lanes, begin + 64);
            for (u64 i = begin; i < end; ++i)
                results[i] = render_scalar_lane(c, u32(i));
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < n; ++t)
        pool.emplace_back(work);
    work();
    for (auto &t : pool)
        t.join();
    for (u64 i = 0; i < lanes; ++i)
        if (results[i].status != RP_SAMPLE_SUCCESS)
            return 1;
    return 0;
}

// shaders/medium.h probes: each query is (sigma_a, sigma_s, Le, distance, sigma_t, u,
// wo.xyz, wi.xyz, g, ux, uy); each result is (transmission, emission, valid, flight, phase,
// sampled direction xyz).
void or_probe_medium(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 15 * i;
        float *o = r + 8 * i;
        const Segment seg = segment(a[0], a[1], a[2], a[3]);
        o[0] = seg.transmission;
        o[1] = seg.emission;
        o[2] = seg.valid ? 1.0f : 0.0f;
        o[3] = flight(a[4], a[5]);
        o[4] = phase(F3{a[6], a[7], a[8]}, F3{a[9], a[10], a[11]}, a[12]);
        const F3 w = phase_sample(F3{a[6], a[7], a[8]}, a[12], a[13], a[14]);
        o[5] = w.x;
        o[6] = w.y;
        o[7] = w.z;
    }
}

// FilmBatch::add for scalar samples (src/render.cpp:2355-2385) followed by the per-pixel
// second moments; film rows are rp_film_pixel.  Returns 0, or 1 on an invalid sample.
int or_scalar_film_add(const rp_scalar_result *results, size_t count, const double *cie_xyz, uint32_t pixel_count,
                       rp_film_pixel *film, int demo) {
    // the demo film's scale (wavelength_xyz, src/render.cpp:2131-2145; integrate_y, :70-77)
    double integral = (cie_xyz[1] + cie_xyz[3 * 470 + 1]) / 2;
    for (int i = 1; i + 1 < 471; ++i)
        integral += cie_xyz[3 * i + 1];
    const double scale = 470.0 / integral;
    for (size_t i = 0; i < count; ++i) {
        const rp_scalar_result &r = results[i];
        if (r.pixel >= pixel_count || r.status != RP_SAMPLE_SUCCESS || !(r.wavelength >= 360 && r.wavelength <= 830) ||
            !std::isfinite(r.radiance) || r.radiance < 0)
            return 1;
        rp_film_pixel &f = film[r.pixel];
        double xyz[3], weighted;
        if (demo) {
            const double offset = double(r.wavelength) - 360.0;
            const size_t lower = size_t(offset), upper = std::min<size_t>(lower + 1, 470);
            for (int c = 0; c < 3; ++c)
                xyz[c] = std::lerp(cie_xyz[3 * lower + c], cie_xyz[3 * upper + c], offset - double(lower)) * scale;
            weighted = double(r.radiance);
        } else {
            const size_t row = size_t(std::round(double(r.wavelength)) - 360.0);
            for (int c = 0; c < 3; ++c)
                xyz[c] = cie_xyz[3 * row + c];
            weighted = 470.0 * double(r.radiance);
        }
        for (int c = 0; c < 3; ++c) {
            const double v = xyz[c] * weighted;
            const double next = f.sum[c] + v;
            f.correction[c] += std::fabs(f.sum[c]) >= std::fabs(v) ? (f.sum[c] - next) + v : (v - next) + f.sum[c];
            f.sum[c] = next;
            f.square[c] += v * v;
        }
        const double next = f.weight_sum + 1.0;
        f.weight_correction +=
            std::fabs(f.weight_sum) >= 1.0 ? (f.weight_sum - next) + 1.0 : (1.0 - next) + f.weight_sum;
        f.weight_sum = next;
        ++f.count;
    }
    return 0;
}

} // extern "C"
