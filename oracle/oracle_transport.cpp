// ORACLE -- test infrastructure only (see oracle_math.hpp).  The hero-wavelength path
// tracer of rypath_render_packets (shaders/render.metal:2424-2469), one lane at a time.
#include "oracle.h"
#include "oracle_scene.hpp"
#include "oracle_sampling.hpp"

#include <atomic>
#include <cstdio>
#include <memory>
#include <thread>

namespace oracle {

// ---------------------------------------------------------------- vertices
enum : u32 { camera_vertex = 0, surface_vertex = 1, light_vertex = 2, environment_vertex = 3 };
struct Vertex {
    u32 type = camera_vertex;
    SurfacePoint point;
    Frame frame{};
    HeroBsdf bsdf{};
    F4 beta;
    F3 wo;
    float u = 0, v = 0;
    u32 instance = RP_NONE, primitive = 0, light = RP_NONE;
    u32 material = RP_NONE; // the resolved material of a surface vertex
    bool pair_valid = false, delta = false, connectible = false, delta_light = false;
    F3 sampled_wo_local, sampled_wi_local;
};
inline bool infinite(const Vertex &v) { return v.type == environment_vertex; }
inline bool on_surface(const Vertex &v) { return any_nonzero3(v.point.geometric_normal); }

// shaders/packet_transport.h:77-83
static F3 offset(const Vertex &v, F3 direction) {
    if (!on_surface(v))
        return v.point.position;
    const F3 n = dot(direction, v.point.geometric_normal) < 0 ? -v.point.geometric_normal
                                                              : v.point.geometric_normal;
    return round_out(v.point.position + dot(fabs3(n), v.point.error) * n, n);
}

// shaders/packet_walk.h:22-57 (packet_reflectance) for sampled/constant/blackbody/image; image:
// the hit's filtered, scaled linear RGB
bool reflectance(const Scene &s, const Material &m, float w, const Rgb *image, float &rho) {
    if (m.scattering != 0) {
        rho = 1;
    } else if (m.kind == RP_REFLECTANCE_IMAGE && image && m.image_texture < s.images.textures.size()) {
        rho = srgb_spectrum(s.images.rgb_table.data(), *image, w);
    } else if (m.kind == RP_REFLECTANCE_KNOTS && m.knot_count >= 2 &&
               m.knot_begin <= s.knots.size() && m.knot_count <= s.knots.size() - m.knot_begin) {
        rho = pbrt_reflectance(s.knots.data() + m.knot_begin, m.knot_count, w);
    } else if (m.kind == RP_REFLECTANCE_CONSTANT) {
        rho = m.scalar_value;
    } else if (m.kind == RP_REFLECTANCE_BLACKBODY) {
        rho = blackbody_reflectance(m.scalar_value, w);
    } else if (m.kind == RP_REFLECTANCE_RGB) {
        // shaders/render.metal:576-588 (sigmoid_reflectance)
        const float q = std::fma(std::fma(m.coefficients[0], w, m.coefficients[1]), w, m.coefficients[2]);
        if (!std::isfinite(q)) {
            rho = NAN;
        } else if (std::fabs(q) <= 1.0f) {
            rho = 0.5f + 0.5f * (q / std::sqrt(1.0f + q * q));
        } else {
            const float inverse = 1.0f / q;
            rho = 0.5f + 0.5f * std::copysign(1.0f / std::sqrt(1.0f + inverse * inverse), q);
        }
    } else
        return false;
    return std::isfinite(rho) && rho >= 0 && rho <= 1;
}
// shaders/hero_current_bsdf.h:72-101 with prepare_scattering (shaders/render.metal:2079-2160)
static bool prepare_bsdf(const Scene &s, const Material &m, const Wavelengths &l, u32 mask,
                         HeroBsdf &out, const Rgb *image = nullptr) {
    out = HeroBsdf{};
    out.active_mask = mask;
    for (int k = 0; k < 4; ++k) {
        LaneBsdf lane{};
        lane.kind = m.scattering;
        if (!(mask & (1u << k))) {
            out.lane[k] = lane;
            continue;
        }
        float rho;
        if (!reflectance(s, m, l.lambda[k], image, rho))
            return false;
        if (m.scattering == 0) {
            lane.reflectance = rho;
        } else {
            const u32 total = u32(s.knots.size());
            const float eta = optical_value(s.knots.data(), m.eta_begin, m.eta_count, total,
                                            (m.optical_extensions & 1u) != 0, l.lambda[k]);
            const float kk = optical_value(s.knots.data(), m.k_begin, m.k_count, total,
                                           (m.optical_extensions & 2u) != 0, l.lambda[k]);
            if (m.scattering == 1) {
                if (!conductor_prepare(eta, kk, m.u_roughness, m.v_roughness, m.remap != 0, lane.conductor))
                    return false;
            } else if (m.scattering == 2) {
                if (!dielectric_prepare(eta, m.u_roughness, m.v_roughness, m.remap != 0, lane.dielectric))
                    return false;
            } else
                return false;
        }
        out.lane[k] = lane;
    }
    // hero_current_structure (shaders/hero_current_bsdf.h:9-14)
    return (mask & 1u) && !(mask & ~15u) && m.scattering <= 2;
}

// ---------------------------------------------------------------- emission
// shaders/render.metal:1811-1830 (area_radiance, plain spectrum)
static bool emitted(const Scene &s, const Vertex &v, F3 direction, const Wavelengths &l, F4 &rad) {
    if (infinite(v)) {
        // shaders/packet_transport.h:92-101: the environment image when there is one
        for (int k = 0; k < 4; ++k)
            rad[k] = s.images.env_image != RP_NONE ? env_image_radiance(s.images, direction, l.lambda[k])
                                                   : s.environment[dense_index(l.lambda[k])];
        return finite_nonnegative4(rad);
    }
    rad = f4(0);
    if (v.instance >= s.instances.size())
        return true;
    const Instance &in = s.instances[v.instance];
    if (in.emission == RP_NONE)
        return true;
    if (!s.emission_two_sided[in.emission] && dot(v.point.geometric_normal, direction) <= 0)
        return true;
    for (int k = 0; k < 4; ++k)
        rad[k] = v.point.inverse_area_pdf == 0 ? 0.f : s.emission[in.emission][dense_index(l.lambda[k])];
    return finite_nonnegative4(rad);
}

// ---------------------------------------------------------------- lane state
// Path-replay adjoint state of one lane (FP64): d loss / d radiance per wavelength lane, the
// parameter materials of the diffuse vertices so far, and the gradient being accumulated.
struct AdjointLane {
    const std::vector<u32> *slot = nullptr; // per scene material: first gradient entry or RP_NONE
    double w[4] = {0, 0, 0, 0};
    u32 history[16];
    u32 history_count = 0;
    double *grad = nullptr;
};

struct LaneState {
    AdjointLane *adj = nullptr;
    Vertex latest;
    F3 preceding_position{};
    u32 preceding_type = 0;
    Sample sample;
    Wavelengths lambda{};
    F4 radiance, beta;
    F3 ray_o, ray_d;
    HeroTrack hero;
    u64 index = 0;
    u32 count = 1, crossings = 0;
    bool complete = false;
};

struct Ctx {
    const Scene &s;
    const Bvh &bvh;
    const Params &p;
};

// shaders/hero_pt_helpers.h:122-132 (hero_represented_pdf)
static F4 represented_pdf(const Vertex &v, const Vertex &previous, const Vertex &next) {
    const F3 before = infinite(previous) ? -previous.point.geometric_normal
                                         : previous.point.position - v.point.position;
    const F3 after = infinite(next) ? -next.point.geometric_normal : next.point.position - v.point.position;
    if (zero3(before) || zero3(after))
        return f4(0);
    const HeroEval e = hero_evaluate(v.bsdf, v.frame.local(normalize3(before)), v.frame.local(normalize3(after)));
    return e.valid ? e.pdf : f4(NAN);
}
// shaders/hero_pt_helpers.h:133-148
static F4 hero_weight(Sample &smp, const Density &prefix, F4 value, F4 sampled, F4 other) {
    if (!finite_nonnegative4(value) || !finite_nonnegative4(sampled) || !finite_nonnegative4(other)) {
        smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return f4(0);
    }
    if (mixture(prefix, other).fraction == 0)
        return value;
    const auto r = balance_contribution(prefix, value, sampled, other);
    if (!r.valid) {
        smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return f4(0);
    }
    return r.value;
}
// shaders/packet_transport.h:740-758 (direct_pdf / hero_history_light_pdf)
static float light_pdf(const Ctx &c, const Vertex &from, const Vertex &light) {
    const float selection = light_pmf(c.s, from.point.position, from.point.shading_normal, light.light);
    if (infinite(light)) {
        // shaders/packet_transport.h:102-108: unidirectional PT samples the image's compensated
        // table; a constant environment has no proposal
        if (c.s.images.env_image != RP_NONE)
            return env_image_pdf(c.s.images, -light.point.geometric_normal, true) * selection;
        return 0.0f * selection;
    }
    const F3 delta = light.point.position - from.point.position;
    if (!(dot(delta, delta) > 0))
        return 0;
    if (!on_surface(light))
        return 0;
    const u32 emitter = light.light; // area emitters occupy the first light slots
    return selection * light_geometry_pdf(c.s, emitter, from.point.position, from.point.shading_normal,
                                          light.point);
}
// shaders/hero_pt_helpers.h:157-184
static F4 hero_endpoint(const Ctx &c, Sample &smp, const Wavelengths &l, const Vertex &pt,
                        const Vertex &previous, const Vertex &before, u32 t, const Density &prev_density) {
    F4 rad;
    bool ok;
    if (infinite(pt))
        ok = emitted(c.s, pt, -pt.point.geometric_normal, l, rad);
    else {
        const F3 delta = previous.point.position - pt.point.position;
        if (zero3(delta)) {
            rad = f4(0);
            ok = true;
        } else
            ok = emitted(c.s, pt, normalize3(delta), l, rad);
    }
    if (!ok) {
        smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return f4(0);
    }
    const F4 value = pt.beta * rad;
    if (t <= 2 || previous.delta || !nonzero4(value))
        return value;
    const F4 bsdf_pdf = represented_pdf(previous, before, pt);
    const float lp = light_pdf(c, previous, pt);
    return hero_weight(smp, prev_density, value, bsdf_pdf, f4(lp));
}
// shaders/packet_transport.h:377-446 (visible): any surface occludes in an opaque scene; with
// pass-through instances, nearest hits along the segment, restarting past each pass-through one
static bool visible(const Ctx &c, Sample &smp, const Vertex &a, const Vertex &b) {
    const F3 direction = b.point.position - a.point.position;
    if (zero3(direction))
        return false;
    const F3 origin = offset(a, direction);
    const F3 target = offset(b, -direction);
    const Scene &s = c.s;
    if (!std::any_of(s.instances.begin(), s.instances.end(), [&](const Instance &in) { return pass_through(s, in); })) {
        ++smp.shadow_walks;
        return !trace_any(s, c.bvh, origin, target - origin, 0x1.fffffep-1f);
    }
    F3 o = origin, d = target - origin;
    for (u32 crossings = 0; crossings <= c.p.boundary_limit; ++crossings) {
        ++smp.shadow_walks;
        const Hit h = trace_closest(s, c.bvh, o, d, 0x1.fffffep-1f);
        if (h.prim == RP_NONE)
            return true;
        const u32 inst = s.tri_instance[h.prim];
        const Instance &in = s.instances[inst];
        if (in.material >= s.materials.size()) {
            smp.status = RP_SAMPLE_INVALID_HIT;
            return false;
        }
        if (!pass_through(s, in))
            return false;
        SurfacePoint pt;
        F3 next;
        if (!hit_surface_point(s, h.prim, inst, s.tri_local[h.prim], h.b1, h.b2, pt) ||
            !spawn_boundary(o, d, h.t, pt, normalize3(d), next)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            return false;
        }
        o = next;
        d = target - next;
    }
    smp.status = RP_SAMPLE_BOUNDARY_EXHAUSTION;
    return false;
}
// shaders/packet_transport.h:470-553 (sample_li): area emitters and positional lights
static bool sample_li(const Ctx &c, const Vertex &ref, const Wavelengths &l, float u0, float u1, float u2,
                      Vertex &v, F3 &direction, float &pdf) {
    const Scene &s = c.s;
    const auto choice = light_sample(s, ref.point.position, ref.point.shading_normal, u0);
    const u32 sel = choice.light;
    v = Vertex{};
    v.type = light_vertex;
    v.light = sel;
    v.connectible = true;
    if (!(choice.pmf > 0)) {
        v.beta = f4(0);
        pdf = 0;
        return true;
    }
    const u32 emitter_count = u32(s.emitters.size());
    const u32 positional_count = u32(s.positional.size());
    F4 rad;
    if (sel < emitter_count) {
        const auto &e = s.emitters[sel];
        v.instance = e.instance;
        v.primitive = e.primitive;
        if (!light_geometry_sample(s, sel, ref.point.position, ref.point.shading_normal, u1, u2, v.u,
                                   v.v, v.point, pdf))
            return false;
        pdf *= choice.pmf;
        if (v.point.inverse_area_pdf == 0) {
            v.beta = f4(0);
            pdf = 0;
            return true;
        }
        const F3 delta = v.point.position - ref.point.position;
        const float d2 = dot(delta, delta);
        if (!(d2 > 0)) {
            v.beta = f4(0);
            pdf = 0;
            return true;
        }
        direction = delta * (1.0f / std::sqrt(d2));
        if (!emitted(s, v, -direction, l, rad))
            return false;
    } else if (sel < emitter_count + positional_count) {
        const Positional &L = s.positional[sel - emitter_count];
        v.delta_light = true;
        v.point.position = L.position;
        const F3 delta = v.point.position - ref.point.position;
        const float d2 = dot(delta, delta);
        if (!(d2 > 0)) {
            v.beta = f4(0);
            pdf = 0;
            return true;
        }
        direction = delta * (1.0f / std::sqrt(d2));
        // shaders/packet_transport.h:238-251 (positional_radiance)
        for (int k = 0; k < 4; ++k) {
            float intensity = L.intensity[dense_index(l.lambda[k])];
            if (!positional_intensity(L, direction, intensity))
                return false;
            rad[k] = intensity / d2;
        }
        pdf = choice.pmf;
    } else if (s.images.env_image != RP_NONE) {
        // shaders/packet_transport.h:536-552 with sample_environment (:109-123)
        v.type = environment_vertex;
        if (!env_image_sample(s.images, u1, u2, true, direction, pdf))
            return false;
        for (int k = 0; k < 4; ++k)
            rad[k] = env_image_radiance(s.images, direction, l.lambda[k]);
        pdf *= choice.pmf;
        v.point.position = ref.point.position + 2 * s.scene_radius * direction;
        v.point.geometric_normal = -direction;
        v.point.shading_normal = -direction;
    } else {
        // constant environment: not sampleable by unidirectional PT (pdf 0)
        v.type = environment_vertex;
        direction = F3{0, 0, 1};
        pdf = 0;
        rad = f4(0);
        v.point.position = ref.point.position + 2 * s.scene_radius * direction;
        v.point.geometric_normal = -direction;
        v.point.shading_normal = -direction;
    }
    v.beta = pdf > 0 ? F4{{rad[0] / pdf, rad[1] / pdf, rad[2] / pdf, rad[3] / pdf}} : f4(0);
    return finite_nonnegative4(v.beta);
}
// shaders/hero_pt_helpers.h:185-221
static F4 hero_direct(const Ctx &c, Sample &smp, const Wavelengths &l, u64 index, const Vertex &pt,
                      const Vertex &before, u32 t, F4 beta, const Density &prefix) {
    if (pt.type != surface_vertex || !pt.connectible)
        return f4(0);
    const U4 w = draw_words(c.s, c.p, smp, index, 133 + t - 2);
    Vertex sampled;
    F3 direction{};
    float sampled_pdf = 0;
    if (!sample_li(c, pt, l, sample_uniform(c.p, w.x), sample_uniform(c.p, w.y),
                   sample_uniform(c.p, w.z), sampled, direction, sampled_pdf) ||
        !std::isfinite(sampled_pdf) || sampled_pdf < 0) {
        smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return f4(0);
    }
    if (!(sampled_pdf > 0) || !nonzero4(sampled.beta))
        return f4(0);
    const HeroEval e = hero_evaluate(pt.bsdf, pt.pair_valid ? pt.sampled_wo_local : pt.frame.local(pt.wo),
                                     pt.frame.local(direction));
    if (!e.valid) {
        smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        return f4(0);
    }
    const F4 value = beta * e.f * sampled.beta * std::fabs(dot(pt.point.shading_normal, direction));
    if (!nonzero4(value) || !visible(c, smp, pt, sampled))
        return f4(0);
    if (sampled.delta_light)
        return value;
    sampled_pdf = light_pdf(c, pt, sampled);
    const F4 bsdf_pdf = represented_pdf(pt, before, sampled);
    return hero_weight(smp, prefix, value, f4(sampled_pdf), bsdf_pdf);
}

// d loss / d knots of one contribution: contribution * w / rho over the history's vertices,
// rho piecewise linear in the knots (pbrt_reflectance), all in FP64.
static void adjoint_accumulate(const Scene &s, AdjointLane &a, const Wavelengths &l, F4 contribution) {
    for (u32 j = 0; j < a.history_count; ++j) {
        const u32 m = a.history[j];
        const Material &M = s.materials[m];
        const Knot *kn = s.knots.data() + M.knot_begin;
        const u32 slot = (*a.slot)[m];
        for (int k = 0; k < 4; ++k) {
            const double g0 = a.w[k] * double(contribution[k]);
            const float x = l.lambda[k];
            if (g0 == 0 || !(x >= kn[0].wavelength && x <= kn[M.knot_count - 1].wavelength))
                continue;
            u32 lo = 0, hi = M.knot_count - 1;
            while (hi - lo > 1) {
                const u32 mid = lo + (hi - lo) / 2;
                if (x < kn[mid].wavelength)
                    hi = mid;
                else
                    lo = mid;
            }
            const double t = lo == hi ? 0.0
                                      : (double(x) - kn[lo].wavelength) / (double(kn[hi].wavelength) - kn[lo].wavelength);
            const double rho = kn[lo].value + (double(kn[hi].value) - kn[lo].value) * t;
            if (!(rho > 0))
                continue;
            const double g = g0 / rho;
            a.grad[slot + lo] += g * (1.0 - t);
            if (hi != lo)
                a.grad[slot + hi] += g * t;
        }
    }
}

// shaders/packet_pt_event_body.inc:11-461 (one hero event, vacuum, opaque surfaces)
static void hero_step(const Ctx &c, LaneState &st) {
    if (st.complete)
        return;
    const Scene &s = c.s;
    const Params &p = c.p;
    Sample &smp = st.sample;
    const Wavelengths &l = st.lambda;
    F4 &beta = st.beta;
    u32 &count = st.count;
    const Density previous_density = st.hero.previous;
    Density direct_density = st.hero.density;
    F4 direct_beta = beta;
    bool direct_allowed = true;
    const u32 capacity = p.max_depth + 2;
    F3 ro = st.ray_o, rd = st.ray_d;
    const u32 old_count = count;
    bool terminated = true;
    Vertex current{};
    do {
        if (count >= capacity || !nonzero4(beta))
            break;
        if (!finite3(ro) || !finite3(rd) || !finite_nonnegative4(beta)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        ++smp.closest_walks;
        const Hit hit = trace_closest(s, c.bvh, ro, rd, INFINITY);
        if (hit.prim == RP_NONE) {
            Vertex &v = current;
            v.type = environment_vertex;
            v.light = s.environment_light;
            v.point.position = ro + rd;
            v.point.geometric_normal = -rd;
            v.point.shading_normal = -rd;
            v.wo = -rd;
            v.beta = beta;
            v.connectible = true;
            ++count;
            break;
        }
        if (!std::isfinite(hit.t) || hit.t < 0 || !std::isfinite(hit.b1) || !std::isfinite(hit.b2)) {
            smp.status = RP_SAMPLE_INVALID_HIT;
            break;
        }
        const u32 inst = s.tri_instance[hit.prim], local = s.tri_local[hit.prim];
        const Instance &instance = s.instances[inst];
        if (instance.material >= s.materials.size()) {
            smp.status = RP_SAMPLE_INVALID_HIT;
            break;
        }
        Vertex &v = current;
        v.type = surface_vertex;
        v.instance = inst;
        v.primitive = local;
        v.u = hit.b1;
        v.v = hit.b2;
        v.light = instance.emission == RP_NONE ? RP_NONE : instance.emitter_begin + local;
        v.wo = -rd;
        if (!hit_surface_point(s, hit.prim, inst, local, hit.b1, hit.b2, v.point)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        // shaders/packet_pt_event_body.inc:130-145: a pass-through surface makes no vertex; the
        // next event continues the ray from past it
        if (pass_through(s, instance)) {
            if (st.crossings++ >= p.boundary_limit) {
                smp.status = RP_SAMPLE_BOUNDARY_EXHAUSTION;
                break;
            }
            F3 origin;
            if (!spawn_boundary(ro, rd, hit.t, v.point, rd, origin)) {
                smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
                break;
            }
            ro = origin;
            terminated = false;
            break;
        }
        // :165-190: mix materials resolve at the hit
        u32 material_index = instance.material;
        if (const u32 mix_status = resolve_mix(s, v.point.position, -rd, material_index)) {
            smp.status = mix_status;
            break;
        }
        v.material = material_index;
        const Material &material = s.materials[material_index];
        // :147-163 and shaders/packet_walk.h:39-49: an image reflectance reads the texture at the
        // hit's footprint (the context of its root material; here, of the image material)
        Rgb image_rgb;
        const Rgb *image = nullptr;
        if (material.scattering == RP_DIFFUSE && material.kind == RP_REFLECTANCE_IMAGE &&
            material.image_texture < s.images.textures.size()) {
            F2 uvst, dstdx, dstdy;
            if (!texture_context(s, p, smp, inst, local, hit.b1, hit.b2, v.point.geometric_normal, rd, count - 1,
                                 uvst, dstdx, dstdy)) {
                smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
                break;
            }
            const rp_image_texture &t = s.images.textures[material.image_texture];
            image_rgb = image_lookup(s.images, t, uvst, dstdx, dstdy, false, false);
            image_rgb = {image_rgb.r * t.scale, image_rgb.g * t.scale, image_rgb.b * t.scale};
            if (t.invert)
                image_rgb = {1 - image_rgb.r, 1 - image_rgb.g, 1 - image_rgb.b};
            image = &image_rgb;
        }
        F3 dpdu, dpdv;
        coordinate_system(v.point.shading_normal, dpdu, dpdv);
        if (!scattering_frame(v.point.shading_normal, dpdu, v.frame) ||
            !prepare_bsdf(s, material, l, st.hero.active_mask, v.bsdf, image)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        F3 ray_position, ray_error;
        ray_point(ro, rd, hit.t, v.point.curved, ray_position, ray_error);
        v.point.error = v.point.error + (fabs3(v.point.position - ray_position) + ray_error);
        if (!finite3(v.point.error)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        v.beta = beta;
        v.connectible = hero_connectible(v.bsdf);
        ++count;
        st.crossings = 0;
        if (count == capacity)
            break;
        if (count - 2 >= p.emergency_limit) {
            smp.status = RP_SAMPLE_EMERGENCY_DEPTH;
            break;
        }
        const U4 draws = draw_words(s, p, smp, st.index, 4 + count - 2);
        const F3 wo_local = v.frame.local(v.wo);
        // hero_prepare_future (shaders/hero_pt_helpers.h:38-50): no single-hero families here
        current.bsdf.active_mask = st.hero.active_mask;
        direct_density = st.hero.density;
        direct_allowed = hero_continue(beta, st.hero, count - 1, sample_uniform(p, draws.w));
        direct_beta = beta;
        current.connectible = hero_connectible(current.bsdf);
        if (!direct_allowed)
            break;
        const HeroSample proposed = hero_sample(current.bsdf, wo_local, sample_uniform(p, draws.x),
                                                sample_uniform(p, draws.y), sample_uniform(p, draws.z));
        bool cont_valid = proposed.valid;
        const bool cont_accepted = proposed.accepted;
        if (proposed.valid && proposed.accepted) {
            st.hero.previous = direct_density;
            const Update adv = advance(direct_density, beta, proposed.numerator, proposed.pdf);
            cont_valid = adv.valid;
            if (adv.valid) {
                beta = adv.beta;
                st.hero.density = adv.density;
            }
            hero_account_eta(st.hero, proposed.eta, proposed.transmission);
            st.hero.active_mask = 1;
            for (int k = 1; k < 4; ++k)
                if (st.hero.density.lane[k].fraction > 0 || (fbits(beta[k]) & 0x7fffffffu))
                    st.hero.active_mask |= 1u << k;
        }
        if (!cont_valid) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        if (!cont_accepted)
            break;
        current.sampled_wo_local = wo_local;
        current.sampled_wi_local = proposed.wi;
        current.pair_valid = true;
        F3 wi = v.frame.world(proposed.wi);
        if (!unit_vector(wi, wi)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        if (!finite_nonnegative4(beta)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        if (proposed.delta)
            current.delta = true;
        const F3 origin = offset(v, wi);
        if (!finite3(origin)) {
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
            break;
        }
        ro = origin;
        rd = wi;
        terminated = false;
    } while (false);
    st.ray_o = ro;
    st.ray_d = rd;
    st.complete = terminated || smp.status != RP_SAMPLE_SUCCESS || count >= capacity || !nonzero4(beta);
    if (count != old_count && smp.status == RP_SAMPLE_SUCCESS) {
        Vertex before{};
        if (count > 2) {
            before.type = st.preceding_type;
            before.point.position = st.preceding_position;
        }
        const F4 endpoint = hero_endpoint(c, smp, l, current, st.latest, before, count, previous_density);
        st.radiance = st.radiance + endpoint;
        if (st.adj) {
            if (smp.status == RP_SAMPLE_SUCCESS && nonzero4(endpoint))
                adjoint_accumulate(s, *st.adj, l, endpoint);
            if (current.type == surface_vertex && smp.status == RP_SAMPLE_SUCCESS) {
                const u32 m = current.material;
                if (s.materials[m].scattering == RP_DIFFUSE && (*st.adj->slot)[m] != RP_NONE &&
                    st.adj->history_count < 16)
                    st.adj->history[st.adj->history_count++] = m;
            }
        }
        if (smp.status == RP_SAMPLE_SUCCESS && count < capacity && direct_allowed) {
            const F4 direct = hero_direct(c, smp, l, st.index, current, st.latest, count, direct_beta, direct_density);
            st.radiance = st.radiance + direct;
            if (st.adj && smp.status == RP_SAMPLE_SUCCESS && nonzero4(direct))
                adjoint_accumulate(s, *st.adj, l, direct);
        }
        if (!finite_nonnegative4(st.radiance))
            smp.status = RP_SAMPLE_INVALID_ARITHMETIC;
        if (smp.status != RP_SAMPLE_SUCCESS)
            st.complete = true;
    }
    if (count != old_count) {
        st.preceding_position = st.latest.point.position;
        st.preceding_type = st.latest.type;
        st.latest = current;
    }
}

// shaders/render.metal:2424-2469 (hero branch) + packet_pt_result (shaders/packet_pt_step.h:225-239)
static rp_packet_result render_lane(const Ctx &c, u32 lane, AdjointLane *adj = nullptr) {
    const Scene &s = c.s;
    LaneState st;
    st.adj = adj;
    u64 index = 0;
    st.sample = begin_sample(s, c.p, lane, index);
    st.index = index;
    const float uw = sample_uniform(c.p, st.sample.words[2]);
    st.lambda = s.hero_mode == RP_HERO_VISIBLE ? sample_visible(uw) : sample_uniform(uw);
    F3 o, d;
    primary_ray(s, c.p, st.sample, o, d);
    st.ray_o = o;
    st.ray_d = d;
    st.beta = f4(1);
    st.count = 1;
    Vertex cam{};
    cam.type = camera_vertex;
    cam.point.position = o;
    cam.beta = f4(1);
    cam.connectible = true;
    st.latest = cam;
    if (st.sample.status != RP_SAMPLE_SUCCESS || !finite3(o) || !finite3(d)) {
        st.sample.status = RP_SAMPLE_INVALID_ARITHMETIC;
        st.complete = true;
    }
    while (!st.complete)
        hero_step(c, st);
    rp_packet_result r{};
    r.status = st.complete ? st.sample.status : u32(RP_SAMPLE_INVALID_ARITHMETIC);
    r.pixel = st.sample.pixel;
    r.sample_low = st.sample.sample_low;
    r.sample_high = st.sample.sample_high;
    r.filter_weight = s.filter_weight;
    for (int k = 0; k < 4; ++k) {
        r.wavelengths[k] = st.lambda.lambda[k];
        r.wavelength_pdfs[k] = st.lambda.pdf[k];
        r.radiance[k] = st.radiance[k];
    }
    // the reserved words, unread by rypath, carry the lane's traversal counts
    r.reserved[0] = st.sample.closest_walks;
    r.reserved[1] = st.sample.shadow_walks;
    return r;
}

} // namespace oracle

using namespace oracle;


static void put_diag(char *diag, size_t cap, const std::string &msg) {
    if (diag && cap) {
        std::snprintf(diag, cap, "%s", msg.c_str());
    }
}

extern "C" {

or_scene *or_scene_create(const rp_scene_desc *desc, char *diag, size_t cap) {
    if (!desc || desc->abi_version != RP_ABI_VERSION || !desc->sobol_tables) {
        put_diag(diag, cap, "invalid scene description");
        return nullptr;
    }
    auto out = std::make_unique<or_scene>();
    std::string error;
    if (!load_scene(*desc, out->scene, error)) {
        put_diag(diag, cap, error);
        return nullptr;
    }
    build_lbvh(out->scene.world, out->bvh);
    return out.release();
}

void or_scene_destroy(or_scene *scene) { delete scene; }
uint32_t or_scene_light_count(const or_scene *scene) { return scene->scene.light_count; }

int or_sample(const or_scene *scene, const rp_request *request, rp_packet_result *results,
              size_t capacity, int threads) {
    const u64 lanes = u64(request->pixel_count) * request->sample_count;
    if (lanes > capacity || request->pixel_count == 0)
        return -1;
    const Params p = make_params(scene->scene, *request);
    const Ctx c{scene->scene, scene->bvh, p};
    unsigned n = threads > 0 ? unsigned(threads) : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<u64> next{0};
    auto work = [&]() {
        for (;;) {
            const u64 begin = next.fetch_add(256);
            if (begin >= lanes)
                return;
            const u64 end = std::min(lanes, begin + 256);
            for (u64 i = begin; i < end; ++i)
                results[i] = render_lane(c, u32(i));
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

// The FP64 path-replay adjoint of a film render: d loss / d knots of the listed materials
// given d loss / d film-mean XYZ per pixel (the rp_cuda_adjoint_device contract, in double).
int or_adjoint(const or_scene *scene, const rp_film_request *f, const uint32_t *materials, uint32_t count,
               const double *d_loss_d_xyz, const double *cie, double *grad, int threads) {
    const Scene &s = scene->scene;
    std::vector<u32> slot(s.materials.size(), RP_NONE);
    u32 params = 0;
    for (u32 i = 0; i < count; ++i) {
        const u32 m = materials[i];
        if (m >= s.materials.size() || slot[m] != RP_NONE || s.materials[m].scattering != RP_DIFFUSE ||
            s.materials[m].kind != RP_REFLECTANCE_KNOTS)
            return -1;
        slot[m] = params;
        params += s.materials[m].knot_count;
    }
    rp_request q{};
    q.width = f->width;
    q.height = f->height;
    q.seed = f->seed;
    q.pixel_count = f->width * f->height;
    q.sample_begin = f->sample_begin;
    q.sample_count = u32(f->sample_count);
    q.emergency_limit = f->emergency_limit;
    q.sampler_kind = f->sampler_kind;
    q.randomization = f->randomization;
    const Params p = make_params(s, q);
    const Ctx c{s, scene->bvh, p};
    const u64 lanes = u64(q.pixel_count) * q.sample_count;
    const unsigned n = threads > 0 ? unsigned(threads) : std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<double>> local(n, std::vector<double>(params, 0.0));
    std::atomic<u64> next{0};
    std::atomic<u32> failures{0};
    auto work = [&](unsigned t) {
        for (;;) {
            const u64 begin = next.fetch_add(256);
            if (begin >= lanes)
                return;
            for (u64 i = begin; i < std::min(lanes, begin + 256); ++i) {
                u64 index = 0;
                const Sample smp = begin_sample(s, p, u32(i), index);
                const float uw = sample_uniform(p, smp.words[2]);
                const Wavelengths l = s.hero_mode == RP_HERO_VISIBLE ? sample_visible(uw) : sample_uniform(uw);
                AdjointLane a;
                a.slot = &slot;
                a.grad = local[t].data();
                for (int k = 0; k < 4; ++k) {
                    if (l.pdf[k] == 0 || !(l.lambda[k] >= 360 && l.lambda[k] <= 830))
                        continue;
                    const size_t row = size_t(std::round(double(l.lambda[k])) - 360.0);
                    double g = 0;
                    for (int ch = 0; ch < 3; ++ch)
                        g += d_loss_d_xyz[3 * size_t(smp.pixel) + ch] * cie[3 * row + ch];
                    a.w[k] = g / (double(l.pdf[k]) * 4.0) / double(q.sample_count);
                }
                if (render_lane(c, u32(i), &a).status != RP_SAMPLE_SUCCESS)
                    ++failures;
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < n; ++t)
        pool.emplace_back(work, t);
    work(0);
    for (auto &t : pool)
        t.join();
    for (u32 j = 0; j < params; ++j) {
        double sum = 0;
        for (unsigned t = 0; t < n; ++t)
            sum += local[t][j];
        grad[j] = sum;
    }
    return failures ? 1 : 0;
}

// The Gaussian filter table (compile_gaussian_filter) and its inverse as the device samples it
// (gaussian_filter_offsets): cdf receives the conditional rows then the marginal; samples
// receive (x, y) for each of count (u, v) pairs.  Returns the table size in floats, or -1.
int or_gaussian_filter(float x_radius, float y_radius, float sigma, float *cdf, size_t capacity, uint32_t *size,
                       float *integral, const float *uv, uint32_t count, float *samples) {
    Scene s;
    s.filter_kind = RP_FILTER_GAUSSIAN;
    s.filter_x = x_radius;
    s.filter_y = y_radius;
    if (!gaussian_filter_table(x_radius, y_radius, sigma, s.gauss_cdf, s.gauss_w, s.gauss_h, *integral).empty() ||
        s.gauss_cdf.size() > capacity)
        return -1;
    std::copy(s.gauss_cdf.begin(), s.gauss_cdf.end(), cdf);
    size[0] = s.gauss_w;
    size[1] = s.gauss_h;
    for (uint32_t i = 0; i < count; ++i)
        gaussian_filter_offsets(s, uv[2 * i], uv[2 * i + 1], samples[2 * i], samples[2 * i + 1]);
    return int(s.gauss_cdf.size());
}

// Halton / ZSobol probe in the layout of rypath's QMC known answers
// (tests/qmc_sampling_tests.cpp:184-219): query (kind, width, height, x, y, sample, dimension,
// mode, seed, spp) as 10 int64, result 6 uint64 (index, camera x/y and three draws, as float
// bits except the ZSobol index).
void or_probe_qmc(const void *sobol_tables, const int64_t *queries, uint32_t count, uint64_t *results) {
    const SobolTables &t = *static_cast<const SobolTables *>(sobol_tables);
    for (uint32_t i = 0; i < count; ++i) {
        const int64_t *q = queries + 10 * i;
        const u32 w = u32(q[1]), h = u32(q[2]), x = u32(q[3]), y = u32(q[4]), d = u32(q[6]), mode = u32(q[7]),
                  seed = u32(q[8]), spp = u32(q[9]);
        const u64 sample = u64(q[5]);
        uint64_t *a = results + 6 * i;
        if (q[0] == RP_SAMPLER_HALTON) {
            const u64 index = halton_index(w, h, x, y, sample);
            a[0] = 0;
            a[1] = fbits(halton_camera(0, w, index));
            a[2] = fbits(halton_camera(1, h, index));
            a[3] = a[4] = fbits(qmc_radical(d, index, mode, seed));
            a[5] = fbits(qmc_radical(d + 1, index, mode, seed));
        } else {
            const u32 m = sobol_scale_exponent(w, h);
            const u32 log = 31 - __builtin_clz(spp);
            const u64 morton = zsobol_morton(x, y, log, sample);
            a[0] = zsobol_index(morton, d, m, log);
            a[1] = fbits(sobol_uniform(zsobol_word(t, morton, 1, 0, true, m, log, mode, seed)));
            a[2] = fbits(sobol_uniform(zsobol_word(t, morton, 1, 1, true, m, log, mode, seed)));
            a[3] = fbits(sobol_uniform(zsobol_word(t, morton, d, 0, false, m, log, mode, seed)));
            a[4] = fbits(sobol_uniform(zsobol_word(t, morton, d, 0, true, m, log, mode, seed)));
            a[5] = fbits(sobol_uniform(zsobol_word(t, morton, d, 1, true, m, log, mode, seed)));
        }
    }
}

void or_probe_sobol(const void *tables, const uint32_t *q, uint32_t count, uint32_t *r) {
    const auto &t = *static_cast<const SobolTables *>(tables);
    for (u32 i = 0; i < count; ++i) {
        const u32 *a = q + 8 * i;
        const u64 index = sobol_index(t, a[0], a[1], a[2], (u64(a[4]) << 32) | a[3]);
        const u32 value = sobol_word(t, index, a[5], a[6], a[7]);
        const u32 camera = sobol_word(t, index, 0, 0, 0);
        u32 *o = r + 6 * i;
        o[0] = u32(index);
        o[1] = u32(index >> 32);
        o[2] = value;
        o[3] = sobol_dimension_hash(a[5], a[7]);
        o[4] = fbits(sobol_uniform(value));
        o[5] = fbits(sobol_camera_uniform(camera, a[0], a[1]));
    }
}

void or_probe_philox(const uint32_t *q, uint32_t count, uint32_t *r) {
    for (u32 i = 0; i < count; ++i) {
        const u32 *a = q + 6 * i;
        const U4 w = philox(U4{a[0], a[1], a[2], a[3]}, a[4], a[5]);
        r[4 * i] = w.x;
        r[4 * i + 1] = w.y;
        r[4 * i + 2] = w.z;
        r[4 * i + 3] = w.w;
    }
}

void or_probe_wavelengths(const float *u, uint32_t count, uint32_t mode, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const Wavelengths w = mode == RP_HERO_VISIBLE ? sample_visible(u[i]) : sample_uniform(u[i]);
        for (int k = 0; k < 4; ++k) {
            r[8 * i + k] = w.lambda[k];
            r[8 * i + 4 + k] = w.pdf[k];
        }
    }
}

int or_probe_raygen(const or_scene *scene, const rp_request *request, uint32_t *words, float *rays,
                    size_t capacity) {
    const u64 lanes = u64(request->pixel_count) * request->sample_count;
    if (lanes > capacity)
        return -1;
    const Params p = make_params(scene->scene, *request);
    for (u64 i = 0; i < lanes; ++i) {
        u64 index = 0;
        const Sample smp = begin_sample(scene->scene, p, u32(i), index);
        u32 *w = words + 11 * i;
        w[0] = smp.pixel;
        w[1] = smp.sample_low;
        w[2] = smp.sample_high;
        w[3] = u32(index);
        w[4] = u32(index >> 32);
        for (int k = 0; k < 4; ++k)
            w[5 + k] = smp.words[k];
        w[9] = smp.lens_words[0];
        w[10] = smp.lens_words[1];
        F3 o, d;
        primary_ray(scene->scene, p, smp, o, d);
        float *r = rays + 6 * i;
        for (int a = 0; a < 3; ++a) {
            r[a] = o[a];
            r[3 + a] = d[a];
        }
    }
    return 0;
}

void or_probe_bsdf(const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 16 * i;
        float *o = r + 12 * i;
        std::fill(o, o + 12, 0.0f);
        LaneBsdf lane{};
        lane.kind = u32(a[0]);
        bool ok = true;
        if (lane.kind == 0)
            lane.reflectance = a[1];
        else if (lane.kind == 1)
            ok = conductor_prepare(a[1], a[2], a[3], a[4], a[5] != 0, lane.conductor);
        else
            ok = dielectric_prepare(a[1], a[3], a[4], a[5] != 0, lane.dielectric);
        if (!ok) {
            o[2] = -1;
            continue;
        }
        const F3 wo{a[6], a[7], a[8]}, wi{a[9], a[10], a[11]};
        const Eval e = scalar_evaluate(lane, wo, wi);
        o[0] = e.f;
        o[1] = e.pdf;
        o[2] = e.valid ? 1.f : 0.f;
        float eta;
        const BSample smp = scalar_sample(lane, wo, a[12], a[13], a[14], eta);
        o[3] = smp.wi.x;
        o[4] = smp.wi.y;
        o[5] = smp.wi.z;
        o[6] = smp.weight;
        o[7] = smp.pdf;
        o[8] = float((smp.delta ? 1 : 0) | (smp.accepted ? 2 : 0) | (smp.valid ? 4 : 0));
        o[9] = eta;
    }
}

int or_export_bvh(const or_scene *scene, uint32_t *nodes, uint32_t *leaf_order, uint64_t *keys,
                  float *bounds, size_t capacity) {
    const Bvh &b = scene->bvh;
    if (b.n > capacity)
        return -1;
    for (u32 i = 0; i < b.n; ++i) {
        leaf_order[i] = b.order[i];
        keys[i] = b.keys[i];
        for (int a = 0; a < 3; ++a) {
            bounds[6 * (b.n - 1 + i) + a] = b.leaf_box[i].lo[a];
            bounds[6 * (b.n - 1 + i) + 3 + a] = b.leaf_box[i].hi[a];
        }
    }
    for (u32 i = 0; i + 1 < b.n; ++i) {
        nodes[3 * i] = b.left[i];
        nodes[3 * i + 1] = b.right[i];
        nodes[3 * i + 2] = b.parent[i];
        for (int a = 0; a < 3; ++a) {
            bounds[6 * i + a] = b.node_box[i].lo[a];
            bounds[6 * i + 3 + a] = b.node_box[i].hi[a];
        }
    }
    return int(b.n);
}

void or_trace_rays(const or_scene *scene, const float *rays, uint32_t count, int any_hit, int brute,
                   float *hits) {
    for (u32 i = 0; i < count; ++i) {
        const float *r = rays + 7 * i;
        const F3 o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
        float *h = hits + 4 * i;
        if (any_hit) {
            const bool occ = brute ? trace_closest_brute(scene->scene, o, d, r[6]).prim != RP_NONE
                                   : trace_any(scene->scene, scene->bvh, o, d, r[6]);
            h[0] = occ ? 1.f : 0.f;
            h[1] = h[2] = 0;
            h[3] = ffrom(RP_NONE);
            continue;
        }
        const Hit hit = brute ? trace_closest_brute(scene->scene, o, d, r[6])
                              : trace_closest(scene->scene, scene->bvh, o, d, r[6]);
        h[0] = hit.prim == RP_NONE ? INFINITY : hit.t;
        h[1] = hit.b1;
        h[2] = hit.b2;
        h[3] = ffrom(hit.prim);
    }
}

void or_probe_advance(const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 20 * i;
        Density prefix;
        F4 beta, num, pdf;
        for (int k = 0; k < 4; ++k) {
            prefix.lane[k].fraction = a[k];
            prefix.lane[k].exponent = int(a[4 + k]);
            beta[k] = a[8 + k];
            num[k] = a[12 + k];
            pdf[k] = a[16 + k];
        }
        const Update u = advance(prefix, beta, num, pdf);
        float *o = r + 13 * i;
        for (int k = 0; k < 4; ++k) {
            o[k] = u.beta[k];
            o[4 + k] = u.density.lane[k].fraction;
            o[8 + k] = float(u.density.lane[k].exponent);
        }
        o[12] = u.valid ? 1.f : 0.f;
    }
}

// Hero BSDF probe: per query 32 floats {kind, active mask, remap, unused, 4 lanes x {eta or
// reflectance, k, roughness u, roughness v}, wo[3], wi[3], uc, ux, uy, unused[3]} -> 32 floats
// {sample: wi[3], numerator[4], pdf[4], eta[4], flags (delta 1, transmission 2, accepted 4,
// valid 8); evaluation at wi: f[4], pdf[4], valid; Dirac lane 0 at wi: mass, pdf, eta, ok;
// connectible; prepared 1 / failed 0; unused}.  kind 0 diffuse, 1 conductor, 2 dielectric.
void or_probe_hero(const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 32 * i;
        float *o = r + 32 * i;
        std::fill(o, o + 32, 0.0f);
        HeroBsdf p;
        p.active_mask = u32(a[1]);
        const bool remap = a[2] != 0;
        bool ok = true;
        for (int k = 0; k < 4; ++k) {
            const float *l = a + 4 + 4 * k;
            LaneBsdf &lane = p.lane[k];
            lane.kind = u32(a[0]);
            if (lane.kind == 0)
                lane.reflectance = l[0];
            else if (lane.kind == 1)
                ok = conductor_prepare(l[0], l[1], l[2], l[3], remap, lane.conductor) && ok;
            else
                ok = dielectric_prepare(l[0], l[2], l[3], remap, lane.dielectric) && ok;
        }
        o[30] = ok ? 1.f : 0.f;
        if (!ok)
            continue;
        const F3 wo{a[20], a[21], a[22]}, wi{a[23], a[24], a[25]};
        const HeroSample smp = hero_sample(p, wo, a[26], a[27], a[28]);
        o[0] = smp.wi.x;
        o[1] = smp.wi.y;
        o[2] = smp.wi.z;
        for (int k = 0; k < 4; ++k) {
            o[3 + k] = smp.numerator[k];
            o[7 + k] = smp.pdf[k];
            o[11 + k] = smp.eta[k];
        }
        o[15] = float((smp.delta ? 1 : 0) | (smp.transmission ? 2 : 0) | (smp.accepted ? 4 : 0) | (smp.valid ? 8 : 0));
        const HeroEval e = hero_evaluate(p, wo, wi);
        for (int k = 0; k < 4; ++k) {
            o[16 + k] = e.f[k];
            o[20 + k] = e.pdf[k];
        }
        o[24] = e.valid ? 1.f : 0.f;
        float mass, density, eta;
        const bool dirac = dirac_lane(p.lane[0], wo, wi, a[27], a[28], mass, density, eta);
        o[25] = mass;
        o[26] = density;
        o[27] = eta;
        o[28] = dirac ? 1.f : 0.f;
        o[29] = hero_connectible(p) ? 1.f : 0.f;
    }
}

// Roulette probe: per query 16 floats {beta[4], eta scale[4], roulette enabled, depth, u,
// transmission, eta[4]} -> 12 floats {continues, beta after[4], eta scale after accounting
// eta[4], roulette enabled after, unused[2]}: hero_continue, then hero_account_eta on the
// query's track (shaders/hero_pt_helpers.h:56-98).
void or_probe_roulette(const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 16 * i;
        float *o = r + 12 * i;
        std::fill(o, o + 12, 0.0f);
        HeroTrack track;
        F4 beta, eta;
        for (int k = 0; k < 4; ++k) {
            beta[k] = a[k];
            track.eta_scale[k] = a[4 + k];
            eta[k] = a[12 + k];
        }
        track.roulette_enabled = a[8] != 0;
        const bool alive = hero_continue(beta, track, u32(a[9]), a[10]);
        hero_account_eta(track, eta, a[11] != 0);
        o[0] = alive ? 1.f : 0.f;
        for (int k = 0; k < 4; ++k) {
            o[1 + k] = beta[k];
            o[5 + k] = track.eta_scale[k];
        }
        o[9] = track.roulette_enabled ? 1.f : 0.f;
    }
}

// MIS weight probe: per query 20 floats {prefix fractions[4], prefix exponents[4], value[4],
// sampled[4], other[4]} -> 5 floats {weighted contribution[4], failed}
// (hero_weight, shaders/hero_pt_helpers.h:122-138).
void or_probe_hero_weight(const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 20 * i;
        float *o = r + 5 * i;
        Density prefix;
        F4 value, sampled, other;
        for (int k = 0; k < 4; ++k) {
            prefix.lane[k].fraction = a[k];
            prefix.lane[k].exponent = int(a[4 + k]);
            value[k] = a[8 + k];
            sampled[k] = a[12 + k];
            other[k] = a[16 + k];
        }
        Sample smp;
        const F4 w = hero_weight(smp, prefix, value, sampled, other);
        for (int k = 0; k < 4; ++k)
            o[k] = w[k];
        o[4] = smp.status != RP_SAMPLE_SUCCESS ? 1.f : 0.f;
    }
}

int or_build_light_tables(const double *rows, uint32_t count, uint32_t *alias, uint32_t *records,
                          uint32_t *nodes, uint32_t *infinite, uint32_t *infinite_count) {
    std::vector<LightInput> in(count);
    for (u32 i = 0; i < count; ++i) {
        const double *r = rows + 16 * i;
        in[i].power = r[0];
        in[i].bounds_power = r[1];
        for (int a = 0; a < 3; ++a) {
            in[i].low[a] = float(r[2 + a]);
            in[i].high[a] = float(r[5 + a]);
            in[i].direction[a] = float(r[8 + a]);
        }
        in[i].cos_outer = float(r[11]);
        in[i].cos_emission = float(r[12]);
        in[i].two_sided = r[13] != 0;
        in[i].infinite = r[14] != 0;
    }
    LightTables t;
    std::string error;
    if (!build_light_tables(in, t, error))
        return -1;
    std::memcpy(alias, t.alias.data(), t.alias.size() * sizeof(LightAlias));
    std::memcpy(records, t.records.data(), t.records.size() * sizeof(LightRecord));
    std::memcpy(nodes, t.nodes.data(), t.nodes.size() * sizeof(LightBounds));
    std::memcpy(infinite, t.infinite.data(), t.infinite.size() * sizeof(u32));
    *infinite_count = u32(t.infinite.size());
    return int(t.nodes.size());
}

void or_probe_light_select(const or_scene *scene, const float *q, uint32_t count, float *r) {
    for (u32 i = 0; i < count; ++i) {
        const float *a = q + 8 * i;
        const F3 pos{a[0], a[1], a[2]}, n{a[3], a[4], a[5]};
        const Selected sel = light_sample(scene->scene, pos, n, a[6]);
        r[3 * i] = ffrom(sel.light);
        r[3 * i + 1] = sel.pmf;
        r[3 * i + 2] = light_pmf(scene->scene, pos, n, fbits(a[7]));
    }
}

// src/packet_film.cpp:10-14 (Neumaier step), :102-114 (packet_sensor_xyz), :198-265 (add)
static void add_compensated(double value, double &sum, double &correction) {
    const double next = sum + value;
    correction += std::abs(sum) >= std::abs(value) ? (sum - next) + value : (value - next) + sum;
    sum = next;
}
int or_film_add_clamped(const rp_packet_result *results, size_t count, const double *cie, uint32_t pixel_count,
                        double exposure, double max_component_value, rp_film_pixel *film);
int or_film_add(const rp_packet_result *results, size_t count, const double *cie, uint32_t pixel_count,
                rp_film_pixel *film) {
    return or_film_add_clamped(results, count, cie, pixel_count, 1.0, INFINITY, film);
}
// PacketFilmBatch::add (src/packet_film.cpp:198-265) without splats, with the compatibility
// planes of a finite clamp (clamp_sensor, :39-47)
int or_film_add_clamped(const rp_packet_result *results, size_t count, const double *cie, uint32_t pixel_count,
                        double exposure, double max_component_value, rp_film_pixel *film) {
    const bool clamp = std::isfinite(max_component_value) && max_component_value > 0;
    for (size_t i = 0; i < count; ++i) {
        const auto &s = results[i];
        if (s.pixel >= pixel_count)
            return -1;
        double xyz[3] = {0, 0, 0};
        for (int k = 0; k < 4; ++k) {
            if (s.wavelength_pdfs[k] == 0)
                continue;
            const double w = s.wavelengths[k];
            if (!(w >= 360 && w <= 830))
                continue;
            const size_t row = size_t(std::round(w) - 360);
            const double weight = double(s.radiance[k]) / s.wavelength_pdfs[k] / 4;
            for (int c = 0; c < 3; ++c)
                xyz[c] += weight * cie[3 * row + c];
        }
        auto &px = film[s.pixel];
        for (int c = 0; c < 3; ++c) {
            const double v = xyz[c] * s.filter_weight;
            add_compensated(v, px.sum[c], px.correction[c]);
            px.square[c] += v * v;
        }
        if (clamp) {
            double e[3] = {xyz[0] * exposure, xyz[1] * exposure, xyz[2] * exposure};
            const double maximum = std::max(std::max(e[0], e[1]), e[2]);
            if (maximum > max_component_value)
                for (double &v : e)
                    v *= max_component_value / maximum;
            for (int c = 0; c < 3; ++c)
                add_compensated(e[c] * s.filter_weight, px.compatibility_sum[c], px.compatibility_correction[c]);
        }
        add_compensated(s.filter_weight, px.weight_sum, px.weight_correction);
        ++px.count;
    }
    return 0;
}

} // extern "C"
