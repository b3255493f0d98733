// Test infrastructure only: rypath's hero-transport shader headers compiled where they lie
// (oracle/ref.mk), behind the host stand-in for <metal_stdlib>, as a C ABI that pins the
// oracle's restatement.  The hero scattering header (shaders/hero_scattering.h, with the
// packet BSDF headers it includes) and the hero path helpers (shaders/hero_pt_helpers.h) are
// rypath's own code; the few declarations below only give the helpers' unused functions
// something to name (rypath includes them inside its transport namespace, after the light,
// visibility and random-number helpers): none of them is called.
#include <metal_stdlib>
#include "hero_spectrum_shared.h"
#include "packet_spectrum_shared.h"
#include "render_wire.h"
#include "replay_shared.h"
#include "hero_scattering.h"

#include <algorithm>
#include <cstdint>

namespace rypath_light_sampling {
template <class... A> float pmf(A &&...);
}
namespace rypath_light_geometry {
template <class... A> float pdf(A &&...);
}
namespace ref_hero {
namespace wire = rypath::render_wire;
using Wavelengths = rypath_packet_spectrum::Wavelengths;
using Mode = rypath_packet::TransportMode;
enum : uint { camera_vertex, surface_vertex, light_vertex, environment_vertex };
// shaders/render.metal:2418 and shaders/packet_transport.h:49-50, as the helpers name them
inline bool packet_hero_enabled(const wire::Parameters &) { return true; }
inline bool nonzero(float4 v) { return any(v > 0); }
inline bool finite_nonnegative(float4 v) { return all(isfinite(v)) && all(v >= 0); }
// names the light-sample and random-number templates refer to (never instantiated)
struct Alpha {
    const wire::Parameters *parameters;
    const device uint *material_data;
};
struct Resources {
    Alpha alpha;
};
template <typename T> struct HeroDirectEndpoint {
    using Type = T;
};
uint4 random(const Resources &, const wire::Sample &, ulong, uint, const rypath_replay::ReplayState *);
float4 uniforms4(const wire::Parameters &, uint4);
#include "hero_frozen_bsdf.h"
bool hero_current_connectible(const HeroFrozenBSDF &);
bool hero_current_requires_single(const HeroFrozenBSDF &);
#include "hero_pt_helpers.h"
} // namespace ref_hero

namespace {
namespace hs = rypath_hero_scattering;

// One packet BSDF of four lanes of one family from a probe query (layout: or_probe_hero).
bool prepare_query(const float *a, rypath_packet::Prepared &p) {
    p = {};
    p.active_mask = unsigned(a[1]);
    const bool remap = a[2] != 0;
    bool ok = true;
    for (int k = 0; k < 4; ++k) {
        const float *l = a + 4 + 4 * k;
        rypath_scattering::Prepared &lane = p.lane[k];
        lane.kind = unsigned(a[0]);
        if (lane.kind == 0)
            lane.reflectance = l[0];
        else if (lane.kind == 1)
            ok = rypath_conductor::prepare(l[0], l[1], l[2], l[3], remap, lane.conductor) && ok;
        else
            ok = rypath_dielectric::prepare(l[0], l[2], l[3], remap, lane.dielectric) && ok;
    }
    return ok;
}
} // namespace

extern "C" {

// rypath_hero_scattering::sample / evaluate / dirac_lane (shaders/hero_scattering.h:67-231) and
// hero_connectible (shaders/hero_pt_helpers.h:18-23); query and result layout of or_probe_hero.
void ref_probe_hero(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 32 * i;
        float *o = r + 32 * i;
        std::fill(o, o + 32, 0.0f);
        rypath_packet::Prepared p;
        const bool ok = prepare_query(a, p);
        o[30] = ok ? 1.f : 0.f;
        if (!ok)
            continue;
        const float3 wo(a[20], a[21], a[22]), wi(a[23], a[24], a[25]);
        const float2 u(a[27], a[28]);
        const hs::Sample s = hs::sample(p, wo, a[26], u, 0);
        o[0] = s.wi.x;
        o[1] = s.wi.y;
        o[2] = s.wi.z;
        for (int k = 0; k < 4; ++k) {
            o[3 + k] = s.numerator[k];
            o[7 + k] = s.pdf[k];
            o[11 + k] = s.eta[k];
        }
        o[15] = float((s.delta ? 1 : 0) | (s.transmission ? 2 : 0) | (s.accepted ? 4 : 0) | (s.valid ? 8 : 0));
        const hs::Evaluation e = hs::evaluate(p, wo, wi, 0);
        for (int k = 0; k < 4; ++k) {
            o[16 + k] = e.f[k];
            o[20 + k] = e.pdf[k];
        }
        o[24] = e.valid ? 1.f : 0.f;
        float mass, density, eta;
        const bool dirac = hs::dirac_lane(p.lane[0], wo, wi, u, rypath_packet::TransportMode::Radiance, mass, density, eta);
        o[25] = mass;
        o[26] = density;
        o[27] = eta;
        o[28] = dirac ? 1.f : 0.f;
        o[29] = ref_hero::hero_connectible(p) ? 1.f : 0.f;
    }
}

// hero_continue then hero_account_eta (shaders/hero_pt_helpers.h:56-98); layout of or_probe_roulette.
void ref_probe_roulette(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 16 * i;
        float *o = r + 12 * i;
        std::fill(o, o + 12, 0.0f);
        ref_hero::HeroTrack track;
        float4 beta, eta;
        for (int k = 0; k < 4; ++k) {
            beta[k] = a[k];
            track.eta_scale[k] = a[4 + k];
            eta[k] = a[12 + k];
        }
        track.roulette_enabled = a[8] != 0;
        const bool alive = ref_hero::hero_continue(beta, track, unsigned(a[9]), a[10]);
        ref_hero::hero_account_eta(track, eta, a[11] != 0);
        o[0] = alive ? 1.f : 0.f;
        for (int k = 0; k < 4; ++k) {
            o[1 + k] = beta[k];
            o[5 + k] = track.eta_scale[k];
        }
        o[9] = track.roulette_enabled ? 1.f : 0.f;
    }
}

// hero_weight (shaders/hero_pt_helpers.h:122-138); layout of or_probe_hero_weight.
void ref_probe_hero_weight(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 20 * i;
        float *o = r + 5 * i;
        rypath_hero::Density prefix;
        float4 value, sampled, other;
        for (int k = 0; k < 4; ++k) {
            prefix.lane[k].fraction = a[k];
            prefix.lane[k].exponent = int(a[4 + k]);
            value[k] = a[8 + k];
            sampled[k] = a[12 + k];
            other[k] = a[16 + k];
        }
        rypath::render_wire::Sample sample{};
        sample.status = rypath::render_wire::success;
        const float4 w = ref_hero::hero_weight(sample, prefix, value, sampled, other);
        for (int k = 0; k < 4; ++k)
            o[k] = w[k];
        o[4] = sample.status != rypath::render_wire::success ? 1.f : 0.f;
    }
}

} // extern "C"
