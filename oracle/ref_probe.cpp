// Test infrastructure only: a C ABI over rypath's OWN host-compilable sources, compiled
// where they lie (oracle/ref.mk), used to pin the oracle's restatement.  Nothing here is
// shipped; the built library lives in oracle/_ref/.
#include "sobol_shared.h"
#include "qmc_shared.h"
#include "hero_spectrum_shared.h"
#include "packet_roulette_shared.h"
#include "offset_rounding_shared.h"
#include "light_geometry_sampling_shared.h"
#include "replay_shared.h"
#include "light_sampling.hpp"
#include "render.hpp"
#include "rgb_spectrum.hpp"
#include <metal_stdlib>
#include "conductor.h"
#include "dielectric.h"
#include "transmission.h"
#include "medium.h"

#include <cstring>
#include <vector>

namespace {
const rypath::sobol::Tables ref_tables{
#include "../third_party/pbrt/sobol_tables.inc"
};
}

extern "C" {

const void *ref_sobol_tables(void) { return &ref_tables; }

void ref_probe_sobol(const uint32_t *q, uint32_t count, uint32_t *r) {
    namespace s = rypath::sobol;
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t *a = q + 8 * i;
        const uint64_t index = s::index(ref_tables, a[0], a[1], a[2], (uint64_t(a[4]) << 32) | a[3]);
        const uint32_t value = s::word(ref_tables, index, a[5], a[6], a[7]);
        const uint32_t camera = s::word(ref_tables, index, 0, s::no_randomization, 0);
        uint32_t *o = r + 6 * i;
        o[0] = uint32_t(index);
        o[1] = uint32_t(index >> 32);
        o[2] = value;
        o[3] = s::dimension_hash(a[5], a[7]);
        const float u = s::uniform(value), c = s::camera_uniform(camera, a[0], a[1]);
        std::memcpy(o + 4, &u, 4);
        std::memcpy(o + 5, &c, 4);
    }
}

void ref_probe_philox(const uint32_t *q, uint32_t count, uint32_t *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t *a = q + 6 * i;
        const auto w = rypath_replay::philox({a[0], a[1], a[2], a[3]}, {a[4], a[5]});
        r[4 * i] = w.x;
        r[4 * i + 1] = w.y;
        r[4 * i + 2] = w.z;
        r[4 * i + 3] = w.w;
    }
}

void ref_probe_wavelengths(const float *u, uint32_t count, uint32_t mode, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const auto w = mode == 1 ? rypath_hero::sample_visible(u[i]) : rypath_hero::sample_uniform(u[i]);
        for (int k = 0; k < 4; ++k) {
            r[8 * i + k] = w.lambda[k];
            r[8 * i + 4 + k] = w.pdf[k];
        }
    }
}

void ref_probe_advance(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 20 * i;
        rypath_hero::Density prefix;
        rypath_hero::Vector beta, num, pdf;
        for (int k = 0; k < 4; ++k) {
            prefix.lane[k].fraction = a[k];
            prefix.lane[k].exponent = int(a[4 + k]);
            beta[k] = a[8 + k];
            num[k] = a[12 + k];
            pdf[k] = a[16 + k];
        }
        const auto u = rypath_hero::advance(prefix, beta, num, pdf);
        float *o = r + 13 * i;
        for (int k = 0; k < 4; ++k) {
            o[k] = u.beta[k];
            o[4 + k] = u.density.lane[k].fraction;
            o[8 + k] = float(u.density.lane[k].exponent);
        }
        o[12] = u.valid ? 1.f : 0.f;
    }
}

// Same layout as or_probe_bsdf.
void ref_probe_bsdf(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 16 * i;
        float *o = r + 12 * i;
        std::fill(o, o + 12, 0.0f);
        const float3 wo(a[6], a[7], a[8]), wi(a[9], a[10], a[11]);
        const float2 u(a[13], a[14]);
        const unsigned kind = unsigned(a[0]);
        rypath_conductor::Evaluation e{0, 0, false};
        rypath_conductor::Sample s{};
        float eta = 1;
        if (kind == 0) {
            e = rypath_transmission::diffuse_evaluate(a[1], 0, wo, wi);
            // packet diffuse sampling uses the concentric map (shaders/packet_scattering.h)
            o[2] = e.valid ? 1.f : 0.f;
            o[0] = e.f;
            o[1] = e.pdf;
            o[8] = -1; // sampling not probed here
            continue;
        } else if (kind == 1) {
            rypath_conductor::Parameters p;
            if (!rypath_conductor::prepare(a[1], a[2], a[3], a[4], a[5] != 0, p)) {
                o[2] = -1;
                continue;
            }
            e = rypath_conductor::evaluate(p, wo, wi);
            s = rypath_conductor::sample(p, wo, u);
        } else {
            rypath_dielectric::Parameters p;
            if (!rypath_dielectric::prepare(a[1], a[3], a[4], a[5] != 0, p)) {
                o[2] = -1;
                continue;
            }
            e = rypath_dielectric::evaluate(p, wo, wi);
            s = rypath_dielectric::sample(p, wo, a[12], u, eta);
        }
        o[0] = e.f;
        o[1] = e.pdf;
        o[2] = e.valid ? 1.f : 0.f;
        o[3] = s.wi.x;
        o[4] = s.wi.y;
        o[5] = s.wi.z;
        o[6] = s.weight;
        o[7] = s.pdf;
        o[8] = float((s.delta ? 1 : 0) | (s.accepted ? 2 : 0) | (s.valid ? 4 : 0));
        o[9] = eta;
    }
}

int ref_build_light_tables(const double *rows, uint32_t count, uint32_t *alias, uint32_t *records,
                           uint32_t *nodes, uint32_t *infinite, uint32_t *infinite_count) {
    std::vector<rypath::LightSamplingInput> in(count);
    for (uint32_t i = 0; i < count; ++i) {
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
    std::string error;
    const auto t = rypath::build_light_sampling(in, SIZE_MAX, error);
    if (!t)
        return -1;
    std::memcpy(alias, t->alias.data(), t->alias.size() * 16);
    std::memcpy(records, t->records.data(), t->records.size() * 16);
    std::memcpy(nodes, t->nodes.data(), t->nodes.size() * 64);
    std::memcpy(infinite, t->infinite.data(), t->infinite.size() * 4);
    *infinite_count = uint32_t(t->infinite.size());
    return int(t->nodes.size());
}

double ref_light_spectrum_power(const float *spectrum) {
    std::array<float, 471> s;
    std::copy(spectrum, spectrum + 471, s.begin());
    return rypath::light_spectrum_power(s);
}

uint32_t ref_outward(uint32_t bits, int toward_negative, int *valid) {
    const auto r = rypath_offset_rounding::outward(bits, toward_negative != 0);
    *valid = r.valid;
    return r.bits;
}

// Packet film reduction through the reference's own PacketFilmBatch
// (src/packet_film.cpp); pbrt_cie_xyz is supplied below from the same CIE table.
static std::vector<double> g_cie;
// shaders/medium.h, in the or_probe_medium layout (oracle.h)
void ref_probe_medium(const float *q, uint32_t count, float *r) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 15 * i;
        float *o = r + 8 * i;
        const auto seg = rypath_medium::segment(a[0], a[1], a[2], a[3]);
        o[0] = seg.transmission;
        o[1] = seg.emission;
        o[2] = seg.valid ? 1.0f : 0.0f;
        o[3] = rypath_medium::flight(a[4], a[5]);
        o[4] = rypath_medium::phase(float3(a[6], a[7], a[8]), float3(a[9], a[10], a[11]), a[12]);
        const float3 w = rypath_medium::phase_sample(float3(a[6], a[7], a[8]), a[12], float2(a[13], a[14]));
        o[5] = w.x;
        o[6] = w.y;
        o[7] = w.z;
    }
}

// src/qmc_shared.h in the or_probe_qmc layout
void ref_probe_qmc(const int64_t *queries, uint32_t count, uint64_t *results) {
    namespace q = rypath::qmc;
    namespace s = rypath::sobol;
    for (uint32_t i = 0; i < count; ++i) {
        const int64_t *a = queries + 10 * i;
        const unsigned w = unsigned(a[1]), h = unsigned(a[2]), x = unsigned(a[3]), y = unsigned(a[4]),
                       d = unsigned(a[6]), mode = unsigned(a[7]), seed = unsigned(a[8]), spp = unsigned(a[9]);
        const uint64_t sample = uint64_t(a[5]);
        uint64_t *o = results + 6 * i;
        if (a[0] == 2) {
            const auto index = q::halton_index(w, h, x, y, sample);
            o[0] = 0;
            o[1] = q::float_bits(q::halton_camera(0, w, index));
            o[2] = q::float_bits(q::halton_camera(1, h, index));
            o[3] = o[4] = q::float_bits(q::radical(d, index, mode, seed));
            o[5] = q::float_bits(q::radical(d + 1, index, mode, seed));
        } else {
            const unsigned v = std::max({w, h, 1u}) - 1;
            const unsigned m = v == 0 ? 0 : 32 - __builtin_clz(v);
            const unsigned log = 31 - __builtin_clz(spp);
            const auto morton = q::morton(x, y, log, sample);
            o[0] = q::zindex(morton, d, m, log);
            o[1] = q::float_bits(s::uniform(q::zword(ref_tables, morton, 1, 0, true, m, log, mode, seed)));
            o[2] = q::float_bits(s::uniform(q::zword(ref_tables, morton, 1, 1, true, m, log, mode, seed)));
            o[3] = q::float_bits(s::uniform(q::zword(ref_tables, morton, d, 0, false, m, log, mode, seed)));
            o[4] = q::float_bits(s::uniform(q::zword(ref_tables, morton, d, 0, true, m, log, mode, seed)));
            o[5] = q::float_bits(s::uniform(q::zword(ref_tables, morton, d, 1, true, m, log, mode, seed)));
        }
    }
}

void ref_set_cie(const double *cie) { g_cie.assign(cie, cie + 3 * 471); }
// PacketFilmBatch with a film clamp: per pixel sum[3], correction[3], weight sum, weight
// correction, count, compatibility sum[3], compatibility correction[3] (15 doubles).
int ref_film_add_clamped(const uint32_t *words, size_t count, uint32_t width, uint32_t height, double exposure,
                         double max_component_value, double *out);
int ref_film_add(const uint32_t *words, size_t count, uint32_t width, uint32_t height,
                 double *out_sum_weight_count) {
    std::vector<double> full(size_t(width) * height * 15);
    const int rc = ref_film_add_clamped(words, count, width, height, 1.0, INFINITY, full.data());
    for (size_t p = 0; rc == 0 && p < size_t(width) * height; ++p)
        std::memcpy(out_sum_weight_count + 9 * p, full.data() + 15 * p, 9 * sizeof(double));
    return rc;
}
int ref_film_add_clamped(const uint32_t *words, size_t count, uint32_t width, uint32_t height, double exposure,
                         double max_component_value, double *out) {
    rypath::RenderScene scene{};
    scene.model = rypath::RenderModel::pbrt;
    scene.exposure = exposure;
    scene.max_component_value = max_component_value;
    rypath::RenderSettings settings{};
    settings.width = width;
    settings.height = height;
    auto film = rypath::make_packet_film(scene, settings);
    const size_t pixels = size_t(width) * height;
    if (count % pixels)
        return -2;
    rypath::PacketFilmBatch batch(film, count / pixels);
    std::vector<rypath::PacketSample> samples(count);
    for (size_t i = 0; i < count; ++i) {
        const uint32_t *w = words + 20 * i; // rp_packet_result layout
        auto &s = samples[i];
        s.pixel = w[1];
        s.sample = (uint64_t(w[3]) << 32) | w[2];
        std::memcpy(s.wavelengths.data(), w + 5, 16);
        std::memcpy(s.wavelength_pdfs.data(), w + 9, 16);
        std::memcpy(s.radiance.data(), w + 13, 16);
        std::memcpy(&s.filter_weight, w + 17, 4);
    }
    if (!batch.add(samples, {}).empty())
        return -1;
    if (!batch.commit(film).empty())
        return -3;
    for (size_t p = 0; p < pixels; ++p) {
        const auto &px = film.pixels[p];
        double *o = out + 15 * p;
        for (int c = 0; c < 3; ++c) {
            o[c] = px.sum[c];
            o[3 + c] = px.correction[c];
            o[9 + c] = px.compatibility_sum[c];
            o[12 + c] = px.compatibility_correction[c];
        }
        o[6] = px.weight_sum;
        o[7] = px.weight_correction;
        o[8] = double(px.count);
    }
    return 0;
}

} // extern "C"

namespace rypath {
std::array<double, 3> pbrt_cie_xyz(double wavelength) {
    if (!(wavelength >= 360 && wavelength <= 830) || g_cie.empty())
        return {};
    const size_t row = size_t(std::round(wavelength) - 360);
    return {g_cie[3 * row], g_cie[3 * row + 1], g_cie[3 * row + 2]};
}
} // namespace rypath

// Link stand-ins for reference symbols that live in translation units this pin does not
// compile (src/render.cpp, src/rgb_spectrum.cpp, src/image_texture.cpp).  Only make_film
// is reached by the probes above; the image/sRGB entries are never called.
namespace rypath {
Film make_film(std::uint32_t width, std::uint32_t height, RenderModel model, double exposure) {
    Film f{};
    f.width = width;
    f.height = height;
    f.pixels.resize(std::size_t(width) * height);
    f.model = model;
    f.exposure = exposure;
    return f;
}
std::array<double, 3> film_mean(const FilmPixel &) { return {}; }
std::optional<RgbSpectrum> reconstruct_srgb(const std::array<float, 3> &) { return {}; }
float evaluate_srgb(const RgbSpectrum &, float) { return 0; }
std::optional<std::array<float, 3>> image_base_texel_linear_rgb(const ImagePyramid &, unsigned, unsigned) {
    return {};
}
const std::array<float, 471> &pbrt_d65() {
    static const std::array<float, 471> zero{};
    return zero;
}
} // namespace rypath
