// C ABI of the B200 spectral path-tracing backend (include/rypath_cuda.h): scene upload,
// light-selection tables, LBVH build, wave scheduling of the wavefront kernels, device film
// and probes.  No exception crosses the boundary; every entry point returns an rp_status.
#include "../../include/rypath_cuda.h"
#include "rp_build.cuh"
#include "rp_probes.cuh"
#include "rp_volpath.cuh"
#include "rp_batch.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cfloat>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <numbers>
#include <string>
#include <vector>

using namespace rp;

namespace {

void set_diag(char *diag, size_t cap, const char *fmt, ...) {
    if (!diag || !cap)
        return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(diag, cap, fmt, ap);
    va_end(ap);
}

struct CudaError {
    cudaError_t code;
    const char *what;
};
#define RP_CHECK(call)                                                                                                 \
    do {                                                                                                               \
        const cudaError_t rp_e = (call);                                                                               \
        if (rp_e != cudaSuccess)                                                                                       \
            throw CudaError{rp_e, #call};                                                                              \
    } while (0)

struct Invalid {
    std::string what;
};
// A valid request for a part of the reference this backend does not build.
struct NotBuilt {
    std::string what;
};

// ---------------------------------------------------------------- host light tables
// PBRT light-BVH construction as rypath performs it on the host (src/light_sampling.cpp:217-572).
struct LightInput {
    double power = 0, bounds_power = -1;
    float low[3] = {0, 0, 0}, high[3] = {0, 0, 0}, direction[3] = {0, 0, 1};
    float cos_outer = -1, cos_emission = 0;
    bool two_sided = true, infinite = false;
};

// Mix materials (src/render.cpp:302-315, :1955-1995): finite amounts, children in range, no
// cycle, at most 64 nested levels, and no null interface as a child.  Empty when valid.
// validate_analytic (src/analytic.hpp:14-50): known shapes with finite, representable
// parameters inside the shaders' numerical domain.
std::string validate_analytic(const rp_analytic &a) {
    if (a.subtype < RP_ANALYTIC_SPHERE || a.subtype > RP_ANALYTIC_CYLINDER)
        return "Unknown analytic shape kind";
    for (const float x : {a.radius, a.z_min, a.z_max, a.phi_max, a.inner_radius, a.height})
        if (!std::isfinite(x))
            return "Analytic shape parameters must be finite";
    if (!(a.radius > 0 && std::isnormal(a.radius)) ||
        !(std::isnormal(a.phi_max) && a.phi_max > 0 && a.phi_max <= 2 * std::numbers::pi_v<float>))
        return "Analytic radius and angular extent must be positive and representable";
    if (a.subtype == RP_ANALYTIC_DISK) {
        if (!(a.inner_radius >= 0 && a.inner_radius < a.radius))
            return "Analytic disk requires 0 <= inner radius < radius";
    } else {
        if (!(a.z_min < a.z_max))
            return "Analytic surface requires positive height";
        if (!std::isnormal(a.z_max - a.z_min))
            return "Analytic surface height overflows or collapses in binary32";
        if (a.subtype == RP_ANALYTIC_SPHERE && (a.z_min < -a.radius || a.z_max > a.radius))
            return "Analytic sphere clipping lies outside its radius";
        if (a.subtype == RP_ANALYTIC_SPHERE && !(std::acos(a.z_min / a.radius) > std::acos(a.z_max / a.radius)))
            return "Analytic sphere angular parameterization collapses in binary32";
    }
    constexpr float minimum = 0x1p-16f, maximum = 0x1p16f;
    if (a.radius < minimum || a.radius > maximum || a.phi_max < minimum || std::abs(a.z_min) > maximum ||
        std::abs(a.z_max) > maximum || std::abs(a.height) > maximum ||
        (a.subtype == RP_ANALYTIC_DISK ? a.radius - a.inner_radius < minimum
                                       : (a.z_max - a.z_min < minimum || a.z_max - a.z_min > maximum)))
        return "Analytic parameters exceed the shader numerical domain (lengths 2^-16..2^16, angular extent >= 2^-16)";
    return {};
}

// The world-to-object map of a row-major object-to-world 3x4 matrix, in double and rounded
// once; false for a singular or non-finite matrix.
bool invert_affine(const float *m, float *out) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = f * g - d * i, Cc = d * h - e * g;
    const double det = a * A + b * B + c * Cc;
    if (!(std::abs(det) > 0) || !std::isfinite(det))
        return false;
    const double inv[9] = {A / det, (c * h - b * i) / det, (b * f - c * e) / det,
                           B / det, (a * i - c * g) / det, (c * d - a * f) / det,
                           Cc / det, (b * g - a * h) / det, (a * e - b * d) / det};
    const double t[3] = {m[3], m[7], m[11]};
    for (int r = 0; r < 3; ++r) {
        double shift = 0;
        for (int k = 0; k < 3; ++k) {
            out[4 * r + k] = float(inv[3 * r + k]);
            shift -= inv[3 * r + k] * t[k];
        }
        out[4 * r + 3] = float(shift);
    }
    for (int k = 0; k < 12; ++k)
        if (!std::isfinite(out[k]))
            return false;
    return true;
}

std::string validate_mix(const rp_scene_desc *d) {
    const u32 n = d->material_count;
    std::vector<unsigned char> state(n, 0); // 0 unvisited, 1 on the walk, 2 done
    std::vector<u32> depth(n, 0);
    std::vector<std::pair<u32, bool>> stack;
    for (u32 root = 0; root < n; ++root) {
        if (state[root] == 2)
            continue;
        stack.emplace_back(root, false);
        while (!stack.empty()) {
            const auto [index, leaving] = stack.back();
            stack.pop_back();
            if (index >= n)
                return "Mix material references an invalid child";
            const rp_material &m = d->materials[index];
            if (leaving) {
                if (m.scattering == RP_MIX) {
                    depth[index] = 1 + std::max(depth[m.first_material], depth[m.second_material]);
                    if (depth[index] > 64)
                        return "Mix material nesting exceeds 64 levels";
                }
                state[index] = 2;
                continue;
            }
            if (state[index] == 2)
                continue;
            if (state[index] == 1)
                return "Cyclic mix materials are unsupported";
            state[index] = 1;
            stack.emplace_back(index, true);
            if (m.scattering == RP_MIX) {
                if (!std::isfinite(m.mix_amount))
                    return "Mix material requires a finite amount and child-owned surface detail";
                if (m.first_material < n && m.second_material < n &&
                    (d->materials[m.first_material].scattering == RP_INTERFACE ||
                     d->materials[m.second_material].scattering == RP_INTERFACE))
                    return "Mix materials cannot contain null boundaries";
                stack.emplace_back(m.second_material, false);
                stack.emplace_back(m.first_material, false);
            }
        }
    }
    return {};
}

// The per-node terms of light_importance in the device's float operations (host compiled
// without contraction): center, squared half-diagonal, its square root, sine of the cone.
void light_node_terms(DLightBounds &node) {
    float d[3];
    for (int a = 0; a < 3; ++a) {
        node.center[a] = (node.low[a] + node.high[a]) * .5f;
        d[a] = node.high[a] - node.low[a];
    }
    node.r2 = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * .25f;
    node.radius = std::sqrt(node.r2);
    node.sin_outer = std::sqrt(std::max(0.f, 1 - node.cos_outer * node.cos_outer));
}

struct LightTables {
    std::vector<DLightAlias> alias;
    std::vector<DLightRecord> records;
    std::vector<DLightBounds> nodes;
    std::vector<u32> infinite;
};
using D3 = std::array<double, 3>;
double d3dot(D3 a, D3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double d3norm(D3 a) { return std::sqrt(d3dot(a, a)); }
D3 d3of(const float *a) { return {a[0], a[1], a[2]}; }

// union of two light bounds with a conservative normal cone (src/light_sampling.cpp:226-276)
LightInput light_union(const LightInput &a, const LightInput &b) {
    if (a.power == 0)
        return b;
    if (b.power == 0)
        return a;
    LightInput r = a;
    r.power = a.power + b.power;
    r.two_sided = a.two_sided || b.two_sided;
    r.cos_emission = std::min(a.cos_emission, b.cos_emission);
    for (int i = 0; i < 3; ++i) {
        r.low[i] = std::min(a.low[i], b.low[i]);
        r.high[i] = std::max(a.high[i], b.high[i]);
    }
    const double pi = std::numbers::pi;
    const double ta = std::acos(std::clamp(double(a.cos_outer), -1., 1.));
    const double tb = std::acos(std::clamp(double(b.cos_outer), -1., 1.));
    const D3 wa = d3of(a.direction), wb = d3of(b.direction);
    const double angle = std::acos(std::clamp(d3dot(wa, wb), -1., 1.));
    if (std::min(angle + tb, pi) <= ta)
        return r;
    if (std::min(angle + ta, pi) <= tb) {
        std::copy(b.direction, b.direction + 3, r.direction);
        r.cos_outer = b.cos_outer;
        return r;
    }
    const double theta = (ta + tb + angle) / 2 + 1e-6;
    if (theta >= pi) {
        r.cos_outer = -1;
        r.direction[0] = r.direction[1] = 0;
        r.direction[2] = 1;
        return r;
    }
    D3 tangent;
    for (int i = 0; i < 3; ++i)
        tangent[i] = wb[i] - d3dot(wa, wb) * wa[i];
    double length = d3norm(tangent);
    if (length < 1e-12) {
        const int axis = std::abs(wa[0]) < .8 ? 0 : 1;
        D3 basis{0, 0, 0};
        basis[axis] = 1;
        for (int i = 0; i < 3; ++i)
            tangent[i] = basis[i] - wa[axis] * wa[i];
        length = d3norm(tangent);
    }
    const double rotate = theta - ta;
    for (int i = 0; i < 3; ++i)
        r.direction[i] = float(std::cos(rotate) * wa[i] + std::sin(rotate) * tangent[i] / length);
    const double dl = d3norm(d3of(r.direction));
    for (int i = 0; i < 3; ++i)
        r.direction[i] = float(r.direction[i] / dl);
    r.cos_outer = std::nextafter(float(std::cos(theta)), -INFINITY);
    return r;
}
// PBRT EvaluateCost (src/light_sampling.cpp:277-292)
double light_cost(const LightInput &b, const LightInput &all, int axis) {
    if (b.power == 0)
        return 0;
    const double pi = std::numbers::pi;
    const double o = std::acos(std::clamp(double(b.cos_outer), -1., 1.));
    const double e = std::acos(std::clamp(double(b.cos_emission), -1., 1.));
    const double w = std::min(o + e, pi);
    const double omega =
        2 * pi * (1 - b.cos_outer) + pi / 2 * (2 * w * std::sin(o) - std::cos(o - 2 * w) - 2 * o * std::sin(o) + b.cos_outer);
    const D3 d{double(b.high[0]) - b.low[0], double(b.high[1]) - b.low[1], double(b.high[2]) - b.low[2]};
    const D3 ad{double(all.high[0]) - all.low[0], double(all.high[1]) - all.low[1], double(all.high[2]) - all.low[2]};
    if (ad[axis] <= 0)
        return INFINITY;
    return b.power * omega * (std::max({ad[0], ad[1], ad[2]}) / ad[axis]) * 2 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
}
// src/light_sampling.cpp:384-572
bool build_light_tables(const std::vector<LightInput> &in, LightTables &out, std::string &error) {
    out = {};
    out.records.assign(in.size(), {kNone, 0, 0, 0});
    out.alias.assign(in.size(), {0, 0, 0, 0});
    if (in.empty())
        return true;
    double total = 0, bounds_total = 0;
    std::vector<double> prob(in.size());
    std::vector<LightInput> bvh(in.begin(), in.end());
    std::vector<u32> finite;
    for (size_t i = 0; i < in.size(); ++i) {
        const auto &v = in[i];
        if (!(v.power >= 0 && std::isfinite(v.power))) {
            error = "Invalid light sampling power";
            return false;
        }
        auto &b = bvh[i];
        b.power = v.bounds_power < 0 ? v.power : v.bounds_power;
        if (b.power == 0 && v.power > 0)
            b.power = v.power;
        prob[i] = v.power == 0 && b.power > 0 ? b.power : v.power;
        total += prob[i];
        if (!v.infinite)
            bounds_total += b.power;
        if (v.infinite) {
            out.infinite.push_back(u32(i));
            out.records[i].flags = 1;
        } else if (b.power > 0)
            finite.push_back(u32(i));
    }
    if (!std::isfinite(total) || !std::isfinite(bounds_total)) {
        error = "Light sampling total power overflow";
        return false;
    }
    // Walker alias table (Vose)
    std::vector<u32> small, large;
    for (size_t i = 0; i < in.size(); ++i) {
        const double p = total > 0 ? prob[i] / total : 1. / double(in.size());
        out.alias[i].pmf = float(p);
        prob[i] = p * double(in.size());
        (prob[i] < 1 ? small : large).push_back(u32(i));
    }
    while (!small.empty() && !large.empty()) {
        const u32 s = small.back();
        small.pop_back();
        const u32 l = large.back();
        large.pop_back();
        out.alias[s].threshold = float(prob[s]);
        out.alias[s].alias = l;
        prob[l] -= 1 - prob[s];
        (prob[l] < 1 ? small : large).push_back(l);
    }
    for (u32 i : small)
        out.alias[i] = {1, out.alias[i].pmf, i, 0};
    for (u32 i : large)
        out.alias[i] = {1, out.alias[i].pmf, i, 0};
    auto bucket_of = [](const LightInput &v, int axis, const double *clo, const double *chi) {
        return std::min(11u, unsigned(12 * ((double(v.low[axis]) + v.high[axis]) / 2 - clo[axis]) / (chi[axis] - clo[axis])));
    };
    std::function<u32(size_t, size_t, u32, unsigned)> build = [&](size_t begin, size_t end, u32 parent,
                                                                 unsigned depth) -> u32 {
        const u32 index = u32(out.nodes.size());
        out.nodes.emplace_back();
        LightInput bounds;
        double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (size_t k = begin; k < end; ++k) {
            const auto &v = bvh[finite[k]];
            bounds = light_union(bounds, v);
            for (int a = 0; a < 3; ++a) {
                const double c = (double(v.low[a]) + v.high[a]) / 2;
                clo[a] = std::min(clo[a], c);
                chi[a] = std::max(chi[a], c);
            }
        }
        DLightBounds node{};
        node.parent = parent;
        node.light = kNone;
        for (int a = 0; a < 3; ++a) {
            node.low[a] = bounds.low[a];
            node.high[a] = bounds.high[a];
            node.direction[a] = bounds.direction[a];
        }
        node.power = float(bounds.power / bounds_total);
        node.cos_outer = bounds.cos_outer;
        node.cos_emission = bounds.cos_emission;
        node.flags = bounds.two_sided ? 1 : 0;
        light_node_terms(node);
        if (end - begin == 1) {
            node.light = finite[begin];
            out.records[finite[begin]].leaf = index;
        } else {
            double best = INFINITY;
            int split_axis = 0;
            unsigned split_bucket = 0;
            bool found = false;
            if (depth < 48)
                for (int axis = 0; axis < 3; ++axis) {
                    if (clo[axis] == chi[axis])
                        continue;
                    std::array<LightInput, 12> buckets{};
                    for (size_t k = begin; k < end; ++k) {
                        const auto &v = bvh[finite[k]];
                        const unsigned b = bucket_of(v, axis, clo, chi);
                        buckets[b] = light_union(buckets[b], v);
                    }
                    for (unsigned split = 1; split < 11; ++split) {
                        LightInput l, r;
                        for (unsigned k = 0; k <= split; ++k)
                            l = light_union(l, buckets[k]);
                        for (unsigned k = split + 1; k < 12; ++k)
                            r = light_union(r, buckets[k]);
                        const double c = light_cost(l, bounds, axis) + light_cost(r, bounds, axis);
                        if (c > 0 && c < best) {
                            best = c;
                            split_axis = axis;
                            split_bucket = split;
                            found = true;
                        }
                    }
                }
            size_t mid = begin + (end - begin) / 2;
            if (found) {
                auto it = std::stable_partition(finite.begin() + std::ptrdiff_t(begin), finite.begin() + std::ptrdiff_t(end),
                                                [&](u32 id) { return bucket_of(bvh[id], split_axis, clo, chi) <= split_bucket; });
                const size_t candidate = size_t(it - finite.begin());
                if (candidate > begin && candidate < end)
                    mid = candidate;
            }
            build(begin, mid, index, depth + 1);
            node.child = build(mid, end, index, depth + 1);
        }
        out.nodes[index] = node;
        return index;
    };
    if (!finite.empty())
        build(0, finite.size(), kNone, 0);
    return true;
}

// src/packet_spectrum_shared.h:33-59 and src/light_sampling.cpp:17-27
double light_spectrum_power(const float *spectrum) {
    double value = 0;
    for (int i = 0; i < 4; ++i) {
        float up = .5f + float(i) * .25f;
        if (up > 1)
            up -= 1;
        float w = 538 - 138.888889f * std::atanh(.85691062f - 1.82750197f * up);
        w = std::clamp(w, 360.f, 830.f);
        const float c = std::cosh(.0072f * (w - 538));
        const float pdf = .0039398042f / (c * c);
        value += double(spectrum[unsigned(std::round(w) - 360)]) / pdf / 4;
    }
    if (value == 0)
        for (int i = 0; i < 471; ++i)
            value += spectrum[i];
    return value;
}

// ---------------------------------------------------------------- images on the host
// The scene-build side of the image inputs: texel decoding for the environment tables and
// light power, rypath's host sRGB reconstruction (src/rgb_spectrum.cpp:62-127), the
// environment importance tables (src/environment_sampling.cpp:20-115) and the environment
// light's power (src/light_sampling.cpp:28-95).
float half_to_float_host(u32 bits) {
    const u32 sign = (bits & 0x8000u) << 16, e = (bits >> 10) & 31u, m = bits & 1023u;
    u32 out;
    if (e == 0) {
        if (m == 0)
            out = sign;
        else {
            const u32 top = 31u - u32(__builtin_clz(m));
            out = sign | ((103u + top) << 23) | ((m << (23u - top)) & 0x7fffffu);
        }
    } else {
        out = sign | ((e == 31u ? 255u : e + 112u) << 23) | (m << 13);
    }
    float f;
    memcpy(&f, &out, 4);
    return f;
}
u32 texel_words(u32 format) { return format == RP_TEXELS_FLOAT ? 4u : format == RP_TEXELS_HALF ? 2u : 1u; }
// Linear RGB of texel (x, y) of a level; false when a channel is not finite
// (image_base_texel_linear_rgb, src/image_texture.cpp:1324-1332).
bool host_texel(const rp_images &im, const rp_image_texture &t, const rp_texture_level &l, u32 x, u32 y,
                float rgb[3]) {
    const size_t index = size_t(y) * l.width + x;
    if (t.texel_format == RP_TEXELS_FLOAT) {
        memcpy(rgb, im.texels + l.offset + 4 * index, 12);
    } else if (t.texel_format == RP_TEXELS_HALF) {
        const u32 rg = im.texels[l.offset + 2 * index], b = im.texels[l.offset + 2 * index + 1];
        rgb[0] = half_to_float_host(rg & 0xffffu);
        rgb[1] = half_to_float_host(rg >> 16);
        rgb[2] = half_to_float_host(b & 0xffffu);
    } else {
        const u32 v = im.texels[l.offset + index];
        const float *lut = im.transfer + t.transfer_offset;
        rgb[0] = lut[v & 255u];
        rgb[1] = lut[(v >> 8) & 255u];
        rgb[2] = lut[(v >> 16) & 255u];
    }
    return std::isfinite(rgb[0]) && std::isfinite(rgb[1]) && std::isfinite(rgb[2]);
}
// reconstruct_srgb + evaluate_srgb at one wavelength; rgb in [0, 1]
bool host_srgb_spectrum(const float *table, const float rgb[3], float wavelength, float &value) {
    for (int c = 0; c < 3; ++c)
        if (!std::isfinite(rgb[c]) || rgb[c] < 0 || rgb[c] > 1)
            return false;
    if (rgb[0] == rgb[1] && rgb[1] == rgb[2]) {
        value = rgb[0];
        return true;
    }
    int top = 0; // the last of tied maxima
    for (int c = 1; c < 3; ++c)
        if (rgb[c] >= rgb[top])
            top = c;
    const float z = rgb[top];
    const float x = rgb[(top + 1) % 3] * 63 / z, y = rgb[(top + 2) % 3] * 63 / z;
    const int xi = std::min(int(x), 62), yi = std::min(int(y), 62);
    const float *nodes = table;
    const int zi = int(std::lower_bound(nodes + 1, nodes + 63, z) - nodes) - 1;
    const float dx = x - float(xi), dy = y - float(yi), dz = (z - nodes[zi]) / (nodes[zi + 1] - nodes[zi]);
    const auto lerp = [](float t, float a, float b) { return (1.0f - t) * a + t * b; };
    float co[3];
    for (int i = 0; i < 3; ++i) {
        const auto at = [&](int ox, int oy, int oz) {
            return table[64 + 3 * (((top * 64 + zi + oz) * 64 + yi + oy) * 64 + xi + ox) + i];
        };
        co[i] = lerp(dz, lerp(dy, lerp(dx, at(0, 0, 0), at(1, 0, 0)), lerp(dx, at(0, 1, 0), at(1, 1, 0))),
                     lerp(dy, lerp(dx, at(0, 0, 1), at(1, 0, 1)), lerp(dx, at(0, 1, 1), at(1, 1, 1))));
    }
    const float poly = std::fma(wavelength, std::fma(wavelength, co[0], co[1]), co[2]);
    if (!std::isfinite(poly)) {
        value = NAN;
        return true;
    }
    if (std::abs(poly) <= 1.0f) {
        value = 0.5f + 0.5f * (poly / std::sqrt(1.0f + poly * poly));
    } else {
        const float r = 1.0f / poly;
        value = 0.5f + 0.5f * std::copysign(1.0f / std::sqrt(1.0f + r * r), poly);
    }
    return true;
}
// light_rgb_power (src/light_sampling.cpp:28-44): the RGB illuminant's spectrum at the four
// visible hero wavelengths of u = 0.5, over their densities.
bool light_rgb_power(const rp_images &im, const float rgb[3], double &value) {
    const float amplitude = 2 * std::max({rgb[0], rgb[1], rgb[2]});
    value = 0;
    if (amplitude == 0)
        return true;
    if (!std::isfinite(amplitude))
        return false;
    const float normalized[3] = {rgb[0] / amplitude, rgb[1] / amplitude, rgb[2] / amplitude};
    for (int i = 0; i < 3; ++i)
        if (!(normalized[i] >= 0 && normalized[i] <= 1))
            return false;
    for (int i = 0; i < 4; ++i) {
        float up = .5f + float(i) * .25f;
        if (up > 1)
            up -= 1;
        float w = 538 - 138.888889f * std::atanh(.85691062f - 1.82750197f * up);
        w = std::clamp(w, 360.f, 830.f);
        const float c = std::cosh(.0072f * (w - 538));
        const float pdf = .0039398042f / (c * c);
        const unsigned bin = unsigned(std::round(w) - 360);
        float spectral;
        host_srgb_spectrum(im.rgb_table, normalized, float(bin + 360), spectral);
        value += double(amplitude) * spectral * im.illuminant[bin] / pdf / 4;
    }
    return true;
}
// The environment image's full and compensated importance tables (a marginal CDF then one
// conditional CDF per row, each width + 1 floats; the compensated table keeps only the mass
// above the mean) and its mean RGB power (light_image_power).
std::string environment_tables(const rp_images &im, std::vector<float> &cdf, u32 &width, u32 &compensated_offset,
                               double &mean_power) {
    const rp_image_texture &t = im.textures[im.environment_image];
    const rp_texture_level &l = im.levels[t.level_begin];
    if (t.level_count != 1 || l.width != l.height)
        return "Environment sampling requires a square native image base";
    width = l.width;
    const size_t side = size_t(width) + 1;
    compensated_offset = u32(side * side);
    cdf.assign(2 * side * side, 0.f);
    std::vector<double> mass(size_t(width) * width), full_rows(width), comp_rows(width), full_prefix(side),
        comp_prefix(side);
    double total = 0, power = 0;
    for (u32 y = 0; y < width; ++y) {
        double row = 0;
        for (u32 x = 0; x < width; ++x) {
            float rgb[3];
            if (!host_texel(im, t, l, x, y, rgb))
                return "Environment sampling texel is invalid";
            const double v =
                (double(std::max(rgb[0], 0.f)) + double(std::max(rgb[1], 0.f)) + double(std::max(rgb[2], 0.f))) / 3;
            mass[size_t(y) * width + x] = v;
            row += v;
            double p;
            if (!light_rgb_power(im, rgb, p))
                return "Invalid environment light sampling image";
            power += p;
        }
        full_rows[y] = row;
        total += row;
    }
    mean_power = power / (double(width) * width);
    const double average = total / (double(width) * width);
    const auto write_prefix = [&](size_t offset, const std::vector<double> &prefix, double sum) {
        for (u32 x = 1; x <= width; ++x)
            cdf[offset + x] = sum > 0 ? float(prefix[x] / sum) : float(x) / float(width);
        cdf[offset + width] = 1.f;
    };
    double comp_total = 0;
    for (u32 y = 0; y < width; ++y) {
        full_prefix[0] = comp_prefix[0] = 0;
        for (u32 x = 0; x < width; ++x) {
            const double v = mass[size_t(y) * width + x];
            full_prefix[x + 1] = full_prefix[x] + v;
            comp_prefix[x + 1] = comp_prefix[x] + std::max(v - average, 0.);
        }
        comp_rows[y] = comp_prefix[width];
        comp_total += comp_rows[y];
        write_prefix(side * (y + 1), full_prefix, full_rows[y]);
        write_prefix(compensated_offset + side * (y + 1), comp_prefix, comp_rows[y]);
    }
    double full_sum = 0, comp_sum = 0;
    for (u32 y = 0; y < width; ++y) {
        full_sum += full_rows[y];
        comp_sum += comp_rows[y];
        cdf[y + 1] = total > 0 ? float(full_sum / total) : float(y + 1) / float(width);
        cdf[compensated_offset + y + 1] = comp_total > 0 ? float(comp_sum / comp_total) : float(y + 1) / float(width);
    }
    cdf[width] = cdf[compensated_offset + width] = 1.f;
    return {};
}
// Structural checks of the image inputs (valid ranges and sizes; texel values are checked
// where they are read).
std::string validate_images(const rp_scene_desc *d) {
    const rp_images *im = d->images;
    if (!im)
        return {};
    if ((im->texture_count && !im->textures) || (im->level_count && !im->levels) ||
        (im->texel_word_count && !im->texels) || (im->transfer_count && !im->transfer))
        return "image arrays must be given with their counts";
    if (im->texture_count && (!im->rgb_table || !im->illuminant))
        return "images need the sRGB reconstruction table and the D65 illuminant";
    for (u32 i = 0; i < im->texture_count; ++i) {
        const rp_image_texture &t = im->textures[i];
        if (t.gltf)
            return "glTF image textures are not built";
        if (t.level_count == 0 || t.level_count > 14 || t.level_begin > im->level_count ||
            t.level_count > im->level_count - t.level_begin || t.texel_format > RP_TEXELS_FLOAT || t.wrap > 2 ||
            t.filter > RP_TEXTURE_EWA || (t.channels != 1 && t.channels != 3 && t.channels != 4))
            return "invalid image texture descriptor";
        if (t.texel_format < RP_TEXELS_HALF && (t.transfer_offset > im->transfer_count ||
                                                im->transfer_count - t.transfer_offset < 256))
            return "8-bit image texture needs 256 transfer values";
        for (u32 k = 0; k < t.level_count; ++k) {
            const rp_texture_level &l = im->levels[t.level_begin + k];
            const uint64_t words = uint64_t(l.width) * l.height * texel_words(t.texel_format);
            if (l.width == 0 || l.height == 0 || l.width > 8192 || l.height > 8192 || l.offset > im->texel_word_count ||
                words > im->texel_word_count - l.offset)
                return "image level outside the texel words";
        }
    }
    if (im->environment_image != RP_NONE) {
        if (im->environment_image >= im->texture_count)
            return "environment image out of range";
        if (!std::isfinite(im->environment_scale) || im->environment_scale < 0)
            return "environment image scale must be finite and nonnegative";
        for (float v : im->environment_from_world)
            if (!std::isfinite(v))
                return "environment transform must be finite";
    }
    return {};
}

// ---------------------------------------------------------------- Gaussian pixel filter
// compile_gaussian_filter (src/gaussian_filter.cpp:84-137): PBRT's Gaussian filter minus its
// value at the radius, tabulated at 32 cells per unit radius at cell midpoints, with PBRT's
// FastExp, normalised as a 2-D piecewise-constant distribution (conditional rows of width + 1
// entries, then the marginal of height + 1).
struct GaussianTable {
    u32 width = 0, height = 0;
    std::vector<float> conditional, marginal;
    float integral = 0;
};
float pbrt_fast_exp(float x) {
    if (x < -100.f)
        return 0;
    const float xp = x * 1.442695041f;
    const float fxp = std::floor(xp);
    const float f = xp - fxp;
    const int i = int(fxp);
    const float poly = std::fma(f, std::fma(f, std::fma(f, 0.0781455737f, 0.226173572f), 0.695556856f), 1.f);
    uint32_t bits;
    memcpy(&bits, &poly, 4);
    const int exponent = int((bits >> 23) & 255) - 127 + i;
    if (exponent < -126)
        return 0;
    bits = (bits & 0x807fffffu) | (uint32_t(exponent + 127) << 23);
    float out;
    memcpy(&out, &bits, 4);
    return out;
}
float lerp_pbrt(float t, float a, float b) { return (1 - t) * a + t * b; }
bool cdf_of(const float *values, size_t n, float radius, float *cdf, float &integral) {
    cdf[0] = 0;
    for (size_t i = 0; i < n; ++i) {
        cdf[i + 1] = cdf[i] + values[i] * (2 * radius) / float(n);
        if (!std::isfinite(cdf[i + 1]))
            return false;
    }
    integral = cdf[n];
    if (integral > 0 && !std::isnormal(integral))
        return false;
    if (integral == 0) {
        for (size_t i = 1; i <= n; ++i)
            cdf[i] = float(i) / float(n);
    } else {
        for (size_t i = 1; i <= n; ++i)
            cdf[i] /= integral;
    }
    for (size_t i = 1; i <= n; ++i) {
        const float gap = cdf[i] - cdf[i - 1];
        if (!std::isfinite(cdf[i]) || (cdf[i] > 0 && !std::isnormal(cdf[i])) || (gap > 0 && !std::isnormal(gap)))
            return false;
    }
    return true;
}
std::string gaussian_table(float xr, float yr, float sigma, GaussianTable &g) {
    if (!std::isnormal(xr) || xr <= 0 || !std::isnormal(yr) || yr <= 0 || !std::isnormal(sigma) || sigma <= 0)
        return "Gaussian radii and sigma must be positive normal binary32 values";
    const float nx = 32 * xr, ny = 32 * yr;
    if (!(nx >= 1 && nx < 4096 + 1.f && ny >= 1 && ny < 4096 + 1.f))
        return "Gaussian table axis must contain 1 to 4096 cells";
    g.width = u32(nx);
    g.height = u32(ny);
    if (uint64_t(g.width) * g.height > 1048576)
        return "Gaussian table exceeds the 1048576-cell limit";
    const float denominator = 2 * std::numbers::pi_v<float> * sigma * sigma;
    const float two_sigma_squared = 2 * sigma * sigma;
    const float scale = 1 / std::sqrt(denominator);
    if (!(denominator > 0 && std::isfinite(denominator) && two_sigma_squared > 0 && std::isfinite(two_sigma_squared) &&
          std::isfinite(scale)))
        return "Gaussian sigma arithmetic overflows or collapses in binary32";
    auto gaussian = [&](float x) { return scale * pbrt_fast_exp(-(x * x) / two_sigma_squared); };
    const float exp_x = gaussian(xr), exp_y = gaussian(yr);
    g.conditional.assign(size_t(g.height) * (g.width + 1), 0.f);
    g.marginal.assign(g.height + 1, 0.f);
    std::vector<float> values(g.width), rows(g.height);
    for (u32 y = 0; y < g.height; ++y) {
        const float py = lerp_pbrt((float(y) + 0.5f) / float(g.height), -yr, yr);
        const float fy = std::max(0.f, gaussian(py) - exp_y);
        for (u32 x = 0; x < g.width; ++x) {
            const float px = lerp_pbrt((float(x) + 0.5f) / float(g.width), -xr, xr);
            values[x] = std::max(0.f, gaussian(px) - exp_x) * fy;
            if (!std::isfinite(values[x]))
                return "Gaussian table contains nonfinite binary32 values";
        }
        if (!cdf_of(values.data(), g.width, xr, g.conditional.data() + size_t(y) * (g.width + 1), rows[y]))
            return "Gaussian conditional distribution overflows or collapses in binary32";
    }
    float integral = 0;
    if (!cdf_of(rows.data(), g.height, yr, g.marginal.data(), integral) || !(integral > 0))
        return "Gaussian table has a zero or nonfinite binary32 integral";
    g.integral = integral;
    return {};
}

// ---------------------------------------------------------------- device buffers
// Device memory comes from the device's stream-ordered pool, configured to keep freed memory
// for reuse by the next scene or pool in this process (no trip to the driver per render job).
// cudaGetDeviceProperties queries every property (milliseconds); scene creation asks once per
// device and process.
const cudaDeviceProp &device_properties(int device) {
    static std::mutex mutex;
    static std::map<int, cudaDeviceProp> cache;
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find(device);
    if (it == cache.end()) {
        cudaDeviceProp prop;
        RP_CHECK(cudaGetDeviceProperties(&prop, device));
        it = cache.emplace(device, prop).first;
    }
    return it->second;
}
void retain_pool(int device) {
    static bool configured[64] = {};
    if (device >= 0 && device < 64 && !configured[device]) {
        cudaMemPool_t pool;
        RP_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t threshold = UINT64_MAX;
        RP_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        configured[device] = true;
    }
}
template <class T> T *dalloc(std::vector<void *> &owned, size_t count, cudaStream_t st = nullptr) {
    void *p = nullptr;
    RP_CHECK(cudaMallocAsync(&p, std::max<size_t>(1, count) * sizeof(T), st));
    owned.push_back(p);
    return static_cast<T *>(p);
}
template <class T> T *dupload(std::vector<void *> &owned, const T *src, size_t count, cudaStream_t st) {
    T *p = dalloc<T>(owned, count, st);
    if (count)
        RP_CHECK(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    return p;
}

// Upload a description's images in their wire layout; an environment image also gets its
// importance tables and its light power (mean RGB illuminant power times its scale; -1 when
// there is no environment image).
void upload_images(const rp_images *im, u32 instances, DImages &g, std::vector<void *> &own, cudaStream_t stm,
                   double &env_power) {
    static_assert(sizeof(DImageTexture) == sizeof(rp_image_texture) && sizeof(DLevel) == sizeof(rp_texture_level));
    g = DImages{};
    g.env_image = kNone;
    env_power = -1;
    if (!im)
        return;
    g.textures = dupload(own, reinterpret_cast<const DImageTexture *>(im->textures), im->texture_count, stm);
    g.levels = dupload(own, reinterpret_cast<const DLevel *>(im->levels), im->level_count, stm);
    g.texels = dupload(own, im->texels, im->texel_word_count, stm);
    g.transfer = dupload(own, im->transfer, im->transfer_count, stm);
    g.texture_count = im->texture_count;
    g.level_count = im->level_count;
    g.texel_word_count = im->texel_word_count;
    g.transfer_count = im->transfer_count;
    g.uvs = dupload(own, reinterpret_cast<const float2 *>(im->uvs), im->uv_count, stm);
    g.uv_count = im->uv_count;
    g.frames = dupload(own, im->frames, size_t(6) * im->frame_count, stm);
    g.frame_count = im->frame_count;
    if (im->instance_uv_begin)
        g.inst_uv_begin = dupload(own, im->instance_uv_begin, instances, stm);
    if (im->instance_frame_begin)
        g.inst_frame_begin = dupload(own, im->instance_frame_begin, instances, stm);
    if (im->ewa_weights)
        g.ewa_weights = dupload(own, im->ewa_weights, 128, stm);
    memcpy(g.world_from_camera, im->world_from_camera, sizeof(g.world_from_camera));
    memcpy(g.camera_from_world, im->camera_from_world, sizeof(g.camera_from_world));
    if (im->texture_count) {
        g.rgb_table = dupload(own, im->rgb_table, RP_RGB_TABLE_FLOATS, stm);
        g.illuminant = dupload(own, im->illuminant, 471, stm);
    }
    if (im->environment_image != RP_NONE) {
        std::vector<float> cdf;
        u32 width = 0, offset = 0;
        double mean = 0;
        const std::string err = environment_tables(*im, cdf, width, offset, mean);
        if (!err.empty())
            throw Invalid{err};
        g.env_cdf = dupload(own, cdf.data(), cdf.size(), stm);
        g.env_width = width;
        g.env_comp_offset = offset;
        g.env_cdf_count = u32(cdf.size());
        g.env_image = im->environment_image;
        g.env_scale = im->environment_scale;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                g.env_from_world[3 * r + c] = im->environment_from_world[3 * r + c];
                g.world_from_env[3 * c + r] = im->environment_from_world[3 * r + c];
            }
        env_power = mean * im->environment_scale;
    }
}

// One image probe: upload the images (and environment tables) and the queries, run `launch`,
// read back `out_per` floats per query.
template <class Launch>
rp_status image_probe(const rp_images *images, const float *queries, u32 count, u32 in_per, u32 out_per,
                      float *results, char *diag, size_t cap, Launch launch) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!images || !queries || !results)
            throw Invalid{"null argument"};
        rp_scene_desc d{};
        d.images = images;
        if (const std::string err = validate_images(&d); !err.empty())
            throw Invalid{err};
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        DImages g;
        double power;
        upload_images(images, 0, g, own, nullptr, power);
        const float *q = dupload(own, queries, size_t(in_per) * count, nullptr);
        float *r = dalloc<float>(own, size_t(out_per) * count);
        launch(g, q, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(out_per) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

int grid_for(int sm_count, u32 work, int block, int per_sm) {
    const u32 needed = (work + block - 1) / block;
    return int(std::max<u32>(1, std::min<u32>(needed, u32(sm_count * per_sm))));
}

// The structure-of-arrays carve of a path pool of `lanes` slots over `base` (nullptr: only
// the size is computed): the 16-byte arrays, the queues and family bins, the counters, and,
// when `full`, the arrays only some runs read (shadow targets and resolved materials of
// scenes with pass-through or mix surfaces, per-lane walk counts of counting runs).  Every
// slice starts on a 256-byte boundary.  The scene pool and the allocation-free scratch both
// carve through here, so a new PathPool array is added in one place; a pool without `full`
// leaves those pointers null, and only scenes without pass-through or mix surfaces, without
// counting and without the adjoint may run on it.
constexpr size_t pool_bytes(u32 lanes, bool full) {
    const size_t v16 = (size_t(lanes) * 16 + 255) & ~size_t(255), v4 = (size_t(lanes) * 4 + 255) & ~size_t(255);
    return 33 * v16 + 9 * v4 + 256 + (full ? v16 + 3 * v4 : 0);
}
size_t carve_pool(unsigned char *base, u32 lanes, bool full, PathPool *out) {
    const size_t v16 = (size_t(lanes) * 16 + 255) & ~size_t(255), v4 = (size_t(lanes) * 4 + 255) & ~size_t(255);
    size_t off = 0;
    auto take = [&](size_t n) {
        unsigned char *p = base ? base + off : nullptr;
        off += n;
        return p;
    };
    PathPool q{};
    q.ident = reinterpret_cast<uint4 *>(take(v16));
    q.cursor = reinterpret_cast<uint4 *>(take(v16));
    float4 **f4[] = {&q.lambda, &q.lambda_pdf, &q.beta, &q.radiance, &q.dens_f, &q.prev_f, &q.eta_scale, &q.ray_o,
                     &q.ray_d, &q.latest_p, &q.latest_n, &q.latest_param, &q.latest_k, &q.preceding, &q.hit,
                     &q.sh_o, &q.sh_d, &q.sh_c};
    for (auto p : f4)
        *p = reinterpret_cast<float4 *>(take(v16));
    q.dens_e = reinterpret_cast<int4 *>(take(v16));
    q.prev_e = reinterpret_cast<int4 *>(take(v16));
    float4 **nee[] = {&q.nee_p, &q.nee_n, &q.nee_g, &q.nee_e, &q.nee_wo, &q.nee_prev, &q.nee_beta, &q.nee_df,
                      &q.nee_param, &q.nee_k};
    for (auto p : nee)
        *p = reinterpret_cast<float4 *>(take(v16));
    q.nee_de = reinterpret_cast<int4 *>(take(v16));
    q.queue[0] = reinterpret_cast<u32 *>(take(v4));
    q.queue[1] = reinterpret_cast<u32 *>(take(v4));
    q.bins = reinterpret_cast<u32 *>(take(4 * v4));
    q.nee_queue = reinterpret_cast<u32 *>(take(3 * v4));
    q.counters = reinterpret_cast<u32 *>(take(256));
    if (full) {
        q.sh_t = reinterpret_cast<float4 *>(take(v16));
        q.material = reinterpret_cast<u32 *>(take(v4));
        q.lane_closest = reinterpret_cast<u32 *>(take(v4));
        q.lane_shadow = reinterpret_cast<u32 *>(take(v4));
    }
    q.bin_capacity = lanes;
    if (off != pool_bytes(lanes, full))
        throw std::logic_error("carve_pool and pool_bytes disagree");
    if (out)
        *out = q;
    return off;
}
// Every PathPool member is a pointer carved above, set elsewhere (stats, the adjoint's), or
// a count: a new member changes this size and so comes past this check.
static_assert(sizeof(PathPool) == 50 * sizeof(void *) + 16, "PathPool changed: review carve_pool");

} // namespace

// ---------------------------------------------------------------- scene
struct rp_scene {
    int device = 0, sm_count = 148;
    cudaStream_t stream = nullptr;
    // the shadow walks of one event run on `side` while the next event's closest-hit walk runs
    // on `stream`; `forked` and `joined` order the two (timing disabled)
    cudaStream_t side = nullptr;
    cudaEvent_t forked = nullptr, joined = nullptr;
    // Owen prefix table of the draw blocks (attach_owen_prefix), built for one seed
    unsigned short *owen_prefix = nullptr;
    u32 owen_capacity = 0, owen_blocks = 0, owen_seed = 0;
    bool owen_built = false;
    // the shade kernels of BSDF families 1-3 run on their own streams beside family 0's
    cudaStream_t family[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t family_done[3] = {nullptr, nullptr, nullptr};
    std::vector<void *> owned;   // scene lifetime
    std::vector<void *> pool_owned;
    DeviceScene ds{};
    u32 n = 0;
    // build products kept for export
    u64 *keys = nullptr;
    u32 *order = nullptr;
    BuildTmp tmp{};
    u32 tree_levels = 0;     // most internal nodes on a root-to-leaf path of the LBVH
    u32 wide_levels = 0;     // levels of the compressed 8-wide traversal tree
    bool resolve = false;    // hero scene with pass-through or mix-root instances
    bool dielectrics = false; // a dielectric material: the QMC samplers' depth limit
    bool scalar_full = false; // conductors, dielectrics or procedural primitives: the full scalar step kernel
    u32 tex_width = 0, tex_height = 0; // film size the texture camera differentials were found for
    double demo_film_scale = 0;        // demo film: 470 / integral of the CIE y table
    float4 *world = nullptr; // world-space triangle vertices in original order
    BNode *nodes = nullptr;  // traversal layout (ds.nodes, ds.leaf_v)
    float4 *leaf_v = nullptr;
    // wavefront pool
    PathPool pool{};
    u32 capacity = 0;
    u32 *lane_closest = nullptr, *lane_shadow = nullptr; // per-lane walk counts (pool.lane_* while counting)
    unsigned char *static_base = nullptr; // device address of the allocation-free scratch, once looked up
    unsigned long long *stats = nullptr;
    double *cie = nullptr;
    rp_film_pixel *film_stage = nullptr;
    size_t film_stage_pixels = 0;
    bool counting = false;
    rp_timing timing{};
    std::vector<cudaEvent_t> events;
    size_t event_cursor = 0;
    std::vector<int> event_kind;
    double light_power_total = 0;
    u32 transport = RP_TRANSPORT_HERO;
    // scalar transport: one 16-byte record per lane, regeneration and failure counters
    uint4 *scalar_records = nullptr;
    float4 *scalar_fresh_ray = nullptr;
    uint2 *scalar_fresh_index = nullptr;
    u32 *scalar_counters = nullptr;
    u32 scalar_capacity = 0;
    // scalar transport slots of the wavefront form (paths, connections, modes, hits)
    void *slot_storage = nullptr;
    u32 slot_capacity = 0;
    int step_blocks = 0; // resident k_scalar_step blocks per SM
    // adjoint: per-lane history and lane weights
    void *adjoint_storage = nullptr;
    u32 adjoint_capacity = 0;

    ~rp_scene() {
        if (device >= 0)
            cudaSetDevice(device);
        for (void *p : pool_owned)
            cudaFreeAsync(p, stream);
        for (void *p : owned)
            cudaFreeAsync(p, stream);
        if (scalar_records)
            cudaFreeAsync(scalar_records, stream);
        if (slot_storage)
            cudaFreeAsync(slot_storage, stream);
        if (owen_prefix)
            cudaFreeAsync(owen_prefix, stream);
        if (adjoint_storage)
            cudaFreeAsync(adjoint_storage, stream);
        if (film_stage)
            cudaFreeAsync(film_stage, stream);
        if (stream)
            cudaStreamSynchronize(stream);
        for (auto e : events)
            cudaEventDestroy(e);
        for (auto e : family_events)
            cudaEventDestroy(e);
        for (int k = 0; k < 3; ++k) {
            if (family_done[k])
                cudaEventDestroy(family_done[k]);
            if (family[k])
                cudaStreamDestroy(family[k]);
        }
        if (forked)
            cudaEventDestroy(forked);
        if (joined)
            cudaEventDestroy(joined);
        if (side)
            cudaStreamDestroy(side);
        if (stream)
            cudaStreamDestroy(stream);
    }

    // timing: pairs of events around launches, grouped by kind (0 trace, 1 shadow, 2 shade, 3 other)
    uint64_t launches = 0;
    void mark(int kind, int kernels = 1, cudaStream_t on = nullptr) {
        launches += kernels;
        if (event_cursor + 2 > events.size()) {
            for (int k = 0; k < 64; ++k) {
                cudaEvent_t e;
                RP_CHECK(cudaEventCreate(&e));
                events.push_back(e);
            }
        }
        RP_CHECK(cudaEventRecord(events[event_cursor], on ? on : stream));
        event_kind.push_back(kind);
    }
    void done(cudaStream_t on = nullptr) {
        RP_CHECK(cudaEventRecord(events[event_cursor + 1], on ? on : stream));
        event_cursor += 2;
    }
    // forget the recorded pairs without reading them (asynchronous calls)
    void discard_marks() {
        launches = 0;
        event_kind.clear();
        event_cursor = 0;
        family_kind.clear();
    }
    // per-family shade timing of counting runs: a pair of events around each family kernel, on
    // that kernel's stream, apart from the group pairs above
    std::vector<cudaEvent_t> family_events;
    std::vector<int> family_kind;
    void mark_family(int family_index, cudaStream_t on) {
        if (2 * family_kind.size() + 2 > family_events.size()) {
            for (int k = 0; k < 64; ++k) {
                cudaEvent_t e;
                RP_CHECK(cudaEventCreate(&e));
                family_events.push_back(e);
            }
        }
        RP_CHECK(cudaEventRecord(family_events[2 * family_kind.size()], on));
        family_kind.push_back(family_index);
    }
    void done_family(cudaStream_t on) { RP_CHECK(cudaEventRecord(family_events[2 * family_kind.size() - 1], on)); }
    void collect() {
        RP_CHECK(cudaStreamSynchronize(stream));
        double sums[4] = {0, 0, 0, 0};
        uint64_t counts[4] = {0, 0, 0, 0};
        for (size_t i = 0; i < event_kind.size(); ++i) {
            float ms = 0;
            RP_CHECK(cudaEventElapsedTime(&ms, events[2 * i], events[2 * i + 1]));
            sums[event_kind[i]] += ms;
            ++counts[event_kind[i]];
        }
        for (int k = 0; k < 4; ++k)
            timing.shade_family_ms[k] = 0;
        for (size_t i = 0; i < family_kind.size(); ++i) {
            float ms = 0;
            RP_CHECK(cudaEventElapsedTime(&ms, family_events[2 * i], family_events[2 * i + 1]));
            timing.shade_family_ms[family_kind[i]] += ms;
        }
        family_kind.clear();
        timing.trace_launches = counts[0];
        timing.shadow_launches = counts[1];
        timing.shade_launches = counts[2];
        timing.other_launches = counts[3];
        timing.trace_ms = sums[0];
        timing.shadow_ms = sums[1];
        timing.shade_ms = sums[2];
        timing.other_ms = sums[3];
        timing.kernel_launches = launches;
        launches = 0;
        event_kind.clear();
        event_cursor = 0;
    }

    void ensure_scalar(u32 lanes) {
        if (lanes <= scalar_capacity)
            return;
        if (scalar_records)
            cudaFreeAsync(scalar_records, stream);
        scalar_records = nullptr;
        scalar_capacity = 0;
        // records (16 B), raygen directions and wavelengths (16 B), Sobol indices (8 B), counters
        const size_t n = size_t(lanes);
        const size_t bytes = n * 16 + n * 16 + ((n * 8 + 255) & ~size_t(255)) + 256;
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&scalar_records), bytes, stream));
        unsigned char *base = reinterpret_cast<unsigned char *>(scalar_records);
        scalar_fresh_ray = reinterpret_cast<float4 *>(base + n * 16);
        scalar_fresh_index = reinterpret_cast<uint2 *>(base + n * 32);
        scalar_counters = reinterpret_cast<u32 *>(base + n * 32 + ((n * 8 + 255) & ~size_t(255)));
        scalar_capacity = lanes;
    }

    void ensure_pool(u32 lanes) {
        if (lanes <= capacity)
            return;
        for (void *p : pool_owned)
            cudaFreeAsync(p, stream);
        pool_owned.clear();
        capacity = 0;
        // one allocation carved into the SoA arrays
        const size_t bytes = carve_pool(nullptr, lanes, true, nullptr);
        unsigned char *base = dalloc<unsigned char>(pool_owned, bytes, stream);
        PathPool q;
        carve_pool(base, lanes, true, &q);
        lane_closest = q.lane_closest;
        lane_shadow = q.lane_shadow;
        q.lane_closest = q.lane_shadow = nullptr; // set by counting waves
        q.stats = stats;
        // the adjoint's members are set per run
        q.hist = pool.hist;
        q.adj_w = pool.adj_w;
        q.adj_slot = pool.adj_slot;
        q.adj_grad = pool.adj_grad;
        q.adj_g = pool.adj_g;
        q.adj_cie = pool.adj_cie;
        q.adj_inv_weight = pool.adj_inv_weight;
        q.adj_params = pool.adj_params;
        pool = q;
        capacity = lanes;
    }
};

namespace {

// The film clamp of a request: on for a finite positive maximum component (0 or infinity:
// off); its exposure must then be finite and nonnegative (src/packet_film.cpp:151-160).
FilmClamp film_clamp(double exposure, double max_component_value) {
    FilmClamp c{exposure, max_component_value, max_component_value > 0 && std::isfinite(max_component_value)};
    if (!(max_component_value >= 0) && !std::isinf(max_component_value))
        throw Invalid{"film clamp must be positive (or 0 / infinity for none)"};
    if (c.on && !(exposure >= 0 && std::isfinite(exposure)))
        throw Invalid{"film exposure must be finite and nonnegative"};
    return c;
}

// prepare_texture_camera_differentials (src/texture_footprint.cpp:199-232, PBRT's
// Camera::FindMinimumDifferentials): over 512 camera rays along the film's diagonal, the
// smallest change of a ray's direction, in the ray's own frame, for one pixel right (dx) and
// one pixel down (dy).  Empty on success.
std::string texture_camera_differentials(V3 corner, V3 dx, V3 dy, u32 width, u32 height, float *min_dx,
                                         float *min_dy) {
    if (width == 0 || height == 0)
        return "Texture camera raster extent must be positive";
    using Vd = std::array<double, 3>;
    const Vd c{corner.x, corner.y, corner.z}, u{dx.x, dx.y, dx.z}, v{dy.x, dy.y, dy.z};
    const auto dotd = [](const Vd &a, const Vd &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const auto unit = [](Vd a, Vd &out) {
        const double len = std::hypot(a[0], a[1], a[2]);
        if (!(len > 0 && std::isfinite(len)))
            return false;
        for (auto &x : a)
            x /= len;
        out = a;
        return true;
    };
    const auto ray = [&](double x, double y, Vd &out) {
        Vd d;
        for (int i = 0; i < 3; ++i) {
            d[i] = std::fma(y, v[i], std::fma(x, u[i], c[i]));
            if (!(std::abs(d[i]) <= double(FLT_MAX)))
                return false;
        }
        return unit(d, out);
    };
    const double px = 1. / width, py = 1. / height;
    Vd bx{}, by{};
    double lx = INFINITY, ly = INFINITY;
    for (unsigned i = 0; i < 512; ++i) {
        const double t = double(i) / 511;
        Vd d, xr, yr;
        if (!ray(t, t, d) || !ray(t + px, t, xr) || !ray(t, t + py, yr))
            return "Texture camera differential ray is unrepresentable or zero";
        // CoordinateSystem of the ray (Duff et al. 2017)
        const double sign = std::copysign(1., d[2]), a = -1 / (sign + d[2]), b = d[0] * d[1] * a;
        const Vd e0{1 + sign * d[0] * d[0] * a, sign * b, -sign * d[0]}, e1{b, sign + d[1] * d[1] * a, -d[1]};
        const auto local = [&](const Vd &r) { return Vd{dotd(e0, r), dotd(e1, r), dotd(d, r)}; };
        const Vd base = local(d);
        Vd x, y;
        if (!unit(local(xr), x) || !unit(local(yr), y))
            return "Texture camera differential ray collapses in its local frame";
        const Vd ex{x[0] - base[0], x[1] - base[1], x[2] - base[2]}, ey{y[0] - base[0], y[1] - base[1], y[2] - base[2]};
        if (dotd(ex, ex) < lx) {
            lx = dotd(ex, ex);
            bx = ex;
        }
        if (dotd(ey, ey) < ly) {
            ly = dotd(ey, ey);
            by = ey;
        }
    }
    for (int k = 0; k < 3; ++k) {
        min_dx[k] = float(bx[k]);
        min_dy[k] = float(by[k]);
    }
    return {};
}

// The footprint inputs of a request on a scene with image reflectance (src/metal_render.mm:
// 1940-1963): a fixed sample budget containing the request's samples, the differential scale
// max(1/8, 1/sqrt(budget)) and the camera's minimum differentials for the film size (found once
// per size).  They go into the scene's device parameters for the launches that follow.
void apply_texture_request(rp_scene *s, const rp_request &r) {
    DImages &im = s->ds.img;
    if (!im.textured)
        return;
    if (r.total_samples == 0 || r.sample_begin >= r.total_samples || r.sample_count > r.total_samples - r.sample_begin)
        throw Invalid{"Image texture request requires a fixed total sample budget containing the sample range"};
    if (s->tex_width != r.width || s->tex_height != r.height) {
        const std::string err =
            texture_camera_differentials(s->ds.forward, s->ds.right, s->ds.up, r.width, r.height, im.tex_min_dx, im.tex_min_dy);
        if (!err.empty())
            throw Invalid{err};
        s->tex_width = r.width;
        s->tex_height = r.height;
    }
    im.tex_spp_scale = float(std::max(0.125, 1.0 / std::sqrt(double(r.total_samples))));
}

WaveParams wave_params(const rp_request &r) {
    WaveParams p{};
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
    u32 v = std::max(std::max(r.width, r.height), 1u) - 1;
    const bool sobol_scale = r.sampler_kind == RP_SAMPLER_SOBOL || r.sampler_kind == RP_SAMPLER_ZSOBOL;
    p.m = sobol_scale ? (v == 0 ? 0 : 32 - __builtin_clz(v)) : 0;
    p.emergency_limit = r.emergency_limit ? r.emergency_limit : 1024;
    p.lanes = r.pixel_count * r.sample_count;
    // src/metal_render.mm:1979-1981: floor(log2(total samples)) for ZSobol
    p.log_spp = r.sampler_kind == RP_SAMPLER_ZSOBOL && r.total_samples ? 63 - __builtin_clzll(r.total_samples) : 0;
    p.boundary_limit = r.boundary_limit ? r.boundary_limit : 4096; // medium_boundary_limit, src/render.hpp:26
    return p;
}
u32 halton_scale(u32 resolution, u32 base) {
    u32 scale = 1;
    while (scale < std::min(resolution, 128u))
        scale *= base;
    return scale;
}

// validate_sampler_range (src/sampling.cpp:51-113)
std::string validate_sampler_range(const rp_request &r) {
    if (r.sample_begin > UINT64_MAX - (r.sample_count - 1))
        return "Sampler range must be nonempty and fit the absolute sample indices";
    if (r.sampler_kind == RP_SAMPLER_INDEPENDENT)
        return {};
    if (r.sampler_kind > RP_SAMPLER_ZSOBOL)
        return "Invalid render sampler kind";
    if (r.randomization > 3)
        return "Invalid QMC randomization mode";
    if (r.seed != uint64_t(int64_t(int32_t(uint32_t(r.seed)))))
        return "QMC seed must have a canonical signed 32-bit encoding";
    const uint64_t last = r.sample_begin + (r.sample_count - 1);
    if (r.sampler_kind == RP_SAMPLER_HALTON) {
        if (r.randomization == RP_RANDOMIZE_FASTOWEN)
            return "Halton does not support fastowen randomization";
        const uint64_t stride = uint64_t(halton_scale(r.width, 2)) * halton_scale(r.height, 3);
        if (last > (uint64_t(INT64_MAX) - (stride - 1)) / stride)
            return "Halton absolute sample range exceeds the signed 64-bit index capacity";
        return {};
    }
    const u32 v = std::max(std::max(r.width, r.height), 1u) - 1;
    const u32 m = v == 0 ? 0 : 32 - __builtin_clz(v);
    if (m > (r.sampler_kind == RP_SAMPLER_ZSOBOL ? 26u : 25u))
        return r.sampler_kind == RP_SAMPLER_ZSOBOL ? "ZSobol film dimensions must be positive and at most 2^26"
                                                   : "Sobol film dimensions must be positive and at most 2^25";
    if (r.sampler_kind == RP_SAMPLER_ZSOBOL) {
        if (r.total_samples == 0 || (r.total_samples & (r.total_samples - 1)) != 0)
            return "ZSobol requires a fixed power-of-two total sample budget";
        const u32 log_spp = 63 - __builtin_clzll(r.total_samples);
        if (2 * m + log_spp > 52)
            return "ZSobol resolution and total sample budget exceed the 52-bit index capacity";
        if (r.sample_begin >= r.total_samples || r.sample_count > r.total_samples - r.sample_begin)
            return "ZSobol absolute sample range exceeds its fixed total sample budget";
        return {};
    }
    if (last >= (uint64_t(1) << (52 - 2 * m)))
        return "Sobol absolute sample range exceeds the 52-bit interval index capacity";
    return {};
}

std::string validate_request(const rp_scene *s, const rp_request &r) {
    if (!r.width || !r.height || !r.pixel_count || !r.sample_count)
        return "Render request must have nonzero film, pixel and sample counts";
    if (uint64_t(r.pixel_begin) + r.pixel_count > uint64_t(r.width) * r.height)
        return "Render request pixels exceed the film";
    if (uint64_t(r.pixel_count) * r.sample_count > 0xffffffffull)
        return "Render request lanes exceed 2^32";
    const std::string range = validate_sampler_range(r);
    if (!range.empty())
        return range;
    // sampler_max_depth (src/sampling.cpp:129-135) as MetalRenderScene::sample applies it
    // (src/metal_render.mm:1898-1904): QMC samplers need the PBRT model within their dimensions
    if (s && r.sampler_kind != RP_SAMPLER_INDEPENDENT) {
        const u32 limit = r.sampler_kind == RP_SAMPLER_HALTON ? (s->dielectrics ? 110u : 124u)
                                                              : (s->dielectrics ? 113u : 127u);
        if (s->ds.model != kModelPbrt || s->ds.max_depth > limit)
            return "QMC sampling requires PBRT rendering with maxdepth at most " + std::to_string(limit);
    }
    return {};
}

// The scalar step kernel: the plain one, or the full one for scenes with conductors,
// dielectrics or procedural primitives.
void launch_scalar_step(const rp_scene *s, unsigned grid, const WaveParams &p, const ScalarParams &q,
                        const ScalarSlots &w, int parity) {
    if (s->scalar_full)
        k_scalar_step<true><<<grid, kTraceBlock, 0, s->stream>>>(s->ds, p, q, w, parity);
    else
        k_scalar_step<false><<<grid, kTraceBlock, 0, s->stream>>>(s->ds, p, q, w, parity);
}

// The closest-hit and shadow kernels with the traversal stack the built tree needs, resolving
// pass-through and mix-root hits when the scene has them.
template <bool Count, int Block, int Stack>
void launch_trace_stack(const rp_scene *s, const PathPool &pool, int in, unsigned grid, cudaStream_t st, u32 limit) {
    if (s->resolve)
        k_trace<Count, Block, Stack, true><<<grid, Block, 0, st>>>(s->ds, pool, in, limit);
    else
        k_trace<Count, Block, Stack, false><<<grid, Block, 0, st>>>(s->ds, pool, in, limit);
}
template <bool Count, int Block>
void launch_trace(const rp_scene *s, const PathPool &pool, int in, unsigned grid, cudaStream_t st, u32 limit) {
    if (s->wide_levels <= u32(kShortStack))
        launch_trace_stack<Count, Block, kShortStack>(s, pool, in, grid, st, limit);
    else
        launch_trace_stack<Count, Block, kStackDepth>(s, pool, in, grid, st, limit);
}
template <bool Count, int Block, bool Adjoint, int Stack>
void launch_shadow_stack(const rp_scene *s, const PathPool &pool, unsigned grid, size_t smem, cudaStream_t st,
                         u32 limit) {
    if (s->resolve)
        k_shadow<Count, Block, Adjoint, Stack, true><<<grid, Block, smem, st>>>(s->ds, pool, limit);
    else
        k_shadow<Count, Block, Adjoint, Stack, false><<<grid, Block, smem, st>>>(s->ds, pool, limit);
}
template <bool Count, int Block, bool Adjoint>
void launch_shadow(const rp_scene *s, const PathPool &pool, unsigned grid, size_t smem, cudaStream_t st, u32 limit) {
    if (s->wide_levels <= u32(kShortStack))
        launch_shadow_stack<Count, Block, Adjoint, kShortStack>(s, pool, grid, smem, st, limit);
    else
        launch_shadow_stack<Count, Block, Adjoint, kStackDepth>(s, pool, grid, smem, st, limit);
}

// The four shade kernels of one event (one per BSDF family), run side by side: family 0 on
// the scene stream, families 1-3 on their own streams, joined back before the shadow walks.
// Each reads only its own bin and appends to the path and shadow queues with atomics, so the
// queue order may differ from a serial launch but no path's result does (every later kernel
// reads a path by its id, and the film reduces by lane).
template <bool Adjoint, bool Img>
void launch_shade_img(rp_scene *s, const WaveParams &p, const PathPool &pool, int in, unsigned grid, size_t smem) {
    RP_CHECK(cudaEventRecord(s->forked, s->stream));
    for (int k = 0; k < 3; ++k)
        RP_CHECK(cudaStreamWaitEvent(s->family[k], s->forked, 0));
    // counting runs time each family kernel alone: the four run one after another on the scene
    // stream, so each one's events bracket its own work (side by side they share the SMs)
    const bool timed = s->counting;
    cudaStream_t on[4] = {s->stream, s->family[0], s->family[1], s->family[2]};
    if (timed)
        on[1] = on[2] = on[3] = s->stream;
    if (timed)
        s->mark_family(0, on[0]);
    k_shade<0, 128, Adjoint, Img><<<grid, 128, smem, on[0]>>>(s->ds, p, pool, in);
    k_nee<0, 128, Img><<<grid, 128, 0, on[0]>>>(s->ds, p, pool);
    if (timed) {
        s->done_family(on[0]);
        s->mark_family(1, on[1]);
    }
    k_shade<1, 128, Adjoint, Img><<<grid, 128, smem, on[1]>>>(s->ds, p, pool, in);
    k_nee<1, 128, Img><<<grid, 128, 0, on[1]>>>(s->ds, p, pool);
    if (timed) {
        s->done_family(on[1]);
        s->mark_family(2, on[2]);
    }
    k_shade<2, 128, Adjoint, Img><<<grid, 128, smem, on[2]>>>(s->ds, p, pool, in);
    k_nee<2, 128, Img><<<grid, 128, 0, on[2]>>>(s->ds, p, pool);
    if (timed) {
        s->done_family(on[2]);
        s->mark_family(3, on[3]);
    }
    k_shade<3, 128, Adjoint, Img><<<grid, 128, smem, on[3]>>>(s->ds, p, pool, in);
    if (timed)
        s->done_family(on[3]);
    for (int k = 0; k < 3; ++k) {
        RP_CHECK(cudaEventRecord(s->family_done[k], s->family[k]));
        RP_CHECK(cudaStreamWaitEvent(s->stream, s->family_done[k], 0));
    }
}
// The plain shade kernels for scenes without images (the adjoint keeps the full ones).
template <bool Adjoint>
void launch_shade(rp_scene *s, const WaveParams &p, const PathPool &pool, int in, unsigned grid, size_t smem) {
    if constexpr (!Adjoint) {
        if (!s->ds.img.textured && s->ds.img.env_image == kNone) {
            launch_shade_img<false, false>(s, p, pool, in, grid, smem);
            return;
        }
    }
    launch_shade_img<Adjoint, true>(s, p, pool, in, grid, smem);
}

// Sobol sampler with Owen randomisation: attaches the table of the first kOwenPrefixBits
// scrambling rounds of the continuation and light-sample draw blocks (one block per vertex up to
// the maximum depth), building it on the scene stream when the seed or depth changed.  Every
// word drawn through it equals the fully computed word.
void attach_owen_prefix(rp_scene *s, WaveParams &p) {
    p.owen_prefix = nullptr;
    p.owen_blocks = 0;
    if (p.sampler != RP_SAMPLER_SOBOL || p.randomization != RP_RANDOMIZE_OWEN)
        return;
    const u32 blocks = std::min<u32>(std::max<u32>(s->ds.max_depth, 1), 129);
    if (s->owen_capacity < blocks) {
        if (s->owen_prefix)
            cudaFreeAsync(s->owen_prefix, s->stream);
        s->owen_prefix = nullptr;
        s->owen_capacity = 0;
        s->owen_built = false;
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&s->owen_prefix),
                                 size_t(2) * blocks * 4 * kOwenPrefixEntries * sizeof(unsigned short), s->stream));
        s->owen_capacity = blocks;
    }
    if (!s->owen_built || s->owen_seed != p.seed_low || s->owen_blocks != blocks) {
        const u32 total = 2 * blocks * 4 * kOwenPrefixEntries;
        k_owen_prefix<<<grid_for(s->sm_count, total, 256, 8), 256, 0, s->stream>>>(s->owen_prefix, blocks, p.seed_low);
        RP_CHECK(cudaGetLastError());
        ++s->launches;
        s->owen_seed = p.seed_low;
        s->owen_blocks = blocks;
        s->owen_built = true;
    }
    p.owen_prefix = s->owen_prefix;
    p.owen_blocks = blocks;
}

// One wave: raygen, then max_depth + 1 events of trace -> shade -> shadow.
// The shadow walks of event e run on the side stream, overlapping the closest-hit walk of
// event e + 1 on the scene stream; the shade kernels of e + 1 wait for them.  The two walks
// share no written data: the shadow walk reads its own queue (written by shade e) and writes
// the radiance and, on a failure, the status of a path; the closest-hit walk reads the rays of
// queued paths and writes their hits and the family bins.  A closest-hit walk that reads a
// path's flags before a concurrent shadow failure marks it complete only computes a hit the
// shade kernel then ignores (it skips complete paths), so every result equals the serial
// order's.
void run_wave(rp_scene *s, const WaveParams &request_params, size_t adjoint_smem = 0) {
    WaveParams p = request_params;
    attach_owen_prefix(s, p);
    s->ensure_pool(p.lanes);
    PathPool &pool = s->pool;
    pool.lane_closest = s->counting ? s->lane_closest : nullptr;
    pool.lane_shadow = s->counting ? s->lane_shadow : nullptr;
    const int sms = s->sm_count;
    s->mark(3);
    RP_CHECK(cudaMemsetAsync(pool.counters, 0, 16 * sizeof(u32), s->stream));
    k_raygen<<<grid_for(sms, p.lanes, 256, 16), 256, 0, s->stream>>>(s->ds, p, pool);
    RP_CHECK(cudaMemcpyAsync(pool.counters, &p.lanes, sizeof(u32), cudaMemcpyHostToDevice, s->stream));
    s->done();
    int in = 0;
    const u32 events = s->ds.max_depth + 1;
    bool shadow_pending = false;
    for (u32 e = 0; e < events; ++e) {
        s->mark(0);
        RP_CHECK(cudaMemsetAsync(pool.counters + 4, 0, 4 * sizeof(u32), s->stream));
        const unsigned trace_grid = grid_for(sms, p.lanes, kTraceBlock, 12);
        if (s->counting)
            launch_trace<true, kTraceBlock>(s, pool, in, trace_grid, s->stream, p.boundary_limit);
        else
            launch_trace<false, kTraceBlock>(s, pool, in, trace_grid, s->stream, p.boundary_limit);
        s->done();
        if (shadow_pending) {
            RP_CHECK(cudaStreamWaitEvent(s->stream, s->joined, 0));
            shadow_pending = false;
        }
        s->mark(2, 7);
        RP_CHECK(cudaMemsetAsync(pool.counters + (in ^ 1), 0, sizeof(u32), s->stream));
        RP_CHECK(cudaMemsetAsync(pool.counters + 2, 0, sizeof(u32), s->stream));
        RP_CHECK(cudaMemsetAsync(pool.counters + 8, 0, 3 * sizeof(u32), s->stream));
        const size_t smem = adjoint_smem;
        const unsigned shade_grid = grid_for(sms, p.lanes, 128, 16);
        if (pool.hist)
            launch_shade<true>(s, p, pool, in, shade_grid, smem);
        else
            launch_shade<false>(s, p, pool, in, shade_grid, 0);
        s->done();
        RP_CHECK(cudaEventRecord(s->forked, s->stream));
        RP_CHECK(cudaStreamWaitEvent(s->side, s->forked, 0));
        s->mark(1, 1, s->side);
        if (pool.hist)
            launch_shadow<false, kTraceBlock, true>(s, pool, trace_grid, smem, s->side, p.boundary_limit);
        else if (s->counting)
            launch_shadow<true, kTraceBlock, false>(s, pool, trace_grid, 0, s->side, p.boundary_limit);
        else
            launch_shadow<false, kTraceBlock, false>(s, pool, trace_grid, 0, s->side, p.boundary_limit);
        s->done(s->side);
        RP_CHECK(cudaEventRecord(s->joined, s->side));
        shadow_pending = true;
        in ^= 1;
    }
    if (shadow_pending)
        RP_CHECK(cudaStreamWaitEvent(s->stream, s->joined, 0));
    RP_CHECK(cudaGetLastError());
}

// Slots of the scalar wavefront: per slot one ScalarPath, one Connection, a mode word and a
// hit, and per trip parity the two step queues.
ScalarSlots scalar_slots(rp_scene *s, u32 count) {
    const size_t a = (size_t(count) * sizeof(ScalarPath) + 255) & ~size_t(255);
    const size_t b = (size_t(count) * sizeof(Connection) + 255) & ~size_t(255);
    const size_t c = (size_t(count) * sizeof(u32) + 255) & ~size_t(255);
    const size_t d = (size_t(count) * sizeof(Hit) + 255) & ~size_t(255);
    const size_t e = (size_t(count) * sizeof(u32) + 255) & ~size_t(255);
    if (s->slot_capacity < count) {
        if (s->slot_storage)
            cudaFreeAsync(s->slot_storage, s->stream);
        s->slot_storage = nullptr;
        s->slot_capacity = 0;
        RP_CHECK(cudaMallocAsync(&s->slot_storage, a + b + c + d + 8 * e, s->stream));
        s->slot_capacity = count;
    }
    unsigned char *base = static_cast<unsigned char *>(s->slot_storage);
    ScalarSlots w;
    w.path = reinterpret_cast<ScalarPath *>(base);
    w.conn = reinterpret_cast<Connection *>(base + a);
    w.mode = reinterpret_cast<u32 *>(base + a + b);
    w.hit = reinterpret_cast<Hit *>(base + a + b + c);
    for (int k = 0; k < 2; ++k) {
        w.queue_connect[k] = reinterpret_cast<u32 *>(base + a + b + c + d + (4 * k) * e);
        w.queue_medium[k] = reinterpret_cast<u32 *>(base + a + b + c + d + (4 * k + 1) * e);
        w.queue_interface[k] = reinterpret_cast<u32 *>(base + a + b + c + d + (4 * k + 2) * e);
        w.queue_path[k] = reinterpret_cast<u32 *>(base + a + b + c + d + (4 * k + 3) * e);
    }
    w.count = count;
    w.remaining = s->scalar_counters + 2;
    w.qcount = s->scalar_counters + 4; // zeroed with the wave's counters
    return w;
}

// Slots of the scalar wavefront (at most this many paths in flight per wave), and the
// walk/step trips between two host reads of the wave's remaining lanes.  262,144 slots of
// about 230 bytes (path, connection, mode, hit, queue entries) keep the path state (60 MB)
// in L2 and give the step kernel several paths per resident thread; measured on the fog box
// (1024x1024, 16 spp) with the step queues: 2^16 slots 314 ms, 2^17 317 ms, 2^18 300 ms;
// without them 2^17 415 ms, 2^19 529 ms, 2^20 634 ms.
constexpr u32 kScalarSlots = 1u << 18;
constexpr int kScalarTripsPerCheck = 8;

// One wave of the scalar transport, one record per lane in s->scalar_records: camera rays,
// then walk / step trips over the slots until every lane's record is written.
void run_scalar_wave(rp_scene *s, const WaveParams &p, u32 boundary_limit) {
    s->ensure_scalar(p.lanes);
    if (!s->step_blocks) {
        int per_sm = 0;
        if (s->scalar_full)
            RP_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scalar_step<true>, kTraceBlock, 0));
        else
            RP_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scalar_step<false>, kTraceBlock, 0));
        s->step_blocks = std::max(1, per_sm);
    }
    s->mark(3);
    RP_CHECK(cudaMemsetAsync(s->scalar_counters, 0, 64, s->stream));
    k_scalar_raygen<<<grid_for(s->sm_count, p.lanes, 256, 16), 256, 0, s->stream>>>(s->ds, p, s->scalar_fresh_ray,
                                                                                     s->scalar_fresh_index);
    s->done();
    ScalarParams q;
    q.boundary_limit = boundary_limit;
    q.out = s->scalar_records;
    q.fresh_ray = s->scalar_fresh_ray;
    q.fresh_index = s->scalar_fresh_index;
    q.next_lane = s->scalar_counters;
    q.stats = s->stats;
    const u32 slots = std::min<u32>(std::max<u32>(p.lanes, 1), kScalarSlots);
    const ScalarSlots w = scalar_slots(s, slots);
    const u32 lanes = p.lanes;
    RP_CHECK(cudaMemcpyAsync(w.remaining, &lanes, sizeof(u32), cudaMemcpyHostToDevice, s->stream));
    const int walk_grid = grid_for(s->sm_count, slots, kTraceBlock, 8);
    const int step_grid = grid_for(s->sm_count, slots, kTraceBlock, s->step_blocks);
    const bool short_stack = s->wide_levels <= u32(kShortStack);
    s->mark(2, 2);
    k_scalar_slots_init<<<grid_for(s->sm_count, slots, 256, 8), 256, 0, s->stream>>>(w.mode, slots);
    launch_scalar_step(s, step_grid, p, q, w, -1);
    const bool walks = s->ds.instance_count != 0; // geometry-free scenes take the sky step
    int parity = 0;
    RP_CHECK(cudaGetLastError());
    // every trip advances each unfinished path by one walk and one step, so a wave ends after
    // at most (its lanes' steps) trips; the bound only guards the host loop
    u32 remaining = lanes;
    for (u64 trip = 0; remaining; trip += kScalarTripsPerCheck) {
        if (trip > (u64(1) << 22))
            throw Invalid{"scalar wave did not finish"};
        for (int k = 0; k < kScalarTripsPerCheck; ++k) {
            if (!walks) {
                launch_scalar_step(s, step_grid, p, q, w, -1);
                s->launches += 1;
                continue;
            }
            const bool procedural = s->ds.prim_count != s->ds.tri_prims;
            if (procedural && s->counting)
                k_scalar_walk<true, kStackDepth, true><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            else if (procedural)
                k_scalar_walk<false, kStackDepth, true><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            else if (s->counting && short_stack)
                k_scalar_walk<true, kShortStack><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            else if (s->counting)
                k_scalar_walk<true, kStackDepth><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            else if (short_stack)
                k_scalar_walk<false, kShortStack><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            else
                k_scalar_walk<false, kStackDepth><<<walk_grid, kTraceBlock, 0, s->stream>>>(s->ds, p, w, parity, s->stats);
            launch_scalar_step(s, step_grid, p, q, w, parity);
            s->launches += 2;
            parity ^= 1;
        }
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpyAsync(&remaining, w.remaining, sizeof(u32), cudaMemcpyDeviceToHost, s->stream));
        RP_CHECK(cudaStreamSynchronize(s->stream));
    }
    s->done();
}

template <class F> rp_status guarded(char *diag, size_t cap, F &&f) {
    try {
        return f();
    } catch (const CudaError &e) {
        set_diag(diag, cap, "CUDA error %s in %s", cudaGetErrorString(e.code), e.what);
        return RP_FAILURE;
    } catch (const Invalid &e) {
        set_diag(diag, cap, "%s", e.what.c_str());
        return RP_INVALID_ARGUMENT;
    } catch (const NotBuilt &e) {
        set_diag(diag, cap, "%s", e.what.c_str());
        return RP_NOT_BUILT;
    } catch (const std::bad_alloc &) {
        set_diag(diag, cap, "host allocation failed");
        return RP_FAILURE;
    } catch (...) {
        set_diag(diag, cap, "unexpected failure");
        return RP_FAILURE;
    }
}

// First half of the LBVH build, launched as soon as the triangles are on the device: the
// build storage, then world-space triangles, their boxes, and the centroid and vertex bounds
// (read back by build_bounds).  The light tables are built on the host meanwhile.
void build_prepare(rp_scene *s, u32 vertex_count) {
    const u32 n = s->ds.prim_count;
    s->n = n;
    auto &own = s->owned;
    cudaStream_t st = s->stream;
    BuildTmp &t = s->tmp;
    t.box_lo = dalloc<float4>(own, n, st);
    t.box_hi = dalloc<float4>(own, n, st);
    t.cbounds = dalloc<int>(own, 16, st);
    t.error = reinterpret_cast<u32 *>(t.cbounds + 12);
    t.levels = t.error + 1;
    t.keys[0] = dalloc<u64>(own, n, st);
    t.keys[1] = dalloc<u64>(own, n, st);
    t.vals[0] = dalloc<u32>(own, n, st);
    t.vals[1] = dalloc<u32>(own, n, st);
    const u32 tiles = (n + kSortTile - 1) / kSortTile;
    t.hist = dalloc<u32>(own, size_t(256) * std::max<u32>(tiles, 1), st);
    t.left = dalloc<u32>(own, n, st);
    t.right = dalloc<u32>(own, n, st);
    t.parent = dalloc<u32>(own, n, st);
    t.leaf_parent = dalloc<u32>(own, n, st);
    t.node_lo = dalloc<float4>(own, n, st);
    t.node_hi = dalloc<float4>(own, n, st);
    t.flags = dalloc<u32>(own, n, st);
    t.refs = dalloc<u32>(own, size_t(2) * n, st);
    t.vertex_count = vertex_count;
    s->world = dalloc<float4>(own, size_t(3) * n, st);
    s->nodes = dalloc<BNode>(own, n, st);
    s->leaf_v = dalloc<float4>(own, size_t(3) * n, st);
    s->ds.nodes = s->nodes;
    s->ds.leaf_v = s->leaf_v;
    const int init[16] = {0x7fffffff,      0x7fffffff,      0x7fffffff,      int(0x80000000), int(0x80000000),
                          int(0x80000000), 0x7fffffff,      0x7fffffff,      0x7fffffff,      int(0x80000000),
                          int(0x80000000), int(0x80000000), 0,               0,               0,
                          0};
    RP_CHECK(cudaMemcpyAsync(t.cbounds, init, sizeof(init), cudaMemcpyHostToDevice, st));
    RP_CHECK(cudaMemsetAsync(t.parent, 0xff, size_t(n) * 4, st));
    RP_CHECK(cudaMemsetAsync(t.leaf_parent, 0xff, size_t(n) * 4, st));
    RP_CHECK(cudaMemsetAsync(t.flags, 0, size_t(n) * 4, st));
    RP_CHECK(cudaMemsetAsync(t.refs, 0, size_t(2) * n * 4, st));
    if (n)
        k_tri_prepare<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(s->ds, s->world, t);
    RP_CHECK(cudaGetLastError());
}

// The bounds of build_prepare: centroid and world-vertex boxes (ordered ints, as in
// BuildTmp::cbounds).  Throws on a vertex index outside the vertex array.
void build_bounds(rp_scene *s, int (&cb)[12]) {
    int out[13];
    RP_CHECK(cudaMemcpyAsync(out, s->tmp.cbounds, sizeof(out), cudaMemcpyDeviceToHost, s->stream));
    RP_CHECK(cudaStreamSynchronize(s->stream));
    if (u32(out[12]) & kBuildVertexRange)
        throw Invalid{"triangle vertex out of range"};
    std::copy(out, out + 12, cb);
}

// The compressed 8-wide traversal tree, collapsed level by level from the checked binary tree
// (one launch per binary level at most: each wide level consumes at least one), then checked:
// every triangle placed once, no allocation beyond the binary tree's size.
void build_wide(rp_scene *s) {
    const u32 n = s->n;
    auto &own = s->owned;
    cudaStream_t st = s->stream;
    BuildTmp &t = s->tmp;
    const u32 capacity = std::max<u32>(n, 2) - 1;
    WNode *wnodes = dalloc<WNode>(own, capacity, st);
    float4 *wtri = dalloc<float4>(own, size_t(3) * std::max<u32>(n, 1), st);
    s->ds.wnodes = wnodes;
    s->ds.wtri = wtri;
    s->ds.wnode_count = 0;
    s->wide_levels = 0;
    if (n == 0)
        return;
    if (n == 1) {
        RP_CHECK(cudaMemcpyAsync(wtri, s->leaf_v, 3 * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        RP_CHECK(cudaStreamSynchronize(st));
        return;
    }
    WideBuild w{};
    w.left = t.left;
    w.right = t.right;
    w.node_lo = t.node_lo;
    w.node_hi = t.node_hi;
    w.box_lo = t.box_lo;
    w.box_hi = t.box_hi;
    w.order = s->order;
    w.leaf_v = s->leaf_v;
    w.wnodes = wnodes;
    w.wtri = wtri;
    w.counters = dalloc<u32>(own, 8, st);
    w.queue[0] = dalloc<uint2>(own, capacity, st);
    w.queue[1] = dalloc<uint2>(own, capacity, st);
    w.capacity = capacity;
    w.n = n;
    const u32 init[8] = {1, 0, 1, 0, 0, 0, 0, 0}; // the root is wide node 0, queued at level 0
    const uint2 root = make_uint2(0, 0);
    RP_CHECK(cudaMemcpyAsync(w.counters, init, sizeof(init), cudaMemcpyHostToDevice, st));
    RP_CHECK(cudaMemcpyAsync(w.queue[0], &root, sizeof(root), cudaMemcpyHostToDevice, st));
    for (u32 level = 0; level < s->tree_levels; ++level) {
        const int parity = int(level & 1);
        RP_CHECK(cudaMemsetAsync(w.counters + 2 + (parity ^ 1), 0, sizeof(u32), st));
        k_wide_level<<<grid_for(s->sm_count, n, 128, 8), 128, 0, st>>>(w, parity, level);
    }
    RP_CHECK(cudaGetLastError());
    u32 result[8];
    RP_CHECK(cudaMemcpyAsync(result, w.counters, sizeof(result), cudaMemcpyDeviceToHost, st));
    RP_CHECK(cudaStreamSynchronize(st));
    if (result[4] || result[1] != n || result[0] > capacity)
        throw Invalid{"wide BVH collapse did not place every triangle once"};
    s->ds.wnode_count = result[0];
    s->wide_levels = result[5];
}

// Second half: Morton codes, radix sort, Karras topology, refit, the traversal layout and the
// structural check (k_tree_refs / k_tree_verify), then one wait for the whole build.
void build_finish(rp_scene *s, const int (&cb)[12]) {
    const u32 n = s->n;
    cudaStream_t st = s->stream;
    BuildTmp &t = s->tmp;
    if (n == 0)
        return;
    const u32 tiles = (n + kSortTile - 1) / kSortTile;
    const float lo[3] = {unordered_host(cb[0]), unordered_host(cb[1]), unordered_host(cb[2])};
    const float hi[3] = {unordered_host(cb[3]), unordered_host(cb[4]), unordered_host(cb[5])};
    const float3 flo = make_float3(lo[0], lo[1], lo[2]);
    const float3 fext = make_float3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    k_morton<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(n, t, flo, fext);
    int cur = 0;
    for (int shift = 0; shift < 64; shift += 8) {
        k_radix_hist<<<tiles, kSortThreads, 0, st>>>(t.keys[cur], n, shift, t.hist, tiles);
        k_radix_scan<<<1, 1024, 0, st>>>(t.hist, 256 * tiles);
        k_radix_scatter<<<tiles, kSortThreads, 0, st>>>(t.keys[cur], t.vals[cur], t.keys[cur ^ 1], t.vals[cur ^ 1], n,
                                                        shift, t.hist, tiles);
        cur ^= 1;
    }
    s->keys = t.keys[cur];
    s->order = t.vals[cur];
    if (n > 1) {
        k_karras<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(s->keys, n, t);
        k_refit<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(n, s->order, t);
        k_tree_refs<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(n, t);
        k_tree_verify<<<grid_for(s->sm_count, 2 * n, 256, 8), 256, 0, st>>>(n, t);
    }
    k_pack<<<grid_for(s->sm_count, n, 256, 8), 256, 0, st>>>(n, s->order, s->world, t, s->nodes, s->leaf_v);
    RP_CHECK(cudaGetLastError());
    u32 result[2] = {0, 0}; // error bits, tree levels
    RP_CHECK(cudaMemcpyAsync(result, t.error, sizeof(result), cudaMemcpyDeviceToHost, st));
    RP_CHECK(cudaStreamSynchronize(st));
    if (result[0] & kBuildTree)
        throw Invalid{"LBVH build produced an invalid tree"};
    s->tree_levels = result[1];
    build_wide(s);
}

} // namespace

extern "C" {

rp_status rp_cuda_device_info(int device, rp_device_info *info, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            set_diag(diag, cap, "no CUDA device");
            return RP_NO_DEVICE;
        }
        if (device < 0 || device >= count)
            throw Invalid{"device index out of range"};
        const cudaDeviceProp &prop = device_properties(device);
        if (info) {
            memset(info, 0, sizeof(*info));
            snprintf(info->name, sizeof(info->name), "%s", prop.name);
            info->device = device;
            info->sm_count = prop.multiProcessorCount;
            info->major = prop.major;
            info->minor = prop.minor;
            info->total_memory = prop.totalGlobalMem;
        }
        return RP_SUCCESS;
    });
}

uint32_t rp_cuda_abi_size(const char *name) {
    const std::string n = name ? name : "";
    if (n == "rp_instance") return sizeof(rp_instance);
    if (n == "rp_analytic") return sizeof(rp_analytic);
    if (n == "rp_material") return sizeof(rp_material);
    if (n == "rp_knot") return sizeof(rp_knot);
    if (n == "rp_area_emission") return sizeof(rp_area_emission);
    if (n == "rp_positional_light") return sizeof(rp_positional_light);
    if (n == "rp_medium") return sizeof(rp_medium);
    if (n == "rp_camera") return sizeof(rp_camera);
    if (n == "rp_scene_desc") return sizeof(rp_scene_desc);
    if (n == "rp_image_texture") return sizeof(rp_image_texture);
    if (n == "rp_texture_level") return sizeof(rp_texture_level);
    if (n == "rp_images") return sizeof(rp_images);
    if (n == "rp_request") return sizeof(rp_request);
    if (n == "rp_packet_result") return sizeof(rp_packet_result);
    if (n == "rp_scalar_result") return sizeof(rp_scalar_result);
    if (n == "rp_film_pixel") return sizeof(rp_film_pixel);
    if (n == "rp_film_request") return sizeof(rp_film_request);
    if (n == "rp_timing") return sizeof(rp_timing);
    if (n == "rp_device_info") return sizeof(rp_device_info);
    if (n == "rp_view") return sizeof(rp_view);
    if (n == "rp_batch_config") return sizeof(rp_batch_config);
    if (n == "rp_batch_request") return sizeof(rp_batch_request);
    if (n == "rp_adjoint_request") return sizeof(rp_adjoint_request);
    if (n == "rp_frame_config") return sizeof(rp_frame_config);
    if (n == "rp_frame_request") return sizeof(rp_frame_request);
    if (n == "rp_frame_info") return sizeof(rp_frame_info);
    return 0;
}

int rp_cuda_build_light_tables(const double *rows, uint32_t count, uint32_t *alias, uint32_t *records, uint32_t *nodes,
                               uint32_t *infinite, uint32_t *infinite_count) {
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
    memcpy(alias, t.alias.data(), t.alias.size() * 16);
    memcpy(records, t.records.data(), t.records.size() * 16);
    for (size_t i = 0; i < t.nodes.size(); ++i) // the 16-word LightBounds head of each node
        memcpy(nodes + 16 * i, &t.nodes[i], 64);
    memcpy(infinite, t.infinite.data(), t.infinite.size() * 4);
    *infinite_count = u32(t.infinite.size());
    return int(t.nodes.size());
}

rp_status rp_cuda_scene_create(const rp_scene_desc *d, int device, rp_scene **out, char *diag, size_t cap) {
    if (out)
        *out = nullptr;
    rp_scene *s = nullptr;
    const rp_status st = guarded(diag, cap, [&]() -> rp_status {
        if (!d || !out)
            throw Invalid{"null scene description or output"};
        if (d->abi_version != RP_ABI_VERSION)
            throw Invalid{"scene description ABI version mismatch"};
        if (!d->sobol_tables)
            throw Invalid{"scene description needs the Sobol tables"};
        if (d->transport != RP_TRANSPORT_HERO && d->transport != RP_TRANSPORT_SCALAR)
            throw NotBuilt{"only the hero-wavelength and scalar transports are built"};
        const bool scalar = d->transport == RP_TRANSPORT_SCALAR;
        bool interfaces = false;
        for (u32 i = 0; i < d->material_count; ++i)
            interfaces = interfaces || d->materials[i].scattering == RP_INTERFACE;
        if (d->camera_medium != RP_NONE && d->camera_medium >= d->medium_count)
            throw Invalid{"camera medium out of range"};
        if (!scalar) {
            // src/render.cpp:1537-1590: hero transport needs every declared medium inactive
            // (all coefficients zero); the camera and instance media are then vacuum
            if (d->max_depth > RP_MAX_DEPTH + 1)
                throw Invalid{"hero transport requires max depth <= 65"};
            for (u32 i = 0; i < d->medium_count; ++i) {
                const auto &m = d->media[i];
                const auto nonzero = [](const float *v) { return std::any_of(v, v + 471, [](float x) { return x != 0; }); };
                if (nonzero(m.sigma_a) || nonzero(m.sigma_s) || nonzero(m.emission))
                    throw Invalid{"Packet/hero spectral transport requires a PBRT scene with vacuum media"};
            }
        }
        if ((d->patch_count && !d->patches) || (d->analytic_count && !d->analytics))
            throw Invalid{"patch or analytic shape array missing"};
        if (const std::string mix = validate_mix(d); !mix.empty())
            throw Invalid{mix};
        if (const std::string images = validate_images(d); !images.empty())
            throw Invalid{images};
        if (d->model > RP_MODEL_DEMO)
            throw Invalid{"invalid scene model"};
        if (d->model == RP_MODEL_DEMO) {
            // src/render.cpp:1823-1895: the demo model renders its sky and sampled reflectance
            if (!scalar)
                throw NotBuilt{"the demo model renders with the scalar transport"};
            if (d->emission_count || d->positional_count || d->images || d->medium_count)
                throw Invalid{"the demo model has no emitters, lights, images or media besides its sky"};
            if (!(d->film_scale > 0) || !std::isfinite(d->film_scale))
                throw Invalid{"the demo camera needs a positive finite film scale"};
        }
        for (u32 i = 0; i < d->material_count; ++i) {
            const rp_material &m = d->materials[i];
            if (m.kind != RP_REFLECTANCE_IMAGE || m.scattering != RP_DIFFUSE)
                continue;
            if (!d->images || m.image_texture >= d->images->texture_count)
                throw Invalid{"image reflectance names no image texture"};
            if (d->images->textures[m.image_texture].filter == RP_TEXTURE_EWA && !d->images->ewa_weights)
                throw Invalid{"an EWA-filtered image needs the EWA weight table"};
            if (!d->images->instance_frame_begin || (d->images->uv_count && !d->images->instance_uv_begin))
                throw Invalid{"image reflectance needs per-instance texture frames"};
        }
        if (d->filter_kind > RP_FILTER_GAUSSIAN)
            throw Invalid{"unsupported pixel filter"};
        if (!(d->lens_radius >= 0) || !std::isfinite(d->lens_radius) ||
            (d->lens_radius > 0 && (!(d->focal_distance > 0) || !std::isfinite(d->focal_distance))))
            throw Invalid{"lens radius must be finite and nonnegative, with a positive finite focal distance"};
        if (d->light_sampler > RP_LIGHTS_UNIFORM)
            throw Invalid{"invalid light sampler"};
        if (d->positional_count > RP_MAX_POSITIONAL)
            throw Invalid{"too many positional lights"};
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            set_diag(diag, cap, "no CUDA device");
            return RP_NO_DEVICE;
        }
        RP_CHECK(cudaSetDevice(device));
        retain_pool(device);
        const auto t_begin = std::chrono::steady_clock::now();
        s = new rp_scene();
        s->device = device;
        s->sm_count = device_properties(device).multiProcessorCount;
        RP_CHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        RP_CHECK(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
        RP_CHECK(cudaEventCreateWithFlags(&s->forked, cudaEventDisableTiming));
        RP_CHECK(cudaEventCreateWithFlags(&s->joined, cudaEventDisableTiming));
        for (int k = 0; k < 3; ++k) {
            RP_CHECK(cudaStreamCreateWithFlags(&s->family[k], cudaStreamNonBlocking));
            RP_CHECK(cudaEventCreateWithFlags(&s->family_done[k], cudaEventDisableTiming));
        }
        cudaStream_t stm = s->stream;
        auto &own = s->owned;
        DeviceScene &ds = s->ds;
        // validation of indices: the vertex indices of emitting triangles here (the host reads
        // their vertices for the light tables), those of every triangle on the device
        // (k_tri_prepare, reported by build_bounds)
        u64 prims = 0;
        for (u32 i = 0; i < d->instance_count; ++i) {
            const auto &in = d->instances[i];
            if (uint64_t(in.triangle_begin) + in.triangle_count > d->triangle_count)
                throw Invalid{"instance triangles out of range"};
            if (in.material >= d->material_count)
                throw Invalid{"instance material out of range"};
            if (in.emission != RP_NONE && in.emission >= d->emission_count)
                throw Invalid{"instance emission out of range"};
            if ((in.patch_count && uint64_t(in.patch_begin) + in.patch_count > d->patch_count) ||
                (in.analytic_count && uint64_t(in.analytic_begin) + in.analytic_count > d->analytic_count))
                throw Invalid{"instance patches or analytic shapes out of range"};
            if ((in.patch_count || in.analytic_count) && in.emission != RP_NONE)
                throw NotBuilt{"area emission from bilinear patches and analytic shapes is not built"};
            if ((in.patch_count || in.analytic_count) && d->materials[in.material].kind == RP_REFLECTANCE_IMAGE)
                throw NotBuilt{"image reflectance on bilinear patches and analytic shapes is not built"};
            for (u32 k = 0; k < in.analytic_count; ++k)
                if (const std::string e = validate_analytic(d->analytics[in.analytic_begin + k]); !e.empty())
                    throw Invalid{e};
            prims += uint64_t(in.patch_count) + in.analytic_count;
            if (in.emission != RP_NONE)
                for (u32 t = 0; t < in.triangle_count; ++t)
                    for (int k = 0; k < 3; ++k)
                        if (uint64_t(in.vertex_begin) + d->triangles[3 * (size_t(in.triangle_begin) + t) + k] >=
                            d->vertex_count)
                            throw Invalid{"triangle vertex out of range"};
            prims += in.triangle_count;
        }
        if (prims >= (1u << 30))
            throw Invalid{"a scene holds fewer than 2^30 triangle instances"};
        for (u32 i = 0; i < d->material_count; ++i) {
            const u32 f = d->materials[i].scattering;
            if (f > RP_DIELECTRIC && f != RP_INTERFACE && f != RP_MIX)
                throw NotBuilt{"unsupported scattering family (diffuse, conductor, dielectric, mix and null "
                               "interfaces are built)"};
            s->dielectrics = s->dielectrics || f == RP_DIELECTRIC; // scene_has_dielectrics (src/render.cpp:927-932)
            s->scalar_full = s->scalar_full || f == RP_CONDUCTOR || f == RP_DIELECTRIC;
        }
        for (u32 i = 0; i < d->instance_count; ++i) {
            const auto &in = d->instances[i];
            if ((in.inside_medium != RP_NONE && in.inside_medium >= d->medium_count) ||
                (in.outside_medium != RP_NONE && in.outside_medium >= d->medium_count))
                throw Invalid{"instance medium out of range"};
        }
        for (u32 i = 0; i < d->medium_count; ++i) {
            const auto &m = d->media[i];
            for (int k = 0; k < RP_SPECTRUM_BINS; ++k)
                if (!(m.sigma_a[k] >= 0 && std::isfinite(m.sigma_a[k]) && m.sigma_s[k] >= 0 &&
                      std::isfinite(m.sigma_s[k]) && m.emission[k] >= 0 && std::isfinite(m.emission[k])))
                    throw Invalid{"medium coefficients must be finite and nonnegative"};
            if (!std::isfinite(m.g))
                throw Invalid{"medium asymmetry must be finite"};
        }
        // flattened triangles (k_flatten) and emitters (src/metal_render.mm:1174-1210)
        std::vector<u32> prim_begin(d->instance_count), em_inst, em_local;
        std::vector<DInstance> instances(d->instance_count);
        u32 next_prim = 0;
        for (u32 i = 0; i < d->instance_count; ++i) {
            const auto &q = d->instances[i];
            DInstance &in = instances[i];
            memcpy(in.m, q.matrix, sizeof(in.m));
            in.vertex_begin = q.vertex_begin;
            in.triangle_begin = q.triangle_begin;
            in.triangle_count = q.triangle_count;
            in.material = q.material;
            in.reverse = q.reverse_orientation;
            in.emission = q.emission;
            in.normal_begin = q.normal_begin;
            in.emitter_begin = kNone;
            // the hero transport is vacuum: its camera and instance media are cleared
            // (src/render.cpp:1587-1590)
            in.inside_medium = scalar ? q.inside_medium : RP_NONE;
            in.outside_medium = scalar ? q.outside_medium : RP_NONE;
            const u32 root = d->materials[q.material].scattering;
            in.resolve = (!scalar && (q.invisible_emitter != 0 || root == RP_INTERFACE) ? kPassThrough : 0u) |
                         (root == RP_MIX ? kMixRoot : 0u);
            s->resolve = s->resolve || (!scalar && in.resolve != 0);
            if (q.emission != RP_NONE) {
                in.emitter_begin = u32(em_inst.size());
                for (u32 t = 0; t < q.triangle_count; ++t) {
                    em_inst.push_back(i);
                    em_local.push_back(t);
                }
            }
            prim_begin[i] = next_prim;
            next_prim += q.triangle_count;
            in.patch_begin = q.patch_count ? q.patch_begin : 0;
            in.patch_count = q.patch_count;
            in.analytic_begin = q.analytic_count ? q.analytic_begin : 0;
            in.analytic_count = q.analytic_count;
        }
        // procedural primitives follow the triangles: every instance's patches, then every
        // instance's analytic shapes, each range in instance order
        std::vector<u32> patch_begin(d->instance_count), analytic_begin(d->instance_count);
        u32 patch_prims = 0, analytic_prims = 0;
        for (u32 i = 0; i < d->instance_count; ++i) {
            patch_begin[i] = patch_prims;
            patch_prims += d->instances[i].patch_count;
        }
        for (u32 i = 0; i < d->instance_count; ++i) {
            analytic_begin[i] = analytic_prims;
            analytic_prims += d->instances[i].analytic_count;
        }
        // the hero walks test procedural leaves in the kernels that resolve hits
        if (!scalar && (patch_prims || analytic_prims))
            s->resolve = true;
        s->scalar_full = s->scalar_full || patch_prims || analytic_prims;
        // world-to-object maps of the instances (procedural hits test the ray in object space)
        std::vector<float> inverse(size_t(12) * std::max<u32>(d->instance_count, 1), 0.0f);
        for (u32 i = 0; i < d->instance_count; ++i) {
            if (!d->instances[i].patch_count && !d->instances[i].analytic_count)
                continue;
            if (!invert_affine(d->instances[i].matrix, inverse.data() + 12 * size_t(i)))
                throw Invalid{"an instance with patches or analytic shapes needs an invertible transform"};
        }
        ds.positions = dupload(own, d->positions, size_t(3) * d->vertex_count, stm);
        ds.normals = dupload(own, d->normals, size_t(3) * d->normal_count, stm);
        ds.normal_count = d->normal_count;
        ds.triangles = dupload(own, d->triangles, size_t(3) * d->triangle_count, stm);
        ds.instances = dupload(own, instances.data(), instances.size(), stm);
        ds.instance_count = d->instance_count;
        std::vector<DMaterial> mats(d->material_count);
        for (u32 i = 0; i < d->material_count; ++i) {
            const auto &m = d->materials[i];
            mats[i] = {m.scattering, m.kind,        m.knot_begin,        m.knot_count,      m.scalar_value,
                       m.eta_begin,  m.eta_count,   m.k_begin,           m.k_count,         m.optical_extensions,
                       m.u_roughness, m.v_roughness, m.remap_roughness,    m.first_material,  m.second_material,
                       m.mix_amount,  m.image_texture, {m.coefficients[0], m.coefficients[1], m.coefficients[2]},
                       {m.reflectance[0], m.reflectance[1], m.reflectance[2], m.reflectance[3], m.reflectance[4],
                        m.reflectance[5], m.reflectance[6], m.reflectance[7]}};
        }
        ds.materials = dupload(own, mats.data(), mats.size(), stm);
        ds.material_count = d->material_count;
        const u32 all_prims = next_prim + patch_prims + analytic_prims;
        ds.prim_count = all_prims;
        ds.tri_prims = next_prim;
        ds.patch_prims = patch_prims;
        u32 *tri_instance = dalloc<u32>(own, all_prims, stm), *tri_local = dalloc<u32>(own, all_prims, stm);
        unsigned char *tri_family = dalloc<unsigned char>(own, all_prims, stm);
        ds.tri_instance = tri_instance;
        ds.tri_local = tri_local;
        ds.tri_family = tri_family;
        const std::vector<u32> *ranges[3] = {&prim_begin, &patch_begin, &analytic_begin};
        const u32 range_base[3] = {0, next_prim, next_prim + patch_prims};
        const u32 range_count[3] = {next_prim, patch_prims, analytic_prims};
        for (int k = 0; k < 3; ++k) {
            if (!range_count[k])
                continue;
            const u32 *begin_dev = dupload(own, ranges[k]->data(), ranges[k]->size(), stm);
            k_flatten<<<grid_for(s->sm_count, range_count[k], 256, 8), 256, 0, stm>>>(
                ds.instances, begin_dev, d->instance_count, ds.materials, range_count[k], tri_instance + range_base[k],
                tri_local + range_base[k], tri_family + range_base[k]);
        }
        ds.patches = dupload(own, d->patches, size_t(4) * d->patch_count, stm);
        std::vector<DAnalytic> analytics(d->analytic_count);
        for (u32 i = 0; i < d->analytic_count; ++i) {
            const rp_analytic &a = d->analytics[i];
            analytics[i] = {a.kind, a.subtype, a.radius, a.z_min, a.z_max, a.phi_max, a.inner_radius, a.height};
        }
        ds.analytics = dupload(own, analytics.data(), analytics.size(), stm);
        ds.inverse = dupload(own, inverse.data(), inverse.size(), stm);
        const auto t_prepare = std::chrono::steady_clock::now();
        build_prepare(s, d->vertex_count);
        const auto t_prepared = std::chrono::steady_clock::now();
        ds.knots = dupload(own, reinterpret_cast<const float2 *>(d->knots), d->knot_count, stm);
        ds.knot_count = d->knot_count;
        // spectra: emissions, positional intensities, environment
        std::vector<float> spectra;
        std::vector<u32> two_sided(d->emission_count);
        for (u32 i = 0; i < d->emission_count; ++i) {
            spectra.insert(spectra.end(), d->emissions[i].radiance, d->emissions[i].radiance + 471);
            two_sided[i] = d->emissions[i].two_sided;
        }
        std::vector<DPositional> pos(d->positional_count);
        for (u32 i = 0; i < d->positional_count; ++i) {
            const auto &q = d->positional[i];
            if (q.kind > RP_SPOT_LIGHT)
                throw Invalid{"unsupported positional light kind (point and spot are built)"};
            DPositional &L = pos[i];
            memcpy(L.position, q.position, sizeof(L.position));
            L.kind = q.kind;
            memcpy(L.light_from_world, q.light_from_world, sizeof(L.light_from_world));
            L.cos_falloff_start = q.cos_falloff_start;
            L.cos_falloff_end = q.cos_falloff_end;
            L.spectrum = u32(spectra.size());
            spectra.insert(spectra.end(), q.intensity, q.intensity + 471);
        }
        bool has_environment = false;
        ds.environment = kNone;
        if (d->environment) {
            has_environment = std::any_of(d->environment, d->environment + 471, [](float v) { return v > 0; });
            ds.environment = u32(spectra.size());
            spectra.insert(spectra.end(), d->environment, d->environment + 471);
        }
        ds.spectra = dupload(own, spectra.data(), spectra.size(), stm);
        ds.emission_two_sided = dupload(own, two_sided.data(), two_sided.size(), stm);
        ds.emission_count = d->emission_count;
        ds.positional = dupload(own, pos.data(), pos.size(), stm);
        ds.positional_count = d->positional_count;
        ds.emitter_instance = dupload(own, em_inst.data(), em_inst.size(), stm);
        ds.emitter_local = dupload(own, em_local.data(), em_local.size(), stm);
        ds.emitter_count = u32(em_inst.size());
        // images (RenderScene::image_textures ... environment_image, src/render.hpp:251-261),
        // uploaded in rypath's wire layout
        double env_power = -1;
        upload_images(d->images, d->instance_count, ds.img, own, stm, env_power);
        for (u32 i = 0; i < d->material_count; ++i)
            if (d->materials[i].kind == RP_REFLECTANCE_IMAGE && d->materials[i].scattering == RP_DIFFUSE)
                ds.img.textured = 1;
        s->scalar_full = s->scalar_full || ds.img.textured;
        // scene sphere (src/metal_render.mm:213-276) over the world vertices of k_tri_prepare
        int bounds[12];
        const auto t_wait = std::chrono::steady_clock::now();
        build_bounds(s, bounds);
        const auto t_bounds = std::chrono::steady_clock::now();
        double lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = unordered_host(bounds[6 + a]);
            hi[a] = unordered_host(bounds[9 + a]);
        }
        float scene_radius = 1;
        if (next_prim) {
            double c[3], e[3];
            for (int a = 0; a < 3; ++a) {
                c[a] = float(lo[a] / 2 + hi[a] / 2);
                e[a] = std::max(std::abs(lo[a] - c[a]), std::abs(hi[a] - c[a]));
                e[a] += 32 * FLT_EPSILON * std::max(std::abs(lo[a]), std::abs(hi[a]));
            }
            scene_radius = std::nextafter(float(std::hypot(e[0], e[1], e[2])), INFINITY);
        }
        ds.scene_radius = scene_radius;
        // light inputs (src/metal_render.mm:525-660, :1565-1660)
        std::vector<LightInput> input;
        const double pi = std::numbers::pi;
        std::vector<double> means(d->emission_count, -1), bounds_mean(d->emission_count, -1);
        for (u32 ii = 0; ii < d->instance_count; ++ii) {
            const DInstance &in = instances[ii];
            if (in.emission == kNone)
                continue;
            double &mean = means[in.emission], &bound = bounds_mean[in.emission];
            const float *rad = d->emissions[in.emission].radiance;
            if (mean < 0) {
                mean = light_spectrum_power(rad);
                bound = *std::max_element(rad, rad + 471);
            }
            const bool two = d->emissions[in.emission].two_sided != 0;
            for (u32 t = 0; t < in.triangle_count; ++t) {
                D3 p[3];
                for (int k = 0; k < 3; ++k) {
                    const float *q = d->positions + 3 * size_t(in.vertex_begin + d->triangles[3 * (in.triangle_begin + t) + k]);
                    for (int a = 0; a < 3; ++a)
                        p[k][a] = double(in.m[4 * a]) * q[0] + double(in.m[4 * a + 1]) * q[1] +
                                  double(in.m[4 * a + 2]) * q[2] + double(in.m[4 * a + 3]);
                }
                const D3 e1{p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
                const D3 e2{p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
                D3 nrm{e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
                if (in.reverse)
                    for (auto &v : nrm)
                        v = -v;
                LightInput li;
                for (int a = 0; a < 3; ++a) {
                    li.low[a] = INFINITY;
                    li.high[a] = -INFINITY;
                }
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a) {
                        li.low[a] = std::min(li.low[a], float(p[k][a]));
                        li.high[a] = std::max(li.high[a], float(p[k][a]));
                    }
                const double length = std::hypot(nrm[0], nrm[1], nrm[2]);
                const double area = .5 * length;
                li.power = pi * area * mean * 1 * (two ? 2 : 1);
                li.bounds_power = pi * area * bound * 1;
                li.two_sided = two;
                if (length > 0) {
                    for (int a = 0; a < 3; ++a)
                        li.direction[a] = float(nrm[a] / length);
                    li.cos_outer = std::nextafter(1.f, 0.f);
                }
                input.push_back(li);
            }
        }
        for (u32 i = 0; i < d->positional_count; ++i) {
            const auto &q = d->positional[i];
            LightInput li;
            for (int a = 0; a < 3; ++a)
                li.low[a] = li.high[a] = q.position[a];
            li.two_sided = false;
            li.bounds_power = 4 * pi * *std::max_element(q.intensity, q.intensity + 471);
            if (q.kind == RP_POINT_LIGHT) {
                li.power = 4 * pi * light_spectrum_power(q.intensity);
            } else {
                li.power = 2 * pi * ((1 - q.cos_falloff_start) + (q.cos_falloff_start - q.cos_falloff_end) / 2) *
                           light_spectrum_power(q.intensity);
                float cos_emission =
                    float(std::cos(std::acos(double(q.cos_falloff_end)) - std::acos(double(q.cos_falloff_start))));
                if (cos_emission == 1)
                    cos_emission = q.cos_falloff_end != q.cos_falloff_start ? .999f : std::nextafter(1.f, 0.f);
                // src/light_sampling.cpp:314-337 (light_positional_cone)
                const float *m = q.light_from_world;
                const D3 a{m[0], m[1], m[2]}, b{m[3], m[4], m[5]}, c{m[6], m[7], m[8]};
                const double aa = d3dot(a, a), bb = d3dot(b, b), cc = d3dot(c, c), tol = 0x1p-20 * aa;
                li.cos_outer = -1;
                li.cos_emission = 0;
                if ((aa > 0 && std::isfinite(aa)) && !(std::abs(aa - bb) > tol) && !(std::abs(aa - cc) > tol) &&
                    !(std::abs(d3dot(a, b)) > tol) && !(std::abs(d3dot(a, c)) > tol) && !(std::abs(d3dot(b, c)) > tol)) {
                    const D3 axis{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
                    const double det = d3dot(axis, c);
                    if (std::abs(det) > 0) {
                        const double length = d3norm(axis);
                        for (int k = 0; k < 3; ++k)
                            li.direction[k] = float(axis[k] / std::copysign(length, det));
                        li.cos_outer = float(std::cos(
                            std::min(pi, std::acos(std::clamp(double(q.cos_falloff_start), -1., 1.)) + 2e-6)));
                        li.cos_outer = std::max(-1.f, std::nextafter(li.cos_outer, -INFINITY));
                        li.cos_emission = cos_emission;
                    }
                }
            }
            input.push_back(li);
        }
        ds.environment_light = kNone;
        if (has_environment || env_power >= 0) {
            // an environment image replaces the constant environment (src/metal_render.mm:617-630)
            LightInput li;
            li.infinite = true;
            const double radius = std::max(double(scene_radius), 1e-8);
            li.power = 4 * pi * pi * radius * radius * (env_power >= 0 ? env_power : light_spectrum_power(d->environment));
            ds.environment_light = u32(input.size());
            input.push_back(li);
        }
        LightTables lt;
        std::string error;
        if (!build_light_tables(input, lt, error))
            throw Invalid{error};
        ds.light_nodes = dupload(own, lt.nodes.data(), lt.nodes.size(), stm);
        ds.light_alias = dupload(own, lt.alias.data(), lt.alias.size(), stm);
        ds.light_records = dupload(own, lt.records.data(), lt.records.size(), stm);
        ds.infinite_lights = dupload(own, lt.infinite.data(), lt.infinite.size(), stm);
        ds.light_node_count = u32(lt.nodes.size());
        ds.infinite_count = u32(lt.infinite.size());
        ds.light_count = u32(input.size());
        ds.light_sampler = d->light_sampler;
        // Sobol tables (sobol::Tables layout, src/sobol_shared.h:36-52)
        const unsigned char *tb = static_cast<const unsigned char *>(d->sobol_tables);
        ds.sobol.directions = dupload(own, reinterpret_cast<const u32 *>(tb), 1024 * 52, stm);
        ds.sobol.intervals = dupload(own, reinterpret_cast<const u64 *>(tb + 212992), 25 * 52, stm);
        ds.sobol.inverse = dupload(own, reinterpret_cast<const u64 *>(tb + 223392), 26 * 52, stm);
        ds.origin = v3(d->camera.origin[0], d->camera.origin[1], d->camera.origin[2]);
        ds.forward = v3(d->camera.corner[0], d->camera.corner[1], d->camera.corner[2]);
        ds.right = v3(d->camera.dx[0], d->camera.dx[1], d->camera.dx[2]);
        ds.up = v3(d->camera.dy[0], d->camera.dy[1], d->camera.dy[2]);
        ds.model = d->model == RP_MODEL_DEMO ? kModelDemo : kModelPbrt;
        ds.film_scale = d->film_scale;
        ds.filter_kind = d->filter_kind;
        ds.filter_x = d->filter_x_radius;
        ds.filter_y = d->filter_y_radius;
        ds.filter_weight = 1;
        ds.gauss_cdf = nullptr;
        ds.gauss_w = ds.gauss_h = 0;
        if (d->filter_kind == RP_FILTER_GAUSSIAN) {
            GaussianTable g;
            const std::string err = gaussian_table(d->filter_x_radius, d->filter_y_radius, d->filter_sigma, g);
            if (!err.empty())
                throw Invalid{err};
            std::vector<float> cdf(g.conditional);
            cdf.insert(cdf.end(), g.marginal.begin(), g.marginal.end());
            ds.gauss_cdf = dupload(own, cdf.data(), cdf.size(), stm);
            ds.gauss_w = g.width;
            ds.gauss_h = g.height;
            // the packet film weight of the hero transport (src/metal_render.mm:4851-4861)
            ds.filter_weight = d->transport == RP_TRANSPORT_HERO ? g.integral : 1.0f;
        }
        {
            // the first 1000 primes, the Halton bases (src/qmc_shared.h:14-18)
            std::vector<u32> primes;
            for (u32 n = 2; primes.size() < 1000; ++n) {
                bool prime = true;
                for (u32 q : primes) {
                    if (q * q > n)
                        break;
                    if (n % q == 0) {
                        prime = false;
                        break;
                    }
                }
                if (prime)
                    primes.push_back(n);
            }
            ds.primes = dupload(own, primes.data(), primes.size(), stm);
        }
        ds.lens_radius = d->lens_radius;
        ds.focal_distance = d->lens_radius > 0 ? d->focal_distance : 1e6f;
        ds.lens_x = v3(d->lens_x[0], d->lens_x[1], d->lens_x[2]);
        ds.lens_y = v3(d->lens_y[0], d->lens_y[1], d->lens_y[2]);
        ds.max_depth = d->max_depth;
        ds.hero_mode = d->hero_wavelengths;
        s->transport = d->transport;
        {
            std::vector<float> media(size_t(d->medium_count) * kMediumStride, 0.0f);
            for (u32 i = 0; i < d->medium_count; ++i) {
                float *m = media.data() + size_t(i) * kMediumStride;
                std::copy(d->media[i].sigma_a, d->media[i].sigma_a + 471, m);
                std::copy(d->media[i].sigma_s, d->media[i].sigma_s + 471, m + 471);
                std::copy(d->media[i].emission, d->media[i].emission + 471, m + 942);
                m[1413] = d->media[i].g;
            }
            ds.media = dupload(own, media.data(), media.size(), stm);
            ds.medium_count = d->medium_count;
            ds.camera_medium = scalar ? d->camera_medium : RP_NONE;
            ds.media_enabled = scalar && (d->medium_count > 0 || interfaces || d->camera_medium != RP_NONE);
        }
        {
            const float u = 0x1.0p-24f;
            const float g3 = 3.0f * u / (1.0f - 3.0f * u);
            ds.slab_scale = 1 + 2 * g3;
        }
        s->stats = dalloc<unsigned long long>(own, 8, stm);
        RP_CHECK(cudaMemsetAsync(s->stats, 0, 8 * sizeof(unsigned long long), stm));
        const auto t_host = std::chrono::steady_clock::now();
        build_finish(s, bounds);
        const auto t_end = std::chrono::steady_clock::now();
        s->timing.build_ms = std::chrono::duration<double, std::milli>(t_end - t_begin).count();
        // LBVH time: the two build halves' launches and device waits; host time: the rest
        using ms = std::chrono::duration<double, std::milli>;
        s->timing.build_bvh_ms =
            ms(t_end - t_host).count() + ms(t_bounds - t_wait).count() + ms(t_prepared - t_prepare).count();
        s->timing.build_host_ms = s->timing.build_ms - s->timing.build_bvh_ms;
        *out = s;
        return RP_SUCCESS;
    });
    if (st != RP_SUCCESS)
        delete s;
    return st;
}

void rp_cuda_scene_destroy(rp_scene *scene) { delete scene; }

rp_status rp_cuda_set_counting(rp_scene *s, int enabled) {
    if (!s)
        return RP_INVALID_ARGUMENT;
    s->counting = enabled != 0;
    return RP_SUCCESS;
}

rp_status rp_cuda_last_timing(rp_scene *s, rp_timing *t) {
    // build_* fields always describe scene creation
    if (!s || !t)
        return RP_INVALID_ARGUMENT;
    *t = s->timing;
    return RP_SUCCESS;
}

static rp_status sample_impl(rp_scene *s, const rp_request *request, rp_packet_result *out, size_t capacity, bool host,
                             cudaStream_t user, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request || !out)
            throw Invalid{"null argument"};
        const std::string err = validate_request(s, *request);
        if (!err.empty())
            throw Invalid{err};
        if (s->transport != RP_TRANSPORT_HERO)
            throw Invalid{"the scene was built for the scalar transport; sample it with rp_cuda_sample_scalar"};
        apply_texture_request(s, *request);
        const WaveParams p = wave_params(*request);
        if (capacity < p.lanes)
            throw Invalid{"output capacity is smaller than the request lanes"};
        RP_CHECK(cudaSetDevice(s->device));
        cudaEvent_t start, stop;
        RP_CHECK(cudaEventCreate(&start));
        RP_CHECK(cudaEventCreate(&stop));
        if (user) {
            RP_CHECK(cudaEventRecord(start, user));
            RP_CHECK(cudaStreamWaitEvent(s->stream, start, 0));
        }
        RP_CHECK(cudaEventRecord(start, s->stream));
        if (s->counting)
            RP_CHECK(cudaMemsetAsync(s->stats, 0, 8 * sizeof(unsigned long long), s->stream));
        run_wave(s, p);
        PacketResult *dst = reinterpret_cast<PacketResult *>(out);
        PacketResult *staging = nullptr;
        if (host) {
            RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&staging), size_t(p.lanes) * sizeof(PacketResult), s->stream));
            dst = staging;
        }
        s->mark(3);
        k_results<<<grid_for(s->sm_count, p.lanes, 256, 16), 256, 0, s->stream>>>(s->pool, p.lanes, s->ds.filter_weight, dst);
        s->done();
        u32 failures = 0;
        if (host) {
            RP_CHECK(cudaMemcpyAsync(out, staging, size_t(p.lanes) * sizeof(PacketResult), cudaMemcpyDeviceToHost, s->stream));
            RP_CHECK(cudaFreeAsync(staging, s->stream));
        }
        RP_CHECK(cudaEventRecord(stop, s->stream));
        if (user)
            RP_CHECK(cudaStreamWaitEvent(user, stop, 0));
        s->collect();
        float total = 0;
        RP_CHECK(cudaEventElapsedTime(&total, start, stop));
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        s->timing.total_ms = total;
        s->timing.samples = p.lanes;
        if (s->counting) {
            unsigned long long st[6];
            RP_CHECK(cudaMemcpy(st, s->stats, sizeof(st), cudaMemcpyDeviceToHost));
            s->timing.nodes_visited = st[0];
            s->timing.triangles_tested = st[1];
            s->timing.closest_rays = st[2];
            s->timing.shadow_rays = st[3];
            s->timing.shadow_nodes_visited = st[4];
            s->timing.shadow_triangles_tested = st[5];
        }
        if (host) {
            for (u32 i = 0; i < p.lanes; ++i)
                if (out[i].status != RP_SAMPLE_SUCCESS) {
                    if (!failures)
                        set_diag(diag, cap, "Metal render sample failed with status %u at lane %u", out[i].status, i);
                    ++failures;
                }
        }
        return failures ? RP_FAILURE : RP_SUCCESS;
    });
}

rp_status rp_cuda_sample(rp_scene *s, const rp_request *request, rp_packet_result *results, size_t capacity, char *diag,
                         size_t cap) {
    return sample_impl(s, request, results, capacity, true, nullptr, diag, cap);
}

rp_status rp_cuda_sample_device(rp_scene *s, const rp_request *request, rp_packet_result *results, size_t capacity,
                                void *stream, char *diag, size_t cap) {
    return sample_impl(s, request, results, capacity, false, static_cast<cudaStream_t>(stream), diag, cap);
}

static_assert(sizeof(ScalarResult) == sizeof(rp_scalar_result), "scalar result layout");

rp_status rp_cuda_sample_scalar(rp_scene *s, const rp_request *request, rp_scalar_result *out, size_t capacity,
                                char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request || !out)
            throw Invalid{"null argument"};
        const std::string err = validate_request(s, *request);
        if (!err.empty())
            throw Invalid{err};
        if (s->transport != RP_TRANSPORT_SCALAR)
            throw Invalid{"the scene was built for the hero transport; sample it with rp_cuda_sample"};
        apply_texture_request(s, *request);
        const WaveParams p = wave_params(*request);
        if (capacity < p.lanes)
            throw Invalid{"output capacity is smaller than the request lanes"};
        RP_CHECK(cudaSetDevice(s->device));
        cudaEvent_t start, stop;
        RP_CHECK(cudaEventCreate(&start));
        RP_CHECK(cudaEventCreate(&stop));
        RP_CHECK(cudaEventRecord(start, s->stream));
        if (s->counting)
            RP_CHECK(cudaMemsetAsync(s->stats, 0, 8 * sizeof(unsigned long long), s->stream));
        run_scalar_wave(s, p, request->boundary_limit ? request->boundary_limit : 4096u);
        ScalarResult *staging = nullptr;
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&staging), size_t(p.lanes) * sizeof(ScalarResult), s->stream));
        s->mark(3);
        k_scalar_results<<<grid_for(s->sm_count, p.lanes, 256, 16), 256, 0, s->stream>>>(s->ds, p, s->scalar_records,
                                                                                          staging);
        s->done();
        RP_CHECK(cudaMemcpyAsync(out, staging, size_t(p.lanes) * sizeof(ScalarResult), cudaMemcpyDeviceToHost,
                                 s->stream));
        RP_CHECK(cudaFreeAsync(staging, s->stream));
        RP_CHECK(cudaEventRecord(stop, s->stream));
        s->collect();
        float total = 0;
        RP_CHECK(cudaEventElapsedTime(&total, start, stop));
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        s->timing.total_ms = total;
        s->timing.samples = p.lanes;
        if (s->counting) {
            unsigned long long st[6];
            RP_CHECK(cudaMemcpy(st, s->stats, sizeof(st), cudaMemcpyDeviceToHost));
            s->timing.nodes_visited = st[0];
            s->timing.triangles_tested = st[1];
            s->timing.closest_rays = st[2];
            s->timing.shadow_rays = st[3];
            s->timing.shadow_nodes_visited = st[4];
            s->timing.shadow_triangles_tested = st[5];
        }
        u32 failures = 0;
        for (u32 i = 0; i < p.lanes; ++i)
            if (out[i].status != RP_SAMPLE_SUCCESS) {
                if (!failures)
                    set_diag(diag, cap, "Metal render sample failed with status %u at lane %u", out[i].status, i);
                ++failures;
            }
        return failures ? RP_FAILURE : RP_SUCCESS;
    });
}

static rp_status film_impl(rp_scene *s, const rp_film_request *r, rp_film_pixel *film, bool host, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !r || !film)
            throw Invalid{"null argument"};
        if (!r->width || !r->height || !r->sample_count || !r->batch_size)
            throw Invalid{"film request needs nonzero film size, samples and batch size"};
        const FilmClamp clamp = film_clamp(r->exposure, r->max_component_value);
        if (clamp.on && s && s->transport == RP_TRANSPORT_SCALAR)
            throw Invalid{"BDPT and finite film clamping require packet or hero spectral transport"};
        const u32 pixels = r->width * r->height;
        RP_CHECK(cudaSetDevice(s->device));
        if (!s->cie) {
            // CIE 1931 2-degree table at 1 nm is supplied by the caller's scene data; it is
            // uploaded lazily from the package data through rp_cuda_set_cie.
            throw Invalid{"CIE table not set (rp_cuda_set_cie)"};
        }
        // waves of whole sample indices over every pixel (canonical order within a batch)
        const u64 max_lanes = 1u << 23;
        const u64 samples_per_wave = std::max<u64>(1, std::min<u64>(r->batch_size, max_lanes / pixels));
        cudaEvent_t start, stop;
        RP_CHECK(cudaEventCreate(&start));
        RP_CHECK(cudaEventCreate(&stop));
        RP_CHECK(cudaEventRecord(start, s->stream));
        rp_film_pixel *committed = film;
        if (host) {
            if (s->film_stage_pixels < pixels) {
                if (s->film_stage)
                    cudaFreeAsync(s->film_stage, s->stream);
                RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&s->film_stage),
                                         size_t(pixels) * 2 * sizeof(rp_film_pixel), s->stream));
                s->film_stage_pixels = pixels;
            }
            committed = s->film_stage + pixels;
            if (r->flags & RP_FILM_FRESH)
                RP_CHECK(cudaMemsetAsync(committed, 0, size_t(pixels) * sizeof(rp_film_pixel), s->stream));
            else
                RP_CHECK(cudaMemcpyAsync(committed, film, size_t(pixels) * sizeof(rp_film_pixel),
                                         cudaMemcpyHostToDevice, s->stream));
        } else if (s->film_stage_pixels < pixels) {
            if (s->film_stage)
                cudaFreeAsync(s->film_stage, s->stream);
            RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&s->film_stage), size_t(pixels) * 2 * sizeof(rp_film_pixel),
                                     s->stream));
            s->film_stage_pixels = pixels;
        }
        rp_film_pixel *staged = s->film_stage;
        if (!host && (r->flags & RP_FILM_FRESH))
            RP_CHECK(cudaMemsetAsync(committed, 0, size_t(pixels) * sizeof(rp_film_pixel), s->stream));
        if (s->counting)
            RP_CHECK(cudaMemsetAsync(s->stats, 0, 8 * sizeof(unsigned long long), s->stream));
        u64 done = 0;
        u32 failed_batches = 0;
        while (done < r->sample_count) {
            const u64 batch = std::min<u64>(r->batch_size, r->sample_count - done);
            RP_CHECK(cudaMemcpyAsync(staged, committed, size_t(pixels) * sizeof(rp_film_pixel), cudaMemcpyDeviceToDevice,
                                     s->stream));
            // waves of whole sample indices over every pixel: each wave holds every BSDF family
            // of the image, so the family shade kernels, which run side by side, stay balanced
            // (waves over pixel bands, whose rows would be final early enough to read back beside
            // the render, measured slower: the bands' family mixes are uneven)
            u32 failures = 0;
            u64 in_batch = 0;
            while (in_batch < batch) {
                const u64 spw = std::min<u64>(samples_per_wave, batch - in_batch);
                rp_request q{};
                q.width = r->width;
                q.height = r->height;
                q.seed = r->seed;
                q.pixel_begin = 0;
                q.pixel_count = pixels;
                q.sample_begin = r->sample_begin + done + in_batch;
                q.sample_count = u32(spw);
                q.emergency_limit = r->emergency_limit;
                q.sampler_kind = r->sampler_kind;
                q.randomization = r->randomization;
                q.total_samples = r->total_samples ? r->total_samples : r->sample_begin + r->sample_count;
                const std::string err = validate_request(s, q);
                if (!err.empty())
                    throw Invalid{err};
                apply_texture_request(s, q);
                const WaveParams p = wave_params(q);
                u32 f = 0;
                if (s->transport == RP_TRANSPORT_SCALAR) {
                    run_scalar_wave(s, p, 4096u);
                    s->mark(3);
                    k_scalar_film<<<grid_for(s->sm_count, pixels, 128, 16), 128, 0, s->stream>>>(
                        s->scalar_records, pixels, u32(spw), s->cie, reinterpret_cast<FilmPixel *>(staged),
                        s->scalar_counters + 1, s->ds.model == kModelDemo ? 1u : 0u, s->demo_film_scale);
                    s->done();
                    RP_CHECK(cudaMemcpyAsync(&f, s->scalar_counters + 1, 4, cudaMemcpyDeviceToHost, s->stream));
                } else {
                    run_wave(s, p);
                    s->mark(3);
                    k_film<<<grid_for(s->sm_count, pixels, 128, 16), 128, 0, s->stream>>>(
                        s->pool, pixels, u32(spw), s->cie, double(s->ds.filter_weight), clamp,
                        reinterpret_cast<FilmPixel *>(staged));
                    s->done();
                    RP_CHECK(cudaMemcpyAsync(&f, s->pool.counters + 3, 4, cudaMemcpyDeviceToHost, s->stream));
                }
                RP_CHECK(cudaStreamSynchronize(s->stream));
                failures += f;
                in_batch += spw;
            }
            if (failures) {
                ++failed_batches;
                break; // keep the previously committed film (src/render_driver.cpp:201-214)
            }
            std::swap(staged, committed);
            done += batch;
        }
        if (host)
            RP_CHECK(cudaMemcpyAsync(film, committed, size_t(pixels) * sizeof(rp_film_pixel), cudaMemcpyDeviceToHost,
                                     s->stream));
        else if (committed != film)
            RP_CHECK(cudaMemcpyAsync(film, committed, size_t(pixels) * sizeof(rp_film_pixel), cudaMemcpyDeviceToDevice,
                                     s->stream));
        RP_CHECK(cudaEventRecord(stop, s->stream));
        s->collect();
        float total = 0;
        RP_CHECK(cudaEventElapsedTime(&total, start, stop));
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        s->timing.total_ms = total;
        s->timing.samples = done * pixels;
        if (s->counting) {
            unsigned long long st[6];
            RP_CHECK(cudaMemcpy(st, s->stats, sizeof(st), cudaMemcpyDeviceToHost));
            s->timing.nodes_visited = st[0];
            s->timing.triangles_tested = st[1];
            s->timing.closest_rays = st[2];
            s->timing.shadow_rays = st[3];
            s->timing.shadow_nodes_visited = st[4];
            s->timing.shadow_triangles_tested = st[5];
        }
        if (failed_batches) {
            set_diag(diag, cap, "a render batch failed; the committed film is unchanged");
            return RP_FAILURE;
        }
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_set_cie(rp_scene *s, const double *cie_xyz) {
    if (!s || !cie_xyz)
        return RP_INVALID_ARGUMENT;
    return guarded(nullptr, 0, [&]() -> rp_status {
        RP_CHECK(cudaSetDevice(s->device));
        if (!s->cie)
            s->cie = dalloc<double>(s->owned, 3 * 471, s->stream);
        RP_CHECK(cudaMemcpyAsync(s->cie, cie_xyz, 3 * 471 * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        RP_CHECK(cudaStreamSynchronize(s->stream));
        // the demo film's scale: 470 / the trapezoidal integral of y (integrate_y,
        // src/render.cpp:70-77)
        double integral = (cie_xyz[1] + cie_xyz[3 * 470 + 1]) / 2;
        for (int i = 1; i + 1 < 471; ++i)
            integral += cie_xyz[3 * i + 1];
        s->demo_film_scale = 470.0 / integral;
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_render_film(rp_scene *s, const rp_film_request *r, rp_film_pixel *film, char *diag, size_t cap) {
    return film_impl(s, r, film, true, diag, cap);
}
rp_status rp_cuda_render_film_device(rp_scene *s, const rp_film_request *r, rp_film_pixel *film, char *diag, size_t cap) {
    return film_impl(s, r, film, false, diag, cap);
}

// ---- differentiation

rp_status rp_cuda_set_knot_values(rp_scene *s, uint32_t first, uint32_t count, const float *values, char *diag,
                                  size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || (!values && count))
            throw Invalid{"null argument"};
        if (uint64_t(first) + count > s->ds.knot_count)
            throw Invalid{"knot range out of range"};
        for (u32 i = 0; i < count; ++i)
            if (!std::isfinite(values[i]))
                throw Invalid{"knot values must be finite"};
        RP_CHECK(cudaSetDevice(s->device));
        if (count) {
            float2 *dst = const_cast<float2 *>(s->ds.knots) + first;
            RP_CHECK(cudaMemcpy2DAsync(reinterpret_cast<float *>(dst) + 1, sizeof(float2), values, sizeof(float),
                                       sizeof(float), count, cudaMemcpyHostToDevice, s->stream));
            RP_CHECK(cudaStreamSynchronize(s->stream));
        }
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_adjoint_device(rp_scene *s, const rp_adjoint_request *r, const double *d_loss_d_xyz, float *gradient,
                                 char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !r || !d_loss_d_xyz || !gradient || (r->material_count && !r->materials))
            throw Invalid{"null argument"};
        if (s->transport != RP_TRANSPORT_HERO)
            throw Invalid{"the adjoint differentiates hero-transport renders"};
        const rp_film_request &f = r->film;
        if (!f.width || !f.height || !f.sample_count || !f.batch_size)
            throw Invalid{"film request needs nonzero film size, samples and batch size"};
        if (s->ds.max_depth > 15)
            throw Invalid{"the adjoint records at most 16 vertices: max depth must be at most 15"};
        if (s->ds.material_count > 255)
            throw Invalid{"the adjoint addresses at most 255 materials"};
        // gradient slots of the parameter materials
        std::vector<u32> slot(std::max<u32>(1, s->ds.material_count), kNone);
        std::vector<DMaterial> mats(s->ds.material_count);
        RP_CHECK(cudaSetDevice(s->device));
        RP_CHECK(cudaMemcpy(mats.data(), s->ds.materials, mats.size() * sizeof(DMaterial), cudaMemcpyDeviceToHost));
        u32 params = 0;
        for (u32 i = 0; i < r->material_count; ++i) {
            const u32 m = r->materials[i];
            if (m >= s->ds.material_count)
                throw Invalid{"adjoint material out of range"};
            if (slot[m] != kNone)
                throw Invalid{"adjoint material listed twice"};
            if (mats[m].scattering != RP_DIFFUSE || mats[m].kind != RP_REFLECTANCE_KNOTS || mats[m].knot_count < 2)
                throw Invalid{"adjoint materials must be diffuse with knot reflectance"};
            slot[m] = params;
            params += mats[m].knot_count;
        }
        if (params > 2048)
            throw Invalid{"the adjoint accumulates at most 2048 gradient entries"};
        if (!s->cie)
            throw Invalid{"CIE table not set (rp_cuda_set_cie)"};
        const u32 pixels = f.width * f.height;
        const u64 max_lanes = 1u << 23;
        const u64 samples_per_wave = std::max<u64>(1, std::min<u64>(f.batch_size, max_lanes / pixels));
        const u32 lanes_cap = u32(std::min<u64>(max_lanes, samples_per_wave * pixels));
        s->ensure_pool(lanes_cap);
        if (s->adjoint_capacity < s->capacity) {
            if (s->adjoint_storage)
                cudaFreeAsync(s->adjoint_storage, s->stream);
            s->adjoint_storage = nullptr;
            s->adjoint_capacity = 0;
            RP_CHECK(cudaMallocAsync(&s->adjoint_storage, size_t(s->capacity) * 32, s->stream));
            s->adjoint_capacity = s->capacity;
        }
        u32 *slot_dev = nullptr;
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&slot_dev), slot.size() * 4, s->stream));
        RP_CHECK(cudaMemcpyAsync(slot_dev, slot.data(), slot.size() * 4, cudaMemcpyHostToDevice, s->stream));
        RP_CHECK(cudaMemsetAsync(gradient, 0, size_t(std::max<u32>(params, 1)) * sizeof(float), s->stream));
        PathPool &pool = s->pool;
        const PathPool saved = pool;
        pool.hist = reinterpret_cast<uint4 *>(s->adjoint_storage);
        pool.adj_w = reinterpret_cast<float4 *>(static_cast<unsigned char *>(s->adjoint_storage) +
                                                size_t(s->adjoint_capacity) * 16);
        pool.adj_slot = slot_dev;
        pool.adj_grad = gradient;
        pool.adj_g = d_loss_d_xyz;
        pool.adj_cie = s->cie;
        pool.adj_inv_weight = 1.0 / double(f.sample_count);
        pool.adj_params = params;
        cudaEvent_t start, stop;
        RP_CHECK(cudaEventCreate(&start));
        RP_CHECK(cudaEventCreate(&stop));
        RP_CHECK(cudaEventRecord(start, s->stream));
        u32 failures = 0;
        try {
            u64 done = 0;
            while (done < f.sample_count) {
                const u64 spw = std::min<u64>(samples_per_wave, f.sample_count - done);
                rp_request q{};
                q.width = f.width;
                q.height = f.height;
                q.seed = f.seed;
                q.pixel_count = pixels;
                q.sample_begin = f.sample_begin + done;
                q.sample_count = u32(spw);
                q.emergency_limit = f.emergency_limit;
                q.sampler_kind = f.sampler_kind;
                q.randomization = f.randomization;
                q.total_samples = f.total_samples ? f.total_samples : f.sample_begin + f.sample_count;
                const std::string err = validate_request(s, q);
                if (!err.empty())
                    throw Invalid{err};
                apply_texture_request(s, q);
                const WaveParams p = wave_params(q);
                run_wave(s, p, size_t(params) * sizeof(float));
                // a failed lane (as in the forward film) fails the gradient
                s->mark(3);
                k_count_failures<<<grid_for(s->sm_count, p.lanes, 256, 8), 256, 0, s->stream>>>(pool, p.lanes);
                s->done();
                u32 wave_failures = 0;
                RP_CHECK(cudaMemcpyAsync(&wave_failures, pool.counters + 3, 4, cudaMemcpyDeviceToHost, s->stream));
                RP_CHECK(cudaStreamSynchronize(s->stream));
                failures += wave_failures;
                done += spw;
            }
            RP_CHECK(cudaEventRecord(stop, s->stream));
            s->collect();
        } catch (...) {
            pool = saved;
            cudaFreeAsync(slot_dev, s->stream);
            cudaEventDestroy(start);
            cudaEventDestroy(stop);
            throw;
        }
        pool = saved;
        cudaFreeAsync(slot_dev, s->stream);
        float total = 0;
        RP_CHECK(cudaEventElapsedTime(&total, start, stop));
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        s->timing.total_ms = total;
        s->timing.samples = f.sample_count * pixels;
        if (failures) {
            set_diag(diag, cap, "%u lanes failed; the gradient is not valid", failures);
            return RP_FAILURE;
        }
        return RP_SUCCESS;
    });
}

// ---- batched views

} // extern "C"

namespace {

struct BatchPlan {
    std::vector<DView> views;
    std::vector<WaveDesc> waves;
    unsigned long long lanes = 0, film_pixels = 0;
};

u32 sobol_scale_exponent(u32 width, u32 height) {
    const u32 v = std::max(std::max(width, height), 1u) - 1;
    return v == 0 ? 0 : 32 - __builtin_clz(v);
}

BatchPlan plan_batch(const rp_view *views, u32 count, const rp_batch_request &r, u32 wave_lanes) {
    if (!views || !count)
        throw Invalid{"a batch needs at least one view"};
    if (r.sampler_kind != RP_SAMPLER_SOBOL && r.sampler_kind != RP_SAMPLER_INDEPENDENT)
        throw Invalid{"batched views use the independent or Sobol sampler"};
    if (r.sampler_kind == RP_SAMPLER_SOBOL && r.randomization > 3)
        throw Invalid{"Invalid Sobol randomization"};
    BatchPlan plan;
    unsigned long long film_end = 0;
    for (u32 i = 0; i < count; ++i) {
        const rp_view &v = views[i];
        if (!v.width || !v.height || !v.sample_count)
            throw Invalid{"every view needs a nonzero film and sample count"};
        if (uint64_t(v.width) * v.height > 0xffffffffull || v.sample_count > 0xffffffffull)
            throw Invalid{"view film or sample count too large"};
        if (r.sampler_kind == RP_SAMPLER_SOBOL && std::max(v.width, v.height) > (1u << 25))
            throw Invalid{"Sobol film exceeds 2^25 pixels per side"};
        if (v.sample_begin > UINT64_MAX - (v.sample_count - 1))
            throw Invalid{"Sampler range must fit the absolute sample indices"};
        if (v.film_offset < film_end)
            throw Invalid{"view films must be in view order and must not overlap"};
        DView d{};
        d.cam = RasterCam{v3(v.camera.origin[0], v.camera.origin[1], v.camera.origin[2]),
                          v3(v.camera.corner[0], v.camera.corner[1], v.camera.corner[2]),
                          v3(v.camera.dx[0], v.camera.dx[1], v.camera.dx[2]),
                          v3(v.camera.dy[0], v.camera.dy[1], v.camera.dy[2])};
        d.width = v.width;
        d.height = v.height;
        d.m = r.sampler_kind == RP_SAMPLER_SOBOL ? sobol_scale_exponent(v.width, v.height) : 0;
        d.pixels = v.width * v.height;
        d.sample_low = u32(v.sample_begin);
        d.sample_high = u32(v.sample_begin >> 32);
        d.spp = u32(v.sample_count);
        d.lane_begin = plan.lanes;
        d.film_begin = v.film_offset;
        plan.lanes += uint64_t(d.pixels) * d.spp;
        film_end = v.film_offset + d.pixels;
        plan.views.push_back(d);
    }
    plan.film_pixels = film_end;
    wave_lanes = std::max<u32>(1, std::min<u32>(wave_lanes, 1u << 23));
    for (unsigned long long l = 0; l < plan.lanes; l += wave_lanes)
        plan.waves.push_back(WaveDesc{l, u32(std::min<unsigned long long>(wave_lanes, plan.lanes - l)), 0});
    return plan;
}

WaveParams batch_params(const rp_batch_request &r) {
    WaveParams p{};
    p.seed_low = u32(r.seed);
    p.seed_high = u32(r.seed >> 32);
    p.sampler = r.sampler_kind;
    p.randomization = r.randomization;
    p.emergency_limit = r.emergency_limit ? r.emergency_limit : 1024;
    p.boundary_limit = 4096;
    return p;
}

template <int TB, int SB>
void batch_wave_kernels(rp_scene *s, const WaveParams &p, const Batch &b, u32 wave_lanes, u32 blocks_per_sm,
                        const FilmClamp &clamp, FilmPixel *film) {
    PathPool &pool = s->pool;
    const int sms = s->sm_count;
    cudaStream_t st = s->stream;
    RP_CHECK(cudaMemsetAsync(pool.counters, 0, 16 * sizeof(u32), st));
    k_raygen_views<<<grid_for(sms, wave_lanes, 256, 16), 256, 0, st>>>(s->ds, p, b, pool);
    const int trace_grid = grid_for(sms, wave_lanes, TB, int(blocks_per_sm * 128 / TB));
    const int shade_grid = grid_for(sms, wave_lanes, SB, int(blocks_per_sm * 128 / SB));
    // the same stream layout as run_wave: family shade kernels side by side, each event's
    // shadow walks beside the next event's closest-hit walk (in a captured graph these forks
    // and joins become parallel branches)
    int in = 0;
    bool shadow_pending = false;
    for (u32 e = 0; e <= s->ds.max_depth; ++e) {
        RP_CHECK(cudaMemsetAsync(pool.counters + 4, 0, 4 * sizeof(u32), st));
        launch_trace<false, TB>(s, pool, in, trace_grid, st, p.boundary_limit);
        if (shadow_pending) {
            RP_CHECK(cudaStreamWaitEvent(st, s->joined, 0));
            shadow_pending = false;
        }
        RP_CHECK(cudaMemsetAsync(pool.counters + (in ^ 1), 0, sizeof(u32), st));
        RP_CHECK(cudaMemsetAsync(pool.counters + 2, 0, sizeof(u32), st));
        RP_CHECK(cudaMemsetAsync(pool.counters + 8, 0, 3 * sizeof(u32), st));
        RP_CHECK(cudaEventRecord(s->forked, st));
        for (int k = 0; k < 3; ++k)
            RP_CHECK(cudaStreamWaitEvent(s->family[k], s->forked, 0));
        k_shade<0, SB><<<shade_grid, SB, 0, st>>>(s->ds, p, pool, in);
        k_nee<0, SB><<<shade_grid, SB, 0, st>>>(s->ds, p, pool);
        k_shade<1, SB><<<shade_grid, SB, 0, s->family[0]>>>(s->ds, p, pool, in);
        k_nee<1, SB><<<shade_grid, SB, 0, s->family[0]>>>(s->ds, p, pool);
        k_shade<2, SB><<<shade_grid, SB, 0, s->family[1]>>>(s->ds, p, pool, in);
        k_nee<2, SB><<<shade_grid, SB, 0, s->family[1]>>>(s->ds, p, pool);
        k_shade<3, SB><<<shade_grid, SB, 0, s->family[2]>>>(s->ds, p, pool, in);
        for (int k = 0; k < 3; ++k) {
            RP_CHECK(cudaEventRecord(s->family_done[k], s->family[k]));
            RP_CHECK(cudaStreamWaitEvent(st, s->family_done[k], 0));
        }
        RP_CHECK(cudaEventRecord(s->forked, st));
        RP_CHECK(cudaStreamWaitEvent(s->side, s->forked, 0));
        launch_shadow<false, TB, false>(s, pool, trace_grid, 0, s->side, p.boundary_limit);
        RP_CHECK(cudaEventRecord(s->joined, s->side));
        shadow_pending = true;
        in ^= 1;
    }
    if (shadow_pending)
        RP_CHECK(cudaStreamWaitEvent(st, s->joined, 0));
    k_film_views<<<grid_for(sms, wave_lanes, 128, 16), 128, 0, st>>>(pool, b, s->cie, double(s->ds.filter_weight), clamp,
                                                                       film);
    k_next_wave<<<1, 32, 0, st>>>(b);
    RP_CHECK(cudaGetLastError());
}

void batch_wave(rp_scene *s, const WaveParams &p, const Batch &b, const rp_batch_config &c, const FilmClamp &clamp,
                FilmPixel *film) {
    const u32 w = c.wave_lanes, bpm = c.blocks_per_sm;
    if (c.trace_block == 64 && c.shade_block == 128)
        batch_wave_kernels<64, 128>(s, p, b, w, bpm, clamp, film);
    else if (c.trace_block == 64 && c.shade_block == 256)
        batch_wave_kernels<64, 256>(s, p, b, w, bpm, clamp, film);
    else if (c.trace_block == 128 && c.shade_block == 256)
        batch_wave_kernels<128, 256>(s, p, b, w, bpm, clamp, film);
    else
        batch_wave_kernels<128, 128>(s, p, b, w, bpm, clamp, film);
}

void check_config(const rp_batch_config &c) {
    if (c.trace_block != 64 && c.trace_block != 128)
        throw Invalid{"trace block must be 64 or 128 threads"};
    if (c.shade_block != 128 && c.shade_block != 256)
        throw Invalid{"shade block must be 128 or 256 threads"};
    if (c.blocks_per_sm < 1 || c.blocks_per_sm > 32)
        throw Invalid{"blocks per SM must be 1..32"};
    if (!c.wave_lanes || c.wave_lanes > (1u << 23))
        throw Invalid{"wave lanes must be 1..2^23"};
}

// Device copies of a plan; freed on the scene stream when the holder goes out of scope.
struct BatchBuffers {
    rp_scene *s;
    DView *views = nullptr;
    WaveDesc *waves = nullptr;
    u32 *cursor = nullptr;
    BatchBuffers(rp_scene *scene, const BatchPlan &plan) : s(scene) {
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&views), plan.views.size() * sizeof(DView), s->stream));
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&waves), plan.waves.size() * sizeof(WaveDesc), s->stream));
        RP_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&cursor), 64, s->stream));
        RP_CHECK(cudaMemcpyAsync(views, plan.views.data(), plan.views.size() * sizeof(DView), cudaMemcpyHostToDevice,
                                 s->stream));
        RP_CHECK(cudaMemcpyAsync(waves, plan.waves.data(), plan.waves.size() * sizeof(WaveDesc),
                                 cudaMemcpyHostToDevice, s->stream));
        RP_CHECK(cudaMemsetAsync(cursor, 0, 64, s->stream));
    }
    ~BatchBuffers() {
        cudaFreeAsync(views, s->stream);
        cudaFreeAsync(waves, s->stream);
        cudaFreeAsync(cursor, s->stream);
        cudaStreamSynchronize(s->stream);
    }
    Batch batch(const BatchPlan &plan) const {
        return Batch{views, u32(plan.views.size()), waves, cursor, plan.film_pixels};
    }
};

// Runs `waves` waves of the plan from wave 0, as graph replays or direct launches; returns the
// device time in ms.
float run_batch(rp_scene *s, const BatchPlan &plan, const BatchBuffers &buf, const rp_batch_request &r,
                const rp_batch_config &c, FilmPixel *film, size_t waves) {
    s->ensure_pool(c.wave_lanes);
    WaveParams p = batch_params(r);
    attach_owen_prefix(s, p);
    const FilmClamp clamp = film_clamp(r.exposure, r.max_component_value);
    const Batch b = buf.batch(plan);
    RP_CHECK(cudaMemsetAsync(buf.cursor, 0, 8, s->stream));
    // the events, the captured graph and its executable are released on every exit, error
    // paths included (a failed launch or timing call throws)
    struct Owned {
        cudaEvent_t start = nullptr, stop = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        ~Owned() {
            if (exec)
                cudaGraphExecDestroy(exec);
            if (graph)
                cudaGraphDestroy(graph);
            if (start)
                cudaEventDestroy(start);
            if (stop)
                cudaEventDestroy(stop);
        }
    } o;
    RP_CHECK(cudaEventCreate(&o.start));
    RP_CHECK(cudaEventCreate(&o.stop));
    if (c.use_graph != 2) {
        RP_CHECK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        try {
            batch_wave(s, p, b, c, clamp, film);
        } catch (...) {
            cudaStreamEndCapture(s->stream, &o.graph);
            throw;
        }
        RP_CHECK(cudaStreamEndCapture(s->stream, &o.graph));
        RP_CHECK(cudaGraphInstantiate(&o.exec, o.graph, 0));
    }
    RP_CHECK(cudaEventRecord(o.start, s->stream));
    for (size_t w = 0; w < waves; ++w) {
        if (o.exec)
            RP_CHECK(cudaGraphLaunch(o.exec, s->stream));
        else
            batch_wave(s, p, b, c, clamp, film);
    }
    RP_CHECK(cudaEventRecord(o.stop, s->stream));
    RP_CHECK(cudaStreamSynchronize(s->stream));
    float ms = 0;
    RP_CHECK(cudaEventElapsedTime(&ms, o.start, o.stop));
    return ms;
}

// Coordinate search over the configuration, one probe wave per candidate (a warm-up replay,
// then a timed one), keeping the fields the request fixes.
rp_batch_config tune_batch(rp_scene *s, const rp_view *views, u32 count, const rp_batch_request &r) {
    rp_batch_config best = r.config;
    const bool fixed_wave = best.wave_lanes != 0, fixed_tb = best.trace_block != 0, fixed_sb = best.shade_block != 0,
               fixed_bpm = best.blocks_per_sm != 0;
    if (!best.use_graph)
        best.use_graph = 1;
    if (!fixed_tb)
        best.trace_block = 128;
    if (!fixed_sb)
        best.shade_block = 128;
    if (!fixed_bpm)
        best.blocks_per_sm = 12;
    const BatchPlan whole = plan_batch(views, count, r, 1u << 23);
    float best_cost = INFINITY;
    auto probe = [&](rp_batch_config c) {
        const BatchPlan plan = plan_batch(views, count, r, c.wave_lanes);
        const BatchBuffers buf(s, plan);
        run_batch(s, plan, buf, r, c, nullptr, 1); // warm-up (module load, pool growth)
        const float ms = run_batch(s, plan, buf, r, c, nullptr, 1);
        const float cost = ms / (float(plan.waves[0].lanes) * 1e-6f);
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    };
    std::vector<u32> sizes;
    if (fixed_wave) {
        sizes.push_back(best.wave_lanes);
    } else {
        for (u32 w = 1u << 20; w <= (1u << 23); w <<= 1)
            if (w <= whole.lanes || sizes.empty())
                sizes.push_back(u32(std::min<unsigned long long>(w, whole.lanes)));
    }
    rp_batch_config c = best;
    for (u32 w : sizes) {
        c.wave_lanes = w;
        probe(c);
    }
    c = best;
    if (!fixed_tb)
        for (u32 tb : {64u, 128u})
            if (tb != best.trace_block) {
                c = best;
                c.trace_block = tb;
                probe(c);
            }
    if (!fixed_sb)
        for (u32 sb : {128u, 256u})
            if (sb != best.shade_block) {
                c = best;
                c.shade_block = sb;
                probe(c);
            }
    if (!fixed_bpm)
        for (u32 bpm : {8u, 16u})
            if (bpm != best.blocks_per_sm) {
                c = best;
                c.blocks_per_sm = bpm;
                probe(c);
            }
    best.probe_ms_per_mlane = best_cost;
    return best;
}

} // namespace

// A float-in, float-out probe kernel over `count` queries of `in` and `out` floats each.
template <typename Launch>
rp_status float_probe(const float *queries, uint32_t count, u32 in, u32 out, float *results, char *diag, size_t cap,
                      Launch launch) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        if (count == 0)
            return RP_SUCCESS;
        const float *q = dupload(own, queries, size_t(in) * count, nullptr);
        float *r = dalloc<float>(own, size_t(out) * count);
        launch(q, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(out) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

extern "C" {

rp_status rp_cuda_tune_views(rp_scene *s, const rp_view *views, uint32_t count, const rp_batch_request *request,
                             rp_batch_config *chosen, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request || !chosen)
            throw Invalid{"null argument"};
        if (s->transport != RP_TRANSPORT_HERO)
            throw Invalid{"batched views render hero-transport scenes"};
        if (s->ds.lens_radius > 0)
            throw Invalid{"batched views render pinhole cameras"};
        if (s->ds.img.textured)
            throw NotBuilt{"batched views of scenes with image reflectance are not built (their texture cameras differ per view)"};
        RP_CHECK(cudaSetDevice(s->device));
        if (!s->cie)
            throw Invalid{"CIE table not set (rp_cuda_set_cie)"};
        *chosen = tune_batch(s, views, count, *request);
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_render_views_device(rp_scene *s, const rp_view *views, uint32_t count, const rp_batch_request *request,
                                      rp_film_pixel *device_film, rp_batch_config *used, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request || !device_film)
            throw Invalid{"null argument"};
        if (s->transport != RP_TRANSPORT_HERO)
            throw Invalid{"batched views render hero-transport scenes"};
        if (s->ds.lens_radius > 0)
            throw Invalid{"batched views render pinhole cameras"};
        if (s->ds.img.textured)
            throw NotBuilt{"batched views of scenes with image reflectance are not built (their texture cameras differ per view)"};
        RP_CHECK(cudaSetDevice(s->device));
        if (!s->cie)
            throw Invalid{"CIE table not set (rp_cuda_set_cie)"};
        rp_batch_config c = request->config;
        if (!c.wave_lanes || !c.trace_block || !c.shade_block || !c.blocks_per_sm)
            c = tune_batch(s, views, count, *request);
        if (!c.use_graph)
            c.use_graph = 1;
        check_config(c);
        const BatchPlan plan = plan_batch(views, count, *request, c.wave_lanes);
        const BatchBuffers buf(s, plan);
        const float ms = run_batch(s, plan, buf, *request, c, reinterpret_cast<FilmPixel *>(device_film),
                                   plan.waves.size());
        u32 failures = 0;
        RP_CHECK(cudaMemcpy(&failures, buf.cursor + 1, 4, cudaMemcpyDeviceToHost));
        const rp_timing build = s->timing;
        s->timing = rp_timing{};
        s->timing.build_ms = build.build_ms;
        s->timing.build_host_ms = build.build_host_ms;
        s->timing.build_bvh_ms = build.build_bvh_ms;
        s->timing.total_ms = ms;
        s->timing.samples = plan.lanes;
        s->timing.kernel_launches = uint64_t(plan.waves.size()) * (3 + 6 * (s->ds.max_depth + 1));
        if (used)
            *used = c;
        if (failures) {
            set_diag(diag, cap, "%u lanes of the batch failed", failures);
            return RP_FAILURE;
        }
        return RP_SUCCESS;
    });
}

// ---- probes

rp_status rp_cuda_probe_sobol(const void *tables, const uint32_t *queries, uint32_t count, uint32_t *results, char *diag,
                              size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const unsigned char *tb = static_cast<const unsigned char *>(tables);
        SobolTables t;
        t.directions = dupload(own, reinterpret_cast<const u32 *>(tb), 1024 * 52, nullptr);
        t.intervals = dupload(own, reinterpret_cast<const u64 *>(tb + 212992), 25 * 52, nullptr);
        t.inverse = dupload(own, reinterpret_cast<const u64 *>(tb + 223392), 26 * 52, nullptr);
        const u32 *q = dupload(own, queries, size_t(8) * count, nullptr);
        u32 *r = dalloc<u32>(own, size_t(6) * count);
        k_probe_sobol<<<(count + 127) / 128, 128>>>(t, q, count, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(6) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_philox(const uint32_t *queries, uint32_t count, uint32_t *results, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const u32 *q = dupload(own, queries, size_t(6) * count, nullptr);
        u32 *r = dalloc<u32>(own, size_t(4) * count);
        k_probe_philox<<<(count + 127) / 128, 128>>>(q, count, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(4) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_bilinear(const float *queries, uint32_t count, float *results, char *diag, size_t cap) {
    return float_probe(queries, count, 20, 4, results, diag, cap, [&](const float *q, float *r) {
        k_probe_bilinear<<<(count + 127) / 128, 128>>>(q, count, r);
    });
}

rp_status rp_cuda_probe_analytic(const float *queries, uint32_t count, float *results, char *diag, size_t cap) {
    return float_probe(queries, count, 16, 16, results, diag, cap, [&](const float *q, float *r) {
        k_probe_analytic<<<(count + 127) / 128, 128>>>(q, count, r);
    });
}

rp_status rp_cuda_probe_wavelengths(const float *u, uint32_t count, uint32_t mode, float *results, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const float *q = dupload(own, u, count, nullptr);
        float *r = dalloc<float>(own, size_t(8) * count);
        k_probe_wavelengths<<<(count + 127) / 128, 128>>>(q, count, mode, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(8) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_bsdf(const float *queries, uint32_t count, float *results, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const float *q = dupload(own, queries, size_t(16) * count, nullptr);
        float *r = dalloc<float>(own, size_t(12) * count);
        k_probe_bsdf<<<(count + 127) / 128, 128>>>(q, count, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(12) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_image_lookup(const rp_images *images, uint32_t index, const float *queries, uint32_t count,
                                     float *results, char *diag, size_t cap) {
    if (images && index >= images->texture_count)
        return guarded(diag, cap, []() -> rp_status { throw Invalid{"texture index out of range"}; });
    return image_probe(images, queries, count, 6, 4, results, diag, cap, [&](const DImages &g, const float *q, float *r) {
        k_probe_image_lookup<<<(count + 127) / 128, 128>>>(g, index, q, count, r);
    });
}

rp_status rp_cuda_probe_rgb_spectrum(const rp_images *images, const float *queries, uint32_t count, float *results,
                                     char *diag, size_t cap) {
    if (images && !images->rgb_table)
        return guarded(diag, cap, []() -> rp_status { throw Invalid{"no sRGB reconstruction table"}; });
    return image_probe(images, queries, count, 4, 2, results, diag, cap, [&](const DImages &g, const float *q, float *r) {
        k_probe_rgb_spectrum<<<(count + 127) / 128, 128>>>(g.rgb_table, q, count, r);
    });
}

rp_status rp_cuda_probe_environment(const rp_images *images, const float *queries, uint32_t count, float *results,
                                    char *diag, size_t cap) {
    if (images && images->environment_image == RP_NONE)
        return guarded(diag, cap, []() -> rp_status { throw Invalid{"no environment image"}; });
    return image_probe(images, queries, count, 8, 12, results, diag, cap, [&](const DImages &g, const float *q, float *r) {
        k_probe_environment<<<(count + 127) / 128, 128>>>(g, q, count, r);
    });
}

rp_status rp_cuda_probe_texture_footprint(const float *queries, uint32_t count, float *results, char *diag,
                                          size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const float *q = dupload(own, queries, size_t(48) * count, nullptr);
        float *r = dalloc<float>(own, size_t(24) * count);
        k_probe_texture_footprint<<<(count + 127) / 128, 128>>>(q, count, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(24) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_texture_camera_differentials(const rp_camera *camera, uint32_t width, uint32_t height,
                                               float *minimum_dx, float *minimum_dy, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!camera || !minimum_dx || !minimum_dy)
            throw Invalid{"null argument"};
        const std::string err = texture_camera_differentials(
            v3(camera->corner[0], camera->corner[1], camera->corner[2]), v3(camera->dx[0], camera->dx[1], camera->dx[2]),
            v3(camera->dy[0], camera->dy[1], camera->dy[2]), width, height, minimum_dx, minimum_dy);
        if (!err.empty())
            throw Invalid{err};
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_environment_tables(const rp_images *images, float *cdf, size_t capacity, uint32_t *width,
                                     uint32_t *compensated_offset, double *mean_power, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!images || !cdf || !width || !compensated_offset || !mean_power)
            throw Invalid{"null argument"};
        rp_scene_desc d{};
        d.images = images;
        if (const std::string err = validate_images(&d); !err.empty())
            throw Invalid{err};
        if (images->environment_image == RP_NONE)
            throw Invalid{"no environment image"};
        std::vector<float> tables;
        const std::string err = environment_tables(*images, tables, *width, *compensated_offset, *mean_power);
        if (!err.empty())
            throw Invalid{err};
        if (tables.size() > capacity)
            throw Invalid{"capacity too small"};
        std::copy(tables.begin(), tables.end(), cdf);
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_hero(const float *queries, uint32_t count, float *results, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *p : o)
                    cudaFreeAsync(p, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const float *q = dupload(own, queries, size_t(32) * count, nullptr);
        float *r = dalloc<float>(own, size_t(32) * count);
        k_probe_hero<<<(count + 127) / 128, 128>>>(q, count, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpy(results, r, size_t(32) * count * 4, cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_probe_raygen(rp_scene *s, const rp_request *request, uint32_t *words, float *rays, size_t capacity,
                               char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request)
            throw Invalid{"null argument"};
        const std::string err = validate_request(s, *request);
        if (!err.empty())
            throw Invalid{err};
        const WaveParams p = wave_params(*request);
        if (capacity < p.lanes)
            throw Invalid{"capacity too small"};
        RP_CHECK(cudaSetDevice(s->device));
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *q : o)
                    cudaFreeAsync(q, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        u32 *w = dalloc<u32>(own, size_t(11) * p.lanes);
        float *r = dalloc<float>(own, size_t(6) * p.lanes);
        k_probe_raygen<<<(p.lanes + 127) / 128, 128, 0, s->stream>>>(s->ds, p, w, r);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpyAsync(words, w, size_t(11) * p.lanes * 4, cudaMemcpyDeviceToHost, s->stream));
        RP_CHECK(cudaMemcpyAsync(rays, r, size_t(6) * p.lanes * 4, cudaMemcpyDeviceToHost, s->stream));
        RP_CHECK(cudaStreamSynchronize(s->stream));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_scene_export_wide(rp_scene *s, void *nodes, size_t node_capacity, float *triangles,
                                    size_t triangle_capacity, uint32_t *node_count, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !node_count)
            throw Invalid{"null argument"};
        *node_count = s->ds.wnode_count;
        if (node_capacity < s->ds.wnode_count || triangle_capacity < s->n)
            throw Invalid{"capacity too small"};
        RP_CHECK(cudaSetDevice(s->device));
        if (s->ds.wnode_count)
            RP_CHECK(cudaMemcpy(nodes, s->ds.wnodes, size_t(s->ds.wnode_count) * sizeof(WNode), cudaMemcpyDeviceToHost));
        if (s->n)
            RP_CHECK(cudaMemcpy(triangles, s->ds.wtri, size_t(s->n) * 3 * sizeof(float4), cudaMemcpyDeviceToHost));
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_scene_export_bvh(rp_scene *s, uint32_t *nodes, uint32_t *leaf_order, uint64_t *keys, float *bounds,
                                   size_t capacity, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s)
            throw Invalid{"null scene"};
        const u32 n = s->n;
        if (capacity < n)
            throw Invalid{"capacity too small"};
        RP_CHECK(cudaSetDevice(s->device));
        if (n == 0)
            return RP_SUCCESS;
        RP_CHECK(cudaMemcpy(leaf_order, s->order, size_t(n) * 4, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(keys, s->keys, size_t(n) * 8, cudaMemcpyDeviceToHost));
        std::vector<u32> l(n), r(n), p(n);
        std::vector<float4> lo(n), hi(n), blo(n), bhi(n);
        RP_CHECK(cudaMemcpy(l.data(), s->tmp.left, size_t(n) * 4, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(r.data(), s->tmp.right, size_t(n) * 4, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(p.data(), s->tmp.parent, size_t(n) * 4, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(lo.data(), s->tmp.node_lo, size_t(n) * 16, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(hi.data(), s->tmp.node_hi, size_t(n) * 16, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(blo.data(), s->tmp.box_lo, size_t(n) * 16, cudaMemcpyDeviceToHost));
        RP_CHECK(cudaMemcpy(bhi.data(), s->tmp.box_hi, size_t(n) * 16, cudaMemcpyDeviceToHost));
        for (u32 i = 0; i + 1 < n; ++i) {
            nodes[3 * i] = l[i];
            nodes[3 * i + 1] = r[i];
            nodes[3 * i + 2] = p[i];
            const float b[6] = {lo[i].x, lo[i].y, lo[i].z, hi[i].x, hi[i].y, hi[i].z};
            memcpy(bounds + 6 * i, b, sizeof(b));
        }
        for (u32 j = 0; j < n; ++j) {
            const u32 prim = leaf_order[j];
            const float b[6] = {blo[prim].x, blo[prim].y, blo[prim].z, bhi[prim].x, bhi[prim].y, bhi[prim].z};
            memcpy(bounds + 6 * (size_t(n) - 1 + j), b, sizeof(b));
        }
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_trace_rays(rp_scene *s, const float *rays, uint32_t count, int any_hit, float *hits, char *diag,
                             size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s)
            throw Invalid{"null scene"};
        RP_CHECK(cudaSetDevice(s->device));
        std::vector<void *> own;
        struct Free {
            std::vector<void *> &o;
            ~Free() {
                for (void *q : o)
                    cudaFreeAsync(q, nullptr);
                cudaStreamSynchronize(nullptr);
            }
        } fr{own};
        const float *q = dupload(own, rays, size_t(7) * count, s->stream);
        float *h = dalloc<float>(own, size_t(4) * count);
        k_probe_trace<<<(count + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, s->stream>>>(s->ds, q, count, any_hit, h);
        RP_CHECK(cudaGetLastError());
        RP_CHECK(cudaMemcpyAsync(hits, h, size_t(4) * count * 4, cudaMemcpyDeviceToHost, s->stream));
        RP_CHECK(cudaStreamSynchronize(s->stream));
        return RP_SUCCESS;
    });
}

} // extern "C"

// ---------------------------------------------------------------- frame sessions
// FrameSession (src/frame_session.hpp:182-212), independent estimator: one absolute sample of
// every pixel per frame, raw XYZ on the device, two frame slots, asynchronous on the scene's
// stream.  A frame is one wave of the scene's wavefront (hero or scalar transport) followed by
// the frame-sensor kernel; its camera, when the request names one, is the scene camera for
// that wave.
struct rp_frame_session {
    rp_scene *scene = nullptr;
    rp_frame_config config{};
    bool camera_set = false;
    rp_camera camera{};
    struct Slot {
        float *xyz = nullptr;   // 3 floats per pixel (device)
        u32 *failures = nullptr; // device counter
        u32 *host_failures = nullptr; // pinned copy, valid once `done` has completed
        cudaEvent_t start = nullptr, done = nullptr;
        bool held = false;
        uint64_t sample_index = 0, epoch = 0;
    } slot[2];
    ~rp_frame_session() {
        if (scene && scene->device >= 0)
            cudaSetDevice(scene->device);
        for (Slot &f : slot) {
            if (f.done)
                cudaEventSynchronize(f.done);
            if (f.xyz)
                cudaFree(f.xyz);
            if (f.failures)
                cudaFree(f.failures);
            if (f.host_failures)
                cudaFreeHost(f.host_failures);
            if (f.start)
                cudaEventDestroy(f.start);
            if (f.done)
                cudaEventDestroy(f.done);
        }
    }
};

namespace {

// The scene camera fields a frame's raygen reads (PBRT raster basis), swapped in for one wave.
void set_camera(DeviceScene &ds, const rp_camera &c) {
    ds.origin = v3(c.origin[0], c.origin[1], c.origin[2]);
    ds.forward = v3(c.corner[0], c.corner[1], c.corner[2]);
    ds.right = v3(c.dx[0], c.dx[1], c.dx[2]);
    ds.up = v3(c.dy[0], c.dy[1], c.dy[2]);
}

rp_frame_info frame_info(const rp_frame_session *fs, u32 k, bool complete) {
    const rp_frame_session::Slot &f = fs->slot[k];
    rp_frame_info info{};
    info.width = fs->config.width;
    info.height = fs->config.height;
    info.sample_index = f.sample_index;
    info.epoch = f.epoch;
    info.status = RP_FRAME_PENDING;
    if (complete) {
        info.failed_pixels = *f.host_failures;
        info.status = info.failed_pixels ? RP_FRAME_FAILED : RP_FRAME_COMPLETE;
        info.completed_samples = uint64_t(info.width) * info.height - info.failed_pixels;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, f.start, f.done) == cudaSuccess)
            info.gpu_ms = ms;
    }
    return info;
}

} // namespace

extern "C" {

rp_status rp_cuda_frame_session_create(rp_scene *s, const rp_frame_config *config, rp_frame_session **out, char *diag,
                                       size_t cap) {
    if (out)
        *out = nullptr;
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !config || !out)
            throw Invalid{"null argument"};
        if (s->ds.img.textured)
            throw NotBuilt{"frame sessions of scenes with image reflectance are not built (the texture camera follows the scene camera)"};
        if (s->ds.model == kModelDemo)
            throw NotBuilt{"frame sessions of demo-model scenes are not built (their sensor weights differ)"};
        rp_request q{};
        q.width = config->width;
        q.height = config->height;
        q.seed = config->seed;
        q.pixel_count = config->width * config->height;
        q.sample_count = 1;
        q.sampler_kind = config->sampler_kind;
        q.randomization = config->randomization;
        q.total_samples = config->footprint_samples ? config->footprint_samples : 1;
        const std::string err = validate_request(s, q);
        if (!err.empty())
            throw Invalid{err};
        if (q.pixel_count > (1u << 23))
            throw Invalid{"frame sessions render at most 2^23 pixels"};
        if (!s->cie)
            throw Invalid{"CIE table not set (rp_cuda_set_cie)"};
        RP_CHECK(cudaSetDevice(s->device));
        auto fs = std::make_unique<rp_frame_session>();
        fs->scene = s;
        fs->config = *config;
        for (auto &f : fs->slot) {
            RP_CHECK(cudaMalloc(reinterpret_cast<void **>(&f.xyz), size_t(q.pixel_count) * 3 * sizeof(float)));
            RP_CHECK(cudaMalloc(reinterpret_cast<void **>(&f.failures), sizeof(u32)));
            RP_CHECK(cudaMallocHost(reinterpret_cast<void **>(&f.host_failures), sizeof(u32)));
            RP_CHECK(cudaEventCreate(&f.start));
            RP_CHECK(cudaEventCreate(&f.done));
        }
        *out = fs.release();
        return RP_SUCCESS;
    });
}

void rp_cuda_frame_session_destroy(rp_frame_session *fs) { delete fs; }

rp_status rp_cuda_frame_submit(rp_frame_session *fs, const rp_frame_request *request, uint32_t *frame, int *busy,
                               char *diag, size_t cap) {
    if (busy)
        *busy = 0;
    return guarded(diag, cap, [&]() -> rp_status {
        if (!fs || !request || !frame)
            throw Invalid{"null argument"};
        u32 k = 0;
        while (k < 2 && fs->slot[k].held)
            ++k;
        if (k == 2) {
            if (busy)
                *busy = 1;
            set_diag(diag, cap, "both frame slots are held; release a frame first");
            return RP_FAILURE;
        }
        rp_scene *s = fs->scene;
        const rp_frame_config &c = fs->config;
        rp_request q{};
        q.width = c.width;
        q.height = c.height;
        q.seed = c.seed;
        q.pixel_count = c.width * c.height;
        q.sample_begin = request->sample_index;
        q.sample_count = 1;
        q.emergency_limit = 1024;
        q.sampler_kind = c.sampler_kind;
        q.randomization = c.randomization;
        q.boundary_limit = 4096;
        q.total_samples = c.footprint_samples ? c.footprint_samples : request->sample_index + 1;
        const std::string err = validate_request(s, q);
        if (!err.empty())
            throw Invalid{err};
        if (request->camera) {
            fs->camera = *request->camera;
            fs->camera_set = true;
        }
        RP_CHECK(cudaSetDevice(s->device));
        rp_frame_session::Slot &f = fs->slot[k];
        f.held = true;
        f.sample_index = request->sample_index;
        f.epoch = request->epoch;
        const DeviceScene scene_camera = s->ds;
        try {
            if (fs->camera_set)
                set_camera(s->ds, fs->camera);
            const WaveParams p = wave_params(q);
            RP_CHECK(cudaEventRecord(f.start, s->stream));
            RP_CHECK(cudaMemsetAsync(f.failures, 0, sizeof(u32), s->stream));
            const unsigned grid = grid_for(s->sm_count, p.lanes, 128, 16);
            if (s->transport == RP_TRANSPORT_SCALAR) {
                run_scalar_wave(s, p, q.boundary_limit);
                k_frame_scalar<<<grid, 128, 0, s->stream>>>(s->scalar_records, p.lanes, s->cie, f.xyz, f.failures);
            } else {
                run_wave(s, p);
                k_frame_packet<<<grid, 128, 0, s->stream>>>(s->pool, p.lanes, 0, p.sample_low, p.sample_high, s->cie,
                                                             f.xyz, f.failures);
            }
            RP_CHECK(cudaGetLastError());
            RP_CHECK(cudaMemcpyAsync(f.host_failures, f.failures, sizeof(u32), cudaMemcpyDeviceToHost, s->stream));
            RP_CHECK(cudaEventRecord(f.done, s->stream));
        } catch (...) {
            s->ds = scene_camera;
            f.held = false;
            s->discard_marks();
            throw;
        }
        s->ds = scene_camera;
        // a frame is asynchronous: its per-kernel timing events are not read back
        s->discard_marks();
        *frame = k;
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_frame_poll(rp_frame_session *fs, uint32_t frame, rp_frame_info *info) {
    if (!fs || !info || frame > 1 || !fs->slot[frame].held)
        return RP_INVALID_ARGUMENT;
    const cudaError_t q = cudaEventQuery(fs->slot[frame].done);
    if (q != cudaSuccess && q != cudaErrorNotReady)
        return RP_FAILURE;
    *info = frame_info(fs, frame, q == cudaSuccess);
    return RP_SUCCESS;
}

rp_status rp_cuda_frame_wait(rp_frame_session *fs, uint32_t frame, rp_frame_info *info) {
    if (!fs || !info || frame > 1 || !fs->slot[frame].held)
        return RP_INVALID_ARGUMENT;
    if (cudaEventSynchronize(fs->slot[frame].done) != cudaSuccess)
        return RP_FAILURE;
    *info = frame_info(fs, frame, true);
    return RP_SUCCESS;
}

rp_status rp_cuda_frame_capture(rp_frame_session *fs, uint32_t frame, float *host_xyz, size_t capacity, char *diag,
                                size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!fs || !host_xyz || frame > 1 || !fs->slot[frame].held)
            throw Invalid{"no such frame"};
        const size_t pixels = size_t(fs->config.width) * fs->config.height;
        if (capacity < pixels)
            throw Invalid{"capture capacity is smaller than the frame"};
        RP_CHECK(cudaSetDevice(fs->scene->device));
        RP_CHECK(cudaEventSynchronize(fs->slot[frame].done));
        RP_CHECK(cudaMemcpy(host_xyz, fs->slot[frame].xyz, pixels * 3 * sizeof(float), cudaMemcpyDeviceToHost));
        const u32 failed = *fs->slot[frame].host_failures;
        if (failed) {
            set_diag(diag, cap, "frame failed: %u pixel samples failed", failed);
            return RP_FAILURE;
        }
        return RP_SUCCESS;
    });
}

rp_status rp_cuda_frame_device_xyz(rp_frame_session *fs, uint32_t frame, const float **device_xyz) {
    if (!fs || !device_xyz || frame > 1 || !fs->slot[frame].held)
        return RP_INVALID_ARGUMENT;
    *device_xyz = fs->slot[frame].xyz;
    return RP_SUCCESS;
}

rp_status rp_cuda_frame_release(rp_frame_session *fs, uint32_t frame) {
    if (!fs || frame > 1 || !fs->slot[frame].held)
        return RP_INVALID_ARGUMENT;
    cudaSetDevice(fs->scene->device);
    const cudaError_t e = cudaEventSynchronize(fs->slot[frame].done);
    fs->slot[frame].held = false;
    return e == cudaSuccess ? RP_SUCCESS : RP_FAILURE;
}

} // extern "C"

// ---------------------------------------------------------------- allocation-free sampling
// The scratch of rp_cuda_sample_device_static: one file-scope device array, shared by every
// call on a device (see include/rypath_cuda.h).  Host code must not use its name as an
// address: the device address is looked up with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_static_scratch[RP_STATIC_SCRATCH_BYTES];

namespace {

static_assert(pool_bytes(RP_STATIC_MAX_LANES, false) <= RP_STATIC_SCRATCH_BYTES &&
                  pool_bytes(RP_STATIC_MAX_LANES + 1, false) > RP_STATIC_SCRATCH_BYTES,
              "RP_STATIC_MAX_LANES is the largest request that fits the static scratch");

// Device address of the scratch array in the current device's context.  The caller keeps it
// with the scene, whose own device memory lives in the same context: a scene cannot outlive
// a reset of its device, so neither can the cached address.
unsigned char *static_scratch(cudaError_t &err) {
    void *ptr = nullptr;
    err = cudaGetSymbolAddress(&ptr, g_static_scratch);
    return err == cudaSuccess ? static_cast<unsigned char *>(ptr) : nullptr;
}

// The pool of the allocation-free entry point: the scene pool's carve without the optional
// arrays (the entry point refuses scenes with pass-through or mix surfaces and never counts).
PathPool static_pool(unsigned char *base, u32 lanes, unsigned long long *stats) {
    PathPool q;
    carve_pool(base, lanes, false, &q);
    q.stats = stats;
    return q;
}

__global__ void k_static_set_lanes(u32 *counter, u32 lanes) { *counter = lanes; }

} // namespace

extern "C" {

rp_status rp_cuda_sample_device_static(rp_scene *s, const rp_request *request, rp_packet_result *device_results,
                                       size_t capacity, void *stream, char *diag, size_t cap) {
    return guarded(diag, cap, [&]() -> rp_status {
        if (!s || !request || !device_results)
            throw Invalid{"null argument"};
        const std::string err = validate_request(s, *request);
        if (!err.empty())
            throw Invalid{err};
        if (s->transport != RP_TRANSPORT_HERO)
            throw Invalid{"the allocation-free entry point samples hero-transport scenes"};
        apply_texture_request(s, *request);
        const WaveParams p = wave_params(*request);
        if (capacity < p.lanes)
            throw Invalid{"output capacity is smaller than the request lanes"};
        if (s->resolve)
            throw Invalid{"the allocation-free entry point renders scenes without pass-through, mix or procedural surfaces"};
        const u32 max_lanes = RP_STATIC_MAX_LANES;
        if (p.lanes > max_lanes) {
            set_diag(diag, cap,
                     "request has %u lanes; the allocation-free entry point accepts at most %u lanes "
                     "(%u bytes of static scratch)",
                     p.lanes, max_lanes, RP_STATIC_SCRATCH_BYTES);
            return RP_INVALID_ARGUMENT;
        }
        RP_CHECK(cudaSetDevice(s->device));
        if (!s->static_base) {
            // the scene's first call: look the array up once, with the scene's device current
            cudaError_t e;
            s->static_base = static_scratch(e);
            if (!s->static_base) {
                set_diag(diag, cap, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
                return RP_FAILURE;
            }
        }
        unsigned char *base = s->static_base;
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
        PathPool pool = static_pool(base, p.lanes, s->stats);
        const int sms = s->sm_count;
        // counters start at zero on every call; every other array is written before it is read
        RP_CHECK(cudaMemsetAsync(pool.counters, 0, 256, st));
        k_raygen<<<grid_for(sms, p.lanes, 256, 16), 256, 0, st>>>(s->ds, p, pool);
        k_static_set_lanes<<<1, 1, 0, st>>>(pool.counters, p.lanes);
        int in = 0;
        for (u32 ev = 0; ev < s->ds.max_depth + 1; ++ev) {
            RP_CHECK(cudaMemsetAsync(pool.counters + 4, 0, 4 * sizeof(u32), st));
            launch_trace<false, kTraceBlock>(s, pool, in, grid_for(sms, p.lanes, kTraceBlock, 12), st, p.boundary_limit);
            RP_CHECK(cudaMemsetAsync(pool.counters + (in ^ 1), 0, sizeof(u32), st));
            RP_CHECK(cudaMemsetAsync(pool.counters + 2, 0, sizeof(u32), st));
            RP_CHECK(cudaMemsetAsync(pool.counters + 8, 0, 3 * sizeof(u32), st));
            const unsigned shade_grid = grid_for(sms, p.lanes, 128, 16);
            k_shade<0><<<shade_grid, 128, 0, st>>>(s->ds, p, pool, in);
            k_nee<0><<<shade_grid, 128, 0, st>>>(s->ds, p, pool);
            k_shade<1><<<shade_grid, 128, 0, st>>>(s->ds, p, pool, in);
            k_nee<1><<<shade_grid, 128, 0, st>>>(s->ds, p, pool);
            k_shade<2><<<shade_grid, 128, 0, st>>>(s->ds, p, pool, in);
            k_nee<2><<<shade_grid, 128, 0, st>>>(s->ds, p, pool);
            k_shade<3><<<shade_grid, 128, 0, st>>>(s->ds, p, pool, in);
            launch_shadow<false, kTraceBlock, false>(s, pool, grid_for(sms, p.lanes, kTraceBlock, 12), 0, st, p.boundary_limit);
            in ^= 1;
        }
        k_results<<<grid_for(sms, p.lanes, 256, 16), 256, 0, st>>>(pool, p.lanes, s->ds.filter_weight,
                                                                   reinterpret_cast<PacketResult *>(device_results));
        RP_CHECK(cudaGetLastError());
        return RP_SUCCESS;
    });
}

} // extern "C"
