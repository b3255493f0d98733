// ORACLE -- test infrastructure only (see oracle_math.hpp).
#include "oracle_scene.hpp"

#include <numbers>

namespace oracle {

// ================================================================= light tables
// src/packet_spectrum_shared.h:33-59
Wavelengths packet_sample_visible(float u) {
    Wavelengths w{};
    if (!(u >= 0 && u < 1)) {
        for (int i = 0; i < 4; ++i)
            w.lambda[i] = w.pdf[i] = NAN;
        return w;
    }
    for (int i = 0; i < 4; ++i) {
        float up = u + float(i) * .25f;
        if (up > 1)
            up -= 1;
        w.lambda[i] = 538 - 138.888889f * std::atanh(.85691062f - 1.82750197f * up);
        if (w.lambda[i] < 360)
            w.lambda[i] = 360;
        if (w.lambda[i] > 830)
            w.lambda[i] = 830;
        w.pdf[i] = visible_pdf(w.lambda[i]);
    }
    return w;
}

// src/light_sampling.cpp:17-27
double light_spectrum_power(const float *spectrum) {
    const auto lambda = packet_sample_visible(.5f);
    double value = 0;
    for (int i = 0; i < 4; ++i)
        value += double(spectrum[unsigned(std::round(lambda.lambda[i]) - 360)]) / lambda.pdf[i] / 4;
    if (value == 0)
        for (int i = 0; i < 471; ++i)
            value += spectrum[i];
    return value;
}

namespace {
using V = std::array<double, 3>;
double vdot(V a, V b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double vnorm(V a) { return std::sqrt(vdot(a, a)); }
V vec(const float *a) { return {a[0], a[1], a[2]}; }

// src/light_sampling.cpp:226-276 (PBRT LightBounds union with a normal cone)
LightInput unite(const LightInput &a, const LightInput &b) {
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
    const V wa = vec(a.direction), wb = vec(b.direction);
    const double angle = std::acos(std::clamp(vdot(wa, wb), -1., 1.));
    if (std::min(angle + tb, pi) <= ta)
        return r;
    if (std::min(angle + ta, pi) <= tb) {
        for (int i = 0; i < 3; ++i)
            r.direction[i] = b.direction[i];
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
    V tangent;
    for (int i = 0; i < 3; ++i)
        tangent[i] = wb[i] - vdot(wa, wb) * wa[i];
    double length = vnorm(tangent);
    if (length < 1e-12) {
        const int axis = std::abs(wa[0]) < .8 ? 0 : 1;
        V basis{0, 0, 0};
        basis[axis] = 1;
        for (int i = 0; i < 3; ++i)
            tangent[i] = basis[i] - wa[axis] * wa[i];
        length = vnorm(tangent);
    }
    const double rotate = theta - ta;
    for (int i = 0; i < 3; ++i)
        r.direction[i] = float(std::cos(rotate) * wa[i] + std::sin(rotate) * tangent[i] / length);
    const double dl = vnorm(vec(r.direction));
    for (int i = 0; i < 3; ++i)
        r.direction[i] = float(r.direction[i] / dl);
    r.cos_outer = std::nextafter(float(std::cos(theta)), -INFINITY);
    return r;
}
// src/light_sampling.cpp:277-292 (PBRT EvaluateCost)
double cost(const LightInput &b, const LightInput &all, int axis) {
    if (b.power == 0)
        return 0;
    const double pi = std::numbers::pi;
    const double o = std::acos(std::clamp(double(b.cos_outer), -1., 1.));
    const double e = std::acos(std::clamp(double(b.cos_emission), -1., 1.));
    const double w = std::min(o + e, pi);
    const double omega = 2 * pi * (1 - b.cos_outer) +
                         pi / 2 * (2 * w * std::sin(o) - std::cos(o - 2 * w) - 2 * o * std::sin(o) +
                                   b.cos_outer);
    const V d{double(b.high[0]) - b.low[0], double(b.high[1]) - b.low[1], double(b.high[2]) - b.low[2]};
    const V ad{double(all.high[0]) - all.low[0], double(all.high[1]) - all.low[1],
               double(all.high[2]) - all.low[2]};
    if (ad[axis] <= 0)
        return INFINITY;
    return b.power * omega * (std::max({ad[0], ad[1], ad[2]}) / ad[axis]) * 2 *
           (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
}
} // namespace

// src/light_sampling.cpp:384-572 (build_light_sampling)
bool build_light_tables(const std::vector<LightInput> &in, LightTables &out, std::string &error) {
    out = {};
    out.records.assign(in.size(), {RP_NONE, 0, 0, 0});
    out.alias.assign(in.size(), {0, 0, 0, 0});
    if (in.empty())
        return true;
    double total = 0, bounds_total = 0;
    std::vector<double> probabilities(in.size());
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
        probabilities[i] = v.power == 0 && b.power > 0 ? b.power : v.power;
        total += probabilities[i];
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
    std::vector<u32> small, large;
    for (size_t i = 0; i < in.size(); ++i) {
        const double p = total > 0 ? probabilities[i] / total : 1. / double(in.size());
        out.alias[i].pmf = float(p);
        probabilities[i] = p * double(in.size());
        (probabilities[i] < 1 ? small : large).push_back(u32(i));
    }
    while (!small.empty() && !large.empty()) {
        const u32 s = small.back();
        small.pop_back();
        const u32 l = large.back();
        large.pop_back();
        out.alias[s].threshold = float(probabilities[s]);
        out.alias[s].alias = l;
        probabilities[l] -= 1 - probabilities[s];
        (probabilities[l] < 1 ? small : large).push_back(l);
    }
    for (u32 i : small) {
        out.alias[i].threshold = 1;
        out.alias[i].alias = i;
    }
    for (u32 i : large) {
        out.alias[i].threshold = 1;
        out.alias[i].alias = i;
    }
    std::function<u32(size_t, size_t, u32, unsigned)> build = [&](size_t begin, size_t end, u32 parent,
                                                                 unsigned depth) -> u32 {
        const u32 index = u32(out.nodes.size());
        out.nodes.emplace_back();
        LightInput bounds;
        double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (size_t k = begin; k < end; ++k) {
            const auto &v = bvh[finite[k]];
            bounds = unite(bounds, v);
            for (int a = 0; a < 3; ++a) {
                const double c = (double(v.low[a]) + v.high[a]) / 2;
                clo[a] = std::min(clo[a], c);
                chi[a] = std::max(chi[a], c);
            }
        }
        LightBounds node{};
        node.parent = parent;
        node.light = RP_NONE;
        for (int a = 0; a < 3; ++a) {
            node.low[a] = bounds.low[a];
            node.high[a] = bounds.high[a];
            node.direction[a] = bounds.direction[a];
        }
        node.power = float(bounds.power / bounds_total);
        node.cos_outer = bounds.cos_outer;
        node.cos_emission = bounds.cos_emission;
        node.flags = bounds.two_sided ? 1 : 0;
        if (end - begin == 1) {
            const u32 id = finite[begin];
            node.light = id;
            out.records[id].leaf = index;
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
                        const unsigned b = std::min(
                            11u, unsigned(12 * ((double(v.low[axis]) + v.high[axis]) / 2 - clo[axis]) /
                                          (chi[axis] - clo[axis])));
                        buckets[b] = unite(buckets[b], v);
                    }
                    for (unsigned split = 1; split < 11; ++split) {
                        LightInput l, r;
                        for (unsigned k = 0; k <= split; ++k)
                            l = unite(l, buckets[k]);
                        for (unsigned k = split + 1; k < 12; ++k)
                            r = unite(r, buckets[k]);
                        const double c = cost(l, bounds, axis) + cost(r, bounds, axis);
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
                auto it = std::stable_partition(
                    finite.begin() + std::ptrdiff_t(begin), finite.begin() + std::ptrdiff_t(end),
                    [&](u32 id) {
                        const auto &v = bvh[id];
                        const unsigned b = std::min(
                            11u, unsigned(12 *
                                          ((double(v.low[split_axis]) + v.high[split_axis]) / 2 -
                                           clo[split_axis]) /
                                          (chi[split_axis] - clo[split_axis])));
                        return b <= split_bucket;
                    });
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
        build(0, finite.size(), RP_NONE, 0);
    return true;
}

// ================================================================= scene loading
static F3 world_point(const Instance &in, F3 p) {
    // shaders/light_geometry_sampling.h:10-15
    return F3{dot(F3{in.m[0], in.m[1], in.m[2]}, p), dot(F3{in.m[4], in.m[5], in.m[6]}, p),
              dot(F3{in.m[8], in.m[9], in.m[10]}, p)} +
           F3{in.m[3], in.m[7], in.m[11]};
}

// The world-to-object map of a row-major object-to-world 3x4 matrix, in double and rounded
// once (as the backend's host code computes it).
static bool invert_affine(const float *m, float *out) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = f * g - d * i, Cc = d * h - e * g;
    const double det = a * A + b * B + c * Cc;
    if (!(std::abs(det) > 0) || !std::isfinite(det))
        return false;
    const double inv[9] = {A / det,  (c * h - b * i) / det, (b * f - c * e) / det,
                           B / det,  (a * i - c * g) / det, (c * d - a * f) / det,
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

// The world box of procedural primitive `prim` as the device builder forms it: the patch's
// corners or the corners of the shape's object box, in world space, widened by 2^-18 of their
// magnitude and extent.
void procedural_box(const Scene &s, u32 prim, F3 &lo, F3 &hi) {
    const Instance &in = s.instances[s.tri_instance[prim]];
    const u32 local = s.tri_local[prim];
    lo = F3{INFINITY, INFINITY, INFINITY};
    hi = -lo;
    auto grow = [&](F3 w) {
        lo = F3{std::fmin(lo.x, w.x), std::fmin(lo.y, w.y), std::fmin(lo.z, w.z)};
        hi = F3{std::fmax(hi.x, w.x), std::fmax(hi.y, w.y), std::fmax(hi.z, w.z)};
    };
    if (prim - s.tri_prims < s.patch_prims) {
        for (int k = 0; k < 4; ++k)
            grow(world_point(in, s.positions[in.vertex_begin + s.patches[in.patch_begin + local][k]]));
    } else {
        const Analytic &a = s.analytics[in.analytic_begin + local];
        const float r = a.radius;
        const float ol[3] = {-r, -r, a.subtype == 2u ? a.height : (a.subtype == 1u ? std::fmax(a.z_min, -r) : a.z_min)};
        const float oh[3] = {r, r, a.subtype == 2u ? a.height : (a.subtype == 1u ? std::fmin(a.z_max, r) : a.z_max)};
        for (int k = 0; k < 8; ++k)
            grow(world_point(in, F3{k & 1 ? oh[0] : ol[0], k & 2 ? oh[1] : ol[1], k & 4 ? oh[2] : ol[2]}));
    }
    const F3 m{std::fmax(std::fabs(lo.x), std::fabs(hi.x)), std::fmax(std::fabs(lo.y), std::fabs(hi.y)),
               std::fmax(std::fabs(lo.z), std::fabs(hi.z))};
    const F3 pad = 0x1p-18f * (m + (hi - lo)) + F3{1e-30f, 1e-30f, 1e-30f};
    lo = lo - pad;
    hi = hi + pad;
}

bool load_scene(const rp_scene_desc &d, Scene &s, std::string &error) {
    s = Scene{};
    s.positions.resize(d.vertex_count);
    for (u32 i = 0; i < d.vertex_count; ++i)
        s.positions[i] = F3{d.positions[3 * i], d.positions[3 * i + 1], d.positions[3 * i + 2]};
    s.normals.resize(d.normal_count);
    for (u32 i = 0; i < d.normal_count; ++i)
        s.normals[i] = F3{d.normals[3 * i], d.normals[3 * i + 1], d.normals[3 * i + 2]};
    s.triangles.resize(d.triangle_count);
    for (u32 i = 0; i < d.triangle_count; ++i)
        s.triangles[i] = {d.triangles[3 * i], d.triangles[3 * i + 1], d.triangles[3 * i + 2]};
    for (u32 i = 0; i < d.material_count; ++i) {
        const auto &m = d.materials[i];
        s.materials.push_back({m.scattering, m.kind, m.knot_begin, m.knot_count, m.scalar_value,
                               m.eta_begin, m.eta_count, m.k_begin, m.k_count, m.optical_extensions,
                               m.u_roughness, m.v_roughness, m.remap_roughness, m.first_material,
                               m.second_material, m.mix_amount, m.image_texture,
                               {m.coefficients[0], m.coefficients[1], m.coefficients[2]},
                               {m.reflectance[0], m.reflectance[1], m.reflectance[2], m.reflectance[3],
                                m.reflectance[4], m.reflectance[5], m.reflectance[6], m.reflectance[7]}});
        if (m.scattering == RP_DIFFUSE && m.kind == RP_REFLECTANCE_IMAGE)
            s.textured = true;
    }
    for (u32 i = 0; i < d.knot_count; ++i)
        s.knots.push_back({d.knots[i].wavelength, d.knots[i].value});
    for (u32 i = 0; i < d.emission_count; ++i) {
        std::array<float, 471> e;
        std::copy(d.emissions[i].radiance, d.emissions[i].radiance + 471, e.begin());
        s.emission.push_back(e);
        s.emission_two_sided.push_back(d.emissions[i].two_sided);
    }
    for (u32 i = 0; i < d.positional_count; ++i) {
        Positional p{};
        const auto &q = d.positional[i];
        p.position = F3{q.position[0], q.position[1], q.position[2]};
        std::copy(q.intensity, q.intensity + 471, p.intensity);
        p.kind = q.kind;
        std::copy(q.light_from_world, q.light_from_world + 9, p.light_from_world);
        p.cos_falloff_start = q.cos_falloff_start;
        p.cos_falloff_end = q.cos_falloff_end;
        s.positional.push_back(p);
    }
    if (d.environment) {
        std::copy(d.environment, d.environment + 471, s.environment.begin());
        s.has_environment = std::any_of(s.environment.begin(), s.environment.end(),
                                        [](float v) { return v > 0; });
    }
    s.model = d.model;
    s.film_scale = d.film_scale;
    if (const std::string images = load_images(d.images, d.instance_count, s.images); !images.empty()) {
        error = images;
        return false;
    }
    // emitters in instance order (src/metal_render.mm:1174-1210)
    for (u32 i = 0; i < d.instance_count; ++i) {
        const auto &q = d.instances[i];
        Instance in{};
        std::copy(q.matrix, q.matrix + 12, in.m);
        in.vertex_begin = q.vertex_begin;
        in.triangle_begin = q.triangle_begin;
        in.triangle_count = q.triangle_count;
        in.material = q.material;
        in.reverse = q.reverse_orientation;
        in.emission = q.emission;
        in.normal_begin = q.normal_begin;
        in.emitter_begin = RP_NONE;
        in.inside_medium = q.inside_medium;
        in.outside_medium = q.outside_medium;
        in.invisible = q.invisible_emitter;
        in.patch_begin = q.patch_count ? q.patch_begin : 0;
        in.patch_count = q.patch_count;
        in.analytic_begin = q.analytic_count ? q.analytic_begin : 0;
        in.analytic_count = q.analytic_count;
        if ((q.patch_count && uint64_t(q.patch_begin) + q.patch_count > d.patch_count) ||
            (q.analytic_count && uint64_t(q.analytic_begin) + q.analytic_count > d.analytic_count)) {
            error = "instance patches or analytic shapes out of range";
            return false;
        }
        if ((q.patch_count || q.analytic_count) && !invert_affine(q.matrix, in.inverse)) {
            error = "an instance with patches or analytic shapes needs an invertible transform";
            return false;
        }
        if (q.emission != RP_NONE) {
            in.emitter_begin = u32(s.emitters.size());
            for (u32 t = 0; t < q.triangle_count; ++t)
                s.emitters.push_back({i, t});
        }
        s.instances.push_back(in);
        for (u32 t = 0; t < q.triangle_count; ++t) {
            const auto &tri = s.triangles[q.triangle_begin + t];
            std::array<F3, 3> w;
            for (int k = 0; k < 3; ++k)
                w[k] = world_point(in, s.positions[q.vertex_begin + tri[k]]);
            s.world.push_back(w);
            s.tri_instance.push_back(i);
            s.tri_local.push_back(t);
        }
    }
    // procedural primitives after the triangles: every instance's patches, then every
    // instance's analytic shapes
    s.tri_prims = u32(s.world.size());
    for (u32 i = 0; i < d.patch_count; ++i)
        s.patches.push_back({d.patches[4 * i], d.patches[4 * i + 1], d.patches[4 * i + 2], d.patches[4 * i + 3]});
    for (u32 i = 0; i < d.analytic_count; ++i) {
        const rp_analytic &a = d.analytics[i];
        // validate_analytic (src/analytic.hpp:14-50), the checks the backend makes
        bool ok = a.subtype >= 1 && a.subtype <= 3 && std::isfinite(a.radius) && std::isfinite(a.z_min) &&
                  std::isfinite(a.z_max) && std::isfinite(a.phi_max) && std::isfinite(a.inner_radius) &&
                  std::isfinite(a.height) && a.radius > 0 && std::isnormal(a.radius) && std::isnormal(a.phi_max) &&
                  a.phi_max > 0 && a.phi_max <= 2 * float(M_PI);
        if (ok && a.subtype == 2)
            ok = a.inner_radius >= 0 && a.inner_radius < a.radius && a.radius - a.inner_radius >= 0x1p-16f;
        else if (ok)
            ok = a.z_min < a.z_max && std::isnormal(a.z_max - a.z_min) && a.z_max - a.z_min >= 0x1p-16f &&
                 a.z_max - a.z_min <= 0x1p16f &&
                 (a.subtype != 1 || (a.z_min >= -a.radius && a.z_max <= a.radius &&
                                     std::acos(a.z_min / a.radius) > std::acos(a.z_max / a.radius)));
        ok = ok && a.radius >= 0x1p-16f && a.radius <= 0x1p16f && a.phi_max >= 0x1p-16f && std::fabs(a.z_min) <= 0x1p16f &&
             std::fabs(a.z_max) <= 0x1p16f && std::fabs(a.height) <= 0x1p16f;
        if (!ok) {
            error = "invalid analytic shape";
            return false;
        }
        s.analytics.push_back({a.kind, a.subtype, a.radius, a.z_min, a.z_max, a.phi_max, a.inner_radius, a.height});
    }
    for (u32 i = 0; i < d.instance_count; ++i)
        for (u32 k = 0; k < d.instances[i].patch_count; ++k) {
            for (u32 c = 0; c < 4; ++c)
                if (uint64_t(d.instances[i].vertex_begin) + s.patches[d.instances[i].patch_begin + k][c] >= d.vertex_count) {
                    error = "patch vertex out of range";
                    return false;
                }
            s.tri_instance.push_back(i);
            s.tri_local.push_back(k);
            ++s.patch_prims;
        }
    for (u32 i = 0; i < d.instance_count; ++i)
        for (u32 k = 0; k < d.instances[i].analytic_count; ++k) {
            s.tri_instance.push_back(i);
            s.tri_local.push_back(k);
        }
    s.procedural_prims = u32(s.tri_instance.size()) - s.tri_prims;
    // camera (src/metal_render.mm:158-191)
    s.origin = F3{d.camera.origin[0], d.camera.origin[1], d.camera.origin[2]};
    s.forward = F3{d.camera.corner[0], d.camera.corner[1], d.camera.corner[2]};
    s.right = F3{d.camera.dx[0], d.camera.dx[1], d.camera.dx[2]};
    s.up = F3{d.camera.dy[0], d.camera.dy[1], d.camera.dy[2]};
    s.filter_kind = d.filter_kind;
    s.filter_x = d.filter_x_radius;
    s.filter_y = d.filter_y_radius;
    if (d.filter_kind == RP_FILTER_GAUSSIAN) {
        float integral = 0;
        error = gaussian_filter_table(d.filter_x_radius, d.filter_y_radius, d.filter_sigma, s.gauss_cdf, s.gauss_w,
                                      s.gauss_h, integral);
        if (!error.empty())
            return false;
        s.filter_weight = d.transport == RP_TRANSPORT_HERO ? integral : 1.0f;
    }
    s.lens_radius = d.lens_radius;
    s.focal_distance = d.lens_radius > 0 ? d.focal_distance : 1e6f;
    s.lens_x = F3{d.lens_x[0], d.lens_x[1], d.lens_x[2]};
    s.lens_y = F3{d.lens_y[0], d.lens_y[1], d.lens_y[2]};
    s.max_depth = d.max_depth;
    s.light_sampler = d.light_sampler;
    s.hero_mode = d.hero_wavelengths;
    s.transport = d.transport;
    s.camera_medium = d.camera_medium;
    bool interfaces = false;
    for (const auto &m : s.materials)
        interfaces = interfaces || m.scattering == RP_INTERFACE;
    for (u32 i = 0; i < d.medium_count; ++i) {
        Medium m;
        std::copy(d.media[i].sigma_a, d.media[i].sigma_a + 471, m.sigma_a.begin());
        std::copy(d.media[i].sigma_s, d.media[i].sigma_s + 471, m.sigma_s.begin());
        std::copy(d.media[i].emission, d.media[i].emission + 471, m.emission.begin());
        m.g = d.media[i].g;
        s.media.push_back(m);
    }
    s.media_enabled = d.medium_count > 0 || interfaces || d.camera_medium != RP_NONE;
    s.sobol_storage.assign((const unsigned char *)d.sobol_tables,
                           (const unsigned char *)d.sobol_tables + sizeof(SobolTables));
    s.sobol = reinterpret_cast<const SobolTables *>(s.sobol_storage.data());
    // scene sphere (src/metal_render.mm:213-276)
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (const auto &w : s.world)
        for (const auto &p : w)
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], double(p[a]));
                hi[a] = std::max(hi[a], double(p[a]));
            }
    for (u32 k = 0; k < s.procedural_prims; ++k) {
        F3 blo, bhi;
        procedural_box(s, s.tri_prims + k, blo, bhi);
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], double(blo[a]));
            hi[a] = std::max(hi[a], double(bhi[a]));
        }
    }
    if (s.tri_instance.empty()) {
        s.scene_radius = 1;
    } else {
        double c[3], e[3];
        for (int a = 0; a < 3; ++a) {
            c[a] = float(lo[a] / 2 + hi[a] / 2);
            e[a] = std::max(std::abs(lo[a] - c[a]), std::abs(hi[a] - c[a]));
            e[a] += 32 * FLT_EPSILON * std::max(std::abs(lo[a]), std::abs(hi[a]));
        }
        s.scene_center = F3{float(c[0]), float(c[1]), float(c[2])};
        s.scene_radius = std::nextafter(float(std::hypot(e[0], e[1], e[2])), INFINITY);
    }
    // light inputs (src/metal_render.mm:525-660, :1565-1660)
    std::vector<LightInput> input;
    const double pi = std::numbers::pi;
    std::vector<double> means(s.emission.size(), -1), bound_means(s.emission.size(), -1);
    for (const auto &in : s.instances) {
        if (in.emission == RP_NONE)
            continue;
        double &mean = means[in.emission], &bound = bound_means[in.emission];
        if (mean < 0) {
            mean = light_spectrum_power(s.emission[in.emission].data());
            bound = *std::max_element(s.emission[in.emission].begin(), s.emission[in.emission].end());
        }
        const bool two_sided = s.emission_two_sided[in.emission] != 0;
        for (u32 t = 0; t < in.triangle_count; ++t) {
            const auto &tri = s.triangles[in.triangle_begin + t];
            V p[3];
            for (int k = 0; k < 3; ++k) {
                const F3 q = s.positions[in.vertex_begin + tri[k]];
                for (int a = 0; a < 3; ++a)
                    p[k][a] = double(in.m[4 * a]) * q.x + double(in.m[4 * a + 1]) * q.y +
                              double(in.m[4 * a + 2]) * q.z + double(in.m[4 * a + 3]);
            }
            const V e1{p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
            const V e2{p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
            V n{e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                e1[0] * e2[1] - e1[1] * e2[0]};
            if (in.reverse)
                for (auto &v : n)
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
            const double area = .5 * std::hypot(n[0], n[1], n[2]);
            li.power = pi * area * mean * 1 * (two_sided ? 2 : 1);
            li.bounds_power = pi * area * bound * 1;
            li.two_sided = two_sided;
            const double length = std::hypot(n[0], n[1], n[2]);
            if (length > 0) {
                for (int a = 0; a < 3; ++a)
                    li.direction[a] = float(n[a] / length);
                li.cos_outer = std::nextafter(1.f, 0.f);
                li.two_sided = two_sided;
            }
            input.push_back(li);
        }
    }
    for (const auto &l : s.positional) {
        LightInput li;
        for (int a = 0; a < 3; ++a)
            li.low[a] = li.high[a] = l.position[a];
        const double maxi = *std::max_element(l.intensity, l.intensity + 471);
        li.two_sided = false;
        li.bounds_power = 4 * pi * maxi;
        if (l.kind == RP_POINT_LIGHT) {
            li.power = 4 * pi * light_spectrum_power(l.intensity);
        } else {
            li.power = 2 * pi *
                       ((1 - l.cos_falloff_start) + (l.cos_falloff_start - l.cos_falloff_end) / 2) *
                       light_spectrum_power(l.intensity);
            float cos_emission = float(std::cos(std::acos(double(l.cos_falloff_end)) -
                                                std::acos(double(l.cos_falloff_start))));
            if (cos_emission == 1)
                cos_emission = l.cos_falloff_end != l.cos_falloff_start ? .999f
                                                                        : std::nextafter(1.f, 0.f);
            // src/light_sampling.cpp:314-337 (light_positional_cone)
            const float *m = l.light_from_world;
            const V a{m[0], m[1], m[2]}, b{m[3], m[4], m[5]}, c{m[6], m[7], m[8]};
            const double aa = vdot(a, a), bb = vdot(b, b), cc = vdot(c, c), tol = 0x1p-20 * aa;
            li.two_sided = false;
            li.cos_outer = -1;
            li.cos_emission = 0;
            if ((aa > 0 && std::isfinite(aa)) && !(std::abs(aa - bb) > tol) &&
                !(std::abs(aa - cc) > tol) && !(std::abs(vdot(a, b)) > tol) &&
                !(std::abs(vdot(a, c)) > tol) && !(std::abs(vdot(b, c)) > tol)) {
                const V axis{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                             a[0] * b[1] - a[1] * b[0]};
                const double det = vdot(axis, c);
                if (std::abs(det) > 0) {
                    const double length = vnorm(axis);
                    for (int k = 0; k < 3; ++k)
                        li.direction[k] = float(axis[k] / std::copysign(length, det));
                    li.cos_outer = float(std::cos(std::min(
                        pi, std::acos(std::clamp(double(l.cos_falloff_start), -1., 1.)) + 2e-6)));
                    li.cos_outer = std::max(-1.f, std::nextafter(li.cos_outer, -INFINITY));
                    li.cos_emission = cos_emission;
                }
            }
        }
        input.push_back(li);
    }
    s.environment_light = RP_NONE;
    const bool env_image = s.images.env_image != RP_NONE;
    if (s.has_environment || env_image) {
        // src/metal_render.mm:617-630: an environment image replaces the constant environment
        LightInput li;
        li.infinite = true;
        const double radius = std::max(double(s.scene_radius), 1e-8);
        li.power = 4 * pi * pi * radius * radius *
                   (env_image ? s.images.env_power * s.images.env_scale : light_spectrum_power(s.environment.data()));
        s.environment_light = u32(input.size());
        input.push_back(li);
    }
    if (!build_light_tables(input, s.lights, error))
        return false;
    s.light_count = u32(input.size());
    return true;
}

// ================================================================= binary LBVH
static inline u32 spread21(u32 v) {
    u64 x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return 0; // unused (see morton63)
}
static inline u64 spread(u64 x) {
    x &= 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
// 63-bit Morton code of a centroid quantised to 2^21 cells per axis.
static inline u64 morton63(F3 c, F3 lo, F3 ext) {
    u64 q[3];
    for (int a = 0; a < 3; ++a) {
        float t = ext[a] > 0 ? (c[a] - lo[a]) / ext[a] : 0.0f;
        float cell = t * 2097152.0f;
        cell = std::min(std::max(cell, 0.0f), 2097151.0f);
        q[a] = u64(cell);
    }
    return (spread(q[0]) << 2) | (spread(q[1]) << 1) | spread(q[2]);
}
static inline int clz64(u64 x) { return x ? std::countl_zero(x) : 64; }

void build_lbvh(const std::vector<std::array<F3, 3>> &tris, Bvh &b) {
    (void)spread21;
    const u32 n = u32(tris.size());
    b = Bvh{};
    b.n = n;
    if (n == 0)
        return;
    std::vector<Box> box(n);
    std::vector<F3> centroid(n);
    F3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    for (u32 i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            box[i].lo[a] = std::min(std::min(tris[i][0][a], tris[i][1][a]), tris[i][2][a]);
            box[i].hi[a] = std::max(std::max(tris[i][0][a], tris[i][1][a]), tris[i][2][a]);
            centroid[i][a] = 0.5f * box[i].lo[a] + 0.5f * box[i].hi[a];
            lo[a] = std::min(lo[a], centroid[i][a]);
            hi[a] = std::max(hi[a], centroid[i][a]);
        }
    }
    const F3 ext = hi - lo;
    // bit 63: a box side longer than 1/16 of the largest centroid extent (the device builder's
    // large-triangle split at the root, rypath_b200/csrc/rp_build.cuh k_morton)
    const float large = std::max(std::max(ext[0], ext[1]), ext[2]) * 0.0625f;
    std::vector<std::pair<u64, u32>> items(n);
    for (u32 i = 0; i < n; ++i) {
        const bool is_large = box[i].hi[0] - box[i].lo[0] > large || box[i].hi[1] - box[i].lo[1] > large ||
                              box[i].hi[2] - box[i].lo[2] > large;
        items[i] = {(is_large ? 1ull << 63 : 0ull) | morton63(centroid[i], lo, ext), i};
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const auto &x, const auto &y) { return x.first < y.first; });
    b.keys.resize(n);
    b.order.resize(n);
    for (u32 i = 0; i < n; ++i) {
        b.keys[i] = items[i].first;
        b.order[i] = items[i].second;
    }
    b.leaf_box.resize(n);
    for (u32 i = 0; i < n; ++i)
        b.leaf_box[i] = box[b.order[i]];
    b.leaf_parent.assign(n, RP_NONE);
    if (n == 1)
        return;
    const u32 m = n - 1;
    b.left.resize(m);
    b.right.resize(m);
    b.parent.assign(m, RP_NONE);
    b.node_box.resize(m);
    // Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees and k-d trees".
    auto delta = [&](long i, long j) -> int {
        if (j < 0 || j >= long(n))
            return -1;
        const u64 a = b.keys[i], c = b.keys[j];
        if (a != c)
            return clz64(a ^ c);
        return 64 + std::countl_zero(u32(i) ^ u32(j));
    };
    for (long i = 0; i < long(m); ++i) {
        const int d = (delta(i, i + 1) - delta(i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(i, i - d);
        long lmax = 2;
        while (delta(i, i + lmax * d) > dmin)
            lmax *= 2;
        long l = 0;
        for (long t = lmax / 2; t >= 1; t /= 2)
            if (delta(i, i + (l + t) * d) > dmin)
                l += t;
        const long j = i + l * d;
        const int dnode = delta(i, j);
        long s = 0;
        for (long div = 2;; div *= 2) {
            const long t = (l + div - 1) / div;
            if (delta(i, i + (s + t) * d) > dnode)
                s += t;
            if (t == 1)
                break;
        }
        const long gamma = i + s * d + std::min(d, 0);
        const long first = std::min(i, j), last = std::max(i, j);
        const u32 lc = first == gamma ? (0x80000000u | u32(gamma)) : u32(gamma);
        const u32 rc = last == gamma + 1 ? (0x80000000u | u32(gamma + 1)) : u32(gamma + 1);
        b.left[i] = lc;
        b.right[i] = rc;
        for (u32 c : {lc, rc}) {
            if (c & 0x80000000u)
                b.leaf_parent[c & 0x7fffffffu] = u32(i);
            else
                b.parent[c] = u32(i);
        }
    }
    // bottom-up refit (post-order; min/max is order independent)
    std::function<Box(u32)> fit = [&](u32 c) -> Box {
        if (c & 0x80000000u)
            return b.leaf_box[c & 0x7fffffffu];
        const Box l = fit(b.left[c]), r = fit(b.right[c]);
        Box u;
        for (int a = 0; a < 3; ++a) {
            u.lo[a] = std::min(l.lo[a], r.lo[a]);
            u.hi[a] = std::max(l.hi[a], r.hi[a]);
        }
        b.node_box[c] = u;
        return u;
    };
    // iterative to avoid deep recursion on degenerate inputs
    std::vector<u32> post;
    std::vector<std::pair<u32, bool>> st{{0, false}};
    while (!st.empty()) {
        auto [c, done] = st.back();
        st.pop_back();
        if (c & 0x80000000u)
            continue;
        if (done) {
            post.push_back(c);
            continue;
        }
        st.push_back({c, true});
        st.push_back({b.right[c], false});
        st.push_back({b.left[c], false});
    }
    for (u32 c : post) {
        const auto child = [&](u32 x) { return (x & 0x80000000u) ? b.leaf_box[x & 0x7fffffffu] : b.node_box[x]; };
        const Box l = child(b.left[c]), r = child(b.right[c]);
        Box u;
        for (int a = 0; a < 3; ++a) {
            u.lo[a] = std::min(l.lo[a], r.lo[a]);
            u.hi[a] = std::max(l.hi[a], r.hi[a]);
        }
        b.node_box[c] = u;
    }
    (void)fit;
}

// Watertight ray/triangle intersection (Woop, Benthin and Wald, JCGT 2(1), 2013).  The
// operation sequence is fixed (explicit fma) so the CUDA kernels round identically.
bool intersect_triangle(F3 o, F3 d, const std::array<F3, 3> &v, float tmax, float &t, float &b1,
                        float &b2) {
    const F3 ad = fabs3(d);
    int kz = ad.x > ad.y ? (ad.x > ad.z ? 0 : 2) : (ad.y > ad.z ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (d[kz] < 0)
        std::swap(kx, ky);
    const float sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0f / d[kz];
    const F3 A = v[0] - o, B = v[1] - o, C = v[2] - o;
    const float ax = std::fma(-sx, A[kz], A[kx]), ay = std::fma(-sy, A[kz], A[ky]);
    const float bx = std::fma(-sx, B[kz], B[kx]), by = std::fma(-sy, B[kz], B[ky]);
    const float cx = std::fma(-sx, C[kz], C[kx]), cy = std::fma(-sy, C[kz], C[ky]);
    float U = std::fma(cx, by, -(cy * bx));
    float Vv = std::fma(ax, cy, -(ay * cx));
    float W = std::fma(bx, ay, -(by * ax));
    if (U == 0 || Vv == 0 || W == 0) {
        U = float(double(cx) * double(by) - double(cy) * double(bx));
        Vv = float(double(ax) * double(cy) - double(ay) * double(cx));
        W = float(double(bx) * double(ay) - double(by) * double(ax));
    }
    if ((U < 0 || Vv < 0 || W < 0) && (U > 0 || Vv > 0 || W > 0))
        return false;
    const float det = U + Vv + W;
    if (det == 0)
        return false;
    const float az = sz * A[kz], bz = sz * B[kz], cz = sz * C[kz];
    const float T = std::fma(U, az, std::fma(Vv, bz, W * cz));
    if (det > 0 ? (T <= 0 || T >= tmax * det) : (T >= 0 || T <= tmax * det))
        return false;
    const float rcp = 1.0f / det;
    t = T * rcp;
    b1 = Vv * rcp;
    b2 = W * rcp;
    return t > 0 && t < tmax;
}

// Conservative slab test (Ize, "Robust BVH ray traversal", JCGT 2(2), 2013).
static inline bool slab(const Box &b, F3 o, F3 inv, float tmax, float &tenter) {
    float t0 = 0, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        float tn = (b.lo[a] - o[a]) * inv[a];
        float tf = (b.hi[a] - o[a]) * inv[a];
        if (tn > tf)
            std::swap(tn, tf);
        tf *= 1 + 2 * gamma_bound(3);
        t0 = tn > t0 ? tn : t0;
        t1 = tf < t1 ? tf : t1;
        if (!(t0 <= t1))
            return false;
    }
    tenter = t0;
    return true;
}

static inline bool better(float t, u32 prim, const Hit &h) {
    return t < h.t || (t == h.t && prim < h.prim);
}

static ShapeHit procedural_hit(const Scene &s, u32 prim, F3 o, F3 d, float tmax);
// The procedural primitives, tested one by one after the triangle tree (the device tree holds
// them with the triangles; the closest hit is the same).
static void procedural_closest(const Scene &s, F3 o, F3 d, float tmax, Hit &h) {
    for (u32 k = 0; k < s.procedural_prims; ++k) {
        const u32 prim = s.tri_prims + k;
        const ShapeHit ph = procedural_hit(s, prim, o, d, tmax);
        if (ph.hit && better(ph.t, prim, h))
            h = Hit{ph.t, ph.u, ph.v, prim};
    }
}

Hit trace_closest(const Scene &s, const Bvh &b, F3 o, F3 d, float tmax) {
    Hit h = trace_triangles(s, b, o, d, tmax);
    if (s.procedural_prims) {
        if (h.prim == RP_NONE)
            h.t = tmax;
        procedural_closest(s, o, d, tmax, h);
        if (h.prim == RP_NONE)
            return Hit{};
    }
    return h;
}

Hit trace_triangles(const Scene &s, const Bvh &b, F3 o, F3 d, float tmax) {
    Hit h;
    h.t = tmax;
    if (b.n == 0)
        return Hit{};
    const F3 inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    auto test_leaf = [&](u32 slot) {
        const u32 prim = b.order[slot];
        float t, b1, b2;
        if (intersect_triangle(o, d, s.world[prim], tmax, t, b1, b2) && better(t, prim, h))
            h = Hit{t, b1, b2, prim};
    };
    if (b.n == 1) {
        test_leaf(0);
    } else {
        u32 stack[128];
        int sp = 0;
        u32 node = 0;
        float te;
        if (!slab(b.node_box[0], o, inv, h.t, te))
            return h.prim == RP_NONE ? Hit{} : h;
        for (;;) {
            const u32 c[2] = {b.left[node], b.right[node]};
            float tc[2];
            bool hitc[2];
            for (int k = 0; k < 2; ++k) {
                const Box &bx = (c[k] & 0x80000000u) ? b.leaf_box[c[k] & 0x7fffffffu] : b.node_box[c[k]];
                hitc[k] = slab(bx, o, inv, h.t, tc[k]);
            }
            u32 next = RP_NONE;
            for (int k = 0; k < 2; ++k)
                if (hitc[k] && (c[k] & 0x80000000u)) {
                    test_leaf(c[k] & 0x7fffffffu);
                    hitc[k] = false;
                }
            if (hitc[0] && hitc[1]) {
                const int first = tc[1] < tc[0] ? 1 : 0;
                stack[sp++] = c[1 - first];
                next = c[first];
            } else if (hitc[0])
                next = c[0];
            else if (hitc[1])
                next = c[1];
            if (next == RP_NONE) {
                if (sp == 0)
                    break;
                next = stack[--sp];
            }
            node = next;
        }
    }
    if (h.prim == RP_NONE)
        return Hit{};
    return h;
}

bool trace_any(const Scene &s, const Bvh &b, F3 o, F3 d, float tmax) {
    for (u32 k = 0; k < s.procedural_prims; ++k)
        if (procedural_hit(s, s.tri_prims + k, o, d, tmax).hit)
            return true;
    if (b.n == 0)
        return false;
    const F3 inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t, b1, b2, te;
    if (b.n == 1)
        return intersect_triangle(o, d, s.world[b.order[0]], tmax, t, b1, b2);
    u32 stack[128];
    int sp = 0;
    if (!slab(b.node_box[0], o, inv, tmax, te))
        return false;
    stack[sp++] = 0;
    while (sp) {
        const u32 node = stack[--sp];
        for (u32 c : {b.left[node], b.right[node]}) {
            const Box &bx = (c & 0x80000000u) ? b.leaf_box[c & 0x7fffffffu] : b.node_box[c];
            if (!slab(bx, o, inv, tmax, te))
                continue;
            if (c & 0x80000000u) {
                if (intersect_triangle(o, d, s.world[b.order[c & 0x7fffffffu]], tmax, t, b1, b2))
                    return true;
            } else
                stack[sp++] = c;
        }
    }
    return false;
}

Hit trace_closest_brute(const Scene &s, F3 o, F3 d, float tmax) {
    Hit h;
    h.t = tmax;
    for (u32 p = 0; p < s.world.size(); ++p) {
        float t, b1, b2;
        if (intersect_triangle(o, d, s.world[p], tmax, t, b1, b2) && better(t, p, h))
            h = Hit{t, b1, b2, p};
    }
    procedural_closest(s, o, d, tmax, h);
    return h.prim == RP_NONE ? Hit{} : h;
}

// ================================================================= Gaussian pixel filter
// PBRT FastExp (as in src/gaussian_filter.cpp:19-35)
static float fast_exp(float x) {
    if (x < -100.f)
        return 0;
    const float xp = x * 1.442695041f;
    const float fxp = std::floor(xp);
    const float f = xp - fxp;
    const int i = int(fxp);
    const float polynomial = std::fma(f, std::fma(f, std::fma(f, 0.0781455737f, 0.226173572f), 0.695556856f), 1.f);
    u32 bits = fbits(polynomial);
    const int exponent = int((bits >> 23) & 255) - 127 + i;
    if (exponent < -126)
        return 0;
    bits = (bits & 0x807fffffu) | (u32(exponent + 127) << 23);
    return ffrom(bits);
}
// src/gaussian_filter.cpp:39-68 (normalised piecewise-constant CDF of n values over 2 radius)
static bool table_cdf(const float *values, size_t n, float radius, float *cdf, float &integral) {
    cdf[0] = 0;
    for (size_t i = 0; i < n; ++i) {
        cdf[i + 1] = cdf[i] + values[i] * (2 * radius) / float(n);
        if (!std::isfinite(cdf[i + 1]))
            return false;
    }
    integral = cdf[n];
    if (integral > 0 && !std::isnormal(integral))
        return false;
    for (size_t i = 1; i <= n; ++i)
        cdf[i] = integral == 0 ? float(i) / float(n) : cdf[i] / integral;
    for (size_t i = 1; i <= n; ++i) {
        const float gap = cdf[i] - cdf[i - 1];
        if (!std::isfinite(cdf[i]) || (cdf[i] > 0 && !std::isnormal(cdf[i])) || (gap > 0 && !std::isnormal(gap)))
            return false;
    }
    return true;
}
std::string gaussian_filter_table(float xr, float yr, float sigma, std::vector<float> &cdf, u32 &width, u32 &height,
                                  float &integral) {
    if (!std::isnormal(xr) || xr <= 0 || !std::isnormal(yr) || yr <= 0 || !std::isnormal(sigma) || sigma <= 0)
        return "Gaussian radii and sigma must be positive normal binary32 values";
    const float nx = 32 * xr, ny = 32 * yr;
    if (!(nx >= 1 && nx < 4097.f && ny >= 1 && ny < 4097.f))
        return "Gaussian table axis must contain 1 to 4096 cells";
    width = u32(nx);
    height = u32(ny);
    if (u64(width) * height > 1048576)
        return "Gaussian table exceeds the 1048576-cell limit";
    const float denominator = 2 * 3.14159265358979323846f * sigma * sigma;
    const float tss = 2 * sigma * sigma;
    const float scale = 1 / std::sqrt(denominator);
    if (!(denominator > 0 && std::isfinite(denominator) && tss > 0 && std::isfinite(tss) && std::isfinite(scale)))
        return "Gaussian sigma arithmetic overflows or collapses in binary32";
    const auto gaussian = [&](float x) { return scale * fast_exp(-(x * x) / tss); };
    const auto lerp = [](float t, float a, float b) { return (1 - t) * a + t * b; };
    const float ex = gaussian(xr), ey = gaussian(yr);
    cdf.assign(size_t(height) * (width + 1) + height + 1, 0.f);
    std::vector<float> values(width), rows(height);
    for (u32 y = 0; y < height; ++y) {
        const float py = lerp((float(y) + 0.5f) / float(height), -yr, yr);
        const float fy = std::max(0.f, gaussian(py) - ey);
        for (u32 x = 0; x < width; ++x) {
            const float px = lerp((float(x) + 0.5f) / float(width), -xr, xr);
            values[x] = std::max(0.f, gaussian(px) - ex) * fy;
            if (!std::isfinite(values[x]))
                return "Gaussian table contains nonfinite binary32 values";
        }
        if (!table_cdf(values.data(), width, xr, cdf.data() + size_t(y) * (width + 1), rows[y]))
            return "Gaussian conditional distribution overflows or collapses in binary32";
    }
    if (!table_cdf(rows.data(), height, yr, cdf.data() + size_t(height) * (width + 1), integral) || !(integral > 0))
        return "Gaussian table has a zero or nonfinite binary32 integral";
    return {};
}

// ================================================================= surface points
static float triangle_extent(F3 e1, F3 e2) {
    // shaders/render.metal:865-868
    const F3 a = fabs3(e1), b = fabs3(e2), c = fabs3(e2 - e1);
    const F3 m{std::max(a.x, std::max(b.x, c.x)), std::max(a.y, std::max(b.y, c.y)),
               std::max(a.z, std::max(b.z, c.z))};
    return max3(m);
}
// shaders/render.metal:885-968
bool triangle_surface_point(const Scene &s, u32 instance, u32 local, float u, float v,
                            bool native_hit, SurfacePoint &point) {
    const Instance &in = s.instances[instance];
    point.curved = false;
    const auto &tri = s.triangles[in.triangle_begin + local];
    const F3 p0 = s.positions[in.vertex_begin + tri[0]];
    const F3 p1 = s.positions[in.vertex_begin + tri[1]];
    const F3 p2 = s.positions[in.vertex_begin + tri[2]];
    const F3 ax{in.m[0], in.m[1], in.m[2]}, ay{in.m[4], in.m[5], in.m[6]}, az{in.m[8], in.m[9], in.m[10]};
    const F3 shift{in.m[3], in.m[7], in.m[11]};
    const F3 e1 = p1 - p0, e2 = p2 - p0;
    const F3 we1{dot(ax, e1), dot(ay, e1), dot(az, e1)};
    const F3 we2{dot(ax, e2), dot(ay, e2), dot(az, e2)};
    const F3 ce = cross(we1, we2);
    const float n2 = dot(ce, ce);
    if (n2 == 0.0f && !native_hit) {
        point = SurfacePoint{};
        return true;
    }
    if (!(n2 > 0.0f) || !std::isfinite(n2))
        return false;
    const float nl = std::sqrt(n2);
    point.inverse_area_pdf = 0.5f * nl;
    point.world_extent = triangle_extent(we1, we2);
    point.geometric_normal = ce / nl;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    if (in.normal_begin != RP_NONE) {
        const u32 begin = in.normal_begin, nc = u32(s.normals.size());
        if (begin >= nc || tri[0] >= nc - begin || tri[1] >= nc - begin || tri[2] >= nc - begin)
            return false;
        const F3 n0 = s.normals[begin + tri[0]], n1 = s.normals[begin + tri[1]],
                 n2v = s.normals[begin + tri[2]];
        const F3 interp = (1.0f - (u + v)) * n0 + u * n1 + v * n2v;
        if (!finite3(interp))
            return false;
        const float scale = max3(fabs3(interp));
        if (scale > 0.0f) {
            const F3 scaled = interp / scale;
            point.shading_normal = normalize3(scaled);
            if (dot(point.geometric_normal, scaled) < 0.0f)
                point.geometric_normal = -point.geometric_normal;
        }
    }
    const F3 lp = p0 + (u * e1 + v * e2);
    point.position = F3{dot(ax, lp), dot(ay, lp), dot(az, lp)} + shift;
    F3 local_error = gamma_bound(7.0f) * (fabs3(p0) + fabs3(u * e1) + fabs3(v * e2));
    if (native_hit) {
        constexpr float allowance = 64.0f * 0x1.0p-23f;
        const float traversal = gamma_bound(7.0f) * triangle_extent(e1, e2);
        local_error = (local_error + allowance * (fabs3(e1) + fabs3(e2))) + F3{traversal, traversal, traversal};
    }
    const F3 ein = local_error + gamma_bound(4.0f) * fabs3(lp);
    point.error = F3{dot(fabs3(ax), ein), dot(fabs3(ay), ein), dot(fabs3(az), ein)} +
                  gamma_bound(4.0f) * fabs3(shift);
    return finite3(point.position) && finite3(point.error) && finite3(point.geometric_normal) &&
           finite3(point.shading_normal);
}

// shaders/render.metal:970-1062 (patch_surface_point)
static bool patch_surface_point(const Scene &s, u32 instance, u32 local, float u, float v, SurfacePoint &point) {
    const Instance &in = s.instances[instance];
    point.curved = true;
    const auto &idx = s.patches[in.patch_begin + local];
    F3 p[4];
    for (int i = 0; i < 4; ++i)
        p[i] = s.positions[in.vertex_begin + idx[i]];
    const F3 ax{in.m[0], in.m[1], in.m[2]}, ay{in.m[4], in.m[5], in.m[6]}, az{in.m[8], in.m[9], in.m[10]};
    const F3 e10 = p[1] - p[0], e32 = p[3] - p[2], e20 = p[2] - p[0], e31 = p[3] - p[1];
    const F3 du = e10 + v * (e32 - e10), dv = e20 + u * (e31 - e20);
    const F3 wu{dot(ax, du), dot(ay, du), dot(az, du)}, wv{dot(ax, dv), dot(ay, dv), dot(az, dv)};
    const F3 c = cross(wu, wv);
    const float squared = dot(c, c);
    if (!(squared >= FLT_MIN) || !std::isfinite(squared))
        return false;
    point.inverse_area_pdf = std::sqrt(squared);
    point.geometric_normal = c / point.inverse_area_pdf;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    if (in.normal_begin != RP_NONE) {
        F3 n[4];
        for (int i = 0; i < 4; ++i) {
            if (in.normal_begin >= s.normals.size() || idx[i] >= s.normals.size() - in.normal_begin)
                return false;
            n[i] = s.normals[in.normal_begin + idx[i]];
        }
        const F3 a = n[0] + v * (n[2] - n[0]), b = n[1] + v * (n[3] - n[1]);
        const F3 interp = a + u * (b - a);
        if (!finite3(interp))
            return false;
        const float scale = std::fmax(std::fmax(std::fabs(interp.x), std::fabs(interp.y)), std::fabs(interp.z));
        if (scale > 0) {
            const F3 sc = interp / scale;
            point.shading_normal = sc / std::sqrt(dot(sc, sc));
            if (dot(point.geometric_normal, sc) < 0)
                point.geometric_normal = -point.geometric_normal;
        }
    }
    Pair lp[3];
    const F3 magnitude = ((fabs3(p[0]) + fabs3(p[1])) + fabs3(p[2])) + fabs3(p[3]);
    for (int a = 0; a < 3; ++a) {
        const Pair lo = pr(p[0][a]) + (pr(p[2][a]) - pr(p[0][a])) * pr(v);
        const Pair hi = pr(p[1][a]) + (pr(p[3][a]) - pr(p[1][a])) * pr(v);
        lp[a] = lo + (hi - lo) * pr(u);
    }
    const bool identity = in.m[3] == 0 && in.m[7] == 0 && in.m[11] == 0 && in.m[0] == 1 && in.m[1] == 0 &&
                          in.m[2] == 0 && in.m[4] == 0 && in.m[5] == 1 && in.m[6] == 0 && in.m[8] == 0 &&
                          in.m[9] == 0 && in.m[10] == 1;
    for (int a = 0; a < 3; ++a) {
        Pair world = pr(in.m[4 * a + 3]);
        float bound = std::fabs(in.m[4 * a + 3]);
        for (int j = 0; j < 3; ++j) {
            world = world + lp[j] * pr(in.m[4 * a + j]);
            bound += magnitude[j] * std::fabs(in.m[4 * a + j]);
        }
        point.position[a] = world.hi;
        const float traversal = identity ? 0.0f : 0x1p-20f * bound;
        point.error[a] = ((std::fabs(world.lo) + 0x1p-40f * bound) + traversal) + 128.0f * FLT_MIN;
    }
    point.world_extent = 0;
    for (int i = 1; i < 4; ++i) {
        const F3 e = p[i] - p[0];
        const F3 w = fabs3(F3{dot(ax, e), dot(ay, e), dot(az, e)});
        point.world_extent = std::fmax(point.world_extent, std::fmax(w.x, std::fmax(w.y, w.z)));
    }
    return finite3(point.position) && finite3(point.error) && finite3(point.geometric_normal) &&
           finite3(point.shading_normal);
}
// shaders/analytic.h:81-85
static float stable_length(F3 v) {
    const float scale = std::fmax(std::fabs(v.x), std::fmax(std::fabs(v.y), std::fabs(v.z)));
    return scale > 0 ? scale * length3(v / scale) : 0;
}
// shaders/render.metal:1080-1118 (analytic_surface_point)
static bool analytic_surface_point(const Scene &s, u32 instance, u32 local, float u, float v, SurfacePoint &point) {
    const Instance &in = s.instances[instance];
    point.curved = true;
    if (local >= in.analytic_count)
        return false;
    const Analytic &rec = s.analytics[in.analytic_begin + local];
    const AnalyticSurface ls = evaluate_analytic(rec, u, v);
    if (!ls.valid)
        return false;
    const F3 a{in.m[0], in.m[1], in.m[2]}, b{in.m[4], in.m[5], in.m[6]}, c{in.m[8], in.m[9], in.m[10]};
    const F3 cofactor{dot(cross(b, c), ls.normal), dot(cross(c, a), ls.normal), dot(cross(a, b), ls.normal)};
    const float jacobian = stable_length(cofactor);
    if (!(jacobian > 0) || !std::isfinite(jacobian))
        return false;
    point.geometric_normal = cofactor / jacobian;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    const F3 shift{in.m[3], in.m[7], in.m[11]};
    point.position = F3{dot(a, ls.position), dot(b, ls.position), dot(c, ls.position)} + shift;
    point.error = F3{dot(fabs3(a), ls.error), dot(fabs3(b), ls.error), dot(fabs3(c), ls.error)} +
                  gamma_bound(5) * (fabs3(point.position) + fabs3(shift));
    point.inverse_area_pdf = analytic_area(rec) * jacobian;
    point.world_extent = 2 * rec.radius * std::fmax(length3(a), std::fmax(length3(b), length3(c)));
    return finite3(point.position) && finite3(point.error) && std::isfinite(point.inverse_area_pdf) &&
           point.inverse_area_pdf >= FLT_MIN;
}
bool hit_surface_point(const Scene &s, u32 prim, u32 instance, u32 local, float b1, float b2, SurfacePoint &p) {
    if (prim < s.tri_prims)
        return triangle_surface_point(s, instance, local, b1, b2, true, p);
    if (prim - s.tri_prims < s.patch_prims)
        return patch_surface_point(s, instance, local, b1, b2, p);
    return analytic_surface_point(s, instance, local, b1, b2, p);
}
void ray_point(F3 o, F3 d, float t, bool curved, F3 &position, F3 &error) {
    position = fma3(F3{t, t, t}, d, o);
    error = gamma_bound(2) * (fabs3(t * d) + fabs3(o));
    if (curved)
        for (int a = 0; a < 3; ++a) {
            const Pair value = pr(t) * pr(d[a]) + pr(o[a]);
            position[a] = value.hi;
            error[a] = (std::fabs(value.lo) + 0x1p-40f * (std::fabs(t * d[a]) + std::fabs(o[a]))) + 128.0f * FLT_MIN;
        }
}
// The hit of the world ray o + t d, t in [0, tmax], on procedural primitive `prim`.
static ShapeHit procedural_hit(const Scene &s, u32 prim, F3 o, F3 d, float tmax) {
    const Instance &in = s.instances[s.tri_instance[prim]];
    const u32 local = s.tri_local[prim];
    const float *w = in.inverse;
    const F3 r0{w[0], w[1], w[2]}, r1{w[4], w[5], w[6]}, r2{w[8], w[9], w[10]};
    const F3 oo = F3{dot(r0, o), dot(r1, o), dot(r2, o)} + F3{w[3], w[7], w[11]};
    const F3 od{dot(r0, d), dot(r1, d), dot(r2, d)};
    if (prim - s.tri_prims < s.patch_prims) {
        const auto &idx = s.patches[in.patch_begin + local];
        return intersect_bilinear(s.positions[in.vertex_begin + idx[0]], s.positions[in.vertex_begin + idx[1]],
                                  s.positions[in.vertex_begin + idx[2]], s.positions[in.vertex_begin + idx[3]], oo, od,
                                  0.0f, tmax);
    }
    return intersect_analytic(s.analytics[in.analytic_begin + local], oo, od, 0.0f, tmax);
}

// shaders/render.metal:1939-1977
bool spawn_boundary(F3 o, F3 d, float t, const SurfacePoint &pt, F3 direction, F3 &origin) {
    if (!(t >= 0) || !std::isfinite(t))
        return false;
    const F3 ng = pt.geometric_normal;
    const F3 n = dot(ng, direction) < 0 ? -ng : ng;
    const float facing = dot(n, direction);
    if (!(facing > gamma_bound(5) * dot(fabs3(n), fabs3(direction))))
        return false;
    F3 position, ray_error;
    ray_point(o, d, t, pt.curved, position, ray_error);
    const F3 error = (pt.error + fabs3(pt.position - position)) + ray_error;
    const float norm_lower = dot(n, n) * (1 - gamma_bound(4));
    const float height = dot(fabs3(n), error) * (1 + gamma_bound(8)) / norm_lower;
    origin = round_out(fma3(F3{height, height, height}, n, position), n);
    if (!(norm_lower > 0) || !std::isfinite(height) || !finite3(origin) ||
        (origin.x == o.x && origin.y == o.y && origin.z == o.z))
        return false;
    const F3 departure = origin - pt.position;
    const float separation = dot(n, departure);
    const float rounding = gamma_bound(5) * dot(fabs3(n), fabs3(departure));
    const float uncertainty = dot(fabs3(n), pt.error) * (1 + gamma_bound(4));
    return std::isfinite(separation) && std::isfinite(rounding) && std::isfinite(uncertainty) &&
           separation - rounding > uncertainty;
}

// shaders/alpha_hash.h:10-36 (PBRT MurmurHash64A over the binary32 words)
float alpha_uniform(F3 origin, F3 direction, u32 t_bits) {
    constexpr u64 m = 0xc6a4a7935bd1e995ull;
    const u32 words[7] = {fbits(origin.x), fbits(origin.y), fbits(origin.z), fbits(direction.x), fbits(direction.y),
                          fbits(direction.z), t_bits};
    u64 h = 28ull * m;
    for (u32 i = 0; i < 6; i += 2) {
        u64 k = u64(words[i]) | (u64(words[i + 1]) << 32);
        k *= m;
        k ^= k >> 47;
        k *= m;
        h ^= k;
        h *= m;
    }
    h ^= u64(words[6]);
    h *= m;
    h ^= h >> 47;
    h *= m;
    h ^= h >> 47;
    return float(u32(h)) * 0x1p-32f;
}
// shaders/packet_pt_event_body.inc:165-190 and shaders/scalar_transport.h:566-587 (constant amounts)
u32 resolve_mix(const Scene &s, F3 position, F3 toward_origin, u32 &material) {
    for (u32 depth = 0; depth <= 64; ++depth) {
        const Material &node = s.materials[material];
        if (node.scattering != 9)
            return RP_SAMPLE_SUCCESS;
        const float amount = node.mix_amount;
        if (depth == 64 || !std::isfinite(amount))
            return RP_SAMPLE_INVALID_ARITHMETIC;
        const float selector = alpha_uniform(position, toward_origin, material);
        material = amount <= 0         ? node.first
                   : amount >= 1       ? node.second
                   : selector < amount ? node.second
                                       : node.first;
        if (material >= s.materials.size())
            return RP_SAMPLE_INVALID_HIT;
    }
    return RP_SAMPLE_SUCCESS;
}
bool pass_through(const Scene &s, const Instance &in) {
    return in.invisible != 0 || s.materials[in.material].scattering == RP_INTERFACE;
}

// ================================================================= light selection
// shaders/light_sampling.h:19-42
static float importance(const LightBounds &b, F3 position, F3 normal) {
    const F3 lo{b.low[0], b.low[1], b.low[2]}, hi{b.high[0], b.high[1], b.high[2]};
    const F3 center = (lo + hi) * .5f;
    const F3 delta = position - center;
    const float r2 = dot(hi - lo, hi - lo) * .25f, d2 = dot(delta, delta);
    const float radius = std::sqrt(r2), distance = std::sqrt(d2);
    const float cb = d2 <= r2 ? -1.f : std::sqrt(std::max(0.f, 1 - r2 / d2));
    const float sb = std::sqrt(std::max(0.f, 1 - cb * cb));
    const F3 wi = distance > 0 ? delta / distance : F3{0, 0, 1};
    float cw = std::clamp(dot(F3{b.direction[0], b.direction[1], b.direction[2]}, wi), -1.f, 1.f);
    if (b.flags & 1)
        cw = std::fabs(cw);
    const float sw = std::sqrt(std::max(0.f, 1 - cw * cw)), co = b.cos_outer,
                so = std::sqrt(std::max(0.f, 1 - co * co));
    const float cx = cw > co ? 1.f : cw * co + sw * so, sx = cw > co ? 0.f : sw * co - cw * so;
    const float cp = cx > cb ? 1.f : cx * cb + sx * sb;
    if (cp <= b.cos_emission)
        return 0;
    float value = b.power * cp / std::max(d2, std::max(radius, FLT_MIN));
    if (any_nonzero3(normal)) {
        const float ci = std::clamp(std::fabs(dot(wi, normal)), 0.f, 1.f);
        const float si = std::sqrt(std::max(0.f, 1 - ci * ci));
        value *= ci > cb ? 1.f : ci * cb + si * sb;
    }
    return std::max(0.f, value);
}
// shaders/light_sampling.h:43-95
Selected light_sample(const Scene &s, F3 position, F3 normal, float u) {
    const u32 count = s.light_count;
    if (!count)
        return {RP_NONE, 0};
    u = std::clamp(u, 0.f, 0x1.fffffep-1f);
    if (s.light_sampler == 2) {
        const u32 id = std::min(u32(u * count), count - 1);
        return {id, 1.f / count};
    }
    if (s.light_sampler == 1) {
        const float v = u * count;
        const u32 i = std::min(u32(v), count - 1);
        const auto &a = s.lights.alias;
        const u32 id = v - i < a[i].threshold ? i : a[i].alias;
        return {id, a[id].pmf};
    }
    const u32 ninf = u32(s.lights.infinite.size()), nodes = u32(s.lights.nodes.size());
    const float infinite = float(ninf) / float(ninf + (nodes ? 1 : 0));
    if (u < infinite) {
        const u32 i = std::min(u32((u / infinite) * ninf), ninf - 1);
        return {s.lights.infinite[i], 1.f / float(ninf + (nodes ? 1 : 0))};
    }
    if (!nodes)
        return {RP_NONE, 0};
    u = std::min((u - infinite) / (1 - infinite), 0x1.fffffep-1f);
    float pmf = 1 - infinite;
    u32 i = 0;
    const auto &tree = s.lights.nodes;
    for (u32 steps = 0; steps < nodes; ++steps) {
        const auto &node = tree[i];
        if (node.light != RP_NONE) {
            if (importance(node, position, normal) <= 0)
                return {RP_NONE, 0};
            return {node.light, pmf};
        }
        const float a = importance(tree[i + 1], position, normal),
                    b = importance(tree[node.child], position, normal), sum = a + b;
        if (!(sum > 0))
            return {RP_NONE, 0};
        const float q = a / sum;
        if (u < q) {
            pmf *= q;
            u = std::min(u / q, 0x1.fffffep-1f);
            i++;
        } else {
            pmf *= 1 - q;
            u = std::min((u - q) / (1 - q), 0x1.fffffep-1f);
            i = node.child;
        }
    }
    return {RP_NONE, 0};
}
// shaders/light_sampling.h:96-126
float light_pmf(const Scene &s, F3 position, F3 normal, u32 id) {
    if (id >= s.light_count)
        return 0;
    if (s.light_sampler == 2)
        return 1.f / s.light_count;
    if (s.light_sampler == 1)
        return s.lights.alias[id].pmf;
    const u32 ninf = u32(s.lights.infinite.size()), nodes = u32(s.lights.nodes.size());
    if (s.lights.records[id].flags & 1)
        return 1.f / float(ninf + (nodes ? 1 : 0));
    u32 i = s.lights.records[id].leaf;
    if (i >= nodes)
        return 0;
    const auto &tree = s.lights.nodes;
    if (importance(tree[i], position, normal) <= 0)
        return 0;
    float result = 1.f - float(ninf) / float(ninf + (nodes ? 1 : 0));
    for (u32 steps = 0; steps < nodes; ++steps) {
        const u32 parent = tree[i].parent;
        if (parent == RP_NONE)
            return result;
        const float a = importance(tree[parent + 1], position, normal),
                    b = importance(tree[tree[parent].child], position, normal), sum = a + b;
        if (!(sum > 0))
            return 0;
        result *= i == parent + 1 ? a / sum : b / sum;
        i = parent;
    }
    return 0;
}

// ================================================================= light geometry (triangles)
// src/light_geometry_sampling_shared.h (PBRT spherical triangle sampling); V3 / float is a
// true division here, as on the GPU.
namespace lg {
constexpr float one_minus_epsilon = 0x1.fffffep-1f;
inline float clamp01(float v) { return std::min(1.f, std::max(0.f, v)); }
inline float safe_sqrt(float v) { return std::sqrt(std::max(0.f, v)); }
inline F3 unitv(F3 v) { return v / length3(v); }
inline bool nonzero(F3 v) { return dot(v, v) > 0; }
// :74-77
inline float angle(F3 a, F3 b) {
    return dot(a, b) < 0 ? pi_f - 2 * std::asin(std::min(1.f, length3(a + b) / 2))
                         : 2 * std::asin(std::min(1.f, length3(a - b) / 2));
}
// :78-80
inline float triangle_area(F3 a, F3 b, F3 c) {
    return std::fabs(2 * std::atan2(dot(a, cross(b, c)), 1 + dot(a, b) + dot(a, c) + dot(b, c)));
}
// :81-85
inline float triangle_solid_angle(F3 p0, F3 p1, F3 p2, F3 r) {
    if (!nonzero(p0 - r) || !nonzero(p1 - r) || !nonzero(p2 - r))
        return 0;
    return triangle_area(unitv(p0 - r), unitv(p1 - r), unitv(p2 - r));
}
inline bool spherical_triangle(float area) { return area >= 3e-4f && area <= 6.22f; }
struct Weights {
    float a, b, c, d;
};
// :91-95
inline Weights normalized_weights(Weights w) {
    const float s = std::max(std::max(w.a, w.b), std::max(w.c, w.d));
    return s > 0 ? Weights{w.a / s, w.b / s, w.c / s, w.d / s} : Weights{1, 1, 1, 1};
}
// :96-100
inline float linear_sample(float u, float a, float b) {
    if (u == 0 && a == 0)
        return 0;
    return std::min(one_minus_epsilon, u * (a + b) / (a + std::sqrt((1 - u) * a * a + u * b * b)));
}
// :101-106
inline void bilinear_sample(float ux, float uy, Weights weights, float &x, float &y) {
    const auto w = normalized_weights(weights);
    y = linear_sample(uy, w.a + w.b, w.c + w.d);
    x = linear_sample(ux, (1 - y) * w.a + y * w.c, (1 - y) * w.b + y * w.d);
}
// :107-115
inline float bilinear_pdf(float ux, float uy, Weights weights) {
    if (ux < 0 || ux > 1 || uy < 0 || uy > 1)
        return 0;
    const auto w = normalized_weights(weights);
    return 4 *
           ((1 - ux) * (1 - uy) * w.a + ux * (1 - uy) * w.b + (1 - ux) * uy * w.c + ux * uy * w.d) /
           (w.a + w.b + w.c + w.d);
}
// :116-121
inline Weights triangle_cosines(F3 a, F3 b, F3 c, F3 r, F3 n) {
    const float wa = std::max(.01f, std::fabs(dot(n, unitv(a - r))));
    const float wb = std::max(.01f, std::fabs(dot(n, unitv(b - r))));
    const float wc = std::max(.01f, std::fabs(dot(n, unitv(c - r))));
    return {wb, wb, wa, wc};
}
// :122-125
inline void triangle_uniform_uv(float ux, float uy, float &b1, float &b2) {
    const float root = std::sqrt(ux);
    b1 = 1 - root;
    b2 = uy * root;
}
// :128-172
inline bool triangle_sample(F3 p0, F3 p1, F3 p2, F3 r, float ux, float uy, float &b1o, float &b2o) {
    const F3 a = unitv(p0 - r), b = unitv(p1 - r), c = unitv(p2 - r);
    const F3 nab = cross(a, b), nca = cross(c, a);
    if (!nonzero(nab) || !nonzero(nca))
        return false;
    const float alpha = angle(unitv(nab), -unitv(nca));
    const float area = triangle_area(a, b, c);
    const float ca = std::cos(alpha), sa = std::sin(alpha);
    const float subarea = ux * area;
    const float sh = std::sin(subarea / 2), st = std::sin(subarea), ct_area = std::cos(subarea);
    const float one_minus_ct = 2 * sh * sh;
    const float sp = sa * ct_area - ca * st;
    const float cp = -ca * ct_area - sa * st;
    const float k1 = -2 * std::sin(alpha - subarea / 2) * sh;
    const float k2 = sa * (.5f * dot(a - b, a - b) - one_minus_ct) - ca * st;
    const float divisor = (k2 * sp + k1 * cp) * sa;
    if (divisor == 0)
        return false;
    const float omc = std::min(2.f, std::max(0.f, (-k2 * one_minus_ct - k1 * st) / divisor));
    const float cosbp = 1 - omc;
    const F3 arc = c - dot(c, a) * a;
    if (!nonzero(arc))
        return false;
    const F3 cprime = cosbp * a + safe_sqrt(omc * (2 - omc)) * unitv(arc);
    const float omct = uy * .5f * dot(cprime - b, cprime - b);
    const float ct = 1 - omct;
    const F3 tangent = cprime - dot(cprime, b) * b;
    if (!nonzero(tangent))
        return false;
    const F3 direction = ct * b + safe_sqrt(omct * (2 - omct)) * unitv(tangent);
    const F3 e1 = p1 - p0, e2 = p2 - p0, s1 = cross(direction, e2);
    const float denom = dot(s1, e1);
    if (denom == 0)
        return false;
    const F3 sv = r - p0;
    float b1 = clamp01(dot(sv, s1) / denom), b2 = clamp01(dot(direction, cross(sv, e1)) / denom);
    if (b1 + b2 > 1) {
        const float sum = b1 + b2;
        b1 /= sum;
        b2 /= sum;
    }
    b1o = b1;
    b2o = b2;
    return std::isfinite(b1) && std::isfinite(b2);
}
// :174-182
inline void triangle_inverse(F3 p0, F3 p1, F3 p2, F3 r, F3 dir, float &u0, float &u1) {
    const F3 a = unitv(p0 - r), b = unitv(p1 - r), c = unitv(p2 - r);
    F3 cp = unitv(cross(cross(b, dir), cross(c, a)));
    if (dot(cp, a + c) < 0)
        cp = -cp;
    u0 = clamp01(triangle_area(a, b, cp) / triangle_area(a, b, c));
    u1 = clamp01(dot(dir - b, dir - b) / dot(cp - b, cp - b));
}
} // namespace lg

static void emitter_corners(const Scene &s, u32 emitter, F3 p[3]) {
    // shaders/light_geometry_sampling.h:16-29
    const auto &e = s.emitters[emitter];
    const Instance &in = s.instances[e.instance];
    const auto &tri = s.triangles[in.triangle_begin + e.primitive];
    for (int i = 0; i < 3; ++i)
        p[i] = world_point(in, s.positions[in.vertex_begin + tri[i]]);
}
// shaders/light_geometry_sampling.h:58-67 (area_solid_angle_pdf)
static float area_solid_angle_pdf(float area_density, F3 reference, const SurfacePoint &point) {
    const F3 delta = point.position - reference;
    const float d2 = dot(delta, delta);
    if (!(d2 > 0) || !(area_density > 0))
        return 0;
    const float cosine = std::fabs(dot(point.geometric_normal, delta * (1.0f / std::sqrt(d2))));
    return cosine > 0 ? area_density * d2 / cosine : 0;
}
// shaders/light_geometry_sampling.h:116-153 (pdf), triangles
float light_geometry_pdf(const Scene &s, u32 emitter, F3 reference, F3 normal,
                         const SurfacePoint &point) {
    const F3 delta = point.position - reference;
    if (!(dot(delta, delta) > 0) || !(point.inverse_area_pdf > 0))
        return 0;
    F3 p[3];
    emitter_corners(s, emitter, p);
    const float area = lg::triangle_solid_angle(p[0], p[1], p[2], reference);
    if (lg::spherical_triangle(area)) {
        float u0, u1;
        lg::triangle_inverse(p[0], p[1], p[2], reference, normalize3(delta), u0, u1);
        return (dot(normal, normal) > 0
                    ? lg::bilinear_pdf(u0, u1, lg::triangle_cosines(p[0], p[1], p[2], reference, normal))
                    : 1.f) /
               area;
    }
    // area_pdf (shaders/light_geometry_sampling.h:44-57): triangles have parametric pdf 1
    return area_solid_angle_pdf(1 / point.inverse_area_pdf, reference, point);
}
// shaders/light_geometry_sampling.h:155-209 (sample), triangles
bool light_geometry_sample(const Scene &s, u32 emitter, F3 reference, F3 normal, float ux, float uy,
                           float &b1, float &b2, SurfacePoint &point, float &pdf) {
    if (!std::isfinite(ux) || !std::isfinite(uy) || ux < 0 || uy < 0 || ux > 1 || uy > 1)
        return false;
    ux = std::min(ux, lg::one_minus_epsilon);
    uy = std::min(uy, lg::one_minus_epsilon);
    F3 p[3];
    emitter_corners(s, emitter, p);
    bool selected = false;
    const float area = lg::triangle_solid_angle(p[0], p[1], p[2], reference);
    if (lg::spherical_triangle(area)) {
        if (dot(normal, normal) > 0) {
            float x, y;
            lg::bilinear_sample(ux, uy, lg::triangle_cosines(p[0], p[1], p[2], reference, normal), x, y);
            ux = x;
            uy = y;
        }
        if (!lg::triangle_sample(p[0], p[1], p[2], reference, ux, uy, b1, b2))
            return false;
        selected = true;
    }
    if (!selected)
        lg::triangle_uniform_uv(ux, uy, b1, b2);
    const auto &e = s.emitters[emitter];
    if (!std::isfinite(b1) || !std::isfinite(b2) ||
        !triangle_surface_point(s, e.instance, e.primitive, b1, b2, false, point))
        return false;
    pdf = light_geometry_pdf(s, emitter, reference, normal, point);
    return std::isfinite(pdf) && pdf >= 0;
}

} // namespace oracle

extern "C" {

void or_probe_bilinear(const float *q, uint32_t count, float *out) {
    using namespace oracle;
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 20 * size_t(i);
        const ShapeHit h = intersect_bilinear(F3{a[0], a[1], a[2]}, F3{a[3], a[4], a[5]}, F3{a[6], a[7], a[8]},
                                              F3{a[9], a[10], a[11]}, F3{a[12], a[13], a[14]}, F3{a[15], a[16], a[17]},
                                              a[18], a[19]);
        float *o = out + 4 * size_t(i);
        o[0] = h.hit ? 1.f : 0.f;
        o[1] = h.t;
        o[2] = h.u;
        o[3] = h.v;
    }
}

void or_probe_analytic(const float *q, uint32_t count, float *out) {
    using namespace oracle;
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 16 * size_t(i);
        Analytic rec;
        std::memcpy(&rec.kind, a, 4);
        std::memcpy(&rec.subtype, a + 1, 4);
        rec.radius = a[2];
        rec.z_min = a[3];
        rec.z_max = a[4];
        rec.phi_max = a[5];
        rec.inner_radius = a[6];
        rec.height = a[7];
        const ShapeHit h = intersect_analytic(rec, F3{a[8], a[9], a[10]}, F3{a[11], a[12], a[13]}, a[14], a[15]);
        float *o = out + 16 * size_t(i);
        o[0] = h.hit ? 1.f : 0.f;
        o[1] = h.t;
        o[2] = h.u;
        o[3] = h.v;
        const AnalyticSurface e = evaluate_analytic(rec, h.hit ? h.u : 0.f, h.hit ? h.v : 0.f);
        const F3 vs[4] = {e.position, e.normal, e.dpdu, e.dpdv};
        for (int k = 0; k < 4; ++k) {
            o[4 + 3 * k] = vs[k].x;
            o[5 + 3 * k] = vs[k].y;
            o[6 + 3 * k] = vs[k].z;
        }
    }
}

} // extern "C"
