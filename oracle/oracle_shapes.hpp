// ORACLE -- test infrastructure only (see oracle_math.hpp).
// Procedural primitives: PBRT bilinear patches (shaders/bilinear.h, the ruled-surface solve in
// float pairs) and analytic shapes (shaders/analytic.h: sphere, disk, cylinder), restated for
// the host.  Pinned to rypath's own headers compiled for the host (oracle/_ref/libref_shapes.so).
#pragma once

#include "oracle_math.hpp"

#include <cfloat>
#include <cmath>

namespace oracle {

// ---------------------------------------------------------------- float pairs
struct Pair {
    float hi = 0, lo = 0;
};
inline Pair pr(float v) { return {v, 0.0f}; }
inline Pair operator-(Pair a) { return {-a.hi, -a.lo}; }
// compensated sum: the rounded sum and what it lost (shaders/bilinear.h:33-38)
inline Pair operator+(Pair a, Pair b) {
    const float sum = a.hi + b.hi;
    const float part = sum - a.hi;
    const float err = (a.hi - (sum - part)) + (b.hi - part) + (a.lo + b.lo);
    const float r = sum + err;
    return {r, err - (r - sum)};
}
inline Pair operator-(Pair a, Pair b) { return a + (-b); }
// product with the fma residual (:42-47)
inline Pair operator*(Pair a, Pair b) {
    const float p = a.hi * b.hi;
    const float err = std::fma(a.hi, b.hi, -p) + a.hi * b.lo + a.lo * b.hi;
    const float r = p + err;
    return {r, err - (r - p)};
}
// quotient with one correction step (:49-56)
inline Pair operator/(Pair a, Pair b) {
    const float q = a.hi / b.hi;
    if (!std::isfinite(q))
        return {q, 0.0f};
    const float correction = (a - b * pr(q)).hi / b.hi;
    return pr(q) + pr(correction);
}
inline Pair scaled(Pair a, int e) { return {std::ldexp(a.hi, e), std::ldexp(a.lo, e)}; }

struct Proj {
    Pair x, y, z;
};
inline Proj operator+(const Proj &a, const Proj &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Proj operator-(const Proj &a, const Proj &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Proj operator*(const Proj &a, Pair s) { return {a.x * s, a.y * s, a.z * s}; }
inline Pair cross2(const Proj &a, const Proj &b) { return a.x * b.y - a.y * b.x; }
inline float proj_size(const Proj &a) { return std::fmax(std::fabs(a.x.hi), std::fabs(a.y.hi)); }
// :80-92 (minimum_projected_ruling)
inline float min_ruling(const Proj &edge, const Proj &warp) {
    const float sx = edge.x.hi, sy = edge.y.hi, wx = warp.x.hi, wy = warp.y.hi;
    const float scale = std::fmax(std::fabs(wx), std::fabs(wy));
    if (scale == 0.0f)
        return proj_size(edge);
    const float ux = wx / scale, uy = wy / scale;
    const float t = std::fmin(std::fmax(-(sx * ux + sy * uy) / (scale * (ux * ux + uy * uy)), 0.0f), 1.0f);
    return proj_size(edge + warp * pr(t));
}
inline float axis(F3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
// :94-108 (project_bilinear_corner)
inline Proj project_corner(F3 p, F3 o, F3 d, int exponent, int dominant) {
    const int i = (dominant + 1) % 3, j = (dominant + 2) % 3;
    const Pair x = scaled(pr(axis(p, i)), -exponent) - scaled(pr(axis(o, i)), -exponent);
    const Pair y = scaled(pr(axis(p, j)), -exponent) - scaled(pr(axis(o, j)), -exponent);
    const Pair z = scaled(pr(axis(p, dominant)), -exponent) - scaled(pr(axis(o, dominant)), -exponent);
    const Pair dd = pr(axis(d, dominant));
    return {x * dd - z * pr(axis(d, i)), y * dd - z * pr(axis(d, j)), z};
}
inline bool in_unit(Pair v) { return v.hi >= 0.0f && (v - pr(1.0f)).hi <= 0.0f; }

struct ShapeHit {
    bool hit = false;
    float t = INFINITY, u = 0, v = 0;
};
// :114-155 (consider_bilinear_edge)
inline void bilinear_edge(const Proj &a, const Proj &b, float ua_u, float ua_v, float ub_u, float ub_v, float dd,
                          int ray_exponent, float t_min, ShapeHit &best) {
    const Proj diff = a - b;
    const bool use_x = std::fabs(diff.x.hi) >= std::fabs(diff.y.hi);
    const Pair from = use_x ? a.x : a.y, to = use_x ? b.x : b.y, den = use_x ? diff.x : diff.y;
    if (den.hi == 0.0f || (from.hi > 0.0f && to.hi > 0.0f) || (from.hi < 0.0f && to.hi < 0.0f))
        return;
    const Pair left = a.x * b.y, right = a.y * b.x;
    const float budget = 0x1p-42f * (std::fabs(left.hi) + std::fabs(right.hi));
    if (!(std::fabs((left - right).hi) <= budget))
        return;
    const Pair z = (b.z * from - a.z * to) / den;
    const float t = scaled(z / pr(dd), ray_exponent).hi;
    if (std::isfinite(t) && t >= t_min && t <= best.t) {
        const float f = (from / den).hi;
        best = {true, t, ua_u + (ub_u - ua_u) * f, ua_v + (ub_v - ua_v) * f};
    }
}
// :157-196 (consider_bilinear_root)
inline void bilinear_root(Pair u, const Proj &origin, const Proj &eu, const Proj &ev, const Proj &warp, float dd,
                          int ray_exponent, float t_min, bool swapped, ShapeHit &best) {
    if (!in_unit(u))
        return;
    const Proj delta = origin + eu * u;
    const Proj ruling = ev + warp * u;
    const bool use_x = std::fabs(ruling.x.hi) >= std::fabs(ruling.y.hi);
    const Pair den = use_x ? ruling.x : ruling.y;
    if (den.hi == 0.0f)
        return;
    const Pair v = -(use_x ? delta.x : delta.y) / den;
    if (!in_unit(v))
        return;
    const Proj point = delta + ruling * v;
    const float budget = 0x1p-39f * (proj_size(origin) + proj_size(eu) + proj_size(ev) + proj_size(warp));
    if (!(proj_size(point) <= budget))
        return;
    const float t = scaled(point.z / pr(dd), ray_exponent).hi;
    if (std::isfinite(t) && t >= t_min && t <= best.t)
        best = swapped ? ShapeHit{true, t, v.hi, u.hi} : ShapeHit{true, t, u.hi, v.hi};
}
inline float max_abs3(F3 v) { return std::fmax(std::fabs(v.x), std::fmax(std::fabs(v.y), std::fabs(v.z))); }
// :198-305 (intersect_bilinear_if, every candidate accepted)
inline ShapeHit intersect_bilinear(F3 p00, F3 p10, F3 p01, F3 p11, F3 o, F3 d, float t_min, float t_max) {
    ShapeHit best{false, t_max, 0.0f, 0.0f};
    const float pmax = std::fmax(std::fmax(max_abs3(p00), max_abs3(p10)),
                                 std::fmax(std::fmax(max_abs3(p01), max_abs3(p11)), max_abs3(o)));
    const float dmax = max_abs3(d);
    if (!(pmax > 0.0f && dmax > 0.0f && std::isfinite(pmax) && std::isfinite(dmax)))
        return best;
    int pe, de;
    std::frexp(pmax, &pe);
    std::frexp(dmax, &de);
    d = F3{std::ldexp(d.x, -de), std::ldexp(d.y, -de), std::ldexp(d.z, -de)};
    const F3 m{std::fabs(d.x), std::fabs(d.y), std::fabs(d.z)};
    const int dominant = m.x >= m.y && m.x >= m.z ? 0 : (m.y >= m.z ? 1 : 2);
    const Proj offset = project_corner(p00, o, d, pe, dominant);
    const Proj corner_u = project_corner(p10, o, d, pe, dominant);
    const Proj corner_v = project_corner(p01, o, d, pe, dominant);
    const Proj opposite = project_corner(p11, o, d, pe, dominant);
    Proj eu = corner_u - offset, ev = corner_v - offset;
    const Proj warp = ((opposite - offset) - eu) - ev;
    const int ray_exponent = pe - de;
    const bool swapped = min_ruling(eu, warp) > min_ruling(ev, warp);
    if (swapped)
        std::swap(eu, ev);
    const Pair a = cross2(eu, warp);
    const Pair b = cross2(offset, warp) + cross2(eu, ev);
    const Pair c = cross2(offset, ev);
    if (a.hi == 0.0f && b.hi == 0.0f && c.hi == 0.0f)
        return best;
    const float dd = axis(d, dominant);
    bilinear_edge(offset, corner_u, 0, 0, 1, 0, dd, ray_exponent, t_min, best);
    bilinear_edge(offset, corner_v, 0, 0, 0, 1, dd, ray_exponent, t_min, best);
    bilinear_edge(corner_u, opposite, 1, 0, 1, 1, dd, ray_exponent, t_min, best);
    bilinear_edge(corner_v, opposite, 0, 1, 1, 1, dd, ray_exponent, t_min, best);
    if (a.hi == 0.0f) {
        if (b.hi != 0.0f)
            bilinear_root(-c / b, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
        return best;
    }
    int ce;
    std::frexp(std::fmax(std::fabs(a.hi), std::fmax(std::fabs(b.hi), std::fabs(c.hi))), &ce);
    const Pair sa = scaled(a, -ce), sb = scaled(b, -ce), sc = scaled(c, -ce);
    const Pair disc = sb * sb - (sa * sc) * pr(4.0f);
    if (disc.hi < 0.0f)
        return best;
    if (disc.hi == 0.0f) {
        bilinear_root((sb * pr(-0.5f)) / sa, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
        return best;
    }
    const float root = std::sqrt(disc.hi);
    const Pair correction = (disc - pr(root) * pr(root)) / pr(2.0f * root);
    const Pair sq = pr(root) + correction;
    const Pair q = (sb + (sb.hi < 0.0f ? -sq : sq)) * pr(-0.5f);
    bilinear_root(q / sa, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
    bilinear_root(sc / q, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
    return best;
}

// ---------------------------------------------------------------- analytic shapes
// geometry_wire::Analytic (src/geometry_wire.h:31-40)
struct Analytic {
    u32 kind = 4, subtype = 1;
    float radius = 1, z_min = -1, z_max = 1, phi_max = 6.2831853f, inner_radius = 0, height = 0;
};
// shaders/analytic.h:21-25
inline float analytic_area(const Analytic &s) {
    return s.subtype == 2u ? .5f * s.phi_max * (s.radius - s.inner_radius) * (s.radius + s.inner_radius)
                           : s.phi_max * s.radius * (s.z_max - s.z_min);
}
struct AnalyticSurface {
    F3 position, normal, dpdu, dpdv, dndu, dndv, error;
    bool valid = false;
};
inline F3 abs3(F3 v) { return {std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)}; }
// shaders/analytic.h:26-64 (evaluate_analytic)
inline AnalyticSurface evaluate_analytic(const Analytic &s, float u, float v) {
    const float phi = u * s.phi_max;
    const float c = std::cos(phi), sn = std::sin(phi), r = s.radius, pm = s.phi_max;
    AnalyticSurface out{};
    if (s.subtype == 2u) {
        const float radius = std::fma(v, s.inner_radius - r, r);
        out.position = {radius * c, radius * sn, s.height};
        out.normal = {0, 0, 1};
        const float fr = radius > 0 ? radius : r;
        out.dpdu = {-pm * fr * sn, pm * fr * c, 0};
        out.dpdv = {(s.inner_radius - r) * c, (s.inner_radius - r) * sn, 0};
    } else if (s.subtype == 3u) {
        out.position = {r * c, r * sn, std::fma(v, s.z_max - s.z_min, s.z_min)};
        out.normal = {c, sn, 0};
        out.dpdu = {-pm * r * sn, pm * r * c, 0};
        out.dpdv = {0, 0, s.z_max - s.z_min};
        out.dndu = {-pm * sn, pm * c, 0};
    } else if (s.subtype == 1u) {
        const float t0 = std::acos(std::fmin(std::fmax(s.z_min / r, -1.0f), 1.0f));
        const float t1 = std::acos(std::fmin(std::fmax(s.z_max / r, -1.0f), 1.0f));
        const float dt = t1 - t0, theta = std::fma(v, dt, t0);
        const float st = std::fmax(0.0f, std::sin(theta)), ct = std::cos(theta);
        out.position = {r * st * c, r * st * sn, r * ct};
        out.normal = {st * c, st * sn, ct};
        const float fs = std::fmax(st, 1e-7f);
        out.dpdu = {-pm * r * fs * sn, pm * r * fs * c, 0};
        out.dpdv = {dt * r * ct * c, dt * r * ct * sn, -dt * r * st};
        out.dndu = {-pm * fs * sn, pm * fs * c, 0};
        out.dndv = {dt * ct * c, dt * ct * sn, -dt * st};
    }
    out.error = 0x1p-19f * (abs3(out.position) + F3{s.radius, s.radius, s.radius});
    out.valid = s.subtype >= 1u && s.subtype <= 3u && finite3(out.position) && finite3(out.normal) &&
                finite3(out.dpdu) && finite3(out.dpdv) && finite3(out.dndu) && finite3(out.dndv) && finite3(out.error);
    return out;
}
// shaders/analytic.h:95-180 (intersect_analytic_if, every root accepted)
inline ShapeHit intersect_analytic(const Analytic &s, F3 o, F3 d, float t_min, float t_max) {
    const ShapeHit none{false, INFINITY, 0.0f, 0.0f};
    float roots[2];
    int count = 0;
    if (s.subtype == 2u) {
        if (d.z == 0)
            return none;
        roots[count++] = (s.height - o.z) / d.z;
    } else {
        const F3 oo = s.subtype == 1u ? o : F3{o.x, o.y, 0};
        const F3 dd = s.subtype == 1u ? d : F3{d.x, d.y, 0};
        const float a = dot(dd, dd);
        if (!(a > 0) || !std::isfinite(a))
            return none;
        const float b = 2 * dot(oo, dd);
        const float c = std::fma(oo.x, oo.x, std::fma(oo.y, oo.y, oo.z * oo.z)) - s.radius * s.radius;
        const float projection = -dot(oo, dd) / a;
        const F3 closest{std::fma(projection, dd.x, oo.x), std::fma(projection, dd.y, oo.y),
                         std::fma(projection, dd.z, oo.z)};
        const float distance = std::sqrt(dot(closest, closest));
        const float disc = 4 * a * (s.radius - distance) * (s.radius + distance);
        if (!(disc >= 0) || !std::isfinite(disc))
            return none;
        const float q = -.5f * (b + std::copysign(std::sqrt(disc), b));
        if (q == 0)
            roots[count++] = projection;
        else {
            roots[count++] = q / a;
            roots[count++] = c / q;
            if (roots[0] > roots[1])
                std::swap(roots[0], roots[1]);
        }
    }
    for (int i = 0; i < count; ++i) {
        const float t = roots[i];
        if (!std::isfinite(t) || t < t_min || t > t_max)
            continue;
        F3 p{std::fma(t, d.x, o.x), std::fma(t, d.y, o.y), std::fma(t, d.z, o.z)};
        if (s.subtype == 1u) {
            const float length_p = std::sqrt(dot(p, p));
            if (!(length_p > 0))
                continue;
            const float k = s.radius / length_p;
            p = F3{p.x * k, p.y * k, p.z * k};
        } else if (s.subtype == 3u) {
            const float length_p = std::sqrt(p.x * p.x + p.y * p.y);
            if (!(length_p > 0))
                continue;
            const float k = s.radius / length_p;
            p = F3{p.x * k, p.y * k, p.z};
        }
        float phi = std::atan2(p.y, p.x);
        if (phi < 0)
            phi += 2 * float(M_PI);
        if (phi > s.phi_max)
            continue;
        float v;
        if (s.subtype == 2u) {
            const float radius = std::sqrt(p.x * p.x + p.y * p.y);
            if (radius < s.inner_radius || radius > s.radius)
                continue;
            v = (s.radius - radius) / (s.radius - s.inner_radius);
        } else if (s.subtype == 1u) {
            if ((s.z_min > -s.radius && p.z < s.z_min) || (s.z_max < s.radius && p.z > s.z_max))
                continue;
            const float t0 = std::acos(std::fmin(std::fmax(s.z_min / s.radius, -1.0f), 1.0f));
            const float t1 = std::acos(std::fmin(std::fmax(s.z_max / s.radius, -1.0f), 1.0f));
            v = (std::acos(std::fmin(std::fmax(p.z / s.radius, -1.0f), 1.0f)) - t0) / (t1 - t0);
        } else {
            if (p.z < s.z_min || p.z > s.z_max)
                continue;
            v = (p.z - s.z_min) / (s.z_max - s.z_min);
        }
        const float uu = std::fmin(std::fmax(phi / s.phi_max, 0.0f), 1.0f), vv = std::fmin(std::fmax(v, 0.0f), 1.0f);
        if (std::isfinite(uu) && std::isfinite(vv))
            return {true, t, uu, vv};
    }
    return none;
}

} // namespace oracle
