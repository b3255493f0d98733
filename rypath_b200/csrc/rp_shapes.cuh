// Procedural primitives: PBRT bilinear patches and analytic shapes (sphere, disk, cylinder),
// intersected in the object space of their instance.
//
// The bilinear test is PBRT's ruled-surface solve carried in float pairs (value + rounding
// error) as rypath states it (shaders/bilinear.h): the corners are projected along the ray's
// dominant axis, the quadratic for the ruling parameter is solved with a compensated
// discriminant, the four straight edges are solved on their own so that neighbouring patches
// agree, and each candidate is checked against its residual.  Its arithmetic is plain IEEE
// float (no transcendental), so the device and the host restatement agree bit for bit.  The
// analytic shapes follow shaders/analytic.h (PBRT's quadrics with the reprojection of the hit
// onto the surface).
#pragma once

#include "rp_math.cuh"

namespace rp {

// ---------------------------------------------------------------- float pairs
struct Pair {
    float hi, lo;
};
RP_DEV Pair pr(float v) { return {v, 0.0f}; }
RP_DEV Pair operator-(Pair a) { return {-a.hi, -a.lo}; }
RP_DEV Pair operator+(Pair a, Pair b) {
    const float sum = a.hi + b.hi;
    const float part = sum - a.hi;
    const float err = (a.hi - (sum - part)) + (b.hi - part) + (a.lo + b.lo);
    const float r = sum + err;
    return {r, err - (r - sum)};
}
RP_DEV Pair operator-(Pair a, Pair b) { return a + (-b); }
RP_DEV Pair operator*(Pair a, Pair b) {
    const float p = a.hi * b.hi;
    const float err = fmaf(a.hi, b.hi, -p) + a.hi * b.lo + a.lo * b.hi;
    const float r = p + err;
    return {r, err - (r - p)};
}
RP_DEV Pair operator/(Pair a, Pair b) {
    const float q = a.hi / b.hi;
    if (!isfinite(q))
        return {q, 0.0f};
    const float correction = (a - b * pr(q)).hi / b.hi;
    return pr(q) + pr(correction);
}
RP_DEV Pair scaled(Pair a, int e) { return {ldexpf(a.hi, e), ldexpf(a.lo, e)}; }

struct Proj { // a corner projected perpendicular to the ray, and its dominant coordinate
    Pair x, y, z;
};
RP_DEV Proj operator+(const Proj &a, const Proj &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
RP_DEV Proj operator-(const Proj &a, const Proj &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
RP_DEV Proj operator*(const Proj &a, Pair s) { return {a.x * s, a.y * s, a.z * s}; }
RP_DEV Pair cross2(const Proj &a, const Proj &b) { return a.x * b.y - a.y * b.x; }
RP_DEV float proj_size(const Proj &a) { return fmaxf(fabsf(a.x.hi), fabsf(a.y.hi)); }
// The smallest projected size of the ruling edge + warp t over t in [0, 1].
RP_DEV float min_ruling(const Proj &edge, const Proj &warp) {
    const float sx = edge.x.hi, sy = edge.y.hi, wx = warp.x.hi, wy = warp.y.hi;
    const float scale = fmaxf(fabsf(wx), fabsf(wy));
    if (scale == 0.0f)
        return proj_size(edge);
    const float ux = wx / scale, uy = wy / scale;
    const float t = fminf(fmaxf(-(sx * ux + sy * uy) / (scale * (ux * ux + uy * uy)), 0.0f), 1.0f);
    return proj_size(edge + warp * pr(t));
}
RP_DEV Proj project_corner(V3 p, V3 o, V3 d, int exponent, int dominant) {
    const int i = (dominant + 1) % 3, j = (dominant + 2) % 3;
    const Pair x = scaled(pr(comp(p, i)), -exponent) - scaled(pr(comp(o, i)), -exponent);
    const Pair y = scaled(pr(comp(p, j)), -exponent) - scaled(pr(comp(o, j)), -exponent);
    const Pair z = scaled(pr(comp(p, dominant)), -exponent) - scaled(pr(comp(o, dominant)), -exponent);
    const Pair dd = pr(comp(d, dominant));
    return {x * dd - z * pr(comp(d, i)), y * dd - z * pr(comp(d, j)), z};
}
RP_DEV bool in_unit(Pair v) { return v.hi >= 0.0f && (v - pr(1.0f)).hi <= 0.0f; }

struct ShapeHit {
    bool hit;
    float t, u, v;
};

// A straight boundary from `a` (uv ua) to `b` (uv ub): its crossing with the ray where the
// projected segment brackets the ray and is collinear with it to the pairs' precision.
RP_DEV void bilinear_edge(const Proj &a, const Proj &b, float ua_u, float ua_v, float ub_u, float ub_v, float dd,
                          int ray_exponent, float t_min, ShapeHit &best) {
    const Proj diff = a - b;
    const bool use_x = fabsf(diff.x.hi) >= fabsf(diff.y.hi);
    const Pair from = use_x ? a.x : a.y, to = use_x ? b.x : b.y, den = use_x ? diff.x : diff.y;
    if (den.hi == 0.0f || (from.hi > 0.0f && to.hi > 0.0f) || (from.hi < 0.0f && to.hi < 0.0f))
        return;
    const Pair left = a.x * b.y, right = a.y * b.x;
    const float budget = 0x1p-42f * (fabsf(left.hi) + fabsf(right.hi));
    if (!(fabsf((left - right).hi) <= budget))
        return;
    const Pair z = (b.z * from - a.z * to) / den;
    const float t = scaled(z / pr(dd), ray_exponent).hi;
    if (isfinite(t) && t >= t_min && t <= best.t) {
        const float f = (from / den).hi;
        best = {true, t, ua_u + (ub_u - ua_u) * f, ua_v + (ub_v - ua_v) * f};
    }
}
// A root u of the ruling quadratic: the ruling at u meets the ray at v, checked against the
// projected residual.
RP_DEV void bilinear_root(Pair u, const Proj &origin, const Proj &eu, const Proj &ev, const Proj &warp, float dd,
                          int ray_exponent, float t_min, bool swapped, ShapeHit &best) {
    if (!in_unit(u))
        return;
    const Proj delta = origin + eu * u;
    const Proj ruling = ev + warp * u;
    const bool use_x = fabsf(ruling.x.hi) >= fabsf(ruling.y.hi);
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
    if (isfinite(t) && t >= t_min && t <= best.t)
        best = swapped ? ShapeHit{true, t, v.hi, u.hi} : ShapeHit{true, t, u.hi, v.hi};
}
RP_DEV float max_abs3(V3 v) { return fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z))); }
// The closest hit with t in [t_min, t_max] of the patch p00 p10 p01 p11 (intersect_bilinear,
// shaders/bilinear.h:222-315).
RP_DEV ShapeHit intersect_bilinear(V3 p00, V3 p10, V3 p01, V3 p11, V3 o, V3 d, float t_min, float t_max) {
    ShapeHit best{false, t_max, 0.0f, 0.0f};
    const float pmax = fmaxf(fmaxf(max_abs3(p00), max_abs3(p10)), fmaxf(fmaxf(max_abs3(p01), max_abs3(p11)), max_abs3(o)));
    const float dmax = max_abs3(d);
    if (!(pmax > 0.0f && dmax > 0.0f && isfinite(pmax) && isfinite(dmax)))
        return best;
    int pe, de;
    frexpf(pmax, &pe);
    frexpf(dmax, &de);
    d = v3(ldexpf(d.x, -de), ldexpf(d.y, -de), ldexpf(d.z, -de));
    const V3 m = vabs(d);
    const int dominant = m.x >= m.y && m.x >= m.z ? 0 : (m.y >= m.z ? 1 : 2);
    const Proj offset = project_corner(p00, o, d, pe, dominant);
    const Proj corner_u = project_corner(p10, o, d, pe, dominant);
    const Proj corner_v = project_corner(p01, o, d, pe, dominant);
    const Proj opposite = project_corner(p11, o, d, pe, dominant);
    Proj eu = corner_u - offset, ev = corner_v - offset;
    const Proj warp = ((opposite - offset) - eu) - ev;
    const int ray_exponent = pe - de;
    const bool swapped = min_ruling(eu, warp) > min_ruling(ev, warp);
    if (swapped) {
        const Proj first = eu;
        eu = ev;
        ev = first;
    }
    const Pair a = cross2(eu, warp);
    const Pair b = cross2(offset, warp) + cross2(eu, ev);
    const Pair c = cross2(offset, ev);
    if (a.hi == 0.0f && b.hi == 0.0f && c.hi == 0.0f)
        return best;
    const float dd = comp(d, dominant);
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
    frexpf(fmaxf(fabsf(a.hi), fmaxf(fabsf(b.hi), fabsf(c.hi))), &ce);
    const Pair sa = scaled(a, -ce), sb = scaled(b, -ce), sc = scaled(c, -ce);
    const Pair disc = sb * sb - (sa * sc) * pr(4.0f);
    if (disc.hi < 0.0f)
        return best;
    if (disc.hi == 0.0f) {
        bilinear_root((sb * pr(-0.5f)) / sa, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
        return best;
    }
    const float root = sqrtf(disc.hi);
    const Pair correction = (disc - pr(root) * pr(root)) / pr(2.0f * root);
    const Pair sq = pr(root) + correction;
    const Pair q = (sb + (sb.hi < 0.0f ? -sq : sq)) * pr(-0.5f);
    bilinear_root(q / sa, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
    bilinear_root(sc / q, offset, eu, ev, warp, dd, ray_exponent, t_min, swapped, best);
    return best;
}

// ---------------------------------------------------------------- analytic shapes
// geometry_wire::Analytic (src/geometry_wire.h:31-40)
struct DAnalytic {
    u32 kind, subtype;
    float radius, z_min, z_max, phi_max, inner_radius, height;
};
constexpr u32 kSphere = 1, kDisk = 2, kCylinder = 3;

// shaders/analytic.h:21-25
RP_DEV float analytic_area(const DAnalytic &s) {
    return s.subtype == kDisk ? .5f * s.phi_max * (s.radius - s.inner_radius) * (s.radius + s.inner_radius)
                              : s.phi_max * s.radius * (s.z_max - s.z_min);
}
struct AnalyticSurface {
    V3 position, normal, dpdu, dpdv, dndu, dndv, error;
    bool valid;
};
// The object-space point of parameters (u, v) (evaluate_analytic, shaders/analytic.h:26-64).
RP_DEV AnalyticSurface evaluate_analytic(const DAnalytic &s, float u, float v) {
    const float phi = u * s.phi_max;
    const float c = cosf(phi), sn = sinf(phi), r = s.radius, pm = s.phi_max;
    AnalyticSurface out{};
    if (s.subtype == kDisk) {
        const float radius = fmaf(v, s.inner_radius - r, r);
        out.position = v3(radius * c, radius * sn, s.height);
        out.normal = v3(0, 0, 1);
        const float fr = radius > 0 ? radius : r;
        out.dpdu = v3(-pm * fr * sn, pm * fr * c, 0);
        out.dpdv = v3((s.inner_radius - r) * c, (s.inner_radius - r) * sn, 0);
    } else if (s.subtype == kCylinder) {
        out.position = v3(r * c, r * sn, fmaf(v, s.z_max - s.z_min, s.z_min));
        out.normal = v3(c, sn, 0);
        out.dpdu = v3(-pm * r * sn, pm * r * c, 0);
        out.dpdv = v3(0, 0, s.z_max - s.z_min);
        out.dndu = v3(-pm * sn, pm * c, 0);
    } else if (s.subtype == kSphere) {
        const float t0 = acosf(fminf(fmaxf(s.z_min / r, -1.0f), 1.0f));
        const float t1 = acosf(fminf(fmaxf(s.z_max / r, -1.0f), 1.0f));
        const float dt = t1 - t0, theta = fmaf(v, dt, t0);
        const float st = fmaxf(0.0f, sinf(theta)), ct = cosf(theta);
        out.position = v3(r * st * c, r * st * sn, r * ct);
        out.normal = v3(st * c, st * sn, ct);
        const float fs = fmaxf(st, 1e-7f); // the limiting frame at the poles
        out.dpdu = v3(-pm * r * fs * sn, pm * r * fs * c, 0);
        out.dpdv = v3(dt * r * ct * c, dt * r * ct * sn, -dt * r * st);
        out.dndu = v3(-pm * fs * sn, pm * fs * c, 0);
        out.dndv = v3(dt * ct * c, dt * ct * sn, -dt * st);
    }
    out.error = 0x1p-19f * (vabs(out.position) + v3(s.radius, s.radius, s.radius));
    out.valid = s.subtype >= kSphere && s.subtype <= kCylinder && finite3(out.position) && finite3(out.normal) &&
                finite3(out.dpdu) && finite3(out.dpdv) && finite3(out.dndu) && finite3(out.dndv) && finite3(out.error);
    return out;
}
// The first root in [t_min, t_max] of the object-space ray o + t d on the shape, reprojected
// onto the surface, inside its phi, z and radius bounds (intersect_analytic_if,
// shaders/analytic.h:95-180).
RP_DEV ShapeHit intersect_analytic(const DAnalytic &s, V3 o, V3 d, float t_min, float t_max) {
    const ShapeHit none{false, __int_as_float(0x7f800000), 0.0f, 0.0f};
    float roots[2];
    int count = 0;
    if (s.subtype == kDisk) {
        if (d.z == 0)
            return none;
        roots[count++] = (s.height - o.z) / d.z;
    } else {
        const V3 oo = s.subtype == kSphere ? o : v3(o.x, o.y, 0);
        const V3 dd = s.subtype == kSphere ? d : v3(d.x, d.y, 0);
        const float a = dot(dd, dd);
        if (!(a > 0) || !isfinite(a))
            return none;
        const float b = 2 * dot(oo, dd);
        const float c = fmaf(oo.x, oo.x, fmaf(oo.y, oo.y, oo.z * oo.z)) - s.radius * s.radius;
        const float projection = -dot(oo, dd) / a;
        const V3 closest = fma3(v3(projection, projection, projection), dd, oo);
        const float distance = sqrtf(dot(closest, closest));
        const float disc = 4 * a * (s.radius - distance) * (s.radius + distance);
        if (!(disc >= 0) || !isfinite(disc))
            return none;
        const float q = -.5f * (b + copysignf(sqrtf(disc), b));
        if (q == 0)
            roots[count++] = projection;
        else {
            roots[count++] = q / a;
            roots[count++] = c / q;
            if (roots[0] > roots[1]) {
                const float swap = roots[0];
                roots[0] = roots[1];
                roots[1] = swap;
            }
        }
    }
    for (int i = 0; i < count; ++i) {
        const float t = roots[i];
        if (!isfinite(t) || t < t_min || t > t_max)
            continue;
        V3 p = fma3(v3(t, t, t), d, o);
        if (s.subtype == kSphere) {
            const float length_p = sqrtf(dot(p, p));
            if (!(length_p > 0))
                continue;
            const float k = s.radius / length_p;
            p = v3(p.x * k, p.y * k, p.z * k);
        } else if (s.subtype == kCylinder) {
            const float length_p = sqrtf(p.x * p.x + p.y * p.y);
            if (!(length_p > 0))
                continue;
            const float k = s.radius / length_p;
            p = v3(p.x * k, p.y * k, p.z);
        }
        float phi = atan2f(p.y, p.x);
        if (phi < 0)
            phi += 2 * kPi;
        if (phi > s.phi_max)
            continue;
        float v;
        if (s.subtype == kDisk) {
            const float radius = sqrtf(p.x * p.x + p.y * p.y);
            if (radius < s.inner_radius || radius > s.radius)
                continue;
            v = (s.radius - radius) / (s.radius - s.inner_radius);
        } else if (s.subtype == kSphere) {
            // full-sphere bounds are inactive: reprojection can round a pole just outside them
            if ((s.z_min > -s.radius && p.z < s.z_min) || (s.z_max < s.radius && p.z > s.z_max))
                continue;
            const float t0 = acosf(fminf(fmaxf(s.z_min / s.radius, -1.0f), 1.0f));
            const float t1 = acosf(fminf(fmaxf(s.z_max / s.radius, -1.0f), 1.0f));
            v = (acosf(fminf(fmaxf(p.z / s.radius, -1.0f), 1.0f)) - t0) / (t1 - t0);
        } else {
            if (p.z < s.z_min || p.z > s.z_max)
                continue;
            v = (p.z - s.z_min) / (s.z_max - s.z_min);
        }
        const float uu = fminf(fmaxf(phi / s.phi_max, 0.0f), 1.0f), vv = fminf(fmaxf(v, 0.0f), 1.0f);
        if (isfinite(uu) && isfinite(vv))
            return {true, t, uu, vv};
    }
    return none;
}
// The object-space box of a shape (sphere and cylinder over their z range, disk at its height).
RP_HD void analytic_bounds(const DAnalytic &s, float lo[3], float hi[3]) {
    const float r = s.radius;
    lo[0] = lo[1] = -r;
    hi[0] = hi[1] = r;
    if (s.subtype == kDisk) {
        lo[2] = hi[2] = s.height;
    } else {
        lo[2] = s.subtype == kSphere ? fmaxf(s.z_min, -r) : s.z_min;
        hi[2] = s.subtype == kSphere ? fminf(s.z_max, r) : s.z_max;
    }
}

} // namespace rp
