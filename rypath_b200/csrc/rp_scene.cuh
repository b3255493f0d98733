// Device scene: surface reconstruction, light selection, light geometry sampling and the
// binary LBVH traversal with watertight triangle tests.
#pragma once

#include "rp_image.cuh"
#include "rp_shapes.cuh"

namespace rp {

constexpr u32 kNone = 0xffffffffu;
constexpr u32 kModelPbrt = 0, kModelDemo = 1;
constexpr u32 kLeaf = 0x80000000u;

// wire::Instance subset (src/render_wire.h:168-188), plus the first emitter slot
struct DInstance {
    float m[12];
    u32 vertex_begin, triangle_begin, triangle_count, material, reverse, emission, normal_begin, emitter_begin;
    u32 inside_medium, outside_medium; // kNone = vacuum
    u32 resolve;                       // kPassThrough | kMixRoot: hits resolve before shading
    u32 patch_begin, patch_count, analytic_begin, analytic_count; // procedural primitives
};
constexpr u32 kMixScattering = 9, kInterfaceScattering = 10;
// DInstance::resolve bits: the hero transport passes through the instance (an invisible
// emitter or a null-interface root material), or its root material is a mix.
constexpr u32 kPassThrough = 1, kMixRoot = 2;
// tri_family of triangles whose hits resolve in the closest-hit kernel before binning
constexpr u32 kResolveFamily = 4;
// wire::Material subset (src/render_wire.h:107-130)
struct DMaterial {
    u32 scattering, kind, knot_begin, knot_count;
    float scalar_value;
    u32 eta_begin, eta_count, k_begin, k_count, optical_extensions;
    float u_roughness, v_roughness;
    u32 remap;
    u32 first, second; // mix children
    float mix_amount;
    u32 image_texture; // image reflectance (kind 3)
    float coefficients[3]; // RGB sigmoid reflectance (kind 2)
    float reflectance[8];  // demo-model sampled reflectance at the demo knots
};
struct DPositional {
    float position[3];
    u32 kind;
    float light_from_world[9];
    float cos_falloff_start, cos_falloff_end;
    u32 spectrum; // offset of the 471-bin intensity in the spectra buffer
};
// wire::LightBounds / LightAlias / LightRecord (src/render_wire.h:227-244)
struct DLightBounds {
    float low[3], high[3], direction[3];
    float power, cos_outer, cos_emission;
    u32 child, parent, light, flags;
    // per-node terms of light_importance, computed on the host with the same float operations
    float center[3]; // (low + high) * 0.5
    float r2;        // |high - low|^2 / 4
    float radius;    // sqrt(r2)
    float sin_outer; // sqrt(max(0, 1 - cos_outer^2))
};
static_assert(offsetof(DLightBounds, center) == 64, "the first 16 words are LightBounds");
struct DLightAlias {
    float threshold, pmf;
    u32 alias, padding;
};
struct DLightRecord {
    u32 leaf, flags, padding0, padding1;
};
// Binary BVH node: both child boxes and both child links (64 bytes).
struct __align__(16) BNode {
    float4 a; // left lo.xyz, left hi.x
    float4 b; // left hi.yz, right lo.xy
    float4 c; // right lo.z, right hi.xyz
    uint4 d;  // left, right, unused, unused
};

// Compressed 8-wide BVH node (80 bytes).  Child k's box is bounded per axis by the planes
// p + q 2^e of its 8-bit lo and hi bytes q (the builder widens q until the planes, in real
// arithmetic, enclose the child's box).  Internal children are stored
// contiguously from child_base and leaf triangles from tri_base, each in slot order; slot bit a
// is set when the child's centre lies on the positive side of the node's centre along axis a,
// so a ray visits hit children in the order slot ^ (its direction's negative-axis bits): near
// side first.
struct __align__(16) WNode {
    float4 origin;  // p.x, p.y, p.z; w bits: biased exponents e.x, e.y, e.z (bytes 0-2), internal mask (byte 3)
    uint4 links;    // child_base, tri_base, leaf mask, unused
    uint4 q0;       // lo.x[0..7], lo.y[0..7]
    uint4 q1;       // lo.z[0..7], hi.x[0..7]
    uint4 q2;       // hi.y[0..7], hi.z[0..7]
};

struct DeviceScene {
    const float *positions;
    const float *normals;
    u32 normal_count;
    const u32 *triangles;
    const DInstance *instances;
    u32 instance_count;
    const u32 *tri_instance; // per flattened triangle
    const u32 *tri_local;
    u32 prim_count;
    const BNode *nodes;
    const float4 *leaf_v; // 3 per leaf slot: world v0 (w = prim id bits), v1, v2
    const WNode *wnodes;  // traversal tree (root 0)
    const float4 *wtri;   // 3 per wide leaf, in the wide nodes' tri_base order
    u32 wnode_count;
    const unsigned char *tri_family; // BSDF family of each triangle's material
    const DMaterial *materials;
    u32 material_count;
    const float2 *knots;
    u32 knot_count;
    const float *spectra; // emissions (471 each), positional intensities, environment
    const u32 *emission_two_sided;
    u32 emission_count;
    const DPositional *positional;
    u32 positional_count;
    u32 environment; // offset of the environment spectrum or kNone
    const u32 *emitter_instance;
    const u32 *emitter_local;
    u32 emitter_count;
    const DLightBounds *light_nodes;
    const DLightAlias *light_alias;
    const DLightRecord *light_records;
    const u32 *infinite_lights;
    u32 light_node_count, infinite_count, light_count, light_sampler, environment_light;
    float scene_radius;
    SobolTables sobol;
    V3 origin, forward, right, up;
    u32 filter_kind;
    float filter_x, filter_y;
    u32 max_depth, hero_mode;
    float slab_scale; // 1 + 2 gamma(3), the conservative far-plane factor
    // homogeneous media (scalar transport): kMediumStride floats each -- sigma_a[471],
    // sigma_s[471], emission[471], g
    const float *media;
    u32 medium_count, camera_medium;
    u32 media_enabled; // any medium or null interface: shadow connections track media
    // thin lens (lens_radius 0: pinhole)
    float lens_radius, focal_distance;
    V3 lens_x, lens_y;
    // Gaussian filter: tabulated CDFs (gauss_h rows of gauss_w + 1, then the marginal of
    // gauss_h + 1) and the packet film weight (the table's integral; 1 for other filters)
    const float *gauss_cdf;
    u32 gauss_w, gauss_h;
    float filter_weight;
    const u32 *primes; // the first 1000 primes (Halton bases)
    DImages img;       // image textures and the environment image (env_image kNone: none)
    u32 model;         // kModelPbrt or kModelDemo (RenderModel)
    float film_scale;  // demo camera: tan(vertical fov / 2)
    // procedural primitives: flattened primitives [0, tri_prims) are triangles, the next
    // patch_prims bilinear patches, the rest analytic shapes; tri_local holds the index within
    // the instance's primitives of that kind
    u32 tri_prims, patch_prims;
    const u32 *patches;        // 4 vertex indices each (p00 p10 p01 p11), instance-local
    const DAnalytic *analytics;
    const float *inverse;      // per instance: world-to-object 3x4, row-major
};

RP_DEV V3 load3(const float *p) { return v3(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }
RP_DEV float spectrum(const DeviceScene &s, u32 offset, float w) { return __ldg(s.spectra + offset + dense_index(w)); }

// shaders/light_geometry_sampling.h:10-15
RP_DEV V3 world_point(const DInstance &in, V3 p) {
    return v3(dot(v3(in.m[0], in.m[1], in.m[2]), p), dot(v3(in.m[4], in.m[5], in.m[6]), p),
              dot(v3(in.m[8], in.m[9], in.m[10]), p)) +
           v3(in.m[3], in.m[7], in.m[11]);
}

// SurfacePoint subset (shaders/render.metal:870-881)
struct SurfacePoint {
    V3 position, error, geometric_normal, shading_normal;
    float inverse_area_pdf;
    float world_extent;
    bool curved; // a patch or analytic point: ray positions carry their rounding in float pairs
};
// shaders/render.metal:865-868
RP_DEV float triangle_extent(V3 e1, V3 e2) {
    const V3 a = vabs(e1), b = vabs(e2), c = vabs(e2 - e1);
    return fmaxf(fmaxf(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y))), fmaxf(a.z, fmaxf(b.z, c.z)));
}
// shaders/render.metal:885-968 (triangle_surface_point)
__device__ __noinline__ bool triangle_surface_point(const DeviceScene &s, u32 instance, u32 local, float u, float v, bool native_hit,
                                   SurfacePoint &point) {
    const DInstance &in = s.instances[instance];
    const u32 *tri = s.triangles + 3 * (in.triangle_begin + local);
    const u32 i0 = __ldg(tri), i1 = __ldg(tri + 1), i2 = __ldg(tri + 2);
    const V3 p0 = load3(s.positions + 3 * (in.vertex_begin + i0));
    const V3 p1 = load3(s.positions + 3 * (in.vertex_begin + i1));
    const V3 p2 = load3(s.positions + 3 * (in.vertex_begin + i2));
    const V3 ax = v3(in.m[0], in.m[1], in.m[2]), ay = v3(in.m[4], in.m[5], in.m[6]), az = v3(in.m[8], in.m[9], in.m[10]);
    const V3 shift = v3(in.m[3], in.m[7], in.m[11]);
    const V3 e1 = p1 - p0, e2 = p2 - p0;
    const V3 we1 = v3(dot(ax, e1), dot(ay, e1), dot(az, e1));
    const V3 we2 = v3(dot(ax, e2), dot(ay, e2), dot(az, e2));
    const V3 ce = cross(we1, we2);
    const float n2 = dot(ce, ce);
    point.curved = false;
    if (n2 == 0.0f && !native_hit) {
        point.position = point.error = point.geometric_normal = point.shading_normal = v3(0, 0, 0);
        point.inverse_area_pdf = 0;
        point.world_extent = 0;
        return true;
    }
    if (!(n2 > 0.0f) || !isfinite(n2))
        return false;
    const float nl = sqrtf(n2);
    point.inverse_area_pdf = 0.5f * nl;
    point.world_extent = triangle_extent(we1, we2);
    point.geometric_normal = ce / nl;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    if (in.normal_begin != kNone) {
        const u32 begin = in.normal_begin, nc = s.normal_count;
        if (begin >= nc || i0 >= nc - begin || i1 >= nc - begin || i2 >= nc - begin)
            return false;
        const V3 n0 = load3(s.normals + 3 * (begin + i0)), n1 = load3(s.normals + 3 * (begin + i1)),
                 n2v = load3(s.normals + 3 * (begin + i2));
        const V3 interp = (1.0f - (u + v)) * n0 + u * n1 + v * n2v;
        if (!finite3(interp))
            return false;
        const float scale = max3(vabs(interp));
        if (scale > 0.0f) {
            const V3 scaled = interp / scale;
            point.shading_normal = normalize3(scaled);
            if (dot(point.geometric_normal, scaled) < 0.0f)
                point.geometric_normal = -point.geometric_normal;
        }
    }
    const V3 lp = p0 + (u * e1 + v * e2);
    point.position = v3(dot(ax, lp), dot(ay, lp), dot(az, lp)) + shift;
    V3 local_error = gamma_bound(7.0f) * (vabs(p0) + vabs(u * e1) + vabs(v * e2));
    if (native_hit) {
        const float allowance = 64.0f * 0x1.0p-23f;
        const float traversal = gamma_bound(7.0f) * triangle_extent(e1, e2);
        local_error = (local_error + allowance * (vabs(e1) + vabs(e2))) + v3(traversal, traversal, traversal);
    }
    const V3 ein = local_error + gamma_bound(4.0f) * vabs(lp);
    point.error = v3(dot(vabs(ax), ein), dot(vabs(ay), ein), dot(vabs(az), ein)) + gamma_bound(4.0f) * vabs(shift);
    return finite3(point.position) && finite3(point.error) && finite3(point.geometric_normal) &&
           finite3(point.shading_normal);
}

// shaders/render.metal:970-1062 (patch_surface_point): the parametric point, the normal of the
// world-space partials, vertex normals interpolated bilinearly, the position in float pairs
// with its retained roundoff.
__device__ __noinline__ bool patch_surface_point(const DeviceScene &s, u32 instance, u32 local, float u, float v,
                                                 SurfacePoint &point) {
    const DInstance &in = s.instances[instance];
    point.curved = true;
    const u32 *pt = s.patches + 4 * size_t(in.patch_begin + local);
    u32 idx[4];
    V3 p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        idx[i] = __ldg(pt + i);
        p[i] = load3(s.positions + 3 * size_t(in.vertex_begin + idx[i]));
    }
    const V3 ax = v3(in.m[0], in.m[1], in.m[2]), ay = v3(in.m[4], in.m[5], in.m[6]), az = v3(in.m[8], in.m[9], in.m[10]);
    const V3 e10 = p[1] - p[0], e32 = p[3] - p[2], e20 = p[2] - p[0], e31 = p[3] - p[1];
    const V3 du = e10 + (e32 - e10) * v, dv = e20 + (e31 - e20) * u;
    const V3 wu = v3(dot(ax, du), dot(ay, du), dot(az, du)), wv = v3(dot(ax, dv), dot(ay, dv), dot(az, dv));
    const V3 c = cross(wu, wv);
    const float squared = dot(c, c);
    if (!(squared >= kFltMin) || !isfinite(squared))
        return false;
    point.inverse_area_pdf = sqrtf(squared);
    point.geometric_normal = c / point.inverse_area_pdf;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    if (in.normal_begin != kNone) {
        V3 n[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (in.normal_begin >= s.normal_count || idx[i] >= s.normal_count - in.normal_begin)
                return false;
            n[i] = load3(s.normals + 3 * size_t(in.normal_begin + idx[i]));
        }
        const V3 a = n[0] + (n[2] - n[0]) * v, b = n[1] + (n[3] - n[1]) * v;
        const V3 interp = a + (b - a) * u;
        if (!finite3(interp))
            return false;
        const float scale = max3(vabs(interp));
        if (scale > 0) {
            const V3 sc = interp / scale;
            point.shading_normal = normalize3(sc);
            if (dot(point.geometric_normal, sc) < 0)
                point.geometric_normal = -point.geometric_normal;
        }
    }
    Pair local_p[3];
    const V3 magnitude = ((vabs(p[0]) + vabs(p[1])) + vabs(p[2])) + vabs(p[3]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const Pair lo = pr(comp(p[0], a)) + (pr(comp(p[2], a)) - pr(comp(p[0], a))) * pr(v);
        const Pair hi = pr(comp(p[1], a)) + (pr(comp(p[3], a)) - pr(comp(p[1], a))) * pr(v);
        local_p[a] = lo + (hi - lo) * pr(u);
    }
    const bool identity = in.m[3] == 0 && in.m[7] == 0 && in.m[11] == 0 && in.m[0] == 1 && in.m[1] == 0 &&
                          in.m[2] == 0 && in.m[4] == 0 && in.m[5] == 1 && in.m[6] == 0 && in.m[8] == 0 &&
                          in.m[9] == 0 && in.m[10] == 1;
    float pos[3], err[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Pair world = pr(in.m[4 * a + 3]);
        float bound = fabsf(in.m[4 * a + 3]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            world = world + local_p[j] * pr(in.m[4 * a + j]);
            bound += comp(magnitude, j) * fabsf(in.m[4 * a + j]);
        }
        pos[a] = world.hi;
        const float traversal = identity ? 0.0f : 0x1p-20f * bound;
        err[a] = ((fabsf(world.lo) + 0x1p-40f * bound) + traversal) + 128.0f * kFltMin;
    }
    point.position = v3(pos[0], pos[1], pos[2]);
    point.error = v3(err[0], err[1], err[2]);
    point.world_extent = 0;
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        const V3 e = p[i] - p[0];
        const V3 w = vabs(v3(dot(ax, e), dot(ay, e), dot(az, e)));
        point.world_extent = fmaxf(point.world_extent, fmaxf(w.x, fmaxf(w.y, w.z)));
    }
    return finite3(point.position) && finite3(point.error) && finite3(point.geometric_normal) &&
           finite3(point.shading_normal);
}
// shaders/analytic.h:81-85 (analytic_stable_length)
RP_DEV float stable_length(V3 v) {
    const float scale = fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z)));
    return scale > 0 ? scale * length3(v / scale) : 0;
}
// shaders/render.metal:1080-1118 (analytic_surface_point): the shape's point moved to world
// space, its normal by the cofactor matrix, the area density scaled by the transform.
__device__ __noinline__ bool analytic_surface_point(const DeviceScene &s, u32 instance, u32 local, float u, float v,
                                                    SurfacePoint &point) {
    const DInstance &in = s.instances[instance];
    point.curved = true;
    if (local >= in.analytic_count)
        return false;
    const DAnalytic rec = s.analytics[in.analytic_begin + local];
    const AnalyticSurface ls = evaluate_analytic(rec, u, v);
    if (!ls.valid)
        return false;
    const V3 a = v3(in.m[0], in.m[1], in.m[2]), b = v3(in.m[4], in.m[5], in.m[6]), c = v3(in.m[8], in.m[9], in.m[10]);
    const V3 cofactor = v3(dot(cross(b, c), ls.normal), dot(cross(c, a), ls.normal), dot(cross(a, b), ls.normal));
    const float jacobian = stable_length(cofactor);
    if (!(jacobian > 0) || !isfinite(jacobian))
        return false;
    point.geometric_normal = cofactor / jacobian;
    if (in.reverse)
        point.geometric_normal = -point.geometric_normal;
    point.shading_normal = point.geometric_normal;
    const V3 shift = v3(in.m[3], in.m[7], in.m[11]);
    point.position = v3(dot(a, ls.position), dot(b, ls.position), dot(c, ls.position)) + shift;
    point.error = v3(dot(vabs(a), ls.error), dot(vabs(b), ls.error), dot(vabs(c), ls.error)) +
                  gamma_bound(5) * (vabs(point.position) + vabs(shift));
    point.inverse_area_pdf = analytic_area(rec) * jacobian;
    point.world_extent = 2 * rec.radius * fmaxf(length3(a), fmaxf(length3(b), length3(c)));
    return finite3(point.position) && finite3(point.error) && isfinite(point.inverse_area_pdf) &&
           point.inverse_area_pdf >= kFltMin;
}
// surface_point (shaders/render.metal:1120-1132) of flattened primitive `prim` of `instance`
// (its `local` primitive of that kind) at the hit's coordinates.
RP_DEV bool hit_surface_point(const DeviceScene &s, u32 prim, u32 instance, u32 local, float b1, float b2,
                              SurfacePoint &point) {
    if (prim < s.tri_prims)
        return triangle_surface_point(s, instance, local, b1, b2, true, point);
    if (prim - s.tri_prims < s.patch_prims)
        return patch_surface_point(s, instance, local, b1, b2, point);
    return analytic_surface_point(s, instance, local, b1, b2, point);
}
// The float-pair ray point at a patch or analytic point (out of line: triangle hits, the
// common case, do not carry its code).
__device__ __noinline__ void curved_ray_point(V3 o, V3 d, float t, V3 &position, V3 &error) {
    float p[3], e[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const Pair value = pr(t) * pr(comp(d, a)) + pr(comp(o, a));
        p[a] = value.hi;
        e[a] = (fabsf(value.lo) + 0x1p-40f * (fabsf(t * comp(d, a)) + fabsf(comp(o, a)))) + 128.0f * kFltMin;
    }
    position = v3(p[0], p[1], p[2]);
    error = v3(e[0], e[1], e[2]);
}
// The ray's point at t and the rounding that bounds it (shaders/render.metal:1913-1929): in
// plain float at triangles, in float pairs at patch and analytic points.
RP_DEV void ray_point(V3 o, V3 d, float t, bool curved, V3 &position, V3 &error) {
    if (curved) {
        curved_ray_point(o, d, t, position, error);
        return;
    }
    position = fma3(v3(t, t, t), d, o);
    error = gamma_bound(2.0f) * (vabs(t * d) + vabs(o));
}
// The world ray in the object space of an instance (world-to-object 3x4 `w`): the same t.
RP_DEV void object_ray(const float *w, V3 o, V3 d, V3 &oo, V3 &od) {
    const V3 r0 = v3(__ldg(w), __ldg(w + 1), __ldg(w + 2)), r1 = v3(__ldg(w + 4), __ldg(w + 5), __ldg(w + 6)),
             r2 = v3(__ldg(w + 8), __ldg(w + 9), __ldg(w + 10));
    oo = v3(dot(r0, o), dot(r1, o), dot(r2, o)) + v3(__ldg(w + 3), __ldg(w + 7), __ldg(w + 11));
    od = v3(dot(r0, d), dot(r1, d), dot(r2, d));
}
// The hit of the world ray o + t d, t in [0, tmax], on procedural primitive `prim`.
__device__ __noinline__ ShapeHit procedural_hit(const DeviceScene &s, u32 prim, V3 o, V3 d, float tmax) {
    const u32 inst = __ldg(s.tri_instance + prim), local = __ldg(s.tri_local + prim);
    const DInstance &in = s.instances[inst];
    V3 oo, od;
    object_ray(s.inverse + 12 * size_t(inst), o, d, oo, od);
    if (prim - s.tri_prims < s.patch_prims) {
        const u32 *pt = s.patches + 4 * size_t(in.patch_begin + local);
        V3 p[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            p[i] = load3(s.positions + 3 * size_t(in.vertex_begin + __ldg(pt + i)));
        return intersect_bilinear(p[0], p[1], p[2], p[3], oo, od, 0.0f, tmax);
    }
    return intersect_analytic(s.analytics[in.analytic_begin + local], oo, od, 0.0f, tmax);
}

// PBRT's alpha hash (MurmurHash64A over the binary32 words of origin, direction and t;
// shaders/alpha_hash.h:10-36) as a uniform in [0, 1).  t arrives as its bit pattern.
RP_DEV float alpha_uniform(V3 o, V3 d, u32 t_bits) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    const u32 w[6] = {__float_as_uint(o.x), __float_as_uint(o.y), __float_as_uint(o.z),
                      __float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z)};
    u64 h = 28ull * m;
#pragma unroll
    for (int i = 0; i < 6; i += 2) {
        u64 k = u64(w[i]) | (u64(w[i + 1]) << 32);
        k *= m;
        k ^= k >> 47;
        k *= m;
        h ^= k;
        h *= m;
    }
    h ^= u64(t_bits);
    h *= m;
    h ^= h >> 47;
    h *= m;
    h ^= h >> 47;
    return float(u32(h)) * 0x1p-32f;
}
// The material a hit on mix root `material` resolves to (shaders/packet_pt_event_body.inc:
// 165-190): at each mix node, second where the alpha hash of (position, -direction, node
// index) is below the amount, else first.  Returns the sample status: 0, 2 (a 65th level
// or a non-finite amount) or 3 (a child out of range).
RP_DEV u32 resolve_mix(const DeviceScene &s, V3 position, V3 toward_origin, u32 &material) {
    for (u32 depth = 0; depth <= 64; ++depth) {
        const DMaterial &node = s.materials[material];
        if (node.scattering != kMixScattering)
            return 0;
        const float amount = node.mix_amount;
        if (depth == 64 || !isfinite(amount))
            return 2;
        const float selector = alpha_uniform(position, toward_origin, material);
        material = amount <= 0 ? node.first : amount >= 1 ? node.second : selector < amount ? node.second : node.first;
        if (material >= s.material_count)
            return 3;
    }
    return 0;
}

// ------------------------------------------------------------------ light selection (shaders/light_sampling.h)
// :19-42
// Point-light nodes (r2 == 0) take the bound angle's closed form: cos = 1 (or -1 at the light,
// 0 for a NaN distance, as 1 - 0 / d2 gives), sin = 0 (1 when cos is 0).
RP_DEV float light_importance(const DLightBounds &b, V3 position, V3 normal) {
    const V3 center = v3(b.center[0], b.center[1], b.center[2]);
    const V3 delta = position - center;
    const float r2 = b.r2, d2 = dot(delta, delta);
    const float radius = b.radius, distance = sqrtf(d2);
    float cb, sb;
    if (r2 == 0) {
        cb = d2 <= 0 ? -1.f : (d2 == d2 ? 1.f : 0.f);
        sb = cb == 0 ? 1.f : 0.f;
    } else {
        cb = d2 <= r2 ? -1.f : sqrtf(fmaxf(0.f, 1 - r2 / d2));
        sb = sqrtf(fmaxf(0.f, 1 - cb * cb));
    }
    const V3 wi = distance > 0 ? delta / distance : v3(0, 0, 1);
    float cw = fminf(fmaxf(dot(v3(b.direction[0], b.direction[1], b.direction[2]), wi), -1.f), 1.f);
    if (b.flags & 1)
        cw = fabsf(cw);
    const float sw = sqrtf(fmaxf(0.f, 1 - cw * cw)), co = b.cos_outer, so = b.sin_outer;
    const float cx = cw > co ? 1.f : cw * co + sw * so, sx = cw > co ? 0.f : sw * co - cw * so;
    const float cp = cx > cb ? 1.f : cx * cb + sx * sb;
    if (cp <= b.cos_emission)
        return 0;
    float value = b.power * cp / fmaxf(d2, fmaxf(radius, kFltMin));
    if (nonzero3(normal)) {
        const float ci = fminf(fmaxf(fabsf(dot(wi, normal)), 0.f), 1.f);
        const float si = sqrtf(fmaxf(0.f, 1 - ci * ci));
        value *= ci > cb ? 1.f : ci * cb + si * sb;
    }
    return fmaxf(0.f, value);
}
struct Selected {
    u32 light;
    float pmf;
};
// :43-95
__device__ __noinline__ Selected light_sample(const DeviceScene &s, V3 position, V3 normal, float u) {
    const u32 count = s.light_count;
    if (!count)
        return {kNone, 0};
    u = fminf(fmaxf(u, 0.f), kOneMinusEps);
    if (s.light_sampler == 2) {
        const u32 id = min(u32(u * count), count - 1);
        return {id, 1.f / count};
    }
    if (s.light_sampler == 1) {
        const float v = u * count;
        const u32 i = min(u32(v), count - 1);
        const u32 id = v - i < s.light_alias[i].threshold ? i : s.light_alias[i].alias;
        return {id, s.light_alias[id].pmf};
    }
    const u32 ninf = s.infinite_count, nodes = s.light_node_count;
    const float infinite = float(ninf) / float(ninf + (nodes ? 1 : 0));
    if (u < infinite) {
        const u32 i = min(u32((u / infinite) * ninf), ninf - 1);
        return {s.infinite_lights[i], 1.f / float(ninf + (nodes ? 1 : 0))};
    }
    if (!nodes)
        return {kNone, 0};
    u = fminf((u - infinite) / (1 - infinite), kOneMinusEps);
    float pmf = 1 - infinite;
    u32 i = 0;
    float reached = 0; // importance of node i, once a parent has computed it
    for (u32 steps = 0; steps < nodes; ++steps) {
        const DLightBounds &node = s.light_nodes[i];
        if (node.light != kNone) {
            if ((steps == 0 ? light_importance(node, position, normal) : reached) <= 0)
                return {kNone, 0};
            return {node.light, pmf};
        }
        const float a = light_importance(s.light_nodes[i + 1], position, normal),
                    b = light_importance(s.light_nodes[node.child], position, normal), sum = a + b;
        if (!(sum > 0))
            return {kNone, 0};
        const float q = a / sum;
        if (u < q) {
            pmf *= q;
            u = fminf(u / q, kOneMinusEps);
            i++;
            reached = a;
        } else {
            pmf *= 1 - q;
            u = fminf((u - q) / (1 - q), kOneMinusEps);
            i = node.child;
            reached = b;
        }
    }
    return {kNone, 0};
}
// :96-126
__device__ __noinline__ float light_pmf(const DeviceScene &s, V3 position, V3 normal, u32 id) {
    if (id >= s.light_count)
        return 0;
    if (s.light_sampler == 2)
        return 1.f / s.light_count;
    if (s.light_sampler == 1)
        return s.light_alias[id].pmf;
    const u32 ninf = s.infinite_count, nodes = s.light_node_count;
    if (s.light_records[id].flags & 1)
        return 1.f / float(ninf + (nodes ? 1 : 0));
    u32 i = s.light_records[id].leaf;
    if (i >= nodes)
        return 0;
    if (light_importance(s.light_nodes[i], position, normal) <= 0)
        return 0;
    float result = 1.f - float(ninf) / float(ninf + (nodes ? 1 : 0));
    for (u32 steps = 0; steps < nodes; ++steps) {
        const u32 parent = s.light_nodes[i].parent;
        if (parent == kNone)
            return result;
        const float a = light_importance(s.light_nodes[parent + 1], position, normal),
                    b = light_importance(s.light_nodes[s.light_nodes[parent].child], position, normal), sum = a + b;
        if (!(sum > 0))
            return 0;
        result *= i == parent + 1 ? a / sum : b / sum;
        i = parent;
    }
    return 0;
}

// ------------------------------------------------------------------ light geometry (src/light_geometry_sampling_shared.h)
RP_DEV float clamp01(float v) { return fminf(1.f, fmaxf(0.f, v)); }
RP_DEV float safe_sqrt(float v) { return sqrtf(fmaxf(0.f, v)); }
RP_DEV V3 unitv(V3 v) { return v / length3(v); }
RP_DEV bool nonzero_len(V3 v) { return dot(v, v) > 0; }
// :74-77
RP_DEV float sph_angle(V3 a, V3 b) {
    return dot(a, b) < 0 ? kPi - 2 * asinf(fminf(1.f, length3(a + b) / 2)) : 2 * asinf(fminf(1.f, length3(a - b) / 2));
}
// :78-85
RP_DEV float sph_triangle_area(V3 a, V3 b, V3 c) {
    return fabsf(2 * atan2f(dot(a, cross(b, c)), 1 + dot(a, b) + dot(a, c) + dot(b, c)));
}
RP_DEV float triangle_solid_angle(V3 p0, V3 p1, V3 p2, V3 r) {
    if (!nonzero_len(p0 - r) || !nonzero_len(p1 - r) || !nonzero_len(p2 - r))
        return 0;
    return sph_triangle_area(unitv(p0 - r), unitv(p1 - r), unitv(p2 - r));
}
struct W4 {
    float a, b, c, d;
};
// :91-115
RP_DEV W4 normalized_weights(W4 w) {
    const float s = fmaxf(fmaxf(w.a, w.b), fmaxf(w.c, w.d));
    return s > 0 ? W4{w.a / s, w.b / s, w.c / s, w.d / s} : W4{1, 1, 1, 1};
}
RP_DEV float linear_sample(float u, float a, float b) {
    if (u == 0 && a == 0)
        return 0;
    return fminf(kOneMinusEps, u * (a + b) / (a + sqrtf((1 - u) * a * a + u * b * b)));
}
RP_DEV float bilinear_pdf(float ux, float uy, W4 weights) {
    if (ux < 0 || ux > 1 || uy < 0 || uy > 1)
        return 0;
    const W4 w = normalized_weights(weights);
    return 4 * ((1 - ux) * (1 - uy) * w.a + ux * (1 - uy) * w.b + (1 - ux) * uy * w.c + ux * uy * w.d) /
           (w.a + w.b + w.c + w.d);
}
// :116-121
RP_DEV W4 triangle_cosines(V3 a, V3 b, V3 c, V3 r, V3 n) {
    const float wa = fmaxf(.01f, fabsf(dot(n, unitv(a - r))));
    const float wb = fmaxf(.01f, fabsf(dot(n, unitv(b - r))));
    const float wc = fmaxf(.01f, fabsf(dot(n, unitv(c - r))));
    return {wb, wb, wa, wc};
}
// :128-172 (PBRT SampleSphericalTriangle, rationalised)
RP_DEV bool sph_triangle_sample(V3 p0, V3 p1, V3 p2, V3 r, float ux, float uy, float &b1o, float &b2o) {
    const V3 a = unitv(p0 - r), b = unitv(p1 - r), c = unitv(p2 - r);
    const V3 nab = cross(a, b), nca = cross(c, a);
    if (!nonzero_len(nab) || !nonzero_len(nca))
        return false;
    const float alpha = sph_angle(unitv(nab), -unitv(nca));
    const float area = sph_triangle_area(a, b, c);
    const float ca = cosf(alpha), sa = sinf(alpha);
    const float subarea = ux * area;
    const float sh = sinf(subarea / 2), st = sinf(subarea), ct_area = cosf(subarea);
    const float one_minus_ct = 2 * sh * sh;
    const float sp = sa * ct_area - ca * st;
    const float cp = -ca * ct_area - sa * st;
    const float k1 = -2 * sinf(alpha - subarea / 2) * sh;
    const float k2 = sa * (.5f * dot(a - b, a - b) - one_minus_ct) - ca * st;
    const float divisor = (k2 * sp + k1 * cp) * sa;
    if (divisor == 0)
        return false;
    const float omc = fminf(2.f, fmaxf(0.f, (-k2 * one_minus_ct - k1 * st) / divisor));
    const float cosbp = 1 - omc;
    const V3 arc = c - dot(c, a) * a;
    if (!nonzero_len(arc))
        return false;
    const V3 cprime = cosbp * a + safe_sqrt(omc * (2 - omc)) * unitv(arc);
    const float omct = uy * .5f * dot(cprime - b, cprime - b);
    const float ct = 1 - omct;
    const V3 tangent = cprime - dot(cprime, b) * b;
    if (!nonzero_len(tangent))
        return false;
    const V3 direction = ct * b + safe_sqrt(omct * (2 - omct)) * unitv(tangent);
    const V3 e1 = p1 - p0, e2 = p2 - p0, s1 = cross(direction, e2);
    const float denom = dot(s1, e1);
    if (denom == 0)
        return false;
    const V3 sv = r - p0;
    float b1 = clamp01(dot(sv, s1) / denom), b2 = clamp01(dot(direction, cross(sv, e1)) / denom);
    if (b1 + b2 > 1) {
        const float sum = b1 + b2;
        b1 /= sum;
        b2 /= sum;
    }
    b1o = b1;
    b2o = b2;
    return isfinite(b1) && isfinite(b2);
}
// :174-182
RP_DEV void sph_triangle_inverse(V3 p0, V3 p1, V3 p2, V3 r, V3 dir, float &u0, float &u1) {
    const V3 a = unitv(p0 - r), b = unitv(p1 - r), c = unitv(p2 - r);
    V3 cp = unitv(cross(cross(b, dir), cross(c, a)));
    if (dot(cp, a + c) < 0)
        cp = -cp;
    u0 = clamp01(sph_triangle_area(a, b, cp) / sph_triangle_area(a, b, c));
    u1 = clamp01(dot(dir - b, dir - b) / dot(cp - b, cp - b));
}
// shaders/light_geometry_sampling.h:16-29
RP_DEV void emitter_corners(const DeviceScene &s, u32 emitter, V3 p[3]) {
    const DInstance &in = s.instances[s.emitter_instance[emitter]];
    const u32 *tri = s.triangles + 3 * (in.triangle_begin + s.emitter_local[emitter]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        p[i] = world_point(in, load3(s.positions + 3 * (in.vertex_begin + __ldg(tri + i))));
}
// shaders/light_geometry_sampling.h:58-67
RP_DEV float area_solid_angle_pdf(float area_density, V3 reference, const SurfacePoint &point) {
    const V3 delta = point.position - reference;
    const float d2 = dot(delta, delta);
    if (!(d2 > 0) || !(area_density > 0))
        return 0;
    const float cosine = fabsf(dot(point.geometric_normal, delta * (1.0f / sqrtf(d2))));
    return cosine > 0 ? area_density * d2 / cosine : 0;
}
// shaders/light_geometry_sampling.h:116-153 (triangles)
__device__ __noinline__ float light_geometry_pdf(const DeviceScene &s, u32 emitter, V3 reference, V3 normal, const SurfacePoint &point) {
    const V3 delta = point.position - reference;
    if (!(dot(delta, delta) > 0) || !(point.inverse_area_pdf > 0))
        return 0;
    V3 p[3];
    emitter_corners(s, emitter, p);
    const float area = triangle_solid_angle(p[0], p[1], p[2], reference);
    if (area >= 3e-4f && area <= 6.22f) {
        float u0, u1;
        sph_triangle_inverse(p[0], p[1], p[2], reference, normalize3(delta), u0, u1);
        return (dot(normal, normal) > 0 ? bilinear_pdf(u0, u1, triangle_cosines(p[0], p[1], p[2], reference, normal))
                                        : 1.f) /
               area;
    }
    return area_solid_angle_pdf(1 / point.inverse_area_pdf, reference, point);
}
// shaders/light_geometry_sampling.h:155-209 (triangles)
__device__ __noinline__ bool light_geometry_sample(const DeviceScene &s, u32 emitter, V3 reference, V3 normal, float ux, float uy,
                                  SurfacePoint &point, float &pdf) {
    if (!isfinite(ux) || !isfinite(uy) || ux < 0 || uy < 0 || ux > 1 || uy > 1)
        return false;
    ux = fminf(ux, kOneMinusEps);
    uy = fminf(uy, kOneMinusEps);
    V3 p[3];
    emitter_corners(s, emitter, p);
    float b1, b2;
    const float area = triangle_solid_angle(p[0], p[1], p[2], reference);
    if (area >= 3e-4f && area <= 6.22f) {
        if (dot(normal, normal) > 0) {
            const W4 w = normalized_weights(triangle_cosines(p[0], p[1], p[2], reference, normal));
            const float y = linear_sample(uy, w.a + w.b, w.c + w.d);
            const float x = linear_sample(ux, (1 - y) * w.a + y * w.c, (1 - y) * w.b + y * w.d);
            ux = x;
            uy = y;
        }
        if (!sph_triangle_sample(p[0], p[1], p[2], reference, ux, uy, b1, b2))
            return false;
    } else {
        const float root = sqrtf(ux);
        b1 = 1 - root;
        b2 = uy * root;
    }
    if (!isfinite(b1) || !isfinite(b2) ||
        !triangle_surface_point(s, s.emitter_instance[emitter], s.emitter_local[emitter], b1, b2, false, point))
        return false;
    pdf = light_geometry_pdf(s, emitter, reference, normal, point);
    return isfinite(pdf) && pdf >= 0;
}

// ------------------------------------------------------------------ positional lights (shaders/render.metal:654-811)
RP_DEV bool normal_or_zero(float v) {
    const u32 m = fbits(v) & 0x7fffffffu;
    return m == 0 || (m >= 0x00800000u && m < 0x7f800000u);
}
RP_DEV bool spot_product(float a, float b, float &r) {
    if (a != 0 && b != 0 && fabsf(a) < kFltMin / fabsf(b))
        return false;
    r = a * b;
    return normal_or_zero(r) && (r != 0 || a == 0 || b == 0);
}
RP_DEV bool spot_sum(float a, float b, float &r) {
    r = a + b;
    return normal_or_zero(r) && (r != 0 || a == -b);
}
RP_DEV bool spot_divide(float a, float b, float &r) {
    r = a / b;
    return normal_or_zero(r) && (r != 0 || a == 0);
}
RP_DEV bool positional_intensity(const DPositional &L, V3 wi, float &intensity) {
    if (L.kind == 0)
        return true;
    if (L.kind != 1)
        return false;
    float w[3];
    const float nwi[3] = {-wi.x, -wi.y, -wi.z};
#pragma unroll
    for (int row = 0; row < 3; ++row) {
        float terms[3];
#pragma unroll
        for (int col = 0; col < 3; ++col)
            if (!spot_product(L.light_from_world[row * 3 + col], nwi[col], terms[col]))
                return false;
        float sum, c;
        if (!spot_sum(terms[0], terms[1], sum) || !spot_sum(sum, terms[2], c))
            return false;
        w[row] = c;
    }
    const float scale = fmaxf(fmaxf(fabsf(w[0]), fabsf(w[1])), fabsf(w[2]));
    if (!(scale >= kFltMin) || !isfinite(scale))
        return false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float c;
        if (!spot_divide(w[i], scale, c))
            return false;
        w[i] = c;
    }
    float cosine;
    if (!spot_divide(w[2], sqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]), cosine))
        return false;
    const float end = L.cos_falloff_end, start = L.cos_falloff_start;
    const float t = start == end ? (cosine < end ? 0.0f : 1.0f) : fminf(fmaxf((cosine - end) / (start - end), 0.0f), 1.0f);
    const float falloff = start == end ? t : t * t * (3.0f - 2.0f * t);
    intensity *= falloff;
    return isfinite(intensity) && intensity >= 0;
}

// ------------------------------------------------------------------ traversal
// Ray of a traversal walk: origin, direction, the slab reciprocals, and the per-ray part of
// the watertight triangle test (the dominant axis kz, the other two axes kx, ky, swapped when
// the direction along kz is negative to keep the winding, and the shear constants).
struct WalkRay {
    V3 o, d, inv;
    int kx, ky, kz;
    float sx, sy, sz;
};
RP_DEV WalkRay walk_ray(V3 o, V3 d) {
    WalkRay r;
    r.o = o;
    r.d = d;
    r.inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const V3 ad = vabs(d);
    r.kz = ad.x > ad.y ? (ad.x > ad.z ? 0 : 2) : (ad.y > ad.z ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    if (comp(d, r.kz) < 0) {
        const int t0 = r.kx;
        r.kx = r.ky;
        r.ky = t0;
    }
    const float dz = comp(d, r.kz);
    r.sx = comp(d, r.kx) / dz;
    r.sy = comp(d, r.ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}

// Watertight ray/triangle intersection (Woop, Benthin and Wald, JCGT 2(1), 2013).
RP_DEV bool intersect_triangle(const WalkRay &r, V3 v0, V3 v1, V3 v2, float tmax, float &t, float &b1, float &b2) {
    const int kx = r.kx, ky = r.ky, kz = r.kz;
    const float sx = r.sx, sy = r.sy, sz = r.sz;
    const V3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
    const float ax = fmaf(-sx, comp(A, kz), comp(A, kx)), ay = fmaf(-sy, comp(A, kz), comp(A, ky));
    const float bx = fmaf(-sx, comp(B, kz), comp(B, kx)), by = fmaf(-sy, comp(B, kz), comp(B, ky));
    const float cx = fmaf(-sx, comp(C, kz), comp(C, kx)), cy = fmaf(-sy, comp(C, kz), comp(C, ky));
    float U = fmaf(cx, by, -(cy * bx));
    float Vv = fmaf(ax, cy, -(ay * cx));
    float W = fmaf(bx, ay, -(by * ax));
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
    const float az = sz * comp(A, kz), bz = sz * comp(B, kz), cz = sz * comp(C, kz);
    const float T = fmaf(U, az, fmaf(Vv, bz, W * cz));
    if (det > 0 ? (T <= 0 || T >= tmax * det) : (T >= 0 || T <= tmax * det))
        return false;
    const float rcp = 1.0f / det;
    t = T * rcp;
    b1 = Vv * rcp;
    b2 = W * rcp;
    return t > 0 && t < tmax;
}

// Conservative slab test (Ize, JCGT 2(2), 2013), same operation order as the CPU LBVH.  The
// three axes run without early exits and one comparison decides: t0 only grows and t1 only
// shrinks, and neither takes a NaN (a NaN bound loses every comparison), so the answer and
// the entry distance equal those of the per-axis early-exit form.
RP_DEV void slab_axis(float l, float h, float o, float inv, float scale, float &t0, float &t1) {
    const float tn = (l - o) * inv, tf = (h - o) * inv;
    const bool swap = tn > tf;
    const float near = swap ? tf : tn, far = (swap ? tn : tf) * scale;
    t0 = near > t0 ? near : t0;
    t1 = far < t1 ? far : t1;
}
RP_DEV bool slab(float lx, float ly, float lz, float hx, float hy, float hz, V3 o, V3 inv, float tmax, float scale,
                 float &tenter) {
    float t0 = 0, t1 = tmax;
    slab_axis(lx, hx, o.x, inv.x, scale, t0, t1);
    slab_axis(ly, hy, o.y, inv.y, scale, t0, t1);
    slab_axis(lz, hz, o.z, inv.z, scale, t0, t1);
    tenter = t0;
    return t0 <= t1;
}

struct Hit {
    float t, b1, b2;
    u32 prim;
};

// Traversal stack entries (node groups) per thread.  A walk holds at most one entry per level
// of the wide tree, so the wavefront walks take kShortStack entries when the built tree has at
// most that many levels, and kStackDepth otherwise (deeper trees report an invalid hit).
constexpr int kStackDepth = 40, kShortStack = 16;

// Closest-hit triangle test of wide leaf `index`: keeps the minimum (t, primitive id).  Proc:
// the scene has procedural primitives (their leaves take the object-space tests).
template <bool Count, bool Proc>
RP_DEV void closest_leaf(const DeviceScene &s, const WalkRay &r, float tmax, Hit &h, u32 index, u32 &tris_tested) {
    const float4 a = __ldg(s.wtri + 3 * index), b = __ldg(s.wtri + 3 * index + 1), c = __ldg(s.wtri + 3 * index + 2);
    const u32 prim = __float_as_uint(a.w);
    float t, b1, b2;
    if (Count)
        ++tris_tested;
    if (Proc && prim >= s.tri_prims) {
        const ShapeHit ph = procedural_hit(s, prim, r.o, r.d, tmax);
        if (ph.hit && (ph.t < h.t || (ph.t == h.t && prim < h.prim))) {
            h.t = ph.t;
            h.b1 = ph.u;
            h.b2 = ph.v;
            h.prim = prim;
        }
        return;
    }
    if (intersect_triangle(r, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z), tmax, t, b1, b2) &&
        (t < h.t || (t == h.t && prim < h.prim))) {
        h.t = t;
        h.b1 = b1;
        h.b2 = b2;
        h.prim = prim;
    }
}
// Any-hit triangle test of wide leaf `index` in (0, tmax).
template <bool Count, bool Proc>
RP_DEV bool any_leaf(const DeviceScene &s, const WalkRay &r, float tmax, u32 index, u32 &tris_tested) {
    const float4 a = __ldg(s.wtri + 3 * index), b = __ldg(s.wtri + 3 * index + 1), c = __ldg(s.wtri + 3 * index + 2);
    float t, b1, b2;
    if (Count)
        ++tris_tested;
    const u32 prim = __float_as_uint(a.w);
    if (Proc && prim >= s.tri_prims)
        return procedural_hit(s, prim, r.o, r.d, tmax).hit;
    return intersect_triangle(r, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z), tmax, t, b1, b2);
}

// The quantized planes of a wide node against a ray, in interval arithmetic.  Along an axis
// the plane of byte q lies at p + q s (real arithmetic; the builder guarantees lo planes at
// or below and hi planes at or above the child's box), and the ray reaches it at
// t = (p - o) / d + q s / d.  With [a_lo, a_hi] containing (p - o) / d - 2^23 s / d and
// [b_lo, b_hi] containing s / d, a lower bound of t is fmaf_rd(2^23 + q, b_lo, a_lo) and an upper
// bound fmaf_ru(2^23 + q, b_hi, a_hi), where 2^23 + q is the float whose bits are 0x4b0000qq
// (one byte permute).  A direction component of zero (or one whose reciprocal overflows) makes
// that axis's bounds NaN or infinite in the direction that leaves the axis unconstrained; the
// NaN-ignoring min and max then skip it, which is conservative.
struct WideRay {
    float a_lo[3], a_hi[3], b_lo[3], b_hi[3]; // per axis, for the node being visited
    float rcp_lo[3], rcp_hi[3];                // directed-rounding bounds of 1 / d
    u32 negative;                              // axis bits: d < 0 (the near plane is the hi one)
};
RP_DEV WideRay wide_ray(V3 d) {
    WideRay w;
    const float dd[3] = {d.x, d.y, d.z};
    w.negative = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        w.rcp_lo[a] = __frcp_rd(dd[a]);
        w.rcp_hi[a] = __frcp_ru(dd[a]);
        w.negative |= (__float_as_uint(dd[a]) >> 31) << a;
    }
    return w;
}
// [lo, hi] bounds of x * y for x in [x_lo, x_hi] and y in [y_lo, y_hi] with y of one sign.
RP_DEV void interval_mul(float x_lo, float x_hi, float y_lo, float y_hi, bool y_negative, float &lo, float &hi) {
    if (!y_negative) {
        lo = __fmul_rd(x_lo, x_lo >= 0 ? y_lo : y_hi);
        hi = __fmul_ru(x_hi, x_hi >= 0 ? y_hi : y_lo);
    } else {
        lo = __fmul_rd(x_hi, x_hi >= 0 ? y_lo : y_hi);
        hi = __fmul_ru(x_lo, x_lo >= 0 ? y_hi : y_lo);
    }
}
RP_DEV float qfloat(u32 word, int byte) { return __uint_as_float(__byte_perm(word, 0x4b000000u, 0x7540u | u32(byte))); }

// The children of a wide node whose boxes the ray's segment [0, tmax] may enter: internal ones
// as bits at slot ^ order (near side first), leaves as bits at their slot.  Conservative: the
// computed entry is at or below the true one and the exit at or above, so no child that holds
// a hit in [0, tmax] is missed; all eight slots are tested without branches and masked.
RP_DEV void wide_children(const WNode &n, V3 o, WideRay &w, float tmax, u32 order, u32 &inner, u32 &leaves) {
    const u32 meta = __float_as_uint(n.origin.w);
    const u32 imask = meta >> 24, lmask = n.links.z;
    const float p[3] = {n.origin.x, n.origin.y, n.origin.z}, oo[3] = {o.x, o.y, o.z};
    // byte words of each bound row: lo.x, lo.y, lo.z, hi.x, hi.y, hi.z (slots 0-3, 4-7)
    const u32 rows[6][2] = {{n.q0.x, n.q0.y}, {n.q0.z, n.q0.w}, {n.q1.x, n.q1.y},
                            {n.q1.z, n.q1.w}, {n.q2.x, n.q2.y}, {n.q2.z, n.q2.w}};
    u32 near_w[3][2], far_w[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float s = __uint_as_float(((meta >> (8 * a)) & 0xffu) << 23);
        const bool neg = (w.negative >> a) & 1u;
        float d_lo, d_hi, c_lo, c_hi;
        // (p - o) / d, then minus 2^23 s / d
        interval_mul(__fsub_rd(p[a], oo[a]), __fsub_ru(p[a], oo[a]), w.rcp_lo[a], w.rcp_hi[a], neg, d_lo, d_hi);
        w.b_lo[a] = __fmul_rd(s, w.rcp_lo[a]);
        w.b_hi[a] = __fmul_ru(s, w.rcp_hi[a]);
        c_lo = __fmaf_rd(-8388608.0f, w.b_hi[a], d_lo);
        c_hi = __fmaf_ru(-8388608.0f, w.b_lo[a], d_hi);
        w.a_lo[a] = c_lo;
        w.a_hi[a] = c_hi;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            near_w[a][h] = neg ? rows[3 + a][h] : rows[a][h];
            far_w[a][h] = neg ? rows[a][h] : rows[3 + a][h];
        }
    }
    u32 hits = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int h = k >> 2, byte = k & 3;
        float t0 = 0.0f, t1 = tmax;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            t0 = fmaxf(t0, __fmaf_rd(qfloat(near_w[a][h], byte), w.b_lo[a], w.a_lo[a]));
            t1 = fminf(t1, __fmaf_ru(qfloat(far_w[a][h], byte), w.b_hi[a], w.a_hi[a]));
        }
        hits |= (t0 <= t1 ? 1u : 0u) << k;
    }
    leaves = hits & lmask;
    u32 m = hits & imask; // to traversal order: bit k moves to k ^ order
    if (order & 1u)
        m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (order & 2u)
        m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (order & 4u)
        m = ((m & 0x0fu) << 4) | ((m >> 4) & 0x0fu);
    inner = m;
}

// Closest hit: minimises (t, primitive id), so the result is independent of visit order.
// `stack` is this thread's slice of a shared-memory stack with stride `stride`; an entry is a
// node group: the parent's child_base and internal mask, and the hit children not yet
// visited.  A walk visits each wide node at most once; a stack deeper than Stack reports a
// failed query.
template <bool Count, int Stack = kStackDepth, bool Proc = false>
RP_DEV bool walk_closest(const DeviceScene &s, V3 o, V3 d, float tmax, Hit &h, uint2 *stack, int stride,
                         u32 &nodes_visited, u32 &tris_tested) {
    h.t = tmax;
    h.b1 = h.b2 = 0;
    h.prim = kNone;
    if (s.prim_count == 0)
        return true;
    const WalkRay r = walk_ray(o, d);
    if (s.prim_count == 1) {
        closest_leaf<Count, Proc>(s, r, tmax, h, 0, tris_tested);
        return true;
    }
    const u32 order = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    WideRay wr = wide_ray(d);
    int sp = 0;
    u32 node = 0;
    for (u32 guard = 0; guard <= s.wnode_count; ++guard) {
        const WNode *np = s.wnodes + node;
        WNode n;
        n.origin = __ldg(&np->origin);
        n.links = __ldg(&np->links);
        n.q0 = __ldg(&np->q0);
        n.q1 = __ldg(&np->q1);
        n.q2 = __ldg(&np->q2);
        if (Count)
            ++nodes_visited;
        u32 inner, leaves;
        wide_children(n, o, wr, h.t, order, inner, leaves);
        const u32 lmask = n.links.z;
        while (leaves) {
            const u32 k = __ffs(leaves) - 1;
            leaves &= leaves - 1;
            closest_leaf<Count, Proc>(s, r, tmax, h, n.links.y + __popc(lmask & ((1u << k) - 1)), tris_tested);
        }
        const u32 imask = __float_as_uint(n.origin.w) >> 24;
        u32 base = n.links.x, group_mask = imask;
        if (!inner) {
            if (sp == 0)
                return true;
            const uint2 e = stack[(sp - 1) * stride];
            base = e.x;
            group_mask = e.y >> 8;
            inner = e.y & 0xffu;
            --sp;
        }
        const u32 b = __ffs(inner) - 1;
        inner &= inner - 1;
        const u32 slot = b ^ order;
        node = base + __popc(group_mask & ((1u << slot) - 1));
        if (inner) {
            if (sp >= Stack)
                return false;
            stack[sp * stride] = make_uint2(base, (group_mask << 8) | inner);
            ++sp;
        }
    }
    return false;
}
template <bool Count>
RP_DEV bool trace_closest(const DeviceScene &s, V3 o, V3 d, float tmax, Hit &h, uint2 *stack, int stride,
                          u32 &nodes_visited, u32 &tris_tested) {
    return walk_closest<Count, kStackDepth, true>(s, o, d, tmax, h, stack, stride, nodes_visited, tris_tested);
}

// Any hit in (0, tmax): the shadow-ray occlusion query, the same walk stopped at the first hit.
template <bool Count, int Stack = kStackDepth, bool Proc = false>
RP_DEV bool walk_any(const DeviceScene &s, V3 o, V3 d, float tmax, bool &occluded, uint2 *stack, int stride,
                     u32 &nodes_visited, u32 &tris_tested) {
    occluded = false;
    if (s.prim_count == 0)
        return true;
    const WalkRay r = walk_ray(o, d);
    if (s.prim_count == 1) {
        occluded = any_leaf<Count, Proc>(s, r, tmax, 0, tris_tested);
        return true;
    }
    const u32 order = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    WideRay wr = wide_ray(d);
    int sp = 0;
    u32 node = 0;
    for (u32 guard = 0; guard <= s.wnode_count; ++guard) {
        const WNode *np = s.wnodes + node;
        WNode n;
        n.origin = __ldg(&np->origin);
        n.links = __ldg(&np->links);
        n.q0 = __ldg(&np->q0);
        n.q1 = __ldg(&np->q1);
        n.q2 = __ldg(&np->q2);
        if (Count)
            ++nodes_visited;
        u32 inner, leaves;
        wide_children(n, o, wr, tmax, order, inner, leaves);
        const u32 lmask = n.links.z;
        while (leaves) {
            const u32 k = __ffs(leaves) - 1;
            leaves &= leaves - 1;
            if (any_leaf<Count, Proc>(s, r, tmax, n.links.y + __popc(lmask & ((1u << k) - 1)), tris_tested)) {
                occluded = true;
                return true;
            }
        }
        const u32 imask = __float_as_uint(n.origin.w) >> 24;
        u32 base = n.links.x, group_mask = imask;
        if (!inner) {
            if (sp == 0)
                return true;
            const uint2 e = stack[(sp - 1) * stride];
            base = e.x;
            group_mask = e.y >> 8;
            inner = e.y & 0xffu;
            --sp;
        }
        const u32 b = __ffs(inner) - 1;
        inner &= inner - 1;
        const u32 slot = b ^ order;
        node = base + __popc(group_mask & ((1u << slot) - 1));
        if (inner) {
            if (sp >= Stack)
                return false;
            stack[sp * stride] = make_uint2(base, (group_mask << 8) | inner);
            ++sp;
        }
    }
    return false;
}
template <bool Count>
RP_DEV bool trace_any(const DeviceScene &s, V3 o, V3 d, float tmax, bool &occluded, uint2 *stack, int stride,
                      u32 &nodes_visited, u32 &tris_tested) {
    return walk_any<Count, kStackDepth, true>(s, o, d, tmax, occluded, stack, stride, nodes_visited, tris_tested);
}

} // namespace rp
