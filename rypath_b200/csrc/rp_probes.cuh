// Fixed-input probe kernels (the counterparts of rypath's rypath_*_probe Metal kernels).
#pragma once

#include "rp_kernels.cuh"

namespace rp {

// rypath_sobol_probe (shaders/render.metal:74-93)
__global__ void k_probe_sobol(SobolTables t, const u32 *q, u32 count, u32 *r) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
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
__global__ void k_probe_philox(const u32 *q, u32 count, u32 *r) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const u32 *a = q + 6 * i;
    const uint4 w = philox(make_uint4(a[0], a[1], a[2], a[3]), a[4], a[5]);
    r[4 * i] = w.x;
    r[4 * i + 1] = w.y;
    r[4 * i + 2] = w.z;
    r[4 * i + 3] = w.w;
}
__global__ void k_probe_wavelengths(const float *u, u32 count, u32 mode, float *r) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    V4 l, p;
    sample_wavelengths(u[i], mode, l, p);
    for (int k = 0; k < 4; ++k) {
        r[8 * i + k] = l.v[k];
        r[8 * i + 4 + k] = p.v[k];
    }
}
// Single-lane BSDF probe in the layout of or_probe_bsdf.
__global__ void k_probe_bsdf(const float *q, u32 count, float *r) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 16 * i;
    float *o = r + 12 * i;
    for (int k = 0; k < 12; ++k)
        o[k] = 0;
    HeroBsdf b;
    b.kind = u32(a[0]);
    b.active_mask = 1;
    for (int k = 0; k < 4; ++k)
        b.param[k] = b.k[k] = 0;
    b.g = {0, 0, true};
    if (b.kind == 0) {
        b.param[0] = a[1];
    } else if (b.kind == 1) {
        const float eta = a[1], kk = a[2], u = a[3], v = a[4];
        if (!isfinite(eta) || !isfinite(kk) || !isfinite(u) || !isfinite(v) || eta < 0 || kk < 0 || u < 0 || v < 0 ||
            (eta == 0 && kk == 0)) {
            o[2] = -1;
            return;
        }
        b.param[0] = eta;
        b.k[0] = kk;
        prepare_roughness(u, v, a[5] != 0, false, b.g);
    } else {
        const float eta = a[1], u = a[3], v = a[4];
        if (!isfinite(eta) || eta < 0 || !isfinite(u) || !isfinite(v) || u < 0 || v < 0) {
            o[2] = -1;
            return;
        }
        b.param[0] = eta == 0 ? 1 : eta;
        prepare_roughness(u, v, a[5] != 0, b.param[0] == 1, b.g);
    }
    const V3 wo = v3(a[6], a[7], a[8]), wi = v3(a[9], a[10], a[11]);
    // lane_evaluate/lane_sample force smooth for eta == 1 exactly as dielectric prepare does
    const Eval e = lane_evaluate(b, 0, wo, wi);
    o[0] = e.f;
    o[1] = e.pdf;
    o[2] = e.valid ? 1.f : 0.f;
    float eta;
    const BSample sm = lane_sample(b, 0, wo, a[12], a[13], a[14], eta);
    o[3] = sm.wi.x;
    o[4] = sm.wi.y;
    o[5] = sm.wi.z;
    o[6] = sm.weight;
    o[7] = sm.pdf;
    o[8] = float((sm.delta ? 1 : 0) | (sm.accepted ? 2 : 0) | (sm.valid ? 4 : 0));
    o[9] = eta;
}
// Hero BSDF probe (shaders/hero_current_bsdf.h:121-203, hero_frozen_bsdf.h:167-250,
// hero_scattering.h:100-138): per query 32 floats {kind, active mask, remap, unused, per
// wavelength {eta or reflectance, k, roughness u, roughness v}, wo[3], wi[3], uc, ux, uy,
// unused[3]} -> 32 floats {sampled wi[3], numerator[4], pdf[4], eta[4], flags (delta 1 |
// transmission 2 | accepted 4 | valid 8), evaluated f[4], evaluated pdf[4], evaluation valid,
// wavelength 0's Dirac mass, pdf and eta, Dirac ok, connectible, prepared, unused}.  A hero
// BSDF shares one roughness over its wavelengths, so wavelength 0's roughness is the one used;
// every wavelength's parameters are checked as the family's prepare checks them.
__global__ void k_probe_hero(const float *queries, u32 count, float *results) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = queries + 32 * i;
    float *o = results + 32 * i;
    for (int j = 0; j < 32; ++j)
        o[j] = 0;
    HeroBsdf p;
    p.kind = u32(a[0]);
    p.active_mask = u32(a[1]);
    p.g = {0, 0, true};
    bool ok = p.kind <= 2;
    for (int k = 0; k < 4; ++k) {
        const float *l = a + 4 + 4 * k;
        p.param[k] = p.kind == 2 && l[0] == 0 ? 1.f : l[0];
        p.k[k] = p.kind == 1 ? l[1] : 0.f;
        if (p.kind == 0)
            continue;
        const bool rough_ok = isfinite(l[2]) && isfinite(l[3]) && l[2] >= 0 && l[3] >= 0;
        if (p.kind == 1)
            ok = ok && rough_ok && isfinite(l[0]) && isfinite(l[1]) && l[0] >= 0 && l[1] >= 0 &&
                 !(l[0] == 0 && l[1] == 0);
        else
            ok = ok && rough_ok && isfinite(l[0]) && l[0] >= 0;
    }
    if (ok && p.kind != 0)
        prepare_roughness(a[6], a[7], a[2] != 0, false, p.g);
    o[30] = ok ? 1.f : 0.f;
    if (!ok)
        return;
    const V3 wo = v3(a[20], a[21], a[22]), wi = v3(a[23], a[24], a[25]);
    const HeroSample sm = p.kind == 0   ? hero_sample_k<0>(p, wo, a[26], a[27], a[28])
                          : p.kind == 1 ? hero_sample_k<1>(p, wo, a[26], a[27], a[28])
                                        : hero_sample_k<2>(p, wo, a[26], a[27], a[28]);
    o[0] = sm.wi.x;
    o[1] = sm.wi.y;
    o[2] = sm.wi.z;
    for (int k = 0; k < 4; ++k) {
        o[3 + k] = sm.numerator.v[k];
        o[7 + k] = sm.pdf.v[k];
        o[11 + k] = sm.eta.v[k];
    }
    o[15] = float((sm.delta ? 1 : 0) | (sm.transmission ? 2 : 0) | (sm.accepted ? 4 : 0) | (sm.valid ? 8 : 0));
    const HeroEval e = hero_evaluate(p, wo, wi);
    for (int k = 0; k < 4; ++k) {
        o[16 + k] = e.f.v[k];
        o[20 + k] = e.pdf.v[k];
    }
    o[24] = e.valid ? 1.f : 0.f;
    float mass, density, eta;
    const bool dirac = dirac_lane(p, 0, wo, wi, a[27], a[28], mass, density, eta);
    o[25] = mass;
    o[26] = density;
    o[27] = eta;
    o[28] = dirac ? 1.f : 0.f;
    o[29] = hero_connectible(p) ? 1.f : 0.f;
}
// Image probes, in the oracle's layouts: texture lookups of texture `index` (6 floats {u, v,
// dudx, dvdx, dudy, dvdy} -> 4 {rgb[3], scalar}); RGB reconstruction (4 {r, g, b, wavelength}
// -> 2 {bounded, unbounded}); environment queries (8 {direction[3], wavelength, u[2], unused[2]}
// -> 12 {radiance, compensated pdf, full pdf, sample ok, direction[3], pdf, full-table sample
// ok, direction[3]}).
__global__ void k_probe_image_lookup(const DImages im, u32 index, const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 6 * i;
    float *o = out + 4 * i;
    const DImageTexture t = im.textures[index];
    const F2 uv = f2(a[0], a[1]), dx = f2(a[2], a[3]), dy = f2(a[4], a[5]);
    const RGB c = lookup_filtered(im, t, uv, dx, dy, false, false);
    o[0] = c.r;
    o[1] = c.g;
    o[2] = c.b;
    o[3] = lookup_filtered(im, t, uv, dx, dy, true, false).r;
}
// Bilinear patch intersection: 20 floats per query -> {hit, t, u, v}.
__global__ void k_probe_bilinear(const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 20 * i;
    const ShapeHit h = intersect_bilinear(v3(a[0], a[1], a[2]), v3(a[3], a[4], a[5]), v3(a[6], a[7], a[8]),
                                          v3(a[9], a[10], a[11]), v3(a[12], a[13], a[14]), v3(a[15], a[16], a[17]),
                                          a[18], a[19]);
    out[4 * i] = h.hit ? 1.f : 0.f;
    out[4 * i + 1] = h.t;
    out[4 * i + 2] = h.u;
    out[4 * i + 3] = h.v;
}
// Analytic shape intersection and evaluation at the hit: 16 words per query -> 16 floats.
__global__ void k_probe_analytic(const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 16 * i;
    DAnalytic rec;
    rec.kind = __float_as_uint(a[0]);
    rec.subtype = __float_as_uint(a[1]);
    rec.radius = a[2];
    rec.z_min = a[3];
    rec.z_max = a[4];
    rec.phi_max = a[5];
    rec.inner_radius = a[6];
    rec.height = a[7];
    const ShapeHit h = intersect_analytic(rec, v3(a[8], a[9], a[10]), v3(a[11], a[12], a[13]), a[14], a[15]);
    float *o = out + 16 * i;
    o[0] = h.hit ? 1.f : 0.f;
    o[1] = h.t;
    o[2] = h.u;
    o[3] = h.v;
    const AnalyticSurface e = evaluate_analytic(rec, h.hit ? h.u : 0.f, h.hit ? h.v : 0.f);
    const V3 vs[4] = {e.position, e.normal, e.dpdu, e.dpdv};
    for (int k = 0; k < 4; ++k) {
        o[4 + 3 * k] = vs[k].x;
        o[5 + 3 * k] = vs[k].y;
        o[6 + 3 * k] = vs[k].z;
    }
}
__global__ void k_probe_rgb_spectrum(const float *table, const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 4 * i;
    const RGB c = rgb3(a[0], a[1], a[2]);
    out[2 * i] = rgb_spectrum(table, c, a[3]);
    out[2 * i + 1] = rgb_spectrum_unbounded(table, c, a[3]);
}
__global__ void k_probe_environment(const DImages im, const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 8 * i;
    float *o = out + 12 * i;
    const V3 d = v3(a[0], a[1], a[2]);
    o[0] = environment_image_radiance(im, d, a[3]);
    o[1] = environment_image_pdf(im, d, true);
    o[2] = environment_image_pdf(im, d, false);
    V3 w = v3(0, 0, 0);
    float pdf = 0;
    o[3] = sample_environment_image(im, a[4], a[5], true, w, pdf) ? 1.f : 0.f;
    o[4] = w.x;
    o[5] = w.y;
    o[6] = w.z;
    o[7] = pdf;
    V3 w2 = v3(0, 0, 0);
    float pdf2 = 0;
    o[8] = sample_environment_image(im, a[4], a[5], false, w2, pdf2) ? 1.f : 0.f;
    o[9] = w2.x;
    o[10] = w2.y;
    o[11] = w2.z;
}
// Texture footprint probe, in the oracle's layout (48 floats {relative p[3], n[3], ray
// direction[3], x ray[3], y ray[3], spp scale, world_from_camera[9], camera_from_world[9],
// minimum dx[3], minimum dy[3], dpdu[3], dpdv[3], unused[2]} -> 24 {primary ok, primary
// dpdx[3], dpdy[3], approximate dpdx[3], dpdy[3], derivatives ok, dstdx[2], dstdy[2],
// texture direction of the x ray[3], unused[3]}).
__global__ void k_probe_texture_footprint(const float *q, u32 count, float *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *a = q + 48 * i;
    float *o = out + 24 * i;
    DImages im{};
    for (int k = 0; k < 9; ++k) {
        im.world_from_camera[k] = a[16 + k];
        im.camera_from_world[k] = a[25 + k];
    }
    for (int k = 0; k < 3; ++k) {
        im.tex_min_dx[k] = a[34 + k];
        im.tex_min_dy[k] = a[37 + k];
    }
    im.tex_spp_scale = a[15];
    const V3 rp = v3(a[0], a[1], a[2]), n = v3(a[3], a[4], a[5]), d = v3(a[6], a[7], a[8]);
    const V3 rx = v3(a[9], a[10], a[11]), ry = v3(a[12], a[13], a[14]);
    V3 pdx = v3(0, 0, 0), pdy = v3(0, 0, 0), adx, ady;
    const bool primary = texture_primary_dp(rp, n, d, rx, ry, a[15], pdx, pdy);
    texture_approximate_dp(im, rp, n, adx, ady);
    F2 sx = f2(0, 0), sy = f2(0, 0);
    const bool ok = texture_uv_derivatives(v3(a[40], a[41], a[42]), v3(a[43], a[44], a[45]), primary ? pdx : adx,
                                           primary ? pdy : ady, sx, sy);
    const V3 td = texture_direction(rx);
    const float v[24] = {primary ? 1.f : 0.f, pdx.x, pdx.y, pdx.z, pdy.x, pdy.y, pdy.z, adx.x, adx.y, adx.z,
                         ady.x, ady.y, ady.z, ok ? 1.f : 0.f, sx.x, sx.y, sy.x, sy.y, td.x, td.y, td.z, 0, 0, 0};
    for (int k = 0; k < 24; ++k)
        o[k] = v[k];
}
__global__ void k_probe_raygen(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams p, u32 *words,
                               float *rays) {
    const u32 lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= p.lanes)
        return;
    const BeginSample b = begin_sample(s, p, lane);
    u32 *w = words + 11 * lane;
    w[0] = b.pixel;
    w[1] = b.sample_low;
    w[2] = b.sample_high;
    w[3] = u32(b.index);
    w[4] = u32(b.index >> 32);
    w[5] = b.words.x;
    w[6] = b.words.y;
    w[7] = b.words.z;
    w[8] = b.words.w;
    w[9] = b.lens_words.x;
    w[10] = b.lens_words.y;
    V3 o, d;
    primary_ray(s, p, b, o, d);
    float *r = rays + 6 * lane;
    r[0] = o.x;
    r[1] = o.y;
    r[2] = o.z;
    r[3] = d.x;
    r[4] = d.y;
    r[5] = d.z;
}
__global__ void __launch_bounds__(kTraceBlock) k_probe_trace(const __grid_constant__ DeviceScene s, const float *rays,
                                                             u32 count, int any_hit, float *hits) {
    __shared__ uint2 stack[kStackDepth * kTraceBlock];
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float *r = rays + 7 * i;
    const V3 o = v3(r[0], r[1], r[2]), d = v3(r[3], r[4], r[5]);
    float *h = hits + 4 * i;
    u32 nv = 0, nt = 0;
    if (any_hit) {
        bool occ;
        const bool ok = trace_any<false>(s, o, d, r[6], occ, stack + threadIdx.x, kTraceBlock, nv, nt);
        h[0] = ok ? (occ ? 1.f : 0.f) : -1.f;
        h[1] = h[2] = 0;
        h[3] = __uint_as_float(kNone);
        return;
    }
    Hit hit;
    const bool ok = trace_closest<false>(s, o, d, r[6], hit, stack + threadIdx.x, kTraceBlock, nv, nt);
    h[0] = hit.prim == kNone ? __int_as_float(0x7f800000) : hit.t;
    h[1] = hit.b1;
    h[2] = hit.b2;
    h[3] = __uint_as_float(ok ? hit.prim : 0xfffffffeu);
}

} // namespace rp
