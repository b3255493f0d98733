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
