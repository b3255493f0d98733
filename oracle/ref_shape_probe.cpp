// Test infrastructure only: rypath's procedural primitive shaders (shaders/bilinear.h, the
// ruled-surface patch test in float pairs, and shaders/analytic.h, the sphere / disk / cylinder
// tests and parameterisations) compiled from the checkout (oracle/ref.mk) behind the host
// stand-in for <metal_stdlib>, as a C ABI that pins the oracle's restatement.  The code of this
// file is only the marshalling, in the layouts of rp_cuda_probe_bilinear / _analytic.
#include <metal_stdlib>
#include "bilinear.h"
#include "analytic.h"

#include <cstdint>
#include <cstring>

extern "C" {

void ref_bilinear(const float *q, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 20 * size_t(i);
        const BilinearIntersection h =
            intersect_bilinear(metal::float3(a[0], a[1], a[2]), metal::float3(a[3], a[4], a[5]),
                               metal::float3(a[6], a[7], a[8]), metal::float3(a[9], a[10], a[11]),
                               metal::float3(a[12], a[13], a[14]), metal::float3(a[15], a[16], a[17]), a[18], a[19]);
        float *o = out + 4 * size_t(i);
        o[0] = h.hit ? 1.f : 0.f;
        o[1] = h.t;
        o[2] = h.uv.x;
        o[3] = h.uv.y;
    }
}

void ref_analytic(const float *q, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float *a = q + 16 * size_t(i);
        rypath::geometry_wire::Analytic rec{};
        std::memcpy(&rec, a, sizeof(rec));
        const AnalyticIntersection h = intersect_analytic(rec, metal::float3(a[8], a[9], a[10]),
                                                          metal::float3(a[11], a[12], a[13]), a[14], a[15]);
        float *o = out + 16 * size_t(i);
        o[0] = h.hit ? 1.f : 0.f;
        o[1] = h.t;
        o[2] = h.uv.x;
        o[3] = h.uv.y;
        const AnalyticSurface e = evaluate_analytic(rec, h.hit ? h.uv : metal::float2(0, 0));
        const metal::float3 vs[4] = {e.position, e.normal, e.dpdu, e.dpdv};
        for (int k = 0; k < 4; ++k) {
            o[4 + 3 * k] = vs[k].x;
            o[5 + 3 * k] = vs[k].y;
            o[6 + 3 * k] = vs[k].z;
        }
    }
}

} // extern "C"
