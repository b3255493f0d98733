// Wavefront kernels of the hero path tracer and the device film reduction.
#pragma once

#include "rp_transport.cuh"

namespace rp {

constexpr int kTraceBlock = 128;

// Warp-aggregated append to a device queue: one atomicAdd per warp.  Every lane of the warp
// must call this together (the shade kernel runs a warp-uniform trip count).
RP_DEV u32 warp_append(u32 *counter, bool want) {
    const u32 ballot = __ballot_sync(0xffffffffu, want);
    const int lane = threadIdx.x & 31;
    u32 base = 0;
    if (lane == 0 && ballot)
        base = atomicAdd(counter, __popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    return base + __popc(ballot & ((1u << lane) - 1));
}

// rypath_render_packets prologue (shaders/render.metal:2424-2460) + packet_pt_initialize
// (shaders/packet_pt_step.h:84-115) for request lane `lane`, stored in pool slot `slot`.
RP_DEV void raygen_lane(const DeviceScene &s, const RasterCam &cam, const WaveParams &p, u32 lane, u32 slot,
                        PathPool &pool) {
    {
        const BeginSample b = begin_sample(s, p, lane);
        V4 lambda, pdf;
        sample_wavelengths(sample_uniform(p, b.words.z), s.hero_mode, lambda, pdf);
        V3 o, d;
        primary_ray_from(s, cam, p, b, o, d);
        u32 flags = 15u | F_ROULETTE | (kCamera << F_LTYPE_SHIFT);
        if (!finite3(o) || !finite3(d))
            flags = set_status(flags, 2) | F_COMPLETE;
        pool.ident[slot] = make_uint4(b.pixel, b.sample_low, b.sample_high, flags);
        pool.cursor[slot] = make_uint4(u32(b.index), u32(b.index >> 32), 1, slot);
        pool.lambda[slot] = to_float4(lambda);
        pool.lambda_pdf[slot] = to_float4(pdf);
        pool.beta[slot] = make_float4(1, 1, 1, 1);
        pool.radiance[slot] = make_float4(0, 0, 0, 0);
        pool.dens_f[slot] = pool.prev_f[slot] = make_float4(.5f, .5f, .5f, .5f);
        pool.dens_e[slot] = pool.prev_e[slot] = make_int4(1, 1, 1, 1);
        pool.eta_scale[slot] = make_float4(1, 1, 1, 1);
        pool.ray_o[slot] = make_float4(o.x, o.y, o.z, 0);
        pool.ray_d[slot] = make_float4(d.x, d.y, d.z, 0);
        pool.latest_p[slot] = make_float4(o.x, o.y, o.z, 0);
        pool.latest_n[slot] = make_float4(0, 0, 0, 0);
        pool.queue[0][slot] = slot;
        if (pool.lane_closest) {
            pool.lane_closest[slot] = 0;
            pool.lane_shadow[slot] = 0;
        }
        if (pool.hist) {
            pool.hist[slot] = empty_history();
            pool.adj_w[slot] = adjoint_lane_weight(pool, b.pixel, lambda, pdf);
        }
    }
}
__global__ void k_raygen(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams p, PathPool pool) {
    const RasterCam cam{s.origin, s.forward, s.right, s.up};
    for (u32 lane = blockIdx.x * blockDim.x + threadIdx.x; lane < p.lanes; lane += gridDim.x * blockDim.x)
        raygen_lane(s, cam, p, lane, lane, pool);
}

// Hit records the shade kernels read as a failed event (rp_sample_status 3, 4, 2).
constexpr u32 kHitInvalid = 0xfffffffeu, kHitExhausted = 0xfffffffdu, kHitArithmetic = 0xfffffffcu;

// A hit on a pass-through or mix-root instance, resolved before shading
// (shaders/packet_pt_event_body.inc:100-205): the same validity checks and surface point as
// the event, then either a crossing (at most boundary_limit in a row, each a new walk from
// the spawned origin, which is written to ray_o) or the mix resolution (the resolved material
// written to pool.material).  Returns the family to bin (3 for a failure or a miss) and sets
// `prim` to the primitive or failure code to record.
template <bool Count, int Stack>
__device__ __noinline__ u32 resolve_hit(const DeviceScene &s, const PathPool &pool, u32 path, V3 ro, V3 rd, Hit &h,
                                        u32 &prim, uint2 *stack, int stride, u32 boundary_limit, u32 &nodes, u32 &tris,
                                        u32 &rays) {
    u32 crossings = 0;
    bool moved = false;
    u32 family = 3;
    for (;;) {
        if (!isfinite(h.t) || h.t < 0 || !isfinite(h.b1) || !isfinite(h.b2)) {
            prim = kHitInvalid;
            break;
        }
        const u32 inst = s.tri_instance[h.prim];
        const DInstance &in = s.instances[inst];
        if (in.material >= s.material_count) {
            prim = kHitInvalid;
            break;
        }
        SurfacePoint pt;
        if (!hit_surface_point(s, h.prim, inst, s.tri_local[h.prim], h.b1, h.b2, pt)) {
            prim = kHitArithmetic;
            break;
        }
        if (in.resolve & kPassThrough) {
            V3 origin;
            if (crossings++ >= boundary_limit) {
                prim = kHitExhausted;
                break;
            }
            if (!spawn_boundary(ro, rd, h.t, pt, rd, origin)) {
                prim = kHitArithmetic;
                break;
            }
            ro = origin;
            moved = true;
            ++rays;
            if (!walk_closest<Count, Stack, true>(s, ro, rd, __int_as_float(0x7f800000), h, stack, stride, nodes, tris)) {
                prim = kHitInvalid;
                break;
            }
            prim = h.prim;
            if (prim == kNone)
                break;
            family = __ldg(s.tri_family + prim);
            if (family != kResolveFamily)
                break;
            continue;
        }
        u32 material = in.material;
        const u32 status = resolve_mix(s, pt.position, -rd, material);
        if (status != 0) {
            prim = status == 2 ? kHitArithmetic : kHitInvalid;
            break;
        }
        pool.material[path] = material;
        prim = h.prim;
        family = s.materials[material].scattering;
        break;
    }
    if (moved)
        pool.ray_o[path] = make_float4(ro.x, ro.y, ro.z, 0);
    return prim >= kHitArithmetic || prim == kNone ? 3u : family;
}

// Closest-hit queries for the active queue; each path is then appended to the bin of the
// BSDF family it hit (0 diffuse, 1 conductor, 2 dielectric, 3 miss or failed query), so the
// shade stage runs one specialised kernel per family ("material-sorted shading").
// Stack: traversal stack entries per thread (kShortStack for shallow trees, whose walks then
// fit eight 128-thread blocks per SM).
// Resolve: the scene has pass-through or mix-root instances (resolve_hit).
template <bool Count, int Block = kTraceBlock, int Stack = kStackDepth, bool Resolve = false>
__global__ void __launch_bounds__(Block, Stack <= kShortStack ? 1024 / Block : 1)
    k_trace(const __grid_constant__ DeviceScene s, PathPool pool, int in, u32 boundary_limit) {
    __shared__ uint2 stack[Stack * Block];
    const u32 count = pool.counters[in];
    const u32 *queue = pool.queue[in];
    u32 nodes = 0, tris = 0, rays = 0;
    const u32 stride = gridDim.x * blockDim.x;
    const u32 trips = (count + stride - 1) / stride;
    const int lane = threadIdx.x & 31;
    for (u32 trip = 0; trip < trips; ++trip) {
        const u32 i = trip * stride + blockIdx.x * blockDim.x + threadIdx.x;
        u32 family = 4, path = 0;
        if (i < count) {
            path = queue[i];
            if (!(pool.ident[path].w & F_COMPLETE)) {
                const float4 o = pool.ray_o[path], d = pool.ray_d[path];
                const u32 walks_before = rays;
                Hit h;
                const bool ok = walk_closest<Count, Stack, Resolve>(s, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z),
                                                           __int_as_float(0x7f800000), h, stack + threadIdx.x, Block,
                                                           nodes, tris);
                ++rays;
                u32 prim = ok ? h.prim : kHitInvalid;
                family = (!ok || h.prim == kNone) ? 3u : u32(__ldg(s.tri_family + h.prim));
                if (Resolve && family == kResolveFamily)
                    family = resolve_hit<Count, Stack>(s, pool, path, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), h, prim,
                                                       stack + threadIdx.x, Block, boundary_limit, nodes, tris, rays);
                pool.hit[path] = make_float4(h.t, h.b1, h.b2, __uint_as_float(prim));
                if (Count && pool.lane_closest)
                    pool.lane_closest[path] += rays - walks_before;
            }
        }
        const u32 peers = __match_any_sync(0xffffffffu, family);
        const int leader = __ffs(peers) - 1;
        u32 base = 0;
        if (lane == leader && family < 4)
            base = atomicAdd(pool.counters + 4 + family, __popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (family < 4)
            pool.bins[size_t(family) * pool.bin_capacity + base + __popc(peers & ((1u << lane) - 1))] = path;
    }
    if (Count) {
        atomicAdd(pool.stats + 0, (unsigned long long)nodes);
        atomicAdd(pool.stats + 1, (unsigned long long)tris);
        atomicAdd(pool.stats + 2, (unsigned long long)rays);
    }
}

// One hero event after its closest hit (shaders/packet_pt_event_body.inc:11-461), for the paths
// whose hit is of BSDF family F (3: no surface -- environment or a failed query).
// Adjoint: the path-replay adjoint hooks are compiled in (the plain forward kernel carries none
// of their registers).  The minimum of 512 resident threads per SM caps registers at 128, so
// four 128-thread blocks fit an SM; the escape kernel (F = 3) fits without spilling, the
// other families spill about 500 bytes to L1 and still run a little faster than three blocks
// at 168 registers (113.5 against 115.0 ms per 1080p 16-spp frame of the mixed scene).
// Img: the scene has image reflectance or an environment image (their code is compiled out of
// the plain kernels).
template <int F, int Block = 128, bool Adjoint = false, bool Img = true>
__global__ void __launch_bounds__(Block, 512 / Block) k_shade(const __grid_constant__ DeviceScene s,
                                                              const __grid_constant__ WaveParams p, PathPool pool, int in) {
    extern __shared__ float sgrad[]; // adjoint only
    if (Adjoint)
        adjoint_begin(pool, sgrad);
    const u32 count = pool.counters[4 + F];
    const u32 *queue = pool.bins + size_t(F) * pool.bin_capacity;
    u32 *out_queue = pool.queue[in ^ 1];
    u32 *out_count = pool.counters + (in ^ 1);
    const u32 capacity = s.max_depth + 2;
    // uniform trip count so warp-level appends see every lane of the warp
    const u32 stride = gridDim.x * blockDim.x;
    const u32 trips = (count + stride - 1) / stride;
    for (u32 trip = 0; trip < trips; ++trip) {
        const u32 i = trip * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool keep = false, nee = false;
        u32 path = 0;
        if (i < count) {
            path = queue[i];
            uint4 ident = pool.ident[path];
            u32 flags = ident.w;
            if (!(flags & F_COMPLETE)) {
                uint4 cursor = pool.cursor[path];
                const u64 index = (u64(cursor.y) << 32) | cursor.x;
                u32 cnt = cursor.z;
                const V4 lambda = from_float4(pool.lambda[path]);
                V4 beta = from_float4(pool.beta[path]);
                V4 radiance = from_float4(pool.radiance[path]);
                Density density = load_density(pool.dens_f[path], pool.dens_e[path]);
                const Density previous_density = load_density(pool.prev_f[path], pool.prev_e[path]);
                Density hero_previous = previous_density;
                V4 eta_scale = from_float4(pool.eta_scale[path]);
                bool roulette = (flags & F_ROULETTE) != 0;
                u32 active_mask = flags & F_MASK;
                const float4 ro4 = pool.ray_o[path], rd4 = pool.ray_d[path];
                V3 ro = v3(ro4.x, ro4.y, ro4.z), rd = v3(rd4.x, rd4.y, rd4.z);
                const float4 hit = pool.hit[path];
                u32 status = get_status(flags);
                Density direct_density = density;
                V4 direct_beta = beta;
                bool direct_allowed = true;
                const u32 old_count = cnt;
                bool terminated = true;
                // current vertex
                u32 ctype = kSurface, cinst = kNone, clocal = 0, clight = kNone, cmat = kNone;
                SurfacePoint cp;
                cp.position = cp.error = cp.geometric_normal = cp.shading_normal = v3(0, 0, 0);
                cp.inverse_area_pdf = 0;
                Frame cframe;
                HeroBsdf cbsdf;
                cbsdf.kind = 0;
                cbsdf.active_mask = active_mask;
                cbsdf.g = {0, 0, true};
                V4 cbeta = beta;
                V3 cwo = v3(0, 0, 0), swo = v3(0, 0, 0);
                bool pair_valid = false, cdelta = false, connectible = false;
                do {
                    if (cnt >= capacity || !nonzero4(beta))
                        break;
                    if (!finite3(ro) || !finite3(rd) || !finite_nonnegative4(beta)) {
                        status = 2;
                        break;
                    }
                    const u32 prim = __float_as_uint(hit.w);
                    if (prim >= kHitArithmetic && prim != kNone) {
                        status = prim == kHitInvalid ? 3u : prim == kHitExhausted ? 4u : 2u;
                        break;
                    }
                    if (prim == kNone) {
                        ctype = kEnvironment;
                        clight = s.environment_light;
                        cp.position = ro + rd;
                        cp.geometric_normal = -rd;
                        cp.shading_normal = -rd;
                        cwo = -rd;
                        cbeta = beta;
                        connectible = true;
                        ++cnt;
                        break;
                    }
                    if constexpr (F == 3) {
                        status = 3; // a surface hit never reaches the no-surface bin
                        break;
                    } else {
                        const float t = hit.x, b1 = hit.y, b2 = hit.z;
                        if (!isfinite(t) || t < 0 || !isfinite(b1) || !isfinite(b2) || prim >= s.prim_count) {
                            status = 3;
                            break;
                        }
                        cinst = s.tri_instance[prim];
                        clocal = s.tri_local[prim];
                        const DInstance &instance = s.instances[cinst];
                        if (instance.material >= s.material_count) {
                            status = 3;
                            break;
                        }
                        // a mix root's hit was resolved by the closest-hit kernel
                        cmat = (instance.resolve & kMixRoot) ? pool.material[path] : instance.material;
                        ctype = kSurface;
                        clight = instance.emission == kNone ? kNone : instance.emitter_begin + clocal;
                        cwo = -rd;
                        if (!hit_surface_point(s, prim, cinst, clocal, b1, b2, cp)) {
                            status = 2;
                            break;
                        }
                        const DMaterial material = s.materials[cmat];
                        // an image reflectance reads its texture at the hit's footprint
                        // (shaders/packet_pt_event_body.inc:147-163, packet_walk.h:39-49)
                        RgbPolynomial image_rgb;
                        bool image = false;
                        if constexpr (F == 0) {
                            if (Img && s.img.textured && material.kind == 3 && material.image_texture < s.img.texture_count) {
                                F2 st, dstdx, dstdy;
                                if (!texture_context(s, p, ident.x, ident.y, ident.z, cinst, clocal, b1, b2,
                                                     cp.geometric_normal, rd, cnt - 1, st, dstdx, dstdy)) {
                                    status = 2;
                                    break;
                                }
                                image_rgb = rgb_polynomial(
                                    s.img.rgb_table, image_reflectance_rgb(s.img, material.image_texture, st, dstdx, dstdy));
                                image = true;
                            }
                        }
                        if (!shading_frame(cp.shading_normal, cframe) ||
                            !prepare_bsdf<F>(s, material, lambda, active_mask, cbsdf, image ? &image_rgb : nullptr)) {
                            status = 2;
                            break;
                        }
                        V3 ray_position, ray_error;
                        ray_point(ro, rd, t, cp.curved, ray_position, ray_error);
                        cp.error = cp.error + (vabs(cp.position - ray_position) + ray_error);
                        if (!finite3(cp.error)) {
                            status = 2;
                            break;
                        }
                        cbeta = beta;
                        connectible = hero_connectible(cbsdf);
                        ++cnt;
                        if (cnt == capacity)
                            break;
                        if (cnt - 2 >= p.emergency_limit) {
                            status = 1;
                            break;
                        }
                        const uint4 draws = draw_words(s, p, ident.x, ident.y, ident.z, index, 4 + cnt - 2);
                        swo = to_local(cframe, cwo);
                        cbsdf.active_mask = active_mask;
                        direct_density = density;
                        direct_allowed = hero_continue(beta, eta_scale, roulette, cnt - 1, sample_uniform(p, draws.w));
                        direct_beta = beta;
                        connectible = hero_connectible(cbsdf);
                        if (!direct_allowed)
                            break;
                        const HeroSample proposed = hero_sample_k<F>(cbsdf, swo, sample_uniform(p, draws.x),
                                                                sample_uniform(p, draws.y), sample_uniform(p, draws.z));
                        bool cont_valid = proposed.valid;
                        if (proposed.valid && proposed.accepted) {
                            hero_previous = direct_density;
                            const Update adv = advance(direct_density, beta, proposed.numerator, proposed.pdf);
                            cont_valid = adv.valid;
                            if (adv.valid) {
                                beta = adv.beta;
                                density = adv.density;
                            }
                            hero_account_eta(eta_scale, roulette, proposed.eta, proposed.transmission);
                            active_mask = 1;
    #pragma unroll
                            for (int k = 1; k < 4; ++k)
                                if (density.lane[k].fraction > 0 || (fbits(beta.v[k]) & 0x7fffffffu))
                                    active_mask |= 1u << k;
                        }
                        if (!cont_valid) {
                            status = 2;
                            break;
                        }
                        if (!proposed.accepted)
                            break;
                        pair_valid = true;
                        V3 wi = to_world(cframe, proposed.wi);
                        if (!unit_vector(wi, wi)) {
                            status = 2;
                            break;
                        }
                        if (!finite_nonnegative4(beta)) {
                            status = 2;
                            break;
                        }
                        if (proposed.delta)
                            cdelta = true;
                        const V3 origin = offset_point(cp.position, cp.error, cp.geometric_normal, wi);
                        if (!finite3(origin)) {
                            status = 2;
                            break;
                        }
                        ro = origin;
                        rd = wi;
                        terminated = false;
                    }
                } while (false);
                bool complete = terminated || status != 0 || cnt >= capacity || !nonzero4(beta);
                // latest vertex (the previous event's) for MIS
                const float4 lp4 = pool.latest_p[path], ln4 = pool.latest_n[path];
                Latest latest;
                latest.type = (flags >> F_LTYPE_SHIFT) & 3u;
                latest.kind = (flags >> F_LKIND_SHIFT) & 3u;
                latest.mask = (flags >> F_LMASK_SHIFT) & 15u;
                latest.delta = (flags & F_LDELTA) != 0;
                latest.smooth = (flags & F_LSMOOTH) != 0;
                latest.position = v3(lp4.x, lp4.y, lp4.z);
                latest.shading_normal = v3(ln4.x, ln4.y, ln4.z);
                latest.alpha_x = lp4.w;
                latest.alpha_y = ln4.w;
                if (cnt != old_count && status == 0) {
                    // hero_endpoint (shaders/hero_pt_helpers.h:157-184)
                    V4 rad = v4(0);
                    bool emission_ok = true;
                    if (ctype == kEnvironment) {
                        if (Img && s.img.env_image != kNone) {
                            rad = environment_image_radiance4(s.img, rd, lambda);
                        } else if (s.environment != kNone) {
#pragma unroll
                            for (int k = 0; k < 4; ++k)
                                rad.v[k] = spectrum(s, s.environment, lambda.v[k]);
                        }
                        emission_ok = finite_nonnegative4(rad);
                    } else {
                        const V3 delta = latest.position - cp.position;
                        const DInstance &instance = s.instances[cinst];
                        if (!zero3(delta) && instance.emission != kNone) {
                            const V3 dir = normalize3(delta);
                            if (s.emission_two_sided[instance.emission] || dot(cp.geometric_normal, dir) > 0) {
                                const u32 off = instance.emission * 471u;
#pragma unroll
                                for (int k = 0; k < 4; ++k)
                                    rad.v[k] = cp.inverse_area_pdf == 0 ? 0.f : spectrum(s, off, lambda.v[k]);
                                emission_ok = finite_nonnegative4(rad);
                            }
                        }
                    }
                    V4 endpoint = v4(0);
                    if (!emission_ok) {
                        status = 2;
                    } else {
                        const V4 value = mul4(cbeta, rad);
                        if (cnt <= 2 || latest.delta || !nonzero4(value)) {
                            endpoint = value;
                        } else {
                            latest.param = from_float4(pool.latest_param[path]);
                            latest.k = from_float4(pool.latest_k[path]);
                            const float4 pre = pool.preceding[path];
                            bool ok;
                            const V4 bsdf_pdf = represented_pdf<-1>(latest_bsdf(latest), latest.shading_normal, latest.position,
                                                                v3(pre.x, pre.y, pre.z), ctype == kEnvironment,
                                                                ctype == kEnvironment ? rd : cp.position, ok);
                            // hero_history_light_pdf / direct_pdf (shaders/packet_transport.h:740-758)
                            float lpdf = 0;
                            const float selection = light_pmf(s, latest.position, latest.shading_normal, clight);
                            if (ctype == kEnvironment) {
                                // the constant environment has no unidirectional proposal;
                                // the image's is its compensated table
                                lpdf = (Img && s.img.env_image != kNone) ? environment_image_pdf(s.img, rd, true) * selection
                                                                : 0.0f * selection;
                            } else {
                                const V3 dl = cp.position - latest.position;
                                if (dot(dl, dl) > 0 && nonzero3(cp.geometric_normal) && clight < s.emitter_count)
                                    lpdf = selection * light_geometry_pdf(s, clight, latest.position,
                                                                          latest.shading_normal, cp);
                            }
                            if (!ok || !hero_weight(previous_density, value, ok ? bsdf_pdf : v4(__int_as_float(0x7fffffff)),
                                                    v4(lpdf), endpoint))
                                status = 2;
                        }
                    }
                    radiance = add4(radiance, endpoint);
                    if (Adjoint) {
                        // replay: the emission's gradient over the vertices before this one,
                        // then this diffuse vertex joins the history of what follows it
                        uint4 h = pool.hist[path];
                        if (status == 0 && nonzero4(endpoint))
                            adjoint_accumulate(s, pool, sgrad, h, lambda, endpoint, pool.adj_w[path]);
                        if (F == 0 && ctype == kSurface && status == 0) {
                            const u32 m = cmat;
                            if (__ldg(pool.adj_slot + m) != kNone) {
                                h = history_push(h, m);
                                pool.hist[path] = h;
                            }
                        }
                    }
                    // hero_direct (shaders/hero_pt_helpers.h:185-221) runs in the light-sample kernel
                    // (k_nee), from the request this event leaves (write_nee_request); its failures fail the
                    // path there.
                    nee = F != 3 && status == 0 && cnt < capacity && direct_allowed && ctype == kSurface && connectible;
                    if (!finite_nonnegative4(radiance))
                        status = 2;
                    if (status != 0) {
                        complete = true;
                        nee = false;
                    }
                    if (nee) {
                        Density dd = direct_density;
                        write_nee_request(pool, path, cnt, cp, cbsdf, cwo, latest.position, direct_beta, dd);
                    }
                }
                // A complete path is read again only for its identity, status and radiance (the
                // shadow walk, the film and the packet results), so the rest of its state is not
                // written back.
                if (cnt != old_count) {
                    // preceding = latest; latest = current (shaders/packet_pt_event_body.inc:453-460)
                    flags = (flags & ~(3u << F_PTYPE_SHIFT)) | (latest.type << F_PTYPE_SHIFT);
                    if (!complete) {
                        pool.preceding[path] = make_float4(latest.position.x, latest.position.y, latest.position.z, 0);
                        pool.latest_p[path] =
                            make_float4(cp.position.x, cp.position.y, cp.position.z, cbsdf.g.alpha_x);
                        pool.latest_n[path] =
                            make_float4(cp.shading_normal.x, cp.shading_normal.y, cp.shading_normal.z, cbsdf.g.alpha_y);
                        pool.latest_param[path] =
                            make_float4(cbsdf.param[0], cbsdf.param[1], cbsdf.param[2], cbsdf.param[3]);
                        pool.latest_k[path] = make_float4(cbsdf.k[0], cbsdf.k[1], cbsdf.k[2], cbsdf.k[3]);
                    }
                    flags &= ~((3u << F_LTYPE_SHIFT) | F_LDELTA | (3u << F_LKIND_SHIFT) | (15u << F_LMASK_SHIFT) | F_LSMOOTH);
                    flags |= (ctype << F_LTYPE_SHIFT) | (cdelta ? F_LDELTA : 0u) | ((cbsdf.kind & 3u) << F_LKIND_SHIFT) |
                             ((cbsdf.active_mask & 15u) << F_LMASK_SHIFT) | (cbsdf.g.smooth ? F_LSMOOTH : 0u);
                }
                flags = (flags & ~(F_MASK | F_ROULETTE)) | active_mask | (roulette ? F_ROULETTE : 0u);
                flags = set_status(flags, status) | (complete ? F_COMPLETE : 0u);
                ident.w = flags;
                pool.ident[path] = ident;
                pool.radiance[path] = to_float4(radiance);
                if (!complete) {
                    cursor.z = cnt;
                    pool.cursor[path] = cursor;
                    pool.beta[path] = to_float4(beta);
                    float4 f;
                    int4 e;
                    store_density(density, f, e);
                    pool.dens_f[path] = f;
                    pool.dens_e[path] = e;
                    store_density(hero_previous, f, e);
                    pool.prev_f[path] = f;
                    pool.prev_e[path] = e;
                    pool.eta_scale[path] = to_float4(eta_scale);
                    pool.ray_o[path] = make_float4(ro.x, ro.y, ro.z, 0);
                    pool.ray_d[path] = make_float4(rd.x, rd.y, rd.z, 0);
                }
                keep = !complete;
            }
        }
        const u32 slot = warp_append(out_count, keep);
        if (keep)
            out_queue[slot] = path;
        if (F != 3) {
            const u32 nslot = warp_append(pool.counters + 8 + F, nee);
            if (nee)
                pool.nee_queue[size_t(F) * pool.bin_capacity + nslot] = path;
        }
    }
    if (Adjoint)
        adjoint_end(pool, sgrad);
}

// The light sample of one hero event (hero_direct, shaders/hero_pt_helpers.h:185-221) for the
// paths of BSDF family F whose event asked for one: light selection, the light's point and
// radiance, the BSDF on the light direction, the balance weight, and the visibility segment
// queued for the shadow kernel.  Its own failures (invalid arithmetic) fail the path.  Split
// from the shade kernel, which leaves the request (write_nee_request), so that each kernel
// holds half the live state.
template <int F, int Block = 128, bool Img = true>
__global__ void __launch_bounds__(Block, 512 / Block) k_nee(const __grid_constant__ DeviceScene s,
                                                            const __grid_constant__ WaveParams p, PathPool pool) {
    const u32 count = pool.counters[8 + F];
    const u32 *queue = pool.nee_queue + size_t(F) * pool.bin_capacity;
    const u32 stride = gridDim.x * blockDim.x;
    const u32 trips = (count + stride - 1) / stride;
    for (u32 trip = 0; trip < trips; ++trip) {
        const u32 i = trip * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool shadow = false;
        float4 sh_o = make_float4(0, 0, 0, 0), sh_d = sh_o, sh_c = sh_o, sh_t = sh_o;
        if (i < count) {
            const u32 path = queue[i];
            uint4 ident = pool.ident[path];
            const uint4 cursor = pool.cursor[path];
            const u64 index = (u64(cursor.y) << 32) | cursor.x;
            const V4 lambda = from_float4(pool.lambda[path]);
            u32 cnt;
            SurfacePoint cp;
            HeroBsdf cbsdf;
            V3 cwo, previous;
            V4 direct_beta;
            Density direct_density;
            read_nee_request(pool, path, cnt, cp, cbsdf, cwo, previous, direct_beta, direct_density);
            Latest latest;
            latest.position = previous;
            Frame cframe;
            shading_frame(cp.shading_normal, cframe); // succeeded in the shade kernel
            const bool pair_valid = false;
            const V3 swo = v3(0, 0, 0);
            u32 status = 0;
            {
                        // the light-sample draw: its first word selects the light; the next two, a
                        // point on an area light, are drawn only when an area light was selected
                        // (the same words either way)
                        const u32 block = 133 + cnt - 2;
                        const float u0 = sample_uniform(p, draw_word0(s, p, ident.x, ident.y, ident.z, index, block));
                        // sample_li (shaders/packet_transport.h:470-553)
                        const Selected choice = light_sample(s, cp.position, cp.shading_normal, u0);
                        float u1 = 0, u2 = 0;
                        const bool env_image = Img && s.img.env_image != kNone && choice.light == s.environment_light;
                        if (choice.pmf > 0 && (choice.light < s.emitter_count || env_image)) {
                            const uint4 w = draw_words(s, p, ident.x, ident.y, ident.z, index, block);
                            u1 = sample_uniform(p, w.y);
                            u2 = sample_uniform(p, w.z);
                        }
                        V4 lbeta = v4(0);
                        float spdf = 0;
                        bool li_ok = true, delta_light = false;
                        SurfacePoint lp;
                        lp.position = lp.error = lp.geometric_normal = lp.shading_normal = v3(0, 0, 0);
                        lp.inverse_area_pdf = 0;
                        V3 direction = v3(0, 0, 1);
                        const u32 sel = choice.light;
                        if (choice.pmf > 0) {
                            V4 lrad = v4(0);
                            if (sel < s.emitter_count) {
                                if (!light_geometry_sample(s, sel, cp.position, cp.shading_normal, u1, u2, lp, spdf)) {
                                    li_ok = false;
                                } else {
                                    spdf *= choice.pmf;
                                    const V3 dl = lp.position - cp.position;
                                    const float d2 = dot(dl, dl);
                                    if (lp.inverse_area_pdf == 0 || !(d2 > 0)) {
                                        spdf = 0;
                                    } else {
                                        direction = dl * (1.0f / sqrtf(d2));
                                        const DInstance &li = s.instances[s.emitter_instance[sel]];
                                        if (s.emission_two_sided[li.emission] || dot(lp.geometric_normal, -direction) > 0) {
#pragma unroll
                                            for (int k = 0; k < 4; ++k)
                                                lrad.v[k] = spectrum(s, li.emission * 471u, lambda.v[k]);
                                        }
                                        li_ok = finite_nonnegative4(lrad);
                                    }
                                }
                            } else if (sel < s.emitter_count + s.positional_count) {
                                const DPositional &L = s.positional[sel - s.emitter_count];
                                delta_light = true;
                                lp.position = v3(L.position[0], L.position[1], L.position[2]);
                                const V3 dl = lp.position - cp.position;
                                const float d2 = dot(dl, dl);
                                if (!(d2 > 0)) {
                                    spdf = 0;
                                } else {
                                    direction = dl * (1.0f / sqrtf(d2));
#pragma unroll
                                    for (int k = 0; k < 4; ++k) {
                                        float intensity = spectrum(s, L.spectrum, lambda.v[k]);
                                        if (!positional_intensity(L, direction, intensity))
                                            li_ok = false;
                                        lrad.v[k] = intensity / d2;
                                    }
                                    spdf = choice.pmf;
                                }
                            } else if (env_image) {
                                // the environment image's compensated table
                                // (shaders/packet_transport.h:536-552)
                                float epdf = 0;
                                if (!sample_environment_image(s.img, u1, u2, true, direction, epdf)) {
                                    li_ok = false;
                                } else {
                                    lrad = environment_image_radiance4(s.img, direction, lambda);
                                    spdf = epdf * choice.pmf;
                                    lp.position = cp.position + (2 * s.scene_radius) * direction;
                                    lp.geometric_normal = lp.shading_normal = -direction;
                                }
                            } else {
                                spdf = 0; // constant environment: pdf 0 for unidirectional PT
                            }
                            if (li_ok)
                                lbeta = spdf > 0 ? V4{{lrad.v[0] / spdf, lrad.v[1] / spdf, lrad.v[2] / spdf,
                                                       lrad.v[3] / spdf}}
                                                 : v4(0);
                            li_ok = li_ok && finite_nonnegative4(lbeta);
                        }
                        if (!li_ok || !isfinite(spdf) || spdf < 0) {
                            status = 2;
                        } else if (spdf > 0 && nonzero4(lbeta)) {
                            const HeroEval e = hero_evaluate_k<F == 3 ? 0 : F>(
                                cbsdf, pair_valid ? swo : to_local(cframe, cwo), to_local(cframe, direction));
                            if (!e.valid) {
                                status = 2;
                            } else {
                                const V4 value = scale4(mul4(mul4(direct_beta, e.f), lbeta),
                                                        fabsf(dot(cp.shading_normal, direction)));
                                if (nonzero4(value)) {
                                    V4 contribution = value;
                                    bool weight_ok = true;
                                    if (!delta_light) {
                                        const float sel_pmf = light_pmf(s, cp.position, cp.shading_normal, sel);
                                        const float lpdf =
                                            env_image ? environment_image_pdf(s.img, direction, true) * sel_pmf
                                            : nonzero3(lp.geometric_normal)
                                                ? sel_pmf * light_geometry_pdf(s, sel, cp.position, cp.shading_normal, lp)
                                                : 0.0f;
                                        bool ok;
                                        const V4 bsdf_pdf = represented_pdf<F == 3 ? 0 : F>(
                                            cbsdf, cp.shading_normal, cp.position, latest.position, env_image,
                                            env_image ? direction : lp.position, ok);
                                        weight_ok = ok && hero_weight(direct_density, value, v4(lpdf), bsdf_pdf, contribution);
                                    }
                                    // visible(): offset both endpoints (shaders/packet_transport.h:377-446)
                                    const V3 seg = lp.position - cp.position;
                                    if (!zero3(seg)) {
                                        const V3 so = offset_point(cp.position, cp.error, cp.geometric_normal, seg);
                                        const V3 st = offset_point(lp.position, lp.error, lp.geometric_normal, -seg);
                                        const V3 sd = st - so;
                                        shadow = true;
                                        sh_o = make_float4(so.x, so.y, so.z, kOneMinusEps);
                                        sh_d = make_float4(sd.x, sd.y, sd.z, __uint_as_float(path));
                                        sh_t = make_float4(st.x, st.y, st.z, 0);
                                        sh_c = weight_ok ? to_float4(contribution)
                                                         : make_float4(__int_as_float(0x7fffffff), 0, 0, 0);
                                    }
                                }
                            }
                        }
            }
            if (status != 0) {
                ident.w = set_status(ident.w, status) | F_COMPLETE;
                pool.ident[path] = ident;
                shadow = false;
            }
        }
        const u32 sslot = warp_append(pool.counters + 2, shadow);
        if (shadow) {
            pool.sh_o[sslot] = sh_o;
            pool.sh_d[sslot] = sh_d;
            pool.sh_c[sslot] = sh_c;
            if (pool.sh_t)
                pool.sh_t[sslot] = sh_t;
        }
    }
}

// visible() through pass-through surfaces (shaders/packet_transport.h:393-445): nearest hits
// along the segment; an opaque one occludes, a pass-through one restarts the segment past it
// toward the target (at most boundary_limit + 1 walks).  Returns 0 with `occluded` set, or
// the failed sample's status (3 invalid hit, 2 invalid arithmetic, 4 boundary exhaustion).
template <bool Count, int Stack>
__device__ __noinline__ u32 pass_through_visible(const DeviceScene &s, V3 o, V3 d, float tmax, float4 target4,
                                                 bool &occluded, uint2 *stack, int stride, u32 boundary_limit,
                                                 u32 &nodes, u32 &tris, u32 &rays) {
    const V3 target = v3(target4.x, target4.y, target4.z);
    occluded = true;
    for (u32 crossings = 0; crossings <= boundary_limit; ++crossings) {
        Hit h;
        ++rays;
        if (!walk_closest<Count, Stack, true>(s, o, d, tmax, h, stack, stride, nodes, tris))
            return 3;
        if (h.prim == kNone) {
            occluded = false;
            return 0;
        }
        const u32 inst = s.tri_instance[h.prim];
        const DInstance &in = s.instances[inst];
        if (in.material >= s.material_count)
            return 3;
        if (!(in.resolve & kPassThrough))
            return 0;
        SurfacePoint pt;
        if (!hit_surface_point(s, h.prim, inst, s.tri_local[h.prim], h.b1, h.b2, pt))
            return 2;
        V3 next;
        if (!spawn_boundary(o, d, h.t, pt, normalize3(d), next))
            return 2;
        o = next;
        d = target - next;
    }
    return 4;
}

// Visibility of the light samples (visible(), shaders/packet_transport.h:377-446, opaque surfaces)
// Resolve: the scene has pass-through instances, which shadow rays cross (pass_through_visible).
template <bool Count, int Block = kTraceBlock, bool Adjoint = false, int Stack = kStackDepth, bool Resolve = false>
__global__ void __launch_bounds__(Block, Stack <= kShortStack ? 1024 / Block : 1)
    k_shadow(const __grid_constant__ DeviceScene s, PathPool pool, u32 boundary_limit) {
    __shared__ uint2 stack[Stack * Block];
    extern __shared__ float sgrad[]; // adjoint only
    if (Adjoint)
        adjoint_begin(pool, sgrad);
    const u32 count = pool.counters[2];
    u32 nodes = 0, tris = 0, rays = 0;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float4 o = pool.sh_o[i], d = pool.sh_d[i];
        const u32 path = __float_as_uint(d.w);
        const u32 walks_before = rays;
        bool occluded;
        u32 failure = 0;
        if (Resolve) {
            failure = pass_through_visible<Count, Stack>(s, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), o.w, pool.sh_t[i],
                                                         occluded, stack + threadIdx.x, Block, boundary_limit, nodes,
                                                         tris, rays);
        } else {
            if (!walk_any<Count, Stack, false>(s, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), o.w, occluded, stack + threadIdx.x,
                                        Block, nodes, tris))
                failure = 3;
            ++rays;
        }
        if (Count && pool.lane_shadow)
            pool.lane_shadow[path] += rays - walks_before;
        uint4 ident = pool.ident[path];
        if (failure) {
            ident.w = set_status(ident.w, failure) | F_COMPLETE;
            pool.ident[path] = ident;
            continue;
        }
        if (occluded)
            continue;
        const float4 c = pool.sh_c[i];
        if (isnan(c.x)) {
            ident.w = set_status(ident.w, 2) | F_COMPLETE;
            pool.ident[path] = ident;
            continue;
        }
        float4 r = pool.radiance[path];
        r.x += c.x;
        r.y += c.y;
        r.z += c.z;
        r.w += c.w;
        pool.radiance[path] = r;
        if (!finite_nonnegative4(from_float4(r))) {
            ident.w = set_status(ident.w, 2) | F_COMPLETE;
            pool.ident[path] = ident;
        } else if (Adjoint) {
            // replay: the light sample's gradient, over the history including its vertex
            adjoint_accumulate(s, pool, sgrad, pool.hist[path], from_float4(pool.lambda[path]), from_float4(c),
                               pool.adj_w[path]);
        }
    }
    if (Adjoint)
        adjoint_end(pool, sgrad);
    if (Count) {
        atomicAdd(pool.stats + 4, (unsigned long long)nodes);
        atomicAdd(pool.stats + 5, (unsigned long long)tris);
        atomicAdd(pool.stats + 3, (unsigned long long)rays);
    }
}

// packet_pt_result (shaders/packet_pt_step.h:225-239): 80-byte packet result per lane.  The
// reserved words, which rypath leaves unread, carry the lane's closest-hit and any-hit walk
// counts in counting runs (zero otherwise).
struct PacketResult {
    u32 status, pixel, sample_low, sample_high, splat_count;
    float wavelengths[4], wavelength_pdfs[4], radiance[4];
    float filter_weight;
    u32 reserved[2];
};
__global__ void k_results(PathPool pool, u32 lanes, float filter_weight, PacketResult *out) {
    for (u32 lane = blockIdx.x * blockDim.x + threadIdx.x; lane < lanes; lane += gridDim.x * blockDim.x) {
        const uint4 id = pool.ident[lane];
        const float4 l = pool.lambda[lane], pdf = pool.lambda_pdf[lane], r = pool.radiance[lane];
        PacketResult res;
        res.status = (id.w & F_COMPLETE) ? get_status(id.w) : 2u;
        res.pixel = id.x;
        res.sample_low = id.y;
        res.sample_high = id.z;
        res.splat_count = 0;
        res.wavelengths[0] = l.x;
        res.wavelengths[1] = l.y;
        res.wavelengths[2] = l.z;
        res.wavelengths[3] = l.w;
        res.wavelength_pdfs[0] = pdf.x;
        res.wavelength_pdfs[1] = pdf.y;
        res.wavelength_pdfs[2] = pdf.z;
        res.wavelength_pdfs[3] = pdf.w;
        res.radiance[0] = r.x;
        res.radiance[1] = r.y;
        res.radiance[2] = r.z;
        res.radiance[3] = r.w;
        res.filter_weight = filter_weight;
        res.reserved[0] = pool.lane_closest ? pool.lane_closest[lane] : 0u;
        res.reserved[1] = pool.lane_shadow ? pool.lane_shadow[lane] : 0u;
        out[lane] = res;
    }
}

// Device film pixel: FP64 Neumaier sums (src/packet_film.cpp:10-14, :198-265) plus second moments.
struct FilmPixel {
    double sum[3], correction[3];
    double weight_sum, weight_correction;
    double square[3];
    unsigned long long count;
    double compatibility_sum[3], compatibility_correction[3];
};
// A finite film clamp (on: max_component_value finite and positive).
struct FilmClamp {
    double exposure, max_component_value;
    bool on;
};
RP_DEV void add_compensated(double value, double &sum, double &correction) {
    const double next = __dadd_rn(sum, value);
    correction = __dadd_rn(correction, fabs(sum) >= fabs(value) ? __dadd_rn(__dsub_rn(sum, next), value)
                                                                  : __dadd_rn(__dsub_rn(value, next), sum));
    sum = next;
}
// packet_sensor_xyz (src/packet_film.cpp:102-114) of one lane added to its pixel; false when
// the lane failed (a failed lane fails its batch).
// clamp_sensor + add_xyz into the compatibility planes (src/packet_film.cpp:39-56, :217-220)
RP_DEV void film_add_compatibility(const double (&xyz)[3], double weight, const FilmClamp &c, FilmPixel &f) {
    double v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        v[k] = __dmul_rn(xyz[k], c.exposure);
    double maximum = v[0];
    if (v[1] > maximum)
        maximum = v[1];
    if (v[2] > maximum)
        maximum = v[2];
    if (maximum > c.max_component_value) {
        const double scale = __ddiv_rn(c.max_component_value, maximum);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            v[k] = __dmul_rn(v[k], scale);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
        add_compensated(__dmul_rn(v[k], weight), f.compatibility_sum[k], f.compatibility_correction[k]);
}
RP_DEV bool film_add_lane(const PathPool &pool, u32 lane, const double *cie, double weight, const FilmClamp &clamp,
                          FilmPixel &f) {
    const uint4 id = pool.ident[lane];
    const u32 status = (id.w & F_COMPLETE) ? get_status(id.w) : 2u;
    if (status != 0)
        return false;
    const float4 l4 = pool.lambda[lane], p4 = pool.lambda_pdf[lane], r4 = pool.radiance[lane];
    const float lam[4] = {l4.x, l4.y, l4.z, l4.w}, pdf[4] = {p4.x, p4.y, p4.z, p4.w}, rad[4] = {r4.x, r4.y, r4.z, r4.w};
    double xyz[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (pdf[k] == 0)
            continue;
        const float w = lam[k];
        if (!(w >= 360 && w <= 830))
            continue;
        const u32 row = u32(round(double(w)) - 360.0);
        const double weight = __ddiv_rn(__ddiv_rn(double(rad[k]), double(pdf[k])), 4.0);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            xyz[c] = __dadd_rn(xyz[c], __dmul_rn(weight, __ldg(cie + 3 * row + c)));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double v = __dmul_rn(xyz[c], weight); // add_xyz (src/packet_film.cpp:46-56)
        add_compensated(v, f.sum[c], f.correction[c]);
        f.square[c] = __dadd_rn(f.square[c], __dmul_rn(v, v));
    }
    if (clamp.on)
        film_add_compatibility(xyz, weight, clamp, f);
    add_compensated(weight, f.weight_sum, f.weight_correction);
    ++f.count;
    return true;
}
// Failed lanes of a wave (counters[3]), for passes that produce no film.  counters[3] is
// cleared with the wave's counters, so callers accumulate it per wave.
__global__ void k_count_failures(PathPool pool, u32 lanes) {
    for (u32 lane = blockIdx.x * blockDim.x + threadIdx.x; lane < lanes; lane += gridDim.x * blockDim.x) {
        const u32 w = pool.ident[lane].w;
        if (!(w & F_COMPLETE) || get_status(w) != 0)
            atomicAdd(pool.counters + 3, 1u);
    }
}
// Every sample of a wave reduced per pixel in canonical (absolute sample, pixel) order.
// Owen prefix table (owen_prefix_rounds of every prefix) of the draw blocks [4, 4 + blocks)
// and [133, 133 + blocks), four dimensions each.
__global__ void k_owen_prefix(unsigned short *table, u32 blocks, u32 seed) {
    const u32 total = 2 * blocks * 4 * kOwenPrefixEntries;
    for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const u32 slot = e / (4 * kOwenPrefixEntries), k = (e / kOwenPrefixEntries) & 3u, prefix = e % kOwenPrefixEntries;
        const u32 block = slot < blocks ? 4 + slot : 133 + (slot - blocks);
        table[e] = (unsigned short)owen_prefix_rounds(prefix, sobol_dimension_hash(4 * block + k, seed));
    }
}

__global__ void k_film(PathPool pool, u32 pixel_count, u32 samples, const double *cie, double weight, FilmClamp clamp,
                       FilmPixel *film) {
    for (u32 px = blockIdx.x * blockDim.x + threadIdx.x; px < pixel_count; px += gridDim.x * blockDim.x) {
        FilmPixel f = film[px];
        for (u32 si = 0; si < samples; ++si)
            if (!film_add_lane(pool, si * pixel_count + px, cie, weight, clamp, f))
                atomicAdd(pool.counters + 3, 1u);
        film[px] = f;
    }
}

// The frame sensor of a packet lane (shaders/frame_sensor.h:33-52): raw XYZ of one camera
// sample, sum over the valid wavelength lanes of the matching functions at the nearest
// nanometre times radiance / pdf / 4, in binary32 (the filter weight cancels against its own
// normalisation).  A failed or inconsistent lane (status, identity, a companion terminated
// beside a surviving one, a non-finite value) writes zero and counts a failure.
__global__ void k_frame_packet(PathPool pool, u32 pixel_count, u32 pixel_begin, u32 sample_low, u32 sample_high,
                               const double *cie, float *xyz, u32 *failures) {
    for (u32 px = blockIdx.x * blockDim.x + threadIdx.x; px < pixel_count; px += gridDim.x * blockDim.x) {
        const uint4 id = pool.ident[px];
        bool valid = (id.w & F_COMPLETE) && get_status(id.w) == 0 && id.x == pixel_begin + px && id.y == sample_low &&
                     id.z == sample_high;
        const float4 l4 = pool.lambda[px], p4 = pool.lambda_pdf[px], r4 = pool.radiance[px];
        const float lam[4] = {l4.x, l4.y, l4.z, l4.w}, pdf[4] = {p4.x, p4.y, p4.z, p4.w}, rad[4] = {r4.x, r4.y, r4.z, r4.w};
        bool secondary = false, terminated = false;
        float v[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool good = lam[k] >= 360 && lam[k] <= 830 && isfinite(pdf[k]) && pdf[k] >= 0 && (k != 0 || pdf[k] > 0) &&
                              isfinite(rad[k]) && rad[k] >= 0;
            valid = valid && good;
            if (k > 0) {
                secondary = secondary || pdf[k] > 0;
                terminated = terminated || pdf[k] == 0;
            }
            if (good && pdf[k] > 0) {
                const u32 row = u32(floorf(lam[k] + .5f) - 360.f);
                const float w = rad[k] / pdf[k] / 4.f;
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    v[c] = v[c] + float(__ldg(cie + 3 * row + c)) * w;
            }
        }
        valid = valid && !(secondary && terminated) && isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]);
        if (!valid) {
            v[0] = v[1] = v[2] = 0;
            atomicAdd(failures, 1u);
        }
        xyz[3 * size_t(px)] = v[0];
        xyz[3 * size_t(px) + 1] = v[1];
        xyz[3 * size_t(px) + 2] = v[2];
    }
}

} // namespace rp
