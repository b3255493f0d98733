// Batched rendering: many camera views of one scene, of uneven resolution and sample count,
// rendered as one wavefront.  The batch's lanes are the concatenation, view by view, of each
// view's (absolute sample, pixel) lanes in canonical order; a wave is a contiguous range of
// them, so small views share waves instead of each running a short, launch-bound wavefront.
// Every lane is the lane the view would have in a plain render (same pixel, sample index,
// Sobol index and camera ray), so each view's film equals its plain render bit for bit.
//
// The per-wave kernel sequence reads its wave from a device table and the last kernel of
// the wave advances the wave cursor, so one CUDA graph of the sequence replays every wave.
#pragma once

#include "rp_kernels.cuh"

namespace rp {

struct DView {
    RasterCam cam;
    u32 width, height, m, pixels;   // m: Sobol scale exponent of the view's film
    u32 sample_low, sample_high;    // first absolute sample of the view in this batch
    u32 spp, pad;                   // samples of the view in this batch
    unsigned long long lane_begin;  // first batch lane of the view
    unsigned long long film_begin;  // first film pixel of the view
};
struct WaveDesc {
    unsigned long long lane_begin; // first batch lane of the wave
    u32 lanes, pad;
};
struct Batch {
    const DView *views;
    u32 view_count;
    const WaveDesc *waves;
    u32 *cursor;   // [0] current wave, [1] failed lanes
    unsigned long long film_pixels;
};

// last view whose first lane (or film pixel) is <= x
RP_DEV u32 find_view_by_lane(const Batch &b, unsigned long long x) {
    u32 lo = 0, hi = b.view_count;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) / 2;
        if (b.views[mid].lane_begin <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}
RP_DEV u32 find_view_by_pixel(const Batch &b, unsigned long long x) {
    u32 lo = 0, hi = b.view_count;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) / 2;
        if (b.views[mid].film_begin <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Camera rays of the current wave: batch lane -> (view, sample, pixel) -> raygen_lane with
// the view's film and camera.  Also sets the wave's active-queue length.
__global__ void k_raygen_views(const __grid_constant__ DeviceScene s, const __grid_constant__ WaveParams base, Batch b,
                               PathPool pool) {
    const WaveDesc w = b.waves[*b.cursor];
    if (blockIdx.x == 0 && threadIdx.x == 0)
        pool.counters[0] = w.lanes;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < w.lanes; i += gridDim.x * blockDim.x) {
        const unsigned long long g = w.lane_begin + i;
        const DView &v = b.views[find_view_by_lane(b, g)];
        const unsigned long long local = g - v.lane_begin;
        const u32 sample = u32(local / v.pixels), px = u32(local % v.pixels);
        const unsigned long long absolute = ((unsigned long long)v.sample_high << 32 | v.sample_low) + sample;
        WaveParams p = base;
        p.width = v.width;
        p.height = v.height;
        p.m = v.m;
        p.pixel_begin = 0;
        p.pixel_count = v.pixels;
        p.sample_low = u32(absolute);
        p.sample_high = u32(absolute >> 32);
        raygen_lane(s, v.cam, p, px, i, pool);
    }
}

// The current wave's samples reduced into the batch film, per view pixel in canonical order
// (k_film), then the wave cursor advances.  film == nullptr: count failures only (tuning).
__global__ void k_film_views(PathPool pool, Batch b, const double *cie, double weight, FilmClamp clamp,
                             FilmPixel *film) {
    const WaveDesc w = b.waves[*b.cursor];
    const unsigned long long first = w.lane_begin, last = w.lane_begin + w.lanes; // [first, last)
    // the views the wave overlaps are contiguous, and so are their film pixels
    const DView &va = b.views[find_view_by_lane(b, first)], &vb = b.views[find_view_by_lane(b, last - 1)];
    const unsigned long long slot_end = vb.film_begin + vb.pixels;
    for (unsigned long long slot = va.film_begin + blockIdx.x * blockDim.x + threadIdx.x; slot < slot_end;
         slot += gridDim.x * blockDim.x) {
        const DView &v = b.views[find_view_by_pixel(b, slot)];
        const unsigned long long px = slot - v.film_begin;
        if (px >= v.pixels)
            continue; // a gap between view films
        const unsigned long long base = v.lane_begin + px; // lane of sample 0
        const unsigned long long span = (unsigned long long)v.spp * v.pixels;
        if (last <= base || first >= v.lane_begin + span)
            continue;
        // samples s with first <= base + s * pixels < last
        const unsigned long long s0 = first <= base ? 0 : (first - base + v.pixels - 1) / v.pixels;
        unsigned long long s1 = (last - 1 - base) / v.pixels + 1;
        if (s1 > v.spp)
            s1 = v.spp;
        if (s0 >= s1)
            continue;
        FilmPixel f;
        if (film)
            f = film[slot];
        for (unsigned long long si = s0; si < s1; ++si) {
            const u32 lane = u32(base + si * v.pixels - first);
            FilmPixel scratch{};
            if (!film_add_lane(pool, lane, cie, weight, clamp, film ? f : scratch))
                atomicAdd(b.cursor + 1, 1u);
        }
        if (film)
            film[slot] = f;
    }
}

// Advances the wave cursor once every kernel of the wave has run (the graph's last node).
__global__ void k_next_wave(Batch b) {
    if (threadIdx.x == 0)
        ++b.cursor[0];
}

} // namespace rp
