// GPU LBVH construction: world-space triangles, 63-bit Morton codes of their centroids, a
// stable LSB radix sort, Karras's binary radix-tree topology and an atomic bottom-up refit.
// Every step is exact (integer work, min/max), so the tree equals a CPU build of the same
// algorithm bit for bit.
#pragma once

#include "rp_scene.cuh"

namespace rp {

RP_DEV int ordered(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
RP_HD float unordered_host(int i) {
    const int v = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    memcpy(&f, &v, 4);
    return f;
}

struct BuildTmp {
    float4 *box_lo, *box_hi; // per triangle (original order)
    int *cbounds;            // ordered ints: centroid min[3], max[3], then vertex min[3], max[3]
    u64 *keys[2];
    u32 *vals[2];
    u32 *hist;
    u32 *left, *right, *parent, *leaf_parent;
    float4 *node_lo, *node_hi; // internal node bounds
    u32 *flags;
    u32 *error;                // kBuildVertexRange | kBuildTree bits
    u32 *levels;               // most internal nodes on a root-to-leaf path
    u32 *refs;                 // references to internal nodes [0, n-1) and leaves [n-1, 2n-1)
    u32 vertex_count;
};
constexpr u32 kBuildVertexRange = 1, kBuildTree = 2;
// a path from a leaf to the root is shorter than 64 + 32 levels for unique-by-index keys
constexpr int kMaxTreeLevels = 160;

// Flattened triangle i -> (instance, triangle within the instance, BSDF family of its
// material, or kResolveFamily for pass-through and mix-root instances).  prim_begin: the first flattened triangle of each instance (an exclusive prefix
// of the instances' triangle counts), so the instance of i is the last one beginning at or
// before i.
__global__ void k_flatten(const DInstance *instances, const u32 *prim_begin, u32 instance_count,
                          const DMaterial *materials, u32 n, u32 *tri_instance, u32 *tri_local,
                          unsigned char *tri_family) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u32 lo = 0, hi = instance_count;
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) / 2;
            if (prim_begin[mid] <= i)
                lo = mid;
            else
                hi = mid;
        }
        tri_instance[i] = lo;
        tri_local[i] = i - prim_begin[lo];
        const DInstance &in = instances[lo];
        tri_family[i] = (unsigned char)(in.resolve ? kResolveFamily : materials[in.material].scattering);
    }
}

// Block reduction of six (min, max) pairs; pair a < 3 goes to gmin[a], gmax[a], pair a >= 3
// to gmin[a + 3], gmax[a + 3].
RP_DEV void block_min_max(int (&lmin)[6], int (&lmax)[6], int *gmin, int *gmax) {
    __shared__ int smin[6][32], smax[6][32];
#pragma unroll
    for (int a = 0; a < 6; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lmin[a] = min(lmin[a], __shfl_xor_sync(0xffffffffu, lmin[a], o));
            lmax[a] = max(lmax[a], __shfl_xor_sync(0xffffffffu, lmax[a], o));
        }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int a = 0; a < 6; ++a) {
            smin[a][warp] = lmin[a];
            smax[a][warp] = lmax[a];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        int mn = 0x7fffffff, mx = int(0x80000000);
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            mn = min(mn, smin[a][w]);
            mx = max(mx, smax[a][w]);
        }
        atomicMin(gmin + (a < 3 ? a : a + 3), mn);
        atomicMax(gmax + (a < 3 ? a : a + 3), mx);
    }
}

// The world box of procedural primitive `prim`: the patch's corners, or the corners of the
// shape's object box, moved to world space and widened by 2^-18 of their magnitude and extent
// (the hit test runs on the ray moved to object space, whose rounding the slab test must not
// cut off).  False for a patch corner outside the vertex array.
RP_DEV bool procedural_box(const DeviceScene &s, const DInstance &in, u32 prim, u32 vertex_count, V3 &lo, V3 &hi) {
    const float inf = __int_as_float(0x7f800000);
    lo = v3(inf, inf, inf);
    hi = -lo;
    const u32 local = s.tri_local[prim];
    if (prim - s.tri_prims < s.patch_prims) {
        const u32 *pt = s.patches + 4 * size_t(in.patch_begin + local);
        for (int k = 0; k < 4; ++k) {
            if ((unsigned long long)in.vertex_begin + pt[k] >= vertex_count)
                return false;
            const V3 w = world_point(in, load3(s.positions + 3 * size_t(in.vertex_begin + pt[k])));
            lo = v3(fminf(lo.x, w.x), fminf(lo.y, w.y), fminf(lo.z, w.z));
            hi = v3(fmaxf(hi.x, w.x), fmaxf(hi.y, w.y), fmaxf(hi.z, w.z));
        }
    } else {
        float ol[3], oh[3];
        analytic_bounds(s.analytics[in.analytic_begin + local], ol, oh);
        for (int k = 0; k < 8; ++k) {
            const V3 w = world_point(in, v3(k & 1 ? oh[0] : ol[0], k & 2 ? oh[1] : ol[1], k & 4 ? oh[2] : ol[2]));
            lo = v3(fminf(lo.x, w.x), fminf(lo.y, w.y), fminf(lo.z, w.z));
            hi = v3(fmaxf(hi.x, w.x), fmaxf(hi.y, w.y), fmaxf(hi.z, w.z));
        }
    }
    const V3 pad = 0x1p-18f * (v3(fmaxf(fabsf(lo.x), fabsf(hi.x)), fmaxf(fabsf(lo.y), fabsf(hi.y)),
                                  fmaxf(fabsf(lo.z), fabsf(hi.z))) +
                               (hi - lo)) +
                   v3(1e-30f, 1e-30f, 1e-30f);
    lo = lo - pad;
    hi = hi + pad;
    return finite3(lo) && finite3(hi);
}

// World-space vertices, boxes, centroid bounds and vertex bounds of every triangle.  A vertex
// index outside the vertex array sets kBuildVertexRange and is not read.
__global__ void k_tri_prepare(const __grid_constant__ DeviceScene s, float4 *world, BuildTmp t) {
    // [0, 3): centroid axes (into cbounds), [3, 6): vertex axes (into vbounds)
    int lmin[6], lmax[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        lmin[a] = 0x7fffffff;
        lmax[a] = int(0x80000000);
    }
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < s.prim_count; i += gridDim.x * blockDim.x) {
        const DInstance &in = s.instances[s.tri_instance[i]];
        V3 lo, hi;
        if (i >= s.tri_prims) {
            if (!procedural_box(s, in, i, t.vertex_count, lo, hi)) {
                atomicOr(t.error, kBuildVertexRange);
                continue;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k)
                world[3 * size_t(i) + k] = make_float4(0, 0, 0, 0);
        } else {
            const u32 *tri = s.triangles + 3 * size_t(in.triangle_begin + s.tri_local[i]);
            bool valid = true;
#pragma unroll
            for (int k = 0; k < 3; ++k)
                valid = valid && (unsigned long long)in.vertex_begin + tri[k] < t.vertex_count;
            if (!valid) {
                atomicOr(t.error, kBuildVertexRange);
                continue;
            }
            V3 v[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                v[k] = world_point(in, load3(s.positions + 3 * size_t(in.vertex_begin + tri[k])));
                world[3 * size_t(i) + k] = make_float4(v[k].x, v[k].y, v[k].z, 0);
            }
            lo = v3(fminf(fminf(v[0].x, v[1].x), v[2].x), fminf(fminf(v[0].y, v[1].y), v[2].y),
                    fminf(fminf(v[0].z, v[1].z), v[2].z));
            hi = v3(fmaxf(fmaxf(v[0].x, v[1].x), v[2].x), fmaxf(fmaxf(v[0].y, v[1].y), v[2].y),
                    fmaxf(fmaxf(v[0].z, v[1].z), v[2].z));
        }
        t.box_lo[i] = make_float4(lo.x, lo.y, lo.z, 0);
        t.box_hi[i] = make_float4(hi.x, hi.y, hi.z, 0);
        const float c[3] = {0.5f * lo.x + 0.5f * hi.x, 0.5f * lo.y + 0.5f * hi.y, 0.5f * lo.z + 0.5f * hi.z};
        const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lmin[a] = min(lmin[a], ordered(c[a]));
            lmax[a] = max(lmax[a], ordered(c[a]));
            lmin[3 + a] = min(lmin[3 + a], ordered(l[a]));
            lmax[3 + a] = max(lmax[3 + a], ordered(h[a]));
        }
    }
    block_min_max(lmin, lmax, t.cbounds, t.cbounds + 3);
}

RP_DEV u64 spread21(u64 x) {
    x &= 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
// Sort key of a triangle: the 63-bit Morton code of its centroid, with bit 63 set for a large
// triangle (a box side longer than 1/16 of the largest centroid extent).  Large triangles then
// sort after all others and Karras's topology splits them off at the root, so their boxes do
// not inflate the nodes above the small triangles near their centroids (a ground plane of two
// triangles would otherwise widen every node on its two root-to-leaf paths).
__global__ void k_morton(u32 n, BuildTmp t, float3 lo, float3 ext) {
    const float large = fmaxf(fmaxf(ext.x, ext.y), ext.z) * 0.0625f;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 bl = t.box_lo[i], bh = t.box_hi[i];
        const bool is_large = bh.x - bl.x > large || bh.y - bl.y > large || bh.z - bl.z > large;
        const float c[3] = {0.5f * bl.x + 0.5f * bh.x, 0.5f * bl.y + 0.5f * bh.y, 0.5f * bl.z + 0.5f * bh.z};
        const float l[3] = {lo.x, lo.y, lo.z}, e[3] = {ext.x, ext.y, ext.z};
        u64 q[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float tt = e[a] > 0 ? (c[a] - l[a]) / e[a] : 0.0f;
            float cell = tt * 2097152.0f;
            cell = fminf(fmaxf(cell, 0.0f), 2097151.0f);
            q[a] = u64(cell);
        }
        t.keys[0][i] = (is_large ? 1ull << 63 : 0ull) | (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
        t.vals[0][i] = i;
    }
}

// ---- stable LSB radix sort, 8-bit digits, tiles of 256 threads x 8 items
constexpr int kSortThreads = 256, kSortItems = 8, kSortTile = kSortThreads * kSortItems;

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const u64 *keys, u32 n, int shift, u32 *hist, u32 tiles) {
    __shared__ u32 h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const u32 base = blockIdx.x * kSortTile;
    for (int c = 0; c < kSortItems; ++c) {
        const u32 i = base + c * kSortThreads + threadIdx.x;
        if (i < n)
            atomicAdd(h + u32((keys[i] >> shift) & 0xff), 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}
// exclusive scan of hist (digit-major) in one block
__global__ void __launch_bounds__(1024) k_radix_scan(u32 *hist, u32 total) {
    __shared__ u32 warp_sums[32];
    __shared__ u32 carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (u32 base = 0; base < total; base += 1024) {
        const u32 i = base + threadIdx.x;
        const u32 v = i < total ? hist[i] : 0;
        u32 x = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            u32 w = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const u32 y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o)
                    w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const u32 incl = x + (warp > 0 ? warp_sums[warp - 1] : 0) + carry;
        if (i < total)
            hist[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry = incl;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const u64 *kin, const u32 *vin, u64 *kout, u32 *vout,
                                                                 u32 n, int shift, const u32 *hist, u32 tiles) {
    __shared__ u32 digit_base[256];
    __shared__ u32 warp_counts[kSortThreads / 32][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    digit_base[threadIdx.x] = hist[threadIdx.x * tiles + blockIdx.x];
    for (int w = 0; w < kSortThreads / 32; ++w)
        warp_counts[w][threadIdx.x] = 0;
    __syncthreads();
    const u32 base = blockIdx.x * kSortTile;
    for (int c = 0; c < kSortItems; ++c) {
        const u32 i = base + c * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const u64 key = valid ? kin[i] : 0;
        const u32 val = valid ? vin[i] : 0;
        const u32 d = valid ? u32((key >> shift) & 0xff) : 0x100u;
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 rank = __popc(peers & ((1u << lane) - 1));
        if (valid && rank == 0)
            warp_counts[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            u32 offset = digit_base[d] + rank;
            for (int w = 0; w < warp; ++w)
                offset += warp_counts[w][d];
            kout[offset] = key;
            vout[offset] = val;
        }
        __syncthreads();
        u32 sum = 0;
        for (int w = 0; w < kSortThreads / 32; ++w) {
            sum += warp_counts[w][threadIdx.x];
            warp_counts[w][threadIdx.x] = 0;
        }
        digit_base[threadIdx.x] += sum;
        __syncthreads();
    }
}

// Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees and k-d trees".
RP_DEV int karras_delta(const u64 *keys, u32 n, long i, long j) {
    if (j < 0 || j >= long(n))
        return -1;
    const u64 a = keys[i], c = keys[j];
    if (a != c)
        return __clzll(a ^ c);
    return 64 + __clz(u32(i) ^ u32(j));
}
__global__ void k_karras(const u64 *keys, u32 n, BuildTmp t) {
    for (u32 ii = blockIdx.x * blockDim.x + threadIdx.x; ii + 1 < n; ii += gridDim.x * blockDim.x) {
        const long i = ii;
        const int d = (karras_delta(keys, n, i, i + 1) - karras_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = karras_delta(keys, n, i, i - d);
        long lmax = 2;
        while (karras_delta(keys, n, i, i + lmax * d) > dmin)
            lmax *= 2;
        long l = 0;
        for (long s = lmax / 2; s >= 1; s /= 2)
            if (karras_delta(keys, n, i, i + (l + s) * d) > dmin)
                l += s;
        const long j = i + l * d;
        const int dnode = karras_delta(keys, n, i, j);
        long s = 0;
        for (long div = 2;; div *= 2) {
            const long step = (l + div - 1) / div;
            if (karras_delta(keys, n, i, i + (s + step) * d) > dnode)
                s += step;
            if (step == 1)
                break;
        }
        const long gamma = i + s * d + (d < 0 ? d : 0);
        const long first = i < j ? i : j, last = i < j ? j : i;
        const u32 lc = first == gamma ? (kLeaf | u32(gamma)) : u32(gamma);
        const u32 rc = last == gamma + 1 ? (kLeaf | u32(gamma + 1)) : u32(gamma + 1);
        t.left[i] = lc;
        t.right[i] = rc;
        if (lc & kLeaf)
            t.leaf_parent[lc & ~kLeaf] = u32(i);
        else
            t.parent[lc] = u32(i);
        if (rc & kLeaf)
            t.leaf_parent[rc & ~kLeaf] = u32(i);
        else
            t.parent[rc] = u32(i);
    }
}
// Bottom-up refit: the second child to arrive at a node writes its bounds.
__global__ void k_refit(u32 n, const u32 *order, BuildTmp t) {
    for (u32 slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        u32 node = t.leaf_parent[slot];
        for (int level = 0; node != kNone && level < kMaxTreeLevels; ++level) {
            __threadfence();
            if (atomicAdd(t.flags + node, 1u) == 0)
                break;
            __threadfence();
            float4 lo[2], hi[2];
            const u32 ch[2] = {t.left[node], t.right[node]};
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (ch[k] & kLeaf) {
                    const u32 prim = order[ch[k] & ~kLeaf];
                    lo[k] = __ldcg(t.box_lo + prim);
                    hi[k] = __ldcg(t.box_hi + prim);
                } else {
                    lo[k] = __ldcg(t.node_lo + ch[k]);
                    hi[k] = __ldcg(t.node_hi + ch[k]);
                }
            }
            __stcg(t.node_lo + node, make_float4(fminf(lo[0].x, lo[1].x), fminf(lo[0].y, lo[1].y), fminf(lo[0].z, lo[1].z), 0));
            __stcg(t.node_hi + node, make_float4(fmaxf(hi[0].x, hi[1].x), fmaxf(hi[0].y, hi[1].y), fmaxf(hi[0].z, hi[1].z), 0));
            node = t.parent[node];
        }
    }
}
// Traversal layout: child boxes inside each node; leaf triangles in leaf-slot order.
__global__ void k_pack(u32 n, const u32 *order, const float4 *world, BuildTmp t, BNode *nodes, float4 *leaf_v) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u32 prim = order[i];
        const float4 a = world[3 * prim];
        leaf_v[3 * i] = make_float4(a.x, a.y, a.z, __uint_as_float(prim));
        leaf_v[3 * i + 1] = world[3 * prim + 1];
        leaf_v[3 * i + 2] = world[3 * prim + 2];
        if (i + 1 < n) {
            float4 lo[2], hi[2];
            const u32 ch[2] = {t.left[i], t.right[i]};
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (ch[k] & kLeaf) {
                    const u32 p = order[ch[k] & ~kLeaf];
                    lo[k] = t.box_lo[p];
                    hi[k] = t.box_hi[p];
                } else {
                    lo[k] = t.node_lo[ch[k]];
                    hi[k] = t.node_hi[ch[k]];
                }
            }
            BNode b;
            b.a = make_float4(lo[0].x, lo[0].y, lo[0].z, hi[0].x);
            b.b = make_float4(hi[0].y, hi[0].z, lo[1].x, lo[1].y);
            b.c = make_float4(lo[1].z, hi[1].x, hi[1].y, hi[1].z);
            b.d = make_uint4(ch[0], ch[1], 0, 0);
            nodes[i] = b;
        }
    }
}

// ---- compressed 8-wide tree, collapsed top-down from the binary one
struct WideBuild {
    const u32 *left, *right;          // binary topology
    const float4 *node_lo, *node_hi;  // binary internal boxes
    const float4 *box_lo, *box_hi;    // triangle boxes (original order)
    const u32 *order;                 // leaf slot -> triangle
    const float4 *leaf_v;             // triangles by leaf slot
    WNode *wnodes;
    float4 *wtri;
    u32 *counters;                    // [0] wide nodes, [1] wide leaves, [2] [3] level queue lengths, [4] error, [5] levels
    uint2 *queue[2];                  // (binary internal node, wide node index) per level
    u32 capacity;                     // wide nodes available (binary internal nodes)
    u32 n;                            // triangles
};

RP_DEV float box_area(float4 lo, float4 hi) {
    const float x = hi.x - lo.x, y = hi.y - lo.y, z = hi.z - lo.z;
    return x * y + y * z + z * x;
}

// Biased exponent of the power-of-two step that spans [lo, hi] in 255 steps, and the 8-bit
// bounds of every child along this axis: each plane lo + q step (in real arithmetic, checked
// with directed rounding) is at or below the child's low bound (or at or above its high
// bound).  A larger step is taken when 255 steps fall short.
RP_DEV u32 quantize_axis(float lo, float hi, const float *clo, const float *chi, int count, unsigned char *qlo,
                         unsigned char *qhi) {
    const float extent = hi - lo;
    int e = -126;
    if (extent > 0 && isfinite(extent)) {
        frexpf(extent / 255.0f, &e); // extent / 255 < 2^e
        e = max(e, -126);
    }
    for (; e <= 127; ++e) {
        const float step = __uint_as_float(u32(e + 127) << 23);
        bool ok = true;
        for (int k = 0; k < count && ok; ++k) {
            // clamped in float first: a NaN bound clamps to 0 (and a NaN decode never passes)
            int a = int(fminf(fmaxf(floorf((clo[k] - lo) / step), 0.0f), 255.0f));
            int b = int(fminf(fmaxf(ceilf((chi[k] - lo) / step), 0.0f), 255.0f));
            // the real planes lo + q step: at or below clo, at or above chi
            while (a > 0 && !(__fmaf_ru(float(a), step, lo) <= clo[k]))
                --a;
            while (b < 255 && !(__fmaf_rd(float(b), step, lo) >= chi[k]))
                ++b;
            ok = __fmaf_rd(float(b), step, lo) >= chi[k] || !(chi[k] == chi[k]);
            qlo[k] = (unsigned char)a;
            qhi[k] = (unsigned char)b;
        }
        if (ok)
            break;
    }
    return u32(min(e, 127) + 127);
}

// One level of the collapse: each queued binary node becomes a wide node of up to 8 children,
// expanding the internal child of largest surface area until 8 are reached or none is left.
// Internal children are queued for the next level with the wide indices allocated for them.
__global__ void k_wide_level(WideBuild w, int parity, u32 level) {
    const u32 count = min(w.counters[2 + parity], w.capacity); // an overflowing level has set the error bit
    const uint2 *in = w.queue[parity];
    uint2 *out = w.queue[parity ^ 1];
    u32 *out_count = w.counters + 2 + (parity ^ 1);
    if (count && blockIdx.x == 0 && threadIdx.x == 0)
        atomicMax(w.counters + 5, level + 1);
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint2 item = in[i];
        u32 ch[8];
        int nc = 2;
        ch[0] = w.left[item.x];
        ch[1] = w.right[item.x];
        while (nc < 8) {
            int best = -1;
            float best_area = -1;
            for (int k = 0; k < nc; ++k)
                if (!(ch[k] & kLeaf)) {
                    const float a = box_area(w.node_lo[ch[k]], w.node_hi[ch[k]]);
                    if (a > best_area) {
                        best_area = a;
                        best = k;
                    }
                }
            if (best < 0)
                break;
            const u32 c = ch[best];
            ch[best] = w.left[c];
            ch[nc++] = w.right[c];
        }
        // child boxes and the node box
        float4 lo[8], hi[8];
        float4 nlo = make_float4(INFINITY, INFINITY, INFINITY, 0), nhi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0);
        for (int k = 0; k < nc; ++k) {
            if (ch[k] & kLeaf) {
                const u32 prim = w.order[ch[k] & ~kLeaf];
                lo[k] = w.box_lo[prim];
                hi[k] = w.box_hi[prim];
            } else {
                lo[k] = w.node_lo[ch[k]];
                hi[k] = w.node_hi[ch[k]];
            }
            nlo = make_float4(fminf(nlo.x, lo[k].x), fminf(nlo.y, lo[k].y), fminf(nlo.z, lo[k].z), 0);
            nhi = make_float4(fmaxf(nhi.x, hi[k].x), fmaxf(nhi.y, hi[k].y), fmaxf(nhi.z, hi[k].z), 0);
        }
        // slots: each child to the free slot whose octant direction best matches its offset
        // from the node centre (children with the largest offsets choose first)
        const float cx = 0.5f * nlo.x + 0.5f * nhi.x, cy = 0.5f * nlo.y + 0.5f * nhi.y, cz = 0.5f * nlo.z + 0.5f * nhi.z;
        float ox[8], oy[8], oz[8];
        int slot_of[8];
        bool placed[8];
        for (int k = 0; k < nc; ++k) {
            ox[k] = (0.5f * lo[k].x + 0.5f * hi[k].x) - cx;
            oy[k] = (0.5f * lo[k].y + 0.5f * hi[k].y) - cy;
            oz[k] = (0.5f * lo[k].z + 0.5f * hi[k].z) - cz;
            placed[k] = false;
        }
        u32 used = 0;
        for (int round = 0; round < nc; ++round) {
            int pick = -1;
            float reach = -1;
            for (int k = 0; k < nc; ++k)
                if (!placed[k]) {
                    const float m = fabsf(ox[k]) + fabsf(oy[k]) + fabsf(oz[k]);
                    if (m > reach) {
                        reach = m;
                        pick = k;
                    }
                }
            int best_slot = -1;
            float best_score = -INFINITY;
            for (int sl = 0; sl < 8; ++sl)
                if (!((used >> sl) & 1u)) {
                    const float score = ((sl & 1) ? ox[pick] : -ox[pick]) + ((sl & 2) ? oy[pick] : -oy[pick]) +
                                        ((sl & 4) ? oz[pick] : -oz[pick]);
                    if (score > best_score) {
                        best_score = score;
                        best_slot = sl;
                    }
                }
            placed[pick] = true;
            slot_of[pick] = best_slot;
            used |= 1u << best_slot;
        }
        int child_at[8];
        for (int sl = 0; sl < 8; ++sl)
            child_at[sl] = -1;
        for (int k = 0; k < nc; ++k)
            child_at[slot_of[k]] = k;
        u32 imask = 0, lmask = 0, internal = 0, leaves = 0;
        for (int sl = 0; sl < 8; ++sl)
            if (child_at[sl] >= 0) {
                if (ch[child_at[sl]] & kLeaf) {
                    lmask |= 1u << sl;
                    ++leaves;
                } else {
                    imask |= 1u << sl;
                    ++internal;
                }
            }
        const u32 base = internal ? atomicAdd(w.counters + 0, internal) : 0;
        const u32 tri_base = leaves ? atomicAdd(w.counters + 1, leaves) : 0;
        if (base + internal > w.capacity || tri_base + leaves > w.n) {
            atomicOr(w.counters + 4, 1u);
            continue;
        }
        // quantized bounds, slot order
        float clo[8], chi[8];
        unsigned char q[6][8];
        for (int sl = 0; sl < 8; ++sl)
            for (int a = 0; a < 6; ++a)
                q[a][sl] = 0;
        u32 ebytes = 0;
        const float nl[3] = {nlo.x, nlo.y, nlo.z}, nh[3] = {nhi.x, nhi.y, nhi.z};
        for (int a = 0; a < 3; ++a) {
            int m = 0;
            int slots[8];
            for (int sl = 0; sl < 8; ++sl)
                if (child_at[sl] >= 0) {
                    const int k = child_at[sl];
                    clo[m] = a == 0 ? lo[k].x : a == 1 ? lo[k].y : lo[k].z;
                    chi[m] = a == 0 ? hi[k].x : a == 1 ? hi[k].y : hi[k].z;
                    slots[m++] = sl;
                }
            unsigned char ql[8], qh[8];
            const u32 eb = quantize_axis(nl[a], nh[a], clo, chi, m, ql, qh);
            ebytes |= eb << (8 * a);
            for (int j = 0; j < m; ++j) {
                q[a][slots[j]] = ql[j];
                q[3 + a][slots[j]] = qh[j];
            }
        }
        auto pack = [&](int row, int half) {
            u32 v = 0;
            for (int b = 0; b < 4; ++b)
                v |= u32(q[row][4 * half + b]) << (8 * b);
            return v;
        };
        WNode node;
        node.origin = make_float4(nlo.x, nlo.y, nlo.z, __uint_as_float(ebytes | (imask << 24)));
        node.links = make_uint4(base, tri_base, lmask, 0);
        node.q0 = make_uint4(pack(0, 0), pack(0, 1), pack(1, 0), pack(1, 1));
        node.q1 = make_uint4(pack(2, 0), pack(2, 1), pack(3, 0), pack(3, 1));
        node.q2 = make_uint4(pack(4, 0), pack(4, 1), pack(5, 0), pack(5, 1));
        w.wnodes[item.y] = node;
        u32 ji = 0, jl = 0;
        for (int sl = 0; sl < 8; ++sl) {
            const int k = child_at[sl];
            if (k < 0)
                continue;
            if (ch[k] & kLeaf) {
                const u32 slot = ch[k] & ~kLeaf, dst = tri_base + jl++;
                w.wtri[3 * size_t(dst)] = w.leaf_v[3 * size_t(slot)];
                w.wtri[3 * size_t(dst) + 1] = w.leaf_v[3 * size_t(slot) + 1];
                w.wtri[3 * size_t(dst) + 2] = w.leaf_v[3 * size_t(slot) + 2];
            } else {
                const u32 at = atomicAdd(out_count, 1u);
                if (at < w.capacity)
                    out[at] = make_uint2(ch[k], base + ji);
                else
                    atomicOr(w.counters + 4, 1u);
                ++ji;
            }
        }
    }
}

// Structural check of the topology before any traversal.  k_tree_refs counts the references
// to every internal node and leaf (a child index out of range sets kBuildTree); k_tree_verify
// requires exactly one reference to each node but the root (none) and each leaf, and a walk
// from every leaf up its parents that reaches the root within kMaxTreeLevels.  Together they
// make the topology a tree of all 2n - 1 nodes: a part unreachable from the root would give
// one of its leaves a parent chain that never reaches the root.  Traversal loops are then
// finite, and k_refit (bounded by the same level count) has refit every node.
__global__ void k_tree_refs(u32 n, BuildTmp t) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x) {
        const u32 ch[2] = {t.left[i], t.right[i]};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const u32 c = ch[k] & ~kLeaf;
            const bool leaf = (ch[k] & kLeaf) != 0;
            if (leaf ? c >= n : c >= n - 1) {
                atomicOr(t.error, kBuildTree);
                continue;
            }
            atomicAdd(t.refs + (leaf ? n - 1 + c : c), 1u);
        }
    }
}
__global__ void k_tree_verify(u32 n, BuildTmp t) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n - 1; i += gridDim.x * blockDim.x) {
        if (t.refs[i] != (i == 0 ? 0u : 1u)) {
            atomicOr(t.error, kBuildTree);
            continue;
        }
        if (i < n - 1)
            continue;
        u32 node = t.leaf_parent[i - (n - 1)];
        int level = 0;
        while (node != 0 && node < n - 1 && level + 1 < kMaxTreeLevels) {
            node = t.parent[node];
            ++level;
        }
        if (node != 0)
            atomicOr(t.error, kBuildTree);
        else
            atomicMax(t.levels, u32(level + 1));
    }
}

} // namespace rp
