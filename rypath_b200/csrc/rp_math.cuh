// Device arithmetic of the hero spectral path: sampling words, wavelength sampling,
// scaled-likelihood MIS, Russian roulette and the diffuse / GGX conductor / GGX dielectric
// BSDFs.  Each function names the rypath source it reproduces.  The translation unit is
// compiled with --fmad=false so binary32 expressions round exactly as written; where rypath
// calls fma() explicitly, so does this code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rp {

typedef uint32_t u32;
typedef uint64_t u64;

#define RP_DEV __device__ __forceinline__
#define RP_HD __host__ __device__ __forceinline__

constexpr float kPi = 3.14159265358979323846f;
constexpr float kOneMinusEps = 0x1.fffffep-1f;
constexpr float kFltMin = 1.17549435e-38f;
constexpr float kFltEps = 1.1920929e-7f;

// ------------------------------------------------------------------ vectors
struct V3 {
    float x, y, z;
};
RP_HD V3 v3(float x, float y, float z) { return {x, y, z}; }
RP_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
RP_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
RP_HD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
RP_HD V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
RP_HD V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
RP_HD V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
RP_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RP_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
RP_DEV V3 vabs(V3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
RP_DEV bool finite3(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
RP_DEV bool zero3(V3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
RP_DEV bool nonzero3(V3 a) { return a.x != 0 || a.y != 0 || a.z != 0; }
RP_DEV bool eq3(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
RP_DEV float length3(V3 a) { return sqrtf(dot(a, a)); }
RP_DEV V3 normalize3(V3 a) { return a / sqrtf(dot(a, a)); }
RP_DEV float max3(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
RP_DEV V3 fma3(V3 a, V3 b, V3 c) { return {fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z)}; }
RP_DEV float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct V4 {
    float v[4];
};
RP_DEV V4 v4(float s) { return {{s, s, s, s}}; }
RP_DEV V4 mul4(V4 a, V4 b) { return {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
RP_DEV V4 scale4(V4 a, float s) { return {{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
RP_DEV V4 add4(V4 a, V4 b) { return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}}; }
// shaders/packet_transport.h:49-50
RP_DEV bool nonzero4(V4 a) { return a.v[0] > 0 || a.v[1] > 0 || a.v[2] > 0 || a.v[3] > 0; }
RP_DEV bool finite_nonnegative4(V4 a) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (!isfinite(a.v[i]) || !(a.v[i] >= 0))
            return false;
    return true;
}
RP_DEV V4 from_float4(float4 a) { return {{a.x, a.y, a.z, a.w}}; }
RP_DEV float4 to_float4(V4 a) { return make_float4(a.v[0], a.v[1], a.v[2], a.v[3]); }

RP_DEV u32 fbits(float x) { return __float_as_uint(x); }
RP_DEV float ffrom(u32 x) { return __uint_as_float(x); }

// ------------------------------------------------------------------ Sobol (src/sobol_shared.h)
constexpr u32 kSobolMatrix = 52;
struct SobolTables {
    const u32 *directions; // 1024 x 52
    const u64 *intervals;  // 25 x 52
    const u64 *inverse;    // 26 x 52
};
// src/sobol_shared.h:56-76
RP_DEV u64 sobol_index(const SobolTables &t, u32 m, u32 x, u32 y, u64 sample) {
    if (m == 0)
        return sample;
    const u32 row = (m - 1) * kSobolMatrix;
    u64 result = sample << (2 * m);
    u64 delta = 0;
    for (u32 c = row; sample != 0; ++c, sample >>= 1)
        if (sample & 1)
            delta ^= __ldg(t.intervals + c);
    u64 bits = ((u64(x) << m) | y) ^ delta;
    for (u32 c = row; bits != 0; ++c, bits >>= 1)
        if (bits & 1)
            result ^= __ldg(t.inverse + c);
    return result;
}
// src/sobol_shared.h:79-89
RP_DEV u32 sobol_dimension_hash(u32 dimension, u32 seed) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    u64 block = ((u64(seed) << 32) | dimension) * m;
    block ^= block >> 47;
    block *= m;
    u64 h = (8 * m ^ block) * m;
    h ^= h >> 47;
    h *= m;
    return u32(h ^ (h >> 47));
}
// src/sobol_shared.h:99-105
RP_DEV u64 mix_bits(u64 v) {
    v ^= v >> 31;
    v *= 0x7fb5d329728ea185ull;
    v ^= v >> 27;
    v *= 0x81dadef4bc2dd44dull;
    return v ^ (v >> 33);
}
// XOR of the direction numbers selected by the set bits of the index: the generator-matrix
// product of src/sobol_shared.h:110-114, walking set bits with ffs.
RP_DEV u32 sobol_raw(const SobolTables &t, u64 index, u32 dimension) {
    u32 value = 0;
    const u32 *col = t.directions + dimension * kSobolMatrix;
    u32 lo = u32(index), hi = u32(index >> 32);
    while (lo) {
        const int b = __ffs(lo) - 1;
        value ^= __ldg(col + b);
        lo &= lo - 1;
    }
    while (hi) {
        const int b = __ffs(hi) - 1;
        value ^= __ldg(col + 32 + b);
        hi &= hi - 1;
    }
    return value;
}
// The randomisations of a 32-bit sample word with a 32-bit hash: none, permute digits (xor),
// fast Owen (Laine-Karras style hash), Owen (src/sobol_shared.h:115-141, src/qmc_shared.h:190-212)
RP_DEV u32 scramble_word(u32 value, u32 mode, u32 hash) {
    if (mode == 0)
        return value;
    if (mode == 1)
        return value ^ hash;
    if (mode == 2) {
        value = __brev(value);
        value ^= value * 0x3d20adeau;
        value += hash;
        value *= (hash >> 16) | 1;
        value ^= value * 0x05526c56u;
        value ^= value * 0x53a22864u;
        return __brev(value);
    }
    value ^= (hash & 1) << 31;
#pragma unroll 1
    for (u32 bit = 1; bit < 32; ++bit) {
        const u32 prefix = value & (~u32(0) << (32 - bit));
        if (u32(mix_bits(prefix ^ hash)) & (u32(1) << bit))
            value ^= u32(1) << (31 - bit);
    }
    return value;
}
// src/sobol_shared.h:108-141
RP_DEV u32 sobol_word(const SobolTables &t, u64 index, u32 dimension, u32 mode, u32 seed) {
    const u32 value = sobol_raw(t, index, dimension);
    if (mode == 0)
        return value;
    return scramble_word(value, mode, sobol_dimension_hash(dimension, seed));
}
// Owen scrambling rounds 0 .. kOwenPrefixBits - 1 decide the top kOwenPrefixBits bits of a
// word from those bits alone (round b flips bit 31 - b from the b bits above it), so a table
// of every prefix per dimension replaces them.
constexpr u32 kOwenPrefixBits = 12, kOwenPrefixEntries = 1u << kOwenPrefixBits;
RP_DEV u32 owen_prefix_rounds(u32 prefix, u32 hash) {
    u32 value = (prefix << (32 - kOwenPrefixBits)) ^ ((hash & 1) << 31);
    for (u32 bit = 1; bit < kOwenPrefixBits; ++bit)
        if (u32(mix_bits((value & (~u32(0) << (32 - bit))) ^ hash)) & (u32(1) << bit))
            value ^= u32(1) << (31 - bit);
    return value >> (32 - kOwenPrefixBits);
}
// Four consecutive dimensions [dimension, dimension + 4) of one Sobol index, each equal to
// sobol_word of its dimension.  `prefix` (optional, Owen only): the four dimensions' tables of
// owen_prefix_rounds, kOwenPrefixEntries entries each.  The four generator products share the walk over the index
// bits, and the four Owen bit loops run in lockstep: each loop is a chain of dependent 64-bit
// hashes, so four independent chains keep the pipelines busy where one would stall on each
// hash.
RP_DEV uint4 sobol_words4(const SobolTables &t, u64 index, u32 dimension, u32 mode, u32 seed,
                          const unsigned short *prefix = nullptr) {
    const u32 *col = t.directions + dimension * kSobolMatrix;
    u32 v[4] = {0, 0, 0, 0};
    u32 lo = u32(index), hi = u32(index >> 32);
    while (lo) {
        const int b = __ffs(lo) - 1;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] ^= __ldg(col + k * kSobolMatrix + b);
        lo &= lo - 1;
    }
    while (hi) {
        const int b = __ffs(hi) - 1;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] ^= __ldg(col + k * kSobolMatrix + 32 + b);
        hi &= hi - 1;
    }
    if (mode == 0)
        return make_uint4(v[0], v[1], v[2], v[3]);
    u32 h[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        h[k] = sobol_dimension_hash(dimension + k, seed);
    if (mode != 3) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] = scramble_word(v[k], mode, h[k]);
        return make_uint4(v[0], v[1], v[2], v[3]);
    }
    // Owen (the mode-3 loop of scramble_word), four words at once
    u32 first = 1;
    if (prefix) {
        constexpr u32 low = 32 - kOwenPrefixBits;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] = (v[k] & ((u32(1) << low) - 1)) | (u32(__ldg(prefix + k * kOwenPrefixEntries + (v[k] >> low))) << low);
        first = kOwenPrefixBits;
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] ^= (h[k] & 1) << 31;
    }
#pragma unroll 1
    for (u32 bit = first; bit < 32; ++bit) {
        const u32 mask = ~u32(0) << (32 - bit), flip = u32(1) << (31 - bit);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (u32(mix_bits((v[k] & mask) ^ h[k])) & (u32(1) << bit))
                v[k] ^= flip;
    }
    return make_uint4(v[0], v[1], v[2], v[3]);
}
// sobol_word of one dimension; with Owen randomisation and that dimension's table of
// owen_prefix_rounds (`prefix`, optional), the table replaces the first kOwenPrefixBits rounds.
RP_DEV u32 sobol_word_prefixed(const SobolTables &t, u64 index, u32 dimension, u32 mode, u32 seed,
                               const unsigned short *prefix) {
    if (mode != 3 || !prefix)
        return sobol_word(t, index, dimension, mode, seed);
    constexpr u32 low = 32 - kOwenPrefixBits;
    u32 v = sobol_raw(t, index, dimension);
    const u32 h = sobol_dimension_hash(dimension, seed);
    v = (v & ((u32(1) << low) - 1)) | (u32(__ldg(prefix + (v >> low))) << low);
#pragma unroll 1
    for (u32 bit = kOwenPrefixBits; bit < 32; ++bit)
        if (u32(mix_bits((v & (~u32(0) << (32 - bit))) ^ h)) & (u32(1) << bit))
            v ^= u32(1) << (31 - bit);
    return v;
}
// src/sobol_shared.h:143-154
RP_DEV float sobol_uniform(u32 v) {
    const float unit = float(v) * 0x1p-32f;
    return unit < kOneMinusEps ? unit : kOneMinusEps;
}
RP_DEV float sobol_camera_uniform(u32 global, u32 m, u32 pixel) {
    const float local = sobol_uniform(global) * float(u32(1) << m) - float(pixel);
    if (local < 0.0f)
        return 0.0f;
    return local < kOneMinusEps ? local : kOneMinusEps;
}

// ------------------------------------------------------------------ Halton and ZSobol (src/qmc_shared.h, PBRT v4)
RP_DEV float bits_float(u32 x) { return __uint_as_float(x); }
RP_DEV u32 float_bits(float x) { return __float_as_uint(x); }
// :20-40 (MurmurHash64A of two or three words)
RP_DEV u64 qmc_hash2(u32 a, u32 b) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    u64 k = ((u64(b) << 32) | a) * m;
    k ^= k >> 47;
    k *= m;
    u64 h = (8 * m ^ k) * m;
    h ^= h >> 47;
    h *= m;
    return h ^ (h >> 47);
}
RP_DEV u64 qmc_hash3(u32 a, u32 b, u32 c) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    u64 k = ((u64(b) << 32) | a) * m;
    k ^= k >> 47;
    k *= m;
    u64 h = (12 * m ^ k) * m;
    h ^= c;
    h *= m;
    h ^= h >> 47;
    h *= m;
    return h ^ (h >> 47);
}
// :41-66 element i of a hashed permutation of [0, l): cycle-walks a bijection on [0, w],
// w + 1 the next power of two, so it ends within w + 1 steps
RP_DEV u32 qmc_permutation(u32 i, u32 l, u32 p) {
    u32 w = l - 1;
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    for (u32 guard = 0; guard <= w; ++guard) {
        i ^= p;
        i *= 0xe170893du;
        i ^= p >> 16;
        i ^= (i & w) >> 4;
        i ^= p >> 8;
        i *= 0x0929eb3fu;
        i ^= p >> 23;
        i ^= (i & w) >> 1;
        i *= 1 | p >> 27;
        i *= 0x6935fa69u;
        i ^= (i & w) >> 11;
        i *= 0x74dcb303u;
        i ^= (i & w) >> 2;
        i *= 0x9e501cc3u;
        i ^= (i & w) >> 2;
        i *= 0xc860a3dfu;
        i &= w;
        i ^= i >> 5;
        if (i < l)
            break;
    }
    return (i + p) % l;
}
// :84-106 scrambled radical inverse of `a` in the base of `dimension`
RP_DEV float qmc_radical(const u32 *primes, u32 dimension, u64 a, u32 mode, u32 seed) {
    const u32 base = __ldg(primes + dimension);
    const u64 limit = ~u64(0) / base - base;
    const float inv = 1.f / float(base);
    float inv_m = 1;
    u64 reversed = 0;
    u32 digit_index = 0;
    const u32 owen_hash = u32(mix_bits(1 + (dimension << 4)));
    while ((mode == 0 ? a != 0 : (mode == 1 ? 1.f - float(base - 1) * inv_m < 1.f : 1.f - inv_m < 1.f)) &&
           reversed < limit) {
        const u64 next = a / base;
        u32 digit = u32(a - next * base);
        if (mode == 1)
            digit = qmc_permutation(digit, base, u32(qmc_hash3(base, digit_index, seed)));
        else if (mode == 3)
            digit = qmc_permutation(digit, base, u32(mix_bits(owen_hash ^ reversed)));
        reversed = reversed * base + digit;
        inv_m *= inv;
        ++digit_index;
        a = next;
    }
    const float value = float(reversed) * inv_m;
    return value < kOneMinusEps ? value : kOneMinusEps;
}
// :107-114
RP_DEV u64 qmc_inverse_radical(u32 a, u32 base, u32 count) {
    u64 result = 0;
    for (u32 i = 0; i < count; ++i) {
        result = result * base + a % base;
        a /= base;
    }
    return result;
}
// :115-129
RP_DEV u32 qmc_base_scale(u32 resolution, u32 base) {
    u32 scale = 1;
    const u32 bound = resolution < 128 ? resolution : 128;
    while (scale < bound)
        scale *= base;
    return scale;
}
RP_DEV u32 qmc_base_exponent(u32 scale, u32 base) {
    u32 e = 0;
    while (scale > 1) {
        scale /= base;
        ++e;
    }
    return e;
}
// :130-138 (scales are at most 243)
RP_DEV u32 qmc_inverse_mod(u32 a, u32 modulus) {
    if (modulus == 1)
        return 0;
    for (u32 i = 1; i < modulus; ++i)
        if ((a * i) % modulus == 1)
            return i;
    return 0;
}
// :139-148 Halton index of sample `sample` of pixel (x, y)
RP_DEV u64 halton_index(u32 width, u32 height, u32 x, u32 y, u64 sample) {
    const u32 sx = qmc_base_scale(width, 2), sy = qmc_base_scale(height, 3), stride = sx * sy;
    u64 offset = 0;
    if (stride > 1) {
        offset = qmc_inverse_radical(x % 128, 2, qmc_base_exponent(sx, 2)) * sy * qmc_inverse_mod(sy, sx);
        offset += qmc_inverse_radical(y % 128, 3, qmc_base_exponent(sy, 3)) * sx * qmc_inverse_mod(sx, sy);
        offset %= stride;
    }
    return offset + sample * stride;
}
// :176-179
RP_DEV float halton_camera(const u32 *primes, u32 axis, u32 resolution, u64 index) {
    const u32 scale = qmc_base_scale(resolution, axis == 0 ? 2 : 3);
    return qmc_radical(primes, axis, index / scale, 0, 0);
}
// :213-220
RP_DEV u64 zsobol_morton(u32 x, u32 y, u32 log_spp, u64 sample) {
    u64 result = 0;
    for (u32 b = 0; b < 26; ++b) {
        result |= u64((x >> b) & 1) << (2 * b);
        result |= u64((y >> b) & 1) << (2 * b + 1);
    }
    return (result << log_spp) | sample;
}
// :221-238 ZSobol index: base-4 digits of the Morton index permuted by a hash of their prefix
RP_DEV u64 zsobol_index(u64 morton_index, u32 dimension, u32 exponent, u32 log_spp) {
    // the 24 permutations of 4 elements, 2 bits each (digit d at bits 2d..2d+1)
    constexpr unsigned char perm[24] = {0xe4, 0xb4, 0xd8, 0x78, 0x6c, 0x9c, 0xe1, 0xb1, 0xc9, 0x39, 0x2d, 0x8d,
                                        0xc6, 0x36, 0xd2, 0x72, 0x4e, 0x1e, 0x27, 0x87, 0x1b, 0x4b, 0x63, 0x93};
    const u32 odd = log_spp & 1;
    const u32 digits = exponent + (log_spp + 1) / 2;
    u64 result = 0;
    for (int i = int(digits) - 1; i >= int(odd); --i) {
        const u32 shift = 2 * u32(i) - odd;
        const u32 digit = u32((morton_index >> shift) & 3);
        const u64 higher = morton_index >> (shift + 2);
        const u32 p = u32((mix_bits(higher ^ u32(0x55555555u * dimension)) >> 24) % 24);
        result |= u64((perm[p] >> (2 * digit)) & 3) << shift;
    }
    if (odd)
        result |= (morton_index & 1) ^ (mix_bits((morton_index >> 1) ^ u32(0x55555555u * dimension)) & 1);
    return result;
}
// :244-249
RP_DEV u32 zsobol_word(const SobolTables &t, u64 morton_index, u32 dimension, u32 axis, bool pair, u32 exponent,
                       u32 log_spp, u32 mode, u32 seed) {
    const u64 index = zsobol_index(morton_index, dimension, exponent, log_spp);
    const u64 hash = qmc_hash2(dimension + (pair ? 2 : 1), seed);
    const u32 random = pair && axis == 1 ? u32(hash >> 32) : u32(hash);
    return scramble_word(sobol_raw(t, index, axis), mode, random);
}

// ------------------------------------------------------------------ Philox (shaders/render.metal:97-111)
RP_DEV uint4 philox(uint4 c, u32 k0, u32 k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const u32 hi0 = __umulhi(0xd2511f53u, c.x), lo0 = 0xd2511f53u * c.x;
        const u32 hi1 = __umulhi(0xcd9e8d57u, c.z), lo1 = 0xcd9e8d57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9e3779b9u;
        k1 += 0xbb67ae85u;
    }
    return c;
}
RP_DEV float u01(u32 w) { return float(w >> 8) * 0x1.0p-24f; }

// ------------------------------------------------------------------ scaled likelihoods
// src/hero_spectrum_shared.h:16-195.  frexp/ldexp are exact binary operations here: every
// fraction handed to them is a normal binary32 value, so they are written on the bit fields.
RP_DEV bool nonnegative_finite(float x) { return fbits(x) < 0x7f800000u || fbits(x) == 0x80000000u; }
struct Number {
    float fraction;
    int exponent;
};
RP_DEV Number zero_number() { return {0.0f, 0}; }
// frexp of a nonzero normal binary32 value
RP_DEV Number split_normal(float x, int exponent) {
    const u32 b = fbits(x);
    const int e = int((b >> 23) & 0xffu) - 126;
    return {ffrom((b & 0x807fffffu) | (126u << 23)), exponent + e};
}
// src/hero_spectrum_shared.h:37-43
RP_DEV Number normalized(float x, int exponent) {
    if (x == 0)
        return zero_number();
    return split_normal(x, exponent);
}
// 2^e for -126 <= e <= 127
RP_DEV float pow2(int e) { return ffrom(u32(e + 127) << 23); }
// exact x * 2^e for normal x, result normal or overflowing (ldexp semantics on that range)
RP_DEV float scale2(float x, int e) {
    const int a = e / 2, b = e - a;
    return __fmul_rn(__fmul_rn(x, pow2(a)), pow2(b));
}
// :44-51
RP_DEV Number number(float x) {
    const u32 w = fbits(x) & 0x7fffffffu;
    if (w == 0)
        return zero_number();
    if ((w & 0x7f800000u) == 0)
        return normalized(float(w), -149);
    return normalized(x, 0);
}
// :52-56
RP_DEV Number nmul(Number a, Number b) {
    if (a.fraction == 0 || b.fraction == 0)
        return zero_number();
    return normalized(a.fraction * b.fraction, a.exponent + b.exponent);
}
// :57-59
RP_DEV Number ndiv(Number a, Number b) { return normalized(a.fraction / b.fraction, a.exponent - b.exponent); }
// :60-74
RP_DEV Number nadd(Number a, Number b) {
    if (a.fraction == 0)
        return b;
    if (b.fraction == 0)
        return a;
    if (a.exponent < b.exponent) {
        const Number t = a;
        a = b;
        b = t;
    }
    const int gap = a.exponent - b.exponent;
    if (gap > 24)
        return a;
    return normalized(a.fraction + scale2(b.fraction, -gap), a.exponent);
}
struct Scalar {
    float value;
    bool valid;
};
// :79-99
RP_DEV Scalar materialize(Number x) {
    if (x.fraction == 0)
        return {0, true};
    if (!(x.fraction >= .5f && x.fraction < 1) || x.exponent > 128)
        return {0, false};
    if (x.exponent >= -125) {
        const float value = scale2(x.fraction, x.exponent);
        return {value, nonnegative_finite(value)};
    }
    if (x.exponent < -149)
        return {0, true};
    const u32 significand = (fbits(x.fraction) & 0x007fffffu) | 0x00800000u;
    const u32 shift = u32(-125 - x.exponent);
    u32 units = significand >> shift;
    const u32 rest = significand & ((1u << shift) - 1);
    const u32 halfway = 1u << (shift - 1);
    units += rest > halfway || (rest == halfway && (units & 1));
    return {ffrom(units), true};
}
struct Density {
    Number lane[4];
};
RP_DEV Density initial_density() {
    Density d;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        d.lane[k] = {0.5f, 1};
    return d;
}
// :109-111
RP_DEV Number total(const Density &p) { return nadd(nadd(p.lane[0], p.lane[1]), nadd(p.lane[2], p.lane[3])); }
// :112-117
RP_DEV Number mixture(const Density &p, V4 pdf) {
    Number t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        t[k] = nmul(p.lane[k], number(pdf.v[k]));
    return nadd(nadd(t[0], t[1]), nadd(t[2], t[3]));
}
struct Update {
    Density density;
    V4 beta;
    bool valid;
};
// :123-144
RP_DEV Update advance(const Density &prefix, V4 beta, V4 numerator, V4 pdf) {
    Update out;
    out.valid = false;
    out.beta = v4(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!nonnegative_finite(pdf.v[k]) || !nonnegative_finite(numerator.v[k]) ||
            !nonnegative_finite(beta.v[k]))
            return out;
        out.density.lane[k] = nmul(prefix.lane[k], number(pdf.v[k]));
    }
    const Number before = total(prefix), after = total(out.density);
    if (!(before.fraction > 0 && after.fraction > 0))
        return out;
    const Number ratio = ndiv(before, after);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const Scalar value = materialize(nmul(nmul(number(beta.v[k]), number(numerator.v[k])), ratio));
        if (!value.valid)
            return out;
        out.beta.v[k] = value.value;
    }
    out.valid = true;
    return out;
}
struct Contribution {
    V4 value;
    bool valid;
};
// :161-180
RP_DEV Contribution balance_contribution(const Density &prefix, V4 value, V4 sampled, V4 other) {
    Contribution r;
    r.valid = false;
    r.value = v4(0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (!nonnegative_finite(value.v[k]) || !nonnegative_finite(sampled.v[k]) ||
            !nonnegative_finite(other.v[k]))
            return r;
    const Number a = mixture(prefix, sampled), b = mixture(prefix, other), sum = nadd(a, b);
    if (!(sum.fraction > 0))
        return r;
    const Number weight = ndiv(a, sum);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const Scalar w = materialize(nmul(number(value.v[k]), weight));
        if (!w.valid)
            return r;
        r.value.v[k] = w.value;
    }
    r.valid = true;
    return r;
}

// ------------------------------------------------------------------ wavelengths
// src/packet_spectrum_shared.h:27-31
RP_DEV float visible_pdf(float lambda) {
    if (lambda < 360 || lambda > 830)
        return 0;
    const float c = coshf(.0072f * (lambda - 538));
    return .0039398042f / (c * c);
}
// src/hero_spectrum_shared.h:199-244
RP_DEV void sample_wavelengths(float u, u32 mode, V4 &lambda, V4 &pdf) {
    if (!(u >= 0 && u < 1)) {
        lambda = v4(__int_as_float(0x7fffffff));
        pdf = lambda;
        return;
    }
#pragma unroll
    for (u32 k = 0; k < 4; ++k) {
        if (mode == 1) {
            const u32 coordinate = u32(u * 16777216.f);
            const float s = float((coordinate + k * 4194304u) & 0x00ffffffu) * 0x1p-24f;
            float w = 538 - 138.888889f * atanhf(.85691062f - 1.82750197f * s);
            w = w < 360 ? 360 : w;
            w = w > 830 ? 830 : w;
            lambda.v[k] = w;
            pdf.v[k] = visible_pdf(w);
        } else {
            float s = u + float(k) * .25f;
            if (s >= 1)
                s -= 1;
            float w = 360 + 470 * s;
            if (w >= 830)
                w = ffrom(fbits(830.f) - 1);
            lambda.v[k] = w;
            pdf.v[k] = 1.f / 470.f;
        }
    }
}

// ------------------------------------------------------------------ Russian roulette
// src/packet_roulette_shared.h:21-28
RP_DEV bool rr_finite(float v) { return (fbits(v) & 0x7fffffffu) < 0x7f800000u; }
RP_DEV bool positive_normal(float v) {
    const u32 w = fbits(v);
    return w >= 0x00800000u && w < 0x7f800000u;
}
RP_DEV bool opposite_hemispheres(float a, float b) { return (a > 0 && b < 0) || (a < 0 && b > 0); }
// shaders/hero_pt_helpers.h:56-85 with rypath_packet_roulette::prepare (:59-94) on a unit scale
RP_DEV bool hero_continue(V4 &beta, V4 eta_scale, bool roulette_enabled, u32 depth, float uniform) {
    if (!roulette_enabled || depth <= 1)
        return true;
    float maximum = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float v = beta.v[k] * eta_scale.v[k];
        if (!isfinite(v) || v < 0 || (beta.v[k] > 0 && !positive_normal(v)))
            return true;
        maximum = fmaxf(maximum, v);
    }
    // prepare(float4(maximum), unit, depth)
    if (!rr_finite(maximum) || ((fbits(maximum) >> 31) && (fbits(maximum) & 0x7fffffffu)))
        return true;
    const float m = maximum * 1.0f;
    if (!positive_normal(m) || m >= 1)
        return true;
    const float q = 1 - m;
    const float survival_p = 1 - q;
    if (!rr_finite(q) || !(q > 0 && q < 1) || !positive_normal(survival_p))
        return true;
    if ((fbits(maximum) & 0x7fffffffu) != 0 && !positive_normal(maximum / survival_p))
        return true;
    const float survival = 1 - q;
    V4 survivor = beta;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (fbits(beta.v[k]) == 0)
            continue;
        survivor.v[k] /= survival;
        if (!positive_normal(survivor.v[k]))
            return true;
    }
    if (uniform < q)
        return false;
    beta = survivor;
    return true;
}
// shaders/hero_pt_helpers.h:86-98 with account_transmission (src/packet_roulette_shared.h:38-51)
RP_DEV void hero_account_eta(V4 &eta_scale, bool &roulette_enabled, V4 eta, bool transmission) {
    if (!transmission || !roulette_enabled)
        return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float e = eta.v[k];
        if (!positive_normal(e)) {
            roulette_enabled = false;
            return;
        }
        const float square = e * e;
        const float next = eta_scale.v[k] * square;
        if (!positive_normal(square) || !positive_normal(next)) {
            roulette_enabled = false;
            return;
        }
        eta_scale.v[k] = next;
    }
}

// ------------------------------------------------------------------ BSDFs
struct Eval {
    float f, pdf;
    bool valid;
};
struct BSample {
    V3 wi;
    float weight, pdf;
    bool delta, accepted, valid;
};
RP_DEV bool randoms(float uc, float ux, float uy) {
    return isfinite(uc) && uc >= 0 && uc < 1 && isfinite(ux) && isfinite(uy) && ux >= 0 && uy >= 0 && ux < 1 &&
           uy < 1;
}
// shaders/transmission.h:52-62 (opaque lane: T = 0)
RP_DEV Eval diffuse_evaluate(float R, V3 wo, V3 wi) {
    if (!isfinite(R) || R < 0 || !finite3(wo) || !finite3(wi))
        return {0, 0, false};
    const float sum = R + 0.0f;
    if (!isfinite(sum))
        return {0, 0, false};
    if (wo.z == 0 || wi.z == 0 || sum == 0)
        return {0, 0, true};
    const float value = (wo.z > 0) == (wi.z > 0) ? R : 0.0f;
    return {value / kPi, value / sum * fabsf(wi.z) / kPi, true};
}
// shaders/packet_scattering.h:170-203
RP_DEV BSample diffuse_reflection_sample(float R, V3 wo, float uc, float ux, float uy) {
    BSample s{{0, 0, 0}, 0, 0, false, false, true};
    const float sum = R + 0.0f;
    if (!isfinite(R) || R < 0 || !isfinite(sum) || !finite3(wo) || !randoms(uc, ux, uy)) {
        s.valid = false;
        return s;
    }
    if (sum == 0 || wo.z == 0)
        return s;
    const float ox = 2 * ux - 1, oy = 2 * uy - 1;
    V3 w;
    if (ox == 0 && oy == 0) {
        w = v3(0, 0, 1);
    } else {
        float radius, theta;
        if (fabsf(ox) > fabsf(oy)) {
            radius = ox;
            theta = (kPi / 4) * (oy / ox);
        } else {
            radius = oy;
            theta = (kPi / 2) - (kPi / 4) * (ox / oy);
        }
        const float dx = radius * cosf(theta), dy = radius * sinf(theta);
        w = v3(dx, dy, sqrtf(fmaxf(0.0f, 1 - (dx * dx + dy * dy))));
    }
    if (wo.z < 0)
        w.z = -w.z;
    s.wi = w;
    s.pdf = R / sum * fabsf(w.z) / kPi;
    s.weight = sum;
    s.accepted = s.pdf > 0;
    return s;
}
// shaders/conductor.h:35-42
RP_DEV bool unit(V3 v, V3 &out) {
    const float s = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
    if (!(s > 0) || !isfinite(s))
        return false;
    v = v / s;
    out = v / sqrtf(dot(v, v));
    return finite3(out);
}
RP_DEV bool complex_ratio_norm(float ax, float ay, float bx, float by, float &out) {
    const float s = fmaxf(fabsf(bx), fabsf(by));
    if (!(s > 0) || !isfinite(s) || !isfinite(ax) || !isfinite(ay))
        return false;
    ax /= s;
    ay /= s;
    bx /= s;
    by /= s;
    out = (ax * ax + ay * ay) / (bx * bx + by * by);
    return isfinite(out);
}
RP_DEV void two_sum(float a, float b, float &sum, float &err) {
    sum = a + b;
    const float bv = sum - a;
    err = (a - (sum - bv)) + (b - bv);
}
// shaders/conductor.h:58-102
RP_DEV bool conductor_fresnel(float cosine, float eta, float k, float &f) {
    if (!isfinite(cosine) || !isfinite(eta) || !isfinite(k) || eta < 0 || k < 0 || (eta == 0 && k == 0))
        return false;
    const float c = fminf(fmaxf(cosine, 0.0f), 1.0f);
    if (eta == 1 && k == 0) {
        f = 0;
        return true;
    }
    if (c == 0) {
        f = 1;
        return true;
    }
    const float n2x = eta * eta - k * k, n2y = 2 * eta * k;
    if (!isfinite(n2x) || !isfinite(n2y))
        return false;
    const float eta2 = eta * eta, k2 = k * k, c2 = c * c;
    float abx, aby, cdx, cdy, tx, ty;
    two_sum(eta2, -k2, abx, aby);
    two_sum(c2, -1, cdx, cdy);
    two_sum(abx, cdx, tx, ty);
    const float correction = aby + cdy + ty + fmaf(eta, eta, -eta2) - fmaf(k, k, -k2) + fmaf(c, c, -c2);
    const float zx = tx + correction, zy = n2y;
    const float scale = fmaxf(fabsf(zx), fabsf(zy));
    float radius = 0;
    if (scale != 0) {
        const float sx = zx / scale, sy = zy / scale;
        radius = scale * sqrtf(sx * sx + sy * sy);
    }
    if (!isfinite(radius))
        return false;
    float qr, qi;
    if (zx >= 0) {
        qr = sqrtf(fmaxf(0.0f, 0.5f * radius + 0.5f * zx));
        qi = qr > 0 ? zy / (2 * qr) : 0;
    } else {
        qi = sqrtf(fmaxf(0.0f, 0.5f * radius - 0.5f * zx));
        qr = qi > 0 ? zy / (2 * qi) : 0;
    }
    float rs, rp;
    if (!complex_ratio_norm(c - qr, 0 - qi, c + qr, 0 + qi, rs) ||
        !complex_ratio_norm(n2x * c - qr, n2y * c - qi, n2x * c + qr, n2y * c + qi, rp))
        return false;
    f = (rs + rp) * 0.5f;
    return isfinite(f) && f >= 0;
}
// shaders/conductor.h:103-119
RP_DEV float ggx_lambda(float ax, float ay, V3 w) {
    const V3 v = v3(1, ax * w.x / w.z, ay * w.y / w.z);
    const float s = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
    return 0.5f * (s * length3(v / s) - 1);
}
RP_DEV float ggx_distribution(float ax, float ay, V3 m) {
    if (m.z * m.z * m.z * m.z < 1e-16f)
        return 0;
    const V3 v = v3(m.x / ax, m.y / ay, m.z);
    const float t = dot(v, v);
    const float den = kPi * ax * ay * t * t;
    if (!isfinite(den) || !(den > 0))
        return __int_as_float(0x7fffffff);
    const float d = 1 / den;
    return d > 0 ? d : __int_as_float(0x7fffffff);
}
struct Ggx {
    float alpha_x, alpha_y;
    bool smooth;
};
// shaders/conductor.h:22-34 and dielectric.h:15-27 (roughness part)
RP_DEV bool prepare_roughness(float u, float v, bool remap, bool force_smooth, Ggx &g) {
    g.alpha_x = remap ? sqrtf(u) : u;
    g.alpha_y = remap ? sqrtf(v) : v;
    g.smooth = force_smooth || fmaxf(g.alpha_x, g.alpha_y) < 1e-3f;
    if (!g.smooth) {
        g.alpha_x = fmaxf(g.alpha_x, 1e-4f);
        g.alpha_y = fmaxf(g.alpha_y, 1e-4f);
    }
    return true;
}
// shaders/conductor.h:120-138
RP_DEV Eval conductor_evaluate(float eta, float k, const Ggx &g, V3 wo, V3 wi) {
    if (!finite3(wo) || !finite3(wi))
        return {0, 0, false};
    if (g.smooth || wo.z == 0 || wi.z == 0 || ((wo.z > 0) != (wi.z > 0)))
        return {0, 0, true};
    V3 m;
    if (!unit(wo + wi, m))
        return {0, 0, false};
    float f;
    if (!conductor_fresnel(fabsf(dot(wo, m)), eta, k, f))
        return {0, 0, false};
    const float lo = ggx_lambda(g.alpha_x, g.alpha_y, wo), li = ggx_lambda(g.alpha_x, g.alpha_y, wi),
                d = ggx_distribution(g.alpha_x, g.alpha_y, m);
    const float value = d * f / (4 * fabsf(wo.z) * fabsf(wi.z) * (1 + lo + li));
    const float pdf = d / (4 * fabsf(wo.z) * (1 + lo));
    const bool valid = isfinite(lo) && isfinite(li) && isfinite(d) && isfinite(value) && isfinite(pdf) &&
                       value >= 0 && pdf >= 0;
    return {value, pdf, valid};
}
// Visible-normal sampling: shaders/conductor.h:157-185, dielectric.h:160-188
RP_DEV bool ggx_visible_normal(float ax, float ay, V3 wo, float ux, float uy, V3 &m) {
    V3 wh;
    if (!unit(v3(ax * wo.x, ay * wo.y, wo.z), wh))
        return false;
    if (wh.z < 0)
        wh = -wh;
    V3 t1;
    if (wh.z < 0.99999f) {
        if (!unit(v3(-wh.y, wh.x, 0), t1))
            return false;
    } else
        t1 = v3(1, 0, 0);
    const V3 t2 = cross(wh, t1);
    const float r = sqrtf(ux), phi = 2 * kPi * uy;
    float dx = r * cosf(phi), dy = r * sinf(phi);
    const float h = sqrtf(fmaxf(0.0f, 1 - dx * dx));
    const float a = (1 + wh.z) * 0.5f;
    const float old_y = dy;
    dy = (1 - a) * h + a * dy;
    const float old_minus_h = old_y > 0 ? -(1 - ux) / (h + old_y) : old_y - h;
    const float z = sqrtf(fmaxf(0.0f, (1 - ux) + (1 - a) * old_minus_h * (old_y + dy)));
    const V3 nh = dx * t1 + dy * t2 + z * wh;
    return unit(v3(ax * nh.x, ay * nh.y, fmaxf(1e-6f, nh.z)), m);
}
// shaders/conductor.h:139-207
RP_DEV BSample conductor_sample(float eta, float k, const Ggx &g, V3 wo, float ux, float uy) {
    BSample s{{0, 0, 0}, 0, 0, g.smooth, false, true};
    if (!finite3(wo) || !isfinite(ux) || !isfinite(uy) || ux < 0 || uy < 0 || ux >= 1 || uy >= 1) {
        s.valid = false;
        return s;
    }
    if (wo.z == 0)
        return s;
    if (g.smooth) {
        s.wi = v3(-wo.x, -wo.y, wo.z);
        s.pdf = 1;
        s.valid = conductor_fresnel(fabsf(wo.z), eta, k, s.weight);
        s.accepted = s.valid && s.weight > 0;
        return s;
    }
    V3 m;
    if (!ggx_visible_normal(g.alpha_x, g.alpha_y, wo, ux, uy, m)) {
        s.valid = false;
        return s;
    }
    s.wi = -wo + 2 * dot(wo, m) * m;
    if (!finite3(s.wi)) {
        s.valid = false;
        return s;
    }
    if (s.wi.z == 0 || ((wo.z > 0) != (s.wi.z > 0)))
        return s;
    float f;
    s.valid = conductor_fresnel(fabsf(dot(wo, m)), eta, k, f);
    if (!s.valid)
        return s;
    const float lo = ggx_lambda(g.alpha_x, g.alpha_y, wo), li = ggx_lambda(g.alpha_x, g.alpha_y, s.wi);
    const float d = ggx_distribution(g.alpha_x, g.alpha_y, m);
    if (d == 0)
        return s;
    s.pdf = d / (4 * fabsf(wo.z) * (1 + lo));
    s.weight = f * (1 + lo) / (1 + lo + li);
    s.valid = isfinite(lo) && isfinite(li) && isfinite(s.pdf) && isfinite(s.weight) && s.weight >= 0 && s.pdf > 0;
    s.accepted = s.valid && s.weight > 0;
    return s;
}
// shaders/dielectric.h:31-70
RP_DEV bool dielectric_optics(float cosine, float eta, float &F, float &etap, float &ct, bool &tir) {
    if (!isfinite(cosine))
        return false;
    etap = cosine < 0 ? 1 / eta : eta;
    const float c = fminf(fabsf(cosine), 1.0f);
    if (!(etap > 0) || !isfinite(etap))
        return false;
    if (etap == 1) {
        F = 0;
        ct = c;
        tir = false;
        return true;
    }
    const float c2 = c * c;
    const float e2 = eta * eta;
    float disc;
    if (cosine < 0) {
        float ax, ay;
        two_sum(1, -e2, ax, ay);
        disc = fmaf(e2, c2, ax) + (ay + fmaf(eta, eta, -e2) * (c2 - 1) + e2 * fmaf(c, c, -c2));
    } else {
        float ax, ay, bx, by;
        two_sum(e2, -1, ax, ay);
        two_sum(ax, c2, bx, by);
        disc = bx + (ay + by + fmaf(eta, eta, -e2) + fmaf(c, c, -c2));
    }
    if (!isfinite(disc))
        return false;
    tir = disc <= 0;
    if (tir) {
        F = 1;
        ct = 0;
        return true;
    }
    ct = sqrtf(disc) / (cosine < 0 ? 1 : eta);
    const float rp = (etap * c - ct) / (etap * c + ct);
    const float rs = (c - etap * ct) / (c + etap * ct);
    F = .5f * (rp * rp + rs * rs);
    return isfinite(ct) && isfinite(F) && F >= 0 && F <= 1;
}
// shaders/dielectric.h:76-126
RP_DEV Eval dielectric_evaluate(float eta, const Ggx &g, V3 wo, V3 wi) {
    if (!finite3(wo) || !finite3(wi))
        return {0, 0, false};
    if (g.smooth || wo.z == 0 || wi.z == 0)
        return {0, 0, true};
    const bool reflection = (wo.z > 0) == (wi.z > 0);
    const bool entering = wo.z > 0;
    const V3 h = reflection ? wo + wi : (entering ? fma3(v3(eta, eta, eta), wi, wo) : fma3(v3(eta, eta, eta), wo, wi));
    V3 m;
    if (zero3(h))
        return {0, 0, true};
    if (!unit(h, m))
        return {0, 0, false};
    if (m.z < 0)
        m = -m;
    const float co = dot(wo, m), ci = dot(wi, m);
    if (co * wo.z < 0 || ci * wi.z < 0)
        return {0, 0, true};
    float F, ct, ep;
    bool tir;
    if (!dielectric_optics(co, eta, F, ep, ct, tir))
        return {0, 0, false};
    const float lo = ggx_lambda(g.alpha_x, g.alpha_y, wo), li = ggx_lambda(g.alpha_x, g.alpha_y, wi);
    const float d = ggx_distribution(g.alpha_x, g.alpha_y, m);
    if (!isfinite(lo) || !isfinite(li) || !isfinite(d))
        return {0, 0, false};
    if (d == 0)
        return {0, 0, true};
    float value, pdf;
    if (reflection) {
        value = d * F / (4 * fabsf(wo.z) * fabsf(wi.z) * (1 + lo + li));
        pdf = d * F / (4 * fabsf(wo.z) * (1 + lo));
    } else {
        const float den = dot(h, m) / (entering ? eta : 1);
        const float jac = fabsf(ci) / (den * den);
        pdf = d * fabsf(co) / (fabsf(wo.z) * (1 + lo)) * jac * (1 - F);
        const float scale = entering ? 1 / (eta * eta) : eta * eta;
        value = d * (1 - F) * fabsf(ci * co) * scale / (fabsf(wo.z) * fabsf(wi.z) * den * den * (1 + lo + li));
    }
    return {value, pdf,
            isfinite(lo) && isfinite(li) && isfinite(d) && isfinite(value) && isfinite(pdf) && value >= 0 &&
                pdf >= 0};
}
// shaders/dielectric.h:129-133
RP_DEV float refraction_coefficient(float eta, float co, float ct) {
    const float c = fabsf(co);
    return co < 0 ? ((eta - 1) * (eta + 1)) / (eta * c + ct) : (((1 - eta) * (1 + eta)) / eta) / (c + eta * ct);
}
// shaders/dielectric.h:134-227
RP_DEV BSample dielectric_sample(float eta, const Ggx &g, V3 wo, float uc, float ux, float uy, float &sampled_eta) {
    sampled_eta = 1;
    BSample s{{0, 0, 0}, 0, 0, g.smooth, false, true};
    if (!finite3(wo) || !isfinite(uc) || uc < 0 || uc >= 1 || !isfinite(ux) || !isfinite(uy) || ux < 0 || uy < 0 ||
        ux >= 1 || uy >= 1) {
        s.valid = false;
        return s;
    }
    if (wo.z == 0)
        return s;
    V3 m = v3(0, 0, 1);
    if (!g.smooth && !ggx_visible_normal(g.alpha_x, g.alpha_y, wo, ux, uy, m)) {
        s.valid = false;
        return s;
    }
    const float co = dot(wo, m);
    float F, ep, ct;
    bool tir;
    if (!dielectric_optics(co, eta, F, ep, ct, tir)) {
        s.valid = false;
        return s;
    }
    const bool reflection = uc < F;
    if (reflection)
        s.wi = -wo + 2 * co * m;
    else {
        if (tir) {
            s.valid = false;
            return s;
        }
        const float coefficient = eta == 1 ? 0 : refraction_coefficient(eta, co, ct);
        s.wi = (co < 0 ? (-eta) * wo : (-wo) / eta) + coefficient * (co < 0 ? -m : m);
    }
    if (!finite3(s.wi)) {
        s.valid = false;
        return s;
    }
    if (s.wi.z == 0 || (((s.wi.z > 0) == (wo.z > 0)) != reflection))
        return s;
    const float scale = reflection ? 1 : (co < 0 ? eta * eta : 1 / (eta * eta));
    if (g.smooth) {
        s.pdf = reflection ? F : 1 - F;
        s.weight = scale;
    } else {
        const float lo = ggx_lambda(g.alpha_x, g.alpha_y, wo), li = ggx_lambda(g.alpha_x, g.alpha_y, s.wi);
        const float d = ggx_distribution(g.alpha_x, g.alpha_y, m);
        if (!isfinite(lo) || !isfinite(li) || !isfinite(d)) {
            s.valid = false;
            return s;
        }
        if (d == 0)
            return s;
        if (reflection)
            s.pdf = d * F / (4 * fabsf(wo.z) * (1 + lo));
        else {
            const float den = refraction_coefficient(eta, co, ct);
            s.pdf = d * fabsf(co) * ct * (1 - F) / (fabsf(wo.z) * (1 + lo) * den * den);
        }
        s.weight = scale * (1 + lo) / (1 + lo + li);
        s.valid = isfinite(lo) && isfinite(li) && isfinite(d);
    }
    s.valid = s.valid && isfinite(s.pdf) && s.pdf > 0 && isfinite(s.weight) && s.weight > 0;
    s.accepted = s.valid;
    if (s.accepted && !reflection)
        sampled_eta = ep;
    return s;
}

// ------------------------------------------------------------------ hero BSDF
// A prepared hero BSDF (HeroFrozenBSDF for families 0-2, shaders/hero_frozen_bsdf.h): one
// family, a shared roughness, and per-wavelength parameters.  param = diffuse reflectance or
// dielectric eta; k = conductor eta/k pairs.
struct HeroBsdf {
    u32 kind, active_mask;
    Ggx g;
    float param[4];
    float k[4];
};
// shaders/scattering.h:25-28, shaders/hero_current_bsdf.h:62-67
RP_DEV bool lane_delta_only(const HeroBsdf &p, int k) {
    return (p.kind == 1 || p.kind == 2) && (p.g.smooth || (p.kind == 2 && p.param[k] == 1));
}
RP_DEV bool hero_connectible(const HeroBsdf &p) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if ((p.active_mask & (1u << k)) && !lane_delta_only(p, k))
            return true;
    return false;
}
// One wavelength of a family-K BSDF; a dielectric lane with eta == 1 is smooth, as
// rypath_dielectric::prepare makes it (shaders/dielectric.h:19).
template <int K> RP_DEV Eval lane_evaluate_k(const HeroBsdf &p, int k, V3 wo, V3 wi) {
    if constexpr (K == 0) {
        return diffuse_evaluate(p.param[k], wo, wi);
    } else if constexpr (K == 1) {
        return conductor_evaluate(p.param[k], p.k[k], p.g, wo, wi);
    } else {
        Ggx g = p.g;
        if (p.param[k] == 1)
            g.smooth = true;
        return dielectric_evaluate(p.param[k], g, wo, wi);
    }
}
template <int K> RP_DEV BSample lane_sample_k(const HeroBsdf &p, int k, V3 wo, float uc, float ux, float uy, float &eta) {
    eta = 1;
    if constexpr (K == 0) {
        return diffuse_reflection_sample(p.param[k], wo, uc, ux, uy);
    } else if constexpr (K == 1) {
        return conductor_sample(p.param[k], p.k[k], p.g, wo, ux, uy);
    } else {
        Ggx g = p.g;
        if (p.param[k] == 1)
            g.smooth = true;
        return dielectric_sample(p.param[k], g, wo, uc, ux, uy, eta);
    }
}
RP_DEV Eval lane_evaluate(const HeroBsdf &p, int k, V3 wo, V3 wi) {
    return p.kind == 0 ? lane_evaluate_k<0>(p, k, wo, wi)
                       : (p.kind == 1 ? lane_evaluate_k<1>(p, k, wo, wi) : lane_evaluate_k<2>(p, k, wo, wi));
}
RP_DEV BSample lane_sample(const HeroBsdf &p, int k, V3 wo, float uc, float ux, float uy, float &eta) {
    return p.kind == 0 ? lane_sample_k<0>(p, k, wo, uc, ux, uy, eta)
                       : (p.kind == 1 ? lane_sample_k<1>(p, k, wo, uc, ux, uy, eta)
                                      : lane_sample_k<2>(p, k, wo, uc, ux, uy, eta));
}
struct HeroEval {
    V4 f, pdf;
    bool valid;
};
// shaders/hero_frozen_bsdf.h:167-250 (radiance mode) for family K; out of line so every
// caller in a kernel shares one copy.
template <int K> __device__ __noinline__ HeroEval hero_evaluate_k(const HeroBsdf &p, V3 wo, V3 wi) {
    HeroEval out{v4(0), v4(0), false};
    if (!(p.active_mask & 1u) || (p.active_mask & ~15u) || !finite3(wo) || !finite3(wi))
        return out;
    out.valid = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!(p.active_mask & (1u << k)))
            continue;
        const Eval e = lane_evaluate_k<K>(p, k, wo, wi);
        out.f.v[k] = e.f;
        out.pdf.v[k] = e.pdf;
        out.valid = out.valid && e.valid;
    }
    if (!finite_nonnegative4(out.f) || !finite_nonnegative4(out.pdf))
        out.valid = false;
    return out;
}
// Any family, dispatched at run time (the latest vertex of a path can be of any family).
__device__ __noinline__ HeroEval hero_evaluate(const HeroBsdf &p, V3 wo, V3 wi) {
    if (p.kind == 0)
        return hero_evaluate_k<0>(p, wo, wi);
    if (p.kind == 1)
        return hero_evaluate_k<1>(p, wo, wi);
    return hero_evaluate_k<2>(p, wo, wi);
}
// shaders/hero_scattering.h:55-66
RP_DEV float event_eta(const HeroBsdf &p, int k, V3 wo, V3 wi) {
    if (!opposite_hemispheres(wo.z, wi.z))
        return 1;
    if (p.kind == 2)
        return wo.z > 0 ? p.param[k] : 1 / p.param[k];
    return 1;
}
// shaders/hero_scattering.h:100-138 (dirac_lane)
RP_DEV bool dirac_lane(const HeroBsdf &p, int k, V3 wo, V3 wi, float ux, float uy, float &mass, float &pdf,
                       float &eta) {
    mass = pdf = 0;
    eta = 1;
    if (wo.z == 0 || wi.z == 0)
        return true;
    const bool transmission = opposite_hemispheres(wo.z, wi.z);
    if (p.kind == 1 && p.g.smooth) {
        if (transmission || !eq3(wi, v3(-wo.x, -wo.y, wo.z)))
            return true;
        pdf = 1;
        return conductor_fresnel(fabsf(wo.z), p.param[k], p.k[k], mass);
    }
    if (p.kind == 2 && (p.g.smooth || p.param[k] == 1)) {
        float F, ep, ct;
        bool tir;
        if (!dielectric_optics(wo.z, p.param[k], F, ep, ct, tir))
            return false;
        const float probability = transmission ? 1 - F : F;
        if (probability == 0)
            return true;
        float sampled_eta;
        Ggx g = p.g;
        g.smooth = true;
        const BSample c = dielectric_sample(p.param[k], g, wo, transmission ? F : 0.f, ux, uy, sampled_eta);
        if (!c.valid)
            return false;
        if (!(c.pdf > 0) || !eq3(c.wi, wi))
            return true;
        pdf = c.pdf;
        mass = c.weight * pdf;
        eta = sampled_eta;
        return isfinite(mass) && mass >= 0;
    }
    return true;
}
struct HeroSample {
    V3 wi;
    V4 numerator, pdf, eta;
    bool delta, transmission, accepted, valid;
};
// shaders/hero_current_bsdf.h:121-203 (hero_current_sample)
template <int K> RP_DEV HeroSample hero_sample_k(const HeroBsdf &p, V3 wo, float uc, float ux, float uy) {
    HeroSample out;
    out.wi = v3(0, 0, 0);
    out.numerator = v4(0);
    out.pdf = v4(0);
    out.eta = v4(1);
    out.delta = out.transmission = out.accepted = out.valid = false;
    if (!(p.active_mask & 1u) || (p.active_mask & ~15u) || p.kind > 2 || !finite3(wo) || !randoms(uc, ux, uy))
        return out;
    float hero_eta;
    const BSample hero = lane_sample_k<K>(p, 0, wo, uc, ux, uy, hero_eta);
    out.valid = hero.valid;
    out.wi = hero.wi;
    out.delta = hero.delta;
    out.transmission = opposite_hemispheres(wo.z, hero.wi.z);
    if (!hero.valid)
        return out;
    if (!isfinite(hero.pdf) || hero.pdf < 0 || !finite3(hero.wi)) {
        out.valid = false;
        return out;
    }
    if (hero.pdf == 0 || wo.z == 0 || hero.wi.z == 0)
        return out;
    if (K != 0 && out.delta) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (p.active_mask & (1u << k)) {
                float mass, density, eta;
                out.valid = dirac_lane(p, k, wo, hero.wi, ux, uy, mass, density, eta) && out.valid;
                out.numerator.v[k] = mass;
                out.pdf.v[k] = density;
                out.eta.v[k] = eta;
            }
    } else {
        const HeroEval e = hero_evaluate_k<K>(p, wo, hero.wi);
        out.numerator = scale4(e.f, fabsf(hero.wi.z));
        out.pdf = e.pdf;
        out.valid = e.valid;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if ((p.active_mask & (1u << k)) && out.pdf.v[k] > 0)
                out.eta.v[k] = event_eta(p, k, wo, hero.wi);
    }
    out.pdf.v[0] = hero.pdf;
    out.eta.v[0] = p.kind == 2 ? hero_eta : event_eta(p, 0, wo, hero.wi);
    bool eta_ok = true;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        eta_ok = eta_ok && isfinite(out.eta.v[k]) && out.eta.v[k] > 0;
    out.valid = out.valid && finite_nonnegative4(out.numerator) && finite_nonnegative4(out.pdf) && eta_ok;
    out.accepted = out.valid && nonzero4(out.numerator);
    return out;
}

// ------------------------------------------------------------------ spectra and geometry helpers
// shaders/render.metal:548-574
RP_DEV float pbrt_reflectance(const float2 *k, u32 count, float w) {
    if (w < k[0].x || w > k[count - 1].x)
        return 0.0f;
    u32 lo = 0, hi = count - 1;
    while (hi - lo > 1) {
        const u32 mid = lo + (hi - lo) / 2;
        if (w < k[mid].x)
            hi = mid;
        else
            lo = mid;
    }
    if (lo == hi)
        return k[lo].y;
    const float a = k[lo].x, b = k[hi].x;
    const float span = b - a;
    const float t = isfinite(span) ? (w - a) / span : (0.5f * w - 0.5f * a) / (0.5f * b - 0.5f * a);
    return k[lo].y + (k[hi].y - k[lo].y) * t;
}
// shaders/render.metal:590-616
RP_DEV float blackbody_reflectance(float factor, float w) {
    if (!(w >= 360.0f && w <= 830.0f))
        return 0.0f;
    if (!(factor > 0.0f && isfinite(factor)))
        return __int_as_float(0x7fffffff);
    const float x = factor / w;
    if (x >= 128.0f)
        return 0.0f;
    const float x_peak = 4.965114268247028f;
    const float log_peak_factor = -0.007001607544495994f;
    const float f = x < 0.0625f ? x * (1.0f + x * (-0.5f + x * (1.0f / 6.0f + x * (-1.0f / 24.0f + x / 120.0f))))
                                : 1.0f - expf(-x);
    const float log_rho = 5.0f * logf(x / x_peak) + x_peak - x + log_peak_factor - logf(f);
    return fminf(fmaxf(expf(log_rho), 0.0f), 1.0f);
}
// shaders/render.metal:627-630
RP_DEV u32 dense_index(float w) {
    const u32 nm = u32(w);
    return nm + u32(w - float(nm) >= 0.5f) - 360u;
}
// shaders/render.metal:1978-1990
RP_DEV float optical_value(const float2 *knots, u32 begin, u32 count, u32 total, bool extend, float w) {
    if (count < 2 || begin > total || count > total - begin)
        return __int_as_float(0x7fffffff);
    const float2 *c = knots + begin;
    if (extend) {
        if (w < c[0].x)
            return c[0].y;
        if (w > c[count - 1].x)
            return c[count - 1].y;
    }
    return pbrt_reflectance(c, count, w);
}
// shaders/render.metal:849-852
RP_DEV float gamma_bound(float n) {
    const float u = 0x1.0p-24f;
    return n * u / (1.0f - n * u);
}
// src/offset_rounding_shared.h:27-41 and shaders/render.metal:854-863
RP_DEV float round_out1(float p, float n) {
    if (n == 0.0f)
        return p;
    const bool toward_negative = signbit(n);
    const u32 bits = fbits(p);
    const u32 m = bits & 0x7fffffffu, s = bits & 0x80000000u;
    if (m > 0x7f7fffffu)
        return p;
    if (m == 0)
        return ffrom((toward_negative ? 0x80000000u : 0u) | 0x00800000u);
    const bool away = ((s != 0) == toward_negative);
    if (away)
        return ffrom(s | (m < 0x00800000u ? 0x00800000u : m + 1u));
    return ffrom(s | (m <= 0x00800000u ? 0u : m - 1u));
}
RP_DEV V3 round_out(V3 p, V3 n) { return v3(round_out1(p.x, n.x), round_out1(p.y, n.y), round_out1(p.z, n.z)); }
// shaders/surface_detail.h:35-43
RP_DEV bool unit_vector(V3 v, V3 &out) {
    const float s = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
    if (!(s > 0.0f) || !finite3(v))
        return false;
    out = normalize3(v / s);
    return finite3(out);
}
struct Frame {
    V3 x, y, z;
};
RP_DEV V3 to_local(const Frame &f, V3 v) { return v3(dot(f.x, v), dot(f.y, v), dot(f.z, v)); }
RP_DEV V3 to_world(const Frame &f, V3 v) { return v.x * f.x + v.y * f.y + v.z * f.z; }
// shaders/surface_detail.h:49-55 followed by scattering_frame (shaders/render.metal:2039-2053)
RP_DEV bool shading_frame(V3 n, Frame &r) {
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    const V3 dpdu = v3(1 + sign * n.x * n.x * a, sign * b, -sign * n.x);
    if (!unit_vector(n, r.z) || !unit_vector(dpdu, r.x))
        return false;
    const float projection = dot(r.x, r.z);
    if (!isfinite(projection))
        return false;
    if (!unit_vector(r.x - projection * r.z, r.x))
        return false;
    if (fabsf(dot(r.x, r.z)) > 64.0f * kFltEps)
        return false;
    r.y = cross(r.z, r.x);
    return finite3(r.y);
}

} // namespace rp
