// ORACLE -- test infrastructure only.  CPU restatement of rypath's spectral path-tracing
// arithmetic, used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
// checker.  Nothing in the product links or calls this code.
//
// Every function names the reference file:line it restates.  Compile with
// -ffp-contract=off so binary32 expressions round exactly as written.
#pragma once

#include <algorithm>
#include <array>
#include <bit>
#include <cfloat>
#include <cmath>
#include <vector>
#include <cstdint>
#include <cstring>

namespace oracle {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

// ---------------------------------------------------------------- small vector types
struct F3 {
    float x = 0, y = 0, z = 0;
    float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline F3 f3(float x, float y, float z) { return {x, y, z}; }
inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
inline F3 operator*(float s, F3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 operator*(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline F3 operator/(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline F3 operator/(F3 a, F3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline F3 fabs3(F3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline bool finite3(F3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline bool zero3(F3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
inline bool any_nonzero3(F3 a) { return a.x != 0 || a.y != 0 || a.z != 0; }
inline bool eq3(F3 a, F3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline float length3(F3 a) { return std::sqrt(dot(a, a)); }
// Metal normalize: v * rsqrt(dot(v, v)); restated as a divide by the exact-rounded root.
inline F3 normalize3(F3 a) { return a / std::sqrt(dot(a, a)); }
inline F3 fma3(F3 a, F3 b, F3 c) {
    return {std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y), std::fma(a.z, b.z, c.z)};
}
inline float max3(F3 a) { return std::max(std::max(a.x, a.y), a.z); }

struct F4 {
    float v[4] = {0, 0, 0, 0};
    float &operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
inline F4 f4(float s) { return {{s, s, s, s}}; }
inline F4 operator*(F4 a, F4 b) {
    return {{a[0] * b[0], a[1] * b[1], a[2] * b[2], a[3] * b[3]}};
}
inline F4 operator*(F4 a, float s) { return {{a[0] * s, a[1] * s, a[2] * s, a[3] * s}}; }
inline F4 operator/(F4 a, float s) { return {{a[0] / s, a[1] / s, a[2] / s, a[3] / s}}; }
inline F4 operator+(F4 a, F4 b) {
    return {{a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3]}};
}
// shaders/packet_transport.h:49-50
inline bool nonzero4(F4 v) { return v[0] > 0 || v[1] > 0 || v[2] > 0 || v[3] > 0; }
inline bool finite_nonnegative4(F4 v) {
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(v[i]) || !(v[i] >= 0))
            return false;
    return true;
}

inline u32 fbits(float x) { return std::bit_cast<u32>(x); }
inline float ffrom(u32 x) { return std::bit_cast<float>(x); }

// ---------------------------------------------------------------- Sobol (src/sobol_shared.h)
constexpr u32 sobol_dimensions = 1024, sobol_matrix = 52, sobol_max_scale = 25;
struct SobolTables {
    u32 directions[sobol_dimensions * sobol_matrix];
    u64 intervals[sobol_max_scale * sobol_matrix];
    u64 inverse[(sobol_max_scale + 1) * sobol_matrix];
};
static_assert(sizeof(SobolTables) == 234208);

// src/sobol_shared.h:56-76
inline u64 sobol_index(const SobolTables &t, u32 m, u32 x, u32 y, u64 sample) {
    if (m == 0)
        return sample;
    const u32 row = (m - 1) * sobol_matrix;
    u64 result = sample << (2 * m);
    u64 delta = 0;
    for (u32 c = row; sample != 0; ++c, sample >>= 1)
        if (sample & 1)
            delta ^= t.intervals[c];
    u64 bits = ((u64(x) << m) | y) ^ delta;
    for (u32 c = row; bits != 0; ++c, bits >>= 1)
        if (bits & 1)
            result ^= t.inverse[c];
    return result;
}
// src/sobol_shared.h:79-89 (MurmurHash64A of LE32(dimension) || LE32(seed))
inline u32 sobol_dimension_hash(u32 dimension, u32 seed) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    u64 block = ((u64(seed) << 32) | dimension) * m;
    block ^= block >> 47;
    block *= m;
    u64 h = (8 * m ^ block) * m;
    h ^= h >> 47;
    h *= m;
    return u32(h ^ (h >> 47));
}
// src/sobol_shared.h:91-97
inline u32 reverse_bits(u32 v) {
    v = (v << 16) | (v >> 16);
    v = ((v & 0x00ff00ffu) << 8) | ((v & 0xff00ff00u) >> 8);
    v = ((v & 0x0f0f0f0fu) << 4) | ((v & 0xf0f0f0f0u) >> 4);
    v = ((v & 0x33333333u) << 2) | ((v & 0xccccccccu) >> 2);
    return ((v & 0x55555555u) << 1) | ((v & 0xaaaaaaaau) >> 1);
}
// src/sobol_shared.h:99-105
inline u64 mix_bits(u64 v) {
    v ^= v >> 31;
    v *= 0x7fb5d329728ea185ull;
    v ^= v >> 27;
    v *= 0x81dadef4bc2dd44dull;
    return v ^ (v >> 33);
}
// src/sobol_shared.h:108-141
// the randomisations of a 32-bit word with a 32-bit hash (src/sobol_shared.h:115-141,
// src/qmc_shared.h:190-212)
inline u32 scramble_word(u32 value, u32 mode, u32 hash) {
    if (mode == 0)
        return value;
    if (mode == 1)
        return value ^ hash;
    if (mode == 2) {
        value = reverse_bits(value);
        value ^= value * 0x3d20adeau;
        value += hash;
        value *= (hash >> 16) | 1;
        value ^= value * 0x05526c56u;
        value ^= value * 0x53a22864u;
        return reverse_bits(value);
    }
    value ^= (hash & 1) << 31;
    for (u32 bit = 1; bit < 32; ++bit) {
        const u32 prefix = value & (~u32(0) << (32 - bit));
        if (u32(mix_bits(prefix ^ hash)) & (u32(1) << bit))
            value ^= u32(1) << (31 - bit);
    }
    return value;
}
inline u32 sobol_raw(const SobolTables &t, u64 index, u32 dimension) {
    u32 value = 0;
    for (u32 c = dimension * sobol_matrix; index != 0; ++c, index >>= 1)
        if (index & 1)
            value ^= t.directions[c];
    return value;
}
inline u32 sobol_word(const SobolTables &t, u64 index, u32 dimension, u32 mode, u32 seed) {
    const u32 value = sobol_raw(t, index, dimension);
    return mode == 0 ? value : scramble_word(value, mode, sobol_dimension_hash(dimension, seed));
}

// ---------------------------------------------------------------- Halton / ZSobol
// src/qmc_shared.h (PBRT v4 HaltonSampler / ZSobolSampler arithmetic)
// the first 1000 primes, the Halton bases (:14-18)
inline const u32 *qmc_primes() {
    static const std::vector<u32> primes = [] {
        std::vector<u32> out;
        for (u32 n = 2; out.size() < 1000; ++n) {
            bool prime = true;
            for (u32 q : out) {
                if (q * q > n)
                    break;
                if (n % q == 0) {
                    prime = false;
                    break;
                }
            }
            if (prime)
                out.push_back(n);
        }
        return out;
    }();
    return primes.data();
}
// :20-40
inline u64 qmc_hash2(u32 a, u32 b) {
    const u64 m = 0xc6a4a7935bd1e995ull;
    u64 k = ((u64(b) << 32) | a) * m;
    k ^= k >> 47;
    k *= m;
    u64 h = (8 * m ^ k) * m;
    h ^= h >> 47;
    h *= m;
    return h ^ (h >> 47);
}
inline u64 qmc_hash3(u32 a, u32 b, u32 c) {
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
// :41-66 (Kensler's hashed permutation by cycle walking)
inline u32 qmc_permutation(u32 i, u32 l, u32 p) {
    u32 w = l - 1;
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    do {
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
    } while (i >= l);
    return (i + p) % l;
}
// :84-106
inline float qmc_radical(u32 dimension, u64 a, u32 mode = 0, u32 seed = 0) {
    const u32 base = qmc_primes()[dimension];
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
    return value < 0x1.fffffep-1f ? value : 0x1.fffffep-1f;
}
// :107-148
inline u32 qmc_base_scale(u32 resolution, u32 base) {
    u32 scale = 1;
    while (scale < std::min(resolution, 128u))
        scale *= base;
    return scale;
}
inline u64 halton_index(u32 width, u32 height, u32 x, u32 y, u64 sample) {
    const u32 sx = qmc_base_scale(width, 2), sy = qmc_base_scale(height, 3), stride = sx * sy;
    const auto exponent = [](u32 scale, u32 base) {
        u32 e = 0;
        for (; scale > 1; scale /= base)
            ++e;
        return e;
    };
    const auto inverse_radical = [](u32 a, u32 base, u32 count) {
        u64 r = 0;
        for (u32 i = 0; i < count; ++i, a /= base)
            r = r * base + a % base;
        return r;
    };
    const auto inverse_mod = [](u32 a, u32 modulus) -> u32 {
        if (modulus == 1)
            return 0;
        for (u32 i = 1; i < modulus; ++i)
            if ((a * i) % modulus == 1)
                return i;
        return 0;
    };
    u64 offset = 0;
    if (stride > 1) {
        offset = inverse_radical(x % 128, 2, exponent(sx, 2)) * sy * inverse_mod(sy, sx);
        offset += inverse_radical(y % 128, 3, exponent(sy, 3)) * sx * inverse_mod(sx, sy);
        offset %= stride;
    }
    return offset + sample * stride;
}
// :176-179
inline float halton_camera(u32 axis, u32 resolution, u64 index) {
    return qmc_radical(axis, index / qmc_base_scale(resolution, axis == 0 ? 2 : 3));
}
// :213-220
inline u64 zsobol_morton(u32 x, u32 y, u32 log_spp, u64 sample) {
    u64 result = 0;
    for (u32 b = 0; b < 26; ++b) {
        result |= u64((x >> b) & 1) << (2 * b);
        result |= u64((y >> b) & 1) << (2 * b + 1);
    }
    return (result << log_spp) | sample;
}
// :221-238
inline u64 zsobol_index(u64 morton, u32 dimension, u32 exponent, u32 log_spp) {
    static const u32 permutations[24][4] = {
        {0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 2, 1}, {0, 3, 1, 2},
        {1, 0, 2, 3}, {1, 0, 3, 2}, {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 2, 0}, {1, 3, 0, 2},
        {2, 1, 0, 3}, {2, 1, 3, 0}, {2, 0, 1, 3}, {2, 0, 3, 1}, {2, 3, 0, 1}, {2, 3, 1, 0},
        {3, 1, 2, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 2, 0, 1}, {3, 0, 2, 1}, {3, 0, 1, 2}};
    const u32 odd = log_spp & 1;
    const u32 digits = exponent + (log_spp + 1) / 2;
    u64 result = 0;
    for (int i = int(digits) - 1; i >= int(odd); --i) {
        const u32 shift = 2 * u32(i) - odd;
        const u32 digit = u32((morton >> shift) & 3);
        const u64 higher = morton >> (shift + 2);
        const u32 p = u32((mix_bits(higher ^ u32(0x55555555u * dimension)) >> 24) % 24);
        result |= u64(permutations[p][digit]) << shift;
    }
    if (odd)
        result |= (morton & 1) ^ (mix_bits((morton >> 1) ^ u32(0x55555555u * dimension)) & 1);
    return result;
}
// :244-249
inline u32 zsobol_word(const SobolTables &t, u64 morton, u32 dimension, u32 axis, bool pair, u32 exponent,
                       u32 log_spp, u32 mode, u32 seed) {
    const u64 index = zsobol_index(morton, dimension, exponent, log_spp);
    const u64 hash = qmc_hash2(dimension + (pair ? 2 : 1), seed);
    const u32 random = pair && axis == 1 ? u32(hash >> 32) : u32(hash);
    return scramble_word(sobol_raw(t, index, axis), mode, random);
}
// src/sobol_shared.h:143-146
inline float sobol_uniform(u32 v) {
    const float unit = float(v) * 0x1p-32f;
    return unit < 0x1.fffffep-1f ? unit : 0x1.fffffep-1f;
}
// src/sobol_shared.h:148-154
inline float sobol_camera_uniform(u32 global, u32 m, u32 pixel) {
    const float local = sobol_uniform(global) * float(u32(1) << m) - float(pixel);
    if (local < 0.0f)
        return 0.0f;
    return local < 0x1.fffffep-1f ? local : 0x1.fffffep-1f;
}
// src/sampling.cpp:41-43 (std::bit_width(max(w, h, 1) - 1))
inline u32 sobol_scale_exponent(u32 w, u32 h) {
    u32 v = std::max(std::max(w, h), 1u) - 1;
    return v == 0 ? 0 : 32 - std::countl_zero(v);
}

// ---------------------------------------------------------------- Philox (shaders/render.metal:97-111)
struct U4 {
    u32 x, y, z, w;
};
inline u32 mulhi(u32 a, u32 b) { return u32((u64(a) * b) >> 32); }
inline U4 philox(U4 c, u32 k0, u32 k1) {
    for (int r = 0; r < 10; ++r) {
        const U4 n{mulhi(0xcd9e8d57u, c.z) ^ c.y ^ k0, 0xcd9e8d57u * c.z,
                   mulhi(0xd2511f53u, c.x) ^ c.w ^ k1, 0xd2511f53u * c.x};
        c = n;
        k0 += 0x9e3779b9u;
        k1 += 0xbb67ae85u;
    }
    return c;
}
// shaders/render.metal:111
inline float u01(u32 w) { return float(w >> 8) * 0x1.0p-24f; }

// ---------------------------------------------------------------- hero likelihoods (src/hero_spectrum_shared.h)
// src/hero_spectrum_shared.h:32
inline bool nonnegative_finite(float x) { return fbits(x) < 0x7f800000u || fbits(x) == 0x80000000u; }
struct Number {
    float fraction = 0;
    int exponent = 0;
};
// :37-43
inline Number normalized(float x, int exponent) {
    if (x == 0)
        return {};
    int e;
    const float m = std::frexp(x, &e);
    return {m, exponent + e};
}
// :44-51
inline Number number(float x) {
    const u32 w = fbits(x) & 0x7fffffffu;
    if (w == 0)
        return {};
    if ((w & 0x7f800000u) == 0)
        return normalized(float(w), -149);
    return normalized(x, 0);
}
// :52-56
inline Number multiply(Number a, Number b) {
    if (a.fraction == 0 || b.fraction == 0)
        return {};
    return normalized(a.fraction * b.fraction, a.exponent + b.exponent);
}
// :57-59
inline Number divide(Number a, Number b) {
    return normalized(a.fraction / b.fraction, a.exponent - b.exponent);
}
// :60-74
inline Number add(Number a, Number b) {
    if (a.fraction == 0)
        return b;
    if (b.fraction == 0)
        return a;
    if (a.exponent < b.exponent)
        std::swap(a, b);
    const int gap = a.exponent - b.exponent;
    if (gap > 24)
        return a;
    return normalized(a.fraction + std::ldexp(b.fraction, -gap), a.exponent);
}
struct Scalar {
    float value = 0;
    bool valid = false;
};
// :79-99
inline Scalar materialize(Number x) {
    if (x.fraction == 0)
        return {0, true};
    if (!(x.fraction >= .5f && x.fraction < 1) || x.exponent > 128)
        return {};
    if (x.exponent >= -125) {
        const float value = std::ldexp(x.fraction, x.exponent);
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
// :103-108
inline Density initial_density() {
    Density d;
    for (int k = 0; k < 4; ++k)
        d.lane[k] = number(1);
    return d;
}
// :109-111
inline Number total(const Density &p) {
    return add(add(p.lane[0], p.lane[1]), add(p.lane[2], p.lane[3]));
}
// :112-117
inline Number mixture(const Density &p, F4 pdf) {
    Number t[4];
    for (int k = 0; k < 4; ++k)
        t[k] = multiply(p.lane[k], number(pdf[k]));
    return add(add(t[0], t[1]), add(t[2], t[3]));
}
struct Update {
    Density density;
    F4 beta;
    bool valid = false;
};
// :123-144
inline Update advance(const Density &prefix, F4 beta, F4 numerator, F4 pdf) {
    Update out{};
    for (int k = 0; k < 4; ++k) {
        if (!nonnegative_finite(pdf[k]) || !nonnegative_finite(numerator[k]) ||
            !nonnegative_finite(beta[k]))
            return out;
        out.density.lane[k] = multiply(prefix.lane[k], number(pdf[k]));
    }
    const Number before = total(prefix), after = total(out.density);
    if (!(before.fraction > 0 && after.fraction > 0))
        return out;
    const Number ratio = divide(before, after);
    for (int k = 0; k < 4; ++k) {
        const auto value = materialize(multiply(multiply(number(beta[k]), number(numerator[k])), ratio));
        if (!value.valid)
            return out;
        out.beta[k] = value.value;
    }
    out.valid = true;
    return out;
}
// :145-153
inline Scalar balance(const Density &prefix, F4 sampled, F4 other) {
    for (int k = 0; k < 4; ++k)
        if (!nonnegative_finite(sampled[k]) || !nonnegative_finite(other[k]))
            return {};
    const Number a = mixture(prefix, sampled), b = mixture(prefix, other), sum = add(a, b);
    if (!(sum.fraction > 0))
        return {};
    return materialize(divide(a, sum));
}
struct Contribution {
    F4 value;
    bool valid = false;
};
// :161-180
inline Contribution balance_contribution(const Density &prefix, F4 value, F4 sampled, F4 other) {
    Contribution r{};
    for (int k = 0; k < 4; ++k)
        if (!nonnegative_finite(value[k]) || !nonnegative_finite(sampled[k]) ||
            !nonnegative_finite(other[k]))
            return r;
    const Number a = mixture(prefix, sampled), b = mixture(prefix, other), sum = add(a, b);
    if (!(sum.fraction > 0))
        return r;
    const Number weight = divide(a, sum);
    for (int k = 0; k < 4; ++k) {
        const auto w = materialize(multiply(number(value[k]), weight));
        if (!w.valid)
            return r;
        r.value[k] = w.value;
    }
    r.valid = true;
    return r;
}
// :183-195
inline Update collapse(const Density &prefix, F4 beta) {
    Update out{};
    if (!(prefix.lane[0].fraction > 0) || !nonnegative_finite(beta[0]))
        return out;
    const auto value = materialize(multiply(number(beta[0]), divide(total(prefix), prefix.lane[0])));
    if (!value.valid)
        return out;
    out.density.lane[0] = number(1);
    out.beta[0] = value.value;
    out.valid = true;
    return out;
}

// ---------------------------------------------------------------- wavelengths
struct Wavelengths {
    float lambda[4], pdf[4];
};
// src/packet_spectrum_shared.h:27-31
inline float visible_pdf(float lambda) {
    if (lambda < 360 || lambda > 830)
        return 0;
    const float c = std::cosh(.0072f * (lambda - 538));
    return .0039398042f / (c * c);
}
// src/hero_spectrum_shared.h:199-202
inline float shifted_cdf(float u, u32 lane) {
    const u32 coordinate = u32(u * 16777216.f);
    return float((coordinate + lane * 4194304u) & 0x00ffffffu) * 0x1p-24f;
}
// src/hero_spectrum_shared.h:203-224
inline Wavelengths sample_visible(float u) {
    Wavelengths out{};
    if (!(u >= 0 && u < 1)) {
        for (int k = 0; k < 4; ++k)
            out.lambda[k] = out.pdf[k] = NAN;
        return out;
    }
    for (u32 k = 0; k < 4; ++k) {
        const float s = shifted_cdf(u, k);
        float w = 538 - 138.888889f * std::atanh(.85691062f - 1.82750197f * s);
        if (w < 360)
            w = 360;
        if (w > 830)
            w = 830;
        out.lambda[k] = w;
        out.pdf[k] = visible_pdf(w);
    }
    return out;
}
// src/hero_spectrum_shared.h:225-244
inline Wavelengths sample_uniform(float u) {
    Wavelengths out{};
    if (!(u >= 0 && u < 1)) {
        for (int k = 0; k < 4; ++k)
            out.lambda[k] = out.pdf[k] = NAN;
        return out;
    }
    for (int k = 0; k < 4; ++k) {
        float s = u + float(k) * .25f;
        if (s >= 1)
            s -= 1;
        float w = 360 + 470 * s;
        if (w >= 830)
            w = ffrom(fbits(830.f) - 1);
        out.lambda[k] = w;
        out.pdf[k] = 1.f / 470.f;
    }
    return out;
}

// ---------------------------------------------------------------- roulette (src/packet_roulette_shared.h)
// :21-25
inline bool rr_finite(float v) { return (fbits(v) & 0x7fffffffu) < 0x7f800000u; }
inline bool positive_normal(float v) {
    const u32 w = fbits(v);
    return w >= 0x00800000u && w < 0x7f800000u;
}
// :28
inline bool opposite_hemispheres(float a, float b) { return (a > 0 && b < 0) || (a < 0 && b > 0); }
struct EtaScale {
    float value = 1;
    bool enabled = true;
};
// :38-51
inline void account_transmission(EtaScale &s, float eta, bool transmission) {
    if (!s.enabled || !transmission)
        return;
    if (!positive_normal(eta)) {
        s.enabled = false;
        return;
    }
    const float square = eta * eta;
    const float next = s.value * square;
    if (!positive_normal(square) || !positive_normal(next)) {
        s.enabled = false;
        return;
    }
    s.value = next;
}
struct Decision {
    F4 survivor;
    float termination = 0;
    bool eligible = false;
};
// :59-94
inline Decision rr_prepare(F4 beta, const EtaScale &s, u32 depth) {
    Decision r{beta, 0, false};
    if (!s.enabled || depth <= 1 || !positive_normal(s.value))
        return r;
    float maximum = 0;
    for (int k = 0; k < 4; ++k) {
        const float v = beta[k];
        if (!rr_finite(v) || ((fbits(v) >> 31) && (fbits(v) & 0x7fffffffu)))
            return r;
        if (v > maximum)
            maximum = v;
    }
    const float m = maximum * s.value;
    if (!positive_normal(m) || m >= 1)
        return r;
    const float q = 1 - m;
    const float survival = 1 - q;
    if (!rr_finite(q) || !(q > 0 && q < 1) || !positive_normal(survival))
        return r;
    for (int k = 0; k < 4; ++k) {
        if ((fbits(beta[k]) & 0x7fffffffu) == 0)
            continue;
        const float v = beta[k] / survival;
        if (!positive_normal(v))
            return Decision{beta, 0, false};
        r.survivor[k] = v;
    }
    r.termination = q;
    r.eligible = true;
    return r;
}

// ---------------------------------------------------------------- hero track (shaders/hero_pt_helpers.h)
struct HeroTrack {
    Density density = initial_density();
    Density previous = initial_density();
    F4 eta_scale = f4(1);
    u32 active_mask = 15;
    bool roulette_enabled = true;
};
// shaders/hero_pt_helpers.h:56-85
inline bool hero_continue(F4 &beta, const HeroTrack &track, u32 depth, float uniform) {
    if (!track.roulette_enabled || depth <= 1)
        return true;
    float maximum = 0;
    for (int k = 0; k < 4; ++k) {
        const float v = beta[k] * track.eta_scale[k];
        if (!std::isfinite(v) || v < 0 || (beta[k] > 0 && !positive_normal(v)))
            return true;
        maximum = std::max(maximum, v);
    }
    const EtaScale unit{};
    const auto d = rr_prepare(f4(maximum), unit, depth);
    if (!d.eligible)
        return true;
    const float survival = 1 - d.termination;
    F4 survivor = beta;
    for (int k = 0; k < 4; ++k) {
        if (fbits(beta[k]) == 0)
            continue;
        survivor[k] /= survival;
        if (!positive_normal(survivor[k]))
            return true;
    }
    if (uniform < d.termination)
        return false;
    beta = survivor;
    return true;
}
// shaders/hero_pt_helpers.h:86-98
inline void hero_account_eta(HeroTrack &track, F4 eta, bool transmission) {
    if (!transmission || !track.roulette_enabled)
        return;
    for (int k = 0; k < 4; ++k) {
        EtaScale lane{track.eta_scale[k], true};
        account_transmission(lane, eta[k], true);
        if (!lane.enabled) {
            track.roulette_enabled = false;
            return;
        }
        track.eta_scale[k] = lane.value;
    }
}

// ---------------------------------------------------------------- BSDFs
constexpr float pi_f = 3.14159265358979323846f;
struct Eval {
    float f, pdf;
    bool valid;
};
struct BSample {
    F3 wi;
    float weight, pdf;
    bool delta, accepted, valid;
};
// shaders/transmission.h:10-12
inline bool randoms(float uc, float ux, float uy) {
    return std::isfinite(uc) && uc >= 0 && uc < 1 && std::isfinite(ux) && std::isfinite(uy) &&
           ux >= 0 && uy >= 0 && ux < 1 && uy < 1;
}
// shaders/transmission.h:52-62 (R, T = 0 for the opaque diffuse lane)
inline Eval diffuse_evaluate(float R, float T, F3 wo, F3 wi) {
    if (!std::isfinite(R) || !std::isfinite(T) || R < 0 || T < 0 || !finite3(wo) || !finite3(wi))
        return {0, 0, false};
    const float sum = R + T;
    if (!std::isfinite(sum))
        return {0, 0, false};
    if (wo.z == 0 || wi.z == 0 || sum == 0)
        return {0, 0, true};
    const float value = (wo.z > 0) == (wi.z > 0) ? R : T;
    return {value / pi_f, value / sum * std::fabs(wi.z) / pi_f, true};
}
// shaders/packet_scattering.h:170-184 (PBRT SampleUniformDiskConcentric + cosine lift)
inline F3 diffuse_concentric_cosine(float ux, float uy) {
    const float ox = 2 * ux - 1, oy = 2 * uy - 1;
    if (ox == 0 && oy == 0)
        return {0, 0, 1};
    float radius, theta;
    if (std::fabs(ox) > std::fabs(oy)) {
        radius = ox;
        theta = (pi_f / 4) * (oy / ox);
    } else {
        radius = oy;
        theta = (pi_f / 2) - (pi_f / 4) * (ox / oy);
    }
    const float dx = radius * std::cos(theta), dy = radius * std::sin(theta);
    return {dx, dy, std::sqrt(std::max(0.0f, 1 - (dx * dx + dy * dy)))};
}
// shaders/packet_scattering.h:185-203
inline BSample diffuse_reflection_sample(float R, F3 wo, float uc, float ux, float uy) {
    BSample s{{0, 0, 0}, 0, 0, false, false, true};
    const float sum = R + 0.0f;
    if (!std::isfinite(R) || R < 0 || !std::isfinite(sum) || !finite3(wo) || !randoms(uc, ux, uy)) {
        s.valid = false;
        return s;
    }
    if (sum == 0 || wo.z == 0)
        return s;
    s.wi = diffuse_concentric_cosine(ux, uy);
    if (wo.z < 0)
        s.wi.z = -s.wi.z;
    s.pdf = R / sum * std::fabs(s.wi.z) / pi_f;
    s.weight = sum;
    s.accepted = s.pdf > 0;
    return s;
}

struct Conductor {
    float eta, k, alpha_x, alpha_y;
    bool smooth;
};
// shaders/conductor.h:22-34
inline bool conductor_prepare(float eta, float k, float u, float v, bool remap, Conductor &p) {
    if (!std::isfinite(eta) || !std::isfinite(k) || !std::isfinite(u) || !std::isfinite(v) ||
        eta < 0 || k < 0 || u < 0 || v < 0 || (eta == 0 && k == 0))
        return false;
    p = {eta, k, remap ? std::sqrt(u) : u, remap ? std::sqrt(v) : v, false};
    p.smooth = std::max(p.alpha_x, p.alpha_y) < 1e-3f;
    if (!p.smooth) {
        p.alpha_x = std::max(p.alpha_x, 1e-4f);
        p.alpha_y = std::max(p.alpha_y, 1e-4f);
    }
    return true;
}
// shaders/conductor.h:35-42
inline bool unit(F3 v, F3 &out) {
    const float s = std::max(std::max(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    if (!(s > 0) || !std::isfinite(s))
        return false;
    v = v / s;
    out = v / std::sqrt(dot(v, v));
    return finite3(out);
}
// shaders/conductor.h:43-51
inline bool complex_ratio_norm(float ax, float ay, float bx, float by, float &out) {
    const float s = std::max(std::fabs(bx), std::fabs(by));
    if (!(s > 0) || !std::isfinite(s) || !std::isfinite(ax) || !std::isfinite(ay))
        return false;
    ax /= s;
    ay /= s;
    bx /= s;
    by /= s;
    out = (ax * ax + ay * ay) / (bx * bx + by * by);
    return std::isfinite(out);
}
// shaders/conductor.h:53-57
inline void two_sum(float a, float b, float &sum, float &err) {
    sum = a + b;
    const float bv = sum - a;
    err = (a - (sum - bv)) + (b - bv);
}
// shaders/conductor.h:58-102
inline bool conductor_fresnel(float cosine, float eta, float k, float &f) {
    if (!std::isfinite(cosine) || !std::isfinite(eta) || !std::isfinite(k) || eta < 0 || k < 0 ||
        (eta == 0 && k == 0))
        return false;
    const float c = std::clamp(cosine, 0.0f, 1.0f);
    if (eta == 1 && k == 0) {
        f = 0;
        return true;
    }
    if (c == 0) {
        f = 1;
        return true;
    }
    const float n2x = eta * eta - k * k, n2y = 2 * eta * k;
    if (!std::isfinite(n2x) || !std::isfinite(n2y))
        return false;
    const float eta2 = eta * eta, k2 = k * k, c2 = c * c;
    float abx, aby, cdx, cdy, tx, ty;
    two_sum(eta2, -k2, abx, aby);
    two_sum(c2, -1, cdx, cdy);
    two_sum(abx, cdx, tx, ty);
    const float correction = aby + cdy + ty + std::fma(eta, eta, -eta2) - std::fma(k, k, -k2) +
                             std::fma(c, c, -c2);
    const float zx = tx + correction, zy = n2y;
    const float scale = std::max(std::fabs(zx), std::fabs(zy));
    float radius = 0;
    if (scale != 0) {
        const float sx = zx / scale, sy = zy / scale;
        radius = scale * std::sqrt(sx * sx + sy * sy);
    }
    if (!std::isfinite(radius))
        return false;
    float qr, qi;
    if (zx >= 0) {
        qr = std::sqrt(std::max(0.0f, 0.5f * radius + 0.5f * zx));
        qi = qr > 0 ? zy / (2 * qr) : 0;
    } else {
        qi = std::sqrt(std::max(0.0f, 0.5f * radius - 0.5f * zx));
        qr = qi > 0 ? zy / (2 * qi) : 0;
    }
    float rs, rp;
    if (!complex_ratio_norm(c - qr, 0 - qi, c + qr, 0 + qi, rs) ||
        !complex_ratio_norm(n2x * c - qr, n2y * c - qi, n2x * c + qr, n2y * c + qi, rp))
        return false;
    f = (rs + rp) * 0.5f;
    return std::isfinite(f) && f >= 0;
}
// shaders/conductor.h:103-107
inline float ggx_lambda(float ax, float ay, F3 w) {
    const F3 v{1, ax * w.x / w.z, ay * w.y / w.z};
    const float s = std::max(std::max(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    return 0.5f * (s * length3(v / s) - 1);
}
// shaders/conductor.h:108-119
inline float ggx_distribution(float ax, float ay, F3 m) {
    if (m.z * m.z * m.z * m.z < 1e-16f)
        return 0;
    const F3 v{m.x / ax, m.y / ay, m.z};
    const float t = dot(v, v);
    const float den = pi_f * ax * ay * t * t;
    if (!std::isfinite(den) || !(den > 0))
        return NAN;
    const float d = 1 / den;
    return d > 0 ? d : NAN;
}
// shaders/conductor.h:120-138
inline Eval conductor_evaluate(const Conductor &p, F3 wo, F3 wi) {
    if (!finite3(wo) || !finite3(wi))
        return {0, 0, false};
    if (p.smooth || wo.z == 0 || wi.z == 0 || ((wo.z > 0) != (wi.z > 0)))
        return {0, 0, true};
    F3 m;
    if (!unit(wo + wi, m))
        return {0, 0, false};
    float f;
    if (!conductor_fresnel(std::fabs(dot(wo, m)), p.eta, p.k, f))
        return {0, 0, false};
    const float lo = ggx_lambda(p.alpha_x, p.alpha_y, wo), li = ggx_lambda(p.alpha_x, p.alpha_y, wi),
                d = ggx_distribution(p.alpha_x, p.alpha_y, m);
    const float value = d * f / (4 * std::fabs(wo.z) * std::fabs(wi.z) * (1 + lo + li));
    const float pdf = d / (4 * std::fabs(wo.z) * (1 + lo));
    const bool valid = std::isfinite(lo) && std::isfinite(li) && std::isfinite(d) &&
                       std::isfinite(value) && std::isfinite(pdf) && value >= 0 && pdf >= 0;
    return {value, pdf, valid};
}
// Visible-normal sampling shared by conductor.h:157-185 and dielectric.h:160-188.
inline bool ggx_visible_normal(float ax, float ay, F3 wo, float ux, float uy, F3 &m) {
    F3 wh;
    if (!unit(F3{ax * wo.x, ay * wo.y, wo.z}, wh))
        return false;
    if (wh.z < 0)
        wh = -wh;
    F3 t1;
    if (wh.z < 0.99999f) {
        if (!unit(F3{-wh.y, wh.x, 0}, t1))
            return false;
    } else
        t1 = F3{1, 0, 0};
    const F3 t2 = cross(wh, t1);
    const float r = std::sqrt(ux), phi = 2 * pi_f * uy;
    float dx = r * std::cos(phi), dy = r * std::sin(phi);
    const float h = std::sqrt(std::max(0.0f, 1 - dx * dx));
    const float a = (1 + wh.z) * 0.5f;
    const float old_y = dy;
    dy = (1 - a) * h + a * dy;
    const float old_minus_h = old_y > 0 ? -(1 - ux) / (h + old_y) : old_y - h;
    const float z = std::sqrt(std::max(0.0f, (1 - ux) + (1 - a) * old_minus_h * (old_y + dy)));
    const F3 nh = dx * t1 + dy * t2 + z * wh;
    return unit(F3{ax * nh.x, ay * nh.y, std::max(1e-6f, nh.z)}, m);
}
// shaders/conductor.h:139-207
inline BSample conductor_sample(const Conductor &p, F3 wo, float ux, float uy) {
    BSample s{{0, 0, 0}, 0, 0, p.smooth, false, true};
    if (!finite3(wo) || !std::isfinite(ux) || !std::isfinite(uy) || ux < 0 || uy < 0 || ux >= 1 ||
        uy >= 1) {
        s.valid = false;
        return s;
    }
    if (wo.z == 0)
        return s;
    if (p.smooth) {
        s.wi = F3{-wo.x, -wo.y, wo.z};
        s.pdf = 1;
        s.valid = conductor_fresnel(std::fabs(wo.z), p.eta, p.k, s.weight);
        s.accepted = s.valid && s.weight > 0;
        return s;
    }
    F3 m;
    if (!ggx_visible_normal(p.alpha_x, p.alpha_y, wo, ux, uy, m)) {
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
    s.valid = conductor_fresnel(std::fabs(dot(wo, m)), p.eta, p.k, f);
    if (!s.valid)
        return s;
    const float lo = ggx_lambda(p.alpha_x, p.alpha_y, wo), li = ggx_lambda(p.alpha_x, p.alpha_y, s.wi);
    const float d = ggx_distribution(p.alpha_x, p.alpha_y, m);
    if (d == 0)
        return s;
    s.pdf = d / (4 * std::fabs(wo.z) * (1 + lo));
    s.weight = f * (1 + lo) / (1 + lo + li);
    s.valid = std::isfinite(lo) && std::isfinite(li) && std::isfinite(s.pdf) &&
              std::isfinite(s.weight) && s.weight >= 0 && s.pdf > 0;
    s.accepted = s.valid && s.weight > 0;
    return s;
}

struct Dielectric {
    float eta, alpha_x, alpha_y;
    bool smooth;
};
// shaders/dielectric.h:15-27
inline bool dielectric_prepare(float eta, float u, float v, bool remap, Dielectric &p) {
    if (!std::isfinite(eta) || eta < 0 || !std::isfinite(u) || !std::isfinite(v) || u < 0 || v < 0)
        return false;
    p = {eta == 0 ? 1 : eta, remap ? std::sqrt(u) : u, remap ? std::sqrt(v) : v, false};
    p.smooth = p.eta == 1 || std::max(p.alpha_x, p.alpha_y) < 1e-3f;
    if (!p.smooth) {
        p.alpha_x = std::max(p.alpha_x, 1e-4f);
        p.alpha_y = std::max(p.alpha_y, 1e-4f);
    }
    return true;
}
// shaders/dielectric.h:31-70
inline bool dielectric_optics(float cosine, float eta, float &F, float &etap, float &ct, bool &tir) {
    if (!std::isfinite(cosine))
        return false;
    etap = cosine < 0 ? 1 / eta : eta;
    const float c = std::min(std::fabs(cosine), 1.0f);
    if (!(etap > 0) || !std::isfinite(etap))
        return false;
    if (etap == 1) {
        F = 0;
        ct = c;
        tir = false;
        return true;
    }
    const float c2 = c * c;
    float disc;
    const float e2 = eta * eta;
    if (cosine < 0) {
        float ax, ay;
        two_sum(1, -e2, ax, ay);
        disc = std::fma(e2, c2, ax) + (ay + std::fma(eta, eta, -e2) * (c2 - 1) + e2 * std::fma(c, c, -c2));
    } else {
        float ax, ay, bx, by;
        two_sum(e2, -1, ax, ay);
        two_sum(ax, c2, bx, by);
        disc = bx + (ay + by + std::fma(eta, eta, -e2) + std::fma(c, c, -c2));
    }
    if (!std::isfinite(disc))
        return false;
    tir = disc <= 0;
    if (tir) {
        F = 1;
        ct = 0;
        return true;
    }
    ct = std::sqrt(disc) / (cosine < 0 ? 1 : eta);
    const float rp = (etap * c - ct) / (etap * c + ct);
    const float rs = (c - etap * ct) / (c + etap * ct);
    F = .5f * (rp * rp + rs * rs);
    return std::isfinite(ct) && std::isfinite(F) && F >= 0 && F <= 1;
}
// shaders/dielectric.h:76-126
inline Eval dielectric_evaluate(const Dielectric &p, F3 wo, F3 wi) {
    if (!finite3(wo) || !finite3(wi))
        return {0, 0, false};
    if (p.smooth || wo.z == 0 || wi.z == 0)
        return {0, 0, true};
    const bool reflection = (wo.z > 0) == (wi.z > 0);
    const bool entering = wo.z > 0;
    const F3 h = reflection ? wo + wi
                            : (entering ? fma3(F3{p.eta, p.eta, p.eta}, wi, wo)
                                        : fma3(F3{p.eta, p.eta, p.eta}, wo, wi));
    F3 m;
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
    if (!dielectric_optics(co, p.eta, F, ep, ct, tir))
        return {0, 0, false};
    const float lo = ggx_lambda(p.alpha_x, p.alpha_y, wo), li = ggx_lambda(p.alpha_x, p.alpha_y, wi);
    const float d = ggx_distribution(p.alpha_x, p.alpha_y, m);
    if (!std::isfinite(lo) || !std::isfinite(li) || !std::isfinite(d))
        return {0, 0, false};
    if (d == 0)
        return {0, 0, true};
    float value, pdf;
    if (reflection) {
        value = d * F / (4 * std::fabs(wo.z) * std::fabs(wi.z) * (1 + lo + li));
        pdf = d * F / (4 * std::fabs(wo.z) * (1 + lo));
    } else {
        const float den = dot(h, m) / (entering ? p.eta : 1);
        const float jac = std::fabs(ci) / (den * den);
        pdf = d * std::fabs(co) / (std::fabs(wo.z) * (1 + lo)) * jac * (1 - F);
        const float scale = entering ? 1 / (p.eta * p.eta) : p.eta * p.eta;
        value = d * (1 - F) * std::fabs(ci * co) * scale /
                (std::fabs(wo.z) * std::fabs(wi.z) * den * den * (1 + lo + li));
    }
    return {value, pdf,
            std::isfinite(lo) && std::isfinite(li) && std::isfinite(d) && std::isfinite(value) &&
                std::isfinite(pdf) && value >= 0 && pdf >= 0};
}
// shaders/dielectric.h:129-133
inline float refraction_coefficient(float eta, float co, float ct) {
    const float c = std::fabs(co);
    return co < 0 ? ((eta - 1) * (eta + 1)) / (eta * c + ct)
                  : (((1 - eta) * (1 + eta)) / eta) / (c + eta * ct);
}
// shaders/dielectric.h:134-227
inline BSample dielectric_sample(const Dielectric &p, F3 wo, float uc, float ux, float uy,
                                 float &sampled_eta) {
    sampled_eta = 1;
    BSample s{{0, 0, 0}, 0, 0, p.smooth, false, true};
    if (!finite3(wo) || !std::isfinite(uc) || uc < 0 || uc >= 1 || !std::isfinite(ux) ||
        !std::isfinite(uy) || ux < 0 || uy < 0 || ux >= 1 || uy >= 1) {
        s.valid = false;
        return s;
    }
    if (wo.z == 0)
        return s;
    F3 m{0, 0, 1};
    if (!p.smooth && !ggx_visible_normal(p.alpha_x, p.alpha_y, wo, ux, uy, m)) {
        s.valid = false;
        return s;
    }
    const float co = dot(wo, m);
    float F, ep, ct;
    bool tir;
    if (!dielectric_optics(co, p.eta, F, ep, ct, tir)) {
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
        const float coefficient = p.eta == 1 ? 0 : refraction_coefficient(p.eta, co, ct);
        s.wi = (co < 0 ? (-p.eta) * wo : (-wo) / p.eta) + coefficient * (co < 0 ? -m : m);
    }
    if (!finite3(s.wi)) {
        s.valid = false;
        return s;
    }
    if (s.wi.z == 0 || (((s.wi.z > 0) == (wo.z > 0)) != reflection))
        return s;
    const float scale = reflection ? 1 : (co < 0 ? p.eta * p.eta : 1 / (p.eta * p.eta));
    if (p.smooth) {
        s.pdf = reflection ? F : 1 - F;
        s.weight = scale;
    } else {
        const float lo = ggx_lambda(p.alpha_x, p.alpha_y, wo),
                    li = ggx_lambda(p.alpha_x, p.alpha_y, s.wi);
        const float d = ggx_distribution(p.alpha_x, p.alpha_y, m);
        if (!std::isfinite(lo) || !std::isfinite(li) || !std::isfinite(d)) {
            s.valid = false;
            return s;
        }
        if (d == 0)
            return s;
        if (reflection)
            s.pdf = d * F / (4 * std::fabs(wo.z) * (1 + lo));
        else {
            const float den = refraction_coefficient(p.eta, co, ct);
            s.pdf = d * std::fabs(co) * ct * (1 - F) / (std::fabs(wo.z) * (1 + lo) * den * den);
        }
        s.weight = scale * (1 + lo) / (1 + lo + li);
        s.valid = std::isfinite(lo) && std::isfinite(li) && std::isfinite(d);
    }
    s.valid = s.valid && std::isfinite(s.pdf) && s.pdf > 0 && std::isfinite(s.weight) && s.weight > 0;
    s.accepted = s.valid;
    if (s.accepted && !reflection)
        sampled_eta = ep;
    return s;
}

// One wavelength of a prepared hero BSDF (rypath_scattering::Prepared, kinds 0-2;
// shaders/scattering.h:11-21).
struct LaneBsdf {
    u32 kind = 0;
    float reflectance = 0;
    Conductor conductor{};
    Dielectric dielectric{};
};
// shaders/scattering.h:25-28
inline bool delta_only(const LaneBsdf &p) {
    return (p.kind == 1 && p.conductor.smooth) || (p.kind == 2 && p.dielectric.smooth);
}
// shaders/packet_scattering.h:133-157 (scalar_evaluate), kinds 0-2
inline Eval scalar_evaluate(const LaneBsdf &p, F3 wo, F3 wi) {
    if (p.kind == 0)
        return diffuse_evaluate(p.reflectance, 0, wo, wi);
    if (p.kind == 1)
        return conductor_evaluate(p.conductor, wo, wi);
    if (p.kind == 2)
        return dielectric_evaluate(p.dielectric, wo, wi);
    return {0, 0, false};
}
// shaders/packet_scattering.h:204-214 (scalar_sample), kinds 0-2
inline BSample scalar_sample(const LaneBsdf &p, F3 wo, float uc, float ux, float uy, float &eta) {
    eta = 1;
    if (p.kind == 0)
        return diffuse_reflection_sample(p.reflectance, wo, uc, ux, uy);
    if (p.kind == 1)
        return conductor_sample(p.conductor, wo, ux, uy);
    if (p.kind == 2)
        return dielectric_sample(p.dielectric, wo, uc, ux, uy, eta);
    return {{0, 0, 0}, 0, 0, false, false, false};
}

// A hero BSDF: four lanes of one family with an active mask (HeroFrozenBSDF,
// shaders/hero_frozen_bsdf.h; evaluation :167-250).
struct HeroBsdf {
    LaneBsdf lane[4];
    u32 active_mask = 15;
};
struct HeroEval {
    F4 f, pdf;
    bool valid;
};
// shaders/hero_current_bsdf.h:62-67 (hero_current_connectible)
inline bool hero_connectible(const HeroBsdf &p) {
    for (int k = 0; k < 4; ++k)
        if ((p.active_mask & (1u << k)) && !delta_only(p.lane[k]))
            return true;
    return false;
}
// shaders/hero_frozen_bsdf.h:167-250 (hero_frozen_evaluate, radiance mode, kinds 0-2)
inline HeroEval hero_evaluate(const HeroBsdf &p, F3 wo, F3 wi) {
    HeroEval out{f4(0), f4(0), false};
    if (!(p.active_mask & 1u) || (p.active_mask & ~15u) || !finite3(wo) || !finite3(wi))
        return out;
    out.valid = true;
    for (int k = 0; k < 4; ++k) {
        if (!(p.active_mask & (1u << k)))
            continue;
        LaneBsdf lane = p.lane[k];
        if (lane.kind == 2 && lane.dielectric.eta == 1)
            lane.dielectric.smooth = true;
        const Eval e = scalar_evaluate(lane, wo, wi);
        out.f[k] = e.f;
        out.pdf[k] = e.pdf;
        out.valid = out.valid && e.valid;
    }
    for (int k = 0; k < 4; ++k)
        if (!std::isfinite(out.f[k]) || !(out.f[k] >= 0) || !std::isfinite(out.pdf[k]) ||
            !(out.pdf[k] >= 0))
            out.valid = false;
    return out;
}
// shaders/hero_scattering.h:55-66 (event_eta), kinds 0-2
inline float event_eta(const LaneBsdf &p, F3 wo, F3 wi) {
    if (!opposite_hemispheres(wo.z, wi.z))
        return 1;
    if (p.kind == 2)
        return wo.z > 0 ? p.dielectric.eta : 1 / p.dielectric.eta;
    return 1;
}
// shaders/hero_scattering.h:100-138 (dirac_lane), kinds 1-2
inline bool dirac_lane(const LaneBsdf &p, F3 wo, F3 wi, float ux, float uy, float &mass, float &pdf,
                       float &eta) {
    mass = pdf = 0;
    eta = 1;
    if (wo.z == 0 || wi.z == 0)
        return true;
    const bool transmission = opposite_hemispheres(wo.z, wi.z);
    if (p.kind == 1 && p.conductor.smooth) {
        if (transmission || !eq3(wi, F3{-wo.x, -wo.y, wo.z}))
            return true;
        pdf = 1;
        return conductor_fresnel(std::fabs(wo.z), p.conductor.eta, p.conductor.k, mass);
    }
    if (p.kind == 2 && (p.dielectric.smooth || p.dielectric.eta == 1)) {
        float F, ep, ct;
        bool tir;
        if (!dielectric_optics(wo.z, p.dielectric.eta, F, ep, ct, tir))
            return false;
        const float probability = transmission ? 1 - F : F;
        if (probability == 0)
            return true;
        float sampled_eta;
        LaneBsdf lane = p;
        if (lane.dielectric.eta == 1)
            lane.dielectric.smooth = true;
        const BSample c = scalar_sample(lane, wo, transmission ? F : 0.f, ux, uy, sampled_eta);
        if (!c.valid)
            return false;
        if (!(c.pdf > 0) || !eq3(c.wi, wi))
            return true;
        pdf = c.pdf;
        mass = c.weight * pdf;
        eta = sampled_eta;
        return std::isfinite(mass) && mass >= 0;
    }
    return true;
}
struct HeroSample {
    F3 wi;
    F4 numerator, pdf, eta;
    bool delta, transmission, accepted, valid;
};
inline bool nonnegative4(F4 v) { return finite_nonnegative4(v); }
// shaders/hero_current_bsdf.h:121-203 (hero_current_sample), kinds 0-2
inline HeroSample hero_sample(const HeroBsdf &p, F3 wo, float uc, float ux, float uy) {
    HeroSample out{};
    out.eta = f4(1);
    out.valid = false;
    const u32 kind = p.lane[0].kind;
    if (!(p.active_mask & 1u) || (p.active_mask & ~15u) || kind > 2 || !finite3(wo) ||
        !randoms(uc, ux, uy))
        return out;
    float hero_eta;
    LaneBsdf lane0 = p.lane[0];
    if (lane0.kind == 2 && lane0.dielectric.eta == 1)
        lane0.dielectric.smooth = true;
    const BSample hero = scalar_sample(lane0, wo, uc, ux, uy, hero_eta);
    out.valid = hero.valid;
    out.wi = hero.wi;
    out.delta = hero.delta;
    out.transmission = opposite_hemispheres(wo.z, hero.wi.z);
    if (!hero.valid)
        return out;
    if (!std::isfinite(hero.pdf) || hero.pdf < 0 || !finite3(hero.wi)) {
        out.valid = false;
        return out;
    }
    if (hero.pdf == 0 || wo.z == 0 || hero.wi.z == 0)
        return out;
    if (hero.delta) {
        for (int k = 0; k < 4; ++k)
            if (p.active_mask & (1u << k)) {
                float mass, density, eta;
                out.valid = dirac_lane(p.lane[k], wo, hero.wi, ux, uy, mass, density, eta) && out.valid;
                out.numerator[k] = mass;
                out.pdf[k] = density;
                out.eta[k] = eta;
            }
    } else {
        const HeroEval e = hero_evaluate(p, wo, hero.wi);
        out.numerator = e.f * std::fabs(hero.wi.z);
        out.pdf = e.pdf;
        out.valid = e.valid;
        for (int k = 0; k < 4; ++k)
            if ((p.active_mask & (1u << k)) && out.pdf[k] > 0)
                out.eta[k] = event_eta(p.lane[k], wo, hero.wi);
    }
    out.pdf[0] = hero.pdf;
    out.eta[0] = kind == 2 ? hero_eta : event_eta(p.lane[0], wo, hero.wi);
    bool eta_ok = true;
    for (int k = 0; k < 4; ++k)
        eta_ok = eta_ok && std::isfinite(out.eta[k]) && out.eta[k] > 0;
    out.valid = out.valid && nonnegative4(out.numerator) && nonnegative4(out.pdf) && eta_ok;
    bool any = false;
    for (int k = 0; k < 4; ++k)
        any = any || out.numerator[k] > 0;
    out.accepted = out.valid && any;
    return out;
}

// ---------------------------------------------------------------- spectra
struct Knot {
    float wavelength, value;
};
// shaders/render.metal:548-574
inline float pbrt_reflectance(const Knot *k, u32 count, float w) {
    if (w < k[0].wavelength || w > k[count - 1].wavelength)
        return 0.0f;
    u32 lo = 0, hi = count - 1;
    while (hi - lo > 1) {
        const u32 mid = lo + (hi - lo) / 2;
        if (w < k[mid].wavelength)
            hi = mid;
        else
            lo = mid;
    }
    if (lo == hi)
        return k[lo].value;
    const float a = k[lo].wavelength, b = k[hi].wavelength;
    const float span = b - a;
    const float t = std::isfinite(span) ? (w - a) / span : (0.5f * w - 0.5f * a) / (0.5f * b - 0.5f * a);
    // Metal mix(x, y, t) = x + (y - x) * t
    return k[lo].value + (k[hi].value - k[lo].value) * t;
}
// shaders/render.metal:590-616
inline float blackbody_reflectance(float factor, float w) {
    if (!(w >= 360.0f && w <= 830.0f))
        return 0.0f;
    if (!(factor > 0.0f && std::isfinite(factor)))
        return NAN;
    const float x = factor / w;
    if (x >= 128.0f)
        return 0.0f;
    constexpr float x_peak = 4.965114268247028f;
    constexpr float log_peak_factor = -0.007001607544495994f;
    const float f = x < 0.0625f
                        ? x * (1.0f + x * (-0.5f + x * (1.0f / 6.0f + x * (-1.0f / 24.0f + x / 120.0f))))
                        : 1.0f - std::exp(-x);
    const float log_rho = 5.0f * std::log(x / x_peak) + x_peak - x + log_peak_factor - std::log(f);
    return std::clamp(std::exp(log_rho), 0.0f, 1.0f);
}
// shaders/render.metal:627-630
inline u32 dense_index(float w) {
    const u32 nm = u32(w);
    return nm + u32(w - float(nm) >= 0.5f) - 360u;
}
// shaders/render.metal:1978-1990
inline float optical_value(const Knot *knots, u32 begin, u32 count, u32 total, bool extend, float w) {
    if (count < 2 || begin > total || count > total - begin)
        return NAN;
    const Knot *c = knots + begin;
    if (extend) {
        if (w < c[0].wavelength)
            return c[0].value;
        if (w > c[count - 1].wavelength)
            return c[count - 1].value;
    }
    return pbrt_reflectance(c, count, w);
}

// ---------------------------------------------------------------- geometry helpers (shaders/render.metal)
// :849-852
inline float gamma_bound(float n) {
    constexpr float u = 0x1.0p-24f;
    return n * u / (1.0f - n * u);
}
// src/offset_rounding_shared.h:27-41
inline u32 outward(u32 bits, bool toward_negative, bool &valid) {
    constexpr u32 sign = 0x80000000u, mag = 0x7fffffffu, minimum = 0x00800000u, maximum = 0x7f7fffffu;
    const u32 m = bits & mag, s = bits & sign;
    valid = true;
    if (m > maximum) {
        valid = false;
        return bits;
    }
    if (m == 0)
        return (toward_negative ? sign : 0u) | minimum;
    const bool away = ((s != 0) == toward_negative);
    if (away) {
        const u32 next = m < minimum ? minimum : m + 1u;
        valid = next <= maximum;
        return s | next;
    }
    return s | (m <= minimum ? 0u : m - 1u);
}
// shaders/render.metal:854-863
inline F3 round_out(F3 p, F3 n) {
    for (int i = 0; i < 3; ++i)
        if (n[i] != 0.0f) {
            bool v;
            p[i] = ffrom(outward(fbits(p[i]), std::signbit(n[i]), v));
        }
    return p;
}
// shaders/surface_detail.h:35-43
inline bool unit_vector(F3 v, F3 &out) {
    const float s = std::max(std::max(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    if (!(s > 0.0f) || !finite3(v))
        return false;
    out = normalize3(v / s);
    return finite3(out);
}
// shaders/surface_detail.h:49-55
inline void coordinate_system(F3 n, F3 &s, F3 &t) {
    const float sign = std::copysign(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    s = F3{1 + sign * n.x * n.x * a, sign * b, -sign * n.x};
    t = F3{b, sign + n.y * n.y * a, -n.y};
}
struct Frame {
    F3 x, y, z;
    F3 local(F3 v) const { return {dot(x, v), dot(y, v), dot(z, v)}; }
    F3 world(F3 v) const { return v.x * x + v.y * y + v.z * z; }
};
// shaders/render.metal:2039-2053
inline bool scattering_frame(F3 n, F3 dpdu, Frame &r) {
    if (!unit_vector(n, r.z) || !unit_vector(dpdu, r.x))
        return false;
    const float projection = dot(r.x, r.z);
    if (!std::isfinite(projection))
        return false;
    if (!unit_vector(r.x - projection * r.z, r.x))
        return false;
    if (std::fabs(dot(r.x, r.z)) > 64.0f * FLT_EPSILON)
        return false;
    r.y = cross(r.z, r.x);
    return finite3(r.y);
}

} // namespace oracle
