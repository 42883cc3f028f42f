// TEST INFRASTRUCTURE ONLY (the oracle). Nothing in the product links this.
//
// Scalar float helpers with the WGSL semantics the reference's shaders are
// written against, restated with explicit IEEE single-precision operations
// (no contraction, IEEE division and square root; this file must be compiled
// with -ffp-contract=off and without -ffast-math).
//
// WGSL builtins follow the WGSL specification:
//   max(e1, e2) = e2 if e1 < e2 else e1;  min(e1, e2) = e2 if e2 < e1 else e1;
//   clamp(e, lo, hi) = min(max(e, lo), hi);  fract(x) = x - floor(x);
//   select(f, t, c) = c ? t : f;  normalize(v) = v / length(v);
//   float -> int conversion saturates (NaN -> 0).
// sin/cos/exp are NOT the platform's: the path uses the project's own
// Cody-Waite reduction plus Taylor polynomials (coefficients 1/n!), written
// identically in the CUDA kernels so both sides round the same way.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

struct f3 { float x, y, z; };
struct i3 { int32_t x, y, z; };

static inline float wmax(float a, float b) { return a < b ? b : a; }
static inline float wmin(float a, float b) { return b < a ? b : a; }
static inline float wclamp(float e, float lo, float hi) { return wmin(wmax(e, lo), hi); }
static inline int32_t imax(int32_t a, int32_t b) { return a < b ? b : a; }
static inline int32_t imin(int32_t a, int32_t b) { return b < a ? b : a; }
static inline uint32_t umin(uint32_t a, uint32_t b) { return b < a ? b : a; }
static inline uint32_t umax(uint32_t a, uint32_t b) { return a < b ? b : a; }

static inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
static inline f3 add(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline f3 sub(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline f3 mul(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline f3 muls(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
static inline f3 divs(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
static inline f3 adds(f3 a, float s) { return f3{a.x + s, a.y + s, a.z + s}; }
static inline f3 neg(f3 a) { return f3{-a.x, -a.y, -a.z}; }
static inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 cross(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float length(f3 a) { return std::sqrt(dot(a, a)); }
static inline f3 normalize(f3 a) { return divs(a, length(a)); }
static inline float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline void setc(f3& a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }
static inline int32_t compi(i3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline f3 tof(i3 a) { return f3{(float)a.x, (float)a.y, (float)a.z}; }

static inline float fract(float x) { return x - std::floor(x); }

// WGSL i32(f32): round toward zero, saturating; NaN -> 0.
static inline int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (-2147483647 - 1);
    return (int32_t)x;
}
// WGSL u32(f32): round toward zero, saturating; NaN -> 0.
static inline uint32_t f2u(float x) {
    if (x != x) return 0u;
    if (x >= 4294967296.0f) return 4294967295u;
    if (x <= 0.0f) return 0u;
    return (uint32_t)x;
}
static inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

static inline uint32_t reverse_bits(uint32_t v) {
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0f0f0f0fu) | ((v & 0x0f0f0f0fu) << 4);
    v = ((v >> 8) & 0x00ff00ffu) | ((v & 0x00ff00ffu) << 8);
    return (v >> 16) | (v << 16);
}

// Own sine/cosine: k = nearest multiple of pi/2 (x * 2/pi rounded), three-part
// Cody-Waite reduction (each part has 12 trailing zero bits so k * part is
// exact), then Taylor polynomials on |r| <= pi/4 (sin to r^11, cos to r^12).
// log2 by exponent split and the atanh series (the device's own_log2, same
// operations): m in [sqrt(1/2), sqrt(2)), ln m = 2 (t + t^3/3 + ... + t^9/9).
static inline float own_log2(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    int e = (int)((b >> 23) & 255u) - 127;
    uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
    float m;
    std::memcpy(&m, &mb, 4);
    if (m > 1.41421354f) {
        m = m * 0.5f;
        e += 1;
    }
    const float t = (m - 1.0f) / (m + 1.0f);
    const float t2 = t * t;
    float p = 0.222222224f;
    p = p * t2 + 0.285714298f;
    p = p * t2 + 0.4f;
    p = p * t2 + 0.666666687f;
    p = p * t2 + 2.0f;
    const float ln_m = p * t;
    return (float)e + ln_m * 1.44269502f;
}

static inline void own_sincos(float x, float* s, float* c) {
    const float two_over_pi = 0x1.45f306p-1f;
    const float p1 = 0x1.92p+0f, p2 = 0x1.fb4p-12f, p3 = 0x1.4442d2p-24f;
    float kf = std::floor(x * two_over_pi + 0.5f);
    int32_t k = f2i(kf);
    float r = ((x - kf * p1) - kf * p2) - kf * p3;
    float r2 = r * r;
    float ps = -0x1.ae6456p-26f;            // -1/11!
    ps = ps * r2 + 0x1.71de3ap-19f;
    ps = ps * r2 - 0x1.a01a02p-13f;
    ps = ps * r2 + 0x1.111112p-7f;
    ps = ps * r2 - 0x1.555556p-3f;
    float sr = r + r * (r2 * ps);
    float pc = 0x1.1eed8ep-29f;             // 1/12!
    pc = pc * r2 - 0x1.27e4fcp-22f;
    pc = pc * r2 + 0x1.a01a02p-16f;
    pc = pc * r2 - 0x1.6c16c2p-10f;
    pc = pc * r2 + 0x1.555556p-5f;
    pc = pc * r2 - 0.5f;
    float cr = 1.0f + r2 * pc;
    switch (k & 3) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

// Own exp: k = round(x / ln2), two-part Cody-Waite reduction, Taylor to f^8
// on |f| <= ln2/2, then scaling by 2^k through the exponent bits.
static inline float own_exp(float x) {
    if (x != x) return x;
    if (x > 88.5f) return INFINITY;
    if (x < -103.0f) return 0.0f;
    const float log2e = 0x1.715476p+0f;
    const float l1 = 0x1.62ep-1f, l2 = 0x1.0bfbe8p-15f;
    float kf = std::floor(x * log2e + 0.5f);
    int32_t k = f2i(kf);
    float f = (x - kf * l1) - kf * l2;
    float p = 0x1.a01a02p-16f;               // 1/8!
    p = p * f + 0x1.a01a02p-13f;
    p = p * f + 0x1.6c16c2p-10f;
    p = p * f + 0x1.111112p-7f;
    p = p * f + 0x1.555556p-5f;
    p = p * f + 0x1.555556p-3f;
    p = p * f + 0.5f;
    p = p * f + 1.0f;
    p = p * f + 1.0f;
    // 2^k in two steps so k down to -149 and up to 128 stay representable.
    int32_t k1 = k / 2, k2 = k - k1;
    float s1 = bitsf((uint32_t)(k1 + 127) << 23);
    float s2 = bitsf((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

}  // namespace orc
