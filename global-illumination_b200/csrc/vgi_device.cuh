// Device-side scalar semantics and hashing shared by the CUDA kernels.
//
// The kernels are compiled with --fmad=false, -prec-div=true, -prec-sqrt=true
// so every float operation is a single IEEE round-to-nearest step, in the
// order the reference's WGSL writes it (shaders/voxel_traversal.wgsl,
// shaders/voxel_path.wgsl). WGSL builtin semantics used throughout:
//   max(a, b) = a < b ? b : a,  min(a, b) = b < a ? b : a,
//   clamp(e, lo, hi) = min(max(e, lo), hi),  fract(x) = x - floor(x),
//   normalize(v) = v / length(v),  float -> int conversion saturates.
// Sine, cosine and exp are the project's own (three-part Cody-Waite
// reduction by pi/2, two-part by ln 2, Taylor polynomials with 1/n!
// coefficients), so results do not depend on any math library.
#pragma once
#include <cstdint>

namespace vgi {

__device__ __forceinline__ float wmax(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float wmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float wclamp(float e, float lo, float hi) { return wmin(wmax(e, lo), hi); }

struct V3 { float x, y, z; };
struct I3 { int x, y, z; };

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return V3{__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 add_s(V3 a, float s) { return V3{__fadd_rn(a.x, s), __fadd_rn(a.y, s), __fadd_rn(a.z, s)}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
    return V3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ float len3(V3 a) { return __fsqrt_rn(dot3(a, a)); }
__device__ __forceinline__ V3 normalize3(V3 a) { return a / len3(a); }
__device__ __forceinline__ V3 itof(I3 a) { return V3{(float)a.x, (float)a.y, (float)a.z}; }

// a / b rounded to nearest, from y = RN(1/b), for a ray's repeated divisions
// by its direction components. Two Markstein corrections of q = RN(a y)
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990): the first brings q within
// one ulp of a / b, so the remainder a - b q is exact in the fma, and the
// second then rounds correctly since y is within half an ulp of 1 / b. The
// traversal calls it with b a direction component, 1e-8 < |b| <= 1 (or
// b = y = 1, where it is exact), and a a difference of positions, so no step
// overflows or underflows and the result equals the IEEE quotient.
__device__ __forceinline__ float div_recip(float a, float b, float y) {
    float q = __fmul_rn(a, y);
    float r = __fmaf_rn(-b, q, a);
    q = __fmaf_rn(r, y, q);
    r = __fmaf_rn(-b, q, a);
    return __fmaf_rn(r, y, q);
}
// The reciprocals div_recip needs for a direction, with 1 for the axes the
// traversal treats as not moving (|d| <= 1e-8), which it divides by 1.
__device__ __forceinline__ V3 direction_recip(V3 d) {
    return V3{fabsf(d.x) > 1e-8f ? __frcp_rn(d.x) : 1.0f, fabsf(d.y) > 1e-8f ? __frcp_rn(d.y) : 1.0f,
              fabsf(d.z) > 1e-8f ? __frcp_rn(d.z) : 1.0f};
}

// WGSL i32(f32) / u32(f32): truncate, saturate, NaN -> 0.
__device__ __forceinline__ int f2i(float x) { return __float2int_rz(x); }
__device__ __forceinline__ uint32_t f2u(float x) { return __float2uint_rz(x); }

__device__ __forceinline__ uint32_t pcg(uint32_t value) {
    uint32_t state = value * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ uint32_t hash_voxel(int x, int y, int z) {
    return pcg(pcg(pcg((uint32_t)x) ^ (uint32_t)y) ^ (uint32_t)z);
}

__device__ __forceinline__ void own_sincos(float x, float* s, float* c) {
    const float two_over_pi = 0x1.45f306p-1f;
    const float p1 = 0x1.92p+0f, p2 = 0x1.fb4p-12f, p3 = 0x1.4442d2p-24f;
    float kf = floorf(__fadd_rn(__fmul_rn(x, two_over_pi), 0.5f));
    int k = f2i(kf);
    float r = __fsub_rn(__fsub_rn(__fsub_rn(x, __fmul_rn(kf, p1)), __fmul_rn(kf, p2)), __fmul_rn(kf, p3));
    float r2 = __fmul_rn(r, r);
    float ps = -0x1.ae6456p-26f;
    ps = __fadd_rn(__fmul_rn(ps, r2), 0x1.71de3ap-19f);
    ps = __fsub_rn(__fmul_rn(ps, r2), 0x1.a01a02p-13f);
    ps = __fadd_rn(__fmul_rn(ps, r2), 0x1.111112p-7f);
    ps = __fsub_rn(__fmul_rn(ps, r2), 0x1.555556p-3f);
    float sr = __fadd_rn(r, __fmul_rn(r, __fmul_rn(r2, ps)));
    float pc = 0x1.1eed8ep-29f;
    pc = __fsub_rn(__fmul_rn(pc, r2), 0x1.27e4fcp-22f);
    pc = __fadd_rn(__fmul_rn(pc, r2), 0x1.a01a02p-16f);
    pc = __fsub_rn(__fmul_rn(pc, r2), 0x1.6c16c2p-10f);
    pc = __fadd_rn(__fmul_rn(pc, r2), 0x1.555556p-5f);
    pc = __fsub_rn(__fmul_rn(pc, r2), 0.5f);
    float cr = __fadd_rn(1.0f, __fmul_rn(r2, pc));
    switch (k & 3) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

// log2 for the selection's key buckets, the same operations as the oracle's
// own_log2: x = m 2^e with m reduced to [sqrt(1/2), sqrt(2)), and
// ln m = 2 atanh(t), t = (m - 1) / (m + 1), by its series t + t^3/3 + ...
// + t^9/9 (|t| < 0.172, so the next term is below 2^-24 of the result).
// Zero and subnormal inputs give e = -127 plus the series of their raw
// significand, which the callers' clamps treat like -infinity.
__device__ __forceinline__ float own_log2(float x) {
    const uint32_t b = __float_as_uint(x);
    int e = (int)((b >> 23) & 255u) - 127;
    float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421354f) {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    const float t = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float t2 = __fmul_rn(t, t);
    float p = 0.222222224f;                     // 2/9
    p = __fadd_rn(__fmul_rn(p, t2), 0.285714298f);  // 2/7
    p = __fadd_rn(__fmul_rn(p, t2), 0.4f);          // 2/5
    p = __fadd_rn(__fmul_rn(p, t2), 0.666666687f);  // 2/3
    p = __fadd_rn(__fmul_rn(p, t2), 2.0f);
    const float ln_m = __fmul_rn(p, t);
    return __fadd_rn((float)e, __fmul_rn(ln_m, 1.44269502f));  // 1 / ln 2
}

__device__ __forceinline__ float own_exp(float x) {
    if (x != x) return x;
    if (x > 88.5f) return __int_as_float(0x7f800000);
    if (x < -103.0f) return 0.0f;
    const float log2e = 0x1.715476p+0f;
    const float l1 = 0x1.62ep-1f, l2 = 0x1.0bfbe8p-15f;
    float kf = floorf(__fadd_rn(__fmul_rn(x, log2e), 0.5f));
    int k = f2i(kf);
    float f = __fsub_rn(__fsub_rn(x, __fmul_rn(kf, l1)), __fmul_rn(kf, l2));
    float p = 0x1.a01a02p-16f;
    p = __fadd_rn(__fmul_rn(p, f), 0x1.a01a02p-13f);
    p = __fadd_rn(__fmul_rn(p, f), 0x1.6c16c2p-10f);
    p = __fadd_rn(__fmul_rn(p, f), 0x1.111112p-7f);
    p = __fadd_rn(__fmul_rn(p, f), 0x1.555556p-5f);
    p = __fadd_rn(__fmul_rn(p, f), 0x1.555556p-3f);
    p = __fadd_rn(__fmul_rn(p, f), 0.5f);
    p = __fadd_rn(__fmul_rn(p, f), 1.0f);
    p = __fadd_rn(__fmul_rn(p, f), 1.0f);
    int k1 = k / 2, k2 = k - k1;
    float s1 = __int_as_float((k1 + 127) << 23);
    float s2 = __int_as_float((k2 + 127) << 23);
    return __fmul_rn(__fmul_rn(p, s1), s2);
}

}  // namespace vgi
