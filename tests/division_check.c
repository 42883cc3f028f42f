/* Host restatement of the traversal's reciprocal division (div_recip in
 * global-illumination_b200/csrc/vgi_device.cuh), checked against IEEE
 * division. Test infrastructure: compiled by tests/test_division.py with
 * -ffp-contract=off, so `*` and `/` are single round-to-nearest steps and
 * fmaf is the fused multiply-add, the operations the device code uses. */
#include <math.h>
#include <stdint.h>
#include <string.h>

static float div_recip(float a, float b, float y) {
    float q = a * y;
    float r = fmaf(-b, q, a);
    q = fmaf(r, y, q);
    r = fmaf(-b, q, a);
    return fmaf(r, y, q);
}

static uint32_t bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
static float from_bits(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static uint64_t next(uint64_t* s) {
    uint64_t x = *s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *s = x;
    return x;
}

/* A direction component: sign, exponent 2^-27 .. 2^-1 and any significand,
 * kept to 1e-8 < |b| <= 1 (1 itself included). */
static float direction_component(uint64_t* s) {
    uint64_t r = next(s);
    if ((r & 1023u) == 0u) return (r & 1024u) ? -1.0f : 1.0f;
    for (;;) {
        r = next(s);
        uint32_t e = 127u - 27u + (uint32_t)(r % 27u);
        uint32_t m = (uint32_t)(r >> 8) & 0x7fffffu;
        float b = from_bits((e << 23) | m);
        if (b > 1e-8f) return (r >> 40) & 1u ? -b : b;
    }
}

/* A position difference: sign, exponent 2^-40 .. 2^14 and any significand,
 * or zero. */
static float difference(uint64_t* s) {
    uint64_t r = next(s);
    if ((r & 63u) == 0u) return 0.0f;
    uint32_t e = 127u - 40u + (uint32_t)((r >> 6) % 55u);
    uint32_t m = (uint32_t)(r >> 20) & 0x7fffffu;
    float a = from_bits((e << 23) | m);
    return (r >> 50) & 1u ? -a : a;
}

static uint64_t compare(float a, float b, float* bad) {
    float y = 1.0f / b;
    if (bits(div_recip(a, b, y)) != bits(a / b)) {
        bad[0] = a;
        bad[1] = b;
        return 1;
    }
    return 0;
}

/* n random pairs; returns mismatches and records the last in bad[2]. */
uint64_t check_random(uint64_t n, uint64_t seed, float* bad) {
    uint64_t s = seed | 1u, miss = 0;
    for (uint64_t i = 0; i < n; ++i) {
        float b = direction_component(&s);
        miss += compare(difference(&s), b, bad);
    }
    return miss;
}

/* n pairs whose quotient lies within a few ulps of a rounding midpoint:
 * a = RN(b * (q + ulp(q)/2)) for random floats q and b. */
uint64_t check_midpoints(uint64_t n, uint64_t seed, float* bad) {
    uint64_t s = seed | 1u, miss = 0;
    for (uint64_t i = 0; i < n; ++i) {
        float b = direction_component(&s);
        float q = difference(&s);
        if (q == 0.0f) continue;
        double half = 0.5 * ((double)nextafterf(fabsf(q), INFINITY) - (double)fabsf(q));
        float a = (float)((double)b * ((double)q + (q > 0 ? half : -half)));
        if (fabsf(a) > 16384.0f || fabsf(a) < 1e-12f) continue;
        miss += compare(a, b, bad);
    }
    return miss;
}

/* Every b with |b| in [lo, 2 lo) for one dividend a. */
uint64_t check_binade(float a, float lo, float* bad) {
    uint64_t miss = 0;
    uint32_t first = bits(lo) & 0x7f800000u;
    for (uint32_t m = 0; m < (1u << 23); ++m) {
        float b = from_bits(first | m);
        miss += compare(a, b, bad);
        miss += compare(a, -b, bad);
    }
    return miss;
}
