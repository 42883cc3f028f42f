// resolve_retention (shaders/voxel_retention.wgsl:9-96), shared by the
// world cache's apply_events and the view tier's retain_view_history.
//
// `events` is the encode_events layout (src/gpu/resident.rs:1326-1414):
// `event_count` headers of three uint4, then bound records of two uint4.
// `reach` is the squared distance beyond which a bound does not apply.
#pragma once
#include "vgi_device.cuh"

namespace vgi {

struct RetentionResult {
    uint32_t limit;          // history cap, or 0xffffffff for none
    float change;            // measured change (known events only)
    bool measured, woken, urgent, urgent_if_binding;
};

// curve_limit / box_distance2 (voxel_retention.wgsl:9-22)
__device__ __forceinline__ uint32_t retention_curve_limit(uint32_t d2) {
    if (d2 >= 36864u) return 0xffffffffu;
    return (d2 * d2 + 10368u) / 20736u;
}
__device__ __forceinline__ uint32_t retention_box_distance2(int lx, int ly, int lz, int hx, int hy, int hz, int px, int py, int pz) {
    int sx = min(max(max(lx - px, px - hx), 0), 4096);
    int sy = min(max(max(ly - py, py - hy), 0), 4096);
    int sz = min(max(max(lz - pz, pz - hz), 0), 4096);
    return (uint32_t)sx * (uint32_t)sx + (uint32_t)sy * (uint32_t)sy + (uint32_t)sz * (uint32_t)sz;
}

__device__ inline RetentionResult resolve_retention(const uint4* events, uint32_t event_count, uint32_t reach, int px, int py, int pz,
                                                    bool measured_mode, uint32_t urgent_measured, uint32_t urgent_curve) {
    uint32_t cap = 0xffffffffu, source_cap = 0xffffffffu;
    float change = 0.0f;
    bool known = true, woken = false, urgent_if_binding = false, urgent = false;
    for (uint32_t e = 0; e < event_count; ++e) {
        uint4 h0 = events[e * 3u], h1 = events[e * 3u + 1u], h2 = events[e * 3u + 2u];
        if ((h0.w & 2u) != 0u) {
            uint32_t limit = h2.x;
            for (uint32_t b = 0; b < h2.w; ++b) {
                uint4 sp = events[event_count * 3u + (h2.z + b) * 2u];
                float dx = __fsub_rn((float)px, __uint_as_float(sp.x)), dy = __fsub_rn((float)py, __uint_as_float(sp.y)),
                      dz = __fsub_rn((float)pz, __uint_as_float(sp.z));
                float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                if (d2 <= __uint_as_float(sp.w)) limit = limit < 4u ? limit : 4u;
            }
            source_cap = source_cap < limit ? source_cap : limit;
            woken = true;
            continue;
        }
        uint32_t outside = retention_box_distance2((int)h0.x, (int)h0.y, (int)h0.z, (int)h1.x, (int)h1.y, (int)h1.z, px, py, pz);
        if (outside > reach) continue;
        woken = true;
        bool exact = known;
        uint32_t nearest = 0xffffffffu;
        for (uint32_t b = 0; b < h2.w; ++b) {
            uint32_t record = event_count * 3u + (h2.z + b) * 2u;
            uint4 b0 = events[record], b1 = events[record + 1u];
            uint32_t d = retention_box_distance2((int)b0.x, (int)b0.y, (int)b0.z, (int)b1.x, (int)b1.y, (int)b1.z, px, py, pz);
            if (d > reach) continue;
            nearest = nearest < d ? nearest : d;
            uint32_t edit_kind = b1.w & 7u;
            if ((b1.w & 8u) != 0u && (edit_kind == 0u || edit_kind == 3u)) {
                if (edit_kind == 3u && measured_mode) urgent_if_binding = urgent_if_binding || d <= urgent_measured;
                else urgent = urgent || d <= urgent_curve;
            }
            if (exact) {
                uint32_t kind = b1.w & 7u;
                if (kind == 0u) {
                    known = false;
                    exact = false;
                } else if (kind != 1u) {
                    float area = 1.0f;
                    if (kind == 2u) area = (float)min(max(((int)b1.w >> 3) + 1 - py, 0), 16);
                    change = __fadd_rn(change, __fdiv_rn(__fmul_rn(__uint_as_float(b0.w), area), __fmul_rn(3.14159265358979f, (float)(d > 1u ? d : 1u))));
                }
            }
        }
        if (nearest != 0xffffffffu) {
            uint32_t c = retention_curve_limit(nearest);
            cap = cap < c ? cap : c;
        }
    }
    RetentionResult r;
    r.measured = measured_mode && known;
    uint32_t other = r.measured ? 0xffffffffu : cap;
    r.limit = source_cap < other ? source_cap : other;
    r.change = change;
    r.woken = woken;
    r.urgent = urgent;
    r.urgent_if_binding = urgent_if_binding;
    return r;
}

}  // namespace vgi
