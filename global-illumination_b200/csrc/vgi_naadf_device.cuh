// 4x4x4 NAADF helpers shared by the region packers (vgi_naadf.cu and
// vgi_pack_static.cu): try_grow and build_aadf (crates/bevy_voxel_gi/src/
// naadf.rs:37-148) on a brick-sized grid, and pack_extents
// (src/gpu_scene.rs:462-467).
#pragma once
#include <cstdint>

namespace vgi {
namespace naadf {

constexpr uint16_t kAir = 256;

// An AADF as six 4-bit extents (NEG_X, POS_X, NEG_Y, POS_Y, NEG_Z, POS_Z).
__device__ __forceinline__ uint32_t ext_get(uint32_t a, int d) { return (a >> (d * 4)) & 15u; }
__device__ __forceinline__ uint32_t ext_inc(uint32_t a, int d) { return a + (1u << (d * 4)); }

// try_grow on a 4x4x4 grid (naadf.rs:117-148): `cur` grows one step in
// direction d towards neighbour n if n is in the grid, unblocked, and covers
// every other extent of cur.
__device__ __forceinline__ uint32_t try_grow4(uint32_t cur, int nx, int ny, int nz, int d, uint64_t blocked, const uint32_t* src) {
    if (nx < 0 || ny < 0 || nz < 0 || nx > 3 || ny > 3 || nz > 3) return cur;
    if (ext_get(cur, d) == 255u) return cur;
    int ni = nx + 4 * (ny + 4 * nz);
    if ((blocked >> ni) & 1ull) return cur;
    uint32_t nb = src[ni];
    int opposite = d ^ 1;
#pragma unroll
    for (int b = 0; b < 6; ++b)
        if (b != opposite && ext_get(nb, b) < ext_get(cur, b)) return cur;
    return ext_inc(cur, d);
}

// build_aadf over a 4^3 grid by one warp: buf holds 2 x 64 words; returns
// with the result in buf[0..63]. Not called for an all-empty grid.
__device__ __forceinline__ void build_aadf4_warp(uint64_t blocked, uint32_t* buf, int lane) {
    uint32_t* src = buf;
    uint32_t* dst = buf + 64;
    src[lane] = 0u;
    src[lane + 32] = 0u;
    __syncwarp();
    if (blocked == ~0ull) return;
    for (int round = 0; round < 3; ++round) {
        for (int axis = 0; axis < 3; ++axis) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int i = lane + 32 * h;
                int x = i & 3, y = (i >> 2) & 3, z = i >> 4;
                uint32_t cur = 0u;
                if (!((blocked >> i) & 1ull)) {
                    cur = src[i];
                    int dx = axis == 0, dy = axis == 1, dz = axis == 2;
                    cur = try_grow4(cur, x - dx, y - dy, z - dz, axis * 2, blocked, src);
                    cur = try_grow4(cur, x + dx, y + dy, z + dz, axis * 2 + 1, blocked, src);
                }
                dst[i] = cur;
            }
            __syncwarp();
            uint32_t* t = src;
            src = dst;
            dst = t;
        }
    }
    // 9 sweeps: the result is in the buffer that started as `dst`; move it.
    uint32_t a = src[lane], b = src[lane + 32];
    __syncwarp();
    buf[lane] = a;
    buf[lane + 32] = b;
    __syncwarp();
}

__device__ __forceinline__ uint32_t pack_extents(uint32_t a) {
    uint32_t bits = 0;
#pragma unroll
    for (int d = 0; d < 6; ++d) bits |= (ext_get(a, d) & 3u) << (d * 2);
    return bits;
}

}  // namespace naadf
}  // namespace vgi
