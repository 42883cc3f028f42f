// NAADF upload path on the GPU: region classification, brick-level and
// voxel-level AADF construction and cell packing, one CTA per 16^3 region.
//
// Behaviour follows (paths within nathanaelneveux/global-illumination,
// crates/bevy_voxel_gi/src/):
//   world.rs:243-319      NaadfRegion::build (Empty / Uniform / mixed)
//   world.rs:352-384      brick_voxel_bounds / brick_bounds
//   naadf.rs:37-148       build_aadf / try_grow (Jacobi sweeps, max(size)-1 rounds)
//   gpu_scene.rs:174-239  header kinds, 64-word brick tables, 32-word bricks
//   gpu_scene.rs:458-467  pack_bytes / pack_extents
//
// B200 layout: a CTA stages its region's 8 KB of voxels in shared memory with
// 16-byte loads, classifies it with block votes, builds the 4^3 brick field and
// then each warp builds the 4^3 voxel field of one mixed brick at a time
// (two cells per lane, __syncwarp between sweeps). Cell space is reserved
// with one atomic per mixed region, so the whole pack is a single streaming
// pass over the voxels. Identical brick payloads are not interned here:
// every mixed brick owns its 32 words (the reference deduplicates them on the
// CPU; traversal reads the same values either way).
#include <cuda_runtime.h>
#include <cstdint>

#include "vgi_naadf_device.cuh"

namespace vgi {
namespace {

using naadf::build_aadf4_warp;
using naadf::kAir;
using naadf::pack_extents;

constexpr int kThreads = 128;

// One CTA per region. headers[r] receives (kind, material or cell offset);
// z and w (top-level extents, stride) are written by the host runtime.
__global__ void __launch_bounds__(kThreads) classify_pack_kernel(const uint16_t* __restrict__ voxels, const uint32_t* __restrict__ regions,
                                                                 uint32_t n, uint4* __restrict__ headers, uint32_t* __restrict__ cells,
                                                                 unsigned long long* __restrict__ alloc, unsigned long long capacity,
                                                                 uint32_t* __restrict__ error) {
    __shared__ __align__(16) uint16_t vox[4096];
    __shared__ uint32_t brick_info[64];   // bit 0 uniform, bit 1 occupied, bits 16.. first material
    __shared__ uint32_t table[64];
    __shared__ uint32_t scratch[4][128];
    __shared__ uint32_t mixed_list[64];
    __shared__ uint32_t n_mixed;
    __shared__ unsigned long long base;
    const uint32_t r = regions ? regions[blockIdx.x] : blockIdx.x;
    if (r >= n) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(voxels + (size_t)r * 4096);
        uint4* dst = reinterpret_cast<uint4*>(vox);
#pragma unroll
        for (int k = 0; k < 4; ++k) dst[tid + k * kThreads] = __ldg(src + tid + k * kThreads);
    }
    if (tid == 0) n_mixed = 0;
    __syncthreads();
    const uint16_t v0 = vox[0];
    bool air = true, same = true;
    for (int i = tid; i < 4096; i += kThreads) {
        air = air && vox[i] == kAir;
        same = same && vox[i] == v0;
    }
    const bool all_air = __syncthreads_and(air);
    const bool all_same = __syncthreads_and(same);
    if (all_air || all_same) {
        if (tid == 0) headers[r] = make_uint4(all_air ? 1u : 2u, (uint32_t)(all_air ? kAir : v0), 0u, 0u);
        return;
    }
    // Per-brick uniformity and occupancy.
    if (tid < 64) {
        int bx = tid & 3, by = (tid >> 2) & 3, bz = tid >> 4;
        uint16_t first = vox[(bx * 4) + 16 * ((by * 4) + 16 * (bz * 4))];
        bool uniform = true, occupied = false;
        for (int v = 0; v < 64; ++v) {
            uint16_t m = vox[(bx * 4 + (v & 3)) + 16 * ((by * 4 + ((v >> 2) & 3)) + 16 * (bz * 4 + (v >> 4)))];
            uniform = uniform && m == first;
            occupied = occupied || m != kAir;
        }
        brick_info[tid] = (uniform ? 1u : 0u) | (occupied ? 2u : 0u) | ((uint32_t)first << 16);
    }
    __syncthreads();
    // Brick-level field (brick_bounds) by warp 0; the mixed-brick list by warp 1.
    if (warp == 0) {
        uint64_t occ = 0;
        for (int b = 0; b < 64; ++b) occ |= (uint64_t)((brick_info[b] >> 1) & 1u) << b;
        build_aadf4_warp(occ, scratch[0], lane);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int b = lane + 32 * h;
            uint32_t info = brick_info[b];
            uint32_t first = info >> 16;
            if ((info & 1u) && first == kAir) table[b] = pack_extents(scratch[0][b]) << 2;
            else if (info & 1u) table[b] = (first << 2) | 1u;
            else table[b] = 2u;
        }
    } else if (warp == 1) {
        // Mixed bricks in table order (ballot + popc keeps the order stable).
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int b = lane + 32 * h;
            bool mixed = !(brick_info[b] & 1u);
            unsigned ballot = __ballot_sync(0xffffffffu, mixed);
            uint32_t before = h == 0 ? 0u : (uint32_t)__popc(__ballot_sync(0xffffffffu, !(brick_info[lane] & 1u)));
            if (mixed) mixed_list[before + __popc(ballot & ((1u << lane) - 1u))] = (uint32_t)b;
            if (h == 1 && lane == 0) n_mixed = before + __popc(ballot);
        }
    }
    __syncthreads();
    const uint32_t words = 64u + 32u * n_mixed;
    if (tid == 0) {
        unsigned long long at = atomicAdd(alloc, (unsigned long long)words);
        if (at + words > capacity) {
            atomicOr(error, 1u);
            base = ~0ull;
        } else {
            base = at;
        }
    }
    __syncthreads();
    if (base == ~0ull) return;
    // Voxel-level fields and payloads: one mixed brick per warp at a time.
    for (uint32_t k = warp; k < n_mixed; k += kThreads / 32) {
        const uint32_t b = mixed_list[k];
        const int bx = b & 3, by = (b >> 2) & 3, bz = b >> 4;
        uint16_t m0, m1;
        {
            int v = lane, w = lane + 32;
            m0 = vox[(bx * 4 + (v & 3)) + 16 * ((by * 4 + ((v >> 2) & 3)) + 16 * (bz * 4 + (v >> 4)))];
            m1 = vox[(bx * 4 + (w & 3)) + 16 * ((by * 4 + ((w >> 2) & 3)) + 16 * (bz * 4 + (w >> 4)))];
        }
        uint64_t blocked = (uint64_t)__ballot_sync(0xffffffffu, m0 != kAir) | ((uint64_t)__ballot_sync(0xffffffffu, m1 != kAir) << 32);
        build_aadf4_warp(blocked, scratch[warp], lane);
        uint32_t c0 = m0 == kAir ? (pack_extents(scratch[warp][lane]) << 1) : (((uint32_t)m0 << 1) | 1u);
        uint32_t c1 = m1 == kAir ? (pack_extents(scratch[warp][lane + 32]) << 1) : (((uint32_t)m1 << 1) | 1u);
        // Cells 2j and 2j+1 share word j: lane l owns cells l and l+32, so
        // word j (j < 16) takes cells 2j, 2j+1 from lanes 2j, 2j+1 (first half)
        // and word 16 + j from their second halves.
        uint32_t lo0 = __shfl_sync(0xffffffffu, c0, (lane & 15) * 2), hi0 = __shfl_sync(0xffffffffu, c0, (lane & 15) * 2 + 1);
        uint32_t lo1 = __shfl_sync(0xffffffffu, c1, (lane & 15) * 2), hi1 = __shfl_sync(0xffffffffu, c1, (lane & 15) * 2 + 1);
        uint32_t word = lane < 16 ? (lo0 | (hi0 << 16)) : (lo1 | (hi1 << 16));
        const unsigned long long ptr = base + 64u + 32u * k;
        cells[ptr + (lane < 16 ? lane : lane)] = word;
        if (lane == 0) table[b] = ((uint32_t)ptr << 2) | 2u;
        __syncwarp();
    }
    __syncthreads();
    if (tid < 64) cells[base + tid] = table[tid];
    if (tid == 0) headers[r] = make_uint4(3u, (uint32_t)base, 0u, 0u);
}

// Brick payload deduplication (the reference's intern_brick,
// gpu_scene.rs:311-335): one thread per brick word of every mixed region.
// Each mixed brick's 32-word payload is hashed into an open-addressing table
// of payload pointers; equal payloads (compared word for word, never by hash
// alone) share the first pointer to claim a slot, and the brick word is
// repointed to it. Traversal reads the same values; the payloads it touches
// shrink to one copy each.
__device__ __forceinline__ uint32_t payload_hash(const uint32_t* p) {
    uint32_t h = 0x9e3779b9u;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
        h ^= p[k] + 0x7f4a7c15u + (h << 6) + (h >> 2);
        h *= 0x85ebca6bu;
    }
    return h ^ (h >> 16);
}

__global__ void dedup_bricks_kernel(const uint4* __restrict__ headers, uint32_t n, uint32_t* __restrict__ cells,
                                    uint32_t* __restrict__ table, uint32_t mask, uint32_t* __restrict__ error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = i >> 6, b = i & 63u;
    if (r >= n) return;
    const uint4 h = headers[r];
    if (h.x != 3u) return;
    const uint32_t word = cells[h.y + b];
    if ((word & 3u) != 2u) return;
    const uint32_t mine = word >> 2;
    const uint32_t* payload = cells + mine;
    uint32_t slot = payload_hash(payload) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        const uint32_t held = atomicCAS(table + slot, 0xffffffffu, mine);
        if (held == 0xffffffffu) return;  // first copy: stays canonical
        bool same = true;
        const uint32_t* other = cells + held;
        for (int k = 0; k < 32 && same; ++k) same = other[k] == payload[k];
        if (same) {
            cells[h.y + b] = (held << 2) | 2u;
            return;
        }
        slot = (slot + 1u) & mask;
    }
    atomicOr(error, 4u);  // table full: the brick keeps its own payload
}

// Voxel edits: 2 words per edit (region index, local index << 16 | value).
__global__ void scatter_edits_kernel(const uint2* __restrict__ edits, uint32_t n, uint16_t* __restrict__ voxels) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint2 e = edits[i];
    voxels[(size_t)e.x * 4096 + (e.y >> 16)] = (uint16_t)(e.y & 0xffffu);
}

// Top-level extents and stride into header words z, w: 2 words per region.
__global__ void set_header_extents_kernel(uint4* __restrict__ headers, const uint2* __restrict__ zw, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint2 v = zw[i];
    headers[i].z = v.x;
    headers[i].w = v.y;
}

// The region header per cell of the dense region grid (kind 0 where the
// grid holds -1, a region the directory does not find), so a ray entering a
// region reads its header with one load instead of an index, then a header.
__global__ void grid_headers_kernel(const int32_t* __restrict__ grid, uint32_t n, const uint4* __restrict__ headers,
                                    uint4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t h = grid[i];
    out[i] = h < 0 ? make_uint4(0u, 0u, 0u, 0u) : headers[h];
}

// Loaded regions into their header slots: region i of the staged upload
// (4096 voxels, 512 x 16 bytes) to slot slots[i] of the voxel store.
__global__ void scatter_regions_kernel(const uint4* __restrict__ staged, const uint32_t* __restrict__ slots, uint32_t n,
                                       uint4* __restrict__ voxels) {
    const uint32_t i = blockIdx.x;
    if (i >= n) return;
    const uint4* src = staged + (size_t)i * 512;
    uint4* dst = voxels + (size_t)slots[i] * 512;
    for (uint32_t k = threadIdx.x; k < 512; k += blockDim.x) dst[k] = src[k];
}

// Unloaded regions' header slots become kind 0 (no region): the packer's
// deduplication and the header grid skip them until a load reuses the slot.
__global__ void clear_headers_kernel(uint4* __restrict__ headers, const uint32_t* __restrict__ slots, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) headers[slots[i]] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace

void launch_scatter_regions(const uint16_t* staged, const uint32_t* slots, uint32_t n, uint16_t* voxels, cudaStream_t s) {
    if (n == 0) return;
    scatter_regions_kernel<<<n, 128, 0, s>>>(reinterpret_cast<const uint4*>(staged), slots, n, reinterpret_cast<uint4*>(voxels));
}

void launch_clear_headers(uint4* headers, const uint32_t* slots, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    clear_headers_kernel<<<(n + 255) / 256, 256, 0, s>>>(headers, slots, n);
}

void launch_grid_headers(const int32_t* grid, uint32_t n, const uint4* headers, uint4* out, cudaStream_t s) {
    if (n == 0) return;
    grid_headers_kernel<<<(n + 255) / 256, 256, 0, s>>>(grid, n, headers, out);
}

void launch_classify_pack(const uint16_t* voxels, const uint32_t* regions, uint32_t grid, uint32_t n, uint4* headers, uint32_t* cells,
                          unsigned long long* alloc, unsigned long long capacity, uint32_t* error, cudaStream_t s) {
    if (grid == 0) return;
    classify_pack_kernel<<<grid, kThreads, 0, s>>>(voxels, regions, n, headers, cells, alloc, capacity, error);
}

void launch_dedup_bricks(const uint4* headers, uint32_t n, uint32_t* cells, uint32_t* table, uint32_t mask, uint32_t* error,
                         cudaStream_t s) {
    if (n == 0) return;
    const uint64_t threads = (uint64_t)n * 64;
    dedup_bricks_kernel<<<(uint32_t)((threads + 255) / 256), 256, 0, s>>>(headers, n, cells, table, mask, error);
}

void launch_scatter_edits(const uint2* edits, uint32_t n, uint16_t* voxels, cudaStream_t s) {
    if (n == 0) return;
    scatter_edits_kernel<<<(n + 255) / 256, 256, 0, s>>>(edits, n, voxels);
}

void launch_set_header_extents(uint4* headers, const uint2* zw, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    set_header_extents_kernel<<<(n + 255) / 256, 256, 0, s>>>(headers, zw, n);
}

}  // namespace vgi
