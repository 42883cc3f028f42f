// Region packing into caller-owned device buffers, without any allocation.
//
// This is the allocation-free variant of the GPU region packer
// (classify_pack_kernel in vgi_naadf.cu). It is for callers that are not
// allowed to allocate device memory. One example is an engine that reserves
// all of its GPU memory up front through its own allocator. Another is a
// caller on a frame-critical thread, where cudaMalloc's implicit device
// synchronisation would stall rendering.
//
// The caller passes the region voxels in and the header and cell buffers out,
// all in its own device memory. The packer's scratch is a file-scope device
// array with room for VGI_STATIC_PACK_MAX_REGIONS regions: a word count, then
// an offset, per region, plus a total and an error word. Each GPU that loads
// the library keeps that array (about 256 KiB) until the process exits.
//
// The packing is done in three passes:
//   1. count the cell words each region needs (one CTA per region);
//   2. scan the counts into offsets in region order (one CTA);
//   3. pack each region at its offset (one CTA per region).
// So, unlike the atomic arena of vgi_upload_regions, the cell layout depends
// only on the input.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/vgi.h"
#include "vgi_naadf_device.cuh"

namespace {

using vgi::naadf::build_aadf4_warp;
using vgi::naadf::kAir;
using vgi::naadf::pack_extents;

constexpr uint32_t kMaxRegions = VGI_STATIC_PACK_MAX_REGIONS;
constexpr int kThreads = 128;
constexpr int kScanThreads = 1024;
// Word layout of the scratch array: [0, kMaxRegions) per-region word counts,
// replaced in place by their exclusive offsets; then the total word count and
// an error word (bit 0: cell capacity exceeded, bit 1: voxel value above 256).
constexpr uint32_t kTotal = kMaxRegions;
constexpr uint32_t kError = kMaxRegions + 1;
constexpr uint32_t kScratchWords = kMaxRegions + 64;

static __device__ __align__(256) uint32_t g_pack_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_address[kMaxDevices] = {};

// The device address of g_pack_scratch on the current device. The first call
// on a device resolves it with cudaGetSymbolAddress (the host-side name of
// the array is only a stand-in and must never reach a kernel).
int scratch_address(uint32_t** out) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return VGI_ERR_CUDA;
    if (device < 0 || device >= kMaxDevices) return VGI_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_pack_scratch) != cudaSuccess || !p) return VGI_ERR_CUDA;
        g_scratch_address[device] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_address[device];
    return VGI_OK;
}

// Stages a region's voxels in shared memory and classifies it: returns the
// kind (1 air, 2 uniform solid, 3 mixed); for kind 3 fills brick_info (bit 0
// uniform, bit 1 occupied, bits 16.. first material) for the 64 bricks.
// Flags voxel values above 256 in `error`.
__device__ uint32_t stage_and_classify(const uint16_t* __restrict__ voxels, uint32_t r, uint16_t* vox, uint32_t* brick_info,
                                       uint32_t* error) {
    const int tid = threadIdx.x;
    const uint4* src = reinterpret_cast<const uint4*>(voxels + (size_t)r * 4096);
    uint4* dst = reinterpret_cast<uint4*>(vox);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[tid + k * kThreads] = __ldg(src + tid + k * kThreads);
    __syncthreads();
    const uint16_t v0 = vox[0];
    bool air = true, same = true, bad = false;
    for (int i = tid; i < 4096; i += kThreads) {
        air = air && vox[i] == kAir;
        same = same && vox[i] == v0;
        bad = bad || vox[i] > kAir;
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0) atomicOr(error, 2u);
        return 0u;
    }
    const bool all_air = __syncthreads_and(air);
    const bool all_same = __syncthreads_and(same);
    if (all_air) return 1u;
    if (all_same) return 2u;
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
    return 3u;
}

// Pass 1: the cell words each region needs (64-word table + 32 per mixed brick).
__global__ void __launch_bounds__(kThreads) count_words_kernel(const uint16_t* __restrict__ voxels, uint32_t* __restrict__ scratch) {
    __shared__ __align__(16) uint16_t vox[4096];
    __shared__ uint32_t brick_info[64];
    const uint32_t r = blockIdx.x;
    const uint32_t kind = stage_and_classify(voxels, r, vox, brick_info, scratch + kError);
    if (kind != 3u) {
        if (threadIdx.x == 0) scratch[r] = 0u;
        return;
    }
    if (threadIdx.x < 32) {
        unsigned a = __ballot_sync(0xffffffffu, !(brick_info[threadIdx.x] & 1u));
        unsigned b = __ballot_sync(0xffffffffu, !(brick_info[threadIdx.x + 32] & 1u));
        if (threadIdx.x == 0) scratch[r] = 64u + 32u * (uint32_t)(__popc(a) + __popc(b));
    }
}

// Pass 2: exclusive scan of the n counts in place; the total goes to kTotal.
__global__ void __launch_bounds__(kScanThreads) scan_words_kernel(uint32_t* __restrict__ scratch, uint32_t n) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const uint32_t per = (n + kScanThreads - 1) / kScanThreads;
    const uint32_t first = threadIdx.x * per;
    const uint32_t last = min(first + per, n);
    uint32_t sum = 0;
    for (uint32_t i = first; i < last; ++i) sum += scratch[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t running = (warp ? warp_sums[warp - 1] : 0u) + incl - sum;
    for (uint32_t i = first; i < last; ++i) {
        uint32_t c = scratch[i];
        scratch[i] = running;
        running += c;
    }
    if (threadIdx.x == kScanThreads - 1) scratch[kTotal] = warp_sums[31];
}

// Pass 3: pack every region at its offset; capacity overruns set error bit 0.
__global__ void __launch_bounds__(kThreads) pack_at_offsets_kernel(const uint16_t* __restrict__ voxels, uint4* __restrict__ headers,
                                                                   uint32_t* __restrict__ cells, unsigned long long capacity,
                                                                   uint32_t* __restrict__ scratch) {
    __shared__ __align__(16) uint16_t vox[4096];
    __shared__ uint32_t brick_info[64];
    __shared__ uint32_t table[64];
    __shared__ uint32_t work[4][128];
    __shared__ uint32_t mixed_list[64];
    __shared__ uint32_t n_mixed;
    const uint32_t r = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t kind = stage_and_classify(voxels, r, vox, brick_info, scratch + kError);
    if (kind == 0u) return;
    if (kind != 3u) {
        if (tid == 0) headers[r] = make_uint4(kind, kind == 1u ? (uint32_t)kAir : (uint32_t)vox[0], 0u, 0u);
        return;
    }
    if (warp == 0) {
        uint64_t occ = 0;
        for (int b = 0; b < 64; ++b) occ |= (uint64_t)((brick_info[b] >> 1) & 1u) << b;
        build_aadf4_warp(occ, work[0], lane);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int b = lane + 32 * h;
            uint32_t info = brick_info[b];
            uint32_t first = info >> 16;
            if ((info & 1u) && first == kAir) table[b] = pack_extents(work[0][b]) << 2;
            else if (info & 1u) table[b] = (first << 2) | 1u;
            else table[b] = 2u;
        }
    } else if (warp == 1) {
        unsigned a = __ballot_sync(0xffffffffu, !(brick_info[lane] & 1u));
        unsigned b = __ballot_sync(0xffffffffu, !(brick_info[lane + 32] & 1u));
        if (!(brick_info[lane] & 1u)) mixed_list[__popc(a & ((1u << lane) - 1u))] = (uint32_t)lane;
        if (!(brick_info[lane + 32] & 1u)) mixed_list[__popc(a) + __popc(b & ((1u << lane) - 1u))] = (uint32_t)(lane + 32);
        if (lane == 0) n_mixed = (uint32_t)(__popc(a) + __popc(b));
    }
    __syncthreads();
    const unsigned long long base = scratch[r];
    const unsigned long long words = 64ull + 32ull * n_mixed;
    if (base + words > capacity) {
        if (tid == 0) atomicOr(scratch + kError, 1u);
        return;
    }
    for (uint32_t k = warp; k < n_mixed; k += kThreads / 32) {
        const uint32_t b = mixed_list[k];
        const int bx = b & 3, by = (b >> 2) & 3, bz = b >> 4;
        const int v = lane, w = lane + 32;
        const uint16_t m0 = vox[(bx * 4 + (v & 3)) + 16 * ((by * 4 + ((v >> 2) & 3)) + 16 * (bz * 4 + (v >> 4)))];
        const uint16_t m1 = vox[(bx * 4 + (w & 3)) + 16 * ((by * 4 + ((w >> 2) & 3)) + 16 * (bz * 4 + (w >> 4)))];
        uint64_t blocked = (uint64_t)__ballot_sync(0xffffffffu, m0 != kAir) | ((uint64_t)__ballot_sync(0xffffffffu, m1 != kAir) << 32);
        build_aadf4_warp(blocked, work[warp], lane);
        uint32_t c0 = m0 == kAir ? (pack_extents(work[warp][lane]) << 1) : (((uint32_t)m0 << 1) | 1u);
        uint32_t c1 = m1 == kAir ? (pack_extents(work[warp][lane + 32]) << 1) : (((uint32_t)m1 << 1) | 1u);
        uint32_t lo0 = __shfl_sync(0xffffffffu, c0, (lane & 15) * 2), hi0 = __shfl_sync(0xffffffffu, c0, (lane & 15) * 2 + 1);
        uint32_t lo1 = __shfl_sync(0xffffffffu, c1, (lane & 15) * 2), hi1 = __shfl_sync(0xffffffffu, c1, (lane & 15) * 2 + 1);
        const unsigned long long ptr = base + 64u + 32u * k;
        cells[ptr + lane] = lane < 16 ? (lo0 | (hi0 << 16)) : (lo1 | (hi1 << 16));
        if (lane == 0) table[b] = ((uint32_t)ptr << 2) | 2u;
        __syncwarp();
    }
    __syncthreads();
    if (tid < 64) cells[base + tid] = table[tid];
    if (tid == 0) headers[r] = make_uint4(3u, (uint32_t)base, 0u, 0u);
}

}  // namespace

extern "C" int vgi_pack_regions_static(const uint16_t* voxels, uint32_t n, uint32_t* headers, uint32_t* cells, uint64_t cells_capacity,
                                       uint64_t* cells_used, void* stream) {
    if (cells_used) *cells_used = 0;
    if (n == 0) return VGI_OK;
    if (!voxels || !headers || !cells || !cells_used) return VGI_ERR_INVALID;
    // Regions are read and headers written as 16-byte words.
    if (reinterpret_cast<uintptr_t>(voxels) % 16 || reinterpret_cast<uintptr_t>(headers) % 16 || reinterpret_cast<uintptr_t>(cells) % 4)
        return VGI_ERR_INVALID;
    if (n > kMaxRegions) return VGI_ERR_CAPACITY;  // more regions than the static scratch holds
    // Brick pointers are 30-bit word offsets.
    const unsigned long long capacity = cells_capacity < (1ull << 30) ? cells_capacity : (1ull << 30);
    uint32_t* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != VGI_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The array keeps the previous call's contents: clear the total and error words.
    if (cudaMemsetAsync(scratch + kTotal, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) return VGI_ERR_CUDA;
    count_words_kernel<<<n, kThreads, 0, s>>>(voxels, scratch);
    scan_words_kernel<<<1, kScanThreads, 0, s>>>(scratch, n);
    pack_at_offsets_kernel<<<n, kThreads, 0, s>>>(voxels, reinterpret_cast<uint4*>(headers), cells, capacity, scratch);
    if (cudaGetLastError() != cudaSuccess) return VGI_ERR_CUDA;
    uint32_t tail[2] = {0u, 0u};
    if (cudaMemcpyAsync(tail, scratch + kTotal, sizeof(tail), cudaMemcpyDeviceToHost, s) != cudaSuccess) return VGI_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return VGI_ERR_CUDA;
    if (tail[1] & 2u) return VGI_ERR_INVALID;
    if (tail[1] & 1u) return VGI_ERR_CAPACITY;
    *cells_used = tail[0];
    return VGI_OK;
}
