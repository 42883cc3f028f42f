// MLP radiance cache on the fifth-generation tensor cores (tcgen05).
//
// The network maps a face's encoded position, normal and albedo to the
// radiance it receives: 81 inputs (12 sine/cosine frequencies per position
// axis, the normal as one-hot, the albedo) padded to 96, four hidden layers
// of 64 with ReLU, and 3 outputs through exp (16 computed, 3 used). Weights
// are BF16 images of FP32 master weights; every product accumulates in FP32.
//
// Forward pass: a persistent kernel of 128-thread CTAs, one 128-query tile
// at a time. The packed weights (38 KB) stay in shared memory for the
// kernel's life. Per layer, the activations (A, 128 x K, BF16) and the
// layer's transposed weights (B, N x K) sit in shared memory in the
// no-swizzle K-major canonical layout: 8-row x 16-byte core matrices, the
// K-neighbouring core matrix 128 bytes on, the next 8 rows (K/8) * 128
// bytes on. One thread issues the layer's K/16 MMAs (M = 128, N = 64 or 16)
// into a TMEM accumulator and commits them to an mbarrier. Every thread then
// reads its own row (TMEM lane = row) with tcgen05.ld, applies ReLU (or exp
// after the last layer) and writes the next layer's A. Waits are bounded:
// a wait that runs out sets the error word and the CTA leaves the loop,
// frees its TMEM and returns.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "vgi_device.cuh"
#include "vgi_types.cuh"

namespace vgi {
namespace mlp {

constexpr int kIn = 96;       // 81 features, zero padded
constexpr int kHidden = 64;
constexpr int kOut = 16;      // 3 used
constexpr int kLayers = 5;
constexpr int kRows = 128;    // queries per tile (MMA M)
constexpr int kThreads = 128;

__host__ __device__ constexpr int in_dim(int l) { return l == 0 ? kIn : kHidden; }
__host__ __device__ constexpr int out_dim(int l) { return l == kLayers - 1 ? kOut : kHidden; }
// Offsets of each layer in the FP32 master weights ([in][out] row-major)
// and in the packed BF16 image (bytes), which share the element order.
__host__ __device__ constexpr int weight_offset(int l) {
    int o = 0;
    for (int i = 0; i < l; ++i) o += in_dim(i) * out_dim(i);
    return o;
}
constexpr int kWeights = weight_offset(kLayers);          // 19456
constexpr int kImageBytes = kWeights * 2;                 // 38912
constexpr int kABytes = kRows * kIn * 2;                  // 24576

// Byte offset of element (row n, column k) of an N x K K-major tile in the
// no-swizzle canonical layout.
__host__ __device__ constexpr uint32_t core_offset(uint32_t n, uint32_t k, uint32_t K) {
    return (n >> 3) * (K / 8u) * 128u + (k >> 3) * 128u + (n & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start, leading (K) and stride (8-row)
// byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t matrix_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128.
__device__ __forceinline__ uint32_t instr_desc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    return done != 0;
}
// Waits for the mbarrier phase, at most `limit` polls (the kernels take the
// limit as an argument: kMlpWaitPolls unless a caller lowers it to make a
// wait run out on purpose).
constexpr uint32_t kWaitLimit = kMlpWaitPolls;
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (bar_try(bar, phase)) return true;
    return false;
}
// A wait that ran out: the error word is set and the CTA leaves its loop, but
// only after the copy or MMAs that were to arrive on the barrier have landed
// (a second wait, at the full limit), so no async write into this CTA's
// shared memory or TMEM is still in flight when it frees its TMEM and exits.
__device__ __forceinline__ void give_up(uint32_t bar, uint32_t phase, uint32_t* abort_flag, uint32_t* error) {
    atomicOr(abort_flag, 1u);
    atomicOr(error, 1u);
    bar_wait(bar, phase, kWaitLimit);
}

// One-dimensional bulk copy global -> this CTA's shared memory on the TMA
// engine (no multicast); completion is counted on the mbarrier in bytes.
// Addresses and size are multiples of 16 bytes.
__device__ __forceinline__ void bulk_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst), "l"(src),
                 "r"(bytes), "r"(bar)
                 : "memory");
}

// Reads 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Two values rounded to BF16 (round to nearest even) in one conversion, a
// in the low half.
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&p);
}

// Writes 8 activations (columns c*8 .. c*8+7) of `row` into a K-major tile.
__device__ __forceinline__ void store8(uint8_t* tile, uint32_t row, uint32_t c, uint32_t K, const float* v) {
    uint4 w = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    *reinterpret_cast<uint4*>(tile + core_offset(row, c * 8u, K)) = w;
}

// FP32 master [in][out] -> BF16 image, each layer's transpose (rows = out)
// in the canonical K-major layout.
__global__ void pack_kernel(const float* master, uint8_t* image) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWeights) return;
    int l = 0;
    while (l + 1 < kLayers && i >= weight_offset(l + 1)) ++l;
    const int local = i - weight_offset(l);
    const int k = local / out_dim(l), n = local % out_dim(l);
    const __nv_bfloat16 b = __float2bfloat16_rn(master[i]);
    *reinterpret_cast<__nv_bfloat16*>(image + weight_offset(l) * 2 + core_offset(n, k, in_dim(l))) = b;
}

// ---- input encoding --------------------------------------------------------
// A face's 96 inputs: for each axis a of the face centre, normalised to
// [0, 1] over the loaded volume, sin and cos of pi 2^k x for k = 0..11
// (features 24a + 2k and 24a + 2k + 1); the normal as one-hot over the face
// index (72..77: +x, -x, +y, -y, +z, -z); the albedo rgb (78..80); zeros
// (81..95). sincospif gives k = 0 and k = 6; the other frequencies follow by
// the double-angle identities sin 2t = 2 sin t cos t, cos 2t = 1 - 2 sin^2 t,
// five doublings at most, so the error stays within a few dozen ulp.
__device__ __forceinline__ void encode_axis(float x, float* v) {
    for (int half = 0; half < 2; ++half) {
        float s, c;
        sincospif(half ? x * 64.0f : x, &s, &c);
        for (int k = 0; k < 6; ++k) {
            v[(half * 6 + k) * 2] = s;
            v[(half * 6 + k) * 2 + 1] = c;
            const float s2 = 2.0f * s * c, c2 = 1.0f - 2.0f * s * s;
            s = s2;
            c = c2;
        }
    }
}

// Writes the encoding of one face into row `row` of a K = 96 tile.
__device__ __forceinline__ void stage_face(uint8_t* tile, uint32_t row, const float* centre, const MlpEncoding& e, uint32_t face,
                                           float r, float g, float b) {
    for (int a = 0; a < 3; ++a) {
        float v[24];
        encode_axis((centre[a] - e.lo[a]) * e.inv[a], v);
        for (int c = 0; c < 3; ++c) store8(tile, row, (uint32_t)(a * 3 + c), kIn, v + c * 8);
    }
    float v[24];
    // The one-hot by compare, not by a dynamic index, keeps v in registers.
    for (int j = 0; j < 24; ++j) v[j] = (uint32_t)j == face ? 1.0f : 0.0f;
    v[6] = r;
    v[7] = g;
    v[8] = b;
    for (int c = 0; c < 3; ++c) store8(tile, row, 9u + (uint32_t)c, kIn, v + c * 8);
}

// The centre of a face (voxel xyz, face index in the low 3 bits of w), in voxels.
__device__ __forceinline__ void face_centre(const uint4& meta, float* centre) {
    const uint32_t face = meta.w & 7u, axis = face >> 1;
    const float side = (face & 1u) ? -0.5f : 0.5f;
    centre[0] = (float)(int)meta.x + 0.5f + (axis == 0 ? side : 0.0f);
    centre[1] = (float)(int)meta.y + 0.5f + (axis == 1 ? side : 0.0f);
    centre[2] = (float)(int)meta.z + 0.5f + (axis == 2 ? side : 0.0f);
}

// One face's 96 inputs as FP32, in the order stage_face writes them.
__device__ __forceinline__ void encode_centre(const float* centre, uint32_t face, float r, float g, float b, const MlpEncoding& enc,
                                              float* f) {
    float v[24];
    for (int a = 0; a < 3; ++a) {
        encode_axis((centre[a] - enc.lo[a]) * enc.inv[a], v);
        for (int j = 0; j < 24; ++j) f[a * 24 + j] = v[j];
    }
    for (int j = 72; j < kIn; ++j) f[j] = 0.0f;
    if (face < 6u) f[72 + face] = 1.0f;
    f[78] = r;
    f[79] = g;
    f[80] = b;
}

// The same from a slot identity word (voxel xyz, face | material << 16).
__device__ __forceinline__ void encode_meta(const uint4& meta, const float4* materials, const MlpEncoding& enc, float* f) {
    const uint32_t face = meta.w & 7u, material = (meta.w >> 16) & 255u;
    const float4 d = materials[material * 4u];
    float centre[3];
    face_centre(meta, centre);
    encode_centre(centre, face, d.x, d.y, d.z, enc, f);
}

// ---- forward pass -----------------------------------------------------------
// Rows of caller-given features: outputs[row] = (exp(net)[0..2], 0).
struct FeatureRows {
    const float* features;
    float4* outputs;
    uint32_t n;
    __device__ uint32_t count() const { return n; }
    __device__ void stage(uint8_t* tile, uint32_t tid, uint32_t row) const {
        float v[8];
        for (uint32_t c = 0; c < kIn / 8; ++c) {
            if (row < n) {
                const float4 a = reinterpret_cast<const float4*>(features + (size_t)row * kIn)[c * 2u];
                const float4 b = reinterpret_cast<const float4*>(features + (size_t)row * kIn)[c * 2u + 1u];
                v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
            } else {
                for (int j = 0; j < 8; ++j) v[j] = 0.0f;
            }
            store8(tile, tid, c, kIn, v);
        }
    }
    __device__ void emit(uint32_t row, float r, float g, float b) const {
        if (row < n) outputs[row] = make_float4(r, g, b, 0.0f);
    }
};

// The trace's queued hits: two float4 per query, (face centre xyz in
// voxels, path index bits) and (albedo rgb, face index bits); the
// prediction goes to out[path] = (rgb, 0). The count is read on the device.
struct PathQueries {
    const float4* queue;
    const uint32_t* counter;
    uint32_t capacity;
    MlpEncoding enc;
    float4* out;
    __device__ uint32_t count() const {
        const uint32_t n = *counter;
        return n < capacity ? n : capacity;
    }
    __device__ void stage(uint8_t* tile, uint32_t tid, uint32_t row) const {
        if (row < count()) {
            const float4 q0 = queue[2u * row], q1 = queue[2u * row + 1u];
            const float centre[3] = {q0.x, q0.y, q0.z};
            stage_face(tile, tid, centre, enc, __float_as_uint(q1.w), q1.x, q1.y, q1.z);
        } else {
            const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (uint32_t c = 0; c < kIn / 8; ++c) store8(tile, tid, c, kIn, z);
        }
    }
    __device__ void emit(uint32_t row, float r, float g, float b) const {
        if (row < count()) out[__float_as_uint(queue[2u * row].w)] = make_float4(r, g, b, 0.0f);
    }
};

// The forward pass of CTA `cta` of `ctas` over `rows`' 128-row tiles, with
// the network in `image` (the kernels below give each CTA its rows).
//
// A CTA holds one copy of the weight image and kGroups groups of 128
// threads. Each group runs its own tiles (worker cta * kGroups + group of
// ctas * kGroups) with its own A tile, mbarrier and 64 TMEM columns, and
// synchronises on its own named barrier, so one group's epilogue overlaps
// another's MMAs. Sharing the image lets 2 CTAs, 6 tiles, be in flight per
// SM where one group per CTA fitted 3.
constexpr int kGroups = 3;
constexpr int kForwardThreads = kThreads * kGroups;                         // 384
constexpr int kForwardTmem = 256;                                           // kGroups x 64 columns, a power of two
constexpr int kForwardSmem = kImageBytes + kGroups * kABytes + 64;          // + mbarriers, TMEM slot, flags
static_assert(kGroups * 64 <= kForwardTmem && 2 * kForwardTmem <= 512, "two CTAs' TMEM per SM");
static_assert(2 * (kForwardSmem + 1024) <= 233472, "two CTAs' shared memory per SM");

__device__ __forceinline__ void group_sync(uint32_t group) {
    asm volatile("bar.sync %0, %1;" ::"r"(1u + group), "r"((uint32_t)kThreads) : "memory");
}

template <class Rows>
__device__ __forceinline__ void forward_tiles(const Rows& rows, const uint8_t* image, uint32_t cta, uint32_t ctas, uint32_t* error,
                                              uint32_t wait_polls) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* weights = smem;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, group = tid / kThreads, gtid = tid % kThreads;
    uint8_t* tile = smem + kImageBytes + group * kABytes;
    // bars[0]: the weight copy; bars[1 + g]: group g's MMAs. flags likewise.
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kImageBytes + kGroups * kABytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 1 + kGroups);
    uint32_t* flags = tmem_slot + 1;
    const uint32_t n = rows.count();
    const uint32_t tiles = (n + kRows - 1) / kRows;
    if (cta * kGroups >= tiles) return;  // uniform per CTA: nothing allocated yet

    if (tid == 0) {
        for (int g = 0; g <= kGroups; ++g) {
            flags[g] = 0u;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + g)), "r"(1u));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        bulk_expect(smem_u32(bars), kImageBytes);
        bulk_load(smem_u32(weights), image, kImageBytes, smem_u32(bars));
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(kForwardTmem));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t group_tmem = tmem + group * 64u;
    const uint32_t lane_base = group_tmem + (((warp & 3u) * 32u) << 16);
    // The weight image (phase 0 of bars[0]).
    if (!bar_wait(smem_u32(bars), 0u, wait_polls)) give_up(smem_u32(bars), 0u, flags, error);
    __syncthreads();
    const uint32_t bar = smem_u32(bars + 1 + group);
    uint32_t* abort_flag = flags + 1 + group;
    uint32_t phase = 0;
    const uint32_t workers = ctas * kGroups;
    const uint32_t first_tile = flags[0] ? tiles : cta * kGroups + group;

    for (uint32_t t = first_tile; t < tiles; t += workers) {
        const uint32_t row = t * kRows + gtid;
        rows.stage(tile, gtid, row);
        bool ok = true;
        for (int l = 0; l < kLayers && ok; ++l) {
            const uint32_t K = in_dim(l), N = out_dim(l);
            fence_async_smem();
            fence_before();
            group_sync(group);
            if (gtid == 0) {
                fence_after();
                const uint32_t a0 = smem_u32(tile), b0 = smem_u32(weights + weight_offset(l) * 2);
                const uint32_t idesc = instr_desc(N);
                for (uint32_t kk = 0; kk < K / 16u; ++kk)
                    mma_bf16(group_tmem, matrix_desc(a0 + kk * 256u, 128u, (K / 8u) * 128u),
                             matrix_desc(b0 + kk * 256u, 128u, (K / 8u) * 128u), idesc, kk > 0 ? 1u : 0u);
                mma_commit(bar);
            }
            if (!bar_wait(bar, phase, wait_polls)) give_up(bar, phase, abort_flag, error);
            phase ^= 1u;
            group_sync(group);
            if (*abort_flag) {
                ok = false;
                break;
            }
            fence_after();
            if (l + 1 < kLayers) {
                // The row in two halves of 32 columns: each half's TMEM
                // loads in flight, then one wait (two CTAs per SM leave 85
                // registers a thread).
#pragma unroll
                for (uint32_t h = 0; h < 64u; h += 32u) {
                    if (h >= N) continue;
                    float v[32];
                    tmem_ld16(lane_base + h, v);
                    tmem_ld16(lane_base + h + 16u, v + 16);
                    tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = v[j] > 0.0f ? v[j] : 0.0f;
#pragma unroll
                    for (uint32_t c = 0; c < 4u; ++c) store8(tile, gtid, h / 8u + c, N, v + c * 8u);
                }
            } else {
                float v[16];
                tmem_ld16(lane_base, v);
                tmem_wait_ld();
                rows.emit(row, expf(v[0]), expf(v[1]), expf(v[2]));
            }
        }
        if (!ok) break;
    }
    fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kForwardTmem));
}

template <class Rows>
__global__ void __launch_bounds__(kForwardThreads, 2) forward_kernel(const Rows rows, const uint8_t* image, uint32_t* error, uint32_t wait_polls) {
    forward_tiles(rows, image, blockIdx.x, gridDim.x, error, wait_polls);
}

// The queued hits of several scenes (the chunks of a batched frame) in one
// launch. Each scene keeps its own queue, encoding, output field, network and
// error word, and owns the CTA range [first_cta, first_cta + ctas) of the
// grid; a CTA finds its scene by binary search (uniform per CTA) and runs
// that scene's tiles. Every row's prediction is the one the scene's own
// query launch gives: a row's outputs depend on its inputs and the weights
// only, whatever tile it lands in.
__global__ void __launch_bounds__(kForwardThreads, 2) forward_scenes_kernel(const MlpSceneQueries* scenes, uint32_t n_scenes, uint32_t wait_polls) {
    uint32_t lo = 0, hi = n_scenes - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (scenes[mid].first_cta <= blockIdx.x) lo = mid;
        else hi = mid - 1u;
    }
    const MlpSceneQueries sc = scenes[lo];
    if (blockIdx.x - sc.first_cta >= sc.ctas) return;  // uniform per CTA
    const PathQueries rows{sc.queue, sc.counter, sc.capacity, sc.enc, sc.out};
    forward_tiles(rows, sc.image, blockIdx.x - sc.first_cta, sc.ctas, sc.error, wait_polls);
}

__global__ void encode_faces_kernel(const uint4* meta, uint32_t n, const float4* materials, MlpEncoding enc, float* features) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) encode_meta(meta[k], materials, enc, features + (size_t)k * kIn);
}

// Training rows from a frame's results: `batch` slots drawn by hash from
// (step, row); features as encode_meta writes them (BF16-rounded by the
// training kernel), target = the slot's frame mean, NaN when the slot had no
// known sample. slot_meta[s * 3] = voxel xyz, face | material << 16;
// results[s * 6] = mean rgb; results[s * 6 + 1].y = samples (float bits).
__global__ void encode_training_kernel(const uint4* slot_meta, const uint4* results, const float4* materials, uint32_t n_slots,
                                       const uint32_t* step, uint32_t batch, MlpEncoding enc, float* features, float4* targets) {
    const uint32_t k = blockIdx.x * kThreads + threadIdx.x;
    if (k >= batch) return;
    const uint32_t salt = pcg(*step * 0x9e3779b9u + 0x7f4a7c15u);
    const uint32_t slot = pcg(k ^ salt) % n_slots;
    encode_meta(slot_meta[(size_t)slot * 3u], materials, enc, features + (size_t)k * kIn);
    const uint4 r0 = results[(size_t)slot * 6u], r1 = results[(size_t)slot * 6u + 1u];
    float4 target = make_float4(__int_as_float(0x7fc00000), 0.0f, 0.0f, 0.0f);
    if (__uint_as_float(r1.y) > 0.0f) target = make_float4(__uint_as_float(r0.x), __uint_as_float(r0.y), __uint_as_float(r0.z), 0.0f);
    targets[k] = target;
}

// Training faces from a frame's network queries (the faces its paths hit
// without a cache answer): row k takes query hash(step, k) mod count and
// becomes a FaceTask (voxel, face, sequence step * samples) plus the row's
// inputs. No queries: the task is marked invalid (face 0xffffffff).
__global__ void query_tasks_kernel(const float4* queue, const uint32_t* counter, uint32_t capacity, const uint32_t* step, uint32_t n,
                                   uint32_t samples, MlpEncoding enc, uint4* tasks, float* features) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t available = *counter < capacity ? *counter : capacity;
    float* f = features + (size_t)k * kIn;
    if (available == 0u) {
        tasks[2u * k] = make_uint4(0u, 0u, 0u, 0xffffffffu);
        tasks[2u * k + 1u] = make_uint4(0u, 0u, 0u, 0u);
        for (int j = 0; j < kIn; ++j) f[j] = 0.0f;
        return;
    }
    const uint32_t salt = pcg(*step * 0x85ebca6bu + 0x3c6ef372u);
    const uint32_t q = pcg(k ^ salt) % available;
    const float4 q0 = queue[2u * q], q1 = queue[2u * q + 1u];
    const uint32_t face = __float_as_uint(q1.w), axis = face >> 1;
    const float side = (face & 1u) ? -0.5f : 0.5f;
    const float centre[3] = {q0.x, q0.y, q0.z};
    int v[3];
    for (int a = 0; a < 3; ++a) v[a] = (int)floorf(centre[a] - 0.5f - ((uint32_t)a == axis ? side : 0.0f));
    tasks[2u * k] = make_uint4((uint32_t)v[0], (uint32_t)v[1], (uint32_t)v[2], face);
    // Each task's samples take their own stretch of the sequence (the step
    // count times the rows, plus the row): a face drawn again in a later
    // frame gets fresh directions, not the ones a shared base would repeat.
    tasks[2u * k + 1u] = make_uint4((*step * n + k) * samples, 0u, 0u, 0u);
    encode_centre(centre, face, q1.x, q1.y, q1.z, enc, f);
}

// targets[k] = the traced mean of row k's face, NaN without a known sample.
// A task left empty by query_tasks_kernel (no queries this frame) gets no
// result from the trace, so its row of `results` still holds an earlier
// frame's (or freed memory's) words: its target is NaN, skipped by training,
// whatever the row holds.
__global__ void query_targets_kernel(const uint4* results, const uint4* tasks, uint32_t n, float4* targets) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float4 target = make_float4(__int_as_float(0x7fc00000), 0.0f, 0.0f, 0.0f);
    if (tasks[2u * k].w != 0xffffffffu) {
        const uint4 r0 = results[(size_t)k * 6u], r1 = results[(size_t)k * 6u + 1u];
        if (__uint_as_float(r1.y) > 0.0f) target = make_float4(__uint_as_float(r0.x), __uint_as_float(r0.y), __uint_as_float(r0.z), 0.0f);
    }
    targets[k] = target;
}


// ---- training ------------------------------------------------------------
// One fused kernel per batch: every CTA (one per SM, 512 TMEM columns) runs
// its 128-sample tiles forward, then backward, and accumulates the weight
// gradients of all layers in TMEM across its tiles:
//     dW_l += h_l^T dz_l        (M = 128 >= in_l, K = 128 samples, N = out_l)
//     dh_l  = dz_l W_l^T        (M = 128 samples, K = out_l, N = in_l)
//     dz_{l-1} = dh_l * (h_l > 0)
// h_l (the input of layer l) is kept transposed (features x samples) for the
// dW products; dz_l is kept both as the next A operand (samples x out_l) and
// transposed (out_l x samples). The transposed tiles put the K-neighbouring
// core matrices 144 bytes apart (not 128), so the four 8-thread groups of a
// warp that write one feature row for 32 samples land in different banks.
// The hidden h_l^T tiles hold 64 feature rows; an M = 128 product also reads
// the 64 rows after them (the next buffer), which only feed accumulator rows
// 64-127, never read out (the last hidden tile's extra rows are the dz^T
// tile, the input tile's are h_1^T). The loss is the relative luminance MSE
// sum_c (p_c - y_c)^2 / (lum(p)^2 + 0.01) / B with lum(p) held constant,
// p = exp(z). Each CTA writes its gradient sums and loss to its own row of
// `partials` (19456 + 1 floats); adam_kernel / reduce_kernel sum the rows in
// CTA order, so the result does not depend on timing.
constexpr uint32_t kLboT = 144, kSboT = 16 * kLboT;   // transposed tiles: K = 128 samples
constexpr uint32_t kHT0 = (kIn / 8) * kSboT;           // 27648
constexpr uint32_t kHT = (kHidden / 8) * kSboT;        // 18432
constexpr uint32_t kWF = 0, kWB = kImageBytes, kAT = 2 * kImageBytes, kH0 = kAT + kABytes;
constexpr uint32_t kH1 = kH0 + kHT0, kDZ = kH1 + 4 * kHT, kBarT = kDZ + kHT;
constexpr int kTrainSmem = kBarT + 64;                 // 222,272 bytes
constexpr int kTrainColumns = 512;
// A CTA's row of partials: gradient sums, its loss at [kWeights], padded to
// a multiple of 4 floats so that every row's float4 stores stay aligned.
constexpr int kPartial = (kWeights + 1 + 3) / 4 * 4;
static_assert(kPartial % 4 == 0 && kWeights % 4 == 0, "float4-aligned partial rows");
__host__ __device__ constexpr uint32_t grad_column(int l) { return 64u + 64u * (uint32_t)l; }
__host__ __device__ constexpr uint32_t ht_offset(int l) { return l == 0 ? kH0 : kH1 + (uint32_t)(l - 1) * kHT; }
// Element (row, sample) of a transposed tile.
__host__ __device__ constexpr uint32_t t_offset(uint32_t row, uint32_t col) {
    return (row >> 3) * kSboT + (col >> 3) * kLboT + (row & 7u) * 16u + (col & 7u) * 2u;
}
// The M = 128 reads of the last transposed tile end at the mbarrier.
static_assert(kH1 + 3 * kHT + 16 * kSboT == kBarT, "transposed-tile overrun leaves the tiles");
static_assert(kH0 + 16 * kSboT <= kBarT, "input-tile overrun leaves the tiles");
static_assert(kTrainSmem <= 232448, "shared memory per CTA");

// Positions of master weight i (layer l, input k, output n) in the forward
// image (rows = out, K = in) and the backward image (rows = in, K = out).
__device__ __forceinline__ void image_positions(int i, uint32_t& fwd, uint32_t& bwd) {
    int l = 0;
    while (l + 1 < kLayers && i >= weight_offset(l + 1)) ++l;
    const int local = i - weight_offset(l);
    const int k = local / out_dim(l), n = local % out_dim(l);
    fwd = (uint32_t)weight_offset(l) * 2u + core_offset(n, k, in_dim(l));
    bwd = (uint32_t)weight_offset(l) * 2u + core_offset(k, n, out_dim(l));
}

// FP32 master [in][out] -> BF16 image with rows = in, K = out: the B
// operand of dh = dz W^T.
__global__ void pack_backward_kernel(const float* master, uint8_t* image) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWeights) return;
    uint32_t fwd, bwd;
    image_positions(i, fwd, bwd);
    *reinterpret_cast<__nv_bfloat16*>(image + bwd) = __float2bfloat16_rn(master[i]);
}

__device__ __forceinline__ void store_t(uint8_t* smem, uint32_t base, uint32_t row, uint32_t col, float v) {
    *reinterpret_cast<__nv_bfloat16*>(smem + base + t_offset(row, col)) = __float2bfloat16_rn(v);
}

// 256 threads: two warps per TMEM lane quadrant. Thread tid serves tile row
// (sample) tid % 128, the lanes of warp (tid / 32) % 4, and half tid / 128 of
// each 64-wide row's columns (32 each); the 16-wide output layer is the
// first half's alone. Two warps per scheduler hide each other's waits.
constexpr uint32_t kTrainThreads = 256;
static_assert(kHidden == 64 && kOut == 16 && kIn == 96, "the column split assumes 96 -> 64 ... 64 -> 16");

__global__ void __launch_bounds__(kTrainThreads) train_kernel(const float* features, const float4* targets, uint32_t batch,
                                                              const uint8_t* image_f, const uint8_t* image_b, float* partials,
                                                              uint32_t* error, uint32_t wait_polls) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kBarT);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kBarT + 8);
    uint32_t* abort_flag = reinterpret_cast<uint32_t*>(smem + kBarT + 12);
    float* loss_warps = reinterpret_cast<float*>(smem + kBarT + 16);  // 8 floats: kBarT + 16 .. + 48
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = tid & (kRows - 1u), half = tid >> 7, col0 = half * 32u;
    const uint32_t bar_addr = smem_u32(bar), s0 = smem_u32(smem);
    // Launched after the previous step's Adam as a programmatic dependent:
    // the set-up below (barrier, zeroed tiles, TMEM) overlaps that kernel,
    // and griddepcontrol.wait holds every read of its outputs (the weight
    // images) and of the batch until it has finished. The next kernel may
    // begin its own set-up as soon as every CTA here has started.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tid == 0) {
        *abort_flag = 0u;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_addr), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Zero the transposed tiles once: rows past a tile's real features are
    // read by the M = 128 products.
    for (uint32_t i = tid; i < (kBarT - kH0) / 16; i += kTrainThreads) reinterpret_cast<uint4*>(smem + kH0)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(kTrainColumns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (tid == 0) {
        bulk_expect(bar_addr, 2u * kImageBytes);
        bulk_load(s0 + kWF, image_f, kImageBytes, bar_addr);
        bulk_load(s0 + kWB, image_b, kImageBytes, bar_addr);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = tmem + (((warp & 3u) * 32u) << 16);
    const uint32_t tiles = (batch + kRows - 1) / kRows;
    bool first = true, ok = true;
    float loss_sum = 0.0f;

    // Every thread calls it; thread 0 has issued the MMAs and the commit (or
    // the copies). Returns false when the wait ran out.
    uint32_t phase = 0;
    auto finish = [&]() -> bool {
        if (!bar_wait(bar_addr, phase, wait_polls)) give_up(bar_addr, phase, abort_flag, error);
        phase ^= 1u;
        __syncthreads();
        if (*abort_flag) return false;
        fence_after();
        return true;
    };
    auto publish = [&]() {
        fence_async_smem();
        fence_before();
        __syncthreads();
    };
    ok = finish();  // the weight images

    for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const uint32_t row = t * kRows + r;
        const bool valid = row < batch;
        // Input: this half's 48 features of A (K = 96) and h_0^T, the 12
        // loads in flight first.
        {
            float4 in[kIn / 8];
            const float4* src = reinterpret_cast<const float4*>(features + (size_t)row * kIn) + half * (kIn / 8);
#pragma unroll
            for (int q = 0; q < kIn / 8; ++q) in[q] = valid ? src[q] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (uint32_t c = 0; c < kIn / 16; ++c) {
                const uint32_t group = half * (kIn / 16) + c;
                const float v[8] = {in[2 * c].x, in[2 * c].y, in[2 * c].z, in[2 * c].w,
                                    in[2 * c + 1].x, in[2 * c + 1].y, in[2 * c + 1].z, in[2 * c + 1].w};
                store8(smem + kAT, r, group, kIn, v);
#pragma unroll
                for (int j = 0; j < 8; ++j) store_t(smem, kH0, group * 8 + j, r, v[j]);
            }
        }
        // Forward.
        float z[16];
#pragma unroll
        for (int l = 0; l < kLayers; ++l) {
            const uint32_t K = in_dim(l), N = out_dim(l);
            publish();
            if (tid == 0) {
                fence_after();
                for (uint32_t kk = 0; kk < K / 16u; ++kk)
                    mma_bf16(tmem, matrix_desc(s0 + kAT + kk * 256u, 128u, (K / 8u) * 128u),
                             matrix_desc(s0 + kWF + weight_offset(l) * 2 + kk * 256u, 128u, (K / 8u) * 128u), instr_desc(N), kk > 0 ? 1u : 0u);
                mma_commit(bar_addr);
            }
            if (!(ok = finish())) break;
            if (l + 1 < kLayers) {
                // This half's 32 columns: both loads in flight, one wait.
                float v[32];
                tmem_ld16(lane_base + col0, v);
                tmem_ld16(lane_base + col0 + 16u, v + 16);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = v[j] > 0.0f ? v[j] : 0.0f;
#pragma unroll
                for (uint32_t c = 0; c < 4u; ++c) store8(smem + kAT, r, half * 4u + c, N, v + c * 8);
#pragma unroll
                for (int j = 0; j < 32; ++j) store_t(smem, ht_offset(l + 1), col0 + j, r, v[j]);
            } else if (half == 0) {
                tmem_ld16(lane_base, z);
                tmem_wait_ld();
            }
        }
        if (!ok) break;
        // Output gradient (the first half: the 16-wide layer is its own).
        float dz[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) dz[j] = 0.0f;
        const float4 y = valid && half == 0 ? targets[row] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (valid && half == 0 && y.x == y.x) {  // a NaN target marks a row without a sample
            const float p0 = expf(z[0]), p1 = expf(z[1]), p2 = expf(z[2]);
            const float lum = 0.2126f * p0 + 0.7152f * p1 + 0.0722f * p2;
            const float inv = 1.0f / ((lum * lum + 0.01f) * (float)batch);
            const float e0 = p0 - y.x, e1 = p1 - y.y, e2 = p2 - y.z;
            loss_sum += (e0 * e0 + e1 * e1 + e2 * e2) * inv;
            dz[0] = 2.0f * e0 * inv * p0;
            dz[1] = 2.0f * e1 * inv * p1;
            dz[2] = 2.0f * e2 * inv * p2;
        }
        // Backward.
#pragma unroll
        for (int l = kLayers - 1; l >= 0; --l) {
            const uint32_t N = out_dim(l), Kin = in_dim(l);
            // dz_l as the A operand (samples x N) and transposed (N x samples):
            // this half's 32 columns of a 64-wide layer, or the first half's
            // 16 of the output layer.
            if (N == 64u) {
#pragma unroll
                for (uint32_t c = 0; c < 4u; ++c) store8(smem + kAT, r, half * 4u + c, N, dz + c * 8);
#pragma unroll
                for (uint32_t o = 0; o < 32u; ++o) store_t(smem, kDZ, col0 + o, r, dz[o]);
            } else if (half == 0) {
#pragma unroll
                for (uint32_t c = 0; c < 2u; ++c) store8(smem + kAT, r, c, N, dz + c * 8);
#pragma unroll
                for (uint32_t o = 0; o < 16u; ++o) store_t(smem, kDZ, o, r, dz[o]);
            }
            publish();
            if (tid == 0) {
                fence_after();
                // dW_l += h_l^T dz_l
                for (uint32_t kk = 0; kk < kRows / 16u; ++kk)
                    mma_bf16(tmem + grad_column(l), matrix_desc(s0 + ht_offset(l) + kk * 2u * kLboT, kLboT, kSboT),
                             matrix_desc(s0 + kDZ + kk * 2u * kLboT, kLboT, kSboT), instr_desc(N), (first && kk == 0) ? 0u : 1u);
                // dh_l = dz_l W_l^T
                if (l > 0)
                    for (uint32_t kk = 0; kk < N / 16u; ++kk)
                        mma_bf16(tmem, matrix_desc(s0 + kAT + kk * 256u, 128u, (N / 8u) * 128u),
                                 matrix_desc(s0 + kWB + weight_offset(l) * 2 + kk * 256u, 128u, (N / 8u) * 128u), instr_desc(Kin),
                                 kk > 0 ? 1u : 0u);
                mma_commit(bar_addr);
            }
            if (!(ok = finish())) break;
            if (l > 0) {
                // dh (Kin = 64) into this half's dz, then the ReLU mask from
                // the kept activations.
                tmem_ld16(lane_base + col0, dz);
                tmem_ld16(lane_base + col0 + 16u, dz + 16);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const __nv_bfloat16 h = *reinterpret_cast<const __nv_bfloat16*>(smem + ht_offset(l) + t_offset(col0 + j, r));
                    dz[j] = (valid && __bfloat162float(h) > 0.0f) ? dz[j] : 0.0f;
                }
            }
        }
        if (!ok) break;
        first = false;
    }
    // This CTA's gradient sums: row r of each layer's accumulator is input
    // feature r; this half writes its 32 columns (the output layer's 16: the
    // first half).
    float* out = partials + (size_t)blockIdx.x * kPartial;
    if (ok && !first) {
        fence_before();
        __syncthreads();
        fence_after();
#pragma unroll
        for (int l = 0; l < kLayers; ++l) {
            const uint32_t N = out_dim(l);
            float v[32];
            if (N == 64u) {
                tmem_ld16(lane_base + grad_column(l) + col0, v);
                tmem_ld16(lane_base + grad_column(l) + col0 + 16u, v + 16);
                tmem_wait_ld();
                if (r < (uint32_t)in_dim(l)) {
#pragma unroll
                    for (uint32_t c = 0; c < 32u; c += 4u)
                        *reinterpret_cast<float4*>(out + weight_offset(l) + r * N + col0 + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                }
            } else if (half == 0) {
                tmem_ld16(lane_base + grad_column(l), v);
                tmem_wait_ld();
                if (r < (uint32_t)in_dim(l)) {
#pragma unroll
                    for (uint32_t c = 0; c < 16u; c += 4u)
                        *reinterpret_cast<float4*>(out + weight_offset(l) + r * N + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_sum += __shfl_xor_sync(0xffffffffu, loss_sum, o);
    if ((tid & 31u) == 0) loss_warps[warp] = loss_sum;
    fence_before();
    __syncthreads();
    // Warps 4-7 (the second half) carry no loss: their terms are zero.
    if (tid == 0)
        out[kWeights] = ((loss_warps[0] + loss_warps[1]) + (loss_warps[2] + loss_warps[3])) +
                        ((loss_warps[4] + loss_warps[5]) + (loss_warps[6] + loss_warps[7]));
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrainColumns));
}

// The CTAs' partial rows summed, for kSumWeights consecutive entries of a
// block (weights, then the loss at kWeights): kSumGroups threads share an
// entry, thread group j summing rows j, j + kSumGroups, ... in order, and the
// group sums are added in a fixed tree, so the result does not depend on
// timing. Four groups put four times as many loads in flight as one thread
// an entry: the partial rows (128 x 78 KB for a 16,384-row step) are read at
// L2 bandwidth instead of one thread's load latency.
constexpr int kSumWeights = 64, kSumGroups = 4, kSumThreads = kSumWeights * kSumGroups;
constexpr int kSumBlocks = (kWeights + 1 + kSumWeights - 1) / kSumWeights;

// Returns the sum for entry `w` in the threads of group 0 (others: 0).
__device__ __forceinline__ float sum_partials(const float* partials, uint32_t parts, int w, float (*scratch)[kSumWeights]) {
    const int t = threadIdx.x % kSumWeights, j = threadIdx.x / kSumWeights;
    float g = 0.0f;
    if (w <= kWeights) {
#pragma unroll 8
        for (uint32_t c = (uint32_t)j; c < parts; c += kSumGroups) g += partials[(size_t)c * kPartial + w];
    }
    scratch[j][t] = g;
    __syncthreads();
    return j == 0 ? (scratch[0][t] + scratch[1][t]) + (scratch[2][t] + scratch[3][t]) : 0.0f;
}
static_assert(kSumGroups == 4, "the fixed tree of sum_partials adds four group sums");

// grads[i] and the loss.
__global__ void __launch_bounds__(kSumThreads) reduce_kernel(const float* partials, uint32_t parts, float* grads, float* loss) {
    __shared__ float scratch[kSumGroups][kSumWeights];
    const int w = blockIdx.x * kSumWeights + (int)(threadIdx.x % kSumWeights);
    const float g = sum_partials(partials, parts, w, scratch);
    if (threadIdx.x >= (unsigned)kSumWeights || w > kWeights) return;
    if (w < kWeights) grads[w] = g;
    else *loss = g;
}

// One Adam step (Kingma & Ba) on the FP32 masters from the CTAs' partial
// gradient rows, then both BF16 images. The step count lives on the device
// (frames replay from a graph): every thread reads it first, and the last
// block to finish stores it advanced by one.
__global__ void __launch_bounds__(kSumThreads) adam_kernel(float* master, float* m, float* v, const float* partials, uint32_t parts, float lr,
                                                          float beta1, float beta2, float eps, uint32_t* steps, uint8_t* image_f,
                                                          uint8_t* image_b, float* loss) {
    __shared__ float scratch[kSumGroups][kSumWeights];
    // A programmatic dependent of the training kernel: nothing it wrote (the
    // partial rows) or the step before it changed is read before
    // griddepcontrol.wait, and the next step's training kernel may begin its
    // set-up once every block here has started.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int i = blockIdx.x * kSumWeights + (int)(threadIdx.x % kSumWeights);
    const uint32_t step = steps[0] + 1u;
    const float g = sum_partials(partials, parts, i, scratch);
    if (threadIdx.x < (unsigned)kSumWeights && i < kWeights) {
        const float mi = beta1 * m[i] + (1.0f - beta1) * g;
        const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / (1.0f - powf(beta1, (float)step)), vh = vi / (1.0f - powf(beta2, (float)step));
        const float w = master[i] - lr * mh / (sqrtf(vh) + eps);
        master[i] = w;
        uint32_t fwd, bwd;
        image_positions(i, fwd, bwd);
        const __nv_bfloat16 b = __float2bfloat16_rn(w);
        *reinterpret_cast<__nv_bfloat16*>(image_f + fwd) = b;
        *reinterpret_cast<__nv_bfloat16*>(image_b + bwd) = b;
    } else if (threadIdx.x < (unsigned)kSumWeights && i == kWeights) {
        *loss = g;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(steps + 1, 1u) == gridDim.x - 1) {  // steps[1]: blocks done
            steps[1] = 0u;
            steps[0] = step;
        }
    }
}

}  // namespace mlp

void launch_mlp_pack_backward(const float* master, uint8_t* image, cudaStream_t s) {
    mlp::pack_backward_kernel<<<(mlp::kWeights + 255) / 256, 256, 0, s>>>(master, image);
}

uint32_t mlp_train_parts(uint32_t batch, uint32_t ctas) {
    const uint32_t tiles = (batch + mlp::kRows - 1) / mlp::kRows;
    return tiles < ctas ? tiles : ctas;
}

uint32_t mlp_partial_floats() { return (uint32_t)mlp::kPartial; }

// A launch that may begin while the kernel before it on the stream is still
// running (programmatic dependent launch); the kernel waits for it with
// griddepcontrol.wait before reading anything it wrote.
template <typename... Params, typename... Args>
static cudaError_t launch_dependent(void (*kernel)(Params...), uint32_t grid, uint32_t block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

cudaError_t launch_mlp_train(const float* features, const float4* targets, uint32_t batch, const uint8_t* image_f, const uint8_t* image_b,
                             float* partials, uint32_t* error, uint32_t ctas, cudaStream_t s, uint32_t wait_polls) {
    if (batch == 0) return cudaSuccess;
    return launch_dependent(mlp::train_kernel, mlp_train_parts(batch, ctas), mlp::kTrainThreads, (size_t)mlp::kTrainSmem, s, features, targets,
                            batch, image_f, image_b, partials, error, wait_polls);
}

void launch_mlp_reduce(const float* partials, uint32_t parts, float* grads, float* loss, cudaStream_t s) {
    mlp::reduce_kernel<<<mlp::kSumBlocks, mlp::kSumThreads, 0, s>>>(partials, parts, grads, loss);
}

void launch_mlp_adam(float* master, float* m, float* v, const float* partials, uint32_t parts, float lr, float beta1, float beta2, float eps,
                     uint32_t* steps, uint8_t* image_f, uint8_t* image_b, float* loss, cudaStream_t s) {
    launch_dependent(mlp::adam_kernel, (uint32_t)mlp::kSumBlocks, (uint32_t)mlp::kSumThreads, 0, s, master, m, v, partials, parts, lr, beta1,
                     beta2, eps, steps, image_f, image_b, loss);
}


void launch_mlp_queries(const float4* queue, const uint32_t* count, uint32_t capacity, const uint8_t* image, const MlpEncoding& enc,
                        float4* out, uint32_t* error, uint32_t ctas, cudaStream_t s, uint32_t wait_polls) {
    if (capacity == 0) return;
    const mlp::PathQueries rows{queue, count, capacity, enc, out};
    mlp::forward_kernel<mlp::PathQueries><<<ctas, mlp::kForwardThreads, mlp::kForwardSmem, s>>>(rows, image, error, wait_polls);
}

void launch_mlp_scene_queries(const MlpSceneQueries* scenes, uint32_t n_scenes, uint32_t ctas, cudaStream_t s, uint32_t wait_polls) {
    if (n_scenes == 0 || ctas == 0) return;
    mlp::forward_scenes_kernel<<<ctas, mlp::kForwardThreads, mlp::kForwardSmem, s>>>(scenes, n_scenes, wait_polls);
}

void launch_mlp_encode_training(const uint4* slot_meta, const uint4* results, const float4* materials, uint32_t n_slots,
                                const uint32_t* step, uint32_t batch, const MlpEncoding& enc, float* features, float4* targets,
                                cudaStream_t s) {
    if (batch == 0 || n_slots == 0) return;
    mlp::encode_training_kernel<<<(batch + mlp::kThreads - 1) / mlp::kThreads, mlp::kThreads, 0, s>>>(slot_meta, results, materials, n_slots,
                                                                                                     step, batch, enc, features, targets);
}

void launch_mlp_encode_faces(const uint4* meta, uint32_t n, const float4* materials, const MlpEncoding& enc, float* features,
                             cudaStream_t s) {
    if (n) mlp::encode_faces_kernel<<<(n + 127) / 128, 128, 0, s>>>(meta, n, materials, enc, features);
}

void launch_mlp_query_tasks(const float4* queue, const uint32_t* count, uint32_t capacity, const uint32_t* step, uint32_t n,
                            uint32_t samples, const MlpEncoding& enc, uint4* tasks, float* features, cudaStream_t s) {
    if (n) mlp::query_tasks_kernel<<<(n + 127) / 128, 128, 0, s>>>(queue, count, capacity, step, n, samples, enc, tasks, features);
}

void launch_mlp_query_targets(const uint4* results, const uint4* tasks, uint32_t n, float4* targets, cudaStream_t s) {
    if (n) mlp::query_targets_kernel<<<(n + 127) / 128, 128, 0, s>>>(results, tasks, n, targets);
}

// Raises the dynamic shared-memory limit of the MLP kernels; called once per
// context before their first launch (outside any stream capture).
cudaError_t mlp_set_attributes() {
    cudaError_t e = cudaFuncSetAttribute(mlp::forward_kernel<mlp::FeatureRows>, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kForwardSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp::forward_kernel<mlp::PathQueries>, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kForwardSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp::forward_scenes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kForwardSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(mlp::train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kTrainSmem);
    return e;
}

void launch_mlp_pack(const float* master, uint8_t* image, cudaStream_t s) {
    mlp::pack_kernel<<<(mlp::kWeights + 255) / 256, 256, 0, s>>>(master, image);
}

cudaError_t launch_mlp_forward(const float* features, const uint8_t* image, float4* outputs, uint32_t n, uint32_t* error, uint32_t ctas,
                               cudaStream_t s, uint32_t wait_polls) {
    if (n == 0) return cudaSuccess;
    const uint32_t tiles = (n + mlp::kRows - 1) / mlp::kRows;
    const uint32_t need = (tiles + mlp::kGroups - 1) / mlp::kGroups;  // CTAs with a tile for their first group
    const mlp::FeatureRows rows{features, outputs, n};
    mlp::forward_kernel<mlp::FeatureRows><<<need < ctas ? need : ctas, mlp::kForwardThreads, mlp::kForwardSmem, s>>>(rows, image, error,
                                                                                                                     wait_polls);
    return cudaGetLastError();
}

uint32_t mlp_weight_count() { return mlp::kWeights; }
uint32_t mlp_image_bytes() { return mlp::kImageBytes; }

}  // namespace vgi
