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

#include "vgi_types.cuh"

namespace vgi {
namespace mlp {

constexpr int kIn = 96;       // 81 features, zero padded
constexpr int kHidden = 64;
constexpr int kOut = 16;      // 3 used
constexpr int kLayers = 5;
constexpr int kRows = 128;    // queries per tile (MMA M)
constexpr int kThreads = 128;
constexpr int kTmemColumns = 64;

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
constexpr int kSmemBytes = kImageBytes + kABytes + 64;    // + mbarrier, TMEM slot, flags

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
// Waits for the mbarrier phase, at most `kWaitLimit` polls.
constexpr uint32_t kWaitLimit = 1u << 22;
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (bar_try(bar, phase)) return true;
    return false;
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

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat16 x = __float2bfloat16_rn(a), y = __float2bfloat16_rn(b);
    return (uint32_t)__bfloat16_as_ushort(x) | ((uint32_t)__bfloat16_as_ushort(y) << 16);
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

// outputs[row][0..3] = exp(network(features[row][0..95]))[0..2], 0
__global__ void __launch_bounds__(kThreads) forward_kernel(const float* features, const uint8_t* image, float4* outputs, uint32_t n,
                                                           uint32_t* error) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* weights = smem;
    uint8_t* tile = smem + kImageBytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kImageBytes + kABytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kImageBytes + kABytes + 8);
    uint32_t* abort_flag = reinterpret_cast<uint32_t*>(smem + kImageBytes + kABytes + 12);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;

    for (uint32_t i = tid; i < kImageBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(weights)[i] = reinterpret_cast<const uint4*>(image)[i];
    if (tid == 0) {
        *abort_flag = 0u;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(kTmemColumns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = tmem + ((warp * 32u) << 16);
    const uint32_t bar_addr = smem_u32(bar);
    uint32_t phase = 0;
    const uint32_t tiles = (n + kRows - 1) / kRows;

    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t row = t * kRows + tid;
        // Layer 0 input: the row's 96 features (zeros past the end).
        {
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
        bool ok = true;
        for (int l = 0; l < kLayers && ok; ++l) {
            const uint32_t K = in_dim(l), N = out_dim(l);
            fence_async_smem();
            fence_before();
            __syncthreads();
            if (tid == 0) {
                fence_after();
                const uint32_t a0 = smem_u32(tile), b0 = smem_u32(weights + weight_offset(l) * 2);
                const uint32_t idesc = instr_desc(N);
                for (uint32_t kk = 0; kk < K / 16u; ++kk)
                    mma_bf16(tmem, matrix_desc(a0 + kk * 256u, 128u, (K / 8u) * 128u), matrix_desc(b0 + kk * 256u, 128u, (K / 8u) * 128u),
                             idesc, kk > 0 ? 1u : 0u);
                mma_commit(bar_addr);
            }
            if (!bar_wait(bar_addr, phase)) {
                atomicOr(abort_flag, 1u);
                atomicOr(error, 1u);
            }
            phase ^= 1u;
            __syncthreads();
            if (*abort_flag) {
                ok = false;
                break;
            }
            fence_after();
            if (l + 1 < kLayers) {
                for (uint32_t c0 = 0; c0 < N; c0 += 16u) {
                    float v[16];
                    tmem_ld16(lane_base + c0, v);
                    tmem_wait_ld();
                    for (int j = 0; j < 16; ++j) v[j] = v[j] > 0.0f ? v[j] : 0.0f;
                    store8(tile, tid, c0 / 8u, N, v);
                    store8(tile, tid, c0 / 8u + 1u, N, v + 8);
                }
            } else {
                float v[16];
                tmem_ld16(lane_base, v);
                tmem_wait_ld();
                if (row < n) outputs[row] = make_float4(expf(v[0]), expf(v[1]), expf(v[2]), 0.0f);
            }
        }
        if (!ok) break;
    }
    fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns));
}

}  // namespace mlp

void launch_mlp_pack(const float* master, uint8_t* image, cudaStream_t s) {
    mlp::pack_kernel<<<(mlp::kWeights + 255) / 256, 256, 0, s>>>(master, image);
}

cudaError_t launch_mlp_forward(const float* features, const uint8_t* image, float4* outputs, uint32_t n, uint32_t* error, uint32_t ctas,
                               cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(mlp::forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kSmemBytes);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (n + mlp::kRows - 1) / mlp::kRows;
    mlp::forward_kernel<<<tiles < ctas ? tiles : ctas, mlp::kThreads, mlp::kSmemBytes, s>>>(features, image, outputs, n, error);
    return cudaGetLastError();
}

uint32_t mlp_weight_count() { return mlp::kWeights; }
uint32_t mlp_image_bytes() { return mlp::kImageBytes; }

}  // namespace vgi
