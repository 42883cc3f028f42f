// Face trace: the distance-skip DDA over NAADF geometry, the cosine-hemisphere
// path estimator with emitter NEE and MIS, the world-cache gather, and the
// per-face moment reduction.
//
// Behaviour follows the reference shaders line for line (paths within
// nathanaelneveux/global-illumination, crates/bevy_voxel_gi/shaders/):
//   voxel_traversal.wgsl:17-219  face_index_of, lookup_region, advance_box,
//                                geometry_ahead, trace_domain_limited
//   voxel_path.wgsl:63-520       cached_energy, emitter selection and light
//                                tree, QMC sampler, hemisphere, direct_at,
//                                sample_emitter, sample_terminal_emission,
//                                advance_path, trace_receiver
//   voxel_trace.wgsl:25-92       trace_moments, write_result,
//                                trace_faces_parallel
//
// Layout on B200: one thread per (face, lane); the lanes of a face are
// adjacent in a warp and trace the strided subsequences i = lane, lane + L, ...
// (PATH_LANES = L). Lane 0 sums the lanes in order with warp shuffles, which
// gives exactly the cooperative kernel's summation order. The material table
// is staged in shared memory; geometry, face index, cache records and emitter
// words are read through the read-only path (they stay resident in the 126 MB
// L2 for the configurations this targets).
#include <cuda_fp16.h>

#include <algorithm>

#include "vgi_device.cuh"
#include "vgi_types.cuh"

namespace vgi {

// Halton scales per dimension: entry k is the reference's `scale` after k + 1
// divisions by the base (index < 2^24 + 1 has at most 25 base-2 digits).
__constant__ float c_halton_scale[12][25];

namespace {

constexpr int kBlock = 256;

template <bool C>
struct Cnt {
    __device__ void ray() {}
    __device__ void step() {}
    __device__ void bytes(uint32_t) {}
    __device__ void tbytes(uint32_t) {}
    __device__ void status(uint32_t) {}
    __device__ void path() {}
    __device__ void unknown() {}
    __device__ void cache_hit() {}
};
// Counters of the counting variant. `tb` is the traversal's share of the
// algorithmic bytes: directory probes, region headers, brick and cell words.
template <>
struct Cnt<true> {
    uint32_t rays = 0, steps = 0, paths = 0, unk = 0, hits = 0, st[4] = {0, 0, 0, 0};
    uint32_t wp[2] = {0, 0}, lp[2] = {0, 0};
    unsigned long long b = 0, tb = 0;
    __device__ void ray() { rays++; }
    __device__ void step() { steps++; }
    __device__ void bytes(uint32_t n) { b += n; }
    __device__ void tbytes(uint32_t n) {
        b += n;
        tb += n;
    }
    __device__ void status(uint32_t s) { st[s & 3]++; }
    __device__ void path() { paths++; }
    __device__ void unknown() { unk++; }
    __device__ void cache_hit() { hits++; }
};

struct Ray {
    I3 voxel;
    uint32_t material;
    V3 position;
    uint32_t status;
    V3 normal;
};

struct Mat {
    float4 diffuse;    // rgb, w unused (0)
    float4 emission;   // rgb, w unused (0)
    float weight;      // emission_extra.y
};

__device__ __forceinline__ uint32_t face_index_of(V3 n) {
    if (n.x != 0.0f) return n.x < 0.0f ? 1u : 0u;
    if (n.y != 0.0f) return n.y < 0.0f ? 3u : 2u;
    if (n.z != 0.0f) return n.z < 0.0f ? 5u : 4u;
    return 6u;
}
__device__ __forceinline__ V3 face_normal(uint32_t face) {
    float s = (face & 1u) != 0u ? -1.0f : 1.0f;
    uint32_t a = face >> 1;
    return V3{a == 0 ? s : 0.0f, a == 1 ? s : 0.0f, a == 2 ? s : 0.0f};
}

template <bool C>
__device__ __forceinline__ uint32_t lookup_region(const TraceArgs& A, int x, int y, int z, Cnt<C>& cnt) {
    uint32_t slot = hash_voxel(x, y, z) & A.dir_mask;
#pragma unroll 1
    for (uint32_t attempt = 0; attempt < 32u; ++attempt) {
        int4 e = __ldg(A.directory + slot);
        cnt.tbytes(16);
        if (e.w == -1) return kNoIndex;
        if (e.x == x && e.y == y && e.z == z) return (uint32_t)e.w;
        slot = (slot + 1u) & A.dir_mask;
    }
    return kNoIndex;
}

__device__ __forceinline__ bool in_bounds(const TraceArgs& A, int x, int y, int z) {
    return x >= A.mn[0] && y >= A.mn[1] && z >= A.mn[2] && x <= A.mx[0] && y <= A.mx[1] && z <= A.mx[2];
}

// advance_box (voxel_traversal.wgsl:90-107): exit normal and distance of the
// ray from the box (cell - neg, cell + pos + 1) * size. It is split in two:
// box_planes picks the exit plane per axis from the direction's sign, and
// advance_planes runs the rest, so a ray that stays in one box can reuse its
// planes. `inv` holds the direction's reciprocals (direction_recip), so each
// division is div_recip.
__device__ __forceinline__ V3 box_planes(V3 d, I3 cell, I3 ng, I3 ps, float size) {
    return V3{d.x > 0.0f ? __fmul_rn((float)(cell.x + ps.x + 1), size) : __fmul_rn((float)(cell.x - ng.x), size),
              d.y > 0.0f ? __fmul_rn((float)(cell.y + ps.y + 1), size) : __fmul_rn((float)(cell.y - ng.y), size),
              d.z > 0.0f ? __fmul_rn((float)(cell.z + ps.z + 1), size) : __fmul_rn((float)(cell.z - ng.z), size)};
}
__device__ __forceinline__ float4 advance_planes(V3 p, V3 d, V3 inv, V3 plane) {
    float tx, ty, tz;
    {
        bool moving = fabsf(d.x) > 1e-8f;
        float raw = div_recip(__fsub_rn(plane.x, p.x), moving ? d.x : 1.0f, inv.x);
        tx = (moving && raw >= -0.001f && raw < 1e30f) ? raw : 1e30f;
    }
    {
        bool moving = fabsf(d.y) > 1e-8f;
        float raw = div_recip(__fsub_rn(plane.y, p.y), moving ? d.y : 1.0f, inv.y);
        ty = (moving && raw >= -0.001f && raw < 1e30f) ? raw : 1e30f;
    }
    {
        bool moving = fabsf(d.z) > 1e-8f;
        float raw = div_recip(__fsub_rn(plane.z, p.z), moving ? d.z : 1.0f, inv.z);
        tz = (moving && raw >= -0.001f && raw < 1e30f) ? raw : 1e30f;
    }
    bool choose_y = ty < wmax(tx, 0.0f);
    float dxy = wmax(choose_y ? ty : tx, 0.0f);
    bool choose_z = tz < dxy;
    float dist = wmax(choose_z ? tz : dxy, 0.0f);
    float ax = (!choose_z && !choose_y) ? 1.0f : 0.0f;
    float ay = (!choose_z && choose_y) ? 1.0f : 0.0f;
    float az = choose_z ? 1.0f : 0.0f;
    bool hit = dist < 1e30f;
    float4 r;
    r.x = hit ? __fmul_rn(ax, d.x > 0.0f ? -1.0f : 1.0f) : 0.0f;
    r.y = hit ? __fmul_rn(ay, d.y > 0.0f ? -1.0f : 1.0f) : 0.0f;
    r.z = hit ? __fmul_rn(az, d.z > 0.0f ? -1.0f : 1.0f) : 0.0f;
    r.w = wmax(__fadd_rn(dist, 0.001f), 0.001f);
    return r;
}
__device__ __forceinline__ float4 advance_box(V3 p, V3 d, V3 inv, I3 cell, I3 ng, I3 ps, float size) {
    return advance_planes(p, d, inv, box_planes(d, cell, ng, ps, size));
}

__device__ __forceinline__ I3 unpack_bytes(uint32_t v) { return I3{(int)(v & 255u), (int)((v >> 8) & 255u), (int)((v >> 16) & 255u)}; }
__device__ __forceinline__ I3 neg_ext(uint32_t b) { return I3{(int)(b & 3u), (int)((b >> 4) & 3u), (int)((b >> 8) & 3u)}; }
__device__ __forceinline__ I3 pos_ext(uint32_t b) { return I3{(int)((b >> 2) & 3u), (int)((b >> 6) & 3u), (int)((b >> 10) & 3u)}; }

// floor(position / 16.0): dividing by a power of two is exact, so multiplying
// by 1/16 rounds to the same value.
__device__ __forceinline__ I3 floor_div16(V3 p) {
    return I3{f2i(floorf(__fmul_rn(p.x, 0.0625f))), f2i(floorf(__fmul_rn(p.y, 0.0625f))), f2i(floorf(__fmul_rn(p.z, 0.0625f)))};
}

// geometry_ahead (voxel_traversal.wgsl:108-121)
template <bool C>
__device__ bool geometry_ahead(const TraceArgs& A, V3 position, V3 dir, V3 inv, float remaining, Cnt<C>& cnt) {
#pragma unroll 1
    for (uint32_t step = 0; step < 2048u; ++step) {
        cnt.step();
        I3 r = floor_div16(position);
        if (remaining < 0.0f || !in_bounds(A, r.x, r.y, r.z)) return false;
        uint32_t index = lookup_region(A, r.x, r.y, r.z, cnt);
        if (index != kNoIndex) {
            cnt.tbytes(16);
            if (__ldg(&A.headers[index].x) != 1u) return true;
        }
        float travel = advance_box(position, dir, inv, r, I3{0, 0, 0}, I3{0, 0, 0}, 16.0f).w;
        position = position + dir * travel;
        remaining = __fsub_rn(remaining, travel);
    }
    return true;
}

// trace_domain_limited (voxel_traversal.wgsl:126-219)
template <bool C>
__device__ Ray trace_domain(const TraceArgs& A, V3 origin, V3 dir, float max_distance, bool visible_geometry, uint32_t max_steps,
                            Cnt<C>& cnt) {
    cnt.ray();
    Ray res;
    res.voxel = I3{0, 0, 0};
    res.material = 0u;
    res.position = V3{0.0f, 0.0f, 0.0f};
    res.status = 0u;
    res.normal = V3{0.0f, 0.0f, 0.0f};
    float nearv = -1e30f, farv = 1e30f;
    V3 normal{0.0f, 0.0f, 0.0f};
    const V3 inv = direction_recip(dir);
    const float mnx = __fmul_rn((float)A.mn[0], 16.0f), mny = __fmul_rn((float)A.mn[1], 16.0f), mnz = __fmul_rn((float)A.mn[2], 16.0f);
    const float mxx = __fmul_rn((float)(A.mx[0] + 1), 16.0f), mxy = __fmul_rn((float)(A.mx[1] + 1), 16.0f),
                mxz = __fmul_rn((float)(A.mx[2] + 1), 16.0f);
#define VGI_SLAB(AX, O, D, Y, MN, MX)                                           \
    if (fabsf(D) <= 1e-8f) {                                                    \
        if (O < MN || O > MX) { cnt.status(0); return res; }                    \
    } else {                                                                    \
        float first = div_recip(__fsub_rn(MN, O), D, Y);                        \
        float second = div_recip(__fsub_rn(MX, O), D, Y);                       \
        if (wmin(first, second) > nearv) {                                      \
            nearv = wmin(first, second);                                        \
            float s = first < second ? -1.0f : 1.0f;                            \
            normal = V3{AX == 0 ? s : 0.0f, AX == 1 ? s : 0.0f, AX == 2 ? s : 0.0f}; \
        }                                                                       \
        farv = wmin(farv, wmax(first, second));                                 \
    }
    VGI_SLAB(0, origin.x, dir.x, inv.x, mnx, mxx)
    VGI_SLAB(1, origin.y, dir.y, inv.y, mny, mxy)
    VGI_SLAB(2, origin.z, dir.z, inv.z, mnz, mxz)
#undef VGI_SLAB
    if (farv < wmax(nearv, 0.0f)) { cnt.status(0); return res; }
    float distance = __fadd_rn(wmax(nearv, 0.0f), 0.001f);
    V3 position = origin + dir * distance;
    int lrx = 0x7fffffff, lry = 0x7fffffff, lrz = 0x7fffffff;
    uint4 meta = make_uint4(0, 0, 0, 0);
#pragma unroll 1
    for (uint32_t step = 0; step < max_steps; ++step) {
        cnt.step();
        if (distance > max_distance) { cnt.status(0); return res; }
        I3 voxel{f2i(floorf(position.x)), f2i(floorf(position.y)), f2i(floorf(position.z))};
        int rx = voxel.x >> 4, ry = voxel.y >> 4, rz = voxel.z >> 4;
        if (!in_bounds(A, rx, ry, rz)) { cnt.status(0); return res; }
        if (lrx != rx || lry != ry || lrz != rz) {
            uint32_t index = lookup_region(A, rx, ry, rz, cnt);
            if (index == kNoIndex) {
                if (visible_geometry) {
                    float4 adv = advance_box(position, dir, inv, I3{rx, ry, rz}, I3{0, 0, 0}, I3{0, 0, 0}, 16.0f);
                    distance = __fadd_rn(distance, adv.w);
                    position = position + dir * adv.w;
                    normal = V3{adv.x, adv.y, adv.z};
                    continue;
                }
                res.status = geometry_ahead(A, position, dir, inv, __fsub_rn(max_distance, distance), cnt) ? 2u : 0u;
                cnt.status(res.status);
                return res;
            }
            cnt.tbytes(16);
            meta = __ldg(A.headers + index);
            lrx = rx; lry = ry; lrz = rz;
        }
        float4 adv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (meta.x == 1u) {
            adv = advance_box(position, dir, inv, I3{rx, ry, rz}, unpack_bytes(meta.z), unpack_bytes(meta.w), 16.0f);
        } else {
            uint32_t material = meta.y;
            if (meta.x == 3u) {
                uint32_t lx = (uint32_t)(voxel.x & 15), ly = (uint32_t)(voxel.y & 15), lz = (uint32_t)(voxel.z & 15);
                uint32_t bx = lx >> 2, by = ly >> 2, bz = lz >> 2;
                uint32_t brick = __ldg(A.cells + meta.y + (bz * 4u + by) * 4u + bx);
                cnt.tbytes(4);
                uint32_t state = brick & 3u;
                if (state == 0u) {
                    uint32_t ext = brick >> 2u;
                    adv = advance_box(position, dir, inv, I3{rx * 4 + (int)bx, ry * 4 + (int)by, rz * 4 + (int)bz}, neg_ext(ext), pos_ext(ext), 4.0f);
                    material = 256u;
                } else if (state == 1u) {
                    material = brick >> 2u;
                } else {
                    uint32_t idx = ((lz & 3u) * 4u + (ly & 3u)) * 4u + (lx & 3u);
                    uint32_t word = __ldg(A.cells + (brick >> 2u) + (idx >> 1));
                    cnt.tbytes(4);
                    uint32_t cell = (word >> ((idx & 1u) * 16u)) & 65535u;
                    material = (cell & 1u) != 0u ? (cell >> 1u) : 256u;
                    if (material == 256u) {
                        uint32_t ext = cell >> 1u;
                        adv = advance_box(position, dir, inv, voxel, neg_ext(ext), pos_ext(ext), 1.0f);
                    }
                }
            }
            if (material != 256u) {
                res.voxel = voxel;
                res.material = material;
                res.position = position;
                res.normal = normal;
                res.status = 1u;
                cnt.status(1);
                return res;
            }
        }
        distance = __fadd_rn(distance, adv.w);
        position = position + dir * adv.w;
        normal = V3{adv.x, adv.y, adv.z};
    }
    res.status = 2u;
    res.material = 0xffffffffu;
    cnt.status(2);
    return res;
}

// ---- estimator ---------------------------------------------------------------
struct Emissive {
    I3 voxel;
    uint32_t face;
    float4 sampling;
};

template <bool C>
__device__ __forceinline__ Emissive load_emitter(const TraceArgs& A, uint32_t index, Cnt<C>& cnt) {
    cnt.bytes(32);
    uint4 a = __ldg(A.emitters + index * 2u);
    uint4 b = __ldg(A.emitters + index * 2u + 1u);
    return Emissive{I3{(int)a.x, (int)a.y, (int)a.z}, a.w,
                    make_float4(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z), __uint_as_float(b.w))};
}

// Light-tree nodes (LightNode, voxel_path.wgsl:93-107) are read through a
// companion record per node, built once per emitter upload by node_aux_kernel:
//   aux[2i]     = (centre xyz, radius): (min + max) * 0.5 and
//                 length(max - min) * 0.5, the values node_importance derives
//                 on every visit, computed with the same operations;
//   aux[2i + 1] = (power, normals, left, right) as raw words.
// The walk then moves 16-32 bytes per node instead of 64. The algorithmic
// byte count still charges the node records the shader loads.
struct NodeLite {
    float4 geo;   // centre xyz, radius
    uint4 link;   // power bits, normals, left, right
};

__device__ __forceinline__ NodeLite load_lite(const TraceArgs& A, uint32_t index) {
    return NodeLite{__ldg(A.node_aux + 2u * index), __ldg(reinterpret_cast<const uint4*>(A.node_aux) + 2u * index + 1u)};
}

// voxel_path.wgsl:108-122
__device__ float node_importance(const NodeLite& node, V3 position, V3 normal) {
    V3 delta = V3{node.geo.x, node.geo.y, node.geo.z} - position;
    float radius = node.geo.w;
    float distance = wmax(len3(delta), 1e-5f);
    V3 direction = delta / distance;
    float spread = wmin(__fdiv_rn(radius, distance), 1.0f);
    float receiver = wclamp(__fadd_rn(dot3(normal, direction), spread), 0.0f, 1.0f);
    const uint32_t normals = node.link.y;
    float px = (normals & 1u) ? -direction.x : -1.0f;
    float py = (normals & 4u) ? -direction.y : -1.0f;
    float pz = (normals & 16u) ? -direction.z : -1.0f;
    float nx = (normals & 2u) ? direction.x : -1.0f;
    float ny = (normals & 8u) ? direction.y : -1.0f;
    float nz = (normals & 32u) ? direction.z : -1.0f;
    float qx = wmax(px, nx), qy = wmax(py, ny), qz = wmax(pz, nz);
    float emitter = wclamp(__fadd_rn(wmax(wmax(qx, qy), qz), spread), 0.0f, 1.0f);
    float num = __fmul_rn(__fmul_rn(__uint_as_float(node.link.x), receiver), emitter);
    float den = __fadd_rn(__fadd_rn(__fmul_rn(distance, distance), __fmul_rn(radius, radius)), 0.25f);
    return __fdiv_rn(num, den);
}

// voxel_path.wgsl:123-131, given the node's children.
template <bool C>
__device__ float node_left_probability(const TraceArgs& A, uint32_t left_index, uint32_t right_index, V3 position, V3 normal, Cnt<C>& cnt) {
    cnt.bytes(128);  // load_node(left) + load_node(right)
    const NodeLite left = load_lite(A, left_index);
    const NodeLite right = load_lite(A, right_index);
    const float lp = __uint_as_float(left.link.x), rp = __uint_as_float(right.link.x);
    float power = __fdiv_rn(lp, __fadd_rn(lp, rp));
    float a = node_importance(left, position, normal);
    float b = node_importance(right, position, normal);
    if (__fadd_rn(a, b) <= 1e-20f) return wclamp(power, 1e-6f, 0.999999f);
    return wclamp(__fadd_rn(__fmul_rn(0.05f, power), __fdiv_rn(__fmul_rn(0.95f, a), __fadd_rn(a, b))), 1e-6f, 0.999999f);
}

// `top`, when given, holds node_left_probability of the nodes at heap slots
// 0..kTreeTopSlots-1 (slot s's children at 2s + 1 and 2s + 2) for this
// position and normal, as wave_begin_kernel keeps them per receiver: the
// same values, so the walk takes the same branches.
template <bool C>
__device__ Emissive tree_emitter(const TraceArgs& A, V3 position, V3 normal, float choice, Cnt<C>& cnt, const float* top = nullptr) {
    uint32_t index = 0, slot = 0;
    float u = choice, probability = 1.0f;
    // Median splits keep the hierarchy balanced (depth <= 33); the host
    // checks that children follow their parent, so the walk ends. The bound
    // only guards malformed words: a zero-probability emitter contributes 0.
#pragma unroll 1
    for (uint32_t depth = 0; depth < 64u; ++depth) {
        cnt.bytes(64);  // load_node(index)
        const uint4 link = __ldg(reinterpret_cast<const uint4*>(A.node_aux) + 2u * index + 1u);
        if (link.z == 0xffffffffu) {
            Emissive e = load_emitter(A, link.w, cnt);
            e.sampling.y = probability;
            return e;
        }
        const float p = (top != nullptr && slot < kTreeTopSlots) ? top[slot] : node_left_probability(A, link.z, link.w, position, normal, cnt);
        if (u < p) {
            probability = __fmul_rn(probability, p);
            u = __fdiv_rn(u, p);
            index = link.z;
            slot = slot < kTreeTopSlots ? 2u * slot + 1u : kTreeTopSlots;
        } else {
            probability = __fmul_rn(probability, __fsub_rn(1.0f, p));
            u = __fdiv_rn(__fsub_rn(u, p), __fsub_rn(1.0f, p));
            index = link.w;
            slot = slot < kTreeTopSlots ? 2u * slot + 2u : kTreeTopSlots;
        }
        u = wmin(u, __uint_as_float(0x3f7fffffu));
    }
    return Emissive{I3{0, 0, 0}, 0u, make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
}

// node_left_probability of the node at heap slot `slot` of the walk (the
// bits of slot + 1 below its leading one, from the top: 0 left, 1 right),
// or -1 when the walk never asks there (a leaf on the way, or the slot's
// node is a leaf).
__device__ float tree_slot_probability(const TraceArgs& A, uint32_t slot, V3 position, V3 normal) {
    Cnt<false> none;
    const uint32_t path = slot + 1u;
    const int depth = 31 - __clz(path);
    uint32_t index = 0;
    for (int b = depth - 1; b >= 0; --b) {
        const uint4 link = __ldg(reinterpret_cast<const uint4*>(A.node_aux) + 2u * index + 1u);
        if (link.z == 0xffffffffu) return -1.0f;
        index = ((path >> b) & 1u) ? link.w : link.z;
    }
    const uint4 link = __ldg(reinterpret_cast<const uint4*>(A.node_aux) + 2u * index + 1u);
    if (link.z == 0xffffffffu) return -1.0f;
    return node_left_probability(A, link.z, link.w, position, normal, none);
}

__device__ __forceinline__ int comp(I3 v, uint32_t i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// key_less (voxel_path.wgsl:150-157) against the node's pivot word (voxel
// xyz, face) and link word (left, right, axis).
__device__ __forceinline__ bool key_less(I3 voxel, uint32_t face, uint4 pivot, uint32_t axis) {
    const I3 p{(int)pivot.x, (int)pivot.y, (int)pivot.z};
#pragma unroll
    for (uint32_t j = 0; j < 3u; ++j) {
        uint32_t i = (axis + j) % 3u;
        int a = comp(voxel, i), b = comp(p, i);
        if (a != b) return a < b;
    }
    return face < pivot.w;
}

template <bool C>
__device__ float tree_probability(const TraceArgs& A, V3 position, V3 normal, I3 voxel, V3 hit_normal, Cnt<C>& cnt) {
    uint32_t face = 0;
#pragma unroll
    for (uint32_t i = 0; i < 6u; ++i) {
        V3 fn = face_normal(i);
        if (fn.x == hit_normal.x && fn.y == hit_normal.y && fn.z == hit_normal.z) face = i;
    }
    uint32_t index = 0;
    float probability = 1.0f;
    const uint32_t first_node = f2u(A.emitter_count) * 2u;
#pragma unroll 1
    for (uint32_t depth = 0; depth < 64u; ++depth) {
        cnt.bytes(64);  // load_node(index)
        const uint4 pivot = __ldg(A.emitters + first_node + index * 4u + 2u);
        const uint4 link = __ldg(A.emitters + first_node + index * 4u + 3u);  // left, right, axis
        if (link.x == 0xffffffffu) {
            Emissive found = load_emitter(A, link.y, cnt);
            bool same = found.voxel.x == voxel.x && found.voxel.y == voxel.y && found.voxel.z == voxel.z && found.face == face;
            return same ? probability : 0.0f;
        }
        float p = node_left_probability(A, link.x, link.y, position, normal, cnt);
        if (key_less(voxel, face, pivot, link.z)) {
            probability = __fmul_rn(probability, p);
            index = link.x;
        } else {
            probability = __fmul_rn(probability, __fsub_rn(1.0f, p));
            index = link.y;
        }
    }
    return 0.0f;
}

// voxel_path.wgsl:178-213 (the Owen scramble is sobol_burley's hash)
__device__ __forceinline__ uint32_t scramble_reverse(uint32_t v, uint32_t seed) {
    v ^= v * 0x3d20adeau;
    v += seed;
    v *= (seed >> 16u) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return v;
}

// The radical inverse of voxel_path.wgsl:191-198: digit k of `index` in base
// BASE times scale_k, where scale_k is the k-th value of the reference's
// running `scale /= f32(base)`. The scales are precomputed with the same IEEE
// divisions (c_halton_scale), and BASE is a compile-time constant, so each
// digit costs a multiply-high instead of an integer and a float division.
template <uint32_t BASE>
__device__ __forceinline__ float radical_inverse(uint32_t index, const float* scale) {
    float value = 0.0f;
    uint32_t k = 0;
#pragma unroll 1
    while (index != 0u) {
        const uint32_t q = index / BASE;
        value = __fadd_rn(value, __fmul_rn((float)(index - q * BASE), scale[k]));
        index = q;
        ++k;
    }
    return value;
}

__device__ float sample_1d(uint32_t stream, uint32_t sequence, uint32_t dimension) {
    if (dimension < 12u) {
        const uint32_t index = (sequence & 0x00ffffffu) + 1u;
        float value;
        switch (dimension) {
            case 0: value = radical_inverse<2>(index, c_halton_scale[0]); break;
            case 1: value = radical_inverse<3>(index, c_halton_scale[1]); break;
            case 2: value = radical_inverse<5>(index, c_halton_scale[2]); break;
            case 3: value = radical_inverse<7>(index, c_halton_scale[3]); break;
            case 4: value = radical_inverse<11>(index, c_halton_scale[4]); break;
            case 5: value = radical_inverse<13>(index, c_halton_scale[5]); break;
            case 6: value = radical_inverse<17>(index, c_halton_scale[6]); break;
            case 7: value = radical_inverse<19>(index, c_halton_scale[7]); break;
            case 8: value = radical_inverse<23>(index, c_halton_scale[8]); break;
            case 9: value = radical_inverse<29>(index, c_halton_scale[9]); break;
            case 10: value = radical_inverse<31>(index, c_halton_scale[10]); break;
            default: value = radical_inverse<37>(index, c_halton_scale[11]); break;
        }
        // x / 2^23 is exact, so the multiply gives the same bits.
        float rotation = __fmul_rn((float)(pcg(stream ^ pcg(dimension)) >> 9u), 0x1p-23f);
        float t = __fadd_rn(value, rotation);
        return __fsub_rn(t, floorf(t));
    }
    uint32_t seed = pcg(stream ^ pcg(dimension / 2u));
    uint32_t index = __brev(scramble_reverse(__brev(sequence), pcg(seed ^ 0x79c68e4au)));
    if ((dimension & 1u) != 0u) {
        index ^= (index >> 1u) & 0x55555555u;
        index ^= (index >> 2u) & 0x33333333u;
        index ^= (index >> 4u) & 0x0f0f0f0fu;
        index ^= (index >> 8u) & 0x00ff00ffu;
        index ^= (index >> 16u) & 0x0000ffffu;
    }
    uint32_t value = __brev(scramble_reverse(index, pcg(seed ^ pcg(dimension))));
    return __fmul_rn((float)(value >> 9u), 0x1p-23f);
}

__device__ __forceinline__ float continuation_sample(uint32_t stream, uint32_t sequence, uint32_t bounce, uint32_t dimension) {
    if (bounce < 3u) {
        uint32_t legacy = dimension == 2u ? 8u + bounce : 2u + bounce * 2u + dimension;
        return sample_1d(stream, sequence, legacy);
    }
    return sample_1d(stream, sequence, 16u + (bounce - 3u) * 3u + dimension);
}

// voxel_path.wgsl:231-238
__device__ V3 hemisphere(V3 n, float u, float v) {
    V3 tangent = fabsf(n.z) < 0.999f ? normalize3(cross3(n, V3{0.0f, 0.0f, 1.0f})) : normalize3(cross3(n, V3{0.0f, 1.0f, 0.0f}));
    V3 bitangent = cross3(n, tangent);
    float phi = __fmul_rn(6.28318530718f, u);
    float s, c;
    own_sincos(phi, &s, &c);
    float sv = __fsqrt_rn(v);
    return (tangent * __fmul_rn(c, sv) + bitangent * __fmul_rn(s, sv)) + n * __fsqrt_rn(__fsub_rn(1.0f, v));
}

__device__ __forceinline__ float cosine_pdf(V3 n, V3 d) { return __fdiv_rn(wmax(dot3(n, d), 0.0f), 3.14159265359f); }

template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
struct Tracer {
    const TraceArgs& A;
    const float4* smat;   // shared material table, 2 float4 per material
    Cnt<C>& cnt;

    __device__ Mat material(uint32_t m) {
        cnt.bytes(64);
        // Material ids are below 256 for every geometry the host accepts.
        m &= 255u;
        float4 d = smat[m * 2u], e = smat[m * 2u + 1u];
        return Mat{make_float4(d.x, d.y, d.z, 0.0f), make_float4(e.x, e.y, e.z, 0.0f), d.w};
    }
    __device__ float reach() const { return LIMITED ? A.reach : A.max_distance; }

    // voxel_path.wgsl:239-243
    __device__ Ray trace(V3 origin, V3 dir, float max_distance) {
        Ray r = trace_domain(A, origin, dir, max_distance, BUDGETED, A.path_steps, cnt);
        if (BUDGETED && r.status == 2u && r.material == 0xffffffffu) r.status = 0u;
        return r;
    }
    // voxel_path.wgsl:271-282
    __device__ Ray trace_diffuse(V3 origin, V3 dir) {
        float r = reach();
        Ray hit = trace(origin, dir, r);
        if (LIMITED && hit.status == 0u && geometry_ahead(A, origin + dir * r, dir, direction_recip(dir), __fsub_rn(A.max_distance, r), cnt)) hit.status = 3u;
        return hit;
    }
    // voxel_path.wgsl:283-307 (value rgb; custom_visible only at the face centre)
    template <bool CUSTOM>
    __device__ void direct_at(V3 position, V3 normal, V3& value, V3& custom, float* value_w = nullptr) {
        value = V3{0.0f, 0.0f, 0.0f};
        custom = V3{0.0f, 0.0f, 0.0f};
        float w = 0.0f;
        V3 origin = position + normal * 0.002f;
#pragma unroll 1
        for (uint32_t i = 0; i < A.light_count; ++i) {
            const float4 Lp = __ldg(A.lights + i * 3u), Le = __ldg(A.lights + i * 3u + 1u), Lx = __ldg(A.lights + i * 3u + 2u);
            cnt.bytes(48);
            V3 pos{Lp.x, Lp.y, Lp.z};
            float distance = A.max_distance;
            float attenuation = 1.0f;
            V3 direction;
            if (Lp.w >= 0.0f) {
                V3 delta = pos - position;
                float d2 = dot3(delta, delta);
                if (d2 <= 0.0000001f || d2 > __fmul_rn(Lp.w, Lp.w)) continue;
                distance = __fsqrt_rn(d2);
                direction = delta / distance;
                distance = __fsub_rn(distance, 0.004f);
                attenuation = __fdiv_rn(1.0f, wmax(d2, 1.0f));
            } else {
                direction = normalize3(pos);
            }
            float cosine = wmax(dot3(normal, direction), 0.0f);
            if (cosine > 0.0f && trace(origin, direction, distance).status == 0u) {
                float k = __fmul_rn(cosine, attenuation);
                value = value + V3{Le.x, Le.y, Le.z} * k;
                if (CUSTOM) {
                    custom = custom + V3{Lx.y, Lx.z, Lx.w} * k;
                    w = __fadd_rn(w, __fmul_rn(Le.w, k));
                }
            }
        }
        if (CUSTOM && value_w) *value_w = w;
    }
    // voxel_path.wgsl:309-324
    __device__ Emissive choose_emitter(V3 position, V3 normal, float choice) {
        uint32_t count = f2u(A.emitter_count);
        if (load_emitter(A, 0u, cnt).sampling.w > 0.0f) return tree_emitter(A, position, normal, choice, cnt);
        uint32_t low = 0, high = count;
#pragma unroll 1
        while (low < high) {
            uint32_t middle = (low + high) / 2u;
            if (load_emitter(A, middle, cnt).sampling.x <= choice) low = middle + 1u;
            else high = middle;
        }
        return load_emitter(A, low < count - 1u ? low : count - 1u, cnt);
    }
    // voxel_path.wgsl:332-364
    __device__ V3 sample_emitter(V3 position, V3 normal, uint32_t source_stream, uint32_t sequence, uint32_t bounce) {
        V3 zero{0.0f, 0.0f, 0.0f};
        if (A.emitter_count == 0.0f) return zero;
        uint32_t stream = source_stream ^ pcg(bounce + 0xa341316cu);
        Emissive em = choose_emitter(position, normal, sample_1d(stream, sequence, 12u));
        V3 en = face_normal(em.face);
        uint32_t axis = em.face / 2u;
        V3 tangent = axis == 0u ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
        V3 bitangent = axis == 2u ? V3{0.0f, 1.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f};
        float s13 = __fsub_rn(sample_1d(stream, sequence, 13u), 0.5f);
        float s14 = __fsub_rn(sample_1d(stream, sequence, 14u), 0.5f);
        V3 lp = ((add_s(itof(em.voxel), 0.5f) + en * 0.5f) + tangent * s13) + bitangent * s14;
        V3 delta = lp - position;
        float d2 = dot3(delta, delta);
        float r = reach();
        if (d2 < 0.0001f || d2 > __fmul_rn(r, r)) return zero;
        float distance = __fsqrt_rn(d2);
        V3 direction = delta / distance;
        float rc = wmax(dot3(normal, direction), 0.0f);
        float ec = wmax(dot3(en, -direction), 0.0f);
        if (rc <= 0.0f || ec <= 0.0f || em.sampling.y <= 0.0f) return zero;
        float light_pdf = __fdiv_rn(__fmul_rn(em.sampling.y, d2), ec);
        float directional_pdf = __fdiv_rn(rc, 3.14159265359f);
        V3 so = position + normal * 0.002f;
        V3 sd = (lp + en * 0.002f) - so;
        float sdist = len3(sd);
        if (trace(so, sd / sdist, sdist).status != 0u) return zero;
        Mat m = material(f2u(em.sampling.z));
        float factor = __fdiv_rn(directional_pdf, __fadd_rn(light_pdf, directional_pdf));
        return V3{m.emission.x, m.emission.y, m.emission.z} * factor;
    }
    // voxel_path.wgsl:368-394
    __device__ V3 sample_terminal_emission(V3 position, V3 normal, uint32_t stream, uint32_t sequence, uint32_t bounce) {
        V3 zero{0.0f, 0.0f, 0.0f};
        if (A.emitter_count == 0.0f) return zero;
        if (continuation_sample(stream, sequence, bounce, 2u) < 0.5f) return sample_emitter(position, normal, stream, sequence, bounce + 1u) * 2.0f;
        V3 direction = hemisphere(normal, continuation_sample(stream, sequence, bounce, 0u), continuation_sample(stream, sequence, bounce, 1u));
        if (dot3(normal, direction) <= 0.0f) return zero;
        float r = reach();
        Ray hit = trace(position + normal * 0.002f, direction, r);
        if (hit.status != 1u) return zero;
        Mat m = material(hit.material);
        float power = m.weight;
        V3 delta = hit.position - position;
        float d2 = dot3(delta, delta);
        if (power == 0.0f || d2 < 0.0001f || d2 > __fmul_rn(r, r)) return zero;
        float selection_pdf = __fdiv_rn(power, wmax(A.emitter_total, 1e-20f));
        if (load_emitter(A, 0u, cnt).sampling.w > 0.0f) selection_pdf = tree_probability(A, position, normal, hit.voxel, hit.normal, cnt);
        float light_pdf = __fdiv_rn(__fmul_rn(selection_pdf, d2), wmax(dot3(hit.normal, -direction), 1e-8f));
        float directional_pdf = cosine_pdf(normal, direction);
        float factor = __fdiv_rn(__fmul_rn(2.0f, directional_pdf), __fadd_rn(directional_pdf, light_pdf));
        return V3{m.emission.x, m.emission.y, m.emission.z} * factor;
    }
    // voxel_path.wgsl:66-87; the slot's record holds (mean rgb, count word).
    __device__ bool cached_energy(I3 voxel, uint32_t face, V3& value) {
        if (face > 5u || A.face_index == nullptr) return false;
        uint4 header = __ldg(A.face_index);
        uint32_t mask = header.x;
        uint32_t slot = (hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u)) & mask;
#pragma unroll 1
        for (uint32_t attempt = 0; attempt < header.y; ++attempt) {
            uint4 e = __ldg(A.face_index + slot + 1u);
            cnt.bytes(16);
            if (e.w == 0xffffffffu) return false;
            if ((int)e.x == voxel.x && (int)e.y == voxel.y && (int)e.z == voxel.z && (e.w >> 29u) == face) {
                float4 rec = __ldg(A.cache + (e.w & 0x1fffffffu));
                cnt.bytes(16);
                uint32_t count = __float_as_uint(rec.w);
                if (count < 16u || (count & 0x80000000u) != 0u) return false;
                value = V3{rec.x, rec.y, rec.z};
                return true;
            }
            slot = (slot + 1u) & mask;
        }
        return false;
    }
    // voxel_path.wgsl:418-496: begin_path + advance_path with DIFFUSE_HITS steps
    // and the terminal mixture; returns the continuation's energy.
    __device__ V3 trace_path(V3 start, V3 direction, V3 normal, uint32_t stream, uint32_t sequence, bool& unknown) {
        V3 energy{0.0f, 0.0f, 0.0f};
        V3 tp{1.0f, 1.0f, 1.0f};
        V3 origin = start;
        float previous_pdf = cosine_pdf(normal, direction);
        V3 previous_position = start - normal * 0.001f;
        V3 previous_normal = normal;
        if (previous_pdf <= 0.0f) return energy;
#pragma unroll 1
        for (uint32_t step = 0; step < HITS; ++step) {
            uint32_t bounce = step;
            Ray hit = trace_diffuse(origin, direction);
            if (hit.status == 0u) {
                float horizon = wclamp(__fadd_rn(__fmul_rn(direction.y, 0.35f), 0.65f), 0.15f, 1.0f);
                energy = energy + (tp * V3{A.env[0], A.env[1], A.env[2]}) * horizon;
                break;
            }
            if (hit.status == 2u) { unknown = true; break; }
            if (hit.status == 3u) break;
            Mat m = material(hit.material);
            V3 direct, unused;
            direct_at<false>(hit.position, hit.normal, direct, unused);
            float emission_weight = m.weight;
            V3 delta = hit.position - origin;
            float selection_pdf = __fdiv_rn(emission_weight, wmax(A.emitter_total, 1e-20f));
            if (emission_weight > 0.0f && A.emitter_count > 0.0f && load_emitter(A, 0u, cnt).sampling.w > 0.0f)
                selection_pdf = tree_probability(A, previous_position, previous_normal, hit.voxel, hit.normal, cnt);
            float light_pdf = __fdiv_rn(__fmul_rn(selection_pdf, dot3(delta, delta)), wmax(dot3(hit.normal, -direction), 1e-8f));
            float mis = 1.0f;
            if (light_pdf > 0.0f) mis = __fdiv_rn(previous_pdf, __fadd_rn(previous_pdf, light_pdf));
            V3 emission{m.emission.x, m.emission.y, m.emission.z};
            V3 diffuse{m.diffuse.x, m.diffuse.y, m.diffuse.z};
            V3 cached;
            if (cached_energy(hit.voxel, face_index_of(hit.normal), cached)) {
                cnt.cache_hit();
                energy = energy + tp * (emission * mis + diffuse * (direct + cached));
                break;
            }
            bool last = step + 1u == HITS;
            V3 nee = last ? sample_terminal_emission(hit.position, hit.normal, stream, sequence, bounce)
                          : sample_emitter(hit.position, hit.normal, stream, sequence, bounce + 1u);
            energy = energy + tp * (emission * mis + diffuse * (direct + nee));
            if (last) break;
            tp = tp * diffuse;
            float maximum = wmax(tp.x, wmax(tp.y, tp.z));
            if (maximum == 0.0f) break;
            if (bounce >= 1u) {
                float survival = wclamp(maximum, 0.1f, 0.95f);
                if (continuation_sample(stream, sequence, bounce, 2u) > survival) break;
                tp = tp / survival;
            }
            origin = hit.position + hit.normal * 0.002f;
            previous_position = hit.position;
            previous_normal = hit.normal;
            direction = hemisphere(hit.normal, continuation_sample(stream, sequence, bounce, 0u), continuation_sample(stream, sequence, bounce, 1u));
            previous_pdf = cosine_pdf(hit.normal, direction);
            if (previous_pdf <= 0.0f) break;
        }
        return energy;
    }
};

template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__global__ void __launch_bounds__(kBlock) trace_faces_kernel(const TraceArgs A) {
    __shared__ float4 smat[512];
    for (int i = threadIdx.x; i < 256; i += kBlock) {
        float4 d = __ldg(A.materials + i * 4), e = __ldg(A.materials + i * 4 + 2), x = __ldg(A.materials + i * 4 + 3);
        smat[i * 2] = make_float4(d.x, d.y, d.z, x.y);
        smat[i * 2 + 1] = make_float4(e.x, e.y, e.z, 0.0f);
    }
    __syncthreads();
    Cnt<C> cnt;
    Tracer<HITS, LIMITED, BUDGETED, C> T{A, smat, cnt};
    const uint32_t lanes = 1u << A.lanes_log2;
    const uint32_t gid = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t face = gid >> A.lanes_log2;
    const uint32_t lane = gid & (lanes - 1u);
    uint4 t0 = make_uint4(0, 0, 0, 0xffffffffu), t1 = make_uint4(0, 0, 0, 0);
    if (face < A.n_tasks) {
        t0 = __ldg(A.tasks + face * 2u);
        t1 = __ldg(A.tasks + face * 2u + 1u);
    }
    const bool valid = face < A.n_tasks && t0.w != 0xffffffffu;
    V3 mean{0.0f, 0.0f, 0.0f}, second{0.0f, 0.0f, 0.0f};
    uint32_t known = 0;
    V3 normal = face_normal(valid ? t0.w : 0u);
    I3 voxel{(int)t0.x, (int)t0.y, (int)t0.z};
    V3 surface = add_s(itof(voxel), 0.5f) + normal * 0.5f;
    if (valid) {
        if (lane == 0) cnt.bytes(32 + 96);
        const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(t0.w + 1u);
#pragma unroll 1
        for (uint32_t i = lane; i < A.samples; i += lanes) {
            const uint32_t sequence = t1.x + i;
            cnt.path();
            // voxel_path.wgsl:504-520 (sample_receiver_path + trace_receiver)
            V3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
            V3 value = T.sample_emitter(surface, normal, stream, sequence, 0u);
            bool unknown = false;
            if (dot3(normal, direction) > 0.0f) {
                V3 cont = T.trace_path(surface + normal * 0.001f, direction, normal, stream, sequence, unknown);
                value = value + cont;
            }
            if (unknown) { cnt.unknown(); continue; }
            mean = mean + value;
            second = second + value * value;
            known += 1u;
        }
    }
    // Lane 0 sums lanes 0..L-1 in order (trace_faces_parallel's reduction);
    // with one lane this is the serial kernel's 0 + sum.
    V3 tm{0.0f, 0.0f, 0.0f}, ts{0.0f, 0.0f, 0.0f};
    uint32_t tk = 0;
    {
        const uint32_t base = (threadIdx.x & 31u) & ~(lanes - 1u);
        for (uint32_t i = 0; i < lanes; ++i) {
            float mx = __shfl_sync(0xffffffffu, mean.x, base + i), my = __shfl_sync(0xffffffffu, mean.y, base + i),
                  mz = __shfl_sync(0xffffffffu, mean.z, base + i);
            float sx = __shfl_sync(0xffffffffu, second.x, base + i), sy = __shfl_sync(0xffffffffu, second.y, base + i),
                  sz = __shfl_sync(0xffffffffu, second.z, base + i);
            uint32_t k = __shfl_sync(0xffffffffu, known, base + i);
            tm = tm + V3{mx, my, mz};
            ts = ts + V3{sx, sy, sz};
            tk += k;
        }
    }
    if (valid && lane == 0) {
        // write_result (voxel_trace.wgsl:25-37)
        V3 dv, dc;
        float dw = 0.0f;
        T.template direct_at<true>(surface, normal, dv, dc, &dw);
        float inverse = __fdiv_rn(1.0f, (float)(tk > 1u ? tk : 1u));
        V3 m = tm * inverse, s = ts * inverse;
        uint4* out = A.results + (size_t)face * 6u;
        out[0] = make_uint4(__float_as_uint(m.x), __float_as_uint(m.y), __float_as_uint(m.z), 0u);
        out[1] = make_uint4(0u, __float_as_uint((float)tk), 0u, 0u);
        out[2] = make_uint4(__float_as_uint(s.x), __float_as_uint(s.y), __float_as_uint(s.z), 0u);
        out[3] = make_uint4(0u, 0u, 0u, 0u);
        out[4] = make_uint4(__float_as_uint(dv.x), __float_as_uint(dv.y), __float_as_uint(dv.z), __float_as_uint(dw));
        out[5] = make_uint4(0u, __float_as_uint(dc.x), __float_as_uint(dc.y), __float_as_uint(dc.z));
    }
    if constexpr (C) {
        // Warp-aggregate the counters, one atomic per counter per warp.
        unsigned long long v[11];
        const Cnt<true>& c = cnt;
        v[0] = c.rays; v[1] = c.paths; v[2] = c.steps; v[3] = c.b; v[4] = c.unk; v[5] = c.hits;
        v[6] = c.st[0]; v[7] = c.st[1]; v[8] = c.st[2]; v[9] = c.st[3]; v[10] = c.tb;
#pragma unroll
        for (int k = 0; k < 11; ++k) {
            unsigned long long x = v[k];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31u) == 0u && x) atomicAdd(A.counters + k, x);
        }
    }
}

template <uint32_t H, bool L, bool B>
void launch_variant(const TraceArgs& a, bool count, cudaStream_t s) {
    uint64_t threads = (uint64_t)a.n_tasks << a.lanes_log2;
    uint32_t blocks = (uint32_t)((threads + kBlock - 1) / kBlock);
    if (blocks == 0) return;
    if (count) trace_faces_kernel<H, L, B, true><<<blocks, kBlock, 0, s>>>(a);
    else trace_faces_kernel<H, L, B, false><<<blocks, kBlock, 0, s>>>(a);
}

template <uint32_t H>
void launch_hits(const TraceArgs& a, bool limited, bool budgeted, bool count, cudaStream_t s) {
    if (limited) {
        if (budgeted) launch_variant<H, true, true>(a, count, s);
        else launch_variant<H, true, false>(a, count, s);
    } else {
        if (budgeted) launch_variant<H, false, true>(a, count, s);
        else launch_variant<H, false, false>(a, count, s);
    }
}

}  // namespace

void launch_trace(const TraceArgs& a, uint32_t hits, bool limited, bool budgeted, bool count, cudaStream_t s) {
    if (hits <= 1) launch_hits<1>(a, limited, budgeted, count, s);
    else if (hits == 2) launch_hits<2>(a, limited, budgeted, count, s);
    else launch_hits<3>(a, limited, budgeted, count, s);
}

}  // namespace vgi

namespace vgi {
namespace {

// Companion light-tree records (see NodeLite): one thread per node.
__global__ void node_aux_kernel(const uint4* __restrict__ emitters, uint32_t first_node, uint32_t nodes, float4* __restrict__ aux) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const uint4 w0 = emitters[first_node + i * 4u], w1 = emitters[first_node + i * 4u + 1u], w3 = emitters[first_node + i * 4u + 3u];
    const V3 mn{__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
    const V3 mx{__uint_as_float(w1.x), __uint_as_float(w1.y), __uint_as_float(w1.z)};
    const V3 centre = (mn + mx) * 0.5f;
    const float radius = __fmul_rn(len3(mx - mn), 0.5f);
    aux[2u * i] = make_float4(centre.x, centre.y, centre.z, radius);
    reinterpret_cast<uint4*>(aux)[2u * i + 1u] = make_uint4(w0.w, w1.w, w3.x, w3.y);
}

}  // namespace

// ---- change footprints (voxel_trace.wgsl:94-202) ------------------------------
namespace {
constexpr int32_t kFootprintBias = 1073741824;

// The last task whose first thread is at most t (first threads ascend).
__device__ uint32_t footprint_task(const int4* fp, uint32_t t) {
    uint32_t lo = 0u, hi = (uint32_t)fp[0].x;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if ((uint32_t)fp[1u + mid * 3u + 2u].x <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// trace_footprints: one thread per tube of a square grid across a changed
// box's diagonal, per directional light. A tube clear on the sun side that
// lands on a surface below adds the reflected power through it to the task's
// flux (x 64) and its voxel to the landing box (biased by 2^30).
__global__ void __launch_bounds__(64) trace_footprints_kernel(const TraceArgs A, const int4* fp, uint32_t threads, uint32_t n_directional,
                                                              uint32_t* sums) {
    const uint32_t id = blockIdx.x * 64u + threadIdx.x;
    if ((uint32_t)fp[0].x == 0u || id >= threads) return;
    Cnt<false> cnt;
    const uint32_t e = footprint_task(fp, id);
    const int4 a = fp[1u + e * 3u], b = fp[1u + e * 3u + 1u], c = fp[1u + e * 3u + 2u];
    const uint32_t grid = (uint32_t)c.y;
    const uint32_t local = id - (uint32_t)c.x;
    if (local >= grid * grid) return;
    const V3 lo{(float)a.x, (float)a.y, (float)a.z};
    const V3 hi = add_s(V3{(float)b.x, (float)b.y, (float)b.z}, 1.0f);
    const V3 center = (lo + hi) * 0.5f;
    const float diagonal = len3(hi - lo);
    const float spacing = __fdiv_rn(diagonal, (float)grid);
    const float half = __fmul_rn(0.5f, diagonal);
    const float ox = __fsub_rn(__fmul_rn(__fadd_rn((float)(local % grid), 0.5f), spacing), half);
    const float oy = __fsub_rn(__fmul_rn(__fadd_rn((float)(local / grid), 0.5f), spacing), half);
    const V3 w{0.2126f, 0.7152f, 0.0722f};
    const uint32_t base = e * 8u;
    float flux = 0.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < n_directional; ++i) {
        const float4 Lp = __ldg(A.lights + i * 3u), Le = __ldg(A.lights + i * 3u + 1u), Lx = __ldg(A.lights + i * 3u + 2u);
        const V3 color{wmax(__fsub_rn(Le.x, Lx.y), 0.0f), wmax(__fsub_rn(Le.y, Lx.z), 0.0f), wmax(__fsub_rn(Le.z, Lx.w), 0.0f)};
        if (color.x == 0.0f && color.y == 0.0f && color.z == 0.0f) continue;
        const V3 direction = normalize3(V3{Lp.x, Lp.y, Lp.z});
        const V3 pick = fabsf(direction.y) > 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
        const V3 u = normalize3(cross3(direction, pick));
        const V3 v = cross3(direction, u);
        const V3 point = (center + u * ox) + v * oy;
        const V3 inverse{__fdiv_rn(1.0f, fabsf(direction.x) < 1e-8f ? 1e-8f : direction.x),
                         __fdiv_rn(1.0f, fabsf(direction.y) < 1e-8f ? 1e-8f : direction.y),
                         __fdiv_rn(1.0f, fabsf(direction.z) < 1e-8f ? 1e-8f : direction.z)};
        const V3 nearv = (lo - point) * inverse, farv = (hi - point) * inverse;
        const float enter = wmax(wmax(wmin(nearv.x, farv.x), wmin(nearv.y, farv.y)), wmin(nearv.z, farv.z));
        const float exit = wmin(wmin(wmax(nearv.x, farv.x), wmax(nearv.y, farv.y)), wmax(nearv.z, farv.z));
        if (enter > exit) continue;
        // Shadowed beyond the box either way: the change cannot matter.
        if (trace_domain(A, point + direction * __fadd_rn(exit, 0.01f), direction, A.max_distance, true, 2048u, cnt).status != 0u) continue;
        const V3 start = point + direction * __fsub_rn(enter, 0.01f);
        const Ray hit = trace_domain(A, start, -direction, A.max_distance, true, 2048u, cnt);
        if (hit.status != 1u || dot3(hit.normal, direction) <= 0.0f || len3(hit.position - start) < 0.02f) continue;
        const float4 d = __ldg(A.materials + hit.material * 4u);
        flux = __fadd_rn(flux, __fmul_rn(__fmul_rn(__fmul_rn(dot3(color, w), dot3(V3{d.x, d.y, d.z}, w)), spacing), spacing));
        const uint32_t px = (uint32_t)(hit.voxel.x + kFootprintBias), py = (uint32_t)(hit.voxel.y + kFootprintBias),
                       pz = (uint32_t)(hit.voxel.z + kFootprintBias);
        atomicMin(sums + base, px);
        atomicMin(sums + base + 1u, py);
        atomicMin(sums + base + 2u, pz);
        atomicMax(sums + base + 3u, px);
        atomicMax(sums + base + 4u, py);
        atomicMax(sums + base + 5u, pz);
    }
    if (flux > 0.0f) atomicAdd(sums + base + 6u, f2u(__fadd_rn(__fmul_rn(flux, 64.0f), 0.5f)));
}

// finish_footprints: each task's landing box becomes its reserved Light
// event (header union and its one bound); nothing landed: the empty bound stays.
__global__ void __launch_bounds__(64) finish_footprints_kernel(const int4* fp, const uint32_t* sums, uint4* events) {
    const uint32_t e = blockIdx.x * 64u + threadIdx.x;
    if (e >= (uint32_t)fp[0].x) return;
    const uint32_t base = e * 8u;
    const uint32_t x = sums[base];
    if (x == 0xffffffffu) return;
    const int mnx = (int)x - kFootprintBias, mny = (int)sums[base + 1u] - kFootprintBias, mnz = (int)sums[base + 2u] - kFootprintBias;
    const int mxx = (int)sums[base + 3u] - kFootprintBias, mxy = (int)sums[base + 4u] - kFootprintBias,
              mxz = (int)sums[base + 5u] - kFootprintBias;
    const float flux = __fdiv_rn((float)sums[base + 6u], 64.0f);
    const uint32_t header = (uint32_t)fp[1u + e * 3u].w, bound = (uint32_t)fp[1u + e * 3u + 1u].w;
    events[header] = make_uint4((uint32_t)mnx, (uint32_t)mny, (uint32_t)mnz, events[header].w);
    events[header + 1u] = make_uint4((uint32_t)mxx, (uint32_t)mxy, (uint32_t)mxz, events[header + 1u].w);
    events[bound] = make_uint4((uint32_t)mnx, (uint32_t)mny, (uint32_t)mnz, __float_as_uint(flux));
    events[bound + 1u] = make_uint4((uint32_t)mxx, (uint32_t)mxy, (uint32_t)mxz, 4u);
}
}  // namespace

// ---- headless discovery: primary rays into the NAADF geometry -----------------
namespace {
// A pixel's primary ray (the camera of vgi_camera): right = normalize(
// forward x up), up' = right x forward; sx = ((2 (x + 0.5)) / W - 1) *
// tan_half * (W / H), sy = (1 - (2 (y + 0.5)) / H) * tan_half; direction =
// normalize((forward + right sx) + up' sy). Host callers normalise forward.
__device__ V3 pixel_ray(const float* cam, uint32_t x, uint32_t y, uint32_t w, uint32_t h) {
    const V3 forward{cam[3], cam[4], cam[5]}, up{cam[6], cam[7], cam[8]};
    const V3 right = normalize3(cross3(forward, up));
    const V3 up2 = cross3(right, forward);
    const float fw = (float)w, fh = (float)h;
    const float sx = __fmul_rn(__fmul_rn(__fsub_rn(__fdiv_rn(__fmul_rn(2.0f, __fadd_rn((float)x, 0.5f)), fw), 1.0f), cam[9]), __fdiv_rn(fw, fh));
    const float sy = __fmul_rn(__fsub_rn(1.0f, __fdiv_rn(__fmul_rn(2.0f, __fadd_rn((float)y, 0.5f)), fh)), cam[9]);
    return normalize3((forward + right * sx) + up2 * sy);
}

__device__ __forceinline__ unsigned long long face_key64(I3 v, uint32_t face) {
    const unsigned long long m = (1ull << 20) - 1ull;
    return ((unsigned long long)((uint32_t)v.x & m)) | ((unsigned long long)((uint32_t)v.y & m) << 20) |
           ((unsigned long long)((uint32_t)v.z & m) << 40) | ((unsigned long long)face << 60);
}

// One thread per pixel: the first hit of the pixel's ray (visible geometry,
// 2048 steps) as (voxel xyz, face (6: none), material, status, distance
// bits, 0); each hit face enters the set once and the thread that inserted
// it appends the face (voxel xyz, face, material) to the list.
__global__ void __launch_bounds__(128) discover_kernel(const TraceArgs A, const float* cam, uint32_t w, uint32_t h, uint4* pixels,
                                                       unsigned long long* set, uint32_t set_mask, int4* faces, uint32_t* count,
                                                       uint32_t capacity, uint32_t* overflow) {
    const uint32_t id = blockIdx.x * 128u + threadIdx.x;
    if (id >= w * h) return;
    Cnt<false> cnt;
    const uint32_t x = id % w, y = id / w;
    const V3 eye{cam[0], cam[1], cam[2]};
    const V3 dir = pixel_ray(cam, x, y, w, h);
    const Ray r = trace_domain(A, eye, dir, A.max_distance, true, 2048u, cnt);
    const uint32_t face = r.status == 1u ? face_index_of(r.normal) : 6u;
    const float distance = r.status == 1u ? len3(r.position - eye) : 0.0f;
    pixels[(size_t)id * 2u] = make_uint4((uint32_t)r.voxel.x, (uint32_t)r.voxel.y, (uint32_t)r.voxel.z, face);
    pixels[(size_t)id * 2u + 1u] = make_uint4(r.material, r.status, __float_as_uint(distance), 0u);
    if (face > 5u) return;
    const unsigned long long key = face_key64(r.voxel, face);
    uint32_t s = (hash_voxel(r.voxel.x, r.voxel.y, r.voxel.z) ^ pcg(face + 1u)) & set_mask;
    // Bounded probing: the set holds at least twice the pixels.
#pragma unroll 1
    for (uint32_t probe = 0; probe <= set_mask; ++probe) {
        const unsigned long long old = atomicCAS(set + s, ~0ull, key);
        if (old == key) return;  // already listed
        if (old == ~0ull) {
            const uint32_t k = atomicAdd(count, 1u);
            // Past the capacity only the count grows: the host reports it.
            if (k < capacity) faces[k] = make_int4(r.voxel.x, r.voxel.y, r.voxel.z, (int)(face | (r.material << 8)));
            return;
        }
        s = (s + 1u) & set_mask;
    }
    atomicOr(overflow, 1u);
}
}  // namespace

void launch_discover(const TraceArgs& a, const float* cam, uint32_t w, uint32_t h, uint4* pixels, unsigned long long* set, uint32_t set_mask,
                     int4* faces, uint32_t* count, uint32_t capacity, uint32_t* overflow, cudaStream_t s) {
    const uint32_t n = w * h;
    if (n) discover_kernel<<<(n + 127) / 128, 128, 0, s>>>(a, cam, w, h, pixels, set, set_mask, faces, count, capacity, overflow);
}

// ---- far tier (voxel_view_pixels.wgsl:53-216) ------------------------------------
// Per-pixel lighting for faces small on screen, without face identity: each
// cell samples one of its pixels per frame, keeps a history reprojected by
// world position and traces a path when that history is short or one frame
// in `rate`. The raster depth and normal the shader reads become one primary
// ray per cell through the NAADF geometry (as in discovery).
namespace {

__device__ __forceinline__ float comp(V3 v, uint32_t a) { return a == 0u ? v.x : (a == 1u ? v.y : v.z); }
__device__ __forceinline__ void set_comp(V3& v, uint32_t a, float x) {
    if (a == 0u) v.x = x;
    else if (a == 1u) v.y = x;
    else v.z = x;
}

// voxel_traversal.wgsl:74-80: a coarse page's block stride (header w bits 28-30).
template <bool C>
__device__ int voxel_stride(const TraceArgs& A, I3 voxel, Cnt<C>& cnt) {
    const int rx = (int)floorf(__fdiv_rn((float)voxel.x, 16.0f)), ry = (int)floorf(__fdiv_rn((float)voxel.y, 16.0f)),
              rz = (int)floorf(__fdiv_rn((float)voxel.z, 16.0f));
    if (!in_bounds(A, rx, ry, rz)) return 1;
    const uint32_t index = lookup_region(A, rx, ry, rz, cnt);
    if (index == kNoIndex) return 1;
    return 1 << ((__ldg(A.headers + index).w >> 28u) & 7u);
}

// voxel_view_runtime.wgsl:26-30
__device__ __forceinline__ bool in_interest(const FarView& F, I3 voxel) {
    if (F.interest_min[3] == 0) return true;
    const int rx = (int)floorf(__fdiv_rn((float)voxel.x, 16.0f)), ry = (int)floorf(__fdiv_rn((float)voxel.y, 16.0f)),
              rz = (int)floorf(__fdiv_rn((float)voxel.z, 16.0f));
    return rx >= F.interest_min[0] && ry >= F.interest_min[1] && rz >= F.interest_min[2] && rx <= F.interest_max[0] &&
           ry <= F.interest_max[1] && rz <= F.interest_max[2];
}

// pixel_owned (voxel_view_pixels.wgsl:53-65), by distance from the camera.
template <bool C>
__device__ bool pixel_owned(const TraceArgs& A, const FarView& F, I3 voxel, uint32_t face, Cnt<C>& cnt) {
    const uint32_t grid = F.grid[3];
    if ((grid & 1u) == 0u || face >= 6u) return false;
    const uint32_t mode = (grid >> 1u) & 3u;
    const int s = mode == 2u ? voxel_stride(A, voxel, cnt) : 1;
    const I3 block{voxel.x & -s, voxel.y & -s, voxel.z & -s};
    const V3 ray = add_s(itof(block), __fmul_rn(0.5f, (float)s)) - V3{F.cam[0], F.cam[1], F.cam[2]};
    if (dot3(ray, V3{F.axis[0], F.axis[1], F.axis[2]}) <= 0.0f) return false;
    const float side = __fdiv_rn(__fmul_rn((float)s, F.axis[3]), len3(ray));
    if (mode == 0u) return side < F.tune[0];
    return __fmul_rn(__fmul_rn(side, side), fabsf(dot3(face_normal(face), normalize3(ray)))) < F.tune[0];
}

// f32 -> f16 bits, round to nearest even (pack2x16float's conversion).
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    return (uint32_t)__half_as_ushort(__float2half_rn(a)) | ((uint32_t)__half_as_ushort(__float2half_rn(b)) << 16u);
}

struct FarCell {
    V3 mean;
    float count;
    V3 surface;
    uint32_t face;
    uint32_t sequence;
};
__device__ __forceinline__ FarCell load_cell(const uint4* cells, uint32_t i) {
    const uint4 a = cells[i * 3u], b = cells[i * 3u + 1u], c = cells[i * 3u + 2u];
    return FarCell{V3{__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z)}, __uint_as_float(a.w),
                   V3{__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z)}, b.w, c.x};
}
__device__ __forceinline__ void store_cell(uint4* cells, uint32_t i, const FarCell& v) {
    cells[i * 3u] = make_uint4(__float_as_uint(v.mean.x), __float_as_uint(v.mean.y), __float_as_uint(v.mean.z), __float_as_uint(v.count));
    cells[i * 3u + 1u] = make_uint4(__float_as_uint(v.surface.x), __float_as_uint(v.surface.y), __float_as_uint(v.surface.z), v.face);
    cells[i * 3u + 2u] = make_uint4(v.sequence, 0u, 0u, 0u);
}

// write_output (voxel_view_pixels.wgsl:76-81) with custom_direct (67-74).
template <class T>
__device__ void far_write(const FarView& F, T& tracer, uint4* output, uint32_t index, const FarCell& v) {
    const uint32_t axis = (v.face & 7u) / 2u;
    V3 shown = v.mean;
    if (F.custom) {
        V3 value, custom;
        tracer.template direct_at<true>(v.surface, face_normal(v.face & 7u), value, custom);
        shown = shown + custom;
    }
    output[4u + index] = make_uint4(pack2(shown.x, shown.y), pack2(shown.z, v.count), v.face, __float_as_uint(comp(v.surface, axis)));
}

// The camera's screen position of a world point: NDC x, y (the previous
// clip matrix's projection), false behind the camera.
__device__ bool project(const float* cam, uint32_t w, uint32_t h, V3 point, float& nx, float& ny) {
    const V3 forward{cam[3], cam[4], cam[5]}, up{cam[6], cam[7], cam[8]};
    const V3 right = normalize3(cross3(forward, up));
    const V3 up2 = cross3(right, forward);
    const V3 v = point - V3{cam[0], cam[1], cam[2]};
    const float depth = dot3(v, forward);
    if (depth <= 0.0f) return false;
    const float scale = __fmul_rn(depth, cam[9]);
    nx = __fdiv_rn(dot3(v, right), __fmul_rn(scale, __fdiv_rn((float)w, (float)h)));
    ny = __fdiv_rn(dot3(v, up2), scale);
    return true;
}

// previous_cell (voxel_view_pixels.wgsl:83-127).
template <bool C>
__device__ void previous_cell(const TraceArgs& A, const FarView& F, const uint4* previous, V3 surface, uint32_t face, I3 voxel, V3& mean,
                              float& count, uint32_t& sequence, Cnt<C>& cnt) {
    mean = V3{0.0f, 0.0f, 0.0f};
    count = 0.0f;
    sequence = 0u;
    const uint32_t prev_stamp = __float_as_uint(F.tune[3]);
    if (prev_stamp == 0xffffffffu) return;
    float nx, ny;
    if (!project(F.prev, F.width, F.height, surface, nx, ny)) return;
    const uint32_t size = F.grid[2];
    const V3 normal = face_normal(face);
    const float ux = __fadd_rn(__fmul_rn(nx, 0.5f), 0.5f), uy = __fadd_rn(__fmul_rn(ny, -0.5f), 0.5f);
    const float px = __fsub_rn(__fdiv_rn(__fmul_rn(ux, (float)F.width), (float)size), 0.5f);
    const float py = __fsub_rn(__fdiv_rn(__fmul_rn(uy, (float)F.height), (float)size), 0.5f);
    // Far off-screen points stay far off the grid (and convert safely).
    const float flx = fminf(fmaxf(floorf(px), -1048576.0f), 1048576.0f), fly = fminf(fmaxf(floorf(py), -1048576.0f), 1048576.0f);
    const int bx = (int)flx, by = (int)fly;
    const float fx = __fsub_rn(px, flx), fy = __fsub_rn(py, fly);
    const float reach = __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, (float)size), len3(surface - V3{F.cam[0], F.cam[1], F.cam[2]})), F.axis[3]);
    const float tolerance = __fadd_rn(__fmul_rn(4.0f, (float)voxel_stride(A, voxel, cnt)), 0.01f);
    const uint32_t expected = face | ((prev_stamp & 0x1fffffffu) << 3u);
    float weight = 0.0f, samples = 0.0f, best = 0.0f;
    V3 sum{0.0f, 0.0f, 0.0f};
    for (int y = 0; y <= 1; ++y) {
        for (int x = 0; x <= 1; ++x) {
            const int qx = bx + x, qy = by + y;
            if (qx < 0 || qy < 0 || qx >= (int)F.grid[0] || qy >= (int)F.grid[1]) continue;
            const FarCell old = load_cell(previous, (uint32_t)qy * F.grid[0] + (uint32_t)qx);
            if (old.face != expected || old.count == 0.0f) continue;
            const V3 delta = old.surface - surface;
            if (fabsf(dot3(delta, normal)) > tolerance || dot3(delta, delta) > __fmul_rn(reach, reach)) continue;
            const float w = __fadd_rn(__fmul_rn(x == 1 ? fx : __fsub_rn(1.0f, fx), y == 1 ? fy : __fsub_rn(1.0f, fy)), 1e-4f);
            sum = sum + old.mean * w;
            samples = __fadd_rn(samples, __fmul_rn(old.count, w));
            weight = __fadd_rn(weight, w);
            if (w > best) {
                best = w;
                sequence = old.sequence;
            }
        }
    }
    if (weight > 0.0f) {
        mean = sum / weight;
        count = __fdiv_rn(samples, weight);
    }
}

// The handoff's receiver lookup: block_receiver (voxel_view_discovery.wgsl:
// 26-35) then previous_owner (voxel_view_runtime.wgsl:110-120).
template <bool C>
__device__ uint32_t far_owner(const TraceArgs& A, const FarView& F, I3 voxel, uint32_t face, Cnt<C>& cnt) {
    if (F.n_receivers == 0u || F.receiver_hash == nullptr) return kNoIndex;
    const V3 normal = face_normal(face);
    I3 key = voxel;
    V3 surface = add_s(itof(voxel), 0.5f) + normal * 0.5f;
    const int s = voxel_stride(A, voxel, cnt);
    if (s != 1) {
        key = I3{voxel.x & -s, voxel.y & -s, voxel.z & -s};
        surface = itof(key) + add_s(normal * 0.5f, 0.5f) * (float)s;
    }
    uint32_t slot = (hash_voxel(key.x, key.y, key.z) ^ pcg(face + 1u)) & F.hash_mask;
#pragma unroll 1
    for (uint32_t step = 0; step < 64u; ++step) {
        const uint32_t value = F.receiver_hash[slot];
        if (value == 0u) return kNoIndex;
        if (value <= F.n_receivers) {
            const uint4 r0 = F.receivers[(value - 1u) * 2u], r1 = F.receivers[(value - 1u) * 2u + 1u];
            if (r0.w == face && (int)r1.x == key.x && (int)r1.y == key.y && (int)r1.z == key.z && __uint_as_float(r0.x) == surface.x &&
                __uint_as_float(r0.y) == surface.y && __uint_as_float(r0.z) == surface.z)
                return value - 1u;
        }
        slot = (slot + 1u) & F.hash_mask;
    }
    return kNoIndex;
}

__device__ __forceinline__ void load_smat(const TraceArgs& A, float4* smat) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        float4 d = __ldg(A.materials + i * 4), e = __ldg(A.materials + i * 4 + 2), x = __ldg(A.materials + i * 4 + 3);
        smat[i * 2] = make_float4(d.x, d.y, d.z, x.y);
        smat[i * 2 + 1] = make_float4(e.x, e.y, e.z, 0.0f);
    }
    __syncthreads();
}

constexpr uint32_t kFarHits = 3u;  // DIFFUSE_HITS's default: the far pipelines do not override it

// classify_pixels (voxel_view_pixels.wgsl:129-192).
template <bool LIMITED>
__global__ void __launch_bounds__(128) far_classify_kernel(const TraceArgs A, const FarView F, const uint4* __restrict__ previous,
                                                           uint4* __restrict__ current, uint4* __restrict__ output, uint32_t* __restrict__ queue,
                                                           uint32_t* __restrict__ stats) {
    __shared__ float4 smat[512];
    load_smat(A, smat);
    Cnt<false> cnt;
    Tracer<kFarHits, LIMITED, true, false> T{A, smat, cnt};
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stamp = F.frame & 0x1fffffffu;
    if (id == 0u) {
        output[0] = make_uint4(__float_as_uint(F.cam[0]), __float_as_uint(F.cam[1]), __float_as_uint(F.cam[2]), 0u);
        output[1] = make_uint4(__float_as_uint(F.axis[0]), __float_as_uint(F.axis[1]), __float_as_uint(F.axis[2]), __float_as_uint(F.axis[3]));
        output[2] = make_uint4(F.grid[0], F.grid[1], F.grid[2], F.grid[3]);
        output[3] = make_uint4(0u, 0u, __float_as_uint(F.tune[0]), stamp);
    }
    if (id >= F.grid[0] * F.grid[1]) return;
    const uint32_t size = F.grid[2];
    const uint32_t cx = id % F.grid[0], cy = id / F.grid[0];
    // One pixel of the cell per frame, cycling through all of them.
    const uint32_t k = (F.frame * 5u + (cx ^ cy)) % (size * size);
    const uint32_t px = cx * size + k % size, py = cy * size + k / size;
    if (px >= F.width || py >= F.height) return;
    const V3 eye{F.cam[0], F.cam[1], F.cam[2]};
    const V3 dir = pixel_ray(F.cam, px, py, F.width, F.height);
    const Ray hit = trace_domain(A, eye, dir, A.max_distance, true, 2048u, cnt);
    if (hit.status != 1u) return;  // nothing drawn at this pixel
    V3 surface = hit.position;
    if (((F.grid[3] >> 1u) & 3u) == 0u && F.axis[3] > __fmul_rn(__fmul_rn(1.05f, F.tune[0]), len3(surface - eye))) return;
    const uint32_t face = face_index_of(hit.normal);
    if (face >= 6u) return;
    const V3 normal = face_normal(face);
    set_comp(surface, face / 2u, rintf(comp(surface, face / 2u)));
    const V3 inner = surface - normal * 0.01f;
    const I3 voxel{(int)floorf(inner.x), (int)floorf(inner.y), (int)floorf(inner.z)};
    if (!in_interest(F, voxel) || !pixel_owned(A, F, voxel, face, cnt)) return;
    atomicAdd(stats + kFarOwned, 1u);
    V3 mean;
    float count;
    uint32_t sequence;
    previous_cell(A, F, previous, surface, face, voxel, mean, count, sequence, cnt);
    if (count > 0.0f) {
        atomicAdd(stats + kFarReprojected, 1u);
    } else {
        // Handoff: a face entering the far band starts from its view receiver's history.
        const uint32_t owner = far_owner(A, F, voxel, face, cnt);
        if (owner != kNoIndex && __uint_as_float(F.estimates[owner * 4u].w) > 0.0f) {
            const uint4 e = F.estimates[owner * 4u];
            mean = V3{__uint_as_float(e.x), __uint_as_float(e.y), __uint_as_float(e.z)};
            count = __uint_as_float(e.w);
            sequence = F.estimates[owner * 4u + 3u].x;
            atomicAdd(stats + kFarSeeded, 1u);
        }
    }
    const float capped = wmin(count, F.tune[1]);
    atomicAdd(stats + kFarHistory, (uint32_t)capped);
    const FarCell value{mean, capped, surface, face | (stamp << 3u), sequence};
    store_cell(current, id, value);
    const uint32_t rate = max((uint32_t)F.tune[2], 1u);
    if (capped < 4.0f || (id + F.frame) % rate == 0u) {
        const uint32_t slot = atomicAdd(queue, 1u);
        queue[1u + slot] = id;
    } else {
        far_write(F, T, output, id, value);
    }
}

// trace_pixel_queue (voxel_view_pixels.wgsl:199-216), grid-stride over the
// dense queue.
template <bool LIMITED>
__global__ void __launch_bounds__(128) far_trace_kernel(const TraceArgs A, const FarView F, const uint32_t* __restrict__ queue,
                                                        uint4* __restrict__ current, uint4* __restrict__ output, uint32_t* __restrict__ stats) {
    __shared__ float4 smat[512];
    load_smat(A, smat);
    Cnt<false> cnt;
    Tracer<kFarHits, LIMITED, true, false> T{A, smat, cnt};
    const uint32_t n = queue[0];
#pragma unroll 1
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t index = queue[1u + i];
        FarCell cell = load_cell(current, index);
        atomicAdd(stats + kFarTraced, 1u);
        const uint32_t stream = pcg(index * 9781u + 0x9e3779b9u);
        const V3 normal = face_normal(cell.face & 7u);
        // trace_receiver (voxel_path.wgsl:504-520)
        const V3 direction = hemisphere(normal, sample_1d(stream, cell.sequence, 0u), sample_1d(stream, cell.sequence, 1u));
        V3 value = T.sample_emitter(cell.surface, normal, stream, cell.sequence, 0u);
        bool unknown = false;
        if (dot3(normal, direction) > 0.0f) value = value + T.trace_path(cell.surface + normal * 0.001f, direction, normal, stream, cell.sequence, unknown);
        cell.sequence += 1u;
        if (!unknown) {
            cell.count = wmin(__fadd_rn(cell.count, 1.0f), F.tune[1]);
            const float t = __fdiv_rn(1.0f, cell.count);
            cell.mean = cell.mean * __fsub_rn(1.0f, t) + value * t;
        }
        store_cell(current, index, cell);
        far_write(F, T, output, index, cell);
    }
}

// The view receivers' owner hash (receiver_hash, voxel_view_runtime.wgsl:
// 96-98): receiver + 1 per slot, linear probing.
__global__ void receiver_hash_kernel(const uint4* receivers, uint32_t n, uint32_t* hash, uint32_t mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 r0 = receivers[i * 2u], r1 = receivers[i * 2u + 1u];
    uint32_t slot = (hash_voxel((int)r1.x, (int)r1.y, (int)r1.z) ^ pcg(r0.w + 1u)) & mask;
#pragma unroll 1
    for (uint32_t step = 0; step <= mask; ++step) {
        if (atomicCAS(hash + slot, 0u, i + 1u) == 0u) return;
        slot = (slot + 1u) & mask;
    }
}

}  // namespace

void launch_far(const TraceArgs& a, const FarView& f, const uint4* previous, uint4* current, uint4* output, uint32_t* queue, uint32_t* stats,
                bool limited, cudaStream_t s) {
    const uint32_t cells = f.grid[0] * f.grid[1];
    if (cells == 0) return;
    const uint32_t blocks = (cells + 127) / 128;
    // The trace pass strides over at most `cells` queued cells.
    const uint32_t trace_blocks = std::min<uint32_t>(blocks, 148u * 8u);
    if (limited) {
        far_classify_kernel<true><<<blocks, 128, 0, s>>>(a, f, previous, current, output, queue, stats);
        far_trace_kernel<true><<<trace_blocks, 128, 0, s>>>(a, f, queue, current, output, stats);
    } else {
        far_classify_kernel<false><<<blocks, 128, 0, s>>>(a, f, previous, current, output, queue, stats);
        far_trace_kernel<false><<<trace_blocks, 128, 0, s>>>(a, f, queue, current, output, stats);
    }
}

void launch_receiver_hash(const uint4* receivers, uint32_t n, uint32_t* hash, uint32_t mask, cudaStream_t s) {
    if (n) receiver_hash_kernel<<<(n + 127) / 128, 128, 0, s>>>(receivers, n, hash, mask);
}

// ---- reconstruction and presentation --------------------------------------------
namespace {

__device__ __forceinline__ float luminance(V3 c) { return dot3(c, V3{0.2126f, 0.7152f, 0.0722f}); }
__device__ __forceinline__ V3 v3w(uint4 w) { return V3{__uint_as_float(w.x), __uint_as_float(w.y), __uint_as_float(w.z)}; }

// mean_variance (voxel_view_runtime.wgsl:383-394): the mean's variance with
// a 64-sample prior and the unseen-light floor `reference / n`.
__device__ float mean_variance(uint4 mean_w, uint4 moment_w, float reference) {
    const V3 mean = v3w(mean_w), moment = v3w(moment_w);
    const float n = wmax(__uint_as_float(mean_w.w), 1.0f);
    const float m = luminance(mean);
    const V3 channel{wmax(__fsub_rn(moment.x, __fmul_rn(mean.x, mean.x)), 0.0f), wmax(__fsub_rn(moment.y, __fmul_rn(mean.y, mean.y)), 0.0f),
                     wmax(__fsub_rn(moment.z, __fmul_rn(mean.z, mean.z)), 0.0f)};
    const float deviation = luminance(V3{__fsqrt_rn(channel.x), __fsqrt_rn(channel.y), __fsqrt_rn(channel.z)});
    const float prior = __fmul_rn(m, m);
    const float rest = wmax(__fsub_rn(n, 1.0f), 0.0f);
    const float shrunk = __fdiv_rn(__fadd_rn(__fmul_rn(__fmul_rn(deviation, deviation), rest), __fmul_rn(prior, 64.0f)), __fadd_rn(rest, 64.0f));
    const float unseen = __fdiv_rn(reference, n);
    return __fadd_rn(__fdiv_rn(shrunk, n), __fmul_rn(unseen, unseen));
}

// coplanar_donor (voxel_view_runtime.wgsl:396-404); every caller-given
// receiver is its own owner.
__device__ bool coplanar_donor(const ViewDisplay& D, uint4 r0, uint4 r1, V3 normal, uint32_t candidate) {
    const uint4 d0 = D.receivers[candidate * 2u];
    if (d0.w != r0.w) return false;
    const V3 delta = v3w(d0) - v3w(r0);
    // receiver_stride: twice the surface's offset from the voxel along the face's next axis.
    const uint32_t u = (r0.w / 2u + 1u) % 3u;
    const float su = u == 0u ? __uint_as_float(r0.x) : (u == 1u ? __uint_as_float(r0.y) : __uint_as_float(r0.z));
    const int vu = u == 0u ? (int)r1.x : (u == 1u ? (int)r1.y : (int)r1.z);
    const float reach = __fmul_rn(16.0f, __fmul_rn(2.0f, __fsub_rn(su, (float)vu)));
    return fabsf(dot3(delta, normal)) <= 0.05f && dot3(delta, delta) <= __fmul_rn(reach, reach);
}

// reconstruct_view (voxel_view_runtime.wgsl:406-474): inverse-variance
// weighting of coplanar donors in the screen tiles around the receiver's,
// with the centre's bias bound, then a temporal blend of the shown value.
// One warp per receiver: lane l takes the window's tiles l, l + 32, ... in
// row-major order (donors of a tile in receiver order) and keeps its own
// partial sums; lane 0 adds the centre's term and then the lanes' partials
// in lane order, so the sums have one fixed order.
__device__ __forceinline__ float shfl_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = wmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__global__ void __launch_bounds__(128) reconstruct_kernel(const ViewDisplay D) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= D.n) return;  // whole warps
    const uint4 r0 = D.receivers[i * 2u], r1 = D.receivers[i * 2u + 1u];
    const uint32_t tile = D.tile_of[i];
    if (r0.w >= 6u || tile >= D.tiles_x * D.tiles_y) return;
    const uint4 c_mean = D.estimates[i * 4u], c_moment = D.estimates[i * 4u + 1u];
    const V3 normal = face_normal(r0.w);
    const int tx = (int)(tile % D.tiles_x), ty = (int)(tile / D.tiles_x);
    const float center_luminance = luminance(v3w(c_mean));
    // The brightest sampled coplanar donor in the 3 x 3 tiles (a maximum: any order).
    float reference = center_luminance;
    for (uint32_t k = lane; k < 9u; k += 32u) {
        const int qx = tx + (int)(k % 3u) - 1, qy = ty + (int)(k / 3u) - 1;
        if (qx < 0 || qy < 0 || qx >= (int)D.tiles_x || qy >= (int)D.tiles_y) continue;
        const uint32_t t = (uint32_t)qy * D.tiles_x + (uint32_t)qx;
        for (uint32_t j = D.tile_start[t]; j < D.tile_start[t + 1u]; ++j) {
            const uint32_t candidate = D.tile_items[j];
            if (candidate == i || !coplanar_donor(D, r0, r1, normal, candidate)) continue;
            const uint4 value = D.estimates[candidate * 4u];
            if (__uint_as_float(value.w) > 0.0f) reference = wmax(reference, luminance(v3w(value)));
        }
    }
    reference = shfl_max(reference);
    const float center_variance = mean_variance(c_mean, c_moment, reference);
    const float tolerance = __fmul_rn(D.display[0], center_luminance);
    const float tol2 = __fmul_rn(tolerance, tolerance);
    const float deficit = __fdiv_rn(center_variance, wmax(tol2, 1e-12f));
    const int radius = (int)wclamp(ceilf(__fmul_rn(__fsqrt_rn(__fdiv_rn(deficit, 3.14159f)), 0.5f)), 1.0f, 4.0f);
    const bool unsampled = __uint_as_float(c_mean.w) <= 0.0f;
    V3 part{0.0f, 0.0f, 0.0f};
    float part_w = 0.0f;
    const bool gather = (unsampled || center_variance > tol2) && D.display[1] > 0.0f;
    if (gather) {
        const uint32_t side = 2u * (uint32_t)radius + 1u;
        for (uint32_t k = lane; k < side * side; k += 32u) {
            const int qx = tx + (int)(k % side) - radius, qy = ty + (int)(k / side) - radius;
            if (qx < 0 || qy < 0 || qx >= (int)D.tiles_x || qy >= (int)D.tiles_y) continue;
            const uint32_t t = (uint32_t)qy * D.tiles_x + (uint32_t)qx;
            for (uint32_t j = D.tile_start[t]; j < D.tile_start[t + 1u]; ++j) {
                const uint32_t candidate = D.tile_items[j];
                if (candidate == i || !coplanar_donor(D, r0, r1, normal, candidate)) continue;
                const uint4 value = D.estimates[candidate * 4u];
                if (__uint_as_float(value.w) <= 0.0f) continue;
                const float variance = mean_variance(value, D.estimates[candidate * 4u + 1u], reference);
                float bias2 = 0.0f;
                if (!unsampled) {
                    const float difference = __fsub_rn(luminance(v3w(value)), center_luminance);
                    bias2 = wmax(__fsub_rn(__fsub_rn(__fmul_rn(difference, difference), variance), center_variance), 0.0f);
                }
                const float w = __fdiv_rn(1.0f, wmax(__fadd_rn(variance, bias2), 1e-12f));
                part = part + v3w(value) * w;
                part_w = __fadd_rn(part_w, w);
            }
        }
    }
    V3 sum{0.0f, 0.0f, 0.0f};
    float weight = 0.0f;
    if (!unsampled) {
        const float w = __fdiv_rn(1.0f, wmax(center_variance, 1e-12f));
        sum = v3w(c_mean) * w;
        weight = w;
    }
    if (gather) {
        for (uint32_t l = 0; l < 32u; ++l) {
            const V3 p{__shfl_sync(0xffffffffu, part.x, l), __shfl_sync(0xffffffffu, part.y, l), __shfl_sync(0xffffffffu, part.z, l)};
            const float pw = __shfl_sync(0xffffffffu, part_w, l);
            sum = sum + p;
            weight = __fadd_rn(weight, pw);
        }
    }
    if (lane != 0u || weight <= 0.0f) return;
    const uint4 c_shown = D.estimates[i * 4u + 2u];
    const float keep = unsampled ? 0.0f : __fsub_rn(1.0f, D.display[1]);
    const V3 desired = (sum / weight) * __fsub_rn(1.0f, keep) + v3w(c_mean) * keep;
    const float blend = __uint_as_float(c_shown.w) > 0.0f ? D.display[2] : 1.0f;
    const V3 shown = v3w(c_shown) * __fsub_rn(1.0f, blend) + desired * blend;
    D.estimates[i * 4u + 2u] = make_uint4(__float_as_uint(shown.x), __float_as_uint(shown.y), __float_as_uint(shown.z), __float_as_uint(1.0f));
}

// publish_view (voxel_view_runtime.wgsl:476-521): a FarPixel per receiver
// (surface, face, irradiance, evidence, sky corner words) and the counters.
template <bool LIMITED, bool BUDGETED>
__global__ void __launch_bounds__(128) publish_kernel(const TraceArgs A, const ViewDisplay D) {
    __shared__ float4 smat[512];
    load_smat(A, smat);
    Cnt<false> cnt;
    Tracer<1u, LIMITED, BUDGETED, false> T{A, smat, cnt};
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const uint4 r0 = D.receivers[i * 2u];
    uint4 out0 = make_uint4(0u, 0u, 0u, 0xffffffffu), out1 = make_uint4(0u, 0u, 0u, 0u), out2 = make_uint4(0u, 0u, 0u, 0u);
    if (r0.w < 6u) {
        const uint4 mean = D.estimates[i * 4u], shown = D.estimates[i * 4u + 2u], identity = D.estimates[i * 4u + 3u];
        V3 irradiance = v3w(shown);
        if (D.custom) {
            V3 value, custom;
            T.template direct_at<true>(v3w(r0), face_normal(r0.w), value, custom);
            irradiance = irradiance + custom;
        }
        const float count = __uint_as_float(mean.w);
        const bool lit = __uint_as_float(shown.w) > 0.0f || irradiance.x > 0.0f || irradiance.y > 0.0f || irradiance.z > 0.0f;
        const float evidence = lit ? wmax(count, 0.001f) : 0.0f;
        uint32_t sky[4];
        for (uint32_t corner = 0; corner < 4u; ++corner) {
            const uint32_t byte = (identity.z >> (corner * 8u)) & 255u;
            sky[corner] = (byte & 15u) | ((byte & 128u) << 24u);
        }
        out0 = r0;
        out1 = make_uint4(__float_as_uint(irradiance.x), __float_as_uint(irradiance.y), __float_as_uint(irradiance.z), __float_as_uint(evidence));
        out2 = make_uint4(sky[0], sky[1], sky[2], sky[3]);
        atomicAdd(D.stats + 0, (uint32_t)count);
        atomicMax(D.stats + 1, (uint32_t)count);
        if (count == 0.0f) atomicAdd(D.stats + 2, 1u);
        if (evidence > 0.0f) atomicAdd(D.stats + 3, 1u);
        if (D.conts[i * 8u + 4u].w == 1u) atomicAdd(D.stats + 4, 1u);
    }
    D.published[i * 3u] = out0;
    D.published[i * 3u + 1u] = out1;
    D.published[i * 3u + 2u] = out2;
}

// display_face (voxel_gi_presentation.wesl:363-371): a published face's
// irradiance and evidence (at most 1), zero where none is published.
__device__ float4 display_face(const ViewDisplay& D, I3 voxel, uint32_t face, int s) {
    const V3 n = face_normal(face);
    const V3 surface = itof(voxel) + add_s(n * 0.5f, 0.5f) * (float)s;
    uint32_t slot = (hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u)) & D.hash_mask;
#pragma unroll 1
    for (uint32_t step = 0; step < 64u; ++step) {
        const uint32_t entry = D.receiver_hash[slot];
        if (entry == 0u) break;
        if (entry <= D.n) {
            const uint4 p0 = D.published[(entry - 1u) * 3u];
            if (p0.w == face && __uint_as_float(p0.x) == surface.x && __uint_as_float(p0.y) == surface.y && __uint_as_float(p0.z) == surface.z) {
                const uint4 p1 = D.published[(entry - 1u) * 3u + 1u];
                return make_float4(__uint_as_float(p1.x), __uint_as_float(p1.y), __uint_as_float(p1.z), wmin(__uint_as_float(p1.w), 1.0f));
            }
        }
        slot = (slot + 1u) & D.hash_mask;
    }
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// corner_value (voxel_gi_presentation.wesl:353-361): the connected
// coplanar faces' evidence-weighted mean at a shared corner.
__device__ V3 corner_value(float4 c, float4 eu, float4 ev, float4 diag) {
    float sx = __fadd_rn(__fadd_rn(__fmul_rn(c.x, c.w), __fmul_rn(eu.x, eu.w)), __fmul_rn(ev.x, ev.w));
    float sy = __fadd_rn(__fadd_rn(__fmul_rn(c.y, c.w), __fmul_rn(eu.y, eu.w)), __fmul_rn(ev.y, ev.w));
    float sz = __fadd_rn(__fadd_rn(__fmul_rn(c.z, c.w), __fmul_rn(eu.z, eu.w)), __fmul_rn(ev.z, ev.w));
    float sw = __fadd_rn(__fadd_rn(c.w, eu.w), ev.w);
    if (eu.w > 0.0f || ev.w > 0.0f) {
        sx = __fadd_rn(sx, __fmul_rn(diag.x, diag.w));
        sy = __fadd_rn(sy, __fmul_rn(diag.y, diag.w));
        sz = __fadd_rn(sz, __fmul_rn(diag.z, diag.w));
        sw = __fadd_rn(sw, diag.w);
    }
    const float d = wmax(sw, 0.000001f);
    return V3{__fdiv_rn(sx, d), __fdiv_rn(sy, d), __fdiv_rn(sz, d)};
}
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float t) { return a * __fsub_rn(1.0f, t) + b * t; }

// corner_irradiance (voxel_gi_presentation.wesl:377-412) at each pixel's
// first hit: rgb and the centre face's evidence.
__global__ void __launch_bounds__(128) present_kernel(const TraceArgs A, const ViewDisplay D, const float* cam, uint32_t w, uint32_t h,
                                                      bool corners, float4* image) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= w * h) return;
    Cnt<false> cnt;
    const V3 eye{cam[0], cam[1], cam[2]};
    const Ray hit = trace_domain(A, eye, pixel_ray(cam, id % w, id / w, w, h), A.max_distance, true, 2048u, cnt);
    if (hit.status != 1u) {
        image[id] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const V3 position = hit.position, normal = hit.normal;
    const V3 inner = position - normal * 0.01f;
    const I3 cell{(int)floorf(inner.x), (int)floorf(inner.y), (int)floorf(inner.z)};
    const int s = voxel_stride(A, cell, cnt);
    const I3 voxel{cell.x & -s, cell.y & -s, cell.z & -s};
    uint32_t face = 0u;
    I3 u{0, s, 0}, v{0, 0, s};
    if (fabsf(normal.y) > 0.5f) {
        face = 2u;
        u = I3{s, 0, 0};
    } else if (fabsf(normal.z) > 0.5f) {
        face = 4u;
        u = I3{s, 0, 0};
        v = I3{0, s, 0};
    }
    const uint32_t axis = face / 2u;
    face += (axis == 0u ? normal.x : (axis == 1u ? normal.y : normal.z)) < 0.0f ? 1u : 0u;
    const float4 center = display_face(D, voxel, face, s);
    if (!corners) {
        image[id] = center;
        return;
    }
    auto at = [&](int du, int dv) {
        return display_face(D, I3{voxel.x + du * u.x + dv * v.x, voxel.y + du * u.y + dv * v.y, voxel.z + du * u.z + dv * v.z}, face, s);
    };
    const float4 left = at(-1, 0), right = at(1, 0), bottom = at(0, -1), top = at(0, 1);
    const V3 c00 = corner_value(center, left, bottom, at(-1, -1));
    const V3 c10 = corner_value(center, right, bottom, at(1, -1));
    const V3 c01 = corner_value(center, left, top, at(-1, 1));
    const V3 c11 = corner_value(center, right, top, at(1, 1));
    const V3 local = (position - itof(voxel)) / (float)(s * s);
    const float ux = wclamp(dot3(local, itof(u)), 0.0f, 1.0f), uy = wclamp(dot3(local, itof(v)), 0.0f, 1.0f);
    const V3 rgb = mix3(mix3(c00, c10, ux), mix3(c01, c11, ux), uy);
    image[id] = make_float4(rgb.x, rgb.y, rgb.z, center.w);
}

}  // namespace

void launch_reconstruct(const TraceArgs& a, const ViewDisplay& d, bool limited, bool budgeted, cudaStream_t s) {
    if (d.n == 0) return;
    const uint32_t blocks = (d.n + 127) / 128;
    reconstruct_kernel<<<(d.n + 3) / 4, 128, 0, s>>>(d);  // a warp per receiver
    if (limited) {
        if (budgeted) publish_kernel<true, true><<<blocks, 128, 0, s>>>(a, d);
        else publish_kernel<true, false><<<blocks, 128, 0, s>>>(a, d);
    } else {
        if (budgeted) publish_kernel<false, true><<<blocks, 128, 0, s>>>(a, d);
        else publish_kernel<false, false><<<blocks, 128, 0, s>>>(a, d);
    }
}

void launch_present(const TraceArgs& a, const ViewDisplay& d, const float* cam, uint32_t w, uint32_t h, bool corners, float4* image,
                    cudaStream_t s) {
    const uint32_t n = w * h;
    if (n) present_kernel<<<(n + 127) / 128, 128, 0, s>>>(a, d, cam, w, h, corners, image);
}

void launch_footprints(const TraceArgs& a, const int4* fp, uint32_t n_tasks, uint32_t threads, uint32_t n_directional, uint32_t* sums,
                       uint4* events, cudaStream_t s) {
    if (n_tasks == 0) return;
    if (threads) trace_footprints_kernel<<<(threads + 63) / 64, 64, 0, s>>>(a, fp, threads, n_directional, sums);
    finish_footprints_kernel<<<(n_tasks + 63) / 64, 64, 0, s>>>(fp, sums, events);
}

void launch_node_aux(const uint4* emitters, uint32_t first_node, uint32_t nodes, float4* aux, cudaStream_t s) {
    if (nodes == 0) return;
    node_aux_kernel<<<(nodes + 255) / 256, 256, 0, s>>>(emitters, first_node, nodes, aux);
}

cudaError_t init_trace_constants() {
    // The reference's running `scale /= f32(base)` (voxel_path.wgsl:195),
    // for as many digits as an index up to 2^24 has in each base.
    static const uint32_t primes[12] = {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u};
    float table[12][25] = {};
    for (int d = 0; d < 12; ++d) {
        uint32_t digits = 0;
        for (uint32_t m = 0x1000000u; m != 0u; m /= primes[d]) ++digits;
        float scale = 1.0f;
        for (uint32_t k = 0; k < digits && k < 25; ++k) {
            scale = scale / (float)primes[d];
            table[d][k] = scale;
        }
    }
    return cudaMemcpyToSymbol(c_halton_scale, table, sizeof(table));
}

}  // namespace vgi

// The wavefront layout shares this translation unit's helpers and constants.
#include "vgi_wave.cuh"
#include "vgi_retention.cuh"
#include "vgi_view.cuh"
