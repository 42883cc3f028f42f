// Wavefront layout of the face trace (included by vgi_trace.cu, so it shares
// the estimator helpers and the Halton table).
//
// The per-path work of trace_receiver / advance_path (voxel_path.wgsl:418-520)
// runs as stages. At each stage a path emits every ray it can launch
// independently: its continuation, one shadow ray per light for direct_at,
// and its emitter NEE or terminal connection. One persistent traversal
// kernel then runs all queued rays. Its lanes refill from the queue as their
// rays finish, so warps stay full whatever the step counts. The next shade
// stage first completes the previous hit's contribution in the shader's
// operation order:
//     energy + tp * (emission * mis + diffuse * (direct + nee))
// then processes the new hit. Every path performs the same float operations
// as the single-kernel layout, so results are bit-identical to it and to the
// oracle.
//
// Launch sequence per frame with DIFFUSE_HITS = H:
//     begin, (traverse, shade) x H, traverse, finalize.
// Ray slots per path and stage: 0 continuation, 1 NEE shadow or terminal ray,
// 2.. one shadow ray per light. Face-centre direct rays follow all path slots.

namespace vgi {
namespace {

constexpr int kWaveBlock = 256;

// Resident blocks per SM each kernel's register budget must allow.
#ifndef VGI_TRAVERSE_MIN_BLOCKS
#define VGI_TRAVERSE_MIN_BLOCKS 4
#endif
#ifndef VGI_BEGIN_MIN_BLOCKS
#define VGI_BEGIN_MIN_BLOCKS 4
#endif
#ifndef VGI_SHADE_MIN_BLOCKS
#define VGI_SHADE_MIN_BLOCKS 4
#endif
#ifndef VGI_SCATTER_MIN_BLOCKS
#define VGI_SCATTER_MIN_BLOCKS 4
#endif
#ifndef VGI_FINALIZE_MIN_BLOCKS
#define VGI_FINALIZE_MIN_BLOCKS 4
#endif

// Path-state fields, each an array of n_paths float4 (SoA for coalescing).
enum : uint32_t {
    kE = 0,    // continuation energy rgb, previous_pdf
    kTP = 1,   // throughput for the next hit rgb, bounce (bits)
    kPP = 2,   // previous position xyz (the last hit point), the path word (bits)
    kTH = 3,   // throughput at the pending hit rgb, the hit's emission MIS weight
    kX = 4,    // cached energy or pending emitter value rgb
    kN0 = 5,   // receiver NEE (pending, then final) rgb
    kFields = 6,
};
static_assert(kFields == kWavePathFields, "path-state fields");

// The path word (kPP.w): flags in bits 0-5, the pending contribution's kind
// in bits 8-10, the previous normal in bits 12-17 (two bits an axis) and the
// pending hit's material in bits 24-31. A pending hit's emission * MIS and
// diffuse are its material's values times kTH.w, formed again where they
// are used with the same operations, so they need no fields of their own.
constexpr uint32_t kFlagContinue = 1u;   // slot 0 holds this stage's continuation ray
constexpr uint32_t kFlagUnknown = 2u;    // reached unloaded space
constexpr uint32_t kFlagRan = 4u;        // the receiver's continuation was traced
constexpr uint32_t kFlagS0 = 8u;         // slot 1 holds the receiver's NEE shadow ray
constexpr uint32_t kFlagN = 16u;         // slot 1 holds the pending hit's NEE or terminal ray
constexpr uint32_t kFlagValid = 32u;     // a traced sample of a valid task

// Pending-contribution kinds (path word bits 8-10).
constexpr uint32_t kKindNone = 0u, kKindCached = 1u, kKindNee = 2u, kKindTermEmitter = 3u, kKindTermCosine = 4u;

__device__ __forceinline__ uint32_t kind_of(uint32_t w) { return (w >> 8) & 7u; }
__device__ __forceinline__ uint32_t with_kind(uint32_t w, uint32_t k) { return (w & ~(7u << 8)) | (k << 8); }
// Normals on the path are face normals or zero: each axis is +0, -0, +1 or
// -1 (the traversal's normals carry signed zeros), coded 0, 1, 2, 3.
__device__ __forceinline__ uint32_t axis_code(float v) { return v > 0.0f ? 2u : (v < 0.0f ? 3u : (__float_as_uint(v) >> 31)); }
__device__ __forceinline__ float axis_value(uint32_t c) { return c == 2u ? 1.0f : (c == 3u ? -1.0f : __uint_as_float(c << 31)); }
__device__ __forceinline__ uint32_t with_normal(uint32_t w, V3 n) {
    return (w & ~(63u << 12)) | ((axis_code(n.x) | (axis_code(n.y) << 2) | (axis_code(n.z) << 4)) << 12);
}
__device__ __forceinline__ V3 normal_of(uint32_t w) { return V3{axis_value((w >> 12) & 3u), axis_value((w >> 14) & 3u), axis_value((w >> 16) & 3u)}; }
__device__ __forceinline__ uint32_t with_material(uint32_t w, uint32_t m) { return (w & 0x00ffffffu) | ((m & 255u) << 24); }
__device__ __forceinline__ uint32_t material_of(uint32_t w) { return w >> 24; }

struct WaveArgs {
    TraceArgs t;
    uint32_t n_paths;
    uint32_t slots;          // ray slots per path: 2 + lights
    float4* state;           // kFields * n_paths
    float4* ray;             // 2 float4 per ray slot: origin xyz + max distance, direction xyz + (full bit)
    uint32_t* status;        // per ray slot
    uint4* hit;              // 3 uint4 per path for slots 0 and 1 (full results): [p*2 + slot]
    uint32_t* queue_in;      // ray slot indices to traverse
    const uint32_t* count_in;
    uint32_t* queue_out;     // rays emitted by this stage
    uint32_t* count_out;
    uint32_t* queue_head;    // traversal cursor
    uint32_t* scatter_queue; // uncached hits: path | bounce << 30
    uint32_t* scatter_count;
    float4* mlp_queue;       // MLP termination (null: off): per uncached hit (face centre, path), (albedo, face)
    uint32_t* mlp_count;
};

__device__ __forceinline__ float4& field(const WaveArgs& W, uint32_t f, uint32_t p) { return W.state[(size_t)f * W.n_paths + p]; }
__device__ __forceinline__ uint32_t bits(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float fl(uint32_t u) { return __uint_as_float(u); }

// Appends `slot` to the output queue (one atomic per warp).
__device__ __forceinline__ void enqueue(const WaveArgs& W, bool want, uint32_t slot) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(W.count_out, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) W.queue_out[base + __popc(mask & ((1u << lane) - 1u))] = slot;
}

// `hit`: 0 for a ray whose status alone is read (shadow rays), else 1 + the
// index of its full hit record (path p's slot k in {0, 1}: 2p + k), which
// the traversal writes when the ray ends.
__device__ __forceinline__ void put_ray(const WaveArgs& W, uint32_t slot, V3 o, V3 d, float maxd, uint32_t hit) {
    W.ray[2u * slot] = make_float4(o.x, o.y, o.z, maxd);
    W.ray[2u * slot + 1u] = make_float4(d.x, d.y, d.z, fl(hit));
}
__device__ __forceinline__ uint32_t hit_of(uint32_t p, uint32_t k) { return 2u * p + k + 1u; }

template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
struct WaveTracer {
    const WaveArgs& W;
    const TraceArgs& A;
    const float4* smat;
    Cnt<C>& cnt;

    __device__ Mat material_nocount(uint32_t m) const {
        m &= 255u;
        float4 d = smat[m * 2u], e = smat[m * 2u + 1u];
        return Mat{make_float4(d.x, d.y, d.z, 0.0f), make_float4(e.x, e.y, e.z, 0.0f), d.w};
    }
    __device__ float reach() const { return LIMITED ? A.reach : A.max_distance; }

    // sample_emitter up to its shadow ray (voxel_path.wgsl:332-358). Returns
    // true with the ray and the value it would add (emission * factor) when a
    // ray is needed; the material is counted when the ray turns out visible.
    __device__ bool prepare_nee(V3 position, V3 normal, uint32_t source_stream, uint32_t sequence, uint32_t bounce, V3& so, V3& sdir,
                                float& sdist, V3& pending, const float* top = nullptr) {
        if (A.emitter_count == 0.0f) return false;
        uint32_t stream = source_stream ^ pcg(bounce + 0xa341316cu);
        // choose_emitter (voxel_path.wgsl:309-324)
        Emissive em;
        {
            const float choice = sample_1d(stream, sequence, 12u);
            uint32_t count = f2u(A.emitter_count);
            if (load_emitter(A, 0u, cnt).sampling.w > 0.0f) {
                em = tree_emitter(A, position, normal, choice, cnt, top);
            } else {
                uint32_t low = 0, high = count;
#pragma unroll 1
                while (low < high) {
                    uint32_t middle = (low + high) / 2u;
                    if (load_emitter(A, middle, cnt).sampling.x <= choice) low = middle + 1u;
                    else high = middle;
                }
                em = load_emitter(A, low < count - 1u ? low : count - 1u, cnt);
            }
        }
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
        if (d2 < 0.0001f || d2 > __fmul_rn(r, r)) return false;
        float distance = __fsqrt_rn(d2);
        V3 direction = delta / distance;
        float rc = wmax(dot3(normal, direction), 0.0f);
        float ec = wmax(dot3(en, -direction), 0.0f);
        if (rc <= 0.0f || ec <= 0.0f || em.sampling.y <= 0.0f) return false;
        float light_pdf = __fdiv_rn(__fmul_rn(em.sampling.y, d2), ec);
        float directional_pdf = __fdiv_rn(rc, 3.14159265359f);
        so = position + normal * 0.002f;
        V3 sd = (lp + en * 0.002f) - so;
        sdist = len3(sd);
        sdir = sd / sdist;
        Mat m = material_nocount(f2u(em.sampling.z));
        float factor = __fdiv_rn(directional_pdf, __fadd_rn(light_pdf, directional_pdf));
        pending = V3{m.emission.x, m.emission.y, m.emission.z} * factor;
        // The material index rides in the ray's spare word for the count.
        return true;
    }

    // direct_at's rays (voxel_path.wgsl:283-307): one per light that faces the point.
    __device__ void emit_direct(V3 position, V3 normal, uint32_t first_slot, bool want) {
        V3 origin = position + normal * 0.002f;
#pragma unroll 1
        for (uint32_t i = 0; i < A.light_count; ++i) {
            bool emit = false;
            V3 direction{0.0f, 0.0f, 0.0f};
            float distance = A.max_distance;
            if (want) {
                const float4 Lp = __ldg(A.lights + i * 3u);
                cnt.bytes(48);
                V3 pos{Lp.x, Lp.y, Lp.z};
                bool skip = false;
                if (Lp.w >= 0.0f) {
                    V3 delta = pos - position;
                    float d2 = dot3(delta, delta);
                    if (d2 <= 0.0000001f || d2 > __fmul_rn(Lp.w, Lp.w)) skip = true;
                    else {
                        distance = __fsqrt_rn(d2);
                        direction = delta / distance;
                        distance = __fsub_rn(distance, 0.004f);
                    }
                } else {
                    direction = normalize3(pos);
                }
                emit = !skip && wmax(dot3(normal, direction), 0.0f) > 0.0f;
                if (emit) put_ray(W, first_slot + i, origin, direction, distance, 0u);
            }
            enqueue(W, emit, first_slot + i);
        }
    }

    // direct_at's value from the shadow rays' statuses, in light order.
    template <bool CUSTOM>
    __device__ V3 gather_direct(V3 position, V3 normal, uint32_t first_slot, V3* custom, float* value_w) {
        V3 value{0.0f, 0.0f, 0.0f}, cv{0.0f, 0.0f, 0.0f};
        float w = 0.0f;
#pragma unroll 1
        for (uint32_t i = 0; i < A.light_count; ++i) {
            const float4 Lp = __ldg(A.lights + i * 3u), Le = __ldg(A.lights + i * 3u + 1u);
            V3 pos{Lp.x, Lp.y, Lp.z};
            float attenuation = 1.0f;
            V3 direction;
            if (Lp.w >= 0.0f) {
                V3 delta = pos - position;
                float d2 = dot3(delta, delta);
                if (d2 <= 0.0000001f || d2 > __fmul_rn(Lp.w, Lp.w)) continue;
                float distance = __fsqrt_rn(d2);
                direction = delta / distance;
                attenuation = __fdiv_rn(1.0f, wmax(d2, 1.0f));
            } else {
                direction = normalize3(pos);
            }
            float cosine = wmax(dot3(normal, direction), 0.0f);
            if (cosine > 0.0f && W.status[first_slot + i] == 0u) {
                float k = __fmul_rn(cosine, attenuation);
                value = value + V3{Le.x, Le.y, Le.z} * k;
                if (CUSTOM) {
                    const float4 Lx = __ldg(A.lights + i * 3u + 2u);
                    cv = cv + V3{Lx.y, Lx.z, Lx.w} * k;
                    w = __fadd_rn(w, __fmul_rn(Le.w, k));
                }
            }
        }
        if (CUSTOM) {
            *custom = cv;
            *value_w = w;
        }
        return value;
    }

    // The status a shadow/continuation ray reports through trace() (BUDGETED fix).
    __device__ uint32_t traced_status(uint32_t slot) const { return W.status[slot]; }

    // Completes the pending hit of path p: energy += tp * (em*mis + diffuse * (direct + X)).
    // `word` is the path word and `position` the pending hit point (kPP).
    __device__ void combine(uint32_t p, uint32_t word, V3 position, float4& e) {
        const uint32_t kind = kind_of(word), flags = word;
        const float4 th = field(W, kTH, p), xv = field(W, kX, p);
        const V3 normal = normal_of(word);
        const Mat mat = material_nocount(material_of(word));
        // The hit's emission * mis and diffuse, as the shade stage formed them.
        const V3 em = V3{mat.emission.x, mat.emission.y, mat.emission.z} * th.w;
        const V3 df{mat.diffuse.x, mat.diffuse.y, mat.diffuse.z};
        const uint32_t base = p * W.slots;
        V3 unused;
        float unused_w;
        V3 direct = gather_direct<false>(position, normal, base + 2u, &unused, &unused_w);
        V3 x{0.0f, 0.0f, 0.0f};
        if (kind == kKindCached) {
            x = V3{xv.x, xv.y, xv.z};
        } else if (kind == kKindNee || kind == kKindTermEmitter) {
            if ((flags & kFlagN) && traced_status(base + 1u) == 0u) {
                cnt.bytes(64);  // sample_emitter's material read
                x = V3{xv.x, xv.y, xv.z};
            }
            if (kind == kKindTermEmitter) x = x * 2.0f;
        } else if (kind == kKindTermCosine && (flags & kFlagN)) {
            // sample_terminal_emission's cosine branch (voxel_path.wgsl:376-393).
            const uint4 h0 = W.hit[((size_t)p * 2u + 1u) * 3u], h1 = W.hit[((size_t)p * 2u + 1u) * 3u + 1u],
                        h2 = W.hit[((size_t)p * 2u + 1u) * 3u + 2u];
            if (h0.x == 1u) {
                const float4 rd = W.ray[2u * (base + 1u) + 1u];
                const V3 direction{rd.x, rd.y, rd.z};
                cnt.bytes(64);
                Mat m = material_nocount(h0.y);
                const V3 hp{fl(h1.y), fl(h1.z), fl(h1.w)}, hn{fl(h2.x), fl(h2.y), fl(h2.z)};
                const I3 hv{(int)h0.z, (int)h0.w, (int)h1.x};
                float power = m.weight;
                V3 delta = hp - position;
                float d2 = dot3(delta, delta);
                float r = reach();
                if (!(power == 0.0f || d2 < 0.0001f || d2 > __fmul_rn(r, r))) {
                    float selection_pdf = __fdiv_rn(power, wmax(A.emitter_total, 1e-20f));
                    if (load_emitter(A, 0u, cnt).sampling.w > 0.0f) selection_pdf = tree_probability(A, position, normal, hv, hn, cnt);
                    float light_pdf = __fdiv_rn(__fmul_rn(selection_pdf, d2), wmax(dot3(hn, -direction), 1e-8f));
                    float directional_pdf = cosine_pdf(normal, direction);
                    float factor = __fdiv_rn(__fmul_rn(2.0f, directional_pdf), __fadd_rn(directional_pdf, light_pdf));
                    x = V3{m.emission.x, m.emission.y, m.emission.z} * factor;
                }
            }
        }
        const V3 tp{th.x, th.y, th.z};
        const V3 t = em + df * (direct + x);
        const V3 energy = V3{e.x, e.y, e.z} + tp * t;
        e.x = energy.x;
        e.y = energy.y;
        e.z = energy.z;
    }
};

template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__device__ __forceinline__ void stage_materials(const TraceArgs& A, float4* smat) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        float4 d = __ldg(A.materials + i * 4), e = __ldg(A.materials + i * 4 + 2), x = __ldg(A.materials + i * 4 + 3);
        smat[i * 2] = make_float4(d.x, d.y, d.z, x.y);
        smat[i * 2 + 1] = make_float4(e.x, e.y, e.z, 0.0f);
    }
    __syncthreads();
}

template <bool C>
__device__ __forceinline__ void flush_counters(const TraceArgs& A, Cnt<C>& cnt) {
    if constexpr (C) {
        unsigned long long v[kCounterWords];
        v[0] = cnt.rays; v[1] = cnt.paths; v[2] = cnt.steps; v[3] = cnt.b; v[4] = cnt.unk; v[5] = cnt.hits;
        v[6] = cnt.st[0]; v[7] = cnt.st[1]; v[8] = cnt.st[2]; v[9] = cnt.st[3]; v[10] = cnt.tb;
        v[11] = cnt.wp[0]; v[12] = cnt.wp[1]; v[13] = cnt.lp[0]; v[14] = cnt.lp[1];
#pragma unroll
        for (int k = 0; k < kCounterWords; ++k) {
            unsigned long long x = v[k];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31u) == 0u && x) atomicAdd(A.counters + k, x);
        }
    }
}

// Stage 0: the receiver sample (voxel_path.wgsl:504-513) of every path, and
// the face-centre direct rays of write_result (voxel_trace.wgsl:28).
template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__global__ void __launch_bounds__(kWaveBlock, VGI_BEGIN_MIN_BLOCKS) wave_begin_kernel(const WaveArgs W) {
    __shared__ float4 smat[512];
    const TraceArgs& A = W.t;
    stage_materials<HITS, LIMITED, BUDGETED, C>(A, smat);
    Cnt<C> cnt;
    WaveTracer<HITS, LIMITED, BUDGETED, C> T{W, A, smat, cnt};
    const uint32_t p = blockIdx.x * kWaveBlock + threadIdx.x;
    const bool in = p < W.n_paths;
    const uint32_t face = in ? p / A.samples : 0u;
    const uint32_t sample = in ? p - face * A.samples : 0u;
    uint4 t0 = make_uint4(0, 0, 0, 0xffffffffu), t1 = make_uint4(0, 0, 0, 0);
    if (in) {
        t0 = __ldg(A.tasks + face * 2u);
        t1 = __ldg(A.tasks + face * 2u + 1u);
    }
    const bool valid = in && t0.w != 0xffffffffu;
    const V3 normal = face_normal(valid ? t0.w : 0u);
    const I3 voxel{(int)t0.x, (int)t0.y, (int)t0.z};
    const V3 surface = add_s(itof(voxel), 0.5f) + normal * 0.5f;
    const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(t0.w + 1u);
    const uint32_t sequence = t1.x + sample;
    const uint32_t base = p * W.slots;
    uint32_t flags = valid ? kFlagValid : 0u;
    bool s0 = false, c0 = false;
    // The receiver's position and normal are the task's, the same every
    // frame, so the light tree's child probabilities on the top levels of
    // its NEE walk are too. A face keeps them in its row (the timed passes;
    // the counting pass walks as the reference does, to count the node
    // reads): on a miss (new face, new tree) the face's lanes compute the
    // row's slots between them, then every lane walks from it. The face's
    // lanes share a warp when the sample count divides 32.
    const float* top = nullptr;
    if constexpr (!C) {
        if (A.tree_rows != nullptr && A.samples != 0u && 32u % A.samples == 0u) {
            uint4* row = A.tree_rows + (size_t)face * kTreeRowWords;
            const bool tree = valid && A.emitter_count != 0.0f && __uint_as_float(__ldg(A.emitters + 1u).w) > 0.0f;
            bool miss = false;
            if (tree) {
                const uint4 key = row[0];
                miss = key.x != t0.x || key.y != t0.y || key.z != t0.z || key.w != t0.w || row[1].x != A.tree_generation;
                if (miss) {
                    float* slots = reinterpret_cast<float*>(row + 2);
                    for (uint32_t j = sample; j < kTreeTopSlots; j += A.samples) slots[j] = tree_slot_probability(A, j, surface, normal);
                }
            }
            __syncwarp();
            if (tree) {
                if (miss && sample == 0u) {
                    row[0] = t0;
                    row[1] = make_uint4(A.tree_generation, 0u, 0u, 0u);
                }
                top = reinterpret_cast<const float*>(row + 2);
            }
        }
    }
    if (valid) {
        cnt.path();
        if (sample == 0u) cnt.bytes(32 + 96);
        V3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
        V3 so, sd, pending;
        float sdist;
        s0 = T.prepare_nee(surface, normal, stream, sequence, 0u, so, sd, sdist, pending, top);
        if (s0) {
            put_ray(W, base + 1u, so, sd, sdist, 0u);
            flags |= kFlagS0;
            field(W, kN0, p) = make_float4(pending.x, pending.y, pending.z, 0.0f);
        } else {
            field(W, kN0, p) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        // Nothing is pending yet (kind 0 in the path word).
        if (dot3(normal, direction) > 0.0f) {
            flags |= kFlagRan;
            const V3 start = surface + normal * 0.001f;
            const float previous_pdf = cosine_pdf(normal, direction);
            const V3 previous_position = start - normal * 0.001f;
            field(W, kE, p) = make_float4(0.0f, 0.0f, 0.0f, previous_pdf);
            field(W, kTP, p) = make_float4(1.0f, 1.0f, 1.0f, fl(0u));
            if (previous_pdf > 0.0f) {
                c0 = true;
                flags |= kFlagContinue;
                put_ray(W, base, start, direction, T.reach(), hit_of(p, 0u));
            }
            field(W, kPP, p) = make_float4(previous_position.x, previous_position.y, previous_position.z, fl(with_normal(flags, normal)));
        } else {
            field(W, kE, p) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            field(W, kPP, p) = make_float4(0.0f, 0.0f, 0.0f, fl(flags));
        }
    } else if (in) {
        field(W, kPP, p) = make_float4(0.0f, 0.0f, 0.0f, fl(0u));
    }
    enqueue(W, s0, base + 1u);
    enqueue(W, c0, base);
    // Face-centre direct rays, one thread per face.
    const uint32_t face_slots = W.n_paths * W.slots;
    T.emit_direct(surface, normal, face_slots + face * A.light_count, valid && sample == 0u);
    flush_counters<C>(A, cnt);
}

// One lane's ray in flight: trace_domain_limited's loop variables.
struct RayRun {
    V3 dir, pos;
    // The direction's reciprocals for div_recip on the axes the traversal
    // treats as moving (|d| > 1e-8), NaN on the others. advance_box gives a
    // non-moving axis the distance 1e30; a NaN quotient fails its range test
    // and takes 1e30 the same way, so the step needs no test of its own.
    V3 inv;
    float dist, maxd;
    int lrx, lry, lrz;
    uint4 meta;
    uint32_t step, slot;
    // The last step's normal, coded two bits an axis (axis_code), expanded
    // when the ray ends.
    uint32_t ncode;
    // Per axis, from the direction's sign: bits 0-5 the code the axis's
    // normal component takes when another axis is the exit (advance_box
    // multiplies 0 by -1 when d > 0: -0), bits 8-13 the code it takes when
    // it is the exit axis, bit 16 + axis set when d > 0 (the box's exit plane
    // is its upper face).
    uint32_t signs;
    // The box of the last step: its exit planes, and the voxel position
    // shifted by the level it was found at (4 region, 2 brick, 0 voxel).
    // While the voxel keeps this key the lookup would find the same box:
    // creep replays the steps of a ray that grazes a face, where the move
    // across the face is lost to rounding, inside one box this way.
    V3 plane;
    int kx, ky, kz;
    uint32_t shift;  // kNoIndex: no box cached
    uint32_t hit;    // 0, or 1 + the index of the ray's full hit record
};

__device__ __forceinline__ V3 decode_normal(uint32_t code) {
    return V3{axis_value(code & 3u), axis_value((code >> 2) & 3u), axis_value((code >> 4) & 3u)};
}

__device__ __forceinline__ uint32_t direction_signs(V3 d) {
    const uint32_t px = d.x > 0.0f ? 1u : 0u, py = d.y > 0.0f ? 1u : 0u, pz = d.z > 0.0f ? 1u : 0u;
    const uint32_t zeros = px | (py << 2) | (pz << 4);
    const uint32_t exits = (px ? 3u : 2u) | ((py ? 3u : 2u) << 2) | ((pz ? 3u : 2u) << 4);
    return zeros | (exits << 8) | (px << 16) | (py << 17) | (pz << 18);
}

__device__ __forceinline__ V3 traversal_recip(V3 d) {
    const float nan = __uint_as_float(0x7fc00000u);
    return V3{fabsf(d.x) > 1e-8f ? __frcp_rn(d.x) : nan, fabsf(d.y) > 1e-8f ? __frcp_rn(d.y) : nan,
              fabsf(d.z) > 1e-8f ? __frcp_rn(d.z) : nan};
}

// advance_box's step from the box's exit planes (voxel_traversal.wgsl:90-107,
// as advance_planes): returns the distance to move and sets the normal's
// code. Every float operation is advance_planes'.
__device__ __forceinline__ float step_planes(V3 p, V3 d, V3 inv, V3 plane, uint32_t signs, uint32_t& ncode) {
    const float rx = div_recip(__fsub_rn(plane.x, p.x), d.x, inv.x);
    const float ry = div_recip(__fsub_rn(plane.y, p.y), d.y, inv.y);
    const float rz = div_recip(__fsub_rn(plane.z, p.z), d.z, inv.z);
    const float tx = (rx >= -0.001f && rx < 1e30f) ? rx : 1e30f;
    const float ty = (ry >= -0.001f && ry < 1e30f) ? ry : 1e30f;
    const float tz = (rz >= -0.001f && rz < 1e30f) ? rz : 1e30f;
    const bool choose_y = ty < wmax(tx, 0.0f);
    const float dxy = wmax(choose_y ? ty : tx, 0.0f);
    const bool choose_z = tz < dxy;
    const float dist = wmax(choose_z ? tz : dxy, 0.0f);
    const uint32_t mask = choose_z ? (3u << 4) : (choose_y ? (3u << 2) : 3u);
    ncode = dist < 1e30f ? (((signs & ~mask) | ((signs >> 8) & mask)) & 63u) : 0u;
    return wmax(__fadd_rn(dist, 0.001f), 0.001f);
}

template <bool BUDGETED>
__device__ __forceinline__ void finish_ray(const WaveArgs& W, RayRun& s, uint32_t status, uint32_t material, I3 voxel, V3 position, V3 normal) {
    if (BUDGETED && status == 2u && material == 0xffffffffu) status = 0u;  // trace()'s budget rule
    W.status[s.slot] = status;
    if (s.hit) {
        uint4* h = W.hit + (size_t)(s.hit - 1u) * 3u;
        h[0] = make_uint4(status, material, (uint32_t)voxel.x, (uint32_t)voxel.y);
        h[1] = make_uint4((uint32_t)voxel.z, bits(position.x), bits(position.y), bits(position.z));
        h[2] = make_uint4(bits(normal.x), bits(normal.y), bits(normal.z), 0u);
    }
    s.slot = kNoIndex;
}

// trace_domain_limited's slab clip (voxel_traversal.wgsl:127-151) of a ray
// against the scene bounds: the near and far distances, whether an axis that
// does not move lies outside the bounds, and the nearest slab's normal code
// (one axis -1, code 3, or +1, code 2; the others +0).
__device__ __forceinline__ uint32_t slab_clip(const TraceArgs& A, V3 origin, V3 dir, V3 inv, float& nearv, float& farv, bool& miss) {
    nearv = -1e30f;
    farv = 1e30f;
    miss = false;
    uint32_t ncode = 0u;
    const float mnx = __fmul_rn((float)A.mn[0], 16.0f), mny = __fmul_rn((float)A.mn[1], 16.0f), mnz = __fmul_rn((float)A.mn[2], 16.0f);
    const float mxx = __fmul_rn((float)(A.mx[0] + 1), 16.0f), mxy = __fmul_rn((float)(A.mx[1] + 1), 16.0f),
                mxz = __fmul_rn((float)(A.mx[2] + 1), 16.0f);
#define VGI_SLAB(AX, O, D, Y, MN, MX)                                  \
    if (fabsf(D) <= 1e-8f) {                                           \
        if (O < MN || O > MX) miss = true;                             \
    } else {                                                           \
        const float first = div_recip(__fsub_rn(MN, O), D, Y);         \
        const float second = div_recip(__fsub_rn(MX, O), D, Y);        \
        if (wmin(first, second) > nearv) {                             \
            nearv = wmin(first, second);                               \
            ncode = (first < second ? 3u : 2u) << (2 * AX);            \
        }                                                              \
        farv = wmin(farv, wmax(first, second));                        \
    }
    VGI_SLAB(0, origin.x, dir.x, inv.x, mnx, mxx)
    VGI_SLAB(1, origin.y, dir.y, inv.y, mny, mxy)
    VGI_SLAB(2, origin.z, dir.z, inv.z, mnz, mxz)
#undef VGI_SLAB
    return ncode;
}

// The normal code is the slab clip's and has not been formed yet (below).
constexpr uint32_t kSlabPending = 1u << 31;

// trace_domain_limited's set-up: the slab clip. A ray that misses finishes
// at once. For an origin strictly inside the bounds on every axis the clip's
// outcome needs no division: every moving axis has one negative and one
// positive slab distance, so the near distance is negative, the far one
// positive, nothing misses and the start distance is 0 + 0.001. Only the
// slab normal needs the quotients, and only a ray that hits before its first
// box step reports it, so that ray forms it when it ends (normal_code).
template <bool BUDGETED, bool C>
__device__ __forceinline__ void start_ray(const WaveArgs& W, RayRun& s, uint32_t slot, Cnt<C>& cnt) {
    const TraceArgs& A = W.t;
    const float4 ro = W.ray[2u * slot], rd = W.ray[2u * slot + 1u];
    s.slot = slot;
    s.hit = bits(rd.w);
    s.dir = V3{rd.x, rd.y, rd.z};
    s.inv = traversal_recip(s.dir);
    s.signs = direction_signs(s.dir);
    s.maxd = ro.w;
    cnt.ray();
    const V3 origin{ro.x, ro.y, ro.z};
    const bool inside = origin.x > __fmul_rn((float)A.mn[0], 16.0f) && origin.x < __fmul_rn((float)(A.mx[0] + 1), 16.0f) &&
                        origin.y > __fmul_rn((float)A.mn[1], 16.0f) && origin.y < __fmul_rn((float)(A.mx[1] + 1), 16.0f) &&
                        origin.z > __fmul_rn((float)A.mn[2], 16.0f) && origin.z < __fmul_rn((float)(A.mx[2] + 1), 16.0f);
    if (inside) {
        s.dist = 0.001f;
        s.ncode = kSlabPending;
    } else {
        float nearv, farv;
        bool miss;
        const uint32_t ncode = slab_clip(A, origin, s.dir, s.inv, nearv, farv, miss);
        if (miss || farv < wmax(nearv, 0.0f)) {
            cnt.status(0);
            const I3 zi{0, 0, 0};
            const V3 zv{0.0f, 0.0f, 0.0f};
            finish_ray<BUDGETED>(W, s, 0u, 0u, zi, zv, zv);
            return;
        }
        s.dist = __fadd_rn(wmax(nearv, 0.0f), 0.001f);
        s.ncode = ncode;
    }
    s.pos = origin + s.dir * s.dist;
    s.lrx = s.lry = s.lrz = 0x7fffffff;
    s.meta = make_uint4(0, 0, 0, 0);
    s.shift = kNoIndex;
    s.step = 0;
}

// The ray's normal code, forming the slab clip's when it is still pending.
__device__ __forceinline__ uint32_t normal_code(const WaveArgs& W, const RayRun& s) {
    if (!(s.ncode & kSlabPending)) return s.ncode;
    const float4 ro = W.ray[2u * s.slot];
    float nearv, farv;
    bool miss;
    return slab_clip(W.t, V3{ro.x, ro.y, ro.z}, s.dir, s.inv, nearv, farv, miss);
}

// Steps of a ray that grazes a face of its box. If some moving axis's exit
// distance lies in [-0.001, 0] and adding dir * 0.001 cannot change that
// coordinate (the move rounds away), then every later step in the same box
// exits at distance 0: advance_box returns exactly 0.001 (any exit distance
// <= 0 makes its selected distance 0), the coordinate stays, and so does the
// exit distance. Those steps are replayed here as what they are, four
// additions each, while the voxel keeps the box's key, and only the last
// one's normal is computed in full. Every value equals the general step's.
// `limit` bounds the replayed step count (it is the step budget once the
// queue is empty, so a lane then finishes its creep in one pass).
template <bool C>
__device__ __forceinline__ void creep(const TraceArgs& A, RayRun& s, Cnt<C>& cnt, uint32_t limit) {
    const V3 c = s.dir * 0.001f;
    bool stuck = false;
#define VGI_STUCK(AX)                                                                                              \
    if (fabsf(s.dir.AX) > 1e-8f) {                                                                                 \
        const float raw = div_recip(__fsub_rn(s.plane.AX, s.pos.AX), s.dir.AX, s.inv.AX);                           \
        if (raw >= -0.001f && raw <= 0.0f && __fadd_rn(s.pos.AX, c.AX) == s.pos.AX) stuck = true;                  \
    }
    VGI_STUCK(x)
    VGI_STUCK(y)
    VGI_STUCK(z)
#undef VGI_STUCK
    if (!stuck) return;
    const uint32_t bytes = s.shift == 4u ? 0u : (s.shift == 2u ? 4u : 8u);
    const uint32_t end = limit < A.path_steps ? limit : A.path_steps;
    V3 last = s.pos;
    bool ran = false;
#pragma unroll 1
    while (s.step < end && !(s.dist > s.maxd)) {
        const int vx = f2i(floorf(s.pos.x)), vy = f2i(floorf(s.pos.y)), vz = f2i(floorf(s.pos.z));
        if ((vx >> s.shift) != s.kx || (vy >> s.shift) != s.ky || (vz >> s.shift) != s.kz) break;
        cnt.step();
        cnt.tbytes(bytes);
        last = s.pos;
        ran = true;
        s.dist = __fadd_rn(s.dist, 0.001f);
        s.pos = s.pos + c;
        s.step += 1u;
    }
    if (ran) step_planes(last, s.dir, s.inv, s.plane, s.signs, s.ncode);
}

constexpr uint32_t kGo = 0xffffffffu;

// The first half of a step: everything up to the box step. It leaves `status`
// at kGo when the ray skips the box in s.plane, or sets the ray's outcome.
//
// Written as one straight pass for every lane rather than as nested branches
// per level: each lookup (region grid and header, brick word, cell word) is a
// load that the lanes needing it make together, and the decode of whatever
// level a lane stopped at is a set of selects. A warp therefore issues the
// lookup once per step, not once per branch some lane takes; the words read,
// the boxes chosen and every float operation are those of the branched form
// (trace_domain_limited, voxel_traversal.wgsl:152-213).
template <bool BUDGETED, bool C>
__device__ __forceinline__ void classify_step(const WaveArgs& W, RayRun& s, Cnt<C>& cnt, uint32_t& status, uint32_t& material, I3& voxel) {
    const TraceArgs& A = W.t;
    const bool out_of_steps = s.step >= A.path_steps;
    voxel = I3{f2i(floorf(s.pos.x)), f2i(floorf(s.pos.y)), f2i(floorf(s.pos.z))};
    const int rx = voxel.x >> 4, ry = voxel.y >> 4, rz = voxel.z >> 4;
    const bool beyond = s.dist > s.maxd;
    // The region's offset in the bounding box: inside when every axis is
    // below the box's size (unsigned, so a region below the box wraps high).
    const uint32_t nx = (uint32_t)(A.mx[0] - A.mn[0] + 1), ny = (uint32_t)(A.mx[1] - A.mn[1] + 1);
    const uint32_t gx = (uint32_t)rx - (uint32_t)A.mn[0], gy = (uint32_t)ry - (uint32_t)A.mn[1], gz = (uint32_t)rz - (uint32_t)A.mn[2];
    const bool inside = gx < nx && gy < ny && gz <= (uint32_t)(A.mx[2] - A.mn[2]);
    const bool lookup = !out_of_steps && !beyond && inside;
    if constexpr (C) {
        if (!out_of_steps) cnt.step();
    }
    // Region: the header of a region entered this step. The timed pass reads
    // it straight from the dense header grid (kind 0 where the directory
    // finds no region), one load; the counting pass probes the directory to
    // count its words. Both give lookup_region's answer.
    const bool new_region = lookup && (s.lrx != rx || s.lry != ry || s.lrz != rz);
    bool missing = false;
    if (new_region) {
        uint4 h;
        if (!C && A.region_headers) {
            h = __ldg(A.region_headers + (gz * ny + gy) * nx + gx);
            missing = h.x == 0u;
        } else {
            const uint32_t index = lookup_region(A, rx, ry, rz, cnt);
            missing = index == kNoIndex;
            if (!missing) {
                cnt.tbytes(16);
                h = __ldg(A.headers + index);
            }
        }
        if (!missing) {
            s.meta = h;
            s.lrx = rx;
            s.lry = ry;
            s.lrz = rz;
        }
    }
    const bool present = lookup && !missing;
    const bool air_region = present && s.meta.x == 1u;
    const bool mixed = present && s.meta.x == 3u;
    const bool solid_region = present && s.meta.x != 1u && s.meta.x != 3u;
    // Brick word of a mixed region, then the cell word of a mixed brick.
    const uint32_t lx = (uint32_t)(voxel.x & 15), ly = (uint32_t)(voxel.y & 15), lz = (uint32_t)(voxel.z & 15);
    uint32_t brick = 0u;
    if (mixed) {
        brick = __ldg(A.cells + s.meta.y + ((lz >> 2) * 4u + (ly >> 2)) * 4u + (lx >> 2));
        cnt.tbytes(4);
    }
    const bool empty_brick = mixed && (brick & 3u) == 0u;
    const bool solid_brick = mixed && (brick & 3u) == 1u;
    const bool mixed_brick = mixed && (brick & 3u) >= 2u;
    const uint32_t idx = ((lz & 3u) * 4u + (ly & 3u)) * 4u + (lx & 3u);
    uint32_t word = 0u;
    if (mixed_brick) {
        word = __ldg(A.cells + (brick >> 2u) + (idx >> 1));
        cnt.tbytes(4);
    }
    const uint32_t c = (word >> ((idx & 1u) * 16u)) & 65535u;
    const bool solid_cell = mixed_brick && (c & 1u) != 0u;
    // The outcome.
    status = kGo;
    if (out_of_steps) {
        status = 2u;
        material = 0xffffffffu;
    } else if (!lookup) {
        status = 0u;
    } else if (solid_region || solid_brick || solid_cell) {
        status = 1u;
        material = solid_region ? s.meta.y : (solid_brick ? brick >> 2u : c >> 1u);
    }
    if (!BUDGETED && missing) {
        // visible_geometry crosses a missing region; otherwise the ray ends
        // as unknown or escaped by geometry_ahead.
        status = geometry_ahead(A, s.pos, s.dir, s.inv, __fsub_rn(s.maxd, s.dist), cnt) ? 2u : 0u;
    }
    if (lookup && status == kGo) {
        // The box the ray skips: the region's top-level box (an air region;
        // a missing region crossed under the budget rule, without extents and
        // not kept, since it is looked up again every step), the brick's box
        // (an empty brick) or the voxel's box (an air cell). Its cell is the
        // voxel shifted by the level (voxel >> 4 is the region, voxel >> 2
        // the brick), and each axis needs one face: the upper one,
        // (cell + pos + 1) * size, when the ray moves up the axis, else the
        // lower one, (cell - neg) * size, as box_planes picks them.
        const bool region_box = air_region || missing;
        const uint32_t level = region_box ? 4u : (empty_brick ? 2u : 0u);
        const float size = region_box ? 16.0f : (empty_brick ? 4.0f : 1.0f);
        const uint32_t e = empty_brick ? (brick >> 2u) : (c >> 1u);
        int face[3];
        const int v[3] = {voxel.x, voxel.y, voxel.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const bool up = (s.signs >> (16 + a)) & 1u;
            // Extents: a byte of the header's neg/pos word (air region), two
            // bits of the brick or cell word (neg at 4a, pos at 4a + 2), none
            // (missing region).
            const uint32_t region_ext = ((up ? s.meta.w : s.meta.z) >> (8 * a)) & 255u;
            const uint32_t cell_ext = (e >> (4 * a + (up ? 2 : 0))) & 3u;
            const int ext = missing ? 0 : (int)(air_region ? region_ext : cell_ext);
            const int cell = v[a] >> level;
            face[a] = up ? cell + ext + 1 : cell - ext;
        }
        s.plane = V3{__fmul_rn((float)face[0], size), __fmul_rn((float)face[1], size), __fmul_rn((float)face[2], size)};
        const uint32_t shift = missing ? kNoIndex : level;
        s.shift = shift;
        if (shift != kNoIndex) {
            s.kx = voxel.x >> shift;
            s.ky = voxel.y >> shift;
            s.kz = voxel.z >> shift;
        }
    }
}

// The second half: the ray ends with its outcome, or takes the box step.
template <bool BUDGETED, bool C>
__device__ __forceinline__ void finish_step(const WaveArgs& W, RayRun& s, Cnt<C>& cnt, uint32_t status, uint32_t material, I3 voxel,
                                            uint32_t creep_limit) {
    if (status != kGo) {
        cnt.status(status);
        const bool hit = status == 1u;
        const V3 zv{0.0f, 0.0f, 0.0f};
        finish_ray<BUDGETED>(W, s, status, material, hit ? voxel : I3{0, 0, 0}, hit ? s.pos : zv, hit ? decode_normal(normal_code(W, s)) : zv);
        return;
    }
    const float w = step_planes(s.pos, s.dir, s.inv, s.plane, s.signs, s.ncode);
    s.dist = __fadd_rn(s.dist, w);
    s.pos = s.pos + s.dir * w;
    s.step += 1u;
    if (w == 0.001f && s.shift != kNoIndex) creep<C>(W.t, s, cnt, creep_limit);
}

// trace() (voxel_path.wgsl:239-243) for every queued ray. Persistent warps
// keep one ray per lane and advance all lanes one DDA step per pass; when
// enough lanes have finished, they take the next rays from the queue (one
// atomic per warp), so a warp is not held by its longest ray.

template <bool BUDGETED, bool C>
__global__ void __launch_bounds__(kWaveBlock, VGI_TRAVERSE_MIN_BLOCKS) wave_traverse_kernel(const WaveArgs W, uint32_t refill_min) {
    const TraceArgs& A = W.t;
    Cnt<C> cnt;
    const uint32_t total = *W.count_in;
    const int lane = threadIdx.x & 31;
    RayRun s;
    s.slot = kNoIndex;
    bool exhausted = false;
    for (;;) {
        const bool need = s.slot == kNoIndex;
        const unsigned want = __ballot_sync(0xffffffffu, need);
        if (!exhausted && (uint32_t)__popc(want) >= (want == 0xffffffffu ? 1u : refill_min)) {
            const int leader = __ffs(want) - 1;
            uint32_t first = 0;
            if (lane == leader) first = atomicAdd(W.queue_head, (uint32_t)__popc(want));
            first = __shfl_sync(0xffffffffu, first, leader);
            const uint32_t mine = first + __popc(want & ((1u << lane) - 1u));
            if (first + __popc(want) >= total) exhausted = true;
            if (need && mine < total) start_ray<BUDGETED, C>(W, s, W.queue_in[mine], cnt);
        }
        const bool idle = s.slot == kNoIndex;
        const unsigned busy = __ballot_sync(0xffffffffu, !idle);
        if (!busy) {
            if (exhausted) break;
            continue;
        }
        if constexpr (C) {
            if (lane == 0) {
                cnt.wp[exhausted ? 1 : 0] += 1u;
                cnt.lp[exhausted ? 1 : 0] += (uint32_t)__popc(busy);
            }
        }
        // One step per busy lane, in two halves. The first half branches by
        // what the ray's position holds (region lookup, air region, brick,
        // voxel); the warp reconverges before the second, so the box step
        // that most lanes take runs once for all of them. While rays remain
        // queued a grazing lane replays at most 64 steps per pass, so it
        // holds up the warp's other lanes only briefly.
        uint32_t status = kGo, material = 0u;
        I3 voxel{0, 0, 0};
        const uint32_t creep_limit = exhausted ? 0xffffffffu : s.step + 64u;
        if (!idle) classify_step<BUDGETED, C>(W, s, cnt, status, material, voxel);
        __syncwarp();
        if (!idle) finish_step<BUDGETED, C>(W, s, cnt, status, material, voxel, creep_limit);
    }
    flush_counters<C>(A, cnt);
}

// The same traversal over the rays of several scenes at once: scene i's
// WaveArgs (this stage's queue, ray and hit arrays, geometry) is scenes[i],
// and the rays are pulled from the concatenation of the scenes' queues by
// one shared head, so one resident grid keeps busy however uneven the
// scenes are. Each lane keeps the scene of its ray; a step reads that
// scene's arrays, so every ray takes exactly the steps it takes alone.
constexpr uint32_t kMaxBatch = 256;

template <bool BUDGETED>
__global__ void __launch_bounds__(kWaveBlock, VGI_TRAVERSE_MIN_BLOCKS)
    wave_traverse_batch_kernel(const WaveArgs* scenes, uint32_t n_scenes, uint32_t* head, uint32_t refill_min) {
    __shared__ uint32_t first_ray[kMaxBatch + 1];  // prefix sums of the scenes' queue counts
    if (threadIdx.x == 0) {
        uint32_t sum = 0;
        for (uint32_t i = 0; i < n_scenes; ++i) {
            first_ray[i] = sum;
            sum += *scenes[i].count_in;
        }
        first_ray[n_scenes] = sum;
    }
    __syncthreads();
    const uint32_t total = first_ray[n_scenes];
    Cnt<false> cnt;
    const int lane = threadIdx.x & 31;
    RayRun s;
    s.slot = kNoIndex;
    uint32_t scene = 0;
    bool exhausted = false;
    for (;;) {
        const bool need = s.slot == kNoIndex;
        const unsigned want = __ballot_sync(0xffffffffu, need);
        if (!exhausted && (uint32_t)__popc(want) >= (want == 0xffffffffu ? 1u : refill_min)) {
            const int leader = __ffs(want) - 1;
            uint32_t first = 0;
            if (lane == leader) first = atomicAdd(head, (uint32_t)__popc(want));
            first = __shfl_sync(0xffffffffu, first, leader);
            const uint32_t mine = first + __popc(want & ((1u << lane) - 1u));
            if (first + __popc(want) >= total) exhausted = true;
            if (need && mine < total) {
                // The last scene whose first ray is at or before `mine`.
                uint32_t lo = 0, hi = n_scenes - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (first_ray[mid] <= mine) lo = mid;
                    else hi = mid - 1;
                }
                scene = lo;
                const WaveArgs& W = scenes[scene];
                start_ray<BUDGETED, false>(W, s, W.queue_in[mine - first_ray[scene]], cnt);
            }
        }
        const bool idle = s.slot == kNoIndex;
        const unsigned busy = __ballot_sync(0xffffffffu, !idle);
        if (!busy) {
            if (exhausted) break;
            continue;
        }
        uint32_t status = kGo, material = 0u;
        I3 voxel{0, 0, 0};
        const uint32_t creep_limit = exhausted ? 0xffffffffu : s.step + 64u;
        const WaveArgs& W = scenes[scene];
        if (!idle) classify_step<BUDGETED, false>(W, s, cnt, status, material, voxel);
        __syncwarp();
        if (!idle) finish_step<BUDGETED, false>(W, s, cnt, status, material, voxel, creep_limit);
    }
}

// Stage s >= 1: complete the pending hit, then the continuation's new hit
// (one iteration of advance_path, voxel_path.wgsl:432-490).
template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__global__ void __launch_bounds__(kWaveBlock, VGI_SHADE_MIN_BLOCKS) wave_shade_kernel(const WaveArgs W, uint32_t stage) {
    __shared__ float4 smat[512];
    const TraceArgs& A = W.t;
    stage_materials<HITS, LIMITED, BUDGETED, C>(A, smat);
    Cnt<C> cnt;
    WaveTracer<HITS, LIMITED, BUDGETED, C> T{W, A, smat, cnt};
    const uint32_t p = blockIdx.x * kWaveBlock + threadIdx.x;
    const bool in = p < W.n_paths;
    float4 pp = in ? field(W, kPP, p) : make_float4(0, 0, 0, 0);
    uint32_t flags = bits(pp.w);
    const uint32_t base = p * W.slots;
    bool emit_c = false, emit_n = false, emit_d = false, scatter = false, query = false;
    uint32_t scatter_entry = 0;
    V3 dpos{0.0f, 0.0f, 0.0f}, dnrm{0.0f, 0.0f, 0.0f};
    float4 q0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), q1 = q0;
    if (in && (flags & kFlagValid)) {
        float4 e = field(W, kE, p);
        // The receiver's NEE from stage 0.
        if (stage == 1u && (flags & kFlagS0)) {
            float4 n0 = field(W, kN0, p);
            if (W.status[base + 1u] == 0u) cnt.bytes(64);
            else n0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            field(W, kN0, p) = n0;
        }
        if (kind_of(flags) != kKindNone) T.combine(p, flags, V3{pp.x, pp.y, pp.z}, e);
        flags &= ~(kFlagS0 | kFlagN);
        uint32_t pending_kind = kKindNone;
        if (flags & kFlagContinue) {
            flags &= ~kFlagContinue;
            const float4 tpw = field(W, kTP, p);
            const uint32_t bounce = bits(tpw.w);
            const V3 tp{tpw.x, tpw.y, tpw.z};
            const float4 ro = W.ray[2u * base], rd = W.ray[2u * base + 1u];
            const V3 origin{ro.x, ro.y, ro.z}, direction{rd.x, rd.y, rd.z};
            const uint4 h0 = W.hit[(size_t)p * 6u], h1 = W.hit[(size_t)p * 6u + 1u], h2 = W.hit[(size_t)p * 6u + 2u];
            uint32_t status = h0.x;
            if (LIMITED && status == 0u &&
                geometry_ahead(A, origin + direction * T.reach(), direction, direction_recip(direction), __fsub_rn(A.max_distance, T.reach()), cnt))
                status = 3u;
            if (status == 0u) {
                float horizon = wclamp(__fadd_rn(__fmul_rn(direction.y, 0.35f), 0.65f), 0.15f, 1.0f);
                V3 en = V3{e.x, e.y, e.z} + (tp * V3{A.env[0], A.env[1], A.env[2]}) * horizon;
                e.x = en.x;
                e.y = en.y;
                e.z = en.z;
            } else if (status == 2u) {
                flags |= kFlagUnknown;
            } else if (status == 1u) {
                const V3 hp{fl(h1.y), fl(h1.z), fl(h1.w)}, hn{fl(h2.x), fl(h2.y), fl(h2.z)};
                const I3 hv{(int)h0.z, (int)h0.w, (int)h1.x};
                cnt.bytes(64);
                const Mat m = T.material_nocount(h0.y);
                const V3 previous_position{pp.x, pp.y, pp.z}, previous_normal = normal_of(flags);
                const float previous_pdf = e.w;
                // direct_at's rays from the hit.
                emit_d = true;
                const float emission_weight = m.weight;
                const V3 delta = hp - origin;
                float selection_pdf = __fdiv_rn(emission_weight, wmax(A.emitter_total, 1e-20f));
                if (emission_weight > 0.0f && A.emitter_count > 0.0f && load_emitter(A, 0u, cnt).sampling.w > 0.0f)
                    selection_pdf = tree_probability(A, previous_position, previous_normal, hv, hn, cnt);
                const float light_pdf = __fdiv_rn(__fmul_rn(selection_pdf, dot3(delta, delta)), wmax(dot3(hn, -direction), 1e-8f));
                float mis = 1.0f;
                if (light_pdf > 0.0f) mis = __fdiv_rn(previous_pdf, __fadd_rn(previous_pdf, light_pdf));
                const V3 diffuse{m.diffuse.x, m.diffuse.y, m.diffuse.z};
                V3 cached;
                V3 xval{0.0f, 0.0f, 0.0f};
                bool have_cache = false;
                {
                    // cached_energy (voxel_path.wgsl:66-87)
                    const uint32_t f = face_index_of(hn);
                    if (f <= 5u && A.face_index != nullptr) {
                        const uint4 header = __ldg(A.face_index);
                        uint32_t s = (hash_voxel(hv.x, hv.y, hv.z) ^ pcg(f + 1u)) & header.x;
#pragma unroll 1
                        for (uint32_t attempt = 0; attempt < header.y; ++attempt) {
                            const uint4 ent = __ldg(A.face_index + s + 1u);
                            cnt.bytes(16);
                            if (ent.w == 0xffffffffu) break;
                            if ((int)ent.x == hv.x && (int)ent.y == hv.y && (int)ent.z == hv.z && (ent.w >> 29u) == f) {
                                const float4 rec = __ldg(A.cache + (ent.w & 0x1fffffffu));
                                cnt.bytes(16);
                                const uint32_t count = __float_as_uint(rec.w);
                                if (!(count < 16u || (count & 0x80000000u) != 0u)) {
                                    cached = V3{rec.x, rec.y, rec.z};
                                    have_cache = true;
                                }
                                break;
                            }
                            s = (s + 1u) & header.x;
                        }
                    }
                }
                if (have_cache) {
                    cnt.cache_hit();
                    pending_kind = kKindCached;
                    xval = cached;
                } else if (W.mlp_queue != nullptr) {
                    // The network's prediction for the hit face replaces the
                    // cache value; the query kernel writes it into kX.
                    pending_kind = kKindCached;
                    query = true;
                    const V3 centre = add_s(itof(hv), 0.5f) + hn * 0.5f;
                    q0 = make_float4(centre.x, centre.y, centre.z, fl(p));
                    q1 = make_float4(diffuse.x, diffuse.y, diffuse.z, fl(face_index_of(hn)));
                } else {
                    // NEE or the terminal connection, and the continuation,
                    // run in wave_scatter_kernel over the paths queued here.
                    pending_kind = kKindNee;
                    scatter = true;
                    scatter_entry = p | (bounce << 30);
                }
                // The hit's emission * mis and diffuse come from its material
                // and the weight kept here (combine).
                field(W, kTH, p) = make_float4(tp.x, tp.y, tp.z, mis);
                field(W, kX, p) = make_float4(xval.x, xval.y, xval.z, 0.0f);
                flags = with_material(with_normal(flags, hn), h0.y);
                pp = make_float4(hp.x, hp.y, hp.z, 0.0f);
                dpos = hp;
                dnrm = hn;
            }
        }
        flags = with_kind(flags, pending_kind);
        field(W, kE, p) = e;
        pp.w = fl(flags);
        field(W, kPP, p) = pp;
    }
    // Warp-collective from here on: every thread takes part.
    T.emit_direct(dpos, dnrm, base + 2u, emit_d);  // direct_at's rays from the hit point
    enqueue(W, emit_n, base + 1u);
    enqueue(W, emit_c, base);
    {
        const unsigned mask = __ballot_sync(0xffffffffu, scatter);
        if (mask) {
            const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
            uint32_t first = 0;
            if (lane == leader) first = atomicAdd(W.scatter_count, (uint32_t)__popc(mask));
            first = __shfl_sync(0xffffffffu, first, leader);
            if (scatter) W.scatter_queue[first + __popc(mask & ((1u << lane) - 1u))] = scatter_entry;
        }
    }
    if (W.mlp_queue != nullptr) {
        const unsigned mask = __ballot_sync(0xffffffffu, query);
        if (mask) {
            const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
            uint32_t first = 0;
            if (lane == leader) first = atomicAdd(W.mlp_count, (uint32_t)__popc(mask));
            first = __shfl_sync(0xffffffffu, first, leader);
            if (query) {
                const uint32_t k = first + __popc(mask & ((1u << lane) - 1u));
                W.mlp_queue[2u * k] = q0;
                W.mlp_queue[2u * k + 1u] = q1;
            }
        }
    }
    flush_counters<C>(A, cnt);
}

// The rest of an uncached hit (advance_path, voxel_path.wgsl:464-489) for the
// paths wave_shade_kernel queued: the emitter NEE, or on the last hit
// sample_terminal_emission's connection, then roulette and the continuation.
// Queue entries are path | bounce << 30; warps stride over the queue.
template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__global__ void __launch_bounds__(kWaveBlock, VGI_SCATTER_MIN_BLOCKS) wave_scatter_kernel(const WaveArgs W) {
    __shared__ float4 smat[512];
    const TraceArgs& A = W.t;
    stage_materials<HITS, LIMITED, BUDGETED, C>(A, smat);
    Cnt<C> cnt;
    WaveTracer<HITS, LIMITED, BUDGETED, C> T{W, A, smat, cnt};
    const uint32_t total = *W.scatter_count;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (kWaveBlock / 32);
    for (uint32_t first = (blockIdx.x * kWaveBlock + threadIdx.x) - lane; first < total; first += warps * 32u) {
        const uint32_t k = first + lane;
        const bool active = k < total;
        const uint32_t entry = active ? W.scatter_queue[k] : 0u;
        const uint32_t p = entry & 0x3fffffffu, bounce = entry >> 30;
        const uint32_t base = p * W.slots;
        bool emit_n = false, emit_c = false;
        if (active) {
            const float4 pp = field(W, kPP, p), th = field(W, kTH, p);
            uint32_t flags = bits(pp.w);
            const Mat mat = T.material_nocount(material_of(flags));
            const V3 hp{pp.x, pp.y, pp.z}, hn = normal_of(flags), tp{th.x, th.y, th.z};
            const V3 diffuse{mat.diffuse.x, mat.diffuse.y, mat.diffuse.z};
            const uint32_t face = p / A.samples, sample = p - face * A.samples;
            const uint4 t0 = __ldg(A.tasks + face * 2u), t1 = __ldg(A.tasks + face * 2u + 1u);
            const uint32_t pstream = hash_voxel((int)t0.x, (int)t0.y, (int)t0.z) ^ pcg(t0.w + 1u);
            const uint32_t sequence = t1.x + sample;
            const bool last = bounce + 1u == HITS;
            uint32_t kind = kKindNee;
            V3 so, sd, pend{0.0f, 0.0f, 0.0f};
            float sdist = 0.0f;
            if (last) {
                // sample_terminal_emission (voxel_path.wgsl:368-394)
                if (A.emitter_count != 0.0f) {
                    if (continuation_sample(pstream, sequence, bounce, 2u) < 0.5f) {
                        kind = kKindTermEmitter;
                        emit_n = T.prepare_nee(hp, hn, pstream, sequence, bounce + 1u, so, sd, sdist, pend);
                        if (emit_n) put_ray(W, base + 1u, so, sd, sdist, 0u);
                    } else {
                        kind = kKindTermCosine;
                        const V3 tdir =
                            hemisphere(hn, continuation_sample(pstream, sequence, bounce, 0u), continuation_sample(pstream, sequence, bounce, 1u));
                        if (dot3(hn, tdir) > 0.0f) {
                            emit_n = true;
                            put_ray(W, base + 1u, hp + hn * 0.002f, tdir, T.reach(), hit_of(p, 1u));
                        }
                    }
                }
            } else {
                emit_n = T.prepare_nee(hp, hn, pstream, sequence, bounce + 1u, so, sd, sdist, pend);
                if (emit_n) put_ray(W, base + 1u, so, sd, sdist, 0u);
                // The continuation (voxel_path.wgsl:472-489).
                V3 tn = tp * diffuse;
                const float maximum = wmax(tn.x, wmax(tn.y, tn.z));
                bool go = maximum != 0.0f;
                if (go && bounce >= 1u) {
                    const float survival = wclamp(maximum, 0.1f, 0.95f);
                    if (continuation_sample(pstream, sequence, bounce, 2u) > survival) go = false;
                    else tn = tn / survival;
                }
                if (go) {
                    const V3 ndir = hemisphere(hn, continuation_sample(pstream, sequence, bounce, 0u), continuation_sample(pstream, sequence, bounce, 1u));
                    const float npdf = cosine_pdf(hn, ndir);
                    float4 e = field(W, kE, p);
                    e.w = npdf;
                    field(W, kE, p) = e;
                    if (npdf > 0.0f) {
                        emit_c = true;
                        flags |= kFlagContinue;
                        put_ray(W, base, hp + hn * 0.002f, ndir, T.reach(), hit_of(p, 0u));
                        field(W, kTP, p) = make_float4(tn.x, tn.y, tn.z, fl(bounce + 1u));
                    }
                }
            }
            if (emit_n) flags |= kFlagN;
            // kTH (the throughput at this hit and its MIS weight) stays.
            field(W, kX, p) = make_float4(pend.x, pend.y, pend.z, 0.0f);
            field(W, kPP, p) = make_float4(pp.x, pp.y, pp.z, fl(with_kind(flags, kind)));
        }
        enqueue(W, emit_n, base + 1u);
        enqueue(W, emit_c, base);
    }
    flush_counters<C>(A, cnt);
}

// Completes each path's last pending hit, then trace_moments + write_result
// (voxel_trace.wgsl:25-92) with the same lane layout as trace_faces_kernel:
// one thread per (face, lane), lanes summing strided samples, lane 0 summing
// the lanes in order.
template <uint32_t HITS, bool LIMITED, bool BUDGETED, bool C>
__global__ void __launch_bounds__(kWaveBlock, VGI_FINALIZE_MIN_BLOCKS) wave_finalize_kernel(const WaveArgs W) {
    __shared__ float4 smat[512];
    const TraceArgs& A = W.t;
    stage_materials<HITS, LIMITED, BUDGETED, C>(A, smat);
    Cnt<C> cnt;
    WaveTracer<HITS, LIMITED, BUDGETED, C> T{W, A, smat, cnt};
    const uint32_t lanes = 1u << A.lanes_log2;
    const uint32_t gid = blockIdx.x * kWaveBlock + threadIdx.x;
    const uint32_t face = gid >> A.lanes_log2;
    const uint32_t lane = gid & (lanes - 1u);
    uint4 t0 = make_uint4(0, 0, 0, 0xffffffffu);
    if (face < A.n_tasks) t0 = __ldg(A.tasks + face * 2u);
    const bool valid = face < A.n_tasks && t0.w != 0xffffffffu;
    V3 mean{0.0f, 0.0f, 0.0f}, second{0.0f, 0.0f, 0.0f};
    uint32_t known = 0;
    if (valid) {
#pragma unroll 1
        for (uint32_t i = lane; i < A.samples; i += lanes) {
            const uint32_t p = face * A.samples + i;
            const float4 pp = field(W, kPP, p);
            const uint32_t flags = bits(pp.w);
            float4 e = field(W, kE, p);
            if (kind_of(flags) != kKindNone) T.combine(p, flags, V3{pp.x, pp.y, pp.z}, e);
            if (flags & kFlagUnknown) {
                cnt.unknown();
                continue;
            }
            const float4 n0 = field(W, kN0, p);
            V3 value{n0.x, n0.y, n0.z};
            if (flags & kFlagRan) value = value + V3{e.x, e.y, e.z};
            mean = mean + value;
            second = second + value * value;
            known += 1u;
        }
    }
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
        const V3 normal = face_normal(t0.w);
        const V3 surface = add_s(itof(I3{(int)t0.x, (int)t0.y, (int)t0.z}), 0.5f) + normal * 0.5f;
        V3 dc;
        float dw = 0.0f;
        const V3 dv = T.template gather_direct<true>(surface, normal, W.n_paths * W.slots + face * A.light_count, &dc, &dw);
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
    flush_counters<C>(A, cnt);
}

template <uint32_t H, bool L, bool B, bool C>
void wave_run(const WaveBuffers& b, const TraceArgs& a, cudaStream_t s) {
    WaveArgs W{};
    W.t = a;
    W.n_paths = a.n_tasks * a.samples;
    W.slots = 2u + a.light_count;
    W.state = b.state;
    W.ray = b.ray;
    W.status = b.status;
    W.hit = b.hit;
    W.queue_head = b.counters + 2;
    W.scatter_queue = b.scatter;
    W.scatter_count = b.counters + 3;
    W.mlp_queue = b.mlp_image ? b.mlp_queue : nullptr;
    W.mlp_count = b.counters + 4;
    const uint32_t path_blocks = (W.n_paths + kWaveBlock - 1) / kWaveBlock;
    const uint32_t face_blocks = (uint32_t)((((uint64_t)a.n_tasks << a.lanes_log2) + kWaveBlock - 1) / kWaveBlock);
    uint32_t* qa = b.queue[0];
    uint32_t* qb = b.queue[1];
    uint32_t* ca = b.counters + 0;
    uint32_t* cb = b.counters + 1;
    cudaMemsetAsync(ca, 0, sizeof(uint32_t), s);
    W.queue_out = qa;
    W.count_out = ca;
    wave_begin_kernel<H, L, B, C><<<path_blocks, kWaveBlock, 0, s>>>(W);
    for (uint32_t stage = 1; stage <= H + 1u; ++stage) {
        // Traverse what the previous stage queued.
        W.queue_in = qa;
        W.count_in = ca;
        cudaMemsetAsync(W.queue_head, 0, sizeof(uint32_t), s);
        if (b.traverse_marks && stage <= 4u) cudaEventRecord(b.traverse_marks[2u * (stage - 1u)], s);
        wave_traverse_kernel<B, C><<<b.traverse_blocks, kWaveBlock, 0, s>>>(W, b.refill_min);
        if (b.traverse_marks && stage <= 4u) cudaEventRecord(b.traverse_marks[2u * (stage - 1u) + 1u], s);
        if (stage == H + 1u) break;
        cudaMemsetAsync(cb, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(W.scatter_count, 0, sizeof(uint32_t), s);
        W.queue_out = qb;
        W.count_out = cb;
        if (W.mlp_queue) cudaMemsetAsync(W.mlp_count, 0, sizeof(uint32_t), s);
        wave_shade_kernel<H, L, B, C><<<path_blocks, kWaveBlock, 0, s>>>(W, stage);
        if (W.mlp_queue) {
            // One diffuse hit: the queued hits take the network's value.
            if (b.mlp_marks) cudaEventRecord(b.mlp_marks[0], s);
            launch_mlp_queries(W.mlp_queue, W.mlp_count, W.n_paths, b.mlp_image, b.mlp_enc, W.state + (size_t)kX * W.n_paths, b.mlp_error,
                               b.mlp_ctas, s, b.mlp_wait);
            if (b.mlp_marks) cudaEventRecord(b.mlp_marks[1], s);
        } else {
            wave_scatter_kernel<H, L, B, C><<<b.traverse_blocks, kWaveBlock, 0, s>>>(W);
        }
        uint32_t* t = qa; qa = qb; qb = t;
        t = ca; ca = cb; cb = t;
    }
    wave_finalize_kernel<H, L, B, C><<<face_blocks, kWaveBlock, 0, s>>>(W);
}

template <uint32_t H>
void wave_hits(const WaveBuffers& b, const TraceArgs& a, bool limited, bool budgeted, bool count, cudaStream_t s) {
#define VGI_WAVE(LL, BB)                                      \
    if (count) wave_run<H, LL, BB, true>(b, a, s);            \
    else wave_run<H, LL, BB, false>(b, a, s);
    if (limited) {
        if (budgeted) { VGI_WAVE(true, true) } else { VGI_WAVE(true, false) }
    } else {
        if (budgeted) { VGI_WAVE(false, true) } else { VGI_WAVE(false, false) }
    }
#undef VGI_WAVE
}

// One scene's WaveArgs for stage k (1-based) of a frame: the queues
// alternate between the two buffers stage after stage, as in wave_run.
WaveArgs stage_args(const WaveBuffers& b, const TraceArgs& a, uint32_t k) {
    WaveArgs W{};
    W.t = a;
    W.n_paths = a.n_tasks * a.samples;
    W.slots = 2u + a.light_count;
    W.state = b.state;
    W.ray = b.ray;
    W.status = b.status;
    W.hit = b.hit;
    W.queue_head = b.counters + 2;
    W.scatter_queue = b.scatter;
    W.scatter_count = b.counters + 3;
    W.mlp_queue = nullptr;
    W.mlp_count = b.counters + 4;
    const bool odd = (k & 1u) != 0u;  // k = 0: begin writes the first stage's queue
    W.queue_in = odd ? b.queue[0] : b.queue[1];
    W.count_in = odd ? b.counters + 0 : b.counters + 1;
    W.queue_out = odd ? b.queue[1] : b.queue[0];
    W.count_out = odd ? b.counters + 1 : b.counters + 0;
    if (k == 0) {
        W.queue_out = b.queue[0];
        W.count_out = b.counters + 0;
    }
    return W;
}

// The node the last launch on a capturing stream added (null when the
// stream is not capturing).
cudaGraphNode_t last_node(cudaStream_t s) {
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t* deps = nullptr;
    size_t n = 0;
    if (cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &n) != cudaSuccess || status != cudaStreamCaptureStatusActive ||
        n != 1)
        return nullptr;
    return deps[0];
}

// Each scene's own kernels run on its side stream, so the scenes' small
// kernels overlap; the side streams join the main stream for each stage's
// batched traversal and fork from it afterwards.
template <uint32_t H, bool L, bool B>
void wave_batch_run(const WaveScene* sc, uint32_t n, const WaveArgs* device_args, const BatchStreams& st, const AccumArgs* acc,
                    cudaGraphNode_t* prepare_nodes, cudaGraphNode_t* accumulate_nodes) {
    auto fork = [&]() {
        cudaEventRecord(st.fork, st.main);
        for (uint32_t i = 0; i < n; ++i) cudaStreamWaitEvent(st.side[i], st.fork, 0);
    };
    auto join = [&]() {
        for (uint32_t i = 0; i < n; ++i) {
            cudaEventRecord(st.join[i], st.side[i]);
            cudaStreamWaitEvent(st.main, st.join[i], 0);
        }
    };
    fork();
    for (uint32_t i = 0; i < n; ++i) {
        const cudaStream_t s = st.side[i];
        if (acc) {
            launch_prepare(acc[i], s);
            if (prepare_nodes) prepare_nodes[i] = last_node(s);
        }
        const WaveArgs W = stage_args(sc[i].b, sc[i].a, 0);
        cudaMemsetAsync(W.count_out, 0, sizeof(uint32_t), s);
        wave_begin_kernel<H, L, B, false><<<(W.n_paths + kWaveBlock - 1) / kWaveBlock, kWaveBlock, 0, s>>>(W);
    }
    for (uint32_t stage = 1; stage <= H + 1u; ++stage) {
        join();
        cudaMemsetAsync(st.head, 0, sizeof(uint32_t), st.main);
        wave_traverse_batch_kernel<B><<<st.blocks, kWaveBlock, 0, st.main>>>(device_args + (size_t)(stage - 1u) * n, n, st.head, st.refill_min);
        fork();
        for (uint32_t i = 0; i < n; ++i) {
            const cudaStream_t s = st.side[i];
            WaveArgs W = stage_args(sc[i].b, sc[i].a, stage);
            if (stage <= H) {
                cudaMemsetAsync(W.count_out, 0, sizeof(uint32_t), s);
                cudaMemsetAsync(W.scatter_count, 0, sizeof(uint32_t), s);
                if (st.mlp_scenes) {
                    // Uncached first hits queue for the network (one query
                    // launch over every scene below), as wave_run's shade.
                    W.mlp_queue = sc[i].b.mlp_queue;
                    cudaMemsetAsync(W.mlp_count, 0, sizeof(uint32_t), s);
                }
                wave_shade_kernel<H, L, B, false><<<(W.n_paths + kWaveBlock - 1) / kWaveBlock, kWaveBlock, 0, s>>>(W, stage);
                if (!st.mlp_scenes) wave_scatter_kernel<H, L, B, false><<<sc[i].b.traverse_blocks, kWaveBlock, 0, s>>>(W);
            } else {
                const uint32_t face_blocks = (uint32_t)((((uint64_t)sc[i].a.n_tasks << sc[i].a.lanes_log2) + kWaveBlock - 1) / kWaveBlock);
                wave_finalize_kernel<H, L, B, false><<<face_blocks, kWaveBlock, 0, s>>>(W);
                if (acc) {
                    launch_accumulate(acc[i], s);
                    if (accumulate_nodes) accumulate_nodes[i] = last_node(s);
                }
            }
        }
        if (st.mlp_scenes && stage <= H) {
            // Every scene's queued hits take their network's prediction in
            // one launch.
            join();
            launch_mlp_scene_queries(st.mlp_scenes, st.mlp_n, st.mlp_ctas, st.main, st.mlp_wait);
            fork();
        }
    }
    join();
}

}  // namespace

uint32_t wave_batch_stages(uint32_t hits) { return (hits <= 1 ? 1u : hits > 3 ? 3u : hits) + 1u; }

size_t wave_args_bytes() { return sizeof(WaveArgs); }

void wave_batch_args(const WaveScene* sc, uint32_t n, uint32_t hits, void* out) {
    WaveArgs* dst = static_cast<WaveArgs*>(out);
    const uint32_t stages = wave_batch_stages(hits);
    for (uint32_t k = 1; k <= stages; ++k)
        for (uint32_t i = 0; i < n; ++i) dst[(size_t)(k - 1u) * n + i] = stage_args(sc[i].b, sc[i].a, k);
}

void launch_wave_batch(const WaveScene* sc, uint32_t n, const void* args, uint32_t hits, bool limited, bool budgeted,
                       const BatchStreams& st, const AccumArgs* acc, cudaGraphNode_t* prepare_nodes, cudaGraphNode_t* accumulate_nodes) {
    if (n == 0 || n > kMaxBatch) return;
    const WaveArgs* device_args = static_cast<const WaveArgs*>(args);
    const uint32_t h = hits <= 1 ? 1u : hits > 3 ? 3u : hits;
#define VGI_BATCH(HH, LL, BB) wave_batch_run<HH, LL, BB>(sc, n, device_args, st, acc, prepare_nodes, accumulate_nodes)
    if (h == 1) {
        if (limited) { if (budgeted) VGI_BATCH(1, true, true); else VGI_BATCH(1, true, false); }
        else { if (budgeted) VGI_BATCH(1, false, true); else VGI_BATCH(1, false, false); }
    } else if (h == 2) {
        if (limited) { if (budgeted) VGI_BATCH(2, true, true); else VGI_BATCH(2, true, false); }
        else { if (budgeted) VGI_BATCH(2, false, true); else VGI_BATCH(2, false, false); }
    } else {
        if (limited) { if (budgeted) VGI_BATCH(3, true, true); else VGI_BATCH(3, true, false); }
        else { if (budgeted) VGI_BATCH(3, false, true); else VGI_BATCH(3, false, false); }
    }
#undef VGI_BATCH
}

void launch_wave(const WaveBuffers& b, const TraceArgs& a, uint32_t hits, bool limited, bool budgeted, bool count, cudaStream_t s) {
    if (a.n_tasks == 0 || a.samples == 0) return;
    if (b.mlp_image) hits = 1;  // the network ends paths at the first hit
    if (hits <= 1) wave_hits<1>(b, a, limited, budgeted, count, s);
    else if (hits == 2) wave_hits<2>(b, a, limited, budgeted, count, s);
    else wave_hits<3>(b, a, limited, budgeted, count, s);
}

uint32_t wave_traverse_blocks_per_sm() {
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, wave_traverse_kernel<false, false>, kWaveBlock, 0);
    return blocks > 0 ? (uint32_t)blocks : 1u;
}

}  // namespace vgi
