// View tier of the face trace (included by vgi_trace.cu, so it shares the
// estimator). Behaviour follows (paths within
// nathanaelneveux/global-illumination, crates/bevy_voxel_gi/shaders/):
//   voxel_view_trace.wgsl:40-72      trace_view_paths
//   voxel_view_trace.wgsl:106-183    advance_view_path (pause/resume, tickets)
//   voxel_view_runtime.wgsl:272-349  trace_visible_paths, retain_view_history
//   voxel_view_cache.wgsl:6-98       shared_slot, load_shared_face
//   voxel_view_cache.wgsl:225-258    store_shared_faces
//   voxel_path.wgsl:418-496          begin_path / advance_path with an explicit
//                                    state, a hit budget and a terminal flag
//
// The caller gives the receivers (one per visible unit face), so every
// receiver owns itself and the owner queue is receiver order; raster
// discovery, reprojection across views and sun-corner records are not part
// of this path. Records keep the shaders'
// layouts (uint4 words): ViewReceiver 2, ViewPath 8, ViewContinuation 8,
// ViewEstimate 4. One thread runs one owner's visits, as the shader does.

namespace vgi {
namespace {

constexpr uint32_t kViewOwners = 0, kViewCompleted = 2, kViewKnown = 3, kViewAttempted = 9, kViewLoads = 10, kViewPromotions = 11,
                   kViewPrefix = 12;

__device__ __forceinline__ V3 f3w(uint4 w) { return V3{__uint_as_float(w.x), __uint_as_float(w.y), __uint_as_float(w.z)}; }
__device__ __forceinline__ uint4 w3(V3 v, uint32_t w) { return make_uint4(__float_as_uint(v.x), __float_as_uint(v.y), __float_as_uint(v.z), w); }
__device__ __forceinline__ uint4 wi3(I3 v, uint32_t w) { return make_uint4((uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z, w); }

// PathState (voxel_path.wgsl:406-416). Spectra carry a fourth component
// that is zero for every record the host builds (spectrum_vec); energy.w
// then stays +0 and throughput.w is 1 until the first diffuse factor, then +0.
struct ViewPathState {
    V3 energy;
    float energy_w;
    bool unknown;
    Ray first;
    V3 tp;
    float tp_w;
    V3 origin, direction, previous_position, previous_normal;
    float previous_pdf;
    uint32_t bounce;
    bool done;
};

// begin_path (voxel_path.wgsl:418-428)
__device__ ViewPathState view_begin(V3 start, V3 direction, V3 normal) {
    ViewPathState s;
    s.energy = V3{0.0f, 0.0f, 0.0f};
    s.energy_w = 0.0f;
    s.unknown = false;
    s.first = Ray{I3{0, 0, 0}, 0u, V3{0.0f, 0.0f, 0.0f}, 0u, V3{0.0f, 0.0f, 0.0f}};
    s.tp = V3{1.0f, 1.0f, 1.0f};
    s.tp_w = 1.0f;
    s.origin = start;
    s.direction = direction;
    s.previous_normal = normal;
    s.previous_pdf = cosine_pdf(normal, direction);
    s.previous_position = start - normal * 0.001f;
    s.bounce = 0;
    s.done = s.previous_pdf <= 0.0f;
    return s;
}

// advance_path (voxel_path.wgsl:429-492): up to `steps` hits; with
// `terminal` the last of them takes the terminal emission mixture.
template <bool LIMITED, bool BUDGETED>
__device__ void view_advance(Tracer<1, LIMITED, BUDGETED, false>& T, ViewPathState& s, uint32_t stream, uint32_t sequence,
                             uint32_t steps, bool terminal) {
    const TraceArgs& A = T.A;
    if (s.done) return;
#pragma unroll 1
    for (uint32_t step = 0; step < steps; ++step) {
        const uint32_t bounce = s.bounce;
        s.done = true;
        Ray hit = T.trace_diffuse(s.origin, s.direction);
        if (bounce == 0u) s.first = hit;
        if (hit.status == 0u) {
            float horizon = wclamp(__fadd_rn(__fmul_rn(s.direction.y, 0.35f), 0.65f), 0.15f, 1.0f);
            s.energy = s.energy + (s.tp * V3{A.env[0], A.env[1], A.env[2]}) * horizon;
            s.energy_w = __fadd_rn(s.energy_w, __fmul_rn(__fmul_rn(s.tp_w, A.env[3]), horizon));
            break;
        }
        if (hit.status == 2u) {
            s.unknown = true;
            break;
        }
        if (hit.status == 3u) break;
        Mat m = T.material(hit.material);
        V3 direct, unused;
        T.template direct_at<false>(hit.position, hit.normal, direct, unused);
        const float emission_weight = m.weight;
        const V3 delta = hit.position - s.origin;
        float selection_pdf = __fdiv_rn(emission_weight, wmax(A.emitter_total, 1e-20f));
        if (emission_weight > 0.0f && A.emitter_count > 0.0f && load_emitter(A, 0u, T.cnt).sampling.w > 0.0f)
            selection_pdf = tree_probability(A, s.previous_position, s.previous_normal, hit.voxel, hit.normal, T.cnt);
        const float light_pdf = __fdiv_rn(__fmul_rn(selection_pdf, dot3(delta, delta)), wmax(dot3(hit.normal, -s.direction), 1e-8f));
        float mis = 1.0f;
        if (light_pdf > 0.0f) mis = __fdiv_rn(s.previous_pdf, __fadd_rn(s.previous_pdf, light_pdf));
        const V3 emission{m.emission.x, m.emission.y, m.emission.z}, diffuse{m.diffuse.x, m.diffuse.y, m.diffuse.z};
        V3 cached;
        if (T.cached_energy(hit.voxel, face_index_of(hit.normal), cached)) {
            s.energy = s.energy + s.tp * (emission * mis + diffuse * (direct + cached));
            s.energy_w = __fadd_rn(s.energy_w, __fmul_rn(s.tp_w, 0.0f));
            break;
        }
        const bool last = terminal && step + 1u == steps;
        const V3 nee = last ? T.sample_terminal_emission(hit.position, hit.normal, stream, sequence, bounce)
                            : T.sample_emitter(hit.position, hit.normal, stream, sequence, bounce + 1u);
        s.energy = s.energy + s.tp * (emission * mis + diffuse * (direct + nee));
        s.energy_w = __fadd_rn(s.energy_w, __fmul_rn(s.tp_w, 0.0f));
        if (last) break;
        s.tp = s.tp * diffuse;
        s.tp_w = __fmul_rn(s.tp_w, 0.0f);
        const float maximum = wmax(s.tp.x, wmax(s.tp.y, s.tp.z));
        if (maximum == 0.0f) break;
        if (bounce >= 1u) {
            const float survival = wclamp(maximum, 0.1f, 0.95f);
            if (continuation_sample(stream, sequence, bounce, 2u) > survival) break;
            s.tp = s.tp / survival;
            s.tp_w = __fdiv_rn(s.tp_w, survival);
        }
        s.origin = hit.position + hit.normal * 0.002f;
        s.previous_position = hit.position;
        s.previous_normal = hit.normal;
        s.direction = hemisphere(hit.normal, continuation_sample(stream, sequence, bounce, 0u), continuation_sample(stream, sequence, bounce, 1u));
        s.previous_pdf = cosine_pdf(hit.normal, s.direction);
        if (s.previous_pdf <= 0.0f) break;
        s.bounce += 1u;
        s.done = false;
    }
}

template <bool LIMITED, bool BUDGETED>
__device__ __forceinline__ void view_stage_materials(const TraceArgs& A, float4* smat) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        float4 d = __ldg(A.materials + i * 4), e = __ldg(A.materials + i * 4 + 2), x = __ldg(A.materials + i * 4 + 3);
        smat[i * 2] = make_float4(d.x, d.y, d.z, x.y);
        smat[i * 2 + 1] = make_float4(e.x, e.y, e.z, 0.0f);
    }
    __syncthreads();
}

// trace_view_paths (voxel_view_trace.wgsl:40-72): one record per
// (receiver, sample), the receiver sample with its first hit kept.
template <bool LIMITED, bool BUDGETED>
__global__ void __launch_bounds__(kBlock) view_trace_paths_kernel(const ViewArgs V, uint32_t samples, uint4* out) {
    __shared__ float4 smat[512];
    const TraceArgs& A = V.t;
    view_stage_materials<LIMITED, BUDGETED>(A, smat);
    Cnt<false> cnt;
    Tracer<1, LIMITED, BUDGETED, false> T{A, smat, cnt};
    const uint64_t id = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (id >= (uint64_t)V.n * samples) return;
    uint4* record = out + id * 8u;
    const uint4 r0 = V.receivers[(id / samples) * 2u], r1 = V.receivers[(id / samples) * 2u + 1u];
    const V3 surface = f3w(r0);
    const I3 voxel{(int)r1.x, (int)r1.y, (int)r1.z};
    const uint32_t face = r0.w;
    const V3 normal = face_normal(face);
    const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u);
    const uint32_t sequence = r1.w + (uint32_t)(id % samples);
    const V3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
    const V3 emitter = T.sample_emitter(surface, normal, stream, sequence, 0u);
    ViewPathState s = view_begin(surface + normal * 0.001f, direction, normal);
    bool unknown = false;
    if (dot3(normal, direction) > 0.0f) {
        view_advance<LIMITED, BUDGETED>(T, s, stream, sequence, V.hits, true);
        unknown = s.unknown;
    } else {
        s.energy = V3{0.0f, 0.0f, 0.0f};
        s.first = Ray{I3{0, 0, 0}, 0u, V3{0.0f, 0.0f, 0.0f}, 0u, V3{0.0f, 0.0f, 0.0f}};
    }
    V3 direct, unused;
    T.template direct_at<false>(surface, normal, direct, unused);
    record[0] = w3(surface, sequence);
    record[1] = wi3(voxel, face);
    record[2] = w3(direction, __float_as_uint(cosine_pdf(normal, direction)));
    record[3] = w3(s.first.position, s.first.status);
    record[4] = wi3(s.first.voxel, face_index_of(s.first.normal));
    record[5] = w3(emitter, unknown ? 0u : 1u);
    record[6] = w3(s.energy, s.first.material);
    record[7] = w3(direct, stream);
}

// advance_view_path (voxel_view_trace.wgsl:106-183), one path per receiver.
template <bool LIMITED, bool BUDGETED>
__device__ void advance_view_path(Tracer<1, LIMITED, BUDGETED, false>& T, const ViewArgs& V, uint32_t index) {
    uint4* record = V.paths + (size_t)index * 8u;
    uint4* stored = V.conts + (size_t)index * 8u;
    const uint4 r0 = V.receivers[index * 2u], r1 = V.receivers[index * 2u + 1u];
    const V3 surface = f3w(r0);
    const I3 voxel{(int)r1.x, (int)r1.y, (int)r1.z};
    const uint32_t face = r0.w;
    const V3 normal = face_normal(face);
    const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u);
    const uint32_t sequence = r1.w;
    const uint32_t status = stored[4].w;
    const uint4 ticket = stored[7];
    const uint4 p0 = record[0], p1 = record[1];
    bool restart = status == 0u || status == 4u || ticket.x != V.ticket[0] || ticket.y != V.ticket[1] || ticket.z != V.ticket[2] ||
                   ticket.w != V.ticket[3];
    restart = restart || __uint_as_float(p0.x) != surface.x || __uint_as_float(p0.y) != surface.y || __uint_as_float(p0.z) != surface.z;
    restart = restart || (int)p1.x != voxel.x || (int)p1.y != voxel.y || (int)p1.z != voxel.z || p1.w != face || p0.w != sequence;
    ViewPathState s;
    uint4 rec[8];
    if (restart) {
        const V3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
        const V3 emitter = T.sample_emitter(surface, normal, stream, sequence, 0u);
        V3 direct, unused;
        T.template direct_at<false>(surface, normal, direct, unused);
        rec[0] = w3(surface, sequence);
        rec[1] = wi3(voxel, face);
        rec[2] = w3(direction, __float_as_uint(cosine_pdf(normal, direction)));
        rec[3] = make_uint4(0u, 0u, 0u, 0u);
        rec[4] = make_uint4(0u, 0u, 0u, 0u);
        rec[5] = w3(emitter, 0u);
        rec[6] = make_uint4(0u, 0u, 0u, 0u);
        rec[7] = w3(direct, stream);
        s = view_begin(surface + normal * 0.001f, direction, normal);
    } else {
        if (status != 1u) return;
        for (int i = 0; i < 8; ++i) rec[i] = record[i];
        const uint4 c0 = stored[0], c1 = stored[1], c2 = stored[2], c3 = stored[3], c4 = stored[4], c5 = stored[5], c6 = stored[6];
        s.energy = f3w(c0);
        s.energy_w = __uint_as_float(c0.w);
        s.unknown = false;
        s.first.voxel = I3{(int)rec[4].x, (int)rec[4].y, (int)rec[4].z};
        s.first.material = rec[6].w;
        s.first.position = f3w(rec[3]);
        s.first.status = rec[3].w;
        s.first.normal = rec[4].w < 6u ? face_normal(rec[4].w) : V3{0.0f, 0.0f, 0.0f};
        s.tp = f3w(c2);
        s.tp_w = __uint_as_float(c2.w);
        s.origin = f3w(c3);
        s.bounce = c3.w;
        s.direction = f3w(c4);
        s.previous_position = f3w(c5);
        s.previous_normal = f3w(c6);
        s.previous_pdf = __uint_as_float(c1.z);
        s.done = false;
    }
    uint32_t steps = V.range[2] < 8u ? V.range[2] : 8u;
    bool terminal = false;
    if (V.range[3] != 0u) {
        const uint32_t used = s.bounce < V.range[3] ? s.bounce : V.range[3];
        const uint32_t left = V.range[3] - used;
        steps = steps < left ? steps : left;
        terminal = s.bounce + steps == V.range[3];
    }
    view_advance<LIMITED, BUDGETED>(T, s, stream, sequence, steps, terminal);
    rec[3] = w3(s.first.position, s.first.status);
    rec[4] = wi3(s.first.voxel, face_index_of(s.first.normal));
    rec[5].w = (s.done && !s.unknown) ? 1u : 0u;
    rec[6] = w3(s.done ? s.energy : V3{0.0f, 0.0f, 0.0f}, s.first.material);
    for (int i = 0; i < 8; ++i) record[i] = rec[i];
    stored[0] = w3(s.energy, __float_as_uint(s.energy_w));
    stored[1] = make_uint4(0u, 0u, __float_as_uint(s.previous_pdf), 0u);
    stored[2] = w3(s.tp, __float_as_uint(s.tp_w));
    stored[3] = w3(s.origin, s.bounce);
    stored[4] = w3(s.direction, s.done ? (s.unknown ? 3u : 2u) : 1u);
    stored[5] = w3(s.previous_position, 0u);
    stored[6] = w3(s.previous_normal, 0u);
    stored[7] = make_uint4(V.ticket[0], V.ticket[1], V.ticket[2], V.ticket[3]);
}

// shared_slot (voxel_view_cache.wgsl:6-26) for the unit face (voxel, face) of `material`.
__device__ uint32_t view_shared_slot_key(const ViewArgs& V, I3 voxel, uint32_t face, uint32_t material) {
    if (!V.shared || V.t.face_index == nullptr) return kNoIndex;
    const uint4 header = V.t.face_index[0];
    uint32_t bucket = (hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u)) & header.x;
#pragma unroll 1
    for (uint32_t attempt = 0; attempt < header.y; ++attempt) {
        const uint4 e = V.t.face_index[bucket + 1u];
        if (e.w == 0xffffffffu) return kNoIndex;
        if ((int)e.x == voxel.x && (int)e.y == voxel.y && (int)e.z == voxel.z && (e.w >> 29u) == face) {
            const uint32_t slot = e.w & 0x1fffffffu;
            const uint32_t key = V.shared_meta[slot * 3u].w;
            if ((key & 8u) == 0u || (key >> 16u) != material) return kNoIndex;
            return slot;
        }
        bucket = (bucket + 1u) & header.x;
    }
    return kNoIndex;
}

__device__ __forceinline__ uint32_t view_shared_slot(const ViewArgs& V, uint32_t index, uint32_t material) {
    const uint4 r0 = V.receivers[index * 2u], r1 = V.receivers[index * 2u + 1u];
    return view_shared_slot_key(V, I3{(int)r1.x, (int)r1.y, (int)r1.z}, r0.w, material);
}

// reproject_paths' share for caller-given receivers: the receiver takes its
// estimate's sequence, and every receiver is its own owner (queue rank = index).
// report_sun_flips (voxel_view_runtime.wgsl:231-270): the flux a face's
// corners gained or lost from the sun between two corner words, queued as
// (voxel, flux) for the scheduler; past kMaxSunFlips records the flips widen
// one overflow box and add to its summed flux.
__device__ void report_sun_flips(const ViewArgs& V, I3 voxel, V3 normal, uint32_t material, uint32_t before, uint32_t after) {
    const V3 w{0.2126f, 0.7152f, 0.0722f};
    float flux = 0.0f;
    uint32_t bit = 0u;
    for (uint32_t i = 0; i < V.n_directional && bit < 4u; ++i) {
        const float4 p = __ldg(V.t.lights + i * 3u), e = __ldg(V.t.lights + i * 3u + 1u), x = __ldg(V.t.lights + i * 3u + 2u);
        const V3 color{wmax(__fsub_rn(e.x, x.y), 0.0f), wmax(__fsub_rn(e.y, x.z), 0.0f), wmax(__fsub_rn(e.z, x.w), 0.0f)};
        if (color.x == 0.0f && color.y == 0.0f && color.z == 0.0f) continue;
        const float cosine = wmax(dot3(normal, normalize3(V3{p.x, p.y, p.z})), 0.0f);
        for (uint32_t corner = 0; corner < 4u; ++corner) {
            const uint32_t a = (before >> (corner * 8u)) & 255u, b = (after >> (corner * 8u)) & 255u;
            if ((a & b & 128u) != 0u && ((a ^ b) & (1u << bit)) != 0u)
                flux = __fadd_rn(flux, __fmul_rn(__fmul_rn(0.25f, dot3(color, w)), cosine));
        }
        bit += 1u;
    }
    if (flux <= 0.0f) return;
    const float4 d = __ldg(V.t.materials + (material & 255u) * 4u);
    flux = __fmul_rn(flux, dot3(V3{d.x, d.y, d.z}, w));
    uint32_t* flips = V.queue + kViewPrefix + 2u * V.n;
    const uint32_t slot = atomicAdd(flips, 1u);
    if (slot >= kMaxSunFlips) {
        uint32_t* overflow = flips + 4u + kMaxSunFlips * 4u;
        const int bias = 1073741824;
        atomicMax(overflow + 0, (uint32_t)(bias - voxel.x));
        atomicMax(overflow + 1, (uint32_t)(bias - voxel.y));
        atomicMax(overflow + 2, (uint32_t)(bias - voxel.z));
        atomicMax(overflow + 3, (uint32_t)(voxel.x + bias));
        atomicMax(overflow + 4, (uint32_t)(voxel.y + bias));
        atomicMax(overflow + 5, (uint32_t)(voxel.z + bias));
        atomicAdd(overflow + 6, (uint32_t)__fadd_rn(__fmul_rn(flux, 64.0f), 0.5f));
        return;
    }
    uint32_t* record = flips + 4u + slot * 4u;
    record[0] = (uint32_t)voxel.x;
    record[1] = (uint32_t)voxel.y;
    record[2] = (uint32_t)voxel.z;
    record[3] = __float_as_uint(flux);
}

// sky_corner_visibility (voxel_path.wgsl:246-266): per directional light
// with visible colour (at most 4) whether the corner sees it; all zero when a
// ray runs out of steps, bit 31 set otherwise.
__device__ uint32_t sky_corner_visibility(const TraceArgs& A, uint32_t n_directional, V3 position) {
    uint32_t word = 0x80000000u, bit = 0u;
    Cnt<false> cnt;
    for (uint32_t i = 0; i < n_directional && bit < 4u; ++i) {
        const float4 p = __ldg(A.lights + i * 3u), e = __ldg(A.lights + i * 3u + 1u), x = __ldg(A.lights + i * 3u + 2u);
        if (wmax(__fsub_rn(e.x, x.y), 0.0f) == 0.0f && wmax(__fsub_rn(e.y, x.z), 0.0f) == 0.0f && wmax(__fsub_rn(e.z, x.w), 0.0f) == 0.0f)
            continue;
        const V3 direction = normalize3(V3{p.x, p.y, p.z});
        const uint32_t status = trace_domain(A, position + direction * 0.002f, direction, A.max_distance, true, 2048u, cnt).status;
        if (status == 2u) {
            word = 0u;
            break;
        }
        if (status == 0u) word |= 1u << bit;
        bit += 1u;
    }
    return word;
}

// reproject_paths (voxel_view_runtime.wgsl:148-215) for caller-given
// receivers: the receiver takes its estimate's sequence, every receiver is
// its own owner (queue rank = index), and a face lit by a directional light
// refreshes its four corner sun words one frame in 4 (staggered by index),
// at once when it is new to the view.
__global__ void __launch_bounds__(kBlock) view_reproject_kernel(const ViewArgs V) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i == 0) {
        for (uint32_t k = 0; k < kViewPrefix; ++k) V.queue[k] = 0u;
        V.queue[kViewOwners] = V.n;
    }
    if (i >= V.n) return;
    const uint4 r0 = V.receivers[i * 2u], r1 = V.receivers[i * 2u + 1u];
    if (r0.w < 6u) {
        const V3 normal = face_normal(r0.w);
        bool lit = false;
        for (uint32_t l = 0; l < V.n_directional; ++l) {
            const float4 p = __ldg(V.t.lights + l * 3u);
            lit = lit || dot3(normal, V3{p.x, p.y, p.z}) > 0.0f;
        }
        const uint32_t old = V.estimates[i * 4u + 3u].z;
        const bool carried = V.has_previous && old != 0u && (V.frame + i) % 4u != 0u;
        uint32_t corners = carried ? old : 0x80808080u;
        if (lit && !carried) {
            V3 u{0.0f, 1.0f, 0.0f}, v{0.0f, 0.0f, 1.0f};
            if (r0.w / 2u == 1u) u = V3{1.0f, 0.0f, 0.0f};
            else if (r0.w / 2u == 2u) {
                u = V3{1.0f, 0.0f, 0.0f};
                v = V3{0.0f, 1.0f, 0.0f};
            }
            const uint32_t a = (r0.w / 2u + 1u) % 3u;
            const float sa = a == 0u ? __uint_as_float(r0.x) : (a == 1u ? __uint_as_float(r0.y) : __uint_as_float(r0.z));
            const int va = a == 0u ? (int)r1.x : (a == 1u ? (int)r1.y : (int)r1.z);
            const float s = __fmul_rn(2.0f, __fsub_rn(sa, (float)va));  // receiver_stride
            u = u * s;
            v = v * s;
            const V3 base = V3{(float)(int)r1.x, (float)(int)r1.y, (float)(int)r1.z} +
                            V3{wmax(normal.x, 0.0f), wmax(normal.y, 0.0f), wmax(normal.z, 0.0f)} * s;
            corners = 0u;
            for (uint32_t corner = 0; corner < 4u; ++corner) {
                const V3 position = (base + u * (float)(corner & 1u)) + v * (float)(corner >> 1u);
                const uint32_t word = sky_corner_visibility(V.t, V.n_directional, position);
                corners |= ((word & 15u) | ((word >> 24u) & 128u)) << (corner * 8u);
            }
            if (V.has_previous && old != 0u)
                report_sun_flips(V, I3{(int)r1.x, (int)r1.y, (int)r1.z}, normal, V.estimates[i * 4u + 3u].y, old, corners);
        }
        V.estimates[i * 4u + 3u].z = corners;
    }
    V.receivers[i * 2u + 1u].w = V.estimates[i * 4u + 3u].x;
    V.queue[kViewPrefix + i] = i;
    V.queue[kViewPrefix + V.n + i] = i;
}

// retain_view_history (voxel_view_runtime.wgsl:327-349)
__global__ void __launch_bounds__(kBlock) view_retain_kernel(const ViewArgs V) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= V.n) return;
    const uint4 r1 = V.receivers[i * 2u + 1u];
    const RetentionResult c = resolve_retention(V.events, V.n_events, V.reach, (int)r1.x, (int)r1.y, (int)r1.z, V.physical > 0.0f, 0u, 0u);
    uint4* e = V.estimates + i * 4u;
    const uint4 identity = e[3];
    if (identity.w == 0u || view_shared_slot(V, i, identity.y) == kNoIndex) {
        if (c.limit != kNoIndex) e[0].w = __float_as_uint(wmin(__uint_as_float(e[0].w), (float)c.limit));
        if (c.measured) e[1].w = __float_as_uint(__fadd_rn(__uint_as_float(e[1].w), c.change));
    }
    if (c.woken && V.conts[i * 8u + 4u].w == 1u) V.conts[i * 8u + 4u].w = 0u;
}

// load_shared_faces (voxel_view_cache.wgsl:28-98, 188-223), its world-cache
// part: hand the world cache's authority to the view estimate and reserve
// this frame's sequence range on the slot (the priors for new receivers are
// view_seed_kernel's).
__global__ void __launch_bounds__(kBlock) view_load_kernel(const ViewArgs V) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= V.n) return;
    uint4* e = V.estimates + i * 4u;
    uint4 mean = e[0], moment = e[1], shown = e[2], identity = e[3];
    const uint32_t slot = view_shared_slot(V, i, identity.y);
    if (slot == kNoIndex) {
        e[3].w = 0u;
        return;
    }
    uint4* base = V.shared_state + slot * 9u;
    const uint32_t incarnation = base[7].x;
    const uint32_t count = base[1].y & 0x7fffffffu;
    const uint32_t next = base[1].z;
    atomicAdd(V.queue + kViewLoads, 1u);
    if (identity.w == incarnation || __uint_as_float(mean.w) <= (float)count) {
        if (identity.w != incarnation) V.conts[i * 8u + 4u].w = 0u;
        const uint4 m = base[0], sec = base[2];
        mean = make_uint4(m.x, m.y, m.z, __float_as_uint((float)count));
        moment = make_uint4(sec.x, sec.y, sec.z, V.shared_meta[slot * 3u + 1u].x);
        identity.x = next;
    } else {
        atomicAdd(V.queue + kViewPromotions, 1u);
        identity.x = identity.x > next ? identity.x : next;
    }
    if (__uint_as_float(shown.w) == 0.0f && count > 0u) {
        const uint4 sh = base[6];
        shown = __uint_as_float(sh.w) > 0.0f ? sh : make_uint4(mean.x, mean.y, mean.z, __float_as_uint(1.0f));
    }
    // A face entering view again compares its fresh corners with those the
    // world slot kept from when it was last seen.
    if (identity.w != incarnation) {
        const uint4 r0 = V.receivers[i * 2u], r1 = V.receivers[i * 2u + 1u];
        report_sun_flips(V, I3{(int)r1.x, (int)r1.y, (int)r1.z}, face_normal(r0.w), identity.y, base[8].x, identity.z);
    }
    identity.w = incarnation;
    const bool pending = V.conts[i * 8u + 4u].w == 1u;
    const uint32_t owners = V.n;
    const uint32_t rank = V.queue[kViewPrefix + V.n + i];
    const uint32_t oc = owners > 1u ? owners : 1u;
    const uint32_t ordinal = (rank + owners - V.range[0] % oc) % oc;
    uint32_t visits = 0;
    const uint32_t span = owners < V.range[1] ? owners : V.range[1];
    if (ordinal < span && V.range[2] > 0u) {
        const uint32_t cap = V.view_first ? 32u : 1u;
        const uint32_t share = (V.range[1] - ordinal + owners - 1u) / owners;
        visits = cap < share ? cap : share;
    }
    const uint32_t first = next > identity.x ? next : identity.x;
    const uint32_t starts = visits - ((pending && visits > 0u) ? 1u : 0u);
    base[1].z = first + starts;
    V.queue[kViewPrefix + V.n + i] = first;
    identity.x = pending ? V.paths[i * 8u].w : first;
    e[0] = mean;
    e[1] = moment;
    e[2] = shown;
    e[3] = identity;
    V.receivers[i * 2u + 1u].w = identity.x;
}

// voxel_material (voxel_traversal.wgsl:48-70): the material of one voxel, 256 for air.
__device__ uint32_t voxel_material(const TraceArgs& A, I3 v) {
    const int rx = (int)floorf(__fdiv_rn((float)v.x, 16.0f)), ry = (int)floorf(__fdiv_rn((float)v.y, 16.0f)),
              rz = (int)floorf(__fdiv_rn((float)v.z, 16.0f));
    if (!in_bounds(A, rx, ry, rz)) return 256u;
    Cnt<false> cnt;
    const uint32_t index = lookup_region(A, rx, ry, rz, cnt);
    if (index == kNoIndex) return 256u;
    const uint4 meta = __ldg(A.headers + index);
    if (meta.x == 1u) return 256u;
    if (meta.x != 3u) return meta.y;
    const uint32_t lx = (uint32_t)(v.x & 15), ly = (uint32_t)(v.y & 15), lz = (uint32_t)(v.z & 15);
    const uint32_t word = __ldg(A.cells + meta.y + ((lz >> 2) * 4u + (ly >> 2)) * 4u + (lx >> 2));
    if ((word & 3u) == 0u) return 256u;
    if ((word & 3u) == 1u) return word >> 2u;
    const uint32_t idx = ((lz & 3u) * 4u + (ly & 3u)) * 4u + (lx & 3u);
    const uint32_t cell = (__ldg(A.cells + (word >> 2u) + idx / 2u) >> ((idx & 1u) * 16u)) & 65535u;
    return (cell & 1u) != 0u ? cell >> 1u : 256u;
}

// prior_air (voxel_view_cache.wgsl:141-144): known air in a loaded region.
__device__ bool prior_air(const TraceArgs& A, I3 v) {
    const int rx = (int)floorf(__fdiv_rn((float)v.x, 16.0f)), ry = (int)floorf(__fdiv_rn((float)v.y, 16.0f)),
              rz = (int)floorf(__fdiv_rn((float)v.z, 16.0f));
    if (!in_bounds(A, rx, ry, rz)) return false;
    Cnt<false> cnt;
    return lookup_region(A, rx, ry, rz, cnt) != kNoIndex && voxel_material(A, v) == 256u;
}

struct FacePrior {
    V3 mean, moment;
    float weight;
};

// prior_donor (voxel_view_cache.wgsl:108-131): the last frame's estimate of
// the receiver on this unit face, or the world cache's slot if it holds more
// samples; at least 16 samples either way.
__device__ FacePrior prior_donor(const ViewArgs& V, I3 voxel, uint32_t face) {
    FacePrior donor{V3{0.0f, 0.0f, 0.0f}, V3{0.0f, 0.0f, 0.0f}, 0.0f};
    const V3 surface = add_s(itof(voxel), 0.5f) + face_normal(face) * 0.5f;
    uint32_t slot = (hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u)) & V.hash_mask;
#pragma unroll 1
    for (uint32_t step = 0; step < 64u; ++step) {
        const uint32_t value = V.receiver_hash[slot];
        if (value == 0u) break;
        if (value <= V.n) {
            const uint4 r0 = V.receivers[(value - 1u) * 2u], r1 = V.receivers[(value - 1u) * 2u + 1u];
            if (r0.w == face && (int)r1.x == voxel.x && (int)r1.y == voxel.y && (int)r1.z == voxel.z && __uint_as_float(r0.x) == surface.x &&
                __uint_as_float(r0.y) == surface.y && __uint_as_float(r0.z) == surface.z) {
                const uint4 m = V.prev_estimates[(value - 1u) * 4u], mo = V.prev_estimates[(value - 1u) * 4u + 1u];
                if (__uint_as_float(m.w) >= 16.0f) donor = FacePrior{f3w(m), f3w(mo), __uint_as_float(m.w)};
                break;
            }
        }
        slot = (slot + 1u) & V.hash_mask;
    }
    const uint32_t cache = view_shared_slot_key(V, voxel, face, voxel_material(V.t, voxel));
    if (cache != kNoIndex) {
        const uint4* base = V.shared_state + cache * 9u;
        const uint32_t count = base[1].y & 0x7fffffffu;
        if (count >= 16u && (float)count > donor.weight) donor = FacePrior{f3w(base[0]), f3w(base[2]), (float)count};
    }
    return donor;
}

__device__ __forceinline__ void add_prior(FacePrior& sum, const FacePrior& donor, float weight) {
    if (donor.weight == 0.0f) return;
    sum.mean = sum.mean + donor.mean * weight;
    sum.moment = sum.moment + donor.moment * weight;
    sum.weight = __fadd_rn(sum.weight, weight);
}

// bootstrap_face (voxel_view_cache.wgsl:146-186) for a receiver whose
// geometry is not pending: a newly exposed face takes the incident light of
// the coplanar faces it connects to, or of the faces around its air cell.
__device__ FacePrior bootstrap_face(const ViewArgs& V, uint4 r0, uint4 r1) {
    FacePrior prior{V3{0.0f, 0.0f, 0.0f}, V3{0.0f, 0.0f, 0.0f}, 0.0f};
    const uint32_t rf = r0.w;
    const I3 origin{(int)r1.x, (int)r1.y, (int)r1.z};
    const V3 nf = face_normal(rf);
    const I3 normal{(int)nf.x, (int)nf.y, (int)nf.z};
    const I3 air{origin.x + normal.x, origin.y + normal.y, origin.z + normal.z};
    // receiver_stride: unit faces only.
    const uint32_t u = (rf / 2u + 1u) % 3u;
    const float su = u == 0u ? __uint_as_float(r0.x) : (u == 1u ? __uint_as_float(r0.y) : __uint_as_float(r0.z));
    const int vu = u == 0u ? origin.x : (u == 1u ? origin.y : origin.z);
    if (__fmul_rn(2.0f, __fsub_rn(su, (float)vu)) != 1.0f) return prior;
    if (voxel_material(V.t, origin) == 256u || !prior_air(V.t, air)) return prior;
    for (uint32_t f = 0; f < 6u; ++f) {
        const V3 o = face_normal(f);
        const I3 off{(int)o.x, (int)o.y, (int)o.z};
        const I3 v{origin.x + off.x, origin.y + off.y, origin.z + off.z};
        const bool covered = off.x == -normal.x && off.y == -normal.y && off.z == -normal.z;
        if (covered || prior_air(V.t, I3{v.x + normal.x, v.y + normal.y, v.z + normal.z})) add_prior(prior, prior_donor(V, v, rf), 1.0f);
    }
    if (prior.weight == 0.0f) {
        for (uint32_t f = 0; f < 6u; ++f) {
            const V3 o = face_normal(f);
            const I3 off{(int)o.x, (int)o.y, (int)o.z};
            const float alignment = dot3(itof(normal), o);
            const float w = alignment > 0.0f ? 1.0f : 0.25f;
            add_prior(prior, prior_donor(V, air, f), w);
            const I3 covered{origin.x - off.x, origin.y - off.y, origin.z - off.z};
            if (covered.x != air.x || covered.y != air.y || covered.z != air.z) add_prior(prior, prior_donor(V, covered, f), w);
            add_prior(prior, prior_donor(V, I3{air.x - off.x, air.y - off.y, air.z - off.z}, f), w);
        }
    }
    if (prior.weight > 0.0f) {
        prior.mean = prior.mean / prior.weight;
        const V3 m2 = prior.moment / prior.weight;
        prior.moment = V3{wmax(m2.x, __fmul_rn(prior.mean.x, prior.mean.x)), wmax(m2.y, __fmul_rn(prior.mean.y, prior.mean.y)),
                          wmax(m2.z, __fmul_rn(prior.mean.z, prior.mean.z))};
        prior.weight = 1.0f;
    }
    return prior;
}

// The priors of load_shared_faces (voxel_view_cache.wgsl:192-212): a new,
// unmeasured receiver (no samples, no sequence, nothing from the world
// cache) starts from its topology prior, or else, with the far tier's
// handoff, from the far cell at its centre (previous_cell over the last far
// frame's cells): one unit of weight, mean and shown = the prior's rgb.
__global__ void __launch_bounds__(kBlock) view_seed_kernel(const ViewArgs V) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= V.n) return;
    const uint4 r0 = V.receivers[i * 2u], r1 = V.receivers[i * 2u + 1u];
    if (r0.w >= 6u) return;
    uint4* e = V.estimates + i * 4u;
    if (__uint_as_float(e[0].w) != 0.0f || e[3].x != 0u) return;
    FacePrior prior{V3{0.0f, 0.0f, 0.0f}, V3{0.0f, 0.0f, 0.0f}, 0.0f};
    if (V.topology) prior = bootstrap_face(V, r0, r1);
    if (prior.weight == 0.0f && V.far_cells) {
        Cnt<false> cnt;
        V3 mean;
        float count;
        uint32_t sequence;
        previous_cell(V.t, V.far, V.far_cells, f3w(r0), r0.w, I3{(int)r1.x, (int)r1.y, (int)r1.z}, mean, count, sequence, cnt);
        if (count > 0.0f) {
            prior = FacePrior{mean, V3{__fmul_rn(mean.x, mean.x), __fmul_rn(mean.y, mean.y), __fmul_rn(mean.z, mean.z)}, 1.0f};
            atomicAdd(V.far_stats + 5, 1u);
        }
    }
    if (prior.weight <= 0.0f) return;
    const uint32_t one = __float_as_uint(prior.weight);
    e[0] = w3(prior.mean, one);
    e[1] = w3(prior.moment, 0u);
    e[2] = w3(prior.mean, __float_as_uint(1.0f));
}

// One receiver's visits of a view frame (trace_visible_paths,
// voxel_view_runtime.wgsl:272-325): completed paths update the estimate's
// discounted running mean and second moment.
template <bool LIMITED, bool BUDGETED>
__device__ __forceinline__ void view_trace_receiver(Tracer<1, LIMITED, BUDGETED, false>& T, const ViewArgs& V, uint32_t id, uint32_t& attempted,
                                                    uint32_t& completed, uint32_t& known) {
    const uint32_t count = V.n;
    const uint32_t index = V.queue[kViewPrefix + (V.range[0] + id) % count];
    const uint32_t cap = V.view_first ? 32u : 1u;
    const uint32_t share = (V.range[1] - id + count - 1u) / count;
    const uint32_t visits = cap < share ? cap : share;
    const bool reserved = V.shared && V.estimates[index * 4u + 3u].w != 0u;
    uint32_t next = V.queue[kViewPrefix + V.n + index];
    if (V.conts[index * 8u + 4u].w != 1u) next += 1u;
#pragma unroll 1
    for (uint32_t visit = 0; visit < visits; ++visit) {
        attempted += 1u;
        advance_view_path<LIMITED, BUDGETED>(T, V, index);
        const uint32_t status = V.conts[index * 8u + 4u].w;
        if (status != 2u && status != 3u) continue;
        completed += 1u;
        uint4* e = V.estimates + index * 4u;
        uint4 identity = e[3];
        if (reserved) {
            identity.x = next;
            next += 1u;
        } else {
            identity.x += 1u;
        }
        V.receivers[index * 2u + 1u].w = identity.x;
        e[3] = identity;
        const uint4* path = V.paths + index * 8u;
        if (path[5].w != 0u) {
            known += 1u;
            const V3 value = f3w(path[5]) + f3w(path[6]);
            V3 mean = f3w(e[0]), moment = f3w(e[1]);
            float weight = __uint_as_float(e[0].w), change = __uint_as_float(e[1].w);
            if (change > 0.0f) {
                const V3 variance{wmax(__fsub_rn(moment.x, __fmul_rn(mean.x, mean.x)), 0.0f),
                                  wmax(__fsub_rn(moment.y, __fmul_rn(mean.y, mean.y)), 0.0f),
                                  wmax(__fsub_rn(moment.z, __fmul_rn(mean.z, mean.z)), 0.0f)};
                const float lum = __fadd_rn(__fadd_rn(__fmul_rn(variance.x, 0.2126f), __fmul_rn(variance.y, 0.7152f)),
                                            __fmul_rn(variance.z, 0.0722f));
                const float keep = __fdiv_rn(__fmul_rn(V.physical, lum), __fmul_rn(change, change));
                weight = wmin(weight, floorf(keep));
                change = 0.0f;
            }
            const float n = wmin(__fadd_rn(weight, 1.0f), 65536.0f);
            const float t = __fdiv_rn(1.0f, n);
            const float u = __fsub_rn(1.0f, t);
            // mix(a, b, t) = a * (1 - t) + b * t
            mean = mean * u + value * t;
            moment = moment * u + (value * value) * t;
            e[0] = w3(mean, __float_as_uint(n));
            e[1] = w3(moment, __float_as_uint(change));
        }
    }
    if (reserved) {
        const uint32_t first = V.queue[kViewPrefix + V.n + index];
        const uint32_t used = V.conts[index * 8u + 4u].w == 1u ? V.paths[index * 8u].w + 1u : V.estimates[index * 4u + 3u].x;
        V.queue[kViewPrefix + V.n + index] = first > used ? first : used;
    }
}

// trace_visible_paths: one thread per owner invocation.
template <bool LIMITED, bool BUDGETED>
__global__ void __launch_bounds__(kBlock) view_trace_kernel(const ViewArgs V) {
    __shared__ float4 smat[512];
    const TraceArgs& A = V.t;
    view_stage_materials<LIMITED, BUDGETED>(A, smat);
    Cnt<false> cnt;
    Tracer<1, LIMITED, BUDGETED, false> T{A, smat, cnt};
    const uint32_t id = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t count = V.n;
    // The frame's counters, summed per warp and added once per warp.
    uint32_t attempted = 0, completed = 0, known = 0;
    if (id < (count < V.range[1] ? count : V.range[1]) && V.range[2] != 0u)
        view_trace_receiver<LIMITED, BUDGETED>(T, V, id, attempted, completed, known);
    attempted = __reduce_add_sync(0xffffffffu, attempted);
    completed = __reduce_add_sync(0xffffffffu, completed);
    known = __reduce_add_sync(0xffffffffu, known);
    if ((threadIdx.x & 31u) == 0u) {
        if (attempted) atomicAdd(V.queue + kViewAttempted, attempted);
        if (completed) atomicAdd(V.queue + kViewCompleted, completed);
        if (known) atomicAdd(V.queue + kViewKnown, known);
    }
}

// store_shared_faces (voxel_view_cache.wgsl:225-258), and the slot's gather
// record with it.
__global__ void __launch_bounds__(kBlock) view_store_kernel(const ViewArgs V) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= V.n) return;
    const uint4* e = V.estimates + i * 4u;
    const uint4 mean = e[0], moment = e[1], shown = e[2], identity = e[3];
    const uint32_t slot = view_shared_slot(V, i, identity.y);
    if (slot == kNoIndex) return;
    uint4* base = V.shared_state + slot * 9u;
    if (identity.w != base[7].x) return;
    const uint32_t count = (uint32_t)__uint_as_float(mean.w);
    const bool changed_count = (base[1].y & 0x7fffffffu) != count;
    const bool changed_mean = base[0].x != mean.x || base[0].y != mean.y || base[0].z != mean.z;
    base[0] = make_uint4(mean.x, mean.y, mean.z, 0u);
    base[2] = make_uint4(moment.x, moment.y, moment.z, 0u);
    const uint32_t word = count | (__uint_as_float(moment.w) > 0.0f ? 0x80000000u : 0u);
    base[1] = make_uint4(0u, word, V.queue[kViewPrefix + V.n + i], shown.x);
    V.shared_meta[slot * 3u + 1u].x = moment.w;
    base[6] = shown;
    if (identity.z != 0u) base[8].x = identity.z;
    base[3] = make_uint4(0u, shown.y, shown.z, shown.w);
    V.shared_cache[slot] = make_float4(__uint_as_float(mean.x), __uint_as_float(mean.y), __uint_as_float(mean.z), __uint_as_float(word));
    if (changed_mean || changed_count) {
        const V3 m = f3w(mean), mo = f3w(moment);
        const float nx = __fdiv_rn(__fsqrt_rn(wmax(__fsub_rn(mo.x, __fmul_rn(m.x, m.x)), 0.0f)), __fadd_rn(0.002f, fabsf(m.x)));
        const float ny = __fdiv_rn(__fsqrt_rn(wmax(__fsub_rn(mo.y, __fmul_rn(m.y, m.y)), 0.0f)), __fadd_rn(0.002f, fabsf(m.y)));
        const float nz = __fdiv_rn(__fsqrt_rn(wmax(__fsub_rn(mo.z, __fmul_rn(m.z, m.z)), 0.0f)), __fadd_rn(0.002f, fabsf(m.z)));
        V.shared_meta[slot * 3u + 2u] = make_uint4(__float_as_uint(wmax(nx, wmax(ny, nz))), V.clock,
                                                   __float_as_uint(wmax(m.x, wmax(m.y, m.z))), 0xa0000000u | count);
    }
}

template <bool LIMITED, bool BUDGETED>
void view_frame_impl(const ViewArgs& V, cudaStream_t s) {
    const uint32_t grid = (V.n + kBlock - 1) / kBlock;
    view_reproject_kernel<<<grid, kBlock, 0, s>>>(V);
    if (V.n_events) view_retain_kernel<<<grid, kBlock, 0, s>>>(V);
    if (V.shared) view_load_kernel<<<grid, kBlock, 0, s>>>(V);
    if (V.far_cells || V.topology) view_seed_kernel<<<grid, kBlock, 0, s>>>(V);
    const uint32_t work = V.n < V.range[1] ? V.n : V.range[1];
    if (work && V.range[2]) view_trace_kernel<LIMITED, BUDGETED><<<(work + kBlock - 1) / kBlock, kBlock, 0, s>>>(V);
    if (V.shared) view_store_kernel<<<grid, kBlock, 0, s>>>(V);
}

}  // namespace

void launch_view_frame(const ViewArgs& V, bool limited, bool budgeted, cudaStream_t s) {
    if (V.n == 0) return;
    if (limited) {
        if (budgeted) view_frame_impl<true, true>(V, s);
        else view_frame_impl<true, false>(V, s);
    } else {
        if (budgeted) view_frame_impl<false, true>(V, s);
        else view_frame_impl<false, false>(V, s);
    }
}

void launch_view_trace_paths(const ViewArgs& V, uint32_t samples, uint4* out, bool limited, bool budgeted, cudaStream_t s) {
    const uint64_t total = (uint64_t)V.n * samples;
    if (total == 0) return;
    const uint32_t grid = (uint32_t)((total + kBlock - 1) / kBlock);
    if (limited) {
        if (budgeted) view_trace_paths_kernel<true, true><<<grid, kBlock, 0, s>>>(V, samples, out);
        else view_trace_paths_kernel<true, false><<<grid, kBlock, 0, s>>>(V, samples, out);
    } else {
        if (budgeted) view_trace_paths_kernel<false, true><<<grid, kBlock, 0, s>>>(V, samples, out);
        else view_trace_paths_kernel<false, false><<<grid, kBlock, 0, s>>>(V, samples, out);
    }
}

}  // namespace vgi
