// Resident face-cache maintenance around the trace: begin_trace and
// mark_changed before it, accumulate (discounted running mean, display EMA,
// stability) after it, and apply_events for retention events.
//
// Behaviour follows (paths within nathanaelneveux/global-illumination,
// crates/bevy_voxel_gi/shaders/):
//   voxel_accumulate.wgsl:130-133  begin_trace
//   voxel_accumulate.wgsl:135-262  accumulate, record_stability, settled_flag
//   voxel_accumulate.wgsl:264-286  sample_noise, required_samples, refinement_error
//   voxel_accumulate.wgsl:295-344  apply_events, binds
//   voxel_accumulate.wgsl:357-425  face_slot, measure_edits, finish_edits
//   voxel_accumulate.wgsl:432-446  mark_changed
//   voxel_retention.wgsl:1-96      curve_limit, box_distance2, resolve_retention
//
// Layout: the reference's slot records (9 uint4 state, 3 uint4 metadata,
// 3 uint4 checkpoint) are kept as arrays of uint4 so each thread moves whole
// 16-byte words and a warp covers contiguous lines. Beside them each slot
// has a 16-byte gather record (mean rgb, count word) that the trace reads for
// the world-cache gather instead of two state words; every kernel that
// changes a slot's mean or count rewrites it.
#include "vgi_device.cuh"
#include "vgi_types.cuh"
#include "vgi_retention.cuh"

namespace vgi {
namespace {

constexpr int kBlock = 256;
constexpr uint32_t kNoLimit = 0xffffffffu;
constexpr uint32_t kUrgent = 0x40000000u;
constexpr uint32_t kMirrorStale = 0x20000000u;

__device__ __forceinline__ float u2f(uint32_t u) { return __uint_as_float(u); }
__device__ __forceinline__ uint32_t f2b(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float lum3(float r, float g, float b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, r), __fmul_rn(0.7152f, g)), __fmul_rn(0.0722f, b));
}
__device__ __forceinline__ float max3(float a, float b, float c) { return wmax(a, wmax(b, c)); }
__device__ __forceinline__ float var1(float s, float m) { return wmax(__fsub_rn(s, __fmul_rn(m, m)), 0.0f); }

__device__ __forceinline__ void write_record(float4* cache, uint32_t slot, const uint4& mean, uint32_t count) {
    cache[slot] = make_float4(u2f(mean.x), u2f(mean.y), u2f(mean.z), u2f(count));
}

// binds (voxel_accumulate.wgsl:336-344)
__device__ bool binds(const uint4* state, uint32_t slot, float change, float physical) {
    uint4 m = state[slot * 9u], s = state[slot * 9u + 2u];
    uint32_t count = state[slot * 9u + 1u].y;
    float mr = u2f(m.x), mg = u2f(m.y), mb = u2f(m.z);
    float variance = lum3(var1(u2f(s.x), mr), var1(u2f(s.y), mg), var1(u2f(s.z), mb));
    bool lit = lum3(mr, mg, mb) >= __fmul_rn(0.05f, change);
    float keep = __fdiv_rn(__fmul_rn(physical, variance), wmax(__fmul_rn(change, change), 1e-30f));
    return !lit || keep < (float)(count & 0x7fffffffu);
}

// prepare's begin_trace and batch stamp (voxel_accumulate.wgsl:114-121),
// then mark_changed (:432-446), one thread per task. With slot_meta null only
// the task's sequence is written (the counting pass's copy of the tasks).
__global__ void __launch_bounds__(kBlock) prepare_kernel(AccumArgs a) {
    uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= a.n) return;
    uint32_t slot = a.slots ? a.slots[i] : i;
    if (slot == kNoIndex) return;
    uint4 meta1 = a.state[slot * 9u + 1u];
    a.tasks[i * 2u + 1u].x = meta1.z;  // begin_trace: the task takes the slot's sequence
    if (a.slot_meta == nullptr) return;
    uint4* sm = a.slot_meta + slot * 3u + 1u;
    uint4 sched = *sm;
    sched.y = (sched.y & 0xfu) | (a.controls[25] << 4);
    sm->y = sched.y;
    float pending = u2f(sched.x);
    if (pending <= 0.0f) return;
    if (binds(a.state, slot, pending, u2f(a.controls[11]))) {
        meta1.y |= 0x80000000u;
        a.state[slot * 9u + 1u].y = meta1.y;
        a.cache[slot].w = u2f(meta1.y);
    } else {
        sm->x = 0u;
    }
}

__device__ float refinement_error(uint4 m, uint4 s, uint32_t count) {
    if (count < 2u) return 1.0f;
    float c = (float)count;
    float ex = __fdiv_rn(__fsqrt_rn(__fdiv_rn(var1(u2f(s.x), u2f(m.x)), c)), __fadd_rn(0.002f, fabsf(u2f(m.x))));
    float ey = __fdiv_rn(__fsqrt_rn(__fdiv_rn(var1(u2f(s.y), u2f(m.y)), c)), __fadd_rn(0.002f, fabsf(u2f(m.y))));
    float ez = __fdiv_rn(__fsqrt_rn(__fdiv_rn(var1(u2f(s.z), u2f(m.z)), c)), __fadd_rn(0.002f, fabsf(u2f(m.z))));
    return wmin(max3(ex, ey, ez), 8.0f);
}
__device__ float sample_noise(uint4 m, uint4 s) {
    float ex = __fdiv_rn(__fsqrt_rn(var1(u2f(s.x), u2f(m.x))), __fadd_rn(0.002f, fabsf(u2f(m.x))));
    float ey = __fdiv_rn(__fsqrt_rn(var1(u2f(s.y), u2f(m.y))), __fadd_rn(0.002f, fabsf(u2f(m.y))));
    float ez = __fdiv_rn(__fsqrt_rn(var1(u2f(s.z), u2f(m.z))), __fadd_rn(0.002f, fabsf(u2f(m.z))));
    return max3(ex, ey, ez);
}

__device__ __forceinline__ float lerp_alpha(float p, float m, float alpha) { return __fadd_rn(p, __fmul_rn(__fsub_rn(m, p), alpha)); }
__device__ __forceinline__ float mix_w(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

// accumulate + record_stability + settled_flag for CPU-owned faces (no GPU picks).
__global__ void __launch_bounds__(kBlock) accumulate_kernel(AccumArgs a) {
    const uint32_t* ctl = a.controls;
    uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= a.n || i >= ctl[0]) return;
    uint32_t slot = a.slots ? a.slots[i] : i;
    if (slot == kNoIndex) return;
    uint4* st = a.state + slot * 9u;
    uint4* out = a.outputs + (size_t)i * 6u;
    uint4* cp = a.checkpoint + slot * 3u;
    uint4 s0 = st[0], s1 = st[1], s2 = st[2], s3 = st[3], s6 = st[6], s7 = st[7];
    cp[0] = s0;
    cp[1] = s2;
    uint4 cp2 = make_uint4(s1.x, s1.y & 0x7fffffffu, s3.x, 0u);
    uint4 o0 = out[0], o1 = out[1], o2 = out[2], o4 = out[4], o5 = out[5];
    uint32_t fresh = f2u(u2f(o1.y));
    uint4* sched_p = a.slot_meta + slot * 3u + 1u;
    uint4 sched = *sched_p;
    float pending = u2f(sched.x);
    if (fresh > 0u) sched.x = 0u;
    uint32_t previous_count = s1.y & 0x7fffffffu;
    float physical = u2f(ctl[11]);
    float change = (s1.y & 0x80000000u) != 0u ? pending : 0.0f;
    if (physical > 0.0f && fresh > 0u && change > 0.0f) {
        float om = lum3(u2f(s0.x), u2f(s0.y), u2f(s0.z));
        float ov = lum3(var1(u2f(s2.x), u2f(s0.x)), var1(u2f(s2.y), u2f(s0.y)), var1(u2f(s2.z), u2f(s0.z)));
        float fv = lum3(var1(u2f(o2.x), u2f(o0.x)), var1(u2f(o2.y), u2f(o0.y)), var1(u2f(o2.z), u2f(o0.z)));
        float variance = om < __fmul_rn(0.05f, change) ? fv : ov;
        float keep = __fdiv_rn(__fmul_rn(physical, variance), __fmul_rn(change, change));
        uint32_t k = f2u(wmin(keep, 65536.0f));
        previous_count = previous_count < k ? previous_count : k;
        cp2.y = cp2.y < previous_count ? cp2.y : previous_count;
    }
    cp[2] = cp2;
    uint32_t count = previous_count + fresh;
    count = count < ctl[3] ? count : ctl[3];
    float recency = u2f(ctl[10]);
    float alpha = fresh > 0u ? wmin(__fdiv_rn(__fmul_rn(recency, (float)fresh), (float)(count > 1u ? count : 1u)), 1.0f) : 0.0f;
    uint4 nm = make_uint4(f2b(lerp_alpha(u2f(s0.x), u2f(o0.x), alpha)), f2b(lerp_alpha(u2f(s0.y), u2f(o0.y), alpha)),
                          f2b(lerp_alpha(u2f(s0.z), u2f(o0.z), alpha)), f2b(lerp_alpha(u2f(s0.w), u2f(o0.w), alpha)));
    uint4 ns = make_uint4(f2b(lerp_alpha(u2f(s2.x), u2f(o2.x), alpha)), f2b(lerp_alpha(u2f(s2.y), u2f(o2.y), alpha)),
                          f2b(lerp_alpha(u2f(s2.z), u2f(o2.z), alpha)), f2b(lerp_alpha(u2f(s2.w), u2f(o2.w), alpha)));
    s1.y = count;
    s1.z += ctl[1];
    float rr = u2f(nm.x), rg = u2f(nm.y), rb = u2f(nm.z);
    float mr = u2f(ns.x), mg = u2f(ns.y), mb = u2f(ns.z);
    float cnt = wmax((float)count, 1.0f);
    float er = __fsqrt_rn(__fdiv_rn(var1(mr, rr), cnt)), eg = __fsqrt_rn(__fdiv_rn(var1(mg, rg), cnt)), eb = __fsqrt_rn(__fdiv_rn(var1(mb, rb), cnt));
    float uncertainty = count < 2u ? 1.0f
                                   : wmin(8.0f, max3(__fdiv_rn(er, __fadd_rn(0.02f, fabsf(rr))), __fdiv_rn(eg, __fadd_rn(0.02f, fabsf(rg))),
                                                     __fdiv_rn(eb, __fadd_rn(0.02f, fabsf(rb)))));
    float noise = count < 2u ? 1.0f
                             : wmin(8.0f, max3(__fdiv_rn(er, __fadd_rn(0.002f, fabsf(rr))), __fdiv_rn(eg, __fadd_rn(0.002f, fabsf(rg))),
                                               __fdiv_rn(eb, __fadd_rn(0.002f, fabsf(rb)))));
    float elapsed = s7.z != 0u ? __fmul_rn((float)(ctl[2] - s7.y), 0.001f) : __fdiv_rn(1.0f, 60.0f);
    float time_alpha = __fsub_rn(1.0f, own_exp(__fdiv_rn(-elapsed, u2f(ctl[4]))));
    float evidence = __fdiv_rn((float)count, __fadd_rn((float)count, 32.0f));
    float blend = wmin(time_alpha, __fdiv_rn(evidence, __fadd_rn(1.0f, __fmul_rn(__fmul_rn(16.0f, noise), noise))));
    float pr = u2f(s6.x), pg = u2f(s6.y), pb = u2f(s6.z), pw = u2f(s6.w);
    float old_weight = __fdiv_rn(__fsub_rn(1.0f, blend), __fadd_rn(0.25f, max3(pr, pg, pb)));
    float new_weight = __fdiv_rn(blend, __fadd_rn(0.25f, max3(rr, rg, rb)));
    float alpha_display = wmin(blend, __fdiv_rn(new_weight, wmax(__fadd_rn(old_weight, new_weight), 0.0000001f)));
    float confidence = wclamp(__fdiv_rn(__fdiv_rn((float)count, __fadd_rn((float)count, 8.0f)), __fadd_rn(1.0f, uncertainty)), 0.125f, 1.0f);
    uint4 disp = make_uint4(f2b(mix_w(pr, rr, alpha_display)), f2b(mix_w(pg, rg, alpha_display)), f2b(mix_w(pb, rb, alpha_display)),
                            f2b(mix_w(pw, confidence, blend)));
    s7.y = ctl[2];
    s7.z = 0xffffffffu;
    s1.w = disp.x;
    s3 = make_uint4(s3.x, disp.y, disp.z, disp.w);
    st[0] = nm;
    st[1] = s1;
    st[2] = ns;
    st[3] = s3;
    st[4] = o4;
    st[5] = o5;
    st[6] = disp;
    st[7] = s7;
    write_record(a.cache, slot, nm, count);
    // record_stability (picked = false)
    uint4* rank_p = a.slot_meta + slot * 3u + 2u;
    bool same_revision = (sched.y & 8u) != 0u && sched.w == ctl[16];
    uint32_t scount = count & 0x7fffffffu;
    float tolerance = u2f(ctl[17]);
    float bx = u2f(s0.x), by = u2f(s0.y), bz = u2f(s0.z);
    float dx = __fdiv_rn(fabsf(__fsub_rn(bx, rr)), __fadd_rn(0.002f, wmax(fabsf(bx), fabsf(rr))));
    float dy = __fdiv_rn(fabsf(__fsub_rn(by, rg)), __fadd_rn(0.002f, wmax(fabsf(by), fabsf(rg))));
    float dz = __fdiv_rn(fabsf(__fsub_rn(bz, rb)), __fadd_rn(0.002f, wmax(fabsf(bz), fabsf(rb))));
    float drift = max3(dx, dy, dz);
    float dispr = u2f(disp.x), dispg = u2f(disp.y), dispb = u2f(disp.z);
    bool settled = max3(fabsf(__fsub_rn(dispr, rr)), fabsf(__fsub_rn(dispg, rg)), fabsf(__fsub_rn(dispb, rb))) <=
                   __fadd_rn(0.001f, __fmul_rn(__fmul_rn(max3(rr, rg, rb), tolerance), 0.5f));
    uint32_t required = max3(rr, rg, rb) < 0.02f ? (ctl[18] > 256u ? ctl[18] : 256u) : ctl[18];
    bool stable_now = same_revision && settled && scount >= required && refinement_error(nm, ns, scount) <= tolerance &&
                      drift <= __fmul_rn(tolerance, 0.5f);
    uint32_t stable = stable_now ? (((sched.y & 7u) + 1u) < 4u ? (sched.y & 7u) + 1u : 4u) : 0u;
    sched.y = (sched.y & 0xfffffff0u) | 8u | stable;
    sched.w = ctl[16];
    *sched_p = sched;
    uint4 rank = *rank_p;
    *rank_p = make_uint4(f2b(sample_noise(nm, ns)), ctl[2], f2b(max3(rr, rg, rb)), 0x80000000u | scount | (rank.w & kMirrorStale));
    uint4 w1 = s1;
    if ((sched.y & 15u) == 12u) w1.y |= 0x80000000u;
    out[0] = nm;
    out[1] = w1;
    out[2] = ns;
    out[3] = s3;
    out[4] = o4;
    out[5] = o5;
}

// apply_events (voxel_accumulate.wgsl:295-332) with resolve_retention
// (vgi_retention.cuh), one thread per slot.
__global__ void __launch_bounds__(kBlock) apply_events_kernel(AccumArgs a, const uint4* events, uint32_t n_slots) {
    const uint32_t* ctl = a.controls;
    uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
    if (slot >= n_slots) return;
    uint4 identity = a.slot_meta[slot * 3u];
    if ((identity.w & 8u) == 0u) return;
    int px = (int)identity.x, py = (int)identity.y, pz = (int)identity.z;
    const uint32_t event_count = ctl[13], reach = ctl[15];
    const float physical = u2f(ctl[11]);
    const bool measured_mode = physical > 0.0f;
    const RetentionResult r = resolve_retention(events, event_count, reach, px, py, pz, measured_mode, ctl[30], ctl[31]);
    const bool measured = r.measured, woken = r.woken, urgent_if_binding = r.urgent_if_binding;
    const uint32_t limit = r.limit;
    const float change = r.change;
    bool urgent = r.urgent;
    if (limit != kNoLimit) {
        uint4* s1p = a.state + slot * 9u + 1u;
        uint32_t y = s1p->y;
        y = y < limit ? y : limit;
        s1p->y = y;
        uint4* rank = a.slot_meta + slot * 3u + 2u;
        rank->w = (rank->w & 0xe0000000u) | (y & 0x1fffffffu);
        uint4* cp2 = a.checkpoint + slot * 3u + 2u;
        cp2->y = cp2->y < limit ? cp2->y : limit;
        a.cache[slot].w = u2f(y);
    }
    uint4* sched = a.slot_meta + slot * 3u + 1u;
    if (measured && change > 0.0f) sched->x = f2b(__fadd_rn(u2f(sched->x), change));
    if (urgent_if_binding) {
        float p = u2f(sched->x);
        urgent = urgent || !measured || (p > 0.0f && binds(a.state, slot, p, physical));
    }
    if (woken || urgent) sched->y &= 0xfffffff0u;
    if (urgent) a.slot_meta[slot * 3u + 2u].w |= kUrgent;
}

// face_slot (voxel_accumulate.wgsl:357-370): the face index's slot for
// (voxel, face), or kNoLimit.
__device__ uint32_t face_slot(const uint4* index, int x, int y, int z, uint32_t face) {
    const uint4 header = index[0];
    uint32_t probe = (hash_voxel(x, y, z) ^ pcg(face + 1u)) & header.x;
#pragma unroll 1
    for (uint32_t attempt = 0; attempt < header.y; ++attempt) {
        const uint4 e = index[probe + 1u];
        if (e.w == 0xffffffffu) return kNoLimit;
        if ((int)e.x == x && (int)e.y == y && (int)e.z == z && (e.w >> 29u) == face) return e.w & 0x1fffffffu;
        probe = (probe + 1u) & header.x;
    }
    return kNoLimit;
}

// measure_edits (voxel_accumulate.wgsl:375-403), one thread per scan
// position: the brightest outgoing luminance (albedo times incident mean and
// direct luminance, plus emission) of the position's traced faces, folded
// into its entry with an atomic max of the float bits (non-negative values
// order like their bits) tagged by the high bit as "observed". Entries are
// laid out by first position, so a binary search finds a position's entry.
__global__ void __launch_bounds__(kBlock) measure_edits_kernel(const uint4* state, const uint4* slot_meta, const uint4* index,
                                                               const float2* material_light, const uint4* measures,
                                                               uint32_t n_entries, uint32_t n_positions, uint32_t* measure_max) {
    const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= n_positions) return;
    uint32_t lo = 0, hi = n_entries;
#pragma unroll 1
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if (measures[mid * 3u].y <= t) lo = mid;
        else hi = mid;
    }
    const uint4 a = measures[lo * 3u], b = measures[lo * 3u + 1u], size = measures[lo * 3u + 2u];
    if (t < a.y || t >= a.y + a.z) return;
    const uint32_t local = t - a.y;
    const int x = (int)b.x + (int)(local % size.x), y = (int)b.y + (int)((local / size.x) % size.y),
              z = (int)b.z + (int)(local / (size.x * size.y));
    float brightest = 0.0f;
    bool observed = false;
#pragma unroll 1
    for (uint32_t face = 0; face < 6u; ++face) {
        const uint32_t slot = face_slot(index, x, y, z, face);
        if (slot == kNoLimit) continue;
        const uint4 identity = slot_meta[slot * 3u];
        if ((identity.w & 8u) == 0u) continue;
        if ((state[slot * 9u + 1u].y & 0x7fffffffu) == 0u) continue;
        observed = true;
        const uint4 m = state[slot * 9u], d = state[slot * 9u + 4u];
        const float incident = __fadd_rn(lum3(u2f(m.x), u2f(m.y), u2f(m.z)), lum3(u2f(d.x), u2f(d.y), u2f(d.z)));
        const float2 light = material_light[identity.w >> 16u];
        brightest = wmax(brightest, __fadd_rn(__fmul_rn(light.x, incident), light.y));
    }
    if (observed) atomicMax(measure_max + lo, f2b(brightest) | 0x80000000u);
}

// finish_edits (voxel_accumulate.wgsl:407-423), one thread per entry: the
// bound's flux becomes its own emission plus the brightest outgoing
// luminance times two faces per changed voxel, and its kind a measured edit
// (3); an edit with no traced face in its scan becomes unknown (0).
__global__ void __launch_bounds__(kBlock) finish_edits_kernel(const uint4* measures, uint32_t n_entries, const uint32_t* measure_max,
                                                              uint4* events) {
    const uint32_t e = blockIdx.x * kBlock + threadIdx.x;
    if (e >= n_entries) return;
    const uint4 a = measures[e * 3u];
    const float base_flux = u2f(measures[e * 3u + 1u].w);
    const uint32_t observation = measure_max[e];
    if ((observation & 0x80000000u) == 0u) {
        events[a.x + 1u].w &= 0xfffffff8u;
        return;
    }
    const float brightest = u2f(observation & 0x7fffffffu);
    events[a.x].w = f2b(__fadd_rn(base_flux, __fmul_rn(__fmul_rn(brightest, 2.0f), (float)a.w)));
    events[a.x + 1u].w = (events[a.x + 1u].w & 0xfffffff8u) | 3u;
}

// A new slot's incarnation (state word 28): the resident allocator numbers
// slots from 1 as it creates them (src/gpu/resident.rs:457-468).
__global__ void __launch_bounds__(kBlock) seed_incarnations_kernel(uint4* state, uint32_t n) {
    const uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
    if (slot < n) state[slot * 9u + 7u].x = slot + 1u;
}

}  // namespace

void launch_seed_incarnations(uint4* state, uint32_t n, cudaStream_t s) {
    if (n) seed_incarnations_kernel<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(state, n);
}

void launch_measure_edits(const uint4* state, const uint4* slot_meta, const uint4* index, const float2* material_light,
                          const uint4* measures, uint32_t n_entries, uint32_t n_positions, uint32_t* measure_max, uint4* events,
                          cudaStream_t s) {
    if (n_entries == 0) return;
    cudaMemsetAsync(measure_max, 0, (size_t)n_entries * 4, s);
    if (n_positions)
        measure_edits_kernel<<<(n_positions + kBlock - 1) / kBlock, kBlock, 0, s>>>(state, slot_meta, index, material_light, measures,
                                                                                   n_entries, n_positions, measure_max);
    finish_edits_kernel<<<(n_entries + kBlock - 1) / kBlock, kBlock, 0, s>>>(measures, n_entries, measure_max, events);
}

const void* prepare_kernel_address() { return reinterpret_cast<const void*>(&prepare_kernel); }
const void* accumulate_kernel_address() { return reinterpret_cast<const void*>(&accumulate_kernel); }

void launch_prepare(const AccumArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    prepare_kernel<<<(a.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
}
void launch_accumulate(const AccumArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    accumulate_kernel<<<(a.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
}
void launch_apply_events(const AccumArgs& a, const uint4* events, uint32_t n_slots, cudaStream_t s) {
    if (n_slots == 0) return;
    apply_events_kernel<<<(n_slots + kBlock - 1) / kBlock, kBlock, 0, s>>>(a, events, n_slots);
}

}  // namespace vgi
