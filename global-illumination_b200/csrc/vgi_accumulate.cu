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
    // record_stability; tasks from batch.x on are GPU picks, whose record
    // reports the merged count and whose CPU mirror becomes stale.
    const bool picked = i >= ctl[24];
    if (picked && a.picks) a.picks[i].z = count;
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
    *rank_p = make_uint4(f2b(sample_noise(nm, ns)), ctl[2], f2b(max3(rr, rg, rb)),
                         0x80000000u | scount | (picked ? kMirrorStale : (rank.w & kMirrorStale)));
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

// ---- GPU selection (voxel_accumulate.wgsl:448-695) ----------------------------
// Controls words as the reference's Controls: counts.z = [2] clock ms;
// limits.z = [14] slots; schedule = [16..19] (revision, stable error bits,
// stable samples, audit interval ms); focus = [20..23] (voxel xyz, pick
// budget); batch = [24..27] (CPU traced faces, batch id, classify range);
// mirror.x = [32] mirror records per batch.
constexpr uint32_t kBootstrap = 8u, kClasses = 4u;
constexpr uint32_t kSelThreshold = 1024u, kSelRemainder = 1028u, kSelTies = 1032u, kSelTotal = 1036u, kSelMirrors = 1037u;

__device__ __forceinline__ int page_axis(int p) { return (p - (p < 0 ? 31 : 0)) / 32; }

// candidate (voxel_accumulate.wgsl:474-511): class (0 coverage, 1 refinement,
// 2 sweep, 3 urgent) << 8 | key bucket, or kNoIndex.
__device__ uint32_t candidate_key(const AccumArgs& a, uint32_t slot) {
    const uint32_t* ctl = a.controls;
    const uint4 identity = a.slot_meta[slot * 3u];
    if ((identity.w & 8u) == 0u) return kNoIndex;
    const uint4 schedule = a.slot_meta[slot * 3u + 1u];
    const uint32_t last_cpu = schedule.y >> 4u;
    if (last_cpu != 0u && ((ctl[25] - last_cpu) & 0x0fffffffu) < 4u) return kNoIndex;
    const uint4 rank = a.slot_meta[slot * 3u + 2u];
    const uint32_t count = rank.w & 0x1fffffffu;
    const bool fresh = (schedule.y & 8u) != 0u && schedule.w == ctl[16];
    const uint32_t since = ctl[2] - rank.y;
    const uint32_t age_ms = rank.w < 0x80000000u ? 0x7fffffffu : (since > 0x7fffffffu ? 0u : since);
    const uint32_t required = u2f(rank.z) < 0.02f ? (ctl[18] > 256u ? ctl[18] : 256u) : ctl[18];
    const bool due = !fresh || count < required || (schedule.y & 7u) < 4u || age_ms >= ctl[19] || (rank.w & kUrgent) != 0u;
    if (!due) return kNoIndex;
    const int px = (int)identity.x, py = (int)identity.y, pz = (int)identity.z;
    const int fx = (int)ctl[20], fy = (int)ctl[21], fz = (int)ctl[22];
    if ((rank.w & kUrgent) != 0u || count < kBootstrap) {
        const float dx = (float)(px - fx), dy = (float)(py - fy), dz = (float)(pz - fz);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        const uint32_t b = f2u(__fmul_rn(own_log2(__fadd_rn(d2, 1.0f)), 8.0f));
        return (((rank.w & kUrgent) != 0u ? 3u : 0u) << 8u) | (b < 255u ? b : 255u);
    }
    const int ax = abs(page_axis(px) - page_axis(fx)), ay = abs(page_axis(py) - page_axis(fy)), az = abs(page_axis(pz) - page_axis(fz));
    const int page_distance = ax > ay ? (ax > az ? ax : az) : (ay > az ? ay : az);
    if (page_distance <= 2) {
        const float age = wmin(__fmul_rn((float)age_ms, 0.001f), 10.0f);
        const float error = count < 2u ? 1.0f : wmin(__fdiv_rn(u2f(rank.x), __fsqrt_rn((float)count)), 8.0f);
        const float priority = __fadd_rn(__fadd_rn(error, __fmul_rn(age, 0.1f)), page_distance <= 1 ? 0.25f : 0.0f);
        const uint32_t b = f2u(__fmul_rn(wmax(__fadd_rn(own_log2(priority), 8.0f), 0.0f), 16.0f));
        return (1u << 8u) | (255u - (b < 255u ? b : 255u));
    }
    const uint32_t b = f2u(__fmul_rn(own_log2(__fadd_rn((float)age_ms, 1.0f)), 8.0f));
    return (2u << 8u) | (255u - (b < 255u ? b : 255u));
}

// select_classify: keys of the slots [batch.z, batch.w); faces whose
// statistics mirror is stale are counted, and emitted up to mirror.x.
__global__ void __launch_bounds__(kBlock) select_classify_kernel(AccumArgs a, uint32_t* keys, uint32_t* selection) {
    __shared__ uint32_t group_mirrors, group_base;
    const uint32_t* ctl = a.controls;
    if (threadIdx.x == 0) group_mirrors = 0u;
    __syncthreads();
    const uint32_t slot = ctl[26] + blockIdx.x * kBlock + threadIdx.x;
    bool stale = false;
    uint32_t mirror_index = 0u;
    if (slot < ctl[27]) {
        keys[slot] = candidate_key(a, slot);
        stale = (a.slot_meta[slot * 3u + 2u].w & kMirrorStale) != 0u && (a.slot_meta[slot * 3u].w & 8u) != 0u;
        if (stale) mirror_index = atomicAdd(&group_mirrors, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) group_base = group_mirrors > 0u ? atomicAdd(selection + kSelMirrors, group_mirrors) : 0u;
    __syncthreads();
    // No statistics mirror here beyond mirror.x records (the CPU mirror is
    // the crate's): a face counted past it keeps its stale flag.
    if (!stale || group_base + mirror_index >= ctl[32]) return;
    a.slot_meta[slot * 3u + 2u].w &= ~kMirrorStale;
}

// select_histogram: per-class 256-bucket histograms of the keys.
__global__ void __launch_bounds__(kBlock) select_histogram_kernel(const uint32_t* keys, uint32_t n_slots, uint32_t* selection) {
    __shared__ uint32_t local[1024];
    for (uint32_t b = threadIdx.x; b < 1024u; b += kBlock) local[b] = 0u;
    __syncthreads();
    const uint32_t id = blockIdx.x * kBlock + threadIdx.x;
    if (id < n_slots) {
        const uint32_t key = keys[id];
        if (key != kNoIndex) atomicAdd(local + ((key >> 8u) < 3u ? (key >> 8u) : 3u) * 256u + (key & 255u), 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < 1024u; b += kBlock)
        if (local[b] != 0u) atomicAdd(selection + b, local[b]);
}

// select_threshold: one block; inclusive scans of the histograms, the
// per-class quotas (urgent first, then 1/4, 1/2, 1/4 with unused share lent
// to refinement, coverage, sweep, urgent), the threshold bucket and the
// ties it takes.
__global__ void __launch_bounds__(kBlock) select_threshold_kernel(const uint32_t* controls_budget, uint32_t budget, uint32_t* selection) {
    __shared__ uint32_t scan[1024];
    __shared__ uint32_t taken[4];
    const uint32_t t = threadIdx.x;
    for (uint32_t c = 0; c < kClasses; ++c) scan[c * 256u + t] = selection[c * 256u + t];
    __syncthreads();
    for (uint32_t step = 1u; step < 256u; step <<= 1u) {
        uint32_t add[4] = {0u, 0u, 0u, 0u};
        for (uint32_t c = 0; c < kClasses; ++c)
            if (t >= step) add[c] = scan[c * 256u + t - step];
        __syncthreads();
        for (uint32_t c = 0; c < kClasses; ++c) scan[c * 256u + t] += add[c];
        __syncthreads();
    }
    if (t == 0u) {
        uint32_t take[4] = {0u, 0u, 0u, 0u};
        const uint32_t u = scan[3u * 256u + 255u], q = budget - budget / 4u;
        take[3] = u < q ? u : q;
        const uint32_t rest = budget - take[3];
        take[0] = rest / 4u < scan[255u] ? rest / 4u : scan[255u];
        take[1] = rest / 2u < scan[256u + 255u] ? rest / 2u : scan[256u + 255u];
        const uint32_t r2 = rest - rest / 4u - rest / 2u;
        take[2] = r2 < scan[512u + 255u] ? r2 : scan[512u + 255u];
        uint32_t spare = budget - take[0] - take[1] - take[2] - take[3];
        const uint32_t lend[4] = {1u, 0u, 2u, 3u};
        for (uint32_t o = 0; o < kClasses; ++o) {
            const uint32_t c = lend[o];
            const uint32_t room = scan[c * 256u + 255u] - take[c];
            const uint32_t extra = spare < room ? spare : room;
            take[c] += extra;
            spare -= extra;
        }
        for (uint32_t c = 0; c < kClasses; ++c) {
            taken[c] = take[c];
            selection[kSelThreshold + c] = 256u;
            selection[kSelRemainder + c] = 0u;
        }
    }
    __syncthreads();
    for (uint32_t c = 0; c < kClasses; ++c) {
        const uint32_t below = t > 0u ? scan[c * 256u + t - 1u] : 0u;
        if (taken[c] > 0u && below < taken[c] && scan[c * 256u + t] >= taken[c]) {
            selection[kSelThreshold + c] = t;
            selection[kSelRemainder + c] = taken[c] - below;
        }
    }
    (void)controls_budget;
}

// select_emit: the picks, appended after the CPU's traced faces: a task
// (voxel, face, current sequence), the pick record and the task's slot.
// Ties at a threshold bucket and picks are reserved per block.
__global__ void __launch_bounds__(kBlock) select_emit_kernel(AccumArgs a, uint32_t n_slots, uint32_t* keys, uint32_t* selection,
                                                             uint32_t* pick_slots) {
    __shared__ uint32_t group_ties[4], group_tie_base[4], group_picks, group_pick_base;
    const uint32_t* ctl = a.controls;
    if (threadIdx.x < kClasses) group_ties[threadIdx.x] = 0u;
    if (threadIdx.x == 0) group_picks = 0u;
    __syncthreads();
    const uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t key = slot < n_slots ? keys[slot] : kNoIndex;
    const uint32_t group = (key >> 8u) < 3u ? (key >> 8u) : 3u, bucket = key & 255u;
    const uint32_t threshold = atomicAdd(selection + kSelThreshold + group, 0u);
    const bool candidate = key != kNoIndex && bucket <= threshold;
    const bool tie = candidate && bucket == threshold;
    uint32_t tie_index = 0u;
    if (tie) tie_index = atomicAdd(group_ties + group, 1u);
    __syncthreads();
    if (threadIdx.x < kClasses) {
        const uint32_t n = group_ties[threadIdx.x];
        group_tie_base[threadIdx.x] = n > 0u ? atomicAdd(selection + kSelTies + threadIdx.x, n) : 0u;
    }
    __syncthreads();
    const bool accept = candidate && (!tie || group_tie_base[group] + tie_index < atomicAdd(selection + kSelRemainder + group, 0u));
    uint32_t pick_index = 0u;
    if (accept) pick_index = atomicAdd(&group_picks, 1u);
    __syncthreads();
    if (threadIdx.x == 0) group_pick_base = group_picks > 0u ? atomicAdd(selection + kSelTotal, group_picks) : 0u;
    __syncthreads();
    const uint32_t pick = group_pick_base + pick_index;
    if (!accept || pick >= ctl[23]) return;
    keys[slot] = kNoIndex;  // re-ranked when its range comes round
    const uint4 identity = a.slot_meta[slot * 3u];
    if ((identity.w & 8u) == 0u) return;  // a stale key of a retired slot: a hole
    const uint32_t task = ctl[24] + pick;
    const uint4* st = a.state + slot * 9u;
    a.tasks[task * 2u] = make_uint4(identity.x, identity.y, identity.z, identity.w & 7u);
    a.tasks[task * 2u + 1u].x = st[1].z;  // begin_trace
    pick_slots[task] = slot;
    a.picks[task] = make_uint4(slot, a.slot_meta[slot * 3u + 1u].z, st[1].y & 0x3fffffffu, st[7].x);
}

// mark_changed (voxel_accumulate.wgsl:432-446) for the traced tasks.
__global__ void __launch_bounds__(kBlock) mark_changed_kernel(AccumArgs a) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= a.n || i >= a.controls[0]) return;
    const uint32_t slot = a.slots ? a.slots[i] : i;
    if (slot == kNoIndex) return;
    uint4* sm = a.slot_meta + slot * 3u + 1u;
    const float pending = u2f(sm->x);
    if (pending <= 0.0f) return;
    if (binds(a.state, slot, pending, u2f(a.controls[11]))) a.state[slot * 9u + 1u].y |= 0x80000000u;
    else sm->x = 0u;
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
void launch_select(const AccumArgs& a, uint32_t n_slots, uint32_t* keys, uint32_t* selection, uint32_t* pick_slots, cudaStream_t s) {
    const uint32_t first = a.controls[26], end = a.controls[27];
    if (end > first) select_classify_kernel<<<(end - first + kBlock - 1) / kBlock, kBlock, 0, s>>>(a, keys, selection);
    const uint32_t blocks = (n_slots + kBlock - 1) / kBlock;
    if (blocks) select_histogram_kernel<<<blocks, kBlock, 0, s>>>(keys, n_slots, selection);
    select_threshold_kernel<<<1, kBlock, 0, s>>>(nullptr, a.controls[23], selection);
    if (blocks) select_emit_kernel<<<blocks, kBlock, 0, s>>>(a, n_slots, keys, selection, pick_slots);
}

void launch_mark_changed(const AccumArgs& a, cudaStream_t s) {
    if (a.n) mark_changed_kernel<<<(a.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
}

void launch_apply_events(const AccumArgs& a, const uint4* events, uint32_t n_slots, cudaStream_t s) {
    if (n_slots == 0) return;
    apply_events_kernel<<<(n_slots + kBlock - 1) / kBlock, kBlock, 0, s>>>(a, events, n_slots);
}

}  // namespace vgi
