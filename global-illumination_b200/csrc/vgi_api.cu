// libvgi C ABI (include/vgi.h): context, device buffers and the per-frame
// sequence. One CUDA stream per context; all device memory is owned here.
#include "../../include/vgi.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "vgi_runtime.h"
#include "vgi_types.cuh"

namespace vgi {
void launch_classify_pack(const uint16_t* voxels, const uint32_t* regions, uint32_t grid, uint32_t n, uint4* headers, uint32_t* cells,
                          unsigned long long* alloc, unsigned long long capacity, uint32_t* error, cudaStream_t s);
void launch_scatter_edits(const uint2* edits, uint32_t n, uint16_t* voxels, cudaStream_t s);
void launch_set_header_extents(uint4* headers, const uint2* zw, uint32_t n, cudaStream_t s);
void launch_grid_headers(const int32_t* grid, uint32_t n, const uint4* headers, uint4* out, cudaStream_t s);
void launch_scatter_regions(const uint16_t* staged, const uint32_t* slots, uint32_t n, uint16_t* voxels, cudaStream_t s);
void launch_clear_headers(uint4* headers, const uint32_t* slots, uint32_t n, cudaStream_t s);
void launch_dedup_bricks(const uint4* headers, uint32_t n, uint32_t* cells, uint32_t* table, uint32_t mask, uint32_t* error,
                         cudaStream_t s);
}  // namespace vgi

namespace {

using namespace vgi;

// Failures injected by vgi_inject_failure for the calling thread (a context
// has one owner thread): the next `alloc` device allocations and `upload`
// host-to-device copies fail without reaching the device.
thread_local uint32_t t_fail_allocs = 0, t_fail_uploads = 0;

// A host-to-device copy on `s`, or the injected failure.
cudaError_t h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (t_fail_uploads) {
        --t_fail_uploads;
        return cudaErrorInvalidValue;
    }
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
}

template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;  // elements allocated
    cudaError_t reserve(size_t n) {
        if (n <= count && ptr) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        if (n == 0) return cudaSuccess;
        if (t_fail_allocs) {
            --t_fail_allocs;
            return cudaErrorMemoryAllocation;
        }
        cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e == cudaSuccess) count = n;
        return e;
    }
    // Grows to at least n elements (half as much again as before, at least),
    // keeping the first `keep` elements; stream-ordered, then synchronised.
    cudaError_t grow(size_t n, size_t keep, cudaStream_t s) {
        if (n <= count && ptr) return cudaSuccess;
        const size_t cap = std::max(n, count + count / 2);
        if (t_fail_allocs) {
            --t_fail_allocs;
            return cudaErrorMemoryAllocation;
        }
        T* fresh = nullptr;
        cudaError_t e = cudaMalloc(&fresh, cap * sizeof(T));
        if (e != cudaSuccess) return e;
        if (ptr && keep) e = cudaMemcpyAsync(fresh, ptr, std::min(keep, count) * sizeof(T), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaFree(fresh);
            return e;
        }
        if (ptr) cudaFree(ptr);
        ptr = fresh;
        count = cap;
        return cudaSuccess;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
};

constexpr uint32_t kHistoryLimit = 65536;
constexpr uint32_t kMlpHistoryFloor = 32;  // above the cache-binding count of 16
constexpr float kMaxPathDistance = 768.0f;

}  // namespace

struct vgi_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;

    // geometry
    std::vector<RegionKey> keys;
    std::unordered_map<RegionKey, uint32_t, RegionKeyHash> where;
    std::vector<uint16_t> host_voxels;
    std::vector<uint8_t> strides;
    std::vector<uint4> host_headers;
    TopLevelField top;
    int32_t bounds[6] = {0, 0, 0, 0, 0, 0};
    uint64_t dir_slots = 0;
    uint64_t cells_used = 0;
    bool geometry = false;
    // Region residency (vgi_load_regions / vgi_unload_regions): keys, voxels,
    // strides and headers are per header slot; `live` marks the slots that
    // hold a region, freed slots are reused last freed first, and the
    // directory is kept on the host and changed in place.
    std::vector<uint8_t> live;
    std::vector<uint32_t> free_slots;
    std::vector<int32_t> host_dir;
    std::vector<uint32_t> host_cells;  // packed geometry only: the cells vgi_patch_packed patches
    bool packed_geometry = false;  // from vgi_upload_packed: no voxels to repack
    DevBuf<uint16_t> staged_voxels;
    DevBuf<uint32_t> slot_list;
    DevBuf<int4> directory;
    DevBuf<int32_t> grid;  // region_grid: header index per region of the bounding box
    DevBuf<uint4> grid_headers;  // the header each grid cell names (kind 0: none)
    uint64_t grid_cells = 0;
    bool has_grid = false;
    DevBuf<uint4> headers;
    DevBuf<uint32_t> cells;
    DevBuf<uint16_t> voxels;
    DevBuf<unsigned long long> alloc;
    DevBuf<uint32_t> pack_error;
    DevBuf<uint2> edit_buf;
    DevBuf<uint2> zw;
    DevBuf<uint32_t> region_list;
    DevBuf<uint32_t> dedup_table;

    // model
    std::vector<float> host_materials = std::vector<float>(256 * 16, 0.0f);
    std::vector<uint32_t> host_emitter_records;  // 8 words per emitter face
    DevBuf<float4> materials;
    DevBuf<float2> material_light;  // (albedo, emission) luminance per material
    DevBuf<uint4> measures;
    DevBuf<uint32_t> measure_max;
    DevBuf<float4> lights;
    uint32_t n_lights = 0, n_directional = 0;
    float env[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    DevBuf<uint4> emitters;
    DevBuf<float4> node_aux;
    // Per slot, the light tree's top child probabilities at its receiver
    // (TraceArgs::tree_rows), checked against the generation of the tree.
    DevBuf<uint4> tree_rows;
    uint32_t tree_generation = 1;
    float emitter_count = 0.0f, emitter_total = 0.0f;
    vgi_transport transport{};

    // face cache
    uint32_t n_slots = 0;
    DevBuf<uint4> tasks, results, state, slot_meta, checkpoint, face_index;
    DevBuf<float4> cache;
    DevBuf<uint4> scratch_tasks, scratch_results;
    // Pipelined batches (vgi_submit_batch): host copies on their own streams
    // through two device staging buffers each way, so a batch's copies
    // overlap the frames around it.
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    DevBuf<uint4> stage_tasks[2], stage_results[2];
    cudaEvent_t tasks_ready[2] = {}, tasks_free[2] = {}, results_ready[2] = {}, results_done[2] = {};
    uint64_t submitted = 0;
    // Scheduled frames (vgi_frame_scheduled): selection keys (kept between
    // frames), selection scratch, and the picks' tasks, slots, records and results.
    DevBuf<uint32_t> sel_keys, selection, pick_slots;
    DevBuf<uint4> pick_tasks, pick_records, pick_results;
    uint32_t pick_budget = 0;
    bool keys_reset = true;  // the face set changed: every key starts as "not a candidate"
    // view tier: receivers, paths, continuations, estimates, owner queue, events
    DevBuf<uint4> v_receivers, v_paths, v_conts, v_estimates, v_events, v_scratch;
    DevBuf<uint32_t> v_queue;
    // MLP radiance cache: FP32 master weights, their packed BF16 image
    DevBuf<float> mlp_master;
    DevBuf<uint8_t> mlp_image;
    DevBuf<uint32_t> mlp_error;               // [0] API calls and training, [1] the frames' queries
    DevBuf<uint8_t> mlp_image_b;              // W (rows = inputs): B operand of the backward pass
    DevBuf<float> mlp_adam;                   // Adam first and second moments, 2 x 19456
    DevBuf<float> mlp_grads;                  // 19456 gradients + the loss of the last batch
    DevBuf<float> mlp_partials;               // per training CTA: gradient sums + loss
    DevBuf<uint32_t> mlp_steps;               // Adam steps taken, blocks done (device words: a frame graph replays them)
    DevBuf<float4> w_mlp_queue;               // 2 per path: the frame's network queries
    DevBuf<float> mlp_features;               // training rows of a frame (batch x steps x 96)
    DevBuf<float4> mlp_targets;
    DevBuf<uint4> mlp_train_tasks;            // the frame's training faces (FaceTasks) and their traced results
    DevBuf<uint4> mlp_train_results;
    DevBuf<uint32_t> mlp_query_count;         // queries of the last terminating frame
    uint32_t mlp_queue_capacity = 0;          // paths of the last terminating frame's trace
    uint32_t mlp_ctas = 0, mlp_sms = 0;
    uint32_t mlp_wait = kMlpWaitPolls;  // polls per tensor-core wait (vgi_mlp_set_wait_limit)
    // MLP termination in vgi_frame: off, or on after `mlp_warm` plain frames
    // that train the network; `mlp_batch` rows x `mlp_train_steps` steps a frame.
    bool mlp_cache = false;
    uint32_t mlp_warm = 0, mlp_batch = 65536, mlp_train_steps = 1, mlp_frames = 0;
    float mlp_lr = 1e-2f;
    // vgi_set_mlp_schedule: 0, or the share of the samples taken since the
    // network began ending paths that a face's mean covers.
    float mlp_history = 0.0f;
    // vgi_set_mlp_schedule: rows of one Adam step (0: samples / steps).
    uint32_t mlp_step_rows = 0;
    bool graph_mlp = false;                   // the captured frame's trace ends paths with the network
    bool mlp_timed = false;                   // the last timed frame recorded mlp_marks
    bool mlp_queried = false;                 // a frame has queried the network (counters[4] holds its count)
    uint32_t n_view = 0;
    // The view receivers' owner hash for the far tier's handoff (stale after
    // vgi_view_set_receivers).
    DevBuf<uint32_t> v_hash;
    uint32_t v_hash_mask = 0;
    bool v_hash_valid = false;
    bool custom_lights = false;               // some light has custom visible RGB
    // discovery and presentation scratch, kept between calls
    DevBuf<float> disc_cam;
    DevBuf<uint4> disc_pixels;
    DevBuf<unsigned long long> disc_set;
    DevBuf<int4> disc_list;
    DevBuf<uint32_t> disc_counters;
    DevBuf<float4> present_image;
    // reconstruction: screen tile per view receiver (CSR lists per tile),
    // the published FarPixels and the publish counters
    DevBuf<uint32_t> v_tile_of, v_tile_start, v_tile_items;
    uint32_t v_tiles[2] = {0, 0};
    uint32_t v_tiles_n = 0;                   // receivers the tiles were given for
    DevBuf<uint4> v_published;
    DevBuf<uint32_t> v_publish_stats;
    bool v_published_valid = false;
    // far tier: cell histories (this frame's and the previous one's), the
    // output cells, the trace queue and the statistics
    DevBuf<uint4> far_cells[2];
    DevBuf<uint4> far_output;
    DevBuf<uint32_t> far_queue, far_stats;
    uint32_t far_current = 0;
    uint32_t far_shape[4] = {0, 0, 0, 0};     // cells x, y, pixels per side, enabled | measure << 1
    uint32_t far_size[2] = {0, 0};            // viewport
    float far_prev[10] = {};
    uint32_t far_last_frame = 0;
    bool far_has_prev = false;
    bool far_handoff = false;                 // view frames seed new receivers from far cells
    bool topology_prior = false;              // view frames seed new receivers from their neighbours
    uint32_t view_frames = 0;                 // view frames since the receivers were set
    DevBuf<uint4> v_prev_estimates;           // the estimates before a frame's seeding
    DevBuf<uint4> events;
    DevBuf<int4> footprints;                 // change-footprint tasks of the last event list
    DevBuf<uint32_t> footprint_sums;
    uint32_t n_events = 0;
    uint64_t n_events_read = 0;  // uint4 words of the last measured event list, readable back
    DevBuf<unsigned long long> counters;
    uint32_t batch_id = 1;

    // frame timing
    bool timing = false;
    // Frame graph: vgi_frame's launches captured once per face set and
    // sample count, replayed with the prepare and accumulate arguments
    // updated per frame. Any setter marks it stale.
    bool use_graph = false;
    bool graph_dirty = true;
    uint32_t graph_samples = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraphNode_t graph_prepare = nullptr, graph_accumulate = nullptr;
    cudaEvent_t marks[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t traverse_marks[8] = {};
    cudaEvent_t mlp_marks[4] = {};            // network queries, then training, of the last timed frame
    uint32_t traverse_launches = 0;  // traversal launches of the last timed wavefront frame

    // trace layout and the wavefront's buffers
    uint32_t layout = VGI_LAYOUT_WAVEFRONT;
    uint32_t traverse_blocks = 0;
    uint32_t refill_min = 8;
    DevBuf<float4> w_state, w_ray;
    DevBuf<uint4> w_hit;
    DevBuf<uint32_t> w_status, w_queue0, w_queue1, w_scatter, w_counters;
};

extern "C" {
static int mlp_frame_training(vgi_ctx* c);
}

namespace {

int fail(vgi_ctx* c, int code, const std::string& what) {
    if (c) c->error = what;
    return code;
}
#define VGI_CUDA(c, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail((c), VGI_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

vgi_transport default_transport() {
    vgi_transport t{};
    t.reach = kMaxPathDistance;
    t.bounces = 3;
    t.path_steps = 2048;
    t.budgeted = 0;
    t.history_limit = 0;
    t.recency = 1.0f;
    t.measured_retention = 1.0f;
    t.response_seconds = 0.075f;
    t.lanes = 0;
    t.transport_revision = 0;
    t.stable_error = 0.12f;
    t.stable_samples = 32;
    return t;
}

// TransportSettings::normalized (src/settings.rs:413-426)
float norm_reach(float r) { return std::isfinite(r) ? std::min(std::max(r, 1.0f), kMaxPathDistance) : kMaxPathDistance; }
uint32_t norm_bounces(uint32_t b) { return std::min(std::max(b, 1u), 3u); }

uint32_t lanes_log2(const vgi_transport& t, uint32_t samples) {
    uint32_t lanes = t.lanes;
    if (lanes == 0) {
        // One thread per sample for small sample counts; cap at 32.
        lanes = 1;
        while (lanes < samples && lanes < 32) lanes <<= 1;
        if (lanes > samples && lanes > 1) lanes >>= 1;
    }
    uint32_t l = 0;
    while ((1u << (l + 1)) <= lanes && l < 5) ++l;
    return l;
}

// The Controls uniform of shaders/voxel_accumulate.wgsl:11-15 as
// src/gpu/resident.rs:708-760 fills it, for a batch of CPU-owned faces.
void fill_controls(const vgi_ctx* c, uint32_t samples, uint32_t clock_ms, uint32_t* w) {
    std::memset(w, 0, 36 * 4);
    const vgi_transport& t = c->transport;
    w[0] = c->n_slots;
    w[1] = samples;
    w[2] = clock_ms;
    w[3] = t.history_limit == 0 ? kHistoryLimit : std::min(t.history_limit, kHistoryLimit);
    if (c->mlp_history > 0.0f && c->mlp_cache && c->mlp_frames >= c->mlp_warm) {
        // The MLP cache's growing window: the count cap is the given share of
        // the samples taken in frames the network answers (this one
        // included), at least kMlpHistoryFloor, so early frames' answers
        // from the untrained network fade from the means.
        const double taken = (double)samples * (double)(c->mlp_frames - c->mlp_warm + 1u);
        const double window = std::max((double)kMlpHistoryFloor, std::ceil((double)c->mlp_history * taken));
        w[3] = (uint32_t)std::min((double)w[3], window);
    }
    w[4] = fbits(std::max(t.response_seconds, 0.001f));
    w[5] = c->n_slots;
    w[10] = fbits(t.recency >= 1.0f ? t.recency : 1.0f);
    w[11] = fbits(std::max(t.measured_retention, 0.0f));
    w[13] = c->n_events;
    w[14] = c->n_slots;
    w[15] = 192u * 192u;  // INFLUENCE_RADIUS^2 (src/retention.rs:33-40)
    w[16] = t.transport_revision;
    w[17] = fbits(t.stable_error);
    w[18] = t.stable_samples;
    w[24] = c->n_slots;
    w[25] = c->batch_id;
    w[30] = 64u * 64u;  // MEASURED_RELIGHT_RADIUS^2 (src/geometry.rs:19)
    w[31] = 48u * 48u;  // RELIGHT_RADIUS^2 (src/geometry.rs:15)
}

TraceArgs trace_args(vgi_ctx* c, const uint4* tasks, uint4* results, uint32_t n, uint32_t samples, bool with_cache) {
    TraceArgs a{};
    a.directory = c->directory.ptr;
    a.headers = c->headers.ptr;
    a.cells = c->cells.ptr;
    a.dir_mask = (uint32_t)(c->dir_slots - 1);
    for (int k = 0; k < 3; ++k) {
        a.mn[k] = c->bounds[k];
        a.mx[k] = c->bounds[3 + k];
    }
    a.materials = c->materials.ptr;
    a.emitters = c->emitters.ptr;
    a.node_aux = c->node_aux.ptr;
    a.emitter_count = c->emitter_count;
    a.emitter_total = c->emitter_total;
    a.max_distance = kMaxPathDistance;
    a.reach = norm_reach(c->transport.reach);
    for (int k = 0; k < 4; ++k) a.env[k] = c->env[k];
    a.light_count = c->n_lights;
    a.lights = c->lights.ptr;
    a.region_grid = c->has_grid ? c->grid.ptr : nullptr;
    a.region_headers = c->has_grid ? c->grid_headers.ptr : nullptr;
    a.face_index = with_cache ? c->face_index.ptr : nullptr;
    // The kept tree rows follow the context's own face tasks only (a shard
    // of them from its first task's row).
    a.tree_rows = nullptr;
    if (tasks && c->tree_rows.ptr && tasks >= c->tasks.ptr && tasks < c->tasks.ptr + (size_t)c->n_slots * 2) {
        const size_t first = (size_t)(tasks - c->tasks.ptr);
        if (first % 2 == 0) a.tree_rows = c->tree_rows.ptr + first / 2 * kTreeRowWords;
    }
    a.tree_generation = c->tree_generation;
    a.cache = with_cache ? c->cache.ptr : nullptr;
    a.tasks = tasks;
    a.results = results;
    a.n_tasks = n;
    a.samples = samples;
    a.path_steps = c->transport.path_steps;
    a.lanes_log2 = lanes_log2(c->transport, samples);
    a.counters = c->counters.ptr;
    return a;
}

AccumArgs accum_args(vgi_ctx* c, uint32_t samples, uint32_t clock_ms) {
    AccumArgs a{};
    a.state = c->state.ptr;
    a.slot_meta = c->slot_meta.ptr;
    a.checkpoint = c->checkpoint.ptr;
    a.outputs = c->results.ptr;
    a.tasks = c->tasks.ptr;
    a.cache = c->cache.ptr;
    a.slots = nullptr;
    a.n = c->n_slots;
    fill_controls(c, samples, clock_ms, a.controls);
    return a;
}

int check_ready(vgi_ctx* c, bool need_faces) {
    if (!c) return VGI_ERR_INVALID;
    if (!c->geometry) return fail(c, VGI_ERR_STATE, "no geometry uploaded");
    if (!c->materials.ptr || !c->lights.ptr || !c->emitters.ptr) return fail(c, VGI_ERR_STATE, "model not set");
    if (need_faces && c->n_slots == 0) return fail(c, VGI_ERR_STATE, "no faces set");
    return VGI_OK;
}

bool transport_limited(const vgi_ctx* c) { return norm_reach(c->transport.reach) < kMaxPathDistance; }

// Releases the frame graph; the next frames launch directly until one is
// captured again.
void drop_graph(vgi_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    c->graph_prepare = c->graph_accumulate = nullptr;
    c->graph_dirty = true;
}

// The dense region grid the timed traversal reads instead of probing the
// directory: built when the bounding box holds at most 2^24 regions (64 MB).
cudaError_t upload_grid(vgi_ctx* c, const int32_t* directory, uint64_t slots) {
    const std::vector<int32_t> grid = region_grid(directory, slots, c->bounds, c->bounds + 3, 1ull << 24);
    c->has_grid = !grid.empty();
    c->grid_cells = grid.size();
    if (!c->has_grid) return cudaSuccess;
    cudaError_t e = c->grid.reserve(grid.size());
    if (e == cudaSuccess) e = c->grid_headers.reserve(grid.size());
    if (e != cudaSuccess) {
        c->has_grid = false;
        return e;
    }
    e = cudaMemcpyAsync(c->grid.ptr, grid.data(), grid.size() * 4, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return e;
    // The staging vector dies here, so the copy completes first.
    return cudaStreamSynchronize(c->stream);
}

// Copies the current headers into the grid's header cells; every call that
// changes the headers or the grid ends with it.
cudaError_t refresh_grid_headers(vgi_ctx* c) {
    if (!c->has_grid) return cudaSuccess;
    launch_grid_headers(c->grid.ptr, (uint32_t)c->grid_cells, c->headers.ptr, c->grid_headers.ptr, c->stream);
    return cudaGetLastError();
}

// Enqueues the face trace for `a` in the context's layout.
// Whether the trace ends uncached first hits with the network's prediction.
bool mlp_terminates(const vgi_ctx* c) {
    return c->mlp_cache && c->mlp_image.ptr && c->mlp_frames >= c->mlp_warm && c->layout == VGI_LAYOUT_WAVEFRONT;
}

// The network's position normalisation: the loaded regions' voxel box.
MlpEncoding mlp_encoding(const vgi_ctx* c) {
    MlpEncoding e{};
    for (int k = 0; k < 3; ++k) {
        const float lo = (float)c->bounds[k] * 16.0f, hi = (float)(c->bounds[3 + k] + 1) * 16.0f;
        e.lo[k] = lo;
        e.inv[k] = 1.0f / std::max(hi - lo, 1.0f);
    }
    return e;
}

// Samples per training face in an MLP-terminated frame's training trace.
#ifndef VGI_MLP_TRAIN_SAMPLES
#define VGI_MLP_TRAIN_SAMPLES 4
#endif
constexpr uint32_t kMlpTrainSamples = VGI_MLP_TRAIN_SAMPLES;

// `marks`: record the frame's timing events (off for the training trace).
// Sizes the context's wavefront buffers for a trace of `a` and describes
// them; drops the frame graph when a buffer moved.
int wave_buffers(vgi_ctx* c, const TraceArgs& a, bool count, bool marks, WaveBuffers& b) {
    const size_t paths = (size_t)a.n_tasks * a.samples;
    const size_t slots = paths * (2 + a.light_count) + (size_t)a.n_tasks * a.light_count;
    if (paths >= (1ull << 30) || slots > 0xffffffffull) return fail(c, VGI_ERR_CAPACITY, "too many paths for the wavefront layout");
    const bool mlp = mlp_terminates(c);
    // An MLP-terminated frame also traces its training faces in these
    // buffers: size them for both, so a captured frame never reallocates.
    size_t room_paths = paths, room_slots = slots;
    if (mlp) {
        const size_t rows = c->mlp_batch, tp = rows * kMlpTrainSamples;
        room_paths = std::max(room_paths, tp);
        room_slots = std::max(room_slots, tp * (2 + a.light_count) + rows * a.light_count);
    }
    const void* before[3] = {c->w_state.ptr, c->w_ray.ptr, c->w_status.ptr};
    VGI_CUDA(c, c->w_state.reserve(std::max<size_t>(room_paths, 1) * kWavePathFields));
    VGI_CUDA(c, c->w_ray.reserve(std::max<size_t>(room_slots, 1) * 2));
    VGI_CUDA(c, c->w_hit.reserve(std::max<size_t>(room_paths, 1) * 6));
    VGI_CUDA(c, c->w_status.reserve(std::max<size_t>(room_slots, 1)));
    VGI_CUDA(c, c->w_queue0.reserve(std::max<size_t>(room_slots, 1)));
    VGI_CUDA(c, c->w_queue1.reserve(std::max<size_t>(room_slots, 1)));
    VGI_CUDA(c, c->w_scatter.reserve(std::max<size_t>(room_paths, 1)));
    VGI_CUDA(c, c->w_counters.reserve(5));
    const void* queue_before = c->w_mlp_queue.ptr;
    if (mlp) VGI_CUDA(c, c->w_mlp_queue.reserve(std::max<size_t>(room_paths, 1) * 2));
    // A captured frame holds the old buffers' addresses.
    if (before[0] != c->w_state.ptr || before[1] != c->w_ray.ptr || before[2] != c->w_status.ptr || queue_before != c->w_mlp_queue.ptr)
        drop_graph(c);
    b = WaveBuffers{};
    b.state = c->w_state.ptr;
    b.ray = c->w_ray.ptr;
    b.hit = c->w_hit.ptr;
    b.status = c->w_status.ptr;
    b.queue[0] = c->w_queue0.ptr;
    b.queue[1] = c->w_queue1.ptr;
    b.scatter = c->w_scatter.ptr;
    b.counters = c->w_counters.ptr;
    b.traverse_blocks = c->traverse_blocks;
    b.refill_min = c->refill_min;
    b.traverse_marks = (c->timing && !count && marks) ? c->traverse_marks : nullptr;
    if (mlp) {
        b.mlp_image = c->mlp_image.ptr;
        b.mlp_queue = c->w_mlp_queue.ptr;
        b.mlp_error = c->mlp_error.ptr + 1;
        b.mlp_ctas = c->mlp_ctas;
        b.mlp_wait = c->mlp_wait;
        b.mlp_enc = mlp_encoding(c);
        if (c->timing && !count && marks) b.mlp_marks = c->mlp_marks;
        if (marks) c->mlp_queue_capacity = (uint32_t)paths;
    }
    if (b.traverse_marks) c->traverse_launches = std::min<uint32_t>((mlp ? 1u : c->transport.bounces) + 1u, 4u);
    return VGI_OK;
}

int run_trace(vgi_ctx* c, const TraceArgs& a, bool count, bool marks = true) {
    if (c->layout == VGI_LAYOUT_SINGLE_KERNEL) {
        if (c->timing && !count) c->traverse_launches = 0;
        launch_trace(a, c->transport.bounces, transport_limited(c), c->transport.budgeted != 0, count, c->stream);
        VGI_CUDA(c, cudaGetLastError());
        return VGI_OK;
    }
    WaveBuffers b;
    if (int e = wave_buffers(c, a, count, marks, b)) return e;
    launch_wave(b, a, c->transport.bounces, transport_limited(c), c->transport.budgeted != 0, count, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    return VGI_OK;
}

int read_counters(vgi_ctx* c, vgi_counters* out) {
    unsigned long long h[kCounterWords];
    VGI_CUDA(c, cudaMemcpyAsync(h, c->counters.ptr, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (out) {
        out->rays = h[0];
        out->paths = h[1];
        out->steps = h[2];
        out->bytes = h[3];
        out->unknown = h[4];
        out->cache_hits = h[5];
        for (int k = 0; k < 4; ++k) out->status[k] = h[6 + k];
        out->traverse_bytes = h[10];
        for (int k = 0; k < 2; ++k) {
            out->warp_passes[k] = h[11 + k];
            out->lane_passes[k] = h[13 + k];
        }
    }
    return VGI_OK;
}

// Headers z/w from the top-level field and strides; uploads them.
int finish_headers(vgi_ctx* c) {
    const uint32_t n = (uint32_t)c->keys.size();
    std::vector<uint2> zw(n, make_uint2(0u, 0u));
    for (uint32_t r = 0; r < n; ++r) {
        if (!c->live.empty() && !c->live[r]) continue;  // a freed slot (kind 0)
        Extents e = c->top.at(c->keys[r].x, c->keys[r].y, c->keys[r].z);
        uint32_t neg = (uint32_t)e[0] | ((uint32_t)e[2] << 8) | ((uint32_t)e[4] << 16);
        uint32_t pos = (uint32_t)e[1] | ((uint32_t)e[3] << 8) | ((uint32_t)e[5] << 16);
        pos |= (uint32_t)c->strides[r] << 28;
        zw[r] = make_uint2(neg, pos);
        c->host_headers[r].z = neg;
        c->host_headers[r].w = pos;
    }
    VGI_CUDA(c, c->zw.reserve(std::max<size_t>(n, 1)));
    VGI_CUDA(c, h2d(c->zw.ptr, zw.data(), n * sizeof(uint2), c->stream));
    launch_set_header_extents(c->headers.ptr, c->zw.ptr, n, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    return VGI_OK;
}

bool region_blocked(const vgi_ctx* c, int32_t x, int32_t y, int32_t z) {
    auto it = c->where.find(RegionKey{x, y, z});
    if (it == c->where.end()) return true;
    return c->host_headers[it->second].x != 1u;
}

// Runs classify_pack over `list` (region indices; null = all) and reads back
// the headers' kind/payload words.
int pack_regions(vgi_ctx* c, const std::vector<uint32_t>* list) {
    const uint32_t n = (uint32_t)c->keys.size();
    // With freed slots a full repack covers the live ones only.
    std::vector<uint32_t> live_list;
    if (!list && !c->free_slots.empty()) {
        for (uint32_t r = 0; r < n; ++r)
            if (c->live[r]) live_list.push_back(r);
        list = &live_list;
    }
    uint32_t grid = n;
    const uint32_t* dlist = nullptr;
    if (list) {
        grid = (uint32_t)list->size();
        VGI_CUDA(c, c->region_list.reserve(std::max<size_t>(grid, 1)));
        VGI_CUDA(c, h2d(c->region_list.ptr, list->data(), grid * 4, c->stream));
        dlist = c->region_list.ptr;
    }
    VGI_CUDA(c, h2d(c->alloc.ptr, &c->cells_used, 8, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->pack_error.ptr, 0, 4, c->stream));
    launch_classify_pack(c->voxels.ptr, dlist, grid, n, c->headers.ptr, c->cells.ptr, c->alloc.ptr, c->cells.count, c->pack_error.ptr,
                         c->stream);
    VGI_CUDA(c, cudaGetLastError());
    // Share identical brick payloads across every region (sized for all
    // bricks mixed, at most half full).
    size_t slots = 1;
    while (slots < (size_t)n * 128) slots <<= 1;
    VGI_CUDA(c, c->dedup_table.reserve(slots));
    VGI_CUDA(c, cudaMemsetAsync(c->dedup_table.ptr, 0xff, slots * 4, c->stream));
    launch_dedup_bricks(c->headers.ptr, n, c->cells.ptr, c->dedup_table.ptr, (uint32_t)(slots - 1), c->pack_error.ptr, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    uint32_t err = 0;
    unsigned long long used = 0;
    VGI_CUDA(c, cudaMemcpyAsync(&err, c->pack_error.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(&used, c->alloc.ptr, 8, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(c->host_headers.data(), c->headers.ptr, n * sizeof(uint4), cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err & 1u) return fail(c, VGI_ERR_CAPACITY, "cell arena exhausted");
    c->cells_used = used;
    return VGI_OK;
}

}  // namespace

extern "C" {

int vgi_create(const vgi_config* config, vgi_ctx** out) {
    if (!out) return VGI_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return VGI_UNAVAILABLE;
    int device = config ? config->device : 0;
    if (device < 0 || device >= count) return VGI_ERR_INVALID;
    // A device that cannot set up a context idles the caller like a missing
    // one (the reference's transport_unavailable after a failed pipeline
    // build, src/tests.rs:38-80): no context, VGI_UNAVAILABLE.
    if (cudaSetDevice(device) != cudaSuccess) return VGI_UNAVAILABLE;
    if (init_trace_constants() != cudaSuccess) return VGI_UNAVAILABLE;
    auto* c = new vgi_ctx();
    c->device = device;
    c->transport = default_transport();
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) sms = 1;
    c->traverse_blocks = (uint32_t)sms * wave_traverse_blocks_per_sm();
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        c->counters.reserve(16) != cudaSuccess || c->alloc.reserve(1) != cudaSuccess || c->pack_error.reserve(1) != cudaSuccess) {
        vgi_destroy(c);
        return VGI_UNAVAILABLE;
    }
    *out = c;
    return VGI_OK;
}

int vgi_destroy(vgi_ctx* c) {
    if (!c) return VGI_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    c->directory.release(); c->headers.release(); c->cells.release(); c->voxels.release(); c->alloc.release();
    c->pack_error.release(); c->edit_buf.release(); c->zw.release(); c->region_list.release(); c->dedup_table.release();
    c->materials.release(); c->lights.release(); c->emitters.release(); c->node_aux.release(); c->tree_rows.release();
    c->tasks.release(); c->results.release(); c->state.release(); c->slot_meta.release(); c->checkpoint.release();
    c->face_index.release(); c->cache.release(); c->grid.release(); c->scratch_tasks.release(); c->scratch_results.release(); c->events.release();
    c->material_light.release(); c->measures.release(); c->measure_max.release();
    c->v_receivers.release(); c->v_paths.release(); c->v_conts.release(); c->v_estimates.release(); c->v_events.release();
    c->v_scratch.release(); c->v_queue.release();
    c->mlp_master.release(); c->mlp_image.release(); c->mlp_error.release();
    c->mlp_image_b.release(); c->mlp_adam.release(); c->mlp_grads.release(); c->mlp_steps.release(); c->mlp_partials.release();
    c->w_mlp_queue.release(); c->mlp_features.release(); c->mlp_targets.release();
    c->footprints.release(); c->footprint_sums.release();
    c->sel_keys.release(); c->selection.release(); c->pick_slots.release();
    c->pick_tasks.release(); c->pick_records.release(); c->pick_results.release();
    c->mlp_train_tasks.release(); c->mlp_train_results.release(); c->mlp_query_count.release();
    c->counters.release();
    c->w_state.release(); c->w_ray.release(); c->w_hit.release(); c->w_status.release();
    c->w_queue0.release(); c->w_queue1.release(); c->w_scatter.release(); c->w_counters.release();
    for (auto& e : c->marks)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->traverse_marks)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->mlp_marks)
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < 2; ++k) {
        c->stage_tasks[k].release();
        c->stage_results[k].release();
        for (cudaEvent_t e : {c->tasks_ready[k], c->tasks_free[k], c->results_ready[k], c->results_done[k]})
            if (e) cudaEventDestroy(e);
    }
    if (c->copy_in) cudaStreamDestroy(c->copy_in);
    if (c->copy_out) cudaStreamDestroy(c->copy_out);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return VGI_OK;
}

const char* vgi_last_error(const vgi_ctx* c) { return c ? c->error.c_str() : "null context"; }

int vgi_stream(vgi_ctx* c, void** stream) {
    if (!c || !stream) return VGI_ERR_INVALID;
    *stream = (void*)c->stream;
    return VGI_OK;
}

int vgi_sync(vgi_ctx* c) {
    if (!c) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_upload_regions(vgi_ctx* c, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || (n && (!coords || !voxels))) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    // Refused inputs leave the context as it was.
    std::vector<RegionKey> keys(n, RegionKey{0, 0, 0});
    std::unordered_map<RegionKey, uint32_t, RegionKeyHash> where;
    for (uint32_t r = 0; r < n; ++r) {
        keys[r] = RegionKey{coords[r * 3], coords[r * 3 + 1], coords[r * 3 + 2]};
        if (!where.emplace(keys[r], r).second) return fail(c, VGI_ERR_INVALID, "duplicate region coordinate");
    }
    for (size_t i = 0; i < (size_t)n * 4096; ++i)
        if (voxels[i] > 256) return fail(c, VGI_ERR_INVALID, "voxel value above 256 (materials are 0..255, 256 is air)");
    // From here a failure (allocation, copy) leaves no geometry: frames and
    // edits are refused with VGI_ERR_STATE until an upload succeeds, and
    // never read half-replaced buffers.
    c->geometry = false;
    c->keys = std::move(keys);
    c->where = std::move(where);
    c->host_voxels.assign(voxels, voxels + (size_t)n * 4096);
    c->strides.assign(n, 0);
    if (strides) std::copy(strides, strides + n, c->strides.begin());
    c->host_headers.assign(n, make_uint4(0, 0, 0, 0));
    // Every region is live: the packer and the header pass read these.
    c->live.assign(n, 1);
    c->free_slots.clear();
    c->host_cells.clear();
    c->packed_geometry = false;
    // Worst case: every region mixed with 64 mixed bricks (64 + 64 * 32 words);
    // brick pointers are 30-bit word offsets.
    unsigned long long capacity = std::min<unsigned long long>((unsigned long long)n * (64 + 64 * 32) + 64, 1ull << 30);
    VGI_CUDA(c, c->voxels.reserve((size_t)std::max<uint32_t>(n, 1) * 4096));
    VGI_CUDA(c, c->headers.reserve(std::max<uint32_t>(n, 1)));
    VGI_CUDA(c, c->cells.reserve(capacity));
    c->cells.count = capacity;
    if (n) VGI_CUDA(c, h2d(c->voxels.ptr, voxels, (size_t)n * 8192, c->stream));
    c->cells_used = 0;
    int rc = pack_regions(c, nullptr);
    if (rc != VGI_OK) return rc;
    // Region bounds and the top-level field grown from an empty scene
    // (TransportScene::with_page_contents from the default scene).
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (n) {
        lo[0] = hi[0] = c->keys[0].x; lo[1] = hi[1] = c->keys[0].y; lo[2] = hi[2] = c->keys[0].z;
        for (const RegionKey& k : c->keys) {
            lo[0] = std::min(lo[0], k.x); lo[1] = std::min(lo[1], k.y); lo[2] = std::min(lo[2], k.z);
            hi[0] = std::max(hi[0], k.x); hi[1] = std::max(hi[1], k.y); hi[2] = std::max(hi[2], k.z);
        }
    }
    for (int a = 0; a < 3; ++a) { c->bounds[a] = lo[a]; c->bounds[3 + a] = hi[a]; }
    c->top = TopLevelField{}.updated(lo, hi, n > 0, [c](int32_t x, int32_t y, int32_t z) { return region_blocked(c, x, y, z); }, {});
    rc = finish_headers(c);
    if (rc != VGI_OK) return rc;
    std::vector<int32_t> dir = build_directory(c->keys);
    c->dir_slots = dir.size() / 4;
    VGI_CUDA(c, c->directory.reserve(c->dir_slots));
    VGI_CUDA(c, h2d(c->directory.ptr, dir.data(), dir.size() * 4, c->stream));
    VGI_CUDA(c, upload_grid(c, dir.data(), c->dir_slots));
    VGI_CUDA(c, refresh_grid_headers(c));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->host_dir = std::move(dir);
    c->geometry = true;
    return VGI_OK;
}

namespace {
// Checks host-packed arrays before they reach the device: every index the
// traversal follows must stay inside the arrays, and every material below 256.
int validate_packed(vgi_ctx* c, const int32_t* directory, uint64_t slots, const uint32_t* headers, uint32_t n_headers,
                    const uint32_t* cells, uint64_t n_cells) {
    for (uint64_t s = 0; s < slots; ++s) {
        int32_t w = directory[s * 4 + 3];
        if (w < -1 || (w >= 0 && (uint32_t)w >= n_headers)) return fail(c, VGI_ERR_INVALID, "directory entry names no header");
    }
    for (uint32_t h = 0; h < n_headers; ++h) {
        const uint32_t kind = headers[h * 4], payload = headers[h * 4 + 1];
        if (kind < 1 || kind > 3) return fail(c, VGI_ERR_INVALID, "region kind outside 1..3");
        if (kind == 2 && payload > 255) return fail(c, VGI_ERR_INVALID, "uniform region material above 255");
        if (kind != 3) continue;
        if ((uint64_t)payload + 64 > n_cells) return fail(c, VGI_ERR_INVALID, "brick table outside the cells");
        for (uint32_t b = 0; b < 64; ++b) {
            const uint32_t word = cells[payload + b];
            if ((word & 3u) == 1u && (word >> 2) > 255) return fail(c, VGI_ERR_INVALID, "uniform brick material above 255");
            if ((word & 3u) == 3u) return fail(c, VGI_ERR_INVALID, "brick word state 3");
            if ((word & 3u) != 2u) continue;
            const uint64_t ptr = word >> 2;
            if (ptr + 32 > n_cells) return fail(c, VGI_ERR_INVALID, "brick payload outside the cells");
            for (uint32_t k = 0; k < 32; ++k)
                for (uint32_t half = 0; half < 2; ++half) {
                    const uint32_t cell = (cells[ptr + k] >> (16 * half)) & 0xffffu;
                    if ((cell & 1u) && (cell >> 1) > 255) return fail(c, VGI_ERR_INVALID, "voxel material above 255");
                }
        }
    }
    return VGI_OK;
}
}  // namespace

int vgi_upload_packed(vgi_ctx* c, const int32_t* directory, uint64_t slots, const uint32_t* headers, uint32_t n_headers,
                      const uint32_t* cells, uint64_t n_cells, const int32_t* bounds6) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !directory || !headers || !bounds6 || slots == 0 || (slots & (slots - 1))) return VGI_ERR_INVALID;
    if (n_cells && !cells) return VGI_ERR_INVALID;
    int rc = validate_packed(c, directory, slots, headers, n_headers, cells, n_cells);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, cudaSetDevice(c->device));
    c->geometry = false;  // until the arrays below are all in place
    VGI_CUDA(c, c->directory.reserve(slots));
    VGI_CUDA(c, c->headers.reserve(std::max<uint32_t>(n_headers, 1)));
    VGI_CUDA(c, c->cells.reserve(std::max<uint64_t>(n_cells, 1)));
    VGI_CUDA(c, h2d(c->directory.ptr, directory, slots * 16, c->stream));
    if (n_headers) VGI_CUDA(c, h2d(c->headers.ptr, headers, (size_t)n_headers * 16, c->stream));
    if (n_cells) VGI_CUDA(c, h2d(c->cells.ptr, cells, n_cells * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dir_slots = slots;
    c->cells_used = n_cells;
    for (int k = 0; k < 6; ++k) c->bounds[k] = bounds6[k];
    VGI_CUDA(c, upload_grid(c, directory, slots));
    VGI_CUDA(c, refresh_grid_headers(c));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->keys.clear();
    c->where.clear();
    c->host_voxels.clear();
    c->live.clear();
    c->free_slots.clear();
    // The host copies of the packed arrays, which vgi_patch_packed patches
    // and checks before any delta reaches the device.
    c->host_dir.assign(directory, directory + slots * 4);
    c->host_headers.resize(n_headers);
    std::memcpy(c->host_headers.data(), headers, (size_t)n_headers * 16);
    c->host_cells.assign(cells, cells + n_cells);
    c->packed_geometry = true;
    c->geometry = true;
    return VGI_OK;
}

int vgi_patch_packed(vgi_ctx* c, uint64_t slots, uint32_t n_headers, uint64_t n_cells, const int32_t* bounds6, int directory_rebuilt,
                     const uint64_t* dir_ranges, uint32_t n_dir_ranges, const int32_t* dir_data, const uint64_t* header_ranges,
                     uint32_t n_header_ranges, const uint32_t* header_data, const uint64_t* cell_ranges, uint32_t n_cell_ranges,
                     const uint32_t* cell_data) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !bounds6 || slots == 0 || (slots & (slots - 1))) return VGI_ERR_INVALID;
    if ((n_dir_ranges && !dir_ranges) || (n_header_ranges && !header_ranges) || (n_cell_ranges && !cell_ranges))
        return VGI_ERR_INVALID;
    if (!c->geometry || !c->packed_geometry) return fail(c, VGI_ERR_STATE, "a packed delta needs geometry from vgi_upload_packed");
    if (!directory_rebuilt && slots != c->dir_slots)
        return fail(c, VGI_ERR_INVALID, "a directory of another capacity must be sent whole (directory_rebuilt)");
    if (directory_rebuilt && !dir_data) return VGI_ERR_INVALID;
    // The ranges' elements, back to back in each data array.
    auto check_ranges = [](const uint64_t* r, uint32_t n, uint64_t length, const void* data, uint64_t* total) {
        *total = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (r[2 * i] > length || r[2 * i + 1] > length - r[2 * i]) return false;
            *total += r[2 * i + 1];
        }
        return *total == 0 || data != nullptr;
    };
    uint64_t dir_total = 0, header_total = 0, cell_total = 0;
    if ((!directory_rebuilt && !check_ranges(dir_ranges, n_dir_ranges, slots, dir_data, &dir_total)) ||
        !check_ranges(header_ranges, n_header_ranges, n_headers, header_data, &header_total) ||
        !check_ranges(cell_ranges, n_cell_ranges, n_cells, cell_data, &cell_total))
        return fail(c, VGI_ERR_INVALID, "a delta range lies outside its array");
    // The patched arrays on the host; grown elements start at zero, as the
    // device's grown tails do below.
    std::vector<int32_t> dir;
    if (directory_rebuilt) {
        dir.assign(dir_data, dir_data + slots * 4);
    } else {
        dir = c->host_dir;
        for (uint32_t i = 0, at = 0; i < n_dir_ranges; at += (uint32_t)dir_ranges[2 * i + 1] * 4, ++i)
            std::copy(dir_data + at, dir_data + at + dir_ranges[2 * i + 1] * 4, dir.begin() + dir_ranges[2 * i] * 4);
    }
    std::vector<uint4> hdr = c->host_headers;
    hdr.resize(n_headers, make_uint4(0u, 0u, 0u, 0u));
    for (uint64_t i = 0, at = 0; i < n_header_ranges; at += header_ranges[2 * i + 1] * 4, ++i)
        std::memcpy(hdr.data() + header_ranges[2 * i], header_data + at, header_ranges[2 * i + 1] * 16);
    std::vector<uint32_t> cl = c->host_cells;
    cl.resize(n_cells, 0u);
    for (uint64_t i = 0, at = 0; i < n_cell_ranges; at += cell_ranges[2 * i + 1], ++i)
        std::copy(cell_data + at, cell_data + at + cell_ranges[2 * i + 1], cl.begin() + cell_ranges[2 * i]);
    int rc = validate_packed(c, dir.data(), slots, reinterpret_cast<const uint32_t*>(hdr.data()), n_headers, cl.data(), n_cells);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, cudaSetDevice(c->device));
    // One transaction on the stream. A longer array grows with its contents
    // copied on the device (the grown tail cleared); only the ranges cross
    // the bus. A failure from here leaves no geometry until the next upload.
    c->geometry = false;
    const size_t old_headers = c->host_headers.size(), old_cells = c->host_cells.size();
    if (directory_rebuilt) {
        VGI_CUDA(c, c->directory.reserve(slots));
        VGI_CUDA(c, h2d(c->directory.ptr, dir.data(), slots * 16, c->stream));
    } else {
        for (uint32_t i = 0, at = 0; i < n_dir_ranges; at += (uint32_t)dir_ranges[2 * i + 1] * 4, ++i)
            if (dir_ranges[2 * i + 1]) VGI_CUDA(c, h2d(c->directory.ptr + dir_ranges[2 * i], dir_data + at, dir_ranges[2 * i + 1] * 16, c->stream));
    }
    VGI_CUDA(c, c->headers.grow(std::max<uint32_t>(n_headers, 1), old_headers, c->stream));
    if (n_headers > old_headers)
        VGI_CUDA(c, cudaMemsetAsync(c->headers.ptr + old_headers, 0, (n_headers - old_headers) * 16, c->stream));
    for (uint64_t i = 0, at = 0; i < n_header_ranges; at += header_ranges[2 * i + 1] * 4, ++i)
        if (header_ranges[2 * i + 1])
            VGI_CUDA(c, h2d(c->headers.ptr + header_ranges[2 * i], header_data + at, header_ranges[2 * i + 1] * 16, c->stream));
    VGI_CUDA(c, c->cells.grow(std::max<uint64_t>(n_cells, 1), old_cells, c->stream));
    if (n_cells > old_cells) VGI_CUDA(c, cudaMemsetAsync(c->cells.ptr + old_cells, 0, (n_cells - old_cells) * 4, c->stream));
    for (uint64_t i = 0, at = 0; i < n_cell_ranges; at += cell_ranges[2 * i + 1], ++i)
        if (cell_ranges[2 * i + 1])
            VGI_CUDA(c, h2d(c->cells.ptr + cell_ranges[2 * i], cell_data + at, cell_ranges[2 * i + 1] * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dir_slots = slots;
    c->cells_used = n_cells;
    for (int k = 0; k < 6; ++k) c->bounds[k] = bounds6[k];
    c->host_dir = std::move(dir);
    c->host_headers = std::move(hdr);
    c->host_cells = std::move(cl);
    VGI_CUDA(c, upload_grid(c, c->host_dir.data(), slots));
    VGI_CUDA(c, refresh_grid_headers(c));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->geometry = true;
    return VGI_OK;
}

int vgi_edit_voxels(vgi_ctx* c, const int32_t* edits, uint32_t n) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || (n && !edits)) return VGI_ERR_INVALID;
    if (!c->geometry || c->keys.empty()) return fail(c, VGI_ERR_STATE, "edits need geometry uploaded as regions");
    VGI_CUDA(c, cudaSetDevice(c->device));
    for (uint32_t e = 0; e < n; ++e)
        if (edits[e * 4 + 3] < 0 || edits[e * 4 + 3] > 256) return fail(c, VGI_ERR_INVALID, "voxel value outside 0..256");
    std::vector<uint64_t> touched;  // region << 16 | voxel within it
    touched.reserve(n);
    std::vector<uint32_t> dirty;
    std::vector<uint8_t> was_blocked(c->keys.size(), 2);
    // Edits apply in order, so a voxel edited twice keeps its last value
    // (the host copy); the device scatter then writes each voxel once.
    for (uint32_t e = 0; e < n; ++e) {
        int32_t x = edits[e * 4], y = edits[e * 4 + 1], z = edits[e * 4 + 2];
        auto it = c->where.find(RegionKey{x >> 4, y >> 4, z >> 4});
        if (it == c->where.end()) continue;
        uint32_t r = it->second;
        uint32_t local = (uint32_t)((x & 15) + 16 * ((y & 15) + 16 * (z & 15)));
        c->host_voxels[(size_t)r * 4096 + local] = (uint16_t)edits[e * 4 + 3];
        touched.push_back(((uint64_t)r << 16) | local);
        if (was_blocked[r] == 2) {
            was_blocked[r] = c->host_headers[r].x != 1u ? 1 : 0;
            dirty.push_back(r);
        }
    }
    if (touched.empty()) return VGI_OK;
    std::sort(touched.begin(), touched.end());
    touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
    std::vector<uint2> packed;
    packed.reserve(touched.size());
    for (uint64_t k : touched) {
        const uint32_t r = (uint32_t)(k >> 16), local = (uint32_t)(k & 0xffffu);
        packed.push_back(make_uint2(r, (local << 16) | (uint32_t)c->host_voxels[(size_t)r * 4096 + local]));
    }
    VGI_CUDA(c, c->edit_buf.reserve(packed.size()));
    VGI_CUDA(c, h2d(c->edit_buf.ptr, packed.data(), packed.size() * sizeof(uint2), c->stream));
    launch_scatter_edits(c->edit_buf.ptr, (uint32_t)packed.size(), c->voxels.ptr, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    // Repack only the edited regions into fresh cell space; a full repack
    // reclaims space once the arena passes three quarters.
    bool full = c->cells_used + (unsigned long long)dirty.size() * (64 + 64 * 32) > c->cells.count * 3 / 4;
    if (full) c->cells_used = 0;
    int rc = pack_regions(c, full ? nullptr : &dirty);
    if (rc != VGI_OK) return rc;
    std::vector<RegionKey> changed;
    for (uint32_t r : dirty) {
        uint8_t now = c->host_headers[r].x != 1u ? 1 : 0;
        if (now != was_blocked[r]) changed.push_back(c->keys[r]);
    }
    if (!changed.empty()) {
        std::sort(changed.begin(), changed.end(), [](const RegionKey& a, const RegionKey& b) {
            if (a.z != b.z) return a.z < b.z;
            if (a.y != b.y) return a.y < b.y;
            return a.x < b.x;
        });
        c->top = c->top.updated(c->bounds, c->bounds + 3, true,
                                [c](int32_t x, int32_t y, int32_t z) { return region_blocked(c, x, y, z); }, changed);
    }
    rc = finish_headers(c);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, refresh_grid_headers(c));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

// Region residency changes, the GPU side of page streaming
// (VoxelGiInput::page_loaded / page_changed / page_unloaded, src/input.rs:54-70):
// TransportScene::with_page_contents (src/world.rs:982-1046) for the scene,
// with region-sized pages, and PackedScene::update (src/gpu_scene.rs:72-309)
// for the packed arrays. Removals come first, then loads (a region both
// removed and loaded ends up loaded). Only the loaded regions are classified
// and packed, into fresh cell space; once the arena would pass three
// quarters, every resident region is repacked from offset 0, which reclaims
// the space of replaced and removed regions and of bricks no region holds
// any longer (the reference's release_bricks, here one compaction instead of
// per-brick reference counts). Header slots of removed regions are freed and
// reused last freed first; the directory changes in place (linear-probing
// insert, backward-shift delete) and is rebuilt only when its capacity
// changes or an insert would probe 32 slots. The top-level field is updated
// incrementally over the touched regions unless every touched region keeps
// its residency and emptiness. World-cache slots are not touched.
static int apply_regions(vgi_ctx* c, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides,
                         const int32_t* removed, uint32_t n_removed) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || (n && (!coords || !voxels)) || (n_removed && !removed)) return VGI_ERR_INVALID;
    if (c->geometry && c->packed_geometry) return fail(c, VGI_ERR_STATE, "host-packed geometry has no regions to load into");
    VGI_CUDA(c, cudaSetDevice(c->device));
    {
        // Refused inputs leave the context as it was.
        std::unordered_map<RegionKey, uint32_t, RegionKeyHash> seen;
        for (uint32_t i = 0; i < n; ++i)
            if (!seen.emplace(RegionKey{coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]}, i).second)
                return fail(c, VGI_ERR_INVALID, "duplicate region coordinate");
        for (size_t i = 0; i < (size_t)n * 4096; ++i)
            if (voxels[i] > 256) return fail(c, VGI_ERR_INVALID, "voxel value above 256 (materials are 0..255, 256 is air)");
    }
    if (!c->geometry) {
        // No geometry yet: the loads start from an empty scene.
        c->keys.clear();
        c->where.clear();
        c->host_voxels.clear();
        c->strides.clear();
        c->host_headers.clear();
        c->live.clear();
        c->free_slots.clear();
        c->host_dir.clear();
        c->host_cells.clear();
        c->top = TopLevelField{};
        c->cells_used = 0;
        c->packed_geometry = false;
    }
    // From here a failure leaves no geometry (frames refused) until an
    // upload or a load succeeds.
    c->geometry = false;
    // Residency and emptiness of every touched region before the change:
    // -1 not loaded, 0 loaded air, 1 loaded with a solid voxel.
    auto status_of = [c](const RegionKey& k) -> int {
        auto it = c->where.find(k);
        if (it == c->where.end()) return -1;
        return c->host_headers[it->second].x != 1u ? 1 : 0;
    };
    std::unordered_map<RegionKey, int, RegionKeyHash> before;
    std::vector<RegionKey> touched;
    std::vector<uint32_t> freed;
    // A loaded region whose voxels and stride equal the resident region's is
    // the same region (build_page_regions keeps the previous Arc), so it is
    // not touched, even when the same call also unloads it
    // (with_page_contents' touched.retain, src/world.rs:1016-1020).
    std::unordered_set<RegionKey, RegionKeyHash> unchanged;
    for (uint32_t i = 0; i < n; ++i) {
        const RegionKey k{coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]};
        auto it = c->where.find(k);
        if (it == c->where.end()) continue;
        const uint8_t stride = strides ? strides[i] : 0;
        if (c->strides[it->second] == stride &&
            std::equal(voxels + (size_t)i * 4096, voxels + (size_t)(i + 1) * 4096, c->host_voxels.begin() + (size_t)it->second * 4096))
            unchanged.insert(k);
    }
    for (uint32_t i = 0; i < n_removed; ++i) {
        const RegionKey k{removed[i * 3], removed[i * 3 + 1], removed[i * 3 + 2]};
        auto it = c->where.find(k);
        if (it == c->where.end()) continue;
        if (!before.count(k)) before[k] = status_of(k);
        const uint32_t slot = it->second;
        c->where.erase(it);
        c->live[slot] = 0;
        c->free_slots.push_back(slot);
        c->host_headers[slot] = make_uint4(0u, 0u, 0u, 0u);
        if (!c->host_dir.empty()) directory_remove(c->host_dir, k);
        freed.push_back(slot);
        if (!unchanged.count(k)) touched.push_back(k);
    }
    const uint32_t old_slots = (uint32_t)c->keys.size();
    std::vector<uint32_t> slots(n);
    std::vector<RegionKey> inserted;
    for (uint32_t i = 0; i < n; ++i) {
        const RegionKey k{coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]};
        if (!before.count(k)) before[k] = status_of(k);
        auto it = c->where.find(k);
        uint32_t slot;
        if (it != c->where.end()) {
            slot = it->second;
        } else {
            if (!c->free_slots.empty()) {
                slot = c->free_slots.back();
                c->free_slots.pop_back();
            } else {
                slot = (uint32_t)c->keys.size();
                c->keys.push_back(k);
                c->live.push_back(0);
                c->strides.push_back(0);
                c->host_headers.push_back(make_uint4(0u, 0u, 0u, 0u));
                c->host_voxels.resize(c->host_voxels.size() + 4096);
            }
            c->keys[slot] = k;
            c->live[slot] = 1;
            c->where[k] = slot;
            inserted.push_back(k);
        }
        std::copy(voxels + (size_t)i * 4096, voxels + (size_t)(i + 1) * 4096, c->host_voxels.begin() + (size_t)slot * 4096);
        c->strides[slot] = strides ? strides[i] : 0;
        slots[i] = slot;
        if (!unchanged.count(k)) touched.push_back(k);
    }
    // A freed slot that a load took again is live.
    freed.erase(std::remove_if(freed.begin(), freed.end(), [c](uint32_t s) { return c->live[s] != 0; }), freed.end());
    const uint32_t total = (uint32_t)c->keys.size();
    uint32_t n_live = 0;
    for (uint8_t l : c->live) n_live += l;
    // Device storage: voxels and headers per slot, the cell arena sized for
    // every live region mixed (brick pointers are 30-bit word offsets).
    VGI_CUDA(c, c->voxels.grow((size_t)std::max<uint32_t>(total, 1) * 4096, (size_t)old_slots * 4096, c->stream));
    VGI_CUDA(c, c->headers.grow(std::max<uint32_t>(total, 1), old_slots, c->stream));
    const unsigned long long capacity = std::min<unsigned long long>((unsigned long long)n_live * (64 + 64 * 32) + 64, 1ull << 30);
    VGI_CUDA(c, c->cells.grow(capacity, c->cells_used, c->stream));
    if (n) {
        VGI_CUDA(c, c->staged_voxels.reserve((size_t)n * 4096));
        VGI_CUDA(c, h2d(c->staged_voxels.ptr, voxels, (size_t)n * 8192, c->stream));
    }
    std::vector<uint32_t> lists(slots);
    lists.insert(lists.end(), freed.begin(), freed.end());
    VGI_CUDA(c, c->slot_list.reserve(std::max<size_t>(lists.size(), 1)));
    if (!lists.empty()) VGI_CUDA(c, h2d(c->slot_list.ptr, lists.data(), lists.size() * 4, c->stream));
    launch_scatter_regions(c->staged_voxels.ptr, c->slot_list.ptr, n, c->voxels.ptr, c->stream);
    launch_clear_headers(c->headers.ptr, c->slot_list.ptr + n, (uint32_t)freed.size(), c->stream);
    VGI_CUDA(c, cudaGetLastError());
    // Pack the loaded regions, or every live one when the arena is short.
    const bool compact = c->cells_used + (unsigned long long)n * (64 + 64 * 32) > c->cells.count * 3 / 4;
    if (compact) c->cells_used = 0;
    std::vector<uint32_t> pack = slots;
    std::sort(pack.begin(), pack.end());
    int rc = pack_regions(c, compact ? nullptr : &pack);
    if (rc != VGI_OK) return rc;
    // Directory: in place, or rebuilt at a new capacity.
    size_t capacity_slots = 1;
    while (capacity_slots < (size_t)n_live * 2) capacity_slots <<= 1;
    bool rebuild = c->host_dir.empty() || capacity_slots * 4 > c->host_dir.size() || capacity_slots * 8 * 4 < c->host_dir.size();
    if (!rebuild)
        for (const RegionKey& k : inserted)
            if (!directory_insert(c->host_dir, k, c->where[k])) {
                rebuild = true;
                break;
            }
    if (rebuild) {
        std::vector<std::pair<RegionKey, uint32_t>> entries;
        entries.reserve(n_live);
        for (uint32_t r = 0; r < total; ++r)
            if (c->live[r]) entries.emplace_back(c->keys[r], r);
        c->host_dir = build_directory(entries);
    }
    c->dir_slots = c->host_dir.size() / 4;
    VGI_CUDA(c, c->directory.reserve(c->dir_slots));
    VGI_CUDA(c, h2d(c->directory.ptr, c->host_dir.data(), c->host_dir.size() * 4, c->stream));
    // Bounds and the top-level field.
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool first = true;
    for (uint32_t r = 0; r < total; ++r) {
        if (!c->live[r]) continue;
        const RegionKey& k = c->keys[r];
        const int32_t v[3] = {k.x, k.y, k.z};
        for (int a = 0; a < 3; ++a) {
            lo[a] = first ? v[a] : std::min(lo[a], v[a]);
            hi[a] = first ? v[a] : std::max(hi[a], v[a]);
        }
        first = false;
    }
    for (int a = 0; a < 3; ++a) {
        c->bounds[a] = lo[a];
        c->bounds[3 + a] = hi[a];
    }
    bool topology_unchanged = true;
    for (const auto& kv : before) {
        const int now = status_of(kv.first);
        if (kv.second < 0 || now < 0 || kv.second != now) topology_unchanged = false;
    }
    if (!topology_unchanged) {
        std::sort(touched.begin(), touched.end(), [](const RegionKey& a, const RegionKey& b) {
            if (a.z != b.z) return a.z < b.z;
            if (a.y != b.y) return a.y < b.y;
            return a.x < b.x;
        });
        touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
        c->top = c->top.updated(lo, hi, n_live > 0, [c](int32_t x, int32_t y, int32_t z) { return region_blocked(c, x, y, z); },
                                touched);
    }
    rc = finish_headers(c);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, upload_grid(c, c->host_dir.data(), c->dir_slots));
    VGI_CUDA(c, refresh_grid_headers(c));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->geometry = true;
    return VGI_OK;
}

int vgi_load_regions(vgi_ctx* c, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides) {
    return apply_regions(c, coords, n, voxels, strides, nullptr, 0);
}

int vgi_unload_regions(vgi_ctx* c, const int32_t* coords, uint32_t n) {
    return apply_regions(c, nullptr, 0, nullptr, nullptr, coords, n);
}

int vgi_update_regions(vgi_ctx* c, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides,
                       const int32_t* removed, uint32_t n_removed) {
    return apply_regions(c, coords, n, voxels, strides, removed, n_removed);
}

int vgi_geometry_info(vgi_ctx* c, uint64_t* sizes3, int32_t* bounds6) {
    if (!c || !sizes3 || !bounds6) return VGI_ERR_INVALID;
    if (!c->geometry) return fail(c, VGI_ERR_STATE, "no geometry uploaded");
    sizes3[0] = c->dir_slots;
    sizes3[1] = c->packed_geometry ? c->host_headers.size() : (c->keys.empty() ? c->headers.count : c->keys.size());
    sizes3[2] = c->cells_used;
    for (int k = 0; k < 6; ++k) bounds6[k] = c->bounds[k];
    return VGI_OK;
}

int vgi_read_geometry(vgi_ctx* c, int32_t* directory, uint32_t* headers, uint32_t* cells) {
    uint64_t sizes[3];
    int32_t b[6];
    int rc = vgi_geometry_info(c, sizes, b);
    if (rc != VGI_OK) return rc;
    if (directory) VGI_CUDA(c, cudaMemcpyAsync(directory, c->directory.ptr, sizes[0] * 16, cudaMemcpyDeviceToHost, c->stream));
    if (headers) VGI_CUDA(c, cudaMemcpyAsync(headers, c->headers.ptr, sizes[1] * 16, cudaMemcpyDeviceToHost, c->stream));
    if (cells && sizes[2]) VGI_CUDA(c, cudaMemcpyAsync(cells, c->cells.ptr, sizes[2] * 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_set_materials(vgi_ctx* c, const float* m) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !m) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    c->host_materials.assign(m, m + 256 * 16);
    VGI_CUDA(c, c->materials.reserve(256 * 4));
    VGI_CUDA(c, h2d(c->materials.ptr, m, 256 * 64, c->stream));
    // The luminance of each material's albedo and emission, for measuring
    // edits (ResidentCache::set_materials, src/gpu/resident.rs:816-838).
    std::vector<float2> light(256);
    for (int i = 0; i < 256; ++i) {
        const float* d = m + i * 16;
        const float* e = m + i * 16 + 8;
        light[i] = make_float2(0.2126f * d[0] + 0.7152f * d[1] + 0.0722f * d[2], 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2]);
    }
    VGI_CUDA(c, c->material_light.reserve(256));
    VGI_CUDA(c, h2d(c->material_light.ptr, light.data(), 256 * sizeof(float2), c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_set_lights(vgi_ctx* c, const float* lights, uint32_t n, uint32_t n_directional) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || (n && !lights) || n_directional > n || n > 4096) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    // An empty light list still uploads one default record (src/gpu.rs:757-759).
    std::vector<float> words(std::max<uint32_t>(n, 1) * 12, 0.0f);
    if (n) std::copy(lights, lights + n * 12, words.begin());
    VGI_CUDA(c, c->lights.reserve(words.size() / 4));
    VGI_CUDA(c, h2d(c->lights.ptr, words.data(), words.size() * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->n_lights = n;
    c->n_directional = n_directional;
    // transport.y of the view's parameters (src/gpu/view.rs:104-116).
    c->custom_lights = false;
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 9; k < 12; ++k) c->custom_lights |= lights[(size_t)i * 12 + k] != 0.0f;
    return VGI_OK;
}

int vgi_set_environment(vgi_ctx* c, const float* rgb3) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !rgb3) return VGI_ERR_INVALID;
    c->env[0] = rgb3[0];
    c->env[1] = rgb3[1];
    c->env[2] = rgb3[2];
    c->env[3] = 0.0f;
    return VGI_OK;
}

int vgi_set_emitters(vgi_ctx* c, const uint32_t* words, uint64_t n_words, uint32_t n_faces, float total_weight) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !words || n_words < 8 || (n_words & 3)) return VGI_ERR_INVALID;
    // Layout check (src/gpu.rs:686-711, src/emission/tree.rs:173-195): face
    // records, then light-tree nodes whose children follow their parent.
    const uint64_t records = n_faces == 0 ? 1 : n_faces;
    if (n_words < records * 8) return fail(c, VGI_ERR_INVALID, "emitter words shorter than the face records");
    if (n_faces > 0) {
        float tree_len_f;
        std::memcpy(&tree_len_f, &words[7], 4);
        if (!(tree_len_f >= 0.0f) || tree_len_f > 4.0e9f) return fail(c, VGI_ERR_INVALID, "bad light-tree length");
        const uint64_t nodes = (uint64_t)tree_len_f;
        if (n_words != records * 8 + nodes * 16) return fail(c, VGI_ERR_INVALID, "emitter word count does not match the tree");
        for (uint64_t f = 0; f < n_faces; ++f) {
            float m;
            std::memcpy(&m, &words[f * 8 + 6], 4);
            if (!(m >= 0.0f && m < 256.0f)) return fail(c, VGI_ERR_INVALID, "emitter material outside 0..255");
        }
        for (uint64_t i = 0; i < nodes; ++i) {
            const uint32_t* w = words + records * 8 + i * 16;
            const uint32_t left = w[12], right = w[13];
            if (left == 0xffffffffu) {
                if (right >= n_faces) return fail(c, VGI_ERR_INVALID, "light-tree leaf names no face");
            } else if (left <= i || right <= i || left >= nodes || right >= nodes) {
                return fail(c, VGI_ERR_INVALID, "light-tree children must follow their parent");
            }
        }
    }
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, c->emitters.reserve(n_words / 4));
    VGI_CUDA(c, h2d(c->emitters.ptr, words, n_words * 4, c->stream));
    c->host_emitter_records.assign(words, words + (size_t)n_faces * 8);
    const uint32_t nodes = (uint32_t)((n_words - records * 8) / 16);
    VGI_CUDA(c, c->node_aux.reserve(2 * (size_t)std::max<uint32_t>(nodes, 1)));
    launch_node_aux(c->emitters.ptr, (uint32_t)(records * 2), nodes, c->node_aux.ptr, c->stream);
    c->tree_generation += 1u;  // every kept tree row is stale now
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->emitter_count = (float)n_faces;
    c->emitter_total = total_weight;
    return VGI_OK;
}

int vgi_build_emitters(vgi_ctx* c) {
    if (!c) return VGI_ERR_INVALID;
    if (c->keys.empty() && c->geometry) return fail(c, VGI_ERR_STATE, "emitters need geometry uploaded as regions");
    EmitterWords e = build_emitters(c->keys, c->host_voxels.data(), c->host_materials.data(), c->live.empty() ? nullptr : &c->live);
    return vgi_set_emitters(c, e.words.data(), e.words.size(), e.faces, e.total_weight);
}

int vgi_set_transport(vgi_ctx* c, const vgi_transport* t) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || !t) return VGI_ERR_INVALID;
    vgi_transport n = *t;
    n.reach = norm_reach(n.reach);
    n.bounces = norm_bounces(n.bounces);
    if (n.path_steps == 0) n.path_steps = 2048;
    if (n.lanes && (n.lanes & (n.lanes - 1))) return fail(c, VGI_ERR_INVALID, "lanes must be a power of two");
    if (n.lanes > 32) return fail(c, VGI_ERR_INVALID, "lanes above 32");
    c->transport = n;
    return VGI_OK;
}

int vgi_set_faces(vgi_ctx* c, const vgi_face* faces, uint32_t n) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c || (n && !faces)) return VGI_ERR_INVALID;
    if (n >= (1u << 29)) return fail(c, VGI_ERR_CAPACITY, "slot index exceeds 29 bits");
    VGI_CUDA(c, cudaSetDevice(c->device));
    std::vector<std::array<int32_t, 4>> keys(n);
    std::vector<uint4> tasks((size_t)n * 2), meta((size_t)n * 3, make_uint4(0, 0, 0, 0));
    for (uint32_t s = 0; s < n; ++s) {
        if (faces[s].face > 5 || faces[s].material > 255) return fail(c, VGI_ERR_INVALID, "face or material out of range");
        keys[s] = {faces[s].voxel[0], faces[s].voxel[1], faces[s].voxel[2], (int32_t)faces[s].face};
        tasks[s * 2] = make_uint4((uint32_t)faces[s].voxel[0], (uint32_t)faces[s].voxel[1], (uint32_t)faces[s].voxel[2], faces[s].face);
        tasks[s * 2 + 1] = make_uint4(0, 0, 0, 0);
        // Slot identity: voxel, face | LIVE (8) | material << 16.
        meta[s * 3] = make_uint4((uint32_t)faces[s].voxel[0], (uint32_t)faces[s].voxel[1], (uint32_t)faces[s].voxel[2],
                                 faces[s].face | 8u | (faces[s].material << 16));
    }
    std::vector<uint32_t> index = build_face_index(keys);
    size_t m = std::max<uint32_t>(n, 1);
    // Until this call succeeds the context has no faces: a failed allocation
    // or copy below leaves frames refused (VGI_ERR_STATE), never reading
    // released buffers with the old slot count.
    c->n_slots = 0;
    VGI_CUDA(c, c->tasks.reserve(m * 2));
    VGI_CUDA(c, c->results.reserve(m * 6));
    VGI_CUDA(c, c->state.reserve(m * 9));
    VGI_CUDA(c, c->slot_meta.reserve(m * 3));
    VGI_CUDA(c, c->checkpoint.reserve(m * 3));
    VGI_CUDA(c, c->cache.reserve(m));
    VGI_CUDA(c, c->tree_rows.reserve(m * kTreeRowWords));
    VGI_CUDA(c, c->face_index.reserve(index.size() / 4));
    VGI_CUDA(c, h2d(c->tasks.ptr, tasks.data(), (size_t)n * 32, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->results.ptr, 0, m * 96, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->state.ptr, 0, m * 144, c->stream));
    launch_seed_incarnations(c->state.ptr, n, c->stream);
    VGI_CUDA(c, h2d(c->slot_meta.ptr, meta.data(), (size_t)n * 48, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->checkpoint.ptr, 0, m * 48, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->cache.ptr, 0, m * 16, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->tree_rows.ptr, 0xff, m * kTreeRowWords * 16, c->stream));  // no key matches
    VGI_CUDA(c, h2d(c->face_index.ptr, index.data(), index.size() * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->n_slots = n;
    c->batch_id = 1;  // a new face set starts a new batch sequence
    c->keys_reset = true;
    return VGI_OK;
}

namespace {
// Sets a captured kernel node's argument (the kernel takes one AccumArgs).
cudaError_t set_accum_node(vgi_ctx* c, cudaGraphNode_t node, const AccumArgs& acc) {
    cudaKernelNodeParams p{};
    cudaError_t e = cudaGraphKernelNodeGetParams(node, &p);
    if (e != cudaSuccess) return e;
    AccumArgs copy = acc;
    void* args[] = {&copy};
    p.kernelParams = args;
    p.extra = nullptr;
    return cudaGraphExecKernelNodeSetParams(c->graph_exec, node, &p);
}

// Captures prepare, trace and accumulate of one frame into c->graph_exec.
int capture_frame(vgi_ctx* c, uint32_t samples, const AccumArgs& acc) {
    VGI_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    launch_prepare(acc, c->stream);
    TraceArgs tr = trace_args(c, c->tasks.ptr, c->results.ptr, c->n_slots, samples, true);
    int rc = run_trace(c, tr, false);
    launch_accumulate(acc, c->stream);
    if (rc == VGI_OK) rc = mlp_frame_training(c);
    c->graph_mlp = mlp_terminates(c);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc != VGI_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc != VGI_OK ? rc : fail(c, VGI_ERR_CUDA, std::string("frame capture: ") + cudaGetErrorString(e));
    }
    c->graph = g;
    VGI_CUDA(c, cudaGraphInstantiate(&c->graph_exec, g, 0));
    size_t n = 0;
    VGI_CUDA(c, cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    VGI_CUDA(c, cudaGraphGetNodes(g, nodes.data(), &n));
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        VGI_CUDA(c, cudaGraphNodeGetType(node, &type));
        if (type != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams p{};
        VGI_CUDA(c, cudaGraphKernelNodeGetParams(node, &p));
        if (p.func == prepare_kernel_address()) c->graph_prepare = node;
        if (p.func == accumulate_kernel_address()) c->graph_accumulate = node;
    }
    if (!c->graph_prepare || !c->graph_accumulate) {
        drop_graph(c);
        return fail(c, VGI_ERR_CUDA, "frame capture lost the accumulation kernels");
    }
    c->graph_samples = samples;
    c->graph_dirty = false;
    return VGI_OK;
}
}  // namespace

int vgi_set_graph(vgi_ctx* c, int enable) {
    if (!c) return VGI_ERR_INVALID;
    drop_graph(c);
    c->use_graph = enable != 0;
    return VGI_OK;
}

int vgi_frame(vgi_ctx* c, uint32_t samples, uint32_t clock_ms) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (samples == 0) return fail(c, VGI_ERR_INVALID, "samples must be positive");
    AccumArgs acc = accum_args(c, samples, clock_ms);
    // The warm-up frames of the MLP cache trace plainly; the first frame
    // that ends paths with the network needs a new capture.
    if (c->graph_exec && c->graph_mlp != mlp_terminates(c)) drop_graph(c);
    if (c->use_graph && !c->timing && c->layout == VGI_LAYOUT_WAVEFRONT && c->n_slots > 0) {
        if (c->graph_exec && c->graph_samples == samples && !c->graph_dirty) {
            VGI_CUDA(c, set_accum_node(c, c->graph_prepare, acc));
            VGI_CUDA(c, set_accum_node(c, c->graph_accumulate, acc));
            VGI_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
            c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
            if (c->batch_id == 0) c->batch_id = 1;
            if (c->mlp_cache) c->mlp_frames += 1;
            return VGI_OK;
        }
        if (!c->graph_dirty && c->graph_samples == samples) {
            // Buffers are sized (the last frame ran directly): capture this one.
            rc = capture_frame(c, samples, acc);
            if (rc != VGI_OK) return rc;
            VGI_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
            c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
            if (c->batch_id == 0) c->batch_id = 1;
            if (c->mlp_cache) c->mlp_frames += 1;
            return VGI_OK;
        }
        drop_graph(c);
        c->graph_dirty = false;
        c->graph_samples = samples;
    }
    if (c->timing) VGI_CUDA(c, cudaEventRecord(c->marks[0], c->stream));
    launch_prepare(acc, c->stream);
    if (c->timing) VGI_CUDA(c, cudaEventRecord(c->marks[1], c->stream));
    TraceArgs tr = trace_args(c, c->tasks.ptr, c->results.ptr, c->n_slots, samples, true);
    rc = run_trace(c, tr, false);
    if (rc != VGI_OK) return rc;
    if (c->timing) VGI_CUDA(c, cudaEventRecord(c->marks[2], c->stream));
    launch_accumulate(acc, c->stream);
    if (c->timing) VGI_CUDA(c, cudaEventRecord(c->marks[3], c->stream));
    const bool timed_mlp = c->timing && mlp_terminates(c);
    if (timed_mlp) VGI_CUDA(c, cudaEventRecord(c->mlp_marks[2], c->stream));
    rc = mlp_frame_training(c);
    if (rc != VGI_OK) return rc;
    if (timed_mlp) VGI_CUDA(c, cudaEventRecord(c->mlp_marks[3], c->stream));
    if (c->timing) c->mlp_timed = timed_mlp;
    VGI_CUDA(c, cudaGetLastError());
    c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
    if (c->batch_id == 0) c->batch_id = 1;
    if (c->mlp_cache) c->mlp_frames += 1;
    return VGI_OK;
}

int vgi_frame_shard(vgi_ctx* c, uint32_t samples, uint32_t clock_ms, uint32_t first, uint32_t n) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (samples == 0 || n == 0) return fail(c, VGI_ERR_INVALID, "samples and the shard's slots must be positive");
    if (first > c->n_slots || n > c->n_slots - first) return fail(c, VGI_ERR_INVALID, "shard outside the slots");
    if (c->mlp_cache) return fail(c, VGI_ERR_STATE, "the MLP cache mode traces whole frames");
    VGI_CUDA(c, cudaSetDevice(c->device));
    // The shard's slots are a contiguous range: every per-slot array starts
    // at `first`, and the traced count is n. The gather still reads every
    // slot's record (the face index covers all faces).
    AccumArgs acc = accum_args(c, samples, clock_ms);
    acc.state += (size_t)first * 9;
    acc.slot_meta += (size_t)first * 3;
    acc.checkpoint += (size_t)first * 3;
    acc.outputs += (size_t)first * 6;
    acc.tasks += (size_t)first * 2;
    acc.cache += first;
    acc.n = n;
    acc.controls[0] = acc.controls[5] = acc.controls[14] = acc.controls[24] = n;
    launch_prepare(acc, c->stream);
    TraceArgs tr = trace_args(c, c->tasks.ptr + (size_t)first * 2, c->results.ptr + (size_t)first * 6, n, samples, true);
    rc = run_trace(c, tr, false, false);
    if (rc != VGI_OK) return rc;
    launch_accumulate(acc, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
    if (c->batch_id == 0) c->batch_id = 1;
    return VGI_OK;
}

int vgi_frame_scheduled(vgi_ctx* c, uint32_t samples, uint32_t clock_ms, const vgi_schedule* sched) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (!sched || samples == 0) return fail(c, VGI_ERR_INVALID, "a schedule and positive samples are required");
    if (sched->budget == 0 || sched->budget > c->n_slots) return fail(c, VGI_ERR_INVALID, "pick budget outside 1..slots");
    if (sched->classify_first > sched->classify_end || sched->classify_end > c->n_slots)
        return fail(c, VGI_ERR_INVALID, "classification range outside the slots");
    if (c->mlp_cache) return fail(c, VGI_ERR_STATE, "the MLP cache mode traces whole frames");
    VGI_CUDA(c, cudaSetDevice(c->device));
    const uint32_t n = c->n_slots, budget = sched->budget;
    VGI_CUDA(c, c->sel_keys.reserve(n));
    // Keys of a new face set start as "not a candidate" until their range is classified.
    if (c->keys_reset) VGI_CUDA(c, cudaMemsetAsync(c->sel_keys.ptr, 0xff, (size_t)n * 4, c->stream));
    c->keys_reset = false;
    VGI_CUDA(c, c->selection.reserve(kSelectionWords));
    VGI_CUDA(c, c->pick_slots.reserve(budget));
    VGI_CUDA(c, c->pick_tasks.reserve((size_t)budget * 2));
    VGI_CUDA(c, c->pick_records.reserve(budget));
    VGI_CUDA(c, c->pick_results.reserve((size_t)budget * 6));
    c->pick_budget = budget;
    AccumArgs acc = accum_args(c, samples, clock_ms);
    acc.tasks = c->pick_tasks.ptr;
    acc.outputs = c->pick_results.ptr;
    acc.slots = c->pick_slots.ptr;
    acc.picks = c->pick_records.ptr;
    acc.n = budget;
    acc.controls[0] = budget;
    acc.controls[19] = sched->audit_ms;
    acc.controls[20] = (uint32_t)sched->focus[0];
    acc.controls[21] = (uint32_t)sched->focus[1];
    acc.controls[22] = (uint32_t)sched->focus[2];
    acc.controls[23] = budget;
    acc.controls[24] = 0;  // no CPU-traced faces: every task is a pick
    acc.controls[26] = sched->classify_first;
    acc.controls[27] = sched->classify_end;
    acc.controls[32] = 0;  // no statistics-mirror records
    VGI_CUDA(c, cudaMemsetAsync(c->selection.ptr, 0, kSelectionWords * 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->pick_slots.ptr, 0xff, (size_t)budget * 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->pick_tasks.ptr, 0xff, (size_t)budget * 32, c->stream));  // face 0xffffffff: no task
    VGI_CUDA(c, cudaMemsetAsync(c->pick_records.ptr, 0xff, (size_t)budget * 16, c->stream));
    launch_select(acc, n, c->sel_keys.ptr, c->selection.ptr, c->pick_slots.ptr, c->stream);
    launch_mark_changed(acc, c->stream);
    const TraceArgs tr = trace_args(c, c->pick_tasks.ptr, c->pick_results.ptr, budget, samples, true);
    rc = run_trace(c, tr, false, false);
    if (rc != VGI_OK) return rc;
    launch_accumulate(acc, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
    if (c->batch_id == 0) c->batch_id = 1;
    return VGI_OK;
}

int vgi_read_selection(vgi_ctx* c, uint32_t* keys, uint32_t* selection, uint32_t* picks4, uint32_t* tasks8, uint32_t* results24) {
    if (!c) return VGI_ERR_INVALID;
    if (!c->selection.ptr) return fail(c, VGI_ERR_STATE, "no scheduled frame has run");
    VGI_CUDA(c, cudaSetDevice(c->device));
    const uint32_t b = c->pick_budget;
    if (keys) VGI_CUDA(c, cudaMemcpyAsync(keys, c->sel_keys.ptr, (size_t)c->n_slots * 4, cudaMemcpyDeviceToHost, c->stream));
    if (selection) VGI_CUDA(c, cudaMemcpyAsync(selection, c->selection.ptr, kSelectionWords * 4, cudaMemcpyDeviceToHost, c->stream));
    if (picks4) VGI_CUDA(c, cudaMemcpyAsync(picks4, c->pick_records.ptr, (size_t)b * 16, cudaMemcpyDeviceToHost, c->stream));
    if (tasks8) VGI_CUDA(c, cudaMemcpyAsync(tasks8, c->pick_tasks.ptr, (size_t)b * 32, cudaMemcpyDeviceToHost, c->stream));
    if (results24) VGI_CUDA(c, cudaMemcpyAsync(results24, c->pick_results.ptr, (size_t)b * 96, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_discover_faces(vgi_ctx* c, const vgi_camera* cam, uint32_t* pixels8, vgi_face* faces, uint32_t capacity, uint32_t* n_faces) {
    if (!c || !cam || (capacity && !faces)) return VGI_ERR_INVALID;
    if (!c->geometry) return fail(c, VGI_ERR_STATE, "no geometry uploaded");
    const uint64_t n = (uint64_t)cam->width * cam->height;
    if (n == 0 || n > (1ull << 26)) return fail(c, VGI_ERR_INVALID, "camera size outside 1..2^26 pixels");
    VGI_CUDA(c, cudaSetDevice(c->device));
    uint32_t mask = 1;
    while (mask < 2 * n) mask <<= 1;
    DevBuf<float>& dcam = c->disc_cam;
    DevBuf<uint4>& pixels = c->disc_pixels;
    DevBuf<unsigned long long>& set = c->disc_set;
    DevBuf<int4>& list = c->disc_list;
    DevBuf<uint32_t>& counters = c->disc_counters;
    VGI_CUDA(c, dcam.reserve(10));
    VGI_CUDA(c, pixels.reserve(n * 2));
    VGI_CUDA(c, set.reserve(mask));
    VGI_CUDA(c, list.reserve(std::max<uint32_t>(capacity, 1)));
    VGI_CUDA(c, counters.reserve(2));
    float host_cam[10] = {cam->eye[0], cam->eye[1], cam->eye[2], cam->forward[0], cam->forward[1], cam->forward[2],
                          cam->up[0], cam->up[1], cam->up[2], cam->tan_half_fov};
    VGI_CUDA(c, h2d(dcam.ptr, host_cam, sizeof(host_cam), c->stream));
    VGI_CUDA(c, cudaMemsetAsync(set.ptr, 0xff, (size_t)mask * 8, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(counters.ptr, 0, 8, c->stream));
    const TraceArgs tr = trace_args(c, nullptr, nullptr, 0, 1, false);
    launch_discover(tr, dcam.ptr, cam->width, cam->height, pixels.ptr, set.ptr, mask - 1, list.ptr, counters.ptr, capacity, counters.ptr + 1,
                    c->stream);
    VGI_CUDA(c, cudaGetLastError());
    uint32_t counts[2] = {0, 0};
    VGI_CUDA(c, cudaMemcpyAsync(counts, counters.ptr, 8, cudaMemcpyDeviceToHost, c->stream));
    if (pixels8) VGI_CUDA(c, cudaMemcpyAsync(pixels8, pixels.ptr, n * 32, cudaMemcpyDeviceToHost, c->stream));
    std::vector<int4> found(std::min(counts[0], capacity));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (n_faces) *n_faces = counts[0];
    if (counts[0] > capacity) return fail(c, VGI_ERR_CAPACITY, "more faces than the list holds: n_faces says how many");
    if (counts[1]) return fail(c, VGI_ERR_CAPACITY, "the face set overflowed");
    if (!found.empty()) VGI_CUDA(c, cudaMemcpy(found.data(), list.ptr, found.size() * 16, cudaMemcpyDeviceToHost));
    // The list order follows the GPU's insertions; sort it by voxel z, y, x
    // and face, the order of the scene's exposed faces.
    std::sort(found.begin(), found.end(), [](const int4& a, const int4& b) {
        if (a.z != b.z) return a.z < b.z;
        if (a.y != b.y) return a.y < b.y;
        if (a.x != b.x) return a.x < b.x;
        return (a.w & 7) < (b.w & 7);
    });
    for (size_t k = 0; k < found.size(); ++k)
        faces[k] = vgi_face{{found[k].x, found[k].y, found[k].z}, (uint32_t)found[k].w & 7u, (uint32_t)found[k].w >> 8};
    return VGI_OK;
}

int vgi_read_cache(vgi_ctx* c, uint32_t first, uint32_t n, float* dst4, int on_device) {
    if (!c || (n && !dst4) || first > c->n_slots || n > c->n_slots - first) return VGI_ERR_INVALID;
    if (n == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, cudaMemcpyAsync(dst4, c->cache.ptr + first, (size_t)n * 16, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                c->stream));
    if (!on_device) VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_write_cache(vgi_ctx* c, uint32_t first, uint32_t n, const float* src4, int on_device) {
    if (!c || (n && !src4) || first > c->n_slots || n > c->n_slots - first) return VGI_ERR_INVALID;
    if (n == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, cudaMemcpyAsync(c->cache.ptr + first, src4, (size_t)n * 16, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                c->stream));
    if (!on_device) VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_set_layout(vgi_ctx* c, uint32_t layout, uint32_t refill_min) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c) return VGI_ERR_INVALID;
    if (layout != VGI_LAYOUT_WAVEFRONT && layout != VGI_LAYOUT_SINGLE_KERNEL) return fail(c, VGI_ERR_INVALID, "unknown layout");
    if (refill_min < 1 || refill_min > 32) return fail(c, VGI_ERR_INVALID, "refill_min outside 1..32");
    c->layout = layout;
    c->refill_min = refill_min;
    return VGI_OK;
}

int vgi_set_timing(vgi_ctx* c, int enable) {
    if (c) drop_graph(c);  // what a frame launches may change
    if (!c) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    if (enable && !c->marks[0]) {
        for (auto& e : c->marks) VGI_CUDA(c, cudaEventCreate(&e));
        for (auto& e : c->traverse_marks) VGI_CUDA(c, cudaEventCreate(&e));
        for (auto& e : c->mlp_marks) VGI_CUDA(c, cudaEventCreate(&e));
    }
    c->timing = enable != 0;
    return VGI_OK;
}

int vgi_frame_times(vgi_ctx* c, float* ms4) {
    if (!c || !ms4) return VGI_ERR_INVALID;
    if (!c->timing) return fail(c, VGI_ERR_STATE, "timing not enabled");
    VGI_CUDA(c, cudaEventSynchronize(c->marks[3]));
    for (int k = 0; k < 3; ++k) VGI_CUDA(c, cudaEventElapsedTime(&ms4[k], c->marks[k], c->marks[k + 1]));
    ms4[3] = 0.0f;
    for (uint32_t k = 0; k < c->traverse_launches; ++k) {
        float ms = 0.0f;
        VGI_CUDA(c, cudaEventElapsedTime(&ms, c->traverse_marks[2 * k], c->traverse_marks[2 * k + 1]));
        ms4[3] += ms;
    }
    return VGI_OK;
}

int vgi_trace_batch(vgi_ctx* c, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t clock_ms, uint32_t* results) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (!tasks || !results || n != c->n_slots) return fail(c, VGI_ERR_INVALID, "one task per slot expected");
    VGI_CUDA(c, h2d(c->tasks.ptr, tasks, (size_t)n * 32, c->stream));
    rc = vgi_frame(c, samples, clock_ms);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, cudaMemcpyAsync(results, c->results.ptr, (size_t)n * 96, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_submit_batch(vgi_ctx* c, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t clock_ms, uint32_t* results,
                     uint64_t* ticket) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (!tasks || !results || n != c->n_slots) return fail(c, VGI_ERR_INVALID, "one task per slot expected");
    VGI_CUDA(c, cudaSetDevice(c->device));
    if (!c->copy_in) {
        VGI_CUDA(c, cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
        VGI_CUDA(c, cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k)
            for (cudaEvent_t* e : {&c->tasks_ready[k], &c->tasks_free[k], &c->results_ready[k], &c->results_done[k]})
                VGI_CUDA(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    const uint64_t k = c->submitted;
    const int b = (int)(k & 1u);
    const bool reused = k >= 2;  // this staging pair served batch k - 2
    VGI_CUDA(c, c->stage_tasks[b].reserve((size_t)n * 2));
    VGI_CUDA(c, c->stage_results[b].reserve((size_t)n * 6));
    // Tasks in: after the frame of batch k - 2 has taken its staged tasks.
    if (reused) VGI_CUDA(c, cudaStreamWaitEvent(c->copy_in, c->tasks_free[b], 0));
    VGI_CUDA(c, h2d(c->stage_tasks[b].ptr, tasks, (size_t)n * 32, c->copy_in));
    VGI_CUDA(c, cudaEventRecord(c->tasks_ready[b], c->copy_in));
    // The frame, between the staged tasks and the staged results.
    VGI_CUDA(c, cudaStreamWaitEvent(c->stream, c->tasks_ready[b], 0));
    VGI_CUDA(c, cudaMemcpyAsync(c->tasks.ptr, c->stage_tasks[b].ptr, (size_t)n * 32, cudaMemcpyDeviceToDevice, c->stream));
    VGI_CUDA(c, cudaEventRecord(c->tasks_free[b], c->stream));
    rc = vgi_frame(c, samples, clock_ms);
    if (rc != VGI_OK) return rc;
    if (reused) VGI_CUDA(c, cudaStreamWaitEvent(c->stream, c->results_done[b], 0));
    VGI_CUDA(c, cudaMemcpyAsync(c->stage_results[b].ptr, c->results.ptr, (size_t)n * 96, cudaMemcpyDeviceToDevice, c->stream));
    VGI_CUDA(c, cudaEventRecord(c->results_ready[b], c->stream));
    // Results out, while the next frames run.
    VGI_CUDA(c, cudaStreamWaitEvent(c->copy_out, c->results_ready[b], 0));
    VGI_CUDA(c, cudaMemcpyAsync(results, c->stage_results[b].ptr, (size_t)n * 96, cudaMemcpyDeviceToHost, c->copy_out));
    VGI_CUDA(c, cudaEventRecord(c->results_done[b], c->copy_out));
    c->submitted = k + 1;
    if (ticket) *ticket = k;
    return VGI_OK;
}

int vgi_complete_batch(vgi_ctx* c, uint64_t ticket) {
    if (!c) return VGI_ERR_INVALID;
    if (ticket >= c->submitted) return fail(c, VGI_ERR_INVALID, "no such batch submitted");
    if (c->submitted - ticket > 2) return VGI_OK;  // its staging pair has been reused since: it completed before that
    VGI_CUDA(c, cudaEventSynchronize(c->results_done[ticket & 1u]));
    return VGI_OK;
}

int vgi_census(vgi_ctx* c, uint32_t samples, vgi_counters* counters) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, c->scratch_tasks.reserve((size_t)c->n_slots * 2));
    VGI_CUDA(c, c->scratch_results.reserve((size_t)c->n_slots * 6));
    // The next frame's tasks: the slot tasks with each slot's sequence.
    VGI_CUDA(c, cudaMemcpyAsync(c->scratch_tasks.ptr, c->tasks.ptr, (size_t)c->n_slots * 32, cudaMemcpyDeviceToDevice, c->stream));
    AccumArgs acc = accum_args(c, samples, 0);
    acc.tasks = c->scratch_tasks.ptr;
    acc.slot_meta = nullptr;  // begin_trace only
    launch_prepare(acc, c->stream);
    VGI_CUDA(c, cudaMemsetAsync(c->counters.ptr, 0, kCounterWords * 8, c->stream));
    TraceArgs tr = trace_args(c, c->scratch_tasks.ptr, c->scratch_results.ptr, c->n_slots, samples, true);
    rc = run_trace(c, tr, true);
    if (rc != VGI_OK) return rc;
    return read_counters(c, counters);
}

int vgi_autotune(vgi_ctx* c, uint32_t samples, uint32_t* layout_out, uint32_t* refill_out, float* ms_out) {
    int rc = check_ready(c, true);
    if (rc != VGI_OK) return rc;
    if (samples == 0) return fail(c, VGI_ERR_INVALID, "samples must be positive");
    VGI_CUDA(c, c->scratch_tasks.reserve((size_t)c->n_slots * 2));
    VGI_CUDA(c, c->scratch_results.reserve((size_t)c->n_slots * 6));
    VGI_CUDA(c, cudaMemcpyAsync(c->scratch_tasks.ptr, c->tasks.ptr, (size_t)c->n_slots * 32, cudaMemcpyDeviceToDevice, c->stream));
    AccumArgs acc = accum_args(c, samples, 0);
    acc.tasks = c->scratch_tasks.ptr;
    acc.slot_meta = nullptr;  // begin_trace only: no slot changes
    launch_prepare(acc, c->stream);
    const TraceArgs tr = trace_args(c, c->scratch_tasks.ptr, c->scratch_results.ptr, c->n_slots, samples, true);
    const uint32_t layout0 = c->layout, refill0 = c->refill_min;
    const bool timing0 = c->timing;
    c->timing = false;
    struct Candidate { uint32_t layout, refill; };
    const Candidate candidates[] = {{VGI_LAYOUT_WAVEFRONT, 4}, {VGI_LAYOUT_WAVEFRONT, 6}, {VGI_LAYOUT_WAVEFRONT, 8},
                                    {VGI_LAYOUT_WAVEFRONT, 12}, {VGI_LAYOUT_WAVEFRONT, 16}, {VGI_LAYOUT_SINGLE_KERNEL, 8}};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    VGI_CUDA(c, cudaEventCreate(&e0));
    VGI_CUDA(c, cudaEventCreate(&e1));
    float best = 1e30f;
    Candidate chosen{layout0, refill0};
    for (const Candidate& k : candidates) {
        c->layout = k.layout;
        c->refill_min = k.refill;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == VGI_OK; ++rep) {  // the first run warms caches and sizes buffers
            cudaEventRecord(e0, c->stream);
            rc = run_trace(c, tr, false);
            cudaEventRecord(e1, c->stream);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
        }
        if (rc != VGI_OK) break;
        if (ms < best) {
            best = ms;
            chosen = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->timing = timing0;
    c->layout = rc == VGI_OK ? chosen.layout : layout0;
    c->refill_min = rc == VGI_OK ? chosen.refill : refill0;
    drop_graph(c);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, cudaGetLastError());
    if (layout_out) *layout_out = chosen.layout;
    if (refill_out) *refill_out = chosen.refill;
    if (ms_out) *ms_out = best;
    return VGI_OK;
}

int vgi_trace_tasks(vgi_ctx* c, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t* results, vgi_counters* counters) {
    int rc = check_ready(c, false);
    if (rc != VGI_OK) return rc;
    if (!tasks || !results) return VGI_ERR_INVALID;
    if (samples == 0) return fail(c, VGI_ERR_INVALID, "samples must be positive");
    if (n == 0) return VGI_OK;
    VGI_CUDA(c, c->scratch_tasks.reserve((size_t)n * 2));
    VGI_CUDA(c, c->scratch_results.reserve((size_t)n * 6));
    VGI_CUDA(c, h2d(c->scratch_tasks.ptr, tasks, (size_t)n * 32, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->counters.ptr, 0, kCounterWords * 8, c->stream));
    bool with_cache = c->n_slots > 0;
    TraceArgs tr = trace_args(c, c->scratch_tasks.ptr, c->scratch_results.ptr, n, samples, with_cache);
    rc = run_trace(c, tr, counters != nullptr);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, cudaMemcpyAsync(results, c->scratch_results.ptr, (size_t)n * 96, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (counters) return read_counters(c, counters);
    return VGI_OK;
}

int vgi_apply_events(vgi_ctx* c, const uint32_t* words, uint32_t n_events, uint64_t n_words) {
    if (!c || (n_words && !words) || (n_words & 3) || (uint64_t)n_events * 12 > n_words) return VGI_ERR_INVALID;
    if (c->n_slots == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, c->events.reserve(std::max<uint64_t>(n_words / 4, 1)));
    if (n_words) VGI_CUDA(c, h2d(c->events.ptr, words, n_words * 4, c->stream));
    c->n_events = n_events;
    AccumArgs acc = accum_args(c, 0, 0);
    launch_apply_events(acc, c->events.ptr, c->n_slots, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->n_events = 0;
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

static int apply_events_impl(vgi_ctx* c, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                             uint32_t n_entries, const int32_t* footprints, uint32_t n_footprints);

int vgi_apply_events_measured(vgi_ctx* c, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                              uint32_t n_entries) {
    return apply_events_impl(c, words, n_events, n_words, measures, n_entries, nullptr, 0);
}

int vgi_apply_events_footprints(vgi_ctx* c, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                                uint32_t n_entries, const int32_t* footprints, uint32_t n_footprints) {
    return apply_events_impl(c, words, n_events, n_words, measures, n_entries, footprints, n_footprints);
}

static int apply_events_impl(vgi_ctx* c, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                             uint32_t n_entries, const int32_t* footprints, uint32_t n_footprints) {
    if (!c || (n_words && !words) || (n_words & 3) || (uint64_t)n_events * 12 > n_words || (n_entries && !measures) ||
        (n_footprints && !footprints))
        return VGI_ERR_INVALID;
    // Footprint tasks: a count record, then (box min, header record) (box
    // max, bound record) (first thread, grid, 0, 0); the first threads tile
    // grid^2 threads per task in order, and both records name event words.
    uint64_t threads = 0;
    if (n_footprints) {
        if (footprints[0] != (int32_t)n_footprints || n_footprints > 4096) return fail(c, VGI_ERR_INVALID, "footprint count record");
        for (uint32_t e = 0; e < n_footprints; ++e) {
            const int32_t* t = footprints + 4 + (size_t)e * 12;
            const int64_t grid = t[9], header = t[3], bound = t[7];
            if (t[8] != (int32_t)threads || grid < 1 || grid > 1024 || header < 0 || bound < 0 || (uint64_t)header + 2 > n_words / 4 ||
                (uint64_t)bound + 2 > n_words / 4 || t[0] > t[4] || t[1] > t[5] || t[2] > t[6])
                return fail(c, VGI_ERR_INVALID, "footprint tasks must tile their threads, span a box and name event records");
            threads += (uint64_t)grid * (uint64_t)grid;
            if (threads > 0x7fffffffull) return fail(c, VGI_ERR_CAPACITY, "too many footprint threads");
        }
    }
    // Entries must tile their positions in order and name a bound record.
    uint64_t positions = 0;
    for (uint32_t e = 0; e < n_entries; ++e) {
        const uint32_t* a = measures + (size_t)e * 12;
        const uint32_t* size = a + 8;
        const uint64_t count = (uint64_t)size[0] * size[1] * size[2];
        if (a[1] != positions || a[2] != count || count == 0 || (uint64_t)a[0] + 2 > n_words / 4 ||
            (uint64_t)a[0] < (uint64_t)n_events * 3)
            return fail(c, VGI_ERR_INVALID, "measured edit entries must tile their scan positions and name a bound record");
        positions += count;
        if (positions > 0x7fffffffull) return fail(c, VGI_ERR_CAPACITY, "too many measured edit positions");
    }
    c->n_events_read = 0;
    if (c->n_slots == 0) return VGI_OK;
    if (n_entries && !c->material_light.ptr) return fail(c, VGI_ERR_STATE, "measured edits need the material table");
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, c->events.reserve(std::max<uint64_t>(n_words / 4, 1)));
    if (n_words) VGI_CUDA(c, h2d(c->events.ptr, words, n_words * 4, c->stream));
    if (n_footprints) {
        // Where each changed box's shadow lands, into its reserved Light
        // event, before the measured edits and retention read the events.
        if (!c->geometry || !c->materials.ptr || !c->lights.ptr) return fail(c, VGI_ERR_STATE, "footprints need geometry and the model");
        std::vector<uint32_t> sums((size_t)n_footprints * 8, 0u);
        for (uint32_t e = 0; e < n_footprints; ++e) sums[(size_t)e * 8] = sums[(size_t)e * 8 + 1] = sums[(size_t)e * 8 + 2] = 0xffffffffu;
        VGI_CUDA(c, c->footprints.reserve((size_t)n_footprints * 3 + 1));
        VGI_CUDA(c, c->footprint_sums.reserve(sums.size()));
        VGI_CUDA(c, h2d(c->footprints.ptr, footprints, ((size_t)n_footprints * 3 + 1) * 16, c->stream));
        VGI_CUDA(c, h2d(c->footprint_sums.ptr, sums.data(), sums.size() * 4, c->stream));
        const TraceArgs tr = trace_args(c, nullptr, nullptr, 0, 1, false);
        launch_footprints(tr, c->footprints.ptr, n_footprints, (uint32_t)threads, c->n_directional, c->footprint_sums.ptr, c->events.ptr,
                          c->stream);
        VGI_CUDA(c, cudaGetLastError());
        VGI_CUDA(c, cudaStreamSynchronize(c->stream));  // the host vector above is the copy's source
    }
    if (n_entries) {
        VGI_CUDA(c, c->measures.reserve((size_t)n_entries * 3));
        VGI_CUDA(c, c->measure_max.reserve(n_entries));
        VGI_CUDA(c, h2d(c->measures.ptr, measures, (size_t)n_entries * 48, c->stream));
        launch_measure_edits(c->state.ptr, c->slot_meta.ptr, c->face_index.ptr, c->material_light.ptr, c->measures.ptr, n_entries,
                             (uint32_t)positions, c->measure_max.ptr, c->events.ptr, c->stream);
        VGI_CUDA(c, cudaGetLastError());
    }
    c->n_events = n_events;
    AccumArgs acc = accum_args(c, 0, 0);
    launch_apply_events(acc, c->events.ptr, c->n_slots, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->n_events = 0;
    c->n_events_read = n_words / 4;
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

// ---- view tier (vgi_view.cuh) --------------------------------------------
namespace {
ViewArgs view_args(vgi_ctx* c) {
    ViewArgs v{};
    v.t = trace_args(c, nullptr, nullptr, 0, 1, c->n_slots > 0);
    v.receivers = c->v_receivers.ptr;
    v.paths = c->v_paths.ptr;
    v.conts = c->v_conts.ptr;
    v.estimates = c->v_estimates.ptr;
    v.queue = c->v_queue.ptr;
    v.shared_state = c->state.ptr;
    v.shared_meta = c->slot_meta.ptr;
    v.shared_cache = c->cache.ptr;
    v.n = c->n_view;
    v.reach = 192u * 192u;  // INFLUENCE_RADIUS^2 (src/retention.rs:33-40)
    v.physical = std::max(c->transport.measured_retention, 0.0f);
    v.hits = c->transport.bounces;
    return v;
}
bool view_ready(vgi_ctx* c) { return c->directory.ptr && c->materials.ptr && c->lights.ptr && c->emitters.ptr; }
}  // namespace

int vgi_view_set_receivers(vgi_ctx* c, const vgi_face* faces, uint32_t n) {
    if (!c || (n && !faces)) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    std::vector<uint4> receivers((size_t)n * 2), estimates((size_t)n * 4, make_uint4(0, 0, 0, 0));
    for (uint32_t i = 0; i < n; ++i) {
        const vgi_face& f = faces[i];
        if (f.face > 5 || f.material > 255) return fail(c, VGI_ERR_INVALID, "receiver face or material out of range");
        // The receiver's surface point: the face centre, voxel + 0.5 + normal * 0.5.
        float s[3];
        for (int a = 0; a < 3; ++a) {
            const float n_a = (int)(f.face >> 1) == a ? ((f.face & 1u) ? -1.0f : 1.0f) : 0.0f;
            s[a] = ((float)f.voxel[a] + 0.5f) + n_a * 0.5f;
        }
        uint32_t bits[3];
        std::memcpy(bits, s, 12);
        receivers[(size_t)i * 2] = make_uint4(bits[0], bits[1], bits[2], f.face);
        receivers[(size_t)i * 2 + 1] = make_uint4((uint32_t)f.voxel[0], (uint32_t)f.voxel[1], (uint32_t)f.voxel[2], 0u);
        estimates[(size_t)i * 4 + 3] = make_uint4(0u, f.material, 0u, 0u);
    }
    const size_t m = std::max<uint32_t>(n, 1);
    VGI_CUDA(c, c->v_receivers.reserve(m * 2));
    VGI_CUDA(c, c->v_paths.reserve(m * 8));
    VGI_CUDA(c, c->v_conts.reserve(m * 8));
    VGI_CUDA(c, c->v_estimates.reserve(m * 4));
    VGI_CUDA(c, c->v_queue.reserve(12 + 2 * m + kSunFlipWords));
    if (n) {
        VGI_CUDA(c, h2d(c->v_receivers.ptr, receivers.data(), (size_t)n * 32, c->stream));
        VGI_CUDA(c, h2d(c->v_estimates.ptr, estimates.data(), (size_t)n * 64, c->stream));
        VGI_CUDA(c, cudaMemsetAsync(c->v_paths.ptr, 0, (size_t)n * 128, c->stream));
        VGI_CUDA(c, cudaMemsetAsync(c->v_conts.ptr, 0, (size_t)n * 128, c->stream));
    }
    VGI_CUDA(c, cudaMemsetAsync(c->v_queue.ptr, 0, (12 + 2 * m + kSunFlipWords) * 4, c->stream));
    c->n_view = n;
    c->view_frames = 0;
    c->v_hash_valid = false;
    c->v_tiles_n = 0;
    c->v_published_valid = false;
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

namespace {
// The view receivers' owner hash (built once per receiver list).
int ensure_receiver_hash(vgi_ctx* c) {
    if (c->n_view == 0 || c->v_hash_valid) return VGI_OK;
    uint32_t mask = 63;
    while (mask + 1 < 2 * c->n_view) mask = mask * 2 + 1;
    VGI_CUDA(c, c->v_hash.reserve((size_t)mask + 1));
    VGI_CUDA(c, cudaMemsetAsync(c->v_hash.ptr, 0, ((size_t)mask + 1) * 4, c->stream));
    launch_receiver_hash(c->v_receivers.ptr, c->n_view, c->v_hash.ptr, mask, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->v_hash_mask = mask;
    c->v_hash_valid = true;
    return VGI_OK;
}
}  // namespace

// ---- far tier (voxel_view_pixels.wgsl) -------------------------------------------
int vgi_far_frame(vgi_ctx* c, const vgi_camera* cam, const vgi_far_settings* settings, uint32_t frame) {
    if (!c || !cam || !settings) return VGI_ERR_INVALID;
    if (!view_ready(c)) return fail(c, VGI_ERR_STATE, "the far tier needs geometry, materials, lights and emitters");
    if (cam->width == 0 || cam->height == 0 || (uint64_t)cam->width * cam->height > (1ull << 26))
        return fail(c, VGI_ERR_INVALID, "camera size outside 1..2^26 pixels");
    if (settings->measure > 2) return fail(c, VGI_ERR_INVALID, "far measure is 0, 1 or 2");
    VGI_CUDA(c, cudaSetDevice(c->device));
    // FarTierSettings::normalized and cell_for (src/settings.rs:140-167).
    const float voxel_pixels = std::isfinite(settings->voxel_pixels) ? std::min(std::max(settings->voxel_pixels, 0.0f), 4096.0f) : 0.0f;
    const float history = std::isfinite(settings->history) ? std::min(std::max(settings->history, 1.0f), 1024.0f) : 32.0f;
    const uint32_t rate = std::min<uint32_t>(std::max<uint32_t>(settings->rate, 1u), 8u);
    const uint32_t steps = std::min<uint32_t>(std::max<uint32_t>(settings->steps, 16u), 2048u);
    uint32_t size = std::min<uint32_t>(settings->cell, 4u);
    if (size == 0) size = (uint32_t)std::min(std::max(std::round((float)cam->height / 480.0f), 1.0f), 4.0f);
    const uint32_t cx = (cam->width + size - 1) / size, cy = (cam->height + size - 1) / size;
    const uint32_t cells = cx * cy;
    const uint32_t flags = (voxel_pixels > 0.0f ? 1u : 0u) | (settings->measure << 1);
    if (cx != c->far_shape[0] || cy != c->far_shape[1] || cam->width != c->far_size[0] || cam->height != c->far_size[1]) {
        for (auto& b : c->far_cells) {
            VGI_CUDA(c, b.reserve((size_t)cells * 3));
            VGI_CUDA(c, cudaMemsetAsync(b.ptr, 0, (size_t)cells * 48, c->stream));
        }
        VGI_CUDA(c, c->far_output.reserve(4 + (size_t)cells));
        VGI_CUDA(c, cudaMemsetAsync(c->far_output.ptr, 0, (4 + (size_t)cells) * 16, c->stream));
        VGI_CUDA(c, c->far_queue.reserve(1 + (size_t)cells));
        VGI_CUDA(c, c->far_stats.reserve(8));
        c->far_has_prev = false;
        c->far_size[0] = cam->width;
        c->far_size[1] = cam->height;
    }
    c->far_shape[0] = cx;
    c->far_shape[1] = cy;
    c->far_shape[2] = size;
    c->far_shape[3] = flags;
    // A camera not drawn last frame loses its history (src/gpu/view/runtime.rs:870-871).
    const bool previous = c->far_has_prev && frame - c->far_last_frame <= 1u;
    FarView f{};
    const float cam_words[10] = {cam->eye[0], cam->eye[1], cam->eye[2], cam->forward[0], cam->forward[1], cam->forward[2],
                                 cam->up[0], cam->up[1], cam->up[2], cam->tan_half_fov};
    std::copy(cam_words, cam_words + 10, f.cam);
    std::copy(previous ? c->far_prev : cam_words, (previous ? c->far_prev : cam_words) + 10, f.prev);
    f.width = cam->width;
    f.height = cam->height;
    f.grid[0] = cx;
    f.grid[1] = cy;
    f.grid[2] = size;
    f.grid[3] = flags;
    const uint32_t prev_bits = previous ? c->far_last_frame : 0xffffffffu;
    f.tune[0] = voxel_pixels;
    f.tune[1] = history;
    f.tune[2] = (float)rate;
    std::memcpy(&f.tune[3], &prev_bits, 4);
    // pixel_axis: the view forward and clip_from_view[1][1] * height / 2.
    f.axis[0] = cam->forward[0];
    f.axis[1] = cam->forward[1];
    f.axis[2] = cam->forward[2];
    f.axis[3] = (1.0f / cam->tan_half_fov) * (float)cam->height * 0.5f;
    for (int k = 0; k < 3; ++k) {
        f.interest_min[k] = settings->interest_min[k];
        f.interest_max[k] = settings->interest_max[k];
    }
    f.interest_min[3] = f.interest_max[3] = settings->bounded ? 1 : 0;
    f.frame = frame;
    f.custom = c->custom_lights ? 1u : 0u;
    if (c->n_view) {
        const int rc = ensure_receiver_hash(c);
        if (rc != VGI_OK) return rc;
        f.receivers = c->v_receivers.ptr;
        f.estimates = c->v_estimates.ptr;
        f.receiver_hash = c->v_hash.ptr;
        f.hash_mask = c->v_hash_mask;
        f.n_receivers = c->n_view;
    }
    TraceArgs a = trace_args(c, nullptr, nullptr, 0, 1, c->n_slots > 0);
    a.path_steps = steps;
    VGI_CUDA(c, cudaMemsetAsync(c->far_queue.ptr, 0, 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->far_stats.ptr, 0, 32, c->stream));
    const uint32_t prev_index = c->far_current;
    c->far_current ^= 1u;
    launch_far(a, f, c->far_cells[prev_index].ptr, c->far_cells[c->far_current].ptr, c->far_output.ptr, c->far_queue.ptr, c->far_stats.ptr,
               transport_limited(c), c->stream);
    VGI_CUDA(c, cudaGetLastError());
    std::copy(cam_words, cam_words + 10, c->far_prev);
    c->far_last_frame = frame;
    c->far_has_prev = true;
    return VGI_OK;
}

int vgi_set_topology_prior(vgi_ctx* c, int enable) {
    if (!c) return VGI_ERR_INVALID;
    c->topology_prior = enable != 0;
    return VGI_OK;
}

int vgi_set_far_handoff(vgi_ctx* c, int enable) {
    if (!c) return VGI_ERR_INVALID;
    c->far_handoff = enable != 0;
    return VGI_OK;
}

int vgi_far_reset(vgi_ctx* c) {
    if (!c) return VGI_ERR_INVALID;
    // A new camera's state: zeroed histories and output (the stale cells a
    // reader skips by their stamp start empty).
    const size_t cells = (size_t)c->far_shape[0] * c->far_shape[1];
    if (cells) {
        VGI_CUDA(c, cudaSetDevice(c->device));
        for (auto& b : c->far_cells) VGI_CUDA(c, cudaMemsetAsync(b.ptr, 0, cells * 48, c->stream));
        VGI_CUDA(c, cudaMemsetAsync(c->far_output.ptr, 0, (4 + cells) * 16, c->stream));
        VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    c->far_current = 0;
    c->far_has_prev = false;
    return VGI_OK;
}

int vgi_far_read(vgi_ctx* c, uint32_t* shape4, uint32_t* output, uint32_t* cells12, uint32_t* stats8) {
    if (!c) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaSetDevice(c->device));
    const size_t cells = (size_t)c->far_shape[0] * c->far_shape[1];
    if (shape4) std::copy(c->far_shape, c->far_shape + 4, shape4);
    if (cells) {
        if (output) VGI_CUDA(c, cudaMemcpyAsync(output, c->far_output.ptr, (4 + cells) * 16, cudaMemcpyDeviceToHost, c->stream));
        if (cells12) VGI_CUDA(c, cudaMemcpyAsync(cells12, c->far_cells[c->far_current].ptr, cells * 48, cudaMemcpyDeviceToHost, c->stream));
        if (stats8) VGI_CUDA(c, cudaMemcpyAsync(stats8, c->far_stats.ptr, 32, cudaMemcpyDeviceToHost, c->stream));
    } else if (stats8) {
        std::fill(stats8, stats8 + 8, 0u);
    }
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

// ---- reconstruction and presentation (voxel_view_runtime.wgsl:380-521,
// voxel_gi_presentation.wesl:350-412) ------------------------------------------------
int vgi_view_set_tiles(vgi_ctx* c, const uint32_t* tiles, uint32_t n, uint32_t tiles_x, uint32_t tiles_y) {
    if (!c || (n && !tiles)) return VGI_ERR_INVALID;
    if (n != c->n_view) return fail(c, VGI_ERR_INVALID, "one tile per view receiver");
    if ((uint64_t)tiles_x * tiles_y > (1u << 24)) return fail(c, VGI_ERR_INVALID, "at most 2^24 tiles");
    VGI_CUDA(c, cudaSetDevice(c->device));
    const uint32_t n_tiles = tiles_x * tiles_y;
    // Lists per tile in receiver order (a counting sort): the donor order of
    // the reconstruction does not depend on the GPU's scheduling.
    std::vector<uint32_t> start((size_t)n_tiles + 1, 0), items(std::max<uint32_t>(n, 1)), tile_of(std::max<uint32_t>(n, 1), 0xffffffffu);
    for (uint32_t i = 0; i < n; ++i)
        if (tiles[i] < n_tiles) ++start[tiles[i] + 1];
    for (uint32_t t = 0; t < n_tiles; ++t) start[t + 1] += start[t];
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (uint32_t i = 0; i < n; ++i) {
        if (tiles[i] >= n_tiles) continue;
        tile_of[i] = tiles[i];
        items[fill[tiles[i]]++] = i;
    }
    VGI_CUDA(c, c->v_tile_of.reserve(tile_of.size()));
    VGI_CUDA(c, c->v_tile_start.reserve(start.size()));
    VGI_CUDA(c, c->v_tile_items.reserve(items.size()));
    VGI_CUDA(c, h2d(c->v_tile_of.ptr, tile_of.data(), tile_of.size() * 4, c->stream));
    VGI_CUDA(c, h2d(c->v_tile_start.ptr, start.data(), start.size() * 4, c->stream));
    VGI_CUDA(c, h2d(c->v_tile_items.ptr, items.data(), items.size() * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    c->v_tiles[0] = tiles_x;
    c->v_tiles[1] = tiles_y;
    c->v_tiles_n = n;
    return VGI_OK;
}

namespace {
ViewDisplay view_display(vgi_ctx* c) {
    ViewDisplay d{};
    d.receivers = c->v_receivers.ptr;
    d.estimates = c->v_estimates.ptr;
    d.conts = c->v_conts.ptr;
    d.tile_of = c->v_tile_of.ptr;
    d.tile_start = c->v_tile_start.ptr;
    d.tile_items = c->v_tile_items.ptr;
    d.tiles_x = c->v_tiles[0];
    d.tiles_y = c->v_tiles[1];
    d.receiver_hash = c->v_hash.ptr;
    d.hash_mask = c->v_hash_mask;
    d.n = c->n_view;
    d.custom = c->custom_lights ? 1u : 0u;
    d.published = c->v_published.ptr;
    d.stats = c->v_publish_stats.ptr;
    return d;
}
}  // namespace

int vgi_view_reconstruct(vgi_ctx* c, const vgi_view_display* display) {
    if (!c || !display) return VGI_ERR_INVALID;
    if (!view_ready(c)) return fail(c, VGI_ERR_STATE, "the view tier needs geometry, materials, lights and emitters");
    if (c->n_view == 0) return VGI_OK;
    if (c->v_tiles_n != c->n_view) return fail(c, VGI_ERR_STATE, "vgi_view_set_tiles first");
    VGI_CUDA(c, cudaSetDevice(c->device));
    int rc = ensure_receiver_hash(c);
    if (rc != VGI_OK) return rc;
    VGI_CUDA(c, c->v_published.reserve((size_t)c->n_view * 3));
    VGI_CUDA(c, c->v_publish_stats.reserve(5));
    VGI_CUDA(c, cudaMemsetAsync(c->v_publish_stats.ptr, 0, 20, c->stream));
    ViewDisplay d = view_display(c);
    d.display[0] = display->evidence_goal;
    d.display[1] = display->spatial;
    d.display[2] = display->temporal;
    launch_reconstruct(trace_args(c, nullptr, nullptr, 0, 1, c->n_slots > 0), d, transport_limited(c), c->transport.budgeted != 0, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->v_published_valid = true;
    return VGI_OK;
}

int vgi_view_read_published(vgi_ctx* c, uint32_t* pixels12, uint32_t* stats5) {
    if (!c) return VGI_ERR_INVALID;
    if (c->n_view && !c->v_published_valid) return fail(c, VGI_ERR_STATE, "nothing published since the receivers changed");
    VGI_CUDA(c, cudaSetDevice(c->device));
    if (c->n_view) {
        if (pixels12) VGI_CUDA(c, cudaMemcpyAsync(pixels12, c->v_published.ptr, (size_t)c->n_view * 48, cudaMemcpyDeviceToHost, c->stream));
        if (stats5) VGI_CUDA(c, cudaMemcpyAsync(stats5, c->v_publish_stats.ptr, 20, cudaMemcpyDeviceToHost, c->stream));
    } else if (stats5) {
        std::fill(stats5, stats5 + 5, 0u);
    }
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_view_present(vgi_ctx* c, const vgi_camera* cam, int corners, float* rgba) {
    if (!c || !cam || !rgba) return VGI_ERR_INVALID;
    if (!c->geometry) return fail(c, VGI_ERR_STATE, "no geometry uploaded");
    if (c->n_view && !c->v_published_valid) return fail(c, VGI_ERR_STATE, "vgi_view_reconstruct first");
    const uint64_t n = (uint64_t)cam->width * cam->height;
    if (n == 0 || n > (1ull << 26)) return fail(c, VGI_ERR_INVALID, "camera size outside 1..2^26 pixels");
    VGI_CUDA(c, cudaSetDevice(c->device));
    DevBuf<float>& dcam = c->disc_cam;
    DevBuf<float4>& image = c->present_image;
    VGI_CUDA(c, dcam.reserve(10));
    VGI_CUDA(c, image.reserve(n));
    const float host_cam[10] = {cam->eye[0], cam->eye[1], cam->eye[2], cam->forward[0], cam->forward[1], cam->forward[2],
                                cam->up[0], cam->up[1], cam->up[2], cam->tan_half_fov};
    VGI_CUDA(c, h2d(dcam.ptr, host_cam, sizeof(host_cam), c->stream));
    ViewDisplay d = view_display(c);
    uint32_t empty = 0;
    DevBuf<uint32_t> no_hash;
    if (c->n_view == 0) {
        // No receivers: every face displays zero.
        VGI_CUDA(c, no_hash.reserve(1));
        VGI_CUDA(c, h2d(no_hash.ptr, &empty, 4, c->stream));
        d.receiver_hash = no_hash.ptr;
        d.hash_mask = 0;
    }
    launch_present(trace_args(c, nullptr, nullptr, 0, 1, false), d, dcam.ptr, cam->width, cam->height, corners != 0, image.ptr, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaMemcpyAsync(rgba, image.ptr, n * 16, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_view_frame(vgi_ctx* c, const vgi_view_wave* wave, const uint32_t* events, uint32_t n_events, uint64_t n_words) {
    if (!c || !wave || (n_words && !events) || (n_words & 3) || (uint64_t)n_events * 12 > n_words) return VGI_ERR_INVALID;
    if (!view_ready(c)) return fail(c, VGI_ERR_STATE, "the view tier needs geometry, materials, lights and emitters");
    if (c->n_view == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    ViewArgs v = view_args(c);
    v.range[0] = wave->first;
    v.range[1] = wave->invocations == 0 ? c->n_view : wave->invocations;
    v.range[2] = wave->max_hits;
    v.range[3] = wave->depth;
    for (int k = 0; k < 4; ++k) v.ticket[k] = wave->ticket[k];
    v.view_first = wave->view_first != 0;
    v.shared = wave->shared != 0 && c->n_slots > 0;
    v.clock = wave->clock_ms;
    if (n_events) {
        VGI_CUDA(c, c->v_events.reserve(n_words / 4));
        VGI_CUDA(c, h2d(c->v_events.ptr, events, n_words * 4, c->stream));
    }
    v.events = c->v_events.ptr;
    v.n_events = n_events;
    if (c->far_handoff && c->far_has_prev && (c->far_shape[3] & 1u)) {
        // The last far frame's cells, seen from its camera.
        FarView& f = v.far;
        std::copy(c->far_prev, c->far_prev + 10, f.cam);
        std::copy(c->far_prev, c->far_prev + 10, f.prev);
        f.width = c->far_size[0];
        f.height = c->far_size[1];
        std::copy(c->far_shape, c->far_shape + 4, f.grid);
        std::memcpy(&f.tune[3], &c->far_last_frame, 4);
        f.axis[0] = c->far_prev[3];
        f.axis[1] = c->far_prev[4];
        f.axis[2] = c->far_prev[5];
        f.axis[3] = (1.0f / c->far_prev[9]) * (float)c->far_size[1] * 0.5f;
        v.far_cells = c->far_cells[c->far_current].ptr;
        v.far_stats = c->far_stats.ptr;
    }
    // Sun-flip reports build up over frames until vgi_view_read_sun_flips
    // delivers them (the reference clears its region only after a timing
    // receipt copied it, src/gpu/view/timing.rs:386-387).
    v.frame = c->view_frames;
    v.has_previous = c->view_frames > 0 ? 1u : 0u;
    v.n_directional = c->n_directional;
    if (c->topology_prior) {
        const int rc = ensure_receiver_hash(c);
        if (rc != VGI_OK) return rc;
        VGI_CUDA(c, c->v_prev_estimates.reserve((size_t)c->n_view * 4));
        VGI_CUDA(c, cudaMemcpyAsync(c->v_prev_estimates.ptr, c->v_estimates.ptr, (size_t)c->n_view * 64, cudaMemcpyDeviceToDevice, c->stream));
        v.topology = 1u;
        v.receiver_hash = c->v_hash.ptr;
        v.hash_mask = c->v_hash_mask;
        v.prev_estimates = c->v_prev_estimates.ptr;
    }
    launch_view_frame(v, transport_limited(c), c->transport.budgeted != 0, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    c->view_frames += 1;
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_view_read_sun_flips(vgi_ctx* c, uint32_t* words) {
    if (!c || !words) return VGI_ERR_INVALID;
    if (c->n_view == 0) {
        std::fill(words, words + kSunFlipWords, 0u);
        return VGI_OK;
    }
    VGI_CUDA(c, cudaSetDevice(c->device));
    uint32_t* region = c->v_queue.ptr + 12 + 2 * (size_t)c->n_view;
    VGI_CUDA(c, cudaMemcpyAsync(words, region, kSunFlipWords * 4, cudaMemcpyDeviceToHost, c->stream));
    // Delivered: the region starts over.
    VGI_CUDA(c, cudaMemsetAsync(region, 0, kSunFlipWords * 4, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_view_read(vgi_ctx* c, uint32_t* receivers8, uint32_t* paths32, uint32_t* conts32, uint32_t* estimates16, uint32_t* queue) {
    if (!c) return VGI_ERR_INVALID;
    const size_t n = c->n_view;
    if (n) {
        if (receivers8) VGI_CUDA(c, cudaMemcpyAsync(receivers8, c->v_receivers.ptr, n * 32, cudaMemcpyDeviceToHost, c->stream));
        if (paths32) VGI_CUDA(c, cudaMemcpyAsync(paths32, c->v_paths.ptr, n * 128, cudaMemcpyDeviceToHost, c->stream));
        if (conts32) VGI_CUDA(c, cudaMemcpyAsync(conts32, c->v_conts.ptr, n * 128, cudaMemcpyDeviceToHost, c->stream));
        if (estimates16) VGI_CUDA(c, cudaMemcpyAsync(estimates16, c->v_estimates.ptr, n * 64, cudaMemcpyDeviceToHost, c->stream));
        if (queue) VGI_CUDA(c, cudaMemcpyAsync(queue, c->v_queue.ptr, (12 + 2 * n) * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_view_trace_paths(vgi_ctx* c, uint32_t samples, uint32_t* paths32) {
    if (!c || (c->n_view && samples && !paths32)) return VGI_ERR_INVALID;
    if (!view_ready(c)) return fail(c, VGI_ERR_STATE, "the view tier needs geometry, materials, lights and emitters");
    const uint64_t total = (uint64_t)c->n_view * samples;
    if (total == 0) return VGI_OK;
    if (total > (1ull << 26)) return fail(c, VGI_ERR_CAPACITY, "at most 2^26 view path records per call");
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, c->v_scratch.reserve(total * 8));
    ViewArgs v = view_args(c);
    launch_view_trace_paths(v, samples, c->v_scratch.ptr, transport_limited(c), c->transport.budgeted != 0, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaMemcpyAsync(paths32, c->v_scratch.ptr, total * 128, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_reference_fp64(vgi_ctx* c, const uint32_t* tasks, uint32_t n, uint32_t samples, uint64_t seed, double* mean3, double* second3,
                       uint32_t* known) {
    if (!c || (n && (!tasks || !mean3))) return VGI_ERR_INVALID;
    if (!view_ready(c)) return fail(c, VGI_ERR_STATE, "the reference needs geometry, materials, lights and emitters");
    if (n == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    // Emitters chosen in proportion to their material's emission weight.
    const size_t ne = c->host_emitter_records.size() / 8;
    std::vector<double> cdf(ne + 1, 0.0);
    std::vector<int4> recs(std::max<size_t>(ne, 1));
    for (size_t i = 0; i < ne; ++i) {
        const uint32_t* w = c->host_emitter_records.data() + i * 8;
        float mf;
        std::memcpy(&mf, &w[6], 4);
        const uint32_t m = (uint32_t)mf & 255u;
        const double weight = (double)c->host_materials[(size_t)m * 16 + 13];
        cdf[i + 1] = cdf[i] + weight;
        recs[i] = make_int4((int)w[0], (int)w[1], (int)w[2], (int)((w[3] & 7u) | (m << 3)));
    }
    DevBuf<double> d_cdf, d_sum, d_second;
    DevBuf<int4> d_recs;
    DevBuf<uint4> d_tasks;
    DevBuf<uint32_t> d_known;
    VGI_CUDA(c, d_cdf.reserve(ne + 1));
    VGI_CUDA(c, d_recs.reserve(recs.size()));
    VGI_CUDA(c, d_tasks.reserve((size_t)n * 2));
    VGI_CUDA(c, d_sum.reserve((size_t)n * 3));
    VGI_CUDA(c, d_second.reserve((size_t)n * 3));
    VGI_CUDA(c, d_known.reserve(n));
    VGI_CUDA(c, h2d(d_cdf.ptr, cdf.data(), cdf.size() * 8, c->stream));
    VGI_CUDA(c, h2d(d_recs.ptr, recs.data(), recs.size() * 16, c->stream));
    VGI_CUDA(c, h2d(d_tasks.ptr, tasks, (size_t)n * 32, c->stream));
    TraceArgs a = trace_args(c, nullptr, nullptr, 0, 1, false);
    launch_reference64(a, d_cdf.ptr, d_recs.ptr, (uint32_t)ne, cdf[ne], d_tasks.ptr, n, samples, seed, d_sum.ptr, d_second.ptr, d_known.ptr,
                       c->stream);
    VGI_CUDA(c, cudaGetLastError());
    std::vector<double> sum((size_t)n * 3), second((size_t)n * 3);
    std::vector<uint32_t> cnt(n);
    VGI_CUDA(c, cudaMemcpyAsync(sum.data(), d_sum.ptr, sum.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(second.data(), d_second.ptr, second.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(cnt.data(), d_known.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    d_cdf.release(); d_recs.release(); d_tasks.release(); d_sum.release(); d_second.release(); d_known.release();
    for (uint32_t i = 0; i < n; ++i) {
        const double k = cnt[i] ? (double)cnt[i] : 1.0;
        for (int j = 0; j < 3; ++j) {
            mean3[(size_t)i * 3 + j] = sum[(size_t)i * 3 + j] / k;
            if (second3) second3[(size_t)i * 3 + j] = second[(size_t)i * 3 + j] / k;
        }
        if (known) known[i] = cnt[i];
    }
    return VGI_OK;
}

int vgi_mlp_set_weights(vgi_ctx* c, const float* master, uint32_t count) {
    if (!c || !master) return VGI_ERR_INVALID;
    if (count != mlp_weight_count()) return fail(c, VGI_ERR_INVALID, "MLP weight count must be 19456");
    VGI_CUDA(c, cudaSetDevice(c->device));
    VGI_CUDA(c, c->mlp_master.reserve(count));
    VGI_CUDA(c, c->mlp_image.reserve(mlp_image_bytes()));
    VGI_CUDA(c, c->mlp_error.reserve(2));
    VGI_CUDA(c, c->mlp_steps.reserve(2));
    VGI_CUDA(c, c->mlp_image_b.reserve(mlp_image_bytes()));
    VGI_CUDA(c, mlp_set_attributes());
    int sms = 148;
    VGI_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    c->mlp_sms = (uint32_t)sms;
    c->mlp_ctas = (uint32_t)sms * 2u;  // 110 KB of shared memory per forward CTA (three 128-row groups)
    VGI_CUDA(c, c->mlp_partials.reserve((size_t)sms * mlp_partial_floats()));
    VGI_CUDA(c, c->mlp_adam.reserve((size_t)count * 2));
    VGI_CUDA(c, c->mlp_grads.reserve((size_t)count + 1));
    VGI_CUDA(c, h2d(c->mlp_master.ptr, master, (size_t)count * 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_adam.ptr, 0, (size_t)count * 8, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_steps.ptr, 0, 8, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_grads.ptr, 0, (size_t)(count + 1) * 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_error.ptr, 0, 8, c->stream));
    launch_mlp_pack(c->mlp_master.ptr, c->mlp_image.ptr, c->stream);
    launch_mlp_pack_backward(c->mlp_master.ptr, c->mlp_image_b.ptr, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_mlp_get_weights(vgi_ctx* c, float* master, uint32_t count) {
    if (!c || !master || count != mlp_weight_count() || !c->mlp_master.ptr) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaMemcpyAsync(master, c->mlp_master.ptr, (size_t)count * 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_mlp_forward(vgi_ctx* c, const float* features, uint32_t n, float* out4) {
    if (!c || (n && (!features || !out4))) return VGI_ERR_INVALID;
    if (!c->mlp_image.ptr) return fail(c, VGI_ERR_STATE, "MLP weights are not set");
    if (n == 0) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    DevBuf<float> in;
    DevBuf<float4> out;
    VGI_CUDA(c, in.reserve((size_t)n * 96));
    VGI_CUDA(c, out.reserve(n));
    VGI_CUDA(c, h2d(in.ptr, features, (size_t)n * 96 * 4, c->stream));
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_error.ptr, 0, 4, c->stream));
    VGI_CUDA(c, launch_mlp_forward(in.ptr, c->mlp_image.ptr, out.ptr, n, c->mlp_error.ptr, c->mlp_ctas, c->stream, c->mlp_wait));
    uint32_t err = 0;
    VGI_CUDA(c, cudaMemcpyAsync(&err, c->mlp_error.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(out4, out.ptr, (size_t)n * 16, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err) return fail(c, VGI_ERR_CUDA, "MLP forward: a tensor-core wait ran out");
    return VGI_OK;
}

// Gradients of the relative-luminance loss over one batch already on the
// device, into mlp_grads (19456 gradients, then the loss).
// The training kernel over one device-resident batch: per-CTA partial rows.
// Returns the number of rows.
static uint32_t mlp_batch_partials(vgi_ctx* c, const float* features, const float4* targets, uint32_t n, int* rc) {
    *rc = VGI_OK;
    const cudaError_t e = launch_mlp_train(features, targets, n, c->mlp_image.ptr, c->mlp_image_b.ptr, c->mlp_partials.ptr,
                                           c->mlp_error.ptr, c->mlp_sms, c->stream, c->mlp_wait);
    if (e != cudaSuccess) *rc = fail(c, VGI_ERR_CUDA, std::string("MLP training launch: ") + cudaGetErrorString(e));
    return mlp_train_parts(n, c->mlp_sms);
}

static int mlp_upload_batch(vgi_ctx* c, const float* features, const float* targets4, uint32_t n, DevBuf<float>& in, DevBuf<float4>& y) {
    VGI_CUDA(c, in.reserve((size_t)n * 96));
    VGI_CUDA(c, y.reserve(n));
    VGI_CUDA(c, h2d(in.ptr, features, (size_t)n * 96 * 4, c->stream));
    VGI_CUDA(c, h2d(y.ptr, targets4, (size_t)n * 16, c->stream));
    return VGI_OK;
}

static int mlp_read_status(vgi_ctx* c, float* loss) {
    uint32_t err = 0;
    VGI_CUDA(c, cudaMemcpyAsync(&err, c->mlp_error.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    if (loss) VGI_CUDA(c, cudaMemcpyAsync(loss, c->mlp_grads.ptr + mlp_weight_count(), 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err) return fail(c, VGI_ERR_CUDA, "MLP training: a tensor-core wait ran out");
    return VGI_OK;
}

int vgi_mlp_gradients(vgi_ctx* c, const float* features, const float* targets4, uint32_t n, float* grads, float* loss) {
    if (!c || !n || !features || !targets4 || !grads) return VGI_ERR_INVALID;
    if (!c->mlp_image.ptr) return fail(c, VGI_ERR_STATE, "MLP weights are not set");
    VGI_CUDA(c, cudaSetDevice(c->device));
    DevBuf<float> in;
    DevBuf<float4> y;
    if (int e = mlp_upload_batch(c, features, targets4, n, in, y)) return e;
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_error.ptr, 0, 4, c->stream));
    int rc = VGI_OK;
    const uint32_t parts = mlp_batch_partials(c, in.ptr, y.ptr, n, &rc);
    if (rc != VGI_OK) return rc;
    launch_mlp_reduce(c->mlp_partials.ptr, parts, c->mlp_grads.ptr, c->mlp_grads.ptr + mlp_weight_count(), c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaMemcpyAsync(grads, c->mlp_grads.ptr, (size_t)mlp_weight_count() * 4, cudaMemcpyDeviceToHost, c->stream));
    return mlp_read_status(c, loss);
}

// One Adam step over a device-resident batch; the images are repacked.
static int mlp_train_step(vgi_ctx* c, const float* features, const float4* targets, uint32_t n, float lr) {
    int rc = VGI_OK;
    const uint32_t parts = mlp_batch_partials(c, features, targets, n, &rc);
    if (rc != VGI_OK) return rc;
    const uint32_t count = mlp_weight_count();
    launch_mlp_adam(c->mlp_master.ptr, c->mlp_adam.ptr, c->mlp_adam.ptr + count, c->mlp_partials.ptr, parts, lr, 0.9f, 0.99f, 1e-8f,
                    c->mlp_steps.ptr, c->mlp_image.ptr, c->mlp_image_b.ptr, c->mlp_grads.ptr + count, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    return VGI_OK;
}

// A frame's online training: `mlp_train_steps` Adam steps, each on
// `mlp_batch` faces drawn from the frame's results. Enqueued only.
//
// `mlp_batch` training samples a frame, split over `mlp_train_steps` Adam
// steps. Plain (warm-up) frames draw them from the frame's own receivers. A
// frame that ended paths with the network trains on the faces those paths
// hit without a cache answer, the faces the network is asked about: that
// many of the frame's queries, drawn by hash, are traced as faces of their
// own (kMlpTrainSamples paths each, one diffuse hit, the network or the
// cache at the next hit).
static int mlp_frame_training(vgi_ctx* c) {
    if (!c->mlp_cache || !c->mlp_image.ptr || c->n_slots == 0) return VGI_OK;
    const MlpEncoding enc = mlp_encoding(c);
    const uint32_t rows = c->mlp_batch, steps = c->mlp_train_steps;
    // Rows a step: a share of the frame's samples, or (with a schedule) a
    // batch that may exceed it, the steps then cycling through the samples.
    const uint32_t batch = c->mlp_step_rows ? std::min(c->mlp_step_rows, rows) : rows / steps;
    if (!mlp_terminates(c)) {
        for (uint32_t k = 0; k < steps; ++k) {
            launch_mlp_encode_training(c->slot_meta.ptr, c->results.ptr, c->materials.ptr, c->n_slots, c->mlp_steps.ptr, batch, enc,
                                       c->mlp_features.ptr, c->mlp_targets.ptr, c->stream);
            if (int e = mlp_train_step(c, c->mlp_features.ptr, c->mlp_targets.ptr, batch, c->mlp_lr)) return e;
        }
        return VGI_OK;
    }
    const uint32_t* queries = c->w_counters.ptr + 4;
    VGI_CUDA(c, cudaMemcpyAsync(c->mlp_query_count.ptr, queries, 4, cudaMemcpyDeviceToDevice, c->stream));
    launch_mlp_query_tasks(c->w_mlp_queue.ptr, queries, c->mlp_queue_capacity, c->mlp_steps.ptr, rows, kMlpTrainSamples, enc,
                           c->mlp_train_tasks.ptr, c->mlp_features.ptr, c->stream);
    const TraceArgs tr = trace_args(c, c->mlp_train_tasks.ptr, c->mlp_train_results.ptr, rows, kMlpTrainSamples, true);
    if (int e = run_trace(c, tr, false, false)) return e;
    launch_mlp_query_targets(c->mlp_train_results.ptr, c->mlp_train_tasks.ptr, rows, c->mlp_targets.ptr, c->stream);
    for (uint32_t k = 0; k < steps; ++k) {
        uint32_t first = (uint32_t)(((uint64_t)k * batch) % rows);
        if (first + batch > rows) first = rows - batch;
        if (int e = mlp_train_step(c, c->mlp_features.ptr + (size_t)first * 96, c->mlp_targets.ptr + first, batch, c->mlp_lr)) return e;
    }
    c->mlp_queried = true;
    return VGI_OK;
}

int vgi_mlp_encode(vgi_ctx* c, const vgi_face* faces, uint32_t n, float* features) {
    if (!c || (n && (!faces || !features))) return VGI_ERR_INVALID;
    if (!c->materials.ptr) return fail(c, VGI_ERR_STATE, "materials are not set");
    if (n == 0) return VGI_OK;
    std::vector<uint4> meta(n);
    for (uint32_t k = 0; k < n; ++k) {
        if (faces[k].face > 5 || faces[k].material > 255) return fail(c, VGI_ERR_INVALID, "face or material out of range");
        meta[k] = make_uint4((uint32_t)faces[k].voxel[0], (uint32_t)faces[k].voxel[1], (uint32_t)faces[k].voxel[2],
                             faces[k].face | (faces[k].material << 16));
    }
    VGI_CUDA(c, cudaSetDevice(c->device));
    DevBuf<uint4> m;
    DevBuf<float> out;
    VGI_CUDA(c, m.reserve(n));
    VGI_CUDA(c, out.reserve((size_t)n * 96));
    VGI_CUDA(c, h2d(m.ptr, meta.data(), (size_t)n * 16, c->stream));
    launch_mlp_encode_faces(m.ptr, n, c->materials.ptr, mlp_encoding(c), out.ptr, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaMemcpyAsync(features, out.ptr, (size_t)n * 96 * 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_set_mlp_cache(vgi_ctx* c, int enable, uint32_t warm_frames, uint32_t batch, uint32_t steps_per_frame, float lr) {
    if (c) drop_graph(c);  // what a frame launches changes
    if (!c) return VGI_ERR_INVALID;
    if (enable && !c->mlp_image.ptr) return fail(c, VGI_ERR_STATE, "MLP weights are not set");
    if (enable && (steps_per_frame == 0 || steps_per_frame > 64 || batch < steps_per_frame || batch > (1u << 22) || !(lr > 0.0f)))
        return fail(c, VGI_ERR_INVALID, "MLP cache: 1..64 steps a frame, steps <= samples <= 2^22, positive learning rate");
    c->mlp_cache = enable != 0;
    if (!c->mlp_cache) return VGI_OK;
    VGI_CUDA(c, cudaSetDevice(c->device));
    const size_t rows = batch;
    VGI_CUDA(c, c->mlp_features.reserve(rows * 96));
    VGI_CUDA(c, c->mlp_targets.reserve(rows));
    VGI_CUDA(c, c->mlp_train_tasks.reserve(rows * 2));
    VGI_CUDA(c, c->mlp_train_results.reserve(rows * 6));
    VGI_CUDA(c, c->mlp_query_count.reserve(1));
    c->mlp_warm = warm_frames;
    c->mlp_batch = batch;
    c->mlp_train_steps = steps_per_frame;
    c->mlp_lr = lr;
    c->mlp_frames = 0;
    return VGI_OK;
}

int vgi_set_mlp_schedule(vgi_ctx* c, uint32_t rows_per_step, float history_share) {
    if (!c) return VGI_ERR_INVALID;
    if (!(history_share >= 0.0f && history_share <= 1.0f)) return fail(c, VGI_ERR_INVALID, "MLP history share must be in [0, 1]");
    if (rows_per_step > (1u << 22)) return fail(c, VGI_ERR_INVALID, "MLP rows per step: at most 2^22");
    drop_graph(c);  // the captured training steps change
    c->mlp_history = history_share;
    c->mlp_step_rows = rows_per_step;
    return VGI_OK;
}

int vgi_mlp_set_wait_limit(vgi_ctx* c, uint32_t polls) {
    if (!c) return VGI_ERR_INVALID;
    drop_graph(c);  // captured query launches carry the old limit
    c->mlp_wait = polls == VGI_MLP_WAIT_DEFAULT ? kMlpWaitPolls : polls;
    return VGI_OK;
}

int vgi_inject_failure(vgi_ctx* c, uint32_t what, uint32_t count) {
    (void)c;
    if (what == VGI_INJECT_ALLOC) t_fail_allocs = count;
    else if (what == VGI_INJECT_UPLOAD) t_fail_uploads = count;
    else return VGI_ERR_INVALID;
    return VGI_OK;
}

int vgi_mlp_stats(vgi_ctx* c, vgi_mlp_status* out) {
    if (!c || !out) return VGI_ERR_INVALID;
    *out = vgi_mlp_status{};
    out->frames = c->mlp_frames;
    out->terminating = mlp_terminates(c) ? 1u : 0u;
    if (!c->mlp_image.ptr) return VGI_OK;
    uint32_t err[2] = {0, 0};
    VGI_CUDA(c, cudaMemcpyAsync(&out->steps, c->mlp_steps.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(&out->loss, c->mlp_grads.ptr + mlp_weight_count(), 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(err, c->mlp_error.ptr, 8, cudaMemcpyDeviceToHost, c->stream));
    if (c->mlp_queried) VGI_CUDA(c, cudaMemcpyAsync(&out->queries, c->mlp_query_count.ptr, 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    out->error = err[0] | err[1];
    if (c->mlp_timed) {
        VGI_CUDA(c, cudaEventElapsedTime(&out->query_ms, c->mlp_marks[0], c->mlp_marks[1]));
        VGI_CUDA(c, cudaEventElapsedTime(&out->train_ms, c->mlp_marks[2], c->mlp_marks[3]));
    }
    return VGI_OK;
}

int vgi_mlp_train(vgi_ctx* c, const float* features, const float* targets4, uint32_t n, float lr, float* loss) {
    if (!c || !n || !features || !targets4 || !(lr > 0.0f)) return VGI_ERR_INVALID;
    if (!c->mlp_image.ptr) return fail(c, VGI_ERR_STATE, "MLP weights are not set");
    VGI_CUDA(c, cudaSetDevice(c->device));
    DevBuf<float> in;
    DevBuf<float4> y;
    if (int e = mlp_upload_batch(c, features, targets4, n, in, y)) return e;
    VGI_CUDA(c, cudaMemsetAsync(c->mlp_error.ptr, 0, 4, c->stream));
    if (int e = mlp_train_step(c, in.ptr, y.ptr, n, lr)) return e;
    return mlp_read_status(c, loss);
}

int vgi_mlp_apply_gradients(vgi_ctx* c, const float* grads, float loss, float lr, int on_device) {
    if (!c || !grads || !(lr > 0.0f)) return VGI_ERR_INVALID;
    if (!c->mlp_image.ptr) return fail(c, VGI_ERR_STATE, "MLP weights are not set");
    VGI_CUDA(c, cudaSetDevice(c->device));
    // The gradient as one partial row (the loss after it), so the step is the
    // Adam kernel's own over one row: a gradient from vgi_mlp_gradients gives
    // the same step as vgi_mlp_train on that batch.
    const uint32_t count = mlp_weight_count();
    VGI_CUDA(c, cudaMemcpyAsync(c->mlp_partials.ptr, grads, (size_t)count * 4, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                c->stream));
    VGI_CUDA(c, cudaMemcpyAsync(c->mlp_partials.ptr + count, &loss, 4, cudaMemcpyHostToDevice, c->stream));
    launch_mlp_adam(c->mlp_master.ptr, c->mlp_adam.ptr, c->mlp_adam.ptr + count, c->mlp_partials.ptr, 1u, lr, 0.9f, 0.99f, 1e-8f,
                    c->mlp_steps.ptr, c->mlp_image.ptr, c->mlp_image_b.ptr, c->mlp_grads.ptr + count, c->stream);
    VGI_CUDA(c, cudaGetLastError());
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_read_events(vgi_ctx* c, uint32_t* words, uint64_t n_words) {
    if (!c || (n_words && !words) || n_words > c->n_events_read * 4) return VGI_ERR_INVALID;
    if (n_words) VGI_CUDA(c, cudaMemcpyAsync(words, c->events.ptr, n_words * 4, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_read_results(vgi_ctx* c, uint32_t first, uint32_t n, uint32_t* words24) {
    if (!c || !words24 || (uint64_t)first + n > c->n_slots) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaMemcpyAsync(words24, c->results.ptr + (size_t)first * 6, (size_t)n * 96, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_read_state(vgi_ctx* c, uint32_t first, uint32_t n, uint32_t* words36) {
    if (!c || !words36 || (uint64_t)first + n > c->n_slots) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaMemcpyAsync(words36, c->state.ptr + (size_t)first * 9, (size_t)n * 144, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_write_state(vgi_ctx* c, uint32_t first, uint32_t n, const uint32_t* words36) {
    if (!c || !words36 || (uint64_t)first + n > c->n_slots) return VGI_ERR_INVALID;
    std::vector<float4> rec(n);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* s = words36 + (size_t)i * 36;
        float r, g, b, w;
        std::memcpy(&r, s + 0, 4);
        std::memcpy(&g, s + 1, 4);
        std::memcpy(&b, s + 2, 4);
        std::memcpy(&w, s + 5, 4);
        rec[i] = make_float4(r, g, b, w);
    }
    VGI_CUDA(c, h2d(c->state.ptr + (size_t)first * 9, words36, (size_t)n * 144, c->stream));
    VGI_CUDA(c, h2d(c->cache.ptr + first, rec.data(), (size_t)n * 16, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

int vgi_read_slot_meta(vgi_ctx* c, uint32_t first, uint32_t n, uint32_t* words12) {
    if (!c || !words12 || (uint64_t)first + n > c->n_slots) return VGI_ERR_INVALID;
    VGI_CUDA(c, cudaMemcpyAsync(words12, c->slot_meta.ptr + (size_t)first * 3, (size_t)n * 48, cudaMemcpyDeviceToHost, c->stream));
    VGI_CUDA(c, cudaStreamSynchronize(c->stream));
    return VGI_OK;
}

void vgi_material_record(const float* diffuse3, const float* emission3, float* out16) {
    // VoxelGiMaterials::bounded (src/world.rs:166-173) then GpuMaterial
    // (src/gpu.rs:713-723): diffuse clamped to [0, 1], emission to [0, 1e12].
    auto bounded = [](float v, float hi) { return std::isfinite(v) ? std::min(std::max(v, 0.0f), hi) : 0.0f; };
    std::memset(out16, 0, 64);
    float emax = 0.0f;
    for (int k = 0; k < 3; ++k) {
        out16[k] = bounded(diffuse3[k], 1.0f);
        out16[8 + k] = bounded(emission3[k], 1.0e12f);
    }
    emax = std::max(out16[8], std::max(out16[9], out16[10]));
    out16[13] = emax;
}

void vgi_directional_light_record(const float* d, const float* radiance3, const float* custom3, float* out12) {
    // GpuLight for a directional source (src/gpu.rs:733-744): glam's
    // normalize_or_zero (v * (1 / length)), range -1.
    std::memset(out12, 0, 48);
    float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    float rcp = 1.0f / len;
    if (std::isfinite(rcp) && rcp > 0.0f) {
        out12[0] = d[0] * rcp;
        out12[1] = d[1] * rcp;
        out12[2] = d[2] * rcp;
    }
    out12[3] = -1.0f;
    for (int k = 0; k < 3; ++k) {
        out12[4 + k] = radiance3[k];
        out12[9 + k] = custom3 ? custom3[k] : 0.0f;
    }
}

// ---- batched frames ---------------------------------------------------------
}  // extern "C"

struct vgi_batch {
    std::vector<vgi_ctx*> ctxs;
    int device = 0;
    cudaStream_t stream = nullptr;           // batched traversals; the frame's start and end
    cudaEvent_t done = nullptr, fork = nullptr;
    std::vector<cudaEvent_t> ready, join;
    std::vector<cudaStream_t> side;          // one per scene: its own kernels
    DevBuf<uint8_t> args;                    // the traversal's argument table on the device
    std::vector<uint8_t> table;              // ... and the host copy it was made from
    DevBuf<uint32_t> head;                   // the batched traversal's shared queue head
    uint32_t blocks = 0, refill_min = 8;
    bool use_graph = false, graph_dirty = true;
    uint32_t graph_samples = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphNode_t> prepare_nodes, accumulate_nodes;
    // Scenes in the MLP cache mode: whether this frame's paths end at the
    // network, and the query launch's scene table (device and host copies).
    bool mlp = false, graph_mlp = false;
    DevBuf<MlpSceneQueries> mlp_table;
    std::vector<MlpSceneQueries> mlp_host;
    uint32_t mlp_ctas = 0;
    std::string error;
};

namespace {
int batch_fail(vgi_batch* b, int code, const std::string& what) {
    b->error = what;
    return code;
}
#define VGI_BCUDA(b, expr)                                                                               \
    do {                                                                                                 \
        cudaError_t err_ = (expr);                                                                       \
        if (err_ != cudaSuccess) return batch_fail(b, VGI_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(err_)); \
    } while (0)

void batch_drop_graph(vgi_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->prepare_nodes.clear();
    b->accumulate_nodes.clear();
    b->graph_dirty = true;
}

// Every context of a batch traces like vgi_frame in the wavefront layout
// with one transport for all.
int batch_check(vgi_batch* b) {
    const vgi_ctx* c0 = b->ctxs[0];
    for (vgi_ctx* c : b->ctxs) {
        if (int e = check_ready(c, true)) return batch_fail(b, e, std::string("scene not ready: ") + c->error);
        if (c->device != b->device) return batch_fail(b, VGI_ERR_INVALID, "batched scenes must share one device");
        if (c->layout != VGI_LAYOUT_WAVEFRONT) return batch_fail(b, VGI_ERR_STATE, "batched scenes trace in the wavefront layout");
        if (c->mlp_cache != c0->mlp_cache || mlp_terminates(c) != mlp_terminates(c0))
            return batch_fail(b, VGI_ERR_STATE, "batched scenes must all trace plainly or all end paths at their network, in the same phase");
        if (c->transport.bounces != c0->transport.bounces || transport_limited(c) != transport_limited(c0) ||
            (c->transport.budgeted != 0) != (c0->transport.budgeted != 0))
            return batch_fail(b, VGI_ERR_STATE, "batched scenes must share bounces, reach limit and step budget");
    }
    return VGI_OK;
}

// The scenes' buffers and trace arguments for `samples` paths a face, over
// the given tasks and results (null: each scene's own). Rebuilds and uploads
// the traversal's argument table when anything in it changed.
int batch_scenes(vgi_batch* b, uint32_t samples, bool scratch, std::vector<WaveScene>& scenes) {
    const uint32_t n = (uint32_t)b->ctxs.size();
    scenes.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        vgi_ctx* c = b->ctxs[i];
        const uint4* tasks = c->tasks.ptr;
        uint4* results = c->results.ptr;
        if (scratch) {
            VGI_BCUDA(b, c->scratch_tasks.reserve((size_t)c->n_slots * 2));
            VGI_BCUDA(b, c->scratch_results.reserve((size_t)c->n_slots * 6));
            tasks = c->scratch_tasks.ptr;
            results = c->scratch_results.ptr;
        }
        scenes[i].a = trace_args(c, tasks, results, c->n_slots, samples, true);
        if (wave_buffers(c, scenes[i].a, false, false, scenes[i].b) != VGI_OK) return batch_fail(b, VGI_ERR_CUDA, c->error);
        const size_t paths = (size_t)c->n_slots * samples;
        if (paths >= (1ull << 30)) return batch_fail(b, VGI_ERR_CAPACITY, "too many paths in a batched scene");
    }
    // A frame that ends paths at the network has one diffuse hit.
    b->mlp = mlp_terminates(b->ctxs[0]);
    const uint32_t hits = b->mlp ? 1u : b->ctxs[0]->transport.bounces;
    std::vector<uint8_t> table((size_t)wave_batch_stages(hits) * n * wave_args_bytes());
    wave_batch_args(scenes.data(), n, hits, table.data());
    if (b->mlp) {
        // The query launch's CTAs, shared out in proportion to the scenes'
        // paths (at least one each).
        size_t total = 0;
        for (uint32_t i = 0; i < n; ++i) total += (size_t)scenes[i].a.n_tasks * samples;
        const uint32_t budget = std::max<uint32_t>(b->ctxs[0]->mlp_ctas, n);
        std::vector<MlpSceneQueries> q(n);
        uint32_t first = 0;
        for (uint32_t i = 0; i < n; ++i) {
            vgi_ctx* c = b->ctxs[i];
            const size_t paths = (size_t)scenes[i].a.n_tasks * samples;
            const uint32_t ctas = std::max<uint32_t>(1u, (uint32_t)((double)budget * (double)paths / (double)std::max<size_t>(total, 1)));
            MlpSceneQueries e;
            std::memset(&e, 0, sizeof e);  // padding too: the table is compared bytewise
            e.queue = scenes[i].b.mlp_queue;
            e.counter = scenes[i].b.counters + 4;
            e.capacity = (uint32_t)paths;
            e.first_cta = first;
            e.ctas = ctas;
            e.enc = scenes[i].b.mlp_enc;
            e.out = scenes[i].b.state + (size_t)4 * paths;  // the pending-value field, as wave_run's query launch
            e.image = scenes[i].b.mlp_image;
            e.error = scenes[i].b.mlp_error;
            std::memcpy(&q[i], &e, sizeof e);
            first += ctas;
            c->mlp_queue_capacity = (uint32_t)paths;  // what the frame's training draws from
        }
        if (q.size() != b->mlp_host.size() || std::memcmp(q.data(), b->mlp_host.data(), q.size() * sizeof(MlpSceneQueries)) != 0) {
            batch_drop_graph(b);
            VGI_BCUDA(b, b->mlp_table.reserve(n));
            VGI_BCUDA(b, h2d(b->mlp_table.ptr, q.data(), n * sizeof(MlpSceneQueries), b->stream));
            VGI_BCUDA(b, cudaStreamSynchronize(b->stream));
            b->mlp_host = q;
        }
        b->mlp_ctas = first;
    }
    if (b->mlp != b->graph_mlp) batch_drop_graph(b);
    b->graph_mlp = b->mlp;
    if (table != b->table) {
        batch_drop_graph(b);
        VGI_BCUDA(b, b->args.reserve(table.size()));
        VGI_BCUDA(b, h2d(b->args.ptr, table.data(), table.size(), b->stream));
        VGI_BCUDA(b, cudaStreamSynchronize(b->stream));
        b->table.swap(table);
    }
    return VGI_OK;
}

void batch_trace(vgi_batch* b, const std::vector<WaveScene>& scenes, const AccumArgs* acc = nullptr, bool capture = false) {
    const vgi_ctx* c0 = b->ctxs[0];
    BatchStreams st{b->stream, b->side.data(), b->fork, b->join.data(), b->head.ptr, b->blocks, b->refill_min};
    if (b->mlp) {
        st.mlp_scenes = b->mlp_table.ptr;
        st.mlp_n = (uint32_t)scenes.size();
        st.mlp_ctas = b->mlp_ctas;
        st.mlp_wait = c0->mlp_wait;
    }
    if (capture) {
        b->prepare_nodes.assign(scenes.size(), nullptr);
        b->accumulate_nodes.assign(scenes.size(), nullptr);
    }
    launch_wave_batch(scenes.data(), (uint32_t)scenes.size(), b->args.ptr, b->mlp ? 1u : c0->transport.bounces, transport_limited(c0),
                      c0->transport.budgeted != 0, st, acc, capture ? b->prepare_nodes.data() : nullptr,
                      capture ? b->accumulate_nodes.data() : nullptr);
}

// Orders the batch stream after every scene's stream.
int batch_enter(vgi_batch* b) {
    for (size_t i = 0; i < b->ctxs.size(); ++i) {
        VGI_BCUDA(b, cudaEventRecord(b->ready[i], b->ctxs[i]->stream));
        VGI_BCUDA(b, cudaStreamWaitEvent(b->stream, b->ready[i], 0));
    }
    return VGI_OK;
}
// ... and every scene's stream after the batch's work.
int batch_leave(vgi_batch* b) {
    VGI_BCUDA(b, cudaEventRecord(b->done, b->stream));
    for (vgi_ctx* c : b->ctxs) VGI_BCUDA(b, cudaStreamWaitEvent(c->stream, b->done, 0));
    return VGI_OK;
}

cudaError_t set_node_args(cudaGraphExec_t exec, cudaGraphNode_t node, const AccumArgs& acc) {
    cudaKernelNodeParams p{};
    cudaError_t e = cudaGraphKernelNodeGetParams(node, &p);
    if (e != cudaSuccess) return e;
    AccumArgs copy = acc;
    void* args[] = {&copy};
    p.kernelParams = args;
    p.extra = nullptr;
    return cudaGraphExecKernelNodeSetParams(exec, node, &p);
}
}  // namespace

extern "C" {

int vgi_batch_create(vgi_ctx* const* ctxs, uint32_t n, vgi_batch** out) {
    if (!ctxs || !out || n == 0) return VGI_ERR_INVALID;
    if (n > kMaxBatchScenes) return VGI_ERR_CAPACITY;
    *out = nullptr;
    for (uint32_t i = 0; i < n; ++i)
        if (!ctxs[i]) return VGI_ERR_INVALID;
    auto* b = new vgi_batch();
    b->ctxs.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->device;
    b->blocks = ctxs[0]->traverse_blocks;
    b->refill_min = ctxs[0]->refill_min;
    b->ready.resize(n, nullptr);
    b->join.resize(n, nullptr);
    b->side.resize(n, nullptr);
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->ready[i], cudaEventDisableTiming);
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = b->head.reserve(1);
    if (e != cudaSuccess) {
        vgi_batch_destroy(b);
        return VGI_ERR_CUDA;
    }
    *out = b;
    return VGI_OK;
}

int vgi_batch_destroy(vgi_batch* b) {
    if (!b) return VGI_ERR_INVALID;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    b->args.release();
    b->head.release();
    for (cudaEvent_t e : b->ready)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : b->side)
        if (s) cudaStreamDestroy(s);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return VGI_OK;
}

const char* vgi_batch_last_error(const vgi_batch* b) { return b ? b->error.c_str() : "null batch"; }

int vgi_batch_set_graph(vgi_batch* b, int enable) {
    if (!b) return VGI_ERR_INVALID;
    batch_drop_graph(b);
    b->use_graph = enable != 0;
    return VGI_OK;
}

int vgi_batch_frame(vgi_batch* b, uint32_t samples, uint32_t clock_ms) {
    if (!b) return VGI_ERR_INVALID;
    if (samples == 0) return batch_fail(b, VGI_ERR_INVALID, "samples must be positive");
    VGI_BCUDA(b, cudaSetDevice(b->device));
    if (int e = batch_check(b)) return e;
    if (int e = batch_enter(b)) return e;
    std::vector<WaveScene> scenes;
    if (int e = batch_scenes(b, samples, false, scenes)) return e;
    const uint32_t n = (uint32_t)b->ctxs.size();
    std::vector<AccumArgs> acc(n);
    for (uint32_t i = 0; i < n; ++i) acc[i] = accum_args(b->ctxs[i], samples, clock_ms);
    if (b->use_graph && b->exec && !b->graph_dirty && b->graph_samples == samples) {
        for (uint32_t i = 0; i < n; ++i) {
            VGI_BCUDA(b, set_node_args(b->exec, b->prepare_nodes[i], acc[i]));
            VGI_BCUDA(b, set_node_args(b->exec, b->accumulate_nodes[i], acc[i]));
        }
        VGI_BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    } else {
        // Captured on the second frame with unchanged buffers; run directly
        // otherwise.
        const bool capture = b->use_graph && !b->graph_dirty && b->graph_samples == samples;
        if (capture) {
            batch_drop_graph(b);
            VGI_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        }
        batch_trace(b, scenes, acc.data(), capture);
        if (capture) {
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            bool found = e == cudaSuccess;
            for (uint32_t i = 0; i < n && found; ++i) found = b->prepare_nodes[i] && b->accumulate_nodes[i];
            if (!found) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                b->prepare_nodes.clear();
                b->accumulate_nodes.clear();
                return batch_fail(b, VGI_ERR_CUDA, "batched frame capture failed");
            }
            b->graph = g;
            VGI_BCUDA(b, cudaGraphInstantiate(&b->exec, g, 0));
            VGI_BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
            b->graph_dirty = false;
        } else if (b->use_graph) {
            b->graph_dirty = false;  // the next frame is captured
        }
        b->graph_samples = samples;
    }
    VGI_BCUDA(b, cudaGetLastError());
    for (vgi_ctx* c : b->ctxs) {
        c->batch_id = (c->batch_id + 1) & 0x0fffffffu;
        if (c->batch_id == 0) c->batch_id = 1;
    }
    if (int e = batch_leave(b)) return e;
    // Each scene's online training, on its own stream after the frame, as
    // vgi_frame runs it (the scenes' training overlaps on the GPU).
    for (vgi_ctx* c : b->ctxs) {
        if (!c->mlp_cache) continue;
        if (int e = mlp_frame_training(c)) return batch_fail(b, e, std::string("MLP training: ") + c->error);
        c->mlp_frames += 1;
    }
    return VGI_OK;
}

int vgi_batch_sync(vgi_batch* b) {
    if (!b) return VGI_ERR_INVALID;
    VGI_BCUDA(b, cudaStreamSynchronize(b->stream));
    return VGI_OK;
}

int vgi_batch_autotune(vgi_batch* b, uint32_t samples, uint32_t* refill_out, uint32_t* blocks_out, float* ms_out) {
    if (!b) return VGI_ERR_INVALID;
    if (samples == 0) return batch_fail(b, VGI_ERR_INVALID, "samples must be positive");
    VGI_BCUDA(b, cudaSetDevice(b->device));
    if (int e = batch_check(b)) return e;
    if (int e = batch_enter(b)) return e;
    // State-free traces of each scene's current tasks into scratch results.
    for (vgi_ctx* c : b->ctxs) {
        VGI_BCUDA(b, c->scratch_tasks.reserve((size_t)c->n_slots * 2));
        VGI_BCUDA(b, cudaMemcpyAsync(c->scratch_tasks.ptr, c->tasks.ptr, (size_t)c->n_slots * 32, cudaMemcpyDeviceToDevice, b->stream));
    }
    std::vector<WaveScene> scenes;
    if (int e = batch_scenes(b, samples, true, scenes)) return e;
    const uint32_t sms = b->ctxs[0]->traverse_blocks / wave_traverse_blocks_per_sm();
    const uint32_t refills[] = {4, 8, 12, 16};
    const uint32_t per_sm[] = {wave_traverse_blocks_per_sm(), wave_traverse_blocks_per_sm() > 2 ? 2u : 1u};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    VGI_BCUDA(b, cudaEventCreate(&e0));
    VGI_BCUDA(b, cudaEventCreate(&e1));
    float best = 1e30f;
    uint32_t best_refill = b->refill_min, best_blocks = b->blocks;
    for (uint32_t ps : per_sm) {
        for (uint32_t r : refills) {
            b->refill_min = r;
            b->blocks = sms * ps;
            float ms = 0.0f;
            for (int rep = 0; rep < 2; ++rep) {  // the first run warms caches
                cudaEventRecord(e0, b->stream);
                batch_trace(b, scenes);
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (ms < best) {
                best = ms;
                best_refill = r;
                best_blocks = b->blocks;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->refill_min = best_refill;
    b->blocks = best_blocks;
    batch_drop_graph(b);
    b->table.clear();  // the frame's table differs from the scratch one
    VGI_BCUDA(b, cudaGetLastError());
    if (refill_out) *refill_out = best_refill;
    if (blocks_out) *blocks_out = best_blocks;
    if (ms_out) *ms_out = best;
    return batch_leave(b);
}

}  // extern "C"
