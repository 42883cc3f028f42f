// Launch records shared by the host API and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vgi {

constexpr uint32_t kNoIndex = 0xffffffffu;
// Counter words of the counting variants, in vgi_counters order.
constexpr int kCounterWords = 15;

// Everything the face trace reads. Geometry and cache arrays are read-only
// for the kernel's lifetime and are loaded through the non-coherent path.
struct TraceArgs {
    // NAADF geometry (binding 1-3 of the reference's layout)
    const int4* directory;
    const uint4* headers;
    const uint32_t* cells;
    uint32_t dir_mask;
    int mn[3], mx[3];
    // model
    const float4* materials;   // 4 float4 per material (GpuMaterial)
    const uint4* emitters;     // GpuEmitter records then light-tree nodes
    const float4* node_aux;    // 2 records per light-tree node (see vgi_trace.cu)
    float emitter_count;       // params.extra.w
    float emitter_total;       // params.extra.z
    float max_distance;        // params.extra.y (768)
    float reach;               // params.transport.x
    float env[4];
    uint32_t light_count;      // counts.w
    const float4* lights;      // 3 float4 per light (GpuLight)
    // world cache
    const int32_t* region_grid;  // lookup_region's answer per region of [mn, mx], x fastest (null: probe the directory)
    const uint4* region_headers; // with region_grid: the header it names per region (kind 0: not found)
    const uint4* face_index;   // [0] = (mask, probes, 0, 0), entries from 1
    const float4* cache;       // per slot: mean rgb, count word (bits)
    // faces
    const uint4* tasks;        // 2 uint4 per task (FaceTask)
    uint4* results;            // 6 uint4 per task (FaceResult)
    uint32_t n_tasks;
    uint32_t samples;          // counts.y
    uint32_t path_steps;       // PATH_STEPS
    uint32_t lanes_log2;       // threads per face = 1 << lanes_log2
    unsigned long long* counters;  // 10 counters (counting variant only)
    // Per task, the light tree's left-child probabilities of the top
    // kTreeTopSlots nodes at the face's receiver point (null: none kept),
    // valid while the row's key equals the task's first word and the tree
    // generation (kTreeRowWords uint4 a task; see wave_begin_kernel).
    uint4* tree_rows;
    uint32_t tree_generation;
};

// The cached top of the light tree: heap slots 0..62 (depths 0-5), in a row
// of a key (the task's first word), the generation, and 64 floats.
constexpr uint32_t kTreeTopSlots = 63;
constexpr uint32_t kTreeRowWords = 18;

struct AccumArgs {
    uint4* state;         // 9 uint4 per slot
    uint4* slot_meta;     // 3 uint4 per slot
    uint4* checkpoint;    // 3 uint4 per slot
    uint4* outputs;       // 6 uint4 per task
    uint4* tasks;         // 2 uint4 per task
    float4* cache;        // per slot gather record
    const uint32_t* slots;  // task -> slot (null: identity)
    uint32_t n;
    uint32_t controls[36];
    uint4* picks;         // GPU picks' records (slot, revision, count, incarnation) per task, or null
};

// The GPU selection of a scheduled frame (vgi_accumulate.cu): selection
// scratch words and the per-slot keys.
constexpr uint32_t kSelectionWords = 1038;
void launch_select(const AccumArgs& a, uint32_t n_slots, uint32_t* keys, uint32_t* selection, uint32_t* pick_slots, cudaStream_t s);
void launch_mark_changed(const AccumArgs& a, cudaStream_t s);

// Device buffers of the wavefront layout (vgi_wave.cuh) for P = tasks x
// samples paths and S = P * (2 + lights) + tasks * lights ray slots.
// Maps voxel coordinates to the MLP's [0, 1] position inputs: (x - lo) * inv
// per axis.
struct MlpEncoding {
    float lo[3];
    float inv[3];
};

// One scene's network queries in a batched frame's single query launch
// (launch_mlp_scene_queries): its hit queue (2 float4 a query) and count, the
// count's bound, the grid's CTAs it owns, its encoding, the path-state field
// the predictions go to, its network image and its error word.
struct MlpSceneQueries {
    const float4* queue;
    const uint32_t* counter;
    uint32_t capacity;
    uint32_t first_cta, ctas;
    MlpEncoding enc;
    float4* out;
    const uint8_t* image;
    uint32_t* error;
};
void launch_mlp_scene_queries(const MlpSceneQueries* scenes, uint32_t n_scenes, uint32_t ctas, cudaStream_t s, uint32_t wait_polls);

// The MLP cache's tensor-core kernels bound every mbarrier wait to
// `wait_polls` polls: kMlpWaitPolls unless a caller lowers it
// (vgi_mlp_set_wait_limit); a wait that runs out sets the error word.
constexpr uint32_t kMlpWaitPolls = 1u << 22;

// float4 fields of path state per path in the wavefront layout.
constexpr uint32_t kWavePathFields = 6;

struct WaveBuffers {
    float4* state;            // kWavePathFields * P path-state words
    float4* ray;              // 2 * S
    uint32_t* status;         // S
    uint4* hit;               // 6 * P (full results of slots 0 and 1)
    uint32_t* queue[2];       // S each
    uint32_t* scatter;        // P: uncached hits awaiting NEE and continuation
    uint32_t* counters;       // queue counts [0], [1]; traversal head [2]; scatter count [3]
    uint32_t traverse_blocks; // persistent traversal grid
    uint32_t refill_min;      // idle lanes that trigger a refill
    cudaEvent_t* traverse_marks;  // optional: start/end events of up to 4 traversal launches
    // MLP termination (null image: off). Uncached first hits are queued
    // (2 float4 each, counter at counters[4]) and take the network's
    // prediction in place of the continuation.
    const uint8_t* mlp_image;
    float4* mlp_queue;        // 2 * P
    uint32_t* mlp_error;
    uint32_t mlp_ctas;
    uint32_t mlp_wait = kMlpWaitPolls;
    MlpEncoding mlp_enc;
    cudaEvent_t* mlp_marks;   // optional: start/end events of the query launch
};

// One scene of a batched frame: its wavefront buffers and trace arguments.
struct WaveScene {
    WaveBuffers b;
    TraceArgs a;
};
// Batched frames (vgi_wave.cuh): the traversal of every stage runs once over
// the rays of all scenes. The argument table holds wave_batch_stages(hits)
// x n records of wave_args_bytes() each, built on the host by
// wave_batch_args and copied to the device once for a set of buffers.
constexpr uint32_t kMaxBatchScenes = 256;
uint32_t wave_batch_stages(uint32_t hits);
size_t wave_args_bytes();
void wave_batch_args(const WaveScene* scenes, uint32_t n, uint32_t hits, void* out);
// The streams of a batched frame: the batched traversals run on `main`,
// each scene's own kernels on side[i]; fork and join[i] order them.
struct BatchStreams {
    cudaStream_t main;
    const cudaStream_t* side;
    cudaEvent_t fork;
    const cudaEvent_t* join;
    uint32_t* head;            // the batched traversal's shared queue head
    uint32_t blocks, refill_min;
    // Scenes that end uncached first hits with their network: the device
    // table of their queries, its length and the query launch's CTAs (null
    // table: plain frames).
    const MlpSceneQueries* mlp_scenes = nullptr;
    uint32_t mlp_n = 0, mlp_ctas = 0, mlp_wait = kMlpWaitPolls;
};
// acc (null: trace only) gives each scene's prepare and accumulate; when
// capturing, their graph nodes are stored in prepare_nodes / accumulate_nodes.
void launch_wave_batch(const WaveScene* scenes, uint32_t n, const void* device_args, uint32_t hits, bool limited, bool budgeted,
                       const BatchStreams& st, const AccumArgs* acc, cudaGraphNode_t* prepare_nodes, cudaGraphNode_t* accumulate_nodes);

// The view tier's buffers and controls (vgi_view.cuh) for n receivers.
// Far tier (vgi_trace.cu, voxel_view_pixels.wgsl): the view uniforms the
// classify and trace passes read, with the camera in place of the clip
// matrices. Cells are 3 uint4 (PixelHistory: mean rgb + count, surface xyz +
// face word, sequence); the output is a 4-uint4 header then one uint4 per
// cell; the queue is a count then cell indices; 8 statistics words.
struct FarView {
    float cam[10];            // eye xyz, forward xyz (unit), up xyz, tan(half vertical fov)
    float prev[10];           // the previous frame's camera
    uint32_t width, height;   // viewport (origin 0, 0)
    uint32_t grid[4];         // cells x, y, pixels per cell side, enabled | measure << 1
    float tune[4];            // threshold px, max history, trace rate, previous stamp (bits; all ones: none)
    float axis[4];            // forward xyz, pixels per unit at depth 1
    int32_t interest_min[4];  // regions, inclusive; w: bounded
    int32_t interest_max[4];
    uint32_t frame;           // this frame's number (history.z)
    uint32_t custom;          // some light has custom visible RGB (transport.y)
    const uint4* receivers;   // view receivers for the handoff (2 uint4 each), may be null
    const uint4* estimates;   // their estimates (4 uint4 each)
    const uint32_t* receiver_hash;  // receiver + 1 per slot, 0 empty
    uint32_t hash_mask;
    uint32_t n_receivers;
};
// Sun-flip reports after a view queue of 12 + 2n words: a count and 3
// zero words, kMaxSunFlips records (voxel xyz, flux bits), then the overflow
// (biased min xyz as max of bias - v, max xyz biased, flux x 64 summed).
constexpr uint32_t kMaxSunFlips = 2048u, kSunFlipWords = 4u + kMaxSunFlips * 4u + 7u;
struct ViewArgs {
    TraceArgs t;
    uint4* receivers;      // 2 per receiver: surface xyz, face | voxel xyz, sequence
    uint4* paths;          // 8 per receiver (ViewPath)
    uint4* conts;          // 8 per receiver (ViewContinuation)
    uint4* estimates;      // 4 per receiver (ViewEstimate)
    uint32_t* queue;       // 12 counters, owners (n), cursor words (n)
    uint4* shared_state;   // the world cache's slots (9 uint4 each)
    uint4* shared_meta;    // 3 uint4 per slot
    float4* shared_cache;  // the slots' gather records
    const uint4* events;
    uint32_t n_events, reach;
    uint32_t n;
    uint32_t range[4];     // ViewWave.range: first owner, invocations, hits per visit, finite depth
    uint32_t ticket[4];
    uint32_t view_first, shared, clock;
    float physical;        // measured retention c
    uint32_t hits;         // DIFFUSE_HITS for trace_view_paths
    // The far tier's handoff (null: off): a new, unmeasured receiver starts
    // from the far cell at its centre; far_stats[5] counts them.
    const uint4* far_cells;
    uint32_t* far_stats;
    FarView far;
    // The topology prior (bootstrap_face; 0: off): donors are the receivers
    // of the owner hash, read from the estimates as they were before this
    // frame's seeding, and the world cache's slots.
    uint32_t topology;
    // Sun corners (reproject_paths): this view frame's number, whether the
    // receivers were in the last view frame, and the directional lights.
    uint32_t frame, has_previous, n_directional;
    const uint32_t* receiver_hash;
    uint32_t hash_mask;
    const uint4* prev_estimates;
};

void launch_trace(const TraceArgs& a, uint32_t hits, bool limited, bool budgeted, bool count, cudaStream_t stream);
void launch_view_frame(const ViewArgs& v, bool limited, bool budgeted, cudaStream_t stream);
void launch_view_trace_paths(const ViewArgs& v, uint32_t samples, uint4* out, bool limited, bool budgeted, cudaStream_t stream);
void launch_wave(const WaveBuffers& b, const TraceArgs& a, uint32_t hits, bool limited, bool budgeted, bool count, cudaStream_t stream);
uint32_t wave_traverse_blocks_per_sm();
void launch_reference64(const TraceArgs& a, const double* cdf, const int4* emitters, uint32_t n_emitters, double total,
                        const uint4* tasks, uint32_t n_tasks, uint32_t samples, uint64_t seed, double* sum, double* second,
                        uint32_t* known, cudaStream_t s);
// The per-frame kernels whose arguments a captured frame graph updates.
const void* prepare_kernel_address();
const void* accumulate_kernel_address();
// Change footprints (vgi_trace.cu): fp = a count record, then 3 records per
// task; sums = 8 words per task (min xyz, max xyz, flux x 64, unused).
void launch_footprints(const TraceArgs& a, const int4* fp, uint32_t n_tasks, uint32_t threads, uint32_t n_directional, uint32_t* sums,
                       uint4* events, cudaStream_t s);
// Headless discovery (vgi_trace.cu): cam = eye xyz, forward xyz, up xyz,
// tan(half vertical fov); set = 64-bit keys, all ones when empty.
void launch_discover(const TraceArgs& a, const float* cam, uint32_t w, uint32_t h, uint4* pixels, unsigned long long* set, uint32_t set_mask,
                     int4* faces, uint32_t* count, uint32_t capacity, uint32_t* overflow, cudaStream_t s);
constexpr uint32_t kFarOwned = 0, kFarTraced = 1, kFarHistory = 2, kFarReprojected = 3, kFarSeeded = 4;
void launch_far(const TraceArgs& a, const FarView& f, const uint4* previous, uint4* current, uint4* output, uint32_t* queue, uint32_t* stats,
                bool limited, cudaStream_t s);
void launch_receiver_hash(const uint4* receivers, uint32_t n, uint32_t* hash, uint32_t mask, cudaStream_t s);
// Reconstruction and presentation of the view receivers (vgi_trace.cu,
// voxel_view_runtime.wgsl:380-521 and voxel_gi_presentation.wesl:350-412).
struct ViewDisplay {
    const uint4* receivers;       // 2 uint4 each
    uint4* estimates;             // 4 uint4 each (shown is written)
    const uint4* conts;           // 8 uint4 each
    const uint32_t* tile_of;      // per receiver: screen tile, all ones: none
    const uint32_t* tile_start;   // CSR over tiles: receivers of tile t are items[start[t] .. start[t + 1])
    const uint32_t* tile_items;
    uint32_t tiles_x, tiles_y;
    const uint32_t* receiver_hash;  // receiver + 1 per slot
    uint32_t hash_mask;
    uint32_t n;
    float display[3];             // evidence goal, spatial strength, temporal blend
    uint32_t custom;              // add custom direct RGB when publishing
    uint4* published;             // FarPixel per receiver: 3 uint4
    uint32_t* stats;              // history, max history, uncovered, displayed, paused
};
void launch_reconstruct(const TraceArgs& a, const ViewDisplay& d, bool limited, bool budgeted, cudaStream_t s);
void launch_present(const TraceArgs& a, const ViewDisplay& d, const float* cam, uint32_t w, uint32_t h, bool corners, float4* image,
                    cudaStream_t s);
// MLP radiance cache (vgi_mlp.cu).
cudaError_t mlp_set_attributes();
void launch_mlp_queries(const float4* queue, const uint32_t* count, uint32_t capacity, const uint8_t* image, const MlpEncoding& enc,
                        float4* out, uint32_t* error, uint32_t ctas, cudaStream_t s, uint32_t wait_polls = kMlpWaitPolls);
void launch_mlp_encode_training(const uint4* slot_meta, const uint4* results, const float4* materials, uint32_t n_slots,
                                const uint32_t* step, uint32_t batch, const MlpEncoding& enc, float* features, float4* targets,
                                cudaStream_t s);
void launch_mlp_query_tasks(const float4* queue, const uint32_t* count, uint32_t capacity, const uint32_t* step, uint32_t n,
                            uint32_t samples, const MlpEncoding& enc, uint4* tasks, float* features, cudaStream_t s);
void launch_mlp_query_targets(const uint4* results, const uint4* tasks, uint32_t n, float4* targets, cudaStream_t s);
void launch_mlp_encode_faces(const uint4* meta, uint32_t n, const float4* materials, const MlpEncoding& enc, float* features,
                             cudaStream_t s);
void launch_mlp_pack(const float* master, uint8_t* image, cudaStream_t s);
cudaError_t launch_mlp_forward(const float* features, const uint8_t* image, float4* outputs, uint32_t n, uint32_t* error, uint32_t ctas,
                               cudaStream_t s, uint32_t wait_polls = kMlpWaitPolls);
void launch_mlp_pack_backward(const float* master, uint8_t* image, cudaStream_t s);
// Training: train writes one partial row (gradient sums, loss) per CTA,
// mlp_train_parts(batch, ctas) rows; reduce sums them into grads and the
// loss; adam sums them, steps the FP32 masters and repacks both images.
uint32_t mlp_train_parts(uint32_t batch, uint32_t ctas);
uint32_t mlp_partial_floats();
cudaError_t launch_mlp_train(const float* features, const float4* targets, uint32_t batch, const uint8_t* image_f, const uint8_t* image_b,
                             float* partials, uint32_t* error, uint32_t ctas, cudaStream_t s, uint32_t wait_polls = kMlpWaitPolls);
void launch_mlp_reduce(const float* partials, uint32_t parts, float* grads, float* loss, cudaStream_t s);
void launch_mlp_adam(float* master, float* m, float* v, const float* partials, uint32_t parts, float lr, float beta1, float beta2, float eps,
                     uint32_t* steps, uint8_t* image_f, uint8_t* image_b, float* loss, cudaStream_t s);
uint32_t mlp_weight_count();
uint32_t mlp_image_bytes();
void launch_seed_incarnations(uint4* state, uint32_t n, cudaStream_t s);
void launch_measure_edits(const uint4* state, const uint4* slot_meta, const uint4* index, const float2* material_light,
                          const uint4* measures, uint32_t n_entries, uint32_t n_positions, uint32_t* measure_max, uint4* events,
                          cudaStream_t s);
void launch_node_aux(const uint4* emitters, uint32_t first_node, uint32_t nodes, float4* aux, cudaStream_t stream);
cudaError_t init_trace_constants();
void launch_prepare(const AccumArgs& a, cudaStream_t stream);
void launch_accumulate(const AccumArgs& a, cudaStream_t stream);
void launch_apply_events(const AccumArgs& a, const uint4* events, uint32_t n_slots, cudaStream_t stream);

}  // namespace vgi
