/*
 * vgi.h -- C ABI of the B200-native voxel diffuse-GI path (libvgi.so).
 *
 * This is the drop-in boundary for bevy_voxel_gi's per-frame GPU transport:
 * NAADF geometry upload and edits, distance-skip DDA traversal, the
 * visible-face cosine-hemisphere trace into the face cache, the world-cache
 * gather and the temporal accumulation with proportional edit discount.
 * Each entry point names the reference interface it replaces (paths within
 * nathanaelneveux/global-illumination, crates/bevy_voxel_gi/).
 *
 * Conventions
 *  - Every function returns an int status: VGI_OK (0), > 0 recoverable,
 *    < 0 fatal for the context. vgi_last_error() describes the last failure.
 *  - A context is owned by one thread at a time (the reference's single trace
 *    worker, src/dispatch.rs:167-275); it is not thread-safe.
 *  - Host buffers passed in are copied before the call returns. Device
 *    buffers belong to the library. Work is enqueued on the context's CUDA
 *    stream; read-back calls synchronise that stream.
 *  - Word layouts are the reference's GPU records (little-endian u32/f32):
 *    GpuMaterial 16 floats, GpuLight 12 floats, FaceTask 8 words,
 *    FaceResult 24 words, resident state 36 words (src/gpu.rs:118-184,
 *    shaders/voxel_trace.wgsl:5-20, shaders/voxel_accumulate.wgsl:1-3).
 */
#ifndef VGI_H
#define VGI_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGI_OK 0
#define VGI_UNAVAILABLE 1       /* no usable CUDA device: transport idles (src/lib.rs:355-357) */
#define VGI_ERR_INVALID (-1)    /* bad argument or size */
#define VGI_ERR_CUDA (-2)       /* a CUDA call failed */
#define VGI_ERR_STATE (-3)      /* call out of order (e.g. frame before geometry) */
#define VGI_ERR_CAPACITY (-4)   /* a size limit was exceeded */

typedef struct vgi_ctx vgi_ctx;

typedef struct {
    int32_t device;   /* CUDA ordinal */
    uint32_t flags;   /* reserved, 0 */
} vgi_config;

/* Transport and accumulation settings (src/settings.rs:393-428 TransportSettings,
 * src/work.rs:11-47 TraceWork history fields, shader override constants
 * shaders/voxel_path.wgsl:4-14 and shaders/voxel_trace.wgsl:3). */
typedef struct {
    float reach;              /* diffuse reach, clamped to [1, 768]; < 768 selects LIMITED_REACH */
    uint32_t bounces;         /* DIFFUSE_HITS, clamped to [1, 3] */
    uint32_t path_steps;      /* PATH_STEPS (default 2048) */
    uint32_t budgeted;        /* BUDGETED_RAYS (0/1) */
    uint32_t history_limit;   /* 0 = 65536 */
    float recency;            /* >= 1; other values select 1 */
    float measured_retention; /* c of the measured discount; 0 = distance curve */
    float response_seconds;   /* display response time constant */
    uint32_t lanes;           /* threads per face (1,2,4,8,16,32); 0 = automatic */
    uint32_t transport_revision;
    float stable_error;
    uint32_t stable_samples;
} vgi_transport;

/* One face-cache slot: the exposed face (voxel, face 0..5 in +X,-X,+Y,-Y,+Z,-Z
 * order) and its voxel's material (slot identity, shaders/voxel_accumulate.wgsl:37-42). */
typedef struct {
    int32_t voxel[3];
    uint32_t face;
    uint32_t material;
} vgi_face;

/* Per-frame work counters (filled by the counting pass, vgi_census). */
typedef struct {
    uint64_t rays;        /* trace_domain_limited calls */
    uint64_t paths;       /* receiver samples */
    uint64_t steps;       /* DDA iterations, including geometry_ahead */
    uint64_t bytes;       /* algorithmic bytes of the trace */
    uint64_t unknown;     /* paths that reached unloaded space */
    uint64_t cache_hits;  /* paths ended by the world-cache gather */
    uint64_t status[4];   /* rays by status: escaped, hit, unknown, reach */
    uint64_t traverse_bytes; /* the traversal's share of `bytes`: directory,
                                header, brick and cell words */
    /* Lane use of the wavefront traversal: passes of its loop made by warps
     * with a ray in flight, and the rays in flight summed over those passes,
     * while rays remained queued [0] and after the queue ran out [1]. Zero in
     * the single-kernel layout. */
    uint64_t warp_passes[2];
    uint64_t lane_passes[2];
} vgi_counters;

/* ---- lifecycle: GpuTracer::new / drop (src/gpu.rs:448-595) ---------------- */
int vgi_create(const vgi_config* config, vgi_ctx** out);
int vgi_destroy(vgi_ctx* ctx);
const char* vgi_last_error(const vgi_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work. */
int vgi_stream(vgi_ctx* ctx, void** stream);
int vgi_sync(vgi_ctx* ctx);

/* ---- geometry: NaadfRegion::build + PackedScene::update + synchronize_geometry
 * (src/world.rs:243-384, src/gpu_scene.rs:72-309, src/gpu/geometry.rs:19-124).
 * `coords` holds 3 region coordinates per region (16^3 voxels each), `voxels`
 * 4096 u16 per region (x fastest; 0..255 solid material, 256 air),
 * `strides` the optional per-region stride log2 (header bits 28-30). The GPU
 * classifies regions, builds brick and voxel AADFs and packs the cells; the
 * host runtime grows the top-level field and the directory. */
int vgi_upload_regions(vgi_ctx* ctx, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides);
/* Parity path: arrays exactly as PackedScene holds them (directory 4 ints per
 * slot, headers 4 words per region, cells) and region bounds min xyz, max xyz. */
int vgi_upload_packed(vgi_ctx* ctx, const int32_t* directory, uint64_t slots, const uint32_t* headers, uint32_t n_headers,
                      const uint32_t* cells, uint64_t n_cells, const int32_t* bounds6);
/* One SceneDelta applied to geometry from vgi_upload_packed, as
 * GpuTracer::synchronize_geometry stages it (src/gpu/geometry.rs:19-124;
 * SceneDelta, src/gpu_scene.rs:49-60). `slots`, `n_headers` and `n_cells` are
 * the arrays' new lengths and `bounds6` the new region bounds. Each range is a
 * (start, count) pair of u64 element indices; each data array holds its
 * ranges' elements back to back (directory 4 ints per slot, headers 4 words
 * per region, cells one word). directory_rebuilt != 0: `dir_data` is the whole
 * new directory (`slots` entries) and dir_ranges is ignored; a directory of
 * another capacity must come this way. An array that grows keeps its contents
 * on the device (its new tail starts at zero); only the ranges cross the bus,
 * all on the context's stream as one transaction, complete when the call
 * returns. The patched arrays are checked on the host copy first, as
 * vgi_upload_packed checks whole arrays: a refused delta (VGI_ERR_INVALID)
 * changes nothing. VGI_ERR_STATE without packed geometry. */
int vgi_patch_packed(vgi_ctx* ctx, uint64_t slots, uint32_t n_headers, uint64_t n_cells, const int32_t* bounds6, int directory_rebuilt,
                     const uint64_t* dir_ranges, uint32_t n_dir_ranges, const int32_t* dir_data, const uint64_t* header_ranges,
                     uint32_t n_header_ranges, const uint32_t* header_data, const uint64_t* cell_ranges, uint32_t n_cell_ranges,
                     const uint32_t* cell_data);
/* Page streaming on the GPU geometry: VoxelGiInput::page_loaded and
 * page_changed (vgi_load_regions) and page_unloaded (vgi_unload_regions),
 * src/input.rs:54-70, applied as TransportScene::with_page_contents
 * (src/world.rs:982-1046) with region-sized pages and PackedScene::update
 * (src/gpu_scene.rs:72-409). Regions keep the vgi_upload_regions layout; a
 * loaded coordinate already resident is replaced, an unloaded one that is
 * not resident is ignored. Only the loaded regions are packed on the GPU;
 * the directory changes in place (linear-probing insert, backward-shift
 * delete; rebuilt when its capacity changes or a probe chain would reach
 * 32); the top-level field is updated incrementally over the touched
 * regions. Every world-cache slot stays as it is. A load on a context
 * without geometry starts from an empty scene. Refused inputs (duplicate
 * coordinates, voxels above 256) change nothing; another failure leaves no
 * geometry until the next successful upload or load. Not for geometry from
 * vgi_upload_packed (VGI_ERR_STATE). Synchronous. */
int vgi_load_regions(vgi_ctx* ctx, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides);
int vgi_unload_regions(vgi_ctx* ctx, const int32_t* coords, uint32_t n);
/* One frame's page events as one scene change, as with_page_contents takes
 * its changed and removed pages together (src/world.rs:982-1046): `removed`
 * (3 ints per region) are unloaded, then `coords`/`voxels` loaded, and the
 * top-level field is updated once over every touched region. A loaded region
 * equal to the resident one (same voxels and stride) is not touched, even if
 * the same call unloads it. The top-level field is an order-dependent fixed
 * point, so one call here and a vgi_unload_regions then vgi_load_regions pair
 * can leave different (equally valid) extents. */
int vgi_update_regions(vgi_ctx* ctx, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides,
                       const int32_t* removed, uint32_t n_removed);
/* VoxelGiInput::edit_voxel batch (src/input.rs:90-93): 4 ints per edit
 * (x, y, z, value). Voxels outside uploaded regions are ignored. The edited
 * regions are repacked on the GPU and the top-level field is updated
 * incrementally (TransportScene::with_page_contents, src/world.rs:982-1046). */
int vgi_edit_voxels(vgi_ctx* ctx, const int32_t* edits, uint32_t n);
/* sizes: directory slots, headers, cells; bounds: min xyz, max xyz. */
int vgi_geometry_info(vgi_ctx* ctx, uint64_t* sizes3, int32_t* bounds6);
int vgi_read_geometry(vgi_ctx* ctx, int32_t* directory, uint32_t* headers, uint32_t* cells);

/* ---- model: GpuTracer's material/light/emitter uploads (src/gpu.rs:680-800) --- */
int vgi_set_materials(vgi_ctx* ctx, const float* materials /* 256 x 16 */);
/* `lights`: n GpuLight records, directional ones first. */
int vgi_set_lights(vgi_ctx* ctx, const float* lights /* n x 12 */, uint32_t n, uint32_t n_directional);
int vgi_set_environment(vgi_ctx* ctx, const float* rgb3);
/* Emitter buffer as the shader reads it (GpuEmitter records then light-tree words). */
int vgi_set_emitters(vgi_ctx* ctx, const uint32_t* words, uint64_t n_words, uint32_t n_faces, float total_weight);
/* EmissionDistribution::build (src/emission.rs:91-165) from the uploaded
 * regions and the current materials, done by the host runtime. */
int vgi_build_emitters(vgi_ctx* ctx);

/* ---- transport settings: select_quality_pipeline (src/gpu.rs:1172-1229) --- */
int vgi_set_transport(vgi_ctx* ctx, const vgi_transport* transport);

/* ---- face cache: resident slots and the face index (src/gpu/resident.rs,
 * src/gpu/face_index.rs). Slots 0..n-1 start empty (sequence 0). */
int vgi_set_faces(vgi_ctx* ctx, const vgi_face* faces, uint32_t n);

/* One frame over every slot: prepare (begin_trace), mark_changed, the face
 * trace with cache gather, then accumulate (submit_compact's resident batch,
 * src/gpu.rs:647-1022). `clock_ms` is the accumulation clock. Enqueued only. */
int vgi_frame(vgi_ctx* ctx, uint32_t samples, uint32_t clock_ms);
/* Layout of the face trace. Both layouts compute bit-identical results.
 * VGI_LAYOUT_WAVEFRONT (default): paths advance in stages whose rays a
 *   persistent traversal kernel runs from a queue.
 * VGI_LAYOUT_SINGLE_KERNEL: one thread per (face, lane) runs whole paths, the
 *   reference's trace_faces_parallel layout (shaders/voxel_trace.wgsl:70-92).
 * `refill_min` (1..32, default 8) is how many idle lanes make a traversal
 * warp take new rays from the queue. */
#define VGI_LAYOUT_WAVEFRONT 0u
#define VGI_LAYOUT_SINGLE_KERNEL 1u
int vgi_set_layout(vgi_ctx* ctx, uint32_t layout, uint32_t refill_min);
/* Autotuner (no counterpart in the reference): times a trace of the current
 * face set at `samples` (tasks as the next frame would trace them, results
 * discarded, no slot changes) for the wavefront layout with refill_min
 * 4, 6, 8, 12 and 16 and for the single-kernel layout, keeps the fastest as
 * the context's layout and reports it. Synchronous. */
int vgi_autotune(vgi_ctx* ctx, uint32_t samples, uint32_t* layout, uint32_t* refill_min, float* trace_ms);
/* Device timing of vgi_frame (the reference's timestamp query pairs,
 * src/gpu.rs:488-500): with timing enabled each frame records CUDA events on
 * the context's stream around prepare, trace and accumulate, and around each
 * traversal launch of the wavefront layout. vgi_frame_times returns the last
 * frame's prepare, trace and accumulate durations and the summed traversal
 * time (0 for the single-kernel layout), in ms; it synchronises the stream. */
int vgi_set_timing(vgi_ctx* ctx, int enable);
/* Frame graphs (no counterpart in the reference, which records wgpu command
 * buffers per batch): with graphs enabled and timing off, the wavefront
 * layout's frame (prepare, the traversal and stage kernels, accumulate) is
 * captured into a CUDA graph on the second frame after any change and
 * replayed afterwards, with each frame's clock and batch id patched into the
 * captured prepare and accumulate nodes. Every setter, and any growth of
 * the trace buffers, drops the graph. Results equal direct launches. */
int vgi_set_graph(vgi_ctx* ctx, int enable);
int vgi_frame_times(vgi_ctx* ctx, float* ms4);
/* The same frame through host buffers (submit_compact + complete_readback):
 * 8-word tasks in (one per slot, in slot order; their sequence words are
 * replaced by the slot's), 24-word results out. Synchronous. */
int vgi_trace_batch(vgi_ctx* ctx, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t clock_ms, uint32_t* results);
/* vgi_trace_batch without the wait: the tasks are copied in and the results
 * out on the context's copy streams through device staging buffers, so a
 * batch's copies overlap the frames before and after it, like the crate's
 * submit_compact / complete_readback with batches in flight (gpu.rs:647-1170).
 * Returns at once with a ticket; vgi_complete_batch(ticket) waits until
 * `results` holds the batch's FaceResults. The host buffers (pinned memory,
 * for copies that overlap) must stay valid and unchanged until then. Two
 * batches may be in flight: submitting a third waits, on the device, for
 * the first's copies. Frames run in submission order on the context's
 * stream; other calls on the context order after the submitted frames. */
int vgi_submit_batch(vgi_ctx* ctx, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t clock_ms, uint32_t* results,
                     uint64_t* ticket);
int vgi_complete_batch(vgi_ctx* ctx, uint64_t ticket);
/* A counting trace of the next frame's work (no state change): rays, paths,
 * steps and algorithmic bytes. Synchronous. */
int vgi_census(vgi_ctx* ctx, uint32_t samples, vgi_counters* counters);
/* Trace explicit tasks against the current cache without accumulating
 * (trace_faces_parallel alone). Synchronous; counters may be null. */
int vgi_trace_tasks(vgi_ctx* ctx, const uint32_t* tasks, uint32_t n, uint32_t samples, uint32_t* results, vgi_counters* counters);

/* Retention events in the encode_events layout (src/gpu/resident.rs:1326-1414):
 * n_events headers of three uint4, then bound records of two uint4.
 * Applied by apply_events to every live slot (shaders/voxel_accumulate.wgsl:295-332). */
int vgi_apply_events(vgi_ctx* ctx, const uint32_t* words, uint32_t n_events, uint64_t n_words);
/* The same with measured edits (the resident batch's measure_edits and
 * finish_edits passes before apply_events, src/gpu/resident.rs:1004-1050;
 * shaders/voxel_accumulate.wgsl:375-425). `measures` holds 12 words per
 * measured edit bound (encode_events' measure records): (bound record index,
 * first scan position, positions, changed voxels), (scan min xyz, own flux
 * bits), (scan size xyz, 0); entries tile the positions in order. Each such
 * bound's flux becomes its own flux plus twice the changed voxels times the
 * brightest outgoing luminance of the traced faces in its scan box, and its
 * kind a measured edit (3), or unknown (0) when no traced face was seen.
 * Needs the material table. The rewritten words stay readable through
 * vgi_read_events until the next call. */
int vgi_apply_events_measured(vgi_ctx* ctx, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                              uint32_t n_entries);
/* Change footprints (trace_footprints, finish_footprints, shaders/voxel_trace.wgsl:
 * 94-202; planned by plan_footprints / encode_footprints, src/gpu/resident.rs:
 * 1218-1325): before the measured edits and retention read the event list,
 * sunlight tubes through each changed box, along each directional light whose
 * sun side is clear, find where the box's shadow lands; that landing box
 * and its reflected power (x 64, rounded) become the task's reserved Light
 * event (its header union and its one bound, kind 4). A task whose tubes
 * land nowhere keeps its empty bound. footprints: (1 + 3 n) records of 4
 * int32 words, encode_footprints' layout: the count, then per task (box min,
 * header record) (box max, bound record) (first thread, grid, 0, 0), with
 * grid^2 threads per task tiling the threads in order. Otherwise as
 * vgi_apply_events_measured; vgi_read_events returns the filled events. */
int vgi_apply_events_footprints(vgi_ctx* ctx, const uint32_t* words, uint32_t n_events, uint64_t n_words, const uint32_t* measures,
                                uint32_t n_entries, const int32_t* footprints, uint32_t n_footprints);
int vgi_read_events(vgi_ctx* ctx, uint32_t* words, uint64_t n_words);

/* ---- view tier: the visible-face path history of the view renderer -----------
 * (shaders/voxel_view_trace.wgsl, voxel_view_runtime.wgsl:272-349,
 * voxel_view_cache.wgsl; src/gpu/view/runtime.rs Stage::ORDER). The caller
 * gives the receivers: one per visible unit face (voxel, face, material),
 * each its own owner; raster discovery, reprojection between views, the
 * topology prior of new faces and sun-corner records are outside this path.
 * Records keep the shaders' layouts: ViewReceiver 8 words, ViewPath 32,
 * ViewContinuation 32, ViewEstimate 16; the queue holds 12 counters, the
 * owner list and one cursor word per receiver. */
typedef struct vgi_view_wave {
    uint32_t first;        /* ViewWave.range.x: first owner of the rotation */
    uint32_t invocations;  /* range.y: owner invocations this frame (0: one per receiver) */
    uint32_t max_hits;     /* range.z: hits a path advances per visit, 1..8 (0: no tracing) */
    uint32_t depth;        /* range.w: finite path depth, 0 for unbiased roulette */
    uint32_t ticket[4];    /* owner generations: a change restarts paused paths */
    uint32_t view_first;   /* view.history.w: up to 32 visits per owner instead of 1 */
    uint32_t shared;       /* view.cache.z: hand faces to and from the world cache */
    uint32_t clock_ms;     /* view.cache.y: worker clock for the cache's rank records */
} vgi_view_wave;
/* Replaces the receiver list; estimates, paths and continuations start empty. */
int vgi_view_set_receivers(vgi_ctx* ctx, const vgi_face* faces, uint32_t n);
/* One view frame: reproject (sequence from the estimate, owner queue),
 * retain_view_history for `n_events` encoded events (vgi_apply_events'
 * layout), load_shared_faces, trace_visible_paths, store_shared_faces.
 * Synchronous. */
int vgi_view_frame(vgi_ctx* ctx, const vgi_view_wave* wave, const uint32_t* events, uint32_t n_events, uint64_t n_words);
/* Snapshots of the view records; each pointer may be null. */
/* The sun-flip reports (report_sun_flips, voxel_view_runtime.wgsl:229-270)
 * of the view frames since the last call (or since vgi_view_set_receivers):
 * faces whose refreshed corner words, or whose corners on re-entering view
 * against those their world slot kept, changed a lit bit. Reports build up
 * across frames and this call clears them after copying, as the reference's
 * timing receipt does (src/gpu/view/timing.rs:386-387), so a caller that
 * reads less often than once a frame loses no change. 8,203 words: the
 * count and 3 zeros; 2,048 records
 * (voxel xyz, flux as f32 bits) in an arbitrary order; then the overflow of
 * flips past 2,048: max of 2^30 - voxel xyz, max of voxel xyz + 2^30, and
 * the sum of round(flux * 64). */
int vgi_view_read_sun_flips(vgi_ctx* ctx, uint32_t* words);
int vgi_view_read(vgi_ctx* ctx, uint32_t* receivers8, uint32_t* paths32, uint32_t* continuations32, uint32_t* estimates16,
                  uint32_t* queue);
/* trace_view_paths: `samples` complete receiver samples per receiver
 * (sequence + i), one ViewPath record each, in receiver-major order. */
int vgi_view_trace_paths(vgi_ctx* ctx, uint32_t samples, uint32_t* paths32);

/* ---- FP64 converged reference ------------------------------------------------
 * No counterpart in the reference's GPU path: an error yardstick. For each
 * FaceTask (8 words; voxel, face, sequence), `samples` independent unbiased
 * samples of the quantity the world cache accumulates (cosine-averaged
 * incident radiance without the face's own direct light), in double
 * precision, without the cache and with Russian roulette instead of a depth
 * cut. mean3 / second3 get the per-face mean and mean square (rgb), known the
 * samples that did not reach unloaded space. `seed` selects the random
 * streams. Synchronous. */
int vgi_reference_fp64(vgi_ctx* ctx, const uint32_t* tasks, uint32_t n, uint32_t samples, uint64_t seed, double* mean3, double* second3,
                       uint32_t* known);

/* ---- MLP radiance cache ------------------------------------------------------
 * No counterpart in the reference: a small network that predicts a face's
 * incident radiance from its position, normal and albedo, run on the
 * tcgen05 tensor cores. 96 inputs (81 features: 12 sine/cosine frequencies
 * per position axis, the normal as one-hot, the albedo; zero padded), four
 * hidden layers of 64 with ReLU, 16 outputs of which the first 3 pass
 * through exp. Weights are FP32 masters, layer after layer, each [in][out]
 * row-major (19,456 floats); the kernels use their BF16 rounding and
 * accumulate in FP32. */
int vgi_mlp_set_weights(vgi_ctx* ctx, const float* master, uint32_t count);
int vgi_mlp_get_weights(vgi_ctx* ctx, float* master, uint32_t count);
/* Forward pass over n feature rows (96 floats each): out4 = (rgb, 0) per row. */
int vgi_mlp_forward(vgi_ctx* ctx, const float* features, uint32_t n, float* out4);
/* Training loss over n rows with targets4 = (rgb, unused) per row: the
 * relative luminance MSE  sum_rows sum_c (p_c - y_c)^2 / (lum(p)^2 + 0.01) / n,
 * with lum(p) = 0.2126 r + 0.7152 g + 0.0722 b held constant in the gradient.
 * vgi_mlp_gradients writes dLoss/dW (19,456 floats, the master order) and the
 * loss without changing the weights; vgi_mlp_train takes one Adam step
 * (beta 0.9 / 0.99, eps 1e-8, learning rate lr) on the FP32 masters and
 * writes the loss before the step. vgi_mlp_set_weights resets Adam. */
int vgi_mlp_gradients(vgi_ctx* ctx, const float* features, const float* targets4, uint32_t n, float* grads, float* loss);
int vgi_mlp_train(vgi_ctx* ctx, const float* features, const float* targets4, uint32_t n, float lr, float* loss);
/* One Adam step from a given gradient (19,456 floats, the master order; host
 * memory, or device memory on the context's device when on_device != 0) and
 * its loss, for data-parallel training: every rank takes vgi_mlp_gradients
 * of its own rows, the ranks average the gradients (an all-reduce), and each
 * applies the average here, so all ranks keep the same weights. The gradient
 * of a batch from vgi_mlp_gradients gives the step vgi_mlp_train takes on
 * that batch. No counterpart in the reference (it has no network).
 * Synchronous. */
int vgi_mlp_apply_gradients(vgi_ctx* ctx, const float* grads, float loss, float lr, int on_device);
/* The network's 96 inputs for n faces (their voxel, face and material), as
 * the frame's queries and training rows compute them: per axis of the face
 * centre x (voxels, normalised to [0, 1] over the loaded regions), sin and
 * cos of pi 2^k x for k = 0..11 (24 per axis), the face one-hot (72..77),
 * the material's diffuse albedo (78..80), zeros. Synchronous. */
int vgi_mlp_encode(vgi_ctx* ctx, const vgi_face* faces, uint32_t n, float* features);
/* MLP cache mode of vgi_frame. Every frame trains the network online on
 * `samples` faces (at most 2^22), split over `steps_per_frame` Adam steps
 * (learning rate lr) of samples / steps_per_frame faces each (input: the
 * face's encoding; target: the frame's traced mean of the quantity the world
 * cache accumulates; faces without a known sample are skipped). The first
 * `warm_frames` frames trace plainly and draw the faces from their own
 * results. Later frames end every first hit that the world cache does not
 * answer with the network's prediction for the hit face instead of
 * continuing the path (the wavefront layout with one diffuse hit), and
 * train on those hit faces: `samples` of the frame's queries are traced as
 * faces of their own, 4 paths each. In the single-kernel layout frames trace
 * plainly. Resets the frame count; the weights and Adam state stay. */
int vgi_set_mlp_cache(vgi_ctx* ctx, int enable, uint32_t warm_frames, uint32_t samples, uint32_t steps_per_frame, float lr);
/* The MLP cache mode's training batches and averaging window. No
 * counterpart in the reference.
 * rows_per_step: the rows of one Adam step; 0 (the default) splits the
 * frame's samples over its steps. A larger batch cycles through the
 * frame's samples (step k starts at k x rows_per_step modulo the samples),
 * so the frame takes the same steps on bigger batches of the same data.
 * history_share: with share > 0, every frame in which the network ends
 * paths caps the faces' sample count (the accumulation's history limit) at
 * share x the samples a face has taken in such frames, this one included,
 * and at least 32 (above the cache's binding count of 16), so the means
 * weight late frames, whose network is trained, above the first ones; the
 * transport's history limit still caps it. 0 (the default) keeps the
 * transport's limit. */
int vgi_set_mlp_schedule(vgi_ctx* ctx, uint32_t rows_per_step, float history_share);
typedef struct vgi_mlp_status {
    uint32_t frames;       /* frames traced since vgi_set_mlp_cache */
    uint32_t steps;        /* Adam steps taken since vgi_mlp_set_weights */
    uint32_t terminating;  /* the next frame ends first hits with the network */
    uint32_t queries;      /* network queries of the last terminating frame */
    float loss;            /* loss of the last training batch */
    uint32_t error;        /* nonzero: a tensor-core wait ran out */
    float query_ms;        /* with vgi_set_timing: the last terminating frame's */
    float train_ms;        /*   query launch and its training, CUDA-event times */
} vgi_mlp_status;
/* Synchronous. */
int vgi_mlp_stats(vgi_ctx* ctx, vgi_mlp_status* out);
/* No counterpart in the reference (its wgpu waits are the driver's). Every
 * mbarrier wait of the MLP cache's tensor-core kernels gives up after
 * `polls` polls (VGI_MLP_WAIT_DEFAULT restores the default, about 4 M): the
 * kernel sets the error word, lets the copy or MMAs it waited for land,
 * frees its TMEM and returns, and the call reports VGI_ERR_CUDA (frames:
 * vgi_mlp_stats' error). 0 makes every wait give up at once, so a caller
 * can check that path and that the context still works afterwards. Applies
 * to launches and frame graphs made after the call. */
#define VGI_MLP_WAIT_DEFAULT 0xffffffffu
int vgi_mlp_set_wait_limit(vgi_ctx* ctx, uint32_t polls);

/* ---- headless discovery ---------------------------------------------------------
 * The face list from the GPU instead of a raster prepass (as NAADF's
 * renderFirstHit): one primary ray per pixel of a pinhole camera through
 * the NAADF geometry (trace_domain_limited with visible geometry, 2048
 * steps). Pixel (x, y): right = normalize(forward x up), up' = right x
 * forward, sx = ((2 (x + 0.5)) / width - 1) tan_half_fov (width / height),
 * sy = (1 - (2 (y + 0.5)) / height) tan_half_fov, direction =
 * normalize((forward + right sx) + up' sy); forward must be unit length.
 * pixels8 (may be null) receives per pixel (voxel xyz, face (6: no hit),
 * material, status, distance (f32 bits), 0); faces receives each hit face
 * once (its voxel, face and the hit's material), sorted by voxel z, y, x and
 * face. *n_faces is the number of distinct faces even when it exceeds
 * `capacity` (then VGI_ERR_CAPACITY). At most 2^26 pixels. Synchronous. */
typedef struct vgi_camera {
    float eye[3];
    float forward[3];
    float up[3];
    float tan_half_fov;
    uint32_t width, height;
} vgi_camera;
int vgi_discover_faces(vgi_ctx* ctx, const vgi_camera* camera, uint32_t* pixels8, vgi_face* faces, uint32_t capacity, uint32_t* n_faces);

/* ---- reconstruction and presentation of the view receivers ------------------------
 * vgi_view_set_tiles gives each view receiver its screen tile (tiles_x x
 * tiles_y, all ones: none; e.g. the 2 x 2-cell tile of the pixel where
 * discovery first saw its face, as the receiver pool's witness). Then
 * vgi_view_reconstruct runs reconstruct_view (inverse-variance weighting of
 * coplanar donors in the tiles around, radius 1..4 tiles from the evidence
 * deficit, a bias bound against the centre, a temporal blend of the shown
 * value; voxel_view_runtime.wgsl:380-474; donors in receiver order per
 * tile) and publish_view (a FarPixel per receiver: surface xyz, face (all
 * ones: none), irradiance rgb = shown plus custom direct light, evidence,
 * four sky corner words; voxel_view_runtime.wgsl:476-521). Counters: summed
 * history, max history, uncovered, displayed, paused. vgi_view_present
 * evaluates the presentation's corner_irradiance at each pixel's first hit
 * (voxel_gi_presentation.wesl:350-412): the face's published irradiance,
 * or with `corners` the evidence-weighted virtual-corner interpolation over
 * coplanar neighbours; rgba = rgb and the face's evidence (at most 1),
 * zeros where the ray hits nothing. */
typedef struct vgi_view_display {
    float evidence_goal; /* display.x: relative noise threshold (the reference's default 0.031) */
    float spatial;       /* display.y: spatial reconstruction strength (default 1) */
    float temporal;      /* display.z: blend of the shown value per frame */
} vgi_view_display;
int vgi_view_set_tiles(vgi_ctx* ctx, const uint32_t* tiles, uint32_t n, uint32_t tiles_x, uint32_t tiles_y);
int vgi_view_reconstruct(vgi_ctx* ctx, const vgi_view_display* display);
int vgi_view_read_published(vgi_ctx* ctx, uint32_t* pixels12, uint32_t* stats5);
int vgi_view_present(vgi_ctx* ctx, const vgi_camera* camera, int corners, float* rgba);

/* ---- far tier ---------------------------------------------------------------------
 * Per-pixel lighting for faces small on screen (FarTierSettings,
 * shaders/voxel_view_pixels.wgsl), headless: each cell of `cell` x `cell`
 * pixels traces one primary ray per frame through the NAADF geometry at one
 * of its pixels (a different one each frame) in place of the raster depth
 * and normal. A hit face far enough to be "small" (measure 0: a voxel's side
 * in pixels under voxel_pixels; 1: its covered area; 2: the same for its LoD
 * block) owns the cell: its history is reprojected from the previous
 * frame's cells through the previous camera, or handed over from the view
 * receiver of the same face, and a path is traced (trace_receiver with 3
 * hits, `steps` traversal steps, budgeted rays) while the history is under 4
 * samples or one frame in `rate`. Frames numbered more than one apart, or a
 * changed viewport, start without history. Settings are normalized as the
 * reference does (voxel_pixels 0..4096, 0 disables; history 1..1024; rate
 * 1..8; steps 16..2048; cell 0..4, 0: round(height / 480) in 1..4).
 * Asynchronous on the context's stream; vgi_far_read waits. */
typedef struct vgi_far_settings {
    float voxel_pixels;
    uint32_t measure;
    uint32_t cell;
    float history;
    uint32_t rate;
    uint32_t steps;
    int32_t interest_min[3]; /* regions, inclusive, when `bounded` */
    int32_t interest_max[3];
    uint32_t bounded;
} vgi_far_settings;
int vgi_far_frame(vgi_ctx* ctx, const vgi_camera* camera, const vgi_far_settings* settings, uint32_t frame);
/* With `enable`, a view frame starts each new, unmeasured view receiver
 * (no samples, no sequence, nothing from the world cache) from the far cell
 * at its centre in the last far frame, seen from that frame's camera, with
 * one unit of weight (load_shared_faces's far handoff); stats8[5] of
 * vgi_far_read counts them. Off by default. */
int vgi_set_far_handoff(vgi_ctx* ctx, int enable);
/* With `enable`, a view frame first gives each new, unmeasured unit-face
 * receiver whose voxel is solid and whose air cell is known its topology
 * prior (bootstrap_face, voxel_view_cache.wgsl:100-186): the mean of the
 * connected coplanar faces' incident light, else a weighted mean over the
 * faces around its air cell; donors are the other receivers as they were
 * before the frame, and world-cache slots, with at least 16 samples. The
 * far handoff applies only where this prior finds nothing. Off by default. */
int vgi_set_topology_prior(vgi_ctx* ctx, int enable);
/* Drop the far tier's history (a camera cut): cell histories and output
 * cells are zeroed and the next frame reprojects nothing. */
int vgi_far_reset(vgi_ctx* ctx);
/* shape4 = (cells x, cells y, pixels per cell side, enabled | measure << 1);
 * output = PixelOutput: 16 header words (camera xyz 0, view forward + pixels
 * per unit at depth 1, shape, 0 0 threshold-bits stamp), then per cell
 * pack2x16float(rg), pack2x16float(b, count), face | stamp << 3, surface
 * coordinate on the face's axis (bits); only owned cells are written each
 * frame. cells12 = PixelHistory per cell (mean rgb, count, surface xyz, face
 * word, sequence, 0, 0, 0). stats8 = owned, traced, history, reprojected,
 * seeded from view receivers, view receivers seeded from far cells (by view
 * frames since this far frame), 0, 0. Any pointer may be null. */
int vgi_far_read(vgi_ctx* ctx, uint32_t* shape4, uint32_t* output, uint32_t* cells12, uint32_t* stats8);

/* ---- scheduled frames: the GPU world-cache scheduler --------------------------
 * The reference's GPU selection of bulk work (shaders/voxel_accumulate.wgsl:
 * 448-695: candidate, select_classify, select_histogram, select_threshold,
 * select_emit; scheduling.rs states the rules): instead of every slot, a
 * frame traces `budget` faces it picks itself. Each live, due face competes
 * in one class: urgent (an edit's change binds it), coverage (fewer than 8
 * samples; nearest the focus first), refinement (within two 32-voxel pages
 * of the focus; highest error + age first) or sweep (elsewhere; oldest
 * first). Urgent faces take up to 3/4 of the budget, the rest goes 1/4,
 * 1/2, 1/4 with unused share lent on; per-class histograms of 256 key
 * buckets give the exact thresholds. Keys persist per slot; each frame
 * re-classifies slots [classify_first, classify_end) (the reference rotates
 * a quarter per batch), and a picked face's key is cleared until its range
 * comes round. A face is due unless fresh in this transport revision, with
 * its required samples, stable for 4 batches and younger than audit_ms.
 * The picks are traced and accumulated as GPU picks: each pick record is
 * (slot, revision tag, merged count, incarnation), and the face's
 * statistics mirror is marked stale (this library keeps no CPU mirror).
 * Ties at a threshold bucket are taken in block order, so which of them are
 * picked can differ from run to run (as on the reference's GPU); the keys,
 * histograms, thresholds and counts do not. */
typedef struct vgi_schedule {
    int32_t focus[3];          /* the camera's voxel */
    uint32_t budget;           /* faces to pick and trace, 1..slots */
    uint32_t classify_first, classify_end;
    uint32_t audit_ms;         /* a fresh, stable face is due again after this long */
} vgi_schedule;
int vgi_frame_scheduled(vgi_ctx* ctx, uint32_t samples, uint32_t clock_ms, const vgi_schedule* schedule);
/* After a scheduled frame: keys (one word per slot), the 1038 selection words
 * (4 x 256 histogram buckets, thresholds, remainders, ties, total, mirror
 * count), and per pick task its record (4 words), FaceTask (8) and
 * FaceResult as accumulate left it (24). Any pointer may be null. */
int vgi_read_selection(vgi_ctx* ctx, uint32_t* keys, uint32_t* selection, uint32_t* picks4, uint32_t* tasks8, uint32_t* results24);

/* ---- face-sharded frames -------------------------------------------------------
 * No counterpart in the reference. Faces are independent given the frame's
 * geometry and the world cache's snapshot, so a frame can be split across
 * GPUs by slot range. Every rank's context holds all faces (vgi_set_faces
 * with the full list: the face index and one 16-byte gather record per
 * slot), but vgi_frame_shard prepares, traces and accumulates only slots
 * [first, first + n). Between frames every rank publishes its range's
 * gather records (vgi_read_cache) and takes the others' (vgi_write_cache),
 * for example with one all-gather; the next frame then gathers from the
 * same snapshot a single GPU would, so every slot's results and state are
 * those of vgi_frame. Records are 4 words: mean rgb, the count word (bits).
 * With on_device set the pointer is device memory of the context's device
 * and the copy is enqueued on the context's stream; otherwise it is host
 * memory and the call is synchronous. */
int vgi_frame_shard(vgi_ctx* ctx, uint32_t samples, uint32_t clock_ms, uint32_t first, uint32_t n);
int vgi_read_cache(vgi_ctx* ctx, uint32_t first, uint32_t n, float* dst4, int on_device);
int vgi_write_cache(vgi_ctx* ctx, uint32_t first, uint32_t n, const float* src4, int on_device);

/* ---- batched scenes ----------------------------------------------------------
 * No counterpart in the reference (its scenes are traced one at a time):
 * several contexts, one per scene, traced together. vgi_batch_frame runs
 * for every scene what vgi_frame runs (prepare, the wavefront trace with
 * cache gather, accumulate), but the traversal of each stage is ONE
 * persistent launch over the rays of all scenes, so scenes of very uneven
 * size share the GPU. Every scene's results and state are those its own
 * vgi_frame would give. The scenes must be ready (geometry, model, faces),
 * on one device, in the wavefront layout, with the same bounces, reach limit
 * and step budget, and with the MLP cache mode off; at most 256 of them.
 * The batch enqueues on its own stream, ordered after and before each
 * scene's stream. vgi_batch_set_graph captures the whole batched frame into
 * one CUDA graph on the second frame after any change, as vgi_set_graph
 * does for one scene. vgi_batch_autotune times state-free batched traces of
 * the scenes' current tasks over the traversal's refill threshold and grid
 * size, keeps the fastest, and reports it. */
typedef struct vgi_batch vgi_batch;
int vgi_batch_create(vgi_ctx* const* ctxs, uint32_t n, vgi_batch** out);
int vgi_batch_destroy(vgi_batch* batch);
const char* vgi_batch_last_error(const vgi_batch* batch);
int vgi_batch_frame(vgi_batch* batch, uint32_t samples, uint32_t clock_ms);
int vgi_batch_set_graph(vgi_batch* batch, int enable);
int vgi_batch_sync(vgi_batch* batch);
int vgi_batch_autotune(vgi_batch* batch, uint32_t samples, uint32_t* refill_min, uint32_t* blocks, float* trace_ms);

/* ---- read-back: bounded snapshots (complete_readback, src/gpu.rs:1024-1170) --- */
int vgi_read_results(vgi_ctx* ctx, uint32_t first, uint32_t n, uint32_t* words24);
int vgi_read_state(vgi_ctx* ctx, uint32_t first, uint32_t n, uint32_t* words36);
int vgi_write_state(vgi_ctx* ctx, uint32_t first, uint32_t n, const uint32_t* words36);
int vgi_read_slot_meta(vgi_ctx* ctx, uint32_t first, uint32_t n, uint32_t* words12);

/* ---- failure injection ---------------------------------------------------------
 * No counterpart in the reference's interface; it plays the part of the
 * reference's injected failures (src/tests.rs:38-80). For the calling
 * thread, the next `count` device allocations (what = VGI_INJECT_ALLOC) or
 * host-to-device copies (what = VGI_INJECT_UPLOAD) made by this library fail
 * without reaching the device, as out of memory or as a failed copy. The
 * call that meets one returns VGI_ERR_CUDA with the reason in
 * vgi_last_error; the context stays usable: an upload or vgi_set_faces that
 * failed leaves no geometry or no faces (frames return VGI_ERR_STATE) until
 * the next successful one. A failure met inside vgi_create gives
 * VGI_UNAVAILABLE and no context, as a device that cannot run the path.
 * count = 0 cancels. ctx may be null. */
#define VGI_INJECT_ALLOC 1u
#define VGI_INJECT_UPLOAD 2u
int vgi_inject_failure(vgi_ctx* ctx, uint32_t what, uint32_t count);

/* ---- region packing without allocation -------------------------------------
 * No counterpart in the reference. This is for callers that must not allocate
 * device memory. One example is an engine that has reserved all of its GPU
 * memory through its own allocator and forbids libraries from taking more.
 * Another is a frame-critical thread, where cudaMalloc's implicit device
 * synchronisation would stall rendering.
 *
 * It packs `n` regions on the calling thread's current device, on `stream`
 * (a cudaStream_t, 0 for the legacy default stream). The regions are n x 4096
 * u16 voxels in the caller's device memory, 16-byte aligned, values 0..256.
 * Outputs, also in the caller's device memory:
 *   headers: n x 4 u32, 16-byte aligned, (kind, material or cell offset, 0, 0):
 *            the kinds and materials vgi_upload_regions' packer writes;
 *   cells:   `cells_capacity` u32 words.
 * On success, *cells_used is the number of cell words written. Cells are laid
 * out in region order, so the layout depends only on the input. Bricks are
 * not deduplicated: every mixed brick gets its own 32 words, where
 * vgi_upload_regions stores identical bricks once, so the cells take more
 * room (about twice as much on the 512x256x512 terrain: 51 MB against
 * 25 MB). The brick words decode to the same voxels and extents.
 *
 * The call allocates nothing. Its scratch is a static device array sized for
 * VGI_STATIC_PACK_MAX_REGIONS regions (about 256 KiB per GPU, held until the
 * process exits). The first call on each device looks up that array's device
 * address and keeps it for the process; make it before any stream capture.
 * A cudaDeviceReset of that device afterwards leaves the kept address stale
 * and is not supported. The call synchronises `stream`. Every call shares
 * the array, so two calls whose work overlaps on the GPU race; serialise
 * them on one stream.
 *
 * Returns VGI_ERR_CAPACITY for n above the maximum or when cells_capacity is
 * too small, and VGI_ERR_INVALID for null or misaligned pointers or voxel
 * values above 256. */
#define VGI_STATIC_PACK_MAX_REGIONS 65536
int vgi_pack_regions_static(const uint16_t* voxels, uint32_t n, uint32_t* headers, uint32_t* cells, uint64_t cells_capacity,
                            uint64_t* cells_used, void* stream);

/* ---- host runtime (no device needed) -------------------------------------- */
/* Record builders with the host-side conventions of src/gpu.rs:717-760
 * (directional: glam normalize_or_zero of the direction, range -1). */
void vgi_material_record(const float* diffuse3, const float* emission3, float* out16);
void vgi_directional_light_record(const float* direction3, const float* radiance3, const float* custom3, float* out12);
/* The emitter words vgi_build_emitters uploads, for a region list and a
 * material table: returns the word count, writes when `capacity` suffices;
 * info = [faces, total_weight bits]. */
int64_t vgi_host_emitters(const int32_t* coords, uint32_t n, const uint16_t* voxels, const float* materials, uint32_t* out,
                          uint64_t capacity, uint32_t* info2);
/* The face index vgi_set_faces uploads (4 ints per face: voxel xyz, face):
 * returns the uint4 count (capacity + 1), writes when `capacity4` suffices. */
int64_t vgi_host_face_index(const int32_t* faces, uint32_t n, uint32_t* out, uint64_t capacity4);
/* The top-level field vgi_upload_regions grows from an empty scene: 6 bytes
 * per cell over the region bounds (x fastest); returns 1 when the field is
 * disabled by its size limits, 0 when written. `solid` holds 1 per region
 * with any solid voxel. */
int vgi_host_top_level(const int32_t* coords, const uint8_t* solid, uint32_t n, uint8_t* out6, uint64_t capacity);

#ifdef __cplusplus
}
#endif
#endif /* VGI_H */
