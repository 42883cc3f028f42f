// TEST INFRASTRUCTURE ONLY (the oracle). C entry points of the CPU
// restatement of bevy_voxel_gi's per-frame diffuse-GI path. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
#include <vector>
#include "oracle_math.h"
namespace orc {
uint32_t pcg(uint32_t value);
uint32_t hash_voxel(int32_t x, int32_t y, int32_t z);
}
extern "C" {
#endif

typedef struct orc_scene orc_scene;

// Work counters: one "ray" is one trace_domain_limited call; one "path" is one
// receiver sample. Bytes follow the algorithmic byte rules of the hot path
// (directory probe 16, header 16, brick word 4, cell word 4, task 32,
// result 96, material 64 per read, light 48, emitter 32, light-tree node 64,
// face-index probe 16, cache record 16).
typedef struct {
    uint64_t rays, paths, steps, bytes, unknown, cache_hits;
    uint64_t status[4];
    uint64_t traverse_bytes;  // the traversal's share of bytes (directory, header, brick, cell)
} orc_counters;

typedef struct {
    uint32_t diffuse_hits;   // DIFFUSE_HITS override (1..3)
    uint32_t limited_reach;  // LIMITED_REACH override
    uint32_t path_steps;     // PATH_STEPS override
    uint32_t budgeted;       // BUDGETED_RAYS override
    uint32_t lanes;          // PATH_LANES: 1 = serial trace_faces order
} orc_pipeline;

int orc_build_aadf(uint32_t sx, uint32_t sy, uint32_t sz, const uint8_t* blocked, uint8_t* out6);
int orc_scene_create(const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides, int top_mode,
                     orc_scene** out);
void orc_scene_free(orc_scene* sc);
int orc_scene_edit(orc_scene* sc, const int32_t* edits, uint32_t n);
int orc_scene_info(const orc_scene* sc, uint64_t* sizes, int32_t* bounds);
int orc_scene_copy(const orc_scene* sc, int32_t* directory, uint32_t* headers, uint32_t* cells);
int orc_scene_top_level(const orc_scene* sc, uint8_t* out6);
int orc_canonical(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                  uint64_t n_cells, const int32_t* coords, uint32_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif
