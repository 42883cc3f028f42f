/*
 * vgi_scenes.h -- seeded synthetic workloads for libvgi (benchmarks, tests).
 *
 * These are not part of the reference's interface: the reference's lab
 * scenes depend on an unvendored noise crate, so the workloads its headline
 * configurations describe are generated here from their stated parameters.
 * Scenes are region lists in the vgi_upload_regions layout (3 ints per
 * region coordinate, 4096 u16 voxels per region, x fastest, 256 = air).
 */
#ifndef VGI_SCENES_H
#define VGI_SCENES_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A dense grid of nx x ny x nz regions starting at region (0, 0, 0): writes
 * the coordinates in (z, y, x) order. Returns the region count. */
uint32_t vgi_scene_grid_coords(uint32_t nx, uint32_t ny, uint32_t nz, int32_t* coords);

/* Stone room: a 32^3 closed box with 1-voxel shell of material 0 and one
 * emissive voxel of material 1 on the floor at (16, 1, 16). 8 regions. */
void vgi_scene_stone_room(uint16_t* voxels);

/* Furnace (16^3 shell from 8 to 23 in a 32^3 page, material 4). 8 regions. */
void vgi_scene_furnace(uint16_t* voxels);

/* Terrain: seeded 3D fBm value noise (octaves, base frequency 1/period,
 * lacunarity 2, gain 0.5) minus a height bias (y - base_height) / falloff;
 * solid where the density is positive. Materials 0..7 by a second noise
 * field; `emitters` emissive voxels (materials 8 + i % 248) are placed on
 * random surface columns. Region grid nx x ny x nz in (z, y, x) order. */
typedef struct {
    uint32_t seed;
    uint32_t octaves;
    float period;
    float base_height;
    float falloff;
    uint32_t emitters;
} vgi_terrain_params;
void vgi_scene_terrain(const vgi_terrain_params* p, uint32_t nx, uint32_t ny, uint32_t nz, uint16_t* voxels);

/* Cave: solid rock (materials 0..7 by a coarse noise field) carved by
 * `worms` seeded worm tunnels, random walks steered by value noise whose
 * radius varies along the walk in [radius_min, radius_max], under a solid
 * roof `roof` voxels thick. `skylights` vertical shafts of radius
 * `skylight_radius` cut through the roof, and the first tunnels start under
 * them. `emitters` emissive voxels sit on tunnel floors, alternately
 * material 8 (green) and 9 (orange). Region grid nx x ny x nz in (z, y, x)
 * order. */
typedef struct {
    uint32_t seed;
    uint32_t worms;
    uint32_t steps;
    float radius_min;
    float radius_max;
    uint32_t roof;
    uint32_t skylights;
    float skylight_radius;
    uint32_t emitters;
} vgi_cave_params;
void vgi_scene_cave(const vgi_cave_params* p, uint32_t nx, uint32_t ny, uint32_t nz, uint16_t* voxels);

/* Exposed faces: a face of a solid voxel whose neighbour is loaded air.
 * Optional filters: a square frustum (eye xyz, forward xyz, half-angle
 * tangent) on the face centre with the face turned towards the eye; or, with
 * `use_facing`, every face turned towards the eye (the six 90-degree frusta
 * of a cube-map camera, without counting faces on their shared planes twice).
 * Faces are written (voxel xyz, face, material), 5 ints each, in region then
 * voxel (z, y, x) then face order; returns the count (writes at most
 * `capacity`). */
typedef struct {
    uint32_t use_frustum;
    float eye[3];
    float forward[3];
    float tan_half;
    uint32_t use_box;
    int32_t box_min[3];
    int32_t box_max[3];
    uint32_t use_facing;
} vgi_face_filter;
uint64_t vgi_scene_faces(const int32_t* coords, uint32_t n, const uint16_t* voxels, const vgi_face_filter* filter, int32_t* out,
                         uint64_t capacity);

#ifdef __cplusplus
}
#endif
#endif /* VGI_SCENES_H */
