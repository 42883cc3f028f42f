// Host runtime of libvgi: the parts of the path the reference also runs on
// its CPU scene worker, kept on the host here because they are sequential,
// order-dependent and small (O(regions) or O(emissive faces)).
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <unordered_map>
#include <vector>

namespace vgi {

// Six u8 extents per cell: NEG_X, POS_X, NEG_Y, POS_Y, NEG_Z, POS_Z.
using Extents = std::array<uint8_t, 6>;

struct RegionKey {
    int32_t x, y, z;
    bool operator==(const RegionKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct RegionKeyHash {
    size_t operator()(const RegionKey& k) const;
};

// TopLevelAadf (src/world.rs:428-713): a dense region-level empty-space field
// over the loaded regions' bounding box, kept as a fixed point of NAADF's
// merging rule and updated incrementally.
class TopLevelField {
public:
    bool present = false;   // any regions
    bool enabled = false;   // field stored (size limits)
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    uint32_t dim[3] = {0, 0, 0};
    std::vector<Extents> cells;
    std::vector<uint8_t> barrier;

    // `blocked(x, y, z)`: missing region or one holding a solid voxel.
    // `changed`: regions whose residency or emptiness changed since *this.
    TopLevelField updated(const int32_t lo_[3], const int32_t hi_[3], bool any,
                          const std::function<bool(int32_t, int32_t, int32_t)>& blocked,
                          const std::vector<RegionKey>& changed) const;
    Extents at(int32_t x, int32_t y, int32_t z) const;
};

// Region directory (src/gpu_scene.rs:411-434): open addressing keyed by
// hash_voxel(region), capacity nextpow2(2n) doubled until every entry sits
// fewer than 32 probes from its home slot.
std::vector<int32_t> build_directory(const std::vector<RegionKey>& keys);
// The same build over (key, header) pairs, for a header array with free slots.
std::vector<int32_t> build_directory(const std::vector<std::pair<RegionKey, uint32_t>>& entries);
// In-place maintenance between builds (src/gpu_scene.rs:337-409): a linear-
// probing insert that refuses a probe chain of 32 or more (the caller then
// rebuilds), and backward-shift deletion, which leaves no tombstones and
// never lengthens a probe chain. Both keep `dir` (4 words a slot) valid for
// lookup_region.
bool directory_insert(std::vector<int32_t>& dir, const RegionKey& key, uint32_t header);
bool directory_remove(std::vector<int32_t>& dir, const RegionKey& key);

// Face index (src/gpu/face_index.rs): (voxel, face) -> slot, capacity 1024
// doubled before half load, rehashing in table order as the worker does.
// Returns [mask, 64, 0, 0] then one uint4 per entry.
std::vector<uint32_t> build_face_index(const std::vector<std::array<int32_t, 4>>& faces);

// EmissionDistribution::build + light tree (src/emission.rs:91-165,
// src/emission/tree.rs:28-75): the shader's emitter words.
struct EmitterWords {
    std::vector<uint32_t> words;
    uint32_t faces = 0;
    float total_weight = 0.0f;
};
// `live` (optional) marks the header slots that hold a region; the others
// are skipped.
EmitterWords build_emitters(const std::vector<RegionKey>& keys, const uint16_t* voxels, const float* materials,
                            const std::vector<uint8_t>* live = nullptr);

uint32_t host_pcg(uint32_t v);
uint32_t host_hash_voxel(int32_t x, int32_t y, int32_t z);

// What lookup_region (shaders/voxel_traversal.wgsl:32-41) returns for every
// region of the bounding box [lo, hi] (x fastest): the header index, or -1
// where the probe finds an empty slot or gives up after 32 probes. Empty when
// the box holds more than `max_cells` regions.
std::vector<int32_t> region_grid(const int32_t* directory, uint64_t slots, const int32_t lo[3], const int32_t hi[3], uint64_t max_cells);

}  // namespace vgi
