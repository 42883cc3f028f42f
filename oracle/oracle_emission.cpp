// TEST INFRASTRUCTURE ONLY (the oracle). CPU restatement of the reference's
// emitter distribution and light hierarchy, the checker of the product's
// emitter builder.
//
// Follows (paths within nathanaelneveux/global-illumination):
//   crates/bevy_voxel_gi/src/emission.rs:91-165      EmissionDistribution::build
//   crates/bevy_voxel_gi/src/emission.rs:205-216     face_point
//   crates/bevy_voxel_gi/src/emission/tree.rs:19-75  key / build
//   crates/bevy_voxel_gi/src/emission/tree.rs:173-195 LightNode::words
//   crates/bevy_voxel_gi/src/gpu.rs:686-711           emitter upload (GpuEmitter, then node words)
#include "oracle.h"

#include <algorithm>
#include <array>
#include <map>
#include <tuple>
#include <vector>

namespace {
using namespace orc;

struct Face { int32_t v[3]; uint32_t face; uint32_t material; float cumulative; float probability; };

const int32_t OFFS[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

struct Node {
    float mn[3], power, mx[3];
    uint32_t normals;
    int32_t pivot[3];
    uint32_t pivot_face, left, right, axis;
};

void face_center(const Face& f, float out[3]) {
    // face_point(face, 0.5, 0.5): voxel + 0.5 + normal * 0.5 + tangent * 0 + bitangent * 0
    uint32_t axis = f.face / 2;
    float t[3] = {axis == 0 ? 0.0f : 1.0f, axis == 0 ? 1.0f : 0.0f, 0.0f};
    float b[3] = {0.0f, axis == 2 ? 1.0f : 0.0f, axis == 2 ? 0.0f : 1.0f};
    for (int a = 0; a < 3; ++a) {
        float n = (float)OFFS[f.face][a];
        out[a] = (((float)f.v[a] + 0.5f) + n * 0.5f + t[a] * (0.5f - 0.5f)) + b[a] * (0.5f - 0.5f);
    }
}

std::tuple<int32_t, int32_t, int32_t, uint32_t> key(const Face& f, uint32_t axis) {
    return {f.v[axis], f.v[(axis + 1) % 3], f.v[(axis + 2) % 3], f.face};
}

uint32_t split(std::vector<Node>& nodes, std::vector<size_t>& idx, size_t lo, size_t hi, const std::vector<Face>& faces) {
    uint32_t index = (uint32_t)nodes.size();
    Node node{};
    for (int a = 0; a < 3; ++a) { node.mn[a] = INFINITY; node.mx[a] = -INFINITY; }
    node.power = 0.0f;
    for (size_t k = lo; k < hi; ++k) {
        const Face& f = faces[idx[k]];
        float c[3];
        face_center(f, c);
        for (int a = 0; a < 3; ++a) {
            float e = (1.0f - std::fabs((float)OFFS[f.face][a])) * 0.5f;
            float lo_v = c[a] - e, hi_v = c[a] + e;
            // glam's Vec3::min/max on SSE: self < rhs ? self : rhs (ties take rhs)
            node.mn[a] = node.mn[a] < lo_v ? node.mn[a] : lo_v;
            node.mx[a] = node.mx[a] > hi_v ? node.mx[a] : hi_v;
        }
        node.power = node.power + f.probability;
        node.normals |= 1u << f.face;
    }
    nodes.push_back(node);
    if (hi - lo == 1) {
        node.left = 0xffffffffu;
        node.right = (uint32_t)idx[lo];
    } else {
        float ext[3] = {node.mx[0] - node.mn[0], node.mx[1] - node.mn[1], node.mx[2] - node.mn[2]};
        node.axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0u : (ext[1] >= ext[2] ? 1u : 2u);
        uint32_t axis = node.axis;
        std::sort(idx.begin() + lo, idx.begin() + hi, [&](size_t a, size_t b) { return key(faces[a], axis) < key(faces[b], axis); });
        size_t mid = (hi - lo) / 2;
        const Face& pivot = faces[idx[lo + mid]];
        for (int a = 0; a < 3; ++a) node.pivot[a] = pivot.v[a];
        node.pivot_face = pivot.face;
        node.left = split(nodes, idx, lo, lo + mid, faces);
        node.right = split(nodes, idx, lo + mid, hi, faces);
    }
    nodes[index] = node;
    return index;
}
}  // namespace

extern "C" {

// Builds the emitter words for a region list (coords, 4096 voxels per region)
// and a material table (16 floats per material; emission_extra.y = weight).
// Writes [n_faces, n_nodes, total_weight bits] to `info` and, when `out` is
// large enough (out_words uint32 values), the uint4 emitter buffer the shader
// reads: one default record when there are no faces.
int64_t orc_emitters(const int32_t* coords, uint32_t n, const uint16_t* voxels, const float* materials, uint32_t* out,
                     uint64_t out_words, uint32_t* info) {
    float weights[256];
    bool any = false;
    for (int m = 0; m < 256; ++m) { weights[m] = materials[m * 16 + 13]; if (weights[m] > 0.0f) any = true; }
    std::map<std::array<int32_t, 3>, uint32_t> index;  // (z, y, x) -> region
    for (uint32_t r = 0; r < n; ++r) index[{coords[r * 3 + 2], coords[r * 3 + 1], coords[r * 3]}] = r;
    auto material_at = [&](int32_t x, int32_t y, int32_t z, bool* loaded) -> uint16_t {
        auto it = index.find({z >> 4, y >> 4, x >> 4});
        if (it == index.end()) { *loaded = false; return 256; }
        *loaded = true;
        return voxels[(size_t)it->second * 4096 + (x & 15) + 16 * ((y & 15) + 16 * (z & 15))];
    };
    std::vector<Face> faces;
    double total = 0.0;
    if (any) {
        for (auto& kv : index) {  // sorted by (z, y, x)
            uint32_t r = kv.second;
            const uint16_t* m = voxels + (size_t)r * 4096;
            bool has = false;
            for (int i = 0; i < 4096; ++i) if (m[i] != 256 && weights[m[i]] > 0.0f) { has = true; break; }
            if (!has) continue;
            for (int32_t z = 0; z < 16; ++z)
                for (int32_t y = 0; y < 16; ++y)
                    for (int32_t x = 0; x < 16; ++x) {
                        uint16_t mat = m[x + 16 * (y + 16 * z)];
                        if (mat == 256 || weights[mat] <= 0.0f) continue;
                        int32_t v[3] = {coords[r * 3] * 16 + x, coords[r * 3 + 1] * 16 + y, coords[r * 3 + 2] * 16 + z};
                        for (uint32_t f = 0; f < 6; ++f) {
                            bool loaded;
                            uint16_t nb = material_at(v[0] + OFFS[f][0], v[1] + OFFS[f][1], v[2] + OFFS[f][2], &loaded);
                            if (loaded && nb != 256) continue;
                            total += (double)weights[mat];
                            faces.push_back(Face{{v[0], v[1], v[2]}, f, mat, (float)total, weights[mat]});
                        }
                    }
        }
    }
    if (total == 0.0) faces.clear();
    float total_weight = (float)total;
    for (auto& f : faces) { f.cumulative = f.cumulative / total_weight; f.probability = f.probability / total_weight; }
    if (!faces.empty()) faces.back().cumulative = 1.0f;
    std::vector<Node> nodes;
    if (faces.size() >= 32) {
        std::vector<size_t> idx(faces.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
        split(nodes, idx, 0, idx.size(), faces);
    }
    size_t records = faces.empty() ? 1 : faces.size();
    uint64_t words = (uint64_t)records * 8 + (uint64_t)nodes.size() * 16;
    info[0] = (uint32_t)faces.size();
    info[1] = (uint32_t)nodes.size();
    info[2] = fbits(faces.empty() ? 0.0f : total_weight);
    if (out == nullptr || out_words < words) return (int64_t)words;
    std::fill(out, out + words, 0u);
    for (size_t i = 0; i < faces.size(); ++i) {
        uint32_t* w = out + i * 8;
        w[0] = (uint32_t)faces[i].v[0]; w[1] = (uint32_t)faces[i].v[1]; w[2] = (uint32_t)faces[i].v[2]; w[3] = faces[i].face;
        w[4] = fbits(faces[i].cumulative); w[5] = fbits(faces[i].probability);
        w[6] = fbits((float)faces[i].material); w[7] = fbits((float)nodes.size());
    }
    uint32_t* t = out + records * 8;
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node& nd = nodes[i];
        uint32_t* w = t + i * 16;
        w[0] = fbits(nd.mn[0]); w[1] = fbits(nd.mn[1]); w[2] = fbits(nd.mn[2]); w[3] = fbits(nd.power);
        w[4] = fbits(nd.mx[0]); w[5] = fbits(nd.mx[1]); w[6] = fbits(nd.mx[2]); w[7] = nd.normals;
        w[8] = (uint32_t)nd.pivot[0]; w[9] = (uint32_t)nd.pivot[1]; w[10] = (uint32_t)nd.pivot[2]; w[11] = nd.pivot_face;
        w[12] = nd.left; w[13] = nd.right; w[14] = nd.axis; w[15] = 0;
    }
    return (int64_t)words;
}

}  // extern "C"
