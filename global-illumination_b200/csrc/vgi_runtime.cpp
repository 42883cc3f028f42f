// Host runtime algorithms (see vgi_runtime.h). Each follows the reference's
// CPU statement exactly, because its output (skip extents, probe layout,
// emitter order and tree) feeds the bit-exact GPU trace.
#include "vgi_runtime.h"
#include "../../include/vgi.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

namespace vgi {

uint32_t host_pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
uint32_t host_hash_voxel(int32_t x, int32_t y, int32_t z) {
    return host_pcg(host_pcg(host_pcg((uint32_t)x) ^ (uint32_t)y) ^ (uint32_t)z);
}
size_t RegionKeyHash::operator()(const RegionKey& k) const { return host_hash_voxel(k.x, k.y, k.z); }

namespace {

// Grid helpers over a W x H x D box, x fastest.
struct Grid {
    uint32_t w, h, d;
    size_t index(uint32_t x, uint32_t y, uint32_t z) const { return x + (size_t)w * (y + (size_t)h * z); }
    void coords(size_t i, int32_t c[3]) const {
        c[0] = (int32_t)(i % w);
        c[1] = (int32_t)((i / w) % h);
        c[2] = (int32_t)(i / ((size_t)w * h));
    }
    bool inside(const int32_t c[3]) const {
        return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < (int32_t)w && c[1] < (int32_t)h && c[2] < (int32_t)d;
    }
    size_t size() const { return (size_t)w * h * d; }
};

const int kStep[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

// NAADF's merge rule (src/naadf.rs:117-148): grow `e` one cell in direction d
// when the neighbour there is inside, unblocked and its box covers e's
// extents in every direction but the opposite one.
bool grow_towards(Extents& e, const int32_t nb[3], int d, const Grid& g, const std::vector<uint8_t>& barrier,
                  const std::vector<Extents>& field) {
    if (!g.inside(nb) || e[d] == 255) return false;
    size_t ni = g.index(nb[0], nb[1], nb[2]);
    if (barrier[ni]) return false;
    const Extents& n = field[ni];
    for (int k = 0; k < 6; ++k)
        if (k != (d ^ 1) && n[k] < e[k]) return false;
    e[d] += 1;
    return true;
}

// Growth (src/world.rs:838-913): a FIFO of cells whose boxes may grow.
class Worklist {
public:
    explicit Worklist(const Grid& g) : g_(g), queued_(g.size(), 0) {}
    void push(size_t i) {
        if (!queued_[i]) {
            queued_[i] = 1;
            fifo_.push_back(i);
        }
    }
    void touch(size_t i) {
        push(i);
        int32_t c[3];
        g_.coords(i, c);
        for (int d = 0; d < 6; ++d) {
            int32_t n[3] = {c[0] + kStep[d][0], c[1] + kStep[d][1], c[2] + kStep[d][2]};
            if (g_.inside(n)) push(g_.index(n[0], n[1], n[2]));
        }
    }
    void drain(std::vector<Extents>& field, const std::vector<uint8_t>& barrier) {
        for (size_t head = 0; head < fifo_.size(); ++head) {
            size_t i = fifo_[head];
            queued_[i] = 0;
            if (barrier[i]) continue;
            int32_t c[3];
            g_.coords(i, c);
            Extents e = field[i];
            for (int d = 0; d < 6; ++d) {
                int32_t n[3] = {c[0] + kStep[d][0], c[1] + kStep[d][1], c[2] + kStep[d][2]};
                grow_towards(e, n, d, g_, barrier, field);
            }
            if (e != field[i]) {
                field[i] = e;
                touch(i);
            }
            if (head > 4096 && head * 2 > fifo_.size()) {
                fifo_.erase(fifo_.begin(), fifo_.begin() + (ptrdiff_t)head + 1);
                head = (size_t)-1;
            }
        }
        fifo_.clear();
    }

private:
    Grid g_;
    std::vector<uint8_t> queued_;
    std::vector<size_t> fifo_;
};

// cut_boxes (src/world.rs:735-833): every box holding a newly blocked cell is
// shrunk along the single direction keeping the most volume, or to its own
// cell; counts come from a summed-volume table over the new barriers.
void cut_boxes(std::vector<Extents>& field, const std::vector<uint8_t>& barrier, const Grid& g,
               const std::vector<std::array<uint32_t, 3>>& fresh, Worklist& work) {
    uint32_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = fresh[0][a]; hi[a] = fresh[0][a]; }
    for (const auto& c : fresh)
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], c[a]); hi[a] = std::max(hi[a], c[a]); }
    Grid t{hi[0] - lo[0] + 2, hi[1] - lo[1] + 2, hi[2] - lo[2] + 2};
    std::vector<uint32_t> sat(t.size(), 0);
    for (const auto& c : fresh) sat[t.index(c[0] - lo[0] + 1, c[1] - lo[1] + 1, c[2] - lo[2] + 1)] += 1;
    for (int axis = 0; axis < 3; ++axis) {
        size_t stride = axis == 0 ? 1 : (axis == 1 ? t.w : (size_t)t.w * t.h);
        for (size_t i = 0; i < sat.size(); ++i) {
            int32_t c[3];
            t.coords(i, c);
            if (c[axis] > 0) sat[i] += sat[i - stride];
        }
    }
    auto count = [&](const int64_t a0[3], const int64_t b0[3]) -> int64_t {
        int64_t a[3], b[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = std::max<int64_t>(a0[k], lo[k]);
            b[k] = std::min<int64_t>(b0[k], hi[k]);
            if (a[k] > b[k]) return 0;
        }
        for (int k = 0; k < 3; ++k) { a[k] -= lo[k]; b[k] = b[k] - lo[k] + 1; }
        auto at = [&](int64_t x, int64_t y, int64_t z) { return (int64_t)sat[t.index((uint32_t)x, (uint32_t)y, (uint32_t)z)]; };
        return at(b[0], b[1], b[2]) - at(a[0], b[1], b[2]) - at(b[0], a[1], b[2]) - at(b[0], b[1], a[2]) + at(a[0], a[1], b[2]) +
               at(a[0], b[1], a[2]) + at(b[0], a[1], a[2]) - at(a[0], a[1], a[2]);
    };
    auto box = [](const Extents& e, const int32_t c[3], int64_t mn[3], int64_t mx[3]) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = (int64_t)c[a] - e[a * 2];
            mx[a] = (int64_t)c[a] + e[a * 2 + 1];
        }
    };
    const Extents zero{0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < g.size(); ++i) {
        if (barrier[i] || field[i] == zero) continue;
        int32_t c[3];
        g.coords(i, c);
        int64_t mn[3], mx[3];
        box(field[i], c, mn, mx);
        if (count(mn, mx) == 0) continue;
        bool have = false;
        uint64_t best_volume = 0;
        Extents best = zero;
        for (int d = 0; d < 6; ++d) {
            auto clear_at = [&](uint8_t v) {
                Extents e = field[i];
                e[d] = v;
                int64_t a[3], b[3];
                box(e, c, a, b);
                return count(a, b) == 0;
            };
            if (!clear_at(0)) continue;
            uint8_t good = 0, bad = field[i][d];
            while (bad - good > 1) {
                uint8_t mid = (uint8_t)(good + (bad - good) / 2);
                if (clear_at(mid)) good = mid;
                else bad = mid;
            }
            Extents e = field[i];
            e[d] = good;
            uint64_t volume = (uint64_t)(e[0] + e[1] + 1) * (uint64_t)(e[2] + e[3] + 1) * (uint64_t)(e[4] + e[5] + 1);
            if (!have || volume > best_volume) {
                have = true;
                best_volume = volume;
                best = e;
            }
        }
        field[i] = have ? best : zero;
        work.push(i);
    }
}

}  // namespace

TopLevelField TopLevelField::updated(const int32_t lo_[3], const int32_t hi_[3], bool any,
                                     const std::function<bool(int32_t, int32_t, int32_t)>& blocked,
                                     const std::vector<RegionKey>& changed) const {
    TopLevelField out;
    if (!any) return out;
    out.present = true;
    for (int a = 0; a < 3; ++a) {
        out.lo[a] = lo_[a];
        out.hi[a] = hi_[a];
        out.dim[a] = (uint32_t)(hi_[a] - lo_[a] + 1);
    }
    Grid g{out.dim[0], out.dim[1], out.dim[2]};
    if (std::max(g.w, std::max(g.h, g.d)) > 255 || (uint64_t)g.w * g.h * g.d > (4ull << 20)) return out;
    out.enabled = true;
    Worklist work(g);
    const bool in_place = enabled && !cells.empty() && lo[0] == lo_[0] && lo[1] == lo_[1] && lo[2] == lo_[2] && dim[0] == g.w &&
                          dim[1] == g.h && dim[2] == g.d;
    if (in_place) {
        out.cells = cells;
        out.barrier = barrier;
    } else {
        out.cells.assign(g.size(), Extents{0, 0, 0, 0, 0, 0});
        out.barrier.assign(g.size(), 1);
        const bool kept = enabled && !cells.empty();
        for (size_t i = 0; i < g.size(); ++i) {
            int32_t c[3];
            g.coords(i, c);
            int32_t wx = c[0] + lo_[0], wy = c[1] + lo_[1], wz = c[2] + lo_[2];
            if (kept && wx >= lo[0] && wy >= lo[1] && wz >= lo[2] && wx <= hi[0] && wy <= hi[1] && wz <= hi[2]) {
                Grid og{dim[0], dim[1], dim[2]};
                size_t old = og.index(wx - lo[0], wy - lo[1], wz - lo[2]);
                out.barrier[i] = barrier[old];
                Extents e = cells[old];
                uint32_t below[3] = {(uint32_t)c[0], (uint32_t)c[1], (uint32_t)c[2]};
                uint32_t above[3] = {g.w - 1 - c[0], g.h - 1 - c[1], g.d - 1 - c[2]};
                for (int a = 0; a < 3; ++a) {
                    e[a * 2] = (uint8_t)std::min<uint32_t>(e[a * 2], std::min<uint32_t>(below[a], 255));
                    e[a * 2 + 1] = (uint8_t)std::min<uint32_t>(e[a * 2 + 1], std::min<uint32_t>(above[a], 255));
                }
                out.cells[i] = e;
            } else {
                out.barrier[i] = blocked(wx, wy, wz) ? 1 : 0;
                if (!out.barrier[i]) work.touch(i);
            }
        }
    }
    std::vector<std::array<uint32_t, 3>> fresh;
    for (const RegionKey& k : changed) {
        if (k.x < lo_[0] || k.y < lo_[1] || k.z < lo_[2] || k.x > hi_[0] || k.y > hi_[1] || k.z > hi_[2]) continue;
        size_t i = g.index(k.x - lo_[0], k.y - lo_[1], k.z - lo_[2]);
        uint8_t now = blocked(k.x, k.y, k.z) ? 1 : 0;
        if (now == out.barrier[i]) continue;
        out.barrier[i] = now;
        if (now) {
            out.cells[i] = Extents{0, 0, 0, 0, 0, 0};
            fresh.push_back({(uint32_t)(k.x - lo_[0]), (uint32_t)(k.y - lo_[1]), (uint32_t)(k.z - lo_[2])});
        } else {
            work.touch(i);
        }
    }
    if (!fresh.empty()) cut_boxes(out.cells, out.barrier, g, fresh, work);
    work.drain(out.cells, out.barrier);
    return out;
}

Extents TopLevelField::at(int32_t x, int32_t y, int32_t z) const {
    if (!enabled) return Extents{0, 0, 0, 0, 0, 0};
    Grid g{dim[0], dim[1], dim[2]};
    return cells[g.index(x - lo[0], y - lo[1], z - lo[2])];
}

std::vector<int32_t> region_grid(const int32_t* directory, uint64_t slots, const int32_t lo[3], const int32_t hi[3], uint64_t max_cells) {
    std::vector<int32_t> grid;
    if (slots == 0) return grid;
    uint64_t cells = 1;
    for (int a = 0; a < 3; ++a) {
        if (hi[a] < lo[a]) return grid;
        cells *= (uint64_t)((int64_t)hi[a] - lo[a] + 1);
        if (cells > max_cells) return grid;
    }
    grid.assign(cells, -1);
    const uint64_t mask = slots - 1;
    size_t i = 0;
    for (int32_t z = lo[2]; z <= hi[2]; ++z)
        for (int32_t y = lo[1]; y <= hi[1]; ++y)
            for (int32_t x = lo[0]; x <= hi[0]; ++x, ++i) {
                uint64_t slot = host_hash_voxel(x, y, z) & mask;
                for (uint32_t attempt = 0; attempt < 32u; ++attempt) {
                    const int32_t* e = directory + slot * 4;
                    if (e[3] == -1) break;
                    if (e[0] == x && e[1] == y && e[2] == z) {
                        grid[i] = e[3];
                        break;
                    }
                    slot = (slot + 1) & mask;
                }
            }
    return grid;
}

std::vector<int32_t> build_directory(const std::vector<RegionKey>& keys) {
    size_t capacity = 1;
    while (capacity < keys.size() * 2) capacity <<= 1;
    for (;;) {
        std::vector<int32_t> dir(capacity * 4, 0);
        for (size_t i = 0; i < capacity; ++i) dir[i * 4 + 3] = -1;
        bool fits = true;
        for (size_t h = 0; h < keys.size(); ++h) {
            size_t slot = host_hash_voxel(keys[h].x, keys[h].y, keys[h].z) & (capacity - 1);
            size_t distance = 0;
            while (dir[slot * 4 + 3] != -1) {
                slot = (slot + 1) & (capacity - 1);
                ++distance;
            }
            if (distance >= 32) {
                fits = false;
                break;
            }
            dir[slot * 4] = keys[h].x;
            dir[slot * 4 + 1] = keys[h].y;
            dir[slot * 4 + 2] = keys[h].z;
            dir[slot * 4 + 3] = (int32_t)h;
        }
        if (fits) return dir;
        capacity *= 2;
    }
}

std::vector<int32_t> build_directory(const std::vector<std::pair<RegionKey, uint32_t>>& entries) {
    size_t capacity = 1;
    while (capacity < entries.size() * 2) capacity <<= 1;
    for (;;) {
        std::vector<int32_t> dir(capacity * 4, 0);
        for (size_t i = 0; i < capacity; ++i) dir[i * 4 + 3] = -1;
        bool fits = true;
        for (const auto& e : entries)
            if (!directory_insert(dir, e.first, e.second)) {
                fits = false;
                break;
            }
        if (fits) return dir;
        capacity *= 2;
    }
}

bool directory_insert(std::vector<int32_t>& dir, const RegionKey& key, uint32_t header) {
    const size_t mask = dir.size() / 4 - 1;
    size_t slot = host_hash_voxel(key.x, key.y, key.z) & mask;
    size_t distance = 0;
    while (dir[slot * 4 + 3] != -1) {
        slot = (slot + 1) & mask;
        if (++distance >= 32) return false;
    }
    dir[slot * 4] = key.x;
    dir[slot * 4 + 1] = key.y;
    dir[slot * 4 + 2] = key.z;
    dir[slot * 4 + 3] = (int32_t)header;
    return true;
}

bool directory_remove(std::vector<int32_t>& dir, const RegionKey& key) {
    const size_t mask = dir.size() / 4 - 1;
    auto at = [&](size_t s) { return RegionKey{dir[s * 4], dir[s * 4 + 1], dir[s * 4 + 2]}; };
    size_t slot = host_hash_voxel(key.x, key.y, key.z) & mask;
    for (size_t probe = 0;; ++probe) {
        if (dir[slot * 4 + 3] == -1 || probe > mask) return false;
        if (at(slot) == key) break;
        slot = (slot + 1) & mask;
    }
    dir[slot * 4 + 3] = -1;
    dir[slot * 4] = dir[slot * 4 + 1] = dir[slot * 4 + 2] = 0;
    size_t hole = slot, next = slot;
    for (;;) {
        next = (next + 1) & mask;
        if (dir[next * 4 + 3] == -1) return true;
        const RegionKey k = at(next);
        const size_t home = host_hash_voxel(k.x, k.y, k.z) & mask;
        // The entry stays when its home lies cyclically in (hole, next].
        const bool stays = hole <= next ? (hole < home && home <= next) : (hole < home || home <= next);
        if (!stays) {
            std::copy(dir.begin() + next * 4, dir.begin() + next * 4 + 4, dir.begin() + hole * 4);
            dir[next * 4 + 3] = -1;
            dir[next * 4] = dir[next * 4 + 1] = dir[next * 4 + 2] = 0;
            hole = next;
        }
    }
}

namespace {
struct FaceHash {
    std::vector<std::array<uint32_t, 4>> slots;
    size_t used = 0;
    static constexpr uint32_t kEmpty = 0xffffffffu;
    explicit FaceHash(size_t capacity) : slots(capacity, {0u, 0u, 0u, kEmpty}) {}
    size_t home(int32_t x, int32_t y, int32_t z, uint32_t face) const {
        return (host_hash_voxel(x, y, z) ^ host_pcg(face + 1u)) & (slots.size() - 1);
    }
    void put(int32_t x, int32_t y, int32_t z, uint32_t face, uint32_t slot) {
        const size_t mask = slots.size() - 1;
        for (size_t j = home(x, y, z, face);; j = (j + 1) & mask) {
            auto& e = slots[j];
            if (e[3] == kEmpty) break;
            if ((int32_t)e[0] == x && (int32_t)e[1] == y && (int32_t)e[2] == z && (e[3] >> 29) == face) {
                e[3] = (face << 29) | slot;
                return;
            }
        }
        if ((used + 1) * 2 > slots.size()) {
            std::vector<std::array<uint32_t, 4>> old(slots.size() * 2, {0u, 0u, 0u, kEmpty});
            old.swap(slots);
            used = 0;
            for (const auto& e : old)
                if (e[3] != kEmpty) put((int32_t)e[0], (int32_t)e[1], (int32_t)e[2], e[3] >> 29, e[3] & 0x1fffffffu);
        }
        size_t j = home(x, y, z, face);
        while (slots[j][3] != kEmpty) j = (j + 1) & (slots.size() - 1);
        slots[j] = {(uint32_t)x, (uint32_t)y, (uint32_t)z, (face << 29) | slot};
        ++used;
    }
};
}  // namespace

std::vector<uint32_t> build_face_index(const std::vector<std::array<int32_t, 4>>& faces) {
    FaceHash h(1024);
    for (size_t s = 0; s < faces.size(); ++s) h.put(faces[s][0], faces[s][1], faces[s][2], (uint32_t)faces[s][3], (uint32_t)s);
    std::vector<uint32_t> out((h.slots.size() + 1) * 4);
    out[0] = (uint32_t)(h.slots.size() - 1);
    out[1] = 64;
    out[2] = 0;
    out[3] = 0;
    std::memcpy(out.data() + 4, h.slots.data(), h.slots.size() * 16);
    return out;
}

namespace {
uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

struct Emitter {
    int32_t v[3];
    uint32_t face, material;
    float cumulative, probability;
};
struct TreeNode {
    float lo[3], power, hi[3];
    uint32_t normals;
    int32_t pivot[3];
    uint32_t pivot_face, left, right, axis;
};

const int kFaceOffset[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// tree::build (src/emission/tree.rs:28-75)
uint32_t tree_split(std::vector<TreeNode>& nodes, std::vector<uint32_t>& order, size_t lo, size_t hi, const std::vector<Emitter>& em) {
    const uint32_t self = (uint32_t)nodes.size();
    TreeNode node{};
    for (int a = 0; a < 3; ++a) {
        node.lo[a] = INFINITY;
        node.hi[a] = -INFINITY;
    }
    for (size_t k = lo; k < hi; ++k) {
        const Emitter& e = em[order[k]];
        const uint32_t axis = e.face / 2;
        for (int a = 0; a < 3; ++a) {
            // face_point(face, 0.5, 0.5) and the square's half extent
            float tangent = (a == 0) ? (axis == 0 ? 0.0f : 1.0f) : (a == 1 ? (axis == 0 ? 1.0f : 0.0f) : 0.0f);
            float bitangent = (a == 0) ? 0.0f : (a == 1 ? (axis == 2 ? 1.0f : 0.0f) : (axis == 2 ? 0.0f : 1.0f));
            float n = (float)kFaceOffset[e.face][a];
            float centre = ((((float)e.v[a] + 0.5f) + n * 0.5f) + tangent * (0.5f - 0.5f)) + bitangent * (0.5f - 0.5f);
            float half = (1.0f - std::fabs(n)) * 0.5f;
            float low = centre - half, high = centre + half;
            node.lo[a] = node.lo[a] < low ? node.lo[a] : low;
            node.hi[a] = node.hi[a] > high ? node.hi[a] : high;
        }
        node.power = node.power + e.probability;
        node.normals |= 1u << e.face;
    }
    nodes.push_back(node);
    if (hi - lo == 1) {
        node.left = 0xffffffffu;
        node.right = order[lo];
    } else {
        const float ex = node.hi[0] - node.lo[0], ey = node.hi[1] - node.lo[1], ez = node.hi[2] - node.lo[2];
        node.axis = (ex >= ey && ex >= ez) ? 0u : (ey >= ez ? 1u : 2u);
        const uint32_t a0 = node.axis, a1 = (node.axis + 1) % 3, a2 = (node.axis + 2) % 3;
        std::sort(order.begin() + (ptrdiff_t)lo, order.begin() + (ptrdiff_t)hi, [&](uint32_t p, uint32_t q) {
            return std::make_tuple(em[p].v[a0], em[p].v[a1], em[p].v[a2], em[p].face) <
                   std::make_tuple(em[q].v[a0], em[q].v[a1], em[q].v[a2], em[q].face);
        });
        const size_t mid = lo + (hi - lo) / 2;
        const Emitter& pv = em[order[mid]];
        node.pivot[0] = pv.v[0];
        node.pivot[1] = pv.v[1];
        node.pivot[2] = pv.v[2];
        node.pivot_face = pv.face;
        node.left = tree_split(nodes, order, lo, mid, em);
        node.right = tree_split(nodes, order, mid, hi, em);
    }
    nodes[self] = node;
    return self;
}
}  // namespace

EmitterWords build_emitters(const std::vector<RegionKey>& keys, const uint16_t* voxels, const float* materials,
                            const std::vector<uint8_t>* live) {
    EmitterWords out;
    float weight[256];
    bool any = false;
    for (int m = 0; m < 256; ++m) {
        weight[m] = materials[m * 16 + 13];
        any = any || weight[m] > 0.0f;
    }
    auto held = [&](uint32_t r) { return !live || (*live)[r] != 0; };
    std::unordered_map<RegionKey, uint32_t, RegionKeyHash> where;
    for (uint32_t r = 0; r < keys.size(); ++r)
        if (held(r)) where[keys[r]] = r;
    std::vector<Emitter> em;
    double total = 0.0;
    if (any) {
        std::vector<uint32_t> order;
        for (uint32_t r = 0; r < keys.size(); ++r) {
            if (!held(r)) continue;
            const uint16_t* m = voxels + (size_t)r * 4096;
            bool emits = false;
            for (int i = 0; i < 4096 && !emits; ++i) emits = m[i] != 256 && weight[m[i]] > 0.0f;
            if (emits) order.push_back(r);
        }
        std::sort(order.begin(), order.end(), [&](uint32_t p, uint32_t q) {
            return std::make_tuple(keys[p].z, keys[p].y, keys[p].x) < std::make_tuple(keys[q].z, keys[q].y, keys[q].x);
        });
        for (uint32_t r : order) {
            const uint16_t* m = voxels + (size_t)r * 4096;
            for (int32_t i = 0; i < 4096; ++i) {
                const uint16_t mat = m[i];
                if (mat == 256 || weight[mat] <= 0.0f) continue;
                const int32_t v[3] = {keys[r].x * 16 + (i & 15), keys[r].y * 16 + ((i >> 4) & 15), keys[r].z * 16 + (i >> 8)};
                for (uint32_t f = 0; f < 6; ++f) {
                    const int32_t n[3] = {v[0] + kFaceOffset[f][0], v[1] + kFaceOffset[f][1], v[2] + kFaceOffset[f][2]};
                    auto it = where.find(RegionKey{n[0] >> 4, n[1] >> 4, n[2] >> 4});
                    if (it != where.end() && voxels[(size_t)it->second * 4096 + (n[0] & 15) + 16 * ((n[1] & 15) + 16 * (n[2] & 15))] != 256)
                        continue;
                    total += (double)weight[mat];
                    em.push_back(Emitter{{v[0], v[1], v[2]}, f, mat, (float)total, weight[mat]});
                }
            }
        }
    }
    if (total == 0.0) em.clear();
    const float total_weight = (float)total;
    for (Emitter& e : em) {
        e.cumulative = e.cumulative / total_weight;
        e.probability = e.probability / total_weight;
    }
    if (!em.empty()) em.back().cumulative = 1.0f;
    std::vector<TreeNode> nodes;
    if (em.size() >= 32) {
        std::vector<uint32_t> order(em.size());
        for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
        tree_split(nodes, order, 0, order.size(), em);
    }
    const size_t records = em.empty() ? 1 : em.size();
    out.words.assign(records * 8 + nodes.size() * 16, 0u);
    for (size_t i = 0; i < em.size(); ++i) {
        uint32_t* w = out.words.data() + i * 8;
        w[0] = (uint32_t)em[i].v[0];
        w[1] = (uint32_t)em[i].v[1];
        w[2] = (uint32_t)em[i].v[2];
        w[3] = em[i].face;
        w[4] = fbits(em[i].cumulative);
        w[5] = fbits(em[i].probability);
        w[6] = fbits((float)em[i].material);
        w[7] = fbits((float)nodes.size());
    }
    for (size_t i = 0; i < nodes.size(); ++i) {
        uint32_t* w = out.words.data() + records * 8 + i * 16;
        const TreeNode& t = nodes[i];
        w[0] = fbits(t.lo[0]);
        w[1] = fbits(t.lo[1]);
        w[2] = fbits(t.lo[2]);
        w[3] = fbits(t.power);
        w[4] = fbits(t.hi[0]);
        w[5] = fbits(t.hi[1]);
        w[6] = fbits(t.hi[2]);
        w[7] = t.normals;
        w[8] = (uint32_t)t.pivot[0];
        w[9] = (uint32_t)t.pivot[1];
        w[10] = (uint32_t)t.pivot[2];
        w[11] = t.pivot_face;
        w[12] = t.left;
        w[13] = t.right;
        w[14] = t.axis;
        w[15] = 0u;
    }
    out.faces = (uint32_t)em.size();
    out.total_weight = em.empty() ? 0.0f : total_weight;
    return out;
}

}  // namespace vgi

// ---- C entry points of the host runtime (include/vgi.h) -------------------
extern "C" {

int64_t vgi_host_emitters(const int32_t* coords, uint32_t n, const uint16_t* voxels, const float* materials, uint32_t* out,
                          uint64_t capacity, uint32_t* info2) {
    std::vector<vgi::RegionKey> keys(n);
    for (uint32_t r = 0; r < n; ++r) keys[r] = vgi::RegionKey{coords[r * 3], coords[r * 3 + 1], coords[r * 3 + 2]};
    vgi::EmitterWords e = vgi::build_emitters(keys, voxels, materials);
    if (info2) {
        info2[0] = e.faces;
        std::memcpy(&info2[1], &e.total_weight, 4);
    }
    if (out && capacity >= e.words.size()) std::memcpy(out, e.words.data(), e.words.size() * 4);
    return (int64_t)e.words.size();
}

int64_t vgi_host_face_index(const int32_t* faces, uint32_t n, uint32_t* out, uint64_t capacity4) {
    std::vector<std::array<int32_t, 4>> keys(n);
    for (uint32_t s = 0; s < n; ++s) keys[s] = {faces[s * 4], faces[s * 4 + 1], faces[s * 4 + 2], faces[s * 4 + 3]};
    std::vector<uint32_t> index = vgi::build_face_index(keys);
    if (out && capacity4 >= index.size() / 4) std::memcpy(out, index.data(), index.size() * 4);
    return (int64_t)(index.size() / 4);
}

int vgi_host_top_level(const int32_t* coords, const uint8_t* solid, uint32_t n, uint8_t* out6, uint64_t capacity) {
    std::unordered_map<vgi::RegionKey, uint32_t, vgi::RegionKeyHash> where;
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (uint32_t r = 0; r < n; ++r) {
        where[vgi::RegionKey{coords[r * 3], coords[r * 3 + 1], coords[r * 3 + 2]}] = r;
        for (int a = 0; a < 3; ++a) {
            if (r == 0 || coords[r * 3 + a] < lo[a]) lo[a] = coords[r * 3 + a];
            if (r == 0 || coords[r * 3 + a] > hi[a]) hi[a] = coords[r * 3 + a];
        }
    }
    vgi::TopLevelField t = vgi::TopLevelField{}.updated(
        lo, hi, n > 0,
        [&](int32_t x, int32_t y, int32_t z) {
            auto it = where.find(vgi::RegionKey{x, y, z});
            return it == where.end() || solid[it->second] != 0;
        },
        {});
    if (!t.enabled) return 1;
    if (capacity < t.cells.size() * 6) return -1;
    for (size_t i = 0; i < t.cells.size(); ++i)
        for (int k = 0; k < 6; ++k) out6[i * 6 + k] = t.cells[i][k];
    return 0;
}

}  // extern "C"
