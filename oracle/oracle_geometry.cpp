// TEST INFRASTRUCTURE ONLY (the oracle). CPU restatement of the reference's
// NAADF construction and GPU packing, used by tests/ as the checker of the
// CUDA upload/edit path and to produce parity scenes. Never linked by the
// product library.
//
// Follows (paths within nathanaelneveux/global-illumination):
//   crates/bevy_voxel_gi/src/naadf.rs:37-148        build_aadf / try_grow
//   crates/bevy_voxel_gi/src/world.rs:243-319       NaadfRegion::build (classification)
//   crates/bevy_voxel_gi/src/world.rs:352-384       brick_voxel_bounds / brick_bounds
//   crates/bevy_voxel_gi/src/world.rs:477-583       TopLevelAadf::updated
//   crates/bevy_voxel_gi/src/world.rs:717-913       clip / cut_boxes / Growth
//   crates/bevy_voxel_gi/src/gpu_scene.rs:72-309    PackedScene::update (full build)
//   crates/bevy_voxel_gi/src/gpu_scene.rs:311-335   intern_brick (deduplication)
//   crates/bevy_voxel_gi/src/gpu_scene.rs:411-471   rebuild_directory, pack_bytes, pack_extents, hash_region
#include "oracle.h"

#include <algorithm>
#include <array>
#include <deque>
#include <map>
#include <set>
#include <vector>

namespace orc {

static const uint16_t AIR = 256;

uint32_t pcg(uint32_t value) {
    uint32_t state = value * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
uint32_t hash_voxel(int32_t x, int32_t y, int32_t z) {
    return pcg(pcg(pcg((uint32_t)x) ^ (uint32_t)y) ^ (uint32_t)z);
}

// ---- naadf.rs:37-148 -------------------------------------------------------
using Aadf = std::array<uint8_t, 6>;  // NEG_X, POS_X, NEG_Y, POS_Y, NEG_Z, POS_Z

static inline size_t lin(uint32_t x, uint32_t y, uint32_t z, uint32_t sx, uint32_t sy) {
    return (size_t)x + (size_t)sx * ((size_t)y + (size_t)sy * z);
}

static void try_grow(Aadf& current, int32_t nx, int32_t ny, int32_t nz, int direction,
                     uint32_t sx, uint32_t sy, uint32_t sz, const std::vector<uint8_t>& blocked,
                     const std::vector<Aadf>& source) {
    if (nx < 0 || ny < 0 || nz < 0 || nx >= (int32_t)sx || ny >= (int32_t)sy || nz >= (int32_t)sz) return;
    if (current[direction] == 255) return;
    size_t ni = lin(nx, ny, nz, sx, sy);
    if (blocked[ni]) return;
    const Aadf& nb = source[ni];
    int opposite = direction ^ 1;
    for (int b = 0; b < 6; ++b)
        if (b != opposite && nb[b] < current[b]) return;
    current[direction] += 1;
}

std::vector<Aadf> build_aadf(uint32_t sx, uint32_t sy, uint32_t sz, const std::vector<uint8_t>& blocked) {
    size_t n = (size_t)sx * sy * sz;
    std::vector<Aadf> source(n, Aadf{0, 0, 0, 0, 0, 0});
    bool all_blocked = true, all_empty = true;
    for (size_t i = 0; i < n; ++i) { if (blocked[i]) all_empty = false; else all_blocked = false; }
    if (all_blocked) return source;
    if (all_empty) {
        for (uint32_t z = 0; z < sz; ++z)
            for (uint32_t y = 0; y < sy; ++y)
                for (uint32_t x = 0; x < sx; ++x)
                    source[lin(x, y, z, sx, sy)] = Aadf{(uint8_t)x, (uint8_t)(sx - x - 1), (uint8_t)y,
                                                        (uint8_t)(sy - y - 1), (uint8_t)z, (uint8_t)(sz - z - 1)};
        return source;
    }
    std::vector<Aadf> destination = source;
    uint32_t rounds = std::max(sx, std::max(sy, sz));
    rounds = rounds > 0 ? rounds - 1 : 0;
    for (uint32_t round = 0; round < rounds; ++round) {
        for (int axis = 0; axis < 3; ++axis) {
            for (uint32_t z = 0; z < sz; ++z)
                for (uint32_t y = 0; y < sy; ++y)
                    for (uint32_t x = 0; x < sx; ++x) {
                        size_t i = lin(x, y, z, sx, sy);
                        if (blocked[i]) { destination[i] = Aadf{0, 0, 0, 0, 0, 0}; continue; }
                        Aadf current = source[i];
                        int dx = axis == 0, dy = axis == 1, dz = axis == 2;
                        try_grow(current, (int)x - dx, (int)y - dy, (int)z - dz, axis * 2, sx, sy, sz, blocked, source);
                        try_grow(current, (int)x + dx, (int)y + dy, (int)z + dz, axis * 2 + 1, sx, sy, sz, blocked, source);
                        destination[i] = current;
                    }
            std::swap(source, destination);
        }
    }
    return source;
}

static uint32_t pack_extents(const Aadf& f) {
    uint32_t bits = 0;
    for (int i = 0; i < 6; ++i) bits |= (uint32_t)f[i] << (i * 2);
    return bits;
}
static uint32_t pack_bytes3(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 8) | (z << 16); }

// ---- world.rs:717-913: top-level field ------------------------------------
struct TopLevel {
    bool any = false;      // any regions at all
    bool enabled = false;  // fields present (size within limits)
    int32_t mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    uint32_t size[3] = {0, 0, 0};
    std::vector<Aadf> fields;
    std::vector<uint8_t> blocked;
};

struct Growth {
    uint32_t sx, sy, sz;
    std::deque<size_t> queue;
    std::vector<uint8_t> queued;
    Growth(uint32_t x, uint32_t y, uint32_t z) : sx(x), sy(y), sz(z), queued((size_t)x * y * z, 0) {}
    void push(size_t i) { if (!queued[i]) { queued[i] = 1; queue.push_back(i); } }
    void cell(size_t i, int32_t& x, int32_t& y, int32_t& z) const {
        x = (int32_t)(i % sx); y = (int32_t)((i / sx) % sy); z = (int32_t)(i / ((size_t)sx * sy));
    }
    void touch(size_t i) {
        push(i);
        int32_t x, y, z; cell(i, x, y, z);
        for (int d = 0; d < 6; ++d) {
            int32_t n[3] = {x, y, z};
            n[d / 2] += (d % 2 == 0) ? -1 : 1;
            if (n[0] >= 0 && n[1] >= 0 && n[2] >= 0 && n[0] < (int32_t)sx && n[1] < (int32_t)sy && n[2] < (int32_t)sz)
                push(lin(n[0], n[1], n[2], sx, sy));
        }
    }
    void run(std::vector<Aadf>& fields, const std::vector<uint8_t>& blocked) {
        while (!queue.empty()) {
            size_t i = queue.front(); queue.pop_front();
            queued[i] = 0;
            if (blocked[i]) continue;
            int32_t x, y, z; cell(i, x, y, z);
            Aadf current = fields[i];
            for (int d = 0; d < 6; ++d) {
                int32_t n[3] = {x, y, z};
                n[d / 2] += (d % 2 == 0) ? -1 : 1;
                try_grow(current, n[0], n[1], n[2], d, sx, sy, sz, blocked, fields);
            }
            if (current != fields[i]) { fields[i] = current; touch(i); }
        }
    }
};

static Aadf clip_field(Aadf f, const uint32_t below[3], const uint32_t above[3]) {
    for (int a = 0; a < 3; ++a) {
        f[a * 2] = std::min<uint32_t>(f[a * 2], std::min<uint32_t>(below[a], 255));
        f[a * 2 + 1] = std::min<uint32_t>(f[a * 2 + 1], std::min<uint32_t>(above[a], 255));
    }
    return f;
}

static void cut_boxes(std::vector<Aadf>& fields, const std::vector<uint8_t>& blocked, const uint32_t size[3],
                      const std::vector<std::array<uint32_t, 3>>& newly, Growth& growth) {
    uint32_t low[3] = {newly[0][0], newly[0][1], newly[0][2]}, high[3] = {newly[0][0], newly[0][1], newly[0][2]};
    for (auto& c : newly)
        for (int a = 0; a < 3; ++a) { low[a] = std::min(low[a], c[a]); high[a] = std::max(high[a], c[a]); }
    uint32_t ts[3];
    for (int a = 0; a < 3; ++a) ts[a] = high[a] - low[a] + 2;
    std::vector<uint32_t> table((size_t)ts[0] * ts[1] * ts[2], 0);
    for (auto& c : newly) table[lin(c[0] - low[0] + 1, c[1] - low[1] + 1, c[2] - low[2] + 1, ts[0], ts[1])] += 1;
    for (int axis = 0; axis < 3; ++axis) {
        size_t step = axis == 0 ? 1 : (axis == 1 ? ts[0] : (size_t)ts[0] * ts[1]);
        for (size_t i = 0; i < table.size(); ++i) {
            size_t co[3] = {i % ts[0], (i / ts[0]) % ts[1], i / ((size_t)ts[0] * ts[1])};
            if (co[axis] > 0) table[i] += table[i - step];
        }
    }
    auto count = [&](const int64_t mn[3], const int64_t mx[3]) -> uint32_t {
        int64_t a[3], b[3];
        for (int k = 0; k < 3; ++k) { a[k] = std::max<int64_t>(mn[k], low[k]); b[k] = std::min<int64_t>(mx[k], high[k]); }
        if (a[0] > b[0] || a[1] > b[1] || a[2] > b[2]) return 0;
        for (int k = 0; k < 3; ++k) { a[k] -= low[k]; b[k] = b[k] - low[k] + 1; }
        auto at = [&](int64_t x, int64_t y, int64_t z) { return (int64_t)table[lin(x, y, z, ts[0], ts[1])]; };
        return (uint32_t)(at(b[0], b[1], b[2]) - at(a[0], b[1], b[2]) - at(b[0], a[1], b[2]) - at(b[0], b[1], a[2]) +
                          at(a[0], a[1], b[2]) + at(a[0], b[1], a[2]) + at(b[0], a[1], a[2]) - at(a[0], a[1], a[2]));
    };
    auto box = [](const Aadf& f, uint32_t x, uint32_t y, uint32_t z, int64_t mn[3], int64_t mx[3]) {
        mn[0] = (int64_t)x - f[0]; mn[1] = (int64_t)y - f[2]; mn[2] = (int64_t)z - f[4];
        mx[0] = (int64_t)x + f[1]; mx[1] = (int64_t)y + f[3]; mx[2] = (int64_t)z + f[5];
    };
    for (uint32_t z = 0; z < size[2]; ++z)
        for (uint32_t y = 0; y < size[1]; ++y)
            for (uint32_t x = 0; x < size[0]; ++x) {
                size_t i = lin(x, y, z, size[0], size[1]);
                if (blocked[i] || fields[i] == Aadf{0, 0, 0, 0, 0, 0}) continue;
                int64_t mn[3], mx[3];
                box(fields[i], x, y, z, mn, mx);
                if (count(mn, mx) == 0) continue;
                bool have = false; uint64_t most = 0; Aadf bestf{};
                for (int d = 0; d < 6; ++d) {
                    auto with = [&](uint8_t e) { Aadf f = fields[i]; f[d] = e; return f; };
                    auto clear = [&](uint8_t e) { int64_t a[3], b[3]; box(with(e), x, y, z, a, b); return count(a, b) == 0; };
                    if (!clear(0)) continue;
                    uint8_t good = 0, bad = fields[i][d];
                    while (bad - good > 1) {
                        uint8_t middle = good + (bad - good) / 2;
                        if (clear(middle)) good = middle; else bad = middle;
                    }
                    Aadf f = with(good);
                    uint64_t volume = (uint64_t)(f[0] + f[1] + 1) * (f[2] + f[3] + 1) * (f[4] + f[5] + 1);
                    if (!have || volume > most) { have = true; most = volume; bestf = f; }
                }
                fields[i] = have ? bestf : Aadf{0, 0, 0, 0, 0, 0};
                growth.push(i);
            }
}

// TopLevelAadf::updated (world.rs:477-583). `is_blocked(cell)` is true for a
// missing region or one with any solid voxel.
template <class Blocked>
static TopLevel top_level_updated(const TopLevel& self, bool any, const int32_t mn[3], const int32_t mx[3],
                                  Blocked is_blocked, const std::vector<std::array<int32_t, 3>>& changed) {
    TopLevel out;
    if (!any) return out;
    out.any = true;
    uint32_t size[3];
    for (int a = 0; a < 3; ++a) { out.mn[a] = mn[a]; out.mx[a] = mx[a]; size[a] = (uint32_t)(mx[a] - mn[a] + 1); out.size[a] = size[a]; }
    uint64_t cells = (uint64_t)size[0] * size[1] * size[2];
    if (std::max(size[0], std::max(size[1], size[2])) > 255 || cells > (4ull << 20)) return out;
    out.enabled = true;
    auto index = [&](int32_t x, int32_t y, int32_t z) { return lin(x - mn[0], y - mn[1], z - mn[2], size[0], size[1]); };
    Growth growth(size[0], size[1], size[2]);
    bool in_place = self.enabled && !self.fields.empty() && self.mn[0] == mn[0] && self.mn[1] == mn[1] && self.mn[2] == mn[2] &&
                    self.size[0] == size[0] && self.size[1] == size[1] && self.size[2] == size[2];
    if (in_place) {
        out.fields = self.fields;
        out.blocked = self.blocked;
    } else {
        out.fields.assign(cells, Aadf{0, 0, 0, 0, 0, 0});
        out.blocked.assign(cells, 1);
        bool kept = self.enabled && !self.fields.empty();
        for (int32_t z = mn[2]; z <= mx[2]; ++z)
            for (int32_t y = mn[1]; y <= mx[1]; ++y)
                for (int32_t x = mn[0]; x <= mx[0]; ++x) {
                    size_t i = index(x, y, z);
                    if (kept && x >= self.mn[0] && y >= self.mn[1] && z >= self.mn[2] && x <= self.mx[0] && y <= self.mx[1] &&
                        z <= self.mx[2]) {
                        size_t old = lin(x - self.mn[0], y - self.mn[1], z - self.mn[2], self.size[0], self.size[1]);
                        out.blocked[i] = self.blocked[old];
                        uint32_t below[3] = {(uint32_t)(x - mn[0]), (uint32_t)(y - mn[1]), (uint32_t)(z - mn[2])};
                        uint32_t above[3] = {(uint32_t)(mx[0] - x), (uint32_t)(mx[1] - y), (uint32_t)(mx[2] - z)};
                        out.fields[i] = clip_field(self.fields[old], below, above);
                    } else {
                        out.blocked[i] = is_blocked(x, y, z) ? 1 : 0;
                        if (!out.blocked[i]) growth.touch(i);
                    }
                }
    }
    std::vector<std::array<uint32_t, 3>> newly;
    for (auto& c : changed) {
        if (c[0] < mn[0] || c[1] < mn[1] || c[2] < mn[2] || c[0] > mx[0] || c[1] > mx[1] || c[2] > mx[2]) continue;
        size_t i = index(c[0], c[1], c[2]);
        uint8_t now = is_blocked(c[0], c[1], c[2]) ? 1 : 0;
        if (now == out.blocked[i]) continue;
        out.blocked[i] = now;
        if (now) {
            out.fields[i] = Aadf{0, 0, 0, 0, 0, 0};
            newly.push_back({(uint32_t)(c[0] - mn[0]), (uint32_t)(c[1] - mn[1]), (uint32_t)(c[2] - mn[2])});
        } else {
            growth.touch(i);
        }
    }
    if (!newly.empty()) cut_boxes(out.fields, out.blocked, size, newly, growth);
    growth.run(out.fields, out.blocked);
    return out;
}

// ---- world.rs:243-384 + gpu_scene.rs:174-239: one region -----------------
struct RegionPack {
    uint32_t kind;       // 1 air, 2 uniform solid, 3 mixed
    uint32_t material;   // kinds 1, 2
    bool any_solid;
    uint32_t table[64];  // kind 3: brick words with the pointer field holding a brick ordinal
    std::vector<std::array<uint32_t, 32>> bricks;  // kind 3: mixed brick payloads in table order
};

static RegionPack classify_region(const uint16_t* m) {
    RegionPack r{};
    bool all_air = true, all_same = true;
    for (int i = 0; i < 4096; ++i) {
        if (m[i] != AIR) all_air = false;
        if (m[i] != m[0]) all_same = false;
    }
    if (all_air) { r.kind = 1; r.material = AIR; r.any_solid = false; return r; }
    if (all_same) { r.kind = 2; r.material = m[0]; r.any_solid = true; return r; }
    r.kind = 3;
    auto mat = [&](uint32_t x, uint32_t y, uint32_t z) { return m[x + 16 * (y + 16 * z)]; };
    std::vector<uint8_t> occupied(64, 0);
    for (uint32_t b = 0; b < 64; ++b) {
        uint32_t bx = b & 3, by = (b >> 2) & 3, bz = b >> 4;
        for (uint32_t v = 0; v < 64; ++v)
            if (mat(bx * 4 + (v & 3), by * 4 + ((v >> 2) & 3), bz * 4 + (v >> 4)) != AIR) occupied[b] = 1;
    }
    r.any_solid = std::any_of(occupied.begin(), occupied.end(), [](uint8_t o) { return o != 0; });
    std::vector<Aadf> brick_bounds = build_aadf(4, 4, 4, occupied);
    for (uint32_t b = 0; b < 64; ++b) {
        uint32_t bx = b & 3, by = (b >> 2) & 3, bz = b >> 4;
        uint16_t first = mat(bx * 4, by * 4, bz * 4);
        bool uniform = true;
        std::vector<uint8_t> blocked(64);
        for (uint32_t v = 0; v < 64; ++v) {
            uint16_t mv = mat(bx * 4 + (v & 3), by * 4 + ((v >> 2) & 3), bz * 4 + (v >> 4));
            uniform = uniform && mv == first;
            blocked[v] = mv != AIR;
        }
        if (uniform && first == AIR) {
            r.table[b] = pack_extents(brick_bounds[b]) << 2;
        } else if (uniform) {
            r.table[b] = ((uint32_t)first << 2) | 1u;
        } else {
            std::vector<Aadf> vb = build_aadf(4, 4, 4, blocked);
            std::array<uint32_t, 32> data{};
            for (uint32_t v = 0; v < 64; ++v) {
                uint16_t mv = mat(bx * 4 + (v & 3), by * 4 + ((v >> 2) & 3), bz * 4 + (v >> 4));
                uint32_t cell = mv == AIR ? (pack_extents(vb[v]) << 1) : (((uint32_t)mv << 1) | 1u);
                data[v / 2] |= cell << ((v & 1) * 16);
            }
            r.table[b] = ((uint32_t)r.bricks.size() << 2) | 2u;
            r.bricks.push_back(data);
        }
    }
    return r;
}

struct Scene {
    std::vector<int32_t> directory;  // 4 words per slot
    std::vector<uint32_t> headers;   // 4 words per region
    std::vector<uint32_t> cells;
    int32_t mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    // Inputs kept for material lookups and incremental updates.
    std::vector<std::array<int32_t, 3>> coords;   // header order = sorted (z, y, x)
    std::vector<uint16_t> voxels;                 // 4096 per region, header order
    std::vector<uint8_t> strides;
    std::map<std::array<int32_t, 3>, uint32_t> index;  // key (z, y, x) -> header
    TopLevel top;
    int top_mode = 0;
};

static std::array<int32_t, 3> zyx(int32_t x, int32_t y, int32_t z) { return {z, y, x}; }

// Full packing from scratch (gpu_scene.rs:72-309 on an empty PackedScene):
// keys sorted (z, y, x), headers and payloads allocated in that order, brick
// payloads interned, directory rebuilt at nextpow2(2n) until every probe
// distance is below 32.
static void pack_scene(Scene& s) {
    size_t n = s.coords.size();
    s.headers.assign(n * 4, 0);
    s.cells.clear();
    std::map<std::array<uint32_t, 32>, uint32_t> lookup;
    for (size_t h = 0; h < n; ++h) {
        RegionPack r = classify_region(&s.voxels[h * 4096]);
        auto c = s.coords[h];
        uint32_t negw = 0, posw = 0;
        if (s.top.enabled) {
            size_t i = lin(c[0] - s.top.mn[0], c[1] - s.top.mn[1], c[2] - s.top.mn[2], s.top.size[0], s.top.size[1]);
            const Aadf& f = s.top.fields[i];
            negw = pack_bytes3(f[0], f[2], f[4]);
            posw = pack_bytes3(f[1], f[3], f[5]);
        }
        posw |= (uint32_t)s.strides[h] << 28;
        uint32_t* hd = &s.headers[h * 4];
        if (r.kind != 3) {
            hd[0] = r.kind; hd[1] = r.material; hd[2] = negw; hd[3] = posw;
            continue;
        }
        uint32_t offset = (uint32_t)s.cells.size();
        s.cells.resize(offset + 64, 0);
        uint32_t table[64];
        for (int b = 0; b < 64; ++b) {
            uint32_t w = r.table[b];
            if ((w & 3u) == 2u) {
                const auto& data = r.bricks[w >> 2];
                auto it = lookup.find(data);
                uint32_t ptr;
                if (it != lookup.end()) {
                    ptr = it->second;
                } else {
                    ptr = (uint32_t)s.cells.size();
                    s.cells.insert(s.cells.end(), data.begin(), data.end());
                    lookup.emplace(data, ptr);
                }
                w = (ptr << 2) | 2u;
            }
            table[b] = w;
        }
        std::copy(table, table + 64, s.cells.begin() + offset);
        hd[0] = 3; hd[1] = offset; hd[2] = negw; hd[3] = posw;
    }
    size_t capacity = 1;
    while (capacity < n * 2) capacity <<= 1;
    for (;;) {
        s.directory.assign(capacity * 4, 0);
        for (size_t i = 0; i < capacity; ++i) s.directory[i * 4 + 3] = -1;
        bool fits = true;
        for (size_t h = 0; h < n && fits; ++h) {
            auto c = s.coords[h];
            size_t slot = hash_voxel(c[0], c[1], c[2]) & (capacity - 1);
            size_t distance = 0;
            while (s.directory[slot * 4 + 3] != -1) { slot = (slot + 1) & (capacity - 1); ++distance; }
            if (distance >= 32) { fits = false; break; }
            s.directory[slot * 4 + 0] = c[0]; s.directory[slot * 4 + 1] = c[1];
            s.directory[slot * 4 + 2] = c[2]; s.directory[slot * 4 + 3] = (int32_t)h;
        }
        if (fits) break;
        capacity *= 2;
    }
}

static void scene_bounds(const std::vector<std::array<int32_t, 3>>& coords, int32_t mn[3], int32_t mx[3]) {
    for (int a = 0; a < 3; ++a) { mn[a] = 0; mx[a] = 0; }
    if (coords.empty()) return;
    for (int a = 0; a < 3; ++a) { mn[a] = coords[0][a]; mx[a] = coords[0][a]; }
    for (auto& c : coords)
        for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], c[a]); mx[a] = std::max(mx[a], c[a]); }
}

static bool region_blocked(const Scene& s, int32_t x, int32_t y, int32_t z) {
    auto it = s.index.find(zyx(x, y, z));
    if (it == s.index.end()) return true;
    const uint16_t* m = &s.voxels[(size_t)it->second * 4096];
    for (int i = 0; i < 4096; ++i)
        if (m[i] != AIR) return true;
    return false;
}

static void build_top(Scene& s, const TopLevel& previous, const std::vector<std::array<int32_t, 3>>& changed) {
    int32_t mn[3], mx[3];
    scene_bounds(s.coords, mn, mx);
    for (int a = 0; a < 3; ++a) { s.mn[a] = mn[a]; s.mx[a] = mx[a]; }
    if (s.top_mode == 2 || s.coords.empty()) {
        s.top = TopLevel{};
        s.top.any = !s.coords.empty();
        return;
    }
    auto blocked = [&](int32_t x, int32_t y, int32_t z) { return region_blocked(s, x, y, z); };
    if (s.top_mode == 1) {
        // Synchronous full build (TopLevelAadf::synchronous, world.rs:587-590).
        TopLevel t = top_level_updated(TopLevel{}, true, mn, mx, blocked, {});
        if (t.enabled) t.fields = build_aadf(t.size[0], t.size[1], t.size[2], t.blocked);
        s.top = t;
        return;
    }
    s.top = top_level_updated(previous, true, mn, mx, blocked, changed);
}

}  // namespace orc

using namespace orc;

struct orc_scene { Scene s; };

extern "C" {

int orc_build_aadf(uint32_t sx, uint32_t sy, uint32_t sz, const uint8_t* blocked, uint8_t* out6) {
    std::vector<uint8_t> b(blocked, blocked + (size_t)sx * sy * sz);
    auto f = build_aadf(sx, sy, sz, b);
    for (size_t i = 0; i < f.size(); ++i)
        for (int k = 0; k < 6; ++k) out6[i * 6 + k] = f[i][k];
    return 0;
}

// Packs `n` regions (4096 voxels each, x fastest) at region coordinates
// `coords` (3 ints each). top_mode: 0 = the reference's incremental field
// grown from an empty scene, 1 = synchronous build_aadf, 2 = disabled.
int orc_scene_create(const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides, int top_mode,
                     orc_scene** out) {
    auto* sc = new orc_scene();
    Scene& s = sc->s;
    s.top_mode = top_mode;
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return zyx(coords[a * 3], coords[a * 3 + 1], coords[a * 3 + 2]) < zyx(coords[b * 3], coords[b * 3 + 1], coords[b * 3 + 2]);
    });
    s.coords.resize(n);
    s.voxels.resize((size_t)n * 4096);
    s.strides.assign(n, 0);
    for (uint32_t h = 0; h < n; ++h) {
        uint32_t i = order[h];
        s.coords[h] = {coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]};
        std::copy(voxels + (size_t)i * 4096, voxels + (size_t)(i + 1) * 4096, s.voxels.begin() + (size_t)h * 4096);
        if (strides) s.strides[h] = strides[i];
        if (!s.index.emplace(zyx(s.coords[h][0], s.coords[h][1], s.coords[h][2]), h).second) { delete sc; return -1; }
    }
    build_top(s, TopLevel{}, {});
    pack_scene(s);
    *out = sc;
    return 0;
}

void orc_scene_free(orc_scene* sc) { delete sc; }

// Writes each voxel edit (x, y, z, value) into the scene, then recomputes the
// top-level field incrementally from the previous one over the changed
// regions (TransportScene::with_page_contents, world.rs:1024-1040) and
// repacks. Edits outside loaded regions are ignored.
int orc_scene_edit(orc_scene* sc, const int32_t* edits, uint32_t n) {
    Scene& s = sc->s;
    std::vector<std::array<int32_t, 3>> touched;
    std::map<std::array<int32_t, 3>, bool> before;
    for (uint32_t e = 0; e < n; ++e) {
        int32_t x = edits[e * 4], y = edits[e * 4 + 1], z = edits[e * 4 + 2];
        uint16_t value = (uint16_t)edits[e * 4 + 3];
        int32_t rx = x >> 4, ry = y >> 4, rz = z >> 4;
        auto it = s.index.find(zyx(rx, ry, rz));
        if (it == s.index.end()) continue;
        auto key = zyx(rx, ry, rz);
        if (!before.count(key)) before[key] = region_blocked(s, rx, ry, rz);
        s.voxels[(size_t)it->second * 4096 + (x & 15) + 16 * ((y & 15) + 16 * (z & 15))] = value;
    }
    bool topology_unchanged = true;
    for (auto& kv : before) {
        auto c = std::array<int32_t, 3>{kv.first[2], kv.first[1], kv.first[0]};
        touched.push_back(c);
        if (region_blocked(s, c[0], c[1], c[2]) != kv.second) topology_unchanged = false;
    }
    if (!topology_unchanged && s.top_mode == 0) {
        std::sort(touched.begin(), touched.end(), [](const std::array<int32_t, 3>& a, const std::array<int32_t, 3>& b) {
            return zyx(a[0], a[1], a[2]) < zyx(b[0], b[1], b[2]);
        });
        TopLevel previous = s.top;
        build_top(s, previous, touched);
    } else if (!topology_unchanged) {
        build_top(s, TopLevel{}, {});
    }
    pack_scene(s);
    return 0;
}

// Loads (or replaces) and unloads regions: TransportScene::with_page_contents
// (world.rs:982-1046) with region-sized pages. Removals come first, then
// loads. The touched regions (removed, loaded or replaced) update the
// top-level field incrementally over the new region map (TopLevelAadf::
// updated, world.rs:473-583) unless every touched region keeps its residency
// and emptiness; then the scene is packed again from scratch (the canonical
// form of PackedScene's incremental update equals a full pack, the property
// gpu_scene.rs's lineage test pins). Unloading a region that is not loaded
// does nothing.
int orc_scene_regions(orc_scene* sc, const int32_t* coords, uint32_t n, const uint16_t* voxels, const uint8_t* strides,
                      const int32_t* removed, uint32_t n_removed) {
    Scene& s = sc->s;
    struct Region {
        std::array<int32_t, 3> c;
        std::vector<uint16_t> v;
        uint8_t stride;
    };
    std::map<std::array<int32_t, 3>, Region> regions;  // keyed (z, y, x)
    for (size_t h = 0; h < s.coords.size(); ++h) {
        const auto& c = s.coords[h];
        regions[zyx(c[0], c[1], c[2])] =
            Region{c, std::vector<uint16_t>(s.voxels.begin() + h * 4096, s.voxels.begin() + (h + 1) * 4096), s.strides[h]};
    }
    auto status = [&](const std::array<int32_t, 3>& key) -> int {
        auto it = regions.find(key);
        if (it == regions.end()) return -1;
        for (uint16_t m : it->second.v)
            if (m != AIR) return 1;
        return 0;
    };
    std::map<std::array<int32_t, 3>, int> before;
    std::vector<std::array<int32_t, 3>> touched;
    // build_page_regions keeps the previous region when the page brings the
    // same materials and stride (src/world.rs:1490-1494), and touched.retain
    // drops a key whose region is the same before and after (:1016-1020),
    // even when the same change also removed it.
    std::set<std::array<int32_t, 3>> unchanged;
    for (uint32_t i = 0; i < n; ++i) {
        const auto key = zyx(coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]);
        auto it = regions.find(key);
        if (it == regions.end()) continue;
        if (it->second.stride == (strides ? strides[i] : (uint8_t)0) &&
            std::equal(it->second.v.begin(), it->second.v.end(), voxels + (size_t)i * 4096))
            unchanged.insert(key);
    }
    for (uint32_t i = 0; i < n_removed; ++i) {
        const std::array<int32_t, 3> c{removed[i * 3], removed[i * 3 + 1], removed[i * 3 + 2]};
        const auto key = zyx(c[0], c[1], c[2]);
        if (!regions.count(key)) continue;
        if (!before.count(key)) before[key] = status(key);
        regions.erase(key);
        if (!unchanged.count(key)) touched.push_back(c);
    }
    for (uint32_t i = 0; i < n; ++i) {
        const std::array<int32_t, 3> c{coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]};
        const auto key = zyx(c[0], c[1], c[2]);
        if (!before.count(key)) before[key] = status(key);
        regions[key] = Region{c, std::vector<uint16_t>(voxels + (size_t)i * 4096, voxels + (size_t)(i + 1) * 4096),
                              strides ? strides[i] : (uint8_t)0};
        if (!unchanged.count(key)) touched.push_back(c);
    }
    bool topology_unchanged = true;
    for (const auto& kv : before) {
        const int now = status(kv.first);
        if (kv.second < 0 || now < 0 || kv.second != now) topology_unchanged = false;
    }
    s.coords.clear();
    s.voxels.clear();
    s.strides.clear();
    s.index.clear();
    for (const auto& kv : regions) {
        s.index[kv.first] = (uint32_t)s.coords.size();
        s.coords.push_back(kv.second.c);
        s.voxels.insert(s.voxels.end(), kv.second.v.begin(), kv.second.v.end());
        s.strides.push_back(kv.second.stride);
    }
    if (!topology_unchanged) {
        std::sort(touched.begin(), touched.end(), [](const std::array<int32_t, 3>& a, const std::array<int32_t, 3>& b) {
            return zyx(a[0], a[1], a[2]) < zyx(b[0], b[1], b[2]);
        });
        touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
        if (s.top_mode == 0) {
            TopLevel previous = s.top;
            build_top(s, previous, touched);
        } else {
            build_top(s, TopLevel{}, {});
        }
    }
    pack_scene(s);
    return 0;
}

// sizes: [directory slots, headers, cells]; bounds: min xyz, max xyz.
int orc_scene_info(const orc_scene* sc, uint64_t* sizes, int32_t* bounds) {
    const Scene& s = sc->s;
    sizes[0] = s.directory.size() / 4;
    sizes[1] = s.headers.size() / 4;
    sizes[2] = s.cells.size();
    for (int a = 0; a < 3; ++a) { bounds[a] = s.mn[a]; bounds[3 + a] = s.mx[a]; }
    return 0;
}

int orc_scene_copy(const orc_scene* sc, int32_t* directory, uint32_t* headers, uint32_t* cells) {
    const Scene& s = sc->s;
    std::copy(s.directory.begin(), s.directory.end(), directory);
    std::copy(s.headers.begin(), s.headers.end(), headers);
    std::copy(s.cells.begin(), s.cells.end(), cells);
    return 0;
}

// The top-level field as 6 bytes per cell over the bounds (x fastest), or
// returns 1 when the field is disabled.
int orc_scene_top_level(const orc_scene* sc, uint8_t* out6) {
    const Scene& s = sc->s;
    if (!s.top.enabled) return 1;
    for (size_t i = 0; i < s.top.fields.size(); ++i)
        for (int k = 0; k < 6; ++k) out6[i * 6 + k] = s.top.fields[i][k];
    return 0;
}

// Canonical, layout-free form of a packed scene for each region coordinate in
// `coords`: 4 words (kind, material or 0, negative bytes, positive|stride)
// then, for kind 3, 64 brick records of 33 words (the brick word with its
// pointer cleared, then the 32 payload words for a mixed brick, else zeros).
// A region missing from the directory (within 32 probes) yields kind 0.
int orc_canonical(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                  uint64_t n_cells, const int32_t* coords, uint32_t n, uint32_t* out) {
    const size_t per = 4 + 64 * 33;
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t* o = out + (size_t)r * per;
        std::fill(o, o + per, 0u);
        int32_t x = coords[r * 3], y = coords[r * 3 + 1], z = coords[r * 3 + 2];
        uint64_t mask = slots - 1;
        uint64_t slot = hash_voxel(x, y, z) & mask;
        int64_t found = -1;
        for (int attempt = 0; attempt < 32; ++attempt) {
            const int32_t* e = directory + slot * 4;
            if (e[3] == -1) break;
            if (e[0] == x && e[1] == y && e[2] == z) { found = e[3]; break; }
            slot = (slot + 1) & mask;
        }
        if (found < 0) continue;
        const uint32_t* h = headers + (size_t)found * 4;
        o[0] = h[0]; o[2] = h[2]; o[3] = h[3];
        if (h[0] != 3) { o[1] = h[1]; continue; }
        for (int b = 0; b < 64; ++b) {
            if ((uint64_t)h[1] + b >= n_cells) return -2;
            uint32_t w = cells[h[1] + b];
            uint32_t* rec = o + 4 + b * 33;
            if ((w & 3u) == 2u) {
                rec[0] = 2u;
                uint32_t p = w >> 2;
                if ((uint64_t)p + 32 > n_cells) return -2;
                for (int k = 0; k < 32; ++k) rec[1 + k] = cells[p + k];
            } else {
                rec[0] = w;
            }
        }
    }
    return 0;
}

}  // extern "C"

namespace orc {
const Scene& scene_of(const orc_scene* sc) { return sc->s; }
}
