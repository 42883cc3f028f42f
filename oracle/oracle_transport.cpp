// TEST INFRASTRUCTURE ONLY (the oracle). CPU restatement of the reference's
// WGSL transport: traversal, path estimator, world-space face trace, cache
// gather, accumulation and the proportional edit discount. tests/ compare the
// CUDA kernels with it; bench.py times it as the CPU baseline. The product
// never links it.
//
// Follows (paths within nathanaelneveux/global-illumination):
//   crates/bevy_voxel_gi/shaders/voxel_traversal.wgsl:17-219   traversal
//   crates/bevy_voxel_gi/shaders/voxel_path.wgsl:63-520         estimator
//   crates/bevy_voxel_gi/shaders/voxel_trace.wgsl:25-92         face trace
//   crates/bevy_voxel_gi/shaders/voxel_accumulate.wgsl:83-446   prepare/accumulate/events
//   crates/bevy_voxel_gi/shaders/voxel_retention.wgsl:1-96      resolve_retention
//   crates/bevy_voxel_gi/src/gpu/face_index.rs:22-145           face index
//   crates/bevy_voxel_gi/src/emission.rs:91-165                 emitter distribution
//   crates/bevy_voxel_gi/src/emission/tree.rs:28-75, 173-195    light tree and its words
//
// Every float expression keeps the shader's operation order; see
// oracle_math.h for the builtin semantics.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <map>
#include <atomic>
#include <thread>
#include <unordered_map>
#include <vector>

namespace orc {

struct Geometry {
    const int32_t* directory;
    const uint32_t* headers;
    const uint32_t* cells;
    uint32_t mask;
    int32_t mn[3], mx[3];
};

struct Model {
    const float* params;      // 24 words (GpuParams)
    const float* materials;   // 16 floats per material
    const float* lights;      // 12 floats per light
    const uint32_t* emitters; // uint4 words
    const uint32_t* state;    // 36 words per slot (9 uint4)
    const uint32_t* index;    // uint4 words; [0] = (mask, probes, 0, 0)
    orc_pipeline pipe;
    // MLP termination: the network's value for each (voxel, face) a path may
    // hit; an uncached hit takes it in place of the continuation.
    const struct PredictedFaces* predicted = nullptr;
};

struct Counters {
    uint64_t rays = 0, paths = 0, steps = 0, bytes = 0, unknown = 0, cache_hits = 0;
    uint64_t status[4] = {0, 0, 0, 0};
    uint64_t traverse_bytes = 0;
    // Bytes the traversal reads (directory probes, headers, brick and cell words).
    void tbytes(uint64_t n) {
        bytes += n;
        traverse_bytes += n;
    }
};

struct Ctx {
    Geometry g;
    Model m;
    Counters c;
    uint32_t pcount(int i) const { return fbits(m.params[i]); }   // counts.*
    int32_t pmin(int i) const { return (int32_t)fbits(m.params[4 + i]); }
    int32_t pmax(int i) const { return (int32_t)fbits(m.params[8 + i]); }
    float env(int i) const { return m.params[12 + i]; }
    float extra(int i) const { return m.params[16 + i]; }
    float transport(int i) const { return m.params[20 + i]; }
};

struct RayResult {
    i3 voxel{0, 0, 0};
    uint32_t material = 0;
    f3 position{0, 0, 0};
    uint32_t status = 0;
    f3 normal{0, 0, 0};
};

// ---- voxel_traversal.wgsl ------------------------------------------------
static uint32_t face_index_of(f3 n) {
    if (n.x != 0.0f) return n.x < 0.0f ? 1u : 0u;
    if (n.y != 0.0f) return n.y < 0.0f ? 3u : 2u;
    if (n.z != 0.0f) return n.z < 0.0f ? 5u : 4u;
    return 6u;
}

static uint32_t lookup_region(Ctx& x, i3 c) {
    uint32_t slot = hash_voxel(c.x, c.y, c.z) & x.g.mask;
    for (uint32_t attempt = 0; attempt < 32u; ++attempt) {
        const int32_t* e = x.g.directory + (size_t)slot * 4;
        x.c.tbytes(16);
        if (e[3] == -1) return 0xffffffffu;
        if (e[0] == c.x && e[1] == c.y && e[2] == c.z) return (uint32_t)e[3];
        slot = (slot + 1u) & x.g.mask;
    }
    return 0xffffffffu;
}

static bool in_bounds(const Ctx& x, i3 r) {
    return r.x >= x.g.mn[0] && r.y >= x.g.mn[1] && r.z >= x.g.mn[2] && r.x <= x.g.mx[0] && r.y <= x.g.mx[1] &&
           r.z <= x.g.mx[2];
}

static i3 unpack_bytes(uint32_t v) { return i3{(int32_t)(v & 255u), (int32_t)((v >> 8) & 255u), (int32_t)((v >> 16) & 255u)}; }
static i3 negative_extents(uint32_t b) { return i3{(int32_t)(b & 3u), (int32_t)((b >> 4) & 3u), (int32_t)((b >> 8) & 3u)}; }
static i3 positive_extents(uint32_t b) { return i3{(int32_t)((b >> 2) & 3u), (int32_t)((b >> 6) & 3u), (int32_t)((b >> 10) & 3u)}; }

struct F4 { float x, y, z, w; };
struct PredictedFaces {
    std::unordered_map<uint64_t, F4> map;
    mutable std::atomic<uint64_t> misses{0};  // hits on faces the table does not hold
    mutable std::atomic<uint64_t> last_miss{0};
};
static uint64_t face_key(int32_t x, int32_t y, int32_t z, uint32_t face) {
    return ((uint64_t)(uint16_t)x) | ((uint64_t)(uint16_t)y << 16) | ((uint64_t)(uint16_t)z << 32) | ((uint64_t)face << 48);
}

// voxel_traversal.wgsl:90-107
static F4 advance_box(f3 p, f3 d, i3 cell, i3 ng, i3 ps, float size) {
    float mnv[3] = {(float)(cell.x - ng.x) * size, (float)(cell.y - ng.y) * size, (float)(cell.z - ng.z) * size};
    float mxv[3] = {(float)(cell.x + ps.x + 1) * size, (float)(cell.y + ps.y + 1) * size, (float)(cell.z + ps.z + 1) * size};
    float pp[3] = {p.x, p.y, p.z}, dd[3] = {d.x, d.y, d.z};
    float travel[3];
    for (int a = 0; a < 3; ++a) {
        bool moving = std::fabs(dd[a]) > 1e-8f;
        float plane = dd[a] > 0.0f ? mxv[a] : mnv[a];
        float raw = (plane - pp[a]) / (moving ? dd[a] : 1.0f);
        travel[a] = (moving && raw >= -0.001f && raw < 1e30f) ? raw : 1e30f;
    }
    bool choose_y = travel[1] < wmax(travel[0], 0.0f);
    float distance_xy = wmax(choose_y ? travel[1] : travel[0], 0.0f);
    bool choose_z = travel[2] < distance_xy;
    float distance = wmax(choose_z ? travel[2] : distance_xy, 0.0f);
    float axis[3] = {0.0f, 0.0f, 0.0f};
    if (choose_z) axis[2] = 1.0f; else if (choose_y) axis[1] = 1.0f; else axis[0] = 1.0f;
    float nrm[3];
    for (int a = 0; a < 3; ++a) nrm[a] = distance < 1e30f ? axis[a] * (dd[a] > 0.0f ? -1.0f : 1.0f) : 0.0f;
    return F4{nrm[0], nrm[1], nrm[2], wmax(distance + 0.001f, 0.001f)};
}

// voxel_traversal.wgsl:108-121
static bool geometry_ahead(Ctx& x, f3 start, f3 dir, float max_distance) {
    f3 position = start;
    float remaining = max_distance;
    for (uint32_t step = 0; step < 2048u; ++step) {
        x.c.steps += 1;
        f3 q = divs(position, 16.0f);
        i3 region{f2i(std::floor(q.x)), f2i(std::floor(q.y)), f2i(std::floor(q.z))};
        if (remaining < 0.0f || !in_bounds(x, region)) return false;
        uint32_t index = lookup_region(x, region);
        if (index != 0xffffffffu) {
            x.c.tbytes(16);
            if (x.g.headers[(size_t)index * 4] != 1u) return true;
        }
        float travel = advance_box(position, dir, region, i3{0, 0, 0}, i3{0, 0, 0}, 16.0f).w;
        position = add(position, muls(dir, travel));
        remaining = remaining - travel;
    }
    return true;
}

// voxel_traversal.wgsl:126-219
static RayResult trace_domain_limited(Ctx& x, f3 origin, f3 dir, float max_distance, bool visible_geometry,
                                      uint32_t max_steps) {
    x.c.rays += 1;
    RayResult result;
    float nearv = -1e30f, farv = 1e30f;
    f3 normal{0.0f, 0.0f, 0.0f};
    float mnv[3] = {(float)x.pmin(0) * 16.0f, (float)x.pmin(1) * 16.0f, (float)x.pmin(2) * 16.0f};
    float mxv[3] = {(float)(x.pmax(0) + 1) * 16.0f, (float)(x.pmax(1) + 1) * 16.0f, (float)(x.pmax(2) + 1) * 16.0f};
    float oo[3] = {origin.x, origin.y, origin.z}, dd[3] = {dir.x, dir.y, dir.z};
    for (int a = 0; a < 3; ++a) {
        if (std::fabs(dd[a]) <= 1e-8f) {
            if (oo[a] < mnv[a] || oo[a] > mxv[a]) { x.c.status[0] += 1; return result; }
            continue;
        }
        float first = (mnv[a] - oo[a]) / dd[a];
        float second = (mxv[a] - oo[a]) / dd[a];
        if (wmin(first, second) > nearv) {
            nearv = wmin(first, second);
            normal = f3{0.0f, 0.0f, 0.0f};
            setc(normal, a, first < second ? -1.0f : 1.0f);
        }
        farv = wmin(farv, wmax(first, second));
    }
    if (farv < wmax(nearv, 0.0f)) { x.c.status[0] += 1; return result; }
    float distance = wmax(nearv, 0.0f) + 0.001f;
    f3 position = add(origin, muls(dir, distance));
    i3 last_region{0x7fffffff, 0x7fffffff, 0x7fffffff};
    uint32_t meta[4] = {0, 0, 0, 0};
    for (uint32_t step = 0; step < max_steps; ++step) {
        x.c.steps += 1;
        if (distance > max_distance) { x.c.status[0] += 1; return result; }
        i3 voxel{f2i(std::floor(position.x)), f2i(std::floor(position.y)), f2i(std::floor(position.z))};
        i3 region{voxel.x >> 4, voxel.y >> 4, voxel.z >> 4};
        if (!in_bounds(x, region)) { x.c.status[0] += 1; return result; }
        if (last_region.x != region.x || last_region.y != region.y || last_region.z != region.z) {
            uint32_t index = lookup_region(x, region);
            if (index == 0xffffffffu) {
                if (visible_geometry) {
                    F4 adv = advance_box(position, dir, region, i3{0, 0, 0}, i3{0, 0, 0}, 16.0f);
                    distance = distance + adv.w;
                    position = add(position, muls(dir, adv.w));
                    normal = f3{adv.x, adv.y, adv.z};
                    continue;
                }
                result.status = geometry_ahead(x, position, dir, max_distance - distance) ? 2u : 0u;
                x.c.status[result.status] += 1;
                return result;
            }
            x.c.tbytes(16);
            const uint32_t* h = x.g.headers + (size_t)index * 4;
            meta[0] = h[0]; meta[1] = h[1]; meta[2] = h[2]; meta[3] = h[3];
            last_region = region;
        }
        F4 adv{0.0f, 0.0f, 0.0f, 0.0f};
        if (meta[0] == 1u) {
            adv = advance_box(position, dir, region, unpack_bytes(meta[2]), unpack_bytes(meta[3]), 16.0f);
        } else {
            uint32_t material = meta[1];
            if (meta[0] == 3u) {
                uint32_t lx = (uint32_t)(voxel.x & 15), ly = (uint32_t)(voxel.y & 15), lz = (uint32_t)(voxel.z & 15);
                uint32_t bx = lx / 4u, by = ly / 4u, bz = lz / 4u;
                uint32_t brick_data = x.g.cells[meta[1] + (bz * 4u + by) * 4u + bx];
                x.c.tbytes(4);
                uint32_t state = brick_data & 3u;
                if (state == 0u) {
                    uint32_t ext = brick_data >> 2u;
                    adv = advance_box(position, dir, i3{region.x * 4 + (int32_t)bx, region.y * 4 + (int32_t)by, region.z * 4 + (int32_t)bz},
                                      negative_extents(ext), positive_extents(ext), 4.0f);
                    material = 256u;
                } else if (state == 1u) {
                    material = brick_data >> 2u;
                } else {
                    uint32_t ix = lx & 3u, iy = ly & 3u, iz = lz & 3u;
                    uint32_t idx = (iz * 4u + iy) * 4u + ix;
                    uint32_t word = x.g.cells[(brick_data >> 2u) + idx / 2u];
                    x.c.tbytes(4);
                    uint32_t cell = (word >> ((idx & 1u) * 16u)) & 65535u;
                    material = (cell & 1u) != 0u ? (cell >> 1u) : 256u;
                    if (material == 256u) {
                        uint32_t ext = cell >> 1u;
                        adv = advance_box(position, dir, voxel, negative_extents(ext), positive_extents(ext), 1.0f);
                    }
                }
            }
            if (material != 256u) {
                result.voxel = voxel;
                result.material = material;
                result.position = position;
                result.normal = normal;
                result.status = 1u;
                x.c.status[1] += 1;
                return result;
            }
        }
        distance = distance + adv.w;
        position = add(position, muls(dir, adv.w));
        normal = f3{adv.x, adv.y, adv.z};
    }
    result.status = 2u;
    result.material = 0xffffffffu;
    x.c.status[2] += 1;
    return result;
}

// ---- voxel_path.wgsl -------------------------------------------------------
struct Energy { F4 value{0, 0, 0, 0}; f3 custom{0, 0, 0}; };

static F4 f4add(F4 a, F4 b) { return F4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
static F4 f4mul(F4 a, F4 b) { return F4{a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
static F4 f4muls(F4 a, float s) { return F4{a.x * s, a.y * s, a.z * s, a.w * s}; }
static F4 f4divs(F4 a, float s) { return F4{a.x / s, a.y / s, a.z / s, a.w / s}; }
static F4 ld4(const float* p) { return F4{p[0], p[1], p[2], p[3]}; }

static F4 material_diffuse(Ctx& x, uint32_t m) { x.c.bytes += 64; return ld4(x.m.materials + (size_t)m * 16); }
static const float* material(Ctx& x, uint32_t m) { x.c.bytes += 64; return x.m.materials + (size_t)m * 16; }

struct Emissive { i3 voxel; uint32_t face; F4 sampling; };
static Emissive load_emitter(Ctx& x, uint32_t index) {
    x.c.bytes += 32;
    const uint32_t* a = x.m.emitters + (size_t)index * 8;
    return Emissive{i3{(int32_t)a[0], (int32_t)a[1], (int32_t)a[2]}, a[3], F4{bitsf(a[4]), bitsf(a[5]), bitsf(a[6]), bitsf(a[7])}};
}
struct LightNode { F4 minimum_power; f3 maximum; uint32_t normals; i3 pivot; uint32_t face; uint32_t children[4]; };
static LightNode load_node(Ctx& x, uint32_t index) {
    x.c.bytes += 64;
    uint32_t offset = f2u(x.extra(3)) * 2u + index * 4u;
    const uint32_t* w = x.m.emitters + (size_t)offset * 4;
    LightNode n;
    n.minimum_power = F4{bitsf(w[0]), bitsf(w[1]), bitsf(w[2]), bitsf(w[3])};
    n.maximum = f3{bitsf(w[4]), bitsf(w[5]), bitsf(w[6])};
    n.normals = w[7];
    n.pivot = i3{(int32_t)w[8], (int32_t)w[9], (int32_t)w[10]};
    n.face = w[11];
    for (int i = 0; i < 4; ++i) n.children[i] = w[12 + i];
    return n;
}

static f3 face_normal(uint32_t face) {
    f3 n{0.0f, 0.0f, 0.0f};
    setc(n, (int)(face / 2u), (face & 1u) != 0u ? -1.0f : 1.0f);
    return n;
}

// voxel_path.wgsl:108-122
static float node_importance(const LightNode& node, f3 position, f3 normal) {
    f3 mnp{node.minimum_power.x, node.minimum_power.y, node.minimum_power.z};
    f3 delta = sub(muls(add(mnp, node.maximum), 0.5f), position);
    float radius = length(sub(node.maximum, mnp)) * 0.5f;
    float distance = wmax(length(delta), 1e-5f);
    f3 direction = divs(delta, distance);
    float spread = wmin(radius / distance, 1.0f);
    float receiver = wclamp(dot(normal, direction) + spread, 0.0f, 1.0f);
    f3 nd = neg(direction);
    float positive[3] = {(node.normals & 1u) ? nd.x : -1.0f, (node.normals & 4u) ? nd.y : -1.0f, (node.normals & 16u) ? nd.z : -1.0f};
    float negative[3] = {(node.normals & 2u) ? direction.x : -1.0f, (node.normals & 8u) ? direction.y : -1.0f,
                         (node.normals & 32u) ? direction.z : -1.0f};
    float projected[3];
    for (int a = 0; a < 3; ++a) projected[a] = wmax(positive[a], negative[a]);
    float emitter = wclamp(wmax(wmax(projected[0], projected[1]), projected[2]) + spread, 0.0f, 1.0f);
    return node.minimum_power.w * receiver * emitter / (distance * distance + radius * radius + 0.25f);
}

// voxel_path.wgsl:123-131
static float node_left_probability(Ctx& x, const LightNode& node, f3 position, f3 normal) {
    LightNode left = load_node(x, node.children[0]);
    LightNode right = load_node(x, node.children[1]);
    float power = left.minimum_power.w / (left.minimum_power.w + right.minimum_power.w);
    float a = node_importance(left, position, normal);
    float b = node_importance(right, position, normal);
    if (a + b <= 1e-20f) return wclamp(power, 1e-6f, 0.999999f);
    return wclamp(0.05f * power + 0.95f * a / (a + b), 1e-6f, 0.999999f);
}

// voxel_path.wgsl:132-149
static Emissive tree_emitter(Ctx& x, f3 position, f3 normal, float choice) {
    uint32_t index = 0;
    float uniform = choice;
    float probability = 1.0f;
    for (;;) {
        LightNode node = load_node(x, index);
        if (node.children[0] == 0xffffffffu) {
            Emissive e = load_emitter(x, node.children[1]);
            e.sampling.y = probability;
            return e;
        }
        float p = node_left_probability(x, node, position, normal);
        if (uniform < p) { probability = probability * p; uniform = uniform / p; index = node.children[0]; }
        else { probability = probability * (1.0f - p); uniform = (uniform - p) / (1.0f - p); index = node.children[1]; }
        uniform = wmin(uniform, bitsf(0x3f7fffffu));
    }
}

// voxel_path.wgsl:150-174
static bool key_less(i3 voxel, uint32_t face, const LightNode& node) {
    uint32_t axis = node.children[2];
    for (uint32_t j = 0; j < 3u; ++j) {
        int i = (int)((axis + j) % 3u);
        if (compi(voxel, i) != compi(node.pivot, i)) return compi(voxel, i) < compi(node.pivot, i);
    }
    return face < node.face;
}
static float tree_probability(Ctx& x, f3 position, f3 normal, i3 voxel, f3 hit_normal) {
    uint32_t face = 0;
    for (uint32_t i = 0; i < 6u; ++i) {
        f3 fn = face_normal(i);
        if (fn.x == hit_normal.x && fn.y == hit_normal.y && fn.z == hit_normal.z) face = i;
    }
    uint32_t index = 0;
    float probability = 1.0f;
    for (;;) {
        LightNode node = load_node(x, index);
        if (node.children[0] == 0xffffffffu) {
            Emissive found = load_emitter(x, node.children[1]);
            bool same = found.voxel.x == voxel.x && found.voxel.y == voxel.y && found.voxel.z == voxel.z && found.face == face;
            return same ? probability : 0.0f;
        }
        float p = node_left_probability(x, node, position, normal);
        if (key_less(voxel, face, node)) { probability = probability * p; index = node.children[0]; }
        else { probability = probability * (1.0f - p); index = node.children[1]; }
    }
}

// voxel_path.wgsl:178-213
static uint32_t scramble_reverse(uint32_t input, uint32_t seed) {
    uint32_t v = input;
    v ^= v * 0x3d20adeau;
    v += seed;
    v *= (seed >> 16u) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return v;
}
static float sample_1d(uint32_t stream, uint32_t sequence, uint32_t dimension) {
    if (dimension < 12u) {
        static const uint32_t primes[12] = {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u};
        uint32_t base = primes[dimension];
        uint32_t index = (sequence & 0x00ffffffu) + 1u;
        float scale = 1.0f, value = 0.0f;
        while (index != 0u) {
            scale = scale / (float)base;
            value = value + (float)(index % base) * scale;
            index = index / base;
        }
        float rotation = (float)(pcg(stream ^ pcg(dimension)) >> 9u) / 8388608.0f;
        return fract(value + rotation);
    }
    uint32_t seed = pcg(stream ^ pcg(dimension / 2u));
    uint32_t index = reverse_bits(scramble_reverse(reverse_bits(sequence), pcg(seed ^ 0x79c68e4au)));
    if ((dimension & 1u) != 0u) {
        index ^= (index >> 1u) & 0x55555555u;
        index ^= (index >> 2u) & 0x33333333u;
        index ^= (index >> 4u) & 0x0f0f0f0fu;
        index ^= (index >> 8u) & 0x00ff00ffu;
        index ^= (index >> 16u) & 0x0000ffffu;
    }
    uint32_t value = reverse_bits(scramble_reverse(index, pcg(seed ^ pcg(dimension))));
    return (float)(value >> 9u) / 8388608.0f;
}
// voxel_path.wgsl:218-224
static float continuation_sample(uint32_t stream, uint32_t sequence, uint32_t bounce, uint32_t dimension) {
    if (bounce < 3u) {
        uint32_t legacy = dimension == 2u ? 8u + bounce : 2u + bounce * 2u + dimension;
        return sample_1d(stream, sequence, legacy);
    }
    return sample_1d(stream, sequence, 16u + (bounce - 3u) * 3u + dimension);
}

// voxel_path.wgsl:231-238
static f3 hemisphere(f3 n, float u, float v) {
    f3 tangent;
    if (std::fabs(n.z) < 0.999f) tangent = normalize(cross(n, f3{0.0f, 0.0f, 1.0f}));
    else tangent = normalize(cross(n, f3{0.0f, 1.0f, 0.0f}));
    f3 bitangent = cross(n, tangent);
    float phi = 6.28318530718f * u;
    float s, c;
    own_sincos(phi, &s, &c);
    return add(add(muls(tangent, c * std::sqrt(v)), muls(bitangent, s * std::sqrt(v))), muls(n, std::sqrt(1.0f - v)));
}

// voxel_path.wgsl:239-243
static RayResult trace(Ctx& x, f3 origin, f3 dir, float max_distance) {
    RayResult r = trace_domain_limited(x, origin, dir, max_distance, x.m.pipe.budgeted != 0, x.m.pipe.path_steps);
    if (x.m.pipe.budgeted && r.status == 2u && r.material == 0xffffffffu) r.status = 0u;
    return r;
}
static float connection_reach(const Ctx& x) { return x.m.pipe.limited_reach ? x.transport(0) : x.extra(1); }

// voxel_path.wgsl:271-282
static RayResult trace_diffuse(Ctx& x, f3 origin, f3 dir) {
    float reach = connection_reach(x);
    RayResult r = trace(x, origin, dir, reach);
    if (x.m.pipe.limited_reach && r.status == 0u &&
        geometry_ahead(x, add(origin, muls(dir, reach)), dir, x.extra(1) - reach))
        r.status = 3u;
    return r;
}

// voxel_path.wgsl:283-307
static Energy direct_at(Ctx& x, f3 position, f3 normal) {
    Energy e;
    f3 origin = add(position, muls(normal, 0.002f));
    uint32_t count = x.pcount(3);
    for (uint32_t i = 0; i < count; ++i) {
        const float* L = x.m.lights + (size_t)i * 12;
        x.c.bytes += 48;
        f3 pos{L[0], L[1], L[2]};
        float distance = x.extra(1);
        float attenuation = 1.0f;
        f3 direction;
        if (L[3] >= 0.0f) {
            f3 delta = sub(pos, position);
            float d2 = dot(delta, delta);
            if (d2 <= 0.0000001f || d2 > L[3] * L[3]) continue;
            distance = std::sqrt(d2);
            direction = divs(delta, distance);
            distance = distance - 0.004f;
            attenuation = 1.0f / wmax(d2, 1.0f);
        } else {
            direction = normalize(pos);
        }
        float cosine = wmax(dot(normal, direction), 0.0f);
        if (cosine > 0.0f && trace(x, origin, direction, distance).status == 0u) {
            float k = cosine * attenuation;
            e.value = f4add(e.value, F4{L[4] * k, L[5] * k, L[6] * k, L[7] * k});
            e.custom = add(e.custom, f3{L[9] * k, L[10] * k, L[11] * k});
        }
    }
    return e;
}

// voxel_path.wgsl:309-324
static Emissive choose_emitter(Ctx& x, f3 position, f3 normal, float choice) {
    uint32_t count = f2u(x.extra(3));
    if (load_emitter(x, 0).sampling.w > 0.0f) return tree_emitter(x, position, normal, choice);
    uint32_t low = 0, high = count;
    while (low < high) {
        uint32_t middle = (low + high) / 2u;
        if (load_emitter(x, middle).sampling.x <= choice) low = middle + 1u;
        else high = middle;
    }
    return load_emitter(x, umin(low, count - 1u));
}

static float cosine_pdf(f3 n, f3 d) { return wmax(dot(n, d), 0.0f) / 3.14159265359f; }

// voxel_path.wgsl:332-364
static Energy sample_emitter(Ctx& x, f3 position, f3 normal, uint32_t source_stream, uint32_t sequence, uint32_t bounce) {
    Energy result;
    if (x.extra(3) == 0.0f) return result;
    uint32_t stream = source_stream ^ pcg(bounce + 0xa341316cu);
    Emissive em = choose_emitter(x, position, normal, sample_1d(stream, sequence, 12u));
    f3 en = face_normal(em.face);
    uint32_t axis = em.face / 2u;
    f3 tangent = axis == 0u ? f3{0.0f, 1.0f, 0.0f} : f3{1.0f, 0.0f, 0.0f};
    f3 bitangent = axis == 2u ? f3{0.0f, 1.0f, 0.0f} : f3{0.0f, 0.0f, 1.0f};
    f3 lp = add(add(add(adds(tof(em.voxel), 0.5f), muls(en, 0.5f)), muls(tangent, sample_1d(stream, sequence, 13u) - 0.5f)),
                muls(bitangent, sample_1d(stream, sequence, 14u) - 0.5f));
    f3 delta = sub(lp, position);
    float d2 = dot(delta, delta);
    float reach = connection_reach(x);
    if (d2 < 0.0001f || d2 > reach * reach) return result;
    float distance = std::sqrt(d2);
    f3 direction = divs(delta, distance);
    float receiver_cosine = wmax(dot(normal, direction), 0.0f);
    float emitter_cosine = wmax(dot(en, neg(direction)), 0.0f);
    if (receiver_cosine <= 0.0f || emitter_cosine <= 0.0f || em.sampling.y <= 0.0f) return result;
    float light_pdf = em.sampling.y * d2 / emitter_cosine;
    float directional_pdf = receiver_cosine / 3.14159265359f;
    f3 shadow_origin = add(position, muls(normal, 0.002f));
    f3 shadow_delta = sub(add(lp, muls(en, 0.002f)), shadow_origin);
    float shadow_distance = length(shadow_delta);
    if (trace(x, shadow_origin, divs(shadow_delta, shadow_distance), shadow_distance).status != 0u) return result;
    const float* mat = material(x, f2u(em.sampling.z));
    float factor = directional_pdf / (light_pdf + directional_pdf);
    result.value = f4muls(ld4(mat + 8), factor);
    return result;
}

// voxel_path.wgsl:368-394
static Energy sample_terminal_emission(Ctx& x, f3 position, f3 normal, uint32_t stream, uint32_t sequence, uint32_t bounce) {
    Energy result;
    if (x.extra(3) == 0.0f) return result;
    if (continuation_sample(stream, sequence, bounce, 2u) < 0.5f) {
        result = sample_emitter(x, position, normal, stream, sequence, bounce + 1u);
        result.value = f4muls(result.value, 2.0f);
        return result;
    }
    f3 direction = hemisphere(normal, continuation_sample(stream, sequence, bounce, 0u), continuation_sample(stream, sequence, bounce, 1u));
    if (dot(normal, direction) <= 0.0f) return result;
    RayResult hit = trace(x, add(position, muls(normal, 0.002f)), direction, connection_reach(x));
    if (hit.status != 1u) return result;
    const float* mat = material(x, hit.material);
    float power = mat[13];
    f3 delta = sub(hit.position, position);
    float d2 = dot(delta, delta);
    float reach = connection_reach(x);
    if (power == 0.0f || d2 < 0.0001f || d2 > reach * reach) return result;
    float selection_pdf = power / wmax(x.extra(2), 1e-20f);
    if (load_emitter(x, 0).sampling.w > 0.0f) selection_pdf = tree_probability(x, position, normal, hit.voxel, hit.normal);
    float light_pdf = selection_pdf * d2 / wmax(dot(hit.normal, neg(direction)), 1e-8f);
    float directional_pdf = cosine_pdf(normal, direction);
    float factor = 2.0f * directional_pdf / (directional_pdf + light_pdf);
    result.value = f4muls(ld4(mat + 8), factor);
    return result;
}

// voxel_path.wgsl:63-87, with the gather reading the slot's 16-byte cache
// record (mean rgb, count word) instead of two state words.
struct Cached { bool found; F4 value; };
static Cached cached_energy(Ctx& x, i3 voxel, uint32_t face) {
    Cached c{false, F4{0, 0, 0, 0}};
    if (face > 5u || !x.m.index) return c;
    const uint32_t* header = x.m.index;
    uint32_t mask = header[0];
    uint32_t slot = (hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u)) & mask;
    for (uint32_t attempt = 0; attempt < header[1]; ++attempt) {
        const uint32_t* e = x.m.index + (size_t)(slot + 1u) * 4;
        x.c.bytes += 16;
        if (e[3] == 0xffffffffu) return c;
        if ((int32_t)e[0] == voxel.x && (int32_t)e[1] == voxel.y && (int32_t)e[2] == voxel.z && (e[3] >> 29u) == face) {
            uint32_t base = (e[3] & 0x1fffffffu) * 9u;
            const uint32_t* words = x.m.state + (size_t)(base + 1u) * 4;
            x.c.bytes += 16;
            if (words[1] < 16u || (words[1] & 0x80000000u) != 0u) return c;
            const uint32_t* m = x.m.state + (size_t)base * 4;
            c.found = true;
            c.value = F4{bitsf(m[0]), bitsf(m[1]), bitsf(m[2]), bitsf(m[3])};
            return c;
        }
        slot = (slot + 1u) & mask;
    }
    return c;
}

struct PathEnergy { Energy energy; bool unknown = false; RayResult first_hit; };
struct PathState {
    PathEnergy result;
    F4 throughput{1.0f, 1.0f, 1.0f, 1.0f};
    f3 origin, direction, previous_position, previous_normal;
    float previous_pdf = 0.0f;
    uint32_t bounce = 0;
    bool done = false;
};

// voxel_path.wgsl:418-428
static PathState begin_path(f3 start, f3 direction, f3 normal) {
    PathState s;
    s.origin = start;
    s.direction = direction;
    s.previous_normal = normal;
    s.previous_pdf = cosine_pdf(normal, direction);
    s.previous_position = sub(start, muls(normal, 0.001f));
    s.done = s.previous_pdf <= 0.0f;
    return s;
}

// voxel_path.wgsl:429-492
static PathState advance_path(Ctx& x, PathState state, uint32_t stream, uint32_t sequence, uint32_t steps, bool terminal) {
    if (state.done) return state;
    for (uint32_t step = 0; step < steps; ++step) {
        uint32_t bounce = state.bounce;
        state.done = true;
        RayResult hit = trace_diffuse(x, state.origin, state.direction);
        if (bounce == 0u) state.result.first_hit = hit;
        if (hit.status == 0u) {
            float horizon = wclamp(state.direction.y * 0.35f + 0.65f, 0.15f, 1.0f);
            F4 env{x.env(0), x.env(1), x.env(2), x.env(3)};
            state.result.energy.value = f4add(state.result.energy.value, f4muls(f4mul(state.throughput, env), horizon));
            break;
        }
        if (hit.status == 2u) { state.result.unknown = true; break; }
        if (hit.status == 3u) break;
        const float* mat = material(x, hit.material);
        F4 diffuse = ld4(mat), emission = ld4(mat + 8);
        Energy direct = direct_at(x, hit.position, hit.normal);
        float emission_weight = mat[13];
        f3 delta = sub(hit.position, state.origin);
        float selection_pdf = emission_weight / wmax(x.extra(2), 1e-20f);
        if (emission_weight > 0.0f && x.extra(3) > 0.0f && load_emitter(x, 0).sampling.w > 0.0f)
            selection_pdf = tree_probability(x, state.previous_position, state.previous_normal, hit.voxel, hit.normal);
        float light_pdf = selection_pdf * dot(delta, delta) / wmax(dot(hit.normal, neg(state.direction)), 1e-8f);
        float mis = 1.0f;
        if (light_pdf > 0.0f) mis = state.previous_pdf / (state.previous_pdf + light_pdf);
        Cached cached = cached_energy(x, hit.voxel, face_index_of(hit.normal));
        if (cached.found) {
            x.c.cache_hits += 1;
            F4 term = f4add(f4muls(emission, mis), f4mul(diffuse, f4add(direct.value, cached.value)));
            state.result.energy.value = f4add(state.result.energy.value, f4mul(state.throughput, term));
            break;
        }
        if (x.m.predicted) {
            // The GPU's MLP cache mode (no reference counterpart): the
            // network's prediction for the hit face ends the path.
            auto it = x.m.predicted->map.find(face_key(hit.voxel.x, hit.voxel.y, hit.voxel.z, face_index_of(hit.normal)));
            const bool missing = it == x.m.predicted->map.end();
            if (missing) {
                x.m.predicted->misses += 1;
                x.m.predicted->last_miss = face_key(hit.voxel.x, hit.voxel.y, hit.voxel.z, face_index_of(hit.normal));
            }
            const F4 value = missing ? F4{0, 0, 0, 0} : it->second;
            F4 term = f4add(f4muls(emission, mis), f4mul(diffuse, f4add(direct.value, value)));
            state.result.energy.value = f4add(state.result.energy.value, f4mul(state.throughput, term));
            break;
        }
        Energy nee;
        if (terminal && step + 1u == steps) nee = sample_terminal_emission(x, hit.position, hit.normal, stream, sequence, bounce);
        else nee = sample_emitter(x, hit.position, hit.normal, stream, sequence, bounce + 1u);
        F4 term = f4add(f4muls(emission, mis), f4mul(diffuse, f4add(direct.value, nee.value)));
        state.result.energy.value = f4add(state.result.energy.value, f4mul(state.throughput, term));
        if (terminal && step + 1u == steps) break;
        state.throughput = f4mul(state.throughput, diffuse);
        float maximum = wmax(state.throughput.x, wmax(state.throughput.y, state.throughput.z));
        if (maximum == 0.0f) break;
        if (bounce >= 1u) {
            float survival = wclamp(maximum, 0.1f, 0.95f);
            if (continuation_sample(stream, sequence, bounce, 2u) > survival) break;
            state.throughput = f4divs(state.throughput, survival);
        }
        state.origin = add(hit.position, muls(hit.normal, 0.002f));
        state.previous_position = hit.position;
        state.previous_normal = hit.normal;
        state.direction = hemisphere(hit.normal, continuation_sample(stream, sequence, bounce, 0u), continuation_sample(stream, sequence, bounce, 1u));
        state.previous_pdf = cosine_pdf(hit.normal, state.direction);
        if (state.previous_pdf <= 0.0f) break;
        state.bounce += 1u;
        state.done = false;
    }
    return state;
}

// voxel_path.wgsl:504-520
struct ReceiverSample { F4 energy; bool known; };
static ReceiverSample trace_receiver(Ctx& x, f3 surface, f3 normal, uint32_t stream, uint32_t sequence) {
    x.c.paths += 1;
    f3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
    Energy emitter = sample_emitter(x, surface, normal, stream, sequence, 0u);
    PathEnergy continuation;
    if (dot(normal, direction) > 0.0f) {
        PathState st = begin_path(add(surface, muls(normal, 0.001f)), direction, normal);
        continuation = advance_path(x, st, stream, sequence, x.m.pipe.diffuse_hits, true).result;
    }
    ReceiverSample r;
    r.known = !continuation.unknown;
    r.energy = f4add(emitter.value, continuation.energy.value);
    if (continuation.unknown) x.c.unknown += 1;
    return r;
}

// voxel_trace.wgsl:44-59 (one lane's strided subsequence)
struct Moments { F4 mean{0, 0, 0, 0}; F4 second{0, 0, 0, 0}; uint32_t known = 0; };
static Moments trace_moments(Ctx& x, const uint32_t* task, uint32_t first, uint32_t step) {
    Moments m;
    i3 voxel{(int32_t)task[0], (int32_t)task[1], (int32_t)task[2]};
    f3 normal = face_normal(task[3]);
    f3 surface = add(adds(tof(voxel), 0.5f), muls(normal, 0.5f));
    uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(task[3] + 1u);
    for (uint32_t i = first; i < x.pcount(1); i += step) {
        ReceiverSample s = trace_receiver(x, surface, normal, stream, task[4] + i);
        if (!s.known) continue;
        m.mean = f4add(m.mean, s.energy);
        m.second = f4add(m.second, f4mul(s.energy, s.energy));
        m.known += 1u;
    }
    return m;
}

// voxel_trace.wgsl:25-37
static void write_result(Ctx& x, const uint32_t* task, const Moments& m, uint32_t* out) {
    f3 normal = face_normal(task[3]);
    i3 voxel{(int32_t)task[0], (int32_t)task[1], (int32_t)task[2]};
    Energy direct = direct_at(x, add(adds(tof(voxel), 0.5f), muls(normal, 0.5f)), normal);
    float inverse = 1.0f / (float)umax(m.known, 1u);
    F4 mean = f4muls(m.mean, inverse), second = f4muls(m.second, inverse);
    float vals[24] = {mean.x, mean.y, mean.z, mean.w, 0.0f, (float)m.known, 0.0f, 0.0f,
                      second.x, second.y, second.z, second.w, 0.0f, 0.0f, 0.0f, 0.0f,
                      direct.value.x, direct.value.y, direct.value.z, direct.value.w,
                      0.0f, direct.custom.x, direct.custom.y, direct.custom.z};
    for (int i = 0; i < 24; ++i) out[i] = fbits(vals[i]);
    out[12] = out[13] = out[14] = out[15] = 0u;
    x.c.bytes += 96 + 32;
}

static void add_counters(Counters& a, const Counters& b) {
    a.rays += b.rays; a.paths += b.paths; a.steps += b.steps; a.bytes += b.bytes;
    a.unknown += b.unknown; a.cache_hits += b.cache_hits;
    for (int i = 0; i < 4; ++i) a.status[i] += b.status[i];
    a.traverse_bytes += b.traverse_bytes;
}

// ---- voxel_retention.wgsl / voxel_accumulate.wgsl ----------------------------
static const uint32_t NO_LIMIT = 0xffffffffu;
static uint32_t curve_limit(uint32_t d2) {
    if (d2 >= 36864u) return NO_LIMIT;
    return (d2 * d2 + 10368u) / 20736u;
}
static uint32_t box_distance2(const int32_t lo[3], const int32_t hi[3], const int32_t p[3]) {
    uint32_t s = 0;
    for (int a = 0; a < 3; ++a) {
        int32_t v = imax(imax(lo[a] - p[a], p[a] - hi[a]), 0);
        v = imin(v, 4096);
        s += (uint32_t)v * (uint32_t)v;
    }
    return s;
}
static float load_height(int32_t top, int32_t y) {
    int32_t v = top + 1 - y;
    v = v < 0 ? 0 : (v > 16 ? 16 : v);
    return (float)v;
}
struct Retention { uint32_t limit; float change; bool measured, woken, urgent, urgent_if_binding; };

// voxel_retention.wgsl:29-96
static Retention resolve_retention(const uint32_t* events, const int32_t p[3], uint32_t event_count, uint32_t reach,
                                   bool measured_mode, uint32_t urgent_measured, uint32_t urgent_curve) {
    uint32_t cap = NO_LIMIT;
    float change = 0.0f;
    bool known = true;
    uint32_t source_cap = NO_LIMIT;
    bool woken = false, urgent_if_binding = false, urgent = false;
    const float PI = 3.14159265358979f;
    for (uint32_t e = 0; e < event_count; ++e) {
        const uint32_t* h0 = events + (size_t)(e * 3u) * 4;
        const uint32_t* h1 = h0 + 4;
        const uint32_t* h2 = h0 + 8;
        if ((h0[3] & 2u) != 0u) {
            uint32_t limit = h2[0];
            for (uint32_t b = 0; b < h2[3]; ++b) {
                const uint32_t* s = events + (size_t)(event_count * 3u + (h2[2] + b) * 2u) * 4;
                f3 d = sub(f3{(float)p[0], (float)p[1], (float)p[2]}, f3{bitsf(s[0]), bitsf(s[1]), bitsf(s[2])});
                if (dot(d, d) <= bitsf(s[3])) limit = umin(limit, 4u);
            }
            source_cap = umin(source_cap, limit);
            woken = true;
            continue;
        }
        int32_t lo[3] = {(int32_t)h0[0], (int32_t)h0[1], (int32_t)h0[2]};
        int32_t hi[3] = {(int32_t)h1[0], (int32_t)h1[1], (int32_t)h1[2]};
        uint32_t outside = box_distance2(lo, hi, p);
        if (outside > reach) continue;
        woken = true;
        bool exact = known;
        uint32_t nearest = NO_LIMIT;
        for (uint32_t b = 0; b < h2[3]; ++b) {
            size_t record = (size_t)event_count * 3u + (h2[2] + b) * 2u;
            const uint32_t* b0 = events + record * 4;
            const uint32_t* b1 = b0 + 4;
            int32_t blo[3] = {(int32_t)b0[0], (int32_t)b0[1], (int32_t)b0[2]};
            int32_t bhi[3] = {(int32_t)b1[0], (int32_t)b1[1], (int32_t)b1[2]};
            uint32_t d = box_distance2(blo, bhi, p);
            if (d > reach) continue;
            nearest = umin(nearest, d);
            uint32_t edit_kind = b1[3] & 7u;
            if ((b1[3] & 8u) != 0u && (edit_kind == 0u || edit_kind == 3u)) {
                if (edit_kind == 3u && measured_mode) urgent_if_binding = urgent_if_binding || d <= urgent_measured;
                else urgent = urgent || d <= urgent_curve;
            }
            if (exact) {
                uint32_t kind = b1[3] & 7u;
                if (kind == 0u) { known = false; exact = false; }
                else if (kind != 1u) {
                    float area = kind == 2u ? load_height(((int32_t)b1[3]) >> 3, p[1]) : 1.0f;
                    change = change + bitsf(b0[3]) * area / (PI * (float)umax(d, 1u));
                }
            }
        }
        if (nearest != NO_LIMIT) cap = umin(cap, curve_limit(nearest));
    }
    bool measured = measured_mode && known;
    uint32_t limit = umin(source_cap, measured ? NO_LIMIT : cap);
    return Retention{limit, change, measured, woken, urgent, urgent_if_binding};
}

static inline float lum(F4 v) { return 0.2126f * v.x + 0.7152f * v.y + 0.0722f * v.z; }
static inline float max3(float a, float b, float c) { return wmax(a, wmax(b, c)); }
static F4 stF4(const uint32_t* s) { return F4{bitsf(s[0]), bitsf(s[1]), bitsf(s[2]), bitsf(s[3])}; }
static void putF4(uint32_t* s, F4 v) { s[0] = fbits(v.x); s[1] = fbits(v.y); s[2] = fbits(v.z); s[3] = fbits(v.w); }

// voxel_accumulate.wgsl:336-344 (controls: display.w = c)
static bool binds(const uint32_t* state, uint32_t slot, float change, float physical) {
    const uint32_t* base = state + (size_t)slot * 36;
    F4 mean = stF4(base);
    F4 second = stF4(base + 8);
    F4 variance{wmax(second.x - mean.x * mean.x, 0.0f), wmax(second.y - mean.y * mean.y, 0.0f), wmax(second.z - mean.z * mean.z, 0.0f), 0};
    bool lit = lum(mean) >= 0.05f * change;
    float keep = physical * lum(variance) / wmax(change * change, 1e-30f);
    return !lit || keep < (float)(base[5] & 0x7fffffffu);
}

}  // namespace orc

using namespace orc;

static Geometry make_geometry(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                              const float* params) {
    Geometry g;
    g.directory = directory; g.headers = headers; g.cells = cells;
    g.mask = (uint32_t)(slots - 1);
    for (int a = 0; a < 3; ++a) { g.mn[a] = (int32_t)fbits(params[4 + a]); g.mx[a] = (int32_t)fbits(params[8 + a]); }
    return g;
}

extern "C" {

// trace_faces / trace_faces_parallel (voxel_trace.wgsl:62-92): `tasks` holds
// 8 words per face (voxel xyz, face, sequence, padding); `results` receives 24
// words per face (FaceResult). With pipe->lanes = L, lane l of a face traces
// samples l, l+L, ... and lane 0 sums the lanes in order, as the cooperative
// kernel does; L = 1 is the serial kernel. `state` (36 words per slot) and
// `index` (face index words) may be null for a cacheless trace.
static uint64_t g_predicted_misses = 0, g_last_miss = 0;

static int trace_faces_impl(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                            const float* params, const float* materials, const float* lights, const uint32_t* emitters,
                            const uint32_t* state, const uint32_t* index, const uint32_t* tasks, uint32_t n_tasks,
                            const orc_pipeline* pipe, uint32_t* results, orc_counters* counters, int threads,
                            const PredictedFaces* predicted) {
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, emitters, state, index, *pipe, predicted};
    uint32_t lanes = pipe->lanes == 0 ? 1 : pipe->lanes;
    Counters total;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<Counters> per((size_t)threads);
    std::atomic<uint64_t> next{0};
    auto worker = [&](int tid) {
        for (;;) {
            uint64_t first = next.fetch_add(16);
            if (first >= n_tasks) break;
            uint64_t last = std::min<uint64_t>(first + 16, n_tasks);
            for (uint64_t t = first; t < last; ++t) {
                Ctx x{g, m, Counters{}};
                const uint32_t* task = tasks + (size_t)t * 8;
                if (task[3] == 0xffffffffu) continue;
                Moments total_m;
                for (uint32_t l = 0; l < lanes; ++l) {
                    Moments lm = trace_moments(x, task, l, lanes);
                    total_m.mean = f4add(total_m.mean, lm.mean);
                    total_m.second = f4add(total_m.second, lm.second);
                    total_m.known += lm.known;
                }
                write_result(x, task, total_m, results + (size_t)t * 24);
                add_counters(per[(size_t)tid], x.c);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    for (auto& c : per) add_counters(total, c);
    if (counters) {
        counters->rays = total.rays; counters->paths = total.paths; counters->steps = total.steps;
        counters->bytes = total.bytes; counters->unknown = total.unknown; counters->cache_hits = total.cache_hits;
        for (int i = 0; i < 4; ++i) counters->status[i] = total.status[i];
        counters->traverse_bytes = total.traverse_bytes;
    }
    return 0;
}

int orc_trace_faces(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                    const float* params, const float* materials, const float* lights, const uint32_t* emitters,
                    const uint32_t* state, const uint32_t* index, const uint32_t* tasks, uint32_t n_tasks,
                    const orc_pipeline* pipe, uint32_t* results, orc_counters* counters, int threads) {
    return trace_faces_impl(directory, slots, headers, cells, params, materials, lights, emitters, state, index, tasks, n_tasks, pipe,
                            results, counters, threads, nullptr);
}

// orc_trace_faces with the MLP cache mode's termination: keys4 = (voxel
// xyz, face) and values3 = the network's rgb for each face a path may hit.
int orc_trace_faces_predicted(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                              const float* params, const float* materials, const float* lights, const uint32_t* emitters,
                              const uint32_t* state, const uint32_t* index, const uint32_t* tasks, uint32_t n_tasks,
                              const orc_pipeline* pipe, const int32_t* keys4, const float* values3, uint32_t n_keys, uint32_t* results,
                              orc_counters* counters, int threads) {
    PredictedFaces predicted;
    predicted.map.reserve(n_keys);
    for (uint32_t k = 0; k < n_keys; ++k)
        predicted.map[face_key(keys4[k * 4], keys4[k * 4 + 1], keys4[k * 4 + 2], (uint32_t)keys4[k * 4 + 3])] =
            F4{values3[k * 3], values3[k * 3 + 1], values3[k * 3 + 2], 0.0f};
    const int rc = trace_faces_impl(directory, slots, headers, cells, params, materials, lights, emitters, state, index, tasks, n_tasks,
                                    pipe, results, counters, threads, &predicted);
    g_predicted_misses = predicted.misses.load();
    g_last_miss = predicted.last_miss.load();
    return rc;
}

// Hits of the last orc_trace_faces_predicted call on faces its table did not
// hold (they took zero), and the key (x | y << 16 | z << 32 | face << 48) of one.
uint64_t orc_predicted_misses(uint64_t* last_key) {
    if (last_key) *last_key = g_last_miss;
    return g_predicted_misses;
}

// One ray through trace_domain_limited (for traversal parity tests):
// out = [voxel xyz, material, position xyz (bits), status, normal xyz (bits), steps].
int orc_trace_ray(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells,
                  const float* params, const float* ray, uint32_t visible_geometry, uint32_t max_steps, uint32_t* out) {
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, nullptr, nullptr, nullptr, nullptr, nullptr, orc_pipeline{1, 0, max_steps, 0, 1}};
    Ctx x{g, m, Counters{}};
    RayResult r = trace_domain_limited(x, f3{ray[0], ray[1], ray[2]}, f3{ray[3], ray[4], ray[5]}, ray[6], visible_geometry != 0, max_steps);
    uint32_t v[12] = {(uint32_t)r.voxel.x, (uint32_t)r.voxel.y, (uint32_t)r.voxel.z, r.material, fbits(r.position.x), fbits(r.position.y),
                      fbits(r.position.z), r.status, fbits(r.normal.x), fbits(r.normal.y), fbits(r.normal.z), (uint32_t)x.c.steps};
    for (int i = 0; i < 12; ++i) out[i] = v[i];
    return 0;
}

// advance_box (voxel_traversal.wgsl:90-107) on one case:
// in = [position xyz, size, direction xyz, cell xyz (as int bits), negative xyz, positive xyz]
int orc_advance_box(const float* in, float* out) {
    const uint32_t* u = (const uint32_t*)in;
    F4 r = advance_box(f3{in[0], in[1], in[2]}, f3{in[4], in[5], in[6]}, i3{(int32_t)u[7], (int32_t)u[8], (int32_t)u[9]},
                       i3{(int32_t)u[10], (int32_t)u[11], (int32_t)u[12]}, i3{(int32_t)u[13], (int32_t)u[14], (int32_t)u[15]}, in[3]);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
    return 0;
}

float orc_sample_1d(uint32_t stream, uint32_t sequence, uint32_t dimension) { return sample_1d(stream, sequence, dimension); }
void orc_hemisphere(const float* n, float u, float v, float* out) {
    f3 r = hemisphere(f3{n[0], n[1], n[2]}, u, v);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void orc_sincos(float x, float* s, float* c) { own_sincos(x, s, c); }
float orc_exp(float x) { return own_exp(x); }
uint32_t orc_pcg(uint32_t v) { return pcg(v); }
uint32_t orc_curve_limit(uint32_t d2) { return curve_limit(d2); }
// resolve_retention for one receiver voxel over encoded events (the
// encode_events layout): out_limit = the history cap (NO_LIMIT for none),
// out_change = the summed predicted change, flags bit 0 measured (every
// change in range has a known flux, with measured_mode), bit 1 woken.
int orc_resolve_retention(const uint32_t* events, uint32_t n_events, const int32_t* p3, uint32_t reach, int measured_mode,
                          uint32_t* out_limit, float* out_change, uint32_t* flags) {
    const Retention r = resolve_retention(events, p3, n_events, reach, measured_mode != 0, 0u, 0u);
    *out_limit = r.limit;
    *out_change = r.change;
    *flags = (r.measured ? 1u : 0u) | (r.woken ? 2u : 0u);
    return 0;
}

// prepare for every traced CPU-owned slot (voxel_accumulate.wgsl:114-133):
// the task takes the slot's current sequence (begin_trace) and the slot's
// schedule word records the batch id (controls batch.y). slot_meta may be null.
int orc_begin_trace(const uint32_t* state, uint32_t* slot_meta, uint32_t* tasks, const uint32_t* slots, uint32_t n,
                    const uint32_t* controls) {
    for (uint32_t i = 0; i < n; ++i) {
        tasks[(size_t)i * 8 + 4] = state[(size_t)slots[i] * 36 + 6];
        if (slot_meta) {
            uint32_t* sched = slot_meta + ((size_t)slots[i] * 3 + 1) * 4;
            sched[1] = (sched[1] & 0xfu) | (controls[25] << 4);
        }
    }
    return 0;
}

// mark_changed (voxel_accumulate.wgsl:432-446); controls = 36 words.
int orc_mark_changed(uint32_t* state, uint32_t* slot_meta, const uint32_t* slots, uint32_t n, const uint32_t* controls) {
    float physical = bitsf(controls[11]);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t slot = slots[i];
        if (slot == 0xffffffffu) continue;
        uint32_t* meta = slot_meta + ((size_t)slot * 3 + 1) * 4;
        float pending = bitsf(meta[0]);
        if (pending <= 0.0f) continue;
        if (binds(state, slot, pending, physical)) state[(size_t)slot * 36 + 5] |= 0x80000000u;
        else meta[0] = 0u;
    }
    return 0;
}

static uint32_t required_samples(const uint32_t* controls, F4 mean) {
    uint32_t s = controls[18];
    return max3(mean.x, mean.y, mean.z) < 0.02f ? umax(s, 256u) : s;
}
static float refinement_error(const uint32_t* base, uint32_t count) {
    if (count < 2u) return 1.0f;
    F4 mean = stF4(base), second = stF4(base + 8);
    float c = (float)count;
    float e[3];
    float mv[3] = {mean.x, mean.y, mean.z}, sv[3] = {second.x, second.y, second.z};
    for (int a = 0; a < 3; ++a) e[a] = std::sqrt(wmax(sv[a] - mv[a] * mv[a], 0.0f) / c) / (0.002f + std::fabs(mv[a]));
    return wmin(max3(e[0], e[1], e[2]), 8.0f);
}
static float sample_noise(const uint32_t* base) {
    F4 mean = stF4(base), second = stF4(base + 8);
    float mv[3] = {mean.x, mean.y, mean.z}, sv[3] = {second.x, second.y, second.z}, e[3];
    for (int a = 0; a < 3; ++a) e[a] = std::sqrt(wmax(sv[a] - mv[a] * mv[a], 0.0f)) / (0.002f + std::fabs(mv[a]));
    return max3(e[0], e[1], e[2]);
}

// accumulate (voxel_accumulate.wgsl:135-227) with record_stability (:237-262).
// Tasks from batch.x (controls[24]) on are GPU picks: their pick record
// (4 words per task, may be null) takes the merged count and the slot's
// statistics mirror becomes stale. outputs: 24 words per task (FaceResult
// in, state words 0..5 out).
static int accumulate_impl(uint32_t* state, uint32_t* slot_meta, uint32_t* checkpoint, uint32_t* outputs, const uint32_t* slots,
                           uint32_t n, const uint32_t* controls, uint32_t* picks) {
    const uint32_t MIRROR_STALE = 0x20000000u;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t slot = slots[i];
        if (i >= controls[0] || slot == 0xffffffffu) continue;
        uint32_t* base = state + (size_t)slot * 36;
        uint32_t* out = outputs + (size_t)i * 24;
        uint32_t* cp = checkpoint + (size_t)slot * 12;
        for (int k = 0; k < 4; ++k) { cp[k] = base[k]; cp[4 + k] = base[8 + k]; }
        cp[8] = base[4]; cp[9] = base[5] & 0x7fffffffu; cp[10] = base[12]; cp[11] = 0u;
        uint32_t fresh = f2u(bitsf(out[5]));
        uint32_t* meta = slot_meta + ((size_t)slot * 3 + 1) * 4;
        float pending = bitsf(meta[0]);
        if (fresh > 0u) meta[0] = 0u;
        uint32_t previous_count = base[5] & 0x7fffffffu;
        float physical = bitsf(controls[11]);
        float change = (base[5] & 0x80000000u) != 0u ? pending : 0.0f;
        if (physical > 0.0f && fresh > 0u && change > 0.0f) {
            F4 om = stF4(base), os = stF4(base + 8), fm = stF4(out), fs = stF4(out + 8);
            F4 ov{wmax(os.x - om.x * om.x, 0.0f), wmax(os.y - om.y * om.y, 0.0f), wmax(os.z - om.z * om.z, 0.0f), 0};
            F4 fv{wmax(fs.x - fm.x * fm.x, 0.0f), wmax(fs.y - fm.y * fm.y, 0.0f), wmax(fs.z - fm.z * fm.z, 0.0f), 0};
            float variance = lum(om) < 0.05f * change ? lum(fv) : lum(ov);
            float keep = physical * variance / (change * change);
            previous_count = umin(previous_count, f2u(wmin(keep, 65536.0f)));
            cp[9] = umin(cp[9], previous_count);
        }
        uint32_t count = umin(previous_count + fresh, controls[3]);
        float recency = bitsf(controls[10]);
        float alpha = fresh > 0u ? wmin(recency * (float)fresh / (float)umax(count, 1u), 1.0f) : 0.0f;
        F4 mean = stF4(out), second = stF4(out + 8), pm = stF4(base), ps = stF4(base + 8);
        F4 nm{pm.x + (mean.x - pm.x) * alpha, pm.y + (mean.y - pm.y) * alpha, pm.z + (mean.z - pm.z) * alpha, pm.w + (mean.w - pm.w) * alpha};
        F4 ns{ps.x + (second.x - ps.x) * alpha, ps.y + (second.y - ps.y) * alpha, ps.z + (second.z - ps.z) * alpha, ps.w + (second.w - ps.w) * alpha};
        putF4(base, nm);
        putF4(base + 8, ns);
        base[5] = count;
        base[6] += controls[1];
        for (int k = 0; k < 4; ++k) { base[16 + k] = out[16 + k]; base[20 + k] = out[20 + k]; }
        F4 radiance = stF4(base), moment = stF4(base + 8);
        float rv[3] = {radiance.x, radiance.y, radiance.z}, mv[3] = {moment.x, moment.y, moment.z};
        float cnt = wmax((float)count, 1.0f), u[3], nz[3];
        for (int a = 0; a < 3; ++a) {
            float err = std::sqrt(wmax(mv[a] - rv[a] * rv[a], 0.0f) / cnt);
            u[a] = err / (0.02f + std::fabs(rv[a]));
            nz[a] = err / (0.002f + std::fabs(rv[a]));
        }
        float uncertainty = count < 2u ? 1.0f : wmin(8.0f, max3(u[0], u[1], u[2]));
        float noise = count < 2u ? 1.0f : wmin(8.0f, max3(nz[0], nz[1], nz[2]));
        float elapsed = base[30] != 0u ? (float)(controls[2] - base[29]) * 0.001f : 1.0f / 60.0f;
        float time_alpha = 1.0f - own_exp(-elapsed / bitsf(controls[4]));
        float evidence = (float)count / ((float)count + 32.0f);
        float blend = wmin(time_alpha, evidence / (1.0f + 16.0f * noise * noise));
        F4 previous = stF4(base + 24);
        float old_weight = (1.0f - blend) / (0.25f + max3(previous.x, previous.y, previous.z));
        float new_weight = blend / (0.25f + max3(radiance.x, radiance.y, radiance.z));
        float alpha_display = wmin(blend, new_weight / wmax(old_weight + new_weight, 0.0000001f));
        float confidence = wclamp((float)count / ((float)count + 8.0f) / (1.0f + uncertainty), 0.125f, 1.0f);
        // mix(a, b, t) = a * (1 - t) + b * t
        F4 disp{previous.x * (1.0f - alpha_display) + radiance.x * alpha_display,
                previous.y * (1.0f - alpha_display) + radiance.y * alpha_display,
                previous.z * (1.0f - alpha_display) + radiance.z * alpha_display,
                previous.w * (1.0f - blend) + confidence * blend};
        putF4(base + 24, disp);
        base[29] = controls[2];
        base[30] = 0xffffffffu;
        base[7] = base[24];
        base[13] = base[25]; base[14] = base[26]; base[15] = base[27];
        for (int k = 0; k < 24; ++k) out[k] = base[k];
        const bool picked = i >= controls[24];
        if (picked && picks) picks[(size_t)i * 4 + 2] = base[5] & 0x7fffffffu;
        // record_stability
        uint32_t* sched = slot_meta + ((size_t)slot * 3 + 1) * 4;
        uint32_t* rank = slot_meta + ((size_t)slot * 3 + 2) * 4;
        uint32_t sy = sched[1], sw = sched[3];
        bool same_revision = (sy & 8u) != 0u && sw == controls[16];
        uint32_t scount = base[5] & 0x7fffffffu;
        F4 after = stF4(base);
        float tolerance = bitsf(controls[17]);
        float bv[3] = {pm.x, pm.y, pm.z}, av[3] = {after.x, after.y, after.z}, dr[3];
        for (int a = 0; a < 3; ++a) dr[a] = std::fabs(bv[a] - av[a]) / (0.002f + wmax(std::fabs(bv[a]), std::fabs(av[a])));
        float drift = max3(dr[0], dr[1], dr[2]);
        F4 display = stF4(base + 24);
        bool settled = max3(std::fabs(display.x - after.x), std::fabs(display.y - after.y), std::fabs(display.z - after.z)) <=
                       0.001f + max3(after.x, after.y, after.z) * tolerance * 0.5f;
        uint32_t stable = (same_revision && settled && scount >= required_samples(controls, after) &&
                           refinement_error(base, scount) <= tolerance && drift <= tolerance * 0.5f)
                              ? umin((sy & 7u) + 1u, 4u)
                              : 0u;
        sched[1] = (sy & 0xfffffff0u) | 8u | stable;
        sched[3] = controls[16];
        uint32_t old_rank_w = rank[3];
        rank[0] = fbits(sample_noise(base));
        rank[1] = controls[2];
        rank[2] = fbits(max3(after.x, after.y, after.z));
        rank[3] = 0x80000000u | scount | (picked ? MIRROR_STALE : (old_rank_w & MIRROR_STALE));
        // settled_flag
        if ((sched[1] & 15u) == 12u) out[5] |= 0x80000000u;
    }
    return 0;
}

int orc_accumulate(uint32_t* state, uint32_t* slot_meta, uint32_t* checkpoint, uint32_t* outputs, const uint32_t* slots,
                   uint32_t n, const uint32_t* controls) {
    return accumulate_impl(state, slot_meta, checkpoint, outputs, slots, n, controls, nullptr);
}

int orc_accumulate_picks(uint32_t* state, uint32_t* slot_meta, uint32_t* checkpoint, uint32_t* outputs, const uint32_t* slots,
                         uint32_t n, const uint32_t* controls, uint32_t* picks) {
    return accumulate_impl(state, slot_meta, checkpoint, outputs, slots, n, controls, picks);
}

// ---- GPU selection (voxel_accumulate.wgsl:448-695), restated serially ----------
static int page_axis(int p) { return (p - (p < 0 ? 31 : 0)) / 32; }

// candidate (voxel_accumulate.wgsl:474-511): class << 8 | bucket, or none.
static uint32_t candidate_key(const uint32_t* slot_meta, uint32_t slot, const uint32_t* ctl) {
    const uint32_t URGENT = 0x40000000u;
    const uint32_t* identity = slot_meta + (size_t)slot * 12;
    if ((identity[3] & 8u) == 0u) return 0xffffffffu;
    const uint32_t* schedule = identity + 4;
    const uint32_t last_cpu = schedule[1] >> 4u;
    if (last_cpu != 0u && ((ctl[25] - last_cpu) & 0x0fffffffu) < 4u) return 0xffffffffu;
    const uint32_t* rank = identity + 8;
    const uint32_t count = rank[3] & 0x1fffffffu;
    const bool fresh = (schedule[1] & 8u) != 0u && schedule[3] == ctl[16];
    const uint32_t since = ctl[2] - rank[1];
    const uint32_t age_ms = rank[3] < 0x80000000u ? 0x7fffffffu : (since > 0x7fffffffu ? 0u : since);
    const uint32_t required = bitsf(rank[2]) < 0.02f ? umax(ctl[18], 256u) : ctl[18];
    const bool due = !fresh || count < required || (schedule[1] & 7u) < 4u || age_ms >= ctl[19] || (rank[3] & URGENT) != 0u;
    if (!due) return 0xffffffffu;
    const int px = (int)identity[0], py = (int)identity[1], pz = (int)identity[2];
    const int fx = (int)ctl[20], fy = (int)ctl[21], fz = (int)ctl[22];
    if ((rank[3] & URGENT) != 0u || count < 8u) {
        const float dx = (float)(px - fx), dy = (float)(py - fy), dz = (float)(pz - fz);
        const float d2 = dx * dx + dy * dy + dz * dz;
        const uint32_t b = f2u(own_log2(d2 + 1.0f) * 8.0f);
        return (((rank[3] & URGENT) != 0u ? 3u : 0u) << 8u) | umin(b, 255u);
    }
    const int ax = std::abs(page_axis(px) - page_axis(fx)), ay = std::abs(page_axis(py) - page_axis(fy)),
              az = std::abs(page_axis(pz) - page_axis(fz));
    const int page_distance = imax(ax, imax(ay, az));
    if (page_distance <= 2) {
        const float age = wmin((float)age_ms * 0.001f, 10.0f);
        const float error = count < 2u ? 1.0f : wmin(bitsf(rank[0]) / std::sqrt((float)count), 8.0f);
        const float priority = (error + age * 0.1f) + (page_distance <= 1 ? 0.25f : 0.0f);
        const uint32_t b = f2u(wmax(own_log2(priority) + 8.0f, 0.0f) * 16.0f);
        return (1u << 8u) | (255u - umin(b, 255u));
    }
    const uint32_t b = f2u(own_log2((float)age_ms + 1.0f) * 8.0f);
    return (2u << 8u) | (255u - umin(b, 255u));
}

// trace_footprints + finish_footprints (voxel_trace.wgsl:94-202), thread by
// thread: fp = (1 + 3 n) records of 4 int32 words, sums = 8 words per task
// (the caller's initial min 0xffffffff, max 0, flux 0), events = event words.
int orc_footprints(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                   const float* materials, const float* lights, const int32_t* fp, uint32_t threads, uint32_t* sums, uint32_t* events) {
    const int32_t BIAS = 1073741824;
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, nullptr, nullptr, nullptr, orc_pipeline{1, 0, 2048, 0, 1}};
    Ctx x{g, m, Counters{}};
    const uint32_t n = (uint32_t)fp[0];
    const uint32_t n_directional = ((const uint32_t*)params)[11];
    const float reach = params[17];
    for (uint32_t id = 0; id < threads && n > 0; ++id) {
        uint32_t lo_t = 0, hi_t = n;
        while (hi_t - lo_t > 1u) {
            const uint32_t mid = (lo_t + hi_t) / 2u;
            if ((uint32_t)fp[(1 + mid * 3 + 2) * 4] <= id) lo_t = mid;
            else hi_t = mid;
        }
        const uint32_t e = lo_t;
        const int32_t* a = fp + (1 + e * 3) * 4;
        const int32_t* b = a + 4;
        const int32_t* c = a + 8;
        const uint32_t grid = (uint32_t)c[1];
        const uint32_t local = id - (uint32_t)c[0];
        if (local >= grid * grid) continue;
        const f3 lo{(float)a[0], (float)a[1], (float)a[2]};
        const f3 hi{(float)b[0] + 1.0f, (float)b[1] + 1.0f, (float)b[2] + 1.0f};
        const f3 center = muls(add(lo, hi), 0.5f);
        const f3 span = sub(hi, lo);
        const float diagonal = std::sqrt(dot(span, span));
        const float spacing = diagonal / (float)grid;
        const float half = 0.5f * diagonal;
        const float ox = ((float)(local % grid) + 0.5f) * spacing - half;
        const float oy = ((float)(local / grid) + 0.5f) * spacing - half;
        const f3 w{0.2126f, 0.7152f, 0.0722f};
        const uint32_t base = e * 8;
        float flux = 0.0f;
        for (uint32_t i = 0; i < n_directional; ++i) {
            const float* L = lights + (size_t)i * 12;
            const f3 color{wmax(L[4] - L[9], 0.0f), wmax(L[5] - L[10], 0.0f), wmax(L[6] - L[11], 0.0f)};
            if (color.x == 0.0f && color.y == 0.0f && color.z == 0.0f) continue;
            const f3 raw{L[0], L[1], L[2]};
            const float len = std::sqrt(dot(raw, raw));
            const f3 direction{raw.x / len, raw.y / len, raw.z / len};
            const f3 pick = std::fabs(direction.y) > 0.9f ? f3{1.0f, 0.0f, 0.0f} : f3{0.0f, 1.0f, 0.0f};
            const f3 uc = cross(direction, pick);
            const float ul = std::sqrt(dot(uc, uc));
            const f3 u{uc.x / ul, uc.y / ul, uc.z / ul};
            const f3 v = cross(direction, u);
            const f3 point = add(add(center, muls(u, ox)), muls(v, oy));
            const f3 inverse{1.0f / (std::fabs(direction.x) < 1e-8f ? 1e-8f : direction.x),
                             1.0f / (std::fabs(direction.y) < 1e-8f ? 1e-8f : direction.y),
                             1.0f / (std::fabs(direction.z) < 1e-8f ? 1e-8f : direction.z)};
            const f3 nearv = mul(sub(lo, point), inverse), farv = mul(sub(hi, point), inverse);
            const float enter = wmax(wmax(wmin(nearv.x, farv.x), wmin(nearv.y, farv.y)), wmin(nearv.z, farv.z));
            const float exit = wmin(wmin(wmax(nearv.x, farv.x), wmax(nearv.y, farv.y)), wmax(nearv.z, farv.z));
            if (enter > exit) continue;
            if (trace_domain_limited(x, add(point, muls(direction, exit + 0.01f)), direction, reach, true, 2048u).status != 0u) continue;
            const f3 start = add(point, muls(direction, enter - 0.01f));
            const RayResult hit = trace_domain_limited(x, start, neg(direction), reach, true, 2048u);
            const f3 gap = sub(hit.position, start);
            if (hit.status != 1u || dot(hit.normal, direction) <= 0.0f || std::sqrt(dot(gap, gap)) < 0.02f) continue;
            const float* mat = materials + (size_t)hit.material * 16;
            flux = flux + ((dot(color, w) * dot(f3{mat[0], mat[1], mat[2]}, w)) * spacing) * spacing;
            const uint32_t p[3] = {(uint32_t)(hit.voxel.x + BIAS), (uint32_t)(hit.voxel.y + BIAS), (uint32_t)(hit.voxel.z + BIAS)};
            for (int k = 0; k < 3; ++k) {
                sums[base + k] = umin(sums[base + k], p[k]);
                sums[base + 3 + k] = umax(sums[base + 3 + k], p[k]);
            }
        }
        if (flux > 0.0f) sums[base + 6] += f2u(flux * 64.0f + 0.5f);
    }
    for (uint32_t e = 0; e < n; ++e) {
        const uint32_t base = e * 8;
        if (sums[base] == 0xffffffffu) continue;
        int32_t mn[3], mx[3];
        for (int k = 0; k < 3; ++k) {
            mn[k] = (int32_t)sums[base + k] - BIAS;
            mx[k] = (int32_t)sums[base + 3 + k] - BIAS;
        }
        const float flux = (float)sums[base + 6] / 64.0f;
        const uint32_t header = (uint32_t)fp[(1 + e * 3) * 4 + 3], bound = (uint32_t)fp[(1 + e * 3 + 1) * 4 + 3];
        uint32_t* h = events + (size_t)header * 4;
        uint32_t* bd = events + (size_t)bound * 4;
        for (int k = 0; k < 3; ++k) {
            h[k] = (uint32_t)mn[k];
            h[4 + k] = (uint32_t)mx[k];
            bd[k] = (uint32_t)mn[k];
            bd[4 + k] = (uint32_t)mx[k];
        }
        bd[3] = fbits(flux);
        bd[7] = 4u;
    }
    return 0;
}

// A pinhole camera's ray through pixel (px, py): cam = eye xyz, forward xyz
// (unit), up xyz, tan(half vertical fov).
static f3 camera_ray(const float* cam, uint32_t px, uint32_t py, uint32_t w, uint32_t h) {
    const f3 forward{cam[3], cam[4], cam[5]}, up{cam[6], cam[7], cam[8]};
    const f3 rc = cross(forward, up);
    const float rl = std::sqrt(dot(rc, rc));
    const f3 right{rc.x / rl, rc.y / rl, rc.z / rl};
    const f3 up2 = cross(right, forward);
    const float fw = (float)w, fh = (float)h;
    const float sx = ((2.0f * ((float)px + 0.5f)) / fw - 1.0f) * cam[9] * (fw / fh);
    const float sy = (1.0f - (2.0f * ((float)py + 0.5f)) / fh) * cam[9];
    const f3 raw = add(add(forward, muls(right, sx)), muls(up2, sy));
    const float len = std::sqrt(dot(raw, raw));
    return f3{raw.x / len, raw.y / len, raw.z / len};
}

// Headless discovery's per-pixel first hits (the GPU's discover kernel):
// cam = eye xyz, forward xyz (unit), up xyz, tan(half vertical fov);
// pixels = 8 words per pixel (voxel xyz, face or 6, material, status,
// distance bits, 0).
int orc_discover(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                 const float* cam, uint32_t w, uint32_t h, uint32_t* pixels, int threads) {
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, nullptr, nullptr, nullptr, nullptr, nullptr, orc_pipeline{1, 0, 2048, 0, 1}};
    const f3 eye{cam[0], cam[1], cam[2]};
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        Ctx x{g, m, Counters{}};
        for (;;) {
            const uint32_t id = next.fetch_add(1);
            if (id >= w * h) break;
            const f3 dir = camera_ray(cam, id % w, id / w, w, h);
            const RayResult r = trace_domain_limited(x, eye, dir, params[17], true, 2048u);
            const uint32_t face = r.status == 1u ? face_index_of(r.normal) : 6u;
            const f3 gap = sub(r.position, eye);
            const float distance = r.status == 1u ? std::sqrt(dot(gap, gap)) : 0.0f;
            uint32_t* o = pixels + (size_t)id * 8;
            o[0] = (uint32_t)r.voxel.x; o[1] = (uint32_t)r.voxel.y; o[2] = (uint32_t)r.voxel.z; o[3] = face;
            o[4] = r.material; o[5] = r.status; o[6] = fbits(distance); o[7] = 0;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return 0;
}

// ---- far tier (voxel_view_pixels.wgsl:53-216), headless ---------------------------
// view = 44 words: camera (10), previous camera (10), width, height, grid
// (cells x, y, pixels per side, enabled | measure << 1), tune (threshold px,
// max history, rate, previous stamp bits), axis (forward xyz, pixels per unit
// at depth 1), interest min (4, w bounded), interest max (4), frame, custom.
namespace far {
struct View {
    const uint32_t* w;
    const float* cam() const { return reinterpret_cast<const float*>(w); }
    const float* prev() const { return reinterpret_cast<const float*>(w + 10); }
    uint32_t width() const { return w[20]; }
    uint32_t height() const { return w[21]; }
    uint32_t grid(int i) const { return w[22 + i]; }
    float tune(int i) const { return bitsf(w[26 + i]); }
    float axis(int i) const { return bitsf(w[30 + i]); }
    int32_t imin(int i) const { return (int32_t)w[34 + i]; }
    int32_t imax(int i) const { return (int32_t)w[38 + i]; }
    uint32_t frame() const { return w[42]; }
    bool custom() const { return w[43] != 0u; }
    f3 eye() const { return f3{cam()[0], cam()[1], cam()[2]}; }
};

static float comp(f3 v, uint32_t a) { return a == 0u ? v.x : (a == 1u ? v.y : v.z); }
static void set_comp(f3& v, uint32_t a, float x) { (a == 0u ? v.x : (a == 1u ? v.y : v.z)) = x; }
static i3 region_of(i3 v) {
    return i3{(int32_t)std::floor((float)v.x / 16.0f), (int32_t)std::floor((float)v.y / 16.0f), (int32_t)std::floor((float)v.z / 16.0f)};
}

// voxel_traversal.wgsl:74-80
static int32_t voxel_stride(Ctx& x, i3 voxel) {
    const i3 r = region_of(voxel);
    if (!in_bounds(x, r)) return 1;
    const uint32_t index = lookup_region(x, r);
    if (index == 0xffffffffu) return 1;
    return 1 << ((x.g.headers[(size_t)index * 4 + 3] >> 28u) & 7u);
}

// voxel_view_runtime.wgsl:26-30
static bool in_interest(const View& v, i3 voxel) {
    if (v.imin(3) == 0) return true;
    const i3 r = region_of(voxel);
    return r.x >= v.imin(0) && r.y >= v.imin(1) && r.z >= v.imin(2) && r.x <= v.imax(0) && r.y <= v.imax(1) && r.z <= v.imax(2);
}

// voxel_view_pixels.wgsl:53-65
static bool pixel_owned(Ctx& x, const View& v, i3 voxel, uint32_t face) {
    const uint32_t grid = v.grid(3);
    if ((grid & 1u) == 0u || face >= 6u) return false;
    const uint32_t mode = (grid >> 1u) & 3u;
    const int32_t s = mode == 2u ? voxel_stride(x, voxel) : 1;
    const f3 block{(float)(voxel.x & -s), (float)(voxel.y & -s), (float)(voxel.z & -s)};
    const f3 ray = sub(adds(block, 0.5f * (float)s), v.eye());
    if (dot(ray, f3{v.axis(0), v.axis(1), v.axis(2)}) <= 0.0f) return false;
    const float side = ((float)s * v.axis(3)) / length(ray);
    if (mode == 0u) return side < v.tune(0);
    return (side * side) * std::fabs(dot(face_normal(face), normalize(ray))) < v.tune(0);
}

// f32 -> f16 bits, IEEE round to nearest even (pack2x16float's conversion).
static uint32_t half_bits(float f) {
    const uint32_t u = fbits(f);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return sign | (a > 0x7f800000u ? 0x7fffu : 0x7c00u);
    if (a >= 0x477ff000u) return sign | 0x7c00u;  // at or past 65520: rounds to infinity
    if (a < 0x38800000u) {                         // under 2^-14: a subnormal half, exact scaling by 2^24
        return sign | (uint32_t)std::nearbyint(bitsf(a) * 16777216.0f);
    }
    uint32_t h = (((a >> 23) - 112u) << 10) | ((a & 0x7fffffu) >> 13);
    const uint32_t rest = a & 0x1fffu;
    if (rest > 0x1000u || (rest == 0x1000u && (h & 1u))) h += 1u;
    return sign | h;
}
static uint32_t pack2(float a, float b) { return half_bits(a) | (half_bits(b) << 16); }

struct Cell { f3 mean; float count; f3 surface; uint32_t face; uint32_t sequence; };
static Cell load(const uint32_t* cells, uint32_t i) {
    const uint32_t* c = cells + (size_t)i * 12;
    return Cell{f3{bitsf(c[0]), bitsf(c[1]), bitsf(c[2])}, bitsf(c[3]), f3{bitsf(c[4]), bitsf(c[5]), bitsf(c[6])}, c[7], c[8]};
}
static void store(uint32_t* cells, uint32_t i, const Cell& v) {
    uint32_t* c = cells + (size_t)i * 12;
    c[0] = fbits(v.mean.x); c[1] = fbits(v.mean.y); c[2] = fbits(v.mean.z); c[3] = fbits(v.count);
    c[4] = fbits(v.surface.x); c[5] = fbits(v.surface.y); c[6] = fbits(v.surface.z); c[7] = v.face;
    c[8] = v.sequence; c[9] = 0; c[10] = 0; c[11] = 0;
}

// write_output + custom_direct (voxel_view_pixels.wgsl:67-81)
static void write_output(Ctx& x, const View& v, uint32_t* output, uint32_t index, const Cell& cell) {
    const uint32_t axis = (cell.face & 7u) / 2u;
    f3 shown = cell.mean;
    if (v.custom()) shown = add(shown, direct_at(x, cell.surface, face_normal(cell.face & 7u)).custom);
    uint32_t* o = output + 16 + (size_t)index * 4;
    o[0] = pack2(shown.x, shown.y);
    o[1] = pack2(shown.z, cell.count);
    o[2] = cell.face;
    o[3] = fbits(comp(cell.surface, axis));
}

// The previous camera's NDC of a world point; false behind it.
static bool project(const float* cam, uint32_t w, uint32_t h, f3 point, float& nx, float& ny) {
    const f3 forward{cam[3], cam[4], cam[5]}, up{cam[6], cam[7], cam[8]};
    const f3 right = normalize(cross(forward, up));
    const f3 up2 = cross(right, forward);
    const f3 d = sub(point, f3{cam[0], cam[1], cam[2]});
    const float depth = dot(d, forward);
    if (depth <= 0.0f) return false;
    const float scale = depth * cam[9];
    nx = dot(d, right) / (scale * ((float)w / (float)h));
    ny = dot(d, up2) / scale;
    return true;
}

// previous_cell (voxel_view_pixels.wgsl:83-127)
static void previous_cell(Ctx& x, const View& v, const uint32_t* previous, f3 surface, uint32_t face, i3 voxel, f3& mean, float& count,
                          uint32_t& sequence) {
    mean = f3{0, 0, 0};
    count = 0.0f;
    sequence = 0;
    const uint32_t prev_stamp = fbits(v.tune(3));
    if (prev_stamp == 0xffffffffu) return;
    float nx, ny;
    if (!project(v.prev(), v.width(), v.height(), surface, nx, ny)) return;
    const uint32_t size = v.grid(2);
    const f3 normal = face_normal(face);
    const float ux = nx * 0.5f + 0.5f, uy = ny * -0.5f + 0.5f;
    const float px = (ux * (float)v.width()) / (float)size - 0.5f;
    const float py = (uy * (float)v.height()) / (float)size - 0.5f;
    const float flx = std::fmin(std::fmax(std::floor(px), -1048576.0f), 1048576.0f);
    const float fly = std::fmin(std::fmax(std::floor(py), -1048576.0f), 1048576.0f);
    const int32_t bx = (int32_t)flx, by = (int32_t)fly;
    const float fx = px - flx, fy = py - fly;
    const float reach = ((2.0f * (float)size) * length(sub(surface, v.eye()))) / v.axis(3);
    const float tolerance = 4.0f * (float)voxel_stride(x, voxel) + 0.01f;
    const uint32_t expected = face | ((prev_stamp & 0x1fffffffu) << 3u);
    float weight = 0.0f, samples = 0.0f, best = 0.0f;
    f3 sum{0, 0, 0};
    for (int32_t yy = 0; yy <= 1; ++yy) {
        for (int32_t xx = 0; xx <= 1; ++xx) {
            const int32_t qx = bx + xx, qy = by + yy;
            if (qx < 0 || qy < 0 || qx >= (int32_t)v.grid(0) || qy >= (int32_t)v.grid(1)) continue;
            const Cell old = load(previous, (uint32_t)qy * v.grid(0) + (uint32_t)qx);
            if (old.face != expected || old.count == 0.0f) continue;
            const f3 delta = sub(old.surface, surface);
            if (std::fabs(dot(delta, normal)) > tolerance || dot(delta, delta) > reach * reach) continue;
            const float wgt = (xx == 1 ? fx : 1.0f - fx) * (yy == 1 ? fy : 1.0f - fy) + 1e-4f;
            sum = add(sum, muls(old.mean, wgt));
            samples = samples + old.count * wgt;
            weight = weight + wgt;
            if (wgt > best) {
                best = wgt;
                sequence = old.sequence;
            }
        }
    }
    if (weight > 0.0f) {
        mean = divs(sum, weight);
        count = samples / weight;
    }
}

// block_receiver then the receiver of the same key (the view receivers are
// unique faces, so a scan finds what the owner hash finds).
static uint32_t owner(Ctx& x, i3 voxel, uint32_t face, const uint32_t* receivers, uint32_t n) {
    const f3 normal = face_normal(face);
    i3 key = voxel;
    f3 surface = add(adds(f3{(float)voxel.x, (float)voxel.y, (float)voxel.z}, 0.5f), muls(normal, 0.5f));
    const int32_t s = n ? voxel_stride(x, voxel) : 1;
    if (s != 1) {
        key = i3{voxel.x & -s, voxel.y & -s, voxel.z & -s};
        surface = add(f3{(float)key.x, (float)key.y, (float)key.z}, muls(adds(muls(normal, 0.5f), 0.5f), (float)s));
    }
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* r = receivers + (size_t)i * 8;
        if (r[3] == face && (int32_t)r[4] == key.x && (int32_t)r[5] == key.y && (int32_t)r[6] == key.z && bitsf(r[0]) == surface.x &&
            bitsf(r[1]) == surface.y && bitsf(r[2]) == surface.z)
            return i;
    }
    return 0xffffffffu;
}
}  // namespace far

int orc_far_frame(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                  const float* materials, const float* lights, const uint32_t* emitters, const uint32_t* state, const uint32_t* index,
                  const orc_pipeline* pipe, const uint32_t* view_words, const uint32_t* receivers, const uint32_t* estimates,
                  uint32_t n_receivers, const uint32_t* previous, uint32_t* current, uint32_t* output, uint32_t* stats, int threads) {
    using namespace far;
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, emitters, state, index, *pipe};
    const View v{view_words};
    const uint32_t stamp = v.frame() & 0x1fffffffu;
    const float* cam = v.cam();
    output[0] = fbits(cam[0]); output[1] = fbits(cam[1]); output[2] = fbits(cam[2]); output[3] = 0;
    for (int i = 0; i < 4; ++i) {
        output[4 + i] = fbits(v.axis(i));
        output[8 + i] = v.grid(i);
    }
    output[12] = 0; output[13] = 0; output[14] = fbits(v.tune(0)); output[15] = stamp;
    const uint32_t n_cells = v.grid(0) * v.grid(1);
    std::vector<uint8_t> queued(n_cells, 0);
    std::atomic<uint32_t> st[8];
    for (auto& a : st) a = 0;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    auto run = [&](auto&& body) {
        std::atomic<uint32_t> next{0};
        auto worker = [&]() {
            Ctx x{g, m, Counters{}};
            for (;;) {
                const uint32_t id = next.fetch_add(1);
                if (id >= n_cells) break;
                body(x, id);
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
        worker();
        for (auto& t : pool) t.join();
    };
    // classify_pixels (voxel_view_pixels.wgsl:129-192)
    run([&](Ctx& x, uint32_t id) {
        const uint32_t size = v.grid(2);
        const uint32_t cx = id % v.grid(0), cy = id / v.grid(0);
        const uint32_t k = (v.frame() * 5u + (cx ^ cy)) % (size * size);
        const uint32_t px = cx * size + k % size, py = cy * size + k / size;
        if (px >= v.width() || py >= v.height()) return;
        const f3 eye = v.eye();
        const RayResult hit = trace_domain_limited(x, eye, camera_ray(cam, px, py, v.width(), v.height()), x.extra(1), true, 2048u);
        if (hit.status != 1u) return;
        f3 surface = hit.position;
        if (((v.grid(3) >> 1u) & 3u) == 0u && v.axis(3) > (1.05f * v.tune(0)) * length(sub(surface, eye))) return;
        const uint32_t face = face_index_of(hit.normal);
        if (face >= 6u) return;
        const f3 normal = face_normal(face);
        set_comp(surface, face / 2u, std::nearbyint(comp(surface, face / 2u)));
        const f3 inner = sub(surface, muls(normal, 0.01f));
        const i3 voxel{(int32_t)std::floor(inner.x), (int32_t)std::floor(inner.y), (int32_t)std::floor(inner.z)};
        if (!in_interest(v, voxel) || !pixel_owned(x, v, voxel, face)) return;
        st[0] += 1;
        f3 mean;
        float count;
        uint32_t sequence;
        previous_cell(x, v, previous, surface, face, voxel, mean, count, sequence);
        if (count > 0.0f) {
            st[3] += 1;
        } else {
            const uint32_t o = owner(x, voxel, face, receivers, n_receivers);
            if (o != 0xffffffffu && bitsf(estimates[(size_t)o * 16 + 3]) > 0.0f) {
                const uint32_t* e = estimates + (size_t)o * 16;
                mean = f3{bitsf(e[0]), bitsf(e[1]), bitsf(e[2])};
                count = bitsf(e[3]);
                sequence = e[12];
                st[4] += 1;
            }
        }
        const float capped = wmin(count, v.tune(1));
        st[2] += (uint32_t)capped;
        const Cell value{mean, capped, surface, face | (stamp << 3u), sequence};
        store(current, id, value);
        const uint32_t rate = std::max((uint32_t)v.tune(2), 1u);
        if (capped < 4.0f || (id + v.frame()) % rate == 0u) queued[id] = 1;
        else write_output(x, v, output, id, value);
    });
    // trace_pixel_queue (voxel_view_pixels.wgsl:199-216)
    run([&](Ctx& x, uint32_t id) {
        if (!queued[id]) return;
        Cell cell = load(current, id);
        st[1] += 1;
        const uint32_t stream = pcg(id * 9781u + 0x9e3779b9u);
        const ReceiverSample sample = trace_receiver(x, cell.surface, face_normal(cell.face & 7u), stream, cell.sequence);
        cell.sequence += 1u;
        if (sample.known) {
            cell.count = wmin(cell.count + 1.0f, v.tune(1));
            const float t = 1.0f / cell.count;
            cell.mean = add(muls(cell.mean, 1.0f - t), muls(f3{sample.energy.x, sample.energy.y, sample.energy.z}, t));
        }
        store(current, id, cell);
        write_output(x, v, output, id, cell);
    });
    for (int i = 0; i < 8; ++i) stats[i] = st[i];
    return 0;
}

// ---- reconstruction and presentation of the view receivers -------------------------
// receivers: 8 words each (surface xyz, face, voxel xyz, sequence);
// estimates: 16 (mean, moment, shown, identity); conts: 32; tile_of: a tile
// per receiver (all ones: none); published: 12 words each (FarPixel).
namespace recon {
static const f3 LUM{0.2126f, 0.7152f, 0.0722f};
static f3 w3(const uint32_t* w) { return f3{bitsf(w[0]), bitsf(w[1]), bitsf(w[2])}; }

// voxel_view_runtime.wgsl:383-394
static float mean_variance(const uint32_t* e, float reference) {
    const f3 mean = w3(e), moment = w3(e + 4);
    const float n = wmax(bitsf(e[3]), 1.0f);
    const float m = dot(mean, LUM);
    const f3 channel{wmax(moment.x - mean.x * mean.x, 0.0f), wmax(moment.y - mean.y * mean.y, 0.0f), wmax(moment.z - mean.z * mean.z, 0.0f)};
    const float deviation = dot(f3{std::sqrt(channel.x), std::sqrt(channel.y), std::sqrt(channel.z)}, LUM);
    const float prior = m * m;
    const float rest = wmax(n - 1.0f, 0.0f);
    const float shrunk = (deviation * deviation * rest + prior * 64.0f) / (rest + 64.0f);
    const float unseen = reference / n;
    return shrunk / n + unseen * unseen;
}

// voxel_view_runtime.wgsl:396-404 (each caller-given receiver owns itself)
static bool coplanar_donor(const uint32_t* receivers, const uint32_t* r, f3 normal, uint32_t candidate) {
    const uint32_t* d = receivers + (size_t)candidate * 8;
    if (d[3] != r[3]) return false;
    const f3 delta = sub(w3(d), w3(r));
    const uint32_t u = (r[3] / 2u + 1u) % 3u;
    const float reach = 16.0f * (2.0f * (bitsf(r[u]) - (float)(int32_t)r[4 + u]));
    return std::fabs(dot(delta, normal)) <= 0.05f && dot(delta, delta) <= reach * reach;
}

static f3 mix3(f3 a, f3 b, float t) { return add(muls(a, 1.0f - t), muls(b, t)); }
}  // namespace recon

int orc_reconstruct(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                    const float* materials, const float* lights, const uint32_t* emitters, const orc_pipeline* pipe, const uint32_t* receivers,
                    uint32_t* estimates, const uint32_t* conts, const uint32_t* tile_of, uint32_t tiles_x, uint32_t tiles_y, uint32_t n,
                    const float* display, uint32_t custom, uint32_t* published, uint32_t* stats) {
    using namespace recon;
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, emitters, nullptr, nullptr, *pipe};
    Ctx x{g, m, Counters{}};
    const uint32_t n_tiles = tiles_x * tiles_y;
    std::vector<std::vector<uint32_t>> lists(n_tiles);
    for (uint32_t i = 0; i < n; ++i)
        if (tile_of[i] < n_tiles) lists[tile_of[i]].push_back(i);
    // Every receiver reads the estimates as they were before this pass.
    const std::vector<uint32_t> before(estimates, estimates + (size_t)n * 16);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* r = receivers + (size_t)i * 8;
        const uint32_t tile = tile_of[i];
        if (r[3] >= 6u || tile >= n_tiles) continue;
        const uint32_t* center = before.data() + (size_t)i * 16;
        const f3 normal = face_normal(r[3]);
        const int32_t tx = (int32_t)(tile % tiles_x), ty = (int32_t)(tile / tiles_x);
        const float center_luminance = dot(w3(center), LUM);
        float reference = center_luminance;
        // body(lane, donor): the window's tiles in row-major order, tile k
        // belonging to lane k mod 32 (the GPU's warp split).
        auto visit = [&](int32_t radius, auto&& body) {
            const int32_t side = 2 * radius + 1;
            for (int32_t k = 0; k < side * side; ++k) {
                const int32_t qx = tx + k % side - radius, qy = ty + k / side - radius;
                if (qx < 0 || qy < 0 || qx >= (int32_t)tiles_x || qy >= (int32_t)tiles_y) continue;
                for (uint32_t candidate : lists[(uint32_t)qy * tiles_x + (uint32_t)qx]) {
                    if (candidate == i || !coplanar_donor(receivers, r, normal, candidate)) continue;
                    body(k % 32, before.data() + (size_t)candidate * 16);
                }
            }
        };
        visit(1, [&](int32_t, const uint32_t* value) {
            if (bitsf(value[3]) > 0.0f) reference = wmax(reference, dot(w3(value), LUM));
        });
        const float center_variance = mean_variance(center, reference);
        const float tolerance = display[0] * center_luminance;
        const float tol2 = tolerance * tolerance;
        const float deficit = center_variance / wmax(tol2, 1e-12f);
        const int32_t radius = (int32_t)wclamp(std::ceil(std::sqrt(deficit / 3.14159f) * 0.5f), 1.0f, 4.0f);
        const bool unsampled = bitsf(center[3]) <= 0.0f;
        f3 sum{0, 0, 0};
        float weight = 0.0f;
        if (!unsampled) {
            const float w = 1.0f / wmax(center_variance, 1e-12f);
            sum = muls(w3(center), w);
            weight = w;
        }
        if ((unsampled || center_variance > tol2) && display[1] > 0.0f) {
            f3 part[32];
            float part_w[32];
            for (int l = 0; l < 32; ++l) {
                part[l] = f3{0, 0, 0};
                part_w[l] = 0.0f;
            }
            visit(radius, [&](int32_t lane, const uint32_t* value) {
                if (bitsf(value[3]) <= 0.0f) return;
                const float variance = mean_variance(value, reference);
                float bias2 = 0.0f;
                if (!unsampled) {
                    const float difference = dot(w3(value), LUM) - center_luminance;
                    bias2 = wmax(difference * difference - variance - center_variance, 0.0f);
                }
                const float w = 1.0f / wmax(variance + bias2, 1e-12f);
                part[lane] = add(part[lane], muls(w3(value), w));
                part_w[lane] = part_w[lane] + w;
            });
            for (int l = 0; l < 32; ++l) {
                sum = add(sum, part[l]);
                weight = weight + part_w[l];
            }
        }
        if (weight <= 0.0f) continue;
        const float keep = unsampled ? 0.0f : 1.0f - display[1];
        const f3 desired = mix3(divs(sum, weight), w3(center), keep);
        const float blend = bitsf(center[11]) > 0.0f ? display[2] : 1.0f;
        const f3 shown = mix3(w3(center + 8), desired, blend);
        uint32_t* out = estimates + (size_t)i * 16 + 8;
        out[0] = fbits(shown.x); out[1] = fbits(shown.y); out[2] = fbits(shown.z); out[3] = fbits(1.0f);
    }
    // publish_view (voxel_view_runtime.wgsl:476-521)
    for (int k = 0; k < 5; ++k) stats[k] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* r = receivers + (size_t)i * 8;
        uint32_t* o = published + (size_t)i * 12;
        std::fill(o, o + 12, 0u);
        o[3] = 0xffffffffu;
        if (r[3] >= 6u) continue;
        const uint32_t* e = estimates + (size_t)i * 16;
        f3 irradiance = w3(e + 8);
        if (custom) irradiance = add(irradiance, direct_at(x, w3(r), face_normal(r[3])).custom);
        const float count = bitsf(e[3]);
        const bool lit = bitsf(e[11]) > 0.0f || irradiance.x > 0.0f || irradiance.y > 0.0f || irradiance.z > 0.0f;
        const float evidence = lit ? wmax(count, 0.001f) : 0.0f;
        o[0] = r[0]; o[1] = r[1]; o[2] = r[2]; o[3] = r[3];
        o[4] = fbits(irradiance.x); o[5] = fbits(irradiance.y); o[6] = fbits(irradiance.z); o[7] = fbits(evidence);
        for (uint32_t corner = 0; corner < 4u; ++corner) {
            const uint32_t byte = (e[14] >> (corner * 8u)) & 255u;
            o[8 + corner] = (byte & 15u) | ((byte & 128u) << 24u);
        }
        stats[0] += (uint32_t)count;
        stats[1] = std::max(stats[1], (uint32_t)count);
        if (count == 0.0f) stats[2] += 1;
        if (evidence > 0.0f) stats[3] += 1;
        if (conts[(size_t)i * 32 + 19] == 1u) stats[4] += 1;
    }
    return 0;
}

// corner_value (voxel_gi_presentation.wesl:353-361); value = rgb, w = weight.
static f3 corner_value(F4 c, F4 eu, F4 ev, F4 diag) {
    float sx = c.x * c.w + eu.x * eu.w + ev.x * ev.w;
    float sy = c.y * c.w + eu.y * eu.w + ev.y * ev.w;
    float sz = c.z * c.w + eu.z * eu.w + ev.z * ev.w;
    float sw = c.w + eu.w + ev.w;
    if (eu.w > 0.0f || ev.w > 0.0f) {
        sx = sx + diag.x * diag.w;
        sy = sy + diag.y * diag.w;
        sz = sz + diag.z * diag.w;
        sw = sw + diag.w;
    }
    const float d = wmax(sw, 0.000001f);
    return f3{sx / d, sy / d, sz / d};
}

int orc_corner_value(const float* center, const float* edge_u, const float* edge_v, const float* diagonal, float* out3) {
    const f3 v = corner_value(ld4(center), ld4(edge_u), ld4(edge_v), ld4(diagonal));
    out3[0] = v.x; out3[1] = v.y; out3[2] = v.z;
    return 0;
}

// corner_irradiance (voxel_gi_presentation.wesl:377-412) at each pixel's first hit.
int orc_present(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                const uint32_t* published, uint32_t n, const float* cam, uint32_t w, uint32_t h, int corners, float* image, int threads) {
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, nullptr, nullptr, nullptr, nullptr, nullptr, orc_pipeline{1, 0, 2048, 0, 1}};
    std::unordered_map<uint64_t, uint32_t> index;  // (face, surface) -> published entry
    auto key = [](uint32_t face, uint32_t a, uint32_t b, uint32_t c) {
        uint64_t k = face;
        k = k * 0x9e3779b97f4a7c15ull ^ a;
        k = k * 0x9e3779b97f4a7c15ull ^ b;
        return k * 0x9e3779b97f4a7c15ull ^ c;
    };
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* p = published + (size_t)i * 12;
        if (p[3] < 6u) index.emplace(key(p[3], p[0], p[1], p[2]), i);
    }
    auto display_face = [&](i3 voxel, uint32_t face, int32_t s) -> F4 {
        const f3 nrm = face_normal(face);
        const f3 surface = add(f3{(float)voxel.x, (float)voxel.y, (float)voxel.z}, muls(adds(muls(nrm, 0.5f), 0.5f), (float)s));
        auto it = index.find(key(face, fbits(surface.x), fbits(surface.y), fbits(surface.z)));
        if (it == index.end()) return F4{0, 0, 0, 0};
        const uint32_t* p = published + (size_t)it->second * 12;
        if (p[3] != face || p[0] != fbits(surface.x) || p[1] != fbits(surface.y) || p[2] != fbits(surface.z)) return F4{0, 0, 0, 0};
        return F4{bitsf(p[4]), bitsf(p[5]), bitsf(p[6]), wmin(bitsf(p[7]), 1.0f)};
    };
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        Ctx x{g, m, Counters{}};
        for (;;) {
            const uint32_t id = next.fetch_add(1);
            if (id >= w * h) break;
            float* o = image + (size_t)id * 4;
            const f3 eye{cam[0], cam[1], cam[2]};
            const RayResult hit = trace_domain_limited(x, eye, camera_ray(cam, id % w, id / w, w, h), x.extra(1), true, 2048u);
            if (hit.status != 1u) {
                o[0] = o[1] = o[2] = o[3] = 0.0f;
                continue;
            }
            const f3 position = hit.position, normal = hit.normal;
            const f3 inner = sub(position, muls(normal, 0.01f));
            const i3 cell{(int32_t)std::floor(inner.x), (int32_t)std::floor(inner.y), (int32_t)std::floor(inner.z)};
            const int32_t s = far::voxel_stride(x, cell);
            const i3 voxel{cell.x & -s, cell.y & -s, cell.z & -s};
            uint32_t face = 0u;
            i3 u{0, s, 0}, v{0, 0, s};
            if (std::fabs(normal.y) > 0.5f) {
                face = 2u;
                u = i3{s, 0, 0};
            } else if (std::fabs(normal.z) > 0.5f) {
                face = 4u;
                u = i3{s, 0, 0};
                v = i3{0, s, 0};
            }
            const uint32_t axis = face / 2u;
            face += (axis == 0u ? normal.x : (axis == 1u ? normal.y : normal.z)) < 0.0f ? 1u : 0u;
            const F4 center = display_face(voxel, face, s);
            if (!corners) {
                o[0] = center.x; o[1] = center.y; o[2] = center.z; o[3] = center.w;
                continue;
            }
            auto at = [&](int32_t du, int32_t dv) {
                return display_face(i3{voxel.x + du * u.x + dv * v.x, voxel.y + du * u.y + dv * v.y, voxel.z + du * u.z + dv * v.z}, face, s);
            };
            const F4 left = at(-1, 0), right = at(1, 0), bottom = at(0, -1), top = at(0, 1);
            const f3 c00 = corner_value(center, left, bottom, at(-1, -1));
            const f3 c10 = corner_value(center, right, bottom, at(1, -1));
            const f3 c01 = corner_value(center, left, top, at(-1, 1));
            const f3 c11 = corner_value(center, right, top, at(1, 1));
            const f3 local = divs(sub(position, f3{(float)voxel.x, (float)voxel.y, (float)voxel.z}), (float)(s * s));
            const float ux = wclamp(dot(local, f3{(float)u.x, (float)u.y, (float)u.z}), 0.0f, 1.0f);
            const float uy = wclamp(dot(local, f3{(float)v.x, (float)v.y, (float)v.z}), 0.0f, 1.0f);
            const f3 rgb = recon::mix3(recon::mix3(c00, c10, ux), recon::mix3(c01, c11, ux), uy);
            o[0] = rgb.x; o[1] = rgb.y; o[2] = rgb.z; o[3] = center.w;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return 0;
}

// candidate keys only, for slots [controls[26], controls[27]).
int orc_classify(const uint32_t* slot_meta, uint32_t* keys, uint32_t n_slots, const uint32_t* ctl) {
    for (uint32_t slot = ctl[26]; slot < ctl[27] && slot < n_slots; ++slot) keys[slot] = candidate_key(slot_meta, slot, ctl);
    return 0;
}

// select_classify, select_histogram, select_threshold and select_emit over
// n_slots slots. keys: one word per slot (kept between calls, as the GPU's);
// selection: 1038 words, zeroed by the caller; emit takes ties and picks in
// slot order. tasks (8 words), pick_slots and picks (4 words) per task from
// batch.x (controls[24]) up to the budget (controls[23]).
int orc_select(const uint32_t* state, uint32_t* slot_meta, uint32_t* keys, uint32_t n_slots, const uint32_t* ctl, uint32_t* selection,
               uint32_t* tasks, uint32_t* pick_slots, uint32_t* picks) {
    const uint32_t MIRROR_STALE = 0x20000000u;
    for (uint32_t slot = ctl[26]; slot < ctl[27] && slot < n_slots; ++slot) {
        keys[slot] = candidate_key(slot_meta, slot, ctl);
        uint32_t* rank = slot_meta + ((size_t)slot * 3 + 2) * 4;
        const bool stale = (rank[3] & MIRROR_STALE) != 0u && (slot_meta[(size_t)slot * 12 + 3] & 8u) != 0u;
        if (stale) {
            if (selection[1037] < ctl[32]) rank[3] &= ~MIRROR_STALE;
            selection[1037] += 1u;
        }
    }
    for (uint32_t slot = 0; slot < n_slots; ++slot)
        if (keys[slot] != 0xffffffffu) selection[umin(keys[slot] >> 8u, 3u) * 256u + (keys[slot] & 255u)] += 1u;
    uint32_t scan[4][256];
    for (uint32_t c = 0; c < 4; ++c) {
        uint32_t sum = 0;
        for (uint32_t t = 0; t < 256; ++t) scan[c][t] = (sum += selection[c * 256u + t]);
    }
    const uint32_t budget = ctl[23];
    uint32_t take[4] = {0, 0, 0, 0};
    take[3] = umin(scan[3][255], budget - budget / 4u);
    const uint32_t rest = budget - take[3];
    take[0] = umin(rest / 4u, scan[0][255]);
    take[1] = umin(rest / 2u, scan[1][255]);
    take[2] = umin(rest - rest / 4u - rest / 2u, scan[2][255]);
    uint32_t spare = budget - take[0] - take[1] - take[2] - take[3];
    const uint32_t lend[4] = {1u, 0u, 2u, 3u};
    for (uint32_t o = 0; o < 4; ++o) {
        const uint32_t c = lend[o];
        const uint32_t extra = umin(spare, scan[c][255] - take[c]);
        take[c] += extra;
        spare -= extra;
    }
    for (uint32_t c = 0; c < 4; ++c) {
        selection[1024 + c] = 256u;
        selection[1028 + c] = 0u;
        for (uint32_t t = 0; t < 256; ++t) {
            const uint32_t below = t > 0 ? scan[c][t - 1] : 0u;
            if (take[c] > 0u && below < take[c] && scan[c][t] >= take[c]) {
                selection[1024 + c] = t;
                selection[1028 + c] = take[c] - below;
            }
        }
    }
    for (uint32_t slot = 0; slot < n_slots; ++slot) {
        const uint32_t key = keys[slot];
        if (key == 0xffffffffu) continue;
        const uint32_t group = umin(key >> 8u, 3u), bucket = key & 255u;
        const uint32_t threshold = selection[1024 + group];
        if (bucket > threshold) continue;
        bool accept = true;
        if (bucket == threshold) accept = selection[1032 + group]++ < selection[1028 + group];
        if (!accept) continue;
        const uint32_t pick = selection[1036]++;
        if (pick >= budget) continue;
        keys[slot] = 0xffffffffu;
        const uint32_t* identity = slot_meta + (size_t)slot * 12;
        if ((identity[3] & 8u) == 0u) continue;
        const uint32_t task = ctl[24] + pick;
        const uint32_t* st = state + (size_t)slot * 36;
        uint32_t* tk = tasks + (size_t)task * 8;
        tk[0] = identity[0]; tk[1] = identity[1]; tk[2] = identity[2]; tk[3] = identity[3] & 7u;
        tk[4] = st[6];
        pick_slots[task] = slot;
        uint32_t* pr = picks + (size_t)task * 4;
        pr[0] = slot; pr[1] = slot_meta[(size_t)slot * 12 + 6]; pr[2] = st[5] & 0x3fffffffu; pr[3] = st[28];
    }
    return 0;
}

// apply_events (voxel_accumulate.wgsl:295-332) over slots [0, n_slots).
int orc_apply_events(uint32_t* state, uint32_t* slot_meta, uint32_t* checkpoint, const uint32_t* events, uint32_t n_slots,
                     const uint32_t* controls) {
    const uint32_t URGENT = 0x40000000u;
    float physical = bitsf(controls[11]);
    for (uint32_t slot = 0; slot < n_slots; ++slot) {
        uint32_t* identity = slot_meta + (size_t)slot * 12;
        if ((identity[3] & 8u) == 0u) continue;
        int32_t p[3] = {(int32_t)identity[0], (int32_t)identity[1], (int32_t)identity[2]};
        Retention r = resolve_retention(events, p, controls[13], controls[15], physical > 0.0f, controls[30], controls[31]);
        bool urgent = r.urgent;
        if (r.limit != NO_LIMIT) {
            uint32_t* base = state + (size_t)slot * 36;
            base[5] = umin(base[5], r.limit);
            uint32_t* rank = slot_meta + ((size_t)slot * 3 + 2) * 4;
            rank[3] = (rank[3] & 0xe0000000u) | (base[5] & 0x1fffffffu);
            checkpoint[(size_t)slot * 12 + 9] = umin(checkpoint[(size_t)slot * 12 + 9], r.limit);
        }
        uint32_t* sched = slot_meta + ((size_t)slot * 3 + 1) * 4;
        if (r.measured && r.change > 0.0f) sched[0] = fbits(bitsf(sched[0]) + r.change);
        if (r.urgent_if_binding) {
            float pending = bitsf(sched[0]);
            urgent = urgent || !r.measured || (pending > 0.0f && binds(state, slot, pending, physical));
        }
        if (r.woken || urgent) sched[1] &= 0xfffffff0u;
        if (urgent) slot_meta[((size_t)slot * 3 + 2) * 4 + 3] |= URGENT;
    }
    return 0;
}

// choose_emitter (voxel_path.wgsl:309-324) for n uniforms at one receiver:
// out gets (voxel xyz, face, selection probability bits) per choice. The
// emitter words are GpuEmitter records then light-tree nodes, as uploaded.
int orc_choose_emitters(const uint32_t* emitters, uint32_t n_emitters, float total, const float* position, const float* normal,
                        const float* choices, uint32_t n, uint32_t* out) {
    float params[24] = {0};
    params[18] = total;
    params[19] = (float)n_emitters;
    Geometry g{};
    Model m{params, nullptr, nullptr, emitters, nullptr, nullptr, orc_pipeline{1, 0, 64, 0, 1}};
    Ctx x{g, m, Counters{}};
    const f3 p{position[0], position[1], position[2]}, nn{normal[0], normal[1], normal[2]};
    for (uint32_t i = 0; i < n; ++i) {
        Emissive e = choose_emitter(x, p, nn, choices[i]);
        uint32_t* o = out + (size_t)i * 5;
        o[0] = (uint32_t)e.voxel.x; o[1] = (uint32_t)e.voxel.y; o[2] = (uint32_t)e.voxel.z; o[3] = e.face;
        o[4] = fbits(e.sampling.y);
    }
    return 0;
}

// The light tree's probability of selecting the emitter face (voxel, face)
// from a receiver (tree_probability, voxel_path.wgsl:159-174).
float orc_emitter_probability(const uint32_t* emitters, uint32_t n_emitters, float total, const float* position, const float* normal,
                              const int32_t* voxel, uint32_t face) {
    float params[24] = {0};
    params[18] = total;
    params[19] = (float)n_emitters;
    Geometry g{};
    Model m{params, nullptr, nullptr, emitters, nullptr, nullptr, orc_pipeline{1, 0, 64, 0, 1}};
    Ctx x{g, m, Counters{}};
    return tree_probability(x, f3{position[0], position[1], position[2]}, f3{normal[0], normal[1], normal[2]},
                            i3{voxel[0], voxel[1], voxel[2]}, face_normal(face));
}

// measure_edits + finish_edits (voxel_accumulate.wgsl:375-425) for the
// measured edit bounds of an encoded event list (encode_events,
// src/gpu/resident.rs:1326-1414). `measures` holds 3 uint4 per entry:
// (bound record, first position, positions, changed voxels),
// (scan min xyz, own flux bits), (scan size xyz, 0). `material_light` holds
// (albedo luminance, emission luminance) per material. For every position of
// an entry's scan box, the brightest outgoing luminance of its traced faces
// (albedo * (mean + direct luminance) + emission) is taken; the bound then
// gets flux = own + brightest * 2 * voxels and kind 3 (measured edit), or
// kind 0 (unknown) when no traced face was seen. Rewrites `events` in place.
int orc_measure_edits(const uint32_t* state, const uint32_t* slot_meta, const uint32_t* index, const float* material_light,
                      const uint32_t* measures, uint32_t n_entries, uint32_t* events) {
    const uint32_t mask = index[0], probes = index[1];
    for (uint32_t e = 0; e < n_entries; ++e) {
        const uint32_t* a = measures + (size_t)e * 12;
        const uint32_t* b = a + 4;
        const uint32_t* c = a + 8;
        float brightest = 0.0f;
        bool observed = false;
        for (uint32_t local = 0; local < a[2]; ++local) {
            const uint32_t off[3] = {local % c[0], (local / c[0]) % c[1], local / (c[0] * c[1])};
            const int32_t p[3] = {(int32_t)b[0] + (int32_t)off[0], (int32_t)b[1] + (int32_t)off[1], (int32_t)b[2] + (int32_t)off[2]};
            for (uint32_t face = 0; face < 6u; ++face) {
                // face_slot (voxel_accumulate.wgsl:357-370)
                uint32_t slot = NO_LIMIT;
                uint32_t probe = (hash_voxel(p[0], p[1], p[2]) ^ pcg(face + 1u)) & mask;
                for (uint32_t attempt = 0; attempt < probes; ++attempt) {
                    const uint32_t* entry = index + ((size_t)probe + 1) * 4;
                    if (entry[3] == 0xffffffffu) break;
                    if ((int32_t)entry[0] == p[0] && (int32_t)entry[1] == p[1] && (int32_t)entry[2] == p[2] && (entry[3] >> 29u) == face) {
                        slot = entry[3] & 0x1fffffffu;
                        break;
                    }
                    probe = (probe + 1u) & mask;
                }
                if (slot == NO_LIMIT) continue;
                const uint32_t* identity = slot_meta + (size_t)slot * 12;
                if ((identity[3] & 8u) == 0u) continue;
                const uint32_t* base = state + (size_t)slot * 36;
                if ((base[5] & 0x7fffffffu) == 0u) continue;
                observed = true;
                const float incident = lum(stF4(base)) + lum(stF4(base + 16));
                const float* light = material_light + (size_t)(identity[3] >> 16) * 2;
                brightest = wmax(brightest, light[0] * incident + light[1]);
            }
        }
        uint32_t* record = events + (size_t)a[0] * 4;
        if (!observed) {
            record[7] &= 0xfffffff8u;
            continue;
        }
        record[3] = fbits(bitsf(b[3]) + brightest * 2.0f * (float)a[3]);
        record[7] = (record[7] & 0xfffffff8u) | 3u;
    }
    return 0;
}

// The (voxel, face) -> slot index as the worker builds it (face_index.rs:36-97):
// capacity 1024, doubled before an insert would exceed half load; faces
// inserted in slot order. out: words of [mask, 64, 0, 0] then entries;
// returns the number of uint4 words written (capacity + 1), or -1 if
// `out_capacity` is too small.
namespace {
struct FaceTable {
    std::vector<uint32_t> e;
    uint64_t len = 0;
    explicit FaceTable(uint64_t cap) : e(cap * 4, 0) { for (uint64_t i = 0; i < cap; ++i) e[i * 4 + 3] = 0xffffffffu; }
    uint64_t cap() const { return e.size() / 4; }
    void insert(int32_t x, int32_t y, int32_t z, uint32_t face, uint32_t slot) {
        uint64_t mask = cap() - 1;
        uint64_t home = (hash_voxel(x, y, z) ^ pcg(face + 1u)) & mask;
        for (uint64_t j = home;; j = (j + 1) & mask) {
            if (e[j * 4 + 3] == 0xffffffffu) break;
            if ((int32_t)e[j * 4] == x && (int32_t)e[j * 4 + 1] == y && (int32_t)e[j * 4 + 2] == z && (e[j * 4 + 3] >> 29) == face) {
                e[j * 4 + 3] = (face << 29) | slot;
                return;
            }
        }
        if ((len + 1) * 2 > cap()) { grow(); mask = cap() - 1; home = (hash_voxel(x, y, z) ^ pcg(face + 1u)) & mask; }
        uint64_t idx = home;
        while (e[idx * 4 + 3] != 0xffffffffu) idx = (idx + 1) & mask;
        e[idx * 4] = (uint32_t)x; e[idx * 4 + 1] = (uint32_t)y; e[idx * 4 + 2] = (uint32_t)z;
        e[idx * 4 + 3] = (face << 29) | slot;
        len += 1;
    }
    void grow() {
        std::vector<uint32_t> old;
        old.swap(e);
        uint64_t old_cap = old.size() / 4;
        e.assign(old_cap * 2 * 4, 0);
        for (uint64_t i = 0; i < old_cap * 2; ++i) e[i * 4 + 3] = 0xffffffffu;
        len = 0;
        for (uint64_t i = 0; i < old_cap; ++i)
            if (old[i * 4 + 3] != 0xffffffffu)
                insert((int32_t)old[i * 4], (int32_t)old[i * 4 + 1], (int32_t)old[i * 4 + 2], old[i * 4 + 3] >> 29,
                       old[i * 4 + 3] & 0x1fffffffu);
    }
};
}  // namespace

int64_t orc_face_index(const int32_t* faces /*4 per face: xyz, face*/, uint32_t n, uint32_t* out, uint64_t out_capacity) {
    FaceTable t(1024);
    for (uint32_t s = 0; s < n; ++s) {
        const int32_t* f = faces + (size_t)s * 4;
        t.insert(f[0], f[1], f[2], (uint32_t)f[3], s);
    }
    uint64_t cap = t.cap();
    if (cap + 1 > out_capacity) return -1;
    out[0] = (uint32_t)(cap - 1); out[1] = 64; out[2] = 0; out[3] = 0;
    std::copy(t.e.begin(), t.e.end(), out + 4);
    return (int64_t)(cap + 1);
}

}  // extern "C"

// ---- view tier -------------------------------------------------------------
// voxel_view_trace.wgsl (trace_view_paths, advance_view_path),
// voxel_view_runtime.wgsl:272-349 (trace_visible_paths, retain_view_history)
// and voxel_view_cache.wgsl:6-98, 188-258 (shared_slot, load_shared_face,
// store_shared_faces), for a receiver list the caller gives (one receiver
// per visible unit face, so every receiver owns itself). Records are the
// shaders' layouts in 32-bit words:
//   ViewReceiver 8       surface xyz, face | voxel xyz, sequence
//   ViewPath 32          surface, sequence | voxel, face | direction, proposal_pdf |
//                        hit_position, hit_status | hit_voxel, hit_face |
//                        emitter, known | continuation, hit_material | direct, stream
//   ViewContinuation 32  radiance | extra | throughput | origin, bounce |
//                        direction, status | previous_position, 0 | previous_normal, 0 | ticket
//                        (status: 0 new, 1 paused, 2 complete known, 3 complete unknown, 4 inactive)
//   ViewEstimate 16      mean | moment | shown | identity (next sequence, material, corners, incarnation)
// `queue` holds 12 counters, the owner list (n) and a word per receiver (n):
// the owner's rank, replaced by its reserved sequence cursor when it loads
// the shared face. The topology prior of new faces (bootstrap_face) and the
// sun-corner records belong to raster discovery and are not restated.
namespace orc {
namespace view {

constexpr uint32_t OWNERS = 0, COMPLETED = 2, KNOWN = 3, ATTEMPTED = 9, CACHE_LOADS = 10, CACHE_PROMOTIONS = 11, PREFIX = 12;

static f3 rf3(const uint32_t* w) { return f3{bitsf(w[0]), bitsf(w[1]), bitsf(w[2])}; }
static i3 ri3(const uint32_t* w) { return i3{(int32_t)w[0], (int32_t)w[1], (int32_t)w[2]}; }
static void wf3(uint32_t* w, f3 v) { w[0] = fbits(v.x); w[1] = fbits(v.y); w[2] = fbits(v.z); }
static void wi3(uint32_t* w, i3 v) { w[0] = (uint32_t)v.x; w[1] = (uint32_t)v.y; w[2] = (uint32_t)v.z; }
static void wF4(uint32_t* w, F4 v) { w[0] = fbits(v.x); w[1] = fbits(v.y); w[2] = fbits(v.z); w[3] = fbits(v.w); }
static F4 rF4(const uint32_t* w) { return F4{bitsf(w[0]), bitsf(w[1]), bitsf(w[2]), bitsf(w[3])}; }
static f3 rgb(F4 v) { return f3{v.x, v.y, v.z}; }

struct Wave { uint32_t range[4]; uint32_t ticket[4]; };

// trace_view_paths (voxel_view_trace.wgsl:40-72) for path `id` of
// receivers x samples.
static void trace_view_path(Ctx& x, const uint32_t* receiver, uint32_t id, uint32_t samples, uint32_t* record) {
    for (int i = 0; i < 32; ++i) record[i] = 0u;
    if (receiver[3] >= 6u) return;
    const f3 surface = rf3(receiver);
    const i3 voxel = ri3(receiver + 4);
    const uint32_t face = receiver[3];
    const f3 normal = face_normal(face);
    const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u);
    const uint32_t sequence = receiver[7] + id % samples;
    // sample_receiver_path (voxel_path.wgsl:504-513)
    const f3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
    const Energy emitter = sample_emitter(x, surface, normal, stream, sequence, 0u);
    PathEnergy continuation;
    if (dot(normal, direction) > 0.0f) {
        PathState st = begin_path(add(surface, muls(normal, 0.001f)), direction, normal);
        continuation = advance_path(x, st, stream, sequence, x.m.pipe.diffuse_hits, true).result;
    }
    const RayResult& hit = continuation.first_hit;
    wf3(record, surface); record[3] = sequence;
    wi3(record + 4, voxel); record[7] = face;
    wf3(record + 8, direction); record[11] = fbits(cosine_pdf(normal, direction));
    wf3(record + 12, hit.position); record[15] = hit.status;
    wi3(record + 16, hit.voxel); record[19] = face_index_of(hit.normal);
    wf3(record + 20, rgb(emitter.value)); record[23] = continuation.unknown ? 0u : 1u;
    wf3(record + 24, rgb(continuation.energy.value)); record[27] = hit.material;
    wf3(record + 28, rgb(direct_at(x, surface, normal).value)); record[31] = stream;
}

// advance_view_path (voxel_view_trace.wgsl:106-183) with one path per receiver.
static void advance_view_path(Ctx& x, const uint32_t* receiver, uint32_t* record, uint32_t* stored, const Wave& wave) {
    if (receiver[3] >= 6u) {
        for (int i = 0; i < 32; ++i) record[i] = 0u;
        stored[19] = 4u;
        for (int i = 0; i < 4; ++i) stored[28 + i] = wave.ticket[i];
        return;
    }
    const f3 surface = rf3(receiver);
    const i3 voxel = ri3(receiver + 4);
    const uint32_t face = receiver[3];
    const f3 normal = face_normal(face);
    const uint32_t stream = hash_voxel(voxel.x, voxel.y, voxel.z) ^ pcg(face + 1u);
    const uint32_t sequence = receiver[7];
    const uint32_t status = stored[19];
    bool restart = status == 0u || status == 4u;
    for (int i = 0; i < 4; ++i) restart = restart || stored[28 + i] != wave.ticket[i];
    const f3 rs = rf3(record);
    restart = restart || rs.x != surface.x || rs.y != surface.y || rs.z != surface.z;
    restart = restart || (int32_t)record[4] != voxel.x || (int32_t)record[5] != voxel.y || (int32_t)record[6] != voxel.z;
    restart = restart || record[7] != face || record[3] != sequence;
    PathState state;
    if (restart) {
        for (int i = 0; i < 32; ++i) record[i] = 0u;
        wf3(record, surface); record[3] = sequence;
        wi3(record + 4, voxel); record[7] = face;
        const f3 direction = hemisphere(normal, sample_1d(stream, sequence, 0u), sample_1d(stream, sequence, 1u));
        wf3(record + 8, direction);
        record[11] = fbits(cosine_pdf(normal, direction));
        wf3(record + 20, rgb(sample_emitter(x, surface, normal, stream, sequence, 0u).value));
        wf3(record + 28, rgb(direct_at(x, surface, normal).value));
        record[31] = stream;
        state = begin_path(add(surface, muls(normal, 0.001f)), direction, normal);
    } else {
        if (status != 1u) return;
        state.result.energy.value = rF4(stored);
        RayResult first;
        first.voxel = ri3(record + 16);
        first.material = record[27];
        first.position = rf3(record + 12);
        first.status = record[15];
        if (record[19] < 6u) first.normal = face_normal(record[19]);
        state.result.first_hit = first;
        state.throughput = rF4(stored + 8);
        state.origin = rf3(stored + 12);
        state.direction = rf3(stored + 16);
        state.previous_position = rf3(stored + 20);
        state.previous_normal = rf3(stored + 24);
        state.previous_pdf = bitsf(stored[6]);
        state.bounce = stored[15];
    }
    uint32_t steps = umin(wave.range[2], 8u);
    bool terminal = false;
    if (wave.range[3] != 0u) {
        steps = umin(steps, wave.range[3] - umin(state.bounce, wave.range[3]));
        terminal = state.bounce + steps == wave.range[3];
    }
    state = advance_path(x, state, stream, sequence, steps, terminal);
    const RayResult& hit = state.result.first_hit;
    wf3(record + 12, hit.position); record[15] = hit.status;
    wi3(record + 16, hit.voxel); record[19] = face_index_of(hit.normal);
    record[27] = hit.material;
    record[23] = (state.done && !state.result.unknown) ? 1u : 0u;
    wf3(record + 24, state.done ? rgb(state.result.energy.value) : f3{0.0f, 0.0f, 0.0f});
    wF4(stored, state.result.energy.value);
    wF4(stored + 4, F4{0.0f, 0.0f, state.previous_pdf, 0.0f});
    wF4(stored + 8, state.throughput);
    wf3(stored + 12, state.origin); stored[15] = state.bounce;
    wf3(stored + 16, state.direction);
    stored[19] = state.done ? (state.result.unknown ? 3u : 2u) : 1u;
    wf3(stored + 20, state.previous_position);
    wf3(stored + 24, state.previous_normal);
    for (int i = 0; i < 4; ++i) stored[28 + i] = wave.ticket[i];
}

struct Shared {
    uint32_t* state;      // world-cache slots, 36 words
    uint32_t* meta;       // 12 words per slot
    const uint32_t* index; // face index words
    bool enabled;
};

// shared_slot (voxel_view_cache.wgsl:6-26) for a unit face.
static uint32_t shared_slot(const Shared& sh, const uint32_t* receiver, uint32_t material) {
    if (!sh.enabled) return NO_LIMIT;
    const i3 v = ri3(receiver + 4);
    const uint32_t face = receiver[3];
    uint32_t bucket = (hash_voxel(v.x, v.y, v.z) ^ pcg(face + 1u)) & sh.index[0];
    for (uint32_t attempt = 0; attempt < sh.index[1]; ++attempt) {
        const uint32_t* e = sh.index + ((size_t)bucket + 1) * 4;
        if (e[3] == 0xffffffffu) return NO_LIMIT;
        if ((int32_t)e[0] == v.x && (int32_t)e[1] == v.y && (int32_t)e[2] == v.z && (e[3] >> 29u) == face) {
            const uint32_t slot = e[3] & 0x1fffffffu;
            const uint32_t key = sh.meta[(size_t)slot * 12 + 3];
            if ((key & 8u) == 0u || (key >> 16u) != material) return NO_LIMIT;
            return slot;
        }
        bucket = (bucket + 1u) & sh.index[0];
    }
    return NO_LIMIT;
}

}  // namespace view

// The topology prior of load_shared_faces (voxel_view_cache.wgsl:100-186).
namespace prior {
// voxel_material (voxel_traversal.wgsl:48-70)
static uint32_t voxel_material(Ctx& x, i3 v) {
    const i3 r = far::region_of(v);
    if (!in_bounds(x, r)) return 256u;
    const uint32_t index = lookup_region(x, r);
    if (index == 0xffffffffu) return 256u;
    const uint32_t* meta = x.g.headers + (size_t)index * 4;
    if (meta[0] == 1u) return 256u;
    if (meta[0] != 3u) return meta[1];
    const uint32_t lx = (uint32_t)(v.x & 15), ly = (uint32_t)(v.y & 15), lz = (uint32_t)(v.z & 15);
    const uint32_t word = x.g.cells[meta[1] + ((lz >> 2) * 4u + (ly >> 2)) * 4u + (lx >> 2)];
    if ((word & 3u) == 0u) return 256u;
    if ((word & 3u) == 1u) return word >> 2u;
    const uint32_t idx = ((lz & 3u) * 4u + (ly & 3u)) * 4u + (lx & 3u);
    const uint32_t cell = (x.g.cells[(word >> 2u) + idx / 2u] >> ((idx & 1u) * 16u)) & 65535u;
    return (cell & 1u) != 0u ? cell >> 1u : 256u;
}
static bool prior_air(Ctx& x, i3 v) {
    const i3 r = far::region_of(v);
    return in_bounds(x, r) && lookup_region(x, r) != 0xffffffffu && voxel_material(x, v) == 256u;
}
struct FacePrior { f3 mean{0, 0, 0}, moment{0, 0, 0}; float weight = 0.0f; };
struct Donors {
    const uint32_t* receivers;
    uint32_t n;
    const uint32_t* before;  // estimates before the seeding, 16 words each
    const view::Shared* sh;
};
static FacePrior prior_donor(Ctx& x, const Donors& d, i3 voxel, uint32_t face) {
    FacePrior donor;
    const f3 surface = add(adds(f3{(float)voxel.x, (float)voxel.y, (float)voxel.z}, 0.5f), muls(face_normal(face), 0.5f));
    for (uint32_t i = 0; i < d.n; ++i) {
        const uint32_t* r = d.receivers + (size_t)i * 8;
        if (r[3] == face && (int32_t)r[4] == voxel.x && (int32_t)r[5] == voxel.y && (int32_t)r[6] == voxel.z && bitsf(r[0]) == surface.x &&
            bitsf(r[1]) == surface.y && bitsf(r[2]) == surface.z) {
            const uint32_t* e = d.before + (size_t)i * 16;
            if (bitsf(e[3]) >= 16.0f) donor = FacePrior{f3{bitsf(e[0]), bitsf(e[1]), bitsf(e[2])}, f3{bitsf(e[4]), bitsf(e[5]), bitsf(e[6])}, bitsf(e[3])};
            break;
        }
    }
    const uint32_t key[8] = {fbits(surface.x), fbits(surface.y), fbits(surface.z), face, (uint32_t)voxel.x, (uint32_t)voxel.y, (uint32_t)voxel.z, 0u};
    const uint32_t slot = view::shared_slot(*d.sh, key, voxel_material(x, voxel));
    if (slot != 0xffffffffu) {
        const uint32_t* base = d.sh->state + (size_t)slot * 36;
        const uint32_t count = base[5] & 0x7fffffffu;
        if (count >= 16u && (float)count > donor.weight)
            donor = FacePrior{f3{bitsf(base[0]), bitsf(base[1]), bitsf(base[2])}, f3{bitsf(base[8]), bitsf(base[9]), bitsf(base[10])}, (float)count};
    }
    return donor;
}
static void add_prior(FacePrior& sum, const FacePrior& donor, float weight) {
    if (donor.weight == 0.0f) return;
    sum.mean = add(sum.mean, muls(donor.mean, weight));
    sum.moment = add(sum.moment, muls(donor.moment, weight));
    sum.weight = sum.weight + weight;
}
static FacePrior bootstrap_face(Ctx& x, const Donors& d, const uint32_t* r) {
    FacePrior prior;
    const uint32_t rf = r[3];
    const i3 origin{(int32_t)r[4], (int32_t)r[5], (int32_t)r[6]};
    const f3 nf = face_normal(rf);
    const i3 normal{(int32_t)nf.x, (int32_t)nf.y, (int32_t)nf.z};
    const i3 air{origin.x + normal.x, origin.y + normal.y, origin.z + normal.z};
    const uint32_t u = (rf / 2u + 1u) % 3u;
    const int32_t vu = u == 0u ? origin.x : (u == 1u ? origin.y : origin.z);
    if (2.0f * (bitsf(r[u]) - (float)vu) != 1.0f) return prior;
    if (voxel_material(x, origin) == 256u || !prior_air(x, air)) return prior;
    for (uint32_t f = 0; f < 6u; ++f) {
        const f3 o = face_normal(f);
        const i3 off{(int32_t)o.x, (int32_t)o.y, (int32_t)o.z};
        const i3 v{origin.x + off.x, origin.y + off.y, origin.z + off.z};
        const bool covered = off.x == -normal.x && off.y == -normal.y && off.z == -normal.z;
        if (covered || prior_air(x, i3{v.x + normal.x, v.y + normal.y, v.z + normal.z})) add_prior(prior, prior_donor(x, d, v, rf), 1.0f);
    }
    if (prior.weight == 0.0f) {
        for (uint32_t f = 0; f < 6u; ++f) {
            const f3 o = face_normal(f);
            const i3 off{(int32_t)o.x, (int32_t)o.y, (int32_t)o.z};
            const float alignment = dot(f3{(float)normal.x, (float)normal.y, (float)normal.z}, o);
            const float w = alignment > 0.0f ? 1.0f : 0.25f;
            add_prior(prior, prior_donor(x, d, air, f), w);
            const i3 covered{origin.x - off.x, origin.y - off.y, origin.z - off.z};
            if (covered.x != air.x || covered.y != air.y || covered.z != air.z) add_prior(prior, prior_donor(x, d, covered, f), w);
            add_prior(prior, prior_donor(x, d, i3{air.x - off.x, air.y - off.y, air.z - off.z}, f), w);
        }
    }
    if (prior.weight > 0.0f) {
        prior.mean = divs(prior.mean, prior.weight);
        const f3 m2 = divs(prior.moment, prior.weight);
        prior.moment = f3{wmax(m2.x, prior.mean.x * prior.mean.x), wmax(m2.y, prior.mean.y * prior.mean.y), wmax(m2.z, prior.mean.z * prior.mean.z)};
        prior.weight = 1.0f;
    }
    return prior;
}
}  // namespace prior
}  // namespace orc

// Every sun flip reported since the log was last cleared, as (voxel xyz, flux
// bits): the full list behind the 2,048 records and the overflow box, so a
// test can check the GPU's records and overflow whatever order its atomics
// took.
static std::vector<uint32_t>& sun_flip_log() {
    static std::vector<uint32_t> log;
    return log;
}

extern "C" {

uint64_t orc_sun_flip_log(uint32_t* out, uint64_t capacity) {
    const std::vector<uint32_t>& log = sun_flip_log();
    const uint64_t n = log.size() / 4;
    if (out) std::copy(log.begin(), log.begin() + (size_t)std::min(n, capacity) * 4, out);
    return n;
}

void orc_sun_flip_log_clear() { sun_flip_log().clear(); }

// trace_view_paths: `paths` gets 32 words per (receiver, sample).
int orc_trace_view_paths(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                         const float* materials, const float* lights, const uint32_t* emitters, const uint32_t* state,
                         const uint32_t* index, const orc_pipeline* pipe, const uint32_t* receivers, uint32_t n_receivers,
                         uint32_t samples, uint32_t* paths) {
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, emitters, state, index, *pipe};
    for (uint64_t id = 0; id < (uint64_t)n_receivers * samples; ++id) {
        Ctx x{g, m, Counters{}};
        view::trace_view_path(x, receivers + (id / samples) * 8, (uint32_t)id, samples, paths + id * 32);
    }
    return 0;
}

// One view frame over the caller's receivers, in the runtime's order
// (runtime.rs Stage::ORDER): reproject (sequence from the estimate, owner
// queue in receiver order), retain_view_history for one event batch,
// load_shared_faces, trace_visible_paths, store_shared_faces.
// `wave` = range (first, count, max hits, depth), ticket[4];
// `view` = (view_first, shared, clock_ms, n_events, reach, measured_retention bits).

int orc_view_frame(const int32_t* directory, uint64_t slots, const uint32_t* headers, const uint32_t* cells, const float* params,
                   const float* materials, const float* lights, const uint32_t* emitters, uint32_t* state, uint32_t* meta,
                   const uint32_t* index, const orc_pipeline* pipe, uint32_t* receivers, uint32_t n, uint32_t* paths, uint32_t* conts,
                   uint32_t* estimates, uint32_t* queue, const uint32_t* wave_words, const uint32_t* view_words, const uint32_t* events,
                   const uint32_t* far_words, const uint32_t* far_cells, uint32_t* far_stats) {
    using namespace view;
    Geometry g = make_geometry(directory, slots, headers, cells, params);
    Model m{params, materials, lights, emitters, state, index, *pipe};
    Wave wave;
    for (int i = 0; i < 4; ++i) { wave.range[i] = wave_words[i]; wave.ticket[i] = wave_words[4 + i]; }
    const bool view_first = view_words[0] != 0u;
    Shared sh{state, meta, index, view_words[1] != 0u};
    const uint32_t clock = view_words[2], n_events = view_words[3], reach = view_words[4];
    const float physical = bitsf(view_words[5]);
    // The owner queue starts over each frame; the sun-flip region after it
    // keeps building up until the caller reads and clears it (the
    // reference's timing receipt, src/gpu/view/timing.rs:386-387).
    for (uint32_t i = 0; i < PREFIX + 2 * n; ++i) queue[i] = 0u;
    // report_sun_flips (voxel_view_runtime.wgsl:231-270)
    auto report_sun_flips = [&](const uint32_t* r, f3 normal, uint32_t material, uint32_t before, uint32_t after) {
        const f3 w{0.2126f, 0.7152f, 0.0722f};
        const uint32_t nd = fbits(params[11]);
        float flux = 0.0f;
        uint32_t bit = 0u;
        for (uint32_t l = 0; l < nd && bit < 4u; ++l) {
            const float* L = lights + (size_t)l * 12;
            const f3 color{wmax(L[4] - L[9], 0.0f), wmax(L[5] - L[10], 0.0f), wmax(L[6] - L[11], 0.0f)};
            if (color.x == 0.0f && color.y == 0.0f && color.z == 0.0f) continue;
            const float cosine = wmax(dot(normal, normalize(f3{L[0], L[1], L[2]})), 0.0f);
            for (uint32_t corner = 0; corner < 4u; ++corner) {
                const uint32_t a = (before >> (corner * 8u)) & 255u, b = (after >> (corner * 8u)) & 255u;
                if ((a & b & 128u) != 0u && ((a ^ b) & (1u << bit)) != 0u) flux = flux + 0.25f * dot(color, w) * cosine;
            }
            bit += 1u;
        }
        if (flux <= 0.0f) return;
        const float* d = materials + (size_t)(material & 255u) * 16;
        flux = flux * dot(f3{d[0], d[1], d[2]}, w);
        sun_flip_log().insert(sun_flip_log().end(), {r[4], r[5], r[6], fbits(flux)});
        uint32_t* flips = queue + PREFIX + 2 * n;
        const uint32_t slot = flips[0]++;
        if (slot >= 2048u) {
            uint32_t* overflow = flips + 4 + 2048 * 4;
            const int32_t bias = 1073741824;
            for (int k = 0; k < 3; ++k) {
                overflow[k] = umax(overflow[k], (uint32_t)(bias - (int32_t)r[4 + k]));
                overflow[3 + k] = umax(overflow[3 + k], (uint32_t)((int32_t)r[4 + k] + bias));
            }
            overflow[6] += (uint32_t)(flux * 64.0f + 0.5f);
            return;
        }
        uint32_t* record = flips + 4 + (size_t)slot * 4;
        record[0] = r[4]; record[1] = r[5]; record[2] = r[6]; record[3] = fbits(flux);
    };
    uint32_t* owners = queue + PREFIX;
    uint32_t* cursor = queue + PREFIX + n;
    // reproject_paths: the receiver's sequence is its estimate's, and every
    // receiver is its own owner.
    // and the sun corners: a face lit by a directional light refreshes its
    // four corner words one frame in 4 (staggered by index), at once when
    // new to the view (voxel_view_runtime.wgsl:168-200).
    const uint32_t frame = view_words[7];
    const bool has_previous = view_words[8] != 0u;
    Ctx cx{g, m, Counters{}};
    const uint32_t n_directional = cx.pcount(11);
    auto sky_corner_visibility = [&](f3 position) {
        uint32_t word = 0x80000000u, bit = 0u;
        for (uint32_t l = 0; l < n_directional && bit < 4u; ++l) {
            const float* L = lights + (size_t)l * 12;
            if (wmax(L[4] - L[9], 0.0f) == 0.0f && wmax(L[5] - L[10], 0.0f) == 0.0f && wmax(L[6] - L[11], 0.0f) == 0.0f) continue;
            const f3 direction = normalize(f3{L[0], L[1], L[2]});
            const uint32_t status = trace_domain_limited(cx, add(position, muls(direction, 0.002f)), direction, cx.extra(1), true, 2048u).status;
            if (status == 2u) { word = 0u; break; }
            if (status == 0u) word |= 1u << bit;
            bit += 1u;
        }
        return word;
    };
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t* r = receivers + (size_t)i * 8;
        if (r[3] >= 6u) continue;
        uint32_t* e = estimates + (size_t)i * 16;
        const f3 normal = face_normal(r[3]);
        bool lit = false;
        for (uint32_t l = 0; l < n_directional; ++l) lit = lit || dot(normal, f3{lights[l * 12], lights[l * 12 + 1], lights[l * 12 + 2]}) > 0.0f;
        const uint32_t old = e[14];
        const bool carried = has_previous && old != 0u && (frame + i) % 4u != 0u;
        uint32_t corners = carried ? old : 0x80808080u;
        if (lit && !carried) {
            f3 u{0, 1, 0}, v{0, 0, 1};
            if (r[3] / 2u == 1u) u = f3{1, 0, 0};
            else if (r[3] / 2u == 2u) { u = f3{1, 0, 0}; v = f3{0, 1, 0}; }
            const uint32_t a = (r[3] / 2u + 1u) % 3u;
            const float s = 2.0f * (bitsf(r[a]) - (float)(int32_t)r[4 + a]);
            u = muls(u, s);
            v = muls(v, s);
            const f3 base = add(f3{(float)(int32_t)r[4], (float)(int32_t)r[5], (float)(int32_t)r[6]},
                                muls(f3{wmax(normal.x, 0.0f), wmax(normal.y, 0.0f), wmax(normal.z, 0.0f)}, s));
            corners = 0u;
            for (uint32_t corner = 0; corner < 4u; ++corner) {
                const f3 position = add(add(base, muls(u, (float)(corner & 1u))), muls(v, (float)(corner >> 1u)));
                const uint32_t word = sky_corner_visibility(position);
                corners |= ((word & 15u) | ((word >> 24u) & 128u)) << (corner * 8u);
            }
            if (has_previous && old != 0u) report_sun_flips(r, normal, e[13], old, corners);
        }
        e[14] = corners;
        r[7] = e[12];
        const uint32_t entry = queue[OWNERS]++;
        owners[entry] = i;
        cursor[i] = entry;
    }
    // retain_view_history
    if (n_events) {
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t* r = receivers + (size_t)i * 8;
            if (r[3] >= 6u) continue;
            uint32_t* e = estimates + (size_t)i * 16;
            const int32_t p[3] = {(int32_t)r[4], (int32_t)r[5], (int32_t)r[6]};
            Retention change = resolve_retention(events, p, n_events, reach, physical > 0.0f, 0u, 0u);
            if (e[15] == 0u || shared_slot(sh, r, e[13]) == NO_LIMIT) {
                if (change.limit != NO_LIMIT) e[3] = fbits(wmin(bitsf(e[3]), (float)change.limit));
                if (change.measured) e[7] = fbits(bitsf(e[7]) + change.change);
            }
            if (change.woken && conts[(size_t)i * 32 + 19] == 1u) conts[(size_t)i * 32 + 19] = 0u;
        }
    }
    const uint32_t owner_count = queue[OWNERS];
    // load_shared_faces (without the topology prior)
    if (sh.enabled) {
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t* r = receivers + (size_t)i * 8;
            if (r[3] >= 6u) continue;
            uint32_t* e = estimates + (size_t)i * 16;
            const uint32_t slot = shared_slot(sh, r, e[13]);
            if (slot == NO_LIMIT) { e[15] = 0u; continue; }
            const uint32_t* base = state + (size_t)slot * 36;
            const uint32_t incarnation = base[28];
            const uint32_t count = base[5] & 0x7fffffffu;
            const uint32_t next = base[6];
            queue[CACHE_LOADS] += 1;
            if (e[15] == incarnation || bitsf(e[3]) <= (float)count) {
                if (e[15] != incarnation) conts[(size_t)i * 32 + 19] = 0u;
                e[0] = base[0]; e[1] = base[1]; e[2] = base[2]; e[3] = fbits((float)count);
                e[4] = base[8]; e[5] = base[9]; e[6] = base[10]; e[7] = meta[(size_t)slot * 12 + 4];
                e[12] = next;
            } else {
                queue[CACHE_PROMOTIONS] += 1;
                e[12] = umax(e[12], next);
            }
            if (bitsf(e[11]) == 0.0f && count > 0u) {
                const F4 shown = rF4(base + 24);
                if (shown.w > 0.0f) wF4(e + 8, shown);
                else { e[8] = e[0]; e[9] = e[1]; e[10] = e[2]; e[11] = fbits(1.0f); }
            }
            if (e[15] != incarnation) report_sun_flips(r, face_normal(r[3]), e[13], base[32], e[14]);
            e[15] = incarnation;
            const bool pending = conts[(size_t)i * 32 + 19] == 1u;
            const uint32_t rank = cursor[i];
            const uint32_t oc = umax(owner_count, 1u);
            const uint32_t ordinal = (rank + owner_count - wave.range[0] % oc) % oc;
            uint32_t visits = 0;
            if (ordinal < umin(owner_count, wave.range[1]) && wave.range[2] > 0u)
                visits = umin(view_first ? 32u : 1u, (wave.range[1] - ordinal + owner_count - 1u) / owner_count);
            const uint32_t first = umax(next, e[12]);
            const uint32_t starts = visits - ((pending && visits > 0u) ? 1u : 0u);
            state[(size_t)slot * 36 + 6] = first + starts;
            cursor[i] = first;
            e[12] = pending ? paths[(size_t)i * 32 + 3] : first;
            r[7] = e[12];
        }
    }
    // The priors of load_shared_faces (voxel_view_cache.wgsl:192-212): a new,
    // unmeasured receiver starts from its topology prior, or else from the
    // far cell at its centre.
    const bool topology = view_words[6] != 0u;
    if (far_words || topology) {
        Ctx fx{g, m, Counters{}};
        const std::vector<uint32_t> before(estimates, estimates + (size_t)n * 16);
        const prior::Donors donors{receivers, n, before.data(), &sh};
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t* r = receivers + (size_t)i * 8;
            if (r[3] >= 6u) continue;
            uint32_t* e = estimates + (size_t)i * 16;
            if (bitsf(e[3]) != 0.0f || e[12] != 0u) continue;
            prior::FacePrior p;
            if (topology) p = prior::bootstrap_face(fx, donors, r);
            if (p.weight == 0.0f && far_words) {
                f3 mean;
                float count;
                uint32_t sequence;
                far::previous_cell(fx, far::View{far_words}, far_cells, f3{bitsf(r[0]), bitsf(r[1]), bitsf(r[2])}, r[3],
                                   i3{(int32_t)r[4], (int32_t)r[5], (int32_t)r[6]}, mean, count, sequence);
                if (count > 0.0f) {
                    p = prior::FacePrior{mean, f3{mean.x * mean.x, mean.y * mean.y, mean.z * mean.z}, 1.0f};
                    far_stats[5] += 1;
                }
            }
            if (p.weight <= 0.0f) continue;
            e[0] = fbits(p.mean.x); e[1] = fbits(p.mean.y); e[2] = fbits(p.mean.z); e[3] = fbits(p.weight);
            e[4] = fbits(p.moment.x); e[5] = fbits(p.moment.y); e[6] = fbits(p.moment.z); e[7] = 0u;
            e[8] = e[0]; e[9] = e[1]; e[10] = e[2]; e[11] = fbits(1.0f);
        }
    }
    // trace_visible_paths
    if (wave.range[2] != 0u) {
        const uint32_t invocations = umin(owner_count, wave.range[1]);
        for (uint32_t id = 0; id < invocations; ++id) {
            const uint32_t i = owners[(wave.range[0] + id) % owner_count];
            uint32_t* r = receivers + (size_t)i * 8;
            uint32_t* e = estimates + (size_t)i * 16;
            uint32_t* record = paths + (size_t)i * 32;
            uint32_t* stored = conts + (size_t)i * 32;
            const uint32_t visits = umin(view_first ? 32u : 1u, (wave.range[1] - id + owner_count - 1u) / owner_count);
            const bool reserved = sh.enabled && e[15] != 0u;
            uint32_t next = cursor[i];
            if (stored[19] != 1u) next += 1u;
            for (uint32_t visit = 0; visit < visits; ++visit) {
                queue[ATTEMPTED] += 1;
                Ctx x{g, m, Counters{}};
                advance_view_path(x, r, record, stored, wave);
                if (stored[19] != 2u && stored[19] != 3u) continue;
                queue[COMPLETED] += 1;
                if (reserved) { e[12] = next; next += 1u; }
                else e[12] += 1u;
                r[7] = e[12];
                if (record[23] != 0u) {
                    queue[KNOWN] += 1;
                    const f3 value = add(rf3(record + 20), rf3(record + 24));
                    F4 mean = rF4(e), moment = rF4(e + 4);
                    if (moment.w > 0.0f) {
                        const float change = moment.w;
                        const f3 variance{wmax(moment.x - mean.x * mean.x, 0.0f), wmax(moment.y - mean.y * mean.y, 0.0f),
                                          wmax(moment.z - mean.z * mean.z, 0.0f)};
                        const float keep = physical * (0.2126f * variance.x + 0.7152f * variance.y + 0.0722f * variance.z) / (change * change);
                        mean.w = wmin(mean.w, floorf(keep));
                        moment.w = 0.0f;
                    }
                    const float count = wmin(mean.w + 1.0f, 65536.0f);
                    const float t = 1.0f / count;
                    // mix(a, b, t) = a * (1 - t) + b * t
                    mean = F4{mean.x * (1.0f - t) + value.x * t, mean.y * (1.0f - t) + value.y * t, mean.z * (1.0f - t) + value.z * t, count};
                    moment = F4{moment.x * (1.0f - t) + value.x * value.x * t, moment.y * (1.0f - t) + value.y * value.y * t,
                                moment.z * (1.0f - t) + value.z * value.z * t, moment.w};
                    wF4(e, mean);
                    wF4(e + 4, moment);
                }
            }
            if (reserved) {
                const uint32_t first = cursor[i];
                const uint32_t used = stored[19] == 1u ? record[3] + 1u : e[12];
                cursor[i] = umax(first, used);
            }
        }
    }
    // store_shared_faces
    if (sh.enabled) {
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t* r = receivers + (size_t)i * 8;
            if (r[3] >= 6u) continue;
            const uint32_t* e = estimates + (size_t)i * 16;
            const uint32_t slot = shared_slot(sh, r, e[13]);
            if (slot == NO_LIMIT) continue;
            uint32_t* base = state + (size_t)slot * 36;
            if (e[15] != base[28]) continue;
            const uint32_t count = (uint32_t)bitsf(e[3]);
            const bool changed_count = (base[5] & 0x7fffffffu) != count;
            const bool changed_mean = base[0] != e[0] || base[1] != e[1] || base[2] != e[2];
            base[0] = e[0]; base[1] = e[1]; base[2] = e[2]; base[3] = 0u;
            base[8] = e[4]; base[9] = e[5]; base[10] = e[6]; base[11] = 0u;
            base[4] = 0u;
            base[12] = 0u;
            base[5] = count | (bitsf(e[7]) > 0.0f ? 0x80000000u : 0u);
            base[6] = cursor[i];
            meta[(size_t)slot * 12 + 4] = e[7];
            for (int k = 0; k < 4; ++k) base[24 + k] = e[8 + k];
            if (e[14] != 0u) base[32] = e[14];
            base[7] = e[8];
            base[13] = e[9]; base[14] = e[10]; base[15] = e[11];
            if (changed_mean || changed_count) {
                const F4 mean = rF4(e), moment = rF4(e + 4);
                auto noise = [](float mo, float me) { return std::sqrt(wmax(mo - me * me, 0.0f)) / (0.002f + std::fabs(me)); };
                const float nz = wmax(noise(moment.x, mean.x), wmax(noise(moment.y, mean.y), noise(moment.z, mean.z)));
                uint32_t* rank = meta + (size_t)slot * 12 + 8;
                rank[0] = fbits(nz);
                rank[1] = clock;
                rank[2] = fbits(wmax(mean.x, wmax(mean.y, mean.z)));
                rank[3] = 0xa0000000u | count;
            }
        }
    }
    return 0;
}

}  // extern "C"
