// Seeded synthetic workloads (include/vgi_scenes.h). Deterministic: integer
// hashing plus float arithmetic in a fixed order, threads over z slabs.
#include "../../include/vgi_scenes.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vgi_runtime.h"

namespace {

using vgi::host_pcg;

inline float lattice(uint32_t seed, int32_t x, int32_t y, int32_t z) {
    uint32_t h = host_pcg(seed ^ host_pcg((uint32_t)x ^ host_pcg((uint32_t)y ^ host_pcg((uint32_t)z))));
    return (float)(h >> 8) * (1.0f / 8388608.0f) - 1.0f;  // [-1, 1)
}
inline float smooth(float t) { return t * t * (3.0f - 2.0f * t); }
inline float value_noise(uint32_t seed, float x, float y, float z) {
    float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int32_t ix = (int32_t)fx, iy = (int32_t)fy, iz = (int32_t)fz;
    float tx = smooth(x - fx), ty = smooth(y - fy), tz = smooth(z - fz);
    float c[8];
    for (int k = 0; k < 8; ++k) c[k] = lattice(seed, ix + (k & 1), iy + ((k >> 1) & 1), iz + (k >> 2));
    float x00 = c[0] + (c[1] - c[0]) * tx, x10 = c[2] + (c[3] - c[2]) * tx;
    float x01 = c[4] + (c[5] - c[4]) * tx, x11 = c[6] + (c[7] - c[6]) * tx;
    float y0 = x00 + (x10 - x00) * ty, y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
}
inline float fbm(uint32_t seed, uint32_t octaves, float frequency, float x, float y, float z) {
    float sum = 0.0f, amplitude = 1.0f;
    for (uint32_t o = 0; o < octaves; ++o) {
        sum += amplitude * value_noise(seed + o * 0x9e3779b9u, x * frequency, y * frequency, z * frequency);
        frequency *= 2.0f;
        amplitude *= 0.5f;
    }
    return sum;
}

template <class F>
void parallel_for(uint32_t n, F f) {
    uint32_t threads = std::max(1u, std::min<uint32_t>(std::thread::hardware_concurrency(), 64u));
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    auto work = [&]() {
        for (uint32_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
    };
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

inline size_t region_voxel(uint32_t region, uint32_t lx, uint32_t ly, uint32_t lz) {
    return (size_t)region * 4096 + lx + 16 * (ly + 16 * lz);
}

void fill_page(uint16_t* voxels, uint16_t (*at)(int32_t, int32_t, int32_t)) {
    // 2 x 2 x 2 regions in (z, y, x) order covering 0..31 on every axis.
    for (uint32_t r = 0; r < 8; ++r) {
        int32_t rx = r & 1, ry = (r >> 1) & 1, rz = r >> 2;
        for (uint32_t i = 0; i < 4096; ++i) {
            int32_t x = rx * 16 + (int32_t)(i & 15), y = ry * 16 + (int32_t)((i >> 4) & 15), z = rz * 16 + (int32_t)(i >> 8);
            voxels[(size_t)r * 4096 + i] = at(x, y, z);
        }
    }
}

}  // namespace

extern "C" {

uint32_t vgi_scene_grid_coords(uint32_t nx, uint32_t ny, uint32_t nz, int32_t* coords) {
    uint32_t r = 0;
    for (uint32_t z = 0; z < nz; ++z)
        for (uint32_t y = 0; y < ny; ++y)
            for (uint32_t x = 0; x < nx; ++x) {
                if (coords) {
                    coords[r * 3] = (int32_t)x;
                    coords[r * 3 + 1] = (int32_t)y;
                    coords[r * 3 + 2] = (int32_t)z;
                }
                ++r;
            }
    return r;
}

void vgi_scene_stone_room(uint16_t* voxels) {
    fill_page(voxels, [](int32_t x, int32_t y, int32_t z) -> uint16_t {
        bool shell = x == 0 || x == 31 || y == 0 || y == 31 || z == 0 || z == 31;
        if (shell) return 0;
        if (x == 16 && y == 1 && z == 16) return 1;
        return 256;
    });
}

void vgi_scene_furnace(uint16_t* voxels) {
    fill_page(voxels, [](int32_t x, int32_t y, int32_t z) -> uint16_t {
        bool inside = x >= 8 && x < 24 && y >= 8 && y < 24 && z >= 8 && z < 24;
        bool wall = x == 8 || x == 23 || y == 8 || y == 23 || z == 8 || z == 23;
        return inside && wall ? 4 : 256;
    });
}

void vgi_scene_terrain(const vgi_terrain_params* p, uint32_t nx, uint32_t ny, uint32_t nz, uint16_t* voxels) {
    const uint32_t X = nx * 16, Y = ny * 16, Z = nz * 16;
    const float frequency = 1.0f / p->period;
    const uint32_t seed = p->seed;
    // Solid where fbm - (y - base) / falloff > 0; material from a coarse field.
    parallel_for(Z, [&](uint32_t z) {
        for (uint32_t y = 0; y < Y; ++y)
            for (uint32_t x = 0; x < X; ++x) {
                float density = fbm(seed, p->octaves, frequency, (float)x, (float)y, (float)z) - ((float)y - p->base_height) / p->falloff;
                uint16_t m = 256;
                if (density > 0.0f) {
                    float v = value_noise(seed ^ 0x5bd1e995u, (float)x * (1.0f / 48.0f), (float)y * (1.0f / 24.0f), (float)z * (1.0f / 48.0f));
                    int32_t k = (int32_t)std::floor((v + 1.0f) * 4.0f);
                    m = (uint16_t)std::min(7, std::max(0, k));
                }
                uint32_t region = (x >> 4) + nx * ((y >> 4) + ny * (z >> 4));
                voxels[region_voxel(region, x & 15, y & 15, z & 15)] = m;
            }
    });
    // Emissive voxels on the surface: the air cell above the top solid of a
    // random column.
    auto at = [&](uint32_t x, uint32_t y, uint32_t z) -> uint16_t& {
        uint32_t region = (x >> 4) + nx * ((y >> 4) + ny * (z >> 4));
        return voxels[region_voxel(region, x & 15, y & 15, z & 15)];
    };
    uint32_t state = host_pcg(seed ^ 0xe7037ed1u);
    uint32_t placed = 0;
    for (uint32_t attempt = 0; attempt < p->emitters * 64 && placed < p->emitters; ++attempt) {
        state = host_pcg(state + attempt);
        uint32_t x = state % X;
        state = host_pcg(state);
        uint32_t z = state % Z;
        int32_t top = -1;
        for (int32_t y = (int32_t)Y - 1; y >= 0; --y)
            if (at(x, (uint32_t)y, z) != 256) { top = y; break; }
        if (top < 0 || top + 1 >= (int32_t)Y) continue;
        uint16_t& cell = at(x, (uint32_t)top + 1, z);
        if (cell != 256) continue;
        cell = (uint16_t)(8 + placed % 248);
        ++placed;
    }
}

void vgi_scene_cave(const vgi_cave_params* p, uint32_t nx, uint32_t ny, uint32_t nz, uint16_t* voxels) {
    const int32_t X = (int32_t)nx * 16, Y = (int32_t)ny * 16, Z = (int32_t)nz * 16;
    const uint32_t seed = p->seed;
    auto at = [&](int32_t x, int32_t y, int32_t z) -> uint16_t& {
        const uint32_t region = (uint32_t)(x >> 4) + nx * ((uint32_t)(y >> 4) + ny * (uint32_t)(z >> 4));
        return voxels[region_voxel(region, x & 15, y & 15, z & 15)];
    };
    // Rock with materials from a coarse field.
    parallel_for((uint32_t)Z, [&](uint32_t z) {
        for (int32_t y = 0; y < Y; ++y)
            for (int32_t x = 0; x < X; ++x) {
                const float v = value_noise(seed ^ 0x5bd1e995u, (float)x * (1.0f / 48.0f), (float)y * (1.0f / 24.0f), (float)z * (1.0f / 48.0f));
                at(x, y, (int32_t)z) = (uint16_t)std::min(7, std::max(0, (int32_t)std::floor((v + 1.0f) * 4.0f)));
            }
    });
    const int32_t ceiling = Y - (int32_t)p->roof;  // tunnels stay below it
    auto carve = [&](float cx, float cy, float cz, float r, int32_t y_max) {
        const int32_t x0 = std::max(0, (int32_t)std::floor(cx - r)), x1 = std::min(X - 1, (int32_t)std::ceil(cx + r));
        const int32_t y0 = std::max(1, (int32_t)std::floor(cy - r)), y1 = std::min(y_max - 1, (int32_t)std::ceil(cy + r));
        const int32_t z0 = std::max(0, (int32_t)std::floor(cz - r)), z1 = std::min(Z - 1, (int32_t)std::ceil(cz + r));
        for (int32_t z = z0; z <= z1; ++z)
            for (int32_t y = y0; y <= y1; ++y)
                for (int32_t x = x0; x <= x1; ++x) {
                    const float dx = (float)x + 0.5f - cx, dy = (float)y + 0.5f - cy, dz = (float)z + 0.5f - cz;
                    if (dx * dx + dy * dy + dz * dz <= r * r) at(x, y, z) = 256;
                }
    };
    uint32_t state = host_pcg(seed ^ 0x68e31da4u);
    auto uniform = [&]() {
        state = host_pcg(state + 0x9e3779b9u);
        return (float)(state >> 8) * (1.0f / 16777216.0f);
    };
    // Skylight shafts through the roof.
    std::vector<std::array<float, 2>> shafts;
    for (uint32_t k = 0; k < p->skylights; ++k) {
        const float sx = p->skylight_radius + uniform() * ((float)X - 2.0f * p->skylight_radius);
        const float sz = p->skylight_radius + uniform() * ((float)Z - 2.0f * p->skylight_radius);
        shafts.push_back({sx, sz});
        for (int32_t y = ceiling - (int32_t)p->radius_max; y < Y; ++y) carve(sx, (float)y + 0.5f, sz, p->skylight_radius, Y);
    }
    // Worm tunnels.
    const float span = p->radius_max - p->radius_min;
    for (uint32_t w = 0; w < p->worms; ++w) {
        const uint32_t ws = host_pcg(seed + 0x1000u * (w + 1u));
        float px, py, pz;
        if (w < shafts.size()) {
            px = shafts[w][0];
            pz = shafts[w][1];
            py = (float)ceiling - p->radius_max;
        } else {
            px = uniform() * (float)X;
            pz = uniform() * (float)Z;
            py = p->radius_max + 1.0f + uniform() * std::max(1.0f, (float)ceiling - 2.0f * p->radius_max - 2.0f);
        }
        float yaw = uniform() * 6.2831853f, pitch = 0.0f;
        for (uint32_t t = 0; t < p->steps; ++t) {
            const float r = p->radius_min + span * (0.5f + 0.5f * value_noise(ws, (float)t * 0.05f, 0.5f, 0.5f));
            carve(px, py, pz, r, ceiling);
            yaw += 0.35f * value_noise(ws ^ 0x27d4eb2du, (float)t * 0.1f, 1.5f, 0.5f);
            pitch = 0.3f * value_noise(ws ^ 0x165667b1u, (float)t * 0.07f, 2.5f, 0.5f);
            const float step = std::max(1.0f, 0.5f * r);
            px += step * std::cos(pitch) * std::cos(yaw);
            pz += step * std::cos(pitch) * std::sin(yaw);
            py += step * std::sin(pitch);
            // Reflect at the sides; stay between the floor and the roof.
            if (px < 0.0f || px >= (float)X) {
                yaw = 3.14159265f - yaw;
                px = std::min(std::max(px, 0.0f), (float)X - 1.0f);
            }
            if (pz < 0.0f || pz >= (float)Z) {
                yaw = -yaw;
                pz = std::min(std::max(pz, 0.0f), (float)Z - 1.0f);
            }
            py = std::min(std::max(py, r + 1.0f), std::max(r + 1.0f, (float)ceiling - r - 1.0f));
        }
    }
    // Emitters on tunnel floors: the lowest air voxel above rock in a random column.
    uint32_t placed = 0;
    for (uint32_t attempt = 0; attempt < p->emitters * 64 && placed < p->emitters; ++attempt) {
        const int32_t x = (int32_t)(uniform() * (float)X), z = (int32_t)(uniform() * (float)Z);
        if (x >= X || z >= Z) continue;
        for (int32_t y = 1; y < ceiling; ++y) {
            if (at(x, y, z) == 256 && at(x, y - 1, z) != 256) {
                at(x, y, z) = (uint16_t)(8 + (placed & 1u));
                ++placed;
                break;
            }
        }
    }
}

uint64_t vgi_scene_faces(const int32_t* coords, uint32_t n, const uint16_t* voxels, const vgi_face_filter* filter, int32_t* out,
                         uint64_t capacity) {
    std::unordered_map<vgi::RegionKey, uint32_t, vgi::RegionKeyHash> where;
    for (uint32_t r = 0; r < n; ++r) where[vgi::RegionKey{coords[r * 3], coords[r * 3 + 1], coords[r * 3 + 2]}] = r;
    std::vector<uint32_t> order(n);
    for (uint32_t r = 0; r < n; ++r) order[r] = r;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        if (coords[a * 3 + 2] != coords[b * 3 + 2]) return coords[a * 3 + 2] < coords[b * 3 + 2];
        if (coords[a * 3 + 1] != coords[b * 3 + 1]) return coords[a * 3 + 1] < coords[b * 3 + 1];
        return coords[a * 3] < coords[b * 3];
    });
    static const int32_t off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    auto material_at = [&](int32_t x, int32_t y, int32_t z, bool* loaded) -> uint16_t {
        auto it = where.find(vgi::RegionKey{x >> 4, y >> 4, z >> 4});
        if (it == where.end()) { *loaded = false; return 256; }
        *loaded = true;
        return voxels[(size_t)it->second * 4096 + (x & 15) + 16 * ((y & 15) + 16 * (z & 15))];
    };
    // Per region, faces in voxel (z, y, x) then face order; regions in (z, y, x)
    // order, which is voxel order within each region row of the grid.
    std::vector<std::vector<int32_t>> per(n);
    parallel_for(n, [&](uint32_t k) {
        uint32_t r = order[k];
        std::vector<int32_t>& dst = per[k];
        const uint16_t* m = voxels + (size_t)r * 4096;
        for (int32_t i = 0; i < 4096; ++i) {
            uint16_t mat = m[i];
            if (mat == 256) continue;
            int32_t v[3] = {coords[r * 3] * 16 + (i & 15), coords[r * 3 + 1] * 16 + ((i >> 4) & 15), coords[r * 3 + 2] * 16 + (i >> 8)};
            for (int f = 0; f < 6; ++f) {
                int32_t nb[3] = {v[0] + off[f][0], v[1] + off[f][1], v[2] + off[f][2]};
                bool loaded;
                if (material_at(nb[0], nb[1], nb[2], &loaded) != 256 || !loaded) continue;
                if (filter && filter->use_box) {
                    bool in = nb[0] >= filter->box_min[0] && nb[1] >= filter->box_min[1] && nb[2] >= filter->box_min[2] &&
                              nb[0] <= filter->box_max[0] && nb[1] <= filter->box_max[1] && nb[2] <= filter->box_max[2];
                    if (!in) continue;
                }
                if (filter && filter->use_facing) {
                    float cx = (float)v[0] + 0.5f + 0.5f * (float)off[f][0] - filter->eye[0];
                    float cy = (float)v[1] + 0.5f + 0.5f * (float)off[f][1] - filter->eye[1];
                    float cz = (float)v[2] + 0.5f + 0.5f * (float)off[f][2] - filter->eye[2];
                    if (cx * (float)off[f][0] + cy * (float)off[f][1] + cz * (float)off[f][2] >= 0.0f) continue;
                }
                if (filter && filter->use_frustum) {
                    float c[3] = {(float)v[0] + 0.5f + 0.5f * (float)off[f][0], (float)v[1] + 0.5f + 0.5f * (float)off[f][1],
                                  (float)v[2] + 0.5f + 0.5f * (float)off[f][2]};
                    float d[3] = {c[0] - filter->eye[0], c[1] - filter->eye[1], c[2] - filter->eye[2]};
                    // Facing the eye.
                    if (d[0] * (float)off[f][0] + d[1] * (float)off[f][1] + d[2] * (float)off[f][2] >= 0.0f) continue;
                    const float* fw = filter->forward;
                    float depth = d[0] * fw[0] + d[1] * fw[1] + d[2] * fw[2];
                    if (depth <= 0.0f) continue;
                    // Right = normalize(forward x up), up' = right x forward; up = +y (or +z when forward is vertical).
                    float up[3] = {0.0f, 1.0f, 0.0f};
                    if (std::fabs(fw[1]) > 0.99f) { up[1] = 0.0f; up[2] = 1.0f; }
                    float rt[3] = {fw[1] * up[2] - fw[2] * up[1], fw[2] * up[0] - fw[0] * up[2], fw[0] * up[1] - fw[1] * up[0]};
                    float rl = std::sqrt(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2]);
                    for (float& q : rt) q /= rl;
                    float u2[3] = {rt[1] * fw[2] - rt[2] * fw[1], rt[2] * fw[0] - rt[0] * fw[2], rt[0] * fw[1] - rt[1] * fw[0]};
                    float sx = d[0] * rt[0] + d[1] * rt[1] + d[2] * rt[2];
                    float sy = d[0] * u2[0] + d[1] * u2[1] + d[2] * u2[2];
                    if (std::fabs(sx) > depth * filter->tan_half || std::fabs(sy) > depth * filter->tan_half) continue;
                }
                dst.push_back(v[0]);
                dst.push_back(v[1]);
                dst.push_back(v[2]);
                dst.push_back(f);
                dst.push_back(mat);
            }
        }
    });
    uint64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        uint64_t count = per[k].size() / 5;
        if (out && total + count <= capacity) std::memcpy(out + total * 5, per[k].data(), per[k].size() * 4);
        total += count;
    }
    return total;
}

}  // extern "C"
