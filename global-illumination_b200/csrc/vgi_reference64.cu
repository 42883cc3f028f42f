// FP64 converged reference of the face trace's estimate, for error metrics.
//
// The quantity is what the world cache accumulates per face: the incident
// radiance averaged with the cosine-weighted hemisphere measure, excluding
// the receiver's own direct light (trace_receiver, shaders/voxel_path.wgsl:
// 498-520, with direct_at reported separately by write_result,
// shaders/voxel_trace.wgsl:25-37). It is estimated here without the world
// cache and without a depth cut: every hit adds its MIS-weighted emission,
// its lights' direct light and an emitter sample, and paths end only by
// escaping (environment), by reaching unloaded space (sample not counted)
// or by Russian roulette after the first hit (survival clamp(max(tp), 0.1,
// 0.95), voxel_path.wgsl:476-480), which keeps the estimate unbiased.
//
// Everything is double precision: positions, directions, the DDA over the
// same NAADF arrays (region, brick and voxel boxes, the trace_domain rules
// of shaders/voxel_traversal.wgsl:122-219 with a 1e-9 step nudge instead of
// 0.001) and the estimator. Random numbers are independent per sample (a
// PCG stream per face, sample and seed) rather than the production QMC
// sequence. Emitters are chosen in proportion to their material's emission
// weight (the records' power), so the light-selection density is
// weight / total for every emitter face. Materials, lights and the
// environment are the same records the FP32 trace uses.
#include <cstdint>
#include <cuda_runtime.h>

#include "vgi_device.cuh"
#include "vgi_types.cuh"

namespace vgi {
namespace {

constexpr int kBlock = 256;
constexpr double kNudge = 1e-9;
constexpr double kOffset = 1e-4;
constexpr double kMaxDistance = 768.0;
constexpr double kPi = 3.141592653589793;

struct D3 { double x, y, z; };
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) { return D3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double comp(D3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct Ref64Args {
    TraceArgs t;
    const double* cdf;      // n + 1 cumulative emitter weights, cdf[n] = total
    const int4* emitters;   // voxel xyz, face | material << 3
    uint32_t n_emitters;
    double total;
    const uint4* tasks;     // FaceTask words (2 uint4)
    uint32_t n_tasks, samples;
    uint64_t seed;
    double* sum;            // 3 per task
    double* second;         // 3 per task
    uint32_t* known;        // per task
};

// PCG-XSH-RR 64/32 stream per (task, sample, seed).
struct Rng {
    uint64_t state, inc;
    __device__ uint32_t next() {
        const uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    __device__ double uniform() { return (double)(((uint64_t)next() << 21) ^ (uint64_t)(next() >> 11)) * 0x1p-53; }
};
__device__ Rng make_rng(uint64_t seed, uint64_t stream) {
    Rng r{0u, (stream << 1u) | 1u};
    r.next();
    r.state += seed;
    r.next();
    return r;
}

struct Hit64 {
    int status;  // 0 escaped or beyond max distance, 1 hit, 2 unloaded space
    int vx, vy, vz;
    uint32_t material;
    D3 position, normal;
};

__device__ __forceinline__ uint32_t region_of(const TraceArgs& A, int x, int y, int z) {
    uint32_t slot = hash_voxel(x, y, z) & A.dir_mask;
    for (uint32_t attempt = 0; attempt < 32u; ++attempt) {
        const int4 e = A.directory[slot];
        if (e.w == -1) return kNoIndex;
        if (e.x == x && e.y == y && e.z == z) return (uint32_t)e.w;
        slot = (slot + 1u) & A.dir_mask;
    }
    return kNoIndex;
}

// Distance-skip DDA in double precision (trace_domain's cell rules).
__device__ Hit64 trace64(const TraceArgs& A, D3 o, D3 d, double max_distance) {
    Hit64 h{0, 0, 0, 0, 0u, D3{0, 0, 0}, D3{0, 0, 0}};
    double lo = 0.0, hi = 1e300;
    D3 normal{0, 0, 0};
    for (int a = 0; a < 3; ++a) {
        const double da = comp(d, a), oa = comp(o, a);
        const double mn = (double)A.mn[a] * 16.0, mx = (double)(A.mx[a] + 1) * 16.0;
        if (fabs(da) < 1e-300) {
            if (oa < mn || oa > mx) return h;
            continue;
        }
        double t0 = (mn - oa) / da, t1 = (mx - oa) / da;
        if (t0 > t1) {
            const double t = t0;
            t0 = t1;
            t1 = t;
        }
        lo = fmax(lo, t0);
        hi = fmin(hi, t1);
    }
    if (hi < lo) return h;
    double dist = lo + kNudge;
    for (int step = 0; step < 1 << 14; ++step) {
        if (dist > max_distance || dist > hi) return h;
        const D3 p = o + d * dist;
        const int vx = (int)floor(p.x), vy = (int)floor(p.y), vz = (int)floor(p.z);
        const int rx = vx >> 4, ry = vy >> 4, rz = vz >> 4;
        if (rx < A.mn[0] || ry < A.mn[1] || rz < A.mn[2] || rx > A.mx[0] || ry > A.mx[1] || rz > A.mx[2]) return h;
        const uint32_t index = region_of(A, rx, ry, rz);
        if (index == kNoIndex) {
            h.status = 2;
            return h;
        }
        const uint4 meta = A.headers[index];
        int cx = rx, cy = ry, cz = rz, nx = 0, ny = 0, nz = 0, px = 0, py = 0, pz = 0;
        double size = 16.0;
        uint32_t material = 0xffffffffu;
        if (meta.x == 1u) {
            nx = meta.z & 255u; ny = (meta.z >> 8) & 255u; nz = (meta.z >> 16) & 255u;
            px = meta.w & 255u; py = (meta.w >> 8) & 255u; pz = (meta.w >> 16) & 255u;
        } else if (meta.x != 3u) {
            material = meta.y;
        } else {
            const uint32_t lx = vx & 15, ly = vy & 15, lz = vz & 15;
            const uint32_t bx = lx >> 2, by = ly >> 2, bz = lz >> 2;
            const uint32_t brick = A.cells[meta.y + (bz * 4u + by) * 4u + bx];
            if ((brick & 3u) == 0u) {
                const uint32_t e = brick >> 2;
                cx = rx * 4 + (int)bx; cy = ry * 4 + (int)by; cz = rz * 4 + (int)bz;
                nx = e & 3u; px = (e >> 2) & 3u; ny = (e >> 4) & 3u; py = (e >> 6) & 3u; nz = (e >> 8) & 3u; pz = (e >> 10) & 3u;
                size = 4.0;
            } else if ((brick & 3u) == 1u) {
                material = brick >> 2;
            } else {
                const uint32_t idx = ((lz & 3u) * 4u + (ly & 3u)) * 4u + (lx & 3u);
                const uint32_t c = (A.cells[(brick >> 2) + (idx >> 1)] >> ((idx & 1u) * 16u)) & 65535u;
                if (c & 1u) {
                    material = c >> 1;
                } else {
                    const uint32_t e = c >> 1;
                    cx = vx; cy = vy; cz = vz;
                    nx = e & 3u; px = (e >> 2) & 3u; ny = (e >> 4) & 3u; py = (e >> 6) & 3u; nz = (e >> 8) & 3u; pz = (e >> 10) & 3u;
                    size = 1.0;
                }
            }
        }
        if (material != 0xffffffffu) {
            h.status = 1;
            h.vx = vx; h.vy = vy; h.vz = vz;
            h.material = material & 255u;
            h.position = p;
            if (normal.x == 0.0 && normal.y == 0.0 && normal.z == 0.0) {
                // Started inside a solid voxel: face the ray.
                const double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
                if (ax >= ay && ax >= az) normal = D3{d.x > 0 ? -1.0 : 1.0, 0, 0};
                else if (ay >= az) normal = D3{0, d.y > 0 ? -1.0 : 1.0, 0};
                else normal = D3{0, 0, d.z > 0 ? -1.0 : 1.0};
            }
            h.normal = normal;
            return h;
        }
        // Exit of the box (cell - neg, cell + pos + 1) * size.
        const int cell[3] = {cx, cy, cz}, ng[3] = {nx, ny, nz}, ps[3] = {px, py, pz};
        double best = 1e300;
        int axis = -1;
        for (int a = 0; a < 3; ++a) {
            const double da = comp(d, a);
            if (fabs(da) < 1e-300) continue;
            const double plane = da > 0.0 ? (double)(cell[a] + ps[a] + 1) * size : (double)(cell[a] - ng[a]) * size;
            const double t = (plane - comp(o, a)) / da;
            if (t < best) {
                best = t;
                axis = a;
            }
        }
        if (axis < 0) return h;
        dist = fmax(best, dist) + kNudge * fmax(1.0, best);
        normal = D3{axis == 0 ? (d.x > 0 ? -1.0 : 1.0) : 0.0, axis == 1 ? (d.y > 0 ? -1.0 : 1.0) : 0.0,
                    axis == 2 ? (d.z > 0 ? -1.0 : 1.0) : 0.0};
    }
    h.status = 2;
    return h;
}

__device__ D3 face_normal64(uint32_t face) {
    const double s = (face & 1u) ? -1.0 : 1.0;
    const uint32_t a = face >> 1;
    return D3{a == 0 ? s : 0.0, a == 1 ? s : 0.0, a == 2 ? s : 0.0};
}

// Cosine-weighted direction about n (any orthonormal frame).
__device__ D3 cosine_direction(D3 n, double u, double v) {
    const D3 helper = fabs(n.x) > 0.5 ? D3{0, 1, 0} : D3{1, 0, 0};
    D3 t{helper.y * n.z - helper.z * n.y, helper.z * n.x - helper.x * n.z, helper.x * n.y - helper.y * n.x};
    const double tl = sqrt(dotd(t, t));
    t = t * (1.0 / tl);
    const D3 b{n.y * t.z - n.z * t.y, n.z * t.x - n.x * t.z, n.x * t.y - n.y * t.x};
    const double r = sqrt(u), phi = 2.0 * kPi * v;
    return t * (r * cos(phi)) + b * (r * sin(phi)) + n * sqrt(fmax(0.0, 1.0 - u));
}

struct Mat64 { D3 diffuse, emission; double weight; };
__device__ Mat64 material64(const TraceArgs& A, uint32_t m) {
    const float4 d = A.materials[m * 4], e = A.materials[m * 4 + 2], x = A.materials[m * 4 + 3];
    return Mat64{D3{d.x, d.y, d.z}, D3{e.x, e.y, e.z}, (double)x.y};
}

// The lights' direct light at p (direct_at, voxel_path.wgsl:283-307).
__device__ D3 direct64(const TraceArgs& A, D3 p, D3 n) {
    D3 value{0, 0, 0};
    const D3 origin = p + n * kOffset;
    for (uint32_t i = 0; i < A.light_count; ++i) {
        const float4 lp = A.lights[i * 3], le = A.lights[i * 3 + 1];
        D3 dir;
        double distance = kMaxDistance, attenuation = 1.0;
        if (lp.w >= 0.0f) {
            const D3 delta = D3{lp.x, lp.y, lp.z} - p;
            const double d2 = dotd(delta, delta);
            if (d2 <= 1e-7 || d2 > (double)lp.w * (double)lp.w) continue;
            distance = sqrt(d2);
            dir = delta * (1.0 / distance);
            distance -= 2.0 * kOffset;
            attenuation = 1.0 / fmax(d2, 1.0);
        } else {
            const D3 l{lp.x, lp.y, lp.z};
            dir = l * (1.0 / sqrt(dotd(l, l)));
        }
        const double c = dotd(n, dir);
        if (c <= 0.0) continue;
        if (trace64(A, origin, dir, distance).status != 0) continue;
        value = value + D3{le.x, le.y, le.z} * (c * attenuation);
    }
    return value;
}

// One emitter sample at p with MIS against cosine sampling: the value is
// L_e * pdf_bsdf / (pdf_light + pdf_bsdf), an estimate of the emitters'
// cosine-averaged incident radiance.
__device__ D3 emitter64(const Ref64Args& R, D3 p, D3 n, Rng& rng) {
    const TraceArgs& A = R.t;
    if (R.n_emitters == 0 || R.total <= 0.0) return D3{0, 0, 0};
    const double u = rng.uniform() * R.total;
    uint32_t lo = 0, hi = R.n_emitters;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if (R.cdf[mid] <= u) lo = mid;
        else hi = mid;
    }
    const int4 e = R.emitters[lo];
    const uint32_t face = (uint32_t)e.w & 7u, material = (uint32_t)e.w >> 3;
    const Mat64 m = material64(A, material);
    const D3 en = face_normal64(face);
    const uint32_t axis = face >> 1;
    const D3 tangent = axis == 0 ? D3{0, 1, 0} : D3{1, 0, 0};
    const D3 bitangent = axis == 2 ? D3{0, 1, 0} : D3{0, 0, 1};
    const double s = rng.uniform() - 0.5, t = rng.uniform() - 0.5;
    const D3 lp = D3{e.x + 0.5, e.y + 0.5, e.z + 0.5} + en * 0.5 + tangent * s + bitangent * t;
    const D3 delta = lp - p;
    const double d2 = dotd(delta, delta);
    if (d2 < 1e-8) return D3{0, 0, 0};
    const double dist = sqrt(d2);
    const D3 dir = delta * (1.0 / dist);
    const double cr = dotd(n, dir), ce = -dotd(en, dir);
    if (cr <= 0.0 || ce <= 0.0) return D3{0, 0, 0};
    if (trace64(A, p + n * kOffset, dir, dist - 2.0 * kOffset).status != 0) return D3{0, 0, 0};
    const double pdf_light = (m.weight / R.total) * d2 / ce;
    const double pdf_bsdf = cr / kPi;
    return m.emission * (pdf_bsdf / (pdf_light + pdf_bsdf));
}

__global__ void __launch_bounds__(kBlock) reference64_kernel(const Ref64Args R) {
    const TraceArgs& A = R.t;
    const uint32_t task = blockIdx.x;
    if (task >= R.n_tasks) return;
    const uint4 t0 = R.tasks[task * 2u], t1 = R.tasks[task * 2u + 1u];
    const D3 n = face_normal64(t0.w);
    const D3 surface = D3{(double)(int)t0.x + 0.5, (double)(int)t0.y + 0.5, (double)(int)t0.z + 0.5} + n * 0.5;
    double s[3] = {0, 0, 0}, q[3] = {0, 0, 0};
    uint32_t known = 0;
    for (uint32_t i = threadIdx.x; i < R.samples; i += kBlock) {
        Rng rng = make_rng(R.seed, ((uint64_t)task << 32) ^ ((uint64_t)t1.x << 20) ^ i);
        D3 L = emitter64(R, surface, n, rng);
        D3 tp{1, 1, 1};
        D3 origin = surface + n * kOffset;
        D3 dir = cosine_direction(n, rng.uniform(), rng.uniform());
        double prev_pdf = dotd(n, dir) / kPi;
        bool unknown = false;
        for (uint32_t bounce = 0; bounce < 1024u && prev_pdf > 0.0; ++bounce) {
            const Hit64 hit = trace64(A, origin, dir, kMaxDistance);
            if (hit.status == 0) {
                const double horizon = fmin(fmax(dir.y * 0.35 + 0.65, 0.15), 1.0);
                L = L + tp * D3{A.env[0], A.env[1], A.env[2]} * horizon;
                break;
            }
            if (hit.status == 2) {
                unknown = true;
                break;
            }
            const Mat64 m = material64(A, hit.material);
            if (m.weight > 0.0 && R.total > 0.0) {
                const D3 delta = hit.position - origin;
                const double pdf_light = (m.weight / R.total) * dotd(delta, delta) / fmax(-dotd(hit.normal, dir), 1e-8);
                L = L + tp * m.emission * (prev_pdf / (prev_pdf + pdf_light));
            } else {
                L = L + tp * m.emission;
            }
            const D3 direct = direct64(A, hit.position, hit.normal);
            const D3 nee = emitter64(R, hit.position, hit.normal, rng);
            L = L + tp * m.diffuse * (direct + nee);
            tp = tp * m.diffuse;
            const double maximum = fmax(tp.x, fmax(tp.y, tp.z));
            if (maximum == 0.0) break;
            if (bounce >= 1u) {
                const double survival = fmin(fmax(maximum, 0.1), 0.95);
                if (rng.uniform() > survival) break;
                tp = tp * (1.0 / survival);
            }
            origin = hit.position + hit.normal * kOffset;
            dir = cosine_direction(hit.normal, rng.uniform(), rng.uniform());
            prev_pdf = dotd(hit.normal, dir) / kPi;
        }
        if (unknown) continue;
        s[0] += L.x; s[1] += L.y; s[2] += L.z;
        q[0] += L.x * L.x; q[1] += L.y * L.y; q[2] += L.z * L.z;
        known += 1u;
    }
    // Block reduction in a fixed order.
    __shared__ double red[kBlock][7];
    red[threadIdx.x][0] = s[0]; red[threadIdx.x][1] = s[1]; red[threadIdx.x][2] = s[2];
    red[threadIdx.x][3] = q[0]; red[threadIdx.x][4] = q[1]; red[threadIdx.x][5] = q[2];
    red[threadIdx.x][6] = (double)known;
    __syncthreads();
    for (int stride = kBlock / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
            for (int k = 0; k < 7; ++k) red[threadIdx.x][k] += red[threadIdx.x + stride][k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) {
            R.sum[task * 3u + k] = red[0][k];
            R.second[task * 3u + k] = red[0][3 + k];
        }
        R.known[task] = (uint32_t)red[0][6];
    }
}

}  // namespace

void launch_reference64(const TraceArgs& a, const double* cdf, const int4* emitters, uint32_t n_emitters, double total,
                        const uint4* tasks, uint32_t n_tasks, uint32_t samples, uint64_t seed, double* sum, double* second,
                        uint32_t* known, cudaStream_t s) {
    if (n_tasks == 0) return;
    Ref64Args r{a, cdf, emitters, n_emitters, total, tasks, n_tasks, samples, seed, sum, second, known};
    reference64_kernel<<<n_tasks, kBlock, 0, s>>>(r);
}

}  // namespace vgi
