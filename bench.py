#!/usr/bin/env python
"""Benchmark of the per-frame voxel diffuse-GI path on B200.

Workload (one "step" = one frame): the seeded fBm terrain of 512x256x512
voxels (4 octaves, base frequency 1/64, lacunarity 2, gain 0.5, height bias),
8 albedo materials U[0.2, 0.8], a sun of radiance 3 towards (0.4, 0.8, 0.3),
256 emissive voxels of radiance U[1, 10]; the faces turned towards a
cube-map camera at (256, 200, 256) (six 90-degree frusta) form the world
cache; every frame traces 8 paths per face with 2 diffuse hits, terminating
at cached faces, and accumulates the result (prepare, trace, accumulate).

Printed metric: rays/s (one ray = one trace_domain_limited call, counted by
the library's counting pass over the same frame). ``e2e`` is the same metric
through the C ABI with pinned host task/result buffers copied every frame.
``mlp_cache`` compares the MLP cache form on the same terrain: 2 paths a
face a frame, first hits that the world cache does not answer end with the
network's prediction, online training inside each frame; it runs from an
empty cache and an untrained network until its relMSE against the FP64
reference reaches the plain trace's (after the plain run's frames), and
reports both forms' ms/frame, rays/s and time to that relMSE, with the
query kernel's tensor-core throughput.
``batched_scenes`` traces 64 seeded scenes of uneven size (32..256 voxels a
side) both as separate per-scene frames and as batched frames (one
traversal launch per stage over all scenes), from the same empty caches.
``next_rows`` times headless discovery, a far-tier frame and the view
receivers' frame, reconstruction and presentation at 1920x1080.
``cave`` traces the 1024x256x1024 cave in 16 uneven chunks as one batch,
plain and in the MLP cache form with the network's queries batched across
the chunks, to the plain trace's relMSE against the FP64 reference.
``stone_room`` runs the reference's stone-room fixture (32^3, 4 spp, 1 hit,
64 steps, history 64) for 64 frames on the GPU and on the oracle, timed in
full, and compares the final results and state word for word.
``--impl reference`` times the CPU oracle (the restatement of the
reference's algorithm; the reference itself is Rust/WGSL and has no CPU
path) on the box's host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "global-illumination_b200"))

EYE = (256.0, 200.0, 256.0)
SPP = 8
BOUNCES = 2
# Kernels vgi_frame launches in the wavefront layout: prepare, begin,
# (traverse, shade, scatter) per diffuse hit, the last traverse, finalize and
# accumulate.
LAUNCHES_PER_FRAME = 2 + 3 * BOUNCES + 1 + 2
METRIC = "rays/s and ms/frame at equal relMSE vs FP64 ref: MLP cache vs plain, 1 B200"
WORKLOAD = "terrain 512x256x512 fBm, sun + 256 emissive voxels, faces facing a cube-map camera at (256,200,256), 8 spp, 2 bounces via world cache, FP32"


def make_scene(seed, regions=(32, 16, 32), eye=EYE):
    import vgi

    coords, vox = vgi.terrain(*regions, seed=seed, octaves=4, period=64.0, base_height=8.0 * regions[1], falloff=25.0 * regions[1],
                              emitters=256)
    rng = np.random.default_rng(seed)
    m = vgi.VoxelGiMaterials()
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        r = float(rng.uniform(1.0, 10.0))
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(r, r, r)))
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    faces = vgi.exposed_faces(coords, vox, facing=eye)
    transport = vgi.TransportSettings(bounces=BOUNCES, path_steps=2048)
    return coords, vox, m.words(), sun.words(), faces, transport


def measured_peak(key="hbm_gbs", fallback=6650.0):
    """A peak from MEASURED_PEAKS.json (HBM copy GB/s, or cuBLAS bf16 TFLOP/s
    as a burst), else the pool's earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)[key]), "measured"
    except Exception:
        return fallback, "fallback"


def profiled_traffic():
    """DRAM bytes per traversal launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "wave_traverse_terrain.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def profiled_stage_traffic():
    """DRAM bytes per frame of the stage kernels (begin, shade, scatter,
    finalize) from the committed ncu summary of the small terrain, per stage
    launch and in all, with that terrain's face count for scaling."""
    path = os.path.join(ROOT, "profiles", "wave_stages_terrain.md")
    out = {}
    try:
        for line in open(path):
            if line.startswith("stage_dram_bytes:"):
                name, value = line.split(":", 1)[1].split("=")
                out[name.strip()] = float(value)
            elif line.startswith("stage_faces:"):
                out["_faces"] = float(line.split(":")[1])
    except OSError:
        return None
    return out if "_faces" in out and len(out) > 1 else None


class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons during timing."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=lambda: self.lines.extend(iter(self.proc.stdout.readline, "")), daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def lane_use(census):
    """Rays in flight per warp pass of the traversal loop, while rays remained
    queued and after the queue ran out, and the drain's share of passes."""
    wp, lp = census["warp_passes"], census["lane_passes"]
    total = max(wp[0] + wp[1], 1)
    return {"queued": lp[0] / max(wp[0], 1), "drain": lp[1] / max(wp[1], 1), "drain_pass_share": wp[1] / total}


LUMA = np.array([0.2126, 0.7152, 0.0722])


def fp64_reference(g, faces, n_faces=4096, spp=16384):
    """The FP64 converged reference (unbiased path tracing, roulette, no
    cache) on a seeded sample of the faces; it depends on the geometry and
    model only, so one run serves every relMSE of the same scene."""
    import vgi

    rng = np.random.default_rng(17)
    sel = np.sort(rng.choice(faces.shape[0], size=min(n_faces, faces.shape[0]), replace=False))
    t0 = time.perf_counter()
    ref, second, known = g.reference_fp64(vgi.tasks_for(faces[sel]), spp, seed=23)
    seconds = time.perf_counter() - t0
    lr = ref @ LUMA
    var_ref = (np.maximum(second - ref ** 2, 0.0) / np.maximum(known, 1)[:, None]) @ (LUMA * LUMA)
    return {"sel": sel, "l_ref": lr, "spp": spp, "seconds": seconds, "noise": float(np.mean(var_ref / (lr ** 2 + 0.01)))}


def relmse_now(g, ref):
    """Relative MSE of the world cache's accumulated face means against the
    reference, in luminance: mean((L - L_ref)^2 / (L_ref^2 + 0.01))."""
    est = g.read_state()[ref["sel"], 0:3].view(np.float32).astype(np.float64)
    return float(np.mean((est @ LUMA - ref["l_ref"]) ** 2 / (ref["l_ref"] ** 2 + 0.01)))


def relmse(g, ref, frames):
    return {"value": relmse_now(g, ref), "faces": int(ref["sel"].size), "reference_spp": ref["spp"], "frames_accumulated": frames,
            "reference_noise": ref["noise"], "reference_seconds": round(ref["seconds"], 3),
            "definition": "luminance, mean over faces of (L - L_ref)^2 / (L_ref^2 + 0.01); "
                          "L = world-cache mean after the frames run, L_ref = FP64 unbiased path tracing (roulette, no cache)"}


# MLP cache arm: spp, plain warm-up frames, training samples a frame, Adam steps a frame, learning rate.
MLP_SPP, MLP_WARM, MLP_SAMPLES, MLP_STEPS, MLP_LR = 2, 16, 65536, 16, 1e-2
# Rows of one Adam step (16,384: the steps cycle four times through the frame's samples, 128
# tiles of 128 rows on the 148 SMs) and the share of the samples since the network began ending
# paths that a face's mean covers (1.0: those samples, not the warm-up frames' before them).
MLP_STEP_ROWS, MLP_HISTORY = 16384, 1.0
# Inference FLOPs per query at the network's real widths (81 inputs, 3 outputs):
# 2 (81*64 + 3*64*64 + 64*3); the kernel computes the padded 96 x 16 shape.
MLP_QUERY_FLOP = 2 * (81 * 64 + 3 * 64 * 64 + 64 * 3)


def mlp_comparison(g, faces, ref, stream, flush, plain, clock, max_frames):
    """The MLP cache form against the plain trace at equal relMSE vs FP64: the
    MLP form starts from an empty cache and an untrained network (seeded
    init), runs graph-replayed frames (training inside them) until its relMSE
    reaches the plain trace's, and reports its frame time, frames and total
    time beside the plain trace's; frames are CUDA-event timed, L2 flushed
    between them outside the timed pair."""
    import torch

    import vgi

    rng = np.random.default_rng(6)
    init = np.concatenate([(rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)) * 0.5).astype(np.float32).reshape(-1)
                           for i, o in vgi.GpuTracer.MLP_LAYERS])
    # A process loads a kernel's module at its first launch: one plain
    # training frame and one network frame load the MLP form's kernels
    # before the timed run, which then starts again from empty caches and
    # the same untrained network.
    g.set_faces(faces)
    g.mlp_set_weights(init)
    g.set_mlp_cache(True, warm_frames=1, samples=MLP_SAMPLES, steps_per_frame=MLP_STEPS, lr=MLP_LR)
    for _ in range(2):
        g.frame(MLP_SPP, clock)
        clock += 16
    g.sync()
    g.set_mlp_cache(False)
    g.set_faces(faces)
    g.mlp_set_weights(init)
    g.set_mlp_cache(True, warm_frames=MLP_WARM, samples=MLP_SAMPLES, steps_per_frame=MLP_STEPS, lr=MLP_LR)
    g.set_mlp_schedule(MLP_STEP_ROWS, MLP_HISTORY)
    g.set_timing(False)
    g.set_graph(True)
    target = plain["relmse"]
    curve, frame_ms, reached = [], [], None
    at_equal_frames = at_equal_time = None
    near = False
    total = 0.0
    for f in range(max_frames):
        with torch.cuda.stream(stream):
            flush.fill_(float(f))
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
        g.frame(MLP_SPP, clock)
        clock += 16
        with torch.cuda.stream(stream):
            e.record(stream)
        e.synchronize()
        frame_ms.append(s.elapsed_time(e))
        total += frame_ms[-1]
        # relMSE is read every 2 frames, every 4 after 64, and every frame
        # once within 15% of the target, so the frame that reaches it is exact.
        every = 1 if near else (2 if f < 64 else 4)
        value = relmse_now(g, ref) if (f + 1) % every == 0 or f + 1 == plain["frames"] else None
        if value is not None:
            near = value <= 1.15 * target
            curve.append([f + 1, round(total, 2), round(value, 6)])
            if f + 1 == plain["frames"]:
                at_equal_frames = value
            if at_equal_time is None and total >= plain["frames"] * plain["ms_per_frame"]:
                at_equal_time = value
            if reached is None and value <= target:
                reached = {"frames": f + 1, "ms": total}
        if reached is not None and f + 1 >= plain["frames"] and at_equal_time is not None:
            break
    g.set_graph(False)
    stats = g.mlp_stats()
    # One directly launched, event-marked frame for the query and training times.
    g.set_timing(True)
    g.frame(MLP_SPP, clock)
    clock += 16
    g.sync()
    timed = g.mlp_stats()
    census = g.census(MLP_SPP)
    g.set_mlp_cache(False)
    g.set_mlp_schedule(0, 0.0)
    steady_ms = float(np.median(frame_ms[MLP_WARM + 2:])) if len(frame_ms) > MLP_WARM + 4 else float(np.median(frame_ms))
    peak, peak_kind = measured_peak("bf16_tflops", 1590.0)
    achieved = timed["queries"] * MLP_QUERY_FLOP / (timed["query_ms"] * 1e-3) / 1e12 if timed["query_ms"] > 0 else None
    plain_total = plain["frames"] * plain["ms_per_frame"]
    out = {
        "config": {"spp": MLP_SPP, "warm_frames": MLP_WARM, "training_samples_per_frame": MLP_SAMPLES, "adam_steps_per_frame": MLP_STEPS,
                   "rows_per_adam_step": MLP_STEP_ROWS, "history_share": MLP_HISTORY, "lr": MLP_LR, "termination": "uncached first hits take the network's prediction",
                   "network": "96 (81 used) -> 4 x 64 ReLU -> 16 (3 used, exp), BF16 tcgen05, FP32 accumulate and Adam masters"},
        "plain": {"spp": SPP, "frames": plain["frames"], "ms_per_frame": plain["ms_per_frame"], "relmse": target,
                  "ms_to_relmse": plain_total},
        "mlp_ms_per_frame": steady_ms,
        "mlp_rays_per_frame": census["rays"],
        "mlp_rays_per_s": census["rays"] / (steady_ms * 1e-3),
        "frames_per_s_ratio": plain["ms_per_frame"] / steady_ms,
        "relmse_at_equal_frames": at_equal_frames,
        "relmse_at_equal_time": at_equal_time,
        "reached_plain_relmse": reached,
        "speedup_at_equal_relmse": (plain_total / reached["ms"]) if reached else None,
        "relmse_curve": curve[::4] + ([curve[-1]] if curve and (len(curve) - 1) % 4 else []),
        "frames_run": len(frame_ms),
        "training": {"adam_steps": stats["steps"], "last_loss": stats["loss"], "error": stats["error"]},
        "kernel_ms": {"queries": timed["query_ms"], "training": timed["train_ms"], "queries_per_frame": timed["queries"]},
        "tensor_roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                            "kernel": "forward_kernel<PathQueries>",
                            "flop_per_query": MLP_QUERY_FLOP},
    }
    return out, clock


def bench_config(n_faces, warmup):
    """The workload both arms report, word for word the same: the GPU arm
    traces whole frames of it, the CPU arm bounded face samples of the same
    frames from the same warm state."""
    return {"workload": WORKLOAD, "scene_seed": 2, "faces": int(n_faces), "spp": SPP, "bounces": BOUNCES, "path_steps": 2048,
            "warm_state": f"world cache after {warmup} frames from empty, then one frame per step",
            "l2": "device arm: a 256 MB buffer written between timed frames, outside the event pair; the host arm has no device L2"}


def oracle_scene(seed=2, regions=(32, 16, 32), eye=EYE):
    """The bench scene made with the oracle library alone (no libvgi): the
    same seeded generator as make_scene, the materials and sun restated as
    their GPU records."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    coords, vox = O.terrain(*regions, seed=seed, octaves=4, period=64.0, base_height=8.0 * regions[1], falloff=25.0 * regions[1],
                            emitters=256)
    rng = np.random.default_rng(seed)
    entries = [((0.45, 0.45, 0.45), (0.0, 0.0, 0.0))] * 256
    for k in range(8):
        entries[k] = (tuple(rng.uniform(0.2, 0.8, 3)), (0.0, 0.0, 0.0))
    for k in range(248):
        r = float(rng.uniform(1.0, 10.0))
        entries[8 + k] = ((0.5, 0.5, 0.5), (r, r, r))
    words = O.material_words(entries)
    sun = O.directional_light_words((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    faces = O.exposed_faces(coords, vox, facing=eye)
    return coords, vox, words, sun, faces


def cpu_baseline(g, coords, vox, words, lights, faces, budget_s=15.0, parity_faces=2048):
    """The oracle on a bounded face sample with the GPU's warm state, on all
    host threads, and the parity leg: the GPU re-traces the sample's first
    chunk (trace_tasks: the same tasks, sequences, cache state and face
    index) and its results are compared with the oracle's word for word. The
    oracle builds its own geometry and emitters from the voxels."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    n = faces.shape[0]
    scene = O.Scene(coords, vox, top_mode=0)
    geometry = scene.arrays()
    emitters, n_emit, total = O.emitters(coords, vox, words)
    state = g.read_state()
    index = O.face_index(faces[:, :4])
    rng = np.random.default_rng(7)
    sample = np.sort(rng.choice(n, size=min(n, parity_faces), replace=False))
    tasks = np.zeros((sample.size, 8), np.uint32)
    tasks[:, 0:3] = faces[sample, 0:3].view(np.uint32)
    tasks[:, 3] = faces[sample, 3]
    tasks[:, 4] = state[sample, 6]
    d = geometry[0]
    params = O.params_words(sample.size, SPP, d.size // 4, 1, geometry[3], 1, (0, 0, 0), total, n_emit)
    threads = os.cpu_count() or 1
    pipe = O.Pipeline(BOUNCES, 0, 2048, 0, SPP)
    gpu_first = g.trace_tasks(tasks, SPP)
    rays = 0
    start = time.perf_counter()
    chunks = 0
    ref_first = None
    while True:
        # Successive chunks trace the sample's next frames (sequence + spp).
        out, cnt = O.trace_faces(geometry, params, words, lights, emitters, tasks, pipe, state, index, threads)
        if ref_first is None:
            ref_first = out
        tasks[:, 4] += SPP
        rays += cnt["rays"]
        chunks += 1
        if time.perf_counter() - start > budget_s or chunks >= 100000:
            break
    elapsed = time.perf_counter() - start
    base = {"value": rays / elapsed, "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": f"{chunks} x {sample.size} of {n} faces (seeded), {SPP} spp, the GPU's warm cache state, {threads} threads, {elapsed:.1f} s"}
    differ = gpu_first != ref_first
    parity = {"faces": int(sample.size), "words": int(differ.size), "words_differ": int(differ.sum()),
              "faces_differ": int(differ.any(axis=1).sum()),
              "how": "GPU trace_tasks vs the oracle on the same seeded faces, tasks, warm state and face index; "
                     "the oracle's geometry and emitters built from the voxels"}
    return base, parity


def run_reference(args):
    """--impl reference: the CPU oracle (the restatement of the reference's
    algorithm; the reference itself is Rust/WGSL with no CPU path) on the
    same workload, all host threads, without loading libvgi. Its warm-up
    runs the GPU arm's warm-up frames in full (so the state is the one the
    GPU arm's timed frames start from: the two are bit-identical); each
    timed step is one frame over a seeded sample of the faces."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    coords, vox, words, lights, faces = oracle_scene(2)
    scene = O.Scene(coords, vox, top_mode=0)
    geometry = scene.arrays()
    emitters, n_emit, total = O.emitters(coords, vox, words)
    n = faces.shape[0]
    threads = os.cpu_count() or 1
    d = geometry[0]

    def params(count, samples):
        return O.params_words(count, samples, d.size // 4, 1, geometry[3], 1, (0, 0, 0), total, n_emit)

    frames = O.Frames(geometry, params, words, lights, emitters, faces, O.transport_settings(bounces=BOUNCES, path_steps=2048),
                      O.Pipeline(BOUNCES, 0, 2048, 0, SPP), threads=threads)
    clock = 0
    t0 = time.perf_counter()
    for _ in range(args.warmup):
        frames.frame(SPP, clock)
        clock += 16
    warm_s = time.perf_counter() - t0
    rng = np.random.default_rng(11)
    per_step = min(n, 8192)
    rays, secs = 0, 0.0
    for _ in range(args.steps):
        sample = np.sort(rng.choice(n, size=per_step, replace=False)).astype(np.uint32)
        t0 = time.perf_counter()
        cnt, _ = frames.frame_slots(SPP, clock, sample)
        secs += time.perf_counter() - t0
        clock += 16
        rays += cnt["rays"]
    value = rays / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(n, args.warmup),
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads, "kind": "port",
                         "sample": f"{args.warmup} full warm-up frames ({warm_s:.1f} s), then {args.steps} frames over "
                                   f"{per_step} seeded faces of {n} each (begin, trace with gather, accumulate), {threads} threads"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# The cave: 1024x256x1024 voxels, cut along x into 16 uneven chunks (widths
# in regions), traced batched; at most this many faces in all.
CAVE_REGIONS = (64, 16, 64)
CAVE_CHUNKS = [2, 2, 3, 3, 3, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 6]
CAVE_FACES = 4_000_000


def cave_chunks(local):
    """The cave workload: seeded worm tunnels (radius 3..12) under a 16-voxel
    roof with 16 skylight shafts, 2,000 emissive voxels (green (0.5, 4, 1)
    and orange (6, 2, 0.3)), 8 rock materials, a sun and a sky. Its exposed
    faces (every k-th, to at most CAVE_FACES) are the world cache. Each chunk
    is one context holding its own regions and faces; a ray that leaves its
    chunk ends in unloaded space, as it would at the edge of loaded pages."""
    import vgi

    coords, vox = vgi.cave(*CAVE_REGIONS, seed=3)
    vox = vox.reshape(-1, 4096)
    m = vgi.VoxelGiMaterials()
    rng = np.random.default_rng(3)
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    m.set(8, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(0.5, 4.0, 1.0)))
    m.set(9, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(6.0, 2.0, 0.3)))
    words = m.words()
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0)).words()
    per_chunk = []
    lo = 0
    for width in CAVE_CHUNKS:
        keep = np.nonzero((coords[:, 0] >= lo) & (coords[:, 0] < lo + width))[0]
        per_chunk.append((coords[keep], np.ascontiguousarray(vox[keep])))
        lo += width
    faces = [vgi.exposed_faces(c, v) for c, v in per_chunk]
    total = sum(len(f) for f in faces)
    keep = min(1.0, CAVE_FACES / max(total, 1))
    faces = [f[np.random.default_rng(100 + k).random(len(f)) < keep].copy() for k, f in enumerate(faces)]
    tracers = []
    for (c, v), f in zip(per_chunk, faces):
        t = vgi.GpuTracer(local)
        t.upload_regions(c, v)
        t.set_materials(words)
        t.set_lights(sun, 1)
        t.set_environment((0.3, 0.4, 0.5))
        t.build_emitters()
        t.set_transport(vgi.TransportSettings(bounces=BOUNCES, path_steps=2048))
        t.set_faces(f)
        tracers.append(t)
    return tracers, faces, total, keep


def cave_run(local, stream, flush, plain_frames=37):
    """The cave (configuration 5): 16 uneven chunks traced as one batch
    (each stage's traversal one launch, graph-replayed, autotuned), plain,
    then in the MLP cache form with the network's queries batched across
    the chunks (one query launch a frame, each chunk its own network trained
    on its own faces, the rows of 65,536 training samples a frame shared out
    by the chunks' paths). Both start from empty caches; the MLP form runs
    until its relMSE against the FP64 reference (4,096 faces drawn over the
    chunks in proportion to their faces) reaches the plain run's after
    `plain_frames` frames. CUDA events from a common start to the last
    chunk's end, L2 flushed in between."""
    import torch

    import vgi

    tracers, faces, total_faces, keep = cave_chunks(local)
    streams = [torch.cuda.ExternalStream(t.stream, device=torch.device("cuda", local)) for t in tracers]
    n_faces = [len(f) for f in faces]
    # FP64 reference per chunk on its share of 4,096 seeded faces.
    refs = []
    for t, f in zip(tracers, faces):
        k = max(1, int(round(4096 * len(f) / sum(n_faces))))
        refs.append(fp64_reference(t, f, n_faces=k))

    def cave_relmse():
        num = []
        for t, ref in zip(tracers, refs):
            est = t.read_state()[ref["sel"], 0:3].view(np.float32).astype(np.float64)
            num.append((est @ LUMA - ref["l_ref"]) ** 2 / (ref["l_ref"] ** 2 + 0.01))
        return float(np.mean(np.concatenate(num)))

    def timed_frame(run, f):
        with torch.cuda.stream(stream):
            flush.fill_(float(f))
            start = torch.cuda.Event(enable_timing=True)
            start.record(stream)
        for st in streams:
            st.wait_event(start)
        run()
        ends = []
        for st in streams:
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            ends.append(e)
        for e in ends:
            e.synchronize()
        return max(start.elapsed_time(e) for e in ends)

    batch = vgi.GpuBatch(tracers)
    tune = batch.autotune(SPP)
    batch.set_graph(True)
    rays = sum(t.census(SPP)["rays"] for t in tracers)
    clock = 0
    plain_ms = []
    for f in range(plain_frames):
        plain_ms.append(timed_frame(lambda: batch.frame(SPP, clock + 16 * f), f))
    clock += 16 * plain_frames
    plain_rel = cave_relmse()
    rays_late = sum(t.census(SPP)["rays"] for t in tracers)
    plain_step = float(np.median(plain_ms[3:]))
    plain_total = float(sum(plain_ms))
    batch.close()

    # The MLP cache form from empty caches and untrained networks.
    rng = np.random.default_rng(6)
    for t, f in zip(tracers, faces):
        init = np.concatenate([(rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)) * 0.5).astype(np.float32).reshape(-1)
                               for i, o in vgi.GpuTracer.MLP_LAYERS])
        t.set_faces(f)
        t.mlp_set_weights(init)
        share = max(MLP_STEPS * 128, int(MLP_SAMPLES * len(f) / sum(n_faces)))
        # Each chunk's network trains on its share of the frame's samples
        # (2k-7k), split over the steps: cycling such small batches through
        # bigger steps, as the terrain's 65,536 samples do, measured worse here.
        t.set_mlp_cache(True, warm_frames=MLP_WARM, samples=share, steps_per_frame=MLP_STEPS, lr=MLP_LR)
    batch = vgi.GpuBatch(tracers)
    batch.set_graph(True)
    mlp_ms, curve, reached = [], [], None
    total = 0.0
    max_frames = 8 * plain_frames
    for f in range(max_frames):
        mlp_ms.append(timed_frame(lambda: batch.frame(MLP_SPP, clock + 16 * f), f))
        total += mlp_ms[-1]
        if (f + 1) % 4 == 0:
            value = cave_relmse()
            curve.append([f + 1, round(total, 2), round(value, 6)])
            if value <= plain_rel:
                reached = {"frames": f + 1, "ms": total}
                break
    mlp_rays = sum(t.census(MLP_SPP)["rays"] for t in tracers)
    stats = [t.mlp_stats() for t in tracers]
    batch.close()
    for t in tracers:
        t.set_mlp_cache(False)
        t.close()
    mlp_step = float(np.median(mlp_ms[MLP_WARM + 2:])) if len(mlp_ms) > MLP_WARM + 4 else float(np.median(mlp_ms))
    return {
        "workload": f"cave {CAVE_REGIONS[0] * 16}x{CAVE_REGIONS[1] * 16}x{CAVE_REGIONS[2] * 16}, 16 uneven chunks "
                    f"({CAVE_CHUNKS} regions wide), worm tunnels, 16 skylights, 2,000 green and orange emitters, sun and sky; "
                    f"{sum(n_faces)} faces (a seeded {keep:.3f} of the {total_faces} exposed), {SPP} spp plain / {MLP_SPP} spp MLP, 2 bounces",
        "chunks": len(tracers), "faces_min_max": [int(min(n_faces)), int(max(n_faces))], "autotune": tune,
        "plain": {"frames": plain_frames, "ms_per_frame": plain_step, "rays_per_frame": int(rays_late),
                  "rays_per_s": rays_late / (plain_step * 1e-3), "relmse": plain_rel, "ms_to_relmse": plain_total,
                  "first_frame_rays": int(rays)},
        "mlp": {"ms_per_frame": mlp_step, "rays_per_frame": int(mlp_rays), "rays_per_s": mlp_rays / (mlp_step * 1e-3),
                "frames_per_s_ratio": plain_step / mlp_step, "reached_plain_relmse": reached,
                "speedup_at_equal_relmse": (plain_total / reached["ms"]) if reached else None,
                "relmse_curve": curve[::4] + ([curve[-1]] if curve and (len(curve) - 1) % 4 else []),
                "queries_last_frame": int(sum(s["queries"] for s in stats)), "errors": int(sum(s["error"] for s in stats)),
                "query_launch": "one launch a frame over every chunk's queued hits (each chunk's network)"},
        "reference": {"faces": int(sum(r["sel"].size for r in refs)), "spp": refs[0]["spp"],
                      "seconds": round(sum(r["seconds"] for r in refs), 3)},
    }


ROOM_SPP, ROOM_FRAMES = 4, 64
ROOM_STEADY_FROM = 8  # frames before the steady-state timing (graph captured by then)


def stone_room_run(local):
    """The reference's stone-room fixture, run in full: the 32^3 room
    (8 regions) with its stone and emissive materials, every exposed face a
    world-cache slot, 4 paths a face a frame, 1 diffuse hit, 64 traversal
    steps, history 64, for 64 frames from an empty cache. The GPU runs them
    graph-replayed (CUDA events around all 64); the oracle runs the same 64
    frames on all host threads; the two final result and state arrays are
    compared word for word. Rays and paths per frame come from a counting
    pass before each frame (the counting pass changes no state)."""
    import torch

    import vgi

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    coords, vox = vgi.stone_room()
    m = vgi.VoxelGiMaterials()
    m.set(0, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5)))
    m.set(1, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(8.0, 4.0, 1.5)))
    words = m.words()
    transport = vgi.TransportSettings(bounces=1, path_steps=64, history_limit=64)
    faces = vgi.exposed_faces(coords, vox)
    g = vgi.GpuTracer(local)
    g.upload_regions(coords, vox)
    g.set_materials(words)
    g.set_lights(np.zeros(0, np.float32), 0)
    g.set_environment((0.0, 0.0, 0.0))
    g.build_emitters()
    g.set_transport(transport)
    g.set_faces(faces)
    geometry = g.geometry()
    # Work per frame (the counting pass), then the frames themselves.
    rays = paths = 0
    shadow = vgi.GpuTracer(local)
    shadow.upload_regions(coords, vox)
    shadow.set_materials(words)
    shadow.set_lights(np.zeros(0, np.float32), 0)
    shadow.set_environment((0.0, 0.0, 0.0))
    shadow.build_emitters()
    shadow.set_transport(transport)
    shadow.set_faces(faces)
    for f in range(ROOM_FRAMES):
        c = shadow.census(ROOM_SPP)
        rays += c["rays"]
        paths += c["paths"]
        shadow.frame(ROOM_SPP, 16 * f)
    shadow.close()
    g.set_graph(True)
    # The events go on the room tracer's own stream, where its frames run.
    stream = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for f in range(ROOM_FRAMES):
        g.frame(ROOM_SPP, 16 * f)
        if f == ROOM_STEADY_FROM - 1:
            ev[1].record(stream)
    ev[2].record(stream)
    torch.cuda.synchronize()
    gpu_ms = ev[0].elapsed_time(ev[2])
    steady_ms = ev[1].elapsed_time(ev[2]) / (ROOM_FRAMES - ROOM_STEADY_FROM)
    g.set_graph(False)
    got_results, got_state = g.read_results(), g.read_state()
    g.close()

    emitters, n_emit, total = vgi.host_emitters(coords, vox, words)

    def params(n, samples):
        return O.params_words(n, samples, geometry[0].size // 4, 0, geometry[3], 0, (0, 0, 0), total, n_emit)

    threads = os.cpu_count() or 1
    ref = O.Frames(geometry, params, words, np.zeros(0, np.float32), emitters, faces, transport, O.Pipeline(1, 0, 64, 0, ROOM_SPP),
                   threads=threads)
    t0 = time.perf_counter()
    for f in range(ROOM_FRAMES):
        ref.frame(ROOM_SPP, 16 * f)
    cpu_s = time.perf_counter() - t0
    differ = int((got_results != ref.results).sum() + (got_state != ref.state).sum())
    return {
        "workload": f"stone room 32^3 (8 regions), {faces.shape[0]} faces, {ROOM_SPP} spp, 1 bounce, 64 steps, history 64, "
                    f"{ROOM_FRAMES} frames from an empty cache",
        "frames": ROOM_FRAMES, "rays": int(rays), "paths": int(paths),
        "gpu": {"ms_per_frame": gpu_ms / ROOM_FRAMES, "rays_per_s": rays / (gpu_ms * 1e-3), "paths_per_s": paths / (gpu_ms * 1e-3),
                "steady_ms_per_frame": steady_ms,
                "timing": "CUDA events around all frames, graph-replayed (the first frame runs directly and the second is "
                          f"captured, both inside the timed run); steady_ms_per_frame: frames {ROOM_STEADY_FROM}..{ROOM_FRAMES - 1}"},
        "cpu_oracle": {"ms_per_frame": 1000.0 * cpu_s / ROOM_FRAMES, "rays_per_s": rays / cpu_s, "paths_per_s": paths / cpu_s,
                       "threads": threads},
        "parity": {"words": int(got_results.size + got_state.size), "words_differ": differ,
                   "how": "final face results and resident state after all frames, GPU vs oracle"},
    }


def make_batch_scenes(n, seed0=100):
    """Seeded scenes of uneven size for the batched form: the terrain
    generator with 2..16 regions (32..256 voxels) per axis drawn uniformly,
    base height half the height, one emissive voxel per 1024 columns (at
    least 4), the same materials and sun as the terrain workload, faces
    facing an eye above the scene's centre (0.8 of its height)."""
    import vgi

    rng = np.random.default_rng(seed0)
    out = []
    for k in range(n):
        nx, ny, nz = (int(v) for v in rng.integers(2, 17, size=3))
        X, Y, Z = 16 * nx, 16 * ny, 16 * nz
        coords, vox = vgi.terrain(nx, ny, nz, seed=seed0 + k, octaves=4, period=64.0, base_height=0.5 * Y, falloff=1.5 * Y,
                                  emitters=max(4, X * Z // 1024))
        faces = vgi.exposed_faces(coords, vox, facing=(0.5 * X, 0.8 * Y, 0.5 * Z))
        out.append((coords, vox, faces, (X, Y, Z)))
    return out


SPHERES_PER_FRAME = 32


def sphere_edits(coords, faces, rng, mean=SPHERES_PER_FRAME):
    """One frame of the batched workload's edit stream for a scene: a
    Poisson(mean) number of spheres of radius 1..5 around surface voxels (the
    voxels of random faces), each carving air or placing one of the 8
    materials, half and half, and one measured retention event per sphere
    box (vgi.encode_edit_events). Returns (edits x, y, z, value; event words;
    event count; measure records)."""
    import vgi

    size = (coords.max(0) + 1) * 16
    k = max(1, int(rng.poisson(mean)))
    rows = faces[rng.integers(0, len(faces), k)]
    edits, boxes = [], []
    for row in rows:
        c = row[:3].astype(np.int64)
        r = int(rng.integers(1, 6))
        value = 256 if rng.random() < 0.5 else int(rng.integers(0, 8))
        g = np.arange(-r, r + 1)
        off = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        off = off[(off * off).sum(1) <= r * r]
        p = c + off
        p = p[np.all((p >= 0) & (p < size), axis=1)]
        edits.append(np.column_stack([p, np.full(len(p), value)]))
        boxes.append((np.maximum(c - r, 0), np.minimum(c + r, size - 1), len(p), 40.0))
    words, n, measures = vgi.encode_edit_events(boxes)
    return np.concatenate(edits).astype(np.int32), words, n, measures


def batch_comparison(local, stream, flush, n_scenes, steps, warmup):
    """Batched scenes: the same frames of every scene three ways, each scene
    graph-replayed: one scene after another (serial, as the reference's
    trace worker runs them), every scene's vgi_frame on its own stream (the
    streams overlap on the GPU), and vgi_batch_frame (one traversal launch
    per stage over all scenes). All start from empty caches, so the ray work
    is identical; frames are CUDA-event timed from a common start to the
    last scene's end, L2 flushed in between."""
    import torch

    import vgi

    scenes = make_batch_scenes(n_scenes)
    rng = np.random.default_rng(2)
    m = vgi.VoxelGiMaterials()
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(float(rng.uniform(1.0, 10.0)),) * 3))
    words = m.words()
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0)).words()
    tracers = []
    for coords, vox, faces, _ in scenes:
        t = vgi.GpuTracer(local)
        t.upload_regions(coords, vox)
        t.set_materials(words)
        t.set_lights(sun, 1)
        t.set_environment((0.0, 0.0, 0.0))
        t.build_emitters()
        t.set_transport(vgi.TransportSettings(bounces=BOUNCES, path_steps=2048))
        t.set_faces(faces)
        tracers.append(t)
    streams = [torch.cuda.ExternalStream(t.stream, device=torch.device("cuda", local)) for t in tracers]

    def timed(run_frame, n_frames, clock0):
        ms = []
        for f in range(n_frames):
            with torch.cuda.stream(stream):
                flush.fill_(float(f))
                start = torch.cuda.Event(enable_timing=True)
                start.record(stream)
            for st in streams:
                st.wait_event(start)
            run_frame(clock0 + 16 * f)
            ends = []
            for st in streams:
                e = torch.cuda.Event(enable_timing=True)
                e.record(st)
                ends.append(e)
            for e in ends:
                e.synchronize()
            ms.append(max(start.elapsed_time(e) for e in ends))
        return ms

    for t in tracers:
        t.set_graph(True)

    def separate(clock):
        for t in tracers:
            t.frame(SPP, clock)

    def serial(clock):
        # One scene after another, as the reference's trace worker runs them.
        for k, t in enumerate(tracers):
            if k:
                e = torch.cuda.Event()
                e.record(streams[k - 1])
                streams[k].wait_event(e)
            t.frame(SPP, clock)

    def reset():
        for t, (_, _, faces, _) in zip(tracers, scenes):
            t.set_faces(faces)  # empty caches again: every run traces the same frames

    warm_ser = timed(serial, warmup, 0)
    census = sum(t.census(SPP)["rays"] for t in tracers)
    ser = timed(serial, steps, 16 * warmup)
    reset()
    warm_sep = timed(separate, warmup, 0)
    sep = timed(separate, steps, 16 * warmup)
    for t in tracers:
        t.set_graph(False)
    reset()
    batch = vgi.GpuBatch(tracers)
    tune = batch.autotune(SPP)
    batch.set_graph(True)
    warm_bat = timed(lambda clock: batch.frame(SPP, clock), warmup, 0)
    bat = timed(lambda clock: batch.frame(SPP, clock), steps, 16 * warmup)
    # The workload's per-frame edit stream (made beforehand): before every
    # batched frame each scene applies its sphere edits (vgi_edit_voxels:
    # repack of the edited regions and the top-level update) and their
    # measured retention events (vgi_apply_events_measured: the edit measure
    # and the discount over the scene's slots). Host wall time, since the
    # edit calls are synchronous.
    erng = np.random.default_rng(31)
    edit_stream = [[sphere_edits(coords, faces, erng) for coords, _, faces, _ in scenes] for _ in range(steps)]
    spheres = int(np.mean([sum(int(n) for _, _, n, _ in frame) for frame in edit_stream]))
    edit_ms, frame_ms = [], []
    clock_e = 16 * (warmup + steps)

    def edit_scene(k, f):
        # One scene's edits and events; scenes are independent contexts, so
        # host threads apply them side by side (each context one thread).
        edits, words_e, n_ev, measures = edit_stream[f][k]
        tracers[k].edit_voxels(edits)
        tracers[k].apply_events_measured(words_e, n_ev, measures, read=False)

    from concurrent.futures import ThreadPoolExecutor
    pool = ThreadPoolExecutor(max_workers=min(16, len(tracers)))
    for f in range(steps):
        t0 = time.perf_counter()
        list(pool.map(lambda k: edit_scene(k, f), range(len(tracers))))
        t1 = time.perf_counter()
        batch.frame(SPP, clock_e + 16 * f)
        batch.sync()
        t2 = time.perf_counter()
        edit_ms.append(1000.0 * (t1 - t0))
        frame_ms.append(1000.0 * (t2 - t1))
    pool.shutdown()
    batch.close()
    for t in tracers:
        t.close()
    sep_ms, bat_ms, ser_ms = float(np.mean(sep)), float(np.mean(bat)), float(np.mean(ser))
    faces_total = int(sum(f.shape[0] for _, _, f, _ in scenes))
    extents = [e for _, _, _, e in scenes]
    return {
        "scenes": n_scenes, "faces": faces_total,
        "faces_min_max": [int(min(f.shape[0] for _, _, f, _ in scenes)), int(max(f.shape[0] for _, _, f, _ in scenes))],
        "extent_voxels_min_max": [int(min(min(e) for e in extents)), int(max(max(e) for e in extents))],
        "spp": SPP, "bounces": BOUNCES, "rays_per_frame": int(census),
        "serial_ms_per_frame": ser_ms, "separate_ms_per_frame": sep_ms, "batched_ms_per_frame": bat_ms,
        "serial_rays_per_s": census / (ser_ms * 1e-3), "separate_rays_per_s": census / (sep_ms * 1e-3),
        "batched_rays_per_s": census / (bat_ms * 1e-3),
        "speedup_vs_serial": ser_ms / bat_ms, "speedup_vs_separate_streams": sep_ms / bat_ms, "autotune": tune,
        "with_edits": {"spheres_per_frame": spheres, "radius": "1..5", "edit_ms_per_frame": float(np.mean(edit_ms)),
                       "frame_ms": float(np.mean(frame_ms)), "total_ms_per_frame": float(np.mean(edit_ms) + np.mean(frame_ms)),
                       "timing": "host wall time: every scene's edits and measured events (16 host threads, one scene each at a "
                                 "time), then the batched frame to completion"},
        "note": "rays per frame from a census after the warm-up frames; both runs trace identical frames from empty caches",
    }


def next_rows(g, stream, steps=5, eye=EYE):
    """The rows either side of the frame, on the bench terrain at 1920x1080
    from the cube-map camera's position: headless discovery (one primary ray
    per pixel and the distinct faces), a far-tier frame at the reference's
    default settings (8-pixel voxels, 2-pixel cells at 1080p, history 32,
    rate 4, 128 steps), and the view receivers' frame, reconstruction and
    presentation over the discovered faces. Discovery, view frames and
    presentation are synchronous calls (host wall time, host sort and copies
    included); far frames and reconstruction are timed with CUDA events."""
    import torch
    import vgi

    w, h = 1920, 1080
    fwd = np.asarray((0.5, -0.45, 0.6), np.float64)
    cam = (eye, (fwd / np.linalg.norm(fwd)).astype(np.float32), (0.0, 1.0, 0.0), 0.5774, w, h)

    def wall(fn):
        fn()
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            out = fn()
            times.append(1000.0 * (time.perf_counter() - t0))
        return float(statistics.median(times)), out

    def events(fn):
        fn()
        torch.cuda.synchronize()
        pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in pairs:
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return float(statistics.median([a.elapsed_time(b) for a, b in pairs]))

    out = {"camera": {"eye": list(eye), "forward": [float(x) for x in cam[1]], "tan_half_fov": cam[3], "width": w, "height": h}}
    ms, (pixels, faces) = wall(lambda: g.discover_faces(*cam))
    ms_faces, _ = wall(lambda: g.discover_faces(*cam, pixels=False))
    out["discovery"] = {"ms": ms, "ms_faces_only": ms_faces, "pixels": w * h, "faces": int(len(faces)),
                        "rays_per_s": w * h / (ms_faces * 1e-3)}

    settings = vgi.FarTierSettings()
    g.far_reset()
    frame = [0]

    def far():
        g.far_frame(*cam, settings=settings, frame=frame[0])
        frame[0] += 1

    for _ in range(6):  # past the four warm-up traces: one trace in `rate` frames
        far()
    ms = events(far)
    shape, _, _, stats = g.far_read()
    cells = int(shape[0] * shape[1])
    out["far_tier"] = {"ms": ms, "cells": cells, "owned": int(stats[0]), "traced": int(stats[1]), "cells_per_s": cells / (ms * 1e-3),
                       "traced_paths_per_s": int(stats[1]) / (ms * 1e-3)}

    g.view_set_receivers(faces)
    gx, gy = w // 4, h // 4
    g.view_set_tiles(vgi.witness_tiles(pixels, faces, gx, gy), (gx + 1) // 2, (gy + 1) // 2)
    clock = [0]

    def view():
        g.view_frame(clock_ms=clock[0])
        clock[0] += 16

    ms_view, _ = wall(view)
    ms_recon = events(lambda: g.view_reconstruct())
    ms_present, _ = wall(lambda: g.view_present(*cam))
    out["view"] = {"receivers": int(len(faces)), "frame_ms": ms_view, "reconstruct_ms": ms_recon, "present_ms": ms_present,
                   "receivers_per_s": len(faces) / (ms_view * 1e-3)}
    g.view_set_receivers(np.zeros((0, 5), np.int32))
    return out


def profile_next(small=False):
    """Only the bench terrain (or, small, the same terrain at 256x128x256,
    with the camera above it at (64, 160, 64) looking the same way) and one
    pass of the next-row workload, for ncu captures of the discovery,
    far-tier and reconstruction kernels."""
    import torch
    import vgi

    eye = (64.0, 160.0, 64.0) if small else EYE
    coords, vox, words, lights, faces, transport = make_scene(2, (16, 8, 16) if small else (32, 16, 32), eye)
    g = vgi.GpuTracer(0)
    g.upload_regions(coords, vox)
    g.set_materials(words)
    g.set_lights(lights, 1)
    g.set_environment((0.0, 0.0, 0.0))
    g.build_emitters()
    g.set_transport(transport)
    g.set_faces(faces)
    g.frame(SPP, 0)
    stream = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", 0))
    print(json.dumps(next_rows(g, stream, steps=1, eye=eye)), flush=True)
    g.close()


def profile_frame(small=False, frames=4):
    """The plain frame for ncu captures of the wavefront kernels: the bench
    terrain (or, small, the same generator at 256x128x256 voxels with the
    eye at (128, 100, 128), 222k faces, about 0.8 GB on the device) and
    `frames` frames in the default layout, so a capture can skip the
    warm-up frames' launches (3 traversal launches a frame)."""
    import vgi

    regions = (16, 8, 16) if small else (32, 16, 32)
    eye = (128.0, 100.0, 128.0) if small else EYE
    coords, vox, words, lights, faces, transport = make_scene(2, regions, eye)
    g = vgi.GpuTracer(0)
    g.upload_regions(coords, vox)
    g.set_materials(words)
    g.set_lights(lights, 1)
    g.set_environment((0.0, 0.0, 0.0))
    g.build_emitters()
    g.set_transport(transport)
    g.set_faces(faces)
    for f in range(frames):
        g.frame(SPP, 16 * f)
    g.sync()
    census = g.census(SPP)
    print(json.dumps({"profile_frame": {"faces": int(faces.shape[0]), "frames": frames, "rays": census["rays"], "steps": census["steps"],
                                        "traverse_bytes": census["traverse_bytes"]}}), flush=True)
    g.close()


def profile_mlp(frames=3):
    """A small MLP cache workload for ncu captures of the network kernels:
    the same generator at 256x256x256 voxels (64 emissive voxels), faces
    facing an eye at (128, 200, 128), 2 paths a face, the network ending
    uncached first hits from the first frame, 65,536 training samples in 16
    Adam steps of 16,384 rows a frame. About 1 GB on the device."""
    import vgi

    coords, vox = vgi.terrain(16, 16, 16, seed=2, octaves=4, period=64.0, base_height=128.0, falloff=400.0, emitters=64)
    rng = np.random.default_rng(2)
    m = vgi.VoxelGiMaterials()
    for k in range(8):
        m.set(k, vgi.MaterialTransport(diffuse=tuple(rng.uniform(0.2, 0.8, 3))))
    for k in range(248):
        m.set(8 + k, vgi.MaterialTransport(diffuse=(0.5, 0.5, 0.5), emission=(5.0, 5.0, 5.0)))
    sun = vgi.DirectionalTransportLight((0.4, 0.8, 0.3), (3.0, 3.0, 3.0))
    faces = vgi.exposed_faces(coords, vox, facing=(128.0, 200.0, 128.0))
    g = vgi.GpuTracer(0)
    g.upload_regions(coords, vox)
    g.set_materials(m.words())
    g.set_lights(sun.words(), 1)
    g.set_environment((0.0, 0.0, 0.0))
    g.build_emitters()
    g.set_transport(vgi.TransportSettings(bounces=BOUNCES, path_steps=2048))
    g.set_faces(faces)
    init = np.concatenate([(rng.normal(0.0, 1.0 / np.sqrt(i), size=(i, o)) * 0.5).astype(np.float32).reshape(-1)
                           for i, o in vgi.GpuTracer.MLP_LAYERS])
    g.mlp_set_weights(init)
    g.set_mlp_cache(True, warm_frames=0, samples=MLP_SAMPLES, steps_per_frame=MLP_STEPS, lr=MLP_LR)
    g.set_mlp_schedule(MLP_STEP_ROWS, MLP_HISTORY)
    for f in range(frames):
        g.frame(MLP_SPP, 16 * f)
    g.sync()
    st = g.mlp_stats()
    print(json.dumps({"profile_mlp": {"faces": int(faces.shape[0]), "frames": frames, "queries_last_frame": st["queries"],
                                      "adam_steps": st["steps"], "error": st["error"]}}), flush=True)
    g.close()
    if st["error"]:
        sys.exit(1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["vgi", "reference"], default="vgi")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default layout (for profiling runs)")
    ap.add_argument("--no-mlp", action="store_true", help="skip the MLP cache comparison")
    ap.add_argument("--profile-mlp", action="store_true", help="only a small MLP cache workload, for ncu captures")
    ap.add_argument("--batch-scenes", type=int, default=64, help="scenes in the batched-scene comparison (0: skip it)")
    ap.add_argument("--no-next-rows", action="store_true", help="skip discovery, far tier and reconstruction timings")
    ap.add_argument("--no-room", action="store_true", help="skip the stone-room run (64 frames on the GPU and the oracle)")
    ap.add_argument("--no-cave", action="store_true", help="skip the cave run (16 batched chunks, plain and MLP cache)")
    ap.add_argument("--only-cave", action="store_true", help="only the cave run, printed as its own JSON object")
    ap.add_argument("--profile-next", action="store_true", help="only the next-row workload once, for ncu captures")
    ap.add_argument("--profile-frame", action="store_true", help="only plain frames of the terrain, for ncu captures")
    ap.add_argument("--small", action="store_true", help="with --profile-next or --profile-frame: the 256x128x256 terrain")
    args = ap.parse_args()
    if args.profile_frame:
        profile_frame(args.small)
        return
    if args.profile_mlp:
        profile_mlp()
        return
    if args.profile_next:
        profile_next(args.small)
        return
    if args.only_cave:
        import torch

        torch.cuda.set_device(0)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
        stream = torch.cuda.current_stream()
        print(json.dumps({"cave": cave_run(0, stream, flush)}), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import vgi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    # Weak scaling: every rank traces its own terrain (seed 2 + rank); no
    # data-path collective, only the timing reduction.
    coords, vox, words, lights, faces, transport = make_scene(2 + rank)
    g = vgi.GpuTracer(local)
    g.upload_regions(coords, vox)
    g.set_materials(words)
    g.set_lights(lights, 1)
    g.set_environment((0.0, 0.0, 0.0))
    g.build_emitters()
    g.set_transport(transport)
    g.set_faces(faces)
    tuned = None if args.no_autotune else g.autotune(SPP)
    g.set_timing(True)
    n = faces.shape[0]
    stream = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    reference = fp64_reference(g, faces) if rank == 0 else None
    # Clocks from the warm-up frames through the device-timed, graph and
    # end-to-end timed runs (all under load).
    sampler = ClockSampler(local)
    sampler.start()
    clock = 0
    for _ in range(args.warmup):
        g.frame(SPP, clock)
        clock += 16
    g.sync()
    before = g.census(SPP)

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    end_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms = []
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))  # L2 flush: 256 MB written between frames, outside the timed pair
            start_ev[k].record(stream)
        g.frame(SPP, clock)
        clock += 16
        with torch.cuda.stream(stream):
            end_ev[k].record(stream)
        kernel_ms.append(g.frame_times())
    torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(start_ev, end_ev)]
    after = g.census(SPP)
    rays_per_frame = 0.5 * (before["rays"] + after["rays"])
    bytes_per_frame = 0.5 * (before["bytes"] + after["bytes"])
    paths_per_frame = before["paths"]
    total_ms = float(sum(step_ms))

    # The same frames replayed from a captured CUDA graph (timing events off).
    g.set_timing(False)
    g.set_graph(True)
    graph_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 2)]
    for k in range(args.steps + 1):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            graph_ev[2 * k].record(stream)
        g.frame(SPP, clock)
        clock += 16
        with torch.cuda.stream(stream):
            graph_ev[2 * k + 1].record(stream)
    torch.cuda.synchronize()
    # The first frame after enabling runs directly and the second is captured.
    graph_ms = float(np.mean([graph_ev[2 * k].elapsed_time(graph_ev[2 * k + 1]) for k in range(2, args.steps + 1)]))
    g.set_graph(False)
    g.set_timing(True)

    # End to end through the C ABI: pinned host tasks in and every frame's
    # results out, two batches in flight (vgi_submit_batch), so one batch's
    # copies overlap the neighbouring frames; graph-replayed frames. Timed on
    # the host from the first timed submit to the last completion.
    tasks_host = torch.empty((n, 8), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    tasks_host[:] = vgi.tasks_for(faces)
    results_host = [torch.empty((n, 24), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32) for _ in range(2)]
    g.set_timing(False)
    g.set_graph(True)

    def pipelined(count, clock):
        tickets = []
        for k in range(count):
            tickets.append(g.submit_batch(tasks_host, SPP, clock, results_host[k % 2]))
            clock += 16
            if k >= 1:
                g.complete_batch(tickets[k - 1])
        g.complete_batch(tickets[-1])
        return clock

    clock = pipelined(args.warmup, clock)
    t0 = time.perf_counter()
    clock = pipelined(args.steps, clock)
    e2e_total = 1000.0 * (time.perf_counter() - t0)
    clocks = sampler.stop()
    clocks["covers"] = "warm-up, device-timed, graph-replayed and end-to-end frames"
    g.set_graph(False)
    g.set_timing(True)

    stats = torch.tensor([total_ms, e2e_total, rays_per_frame * args.steps, float(n)], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        mx = stats.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = stats.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        total_ms, e2e_total = float(mx[0]), float(mx[1])
        total_rays, total_faces = float(sm[2]), float(sm[3])
    else:
        total_rays, total_faces = float(stats[2]), float(stats[3])

    trace_ms = float(np.mean([t[1] for t in kernel_ms]))
    traverse_ms = float(np.mean([t[3] for t in kernel_ms]))
    traverse_launches = BOUNCES + 1
    traverse_bytes = 0.5 * (before["traverse_bytes"] + after["traverse_bytes"])
    peak, peak_kind = measured_peak()
    # Dominant kernel: the persistent traversal (BOUNCES + 1 launches per frame).
    achieved = traverse_bytes / (traverse_ms * 1e-3) / 1e9
    traffic = profiled_traffic()
    stage_traffic = None
    stages = profiled_stage_traffic()
    if stages:
        # Scaled from the small terrain by faces (paths per face and bounces are the bench's).
        scale = n / stages["_faces"]
        per_stage = {k: v * scale for k, v in stages.items() if k != "_faces"}
        algorithmic = bytes_per_frame - traverse_bytes
        stage_traffic = {"dram_bytes_per_frame": per_stage, "dram_bytes_per_frame_total": sum(per_stage.values()),
                         "algorithmic_bytes_per_frame": algorithmic,
                         "traffic_over_algorithmic": sum(per_stage.values()) / algorithmic,
                         "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one frame's stage launches on the "
                                   "256x128x256 terrain (profiles/wave_stages_terrain.md), scaled by faces",
                         "algorithmic": "the frame's algorithmic bytes outside the traversal (counting pass: tasks, results, "
                                        "materials, lights, emitter and tree reads, face-index probes, accepted cache states)"}
    # The whole frame's algorithmic bytes per second.
    frame_bytes = bytes_per_frame + n * (2 * 144 + 48)
    frame_gbs = frame_bytes / (total_ms / args.steps * 1e-3) / 1e9
    if rank == 0:
        plain_frames = 2 * args.warmup + 3 * args.steps + 1  # warm-up, timed, graph, e2e warm-up and e2e frames
        quality = relmse(g, reference, plain_frames)
        base = parity = None
        if world == 1 and not args.no_cpu_baseline:
            base, parity = cpu_baseline(g, coords, vox, words, lights, faces)
        mlp = None
        if not args.no_mlp:
            # After the CPU baseline, which reads the plain trace's warm state.
            plain = {"frames": plain_frames, "ms_per_frame": graph_ms, "relmse": quality["value"]}
            mlp, clock = mlp_comparison(g, faces, reference, stream, flush, plain, clock, max_frames=max(8 * plain_frames, 64))
        batched = None
        if args.batch_scenes > 0:
            batched = batch_comparison(local, stream, flush, args.batch_scenes, args.steps, args.warmup)
        beside = None if args.no_next_rows else next_rows(g, stream)
        room = None if args.no_room else stone_room_run(local)
        cave = None if args.no_cave else cave_run(local, stream, flush)
        line = {
            "metric": METRIC,
            "value": total_rays / (total_ms * 1e-3),
            "unit": "rays/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": bench_config(n, args.warmup),
            "parallelism": f"independent scene per GPU x{world}",
            "parity": parity,
            "detail": {"paths_per_frame": int(paths_per_frame), "rays_per_frame": rays_per_frame,
                       "census": {"steps": before["steps"], "bytes": before["bytes"], "traverse_bytes": before["traverse_bytes"],
                                  "cache_hits": before["cache_hits"],
                                  "unknown": before["unknown"], "status": before["status"]},
                       "traverse_lanes": lane_use(before),
                       "kernel_ms": {"prepare": float(np.mean([t[0] for t in kernel_ms])), "trace": trace_ms,
                                     "traverse": traverse_ms, "accumulate": float(np.mean([t[2] for t in kernel_ms]))},
                       "trace_algorithmic_gbs": bytes_per_frame / (trace_ms * 1e-3) / 1e9,
                       "autotune": tuned,
                       "graph_ms_per_frame": graph_ms,
                       "paths_per_s": paths_per_frame * world / (total_ms * 1e-3 / args.steps),
                       "frames_per_s": 1000.0 * args.steps / total_ms},
            "e2e": {"value": total_rays / (e2e_total * 1e-3), "unit": "rays/s", "h2d_bytes_per_step": int(n * 32), "d2h_bytes_per_step": int(n * 96)},
            "gpu_launches": LAUNCHES_PER_FRAME * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_kind, "kernel": "wave_traverse_kernel",
                         "launches_per_frame": traverse_launches,
                         "bytes_per_launch": traverse_bytes / traverse_launches,
                         "note": "traversal algorithmic bytes (directory, header, brick, cell words; counting pass) / "
                                 "CUDA-event time of the traversal launches, same frame"},
            "frame_roofline": {
                "bound": "hbm", "achieved": frame_gbs, "peak": peak, "unit": "GB/s", "frac": frame_gbs / peak, "peak_source": peak_kind,
                "bytes_per_frame": frame_bytes,
                "definition": "the whole plain frame: the trace's algorithmic bytes (counting pass: geometry words, tasks, results, "
                              "materials, lights, emitter and tree reads, face-index probes, accepted cache states) plus accumulate's "
                              "state read and write (2 x 144 B) and checkpoint (48 B) per face, over the CUDA-event frame time",
                "note": "most of these bytes hit L2 (the geometry, face index and gather records stay resident); the DRAM traffic "
                        "of the frame's kernels is about a third of them (profiles)"},
            "stage_traffic": stage_traffic,
            "clocks": clocks,
            "relmse": quality,
            "mlp_cache": mlp,
            "batched_scenes": batched,
            "next_rows": beside,
            "stone_room": room,
            "cave": cave,
        }
        if base:
            line["cpu_baseline"] = base
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
