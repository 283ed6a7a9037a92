"""Benchmark of the B200 diffuse path tracer through its C ABI.

Headline workload (one step): the ~1.38M-triangle terrain scene (1024x512-quad
heightfield + 256 level-3 icospheres), 1920x1080, 64 spp, maxDepth 5, rendered
by one prt_render call.  Metric: Mrays/s, rays counted as the reference counts
them (one per closest-hit query).  Synthetic, seeded scene data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank renders its own replica of the workload with
its own pass range (weak scaling, no collective on the data path); the timed
region is bracketed by barriers and the max over ranks is reported.
"""

from __future__ import annotations

import argparse
import contextlib
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "embree-benchmark-protoray_b200")
sys.path.insert(0, PKG)

METRIC = "Mrays/s 1080p 64spp"
WORKLOAD = ("terrain: 1024x512-quad heightfield + 256 level-3 icospheres, 1,376,256 tris; "
            "1920x1080, 64 spp, maxDepth 5")
UNIT = "Mrays/s"
W, H, SPP, DEPTH = 1920, 1080, 64, 5
# the 10M-triangle stress configuration, reported beside the headline
C2_WORKLOAD = ("spheres10m: 2000 level-4 icospheres, log-uniform radius 0.1-5 in a 200^3 box, 10,240,000 tris; "
               "camera on the box's front face; 1920x1080, 16 spp, maxDepth 8")
C2_W, C2_H, C2_SPP, C2_DEPTH = 1920, 1080, 16, 8
ALGO_BYTES_PER_RAY = 192   # compulsory wavefront record traffic per ray of the separate-kernel reference design
L2_BYTES = 126 * 1024 * 1024


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def hbm_fraction(mrays):
    """The HBM roofline of a throughput in Mrays/s: the wavefront record
    traffic per ray (ALGO_BYTES_PER_RAY) at that rate over the copy peak."""
    hbm, kind = peaks()
    achieved = mrays * 1e6 * ALGO_BYTES_PER_RAY / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "peak_kind": kind, "algorithmic_bytes_per_ray": ALGO_BYTES_PER_RAY}


def profile_issue():
    """Warp instructions per closest-hit query of the bounce kernel on the
    headline workload, from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_bounce_issue_terrain1080p.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("warp_inst_per_ray="):
            try:
                return float(line.split("=", 1)[1])
            except ValueError:
                return None
    return None


def profile_traffic():
    """DRAM bytes per ray of the bounce kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_bounce_terrain1080p.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_ray="):
            try:
                return float(line.split("=", 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local, backend):
    import torch
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local) if backend == "nccl" else None)
    return dist if world > 1 else None


def rank_pass_range(rank, world, spp):
    """Passes rendered by `rank`: every rank renders `spp` passes of its own
    range (weak scaling), so ranks never repeat a sample."""
    return rank * spp, spp


def max_over_ranks(x, dist, device):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist, device):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


@contextlib.contextmanager
def c_stdout_to_stderr():
    """The reference's host code logs its progress to stdout; while it runs,
    file descriptor 1 points at stderr, so that this script's stdout carries
    only the JSON line."""
    import ctypes
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def cpu_reference_run(steps, warmup, frames_per_step=1, sample_seconds=None, scene="terrain", accel=1):
    with c_stdout_to_stderr():
        return _cpu_reference_run(steps, warmup, frames_per_step, sample_seconds, scene, accel)


CPU_BVH = {1: "project 8-wide AVX2 BVH with 4-triangle leaves (bvh8.triangle4 class) standing in for Embree 3 (absent)",
           2: "project scalar binary FP32 BVH standing in for Embree 3 (absent)"}


def _cpu_reference_run(steps, warmup, frames_per_step=1, sample_seconds=None, scene="terrain", accel=1):
    """Times the reference's own diffuseStream renderer (oracle/_ref) on the
    host cores; one step = `frames_per_step` 1-spp frames.  scene "terrain":
    1920x1080, maxDepth 5; "spheres10m": the 10.24M-triangle icosphere field
    from its in-field camera, 1920x1080, maxDepth 8.  accel 1: the 8-wide
    AVX2 BVH; 2: the scalar binary BVH."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import scenes
    if not oracle.Reference.available():
        return None
    if scene == "terrain":
        mesh, view = scenes.terrain_scene()
        w, h, depth = W, H, DEPTH
    else:
        mesh, _ = scenes.spheres10m_scene()
        view = scenes.field_view(mesh)
        w, h, depth = C2_W, C2_H, C2_DEPTH
    import tempfile
    d = tempfile.mkdtemp(prefix="prt_bench_")
    path = scenes.write_scene(d, scene, mesh, view)
    R = oracle.Reference()
    rs = R.open(path)
    tb = time.perf_counter()
    rs.build(accel)
    build_s = time.perf_counter() - tb
    cores = int(os.environ.get("PRT_REF_THREADS", "0")) or (os.cpu_count() or 1)
    for _ in range(warmup):
        rs.render("diffuseStream", view, w, h, frames_per_step, depth, accel=accel, want_sums=False)
    rays = 0.0
    secs = 0.0
    t0 = time.perf_counter()
    n = 0
    while n < steps:
        _, st = rs.render("diffuseStream", view, w, h, frames_per_step, depth, accel=accel, want_sums=False)
        rays += st["rays"]
        secs += st["seconds"]
        n += 1
        if sample_seconds and time.perf_counter() - t0 > sample_seconds:
            break
    wall = time.perf_counter() - t0
    try:
        os.remove(path)
    except OSError:
        pass
    return {"value": rays / 1e6 / secs, "rays": rays, "seconds": secs, "wall": wall, "frames": n * frames_per_step,
            "cores": cores, "cpu": cpu_model(), "build_s": build_s, "bvh": CPU_BVH[accel]}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    r = cpu_reference_run(args.steps, args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libprotoray_ref.so was not built"}))
        return 0
    r2 = cpu_reference_run(args.steps, 1, accel=2)
    sample = (f"reference diffuseStream renderer (stream 2048, AVX2, GCC -O3) with the {r['bvh']}; terrain scene "
              f"1920x1080, {r['frames']} frames x 1 spp, maxDepth {DEPTH}; {r['cpu']}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(r["value"], 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * r["seconds"] / max(1, r["frames"]), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        # the same workload as the B200 arm; each step renders a bounded sample of
        # it (1 spp of the 64), described in cpu_baseline.sample
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "maxDepth": DEPTH,
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": round(r["value"], 3), "unit": UNIT, "cores": r["cores"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(r["value"], 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "scalar_bvh": {"value": round(r2["value"], 3), "unit": UNIT, "bvh": r2["bvh"], "frames": r2["frames"]},
    }
    print(json.dumps(line))
    return 0


def make_ctx(prt, mesh, device):
    c = prt.Context(device)
    c.load_mesh(mesh.indices, mesh.positions)
    b = c.build()
    return c, b


def batch_workload(scenes, seed=7, n=64):
    """64 requests: W,H in U{128..1024} rounded to multiples of 8, spp U{1..64},
    maxDepth 5, over 8 seeded scenes of 10K-2M triangles."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        w = int(rng.integers(128, 1025)) // 8 * 8
        h = int(rng.integers(128, 1025)) // 8 * 8
        reqs.append({"scene": int(rng.integers(0, 8)), "width": w, "height": h, "spp": int(rng.integers(1, 65)),
                     "maxDepth": 5})
    return reqs


def run_batch(prt, torch, device, reps=2):
    import scenes
    ctxs, views = [], []
    for k in range(8):
        m, v = scenes.batch_scene(k)
        c, _ = make_ctx(prt, m, device)
        ctxs.append(c)
        views.append(v)
    work = batch_workload(scenes)
    reqs = []
    for q in work:
        acc = torch.zeros((q["height"], q["width"], 4), dtype=torch.float32, device=f"cuda:{device}")
        reqs.append({"scene": ctxs[q["scene"]], "camera": prt.camera_from_view(views[q["scene"]], q["width"], q["height"]),
                     "width": q["width"], "height": q["height"], "spp": q["spp"], "maxDepth": q["maxDepth"],
                     "accum": acc})
    batcher = ctxs[0]
    batcher.render_batch(reqs)   # warm-up (graph capture)
    best_b = None
    for _ in range(reps):
        st = batcher.render_batch(reqs)
        best_b = st if best_b is None or st["ms"] < best_b["ms"] else best_b
    # the same requests as sequential plain launches: one prt_render call per
    # frame (one pass), as the reference render loop drives Device::render
    # (main/render/render_window.cpp:204-256), and, for context, one call per
    # request with all its passes
    def sequential(per_frame):
        ms, rays = 0.0, 0
        for q in work:
            c = ctxs[q["scene"]]
            c.init_frame(q["width"], q["height"])
            c.set_view(views[q["scene"]], q["width"], q["height"])
            if per_frame:
                for p in range(q["spp"]):
                    st = c.render(1, q["maxDepth"], accumulate=True)
                    ms += st["ms"]
                    rays += st["ray"]
            else:
                st = c.render(q["spp"], q["maxDepth"], accumulate=False)
                ms += st["ms"]
                rays += st["ray"]
        return ms, rays

    sequential(True)   # warm-up: graph capture of every (size, spp) configuration
    sequential(False)
    f_ms, f_rays = min(sequential(True) for _ in range(reps))
    c_ms, c_rays = min(sequential(False) for _ in range(reps))
    out = {"batched_mray": round(best_b["mray"], 2), "batched_ms": round(best_b["ms"], 2),
           "sequential_mray": round(f_rays / 1e6 / (f_ms / 1e3), 2), "sequential_ms": round(f_ms, 2),
           "sequential_mode": "one prt_render call (one pass) per frame, requests in order",
           "sequential_calls_mray": round(c_rays / 1e6 / (c_ms / 1e3), 2), "sequential_calls_ms": round(c_ms, 2),
           "requests": len(work), "rays": int(best_b["ray"])}
    out["speedup"] = round(out["batched_mray"] / out["sequential_mray"], 3)
    out["speedup_vs_calls"] = round(out["batched_mray"] / out["sequential_calls_mray"], 3)
    out["roofline"] = hbm_fraction(out["batched_mray"])

    # By request size class (paths = width x height x spp): each class's
    # requests as one batched launch vs one prt_render call per request, device
    # time and host wall time (calls include their launch and completion wait).
    classes = {"small (< 1M paths)": lambda n: n < (1 << 20),
               "medium (1M-8M paths)": lambda n: (1 << 20) <= n < (1 << 23),
               "large (>= 8M paths)": lambda n: n >= (1 << 23)}
    by_class = {}
    for name, pick in classes.items():
        idx = [i for i, q in enumerate(work) if pick(q["width"] * q["height"] * q["spp"])]
        if not idx:
            continue
        sub = [reqs[i] for i in idx]
        batcher.render_batch(sub)   # warm-up (graph capture)
        b_best, b_wall = None, None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = batcher.render_batch(sub)
            wall = time.perf_counter() - t0
            if b_best is None or st["ms"] < b_best["ms"]:
                b_best, b_wall = st, wall

        def calls():
            ms, rays = 0.0, 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for i in idx:
                q = work[i]
                c = ctxs[q["scene"]]
                c.init_frame(q["width"], q["height"])
                c.set_view(views[q["scene"]], q["width"], q["height"])
                st = c.render(q["spp"], q["maxDepth"], accumulate=False)
                ms += st["ms"]
                rays += st["ray"]
            return ms, rays, time.perf_counter() - t0

        calls()
        c_best = min((calls() for _ in range(reps)), key=lambda x: x[0])
        by_class[name] = {"requests": len(idx), "rays": int(b_best["ray"]),
                          "batched_mray": round(b_best["mray"], 2), "calls_mray": round(c_best[1] / 1e3 / c_best[0], 2),
                          "speedup_vs_calls": round(b_best["mray"] / (c_best[1] / 1e3 / c_best[0]), 3),
                          "batched_wall_ms": round(1e3 * b_wall, 2), "calls_wall_ms": round(1e3 * c_best[2], 2),
                          "speedup_vs_calls_wall": round(c_best[2] / b_wall, 3)}
    out["by_size_class"] = by_class
    for c in ctxs:
        c.close()
    return out


def run_fwd_bwd(prt, torch, device):
    """512x512, 16 spp, small scene with per-triangle albedo U[0.2,0.8]:
    forward render and path-replay backward of an L2 image loss."""
    import scenes
    mesh, view = scenes.small_scene()
    c, _ = make_ctx(prt, mesh, device)
    alb = torch.from_numpy(scenes.albedo_for(mesh)).to(f"cuda:{device}")
    c.set_albedo(alb)
    Wd, Hd, spp, depth = 512, 512, 16, 5
    c.init_frame(Wd, Hd)
    c.set_view(view, Wd, Hd)
    g = torch.randn((Hd, Wd, 3), dtype=torch.float32, device=f"cuda:{device}")
    d_alb = torch.zeros(mesh.tri_count, dtype=torch.float32, device=f"cuda:{device}")
    d_sky = torch.zeros(1, dtype=torch.float32, device=f"cuda:{device}")
    for _ in range(2):
        c.clear()
        c.render(spp, depth, accumulate=False)
        c.render_backward(0, spp, depth, g, d_alb, d_sky)
    torch.cuda.synchronize()
    fw, fb = [], []
    for _ in range(3):
        c.clear()
        t0 = time.perf_counter()
        st = c.render(spp, depth, accumulate=False)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        c.render_backward(0, spp, depth, g, d_alb, d_sky)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        fw.append(st["ms"])
        fb.append(st["ms"] + (t2 - t1) * 1e3)
    c.close()
    f, b = min(fw), min(fb)
    return {"fwd_ms": round(f, 3), "fwd_bwd_ms": round(b, 3), "ratio": round(b / f, 3),
            "config": "small scene 82K tris, 512x512, 16 spp, maxDepth 5, per-triangle albedo"}


def run_c2(prt, torch, device, steps, warmup, cpu_seconds):
    """The 10.24M-triangle icosphere field at 1920x1080, 16 spp, maxDepth 8:
    build time of a context's first BVH build and of a rebuild, the
    autotuner's launch configuration for it, device and end-to-end Mrays/s (L2
    flushed between timed steps), and the reference's diffuseStream on the
    host cores on the same scene and camera."""
    import scenes
    mesh, _ = scenes.spheres10m_scene()
    view = scenes.field_view(mesh)
    c = prt.Context(device)
    c.load_mesh(mesh.indices, mesh.positions)
    b0 = c.build()
    b1 = c.build()
    c.init_frame(C2_W, C2_H)
    cam = prt.camera_from_view(view, C2_W, C2_H)
    c.set_camera(cam)
    t0 = time.perf_counter()
    tn = c.autotune(C2_SPP, C2_DEPTH)
    tune = {"block": tn["blockSize"], "blocksPerSM": tn["blocksPerSM"], "pathsPerWave": tn["pathsPerWave"],
            "chains": tn["concurrentWaves"], "primaryPackets": tn["primaryPackets"],
            "tuning_s": round(time.perf_counter() - t0, 2)}
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")
    for _ in range(warmup):
        c.set_pass(0)
        c.render(C2_SPP, C2_DEPTH, accumulate=False)
    rays, ms = 0, 0.0
    for s in range(steps):
        flush.fill_(float(s))
        torch.cuda.synchronize()
        c.set_pass(0)
        st = c.render(C2_SPP, C2_DEPTH, accumulate=False)
        rays += st["ray"]
        ms += st["ms"]
    host_img = torch.empty((C2_H, C2_W, 4), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    e_rays = 0
    t0 = time.perf_counter()
    for s in range(steps):
        c.set_camera(cam)
        c.set_pass(0)
        st = c.render(C2_SPP, C2_DEPTH, accumulate=False)
        c.read_accum(host_img)
        e_rays += st["ray"]
    torch.cuda.synchronize()
    e_secs = time.perf_counter() - t0
    c.close()
    out = {"workload": C2_WORKLOAD, "triangles": mesh.tri_count, "width": C2_W, "height": C2_H, "spp": C2_SPP,
           "maxDepth": C2_DEPTH, "steps": steps, "value": round(rays / 1e6 / (ms / 1e3), 2), "unit": UNIT,
           "ms_per_step": round(ms / steps, 3), "rays_per_step": int(rays / steps),
           "e2e": {"value": round(e_rays / 1e6 / e_secs, 2), "unit": UNIT, "h2d_bytes_per_step": 76,
                   "d2h_bytes_per_step": C2_W * C2_H * 16},
           "buildMs_first": round(b0["buildMs"], 2), "buildMs": round(b1["buildMs"], 2),
           "buildMprim": round(mesh.tri_count / 1e3 / b1["buildMs"], 2), "bvh8_nodes": b1["nodeCount"],
           "bvh8_levels": b1["levels"], "launch_config": tune}
    out["roofline"] = hbm_fraction(out["value"])
    if cpu_seconds > 0:
        r = cpu_reference_run(1000, 1, sample_seconds=cpu_seconds, scene="spheres10m")
        if r is not None:
            out["cpu_baseline"] = {
                "value": round(r["value"], 3), "unit": UNIT, "cores": r["cores"], "kind": "reference",
                "build_s": round(r["build_s"], 2),
                "sample": (f"reference diffuseStream renderer with the {r['bvh']}, same scene and camera, "
                           f"{r['frames']} frames x 1 spp, maxDepth {C2_DEPTH}, {r['wall']:.1f} s")}
            out["vs_cpu"] = round(out["value"] / r["value"], 1)
    return out


def run_mesh_build(prt, torch, device):
    """`protoray build` of the terrain scene written as an OBJ (positions and
    faces, 52 MB): OBJ parse on host threads, GPU mesh build from the OBJ's
    indexed form (upload, expansion, de-duplication, Morton reorder), .mesh
    write; beside it the reference's ObjLoader and
    TriangleMeshBuilder (one host thread each) on the same file, when the
    reference build is present."""
    import shutil
    import tempfile
    import scenes
    mesh, _ = scenes.terrain_scene()
    d = tempfile.mkdtemp(prefix="prt_build_")
    try:
        obj = os.path.join(d, "terrain.obj")
        with open(obj, "w") as f:
            np.savetxt(f, mesh.positions, fmt="v %.9g %.9g %.9g")
            np.savetxt(f, mesh.indices + 1, fmt="f %d %d %d")
        c = prt.Context(device)
        best = None
        for _ in range(6):
            t0 = time.perf_counter()
            soup = prt.Soup(obj)
            t1 = time.perf_counter()
            info = c.build_mesh_soup(soup)
            t2 = time.perf_counter()
            soup.close()
            c.save_built_mesh(os.path.join(d, "terrain.mesh"))
            t3 = time.perf_counter()
            r = {"parse_ms": (t1 - t0) * 1e3, "build_device_ms": info["buildMs"], "build_ms": (t2 - t1) * 1e3,
                 "save_ms": (t3 - t2) * 1e3, "e2e_ms": (t3 - t0) * 1e3}
            if best is None or r["e2e_ms"] < best["e2e_ms"]:
                best = r
        c.close()
        out = {"triangles": mesh.tri_count, "unique_vertices": info["vertCount"],
               "obj_mb": round(os.path.getsize(obj) / 1e6, 1), "host_threads": os.cpu_count(),
               "gpu": {k: round(v, 2) for k, v in best.items()},
               "build_mtris_per_s": round(mesh.tri_count / best["build_ms"] / 1e3, 1),
               "build_device_mtris_per_s": round(mesh.tri_count / best["build_device_ms"] / 1e3, 1)}
        ref_so = os.path.join(ROOT, "oracle", "_ref", "libprotoray_ref.so")
        if os.path.exists(ref_so):
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            R = oracle.Reference()
            with c_stdout_to_stderr():
                t0 = time.perf_counter()
                rt, rn = R.load_obj(obj)
                t1 = time.perf_counter()
                build_ms = R.build_soup(rt, rn, os.path.join(d, "terrain_ref.mesh"))
                t2 = time.perf_counter()
            out["reference"] = {"parse_ms": round((t1 - t0) * 1e3, 1), "build_ms": round(build_ms, 1),
                                "e2e_ms": round((t2 - t0) * 1e3, 1),
                                "kind": "reference ObjLoader + TriangleMeshBuilder compiled from source, 1 thread"}
            out["speedup_build"] = round(build_ms / best["build_ms"], 1)
            out["speedup_e2e"] = round((t2 - t0) * 1e3 / best["e2e_ms"], 1)
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_kernel_tour(prt, torch, device):
    """Launches every kernel family of the library once on a case whose inputs
    exceed L2 where the kernel reads bulk data, for profiler captures
    (`ncu ... python bench.py --kernel-tour`); prints one JSON line of
    CUDA-event times.  Phases: BVH build of 2000 level-4 icospheres (10.2M
    triangles); 4M incoherent closest-hit and any-hit queries on the terrain;
    one diffuse2 render (960x540, 4 spp); path-replay forward and backward
    (small scene, 512x512, 4 spp, per-triangle albedo); a batch of 8 requests;
    the LDR resolve of a 3840x2160 frame; the mesh builder on the terrain as a
    soup (1.38M triangles, 138 MB)."""
    import scenes
    dev = f"cuda:{device}"
    out = {}

    def timed(name, fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out[name + "_ms"] = round(a.elapsed_time(b), 3)

    m, _ = scenes.spheres10m_scene()
    c = prt.Context(device)
    c.load_mesh(m.indices, m.positions)
    timed("build_10m", c.build)
    c.close()

    terrain, tview = scenes.terrain_scene()
    c = prt.Context(device)
    c.load_mesh(terrain.indices, terrain.positions)
    c.build()
    n = 1 << 22
    g = torch.Generator(device=dev).manual_seed(5)
    lo, hi = terrain.positions.min(0), terrain.positions.max(0)
    rays = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    for k in range(3):
        rays[:, k] = float(lo[k]) + torch.rand(n, generator=g, device=dev) * float(hi[k] - lo[k])
    d = torch.randn((n, 3), generator=g, device=dev)
    rays[:, 4:7] = d / d.norm(dim=1, keepdim=True)
    rays[:, 7] = 3.0e38
    hits = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    occ = torch.zeros(n, dtype=torch.float32, device=dev)
    timed("intersect_4m", lambda: c.intersect(rays, hits, n))
    timed("occluded_4m", lambda: c.occluded(rays, occ, n))
    c.set_integrator("diffuse2")
    c.init_frame(960, 540)
    c.set_view(tview, 960, 540)
    timed("diffuse2_960x540x4", lambda: c.render(4, 5, accumulate=False))
    c.init_frame(3840, 2160)
    timed("resolve_ldr_4k", c.read_ldr)
    c.close()

    small, sview = scenes.small_scene()
    c = prt.Context(device)
    c.load_mesh(small.indices, small.positions)
    c.set_albedo(torch.from_numpy(scenes.albedo_for(small)).to(dev))
    c.build()
    c.init_frame(512, 512)
    c.set_view(sview, 512, 512)
    gimg = torch.randn((512, 512, 3), dtype=torch.float32, device=dev)
    d_alb = torch.zeros(small.tri_count, dtype=torch.float32, device=dev)
    d_sky = torch.zeros(1, dtype=torch.float32, device=dev)
    timed("replay_fwd_512x4", lambda: c.render_replay(0, 4, 5))
    timed("replay_bwd_512x4", lambda: c.render_backward(0, 4, 5, gimg, d_alb, d_sky))
    c.close()
    c = prt.Context(device)   # batched requests use the constant albedo
    c.load_mesh(small.indices, small.positions)
    c.build()
    reqs = []
    for k in range(8):
        w, h = 128 + 64 * k, 512 - 32 * k
        reqs.append({"scene": c, "camera": prt.camera_from_view(sview, w, h), "width": w, "height": h,
                     "spp": 1 + 3 * k, "maxDepth": 5,
                     "accum": torch.zeros((h, w, 4), dtype=torch.float32, device=dev)})
    timed("batch_8", lambda: c.render_batch(reqs))
    c.close()

    soup = np.zeros(terrain.tri_count, prt.SOUP_DTYPE)
    soup["v"]["pos"] = terrain.positions[terrain.indices]
    c = prt.Context(device)
    timed("mesh_build_1.38m", lambda: c.build_mesh(soup, ["", "Default"]))
    c.close()
    print(json.dumps({"kernel_tour": out}))
    return 0


def main():
    global W, H, SPP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched, fwd+bwd, mesh-build and 10M-triangle measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default launch configuration")
    ap.add_argument("--launch-config", default=None,
                    help="block,blocksPerSM,pathsPerWave,chains,primaryPackets: set this launch configuration "
                         "instead of autotuning (for profiler captures of the configuration a bench run chose)")
    ap.add_argument("--width", type=int, default=W, help="smaller frames are for profiling captures only")
    ap.add_argument("--height", type=int, default=H)
    ap.add_argument("--spp", type=int, default=SPP)
    ap.add_argument("--profile-depths", action="store_true",
                    help="render the headline frame once through prt_render_profile (one launch per bounce and "
                         "wave, no graph), print rays and ms per bounce, and exit (for profiler captures)")
    ap.add_argument("--kernel-tour", action="store_true",
                    help="launch every kernel family once on small cases (for profiler captures) and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        return run_reference(args)
    if args.kernel_tour:
        import torch
        sys.path.insert(0, PKG)
        import prt
        torch.cuda.set_device(0)
        return run_kernel_tour(prt, torch, 0)
    W, H, SPP = args.width, args.height, args.spp
    if args.profile_depths:
        import prt
        import scenes
        mesh, view = scenes.terrain_scene()
        c, _ = make_ctx(prt, mesh, 0)
        c.init_frame(W, H)
        c.set_view(view, W, H)
        if args.launch_config:
            b, per_sm, ppw, ch, pk = (int(x) for x in args.launch_config.split(","))
            c.set_tune(b, per_sm, ppw, ch, pk)
        ms, rays = c.render_profile(SPP, DEPTH)
        print(json.dumps({"ms_per_depth": [round(float(x), 4) for x in ms], "rays_per_depth": [int(x) for x in rays]}))
        c.close()
        return 0

    rank, world, local = dist_env()
    import torch
    import prt
    import scenes
    torch.cuda.set_device(local)
    dist = init_dist(world, local, "nccl")
    dev = f"cuda:{local}"

    mesh, view = scenes.terrain_scene()
    ctx, build = make_ctx(prt, mesh, local)
    ctx.init_frame(W, H)
    ctx.set_view(view, W, H)

    # L2 flush buffer (written between timed steps)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    pass0, npass = rank_pass_range(rank, world, SPP)

    # queue and launch sizes from the library's autotuner, timed on this
    # workload before the warm-up
    tune = None
    if args.launch_config:
        b, per_sm, ppw, ch, pk = (int(x) for x in args.launch_config.split(","))
        ctx.set_tune(b, per_sm, ppw, ch, pk)
    elif not args.no_autotune:
        t0 = time.perf_counter()
        tune = ctx.autotune(npass, DEPTH)
        tune = {"block": tune["blockSize"], "blocksPerSM": tune["blocksPerSM"], "pathsPerWave": tune["pathsPerWave"],
                "chains": tune["concurrentWaves"], "primaryPackets": tune["primaryPackets"],
                "tuning_s": round(time.perf_counter() - t0, 2)}

    def step(pass_base):
        ctx.set_pass(pass_base)
        return ctx.render(npass, DEPTH, accumulate=False)

    for w in range(args.warmup):
        step(pass0)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    launches0 = ctx.launch_count()
    rays, ms = 0, 0.0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            flush.fill_(float(s))
            torch.cuda.synchronize()
            st = step(pass0)
            rays += st["ray"]
            ms += st["ms"]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        wall = time.perf_counter() - t0
    launches = ctx.launch_count() - launches0
    ms_max = max_over_ranks(ms, dist, dev)
    rays_all = sum_over_ranks(rays, dist, dev)
    value = rays_all / 1e6 / (ms_max / 1e3)

    # end-to-end through the C ABI with host buffers: camera in, image out.
    # With N ranks the frame is the sum of the ranks' accumulators (their
    # pass ranges are disjoint): one NCCL reduce into rank 0, which reads it.
    host_img = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    dev_img = torch.empty((H, W, 4), dtype=torch.float32, device=dev) if dist else None
    cam = prt.camera_from_view(view, W, H)

    def frame_out():
        if dist is None:
            ctx.read_accum(host_img)
            return
        ctx.read_accum(dev_img)
        dist.reduce(dev_img, dst=0, op=dist.ReduceOp.SUM)
        if rank == 0:
            host_img.copy_(dev_img)

    ctx.set_camera(cam)
    step(pass0)
    frame_out()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e_rays = 0
    t0 = time.perf_counter()
    for s in range(args.steps):
        ctx.set_camera(cam)
        st = step(pass0)
        frame_out()
        e_rays += st["ray"]
    torch.cuda.synchronize()
    e_secs = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e_value = sum_over_ranks(e_rays, dist, dev) / 1e6 / e_secs

    hbm, peak_kind = peaks()
    achieved = value * 1e6 * ALGO_BYTES_PER_RAY / 1e9 / max(1, world)   # per GPU
    tr = profile_traffic()
    rays_per_step = rays / args.steps
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_kind": peak_kind,
                "traffic": None if tr is None else round(tr * rays_per_step),
                "algorithmic_bytes_per_ray": ALGO_BYTES_PER_RAY,
                "per": "render step (the k_bounce launches of one 64-spp frame, >99% of its device time)"}
    if tr is not None:
        roofline["traffic_bytes_per_ray"] = tr
    # The binding limit of the bounce kernel is instruction issue, not HBM:
    # warp instructions per ray (ncu smsp__inst_executed of the bounce
    # launches of one wave, committed summary) x rays of a step, over the SM
    # issue peak (SMs x 4 schedulers x 1 warp instruction per clock at the
    # median SM clock sampled during the timed steps) x the step's device time.
    ipr = profile_issue()
    roofline_issue = None
    if ipr is not None:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks.summary().get("sm_mhz") or 1965.0
        inst_rate = ipr * rays_per_step / (ms_max / args.steps / 1e3)
        peak_rate = sms * 4 * mhz * 1e6
        roofline_issue = {"bound": "issue", "achieved": round(inst_rate / 1e12, 4), "peak": round(peak_rate / 1e12, 4),
                          "unit": "T warp-inst/s", "frac": round(inst_rate / peak_rate, 4),
                          "warp_inst_per_ray": ipr, "sms": sms, "sm_mhz": mhz,
                          "per": "render step (device time of the whole step; the bounce kernels are >99% of it)"}

    extras = {}
    if rank == 0 and not args.no_extras:
        # each extra block carries the SM clocks sampled while it ran
        with ClockSampler(local) as ck:
            extras["batched"] = run_batch(prt, torch, local)
        extras["batched"]["clocks"] = ck.summary()
        with ClockSampler(local) as ck:
            extras["differentiable"] = run_fwd_bwd(prt, torch, local)
        extras["differentiable"]["clocks"] = ck.summary()
        extras["mesh_build"] = run_mesh_build(prt, torch, local)
        with ClockSampler(local) as ck:
            extras["c2"] = run_c2(prt, torch, local, args.steps, args.warmup,
                                  0 if (args.no_cpu or world > 1) else args.cpu_seconds / 2)
        extras["c2"]["clocks"] = ck.summary()

    cpu = cpu_scalar = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_run(1000, 1, sample_seconds=0.7 * args.cpu_seconds)
        cpu_scalar = cpu_reference_run(1000, 1, sample_seconds=0.3 * args.cpu_seconds, accel=2)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic seeded scene (no public dataset)",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP,
                       "maxDepth": DEPTH, "triangles": mesh.tri_count, "l2": "flushed between timed steps",
                       "parallelism": f"replicas{world}", "buildMs": round(build["buildMs"], 2),
                       "buildMprim": round(build["buildMprim"], 2), "bvh8_nodes": build["nodeCount"],
                       "bvh8_levels": build["levels"],
                       "launch_config": tune or {"autotune": "off", **ctx.get_tune()}},
            "rays_per_step": int(rays / args.steps),
            "wall_s": round(wall, 3),
            "e2e": {"value": round(e_value, 2), "unit": UNIT, "h2d_bytes_per_step": 76,
                    "d2h_bytes_per_step": W * H * 16},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "roofline_issue": roofline_issue,
            "clocks": clocks.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = {
                "value": round(cpu["value"], 3), "unit": UNIT, "cores": cpu["cores"], "kind": "reference",
                "sample": (f"reference diffuseStream renderer with the {cpu['bvh']}, terrain scene 1920x1080, "
                           f"{cpu['frames']} frames x 1 spp, maxDepth 5, {cpu['wall']:.1f} s; {cpu['cpu']}"),
                "scalar_bvh": {"value": round(cpu_scalar["value"], 3), "bvh": cpu_scalar["bvh"],
                               "frames": cpu_scalar["frames"]}}
        line.update(extras)
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
