#!/usr/bin/env python
"""Benchmark of the spectral path-tracing hot path.

A step is one `render_pass` of the full still: the 2,097,152-triangle signet
ring (14k gold, polished/satin slots), noir studio, 1920 x 1080, 256 spp,
max depth 12, 100 mm thin lens at f/16 with autofocus -- 530,841,600 path
samples.  `value` is path-samples/s with the scene resident in HBM, timed on
the device with CUDA events on the library's stream (max over ranks).  `e2e`
is the same metric through the C ABI with host buffers: each step is
argent_render_pass (camera and settings from host memory) plus
argent_film_read of the colour, albedo and normal films into host memory.

Multi-GPU: the path has no exchange step, so N GPUs run N independent
replicas of the workload (weak scaling); value = N * samples / max time.

--impl reference times argent's CPU algorithm (the oracle's restatement, as
the Rust reference cannot be built here) on the host cores, on the same
workload and metric, each step a bounded band of rows of the same frame.
"""

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PUBLISHED_CPU = 17.7e6  # README.md:5-6: 1920x1080 x 256 spp in ~30 s on 32 cores


def dist_setup(n):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as td
        from datetime import timedelta

        backend = "nccl"
        td.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def barrier(world, device=None):
    if world > 1:
        import torch.distributed as td

        td.barrier(device_ids=[device] if device is not None else None)


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as td

    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """dram read+write bytes per launch of the dominant kernel, from the
    committed ncu summary (profiles/ncu_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


def smi_index(device):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",")]
        if device < len(ids) and ids[device].isdigit():
            return int(ids[device])
    return device


# ------------------------------------------------------------------ reference arm (CPU)

def cpu_sample(wl, seconds=12.0, threads=0, rows=None):
    """argent's algorithm (the oracle) on a band of rows of the workload
    frame at the workload's spp.  Returns (samples/s, rows, threads)."""
    import oracle as O

    sc = O.Scene(wl.mesh, wl.desc.c)
    h = wl.height
    mid = h // 2
    if rows is None:
        t0 = time.perf_counter()
        sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed, rows=(mid, mid + 1),
                       threads=threads, want_xyz=False)
        dt = time.perf_counter() - t0
        rows = int(max(1, min(h - mid, seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed, rows=(mid, mid + rows),
                   threads=threads, want_xyz=False)
    dt = time.perf_counter() - t0
    nthr = threads if threads > 0 else (os.cpu_count() or 1)
    return wl.width * rows * wl.spp / dt, rows, nthr, sc


def build_workload(name, tracer=None, spp=None):
    from argent_b200 import workloads as W

    if name == "ring_still":
        return W.ring_still(spp=spp or 16)
    return W.signet_still(tracer, spp=spp or 256)


class OracleTracer:
    """Autofocus probes through argent's own BVH (for the reference arm)."""

    def __init__(self, mesh):
        import oracle as O

        self.bvh = O.Bvh(mesh.positions, mesh.tris)

    def trace_closest(self, rays):
        return self.bvh.intersect(np.ascontiguousarray(rays, np.float32))


def run_reference(args, world, rank):
    if rank != 0:
        return
    from argent_b200 import mesh as M

    m = M.signet() if args.workload == "signet_still" else None
    tracer = OracleTracer(m) if m is not None else None
    from argent_b200 import workloads as W

    wl = W.signet_still(tracer, mesh=m) if m is not None else W.ring_still()
    threads = os.cpu_count() or 1
    _, rows, nthr, sc = cpu_sample(wl, seconds=args.ref_seconds, threads=threads)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed,
                       rows=(wl.height // 2, wl.height // 2 + rows), threads=threads, want_xyz=False)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    per = wl.width * rows * wl.spp
    value = per * len(times) / sum(times)
    sample = f"rows {wl.height // 2}..{wl.height // 2 + rows} of the {wl.width}x{wl.height} frame at {wl.spp} spp ({per} path-samples per step)"
    out = {
        "impl": "reference", "metric": "path-samples/s", "value": value, "unit": "path-samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_CPU, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
                   "triangles": int(wl.mesh.num_tris), "max_depth": int(wl.settings.max_depth),
                   "parallelism": "cpu-threads"},
        "cpu_baseline": {"value": value, "unit": "path-samples/s", "cores": nthr, "kind": "port",
                         "sample": sample + "; argent's Rust path cannot be built here (no cargo), so the C++ "
                                            "restatement (oracle/) runs, OpenMP over rows"},
        "e2e": {"value": value, "unit": "path-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ GPU arm

def run_gpu(args, world, rank, device):
    import torch

    from argent_b200 import mesh as M
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    torch.cuda.set_device(device)
    ctx = Context(device)
    m = M.signet() if args.workload == "signet_still" else M.ring()
    piece = Piece(ctx, m)
    from argent_b200 import workloads as W

    wl = W.signet_still(piece, mesh=m) if args.workload == "signet_still" else W.ring_still()
    if args.spp:
        wl.spp = args.spp  # profiling runs only: the bench line uses the workload's spp
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        film.clear()
        render_pass(ctx, scene, wl.camera, film, wl.settings, wl.spp, wl.seed)

    for _ in range(args.warmup):
        step()
    ctx.sync()

    # Instrumented pass (not timed): traversal visits per ray, rays per sample.
    cf = Film(ctx, wl.width, wl.height)
    ctx.set_counting(True)
    render_pass(ctx, scene, wl.camera, cf, wl.settings, 1, wl.seed)
    counts = ctx.traversal_counts()
    ctx.set_counting(False)
    cf.close()
    px = wl.width * wl.height

    # Timed region (device time, CUDA events on the library stream).
    barrier(world, device)
    torch.cuda.synchronize()
    ctx.sync()
    clocks = Clocks(smi_index(device))
    clocks.start()
    time.sleep(0.3)
    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    ctx.sync()
    launches = ctx.kernel_launches - launches0
    kt = ctx.kernel_times()
    ctx.set_profiling(False)
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, device)
    barrier(world, device)
    samples_per_step = wl.path_samples
    value = world * samples_per_step * args.steps / (ms_max / 1000.0)

    # Roofline of the dominant kernel.
    dom = max(("intersect", "shade", "shadow", "raygen", "film"), key=lambda k: kt[k][0])
    dom_ms, dom_n = kt[dom]
    path_samples_timed = samples_per_step * args.steps
    per_sample = {}
    node_b, tri_b = 80, 48
    rays_c = counts["closest_rays"] / px
    rays_a = counts["any_rays"] / px
    per_sample["intersect"] = (counts["closest_nodes"] * node_b + counts["closest_tris"] * tri_b) / px + rays_c * (
        32 + 16 + 16 + 4)  # ray read, hit write, meta read, queue index
    per_sample["shadow"] = (counts["any_nodes"] * node_b + counts["any_tris"] * tri_b) / px + rays_a * (48 + 16 + 16)
    # shade: path state read+write (o,d,beta,L,lambda,pdf,hit,meta,rng ~ 152 B in, ~ 112 B out),
    # hit attributes (index 16 B + 3 positions + 3 normals 96 B), spectral tables (~64 B)
    per_sample["shade"] = rays_c * (152 + 112 + 112 + 64)
    per_sample["raygen"] = 176.0
    per_sample["film"] = 64.0 + 12.0 * 3 / max(wl.spp, 1)
    alg_bytes_total = per_sample[dom] * path_samples_timed
    achieved = alg_bytes_total / (dom_ms / 1000.0) / 1e9  # GB/s
    peak, peak_kind = peaks()
    traffic = None
    tr = ncu_traffic()
    if tr and tr.get("kernel") == dom and tr.get("workload") == wl.name:
        traffic = tr.get("dram_bytes_per_launch")

    # End-to-end through the C ABI with host buffers.
    e2e_value = None
    h2d = ctypes.sizeof(type(wl.camera)) + ctypes.sizeof(type(wl.settings)) + 8
    d2h = 3 * px * 3 * 4
    if args.e2e_steps > 0:
        c = np.zeros((wl.height, wl.width, 3), np.float32)
        a = np.zeros_like(c)
        nrm = np.zeros_like(c)
        fp = ctypes.POINTER(ctypes.c_float)
        barrier(world, device)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            film.clear()
            render_pass(ctx, scene, wl.camera, film, wl.settings, wl.spp, wl.seed)
            ctx.check(ctx.lib.argent_film_read(film.h, c.ctypes.data_as(fp), a.ctypes.data_as(fp),
                                               nrm.ctypes.data_as(fp)))
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, world, device)
        e2e_value = world * samples_per_step * args.e2e_steps / dt

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, rows, nthr, _ = cpu_sample(wl, seconds=args.ref_seconds, threads=os.cpu_count() or 1)
        cpu = {"value": v, "unit": "path-samples/s", "cores": nthr, "kind": "port",
               "sample": f"rows {wl.height // 2}..{wl.height // 2 + rows} of the frame at {wl.spp} spp; argent's "
                         f"algorithm as restated in oracle/ (Rust reference not buildable here), OpenMP over rows"}

    if rank == 0:
        out = {
            "metric": "path-samples/s", "value": value, "unit": "path-samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_CPU, "dtype": "f32",
            "data": "synthetic (seeded procedural signet, noir studio)",
            "config": {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
                       "triangles": int(m.num_tris), "max_depth": int(wl.settings.max_depth),
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (path state "
                       f"{ctx_wave_mb(ctx)} MB per wave + BVH/triangles {piece.device_bytes / 1e6:.0f} MB)",
                       "vs_baseline_ref": "README.md:5-6 ~17.7M path-samples/s on 32 CPU cores"},
            "clocks": ck,
            "e2e": {"value": e2e_value, "unit": "path-samples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": f"k_{dom}",
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "alg_bytes_per_path_sample": per_sample[dom],
                         "launches": dom_n, "avg_launch_ms": dom_ms / max(dom_n, 1)},
            "kernel_ms": {k: round(v[0], 3) for k, v in kt.items()},
            "traversal_per_path_sample": {k: v / px for k, v in counts.items()},
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)


def ctx_wave_mb(ctx):
    return 224 * 2 ** 21 // 10 ** 6


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="argent", choices=["argent", "reference"])
    ap.add_argument("--workload", default="signet_still", choices=["signet_still", "ring_still"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--spp", type=int, default=0, help="override spp (short profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU only: rank 0 measures, the other ranks have nothing to do.
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), 0)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as td

            td.destroy_process_group()


if __name__ == "__main__":
    main()
