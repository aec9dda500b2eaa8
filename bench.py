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


def dist_setup(n, backend=None):
    """One process per GPU (replicas): rank, world and local rank from the
    launcher's environment; NCCL on GPUs, gloo where there are none.  The
    group's timeout is short so that ranks waiting on a lost peer end."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as td
        from datetime import timedelta

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        td.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def barrier(world, device=None):
    if world > 1:
        import torch.distributed as td

        td.barrier(device_ids=[device] if device is not None and td.get_backend() == "nccl" else None)


def max_over_ranks(x, world, device):
    """The largest of every rank's x (timings are taken as the max over ranks)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as td

    on_gpu = device is not None and td.get_backend() == "nccl"
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}" if on_gpu else "cpu")
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, seconds_max):
    """Replicas: every rank processes the same units; the job's rate is all
    ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max


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
    """DRAM read+write bytes per ray of the traversal kernel and its issue
    activity, from one ncu capture summarised in profiles/ncu_traffic.json
    (the capture's command is in that file), or None."""
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

def cpu_model():
    """The host CPU's model name (the CPU baseline's hardware)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def spread_bands(height, rows, n=8):
    """n bands of `rows` rows spread evenly down a frame: band k is centred
    on row (2k + 1) h / 2n, so together they sample the frame's average
    (sky, piece, floor) rather than its busiest middle."""
    out = []
    for k in range(n):
        c = (2 * k + 1) * height // (2 * n)
        y0 = max(0, min(height - rows, c - rows // 2))
        out.append((y0, y0 + rows))
    return out


def describe_bands(bands):
    return ", ".join(f"{a}..{b}" for a, b in bands)


def cpu_sample(wl, seconds=12.0, threads=0, rows=None):
    """argent's algorithm (the oracle) on 8 bands of rows spread down the
    workload frame at the workload's spp.  Returns (samples/s, bands,
    threads, scene)."""
    import oracle as O

    sc = O.Scene(wl.mesh, wl.desc.c)
    h = wl.height

    def run(bands):
        for y0, y1 in bands:
            sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed, rows=(y0, y1),
                           threads=threads, want_xyz=False)

    if rows is None:
        t0 = time.perf_counter()
        run(spread_bands(h, 1))
        dt = time.perf_counter() - t0
        rows = int(max(1, min(h // 8, seconds / max(dt, 1e-3))))
    bands = spread_bands(h, rows)
    t0 = time.perf_counter()
    run(bands)
    dt = time.perf_counter() - t0
    nthr = threads if threads > 0 else (os.cpu_count() or 1)
    return wl.width * rows * len(bands) * wl.spp / dt, bands, nthr, sc


WORKLOADS = ("signet_still", "ring_still", "gems_still", "reel_batch", "serve_trace")
DATA = {"signet_still": "seeded procedural signet, noir studio",
        "ring_still": "seeded procedural ring, noir studio",
        "gems_still": "seeded procedural 18k setting with a brilliant and 36 side stones, white studio",
        "reel_batch": "seeded procedural signets of 61k/1.1M/3.0M triangles, seeded synthetic HDRI",
        "serve_trace": "seeded procedural signets of 40k..3.0M triangles, Poisson arrivals seed 6"}


def build_mesh(name):
    from argent_b200 import mesh as M

    return {"signet_still": M.signet, "ring_still": M.ring, "gems_still": M.gem_ring}[name]()


def build_workload(name, mesh, tracer=None):
    """The named workload on `mesh`; `tracer` (anything with
    trace_closest) enables thin-lens autofocus where the shot uses it."""
    from argent_b200 import workloads as W

    if name == "ring_still":
        return W.ring_still()
    if name == "gems_still":
        return W.gems_still(tracer, mesh=mesh)
    return W.signet_still(tracer, mesh=mesh)


class OracleTracer:
    """Autofocus probes through argent's own BVH (for the reference arm)."""

    def __init__(self, mesh):
        import oracle as O

        self.bvh = O.Bvh(mesh.positions, mesh.tris)

    def trace_closest(self, rays):
        return self.bvh.intersect(np.ascontiguousarray(rays, np.float32))


def reference_wls(name):
    """The renders the reference arm samples: the still itself, or for the
    batched workload one render per piece (14k gold), whose turntable frame
    follows the step index."""
    from argent_b200 import workloads as W

    if name == "serve_trace":
        # one render of each request class on the 1.0M-triangle piece, gold14k
        nu, nv = W.SERVE_PIECES[4]
        m = W.M.signet(nu=nu, nv=nv)
        out = []
        for cname, (_, w, h, spp, _) in W.SERVE_CLASSES.items():
            cam, turn = W.shot(None, W.hull(m), "hero", 100.0, 0.0, w / h)
            out.append(W.Workload(f"serve_{cname}_{w}x{h}_{spp}spp", m, W.serve_scene(m, "gold14k", turn), cam, w, h,
                                  spp, W.settings(12), 7))
        return out
    if name != "reel_batch":
        m = build_mesh(name)
        return [build_workload(name, m, OracleTracer(m))]

    pieces = {label: W.reel_piece(label) for label, _, _ in W.REEL_PIECES}
    return W.reel_batch(pieces, alloys=("gold14k",), frames=[0])


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle as O

    wls = reference_wls(args.workload)
    scenes = [O.Scene(wl.mesh, wl.desc.c) for wl in wls]
    threads = os.cpu_count() or 1
    reel = args.workload == "reel_batch"
    turn = {}
    if reel:
        from argent_b200 import workloads as W

        for wl in wls:
            _, turn[wl.name] = W.turntable_camera(W.hull(wl.mesh), "hero", 100.0, 0.0, wl.width / wl.height)

    def band(k, rows):
        for wl, sc in zip(wls, scenes):
            if reel:
                sc.set_turntable(W.reel_frame_turn(turn[wl.name], k % W.REEL_FRAMES))
            for y0, y1 in spread_bands(wl.height, rows):
                sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed, rows=(y0, y1),
                               threads=threads, want_xyz=False)

    t0 = time.perf_counter()
    band(0, 1)
    dt = time.perf_counter() - t0
    rows = int(max(1, min(wls[0].height // 8, args.ref_step_seconds / max(dt, 1e-3))))
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        band(i, rows)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    per = sum(wl.width * rows * 8 * wl.spp for wl in wls)
    value = per * len(times) / sum(times)
    wl = wls[0]
    what = (f"{len(wls)} renders (one per piece, 14k gold, turntable frame = step)" if reel else "the frame")
    if args.workload == "serve_trace":
        what = f"{len(wls)} renders (one per request class, 1.0M-triangle piece, 14k gold)"
    sample = (f"8 bands of {rows} rows spread down {what} (rows {describe_bands(spread_bands(wl.height, rows))}), "
              f"{wl.width} wide at {wl.spp} spp ({per} path-samples per step)")
    cfg = {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
           "triangles": int(wl.mesh.num_tris), "max_depth": int(wl.settings.max_depth),
           "parallelism": "cpu-threads"}
    if args.workload == "serve_trace":
        cfg["workload"] = f"serve_trace_{args.serve_rate:g}rps_{args.serve_seconds:g}s"
    if reel:
        cfg["workload"] = (f"reel_batch_{len(W.REEL_PIECES) * len(W.REEL_ALLOYS)}x{W.REEL_FRAMES}frames_"
                           f"{wl.width}x{wl.height}_{wl.spp}spp")
        cfg["triangles"] = {w.extra["piece"]: int(w.mesh.num_tris) for w in wls}
    out = {
        "impl": "reference", "metric": "path-samples/s", "value": value, "unit": "path-samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_CPU, "dtype": "f32", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "path-samples/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
                         "sample": sample + "; argent's Rust path cannot be built here (no cargo), so the C++ "
                                            "restatement (oracle/) runs, OpenMP over pixels"},
        "e2e": {"value": value, "unit": "path-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ GPU arm

class StillPlan:
    """One still per step: film cleared, one render_pass."""

    def __init__(self, ctx, name, tri_test="mt"):
        from argent_b200.gpu import Film, Piece, Scene

        self.mesh = build_mesh(name)
        self.piece = Piece(ctx, self.mesh)
        self.wl = build_workload(name, self.mesh, self.piece)
        self.tri_test = tri_test
        if tri_test == "watertight":
            from argent_b200 import _native as N

            self.piece.set_triangle_test(N.TRI_WATERTIGHT)
        self.scene = Scene(ctx, self.piece, self.wl.desc)
        self.films = [Film(ctx, self.wl.width, self.wl.height)]
        self.cpu_wl = self.wl
        self.name = self.wl.name
        self.renders = 1
        self.triangles = int(self.mesh.num_tris)
        self.device_bytes = self.piece.device_bytes

    def set_spp(self, spp):
        self.wl.spp = spp

    def items(self, k, films=None, spp=None):
        wl = self.wl
        return [(self.scene, wl.camera, (films or self.films)[0], wl.settings, spp or wl.spp, wl.seed)]

    @property
    def path_samples(self):
        return self.wl.path_samples

    @property
    def pixels(self):
        return self.wl.width * self.wl.height

    def config(self):
        wl = self.wl
        out = {"workload": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
               "triangles": self.triangles, "max_depth": int(wl.settings.max_depth)}
        if self.tri_test != "mt":
            out["triangle_test"] = self.tri_test
        return out

    def accuracy_target(self, ctx):
        """(workload, scene, film holding its render at the workload's spp)."""
        return self.wl, self.scene, self.films[0]

    def tuning_target(self):
        return self.wl, self.scene, self.films[0]


class ReelPlan:
    """The batched workload: step k renders turntable frame k (mod 36) of
    every piece x alloy (3 x 4 = 12 renders) as one render_batch."""

    def __init__(self, ctx):
        from argent_b200 import workloads as W
        from argent_b200.gpu import Film, Piece, Scene

        self.W = W
        pieces = {label: W.reel_piece(label) for label, _, _ in W.REEL_PIECES}
        env = W.hdri()
        self.wls = W.reel_batch(pieces, frames=[0], env_rgb=env)
        self.gpu_pieces = {label: Piece(ctx, m) for label, m in pieces.items()}
        self.scenes = [Scene(ctx, self.gpu_pieces[wl.extra["piece"]], wl.desc) for wl in self.wls]
        self.az = {}
        for label, m in pieces.items():
            _, self.az[label] = W.turntable_camera(W.hull(m), "hero", 100.0, 0.0, 1080 / 1920)
        self.films = [Film(ctx, wl.width, wl.height) for wl in self.wls]
        self.cpu_wl = next(wl for wl in self.wls if wl.extra["piece"] == "1.1M")
        wl0 = self.wls[0]
        self.name = f"reel_batch_{len(self.wls)}x{W.REEL_FRAMES}frames_{wl0.width}x{wl0.height}_{wl0.spp}spp"
        self.renders = len(self.wls)
        self.triangles = {label: int(m.num_tris) for label, m in pieces.items()}
        self.device_bytes = sum(p.device_bytes for p in self.gpu_pieces.values())
        self.spp = wl0.spp

    def set_spp(self, spp):
        self.spp = spp

    def items(self, k, films=None, spp=None):
        frame = k % self.W.REEL_FRAMES
        out = []
        for wl, sc, f in zip(self.wls, self.scenes, films or self.films):
            sc.set_turntable(self.W.reel_frame_turn(self.az[wl.extra["piece"]], frame))
            out.append((sc, wl.camera, f, wl.settings, spp or self.spp, wl.seed))
        return out

    @property
    def path_samples(self):
        return sum(wl.width * wl.height for wl in self.wls) * self.spp

    @property
    def pixels(self):
        return sum(wl.width * wl.height for wl in self.wls)

    def config(self):
        wl = self.wls[0]
        return {"workload": self.name, "width": wl.width, "height": wl.height, "spp": self.spp,
                "triangles": self.triangles, "max_depth": int(wl.settings.max_depth),
                "renders_per_step": self.renders, "alloys": list(self.W.REEL_ALLOYS),
                "env": "2048x1024 synthetic HDRI + noir panels (env_pick 0.5)",
                "subset": f"each step is one turntable frame of all {self.renders} piece x alloy renders; "
                          f"steps walk the {self.W.REEL_FRAMES} frames"}

    def tuning_target(self):
        """The 1.1M-triangle render: the batch's middle piece."""
        i = self.wls.index(self.cpu_wl)
        return self.wls[i], self.scenes[i], self.films[i]

    def accuracy_target(self, ctx):
        """The 1.1M-triangle render of turntable frame 0, rendered afresh."""
        run_plan(ctx, self, 0)
        i = self.wls.index(self.cpu_wl)
        return self.wls[i], self.scenes[i], self.films[i]


def run_plan(ctx, plan, k, films=None, spp=None):
    from argent_b200.gpu import render_batch, render_pass

    items = plan.items(k, films, spp)
    for it in items:
        it[2].clear()
    if len(items) == 1:
        render_pass(ctx, *items[0])
    else:
        render_batch(ctx, items)


ORACLE_SPP = 65536
ORACLE_ROWS = 4  # rows per band; 8 bands spread down the frame
CONVERGE_SPP = (1024, 4096, 16384)


def rel_rmse(img, ref):
    """sqrt(sum (I - O)^2) / sqrt(sum O^2) per XYZ channel."""
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    return [float(v) for v in np.sqrt(((img - ref) ** 2).sum(0)) / np.sqrt((ref ** 2).sum(0))]


def render_bands(ctx, wl, scene, bands, spp, seed, flags):
    """The frame's rows [y0, y1) of each band, rendered through band cameras
    in one render_batch; returns the bands' XYZ stacked row-wise."""
    from argent_b200 import workloads as W
    from argent_b200.gpu import Film, render_batch

    films = [Film(ctx, wl.width, y1 - y0, flags) for y0, y1 in bands]
    render_batch(ctx, [(scene, W.band_camera(wl.camera, wl.height, y0, y1), f, wl.settings, spp, seed)
                       for (y0, y1), f in zip(bands, films)])
    out = np.concatenate([f.xyz() for f in films], 0)
    for f in films:
        f.close()
    return out


def accuracy(ctx, plan, cpu_scene, threads, gpu_rate=None, cpu_rate=None):
    """Error against the FP64 oracle: an FP64-accumulated 65,536-spp render
    (on the device, through band cameras, independent seed) of 8 bands of
    ORACLE_ROWS rows spread down the frame, scored by relRMSE per XYZ channel
    for the GPU render of the timed steps and, when `cpu_scene` is given,
    for argent's algorithm (the CPU restatement) at the same spp on the same
    rows.  Then the GPU renders the same bands at CONVERGE_SPP samples: the
    first spp whose error is at most 1 % in every channel, and the frame time
    that spp takes on the GPU and on the CPU at their measured rates."""
    from argent_b200 import _native as N

    wl, scene, film = plan.accuracy_target(ctx)
    bands = spread_bands(wl.height, ORACLE_ROWS)
    full = film.xyz()
    gpu = np.concatenate([full[y0:y1] for y0, y1 in bands], 0)
    t0 = time.perf_counter()
    o = render_bands(ctx, wl, scene, bands, ORACLE_SPP, wl.seed ^ 0x5BD1E995, N.FILM_FP64)
    dt = time.perf_counter() - t0
    out = {"oracle": f"{wl.name}: rows {describe_bands(bands)}, FP64 film, {ORACLE_SPP} spp on the device, "
                     f"independent seed ({dt:.1f} s)",
           "spp": wl.spp, "gpu_relrmse_xyz": rel_rmse(gpu, o)}
    if cpu_scene is not None:
        parts = []
        for y0, y1 in bands:
            _, _, _, xyz = cpu_scene.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed,
                                                 rows=(y0, y1), threads=threads)
            parts.append(xyz[y0:y1] / wl.spp)
        cpu = np.concatenate(parts, 0)
        out["cpu_relrmse_xyz"] = rel_rmse(cpu, o)
        out["gpu_vs_cpu_relrmse_xyz"] = rel_rmse(gpu, cpu)
    # Convergence toward the oracle.  The oracle's own noise is the error
    # at 256 spp scaled by sqrt(256 / 65536); it adds in quadrature.
    curve = [[wl.spp, max(out["gpu_relrmse_xyz"])]]
    for spp in CONVERGE_SPP:
        if spp <= wl.spp:
            continue
        g = render_bands(ctx, wl, scene, bands, spp, wl.seed, N.FILM_KAHAN)
        curve.append([spp, max(rel_rmse(g, o))])
    reach = next((spp for spp, e in curve if e <= 0.01), None)
    e0 = curve[0][1]
    law = wl.spp * (e0 / 0.01) ** 2  # spp where an unbiased estimate's error falls to 1 % (1/sqrt(spp))
    px = wl.width * wl.height
    out["to_1pct"] = {
        "curve_spp_max_relrmse": curve,
        "first_measured_spp_at_or_below_1pct": reach,
        "spp_by_inverse_sqrt_law": law,
        "oracle_noise_relrmse": e0 * (wl.spp / ORACLE_SPP) ** 0.5,
        "gpu_seconds_per_frame": (law * px / gpu_rate) if gpu_rate else None,
        "cpu_seconds_per_frame": (law * px / cpu_rate) if cpu_rate else None,
        "note": "frame time at the 1 % spp from the measured path-samples/s of each side",
    }
    return out


def tune_wanted(args):
    """Launch tuning (argent_autotune, cached per size class by
    argent_b200.tuning): on by default for the batched and served workloads,
    whose contexts run many kinds of render; --tune / --no-tune override."""
    if args.no_tune:
        return False
    return args.tune or args.workload in ("reel_batch", "serve_trace")


def apply_tuning(ctx, scene, wl, count, keep_shape):
    """Applies the cached tuning of `wl`'s size class (searching and caching
    it on a miss).  keep_shape keeps the context's lanes and wave size (the
    serve context chooses those for latency) and takes only the grids."""
    from argent_b200 import tuning as T

    shape = ctx.config()
    t0 = time.perf_counter()
    key, t, cached = T.tuned(ctx, scene, wl.camera, wl.settings, wl.width, wl.height, count)
    if keep_shape:
        t = dict(t, lanes=shape[0], wave_paths=shape[1])
        ctx.set_tuning(t)
    return {"size_class": key, "tuning": ctx.tuning(), "from_cache": cached,
            "search_s": round(time.perf_counter() - t0, 1), "render": f"{wl.width}x{wl.height}x{count}spp"}


def run_gpu(args, world, rank, device):
    import torch

    from argent_b200 import _native as N
    from argent_b200.gpu import Context, Film

    torch.cuda.set_device(device)
    ctx = Context(device, wave_paths=args.wave_paths or STILL_WAVE_PATHS, lanes=args.lanes)
    plan = ReelPlan(ctx) if args.workload == "reel_batch" else StillPlan(ctx, args.workload, args.tri_test)
    if args.share_rays:
        ctx.set_ray_sharing(True)
    if args.spp:
        plan.set_spp(args.spp)  # profiling runs only: the bench line uses the workload's spp
    stream = torch.cuda.ExternalStream(ctx.stream)
    tune_info = None
    if tune_wanted(args):
        wl, scene, _ = plan.tuning_target()
        tune_info = apply_tuning(ctx, scene, wl, wl.spp, keep_shape=False)

    for i in range(args.warmup):
        run_plan(ctx, plan, i)
    ctx.sync()

    # Instrumented pass (not timed): traversal visits per ray, rays per sample.
    cfilms = [Film(ctx, f.width, f.height) for f in plan.films]
    ctx.set_counting(True)
    run_plan(ctx, plan, 0, cfilms, 1)
    counts = ctx.traversal_counts()
    bounce_act, bounce_sh = ctx.bounce_counts()
    hist = ctx.traversal_histogram()
    child_hits = ctx.child_hit_histogram()
    ctx.set_counting(False)
    for f in cfilms:
        f.close()
    px = plan.pixels

    # Timed region (device time, CUDA events on the library stream).
    barrier(world, device)
    torch.cuda.synchronize()
    ctx.sync()
    clocks = Clocks(smi_index(device))
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    tw0 = time.perf_counter()
    e0.record(stream)
    for i in range(args.steps):
        run_plan(ctx, plan, args.warmup + i)
    e1.record(stream)
    e1.synchronize()
    wall_ms = 1e3 * (time.perf_counter() - tw0)
    ctx.sync()
    launches = ctx.kernel_launches - launches0
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, device)
    barrier(world, device)
    samples_per_step = plan.path_samples
    value = whole_job_rate(world, samples_per_step * args.steps, ms_max / 1000.0)

    # Roofline leg (not timed into `value`): one step on ONE lane with CUDA
    # events around every launch.  On one lane each kernel runs alone on the
    # device (the timed steps overlap eight lanes' kernels, so event pairs
    # there bracket other lanes' work too); the per-kernel totals then give
    # each kernel's own average launch time and its share of serialised
    # device time, comparable with the ncu launch list.
    lanes_cfg, wave_cfg = ctx.config()
    ctx.set_config(1, wave_cfg)
    run_plan(ctx, plan, 0)  # lane 0's buffers and graphs warm
    ctx.sync()
    ctx.set_profiling(True)
    run_plan(ctx, plan, 0)
    ctx.sync()
    kt = ctx.kernel_times()
    ctx.set_profiling(False)
    ctx.set_config(lanes_cfg, wave_cfg)
    # "shade" is the sum of the per-class "shade_*" entries
    serial_total = sum(v[0] for k, v in kt.items() if not k.startswith("shade_")) or 1.0

    # Dominant kernel: the single kernel with the largest share of serialised
    # device time (closest-hit traversal here; "shade" totals the five
    # per-class shading kernels, each of which is smaller).
    dom = max(("intersect", "shadow", "raygen", "film"), key=lambda k: kt[k][0])
    dom_ms, dom_n = kt[dom]
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
    # The same traversal in argent's layout (128 B Node4, 48 B Tri); argent's
    # 4-wide tree visits more nodes, so this understates its bytes.
    per_sample_ref = {
        "intersect": (counts["closest_nodes"] * 128 + counts["closest_tris"] * 48) / px + rays_c * (32 + 16 + 16 + 4),
        "shadow": (counts["any_nodes"] * 128 + counts["any_tris"] * 48) / px + rays_a * (48 + 16 + 16)}
    per_sample["film"] = 64.0 + 12.0 * 3 / max(plan.config()["spp"], 1)
    alg_bytes_step = per_sample[dom] * samples_per_step  # one step = the roofline leg's work
    achieved = alg_bytes_step / (dom_ms / 1000.0) / 1e9  # GB/s over the kernel's own launch time
    peak, peak_kind = peaks()
    # DRAM and L2 traffic per launch: bytes per ray from the committed ncu
    # capture of this kernel (profiles/ncu_traffic.json, which names its
    # command) times this run's rays per launch of the roofline leg.
    traffic, issue, l2 = None, None, None
    tr = ncu_traffic()
    if tr and tr.get("kernel") == f"k_{dom}" and tr.get("workload") == plan.name and dom in ("intersect", "shadow"):
        rays_step = (rays_c if dom == "intersect" else rays_a) * samples_per_step
        traffic = tr["dram_bytes_per_ray"] * rays_step / max(dom_n, 1)
        issue = tr.get("issue_active_pct")
        if tr.get("l2_bytes_per_ray"):
            l2_launch = tr["l2_bytes_per_ray"] * rays_step / max(dom_n, 1)
            l2 = {"bytes_per_launch": l2_launch, "gbs": l2_launch / (dom_ms / max(dom_n, 1) / 1000.0) / 1e9,
                  "hit_rate_pct": tr.get("l2_hit_rate_pct")}

    # The batched workload's renders one render_pass at a time (the plain
    # single-render path), device-timed like the batch, for comparison.
    plain = None
    if plan.renders > 1 and args.steps > 0:
        from argent_b200.gpu import render_pass

        # (a) device time of the same renders issued one render_pass each;
        # (b) end to end as argent's render_reel loop runs them
        # (jobs.rs:689-707): each frame's render_image returns its image
        # before the next frame starts, so every render is followed by its
        # film read to host memory.  (b) is compared with the batch's e2e.
        barrier(world, device)
        ctx.sync()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for i in range(args.steps):
            for it in plan.items(args.warmup + i):
                it[2].clear()
                render_pass(ctx, *it)
        p1.record(stream)
        p1.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1), world, device)
        fp = ctypes.POINTER(ctypes.c_float)
        rbuf = [tuple(np.zeros((f.height, f.width, 3), np.float32) for _ in range(3)) for f in plan.films]
        steps_e2e = max(args.e2e_steps, 1)
        barrier(world, device)
        ctx.sync()
        t0 = time.perf_counter()
        for i in range(steps_e2e):
            for it, (c, a, nrm) in zip(plan.items(i), rbuf):
                it[2].clear()
                render_pass(ctx, *it)
                ctx.check(ctx.lib.argent_film_read(it[2].h, c.ctypes.data_as(fp), a.ctypes.data_as(fp),
                                                   nrm.ctypes.data_as(fp)))
        pe = max_over_ranks(time.perf_counter() - t0, world, device)
        plain = {"value": world * samples_per_step * args.steps / (pms / 1000.0), "unit": "path-samples/s",
                 "ms_per_step": pms / args.steps,
                 "e2e": {"value": world * samples_per_step * steps_e2e / pe, "unit": "path-samples/s",
                         "ms_per_step": 1e3 * pe / steps_e2e,
                         "form": "render_reel's loop: each render's render_pass, then its film read to host, "
                                 "before the next render"},
                 "form": f"the same {plan.renders} renders per step, one render_pass each (device time)"}

    # End-to-end through the C ABI with host buffers.
    e2e_value, e2e_split = None, None
    h2d = plan.renders * (ctypes.sizeof(N.ArgentCamera) + ctypes.sizeof(N.ArgentPathSettings) + 8)
    d2h = 3 * px * 3 * 4
    if args.e2e_steps > 0:
        bufs = [tuple(np.zeros((f.height, f.width, 3), np.float32) for _ in range(3)) for f in plan.films]
        fp = ctypes.POINTER(ctypes.c_float)
        # One untimed step through the same calls, then the timed ones.
        run_plan(ctx, plan, 0)
        for f, (c, a, nrm) in zip(plan.films, bufs):
            ctx.check(ctx.lib.argent_film_read(f.h, c.ctypes.data_as(fp), a.ctypes.data_as(fp),
                                               nrm.ctypes.data_as(fp)))
        barrier(world, device)
        t_issue = t_read = 0.0
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            ta = time.perf_counter()
            run_plan(ctx, plan, i)
            tb = time.perf_counter()
            for f, (c, a, nrm) in zip(plan.films, bufs):
                ctx.check(ctx.lib.argent_film_read(f.h, c.ctypes.data_as(fp), a.ctypes.data_as(fp),
                                                   nrm.ctypes.data_as(fp)))
            t_issue += tb - ta
            t_read += time.perf_counter() - tb
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, world, device)
        e2e_value = world * samples_per_step * args.e2e_steps / dt
        # The reads alone, of films already finished.
        tr0 = time.perf_counter()
        for f, (c, a, nrm) in zip(plan.films, bufs):
            ctx.check(ctx.lib.argent_film_read(f.h, c.ctypes.data_as(fp), a.ctypes.data_as(fp),
                                               nrm.ctypes.data_as(fp)))
        e2e_split = {"issue_ms_per_step": 1e3 * t_issue / args.e2e_steps,
                     "wait_and_read_ms_per_step": 1e3 * t_read / args.e2e_steps,
                     "read_ms_per_step": 1e3 * (time.perf_counter() - tr0)}

    cpu, cpu_scene = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        wl = plan.cpu_wl
        v, bands, nthr, cpu_scene = cpu_sample(wl, seconds=args.ref_seconds, threads=os.cpu_count() or 1)
        cpu = {"value": v, "unit": "path-samples/s", "cores": nthr, "kind": "port", "cpu": cpu_model(),
               "sample": f"{wl.name}: 8 bands spread down the frame (rows {describe_bands(bands)}) at {wl.spp} spp; "
                         f"argent's algorithm as restated in oracle/ (Rust reference not buildable here), "
                         f"OpenMP over pixels on every host thread"}
    acc = None
    if rank == 0 and not args.no_oracle:
        acc = accuracy(ctx, plan, cpu_scene, os.cpu_count() or 1, gpu_rate=value / world,
                       cpu_rate=cpu["value"] if cpu else None)

    if rank == 0:
        cfg = plan.config()
        cfg.update({"parallelism": f"replicas{world}", "l2": "inputs larger than L2 (path state "
                    f"{ctx_wave_mb(args)} MB per wave x {args.lanes or 8} lanes + BVH/triangles "
                    f"{plan.device_bytes / 1e6:.0f} MB)",
                    "context": {"lanes": ctx.config()[0], "wave_paths": ctx.config()[1]},
                    "tuning": tune_info,
                    "ray_sharing": bool(args.share_rays),
                    "vs_baseline_ref": "README.md:5-6 ~17.7M path-samples/s on 32 CPU cores"})
        out = {
            "metric": "path-samples/s", "value": value, "unit": "path-samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "wall_ms_per_step": wall_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_CPU, "dtype": "f32",
            "data": f"synthetic ({DATA[args.workload]})",
            "config": cfg,
            "clocks": ck,
            "e2e": {"value": e2e_value, "unit": "path-samples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "split": e2e_split},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": f"k_{dom}",
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "alg_bytes_per_path_sample": per_sample[dom],
                         "alg_bytes_per_path_sample_argent_layout": per_sample_ref.get(dom),
                         "issue_active_pct": issue, "l2": l2,
                         "launches": dom_n, "avg_launch_ms": dom_ms / max(dom_n, 1),
                         "timing": "one step on one lane, CUDA events around each launch (each kernel alone "
                                   "on the device)"},
            "kernel_ms_alone": {k: round(v[0], 3) for k, v in kt.items()},
            "kernel_share_alone": {k: round(v[0] / serial_total, 4) for k, v in kt.items()},
            "traversal_per_path_sample": {k: v / px for k, v in counts.items()},
            "traversal_nodes_per_ray_histogram": hist,
            "traversal_children_entered_per_node_visit": child_hits,
            "rays_per_path_sample_by_bounce": {"closest": [round(x / px, 4) for x in bounce_act],
                                               "shadow": [round(x / px, 4) for x in bounce_sh]},
            "cpu_baseline": cpu,
            "plain_form": plain,
            "error_vs_fp64_oracle": acc,
        }
        return out
    return None


def run_serve(args, world, rank, device):
    """Served requests: a thread submits the Poisson trace on the wall
    clock while this thread steps the scheduler and reads finished films to
    host memory.  value = path-samples served / (last completion - first
    arrival); latency = completion - submission per request class."""
    import torch

    from argent_b200 import _native as N
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Piece, Scene, Serve

    torch.cuda.set_device(device)
    ctx = Context(device, wave_paths=args.wave_paths or SERVE_WAVE_PATHS, lanes=args.lanes)
    if getattr(args, "share_rays", False):
        ctx.set_ray_sharing(True)
    meshes = W.serve_pieces()
    pieces = [Piece(ctx, m) for m in meshes]
    cams, scenes = {}, {}
    for i, m in enumerate(meshes):
        pts = W.hull(m)
        for cname, (_, w, h, _, _) in W.SERVE_CLASSES.items():
            cams[(i, cname)], turn = W.shot(None, pts, "hero", 100.0, 0.0, w / h)
        for j, alloy in enumerate(W.SERVE_ALLOYS):
            scenes[(i, j)] = Scene(ctx, pieces[i], W.serve_scene(m, alloy, turn))
    ps = W.settings(12)
    rate = args.serve_rate
    trace = W.serve_trace(rate, args.serve_seconds)
    tune_info = None
    if tune_wanted(args):
        # A listing of the 1.0M-triangle piece at 16 spp: about one step's
        # worth of work (2^26 path-samples).
        _, lw, lh, _, _ = W.SERVE_CLASSES["listing"]
        twl = W.Workload("serve_tuning", meshes[4], None, cams[(4, "listing")], lw, lh, 16, ps, 7)
        tune_info = apply_tuning(ctx, scenes[(4, 1)], twl, 16, keep_shape=True)
    srv = Serve(ctx, film_budget=32 << 30, max_active=64, step_path_samples=args.serve_step,
                step_path_samples_max=args.serve_step_max, aging_ms=args.serve_aging_ms,
                overlap=not args.serve_no_overlap, max_pending=args.serve_max_pending,
                max_pending_path_samples=int(args.serve_max_pending_work * W.mean_request_path_samples()))

    def submit(cname, i, j):
        _, w, h, spp, prio = W.SERVE_CLASSES[cname]
        return srv.submit(scenes[(i, j)], cams[(i, cname)], ps, w, h, spp, 7, prio)

    # Warm-up before the trace: one request of each class (path state and
    # films reach their full sizes), then previews.
    for k, cname in enumerate(list(W.SERVE_CLASSES) + ["preview"] * args.warmup):
        t = submit(cname, k % len(meshes), k % len(W.SERVE_ALLOYS))
        srv.run()
        srv.read(t)

    launches0 = ctx.kernel_launches
    steps0 = srv.stats()
    tickets, reqs = {}, {}
    done = threading.Event()
    t_origin = srv.now()

    rejected = {c: 0 for c in W.SERVE_CLASSES}

    def driver():
        for (ta, cname, i, j) in trace:
            dt = t_origin + ta - srv.now()
            if dt > 0:
                time.sleep(dt)
            try:
                t = submit(cname, i, j)
            except N.ArgentError as e:
                if e.code != N.E_BUSY:
                    raise
                rejected[cname] += 1
                continue
            reqs[t] = (i, j)
            tickets[t] = cname
        done.set()

    clocks = Clocks(smi_index(device))
    clocks.start()
    th = threading.Thread(target=driver)
    th.start()
    lat = {c: [] for c in W.SERVE_CLASSES}
    kept = {}  # class -> ((mesh, alloy), colour film) of its first finished request
    finished = set()
    d2h = 0
    t_last = t_origin
    while True:
        pending = srv.step()
        for t, cname in list(tickets.items()):
            if t in finished:
                continue
            st = srv.poll(t)
            if st.state == 2:  # done
                lat[cname].append(st.t_done - st.t_submit)
                t_last = max(t_last, st.t_done)
                c, a, n = srv.read(t)
                d2h += c.nbytes + a.nbytes + n.nbytes
                finished.add(t)
                if cname not in kept:
                    kept[cname] = (reqs[t], c)
        if done.is_set() and pending == 0 and len(finished) == len(tickets):
            break
        if pending == 0:
            time.sleep(0.001)
    th.join()
    ck = clocks.stop()
    st = srv.stats()
    served = st["path_samples"] - steps0["path_samples"]
    wall = t_last - t_origin
    value = served / wall
    offered = rate * W.mean_request_path_samples()
    launches = ctx.kernel_launches - launches0

    def pct(v, q):
        return float(np.percentile(v, q)) if v else None

    # The same stream through argent's own discipline (one job at a time).
    plain = None
    if not args.no_plain:
        pv, plat, prej = serve_plain(ctx, trace, scenes, cams, ps, args.serve_max_pending)
        plain = {"value": pv, "unit": "path-samples/s",
                 "latency_s": {c: {"n": len(v), "p50": pct(v, 50), "p99": pct(v, 99), "max": max(v) if v else None}
                               for c, v in list(plat.items()) + [("all", sum(plat.values(), []))]},
                 "rejected": prej,
                 "discipline": "one job at a time in arrival order, render_pass in chunks of 2..64 spp sized to "
                               "about 1.5 s (serve/queue.rs:599-617), film read to host; a job arriving while "
                               f"{max(args.serve_max_pending - 1, 0)} wait is refused (queue.rs:364-366)"}

    # Error of each class's first served film against the FP64 oracle (an
    # FP64-accumulated 65,536-spp render of ORACLE_ROWS rows at mid-frame
    # through a band camera, independent seed); serve hands back camera RGB,
    # so the channels are camera RGB.
    acc = {}
    if not args.no_oracle:
        from argent_b200.gpu import Film, render_pass

        for cname, ((i, j), c) in kept.items():
            _, w, h, spp, _ = W.SERVE_CLASSES[cname]
            y0, y1 = h // 2, h // 2 + ORACLE_ROWS
            ref = Film(ctx, w, y1 - y0, N.FILM_FP64)
            render_pass(ctx, scenes[(i, j)], W.band_camera(cams[(i, cname)], h, y0, y1), ref, ps, ORACLE_SPP,
                        7 ^ 0x5BD1E995)
            o, _, _ = ref.read()
            ref.close()
            acc[cname] = {"spp": spp, "mesh": i, "alloy": W.SERVE_ALLOYS[j],
                          "relrmse_camera_rgb": rel_rmse(c[y0:y1], o)}

    if rank == 0:
        out = {
            "metric": "path-samples/s", "value": value, "unit": "path-samples/s", "n_gpus": world,
            "steps": int(st["steps"] - steps0["steps"]), "warmup": args.warmup,
            "ms_per_step": 1000.0 * wall / max(1, st["steps"] - steps0["steps"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": f"synthetic ({DATA['serve_trace']})",
            "config": {"workload": f"serve_trace_{rate:g}rps_{args.serve_seconds:g}s", "requests": len(trace),
                       "classes": {k: list(v[1:]) for k, v in W.SERVE_CLASSES.items()},
                       "pieces_triangles": [int(m.num_tris) for m in meshes], "alloys": list(W.SERVE_ALLOYS),
                       "offered_path_samples_per_s": offered, "step_path_samples": args.serve_step,
                       "step_path_samples_max": args.serve_step_max or 2 * args.serve_step,
                       "aging_ms": args.serve_aging_ms or 250, "overlap": not args.serve_no_overlap,
                       "ray_sharing": bool(getattr(args, "share_rays", False)),
                       "max_pending": args.serve_max_pending,
                       "max_pending_path_samples": int(args.serve_max_pending_work * W.mean_request_path_samples()),
                       "tuning": tune_info,
                       "parallelism": f"replicas{world}",
                       "timing": "wall clock of the serve loop (latency is a wall-clock quantity); each step "
                                 "synchronises its batch"},
            "latency_s": {c: {"n": len(v), "p50": pct(v, 50), "p99": pct(v, 99), "max": max(v) if v else None}
                          for c, v in list(lat.items()) + [("all", sum(lat.values(), []))]},
            "rejected": rejected,
            "clocks": ck,
            "e2e": {"value": value, "unit": "path-samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": d2h / max(1, len(finished)), "note": "per request: films read to host"},
            "gpu_launches": int(launches),
            "plain_form": plain,
            "error_vs_fp64_oracle": {"oracle": f"rows h/2..h/2+{ORACLE_ROWS} of each class's first served "
                                               f"request, FP64 film, {ORACLE_SPP} spp on the device",
                                     "classes": acc} if acc else None,
        }
        return out
    return None


def serve_plain(ctx, trace, scenes, cams, ps, max_pending=0):
    """argent's own serve discipline on the GPU, for comparison with the
    continuous-batching scheduler on the same request stream: one job at a
    time in arrival order, each rendered by render_pass in chunks that start
    at 2 spp and adapt to about 1.5 s each (capped at 64 spp), then read to
    host memory (serve/queue.rs:599-617); with max_pending, a job that
    arrives while max_pending - 1 wait is refused (queue.rs:364-366).
    Returns (path-samples/s, {class: latencies}, {class: refused})."""
    import queue

    from argent_b200 import workloads as W
    from argent_b200.gpu import Film, render_pass

    q = queue.Queue()
    t0 = time.perf_counter()
    rejected = {c: 0 for c in W.SERVE_CLASSES}

    def driver():
        for (ta, cname, i, j) in trace:
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            if max_pending and q.qsize() >= max_pending - 1:
                rejected[cname] += 1
                continue
            q.put((time.perf_counter(), cname, i, j))
        q.put(None)

    th = threading.Thread(target=driver)
    th.start()
    lat = {c: [] for c in W.SERVE_CLASSES}
    films = {}
    served, t_last = 0, t0
    while True:
        item = q.get()
        if item is None:
            break
        t_sub, cname, i, j = item
        _, w, h, spp, _ = W.SERVE_CLASSES[cname]
        f = films.get((w, h))
        if f is None:
            f = films[(w, h)] = Film(ctx, w, h)
        f.clear()
        done, chunk = 0, 2
        while done < spp:
            n = min(chunk, spp - done)
            t = time.perf_counter()
            render_pass(ctx, scenes[(i, j)], cams[(i, cname)], f, ps, n, 7)
            ctx.sync()
            per = (time.perf_counter() - t) / n
            done += n
            chunk = int(min(max(1.5 / max(per, 1e-4), 1), 64))
        f.read()
        t_last = time.perf_counter()
        lat[cname].append(t_last - t_sub)
        served += w * h * spp
    th.join()
    for f in films.values():
        f.close()
    return served / (t_last - t0), lat, rejected


PATH_STATE_BYTES = 244  # per path slot per lane
STILL_WAVE_PATHS = 1 << 25  # the stills' and batch's context: 2^25-path waves (8 lanes hold 65 GB of path state)
SERVE_WAVE_PATHS = 1 << 23  # the serve context: 2^23-path waves


def ctx_wave_mb(args):
    return PATH_STATE_BYTES * (args.wave_paths or STILL_WAVE_PATHS) // 10 ** 6


def reel_compare(args, device, steps=4):
    """The batched form against the plain single-render path on one frame
    of the batched workload (12 renders: 3 pieces x 4 alloys), all end to
    end with host buffers: the batch is one render_batch and then every
    film's read; the plain path is render_reel's loop (jobs.rs:689-707), one
    render_pass and its film read per render.  A third leg runs the batch
    with ray sharing (argent_ctx_set_ray_sharing): the four alloys of a piece
    trace their common rays once; its films are compared with the unshared
    batch's."""
    from argent_b200.gpu import Context, render_pass

    ctx = Context(device, wave_paths=STILL_WAVE_PATHS)
    plan = ReelPlan(ctx)
    fp = ctypes.POINTER(ctypes.c_float)
    names = ("batched", "batched_shared_rays", "plain")
    bufs = {n: [tuple(np.zeros((f.height, f.width, 3), np.float32) for _ in range(3)) for f in plan.films]
            for n in names}

    def read(f, b):
        c, a, n = b
        ctx.check(ctx.lib.argent_film_read(f.h, c.ctypes.data_as(fp), a.ctypes.data_as(fp), n.ctypes.data_as(fp)))

    def batched(k, name="batched"):
        run_plan(ctx, plan, k)
        for f, b in zip(plan.films, bufs[name]):
            read(f, b)

    def batched_shared(k):
        ctx.set_ray_sharing(True)
        try:
            batched(k, "batched_shared_rays")
        finally:
            ctx.set_ray_sharing(False)

    def plain(k):
        for it, b in zip(plan.items(k), bufs["plain"]):
            it[2].clear()
            render_pass(ctx, *it)
            read(it[2], b)

    forms = tuple(zip(names, (batched, batched_shared, plain)))
    for _, fn in forms:
        fn(0)  # warm-up (graphs captured, buffers grown)
    ctx.sync()
    # The forms alternate frame by frame, so a drift of the device's speed
    # during the leg falls on all of them.
    spent = {name: 0.0 for name, _ in forms}
    for k in range(steps):
        for name, fn in forms:
            t0 = time.perf_counter()
            fn(1 + k)
            spent[name] += time.perf_counter() - t0
    out = {name: {"e2e_path_samples_per_s": plan.path_samples * steps / dt, "s_per_frame": dt / steps}
           for name, dt in spent.items()}
    # The last frame's films: shared against unshared (the same samples,
    # grouped into other waves, so equal to float rounding of the sums).
    worst = 0.0
    for (c1, _, _), (c2, _, _) in zip(bufs["batched_shared_rays"], bufs["batched"]):
        worst = max(worst, float(np.abs(c1 - c2).max() / max(float(np.abs(c2).max()), 1e-30)))
    out["batched_shared_rays"]["max_abs_diff_vs_batched_over_max"] = worst
    out["workload"] = plan.name
    out["renders_per_frame"] = plan.renders
    out["timing"] = (f"wall clock, {steps} turntable frames each, the forms alternating frame by frame, "
                     f"films read to host memory")
    return out


def form_comparisons(args, device):
    """Short legs comparing the batched and served forms with the plain
    single-render path, carried in the default line:
    the batched reel against the plain single-render path, and a served
    Poisson trace against argent's one-job-at-a-time queue at a rate near
    the device's capacity."""
    out = {"reel": reel_compare(args, device, args.extras_reel_frames)}
    import gc

    gc.collect()
    sargs = argparse.Namespace(**vars(args))
    sargs.serve_rate = args.extras_serve_rate
    sargs.serve_seconds = args.extras_serve_seconds
    sargs.no_oracle = True
    sargs.wave_paths = 0
    sargs.warmup = 3
    srv = run_serve(sargs, 1, 0, device)
    keep = ("value", "latency_s", "rejected", "plain_form", "config")
    out["serve"] = {k: srv[k] for k in keep if k in srv}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="argent", choices=["argent", "reference"])
    ap.add_argument("--workload", default="signet_still", choices=list(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-seconds", type=float, default=8.0, help="CPU work of the cpu_baseline sample (GPU arm)")
    ap.add_argument("--ref-step-seconds", type=float, default=3.0,
                    help="--impl reference: CPU work of each step's sample (warm-up and timed steps alike)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-oracle", action="store_true", help="skip the FP64 65,536-spp error measurement")
    ap.add_argument("--no-plain", action="store_true", help="serve_trace: skip the one-job-at-a-time comparison")
    ap.add_argument("--spp", type=int, default=0, help="override spp (short profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="signet_still: skip the short batched-vs-plain reel and served-vs-plain trace legs")
    ap.add_argument("--extras-reel-frames", type=int, default=4)
    ap.add_argument("--extras-serve-rate", type=float, default=8.0)
    ap.add_argument("--extras-serve-seconds", type=float, default=30.0)
    ap.add_argument("--tune", action="store_true", help="apply (search and cache) a launch tuning")
    ap.add_argument("--no-tune", action="store_true", help="no launch tuning, also for reel and serve")
    ap.add_argument("--share-rays", action="store_true",
                    help="batches trace the rays their renders have in common once (argent_ctx_set_ray_sharing)")
    ap.add_argument("--tri-test", default="mt", choices=["mt", "watertight"],
                    help="stills: argent's Moller-Trumbore (default, bit-exact) or the watertight test")
    ap.add_argument("--lanes", type=int, default=0, help="concurrent waves (0 = the library default)")
    ap.add_argument("--wave-paths", type=int, default=0,
                    help="path slots per wave (0 = 2^25 for stills and batches, 2^23 for the serve trace)")
    ap.add_argument("--serve-rate", type=float, default=4.0, help="serve_trace: requests per second")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serve_trace: trace length")
    ap.add_argument("--serve-step", type=int, default=1 << 26, help="serve_trace: least path-samples per step")
    ap.add_argument("--serve-step-max", type=int, default=0, help="serve_trace: most path-samples per step")
    ap.add_argument("--serve-aging-ms", type=int, default=0, help="serve_trace: aging period (0 = default)")
    ap.add_argument("--serve-no-overlap", action="store_true", help="serve_trace: wait for each step's batch")
    ap.add_argument("--serve-max-pending", type=int, default=25,
                    help="serve_trace: requests waiting or rendering at most, both forms (argent: 24 waiting + 1)")
    ap.add_argument("--serve-max-pending-work", type=float, default=25.0,
                    help="serve_trace, served form: pending work bound in mean requests' path-samples "
                         "(0 = none); 25 is the work argent's 25-job bound holds on average")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU only: rank 0 measures, the other ranks have nothing to do.
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), 0)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.workload == "serve_trace":
            out = run_serve(args, world, rank, local)
        else:
            out = run_gpu(args, world, rank, local)
        if out is not None and rank == 0:
            if args.workload == "signet_still" and world == 1 and not args.no_extras:
                import gc

                gc.collect()  # the still's context and its path state go before the extras' contexts
                try:
                    out["forms"] = form_comparisons(args, local)
                except Exception as e:  # the measured line stands; the legs report what stopped them
                    out["forms"] = {"error": f"{type(e).__name__}: {e}"}
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as td

            td.destroy_process_group()


if __name__ == "__main__":
    main()
