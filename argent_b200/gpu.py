"""Python handles over the C ABI (include/argent_gpu.h).

These mirror argent's own objects: `Piece` (scene.rs:10-38), `Scene`
(scene.rs:47-110), `Film` (render.rs:12-63) and `render_pass`
(render.rs:67-115), so callers and tests read like argent's.
"""

import ctypes

import numpy as np

from . import _native as N


def _p(a, t=ctypes.c_void_p):
    if a is None:
        return None
    return a.ctypes.data_as(t)


class Context:
    """One device, one stream (argent_ctx_create)."""

    def __init__(self, device=0, wave_paths=0, memory_budget=0, lanes=0):
        self.lib = N.gpu()
        lim = N.ArgentLimits(wave_paths, memory_budget, lanes, 0)
        h = ctypes.c_void_p()
        N.check(self.lib.argent_ctx_create(device, ctypes.byref(lim), ctypes.byref(h)))
        self.h = h
        # Native objects made on this context (handle -> kind).  The context
        # destroys those still alive before itself: the garbage collector
        # finalises a reference cycle in any order, and a piece, scene, film
        # or serve must never outlive the context it was made on.
        self._owned = {}

    def _own(self, kind, h):
        self._owned[h.value] = kind

    def _release(self, kind, h):
        """Destroys a child's native object unless the context already has."""
        if getattr(self, "h", None) is not None and self._owned.pop(h.value, None) is not None:
            getattr(self.lib, f"argent_{kind}_destroy")(h)

    def close(self):
        if getattr(self, "h", None):
            owned = getattr(self, "_owned", {})
            for kind in ("serve", "film", "scene", "piece"):  # dependents first
                for hv, k in list(owned.items()):
                    if k == kind:
                        del owned[hv]
                        getattr(self.lib, f"argent_{kind}_destroy")(ctypes.c_void_p(hv))
            self.lib.argent_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def check(self, rc):
        return N.check(rc, self.h)

    def sync(self):
        self.check(self.lib.argent_ctx_sync(self.h))

    @property
    def kernel_launches(self):
        return int(self.lib.argent_ctx_kernel_launches(self.h))

    @property
    def stream(self):
        return self.lib.argent_ctx_stream(self.h)

    def set_profiling(self, on):
        self.check(self.lib.argent_ctx_set_profiling(self.h, 1 if on else 0))

    def kernel_times(self):
        """{class: (total_ms, launches)} since the last set_profiling."""
        ms = (ctypes.c_double * len(N.KERNEL_CLASSES))()
        n = (ctypes.c_uint64 * len(N.KERNEL_CLASSES))()
        self.check(self.lib.argent_ctx_kernel_times(self.h, ms, n))
        return {k: (ms[i], int(n[i])) for i, k in enumerate(N.KERNEL_CLASSES)}

    def autotune(self, scene, cam, settings, width, height, count):
        """argent_autotune: times the frame for each (lanes, wave size) and
        keeps the fastest.  Returns [(lanes, wave_paths, path-samples/s)]."""
        res = (N.ArgentTuneResult * 32)()
        n = ctypes.c_uint32()
        self.check(self.lib.argent_autotune(self.h, scene.h, ctypes.byref(cam), ctypes.byref(settings), width, height,
                                            count, res, 32, ctypes.byref(n)))
        return [(r.lanes, r.wave_paths, r.path_samples_per_s) for r in res[: min(n.value, 32)]]

    def config(self):
        """(lanes, wave_paths) in use."""
        lanes, wave = ctypes.c_uint32(), ctypes.c_uint64()
        self.check(self.lib.argent_ctx_config(self.h, ctypes.byref(lanes), ctypes.byref(wave)))
        return lanes.value, wave.value

    def tuning(self):
        """The launch tuning in use, as a dict (argent_ctx_tuning)."""
        t = N.ArgentTuning()
        self.check(self.lib.argent_ctx_tuning(self.h, ctypes.byref(t)))
        return {"lanes": t.lanes, "wave_paths": t.wave_paths, "trace_blocks_per_sm": t.trace_blocks_per_sm,
                "shade_blocks_per_sm": list(t.shade_blocks_per_sm)}

    def set_tuning(self, tuning):
        """argent_ctx_set_tuning from a dict as `tuning()` returns it."""
        t = N.ArgentTuning()
        t.lanes = int(tuning["lanes"])
        t.wave_paths = int(tuning["wave_paths"])
        t.trace_blocks_per_sm = int(tuning.get("trace_blocks_per_sm", 0))
        for i, v in enumerate(tuning.get("shade_blocks_per_sm", [0] * 5)):
            t.shade_blocks_per_sm[i] = int(v)
        self.check(self.lib.argent_ctx_set_tuning(self.h, ctypes.byref(t)))

    def set_config(self, lanes, wave_paths):
        """argent_ctx_set_config: lanes and wave size of the next calls."""
        self.check(self.lib.argent_ctx_set_config(self.h, int(lanes), int(wave_paths)))

    def set_counting(self, on):
        self.check(self.lib.argent_ctx_set_counting(self.h, 1 if on else 0))

    def set_graphs(self, on):
        """Capture and replay repeated renders as CUDA graphs (default on)."""
        self.check(self.lib.argent_ctx_set_graphs(self.h, 1 if on else 0))

    def set_ray_sharing(self, on):
        """Batches trace the rays their renders have in common once
        (argent_ctx_set_ray_sharing; default off)."""
        self.check(self.lib.argent_ctx_set_ray_sharing(self.h, 1 if on else 0))

    def traversal_counts(self):
        out = (ctypes.c_uint64 * 6)()
        self.check(self.lib.argent_ctx_traversal_counts(self.h, out))
        k = ["closest_rays", "closest_nodes", "closest_tris", "any_rays", "any_nodes", "any_tris"]
        return dict(zip(k, [int(x) for x in out]))

    def child_hit_histogram(self):
        """Interior node visits by children entered (0..8): {"closest": [...],
        "any": [...]} since counting was turned on."""
        out = (ctypes.c_uint64 * 18)()
        self.check(self.lib.argent_ctx_child_hit_histogram(self.h, out))
        v = [int(x) for x in out]
        return {"closest": v[0:9], "any": v[9:18]}

    def bounce_counts(self):
        """(paths entering each bounce, shadow rays queued at each bounce),
        trailing zeros dropped, since counting was turned on."""
        out = (ctypes.c_uint64 * 128)()
        self.check(self.lib.argent_ctx_bounce_counts(self.h, out))
        v = [int(x) for x in out]
        act, sh = v[:64], v[64:]
        n = max([i + 1 for i, x in enumerate(act) if x] + [0])
        return act[:n], sh[:n]

    def traversal_histogram(self):
        """Rays by node visits (bins 0, 1, 2-3, 4-7, 8-15, 16-63, 64-255,
        256+) and the largest visit count, per ray kind."""
        out = (ctypes.c_uint64 * 18)()
        self.check(self.lib.argent_ctx_traversal_histogram(self.h, out))
        v = [int(x) for x in out]
        return {"closest": v[0:8], "any": v[8:16], "closest_max": v[16], "any_max": v[17]}


class Piece:
    """`Piece::new`: mesh upload + acceleration structure build.  With
    `device_bvh` the tree is the linear BVH built on the device (faster to
    build, slower to trace; the same closest hits)."""

    def __init__(self, ctx: Context, mesh, device_bvh: bool = False):
        self.ctx = ctx
        self.mesh = mesh
        h = ctypes.c_void_p()
        fp = ctypes.POINTER(ctypes.c_float)
        upload = ctx.lib.argent_piece_upload_device_bvh if device_bvh else ctx.lib.argent_piece_upload
        ctx.check(upload(
            ctx.h, _p(mesh.positions, fp), len(mesh.positions), _p(mesh.normals, fp), _p(mesh.tris, N.c_u32_p),
            len(mesh.tris), _p(mesh.tri_material, N.c_u16_p), _p(mesh.cavity, fp), ctypes.byref(h)))
        self.h = h
        ctx._own("piece", h)

    def close(self):
        if getattr(self, "h", None):
            self.ctx._release("piece", self.h)
            self.h = None

    def __del__(self):
        self.close()

    def bounds(self):
        lo = (ctypes.c_float * 3)()
        hi = (ctypes.c_float * 3)()
        self.ctx.check(self.ctx.lib.argent_piece_bounds(self.h, lo, hi))
        return np.array(lo[:], np.float32), np.array(hi[:], np.float32)

    @property
    def device_bytes(self):
        return int(self.ctx.lib.argent_piece_device_bytes(self.h))

    def ambient_occlusion(self, normals, samples=48, distance=1.2):
        """cavity::ambient_occlusion (argent-mesh cavity.rs:96-135) on the
        device, for the mesh this piece was uploaded from."""
        m = self.mesh
        fp = ctypes.POINTER(ctypes.c_float)
        n = np.ascontiguousarray(normals, np.float32)
        out = np.zeros(len(m.positions), np.float32)
        self.ctx.check(self.ctx.lib.argent_piece_ambient_occlusion(
            self.ctx.h, self.h, _p(m.positions, fp), _p(n, fp), len(m.positions), samples, distance, _p(out, fp)))
        return out

    def patina_mask(self, settings=None):
        """cavity::patina_mask (cavity.rs:52-78) of the uploaded mesh; pass
        the result as Mesh.cavity to upload a piece with its mask."""
        m = self.mesh
        s = settings if settings is not None else N.ArgentPatinaSettings(48, 1.2, 0.4, 0.35, 3)
        fp = ctypes.POINTER(ctypes.c_float)
        out = np.zeros(len(m.positions), np.float32)
        self.ctx.check(self.ctx.lib.argent_piece_patina_mask(
            self.ctx.h, self.h, _p(m.positions, fp), _p(m.normals, fp), len(m.positions), _p(m.tris, N.c_u32_p),
            len(m.tris), ctypes.byref(s), _p(out, fp)))
        return out

    def set_triangle_test(self, test):
        """argent_piece_set_triangle_test: N.TRI_MOLLER_TRUMBORE (argent's,
        bit-exact hits; the default) or N.TRI_WATERTIGHT."""
        self.ctx.check(self.ctx.lib.argent_piece_set_triangle_test(self.ctx.h, self.h, int(test)))

    def trace_closest(self, rays: np.ndarray) -> np.ndarray:
        """rays: (n, 8) float32 [ox oy oz tmax dx dy dz pad] -> hits (n, 4)
        float32 [t u v prim-bits]."""
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((len(rays), 4), np.float32)
        self.ctx.check(self.ctx.lib.argent_trace_closest(self.ctx.h, self.h, _p(rays), len(rays), _p(hits)))
        return hits

    def trace_anyhit(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(len(rays), np.uint8)
        self.ctx.check(self.ctx.lib.argent_trace_anyhit(self.ctx.h, self.h, _p(rays), len(rays), _p(occ)))
        return occ


class Scene:
    """`Scene::new` around a piece, from an ArgentSceneDesc."""

    def __init__(self, ctx: Context, piece: Piece, desc):
        self.ctx = ctx
        self.piece = piece
        self.desc = desc  # keeps the description's arrays alive
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.argent_scene_upload(ctx.h, piece.h, ctypes.byref(desc.c), ctypes.byref(h)))
        self.h = h
        ctx._own("scene", h)

    def close(self):
        if getattr(self, "h", None):
            self.ctx._release("scene", self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_turntable(self, deg):
        self.ctx.check(self.ctx.lib.argent_scene_set_turntable(self.h, float(deg)))


class Film:
    """`Film` (render.rs:12-63): device sums, read back as averages."""

    def __init__(self, ctx: Context, width, height, flags=N.FILM_KAHAN):
        self.ctx = ctx
        self.width, self.height = width, height
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.argent_film_create(ctx.h, width, height, flags, ctypes.byref(h)))
        self.h = h
        ctx._own("film", h)

    def close(self):
        if getattr(self, "h", None):
            self.ctx._release("film", self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def samples(self):
        return int(self.ctx.lib.argent_film_samples(self.h))

    def clear(self):
        self.ctx.check(self.ctx.lib.argent_film_clear(self.h))

    def read(self):
        """(color, albedo, normal) as `Film::color/albedo/normal`, (h, w, 3)."""
        shape = (self.height, self.width, 3)
        c, a, n = np.zeros(shape, np.float32), np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.ctx.check(self.ctx.lib.argent_film_read(self.h, _p(c, fp), _p(a, fp), _p(n, fp)))
        return c, a, n

    def color(self):
        shape = (self.height, self.width, 3)
        c = np.zeros(shape, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.ctx.check(self.ctx.lib.argent_film_read(self.h, _p(c, fp), None, None))
        return c

    def denoised(self):
        """The colour denoised on the device with the film's albedo and
        normal guides (argent-post's à-trous backend)."""
        out = np.zeros((self.height, self.width, 3), np.float32)
        self.ctx.check(self.ctx.lib.argent_film_denoise(self.h, _p(out, ctypes.POINTER(ctypes.c_float))))
        return out

    def developed(self, grade=None, denoise=True):
        """8-bit sRGB (h, w, 3) of the film: render_image's denoise plus
        argent-post's develop, on the device."""
        g = grade if grade is not None else N.ArgentGrade(0.0, N.TM_AGX, N.AGX_PUNCHY, 1.0)
        out = np.zeros((self.height, self.width, 3), np.uint8)
        self.ctx.check(self.ctx.lib.argent_film_develop(self.h, ctypes.byref(g), 1 if denoise else 0, _p(out)))
        return out

    def xyz(self):
        x = np.zeros((self.height, self.width, 3), np.float32)
        self.ctx.check(self.ctx.lib.argent_film_read_xyz(self.h, _p(x, ctypes.POINTER(ctypes.c_float))))
        return x


def render_pass(ctx: Context, scene: Scene, cam, film: Film, settings, count, seed):
    """argent's `render_pass(scene, cam, film, ps, count, seed)`."""
    ctx.check(ctx.lib.argent_render_pass(ctx.h, scene.h, ctypes.byref(cam), film.h, ctypes.byref(settings),
                                         int(count), int(seed)))


def render_batch(ctx: Context, items):
    """items: list of (scene, cam, film, settings, count, seed)."""
    arr = (N.ArgentBatchItem * len(items))()
    for i, (scene, cam, film, ps, count, seed) in enumerate(items):
        arr[i].scene = scene.h
        arr[i].camera = cam
        arr[i].film = film.h
        arr[i].settings = ps
        arr[i].count = int(count)
        arr[i].seed = int(seed)
    ctx.check(ctx.lib.argent_render_batch(ctx.h, arr, len(items)))


class Serve:
    """Continuous batching of render requests (argent_serve_*): the GPU
    counterpart of serve's job queue (argent/src/serve/queue.rs:599-617).
    submit/poll/cancel may come from any thread; step and read belong to
    the thread that owns the context."""

    def __init__(self, ctx: Context, film_budget=0, max_active=0, step_path_samples=0, aging_ms=0,
                 step_path_samples_max=0, overlap=False, max_pending=0, max_pending_path_samples=0):
        self.ctx = ctx
        cfg = N.ArgentServeConfig(int(film_budget), int(max_active), int(aging_ms), int(step_path_samples),
                                  int(step_path_samples_max), 1 if overlap else 0, int(max_pending),
                                  int(max_pending_path_samples))
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.argent_serve_create(ctx.h, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        ctx._own("serve", h)
        self._scenes = {}  # ticket -> scene, kept alive while the request is

    def close(self):
        if getattr(self, "h", None):
            self.ctx._release("serve", self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, scene: Scene, cam, settings, width, height, spp, seed=7, priority=0, flags=N.FILM_KAHAN):
        """A ticket, or N.ArgentError with code E_BUSY when the serve is at
        its max_pending bound (or the film cannot fit its budget)."""
        r = N.ArgentServeRequest()
        r.scene = scene.h
        r.camera = cam
        r.settings = settings
        r.width, r.height, r.spp, r.seed = int(width), int(height), int(spp), int(seed)
        r.film_flags = int(flags)
        r.priority = int(priority)
        t = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.argent_serve_submit(self.h, ctypes.byref(r), ctypes.byref(t)))
        self._scenes[t.value] = (scene, width, height)
        return t.value

    def poll(self, ticket):
        st = N.ArgentServeStatus()
        self.ctx.check(self.ctx.lib.argent_serve_poll(self.h, ticket, ctypes.byref(st)))
        return st

    def cancel(self, ticket):
        self.ctx.check(self.ctx.lib.argent_serve_cancel(self.h, ticket))

    def step(self):
        """One scheduling round; returns the number of requests pending."""
        n = ctypes.c_uint32()
        self.ctx.check(self.ctx.lib.argent_serve_step(self.h, ctypes.byref(n)))
        return int(n.value)

    def run(self):
        """Steps until nothing is queued or active."""
        while self.step():
            pass

    def read(self, ticket):
        """(color, albedo, normal) of a finished request; forgets it."""
        _, w, h = self._scenes[ticket]
        shape = (h, w, 3)
        c, a, n = np.zeros(shape, np.float32), np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.ctx.check(self.ctx.lib.argent_serve_read(self.h, ticket, _p(c, fp), _p(a, fp), _p(n, fp)))
        del self._scenes[ticket]
        return c, a, n

    def release(self, ticket):
        self.ctx.check(self.ctx.lib.argent_serve_release(self.h, ticket))
        self._scenes.pop(ticket, None)

    def stats(self):
        s, p, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.argent_serve_stats(self.h, ctypes.byref(s), ctypes.byref(p), ctypes.byref(b)))
        return {"steps": s.value, "path_samples": p.value, "film_bytes_in_use": b.value}

    def now(self):
        return float(self.ctx.lib.argent_serve_now(self.h))


def denoise_atrous(ctx: Context, color, albedo=None, normal=None):
    """argent-post's `denoise(.., DenoiseBackend::Atrous)` on the device:
    (h, w, 3) float32 images in, the denoised colour out."""
    fp = ctypes.POINTER(ctypes.c_float)
    c = np.ascontiguousarray(color, np.float32)
    a = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
    n = None if normal is None else np.ascontiguousarray(normal, np.float32)
    out = np.zeros_like(c)
    h, w = c.shape[0], c.shape[1]
    ctx.check(ctx.lib.argent_denoise_atrous(ctx.h, w, h, _p(c, fp), _p(a, fp), _p(n, fp), _p(out, fp)))
    return out


def develop(ctx: Context, rgb, grade=None):
    """argent_post::develop on the device: (h, w, 3) scene-linear float32 in,
    8-bit sRGB out."""
    g = grade if grade is not None else N.ArgentGrade(0.0, N.TM_AGX, N.AGX_PUNCHY, 1.0)
    c = np.ascontiguousarray(rgb, np.float32)
    out = np.zeros(c.shape, np.uint8)
    ctx.check(ctx.lib.argent_develop(ctx.h, c.shape[1], c.shape[0], _p(c, ctypes.POINTER(ctypes.c_float)),
                                     ctypes.byref(g), _p(out)))
    return out
