"""ctypes bindings of include/argent_gpu.h and include/argent_host.h.

The GPU library is the product path: if it cannot be loaded the package
raises instead of falling back to anything else.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
GPU_SO = os.path.join(LIB_DIR, "libargent_gpu.so")
HOST_SO = os.path.join(LIB_DIR, "libargent_host.so")

SPEC_LEN = 471
NK_LEN = 95
NO_HIT = 0xFFFFFFFF

OK, E_OOM, E_INVALID, E_TIMEOUT, E_CUDA, E_OVERFLOW, E_BUSY = range(7)
MAT_METAL, MAT_GEM, MAT_PLASTIC, MAT_OPAL, MAT_DIFFUSE, MAT_BLACK = range(6)
GEM_TRANSPARENT, GEM_OPAL, GEM_OPAQUE = range(3)
ENV_GRADIENT, ENV_MAP = range(2)
FILM_KAHAN, FILM_FP64, FILM_PROGRESSIVE = 1, 2, 4
TRI_MOLLER_TRUMBORE, TRI_WATERTIGHT = 0, 1
FILM_FP64_AFTER = 4096

c_float_p = ctypes.POINTER(ctypes.c_float)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_u16_p = ctypes.POINTER(ctypes.c_uint16)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)


class ArgentMaterial(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("gem_kind", ctypes.c_int32), ("alpha", ctypes.c_float), ("eta", ctypes.c_float),
        ("cell_mm", ctypes.c_float), ("strength", ctypes.c_float), ("has_patina", ctypes.c_int32),
        ("patina_strength", ctypes.c_float), ("patina_lo", ctypes.c_float), ("patina_hi", ctypes.c_float),
        ("patina_alpha", ctypes.c_float), ("patina_eta", ctypes.c_float), ("has_opaque_base", ctypes.c_int32),
        ("nk_eta", ctypes.c_float * NK_LEN), ("nk_k", ctypes.c_float * NK_LEN),
        ("spec_a", ctypes.c_float * SPEC_LEN), ("spec_b", ctypes.c_float * SPEC_LEN),
        ("spec_b2", ctypes.c_float * SPEC_LEN),
    ]


class ArgentPanel(ctypes.Structure):
    _fields_ = [
        ("center", ctypes.c_float * 3), ("hu", ctypes.c_float * 3), ("hv", ctypes.c_float * 3),
        ("emits", ctypes.c_int32), ("camera_visible", ctypes.c_int32), ("feather", ctypes.c_float),
        ("emission", ctypes.c_float * SPEC_LEN),
    ]


class ArgentEnv(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("power", ctypes.c_float), ("top", ctypes.c_float * SPEC_LEN),
        ("horizon", ctypes.c_float * SPEC_LEN), ("bottom", ctypes.c_float * SPEC_LEN), ("width", ctypes.c_int32),
        ("height", ctypes.c_int32), ("rgb", c_float_p), ("rotation_deg", ctypes.c_float),
    ]


class ArgentFloor(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int32), ("y", ctypes.c_float), ("material", ctypes.c_int32),
                ("fade_start", ctypes.c_float), ("fade_end", ctypes.c_float)]


class ArgentSceneDesc(ctypes.Structure):
    _fields_ = [
        ("materials", ctypes.POINTER(ArgentMaterial)), ("num_materials", ctypes.c_int32),
        ("panels", ctypes.POINTER(ArgentPanel)), ("num_panels", ctypes.c_int32),
        ("env", ctypes.POINTER(ArgentEnv)), ("floor", ArgentFloor), ("turntable_deg", ctypes.c_float),
        ("has_white", ctypes.c_int32), ("white_xyz", ctypes.c_float * 3),
    ]


class ArgentCamera(ctypes.Structure):
    _fields_ = [
        ("pos", ctypes.c_float * 3), ("forward", ctypes.c_float * 3), ("right", ctypes.c_float * 3),
        ("up", ctypes.c_float * 3), ("half_w", ctypes.c_float), ("half_h", ctypes.c_float),
        ("lens_radius", ctypes.c_float), ("focus_dist", ctypes.c_float), ("shift", ctypes.c_float * 2),
    ]


class ArgentPathSettings(ctypes.Structure):
    _fields_ = [("max_depth", ctypes.c_uint32), ("clamp_indirect", ctypes.c_float), ("rr_depth", ctypes.c_uint32)]


class ArgentRay(ctypes.Structure):
    _fields_ = [("o", ctypes.c_float * 3), ("tmax", ctypes.c_float), ("d", ctypes.c_float * 3),
                ("pad", ctypes.c_float)]


class ArgentHit(ctypes.Structure):
    _fields_ = [("t", ctypes.c_float), ("u", ctypes.c_float), ("v", ctypes.c_float), ("prim", ctypes.c_uint32)]


class ArgentLimits(ctypes.Structure):
    _fields_ = [("wave_paths", ctypes.c_uint64), ("memory_budget", ctypes.c_uint64), ("lanes", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class ArgentBatchItem(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("camera", ArgentCamera), ("film", ctypes.c_void_p),
                ("settings", ArgentPathSettings), ("count", ctypes.c_uint32), ("seed", ctypes.c_uint32)]


class ArgentServeConfig(ctypes.Structure):
    _fields_ = [("film_budget", ctypes.c_uint64), ("max_active", ctypes.c_uint32), ("aging_ms", ctypes.c_uint32),
                ("step_path_samples", ctypes.c_uint64), ("step_path_samples_max", ctypes.c_uint64),
                ("overlap", ctypes.c_uint32), ("max_pending", ctypes.c_uint32),
                ("max_pending_path_samples", ctypes.c_uint64)]


class ArgentServeRequest(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("camera", ArgentCamera), ("settings", ArgentPathSettings),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("seed", ctypes.c_uint32), ("film_flags", ctypes.c_uint32), ("priority", ctypes.c_int32)]


class ArgentServeStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("samples", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("t_submit", ctypes.c_double), ("t_start", ctypes.c_double),
                ("t_done", ctypes.c_double)]


REQ_QUEUED, REQ_ACTIVE, REQ_DONE, REQ_CANCELLED, REQ_FAILED = range(5)


class ArgentGrade(ctypes.Structure):
    _fields_ = [("exposure_ev", ctypes.c_float), ("tonemap", ctypes.c_int32), ("look", ctypes.c_int32),
                ("saturation", ctypes.c_float)]


TM_AGX, TM_ACES, TM_KHRONOS, TM_REINHARD, TM_CLAMP = range(5)
AGX_BASE, AGX_PUNCHY, AGX_GOLDEN = range(3)


class ArgentPatinaSettings(ctypes.Structure):
    _fields_ = [("ao_samples", ctypes.c_uint32), ("ao_distance", ctypes.c_float),
                ("curvature_radius", ctypes.c_float), ("concavity_weight", ctypes.c_float),
                ("smooth_iterations", ctypes.c_uint32)]


class ArgentTuning(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_uint32), ("trace_blocks_per_sm", ctypes.c_uint32), ("wave_paths", ctypes.c_uint64),
                ("shade_blocks_per_sm", ctypes.c_uint32 * 5), ("reserved", ctypes.c_uint32)]


class ArgentTuneResult(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("wave_paths", ctypes.c_uint64),
                ("path_samples_per_s", ctypes.c_double)]


class ArgentMesh(ctypes.Structure):
    _fields_ = [("nv", ctypes.c_uint32), ("nt", ctypes.c_uint32), ("positions", c_float_p), ("normals", c_float_p),
                ("tris", c_u32_p), ("tri_material", c_u16_p)]


# name -> (restype, argtypes)
GPU_FUNCS = {
    "argent_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ArgentLimits), ctypes.POINTER(ctypes.c_void_p)]),
    "argent_ctx_destroy": (None, [ctypes.c_void_p]),
    "argent_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "argent_ctx_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "argent_ctx_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "argent_ctx_kernel_launches": (ctypes.c_uint64, [ctypes.c_void_p]),
    "argent_piece_upload": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_uint32, c_float_p, c_u32_p,
                                           ctypes.c_uint32, c_u16_p, c_float_p, ctypes.POINTER(ctypes.c_void_p)]),
    "argent_piece_upload_device_bvh": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_uint32, c_float_p,
                                                      c_u32_p, ctypes.c_uint32, c_u16_p, c_float_p,
                                                      ctypes.POINTER(ctypes.c_void_p)]),
    "argent_piece_destroy": (None, [ctypes.c_void_p]),
    "argent_piece_bounds": (ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p]),
    "argent_piece_device_bytes": (ctypes.c_uint64, [ctypes.c_void_p]),
    "argent_scene_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ArgentSceneDesc),
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "argent_scene_destroy": (None, [ctypes.c_void_p]),
    "argent_scene_set_turntable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "argent_film_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "argent_film_destroy": (None, [ctypes.c_void_p]),
    "argent_film_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "argent_film_samples": (ctypes.c_uint32, [ctypes.c_void_p]),
    "argent_film_read": (ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, c_float_p]),
    "argent_film_read_xyz": (ctypes.c_int, [ctypes.c_void_p, c_float_p]),
    "argent_render_pass": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ArgentCamera),
                                          ctypes.c_void_p, ctypes.POINTER(ArgentPathSettings), ctypes.c_uint32,
                                          ctypes.c_uint32]),
    "argent_trace_closest": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                            ctypes.c_void_p]),
    "argent_trace_anyhit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.c_void_p]),
    "argent_trace_closest_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_uint64, ctypes.c_void_p]),
    "argent_trace_anyhit_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_uint64, ctypes.c_void_p]),
    "argent_render_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentBatchItem), ctypes.c_uint32]),
    "argent_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ArgentCamera),
                                       ctypes.POINTER(ArgentPathSettings), ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.POINTER(ArgentTuneResult), ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_uint32)]),
    "argent_ctx_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "argent_ctx_set_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64]),
    "argent_ctx_child_hit_histogram": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "argent_ctx_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentTuning)]),
    "argent_ctx_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentTuning)]),
    "argent_piece_set_triangle_test": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "argent_trace_closest_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_uint64, ctypes.c_void_p]),
    "argent_ctx_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "argent_ctx_kernel_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_uint64)]),
    "argent_ctx_set_graphs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "argent_ctx_set_ray_sharing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "argent_ctx_set_counting": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "argent_ctx_traversal_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "argent_ctx_bounce_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "argent_ctx_traversal_histogram": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "argent_denoise_atrous": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, c_float_p, c_float_p,
                                             c_float_p, c_float_p]),
    "argent_film_denoise": (ctypes.c_int, [ctypes.c_void_p, c_float_p]),
    "argent_develop": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, c_float_p,
                                      ctypes.POINTER(ArgentGrade), ctypes.c_void_p]),
    "argent_film_develop": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentGrade), ctypes.c_int,
                                           ctypes.c_void_p]),
    "argent_piece_ambient_occlusion": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_float_p, c_float_p,
                                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, c_float_p]),
    "argent_piece_patina_mask": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_float_p, c_float_p,
                                                ctypes.c_uint32, c_u32_p, ctypes.c_uint32,
                                                ctypes.POINTER(ArgentPatinaSettings), c_float_p]),
    "argent_mesh_smooth_normals": (ctypes.c_int, [c_float_p, ctypes.c_uint32, c_u32_p, ctypes.c_uint32, c_float_p]),
    "argent_mesh_concavity": (ctypes.c_int, [c_float_p, ctypes.c_uint32, c_float_p, c_u32_p, ctypes.c_uint32,
                                             ctypes.c_float, c_float_p]),
    "argent_mesh_smooth": (ctypes.c_int, [c_float_p, ctypes.c_uint32, c_u32_p, ctypes.c_uint32, c_float_p,
                                          ctypes.c_uint32, ctypes.c_float]),
    "argent_serve_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentServeConfig),
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "argent_serve_destroy": (None, [ctypes.c_void_p]),
    "argent_serve_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ArgentServeRequest),
                                           ctypes.POINTER(ctypes.c_uint64)]),
    "argent_serve_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ArgentServeStatus)]),
    "argent_serve_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "argent_serve_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    "argent_serve_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, c_float_p, c_float_p, c_float_p]),
    "argent_serve_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "argent_serve_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "argent_serve_now": (ctypes.c_double, [ctypes.c_void_p]),
}
KERNEL_CLASSES = ["raygen", "intersect", "shade", "shadow", "film", "trace", "shade_terminal", "shade_metal",
                  "shade_coated", "shade_dielectric", "shade_other"]

_f, _i32, _u32, _cp = ctypes.c_float, ctypes.c_int32, ctypes.c_uint32, ctypes.c_char_p
_i32p = ctypes.POINTER(ctypes.c_int32)
HOST_FUNCS = {
    "argent_metal_nk": (ctypes.c_int, [_cp, c_float_p, c_float_p]),
    "argent_alloy_nk": (ctypes.c_int, [_cp, c_float_p, c_float_p]),
    "argent_karat_gold_nk": (ctypes.c_int, [_f, _f, _f, c_float_p, c_float_p]),
    "argent_nk_f0_srgb": (None, [c_float_p, c_float_p, c_float_p]),
    "argent_luminance_y": (_f, [c_float_p]),
    "argent_bake_emitter": (None, [_f, _f, c_float_p]),
    "argent_bake_rgb_albedo": (None, [c_float_p, c_float_p]),
    "argent_rgb_albedo_coefficients": (ctypes.c_int, [c_float_p, c_float_p]),
    "argent_bake_rgb_illuminant": (None, [c_float_p, c_float_p]),
    "argent_reflectance_srgb": (None, [c_float_p, c_float_p]),
    "argent_blackbody_white": (None, [_f, c_float_p]),
    "argent_gem_tables": (ctypes.c_int, [_cp, _i32p, c_float_p, c_float_p, c_float_p]),
    "argent_gem_dispersion": (ctypes.c_int, [_cp, c_float_p, c_float_p, c_float_p]),
    "argent_material_metal": (ctypes.c_int, [_cp, _f, _f, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_metal_nk": (ctypes.c_int, [c_float_p, c_float_p, _f, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_gem": (ctypes.c_int, [_cp, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_opal": (None, [ctypes.c_int, _f, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_plastic": (None, [c_float_p, _f, _f, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_diffuse": (None, [c_float_p, ctypes.POINTER(ArgentMaterial)]),
    "argent_material_black": (None, [ctypes.POINTER(ArgentMaterial)]),
    "argent_studio_build": (ctypes.c_int, [_cp, _f, _f, ctypes.POINTER(ArgentPanel), _i32p, ctypes.POINTER(ArgentEnv),
                                           ctypes.POINTER(ArgentMaterial), ctypes.POINTER(ArgentFloor), _i32p,
                                           c_float_p]),
    "argent_camera_look_at": (None, [c_float_p, c_float_p, c_float_p, _f, _f, _f, ctypes.POINTER(ArgentCamera)]),
    "argent_view_named": (ctypes.c_int, [_cp, c_float_p, c_float_p, c_float_p]),
    "argent_frame": (None, [c_float_p, _u32, _f, _f, _f, _f, _f, _f, ctypes.POINTER(ArgentCamera)]),
    "argent_synth_hdri": (None, [_u32, _u32, _f, _u32, c_float_p]),
    "argent_mesh_free": (None, [ctypes.POINTER(ArgentMesh)]),
    "argent_synth_ring": (ctypes.c_int, [ctypes.c_float, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_uint32, ctypes.POINTER(ArgentMesh)]),
    "argent_synth_gem_ring": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                             ctypes.c_uint32, ctypes.POINTER(ArgentMesh)]),
    "argent_synth_signet": (ctypes.c_int, [ctypes.c_float, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                                           ctypes.c_uint32, ctypes.POINTER(ArgentMesh)]),
}


def _bind(path, table, required=True):
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: run `python -m argent_b200.build` (no CPU fallback exists)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in table.items():
        try:
            f = getattr(lib, name)
        except AttributeError:
            if required:
                raise
            continue
        f.restype = res
        f.argtypes = args
    return lib


_gpu = None
_host = None


def gpu():
    """The CUDA library (raises if it is not built).  ARGENT_GPU_LIB names
    another build of it to load instead, e.g. one compiled with other
    build-time launch constants (`python -m argent_b200.build --variant`)."""
    global _gpu
    if _gpu is None:
        _gpu = _bind(os.environ.get("ARGENT_GPU_LIB") or GPU_SO, GPU_FUNCS)
    return _gpu


def host():
    """The host-side scene-builder library."""
    global _host
    if _host is None:
        _host = _bind(HOST_SO, HOST_FUNCS)
    return _host


class ArgentError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"argent error {code}: {msg}")
        self.code = code


def check(rc, ctx=None):
    if rc != OK:
        msg = gpu().argent_last_error(ctx)
        raise ArgentError(rc, msg.decode() if msg else "")
    return rc
