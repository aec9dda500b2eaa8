"""CPU oracle: a restatement of argent's render hot path (test infrastructure).

liboracle.so restates crates/argent-core/src/{render,integrator,scene,bvh,
camera,sampler,light,envmap,material,bsdf,microfacet,color}.rs and the
argent-spectra primitives they call, operation by operation, compiled with
-ffp-contract=off.  Only the tests, __graft_entry__.smoke() and bench.py's
CPU-baseline leg load it, as the checker; the product never does.

Parity pinning: the BVH build/traversal, Fresnel, GGX, wavelength sampling,
CIE and white-balance restatements are checked against argent's own unit-test
known answers (tests/test_oracle_golden.py).  The sampler's Sobol values come
from argent's unvendored sobol_burley 0.5.0 crate and are replaced by a
published Burley-2020 construction shared with the CUDA path, so exact sample
streams of argent's binary are unpinned (only the oracle/GPU pair is).
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise OSError(f"{SO} missing: run `make -C oracle` (or python -m argent_b200.build)")
        from argent_b200 import _native as N

        L = ctypes.CDLL(SO)
        vp, u32, u64, f = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float
        fp = ctypes.POINTER(ctypes.c_float)
        sig = {
            "oracle_bvh_create": (vp, [vp, u32, vp, u32]),
            "oracle_bvh_destroy": (None, [vp]),
            "oracle_bvh_intersect": (None, [vp, vp, u64, vp, ctypes.c_int]),
            "oracle_bvh_occluded": (None, [vp, vp, u64, vp, ctypes.c_int]),
            "oracle_bvh_intersect_binary": (None, [vp, vp, u64, vp]),
            "oracle_brute_intersect": (None, [vp, vp, u32, vp, u64, vp, ctypes.c_int]),
            "oracle_tri_hit": (ctypes.c_int, [vp, vp, u32, vp, fp, fp, fp]),
            "oracle_bvh_stats": (None, [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u32)]),
            "oracle_scene_create": (vp, [vp, u32, vp, vp, u32, vp, vp, ctypes.POINTER(N.ArgentSceneDesc)]),
            "oracle_scene_destroy": (None, [vp]),
            "oracle_scene_set_turntable": (None, [vp, f]),
            "oracle_render_pass": (None, [vp, ctypes.POINTER(N.ArgentCamera), ctypes.POINTER(N.ArgentPathSettings),
                                          u32, u32, u32, u32, u32, u32, u32, vp, vp, vp, vp, ctypes.c_int]),
            "oracle_trace_sample": (None, [vp, ctypes.POINTER(N.ArgentCamera), ctypes.POINTER(N.ArgentPathSettings),
                                           u32, u32, u32, u32, u32, u32, fp]),
            "oracle_camera_matrix": (None, [ctypes.c_int, fp, fp]),
            "oracle_fresnel_dielectric": (f, [f, f]),
            "oracle_fresnel_conductor": (f, [f, f, f]),
            "oracle_ggx_e": (f, [f, f]),
            "oracle_ggx_sample_h": (None, [f, fp, f, f, fp]),
            "oracle_energy_table": (None, [fp]),
            "oracle_sample_visible": (None, [f, fp, fp]),
            "oracle_to_xyz": (None, [fp, fp, fp, fp]),
            "oracle_xyz_bar": (None, [f, fp]),
            "oracle_linear_rgb": (None, [fp, fp]),
            "oracle_hash32": (u32, [u32]),
            "oracle_sampler_next": (None, [u32, u32, u32, fp]),
            "oracle_sampler_random": (None, [u32, u32, u32, fp]),
            "oracle_sobol_4d": (None, [u32, u32, u32, fp]),
            "oracle_sobol_raw": (None, [u32, ctypes.c_int, ctypes.POINTER(u32)]),
            "oracle_smooth_vertex_normals": (None, [vp, u32, vp, u32, vp]),
            "oracle_ambient_occlusion": (None, [vp, u32, vp, vp, u32, u32, f, vp]),
            "oracle_concavity": (None, [vp, u32, vp, vp, u32, f, vp]),
            "oracle_smooth": (None, [vp, u32, vp, u32, vp, u32, f]),
            "oracle_patina_mask": (None, [vp, u32, vp, vp, u32, u32, f, f, f, u32, vp]),
            "oracle_atrous": (None, [u32, u32, vp, vp, vp, vp]),
            "oracle_tonemap_pixel": (None, [fp, f, ctypes.c_int, ctypes.c_int, f, fp]),
            "oracle_srgb_encode": (f, [f]),
            "oracle_develop": (None, [vp, u64, f, ctypes.c_int, ctypes.c_int, f, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Bvh:
    """argent's BVH (bvh.rs) over a triangle mesh."""

    def __init__(self, positions, tris):
        self.positions = np.ascontiguousarray(positions, np.float32)
        self.tris = np.ascontiguousarray(tris, np.uint32)
        self.h = lib().oracle_bvh_create(_ptr(self.positions), len(self.positions), _ptr(self.tris), len(self.tris))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_bvh_destroy(self.h)
            self.h = None

    @staticmethod
    def _rays(rays):
        """(n, 8) float32 rays, contiguous: the C side reads them as a flat
        array, so a strided view (rays[::2]) must be copied first."""
        return np.ascontiguousarray(rays, np.float32).reshape(-1, 8)

    def intersect(self, rays, threads=0):
        rays = self._rays(rays)
        hits = np.zeros((len(rays), 4), np.float32)
        lib().oracle_bvh_intersect(self.h, _ptr(rays), len(rays), _ptr(hits), threads)
        return hits

    def intersect_binary(self, rays):
        rays = self._rays(rays)
        hits = np.zeros((len(rays), 4), np.float32)
        lib().oracle_bvh_intersect_binary(self.h, _ptr(rays), len(rays), _ptr(hits))
        return hits

    def occluded(self, rays, threads=0):
        rays = self._rays(rays)
        occ = np.zeros(len(rays), np.uint8)
        lib().oracle_bvh_occluded(self.h, _ptr(rays), len(rays), _ptr(occ), threads)
        return occ

    def brute(self, rays, threads=0):
        rays = self._rays(rays)
        hits = np.zeros((len(rays), 4), np.float32)
        lib().oracle_brute_intersect(_ptr(self.positions), _ptr(self.tris), len(self.tris), _ptr(rays), len(rays),
                                     _ptr(hits), threads)
        return hits

    def tri_hit(self, prim, ray):
        t, u, v = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        r = np.ascontiguousarray(ray, np.float32)
        ok = lib().oracle_tri_hit(_ptr(self.positions), _ptr(self.tris), int(prim), _ptr(r), ctypes.byref(t),
                                  ctypes.byref(u), ctypes.byref(v))
        return bool(ok), t.value, u.value, v.value

    def stats(self):
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        lib().oracle_bvh_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value


class Scene:
    """argent's Scene + render_pass on the CPU, from the same C-ABI description."""

    def __init__(self, mesh, desc):
        self.mesh = mesh  # keep arrays alive
        p, n, t, m, c = mesh.positions, mesh.normals, mesh.tris, mesh.tri_material, mesh.cavity
        self.h = lib().oracle_scene_create(_ptr(p), len(p), _ptr(n), _ptr(t), len(t), _ptr(m), _ptr(c),
                                           ctypes.byref(desc))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def set_turntable(self, deg):
        lib().oracle_scene_set_turntable(self.h, float(deg))

    def render_pass(self, cam, settings, w, h, first, count, seed, rows=None, threads=0, want_xyz=True):
        """Film sums as argent accumulates them (camera RGB), plus XYZ sums
        (float64) and the guides.  rows=(y0, y1) restricts to a band."""
        y0, y1 = rows if rows else (0, h)
        color = np.zeros((h, w, 3), np.float32)
        albedo = np.zeros((h, w, 3), np.float32)
        normal = np.zeros((h, w, 3), np.float32)
        xyz = np.zeros((h, w, 3), np.float64) if want_xyz else None
        lib().oracle_render_pass(self.h, ctypes.byref(cam), ctypes.byref(settings), w, h, first, count, seed, y0, y1,
                                 _ptr(color), _ptr(albedo), _ptr(normal), _ptr(xyz), threads)
        return color, albedo, normal, xyz


# ---------------------------------------------------------------- cavity mask (argent-mesh cavity.rs)

def _mesh_arrays(mesh):
    p = np.ascontiguousarray(mesh.positions, np.float32)
    t = np.ascontiguousarray(mesh.tris, np.uint32)
    return p, t


def smooth_vertex_normals(mesh):
    p, t = _mesh_arrays(mesh)
    out = np.zeros_like(p)
    lib().oracle_smooth_vertex_normals(_ptr(p), len(p), _ptr(t), len(t), _ptr(out))
    return out


def ambient_occlusion(mesh, normals, samples=48, distance=1.2):
    p, t = _mesh_arrays(mesh)
    n = np.ascontiguousarray(normals, np.float32)
    out = np.zeros(len(p), np.float32)
    lib().oracle_ambient_occlusion(_ptr(p), len(p), _ptr(n), _ptr(t), len(t), samples, distance, _ptr(out))
    return out


def concavity(mesh, normals, radius):
    p, t = _mesh_arrays(mesh)
    n = np.ascontiguousarray(normals, np.float32)
    out = np.zeros(len(p), np.float32)
    lib().oracle_concavity(_ptr(p), len(p), _ptr(n), _ptr(t), len(t), radius, _ptr(out))
    return out


def smooth(mesh, values, iterations, lam=0.5):
    p, t = _mesh_arrays(mesh)
    v = np.array(values, np.float32)
    lib().oracle_smooth(_ptr(p), len(p), _ptr(t), len(t), _ptr(v), iterations, lam)
    return v


def patina_mask(mesh, normals=None, ao_samples=48, ao_distance=1.2, curvature_radius=0.4, concavity_weight=0.35,
                smooth_iterations=3):
    """cavity.rs:52-78 with PatinaSettings' defaults (cavity.rs:38-42)."""
    p, t = _mesh_arrays(mesh)
    n = None if normals is None else np.ascontiguousarray(normals, np.float32)
    out = np.zeros(len(p), np.float32)
    lib().oracle_patina_mask(_ptr(p), len(p), _ptr(n), _ptr(t), len(t), ao_samples, ao_distance, curvature_radius,
                             concavity_weight, smooth_iterations, _ptr(out))
    return out


def atrous(color, albedo=None, normal=None):
    """argent-post's built-in à-trous denoiser (denoise.rs:653-712) on
    (h, w, 3) float32 images."""
    c = np.ascontiguousarray(color, np.float32)
    a = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
    n = None if normal is None else np.ascontiguousarray(normal, np.float32)
    out = np.zeros_like(c)
    lib().oracle_atrous(c.shape[1], c.shape[0], _ptr(c), _ptr(a), _ptr(n), _ptr(out))
    return out


# ---------------------------------------------------------------- develop (argent-post tonemap.rs)

def tonemap_pixel(rgb, ev=0.0, op=0, look=0, saturation=1.0):
    """tonemap.rs:201-213: exact display-linear result of one pixel."""
    x = (ctypes.c_float * 3)(*[float(v) for v in rgb])
    out = (ctypes.c_float * 3)()
    lib().oracle_tonemap_pixel(x, ev, op, look, saturation, out)
    return np.array(out[:], np.float32)


def srgb_encode(x):
    return float(lib().oracle_srgb_encode(float(x)))


def develop(rgb, ev=0.0, op=0, look=1, saturation=1.0):
    """tonemap.rs:369-391 on an (h, w, 3) image: (8-bit image, encoded
    floats of the fast path)."""
    c = np.ascontiguousarray(rgb, np.float32)
    enc = np.zeros_like(c)
    out = np.zeros(c.shape, np.uint8)
    lib().oracle_develop(_ptr(c), c.size // 3, ev, op, look, saturation, _ptr(enc), _ptr(out))
    return out, enc
