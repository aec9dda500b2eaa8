"""Triangle meshes and the procedural workload pieces.

`Mesh` mirrors what argent's `Piece::new` consumes (core/src/scene.rs:10-32):
positions, normals, triangles, per-triangle material slots and an optional
per-vertex cavity mask.
"""

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as N


@dataclass
class Mesh:
    positions: np.ndarray  # (nv, 3) float32
    tris: np.ndarray  # (nt, 3) uint32
    normals: Optional[np.ndarray] = None  # (nv, 3) float32
    tri_material: Optional[np.ndarray] = None  # (nt,) uint16
    cavity: Optional[np.ndarray] = None  # (nv,) float32

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, np.float32).reshape(-1, 3)
        self.tris = np.ascontiguousarray(self.tris, np.uint32).reshape(-1, 3)
        if self.normals is not None:
            self.normals = np.ascontiguousarray(self.normals, np.float32).reshape(-1, 3)
        if self.tri_material is not None:
            self.tri_material = np.ascontiguousarray(self.tri_material, np.uint16).reshape(-1)
        if self.cavity is not None:
            self.cavity = np.ascontiguousarray(self.cavity, np.float32).reshape(-1)

    @property
    def num_tris(self):
        return len(self.tris)

    def bounds(self):
        return self.positions.min(axis=0), self.positions.max(axis=0)


def _take(m: N.ArgentMesh) -> Mesh:
    nv, nt = m.nv, m.nt
    p = np.ctypeslib.as_array(m.positions, shape=(nv * 3,)).reshape(nv, 3).copy()
    n = np.ctypeslib.as_array(m.normals, shape=(nv * 3,)).reshape(nv, 3).copy()
    t = np.ctypeslib.as_array(m.tris, shape=(nt * 3,)).reshape(nt, 3).copy()
    mat = np.ctypeslib.as_array(m.tri_material, shape=(nt,)).copy()
    N.host().argent_mesh_free(ctypes.byref(m))
    return Mesh(p, t, n, mat)


def ring(R=9.0, r=1.2, nu=512, nv=64, amp=0.15, cell_mm=0.8, seed=1) -> Mesh:
    """The small plain workload's piece: a torus ring, 2*nu*nv triangles,
    radially displaced by seeded value noise (argent_synth_ring)."""
    m = N.ArgentMesh()
    rc = N.host().argent_synth_ring(R, r, nu, nv, amp, cell_mm, seed, ctypes.byref(m))
    if rc != N.OK:
        raise N.ArgentError(rc, "argent_synth_ring failed")
    return _take(m)


def signet(R=9.0, r=1.2, nu=2048, nv=512, bezel_w=14.0, bezel_d=12.0, emboss_mm=0.4, seed=2, mask_seed=3) -> Mesh:
    """The full-still workload's piece: the torus with a flattened, embossed
    14 x 12 mm bezel; 2*nu*nv triangles (2,097,152 at the defaults), two
    metal slots by a seeded mask (argent_synth_signet)."""
    m = N.ArgentMesh()
    rc = N.host().argent_synth_signet(R, r, nu, nv, bezel_w, bezel_d, emboss_mm, seed, mask_seed, ctypes.byref(m))
    if rc != N.OK:
        raise N.ArgentError(rc, "argent_synth_signet failed")
    return _take(m)


def gem_ring(shank_nu=768, shank_nv=440, center_mm=2.0, stone_mm=0.75, seed=4) -> Mesh:
    """The gems workload's piece: an 18k setting (torus shank + 37 prong
    cups, about 0.9M triangles) holding a 4 mm round brilliant and 36 side
    stones of 1.5 mm (argent_synth_gem_ring).  Material slots: 0 metal,
    1 centre stone, 2..5 side-stone gems."""
    m = N.ArgentMesh()
    rc = N.host().argent_synth_gem_ring(shank_nu, shank_nv, center_mm, stone_mm, seed, ctypes.byref(m))
    if rc != N.OK:
        raise N.ArgentError(rc, "argent_synth_gem_ring failed")
    return _take(m)


# ---------------------------------------------------------------- argent-mesh helpers (host)

def smooth_normals(m: Mesh) -> np.ndarray:
    """normals::smooth_vertex_normals (argent-mesh normals.rs:226-242)."""
    out = np.zeros_like(m.positions)
    fp = ctypes.POINTER(ctypes.c_float)
    N.check(N.gpu().argent_mesh_smooth_normals(m.positions.ctypes.data_as(fp), len(m.positions),
                                               m.tris.ctypes.data_as(N.c_u32_p), len(m.tris), out.ctypes.data_as(fp)))
    return out


def concavity(m: Mesh, normals, radius) -> np.ndarray:
    """cavity::concavity (argent-mesh cavity.rs:137-236)."""
    n = np.ascontiguousarray(normals, np.float32)
    out = np.zeros(len(m.positions), np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    N.check(N.gpu().argent_mesh_concavity(m.positions.ctypes.data_as(fp), len(m.positions), n.ctypes.data_as(fp),
                                          m.tris.ctypes.data_as(N.c_u32_p), len(m.tris), radius,
                                          out.ctypes.data_as(fp)))
    return out


def smooth(m: Mesh, values, iterations, lam=0.5) -> np.ndarray:
    """cavity::smooth (argent-mesh cavity.rs:241-299)."""
    v = np.array(values, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    N.check(N.gpu().argent_mesh_smooth(m.positions.ctypes.data_as(fp), len(m.positions),
                                       m.tris.ctypes.data_as(N.c_u32_p), len(m.tris), v.ctypes.data_as(fp),
                                       iterations, lam))
    return v


def patina_settings(radius):
    """Prepared::build's PatinaSettings (core/src/shot.rs:137-141)."""
    return N.ArgentPatinaSettings(48, float(min(max(radius * 0.09, 0.4), 2.5)),
                                  float(min(max(radius * 0.03, 0.15), 1.0)), 0.35, 3)
