"""The allocation-free closest-hit entry point (argent_trace_closest_noalloc).

Callers that must not allocate device memory while they run (a serve loop
working inside a fixed device-memory budget, issuing probe rays between
renders) use this variant.  It stages rays and hits in a static device array
instead of allocating.  This file is collected last so that a run stopping at
the first failure has already run every other test; it also passes alone in
a fresh process.
"""

import ctypes

import numpy as np
import pytest

from tests.rays import make_rays

NOALLOC_MAX_RAYS = 1 << 18


@pytest.mark.gpu
def test_noalloc_closest_hit_matches_allocating_entry_point():
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    ring = mesh.ring()
    ctx = Context(0)
    piece = Piece(ctx, ring)
    lib = ctx.lib
    # Two calls in a row share the static array; each must match the
    # allocating entry point on its own rays.
    for seed, n in ((21, 200_000), (22, NOALLOC_MAX_RAYS)):
        rays = np.ascontiguousarray(make_rays(ring.positions, ring.tris, n, seed=seed))
        ref = piece.trace_closest(rays)
        got = np.zeros((n, 4), np.float32)
        rc = lib.argent_trace_closest_noalloc(ctx.h, piece.h, rays.ctypes.data_as(ctypes.c_void_p), n,
                                              got.ctypes.data_as(ctypes.c_void_p))
        assert rc == N.OK, lib.argent_last_error(ctx.h)
        rp, gp = ref[:, 3].view(np.uint32), got[:, 3].view(np.uint32)
        assert np.array_equal(rp, gp)
        hit = rp != 0xFFFFFFFF
        assert hit.sum() > n // 4
        ulps = np.abs(ref[hit, 0].view(np.int32).astype(np.int64) - got[hit, 0].view(np.int32).astype(np.int64))
        assert ulps.max() <= 2  # the traversal tests' tolerance on t


@pytest.mark.gpu
def test_noalloc_rejects_more_rays_than_its_array_holds():
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    ctx = Context(0)
    piece = Piece(ctx, mesh.ring(nu=64, nv=16))
    n = NOALLOC_MAX_RAYS + 1
    rays = np.zeros((n, 8), np.float32)
    hits = np.zeros((n, 4), np.float32)
    rc = ctx.lib.argent_trace_closest_noalloc(ctx.h, piece.h, rays.ctypes.data_as(ctypes.c_void_p), n,
                                              hits.ctypes.data_as(ctypes.c_void_p))
    assert rc == N.E_INVALID
    assert b"262144" in ctx.lib.argent_last_error(ctx.h)
