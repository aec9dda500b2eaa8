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


def _cudart():
    """The CUDA runtime the library was linked against (already loaded)."""
    return ctypes.CDLL("libcudart.so.12")


def _device_memory_state(rt, device=0):
    """(free bytes on the device, reserved and used bytes of its default
    stream-ordered memory pool)."""
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), device) == 0
    out = [free.value]
    for attr in (5, 7):  # cudaMemPoolAttrReservedMemCurrent, cudaMemPoolAttrUsedMemCurrent
        v = ctypes.c_uint64()
        assert rt.cudaMemPoolGetAttribute(pool, attr, ctypes.byref(v)) == 0
        out.append(v.value)
    return tuple(out), pool


@pytest.mark.gpu
def test_noalloc_allocates_no_device_memory():
    """After a first call (which looks up the array's address and loads the
    kernel), further calls leave the device's free memory and its default
    memory pool exactly as they were."""
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    ring = mesh.ring()
    ctx = Context(0)
    piece = Piece(ctx, ring)
    n = 100_000
    rays = np.ascontiguousarray(make_rays(ring.positions, ring.tris, n, seed=23))
    hits = np.zeros((n, 4), np.float32)

    def call():
        rc = ctx.lib.argent_trace_closest_noalloc(ctx.h, piece.h, rays.ctypes.data_as(ctypes.c_void_p), n,
                                                  hits.ctypes.data_as(ctypes.c_void_p))
        assert rc == N.OK, ctx.lib.argent_last_error(ctx.h)

    call()
    ctx.sync()
    rt = _cudart()
    _, pool = _device_memory_state(rt)
    assert rt.cudaMemPoolTrimTo(pool, ctypes.c_size_t(0)) == 0
    before, _ = _device_memory_state(rt)
    for _ in range(3):
        call()
    after, _ = _device_memory_state(rt)
    assert after == before, (before, after)
    assert (hits[:, 3].view(np.uint32) != 0xFFFFFFFF).sum() > n // 4


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
