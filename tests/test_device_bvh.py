"""The BVH built on the device (argent_piece_upload_device_bvh).

The device tree differs from the host SAH tree, but a closest hit is the
minimum of (t, triangle index) over the triangles whose Moller-Trumbore test
passes, so both trees give the same hit records bit for bit, and both agree
with argent's traversal (restated in the oracle) under the same buckets as
the host tree's parity tests.
"""

import time

import numpy as np
import pytest

from tests.rays import compare_hits, make_rays

pytestmark = pytest.mark.gpu


def _ctx():
    from argent_b200.gpu import Context

    return Context(0)


def test_ring_closest_and_any_hit_match():
    import oracle as O
    from argent_b200 import mesh
    from argent_b200.gpu import Piece

    ring = mesh.ring()
    ctx = _ctx()
    dev = Piece(ctx, ring, device_bvh=True)
    host = Piece(ctx, ring)
    n = 1 << 22
    rays = make_rays(ring.positions, ring.tris, n, seed=21)
    got = dev.trace_closest(rays)
    assert np.array_equal(got.view(np.uint32), host.trace_closest(rays).view(np.uint32))
    bvh = O.Bvh(ring.positions, ring.tris)
    r = compare_hits(bvh.intersect(rays), got, bvh, rays)
    print("device-BVH closest-hit parity (ring, 2^22 rays):", {k: v for k, v in r.items() if k != "mismatch_idx"})
    assert r["mismatch"] == 0, r["mismatch_idx"]
    assert r["t_ulp_fail"] == 0
    assert r["hit_both"] > n // 4
    shadow = make_rays(ring.positions, ring.tris, 1 << 20, seed=22)
    shadow[::2, 3] = np.float32(5.0)
    occ = dev.trace_anyhit(shadow)
    assert np.array_equal(occ, bvh.occluded(shadow))
    assert occ.sum() > 1000


def test_signet_parity_and_bounds():
    import oracle as O
    from argent_b200 import mesh
    from argent_b200.gpu import Piece

    m = mesh.signet()
    ctx = _ctx()
    Piece(ctx, m, device_bvh=True).close()  # warm the allocator and the kernels
    t0 = time.perf_counter()
    dev = Piece(ctx, m, device_bvh=True)
    t1 = time.perf_counter()
    host = Piece(ctx, m)
    t2 = time.perf_counter()
    print(f"signet upload + BVH build: device {1e3 * (t1 - t0):.1f} ms, host {1e3 * (t2 - t1):.1f} ms")
    for a, b in zip(dev.bounds(), host.bounds()):
        assert np.array_equal(a, b)
    n = 1 << 21
    rays = make_rays(m.positions, m.tris, n, seed=23)
    got = dev.trace_closest(rays)
    assert np.array_equal(got.view(np.uint32), host.trace_closest(rays).view(np.uint32))
    bvh = O.Bvh(m.positions, m.tris)
    r = compare_hits(bvh.intersect(rays), got, bvh, rays)
    print("device-BVH closest-hit parity (signet, 2^21 rays):", {k: v for k, v in r.items() if k != "mismatch_idx"})
    assert r["mismatch"] == 0, r["mismatch_idx"]
    assert r["t_ulp_fail"] == 0
    assert r["closer"] <= n // 100000


def test_renders_the_same_image():
    from argent_b200 import workloads as W
    from argent_b200.gpu import Film, Piece, Scene, render_pass

    wl = W.ring_still()
    ctx = _ctx()
    films = []
    for device_bvh in (False, True):
        piece = Piece(ctx, wl.mesh, device_bvh=device_bvh)
        scene = Scene(ctx, piece, wl.desc)
        film = Film(ctx, wl.width, wl.height)
        render_pass(ctx, scene, wl.camera, film, wl.settings, 8, wl.seed)
        films.append(film.xyz())
    assert np.array_equal(films[0], films[1])
    assert films[0].sum() > 0


@pytest.mark.parametrize("case", ["one", "five", "coplanar", "duplicates"])
def test_small_and_degenerate_pieces(case):
    """Few triangles, a flat piece (zero extent on one axis) and many copies
    of one triangle (equal Morton codes): hits equal the host tree's."""
    from argent_b200.gpu import Piece
    from argent_b200.mesh import Mesh

    rng = np.random.default_rng(5)
    if case == "one":
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        tris = np.array([[0, 1, 2]], np.uint32)
    elif case == "five":
        pos = rng.uniform(-1, 1, (15, 3)).astype(np.float32)
        tris = np.arange(15, dtype=np.uint32).reshape(5, 3)
    elif case == "coplanar":
        pos = rng.uniform(-1, 1, (3000, 3)).astype(np.float32)
        pos[:, 2] = 0.25
        tris = np.arange(3000, dtype=np.uint32).reshape(1000, 3)
    else:
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        tris = np.tile(np.array([[0, 1, 2]], np.uint32), (300, 1))
    m = Mesh(pos, tris)
    ctx = _ctx()
    dev = Piece(ctx, m, device_bvh=True)
    host = Piece(ctx, m)
    for a, b in zip(dev.bounds(), host.bounds()):
        assert np.array_equal(a, b)
    rays = np.zeros((4096, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-1.5, 1.5, (4096, 3))
    d = rng.normal(size=(4096, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = np.inf
    rays[:16, 0:3] = [0.2, 0.2, 1.0]
    rays[:16, 4:7] = [0.0, 0.0, -1.0]
    got = dev.trace_closest(rays)
    assert np.array_equal(got.view(np.uint32), host.trace_closest(rays).view(np.uint32))
    assert np.array_equal(dev.trace_anyhit(rays), host.trace_anyhit(rays))
    if case != "five":
        assert np.all(got[:16, 3].view(np.uint32) != 0xFFFFFFFF)
