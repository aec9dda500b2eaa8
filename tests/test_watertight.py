"""The watertight triangle test (argent_piece_set_triangle_test), the
optional alternative to argent's Moller-Trumbore (bvh.rs:391-410).

Moller-Trumbore in argent's operation order stays the default: it is what
makes closest hits bit-exact against argent.  The watertight test (Woop,
Benthin and Wald 2013) guarantees that no ray slips between two triangles
that share an edge.  These tests measure how far its hits are from argent's
(id mismatches, ties, t in ulps) on the same 2^24 rays as the parity gate,
check that it never leaks on rays aimed exactly at the shared vertices and
edges of a closed mesh, and that switching back restores argent's records
bit for bit."""

import numpy as np
import pytest

from tests.rays import make_rays


def leak_rays(m):
    """Rays from 3 mm outside the closed ring toward every vertex and every
    edge midpoint, along the (area-weighted) vertex normal."""
    p = m.positions.astype(np.float32)
    n = m.normals.astype(np.float32)
    t = m.tris.astype(np.int64)
    edges = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    edges = np.unique(np.sort(edges, 1), axis=0)
    tgt = np.concatenate([p, (p[edges[:, 0]] + p[edges[:, 1]]) * np.float32(0.5)])
    nrm = np.concatenate([n, n[edges[:, 0]] + n[edges[:, 1]]])
    nrm = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    o = (tgt + nrm * np.float32(3.0)).astype(np.float32)
    d = (tgt - o).astype(np.float32)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays = np.zeros((len(tgt), 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = np.inf
    rays[:, 4:7] = d
    return rays


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ring", "signet"])
def test_watertight_against_argent_hits_2p24(which):
    """Id mismatch and tie rates of the watertight test against the
    oracle's argent traversal on the closest-hit gate's 2^24 rays."""
    import oracle as O
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    m = mesh.ring() if which == "ring" else mesh.signet()
    ctx = Context(0)
    piece = Piece(ctx, m)
    piece.set_triangle_test(N.TRI_WATERTIGHT)
    bvh = O.Bvh(m.positions, m.tris)
    n = 1 << 24
    rays = make_rays(m.positions, m.tris, n, seed=8)
    got = piece.trace_closest(rays)
    ref = bvh.intersect(rays)
    rp, gp = ref[:, 3].view(np.uint32), got[:, 3].view(np.uint32)
    both = (rp != 0xFFFFFFFF) & (gp != 0xFFFFFFFF)
    only_ref = int(((rp != 0xFFFFFFFF) & (gp == 0xFFFFFFFF)).sum())
    only_wt = int(((rp == 0xFFFFFFFF) & (gp != 0xFFFFFFFF)).sum())
    same = both & (rp == gp)
    ulps = np.abs(ref[same, 0].view(np.int32).astype(np.int64) - got[same, 0].view(np.int32).astype(np.int64))
    other = both & (rp != gp)
    eq_t = int((other & (ref[:, 0] == got[:, 0])).sum())
    print(f"watertight vs argent ({which}, 2^24 rays): hits {int(both.sum())}, same triangle {int(same.sum())}, "
          f"other triangle {int(other.sum())} (equal t {eq_t}), argent-only hits {only_ref}, "
          f"watertight-only hits {only_wt}, t ulps on the same triangle: median {np.median(ulps):.0f}, "
          f"p99 {np.percentile(ulps, 99):.0f}, max {ulps.max()}")
    rate = (int(other.sum()) - eq_t + only_ref + only_wt) / n
    assert rate < 1e-4, rate
    assert np.percentile(ulps, 99) <= 64


@pytest.mark.gpu
def test_watertight_does_not_leak_at_shared_edges():
    """Rays aimed at every vertex and edge midpoint of the closed ring all
    hit with the watertight test; argent's test is reported beside it."""
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    m = mesh.ring()
    ctx = Context(0)
    piece = Piece(ctx, m)
    rays = leak_rays(m)
    mt_miss = int((piece.trace_closest(rays)[:, 3].view(np.uint32) == 0xFFFFFFFF).sum())
    piece.set_triangle_test(N.TRI_WATERTIGHT)
    wt = piece.trace_closest(rays)
    wt_miss = int((wt[:, 3].view(np.uint32) == 0xFFFFFFFF).sum())
    print(f"rays at {len(rays)} vertices and edge midpoints: Moller-Trumbore misses {mt_miss}, watertight {wt_miss}")
    assert wt_miss == 0
    assert piece.trace_anyhit(rays).all()


@pytest.mark.gpu
def test_switching_back_restores_argent_records():
    """Watertight and back: the records equal a fresh upload's, so hits are
    bit-identical to the default piece's."""
    from argent_b200 import _native as N
    from argent_b200 import mesh
    from argent_b200.gpu import Context, Piece

    m = mesh.ring()
    ctx = Context(0)
    fresh, piece = Piece(ctx, m), Piece(ctx, m)
    rays = make_rays(m.positions, m.tris, 1 << 20, seed=31)
    piece.set_triangle_test(N.TRI_WATERTIGHT)
    piece.set_triangle_test(N.TRI_MOLLER_TRUMBORE)
    a, b = fresh.trace_closest(rays), piece.trace_closest(rays)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(fresh.trace_anyhit(rays), piece.trace_anyhit(rays))


@pytest.mark.gpu
def test_watertight_render_matches_argent_render():
    """A render through the watertight test differs from argent's only
    where a ray meets an edge: relRMSE per XYZ channel within 1 % of the
    oracle's Moller-Trumbore render on the same sample streams."""
    import oracle as O
    from argent_b200 import _native as N
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    piece.set_triangle_test(N.TRI_WATERTIGHT)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, wl.spp, wl.seed)
    sc = O.Scene(wl.mesh, wl.desc.c)
    _, _, _, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed)
    ref = (xyz / wl.spp).reshape(-1, 3)
    got = film.xyz().astype(np.float64).reshape(-1, 3)
    e = np.sqrt(((got - ref) ** 2).sum(0)) / np.sqrt((ref ** 2).sum(0))
    print("watertight ring render relRMSE XYZ vs oracle:", e)
    assert np.all(e <= 0.01), e


def test_leak_rays_aim_at_the_surface():
    """The leak rays start outside the ring and point at it (CPU)."""
    from argent_b200 import mesh

    m = mesh.ring(nu=64, nv=16)
    r = leak_rays(m)
    assert len(r) == len(m.positions) + len(m.positions) * 3
    assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1.0, atol=1e-5)
