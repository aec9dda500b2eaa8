"""Ray sharing in batches (argent_ctx_set_ray_sharing): metal variants of
one piece under the same camera, seed and samples trace each common ray
once.  argent renders every variant on its own (jobs.rs:595-713), so the
reference for each film is its render alone, bit for bit: the batch gives
each pixel the same runs of samples per wave as the render alone (served
requests, whose chunks the scheduler sizes, agree to float rounding)."""

import numpy as np
import pytest

from argent_b200 import _native as N
from argent_b200 import workloads as W

ALLOYS = ("sterling", "gold14k", "rose14k")


def variants(wl, alloys=ALLOYS, turn=None):
    """The ring still's scene with each alloy (same panels, floor, turn)."""
    t = wl.desc.c.turntable_deg if turn is None else turn
    return [W._studio_scene(wl.mesh, [W.metal(a, 0.07, 0.8)], "noir", t) for a in alloys]


def films_of(ctx, piece, descs, wl, count, seeds=None, cams=None, share=False, batch=True):
    from argent_b200.gpu import Film, Scene, render_batch, render_pass

    scenes = [Scene(ctx, piece, d) for d in descs]
    films = [Film(ctx, wl.width, wl.height) for _ in descs]
    seeds = seeds or [wl.seed] * len(descs)
    cams = cams or [wl.camera] * len(descs)
    ctx.set_ray_sharing(share)
    items = [(sc, cam, f, wl.settings, count, sd) for sc, cam, f, sd in zip(scenes, cams, films, seeds)]
    if batch:
        render_batch(ctx, items)
    else:
        for it in items:
            render_pass(ctx, *it)
    out = [(f.xyz(), *f.read()[1:]) for f in films]
    ctx.set_ray_sharing(False)
    return out


def assert_films_equal(a, b):
    for (x1, a1, n1), (x2, a2, n2) in zip(a, b):
        assert np.array_equal(x1.view(np.uint32), x2.view(np.uint32))
        assert np.array_equal(a1.view(np.uint32), a2.view(np.uint32))
        assert np.array_equal(n1.view(np.uint32), n2.view(np.uint32))


@pytest.mark.gpu
def test_shared_batch_equals_renders_alone():
    """Three alloys of the ring, 256 x 256 x 8 spp, one wave: every film is
    bit for bit the variant's own render_pass, and the films differ."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    descs = variants(wl)
    alone = films_of(ctx, piece, descs, wl, 8, batch=False)
    shared = films_of(ctx, piece, descs, wl, 8, share=True)
    assert_films_equal(shared, alone)
    assert not np.array_equal(alone[0][0], alone[1][0])


@pytest.mark.gpu
def test_shared_batch_traces_fewer_rays():
    """With sharing, the three variants trace about a third of the closest
    and shadow rays (until Russian roulette parts their paths)."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    descs = variants(wl)
    counts = {}
    for share in (False, True):
        ctx.set_counting(True)
        films_of(ctx, piece, descs, wl, 8, share=share)
        counts[share] = ctx.traversal_counts()
        ctx.set_counting(False)
    print("traced rays without / with sharing:", counts[False], counts[True])
    assert counts[True]["closest_rays"] < 0.40 * counts[False]["closest_rays"]
    assert counts[True]["any_rays"] < 0.40 * counts[False]["any_rays"]


@pytest.mark.gpu
@pytest.mark.parametrize("wave_paths", [1 << 18, 1 << 17])
def test_shared_batch_over_many_waves_equals_renders_alone(wave_paths):
    """Waves of 2^18 (2^17) paths: alone each film takes two (four) waves of
    4 (2) samples per pixel; shared, the three renders take the same runs of
    samples per pixel on a third of the pixels per wave, so every film is
    still bit for bit its render alone."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still()
    ctx = Context(0, wave_paths=wave_paths)
    piece = Piece(ctx, wl.mesh)
    descs = variants(wl)
    alone = films_of(ctx, piece, descs, wl, 8, batch=False)
    shared = films_of(ctx, piece, descs, wl, 8, share=True)
    assert_films_equal(shared, alone)


@pytest.mark.gpu
def test_only_matching_renders_share():
    """A batch of the three alloys plus one with another seed, one at
    another turntable angle and one through another camera: the three share,
    the others are traced on their own, and every film is bit for bit its
    render alone."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    turned = wl.desc.c.turntable_deg + 10.0
    descs = variants(wl) + variants(wl, ("sterling",)) + variants(wl, ("bronze",), turn=turned) + \
        variants(wl, ("gold14k",))
    other_cam = W.shot(None, W.hull(wl.mesh), "top", 100.0, 0.0, 1.0)[0]
    seeds = [wl.seed] * 3 + [wl.seed + 1, wl.seed, wl.seed]
    cams = [wl.camera] * 5 + [other_cam]
    alone = films_of(ctx, piece, descs, wl, 8, seeds=seeds, cams=cams, batch=False)
    shared = films_of(ctx, piece, descs, wl, 8, seeds=seeds, cams=cams, share=True)
    assert_films_equal(shared, alone)


@pytest.mark.gpu
def test_sharing_off_is_the_default_and_leaves_batches_unchanged():
    """Sharing is off by default; turning it on and off again gives the
    unshared batch's films bit for bit."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    descs = variants(wl)
    a = films_of(ctx, piece, descs, wl, 4)
    films_of(ctx, piece, descs, wl, 4, share=True)
    b = films_of(ctx, piece, descs, wl, 4)
    assert_films_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("overlap", [False, True])
def test_served_variants_share_and_equal_their_renders_alone(overlap):
    """Served requests for three alloys of the same piece, size, samples and
    seed (argent's queue renders every job with seed 7, queue.rs:613) plus one
    of another size: with sharing on they are served together, and every
    result equals its render alone to float rounding."""
    from argent_b200.gpu import Context, Film, Piece, Scene, Serve, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scenes = [Scene(ctx, piece, d) for d in variants(wl)]
    cam = lambda w, h: W.shot(None, W.hull(wl.mesh), "hero", 100.0, 0.0, w / h)[0]  # noqa: E731
    reqs = [(0, 96, 96, 8), (1, 96, 96, 8), (2, 96, 96, 8), (1, 64, 128, 4)]
    ctx.set_ray_sharing(True)
    srv = Serve(ctx, step_path_samples=1 << 20, overlap=overlap)
    tickets = [srv.submit(scenes[i], cam(w, h), W.settings(8), w, h, spp, 7, 0) for i, w, h, spp in reqs]
    steps = 0
    while srv.step():
        steps += 1
        assert steps < 1000
    ctx.set_ray_sharing(False)
    for t, (i, w, h, spp) in zip(tickets, reqs):
        st = srv.poll(t)
        assert st.state == N.REQ_DONE and st.samples == spp
        c, a, n = srv.read(t)
        f = Film(ctx, w, h)
        render_pass(ctx, scenes[i], cam(w, h), f, W.settings(8), spp, 7)
        c0, a0, n0 = f.read()
        assert np.allclose(c, c0, rtol=1e-5, atol=1e-7)
        assert np.allclose(a, a0, rtol=1e-5, atol=1e-7)
        assert np.allclose(n, n0, rtol=1e-5, atol=1e-6)
    srv.close()


@pytest.mark.gpu
def test_groups_hold_at_most_sixteen_renders():
    """Seventeen variants (alloys repeated) of a 64 x 64 x 2 spp shot: a group
    of sixteen and one render alone, every film bit for bit its render
    alone."""
    from argent_b200.gpu import Context, Piece

    wl = W.ring_still(spp=2, width=64, height=64)
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    alloys = ("sterling", "gold14k", "rose14k", "bronze") * 4 + ("platinum",)
    descs = variants(wl, alloys)
    alone = films_of(ctx, piece, descs, wl, 2, batch=False)
    shared = films_of(ctx, piece, descs, wl, 2, share=True)
    assert_films_equal(shared, alone)
