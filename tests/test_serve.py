"""Serving: requests rendered together by argent_serve_step give the films
they give alone (serve/queue.rs:611-613 relies on chunked passes continuing
the sample stream), urgent requests finish first, admission keeps films
within the budget, and cancellation stops a request between steps."""

import numpy as np
import pytest

from argent_b200 import _native as N
from argent_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring_setup():
    from argent_b200.gpu import Context, Piece, Scene

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    radius, floor_y = W.piece_radius(wl.mesh)
    scenes = {}
    for alloy in ("sterling", "gold14k"):
        desc = W._studio_scene(wl.mesh, [W.metal(alloy, 0.07, 0.8)], "noir", wl.desc.c.turntable_deg)
        scenes[alloy] = Scene(ctx, piece, desc)
    return ctx, piece, scenes, wl


def _alone(ctx, scene, cam, settings, w, h, spp, seed):
    from argent_b200.gpu import Film, render_pass

    f = Film(ctx, w, h)
    render_pass(ctx, scene, cam, f, settings, spp, seed)
    return f.read()


def _cam(wl, w, h):
    cam, _ = W.shot(None, W.hull(wl.mesh), "hero", 100.0, 0.0, w / h)
    return cam


@pytest.mark.parametrize("overlap", [False, True])
def test_mix_equals_alone(ring_setup, overlap):
    """Every request of a mix equals its standalone render, with batches run
    one at a time or two in flight."""
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    reqs = [("sterling", 64, 64, 4, 7, 0), ("gold14k", 128, 96, 16, 7, 1), ("sterling", 96, 160, 8, 3, 2),
            ("gold14k", 48, 48, 24, 1, 0)]
    # A small step budget splits every request into several chunks that
    # share batches with the others.
    srv = Serve(ctx, step_path_samples=40000, step_path_samples_max=40000, overlap=overlap)
    tickets = []
    for alloy, w, h, spp, seed, prio in reqs:
        tickets.append(srv.submit(scenes[alloy], _cam(wl, w, h), W.settings(8), w, h, spp, seed, prio))
    steps = 0
    while srv.step():
        steps += 1
        assert steps < 1000
    assert srv.stats()["steps"] > len(reqs)
    for t, (alloy, w, h, spp, seed, prio) in zip(tickets, reqs):
        st = srv.poll(t)
        assert st.state == N.REQ_DONE and st.samples == spp
        c, a, n = srv.read(t)
        c0, a0, n0 = _alone(ctx, scenes[alloy], _cam(wl, w, h), W.settings(8), w, h, spp, seed)
        assert np.allclose(c, c0, rtol=1e-5, atol=1e-7), (alloy, w, h)
        assert np.allclose(a, a0, rtol=1e-5, atol=1e-7)
        assert np.allclose(n, n0, rtol=1e-5, atol=1e-6)
    srv.close()


def test_urgent_requests_finish_first(ring_setup):
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    srv = Serve(ctx, step_path_samples=1 << 16)
    big = srv.submit(scenes["sterling"], _cam(wl, 256, 256), W.settings(8), 256, 256, 32, 7, priority=2)
    srv.step()  # the big request starts alone
    small = srv.submit(scenes["gold14k"], _cam(wl, 64, 64), W.settings(8), 64, 64, 4, 7, priority=0)
    srv.run()
    sb, ss = srv.poll(big), srv.poll(small)
    assert sb.state == N.REQ_DONE and ss.state == N.REQ_DONE
    assert ss.t_done < sb.t_done
    # the preview needed one step once admitted
    assert ss.t_done - ss.t_start < sb.t_done - sb.t_start
    srv.release(big)
    srv.release(small)


def test_admission_keeps_films_within_budget(ring_setup):
    """A finished film stays the request's until it is read, so with room
    for one film the requests run one after another."""
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    w, h = 128, 128
    film = 3 * w * h * 16  # Kahan film bytes
    srv = Serve(ctx, film_budget=film + film // 2, step_path_samples=1 << 15)
    ts = [srv.submit(scenes["sterling"], _cam(wl, w, h), W.settings(8), w, h, 4, 7 + i) for i in range(3)]
    read, order = set(), []
    for _ in range(100):
        pending = srv.step()
        assert srv.stats()["film_bytes_in_use"] <= film + film // 2
        assert sum(srv.poll(t).state == N.REQ_ACTIVE for t in ts if t not in read) <= 1
        for t in ts:
            if t not in read and srv.poll(t).state == N.REQ_DONE:
                srv.read(t)
                read.add(t)
                order.append(t)
        if not pending:
            break
    assert order == ts
    # one film alone over the budget is refused at submission
    with pytest.raises(N.ArgentError):
        srv.submit(scenes["sterling"], _cam(wl, 512, 512), W.settings(8), 512, 512, 4, 7)


def test_cancel_between_steps(ring_setup):
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    srv = Serve(ctx, step_path_samples=1 << 14)
    t = srv.submit(scenes["sterling"], _cam(wl, 128, 128), W.settings(8), 128, 128, 64, 7)
    srv.step()
    done_before = srv.poll(t).samples
    assert 0 < done_before < 64
    srv.cancel(t)
    assert srv.step() == 0
    st = srv.poll(t)
    assert st.state == N.REQ_CANCELLED and st.samples == done_before
    with pytest.raises(N.ArgentError):
        srv.read(t)
    srv.release(t)


def test_submission_refuses_foreign_scenes_and_deep_paths(ring_setup):
    """A request whose scene belongs to another context, or whose path depth
    exceeds 64, is refused when submitted, not when its batch runs."""
    from argent_b200.gpu import Context, Piece, Scene, Serve

    ctx, _, scenes, wl = ring_setup
    other = Context(0)
    foreign = Scene(other, Piece(other, wl.mesh), wl.desc)
    srv = Serve(ctx)
    with pytest.raises(N.ArgentError):
        srv.submit(foreign, _cam(wl, 64, 64), W.settings(8), 64, 64, 4, 7)
    with pytest.raises(N.ArgentError):
        srv.submit(scenes["sterling"], _cam(wl, 64, 64), W.settings(65), 64, 64, 4, 7)
    t = srv.submit(scenes["sterling"], _cam(wl, 64, 64), W.settings(8), 64, 64, 4, 7)
    srv.run()
    assert srv.poll(t).state == N.REQ_DONE
    srv.release(t)
    srv.close()


def test_bounded_queue_refuses_beyond_max_pending(ring_setup):
    """With max_pending = 3, a fourth request waiting or rendering is
    refused with E_BUSY (argent's queue refuses a job once 24 wait,
    queue.rs:364-366); once one finishes, a new submit is accepted."""
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    srv = Serve(ctx, max_pending=3)
    cam = _cam(wl, 32, 32)
    tickets = [srv.submit(scenes["sterling"], cam, W.settings(8), 32, 32, 2, 7, 0) for _ in range(3)]
    with pytest.raises(N.ArgentError) as e:
        srv.submit(scenes["sterling"], cam, W.settings(8), 32, 32, 2, 7, 0)
    assert e.value.code == N.E_BUSY
    srv.run()
    for t in tickets:
        assert srv.poll(t).state == N.REQ_DONE
        srv.read(t)
    t = srv.submit(scenes["gold14k"], cam, W.settings(8), 32, 32, 2, 7, 0)
    srv.run()
    assert srv.poll(t).state == N.REQ_DONE


def test_serve_after_autotune():
    """argent_autotune renders on the context with other lane counts and
    wave sizes and frees the lanes it does not keep; a serve on the same
    context afterwards (overlapped batches) renders every request."""
    from argent_b200.gpu import Context, Piece, Scene, Serve

    wl = W.ring_still()
    ctx = Context(0)
    scene = Scene(ctx, Piece(ctx, wl.mesh), wl.desc)
    ctx.autotune(scene, wl.camera, wl.settings, 256, 256, 4)
    t = ctx.tuning()
    ctx.set_tuning(dict(t, lanes=8, wave_paths=1 << 22))
    srv = Serve(ctx, overlap=True, step_path_samples=1 << 17)
    ts = [srv.submit(scene, _cam(wl, w, h), W.settings(8), w, h, spp, 7, prio)
          for w, h, spp, prio in ((64, 64, 4, 0), (256, 256, 16, 1), (128, 96, 8, 2))]
    srv.run()
    for t in ts:
        assert srv.poll(t).state == N.REQ_DONE
        srv.read(t)


def test_work_bound_refuses_beyond_max_pending_path_samples(ring_setup):
    """max_pending_path_samples bounds the work not yet rendered: a request
    that would take it past the bound is refused; one whose priority level
    has nothing pending is taken whatever its size."""
    from argent_b200.gpu import Serve

    ctx, _, scenes, wl = ring_setup
    cam = _cam(wl, 64, 64)
    srv = Serve(ctx, max_pending_path_samples=64 * 64 * 12)
    big = srv.submit(scenes["sterling"], cam, W.settings(8), 64, 64, 32, 7, 0)  # above the bound, nothing pending
    with pytest.raises(N.ArgentError) as e:
        srv.submit(scenes["sterling"], cam, W.settings(8), 64, 64, 1, 7, 0)
    assert e.value.code == N.E_BUSY
    srv.run()
    srv.read(big)
    a = srv.submit(scenes["sterling"], cam, W.settings(8), 64, 64, 8, 7, 0)
    b = srv.submit(scenes["gold14k"], cam, W.settings(8), 64, 64, 4, 7, 0)  # 12 samples of work in all: fits
    with pytest.raises(N.ArgentError):
        srv.submit(scenes["gold14k"], cam, W.settings(8), 64, 64, 1, 7, 0)
    # another priority level with nothing pending is taken past the bound
    c = srv.submit(scenes["gold14k"], cam, W.settings(8), 64, 64, 16, 7, 2)
    with pytest.raises(N.ArgentError):
        srv.submit(scenes["gold14k"], cam, W.settings(8), 64, 64, 1, 7, 2)
    srv.run()
    assert all(srv.poll(t).state == N.REQ_DONE for t in (a, b, c))
