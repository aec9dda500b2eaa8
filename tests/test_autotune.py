"""argent_autotune: measures each (lanes, wave size) that fits, keeps the
fastest, and rendering afterwards still gives the same film."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_picks_the_fastest_and_keeps_results():
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still(width=512, height=512)
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    ref = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, ref, wl.settings, 16, wl.seed)
    res = ctx.autotune(scene, wl.camera, wl.settings, wl.width, wl.height, 16)
    print("autotune:", [(l, w, round(v / 1e6)) for l, w, v in res])
    assert len(res) >= 4
    best = max(res, key=lambda r: r[2])
    assert ctx.config() == (best[0], best[1])
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, 16, wl.seed)
    # different wave sizes group samples differently: FP32 sums differ by rounding only
    assert np.allclose(film.xyz(), ref.xyz(), rtol=1e-5, atol=1e-7)


def test_tuned_grids_render_bit_identical_films():
    """Blocks per SM of the shading classes and traversals change only how
    the queues' work is spread over the SMs: films are bit-identical to the
    default launch (same lanes and wave size)."""
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.gems_still(spp=4, width=108, height=192)
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    base = ctx.tuning()

    def render():
        f = Film(ctx, wl.width, wl.height)
        render_pass(ctx, scene, wl.camera, f, wl.settings, wl.spp, wl.seed)
        return f.xyz()

    want = render()
    for trace, shade in ((4, [2, 3, 8, 5, 6]), (6, [8, 2, 2, 3, 4]), (0, [1, 6, 4, 8, 2])):
        ctx.set_tuning(dict(base, trace_blocks_per_sm=trace, shade_blocks_per_sm=shade))
        assert ctx.tuning()["shade_blocks_per_sm"] == shade
        assert np.array_equal(render(), want)


def test_tuning_cache_round_trip(tmp_path):
    """argent_b200.tuning: the first call searches and caches the size
    class's tuning; a fresh context applies it from the cache."""
    from argent_b200 import tuning as T
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Piece, Scene

    wl = W.ring_still(width=256, height=256)
    path = str(tmp_path / "tune.json")
    ctx = Context(0)
    scene = Scene(ctx, Piece(ctx, wl.mesh), wl.desc)
    key, t, cached = T.tuned(ctx, scene, wl.camera, wl.settings, wl.width, wl.height, 8, path=path)
    assert not cached and key in T.load(path)
    ctx2 = Context(0)
    scene2 = Scene(ctx2, Piece(ctx2, wl.mesh), wl.desc)
    key2, t2, cached2 = T.tuned(ctx2, scene2, wl.camera, wl.settings, wl.width, wl.height, 8, path=path)
    assert cached2 and key2 == key and ctx2.tuning() == t
