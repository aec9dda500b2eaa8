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
