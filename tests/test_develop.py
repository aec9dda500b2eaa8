"""Develop (tone map + dither + 8 bits): argent-post's known answers on the
oracle (crates/argent-post/src/tonemap.rs tests) and the device develop
against the oracle byte for byte."""

import numpy as np
import pytest

AGX, ACES, KHRONOS, REINHARD, CLAMP = range(5)
BASE, PUNCHY, GOLDEN = range(3)


def _luma(v):
    return 0.2126 * v[0] + 0.7152 * v[1] + 0.0722 * v[2]


def _hue(o):
    mx, mn = max(o), min(o)
    if mx - mn < 1e-3:
        return None
    d = mx - mn
    if mx == o[0]:
        return 60.0 * (((o[1] - o[2]) / d) % 6.0)
    if mx == o[1]:
        return 60.0 * ((o[2] - o[0]) / d + 2.0)
    return 60.0 * ((o[0] - o[1]) / d + 4.0)


def test_oracle_agx_black_and_mid_grey():
    """tonemap.rs `agx_black_and_mid_grey`."""
    import oracle as O

    black = O.tonemap_pixel([0, 0, 0], op=AGX, look=BASE)
    assert np.all(black < 1e-4)
    grey = O.tonemap_pixel([0.18] * 3, op=AGX, look=BASE)
    assert 0.45 <= O.srgb_encode(grey[1]) < 0.55
    assert abs(grey[0] - grey[2]) < 2e-3
    assert O.tonemap_pixel([0.18] * 3, op=AGX, look=PUNCHY)[1] < grey[1]
    golden = O.tonemap_pixel([0.18] * 3, op=AGX, look=GOLDEN)
    assert golden[0] > golden[1] > golden[2]


def test_oracle_agx_rolls_off_without_hue_clipping():
    """tonemap.rs `agx_rolls_off_without_hue_clipping`."""
    import oracle as O

    prev, sats = -1.0, []
    for e in range(-4, 15):
        k = 2.0 ** e
        o = O.tonemap_pixel([1.0 * k, 0.5 * k, 0.1 * k], op=AGX, look=BASE)
        assert np.all(np.isfinite(o)) and np.all((o >= 0) & (o <= 1))
        assert o[0] >= o[1] - 2e-3 and o[1] >= o[2] - 2e-3
        assert _luma(o) >= prev - 1e-5
        prev = _luma(o)
        h = _hue(o)
        if h is not None:
            assert 15.0 <= h <= 62.0
        sats.append((o[0] - o[2]) / max(o[0], 1e-6))
    for a, b in zip(sats[8:], sats[9:]):
        assert b <= a + 1e-3
    assert sats[-1] < 0.1
    assert np.all(O.tonemap_pixel([16.0, 8.0, 1.6], op=CLAMP) == 1.0)
    agx = O.tonemap_pixel([16.0, 8.0, 1.6], op=AGX, look=BASE)
    assert agx[0] - agx[2] > 0.15
    huge = O.tonemap_pixel([1e6, 2e5, 1e4], op=AGX, look=BASE)
    assert np.all((huge > 0.9) & (huge <= 1.0))


def test_oracle_other_operators_are_sane():
    """tonemap.rs `other_operators_are_sane`."""
    import oracle as O

    for op in (ACES, KHRONOS, REINHARD, CLAMP):
        assert np.all(np.abs(O.tonemap_pixel([0, 0, 0], op=op)) < 1e-3)
        hi = O.tonemap_pixel([50.0, 40.0, 30.0], op=op)
        assert np.all((hi >= 0) & (hi <= 1))
        assert np.all(np.isfinite(O.tonemap_pixel([np.nan, np.inf, -1.0], op=op)))
    assert abs(O.tonemap_pixel([0.18] * 3, op=ACES)[1] - 0.106) < 0.01
    kn = O.tonemap_pixel([0.5, 0.3, 0.2], op=KHRONOS)
    assert abs(kn[0] - 0.46) < 1e-3 and abs(kn[2] - 0.16) < 1e-3


def test_oracle_saturation_and_exposure():
    """tonemap.rs `saturation_and_exposure`."""
    import oracle as O

    assert abs(O.tonemap_pixel([1, 1, 1], ev=1.0, op=REINHARD)[0] - 2.0 / 3.0) < 1e-5
    o = O.tonemap_pixel([1.0, 0.2, 0.05], op=AGX, look=BASE, saturation=0.0)
    assert abs(o[0] - o[1]) < 2e-3 and abs(o[1] - o[2]) < 2e-3


def ramp_image(w=512, h=64):
    """tonemap.rs tests `test_image`: an exposure ramp over -10..+12 EV
    around 0.18, the hue varying down the rows."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    t = x / np.float32(w - 1)
    ev = np.float32(-10.0) + np.float32(22.0) * t
    c = np.float32(0.18) * np.power(np.float32(2.0), ev)
    hue = y / np.float32(h)
    return np.stack([c * (1 - hue), c * np.float32(0.6), c * hue], -1).astype(np.float32)


def test_oracle_fast_path_matches_exact():
    """tonemap.rs `fast_path_matches_exact`."""
    import oracle as O

    img = ramp_image(128, 16)
    for op, look in [(AGX, BASE), (AGX, PUNCHY), (AGX, GOLDEN), (ACES, 0), (KHRONOS, 0), (REINHARD, 0), (CLAMP, 0)]:
        _, enc = O.develop(img, 0.5, op, look, 1.2)
        worst = 0.0
        for p, e in zip(img.reshape(-1, 3), enc.reshape(-1, 3)):
            exact = O.tonemap_pixel(p, 0.5, op, look, 1.2)
            worst = max(worst, max(abs(e[c] - O.srgb_encode(exact[c])) for c in range(3)))
        assert worst < 2e-4, (op, look, worst)


def test_oracle_develop_dithers_and_keeps_extremes():
    """tonemap.rs `develop_dithers_and_keeps_extremes`."""
    import oracle as O

    img = np.zeros((4, 256, 3), np.float32)
    img[1] = 1e9
    img[2] = 0.18
    out, _ = O.develop(img, op=CLAMP)
    assert np.all(out[0] == 0) and np.all(out[1] == 255)
    row = out[2].astype(np.float32)
    assert abs(row.mean() - O.srgb_encode(0.18) * 255.0) < 0.15
    assert np.any(row != row.flat[0])


@pytest.mark.gpu
def test_gpu_develop_matches_oracle_bytes():
    """Every operator and look, with exposure and saturation, byte for byte."""
    import oracle as O
    from argent_b200 import _native as N
    from argent_b200.gpu import Context, develop

    ctx = Context(0)
    img = ramp_image(512, 64)
    img[0, :8] = [np.nan, np.inf, -1.0]
    for op, look, ev, sat in [(AGX, PUNCHY, 0.0, 1.0), (AGX, BASE, 0.5, 1.2), (AGX, GOLDEN, -1.0, 0.8),
                              (ACES, 0, 0.5, 1.2), (KHRONOS, 0, 0.0, 1.0), (REINHARD, 0, 1.0, 0.0), (CLAMP, 0, 0.0, 1.0)]:
        got = develop(ctx, img, N.ArgentGrade(ev, op, look, sat))
        ref, _ = O.develop(img, ev, op, look, sat)
        diff = np.count_nonzero(got != ref)
        print("develop op", op, "look", look, "bytes differing", diff)
        assert diff == 0


@pytest.mark.gpu
def test_film_develop_equals_steps():
    """argent_film_develop = film read -> a-trous -> develop, all on the device."""
    from argent_b200 import _native as N
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Film, Piece, Scene, denoise_atrous, develop, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, 4, wl.seed)
    g = N.ArgentGrade(0.0, AGX, PUNCHY, 1.0)
    c, a, n = film.read()
    assert np.array_equal(film.developed(g, denoise=False), develop(ctx, c, g))
    assert np.array_equal(film.developed(g, denoise=True), develop(ctx, denoise_atrous(ctx, c, a, n), g))
