"""À-trous denoise: argent-post's known answers on the oracle
(crates/argent-post/src/denoise.rs:713-800 tests), the device filter against
the oracle, and the film hand-off against a host round trip."""

import numpy as np
import pytest


def _hash(x):
    x = np.uint32(x)
    with np.errstate(over="ignore"):
        x ^= x >> np.uint32(16)
        x = np.uint32(x * np.uint32(0x7FEB352D))
        x ^= x >> np.uint32(15)
        x = np.uint32(x * np.uint32(0x846CA68B))
        x ^= x >> np.uint32(16)
    return x


def _gauss(i):
    """denoise.rs tests: a deterministic standard normal sample per index."""
    i = np.asarray(i, np.uint32)
    with np.errstate(over="ignore"):
        u1 = (_hash(i * np.uint32(2)).astype(np.float32) + np.float32(1.0)) / np.float32(4294967296.0)
        u2 = _hash(i * np.uint32(2) + np.uint32(1)).astype(np.float32) / np.float32(4294967296.0)
    return (np.sqrt(np.float32(-2.0) * np.log(u1)) * np.cos(np.float32(2 * np.pi) * u2)).astype(np.float32)


def gradient(w, h, sigma):
    """denoise.rs tests `gradient`: smooth colour ramp plus Gaussian noise,
    flat albedo 0.8 and normal +z."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    t = x / np.float32(w - 1)
    u = y / np.float32(h - 1)
    clean = np.stack([0.1 + 0.8 * t, 0.2 + 0.5 * u, 0.6 - 0.4 * t], -1).astype(np.float32)
    idx = ((np.arange(h)[:, None] * w + np.arange(w)[None, :]) * 3).astype(np.uint32)
    n = np.stack([_gauss(idx), _gauss(idx + 1), _gauss(idx + 2)], -1)
    noisy = np.maximum(clean + np.float32(sigma) * n, 0.0).astype(np.float32)
    albedo = np.full_like(clean, 0.8)
    normal = np.zeros_like(clean)
    normal[..., 2] = 1.0
    return clean, noisy, albedo, normal


def mse(a, b):
    return float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))


def edges_scene():
    """denoise.rs tests `atrous_keeps_material_edges`: two materials meet at x = 64."""
    w, h = 128, 96
    v = np.where(np.arange(w) < 64, 0.2, 0.8).astype(np.float32)
    clean = np.broadcast_to(v[None, :, None], (h, w, 3)).astype(np.float32).copy()
    idx = ((np.arange(h)[:, None] * w + np.arange(w)[None, :]) * 3).astype(np.uint32)
    noise = np.stack([_gauss(idx), _gauss(idx + 1), _gauss(idx + 2)], -1)
    noisy = (clean + np.float32(0.05) * noise).astype(np.float32)
    return clean, noisy, clean.copy()


def band_mse(img, clean):
    return float(np.mean((img[:, 61:67].astype(np.float64) - clean[:, 61:67]) ** 2))


def test_oracle_atrous_reduces_mse():
    """denoise.rs `atrous_reduces_mse`."""
    import oracle as O

    clean, noisy, albedo, normal = gradient(256, 192, 0.08)
    for a, n in [(None, None), (albedo, normal)]:
        out = O.atrous(noisy, a, n)
        assert mse(out, clean) < 0.15 * mse(noisy, clean)


def test_oracle_atrous_keeps_material_edges():
    """denoise.rs `atrous_keeps_material_edges`."""
    import oracle as O

    clean, noisy, albedo = edges_scene()
    out = O.atrous(noisy, albedo)
    assert band_mse(out, clean) < 0.5 * band_mse(noisy, clean)


@pytest.mark.gpu
def test_gpu_atrous_matches_oracle():
    """The device filter against the oracle on argent's test images.  They
    differ only through expf (CUDA against glibc), which moves the edge-stop
    weights by ulps."""
    import oracle as O
    from argent_b200.gpu import Context, denoise_atrous

    ctx = Context(0)
    clean, noisy, albedo, normal = gradient(256, 192, 0.08)
    for a, n in [(None, None), (albedo, None), (albedo, normal)]:
        got = denoise_atrous(ctx, noisy, a, n)
        ref = O.atrous(noisy, a, n)
        err = np.abs(got - ref).max()
        print("atrous gradient aux", a is not None, n is not None, "max |gpu - oracle|", err)
        assert err < 1e-4
        assert mse(got, clean) < 0.15 * mse(noisy, clean)
    c2, n2, a2 = edges_scene()
    got = denoise_atrous(ctx, n2, a2)
    assert np.abs(got - O.atrous(n2, a2)).max() < 1e-4
    assert band_mse(got, c2) < 0.5 * band_mse(n2, c2)


@pytest.mark.gpu
def test_film_denoise_equals_host_round_trip():
    """argent_film_denoise (averages stay on the device) gives what reading
    the film and denoising the host images gives."""
    from argent_b200 import workloads as W
    from argent_b200.gpu import Context, Film, Piece, Scene, denoise_atrous, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, 4, wl.seed)
    c, a, n = film.read()
    assert np.array_equal(film.denoised(), denoise_atrous(ctx, c, a, n))
