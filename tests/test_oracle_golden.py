"""The oracle against argent's own unit-test known answers.

Each test names the argent test it restates (file:line in the argent tree).
These pin the CPU restatement before it is trusted as the parity reference.
"""

import ctypes
import math

import numpy as np
import pytest

import oracle as O


def f3(v):
    return (ctypes.c_float * 3)(*v)


def test_bvh_matches_brute_force():
    """bvh.rs:572-598 — 60x60 wavy grid, 2000 xorshift rays (seed 12345):
    4-wide traversal == binary traversal == brute force (|dt| < 1e-4), and
    occluded == brute force hit."""
    n = 60
    p = []
    for j in range(n + 1):
        for i in range(n + 1):
            x = np.float32(i) / np.float32(n) * np.float32(10.0) - np.float32(5.0)
            z = np.float32(j) / np.float32(n) * np.float32(10.0) - np.float32(5.0)
            y = np.float32(math.sin(np.float32(x * np.float32(0.7)))) * np.float32(math.cos(np.float32(z * np.float32(0.5))))
            p.append([x, y, z])
    w = n + 1
    t = []
    for j in range(n):
        for i in range(n):
            a = j * w + i
            t += [[a, a + 1, a + w], [a + 1, a + w + 1, a + w]]
    bvh = O.Bvh(np.array(p, np.float32), np.array(t, np.uint32))
    s = [12345]

    def rnd():
        x = s[0]
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        s[0] = x
        return np.float32(x) / np.float32(4294967295.0)

    rays = np.zeros((2000, 8), np.float32)
    for k in range(2000):
        o = [rnd() * np.float32(12) - np.float32(6), np.float32(4) + rnd() * np.float32(2), rnd() * np.float32(12) - np.float32(6)]
        d = np.array([rnd() - np.float32(0.5), np.float32(-1.0), rnd() - np.float32(0.5)], np.float32)
        d = d * (np.float32(1.0) / np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
        rays[k, 0:3] = o
        rays[k, 3] = np.inf
        rays[k, 4:7] = d
    a = bvh.intersect(rays)
    a2 = bvh.intersect_binary(rays)
    b = bvh.brute(rays)
    occ = bvh.occluded(rays)
    ah = a[:, 3].view(np.uint32) != 0xFFFFFFFF
    a2h = a2[:, 3].view(np.uint32) != 0xFFFFFFFF
    bh = b[:, 3].view(np.uint32) != 0xFFFFFFFF
    assert (ah == a2h).all()
    assert (ah == bh).all()
    assert np.all(np.abs(a[ah, 0] - b[ah, 0]) < 1e-4)
    assert (occ.astype(bool) == bh).all()
    assert ah.sum() > 500  # the grid is actually hit


def test_fresnel_known_answers():
    """fresnel.rs:122-148."""
    L = O.lib()
    assert abs(L.oracle_fresnel_dielectric(1.0, 1.5) - 0.04) < 1e-4
    assert L.oracle_fresnel_dielectric(-0.1, 1.5) == 1.0
    n, k = 0.2, 3.0
    expect = ((n - 1) ** 2 + k * k) / ((n + 1) ** 2 + k * k)
    assert abs(L.oracle_fresnel_conductor(1.0, n, k) - expect) < 1e-5
    assert L.oracle_fresnel_conductor(0.0, n, k) > 0.999


def test_microfacet_known_answers():
    """microfacet.rs:146-164."""
    L = O.lib()
    assert L.oracle_ggx_e(0.05, 0.8) > 0.97
    e = L.oracle_ggx_e(0.6, 0.5)
    assert 0.5 < e < 0.95
    wo = f3([0.6, 0.0, 0.8])
    h = (ctypes.c_float * 3)()
    for i in range(64):
        L.oracle_ggx_sample_h(0.3, wo, (i + 0.5) / 64.0, 0.37, h)
        assert h[2] > 0.0
        assert abs(math.sqrt(h[0] ** 2 + h[1] ** 2 + h[2] ** 2) - 1.0) < 1e-4


def test_visible_wavelengths():
    """spec.rs:226-245."""
    L = O.lib()
    lam = (ctypes.c_float * 4)()
    pdf = (ctypes.c_float * 4)()
    for i in range(1000):
        L.oracle_sample_visible((i + 0.5) / 1000.0, lam, pdf)
        for kk in range(4):
            assert 360.0 <= lam[kk] <= 830.0
            assert pdf[kk] > 0.0


def test_cie_known_answers():
    """cie.rs:199-211 and 261-271."""
    L = O.lib()
    out = (ctypes.c_float * 3)()
    L.oracle_xyz_bar(555.0, out)
    assert out[1] == 1.0
    L.oracle_xyz_bar(360.0, out)
    assert list(out) == [np.float32(0.0001299), np.float32(3.917e-6), np.float32(0.0006061)]
    L.oracle_xyz_bar(830.0, out)
    assert list(out) == [np.float32(1.251141e-6), np.float32(4.5181e-7), 0.0]
    L.oracle_xyz_bar(359.9, out)
    assert list(out) == [0.0, 0.0, 0.0]
    L.oracle_xyz_bar(float("nan"), out)
    assert list(out) == [0.0, 0.0, 0.0]
    # Monte Carlo luminance of a constant spectrum = 1 +- 2e-3 (4096 stratified u)
    lam = (ctypes.c_float * 4)()
    pdf = (ctypes.c_float * 4)()
    one = (ctypes.c_float * 4)(1, 1, 1, 1)
    xyz = (ctypes.c_float * 3)()
    y = 0.0
    for i in range(4096):
        L.oracle_sample_visible((i + 0.5) / 4096.0, lam, pdf)
        L.oracle_to_xyz(one, lam, pdf, xyz)
        y += xyz[1]
    assert abs(y / 4096.0 - 1.0) < 2e-3


def test_camera_matrix_d65_passthrough():
    """color.rs:66-79 (second half): D65 white passes XYZ->sRGB through."""
    L = O.lib()
    m = (ctypes.c_float * 9)()
    L.oracle_camera_matrix(1, f3([0.95047, 1.0, 1.08883]), m)
    m0 = (ctypes.c_float * 9)()
    L.oracle_camera_matrix(0, None, m0)
    v = np.array([0.3, 0.4, 0.5])
    a = np.array(m[:]).reshape(3, 3) @ v
    b = np.array(m0[:]).reshape(3, 3) @ v
    assert np.all(np.abs(a - b) < 1e-3)


def test_hash32_and_pcg_stream():
    """sampler.rs:18-25, 86-94: exact integer arithmetic."""
    L = O.lib()
    for x in [0, 1, 0xA511E9B3, 12345678, 0xFFFFFFFF]:
        h = x
        h ^= h >> 16
        h = (h * 0x7FEB352D) & 0xFFFFFFFF
        h ^= h >> 15
        h = (h * 0x846CA68B) & 0xFFFFFFFF
        h ^= h >> 16
        assert L.oracle_hash32(x) == h
    # PCG-XSH-RR stream of Sampler::next_random
    out = (ctypes.c_float * 8)()
    L.oracle_sampler_random(7, 3, 8, out)
    rng = ((7 << 32) | 3) ^ 0x9E3779B97F4A7C15
    for i in range(8):
        rng = (rng * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        x = (((rng >> 18) ^ rng) >> 27) & 0xFFFFFFFF
        rot = rng >> 59
        v = ((x >> rot) | (x << ((32 - rot) & 31))) & 0xFFFFFFFF
        assert out[i] == np.float32((v >> 8) * (1.0 / 16777216.0))


def test_sobol_nets():
    """The sampler's Sobol dimensions form (0, m, 2)-nets pairwise for
    dims (0,1), and every dimension is a (0, 1)-sequence: the first 2^m
    points of one padded 4D set, scrambled, put exactly one point in each of
    the 2^m elementary intervals (Burley 2020 preserves this)."""
    L = O.lib()
    out = (ctypes.c_float * 4)()
    m = 8
    n = 1 << m
    pts = np.zeros((n, 4))
    for i in range(n):
        L.oracle_sobol_4d(i, 3, 0xDEADBEEF, out)
        pts[i] = out[:]
    for dmn in range(4):
        cells = np.floor(pts[:, dmn] * n).astype(int)
        assert len(np.unique(cells)) == n
    for a in range(0, m + 1):
        b = m - a
        cx = np.floor(pts[:, 0] * (1 << a)).astype(int)
        cy = np.floor(pts[:, 1] * (1 << b)).astype(int)
        assert len(np.unique(cx * (1 << b) + cy)) == n, (a, b)


def test_tuning_size_class_keys():
    """The tuning cache key buckets triangles and path-samples by powers of
    two and names the scene's material kinds and env-map flag (CPU)."""
    from types import SimpleNamespace

    from argent_b200 import tuning as T
    from argent_b200 import workloads as W

    wl = W.ring_still()
    scene = SimpleNamespace(piece=SimpleNamespace(mesh=wl.mesh), desc=wl.desc)
    k = T.size_class(scene, 256, 256, 16)
    assert k.startswith("t16_p20_") and k.endswith("_e0")
    assert T.size_class(scene, 1920, 1080, 256) != k
