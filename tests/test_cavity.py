"""Cavity (patina) mask: argent-mesh's known answers on the oracle
(crates/argent-mesh/src/cavity/tests.rs), the host halves of the product
against the oracle, and the device ambient occlusion and full mask against
the oracle."""

import numpy as np
import pytest

from argent_b200 import mesh as M
from argent_b200 import workloads as W


def height_field(n, f):
    """cavity/tests.rs:5-25: z = f(x) over [-5, 5]^2 with n x n quads."""
    f32 = np.float32
    pos = []
    for j in range(n + 1):
        for i in range(n + 1):
            x = f32(-5.0) + f32(10.0) * f32(i) / f32(n)
            y = f32(-5.0) + f32(10.0) * f32(j) / f32(n)
            pos.append([x, y, f(x)])
    idx = lambda i, j: j * (n + 1) + i
    tris = []
    for j in range(n):
        for i in range(n):
            tris.append([idx(i, j), idx(i + 1, j), idx(i + 1, j + 1)])
            tris.append([idx(i, j), idx(i + 1, j + 1), idx(i, j + 1)])
    return M.Mesh(np.array(pos, np.float32), np.array(tris, np.uint32))


def _groove_ridge_z(x):
    f32 = np.float32
    g = f32(-0.5) * max(f32(1.0) - abs(x + f32(3.0)) / f32(0.5), f32(0.0))
    r = f32(0.5) * max(f32(1.0) - abs(x - f32(3.0)) / f32(0.5), f32(0.0))
    return f32(g + r)


@pytest.fixture(scope="module")
def groove_ridge():
    """cavity/tests.rs:27-35: a 0.5 mm V-groove at x = -3 and a ridge at x = +3.
    argent's test gives it crease-split normals (normals::compute at 60 deg);
    here it carries the smooth vertex normals patina_mask falls back to."""
    m = height_field(200, _groove_ridge_z)
    m.normals = M.smooth_normals(m)
    return m


def value_near(m, vals, x, y):
    d = (m.positions[:, 0] - x) ** 2 + (m.positions[:, 1] - y) ** 2
    return vals[int(np.argmin(d))]


def test_oracle_groove_dark_ridge_bright(groove_ridge):
    """cavity/tests.rs:49-62."""
    import oracle as O

    m = groove_ridge
    mask = O.patina_mask(m, m.normals)
    assert mask.shape == (len(m.positions),)
    assert value_near(m, mask, -3.0, 0.0) > 0.6
    assert value_near(m, mask, 3.0, 0.0) < 0.05
    assert value_near(m, mask, 0.0, 0.0) < 0.1
    assert np.all((mask >= 0.0) & (mask <= 1.0))


def test_oracle_concavity_signs(groove_ridge):
    """cavity/tests.rs:64-77; the sphere is a UV sphere of radius 4 (argent
    uses an icosphere): H r = -r / R = -0.1 on average."""
    import oracle as O

    m = groove_ridge
    c = O.concavity(m, m.normals, 0.4)
    assert value_near(m, c, -3.0, 0.0) > 0.2
    assert value_near(m, c, 3.0, 0.0) < -0.2
    assert abs(value_near(m, c, 0.0, 0.0)) < 1e-3
    s = W.sphere(4.0, 96)
    cs = O.concavity(s, s.normals, 0.4)
    assert abs(cs.mean() + 0.1) < 0.02, cs.mean()


def split_cuboid(n, half=1.0):
    """A cube whose six faces are separate n x n grids, so every edge and
    corner vertex has copies at one position (what crease splitting makes of
    argent's subdivided_cuboid, cavity/tests.rs:113-114)."""
    pos, tris = [], []
    axes = [(0, 1, 2), (1, 2, 0), (2, 0, 1)]
    for a, b, c in axes:
        for side in (-1.0, 1.0):
            base = len(pos)
            for j in range(n + 1):
                for i in range(n + 1):
                    p = [0.0, 0.0, 0.0]
                    p[a] = -half + 2 * half * i / n
                    p[b] = -half + 2 * half * j / n
                    p[c] = side * half
                    pos.append(p)
            for j in range(n):
                for i in range(n):
                    q = base + j * (n + 1) + i
                    t1, t2 = [q, q + 1, q + n + 2], [q, q + n + 2, q + n + 1]
                    if side < 0:
                        t1, t2 = t1[::-1], t2[::-1]
                    tris += [t1, t2]
    return M.Mesh(np.array(pos, np.float32), np.array(tris, np.uint32))


def test_oracle_smoothing_preserves_constants_and_merges_copies():
    """cavity/tests.rs:111-129."""
    import oracle as O

    m = split_cuboid(4)
    v = O.smooth(m, np.full(len(m.positions), 0.7, np.float32), 5, 0.5)
    assert np.all(np.abs(v - 0.7) < 1e-6)
    spike = np.zeros(len(m.positions), np.float32)
    spike[0] = 1.0
    v = O.smooth(m, spike, 2, 0.5)
    _, inv = np.unique(m.positions, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    for g in np.unique(inv):
        assert len(set(v[inv == g].tolist())) == 1
    assert v[0] < 1.0 and np.count_nonzero(v > 0.0) > 3


def test_host_halves_match_oracle(groove_ridge):
    """The product's host concavity, smoothing and smooth normals against
    the oracle's restatement (no device needed)."""
    import oracle as O

    m = groove_ridge
    n_host, n_or = M.smooth_normals(m), O.smooth_vertex_normals(m)
    assert np.allclose(n_host, n_or, atol=1e-6)
    c_host, c_or = M.concavity(m, m.normals, 0.4), O.concavity(m, m.normals, 0.4)
    assert np.allclose(c_host, c_or, atol=1e-5)
    rng = np.random.default_rng(3)
    vals = rng.random(len(m.positions)).astype(np.float32)
    assert np.allclose(M.smooth(m, vals, 3), O.smooth(m, vals, 3), atol=1e-6)
    c = split_cuboid(6)
    spike = np.zeros(len(c.positions), np.float32)
    spike[5] = 1.0
    assert np.array_equal(M.smooth(c, spike, 4), O.smooth(c, spike, 4))


@pytest.mark.gpu
def test_gpu_ambient_occlusion_matches_oracle(groove_ridge):
    """Device AO (48 rays per vertex) against the oracle's AO on argent's BVH.
    Ray directions use CUDA's cosf/sinf against glibc's, so a ray grazing a
    triangle edge may flip: at most 2 of 48 rays per vertex may differ."""
    import oracle as O
    from argent_b200.gpu import Context, Piece

    m = groove_ridge
    ctx = Context(0)
    piece = Piece(ctx, m)
    ao = piece.ambient_occlusion(m.normals, 48, 1.2)
    ref = O.ambient_occlusion(m, m.normals, 48, 1.2)
    diff = np.abs(ao - ref)
    print("AO: vertices differing", np.count_nonzero(diff), "of", len(ao), "max", diff.max())
    assert diff.max() <= 2.0 / 48 + 1e-6
    assert np.count_nonzero(diff) <= 0.001 * len(ao)
    # raw occlusion (before patina_mask's contrast shaping): the groove
    # bottom sees its walls, the flat sees open sky
    assert value_near(m, ao, -3.0, 0.0) > 0.25 and value_near(m, ao, 0.0, 0.0) == 0.0


@pytest.mark.gpu
def test_gpu_patina_mask_matches_oracle():
    """The full mask on the ring workload's piece, with argent's
    Prepared::build settings for its radius."""
    import oracle as O
    from argent_b200.gpu import Context, Piece

    m = M.ring()
    radius, _ = W.piece_radius(m)
    st = M.patina_settings(radius)
    ctx = Context(0)
    piece = Piece(ctx, m)
    mask = piece.patina_mask(st)
    ref = O.patina_mask(m, m.normals, st.ao_samples, st.ao_distance, st.curvature_radius, st.concavity_weight,
                        st.smooth_iterations)
    d = np.abs(mask - ref)
    print("patina mask: max diff", d.max(), "mean", d.mean(), "mean mask", ref.mean())
    assert d.max() <= 0.05 and d.mean() <= 1e-3
