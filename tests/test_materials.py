"""Render parity for the materials the still, gems and reel workloads do not
reach: precious opal (Voronoi domains of Bragg lattices over a body,
material.rs:98-113, 208-237; bsdf.rs:83-94, 257), the patina layer of a
metal with a cavity mask (material.rs:115-122) and opaque gems (a polished
coat over a body colour, material.rs:126-131).  Each GPU render is compared
with the oracle's render of the same sample streams, relative RMSE per XYZ
channel at most 1 %."""

import numpy as np
import pytest

from argent_b200 import mesh as M
from argent_b200 import workloads as W

RELRMSE_TOL = 0.01  # per XYZ channel, GPU vs oracle at equal spp and seeds
OPAQUE_SIDE = ("onyx", "lapis", "obsidian", "turquoise")


def rel_rmse(img, ref):
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    return np.sqrt(((img - ref) ** 2).sum(0)) / np.sqrt((ref ** 2).sum(0))


def oracle_xyz(wl, want_normal=False):
    import oracle as O

    sc = O.Scene(wl.mesh, wl.desc.c)
    _, _, n, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed)
    return (xyz / wl.spp, n) if want_normal else xyz / wl.spp


def gpu_xyz(wl, ctx=None):
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    ctx = ctx or Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, wl.spp, wl.seed)
    return film.xyz()


def chroma_spread(xyz, where=None):
    """Spread of the chromaticity x over lit pixels (of `where`): opal's
    play of colour makes it large, a grey body alone small."""
    xyz = xyz.reshape(-1, 3)
    s = xyz.sum(1)
    lit = s > 1e-3 * s.max()
    if where is not None:
        lit &= where.reshape(-1)
    x = xyz[lit, 0] / s[lit]
    return float(np.percentile(x, 95) - np.percentile(x, 5))


def piece_pixels(normal):
    """Pixels whose first hit is the piece: a normal guide that is neither
    zero (background, panels) nor the floor's straight-up normal."""
    n = normal.reshape(-1, 3)
    return (np.abs(n).sum(1) > 0) & ~((np.abs(n[:, 0]) < 1e-6) & (np.abs(n[:, 2]) < 1e-6))


def small_gem_ring():
    return M.gem_ring(shank_nu=192, shank_nv=64)


def test_material_classes():
    """Opal shades in the 'other' class, opaque gems in the coated class
    (with plastic), transparent and opal-kind gems in the dielectric
    class: the host's class table and the material records agree."""
    from argent_b200 import _native as N

    assert W.opal(True).kind == N.MAT_OPAL and W.opal(False).kind == N.MAT_OPAL
    for g in OPAQUE_SIDE:
        m = W.gem(g)
        assert m.kind == N.MAT_GEM and m.gem_kind == N.GEM_OPAQUE and m.has_opaque_base
    assert W.gem("black_opal").kind == N.MAT_OPAL
    assert W.gem("ruby").gem_kind == N.GEM_TRANSPARENT


def test_oracle_opal_has_play_of_colour():
    """The oracle's opal is not a grey body: its lattice flashes spread the
    chromaticity far more than a white diffuse ring of the same shot."""
    wl = W.opal_still(black=True, spp=16, width=64, height=64)
    xyz, n = oracle_xyz(wl, want_normal=True)
    grey = W.opal_still(black=True, spp=16, width=64, height=64)
    grey.desc = W._studio_scene(grey.mesh, [W.diffuse([0.5, 0.5, 0.5])], "noir", 0.0)
    gxyz, gn = oracle_xyz(grey, want_normal=True)
    a, b = chroma_spread(xyz, piece_pixels(n)), chroma_spread(gxyz, piece_pixels(gn))
    print("chroma spread on the piece: opal", a, "grey", b)
    assert a > 2.0 * b


def test_oracle_patina_darkens_the_recesses():
    """With the cavity mask attached, the setting's recesses take the dark
    tarnish (material.rs:115-122); without it the metal stays polished."""
    import oracle as O

    m = small_gem_ring()
    radius, _ = W.piece_radius(m)
    st = M.patina_settings(radius)
    mask = O.patina_mask(m, m.normals, st.ao_samples, st.ao_distance, st.curvature_radius, st.concavity_weight,
                         st.smooth_iterations)
    metal_v = np.unique(m.tris[m.tri_material == 0])
    assert (mask[metal_v] > 0.18).mean() > 0.25  # the patina branch is reached
    a = oracle_xyz(W.gems_still(spp=4, width=54, height=96, mesh=W.with_cavity(m, mask)))
    b = oracle_xyz(W.gems_still(spp=4, width=54, height=96, mesh=m))
    assert a[..., 1].sum() < b[..., 1].sum()


@pytest.mark.gpu
@pytest.mark.parametrize("black", [False, True], ids=["white_opal", "black_opal"])
def test_opal_render_matches_oracle(black):
    """The ring carved from opal (cell 0.35 mm), 128 x 128, 8 spp."""
    wl = W.opal_still(black=black)
    got, ref = gpu_xyz(wl), oracle_xyz(wl)
    e = rel_rmse(got, ref)
    print(wl.name, "relRMSE XYZ vs oracle:", e, "chroma spread", chroma_spread(ref))
    assert np.all(e <= RELRMSE_TOL), e


@pytest.mark.gpu
def test_patina_render_matches_oracle():
    """The gems scene on a small setting whose cavity mask comes from the
    product's own patina_mask: the 18k slot's patina darkens the cups and
    gallery; 108 x 192, 8 spp, depth 32."""
    from argent_b200.gpu import Context, Piece

    m = small_gem_ring()
    ctx = Context(0)
    radius, _ = W.piece_radius(m)
    mask = Piece(ctx, m).patina_mask(M.patina_settings(radius))
    metal_v = np.unique(m.tris[m.tri_material == 0])
    assert (mask[metal_v] > 0.18).mean() > 0.25
    wl = W.gems_still(spp=8, width=108, height=192, mesh=W.with_cavity(m, mask))
    got, ref = gpu_xyz(wl, ctx), oracle_xyz(wl)
    plain = oracle_xyz(W.gems_still(spp=8, width=108, height=192, mesh=m))
    e = rel_rmse(got, ref)
    print("patina relRMSE XYZ vs oracle:", e, "patina vs polished", rel_rmse(ref, plain))
    assert np.all(e <= RELRMSE_TOL), e
    assert np.all(rel_rmse(ref, plain) > 2 * RELRMSE_TOL)  # the patina is visible


@pytest.mark.gpu
def test_opaque_gem_render_matches_oracle():
    """A turquoise centre stone with onyx, lapis, obsidian and turquoise
    side stones in the gems setting, 108 x 192, 8 spp, depth 32."""
    wl = W.gems_still(spp=8, width=108, height=192, center="turquoise", side=OPAQUE_SIDE)
    got, ref = gpu_xyz(wl), oracle_xyz(wl)
    e = rel_rmse(got, ref)
    print("opaque gems relRMSE XYZ vs oracle:", e)
    assert np.all(e <= RELRMSE_TOL), e
