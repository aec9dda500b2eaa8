"""Render parity: argent's furnace known answers (tests/furnace.rs) on the
oracle and on the GPU, and GPU renders against the oracle on the same
sample streams (relative RMSE per XYZ channel <= 1 %)."""

import numpy as np
import pytest

from argent_b200 import workloads as W

RELRMSE_TOL = 0.01  # per XYZ channel, GPU vs oracle at equal spp and seeds


def rel_rmse(img, ref):
    """sqrt(sum (I - O)^2) / sqrt(sum O^2) per channel over the film."""
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    return np.sqrt(((img - ref) ** 2).sum(0)) / np.sqrt((ref ** 2).sum(0))


FURNACE = {
    # name: (material factory, check)
    "white_environment_is_white": (lambda: W.diffuse([0.8, 0.8, 0.8]), "bg"),
    "grey_diffuse_sphere_reflects_its_albedo": (lambda: W.diffuse([0.5, 0.5, 0.5]), "grey"),
    "clear_glass_sphere_conserves_energy": (lambda: W.gem("glass"), "vanish05"),
    "diamond_sphere_conserves_energy": (lambda: W.gem("diamond"), "vanish06"),
}


def check_furnace(kind, center, bg):
    """furnace.rs:60-95."""
    if kind == "bg":
        assert np.all(np.abs(bg - 1.0) < 0.03), bg
    elif kind == "grey":
        assert np.all(np.abs(center - 0.5) < 0.04), center
    elif kind == "vanish05":
        assert np.all(np.abs(center - bg) < 0.05), (center, bg)
    else:
        assert np.all(np.abs(center - bg) < 0.06), (center, bg)


@pytest.mark.parametrize("name", sorted(FURNACE))
def test_oracle_furnace(name):
    """The oracle reproduces argent's furnace tests (rows 1 and 32 only)."""
    import oracle as O

    mat, kind = FURNACE[name]
    wl = W.furnace(mat())
    sc = O.Scene(wl.mesh, wl.desc.c)
    out = np.zeros((64, 64, 3), np.float32)
    for y in (1, 32):
        c, _, _, _ = sc.render_pass(wl.camera, wl.settings, 64, 64, 0, 256, 1, rows=(y, y + 1), want_xyz=False)
        out[y] = c[y] / 256.0
    check_furnace(kind, out[32, 32], out[1, 1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FURNACE))
def test_gpu_furnace(name):
    """argent's furnace tests on the CUDA path through the C ABI."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    mat, kind = FURNACE[name]
    wl = W.furnace(mat())
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, 64, 64)
    render_pass(ctx, scene, wl.camera, film, wl.settings, 256, 1)
    img = film.color()
    check_furnace(kind, img[32, 32], img[1, 1])


def _gpu_render(wl, spp=None, flags=1, chunks=None):
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height, flags)
    spp = spp or wl.spp
    for c in (chunks or [spp]):
        render_pass(ctx, scene, wl.camera, film, wl.settings, c, wl.seed)
    assert film.samples == spp
    return film.xyz(), film.read(), ctx


@pytest.mark.gpu
def test_ring_render_matches_oracle():
    """The small plain workload at full size: 256x256, 16 spp, depth 8."""
    import oracle as O

    wl = W.ring_still()
    xyz_gpu, (color, albedo, normal), ctx = _gpu_render(wl)
    sc = O.Scene(wl.mesh, wl.desc.c)
    c, a, n, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed)
    ref = xyz / wl.spp
    e = rel_rmse(xyz_gpu, ref)
    print("ring_still relRMSE XYZ vs oracle:", e, "mean Y gpu/oracle", xyz_gpu[..., 1].mean(), ref[..., 1].mean())
    assert np.all(e <= RELRMSE_TOL), e
    # camera RGB and the guides agree too
    assert np.all(rel_rmse(color, c / wl.spp) <= RELRMSE_TOL)
    assert np.all(rel_rmse(albedo, a / wl.spp) <= RELRMSE_TOL)
    assert ctx.kernel_launches > 0


@pytest.mark.gpu
def test_chunked_passes_continue_the_sample_stream():
    """render.rs:70,86: film.samples is the next sample index, so 2 x 8 spp
    equals 16 spp (serve/queue.rs:611-612 relies on it)."""
    wl = W.ring_still()
    a, _, _ = _gpu_render(wl, 16)
    b, _, _ = _gpu_render(wl, 16, chunks=[8, 8])
    assert np.allclose(a, b, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_fp64_film_matches_kahan_film():
    wl = W.ring_still()
    a, _, _ = _gpu_render(wl, 16, flags=1)
    b, _, _ = _gpu_render(wl, 16, flags=3)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_batch_equals_separate_passes():
    from argent_b200.gpu import Context, Film, Piece, Scene, render_batch, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    f1, f2, g1, g2 = (Film(ctx, wl.width, wl.height) for _ in range(4))
    render_pass(ctx, scene, wl.camera, f1, wl.settings, 8, 7)
    render_pass(ctx, scene, wl.camera, f2, wl.settings, 8, 11)
    render_batch(ctx, [(scene, wl.camera, g1, wl.settings, 8, 7), (scene, wl.camera, g2, wl.settings, 8, 11)])
    assert np.array_equal(f1.xyz(), g1.xyz())
    assert np.array_equal(f2.xyz(), g2.xyz())
    assert not np.array_equal(f1.xyz(), f2.xyz())


@pytest.mark.gpu
def test_batch_items_sharing_a_film_equal_sequential_passes():
    """Two items of one batch render into the same film (3 then 5 samples):
    the film equals two render_pass calls in a row bit for bit.  The second
    item's pixels never share a wave with the first's, since the film pass
    adds a segment's sums without atomics."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_batch, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    f, g = Film(ctx, wl.width, wl.height), Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, f, wl.settings, 3, 7)
    render_pass(ctx, scene, wl.camera, f, wl.settings, 5, 7)
    render_batch(ctx, [(scene, wl.camera, g, wl.settings, 3, 7), (scene, wl.camera, g, wl.settings, 5, 7)])
    assert f.samples == g.samples == 8
    assert np.array_equal(f.xyz().view(np.uint32), g.xyz().view(np.uint32))


@pytest.mark.gpu
def test_gems_render_matches_oracle():
    """The gems workload (diamond + ruby/sapphire/emerald/garnet in an 18k
    setting, white studio, depth 32) at reduced size: 108 x 192, 8 spp."""
    import oracle as O

    wl = W.gems_still(spp=8, width=108, height=192)
    xyz_gpu, _, _ = _gpu_render(wl)
    sc = O.Scene(wl.mesh, wl.desc.c)
    _, _, _, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed)
    e = rel_rmse(xyz_gpu, xyz / wl.spp)
    print("gems_still 108x192x8 relRMSE XYZ vs oracle:", e)
    assert np.all(e <= RELRMSE_TOL), e


@pytest.mark.gpu
def test_signet_render_matches_oracle_on_a_band():
    """The bench workload itself (2.1M triangles, thin lens, two metal slots)
    on rows 500..520 of the 1920 x 1080 frame at 8 spp."""
    import oracle as O
    from argent_b200 import mesh as M
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    m = M.signet()
    ctx = Context(0)
    piece = Piece(ctx, m)
    wl = W.signet_still(piece, spp=8, mesh=m)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, film, wl.settings, wl.spp, wl.seed)
    xyz_gpu = film.xyz()
    sc = O.Scene(m, wl.desc.c)
    _, _, _, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed, rows=(500, 520))
    e = rel_rmse(xyz_gpu[500:520], xyz[500:520] / wl.spp)
    print("signet_still rows 500..520 x 8 spp relRMSE XYZ vs oracle:", e)
    assert np.all(e <= RELRMSE_TOL), e


@pytest.mark.gpu
def test_reel_batch_matches_oracle():
    """The batched workload's scenes (HDRI map plus panels, env_pick 0.5,
    turntable frames, two alloys) through one render_batch at 108 x 192 and
    8 spp; each film against the oracle's render of the same frame."""
    import oracle as O
    from argent_b200.gpu import Context, Film, Piece, Scene, render_batch

    m = W.reel_piece("61k")
    env = W.hdri()
    wls = W.reel_batch({"61k": m}, alloys=("sterling", "bronze"), frames=[0, 9], width=108, height=192, spp=8,
                       env_rgb=env)
    ctx = Context(0)
    piece = Piece(ctx, m)
    scenes = [Scene(ctx, piece, wl.desc) for wl in wls]
    films = [Film(ctx, wl.width, wl.height) for wl in wls]
    render_batch(ctx, [(sc, wl.camera, f, wl.settings, wl.spp, wl.seed) for sc, wl, f in zip(scenes, wls, films)])
    for wl, f in zip(wls, films):
        sc = O.Scene(m, wl.desc.c)
        _, _, _, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, wl.spp, wl.seed)
        e = rel_rmse(f.xyz(), xyz / wl.spp)
        print(wl.name, "relRMSE XYZ vs oracle:", e)
        assert np.all(e <= RELRMSE_TOL), (wl.name, e)


def test_band_camera_maps_band_rows_to_frame_rows():
    """workloads.band_camera: the centre of band pixel (x, r) looks along the
    ray of frame pixel (x, y0 + r), pinhole and thin lens."""
    wl = W.signet_still(spp=1, mesh=W.M.Mesh(np.array([[-5, -5, -5], [5, 5, 5], [5, -5, 5]], np.float32),
                                             np.array([[0, 1, 2]], np.uint32)))
    cam = wl.camera
    cam.lens_radius = 1.5
    cam.focus_dist = 90.0
    cam.shift[1] = 0.1
    H, w, y0, y1 = wl.height, wl.width, 500, 516
    band = W.band_camera(cam, H, y0, y1)
    for x, r in [(0, 0), (w // 2, 7), (w - 1, 15)]:
        sx = ((x + 0.5) * (2.0 / w)) - 1.0
        sy_f = 1.0 - ((y0 + r + 0.5) * (2.0 / H))
        sy_b = 1.0 - ((r + 0.5) * (2.0 / (y1 - y0)))
        for lu, lv in [(0.5, 0.5), (0.1, 0.8)]:
            of, df = W.camera_ray(cam, sx, sy_f, lu, lv)
            ob, db = W.camera_ray(band, sx, sy_b, lu, lv)
            assert np.allclose(of, ob, atol=1e-5) and np.allclose(df, db, atol=1e-6)


@pytest.mark.gpu
def test_band_camera_renders_the_same_rows():
    """A band rendered through band_camera converges to the same rows of the
    full frame (and not to rows 8 lower)."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    full = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, full, wl.settings, 4096, wl.seed)
    y0, y1 = 96, 112
    band = Film(ctx, wl.width, y1 - y0, 2)
    render_pass(ctx, scene, W.band_camera(wl.camera, wl.height, y0, y1), band, wl.settings, 4096, 99)
    f, b = full.xyz(), band.xyz()
    e = rel_rmse(b, f[y0:y1])
    e_off = rel_rmse(b, f[y0 + 8:y1 + 8])
    print("band vs frame rows relRMSE", e, "8 rows off", e_off)
    assert np.all(e < 0.05) and np.all(3 * e < e_off), (e, e_off)


@pytest.mark.gpu
def test_bounce_counts_add_up_to_the_traversal_counts():
    """Instrumentation: paths entering bounce 0 = path-samples; the queues
    shrink with depth; their sums equal the rays the traversals counted."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    film = Film(ctx, wl.width, wl.height)
    ctx.set_counting(True)
    render_pass(ctx, scene, wl.camera, film, wl.settings, 4, wl.seed)
    act, sh = ctx.bounce_counts()
    tc = ctx.traversal_counts()
    ctx.set_counting(False)
    print("paths per bounce", act, "shadow rays per bounce", sh)
    assert act[0] == wl.width * wl.height * 4
    assert all(b <= a for a, b in zip(act, act[1:]))
    assert len(act) <= wl.settings.max_depth
    assert sum(act) == tc["closest_rays"] and sum(sh) == tc["any_rays"]


@pytest.mark.gpu
def test_progressive_film_switches_to_fp64_past_4096_samples():
    """ARGENT_FILM_PROGRESSIVE: FP32 Kahan sums up to 4096 samples (equal to
    a Kahan film bit for bit), FP64 sums once a pass goes past them, seeded
    from the FP32 sums (equal to an FP64 film to the FP32 rounding of the
    first 4000 samples)."""
    from argent_b200 import _native as N
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still(width=64, height=64)
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    prog = Film(ctx, 64, 64, N.FILM_KAHAN | N.FILM_PROGRESSIVE)
    kahan = Film(ctx, 64, 64, N.FILM_KAHAN)
    fp64 = Film(ctx, 64, 64, N.FILM_FP64)
    for f in (prog, kahan, fp64):
        render_pass(ctx, scene, wl.camera, f, wl.settings, 4000, wl.seed)
    assert np.array_equal(prog.xyz(), kahan.xyz())
    for f in (prog, kahan, fp64):
        render_pass(ctx, scene, wl.camera, f, wl.settings, 200, wl.seed)
    assert prog.samples == 4200
    # The FP64 sums start from the compensated FP32 sums of the first 4000
    # samples, whose per-wave partial sums round in FP32 (about 1e-5).
    a, b = prog.xyz(), fp64.xyz()
    assert np.allclose(a, b, rtol=1e-4, atol=1e-8), np.abs(a - b).max()
    assert np.allclose(a, kahan.xyz(), rtol=1e-4, atol=1e-8)


@pytest.mark.gpu
def test_graph_replay_equals_direct_launches():
    """A repeated render replays its captured graph (new films, same waves);
    every film equals the one rendered with graphs off, bit for bit."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_pass

    wl = W.ring_still()
    ctx = Context(0)
    piece = Piece(ctx, wl.mesh)
    scene = Scene(ctx, piece, wl.desc)
    ctx.set_graphs(False)
    ref = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, ref, wl.settings, 8, wl.seed)
    want = ref.xyz()
    ctx.set_graphs(True)
    n0 = ctx.kernel_launches
    for _ in range(3):
        f = Film(ctx, wl.width, wl.height)
        render_pass(ctx, scene, wl.camera, f, wl.settings, 8, wl.seed)
        assert np.array_equal(f.xyz(), want)
    per = (ctx.kernel_launches - n0) // 3
    assert per > 0 and ctx.kernel_launches - n0 == 3 * per
    # a different seed changes only the job record: the graph replays it
    g = Film(ctx, wl.width, wl.height)
    render_pass(ctx, scene, wl.camera, g, wl.settings, 8, wl.seed + 1)
    assert not np.array_equal(g.xyz(), want)


@pytest.mark.gpu
def test_graph_keys_keep_map_and_gradient_waves_apart():
    """Waves whose scenes have no env map shade with kernels that leave the
    map code out.  Two small renders share one wave (so the wave names no
    single scene); a batch of two gradient-studio scenes and then a batch of
    two env-map scenes of the same piece, materials, panels and sizes give
    the same waves, and the second must not replay the first's graph: every
    film equals its render with graphs off, bit for bit."""
    from argent_b200.gpu import Context, Film, Piece, Scene, render_batch

    m = W.reel_piece("61k")
    env = W.hdri(256, 128)
    radius, floor_y = W.piece_radius(m)
    cam, _ = W.turntable_camera(W.hull(m), aspect=1.0)
    ps = W.settings(8)

    def descs(with_map):
        out = []
        for alloy in ("sterling", "bronze"):
            if with_map:
                out.append(W.reel_scene(m, alloy, env, 30.0))
                continue
            panels, grad, fm, fl, white = W.studio("noir", radius, floor_y)
            mats = [W.metal(alloy, 0.05, 0.8), W.metal(alloy, 0.35, 0.8), fm]
            fl.material = len(mats) - 1
            out.append(W.SceneDesc(mats, panels, grad, fl, 30.0, white))
        return out

    ctx = Context(0)
    piece = Piece(ctx, m)
    batches = [[Scene(ctx, piece, d) for d in descs(with_map)] for with_map in (False, True)]

    def render(scenes):
        films = [Film(ctx, 64, 64) for _ in scenes]
        render_batch(ctx, [(sc, cam, f, ps, 4, 7) for sc, f in zip(scenes, films)])
        return [f.xyz() for f in films]

    ctx.set_graphs(False)
    want = [render(b) for b in batches]
    ctx.set_graphs(True)
    for _ in range(2):
        for b, w in zip(batches, want):
            for got, ref in zip(render(b), w):
                assert np.array_equal(got, ref)
    assert not np.array_equal(want[0][0], want[1][0])


@pytest.mark.gpu
def test_fp64_oracle_film_matches_cpu_restatement_at_c1():
    """The FP64 oracle the benchmark scores renders against runs on the
    device; cross-check it against argent's algorithm on the host: the small
    plain workload at full size (256 x 256, depth 8) at 256 spp through an
    FP64 film, against the CPU restatement's FP64 sums of the same sample
    streams.  Both accumulate in double, so what is left is the
    transcendental functions' last bits flipping a rare path."""
    import oracle as O
    from argent_b200 import _native as N

    wl = W.ring_still()
    xyz_gpu, _, _ = _gpu_render(wl, 256, flags=N.FILM_FP64)
    sc = O.Scene(wl.mesh, wl.desc.c)
    _, _, _, xyz = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, 256, wl.seed)
    e = rel_rmse(xyz_gpu, xyz / 256)
    print("FP64 film, ring 256x256x256 relRMSE XYZ vs CPU restatement:", e)
    assert np.all(e <= 2e-3), e


def test_oracle_render_is_independent_of_its_thread_count():
    """The CPU baseline renders pixels in parallel; each pixel's samples are
    summed by one thread in sample order, so the film is the same bit for bit
    on one thread and on four (a band of the ring still, 2 spp; CPU)."""
    import oracle as O

    wl = W.ring_still(spp=2, width=96, height=96)
    sc = O.Scene(wl.mesh, wl.desc.c)
    one = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, 2, wl.seed, rows=(40, 56), threads=1)
    four = sc.render_pass(wl.camera, wl.settings, wl.width, wl.height, 0, 2, wl.seed, rows=(40, 56), threads=4)
    for a, b in zip(one, four):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert np.abs(one[3][40:56]).sum() > 0 and np.abs(one[3][:40]).sum() == 0
