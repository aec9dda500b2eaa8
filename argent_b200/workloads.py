"""Scene assembly for the workloads, mirroring argent's caller side.

argent builds a scene with `Prepared::scene` (core/src/shot.rs:206-245): the
metal slot(s) first, then the stones, then the studio floor's material; the
studio rig scaled to the piece's bounding radius; the camera from
`Prepared::shot` (shot.rs:263-273, framing by views::frame) with the piece
turned by -azimuth, and thin-lens focus from `Prepared::autofocus`
(shot.rs:278-295).  The same steps are done here with the host library
(argent_host.h) and the GPU traversal for the autofocus probes.

Workloads (seeded, procedural; no argent assets are needed):
  ring_still     256 x 256, 16 spp, depth 8: 65,536-tri ring, sterling, noir, pinhole
  signet_still   1920 x 1080, 256 spp, depth 12: 2.1M-tri signet, 14k gold
                 (polished 0.05 / satin 0.35 slots), noir, 100 mm f/16, autofocus
  gems_still     1080 x 1920, 512 spp, depth 32: 18k setting, brilliant and
                 36 side stones, white studio, 100 mm pinhole
  reel_batch     4 alloys x 36 turntable frames x 3 pieces (61k, 1.1M, 3.0M
                 triangles), 1080 x 1920, 64 spp, depth 12, noir panels plus
                 a 2048 x 1024 synthetic HDRI (env_pick 0.5), render seed 11
  serve_trace    Poisson arrivals (seed 6) over 8 resident pieces (40k..3.0M
                 triangles) x 7 alloys: 70 % previews 512^2 x 4 spp, 25 %
                 listings 2000^2 x 128, 5 % finals 1080 x 1920 x 512
"""

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from . import mesh as M


def _f3(v):
    return (ctypes.c_float * 3)(*[float(x) for x in v])


class SceneDesc:
    """An ArgentSceneDesc plus the arrays it points into."""

    def __init__(self, materials, panels=(), env=None, floor=None, turntable_deg=0.0, white=None):
        self.materials = (N.ArgentMaterial * len(materials))(*materials)
        self.panels = (N.ArgentPanel * max(1, len(panels)))(*panels) if panels else None
        self.env = env if env is not None else N.ArgentEnv()
        self._keep = []
        c = N.ArgentSceneDesc()
        c.materials = self.materials
        c.num_materials = len(materials)
        c.panels = self.panels
        c.num_panels = len(panels)
        c.env = ctypes.pointer(self.env)
        if floor is not None:
            c.floor = floor
        c.turntable_deg = float(turntable_deg)
        if white is not None:
            c.has_white = 1
            c.white_xyz = _f3(white)
        self.c = c

    def keep(self, *objs):
        self._keep.extend(objs)


def metal(alloy, roughness=0.07, patina=0.8):
    m = N.ArgentMaterial()
    N.check(N.host().argent_material_metal(alloy.encode(), roughness, patina, ctypes.byref(m)))
    return m


def gem(name):
    m = N.ArgentMaterial()
    N.check(N.host().argent_material_gem(name.encode(), ctypes.byref(m)))
    return m


def diffuse(rgb):
    m = N.ArgentMaterial()
    N.host().argent_material_diffuse(_f3(rgb), ctypes.byref(m))
    return m


def illuminant_table(rgb):
    t = (ctypes.c_float * N.SPEC_LEN)()
    N.host().argent_bake_rgb_illuminant(_f3(rgb), t)
    return t


def studio(name, radius, floor_y):
    """Studio::build + floor_at: (panels, env, floor_material, floor, white)."""
    panels = (N.ArgentPanel * 16)()
    n = ctypes.c_int32()
    env = N.ArgentEnv()
    fm = N.ArgentMaterial()
    fl = N.ArgentFloor()
    hw = ctypes.c_int32()
    wx = (ctypes.c_float * 3)()
    N.check(N.host().argent_studio_build(name.encode(), radius, floor_y, panels, ctypes.byref(n), ctypes.byref(env),
                                         ctypes.byref(fm), ctypes.byref(fl), ctypes.byref(hw), wx))
    return list(panels[: n.value]), env, fm, fl, (list(wx) if hw.value else None)


def piece_radius(m):
    """Prepared::build (shot.rs:135-136): half the bounding-box diagonal."""
    lo, hi = m.bounds()
    return float(max(np.linalg.norm((hi - lo) * np.float32(0.5)), 1e-3)), float(lo[1])


def hull(m):
    """Prepared::build (shot.rs:111-114): every step-th vertex."""
    step = max(len(m.positions) // 4000, 1)
    return np.ascontiguousarray(m.positions[::step], np.float32)


def rot_y(p, deg):
    r = np.float32(deg) * np.float32(math.pi / 180.0)
    s, c = np.float32(math.sin(r)), np.float32(math.cos(r))
    p = np.asarray(p, np.float32)
    return np.stack([c * p[..., 0] + s * p[..., 2], p[..., 1], -s * p[..., 0] + c * p[..., 2]], -1).astype(np.float32)


def frame(points, azimuth, elevation, fill, focal_mm=100.0, f_stop=0.0, aspect=1.0):
    cam = N.ArgentCamera()
    pts = np.ascontiguousarray(points, np.float32)
    N.host().argent_frame(pts.ctypes.data_as(N.c_float_p), len(pts), azimuth, elevation, fill, focal_mm, f_stop,
                          aspect, ctypes.byref(cam))
    return cam


def band_camera(cam, height, y0, y1):
    """The camera whose (y1 - y0)-row frame shows rows y0..y1 of `cam`'s
    `height`-row frame (same width): the screen y of band row r,
    1 - 2 (r + j) / hb, maps to frame row y0 + r through half_h' =
    half_h * hb / H and shift' = (H - 2 y0 + shift * H) / hb - 1."""
    hb = y1 - y0
    b = N.ArgentCamera()
    ctypes.memmove(ctypes.byref(b), ctypes.byref(cam), ctypes.sizeof(cam))
    b.half_h = cam.half_h * hb / height
    b.shift[1] = (height - 2 * y0 + cam.shift[1] * height) / hb - 1.0
    return b


def camera_ray(cam, sx, sy, lu, lv):
    """Camera::ray (camera.rs:57-69) for the autofocus probes."""
    f = np.float32
    pos, fwd, right, up = (np.array(getattr(cam, k)[:], f) for k in ("pos", "forward", "right", "up"))
    x = (f(sx) + f(cam.shift[0])) * f(cam.half_w)
    y = (f(sy) + f(cam.shift[1])) * f(cam.half_h)
    d = fwd + right * x + up * y
    d = d * (f(1.0) / np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
    if cam.lens_radius <= 0:
        return pos, d
    ft = f(cam.focus_dist) / ((d[0] * fwd[0] + d[1] * fwd[1]) + d[2] * fwd[2])
    pf = pos + d * ft
    o = pos  # disk(0.5, 0.5) = (0, 0)
    dd = pf - o
    return o, dd * (f(1.0) / np.sqrt((dd[0] * dd[0] + dd[1] * dd[1]) + dd[2] * dd[2]))


def shot(piece_gpu, points, view="hero", focal_mm=100.0, f_stop=0.0, aspect=1.0):
    """Prepared::shot (shot.rs:263-273): camera on the rig's front, piece
    turned by -azimuth; autofocus (shot.rs:278-295) when f_stop > 0."""
    az, el, fill = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    N.check(N.host().argent_view_named(view.encode(), ctypes.byref(az), ctypes.byref(el), ctypes.byref(fill)))
    turn = -az.value
    pts = rot_y(points, turn)
    cam = frame(pts, 0.0, el.value, fill.value, focal_mm, f_stop, aspect)
    if cam.lens_radius > 0 and piece_gpu is not None:
        probes = [(0.0, 0.0), (0.0, 0.15), (0.0, 0.3), (0.12, 0.22), (-0.12, 0.22), (0.0, 0.42), (0.2, 0.1),
                  (-0.2, 0.1)]
        rays = np.zeros((len(probes), 8), np.float32)
        fwd_obj = rot_y(np.array(cam.forward[:], np.float32), -turn)
        for i, (sx, sy) in enumerate(probes):
            o, d = camera_ray(cam, sx, sy, 0.5, 0.5)
            rays[i, 0:3] = rot_y(o, -turn)
            rays[i, 4:7] = rot_y(d, -turn)
            rays[i, 3] = np.inf
        hits = piece_gpu.trace_closest(rays)
        ts = []
        for i in range(len(probes)):
            if hits[i, 3].view(np.uint32) != 0xFFFFFFFF:
                d = rays[i, 4:7]
                ts.append(np.float32(hits[i, 0]) * ((d[0] * fwd_obj[0] + d[1] * fwd_obj[1]) + d[2] * fwd_obj[2]))
        if ts:
            ts.sort()
            cam.focus_dist = float(ts[len(ts) // 2])
    return cam, turn


@dataclass
class Workload:
    name: str
    mesh: object
    desc: SceneDesc
    camera: object
    width: int
    height: int
    spp: int
    settings: object
    seed: int
    extra: dict = field(default_factory=dict)

    @property
    def path_samples(self):
        return self.width * self.height * self.spp


def settings(max_depth=32, clamp=24.0, rr=6):
    return N.ArgentPathSettings(max_depth, clamp, rr)


def _studio_scene(m, metal_mats, studio_name, turn):
    radius, floor_y = piece_radius(m)
    panels, env, fm, fl, white = studio(studio_name, radius, floor_y)
    mats = list(metal_mats) + [fm]
    fl.material = len(mats) - 1
    return SceneDesc(mats, panels, env, fl, turn, white)


def ring_still(piece_gpu=None, spp=16, width=256, height=256):
    """The small plain workload."""
    m = M.ring()
    cam, turn = shot(None, hull(m), "hero", 100.0, 0.0, width / height)
    desc = _studio_scene(m, [metal("sterling", 0.07, 0.8)], "noir", turn)
    return Workload("ring_still_256x256_16spp", m, desc, cam, width, height, spp, settings(8), 7)


def signet_still(piece_gpu=None, spp=256, width=1920, height=1080, mesh=None):
    """The full still: 1920 x 1080 x 256 spp on the 2.1M-triangle signet.
    `piece_gpu` (a gpu.Piece of the same mesh) enables thin-lens autofocus."""
    m = mesh if mesh is not None else M.signet()
    cam, turn = shot(piece_gpu, hull(m), "hero", 100.0, 16.0, width / height)
    desc = _studio_scene(m, [metal("gold14k", 0.05, 0.8), metal("gold14k", 0.35, 0.8)], "noir", turn)
    return Workload("signet_still_1920x1080_256spp", m, desc, cam, width, height, spp, settings(12), 7)


SIDE_GEMS = ("ruby", "sapphire", "emerald", "garnet")


def gems_still(piece_gpu=None, spp=512, width=1080, height=1920, mesh=None, max_depth=32, center="diamond",
               side=SIDE_GEMS):
    """The gems workload: 18k gold setting (about 0.9M triangles) with a
    diamond brilliant (argent's DIAMOND Sellmeier; `center="diamond_alt"`
    takes the workload's stated alternate fit, n_D about 2.261) and 36 side
    stones drawn from ruby / sapphire / emerald / garnet; white studio,
    1080 x 1920, 512 spp, max depth 32, 100 mm pinhole, hero view.  `center`
    and `side` (four names) swap the stones' materials, e.g. for opaque
    stones (onyx, turquoise, lapis: a coat over a body colour)."""
    m = mesh if mesh is not None else M.gem_ring()
    cam, turn = shot(piece_gpu, hull(m), "hero", 100.0, 0.0, width / height)
    mats = [metal("gold18k", 0.07, 0.8), gem(center)] + [gem(g) for g in side]
    desc = _studio_scene(m, mats, "white", turn)
    return Workload(f"gems_still_{width}x{height}_{spp}spp", m, desc, cam, width, height, spp, settings(max_depth), 7)


def opal(black, cell_mm=0.35):
    """Material::opal (material.rs:63-66): black or white opal."""
    m = N.ArgentMaterial()
    N.host().argent_material_opal(1 if black else 0, cell_mm, ctypes.byref(m))
    return m


def opal_still(black=False, spp=8, width=128, height=128, cell_mm=0.35):
    """The ring piece carved from precious opal (Voronoi domains of Bragg
    lattices over a milky or dark body, material.rs:98-113, 208-237),
    noir studio, 100 mm pinhole, hero view, depth 8."""
    m = M.ring()
    cam, turn = shot(None, hull(m), "hero", 100.0, 0.0, width / height)
    desc = _studio_scene(m, [opal(black, cell_mm)], "noir", turn)
    kind = "black" if black else "white"
    return Workload(f"opal_{kind}_{width}x{height}_{spp}spp", m, desc, cam, width, height, spp, settings(8), 7)


def with_cavity(mesh, cavity):
    """`mesh` carrying the per-vertex cavity mask `cavity`
    (cavity::patina_mask), as Prepared::build attaches it to the piece
    (shot.rs:142): metal slots with a patina then darken the recesses
    (material.rs:115-122)."""
    return M.Mesh(mesh.positions, mesh.tris, mesh.normals, mesh.tri_material, cavity)


def sphere(r=10.0, n=64):
    """tests/furnace.rs:19-44: a UV sphere with analytic normals."""
    f = np.float32
    pos, nrm = [], []
    for i in range(n + 1):
        th = f(math.pi) * f(i) / f(n)
        for j in range(2 * n):
            ph = f(math.pi) * f(j) / f(n)
            p = [f(r) * f(math.sin(th)) * f(math.cos(ph)), f(r) * f(math.cos(th)), f(r) * f(math.sin(th)) * f(math.sin(ph))]
            pos.append(p)
            nrm.append([p[0] / f(r), p[1] / f(r), p[2] / f(r)])
    w = 2 * n
    tris = []
    for i in range(n):
        for j in range(w):
            a = i * w + j
            b = i * w + (j + 1) % w
            c = (i + 1) * w + (j + 1) % w
            d = (i + 1) * w + j
            tris += [[a, c, b], [a, d, c]]
    return M.Mesh(np.array(pos, np.float32), np.array(tris, np.uint32), np.array(nrm, np.float32),
                  np.zeros(len(tris), np.uint16))


def furnace(material):
    """tests/furnace.rs:46-58: a 10 mm sphere in a uniform white
    RgbIlluminant gradient, camera at z=200, 100 mm pinhole, 64 x 64, 256 spp,
    seed 1, default PathSettings."""
    m = sphere(10.0, 64)
    white = illuminant_table([1.0, 1.0, 1.0])
    env = N.ArgentEnv()
    env.kind = N.ENV_GRADIENT
    env.power = 1.0
    env.top = white
    env.horizon = white
    env.bottom = white
    desc = SceneDesc([material], (), env, None, 0.0, None)
    cam = N.ArgentCamera()
    N.host().argent_camera_look_at(_f3([0, 0, 200]), _f3([0, 0, 0]), _f3([0, 1, 0]), 100.0, 0.0, 1.0,
                                   ctypes.byref(cam))
    return Workload("furnace", m, desc, cam, 64, 64, 256, settings(32), 1)


# ---------------------------------------------------------------- batched turntable reels

REEL_ALLOYS = ("sterling", "gold14k", "rose14k", "bronze")
# (label, nu, nv): the signet generator at 2 * nu * nv triangles
REEL_PIECES = (("61k", 256, 120), ("1.1M", 1024, 540), ("3.0M", 2048, 732))
REEL_FRAMES = 36


def reel_piece(label):
    """One of the batched workload's pieces (argent_synth_signet)."""
    for name, nu, nv in REEL_PIECES:
        if name == label:
            return M.signet(nu=nu, nv=nv)
    raise KeyError(label)


def hdri(width=2048, height=1024, sigma=2.0, seed=5):
    """The synthetic equirect map (argent_synth_hdri): (height, width, 3)
    linear sRGB float32."""
    rgb = np.zeros((height, width, 3), np.float32)
    N.host().argent_synth_hdri(width, height, sigma, seed, rgb.ctypes.data_as(N.c_float_p))
    return rgb


def map_env(rgb, rotation_deg=0.0):
    """Env::Map over `rgb` (kept alive by the caller)."""
    env = N.ArgentEnv()
    env.kind = N.ENV_MAP
    env.power = 1.0
    env.height, env.width = int(rgb.shape[0]), int(rgb.shape[1])
    env.rgb = rgb.ctypes.data_as(N.c_float_p)
    env.rotation_deg = float(rotation_deg)
    return env


def turntable_camera(points, view="hero", focal_mm=100.0, f_stop=0.0, aspect=1.0):
    """Prepared::turntable_camera (shot.rs:318-327): frame the hull turned
    through 24 steps of 15 degrees from the front (azimuth 0).  Returns the
    camera and the view's azimuth."""
    az, el, fill = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    N.check(N.host().argent_view_named(view.encode(), ctypes.byref(az), ctypes.byref(el), ctypes.byref(fill)))
    pts = np.concatenate([rot_y(points, 15.0 * k) for k in range(24)])
    return frame(pts, 0.0, el.value, fill.value, focal_mm, f_stop, aspect), az.value


def reel_frame_turn(azimuth, i, n=REEL_FRAMES):
    """render_reel's turntable rig (jobs.rs:617-621): -azimuth + 360 i / n."""
    return -azimuth + 360.0 * float(i) / float(n)


def reel_scene(m, alloy, env_rgb, turn):
    """The batched workload's scene for one piece and alloy: polished (0.05)
    and satin (0.35) slots of the alloy, the noir studio's panels and floor,
    and the map as the environment, so NEE picks the map with probability
    0.5 (scene.rs:105-109)."""
    radius, floor_y = piece_radius(m)
    panels, _, fm, fl, white = studio("noir", radius, floor_y)
    mats = [metal(alloy, 0.05, 0.8), metal(alloy, 0.35, 0.8), fm]
    fl.material = len(mats) - 1
    desc = SceneDesc(mats, panels, map_env(env_rgb), fl, turn, white)
    desc.keep(env_rgb)
    return desc


def reel_batch(pieces=None, alloys=REEL_ALLOYS, frames=range(REEL_FRAMES), width=1080, height=1920, spp=64,
               env_rgb=None):
    """The batched workload as a list of Workloads, piece-major then alloy
    then frame.  `pieces` maps label -> Mesh (built when None)."""
    if pieces is None:
        pieces = {label: reel_piece(label) for label, _, _ in REEL_PIECES}
    if env_rgb is None:
        env_rgb = hdri()
    out = []
    for label, m in pieces.items():
        cam, az = turntable_camera(hull(m), "hero", 100.0, 0.0, width / height)
        for alloy in alloys:
            for i in frames:
                turn = reel_frame_turn(az, i)
                desc = reel_scene(m, alloy, env_rgb, turn)
                out.append(Workload(f"reel_{label}_{alloy}_f{i:02d}_{width}x{height}_{spp}spp", m, desc, cam, width,
                                    height, spp, settings(12), 11, {"piece": label, "alloy": alloy, "frame": i}))
    return out


# ---------------------------------------------------------------- served requests

SERVE_ALLOYS = ("sterling", "gold14k", "gold18k", "rose14k", "white14k", "platinum", "bronze")
# (nu, nv) of the signet generator: 2 * nu * nv triangles, 40k .. 3.0M
SERVE_PIECES = ((200, 100), (250, 200), (500, 250), (500, 500), (1000, 500), (1000, 750), (2048, 512), (2048, 732))
# class: (share, width, height, spp, priority)
SERVE_CLASSES = {"preview": (0.70, 512, 512, 4, 0), "listing": (0.25, 2000, 2000, 128, 1),
                 "final": (0.05, 1080, 1920, 512, 2)}


def serve_pieces():
    """The served workload's eight resident pieces."""
    return [M.signet(nu=nu, nv=nv) for nu, nv in SERVE_PIECES]


def serve_trace(rate, seconds, seed=6):
    """Poisson arrivals at `rate` requests/s for `seconds`: a list of
    (arrival_s, class, piece index, alloy index), drawn from one seeded
    generator in that order per request."""
    rng = np.random.default_rng(seed)
    names = list(SERVE_CLASSES)
    shares = np.array([SERVE_CLASSES[n][0] for n in names])
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= seconds:
            break
        c = names[int(rng.choice(len(names), p=shares))]
        out.append((t, c, int(rng.integers(len(SERVE_PIECES))), int(rng.integers(len(SERVE_ALLOYS)))))
    return out


def serve_scene(m, alloy, turn):
    """A served look: polished and satin slots of the alloy, noir studio,
    the piece turned for the hero view."""
    return _studio_scene(m, [metal(alloy, 0.05, 0.8), metal(alloy, 0.35, 0.8)], "noir", turn)


def mean_request_path_samples():
    return sum(sh * w * h * spp for sh, w, h, spp, _ in SERVE_CLASSES.values())
