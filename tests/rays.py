"""Seeded ray sets for the closest-hit parity gate.

Ray k draws its uniforms from argent's hash32 (sampler.rs:18-25):
u(k, j) = (hash32(hash32(k*16 + j) ^ hash32(seed)) >> 8) / 2^24.
80 % start on a sphere of 3x the bounding radius and aim at a uniform point
in the bounding box; 10 % start anywhere in the enlarged box with a uniform
direction; 10 % start on the surface, lifted by argent's offset_origin
(geom.rs:26-30), with a uniform direction.  A further slice of rays is snapped
to the coordinate axes, which gives direction components of exactly zero.
"""

import numpy as np


def hash32(x):
    x = np.asarray(x, np.uint32).copy()
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x7FEB352D)
    x ^= x >> np.uint32(15)
    x *= np.uint32(0x846CA68B)
    x ^= x >> np.uint32(16)
    return x


def uniforms(k, j, seed):
    h = hash32(hash32((k.astype(np.uint32) * np.uint32(16) + np.uint32(j))) ^ hash32(np.uint32(seed)))
    return (h >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def _normalize(v):
    v = v.astype(np.float32)
    d = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    return v * (np.float32(1.0) / np.sqrt(d))[:, None]


def _uniform_dir(u1, u2):
    z = np.float32(1.0) - np.float32(2.0) * u1
    r = np.sqrt(np.maximum(np.float32(0.0), np.float32(1.0) - z * z))
    phi = np.float32(2.0 * np.pi) * u2
    return _normalize(np.stack([r * np.cos(phi), r * np.sin(phi), z], 1))


def make_rays(positions, tris, n, seed=8, axis_fraction=0.01):
    """(n, 8) float32 rays [o, tmax=inf, d, 0]."""
    positions = np.asarray(positions, np.float32)
    tris = np.asarray(tris, np.uint32)
    lo, hi = positions.min(0), positions.max(0)
    c = (lo + hi) * np.float32(0.5)
    radius = np.float32(np.linalg.norm((hi - lo) * 0.5))
    k = np.arange(n, dtype=np.uint64)
    cls = (k % 10).astype(np.int64)
    u = [uniforms(k, j, seed) for j in range(8)]
    o = np.zeros((n, 3), np.float32)
    d = np.zeros((n, 3), np.float32)

    # 80 %: from a sphere of 3x the bounding radius toward the box.
    s = cls < 8
    sd = _uniform_dir(u[0][s], u[1][s])
    o[s] = c + sd * (np.float32(3.0) * radius)
    tgt = lo + (hi - lo) * np.stack([u[2][s], u[3][s], u[4][s]], 1)
    d[s] = _normalize(tgt - o[s])

    # 10 %: anywhere in the 1.5x box, uniform direction.
    s = cls == 8
    ext = (hi - lo) * np.float32(1.5)
    o[s] = (c - ext * np.float32(0.5)) + ext * np.stack([u[0][s], u[1][s], u[2][s]], 1)
    d[s] = _uniform_dir(u[3][s], u[4][s])

    # 10 %: secondary-like rays leaving the surface.
    s = cls == 9
    m = int(s.sum())
    ti = np.minimum((u[0][s] * np.float32(len(tris))).astype(np.int64), len(tris) - 1)
    a, b, cc = positions[tris[ti, 0]], positions[tris[ti, 1]], positions[tris[ti, 2]]
    r1 = np.sqrt(u[1][s])
    w0 = np.float32(1.0) - r1
    w1 = r1 * (np.float32(1.0) - u[2][s])
    w2 = r1 * u[2][s]
    p = a * w0[:, None] + b * w1[:, None] + cc * w2[:, None]
    e1, e2 = b - a, cc - a
    ng = _normalize(np.cross(e1, e2))
    dd = _uniform_dir(u[3][s], u[4][s])
    # offset_origin (geom.rs:26-30)
    scale = np.float32(1e-4) * (np.float32(1.0) + np.abs(p).max(1))
    side = ((ng[:, 0] * dd[:, 0] + ng[:, 1] * dd[:, 1]) + ng[:, 2] * dd[:, 2]) >= 0
    n_off = np.where(side[:, None], ng, -ng)
    o[s] = p + n_off * scale[:, None]
    d[s] = dd
    assert m == len(dd)

    # Snap a slice of rays to the axes (zero direction components).
    if axis_fraction > 0:
        snap = u[5] < np.float32(axis_fraction)
        ax = np.minimum((u[6][snap] * 3).astype(np.int64), 2)
        sign = np.where(u[7][snap] < 0.5, np.float32(-1.0), np.float32(1.0))
        dz = np.zeros((int(snap.sum()), 3), np.float32)
        dz[np.arange(len(ax)), ax] = sign
        d[snap] = dz
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = np.inf
    rays[:, 4:7] = d
    return rays


def compare_hits(ref, got, bvh, rays, ulps=2):
    """Classify GPU hits against the oracle's (argent's traversal).

    Buckets:
      match       same triangle, t within `ulps` (bit-equal expected)
      tie         another triangle at a bit-equal t (argent keeps the first
                  in its traversal order, the GPU the lower index); the
                  GPU's triangle must then have the lower index of the two
                  (`tie_not_lower` counts those that do not)
      closer      the GPU hit is strictly closer than argent's, or argent
                  misses it, and the oracle's own Moller-Trumbore confirms the
                  GPU triangle at exactly that t: argent's slab test culled a
                  box whose triangle lies at (within rounding) the current
                  best distance.  Brute force agrees with the GPU here.
      mismatch    anything else (the gate: must be 0)
    """
    rp = ref[:, 3].view(np.uint32)
    gp = got[:, 3].view(np.uint32)
    ref_hit = rp != 0xFFFFFFFF
    got_hit = gp != 0xFFFFFFFF
    out = dict(n=len(ref), hit_both=int((ref_hit & got_hit).sum()), miss_both=int((~ref_hit & ~got_hit).sum()))
    same = ref_hit & got_hit & (rp == gp)
    rt = ref[:, 0].view(np.int32).astype(np.int64)
    gt = got[:, 0].view(np.int32).astype(np.int64)
    t_bad = same & (np.abs(rt - gt) > ulps)
    cand = np.nonzero((ref_hit | got_hit) & ~same)[0]
    ties = closer = tie_not_lower = 0
    bad = []
    for i in cand:
        if not got_hit[i]:
            bad.append(i)  # the GPU missed a hit argent found
            continue
        ok, t, _, _ = bvh.tri_hit(gp[i], rays[i])
        if not ok or np.float32(t) != got[i, 0]:
            bad.append(i)
            continue
        if ref_hit[i] and got[i, 0] == ref[i, 0]:
            ties += 1
            tie_not_lower += int(gp[i] > rp[i])
        elif (not ref_hit[i]) or got[i, 0] < ref[i, 0]:
            closer += 1
        else:
            bad.append(i)
    out.update(match=int(same.sum() - t_bad.sum()), tie=ties, tie_not_lower=tie_not_lower, closer=closer,
               t_ulp_fail=int(t_bad.sum()),
               mismatch=len(bad), mismatch_idx=np.array(bad[:20], np.int64))
    return out
