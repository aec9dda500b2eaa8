"""Launch tunings found by argent_autotune, cached per size class.

A tuning (lanes, wave size, blocks per SM of each shading class and of the
traversals) depends on how much work a render hands the device and on what
it shades, not on the exact scene: renders of one size class share it.  The
class is the piece's triangle count and the render's path-samples, each to
the nearest power of two, the material classes its scene can reach, and
whether it has an env map.  Tunings are kept in a JSON file (the path in
ARGENT_TUNE_CACHE, else tune_cache.json in the user's cache directory), so
a later process applies a tuning without searching again.
"""

import json
import math
import os

from . import _native as N


def cache_path():
    p = os.environ.get("ARGENT_TUNE_CACHE")
    if p:
        return p
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "argent_b200", "tune_cache.json")


def size_class(scene, width, height, count):
    """The cache key of a render: log2 buckets of triangles and
    path-samples, the scene's shading-class mask and env-map flag."""
    tris = max(int(scene.piece.mesh.num_tris), 1)
    ps = max(int(width) * int(height) * int(count), 1)
    desc = scene.desc
    env_map = 1 if desc.env.kind == N.ENV_MAP else 0
    kinds = sorted({int(m.kind) * 4 + int(m.gem_kind) for m in desc.materials})
    return f"t{round(math.log2(tris))}_p{round(math.log2(ps))}_m{'-'.join(map(str, kinds))}_e{env_map}"


def load(path=None):
    try:
        with open(path or cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store(key, tuning, rate, path=None):
    path = path or cache_path()
    data = load(path)
    data[key] = {"tuning": tuning, "path_samples_per_s": rate}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned(ctx, scene, cam, settings, width, height, count, path=None, search=True):
    """Applies the cached tuning of this render's size class to `ctx`, or
    (with `search`) runs argent_autotune on the render and caches what it
    finds.  Returns (key, tuning dict, cached: bool)."""
    key = size_class(scene, width, height, count)
    hit = load(path).get(key)
    if hit:
        ctx.set_tuning(hit["tuning"])
        return key, hit["tuning"], True
    if not search:
        return key, ctx.tuning(), False
    res = ctx.autotune(scene, cam, settings, width, height, count)
    best = max((r[2] for r in res), default=0.0)
    t = ctx.tuning()
    store(key, t, best, path)
    return key, t, False
