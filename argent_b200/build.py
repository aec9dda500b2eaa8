"""Build the native libraries in-tree.

  argent_b200/lib/libargent_gpu.so   CUDA kernels + C ABI (include/argent_gpu.h), sm_100a,
                                     with the serve scheduler (host/serve.cpp) over that ABI
  argent_b200/lib/libargent_host.so  host-side scene builders (include/argent_host.h)

The CUDA library is compiled with --fmad=false: argent's Rust code rounds
every multiply and add separately, and the closest-hit parity gate compares
ray/triangle distances bit for bit.

Usage: python -m argent_b200.build [--force]
       python -m argent_b200.build --variant OUT.so NAME=VALUE ...   (a CUDA library with other constants)
"""

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
LIB = os.path.join(ROOT, "lib")

GPU_SO = os.path.join(LIB, "libargent_gpu.so")
HOST_SO = os.path.join(LIB, "libargent_host.so")

GPU_SOURCES = [
    os.path.join(CSRC, "argent_gpu.cu"),
    os.path.join(CSRC, "host", "bvh_build.cpp"),
    os.path.join(CSRC, "host", "scene_prep.cpp"),
    os.path.join(CSRC, "host", "serve.cpp"),
    os.path.join(CSRC, "host", "cavity.cpp"),
    os.path.join(CSRC, "host", "develop.cpp"),
]
HOST_SOURCES = [
    os.path.join(CSRC, "host", "synth.cpp"),
    os.path.join(CSRC, "host", "spectra.cpp"),
    os.path.join(CSRC, "host", "studio.cpp"),
    os.path.join(CSRC, "host", "scene_prep.cpp"),
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _deps():
    out = []
    for d, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                out.append(os.path.join(d, f))
    for f in os.listdir(os.path.join(REPO, "include")):
        out.append(os.path.join(REPO, "include", f))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _host_cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_gpu(force=False, verbose=False, out=None, defines=()):
    """The CUDA library; `out` and `defines` (e.g. ["ARGENT_SHORT_STACK=8"])
    build a variant with other build-time constants at another path, which
    ARGENT_GPU_LIB then selects."""
    out = out or GPU_SO
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    if not force and not defines and not _stale(out, _deps()):
        return out
    cmd = ["nvcc", *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-ccbin", _host_cxx(),
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared", "-o", out + ".tmp",
           *[f"-D{d}" for d in defines], *GPU_SOURCES, "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build_host(force=False):
    os.makedirs(LIB, exist_ok=True)
    srcs = [s for s in HOST_SOURCES if os.path.exists(s)]
    if not force and not _stale(HOST_SO, _deps()):
        return HOST_SO
    cmd = [_host_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-pthread", "-o", HOST_SO + ".tmp", *srcs]
    subprocess.run(cmd, check=True)
    os.replace(HOST_SO + ".tmp", HOST_SO)
    return HOST_SO


def build_oracle(force=False):
    """The CPU oracle is test infrastructure; it is built here so it travels
    with the tree, but nothing in the package loads it."""
    odir = os.path.join(REPO, "oracle")
    if not os.path.exists(os.path.join(odir, "Makefile")):
        return None
    if force:
        subprocess.run(["make", "-C", odir, "-B", "liboracle.so"], check=True)
    else:
        subprocess.run(["make", "-C", odir, "liboracle.so"], check=True)
    return os.path.join(odir, "liboracle.so")


def build_all(force=False, verbose=False):
    build_host(force)
    build_gpu(force, verbose)
    build_oracle(force)


if __name__ == "__main__":
    if "--variant" in sys.argv:
        # python -m argent_b200.build --variant OUT.so NAME=VALUE ...
        i = sys.argv.index("--variant")
        build_gpu(force=True, out=sys.argv[i + 1], defines=sys.argv[i + 2:])
    else:
        build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
