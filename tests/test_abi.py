"""The C-ABI libraries load and export every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(argent_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


@pytest.mark.parametrize("header,lib", [("argent_gpu.h", "libargent_gpu.so"), ("argent_host.h", "libargent_host.so")])
def test_exports(header, lib):
    path = os.path.join(ROOT, "argent_b200", "lib", lib)
    assert os.path.exists(path), f"{lib} not built"
    so = ctypes.CDLL(path)
    names = declared(header)
    assert names, header
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_bindings_cover_headers():
    from argent_b200 import _native as N

    for n in declared("argent_gpu.h"):
        assert n in N.GPU_FUNCS, n
    for n in declared("argent_host.h"):
        assert n in N.HOST_FUNCS, n


def test_struct_sizes_match_c():
    """ctypes mirrors have the C layout (sizes cross-checked against the header)."""
    from argent_b200 import _native as N

    assert ctypes.sizeof(N.ArgentRay) == 32
    assert ctypes.sizeof(N.ArgentHit) == 16
    assert ctypes.sizeof(N.ArgentMaterial) == 13 * 4 + 2 * 95 * 4 + 3 * 471 * 4
    assert ctypes.sizeof(N.ArgentCamera) == 4 * (12 + 4 + 2)
    assert ctypes.sizeof(N.ArgentTuning) == 40
    assert ctypes.sizeof(N.ArgentServeConfig) == 48


def test_error_path_without_device():
    """With no device the context call fails cleanly with a status code."""
    from argent_b200 import _native as N

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except Exception:
        pass
    lib = N.gpu()
    h = ctypes.c_void_p()
    rc = lib.argent_ctx_create(0, None, ctypes.byref(h))
    assert rc == N.E_CUDA
    assert b"device" in lib.argent_last_error(None)


def test_serve_structs_match_c(tmp_path):
    """The serve structs' ctypes mirrors have the compiler's layout."""
    import subprocess

    from argent_b200 import _native as N

    src = tmp_path / "layout.c"
    src.write_text('''#include <stddef.h>
#include <stdio.h>
#include "argent_gpu.h"
int main(void) {
  printf("%zu %zu %zu\\n", sizeof(ArgentServeConfig), offsetof(ArgentServeConfig, step_path_samples), sizeof(ArgentServeRequest));
  printf("%zu %zu %zu %zu\\n", offsetof(ArgentServeRequest, camera), offsetof(ArgentServeRequest, settings), offsetof(ArgentServeRequest, width), offsetof(ArgentServeRequest, priority));
  printf("%zu %zu %zu\\n", sizeof(ArgentServeStatus), offsetof(ArgentServeStatus, t_submit), offsetof(ArgentServeStatus, t_done));
  printf("%zu %zu %zu\\n", sizeof(ArgentBatchItem), offsetof(ArgentBatchItem, film), offsetof(ArgentBatchItem, count));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    C, R, S, B = N.ArgentServeConfig, N.ArgentServeRequest, N.ArgentServeStatus, N.ArgentBatchItem
    want = [ctypes.sizeof(C), C.step_path_samples.offset, ctypes.sizeof(R),
            R.camera.offset, R.settings.offset, R.width.offset, R.priority.offset,
            ctypes.sizeof(S), S.t_submit.offset, S.t_done.offset,
            ctypes.sizeof(B), B.film.offset, B.count.offset]
    assert got == want


def test_serve_rejects_null_arguments():
    """Serve entry points return ARGENT_E_INVALID for NULL handles (no device needed)."""
    from argent_b200 import _native as N

    lib = N.gpu()
    h = ctypes.c_void_p()
    assert lib.argent_serve_create(None, None, ctypes.byref(h)) == N.E_INVALID
    t = ctypes.c_uint64()
    assert lib.argent_serve_submit(None, None, ctypes.byref(t)) == N.E_INVALID
    assert lib.argent_serve_step(None, None) == N.E_INVALID
    assert lib.argent_serve_poll(None, 1, None) == N.E_INVALID
    assert lib.argent_serve_read(None, 1, None, None, None) == N.E_INVALID
    lib.argent_serve_destroy(None)
