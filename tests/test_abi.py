"""The C-ABI library loads and exports every function include/fornos_gpu.h declares."""
import ctypes
import os
import re

from fornos_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fornos_gpu.h")


def declared_functions(path=HEADER):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fk_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_functions():
    decl = set(declared_functions())
    assert set(_lib.exported_symbols()) == decl


def test_library_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, missing


def test_context_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = lib.fk_ctx_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_null_arguments_rejected(lib):
    assert lib.fk_buf_alloc(None, 16, None) == -1
    assert lib.fk_mesh_create(None, None) == -1
    assert lib.fk_bvh_build(None, 8, 8192, None) == -1
    assert lib.fk_samples_cosine(0, 1, 0, None) == -1
    assert lib.fk_last_error(None) == b"null context"
