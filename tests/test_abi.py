"""The C-ABI library loads and exports every function include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

from pusch_b200 import _native

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(pg_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_functions() == set(_native.SIGNATURES)


def test_abi_version():
    assert _native.load().pg_abi_version() == 1


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    cfg = _native.PgConfig(0, 8, 0)
    h = ctypes.c_void_p()
    assert _native.load().pg_create(ctypes.byref(cfg), ctypes.byref(h)) == _native.PG_ERR_NO_DEVICE
