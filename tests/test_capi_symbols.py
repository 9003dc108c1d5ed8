"""The C ABI library loads without a GPU and exports every entry point include/astr_b200.h
declares; the ctypes table matches the header."""
import ctypes
import os
import re

import astr_gpu_b200
from astr_gpu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "astr_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(astr_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert len(names) >= 20
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_library_exports_all_symbols():
    L = _lib.load()
    for n in _declared():
        assert hasattr(L, n), n


def test_init_without_device_fails_cleanly():
    # in a container with no GPU, astr_init returns an error code instead of aborting
    import torch
    if torch.cuda.is_available():
        return
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.astr_init(0, ctypes.byref(h)) != 0
