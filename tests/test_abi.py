"""The C-ABI library loads and exports every entry point include/sbdgpu.h
declares (no compute without a GPU)."""
import ctypes
import os
import re

import sbd_b200
from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sbdgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sbdgpu_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(sbd_b200.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(sbd_b200.EXPORTS) == syms


def test_built_for_sm100a():
    data = open(sbd_b200.LIB_PATH, "rb").read()
    assert b"sm_100a" in data
