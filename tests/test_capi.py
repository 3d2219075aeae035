"""The C-ABI library loads on a host without a GPU and exports every entry
point include/neo_gpu.h declares."""
import ctypes
import os
import re

from nightstream_b200 import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "neo_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(neo_gpu_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(gpu.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(gpu.SIGNATURES)


def test_context_creation_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(gpu.NeoGpuError):
        gpu.Context(0)
