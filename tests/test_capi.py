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


def test_rust_bindings_cover_the_header():
    """nightstream_b200/rust/neo-gpu-sys declares every entry point of
    include/neo_gpu.h (the binding a Rust host such as the reference's shard
    loop links against), with the same parameter count."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(root, "include", "neo_gpu.h")).read(), flags=re.S)
    decl = {n: len([a for a in args.split(",") if a.strip() and a.strip() != "void"])
            for n, args in re.findall(r"^(?:int|uint32_t|const char\*)\s+(neo_\w+)\s*\(([^;]*?)\)\s*;", hdr, re.M | re.S)}
    rs = open(os.path.join(root, "nightstream_b200", "rust", "neo-gpu-sys", "src", "lib.rs")).read()
    got = {n: len([a for a in args.split(",") if a.strip()])
           for n, args in re.findall(r"pub fn (neo_\w+)\(([^)]*)\)", rs)}
    assert decl, "no declarations parsed"
    assert decl == got


def test_tune_table_round_trip(tmp_path):
    """The launch-shape table loads from and saves to its text form, without a GPU."""
    p = tmp_path / "tune.txt"
    p.write_text("ccs 18 13 75776 8 16384\nccs 10 3 37888 0 8192\nbogus line\n")
    assert gpu.tune_load(str(p))
    assert gpu.tune_get(18, 13) == (75776, 8, 16384)
    assert gpu.tune_get(10, 3) == (37888, 0, 8192)
    out = tmp_path / "out.txt"
    gpu.tune_save(str(out))
    lines = out.read_text().split("\n")
    assert "ccs 18 13 75776 8 16384" in lines and "ccs 10 3 37888 0 8192" in lines
