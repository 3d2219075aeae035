"""Build libneo_gpu.so (sm_100a) in-tree with nvcc.

The library is compiled for ``-gencode arch=compute_100a,code=sm_100a`` only
and written next to this file, so that it travels with the source tree.  Each
source is compiled to its own object (in parallel, under ``_build/``), then
the objects are linked into the shared library; an object is rebuilt when its
source or any header is newer.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libneo_gpu.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["core.cu", "commit.cu", "commit_tc.cu", "ccs_oracle.cu", "fold.cu", "batch.cu",
           "mem_oracle.cu", "mixers.cu", "pp_gen.cu", "tune.cu", "transcript.cpp", "transcript_capi.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-ccbin", "/usr/bin/g++",
]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "neo_gpu.h"))
    return [h for h in hs if os.path.exists(h)]


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def _stale(src, hdr_t):
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(src) > t or hdr_t > t


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in sources() + _headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    hdr_t = max(os.path.getmtime(h) for h in _headers())
    todo = [s for s in sources() if force or _stale(s, hdr_t)]

    def compile_one(src):
        cmd = [NVCC] + CFLAGS + ["-c", src, "-o", _obj(src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        for f in [ex.submit(compile_one, s) for s in todo]:
            f.result()
    link = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-o", LIB] + \
        [_obj(s) for s in sources()]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
