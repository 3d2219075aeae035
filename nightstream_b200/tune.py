"""Measure the launch-shape table of the Pi_CCS row rounds on this GPU.

    python -m nightstream_b200.tune [--ells 10 11 ... 20] [--ks 1 13] [--out PATH]

For every (ell_n, k) it builds a seeded R1CS of n = m = 2^ell_n and k
ternary digit matrices, runs neo_gpu_ccs_autotune (every candidate launch
shape timed on the whole row-round sequence with CUDA events) and writes the
table (one line "ccs <ell_n> <k> <nc_threads> <compact_q> <hist_items>" per
shape) to PATH, by default the table the library loads at start
(nightstream_b200/tune_b200.txt).  Shapes without an entry use the built-in
defaults, so the table only speeds launches up; results are bit-identical
for every choice.
"""
import argparse

import numpy as np

from . import gpu, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ells", type=int, nargs="+", default=list(range(10, 21)))
    ap.add_argument("--ks", type=int, nargs="+", default=[1, 13])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=gpu.TUNE_FILE)
    a = ap.parse_args(argv)
    ctx = gpu.Context(0)
    rng = np.random.default_rng(5)
    for ell in a.ells:
        ccs, _ = synth.make_r1cs(ell, 11)
        for k in a.ks:
            Z = rng.integers(-1, 2, size=(k, 54, 1 << ell)).astype(np.int8)
            best = ctx.ccs_autotune(ccs, Z, a.reps)
            print(f"ccs ell_n={ell} k={k}: nc_threads={best[0]} compact_q={best[1]} hist_items={best[2]}", flush=True)
    gpu.tune_save(a.out)
    ctx.close()


if __name__ == "__main__":
    main()
