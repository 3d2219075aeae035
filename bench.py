#!/usr/bin/env python
"""Shard fold-steps/sec of the Neo fold step on B200.

One "step" is one steady-state fold step of a shard (k = 13: the step's MCS
instance plus 12 carried DEC children).  Default workload (single shard with
memory): a seeded synthetic R1CS of n = m = 2^16 constraints whose witness
carries the shared CPU bus of 1024 trace steps (a 2^14-step trace folds in 16
such steps) with one Twist memory of 2^12 cells (one read and one write per
step, addresses 70 % stride-4 sequential / 30 % uniform, 32-bit values) and
one Shout table of 2^16 uniform 32-bit entries (uniform lookups).  A step is
witness decomposition + MCS Ajtai commitment, the Shout and Twist address
pre-time sum-checks, the Pi_CCS sum-check (16 batched-time rounds over the CCS
claim and the six Route-A memory claims + 6 Ajtai rounds), ME outputs with bus
openings, the Twist val-eval batch and val-lane CPU ME claims, and Pi_RLC /
Pi_DEC on both lanes (24 child commitments), with the Poseidon2 Fiat-Shamir
transcript in between.  --workload main drops the memory sidecar.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU runs (torchrun) place one independent shard per rank (replicas):
value = steps of all ranks / max-over-ranks device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q = (1 << 64) - (1 << 32) + 1
METRIC = "shard fold-steps/sec"
UNIT = "fold-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ell", type=int, default=16, help="log2 of the CCS size n = m")
    ap.add_argument("--workload", default="memory", choices=["memory", "main"],
                    help="memory: single shard with Twist + Shout on the shared CPU bus; main: no memory")
    ap.add_argument("--chunk", type=int, default=1024, help="trace steps per fold step (memory workload)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="plain", choices=["plain", "batched", "served", "rounds", "commit"],
                    help="plain: one shard; batched: 64 uneven shards batched vs one at a time; "
                         "served: Poisson arrivals, p50/p99 latency; rounds / commit: the Pi_CCS row-round "
                         "sequence or the commitment alone at --ell (--steps timed repetitions)")
    ap.add_argument("--shards", type=int, default=64)
    ap.add_argument("--batch-reps", type=int, default=3, help="batched runs of the mix; the median is reported")
    ap.add_argument("--shard-steps", type=int, default=3)
    ap.add_argument("--workers", type=int, default=0, help="batch workers (0: min(16, host cores))")
    ap.add_argument("--no-served", action="store_true", help="plain mode without the served (Poisson) sub-result")
    ap.add_argument("--served-requests", type=int, default=24)
    ap.add_argument("--no-large", action="store_true", help="plain mode without the 2^20 large-shard sub-result")
    ap.add_argument("--no-batch", action="store_true",
                    help="plain mode without the batched 64-shard memory mix (batched vs one-at-a-time) sub-result")
    return ap.parse_args()


MEM_TWIST_ELL, MEM_SHOUT_ELL = 12, 16
INT8_DATASHEET_TOPS = 4500.0  # B200 dense int8 tensor throughput, datasheet (TOPS)


class Workload:
    """The benchmarked shard: its CCS, PP, memory instances and, per fold step,
    the witness and the Twist MemInits.  With memory the fold steps prove
    consecutive chunks of one trace (at least 2^14 trace steps): chunk c's
    witness carries chunk c's bus columns and its Twist memory starts from the
    state chunk c-1 left.  Without memory every step reuses one witness."""

    def __init__(self, args, rank, n_steps):
        from nightstream_b200 import synth
        ell = args.ell
        self.pp = np.random.default_rng(99 + rank).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        if args.workload == "memory":
            n = max(n_steps, (1 << 14) // args.chunk)
            self.ccs, self.zs, self.mem, self.inits = synth.make_memory_workload_chunks(
                ell, 1234 + rank, n, args.chunk, MEM_SHOUT_ELL, MEM_TWIST_ELL)
        else:
            self.ccs, z = synth.make_r1cs(ell, 1234 + rank)
            self.zs, self.mem, self.inits = [z], None, None

    def z(self, c):
        return self.zs[c % len(self.zs)]

    def prepare(self, shard, c):
        """Set the MemInits of step c on a GPU shard or an oracle shard (c > 0)."""
        if self.inits and c:
            for i, init in enumerate(self.inits[c % len(self.zs)]):
                shard.set_twist_init(i, init)


def config(args):
    ell = args.ell
    if args.workload == "memory":
        bus_cols = (MEM_SHOUT_ELL + 2) + (2 * MEM_TWIST_ELL + 5)
        return {
            "workload": f"single shard with memory: steady-state fold steps of an R1CS n=m=2^{ell} (k=13), each "
                        f"proving the next chunk of {args.chunk} trace steps of one trace of >= 2^14 steps (the "
                        f"chunk's shared CPU bus in the witness tail, its Twist memory starting from the state the "
                        f"previous chunk left); one Twist memory of "
                        f"2^{MEM_TWIST_ELL} cells (1 read + 1 write per step, 70% stride-4 / 30% uniform "
                        f"addresses, 32-bit values), one Shout table of 2^{MEM_SHOUT_ELL} uniform 32-bit entries "
                        f"(uniform lookups); Route-A batched time claims + Twist val-eval + val lane",
            "n": 1 << ell, "m": 1 << ell, "k": 13, "kappa": 16, "d": 54, "b": 2, "k_rho": 12,
            "trace_steps_per_fold_step": args.chunk, "bus_cols": bus_cols,
            "twist_cells": 1 << MEM_TWIST_ELL, "shout_table": 1 << MEM_SHOUT_ELL,
            "sumcheck_rounds": f"{ell} time (7 claims) + 6 Ajtai + {MEM_SHOUT_ELL} Shout addr + "
                               f"{MEM_TWIST_ELL} Twist addr + {ell} val-eval",
            "commits_per_step": 25,
            "l2": "inputs larger than L2 (PP limbs 453 MB at 2^16, read by every commit)",
            "witness": "seeded synthetic R1CS witness with the bus tail; values in [0, 2^32) except Twist "
                       "increments (field differences); the same witness each step",
        }
    return {
        "workload": f"steady-state fold step, main lane (Pi_CCS + Pi_RLC + Pi_DEC), "
                    f"R1CS n=m=2^{ell}, k=13, no Twist/Shout",
        "n": 1 << ell, "m": 1 << ell, "k": 13, "kappa": 16, "d": 54, "b": 2, "k_rho": 12,
        "sumcheck_rounds": ell + 6, "commits_per_step": 13,
        "l2": "inputs larger than L2 (PP limbs 453 MB at 2^16, read by every commit)",
        "witness": "seeded synthetic R1CS witness, values in [0, 2^32), same witness each step",
    }


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (read + write) of one 12-plane commit_p8_kernel<4> launch per
# witness column, from an ncu capture at m = 2^14 (182.1 MB / 16384: the PP
# limb tiles once plus the window sequences once); the tiles scale with m.
COMMIT_TRAFFIC_PER_M = 182.1e6 / 16384


# DRAM bytes (read + write) of the 18 launches of one 16-round Pi_CCS sequence
# (k = 13), per row, from an ncu capture at 2^16 rows (248.5 MB / 65536).
ROUNDS_TRAFFIC_PER_ROW = 248.5e6 / 65536

# Integer-ALU ceiling of the sequence's largest launch (round 3, the cross
# terms), from ncu --set full at 2^16 rows, k = 13: ALU pipe and issue-slot
# utilisation.
ROUNDS_ALU = {"kernel": "ccs_fast_round_kernel<3,0> (round 3)", "alu_pipe_frac": 0.669, "issue_active_frac": 0.579,
              "source": "ncu --set full -k regex:ccs_fast_round_kernel -s 3 -c 1 on bench.py --mode rounds --ell 16"}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def flush_l2():
    """Write 512 MB (4x the 126 MB L2) so the next launch starts cold."""
    import torch
    buf = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    buf.fill_(1)
    del buf


def rounds_roofline(ctx, ccs, z, ell, stream, reps=3):
    """The Pi_CCS time rounds of a steady-state step (k = 13: the MCS witness
    and 12 carried DEC children), all ell row rounds launched back to back
    through neo_gpu_ccs_oracle_row_rounds_device and timed with CUDA events on
    the library stream. L2 is flushed before each timed sequence.
    Algorithmic bytes B_ccs = 2^ell [(54k + 48) + 32 (54k + 6)]: round 0 reads
    the witness at compact width, every later round reads and writes the
    K-width tables."""
    import torch
    from nightstream_b200 import gpu, synth
    m = 1 << ell
    rng = np.random.default_rng(1234)
    Z0 = ctx.decomp_b2(z)
    Z = np.stack([Z0] + [rng.integers(-1, 2, size=(54, m)).astype(np.int8) for _ in range(12)])
    k = Z.shape[0]
    d = torch.empty((ell, 7, 2), dtype=torch.int64, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    launches = 0
    for rep in range(reps + 1):
        uk = lambda n: synth.uniform_k(rng, n)
        o = gpu.GpuCcsOracle(ctx, ccs, Z, 2, uk(6), uk(6), uk(ell), uk(1)[0], uk(ell), 6, ell, 6)
        ctx.synchronize()
        flush_l2()
        torch.cuda.synchronize()
        l0 = ctx.kernel_launches
        ev0.record(stream)
        o.row_rounds_device(uk(ell), d.data_ptr())
        ev1.record(stream)
        ev1.synchronize()
        if rep:
            times.append(ev0.elapsed_time(ev1))
            launches = ctx.kernel_launches - l0
        o.close()
    ms = statistics.median(times)
    B = m * ((54 * k + 48) + 32 * (54 * k + 6))
    peak = measured_peaks().get("hbm_gbs")
    src = "measured HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
    if not peak:
        peak, src = 6650.0, "fallback 6.65 TB/s"
    achieved = B / (ms * 1e-3) / 1e9
    return {"kernel": f"Pi_CCS time rounds, ternary-digit path: ccs_hist_kernel + ccs_hist_sum_kernel + "
                      f"ccs_fast_round_kernel<MODE>, {ell} rounds, k = {k}, {launches} launches per sequence",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": ROUNDS_TRAFFIC_PER_ROW * m,
            "traffic_source": "ncu dram__bytes_read+write of the 18 launches of one sequence at 2^16 rows, "
                              "k = 13 (ncu --cache-control none -k regex:ccs_ on bench.py --mode rounds --ell 16), "
                              "per row",
            "alu": ROUNDS_ALU,
            "launch_ms": ms / ell, "sequence_ms": ms, "peak_source": src,
            "algorithmic_bytes_per_sequence": B,
            "note": "integer-ALU bound (alu): rounds 0..4 read int8 digit planes and the whole sequence moves "
                    "0.16x B_ccs"}


def commit_roofline(ctx, m, stream, n_vec=12, reps=5):
    """The DEC batch commitment (n_vec ternary digit planes in one call, the
    small-digit tensor-core form) timed with CUDA events on the library
    stream; the PP limb tiles (537 MB at m = 2^16) exceed L2, so consecutive
    launches stream them from HBM."""
    import torch
    digits = torch.randint(-1, 2, (n_vec, 54, m), dtype=torch.int8, device="cuda")
    outc = torch.empty((n_vec, 16, 54), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        ctx.commit_device(digits.data_ptr(), n_vec, m, outc.data_ptr(), small_digits=True)
    ctx.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        ctx.commit_device(digits.data_ptr(), n_vec, m, outc.data_ptr(), small_digits=True)
    ev1.record(stream)
    ev1.synchronize()
    commit_ms = ev0.elapsed_time(ev1) / reps
    ops = 746496 * m * n_vec  # 2 * 8 limbs * kappa * d^2 * m per commitment
    peak, peak_src = int8_peak_tops()
    achieved = ops / (commit_ms * 1e-3) / 1e12
    nv = 4 if n_vec > 1 else 1
    return {"kernel": f"Ajtai commit, {n_vec} digit plane(s) per call, small-digit form (p8_seq_kernel + "
                      f"commit_p8_kernel<{nv}>: tcgen05 kind::i8, N = {64 * nv}, + commit_p8_reduce_kernel<{nv}>)",
            "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOPS", "frac": achieved / peak,
            "traffic": COMMIT_TRAFFIC_PER_M * m if m >= 1 << 14 and n_vec == 12 else None,
            "traffic_source": "ncu dram__bytes_read+write of one 12-plane commit_p8_kernel<4> launch at "
                              "m = 2^14, scaled by m",
            "launch_ms": commit_ms, "peak_source": peak_src, "algorithmic_ops_per_launch": ops,
            "frac_of_datasheet": achieved / INT8_DATASHEET_TOPS,
            "datasheet_peak": INT8_DATASHEET_TOPS}


def run_kernel_mode(args):
    """--mode rounds / commit: one kernel family alone at --ell (profiling and
    tuning; prints one JSON line)."""
    import torch
    from nightstream_b200 import gpu, synth
    ctx = gpu.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    m = 1 << args.ell
    if args.mode == "rounds":
        ccs, z = synth.make_r1cs(args.ell, 3)
        out = rounds_roofline(ctx, ccs, z, args.ell, stream, reps=args.steps)
    else:
        ctx.pp_upload(np.random.default_rng(1).integers(0, Q, size=(16, m, 54), dtype=np.uint64))
        out = {"planes12": commit_roofline(ctx, m, stream, 12, args.steps),
               "mcs1": commit_roofline(ctx, m, stream, 1, args.steps)}
    out["mode"] = args.mode
    out["ell"] = args.ell
    print(json.dumps(out), flush=True)
    ctx.close()


def int8_peak_tops():
    """Dense int8 GEMM throughput via torch._int_mm (cuBLASLt), 8192^3."""
    import torch
    try:
        a = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device="cuda")
        for _ in range(3):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e9
        for _ in range(5):
            s.record()
            for _ in range(5):
                torch._int_mm(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e) / 5)
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12, "measured torch._int_mm 8192^3 (cuBLASLt int8)"
    except Exception as ex:  # pragma: no cover - depends on the box
        pk = measured_peaks().get("bf16_tflops", 1590.0)
        return 2 * pk, f"2x measured bf16 (int8 GEMM unavailable: {type(ex).__name__})"


def cpu_baseline(args, wl):
    """One oracle fold step (C restatement, OpenMP on all host cores) after step 0."""
    from oracle.fold import OracleShard
    sh = OracleShard(wl.ccs, wl.pp, m_in=1, k_rho=12, app_label=b"neo/bench", mem=wl.mem)
    sh.fold_step(wl.z(0))  # step 0 (k = 1)
    wl.prepare(sh, 1)
    t0 = time.perf_counter()
    sh.fold_step(wl.z(1))
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"one steady-state fold step (k=13, {args.workload} workload) at n=m=2^{args.ell} on the C "
                      f"oracle (OpenMP, {os.cpu_count()} threads): {dt:.2f} s"}


BATCH_TWIST_ELL, BATCH_SHOUT_ELL = 10, 12


def pp_setup_result(args, ctx, m, kappa=16, reps=3):
    """Ajtai PP generation (setup_par from a 32-byte ChaCha8 seed) on the device:
    wall time of neo_gpu_pp_generate (host seed derivation, device sampling,
    tensor-core tile layout), and the same PP on the C oracle (OpenMP over the
    chunk streams).  Replaces the bench's PP for this m; run it last."""
    seed = bytes(range(32))
    ctx.pp_generate(seed, kappa, m, 1)  # warm-up (allocation)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ctx.pp_generate(seed, kappa, m, 1)
        ts.append(time.perf_counter() - t0)
    dev_ms = min(ts) * 1e3
    canon = kappa * m * 54 * 8
    out = {"mode": "setup_par", "kappa": kappa, "m": m, "device_ms": dev_ms,
           "canonical_bytes": canon, "device_gbs_canonical": canon / (dev_ms * 1e-3) / 1e9}
    if not args.no_cpu_baseline:
        import oracle
        t0 = time.perf_counter()
        oracle.pp_setup(seed, kappa, m, 1)
        cpu_s = time.perf_counter() - t0
        out.update({"cpu_ms": cpu_s * 1e3, "cpu_cores": os.cpu_count(), "cpu_kind": "port"})
    return out


def shard_mix(n_shards, lo, hi, seed, steps, memory=True):
    """n_shards synthetic shards with log2(n) uniform in [lo, hi]; with memory,
    each carries a Twist memory of 2^10 cells and a 2^12-entry Shout table on
    its shared CPU bus, min(1024, n/64) trace steps per fold step, and its
    `steps` fold steps prove consecutive chunks of one trace (per-step witness
    and Twist MemInit).  Entries: (ell, ccs, witnesses, mem, inits)."""
    from nightstream_b200 import synth
    rng = np.random.default_rng(seed)
    ells = rng.integers(lo, hi + 1, size=n_shards)
    out = []
    for i, ell in enumerate(ells):
        ell = int(ell)
        if memory:
            chunk = min(1024, (1 << ell) // 64)
            ccs, zs, mem, inits = synth.make_memory_workload_chunks(ell, seed * 1000 + i, steps, chunk,
                                                                    BATCH_SHOUT_ELL, BATCH_TWIST_ELL)
        else:
            (ccs, z), mem, inits = synth.make_r1cs(ell, seed * 1000 + i), None, None
            zs = [z] * steps
        out.append((ell, ccs, zs, mem, inits))
    return out


def upload_pps(ctx, ells):
    for ell in sorted(set(ells)):
        pp = np.random.default_rng(7000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        ctx.pp_upload(pp)


def run_mix(mix, shards, steps, workers):
    """Prove every shard of the mix for `steps` fold steps on a Batch with `workers` workers."""
    from nightstream_b200 import gpu
    b = gpu.Batch(0, n_workers=workers)
    t0 = time.perf_counter()
    ids = [b.submit(ccs, zs, steps, app_label=b"neo/mix-%d" % i, mem=mem, inits=inits)
           for i, (ell, ccs, zs, mem, inits) in enumerate(shards)]
    b.wait_all(3600)
    dt = time.perf_counter() - t0
    infos = [b.job_info(j) for j in ids]
    launches = b.kernel_launches
    b.close()
    assert all(i["status"] == 1 for i in infos), [(j, i["status"], i.get("error")) for j, i in enumerate(infos)
                                                  if i["status"] != 1]
    return dt, infos, launches


def batched_result(args):
    from nightstream_b200 import gpu
    workers = args.workers or min(16, os.cpu_count() or 8)
    shards = shard_mix(args.shards, 10, 16, 77, args.shard_steps)
    ctx = gpu.Context(0)
    upload_pps(ctx, [s[0] for s in shards])
    steps = args.shard_steps
    total_steps = steps * len(shards)
    dt_plain, infos_plain, _ = run_mix(None, shards, steps, 1)
    # the batched interval is ~1-2 s of host-bound work, so one run carries the
    # host's jitter: report the median of `batch_reps` runs (each bit-checked)
    runs = [run_mix(None, shards, steps, workers) for _ in range(max(1, args.batch_reps))]
    same = all(np.array_equal(a["transcript_state"], b["transcript_state"])
               for _, infos, _ in runs for a, b in zip(infos_plain, infos))
    dt_b, infos_b, launches = sorted(runs, key=lambda r: r[0])[len(runs) // 2]
    lat = sorted(i["latency_ms"] for i in infos_b)
    # the same mix on 4 workers: a fold step is a single-threaded host chain
    # (the transcript), so throughput follows the worker count up to the cores
    few = min(4, workers)
    runs4 = [run_mix(None, shards, steps, few) for _ in range(max(1, args.batch_reps // 2))]
    same = same and all(np.array_equal(a["transcript_state"], b["transcript_state"])
                        for _, infos, _ in runs4 for a, b in zip(infos_plain, infos))
    dt4 = statistics.median(r[0] for r in runs4)
    ctx.close()
    return {"value": total_steps / dt_b, "plain_value": total_steps / dt_plain, "speedup": dt_plain / dt_b,
            "workers": workers, "shards": len(shards), "steps_per_shard": steps,
            "sizes_log2": [s[0] for s in shards], "bit_identical_to_plain": bool(same),
            "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "gpu_launches": int(launches), "seconds": dt_b, "plain_seconds": dt_plain,
            "runs_fold_steps_per_s": [total_steps / r[0] for r in runs],
            "by_workers": {str(workers): total_steps / dt_b, str(few): total_steps / dt4}}


def run_batched(args):
    r = batched_result(args)
    out = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["shards"] * r["steps_per_shard"],
           "warmup": 0, "ms_per_step": 1e3 / r["value"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u64 (F_q, K = F_q^2), int8 digits", "data": "synthetic",
           "config": {"workload": f"batched: {r['shards']} shards, n=m=2^U with U uniform in [10,16], "
                                  f"{r['steps_per_shard']} fold steps each, each shard with a Twist memory of 2^10 cells and a "
                                  f"2^12-entry Shout table (min(1024, n/64) trace steps per fold step), "
                                  f"{r['workers']} workers vs one worker",
                      "l2": "PP of all sizes (>1 GB) exceeds L2"},
           "batched": r, "gpu_launches": r["gpu_launches"],
           "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None}}
    print(json.dumps(out), flush=True)


def served_result(args, n_req, rates=(2.0, 5.0, 10.0)):
    """Poisson arrivals of shard-prove requests (n log-uniform 2^10..2^18, each
    with a Twist memory and a Shout table) at each rate: p50 / p99 latency
    (arrival to result), fold-steps/s over the run and the longest queue wait."""
    from nightstream_b200 import gpu
    workers = args.workers or min(16, os.cpu_count() or 8)
    shards = shard_mix(n_req, 10, 18, 91, args.shard_steps)
    ctx = gpu.Context(0)
    upload_pps(ctx, [s[0] for s in shards])
    res = []
    for lam in rates:
        rng = np.random.default_rng(int(lam * 100))
        gaps = rng.exponential(1.0 / lam, size=n_req)
        b = gpu.Batch(0, n_workers=workers)
        t0 = time.perf_counter()
        ids = []
        t_next = t0
        for i, (ell, ccs, zs, mem, inits) in enumerate(shards):
            t_next += gaps[i]
            while time.perf_counter() < t_next:
                time.sleep(min(0.005, max(0.0, t_next - time.perf_counter())))
            ids.append(b.submit(ccs, zs, args.shard_steps, app_label=b"neo/req-%d" % i, mem=mem, inits=inits))
        b.wait_all(3600)
        dt = time.perf_counter() - t0
        infos = [b.job_info(j) for j in ids]
        b.close()
        assert all(i["status"] == 1 for i in infos)
        lat = sorted(i["latency_ms"] for i in infos)
        res.append({"rate_per_s": lam, "p50_ms": lat[len(lat) // 2],
                    "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                    "fold_steps_per_s": n_req * args.shard_steps / dt, "max_queue_ms": max(i["queue_ms"] for i in infos)})
    ctx.close()
    return {"requests": n_req, "steps_per_request": args.shard_steps, "workers": workers,
            "sizes_log2": [s[0] for s in shards], "rates": res}


def large_result(args, steps=3):
    """The large single shard: n = m = 2^20, 2^14 trace steps per fold step, a
    Twist memory of 2^16 cells and a Shout table of 2^20 entries (59 bus
    columns), PP from setup_par on the device; steady-state fold steps through
    the C ABI with the witness resident (CUDA events on the library stream)."""
    import torch
    from nightstream_b200 import gpu, synth
    ell = 20
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(ell, 4321, steps + 1, 1 << 14, 20, 16)
    ctx = gpu.Context(0)
    ctx.pp_generate(bytes(range(3, 35)), 16, 1 << ell, 1)
    sh = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/large", mem=mem)
    zt = torch.from_numpy(np.stack(zs).view(np.int64).copy()).cuda()
    stream = torch.cuda.ExternalStream(ctx.stream)
    sh.fold_step_device(zt[0].data_ptr())  # step 0 (k = 1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    ev0.record(stream)
    for c in range(1, steps + 1):
        sh.set_twist_init(0, inits[c][0])
        sh.fold_step_device(zt[c].data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    stats = sh.step_stats()
    sh.close()
    ctx.close()
    return {"workload": "n=m=2^20, 2^14 trace steps per fold step, Twist 2^16 cells, Shout 2^20 entries, k=13",
            "steps": steps, "ms_per_step": ms, "fold_steps_per_s": 1e3 / ms,
            "transcript_permutations_per_step": int(stats.get("transcript_perms", 0))}


def run_served(args):
    r = served_result(args, args.shards)
    best = max(x["fold_steps_per_s"] for x in r["rates"])
    out = {"metric": METRIC, "value": best, "unit": UNIT, "n_gpus": 1, "steps": r["requests"] * r["steps_per_request"],
           "warmup": 0, "ms_per_step": 1e3 / best, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "u64 (F_q, K = F_q^2), int8 digits", "data": "synthetic",
           "config": {"workload": f"served: {r['requests']} shard-prove requests, n=m=2^U, U uniform in [10,18], "
                                  f"{r['steps_per_request']} fold steps each, Twist 2^10 cells + Shout 2^12 table per "
                                  f"shard, Poisson arrivals, {r['workers']} workers"},
           "served": r}
    print(json.dumps(out), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle.fold import OracleShard
    wl = Workload(args, 0, 2 + args.warmup + args.steps)
    sh = OracleShard(wl.ccs, wl.pp, m_in=1, k_rho=12, app_label=b"neo/bench", mem=wl.mem)
    c = 0

    def step():
        nonlocal c
        wl.prepare(sh, c)
        sh.fold_step(wl.z(c))
        c += 1

    step()
    t0 = time.perf_counter()
    step()
    est = time.perf_counter() - t0
    budget = 150.0
    warm = min(args.warmup, max(0, int(budget / 3 / est) - 1))
    steps = max(1, min(args.steps, int(budget / est)))
    for _ in range(warm):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = time.perf_counter() - t0
    value = steps / dt
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
           "warmup": warm, "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u64 (F_q, K = F_q^2), int8 digits", "data": "synthetic",
           "config": config(args), "impl": "reference",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                            "sample": f"{steps} steady-state fold steps ({args.workload} workload) at n=m=2^{args.ell} "
                                      f"on the C restatement "
                                      f"(Rust reference not buildable here: no cargo/rustc)"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def max_over_ranks(ms, dist=None):
    """The slowest rank's time: every rank takes part in one MAX all-reduce
    (the only collective of a run; the ranks prove independent shards)."""
    if not dist:
        return ms
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, steps, ms):
    """Whole-job fold-steps/s of `world` replicas, each proving `steps` steps of
    its own shard in `ms` milliseconds (the slowest rank's)."""
    return world * steps / (ms * 1e-3)


def run_ours(args, rank, world, local_rank):
    import torch
    from nightstream_b200 import gpu
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    n_steps = 1 + args.warmup + 2 * args.steps
    wl = Workload(args, rank, n_steps)
    ccs, pp, mem = wl.ccs, wl.pp, wl.mem
    m = 1 << args.ell
    ctx = gpu.Context(local_rank)
    ctx.pp_upload(pp)
    shard = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/bench", mem=mem)
    stream = torch.cuda.ExternalStream(ctx.stream)
    # every step's witness resident in HBM (one row per fold step)
    zt = torch.from_numpy(np.stack([wl.z(c) for c in range(n_steps)]).view(np.int64).copy()).cuda()
    z_ptr = lambda c: zt.data_ptr() + c * m * 8
    cur = 0

    def step_device():
        nonlocal cur
        wl.prepare(shard, cur)
        shard.fold_step_device(z_ptr(cur))
        cur += 1

    torch.cuda.synchronize()
    step_device()  # step 0: k = 1 -> steady state afterwards
    for _ in range(args.warmup):
        step_device()
    ctx.synchronize()

    def barrier():
        if dist:
            dist.barrier()

    barrier()
    clocks = Clocks(local_rank)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.kernel_launches
    ctx.synchronize()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step_device()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.kernel_launches - l0
    barrier()
    stats = shard.step_stats()
    ms = max_over_ranks(ms, dist)
    value = replica_value(world, args.steps, ms)

    # end-to-end through the C ABI with host buffers: pinned z in, proof words out
    e2e = None
    if not args.no_e2e:
        zp = torch.from_numpy(np.stack([wl.z(c) for c in range(cur, cur + args.steps)]).view(np.int64).copy())
        zh = zp.pin_memory().numpy().view(np.uint64)
        barrier()
        ctx.synchronize()
        ev0.record(stream)
        for i in range(args.steps):
            wl.prepare(shard, cur)
            proof = shard.fold_step(zh[i])
            cur += 1
        ev1.record(stream)
        ev1.synchronize()
        ems = ev0.elapsed_time(ev1)
        ems = max_over_ranks(ems, dist)
        e2e = {"value": replica_value(world, args.steps, ems), "unit": UNIT, "h2d_bytes_per_step": int(zh[0].nbytes),
               "d2h_bytes_per_step": int(proof.nbytes)}
        if wl.mem is not None:
            # the same steps from trace chunks (neo_gpu_shard_fold_step_trace): the
            # CPU witness and the chunk's memory events in; the bus tail, the Twist
            # increments and the next MemInit are computed on the device
            from nightstream_b200 import synth
            n_chunks = len(wl.zs)
            chunks = []
            for i in range(args.steps):
                c = cur + i
                base, sev, tev = synth.trace_events(wl.z(c), wl.mem, m)
                zc = torch.from_numpy(wl.z(c)[:base].view(np.int64).copy()).pin_memory().numpy().view(np.uint64)
                chunks.append((c, zc, sev, tev))
            h2d = int(chunks[0][1].nbytes) + sum(int(a.nbytes) for ev in chunks[0][2] + chunks[0][3] for a in ev)
            barrier()
            ctx.synchronize()
            ev0.record(stream)
            for i, (c, zc, sev, tev) in enumerate(chunks):
                if i == 0 or c % n_chunks == 0:  # the trace restarts: its memory from the chunk's MemInit
                    wl.prepare(shard, c)
                proof = shard.fold_step_trace(zc, sev, tev)
            ev1.record(stream)
            ev1.synchronize()
            tms = max_over_ranks(ev0.elapsed_time(ev1), dist)
            cur += args.steps
            e2e["trace"] = {"value": replica_value(world, args.steps, tms), "unit": UNIT, "h2d_bytes_per_step": h2d,
                            "d2h_bytes_per_step": int(proof.nbytes),
                            "api": "neo_gpu_shard_fold_step_trace (CPU witness + trace events in)"}

    roofline_commit = commit_roofline(ctx, m, stream)
    roofline = rounds_roofline(ctx, ccs, wl.z(0), args.ell, stream)
    # the batched mix runs before the legs that use the host's OpenMP pool
    batched = batched_result(args) if rank == 0 and world == 1 and not args.no_batch else None
    served = served_result(args, args.served_requests) if rank == 0 and world == 1 and not args.no_served else None
    pp_setup = pp_setup_result(args, ctx, m) if rank == 0 else None

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "u64 (F_q, K = F_q^2), int8 digits", "data": "synthetic",
               "config": config(args), "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
               "roofline": roofline, "roofline_commit": roofline_commit}
        perms = stats.pop("transcript_perms", None)
        stats.pop("unused", None)
        out["step_breakdown_ms"] = stats
        out["transcript_permutations_per_step"] = int(perms) if perms is not None else None
        out["pp_setup"] = pp_setup
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args, wl)
        if batched is not None:
            out["batched"] = batched
        if served is not None:
            out["served"] = served
    shard.close()
    ctx.close()
    if rank == 0:
        if world == 1 and not args.no_large:
            out["large"] = large_result(args)
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.mode == "batched":
            if rank == 0:
                run_batched(args)
        elif args.mode == "served":
            if rank == 0:
                run_served(args)
        elif args.mode in ("rounds", "commit"):
            if rank == 0:
                run_kernel_mode(args)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
