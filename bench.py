#!/usr/bin/env python
"""Benchmark: Ozaki-scheme DGEMM on B200 (INT8 precision form on tcgen05).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the metric's configuration): m = n = k = 8192, A and B entries
(U(0,1) - 0.5) * exp(phi * N(0,1)) with phi = 1 from a seeded generator,
alpha = 1, beta = 0; INT8 slices on tcgen05 with INT32 accumulation, digits
chosen per operand until the split is exact, triangular pair set (fastMode).
One step = one cuozblasDgemmI8 call through the C ABI.  Inputs (512 MiB each)
are larger than L2, so no flush is needed between steps.

value   effective TFLOPS = 2 m n k / device time per step (inputs resident in
        HBM), summed over ranks; with N > 1 every rank runs its own replica
        (the path does not shard in this configuration).
e2e     the same metric with host buffers: pinned host -> device copies of A
        and B, the call, and the device -> host copy of C inside each step.
roofline  the tcgen05 product kernel alone (CUDA events around its launch on
        the handle's stream): int8 ops per launch = pairs * 2 m n k.

Extra keys (rank 0): the plain FP64-slice form on the same inputs, the
maximum relative error of both forms against the correctly rounded product
(the library's NearSum plain form, bit-exact to the reference CPU NearSum),
and DOT / CSRMV memory throughput.  The CPU baseline is the reference OzBLAS
CPU library (oracle/_ref) on a bounded row sample of the same problem.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DIM = 8192
PHI = 1.0


def phi_matrix(rows, cols, phi, seed):
    """(U - 0.5) * exp(phi * N(0,1)) with N from Box-Muller on the same U (column-major rows x cols)."""
    import numpy as np

    g = np.random.default_rng(seed)
    r1 = g.random((cols, rows))
    r2 = g.random((cols, rows))
    return (r1 - 0.5) * np.exp(phi * np.sqrt(-2.0 * np.log(r1)) * np.sin(2.0 * np.pi * r2))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_gpu{gpu_index}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_sample(rows_sample=256, threads=None):
    """The reference OzBLAS CPU library (plain ozblasRgemm, FP64 slices) on the
    first `rows_sample` rows of the same 8192^3 problem.  Test-side code: the
    oracle is only imported here, for the CPU baseline."""
    import numpy as np

    from oracle.oracle import Reference, have_reference

    if not have_reference():
        return None, "oracle/_ref/libozblas_ref.so not built"
    threads = threads or os.cpu_count()
    ref = Reference(work_bytes=int(48e9), threads=threads)
    ref.set_flags(sumMode=0, fastMode=0, nSplitMax=0, reproMode=1)
    A = np.ascontiguousarray(phi_matrix(N_DIM, N_DIM, PHI, 1)[:, :rows_sample])  # first rows, column-major
    B = phi_matrix(N_DIM, N_DIM, PHI, 2)
    C = np.zeros((N_DIM, rows_sample))
    t0 = time.perf_counter()
    ref.dgemm("n", "n", rows_sample, N_DIM, N_DIM, 1.0, A, rows_sample, B, N_DIM, 0.0, C, rows_sample)
    t = time.perf_counter() - t0
    ref.close()
    tflops = 2.0 * rows_sample * N_DIM * N_DIM / t / 1e12
    return {"value": tflops, "unit": "TFLOPS", "cores": threads, "kind": "reference",
            "sample": f"reference ozblasRgemm (plain FP64 slices, sumMode 0) on rows 0..{rows_sample - 1} of the "
                      f"8192^3 phi=1 problem ({t:.2f} s, B split included)"}, None


def max_over_ranks(value, dist):
    """The slowest rank's time (or any scalar's maximum) over the process group; `dist` None: one
    process.  NCCL groups reduce on the GPU, gloo groups (CPU tests) on the host."""
    if dist is None:
        return value
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    steps = []
    base = None
    for i in range(args.warmup + args.steps):
        base, err = cpu_reference_sample(rows_sample=args.ref_rows)
        if base is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return 0
        if i >= args.warmup:
            steps.append(base["value"])
    v = statistics.mean(steps)
    base["value"] = v
    line = {"metric": "Ozaki DGEMM TFLOPS n=8192 (INT8 vs FP64 slices, err vs MPFR); DOT/CSRMV GB/s",
            "impl": "reference", "value": v, "unit": "TFLOPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 2.0 * args.ref_rows * N_DIM * N_DIM / v / 1e9,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "ozaki_dgemm m=n=k=8192 phi=1", "m": N_DIM, "n": N_DIM, "k": N_DIM, "phi": PHI,
                       "sample_rows": args.ref_rows},
            "cpu_baseline": base, "e2e": {"value": v, "unit": "TFLOPS", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-rows", type=int, default=256)
    ap.add_argument("--full-pairs", action="store_true", help="headline with the full pair set instead of triangular")
    ap.add_argument("--n", type=int, default=N_DIM, help="m = n = k (default 8192; smaller for profiling captures)")
    ap.add_argument("--memory-only", action="store_true",
                    help="only the DOT / CSRMV / CG measurements (for profiling them; prints their JSON)")
    ap.add_argument("--cg-iters", type=int, default=2000, help="CG iterations of the memory-only run")
    ap.add_argument("--batched-only", action="store_true",
                    help="only the 256-problem grouped INT8 measurement (prints its JSON)")
    ap.add_argument("--mixed-only", action="store_true",
                    help="only the mixed-precision forms <double,float,float> and <float,double,double> at m = n = k "
                         "= --n (prints their JSON)")
    args = ap.parse_args()
    globals()["N_DIM"] = args.n
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import numpy as np
    import torch

    import ozblas_b200 as ozb

    torch.cuda.set_device(local)
    if args.batched_only:
        h = ozb.Handle(work_bytes=24 << 30)
        print(json.dumps({"workload": "batched uneven Ozaki DGEMM, 256 problems", "reps": args.steps,
                          "extras": batched_extras(ozb, h, torch, reps=args.steps)}))
        h.close()
        return 0
    if args.mixed_only:
        h = ozb.Handle(work_bytes=32 << 30)
        print(json.dumps({"workload": f"mixed-precision Ozaki GEMM {args.n}^3, phi = {PHI}", "reps": args.steps,
                          "extras": mixed_extras(ozb, h, torch, args.n, reps=args.steps)}))
        h.close()
        return 0
    if args.memory_only:
        h = ozb.Handle(work_bytes=8 << 30)
        h.nSplitMax = 0
        print(json.dumps({"workload": "memory-bound plain kernels", "reps": args.steps,
                          "extras": memory_extras(ozb, h, torch, reps=args.steps, cg_iters=args.cg_iters)}))
        h.close()
        return 0
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    n = N_DIM
    A_h = torch.from_numpy(phi_matrix(n, n, PHI, 1 + 10 * rank)).pin_memory()
    B_h = torch.from_numpy(phi_matrix(n, n, PHI, 2 + 10 * rank)).pin_memory()
    C_h = torch.empty((n, n), dtype=torch.float64).pin_memory()
    A = A_h.cuda()
    B = B_h.cuda()
    C = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    h = ozb.Handle(work_bytes=40 << 30)
    h.sumMode = 0
    h.nSplitMax = 0
    h.fastMode = 0 if args.full_pairs else 1

    def step():
        ozb.dgemm_i8(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)

    for _ in range(args.warmup):
        step()
    barrier()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kern_ms = []
    launches0 = h.launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        for i in range(args.steps):
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            kern_ms.append(h.t_comp * 1e3)
        barrier()
    launches = (h.launch_count() - launches0) / args.steps
    ms = max_over_ranks(statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev), dist)
    flops = 2.0 * n * n * n
    value = world * flops / (ms * 1e-3) / 1e12
    pairs = h.nSplitC
    nA, nB = h.nSplitA, h.nSplitB

    # ---- end to end: host buffers, copies inside the step ----
    def e2e_step():
        A.copy_(A_h, non_blocking=True)
        B.copy_(B_h, non_blocking=True)
        step()
        C_h.copy_(C, non_blocking=True)

    e2e_step()
    barrier()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        ev2[i][0].record(stream)
        e2e_step()
        ev2[i][1].record(stream)
    barrier()
    ms_e2e = max_over_ranks(statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev2), dist)
    e2e = {"value": world * flops / (ms_e2e * 1e-3) / 1e12, "unit": "TFLOPS", "h2d_bytes_per_step": 2 * n * n * 8,
           "d2h_bytes_per_step": n * n * 8, "ms_per_step": ms_e2e}

    peaks, peak_kind = measured_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]  # dense int8 rate is twice dense bf16 on B200
    kms = statistics.mean(kern_ms)
    achieved = pairs * flops / (kms * 1e-3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        key = f"k_i8_gemm_{'full' if args.full_pairs else 'tri'}_{n}"
        traffic = tj.get(key)
    roofline = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TFLOP/s", "frac": achieved / int8_peak,
                "traffic": traffic, "kernel": "k_i8_gemm (tcgen05.mma kind::i8)", "kernel_ms": kms,
                "peak_note": f"int8 ops/s; peak = 2 x {peak_kind} dense bf16 ({peaks['bf16_tflops']} TFLOP/s burst, "
                             "MEASURED_PEAKS.json)",
                "algorithmic_ops_per_launch": pairs * flops}

    line = {"metric": "Ozaki DGEMM TFLOPS n=8192 (INT8 vs FP64 slices, err vs MPFR); DOT/CSRMV GB/s",
            "value": value, "unit": "TFLOPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic",
            "config": {"workload": f"ozaki_dgemm_int8 m=n=k={n} phi=1", "m": n, "n": n, "k": n, "phi": PHI,
                       "slices": [nA, nB], "pairs": pairs, "pair_set": "full" if args.full_pairs else "triangular",
                       "sumMode": 0, "l2": "inputs 512 MiB each > L2, no flush",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": e2e, "roofline": roofline, "gpu_launches": launches, "clocks": clk.summary()}

    if rank == 0 and not args.no_extras:
        line["extras"] = extras(ozb, h, torch, A, B, C, n)
        line["extras"]["int8_vs_plain_speedup"] = line["extras"]["plain_fp64_slices"]["ms"] / ms
        line["extras"]["int8_vs_plain_int8_digits_speedup"] = (
            line["extras"]["plain_fp64_slices_int8_digits"]["ms"] / ms)
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            base, err = cpu_reference_sample(rows_sample=args.ref_rows)
        except Exception as e:  # the baseline must not take the GPU line down
            base, err = None, repr(e)
        line["cpu_baseline"] = base if base else {"value": None, "unavailable": err}
    h.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def extras(ozb, h, torch, A, B, C, n):
    """Plain form, accuracy vs the correctly rounded product, DOT/CSRMV throughput."""
    out = {}
    flops = 2.0 * n * n * n

    def timed(fn, reps=1):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    C_tri = C.clone()
    h.fastMode = 0
    ms_full = timed(lambda: ozb.dgemm_i8(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n))
    out["int8_full_pairs"] = {"TFLOPS": flops / ms_full / 1e9, "pairs": h.nSplitC, "ms": ms_full}
    C_full = C.clone()
    h.nSplitMax = 0
    # the plain form as the north star defines it: FP64 slices on the FP64 tensor pipe (DMMA)
    os.environ["OZBLAS_PLAIN_DMMA"] = "1"
    h.read_env()
    try:
        ms_plain = timed(lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n))
    finally:
        del os.environ["OZBLAS_PLAIN_DMMA"]
        h.read_env()
    out["plain_fp64_slices"] = {"TFLOPS": flops / ms_plain / 1e9, "pairs": h.nSplitC, "slices": [h.nSplitA, h.nSplitB],
                                "ms": ms_plain, "internal_fp64_TFLOPS": h.nSplitC * flops / ms_plain / 1e9,
                                "pipe": "FP64 tensor (DMMA)"}
    C_plain = C.clone()
    # the library's default plain path: the same exact slice-pair products on INT8 digits (same bits)
    ms_plain_i8 = timed(lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n))
    out["plain_fp64_slices_int8_digits"] = {"TFLOPS": flops / ms_plain_i8 / 1e9, "ms": ms_plain_i8,
                                            "bit_identical_to_dmma": bool(torch.equal(C, C_plain))}
    h.sumMode = 1
    ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
    torch.cuda.synchronize()
    C_rn = C  # correctly rounded product (NearSum over exact slice pairs)
    h.sumMode = 0

    def maxrel(X):
        d = (X - C_rn).abs() / C_rn.abs()
        d = torch.where(C_rn == 0, (X != 0).double() * float("inf"), d)
        return float(d.max().item()), int((X != C_rn).sum().item())

    e_tri, n_tri = maxrel(C_tri)
    e_full, n_full = maxrel(C_full)
    e_plain, n_plain = maxrel(C_plain)
    out["max_rel_err_vs_correctly_rounded"] = {"int8_triangular": e_tri, "int8_full": e_full, "plain_fsum": e_plain,
                                               "inexact_entries": {"int8_triangular": n_tri, "int8_full": n_full,
                                                                   "plain_fsum": n_plain},
                                               "note": "reference = plain form with NearSum (correctly rounded)"}
    del C_tri, C_full, C_plain
    torch.cuda.empty_cache()
    out.update(memory_extras(ozb, h, torch))
    out["batched_uneven_256"] = batched_extras(ozb, h, torch)
    return out


def batched_case(count=256, seed=5):
    """256 problems, m, n, k log-uniform in [64, 2048] (shape seed 5), phi from {0.5, 1, 2, 4}; problem i's A and B
    use seeds 1000 + 2i and 1001 + 2i.  Host arrays (column-major, as phi_matrix)."""
    import numpy as np

    g = np.random.default_rng(seed)
    mnk = np.exp(g.uniform(np.log(64), np.log(2048), (count, 3))).astype(int)
    phis = g.choice([0.5, 1.0, 2.0, 4.0], count)
    probs = []
    for i in range(count):
        m, n, k = (int(v) for v in mnk[i])
        probs.append((m, n, k, float(phis[i]), phi_matrix(m, k, phis[i], 1000 + 2 * i),
                      phi_matrix(k, n, phis[i], 1001 + 2 * i)))
    return probs


def batched_extras(ozb, h, torch, reps=3):
    """Config 5: 256 uneven problems in one grouped INT8 launch vs the same problems looped through the single INT8
    call and through the plain FP64-slice form; max relative error against the correctly rounded product."""
    probs = batched_case()
    flops = sum(2.0 * m * n * k for m, n, k, _, _, _ in probs)
    As = [torch.from_numpy(A).cuda() for *_, A, _ in probs]
    Bs = [torch.from_numpy(B).cuda() for *_, B in probs]
    Cs = [torch.zeros((n, m), dtype=torch.float64, device="cuda") for m, n, *_ in probs]
    ms, ns, ks = [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs]
    one, zero = [1.0] * len(probs), [0.0] * len(probs)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    out = {"problems": len(probs), "flops_effective": flops}
    for fast in (0, 1):
        h.nSplitMax, h.fastMode = 0, fast
        l0 = h.launch_count()
        ms_b = timed(lambda: ozb.dgemm_i8_batched(h, "n", "n", ms, ns, ks, one, As, ms, Bs, ks, zero, Cs, ms), reps)
        launches = (h.launch_count() - l0) / (reps + 1)
        slices = [h.nSplitA, h.nSplitB]
        C_batched = [c.clone() for c in Cs]

        def looped():
            for i in range(len(probs)):
                ozb.dgemm_i8(h, "n", "n", ms[i], ns[i], ks[i], 1.0, As[i], ms[i], Bs[i], ks[i], 0.0, Cs[i], ms[i])

        ms_l = timed(looped, 1)
        key = "full" if fast == 0 else "triangular"
        out[f"int8_grouped_{key}"] = {"ms": ms_b, "TFLOPS": flops / ms_b / 1e9, "launches": launches,
                                      "max_slices": slices}
        out[f"int8_looped_{key}"] = {"ms": ms_l, "TFLOPS": flops / ms_l / 1e9}
        out[f"grouped_identical_to_looped_{key}"] = all(bool(torch.equal(a, b)) for a, b in zip(C_batched, Cs))
        if fast == 0:
            C_full = C_batched
    h.fastMode = 0

    def plain():
        for i in range(len(probs)):
            ozb.dgemm(h, "n", "n", ms[i], ns[i], ks[i], 1.0, As[i], ms[i], Bs[i], ks[i], 0.0, Cs[i], ms[i])

    ms_p = timed(plain, 1)
    out["plain_fp64_slices_looped"] = {"ms": ms_p, "TFLOPS": flops / ms_p / 1e9}
    C_fsum = [c.clone() for c in Cs]
    h.sumMode = 1
    plain()  # correctly rounded products
    torch.cuda.synchronize()
    h.sumMode = 0

    def worst(X):
        w, cnt, where = 0.0, 0, None
        for i, (a, b) in enumerate(zip(X, Cs)):
            d = ((a - b).abs() / b.abs()).nan_to_num(nan=0.0, posinf=float("inf"))
            d = torch.where(b == 0, (a != 0).double() * float("inf"), d)
            di = float(d.max().item())
            if di > w:
                j = int(d.argmax().item())
                w, where = di, {"problem": i, "m": ms[i], "n": ns[i], "k": ks[i], "phi": probs[i][3],
                                "value": float(a.flatten()[j].item()), "correctly_rounded": float(b.flatten()[j].item())}
            cnt += int((a != b).sum().item())
        return w, cnt, where

    (e_i8, n_i8, w_i8), (e_fs, n_fs, w_fs) = worst(C_full), worst(C_fsum)
    out["max_rel_err_vs_correctly_rounded"] = {"int8_full": e_i8, "plain_fsum": e_fs,
                                               "inexact_entries": {"int8_full": n_i8, "plain_fsum": n_fs},
                                               "entries": sum(m * n for m, n, *_ in probs),
                                               "worst_int8": w_i8, "worst_fsum": w_fs}
    out["speedup_grouped_full_vs_plain_looped"] = ms_p / out["int8_grouped_full"]["ms"]
    return out


def binary128_from_phi(a, seed):
    """Binary128 values (uint64 pairs lo, hi) with the phi distribution of the double array `a` and 113
    significant bits: a's sign, exponent and 52 fraction bits, then 60 random low bits."""
    import numpy as np
    bits = np.ascontiguousarray(a, dtype=np.float64).view(np.uint64).ravel()
    sign = bits >> np.uint64(63)
    exp = (bits >> np.uint64(52)) & np.uint64(0x7FF)
    frac = bits & np.uint64((1 << 52) - 1)
    assert np.all((exp > 0) & (exp < 0x7FF)), "normal doubles only"
    low = np.random.default_rng(seed).integers(0, 1 << 60, size=bits.size, dtype=np.uint64)
    hi = (sign << np.uint64(63)) | ((exp - np.uint64(1023) + np.uint64(16383)) << np.uint64(48)) | (frac >> np.uint64(4))
    lo = ((frac & np.uint64(0xF)) << np.uint64(60)) | low
    return np.stack([lo, hi], axis=-1).reshape(a.shape + (2,))


def mixed_extras(ozb, h, torch, n, reps=3):
    """The two mixed forms through the public API on an n^3 phi problem: call time (CUDA events),
    slice counts, and the slice-product throughput of the product kernel (its phase timer)."""
    out = {}
    A64 = torch.from_numpy(phi_matrix(n, n, PHI, 1)).cuda()
    B64 = torch.from_numpy(phi_matrix(n, n, PHI, 2)).cuda()
    forms = (("dsgemm", ozb.dsgemm, A64, B64, torch.float64),
             ("sdgemm", ozb.sdgemm, A64.float(), B64.float(), torch.float32))
    # FP32 SIMT nominal: 148 SMs x 128 lanes x 2 flops at the maximum SM clock
    fp32_nominal = 148 * 128 * 2 * measured_peaks()[0].get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    for name, fn, A, B, dt in forms:
        C = torch.zeros((n, n), dtype=dt, device="cuda")
        fn(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
        torch.cuda.synchronize()
        ts, comp = [], []
        for _ in range(max(reps, 1)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            comp.append(h.t_comp * 1e3)
        ms, kms = min(ts), min(comp)
        pairs = h.nSplitC
        rec = {"ms": ms, "product_kernel_ms": kms, "slices": [h.nSplitA, h.nSplitB], "pairs": pairs,
               "dgemm_equivalent_TFLOPS": 2.0 * n ** 3 / ms / 1e9,
               "slice_product_TFLOPS": 2.0 * n ** 3 * pairs / kms / 1e9}
        if name == "dsgemm":
            if n > 1024:  # rho >= 47: the INT8 slices run on tcgen05 (kind::i8)
                peaks, how = measured_peaks()
                i8_peak = 2.0 * peaks["bf16_tflops"]
                rec["path"] = "int8 tensor cores"
                rec["int8_peak_TOPS"] = i8_peak
                rec["fraction_of_int8_peak"] = rec["slice_product_TFLOPS"] / i8_peak
                rec["peak_source"] = how
            else:
                rec["path"] = "fp32 simt"
                rec["fp32_simt_nominal_TFLOPS"] = fp32_nominal
                rec["fraction_of_fp32_nominal"] = rec["slice_product_TFLOPS"] / fp32_nominal
        out[name] = rec
        del C
    # quad I/O form: binary128 data built from the same phi matrices
    import numpy as np
    Aq = torch.from_numpy(binary128_from_phi(phi_matrix(n, n, PHI, 1), 11).view(np.int64)).cuda()
    Bq = torch.from_numpy(binary128_from_phi(phi_matrix(n, n, PHI, 2), 12).view(np.int64)).cuda()
    Cq = torch.zeros((n, n, 2), dtype=torch.int64, device="cuda")
    one = np.array([0, 0x3FFF000000000000], dtype=np.uint64)
    zero = np.zeros(2, dtype=np.uint64)
    ozb.qgemm(h, "n", "n", n, n, n, one, Aq, n, Bq, n, zero, Cq, n)
    torch.cuda.synchronize()
    ts = []
    for _ in range(max(reps, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ozb.qgemm(h, "n", "n", n, n, n, one, Aq, n, Bq, n, zero, Cq, n)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = min(ts)
    out["qgemm"] = {"ms": ms, "slices": [h.nSplitA, h.nSplitB], "pairs": h.nSplitC,
                    "split_ms": (h.t_SplitA + h.t_SplitB) * 1e3,
                    "dgemm_equivalent_TFLOPS": 2.0 * n ** 3 / ms / 1e9,
                    "slice_product_TFLOPS": 2.0 * n ** 3 * h.nSplitC / ms / 1e9}
    return out


def memory_extras(ozb, h, torch, reps=3, cg_iters=2000):
    """DOT n = 2^24 (phi = 2), GEMV 8192^2 (phi = 1), CSRMV on the 128^3 7-point stencil (both sum modes) and CG
    on 100^3, through the public API."""
    import numpy as np

    out = {}

    def timed(fn, reps=1):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    # DOT n = 2^24, phi = 2
    nv = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(7)
    r1 = torch.rand(nv, dtype=torch.float64, device="cuda", generator=g)
    r2 = torch.rand(nv, dtype=torch.float64, device="cuda", generator=g)
    x = (r1 - 0.5) * torch.exp(2.0 * torch.sqrt(-2 * torch.log(r1)) * torch.sin(2 * torch.pi * r2))
    r1 = torch.rand(nv, dtype=torch.float64, device="cuda", generator=g)
    y = (r1 - 0.5) * torch.exp(2.0 * torch.sqrt(-2 * torch.log(r1)) * torch.sin(2 * torch.pi * r2))
    for sm in (0, 1):
        h.sumMode = sm
        ms = timed(lambda: ozb.ddot(h, nv, x, y), reps=reps)
        out[f"ddot_2p24_sum{sm}"] = {"GBps": 16.0 * nv / ms / 1e6, "ms": ms, "slices": [h.nSplitA, h.nSplitB]}
    del x, y, r1, r2
    # GEMV 8192^2 (phi = 1), y = A x, beta = 0: algorithmic bytes 8 (mn + n + m)
    mg = 8192
    r1 = torch.rand(mg * mg, dtype=torch.float64, device="cuda", generator=g)
    r2 = torch.rand(mg * mg, dtype=torch.float64, device="cuda", generator=g)
    Ag = (r1 - 0.5) * torch.exp(torch.sqrt(-2 * torch.log(r1)) * torch.sin(2 * torch.pi * r2))
    del r1, r2
    r1 = torch.rand(mg, dtype=torch.float64, device="cuda", generator=g)
    xg = (r1 - 0.5) * torch.exp(torch.sqrt(-2 * torch.log(r1)))
    yg = torch.zeros(mg, dtype=torch.float64, device="cuda")
    for sm in (0, 1):
        h.sumMode = sm
        ms = timed(lambda: ozb.dgemv(h, "n", mg, mg, 1.0, Ag, mg, xg, 0.0, yg), reps=reps)
        out[f"dgemv_8192_sum{sm}"] = {"GBps": 8.0 * (mg * mg + 2 * mg) / ms / 1e6, "ms": ms,
                                      "slices": [h.nSplitA, h.nSplitB]}
    del Ag, xg, yg, r1
    torch.cuda.empty_cache()
    # CSRMV: 7-point stencil on 128^3, values and x (U - 0.5) exp(N(0,1)), beta = 0
    g3 = 128
    m = g3 ** 3
    idx = torch.arange(m, device="cuda", dtype=torch.int64)
    xi, yi, zi = idx % g3, (idx // g3) % g3, idx // (g3 * g3)
    offs = [(-g3 * g3, zi > 0), (-g3, yi > 0), (-1, xi > 0), (0, None), (1, xi < g3 - 1), (g3, yi < g3 - 1),
            (g3 * g3, zi < g3 - 1)]
    cols, masks = [], []
    for o, msk in offs:
        cols.append(idx + o)
        masks.append(torch.ones(m, dtype=torch.bool, device="cuda") if msk is None else msk)
    C7 = torch.stack(cols, 1)
    M7 = torch.stack(masks, 1)
    colind = C7[M7].to(torch.int32).contiguous()
    rowptr = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
    rowptr[1:] = torch.cumsum(M7.sum(1), 0)
    rowptr = rowptr.to(torch.int32).contiguous()
    nnz = colind.numel()
    r1 = torch.rand(nnz, dtype=torch.float64, device="cuda", generator=g)
    r2 = torch.rand(nnz, dtype=torch.float64, device="cuda", generator=g)
    val = (r1 - 0.5) * torch.exp(torch.sqrt(-2 * torch.log(r1)) * torch.sin(2 * torch.pi * r2))
    r1 = torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    r2 = torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    xv = (r1 - 0.5) * torch.exp(torch.sqrt(-2 * torch.log(r1)) * torch.sin(2 * torch.pi * r2))
    yv = torch.zeros(m, dtype=torch.float64, device="cuda")
    nbytes = 12.0 * nnz + 4.0 * (m + 1) + 8.0 * m + 8.0 * m
    for sm in (0, 1):
        h.sumMode = sm
        ms = timed(lambda: ozb.dcsrmv(h, "n", m, m, nnz, 1.0, val, colind, rowptr, xv, 0.0, yv), reps=reps)
        out[f"dcsrmv_stencil128_sum{sm}"] = {"GBps": nbytes / ms / 1e6, "ms": ms, "nnz": nnz,
                                             "slices": [h.nSplitA, h.nSplitB]}
    # CG: 7-point Poisson on 100^3 plus 0.01 U(0,1) on the diagonal, b = A x_true,
    # 2000 iterations (tol 0), NearSum, history every iteration (verbose = 1)
    del val, colind, rowptr, xv, yv, C7, M7, cols, masks, idx, xi, yi, zi
    torch.cuda.empty_cache()
    g3 = 100
    m = g3 ** 3
    idx = torch.arange(m, device="cuda", dtype=torch.int64)
    xi, yi, zi = idx % g3, (idx // g3) % g3, idx // (g3 * g3)
    offs = [(-g3 * g3, zi > 0), (-g3, yi > 0), (-1, xi > 0), (0, None), (1, xi < g3 - 1), (g3, yi < g3 - 1),
            (g3 * g3, zi < g3 - 1)]
    C7 = torch.stack([idx + o for o, _ in offs], 1)
    M7 = torch.stack([torch.ones(m, dtype=torch.bool, device="cuda") if k is None else k for _, k in offs], 1)
    V7 = torch.full((m, 7), -1.0, dtype=torch.float64, device="cuda")
    V7[:, 3] = 6.0 + 0.01 * torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    colind = C7[M7].to(torch.int32).contiguous()
    val = V7[M7].contiguous()
    rowptr = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
    rowptr[1:] = torch.cumsum(M7.sum(1), 0)
    rowptr = rowptr.to(torch.int32).contiguous()
    nnz = colind.numel()
    xt = torch.randn(m, dtype=torch.float64, device="cuda", generator=g)
    b = (torch.where(M7, V7 * xt[C7.clamp(0, m - 1)], torch.zeros_like(V7))).sum(1).contiguous()
    xs = torch.zeros(m, dtype=torch.float64, device="cuda")
    iters = cg_iters
    h1 = np.zeros(iters + 1)
    h2 = np.zeros(iters + 1)
    h.sumMode, h.verbose = 1, 1
    ms = timed(lambda: (xs.zero_(), ozb.dcg(h, "n", m, nnz, val, colind, rowptr, b, xs, iters, 0.0, h1, h2)),
               reps=min(reps, 2))
    l0 = h.launch_count()
    xs.zero_()
    ozb.dcg(h, "n", m, nnz, val, colind, rowptr, b, xs, iters, 0.0, h1, h2)
    per_iter_bytes = 12.0 * nnz + 4.0 * (m + 1) + 116.0 * m
    out[f"dcg_100cube_{iters}it"] = {"ms": ms, "ms_per_iter": ms / iters, "GBps": per_iter_bytes * iters / ms / 1e6,
                                 "iterations": h.cg_numiter, "nnz": nnz, "final_rel_res": float(h1[iters]),
                                 "launches_per_iter": (h.launch_count() - l0) / iters,
                                 "bytes_per_iter": per_iter_bytes}
    h.sumMode, h.verbose = 0, 0
    return out


if __name__ == "__main__":
    sys.exit(main())
