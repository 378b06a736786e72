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
roofline  the tcgen05 product kernel alone (its phase timer: CUDA events
        around its launch on the handle's stream): int8 ops per launch =
        pairs * 2 m n k.
cpu_baseline  the reference OzBLAS CPU library (oracle/_ref, built from the
        reference's src/cpu) running its plain ozblasRgemm as one full
        2048^3 call on all host cores; `--impl reference` times the same call
        per step.

extras (rank 0): full pairs and the plain FP64-slice form at the headline
size; config 1 (plain DGEMM 1024^3, bits against the reference CPU library);
config 2 (DOT / NRM2 / GEMV / CSRMV, both sum modes) and config 4 (CG 100^3,
2000 iterations) with HBM rooflines, CPU baselines and bit checks; config 5
(256 uneven problems in one grouped launch); config 3 (the INT8 form over
m = n = k in {2048, 4096, 8192, 16384} x phi in {0.5, 1, 2, 4} x {triangular,
full}, beside the plain form and native FP64 GEMM).  Accuracy everywhere is
measured against the exact product (an exact accumulator of the oracle's C
restatement) on sampled entries, outside the timed regions.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DIM = 8192
PHI = 1.0
METRIC = "Ozaki DGEMM TFLOPS n=8192 (INT8 vs FP64 slices, err vs MPFR); DOT/CSRMV GB/s"

_JSON_FD = None


def claim_stdout():
    """Send everything written to file descriptor 1 from here on (the reference CPU library's own printf
    included) to stderr, so that standard output carries the JSON line alone."""
    global _JSON_FD
    if _JSON_FD is None:
        sys.stdout.flush()
        _JSON_FD = os.dup(1)
        os.dup2(2, 1)


def emit(obj):
    """Write one JSON line to the original standard output."""
    os.write(_JSON_FD if _JSON_FD is not None else 1, (json.dumps(obj) + "\n").encode())


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
        # the raw samples: $OZBLAS_CLOCKS_DIR when set, else the system's temporary directory
        out_dir = os.environ.get("OZBLAS_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_gpu{gpu_index}.csv")

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


# ---------------------------------------------------------------------------
# Checker and CPU-baseline legs.  Everything below that touches oracle/ runs
# outside every timed GPU region: the reference OzBLAS CPU library
# (oracle/_ref, built from the reference's own src/cpu) is timed as the CPU
# baseline and gives the bits the plain form must equal; the C restatement's
# exact accumulator is the accuracy checker.  Neither is on the measured path.
# ---------------------------------------------------------------------------
REF_GEMM_N = 2048  # the reference CPU GEMM baseline: one full call at this size


def _reference(threads=None):
    from oracle.oracle import Reference, have_reference

    if not have_reference():
        return None
    return Reference(work_bytes=int(48e9), threads=threads or os.cpu_count())


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference_gemm(n=REF_GEMM_N, reps=1, phi=PHI, ref=None):
    """The reference CPU library's plain ozblasRgemm (FP64 slices, FSum) as one full n^3 call, B split included,
    min over `reps` calls after one warm-up call (the reference harness: testing/testing_level3.cpp:184-205).
    Returns (baseline dict, C of the last call) or (None, reason)."""
    import numpy as np

    own = ref is None
    ref = ref or _reference()
    if ref is None:
        return None, "oracle/_ref/libozblas_ref.so not built"
    ref.set_flags(sumMode=0, fastMode=0, nSplitMax=0, reproMode=1)
    A = phi_matrix(n, n, phi, 1)
    B = phi_matrix(n, n, phi, 2)
    C = np.zeros((n, n))
    out = ref.dgemm("n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # warm-up
    ts = []
    for _ in range(max(reps, 1)):
        t0 = time.perf_counter()
        out = ref.dgemm("n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
        ts.append(time.perf_counter() - t0)
    info = ref.info()
    cores = ref.threads()
    if own:
        ref.close()
    t = min(ts)
    return {"value": 2.0 * n ** 3 / t / 1e12, "unit": "TFLOPS", "cores": cores, "kind": "reference",
            "cpu_model": _cpu_model(),
            "sample": f"reference ozblasRgemm (plain FP64 slices {int(info['nSplitA'])}x{int(info['nSplitB'])}, "
                      f"sumMode 0) as one full m=n=k={n} phi={phi} call, B split included; min of {len(ts)} after "
                      f"1 warm-up ({t:.3f} s)"}, out

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
    """The reference's own CPU implementation (oracle/_ref) on the host cores: each step one full plain-form
    ozblasRgemm call at m=n=k=REF_GEMM_N (the headline workload's algorithm at a CPU-bounded size)."""
    if rank != 0:
        return 0
    ref = _reference()
    if ref is None:
        emit({"impl": "reference", "unavailable": "oracle/_ref/libozblas_ref.so not built"})
        return 0
    import numpy as np

    n = REF_GEMM_N
    ref.set_flags(sumMode=0, fastMode=0, nSplitMax=0, reproMode=1)
    A = phi_matrix(n, n, PHI, 1)
    B = phi_matrix(n, n, PHI, 2)
    C = np.zeros((n, n))
    ts = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ref.dgemm("n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
        if i >= args.warmup:
            ts.append(time.perf_counter() - t0)
    info = ref.info()
    cores = ref.threads()
    ref.close()
    ms = statistics.mean(ts) * 1e3
    v = 2.0 * n ** 3 / (ms * 1e-3) / 1e12
    base = {"value": v, "unit": "TFLOPS", "cores": cores, "kind": "reference", "cpu_model": _cpu_model(),
            "sample": f"reference ozblasRgemm (plain FP64 slices {int(info['nSplitA'])}x{int(info['nSplitB'])}, "
                      f"sumMode 0), one full m=n=k={n} phi={PHI} call per step, B split included"}
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "TFLOPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"ozaki_dgemm plain m=n=k={n} phi={PHI} (CPU-bounded size of the 8192^3 "
                                   "workload)", "m": n, "n": n, "k": n, "phi": PHI},
            "cpu_baseline": base, "e2e": {"value": v, "unit": "TFLOPS", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    emit(line)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--sweep-sizes", default="2048,4096,8192,16384",
                    help="m = n = k of the INT8 form sweep (comma separated; empty: no sweep)")
    ap.add_argument("--sweep-phis", default="0.5,1,2,4")
    ap.add_argument("--sweep-only", action="store_true", help="only the INT8 form sweep (prints its JSON)")
    ap.add_argument("--full-pairs", action="store_true", help="headline with the full pair set instead of triangular")
    ap.add_argument("--n", type=int, default=N_DIM, help="m = n = k (default 8192; smaller for profiling captures)")
    ap.add_argument("--work-gb", type=int, default=40, help="arena of the headline handle (GB)")
    ap.add_argument("--memory-only", action="store_true",
                    help="only the DOT / CSRMV / CG measurements (for profiling them; prints their JSON)")
    ap.add_argument("--cg-iters", type=int, default=2000, help="CG iterations of the memory-only run")
    ap.add_argument("--batched-only", action="store_true",
                    help="only the 256-problem grouped INT8 measurement (prints its JSON)")
    ap.add_argument("--mixed-only", action="store_true",
                    help="only the mixed-precision forms <double,float,float> and <float,double,double> at m = n = k "
                         "= --n (prints their JSON)")
    args = ap.parse_args()
    claim_stdout()
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
    sizes = [int(v) for v in args.sweep_sizes.split(",") if v.strip()]
    phis = [float(v) for v in args.sweep_phis.split(",") if v.strip()]
    if args.sweep_only:
        emit({"workload": "INT8 form sweep", "extras": sweep_extras(ozb, torch, sizes, phis)})
        return 0
    if args.batched_only:
        h = ozb.Handle(work_bytes=24 << 30)
        emit({"workload": "batched uneven Ozaki DGEMM, 256 problems", "reps": args.steps,
              "extras": batched_extras(ozb, h, torch, reps=args.steps, cpu=not args.no_cpu)})
        h.close()
        return 0
    if args.mixed_only:
        h = ozb.Handle(work_bytes=32 << 30)
        emit({"workload": f"mixed-precision Ozaki GEMM {args.n}^3, phi = {PHI}", "reps": args.steps,
              "extras": mixed_extras(ozb, h, torch, args.n, reps=args.steps)})
        h.close()
        return 0
    if args.memory_only:
        h = ozb.Handle(work_bytes=8 << 30)
        h.nSplitMax = 0
        emit({"workload": "memory-bound plain kernels", "reps": args.steps,
              "extras": memory_extras(ozb, h, torch, reps=args.steps, cg_iters=args.cg_iters,
                                      cpu=not args.no_cpu)})
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
    h = ozb.Handle(work_bytes=args.work_gb << 30)
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
    # the level-blocked kernel unless the handle was switched to the level-wise one
    kname = "k_i8_gemm" if os.environ.get("OZBLAS_I8_LEVELWISE", "0") not in ("", "0") else "k_i8_blk"
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        key = f"{kname}_{'full' if args.full_pairs else 'tri'}_{n}"
        traffic = tj.get(key)
    roofline = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TFLOP/s", "frac": achieved / int8_peak,
                "traffic": traffic, "kernel": f"{kname} (tcgen05.mma kind::i8)", "kernel_ms": kms,
                "peak_note": f"int8 ops/s; peak = 2 x {peak_kind} dense bf16 ({peaks['bf16_tflops']} TFLOP/s burst, "
                             "MEASURED_PEAKS.json)",
                "algorithmic_ops_per_launch": pairs * flops}

    line = {"metric": METRIC,
            "value": value, "unit": "TFLOPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic",
            "config": {"workload": f"ozaki_dgemm_int8 m=n=k={n} phi=1", "m": n, "n": n, "k": n, "phi": PHI,
                       "slices": [nA, nB], "pairs": pairs, "pair_set": "full" if args.full_pairs else "triangular",
                       "sumMode": 0, "l2": "inputs 512 MiB each > L2, no flush",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": e2e, "roofline": roofline, "gpu_launches": launches, "clocks": clk.summary()}

    cpu = rank == 0 and world == 1 and not args.no_cpu
    if rank == 0 and not args.no_extras:
        line["extras"] = extras(ozb, h, torch, A, B, C, n, ms, cpu=cpu, sizes=sizes, phis=phis)
    if cpu:
        try:
            base, err = cpu_reference_gemm()
        except Exception as e:  # the baseline must not take the GPU line down
            base, err = None, repr(e)
        line["cpu_baseline"] = base if base else {"value": None, "unavailable": err}
    h.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        emit(line)
    return 0


def timed_ms(torch, fn, reps=1, warm=1):
    """Minimum CUDA-event time (ms) of `fn` on the current stream over `reps` runs after `warm` untimed runs."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(max(reps, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return min(ts)


def phi_device(torch, rows, cols, phi, seed):
    """(U - 0.5) * exp(phi * N(0,1)) generated on the GPU (seeded), column-major rows x cols (tensor[j, i] = X(i, j))."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    r1 = torch.rand((cols, rows), dtype=torch.float64, device="cuda", generator=g)
    r2 = torch.rand((cols, rows), dtype=torch.float64, device="cuda", generator=g)
    r2.mul_(2.0 * 3.141592653589793).sin_()
    x = torch.log(r1).mul_(-2.0).sqrt_().mul_(r2).mul_(phi).exp_()
    del r2
    return x.mul_(r1.sub_(0.5))


def exact_errors(orc, Arows, Bcols, blocks):
    """Checker (exact accumulator of the C restatement): for each name -> computed block (column-major nr x nc,
    shape (nc, nr)), the max componentwise relative error against the exact product and the number of entries
    that differ from the correctly rounded value."""
    import numpy as np

    out = {}
    for name, Cb in blocks.items():
        rn, rel = orc.exact_gemm_block(Arows, Bcols, Cb)
        Cb = np.ascontiguousarray(Cb, dtype=np.float64).reshape(rn.shape)
        out[name] = {"max_rel_err": float(np.max(rel)) if rel.size else 0.0,
                     "inexact": int(np.count_nonzero(Cb.view(np.int64) != rn.view(np.int64))), "checked": int(rn.size)}
    return out


def merge_errors(acc, new):
    for name, e in new.items():
        a = acc.setdefault(name, {"max_rel_err": 0.0, "inexact": 0, "checked": 0})
        a["max_rel_err"] = max(a["max_rel_err"], e["max_rel_err"])
        a["inexact"] += e["inexact"]
        a["checked"] += e["checked"]
    return acc


def sampled_check(orc, torch, TA, TB, outs, nsamp=64, seed=3, full_lines=False):
    """Exact-oracle accuracy of n x n products (tensors in column-major layout T[j, i]): a seeded 64 x 64 block of
    sampled rows and columns (4096 entries), plus, with full_lines, every entry of row 0 and of column 0."""
    import numpy as np

    from oracle.oracle import Restatement

    orc = orc or Restatement()
    n = TA.shape[0]
    g = np.random.default_rng(seed)
    rows = np.sort(g.choice(n, size=min(nsamp, n), replace=False))
    cols = np.sort(g.choice(n, size=min(nsamp, n), replace=False))
    ri, ci = torch.as_tensor(rows, device="cuda"), torch.as_tensor(cols, device="cuda")
    Arows = TA[:, ri].T.contiguous().cpu().numpy()
    Bcols = TB[ci, :].contiguous().cpu().numpy()
    acc = exact_errors(orc, Arows, Bcols, {k: v[ci][:, ri].contiguous().cpu().numpy() for k, v in outs.items()})
    if full_lines:
        Ball = TB.cpu().numpy()
        merge_errors(acc, exact_errors(orc, TA[:, 0:1].T.contiguous().cpu().numpy(), Ball,
                                       {k: v[:, 0:1].contiguous().cpu().numpy() for k, v in outs.items()}))
        del Ball
        Aall = TA.T.contiguous().cpu().numpy()
        merge_errors(acc, exact_errors(orc, Aall, TB[0:1, :].contiguous().cpu().numpy(),
                                       {k: v[0:1, :].contiguous().cpu().numpy() for k, v in outs.items()}))
    return acc


def i8_roofline(pairs, n, kernel_ms, peak):
    achieved = pairs * 2.0 * n ** 3 / (kernel_ms * 1e-3) / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak}


def sweep_extras(ozb, torch, sizes, phis, plain_max=8192, dmma_max=4096):
    """Config 3: the INT8 form at m = n = k in `sizes` x phi in `phis` x {triangular, full} pair sets, each timed
    through the public API (min of 2 after a warm-up) with its product kernel's time (phase timer), against the
    plain FP64-slice form (INT8-digit products, and DMMA up to dmma_max) and native FP64 GEMM (cuBLAS DGEMM through
    torch, a comparison only); accuracy of every form against the exact product (oracle accumulator) on 4096
    sampled entries, plus full row 0 and column 0 at n <= 4096."""
    from oracle.oracle import Restatement

    orc = Restatement()
    peaks, peak_kind = measured_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    rows = []
    for n in sizes:
        h = ozb.Handle(work_bytes=(110 << 30) if n > 8192 else (48 << 30))
        for phi in phis:
            TA = phi_device(torch, n, n, phi, 1)
            TB = phi_device(torch, n, n, phi, 2)
            C = torch.zeros((n, n), dtype=torch.float64, device="cuda")
            flops = 2.0 * n ** 3
            outs, rec = {}, {"n": n, "phi": phi}
            h.sumMode, h.nSplitMax = 0, 0
            for fast, key in ((1, "int8_triangular"), (0, "int8_full")):
                h.fastMode = fast
                kms = []

                def call():
                    ozb.dgemm_i8(h, "n", "n", n, n, n, 1.0, TA, n, TB, n, 0.0, C, n)
                    kms.append(h.t_comp * 1e3)

                ms = timed_ms(torch, call, reps=2)
                kern = min(kms[1:])
                rec[key] = {"ms": ms, "TFLOPS": flops / ms / 1e9, "kernel_ms": kern, "digits": [h.nSplitA, h.nSplitB],
                            "pairs": h.nSplitC, "roofline": i8_roofline(h.nSplitC, n, kern, int8_peak)}
                outs[key] = C.clone()
            h.fastMode = 0
            if n <= plain_max:
                ms = timed_ms(torch, lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, TA, n, TB, n, 0.0, C, n), reps=1)
                rec["plain_int8_digits"] = {"ms": ms, "TFLOPS": flops / ms / 1e9, "slices": [h.nSplitA, h.nSplitB],
                                            "pairs": h.nSplitC}
                outs["plain_fsum"] = C.clone()
            if n <= dmma_max:
                os.environ["OZBLAS_PLAIN_DMMA"] = "1"
                h.read_env()
                try:
                    ms = timed_ms(torch, lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, TA, n, TB, n, 0.0, C, n),
                                  reps=1)
                finally:
                    del os.environ["OZBLAS_PLAIN_DMMA"]
                    h.read_env()
                rec["plain_dmma"] = {"ms": ms, "TFLOPS": flops / ms / 1e9,
                                     "internal_fp64_TFLOPS": h.nSplitC * flops / ms / 1e9,
                                     "bits_equal_int8_digits": bool(torch.equal(C, outs["plain_fsum"]))}
            ms = timed_ms(torch, lambda: torch.mm(TB, TA, out=C), reps=2)
            rec["native_dgemm_cublas"] = {"ms": ms, "TFLOPS": flops / ms / 1e9, "note": "comparison only"}
            outs["native_dgemm"] = C.clone()
            del C
            rec["accuracy_vs_exact"] = sampled_check(orc, torch, TA, TB, outs, full_lines=n <= 4096)
            if "plain_int8_digits" in rec:
                rec["int8_triangular_vs_plain_speedup"] = rec["plain_int8_digits"]["ms"] / rec["int8_triangular"]["ms"]
            if "plain_dmma" in rec:
                rec["int8_triangular_vs_plain_dmma_speedup"] = rec["plain_dmma"]["ms"] / rec["int8_triangular"]["ms"]
            rows.append(rec)
            del TA, TB, outs
            torch.cuda.empty_cache()
        h.close()
    return {"rows": rows, "int8_peak_TOPS": int8_peak, "peak_source": peak_kind,
            "accuracy_method": "exact accumulator of the C restatement (RN of the exact dot); 64 x 64 sampled "
                               "entries, plus all of row 0 and column 0 at n <= 4096",
            "inputs": "(U - 0.5) exp(phi N(0,1)) generated on the GPU, seeds 1 (A) and 2 (B)"}


def extras(ozb, h, torch, A, B, C, n, ms_headline, cpu=True, sizes=(), phis=()):
    """Everything the line reports beside the headline: full pairs at the headline size, the plain form, accuracy
    against the exact product, configs 1, 2, 4 and 5, the config 3 sweep, and their CPU baselines."""
    out = {}
    flops = 2.0 * n * n * n

    C_tri = C.clone()
    h.fastMode = 0
    ms_full = timed_ms(torch, lambda: ozb.dgemm_i8(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n))
    out["int8_full_pairs"] = {"TFLOPS": flops / ms_full / 1e9, "pairs": h.nSplitC, "ms": ms_full}
    C_full = C.clone()
    h.nSplitMax = 0
    # the plain form as the reference computes it: FP64 slices, here on the FP64 tensor pipe (DMMA)
    os.environ["OZBLAS_PLAIN_DMMA"] = "1"
    h.read_env()
    try:
        ms_plain = timed_ms(torch, lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n), warm=0)
    finally:
        del os.environ["OZBLAS_PLAIN_DMMA"]
        h.read_env()
    out["plain_fp64_slices"] = {"TFLOPS": flops / ms_plain / 1e9, "pairs": h.nSplitC, "slices": [h.nSplitA, h.nSplitB],
                                "ms": ms_plain, "internal_fp64_TFLOPS": h.nSplitC * flops / ms_plain / 1e9,
                                "pipe": "FP64 tensor (DMMA)"}
    C_plain = C.clone()
    # the library's default plain path: the same exact slice-pair products on INT8 digits (same bits)
    ms_plain_i8 = timed_ms(torch, lambda: ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n))
    out["plain_fp64_slices_int8_digits"] = {"TFLOPS": flops / ms_plain_i8 / 1e9, "ms": ms_plain_i8,
                                            "bit_identical_to_dmma": bool(torch.equal(C, C_plain))}
    out["int8_vs_plain_speedup"] = ms_plain / ms_headline
    out["int8_vs_plain_int8_digits_speedup"] = ms_plain_i8 / ms_headline
    out["accuracy_vs_exact"] = sampled_check(None, torch, A, B, {"int8_triangular": C_tri, "int8_full": C_full,
                                                                 "plain_fsum": C_plain})
    out["accuracy_vs_exact"]["method"] = "exact accumulator of the C restatement on 64 x 64 sampled entries"
    del C_tri, C_full, C_plain
    torch.cuda.empty_cache()
    out["config1_plain_dgemm_1024"] = config1_extras(ozb, torch, cpu=cpu)
    out.update(memory_extras(ozb, h, torch, cpu=cpu))
    out["batched_uneven_256"] = batched_extras(ozb, h, torch, cpu=cpu)
    if sizes:
        out["config3_int8_sweep"] = sweep_extras(ozb, torch, sizes, phis)
    return out


def config1_extras(ozb, torch, cpu=True, n=1024):
    """Config 1: plain DGEMM 1024^3, phi = 1, FSum, split until exact: time through the public API, and the bits
    against the reference CPU library on the same host inputs (plus its time, min of 10 after a warm-up)."""
    import numpy as np

    A_h = phi_matrix(n, n, 1.0, 1)
    B_h = phi_matrix(n, n, 1.0, 2)
    A, B = torch.from_numpy(A_h).cuda(), torch.from_numpy(B_h).cuda()
    C = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    h = ozb.Handle(work_bytes=8 << 30)
    h.sumMode, h.nSplitMax, h.fastMode = 0, 0, 0
    kms = []

    def call():
        ozb.dgemm(h, "n", "n", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
        kms.append(h.t_comp * 1e3)

    ms = timed_ms(torch, call, reps=10)
    pairs, nA, nB = h.nSplitC, h.nSplitA, h.nSplitB
    h.close()
    flops = 2.0 * n ** 3
    peaks, _ = measured_peaks()
    digits = (53 - int(ozb.rule_rho(n, 0)) + 1 + 6) // 7  # int8 digit planes per FP64 slice
    kern = min(kms[1:])
    i8_ops = pairs * digits * digits * flops
    rec = {"ms": ms, "TFLOPS": flops / ms / 1e9, "slices": [nA, nB], "pairs": pairs,
           "internal_fp64_TFLOPS": pairs * flops / ms / 1e9, "product_kernel_ms": kern,
           "roofline": {"bound": "tensor", "unit": "TFLOP/s", "achieved": i8_ops / (kern * 1e-3) / 1e12,
                        "peak": 2.0 * peaks["bf16_tflops"],
                        "frac": i8_ops / (kern * 1e-3) / 1e12 / (2.0 * peaks["bf16_tflops"]),
                        "work": f"pairs x {digits}^2 int8 digit-plane products x 2mnk"}}
    if cpu:
        ref = _reference()
        if ref is None:
            rec["cpu_baseline"] = {"value": None, "unavailable": "oracle/_ref not built"}
        else:
            base, C_ref = cpu_reference_gemm(n=n, reps=10, phi=1.0, ref=ref)
            ref.close()
            rec["cpu_baseline"] = base
            out = C.cpu().numpy()
            rec["bit_exact_vs_reference"] = bool(np.array_equal(out.view(np.int64), C_ref.view(np.int64)))
    return rec


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


def batched_extras(ozb, h, torch, reps=3, cpu=True):
    """Config 5: 256 uneven problems in one grouped INT8 launch vs the same problems looped through the single INT8
    call and through the plain FP64-slice form; accuracy of the grouped results and of the plain FSum against the
    exact product (oracle accumulator, 16 x 16 sampled entries per problem); with cpu, the reference CPU library
    looped over problems 0..15."""
    import numpy as np

    from oracle.oracle import Restatement

    probs = batched_case()
    flops = sum(2.0 * m * n * k for m, n, k, _, _, _ in probs)
    As = [torch.from_numpy(A).cuda() for *_, A, _ in probs]
    Bs = [torch.from_numpy(B).cuda() for *_, B in probs]
    Cs = [torch.zeros((n, m), dtype=torch.float64, device="cuda") for m, n, *_ in probs]
    ms, ns, ks = [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs]
    one, zero = [1.0] * len(probs), [0.0] * len(probs)

    out = {"problems": len(probs), "flops_effective": flops}
    peaks, _ = measured_peaks()
    for fast in (0, 1):
        h.nSplitMax, h.fastMode = 0, fast
        l0 = h.launch_count()
        kms, sms = [], []

        def grouped():
            ozb.dgemm_i8_batched(h, "n", "n", ms, ns, ks, one, As, ms, Bs, ks, zero, Cs, ms)
            kms.append(h.t_comp * 1e3)
            sms.append(h.t_SplitA * 1e3)

        ms_b = timed_ms(torch, grouped, reps)
        launches = (h.launch_count() - l0) / (reps + 1)
        slices = [h.nSplitA, h.nSplitB]
        C_batched = [c.clone() for c in Cs]

        def looped():
            for i in range(len(probs)):
                ozb.dgemm_i8(h, "n", "n", ms[i], ns[i], ks[i], 1.0, As[i], ms[i], Bs[i], ks[i], 0.0, Cs[i], ms[i])

        ms_l = timed_ms(torch, looped, 1)
        key = "full" if fast == 0 else "triangular"
        out[f"int8_grouped_{key}"] = {"ms": ms_b, "TFLOPS": flops / ms_b / 1e9, "launches": launches,
                                      "max_slices": slices, "product_kernel_ms": min(kms[1:]),
                                      "split_ms": min(sms[1:])}
        out[f"int8_looped_{key}"] = {"ms": ms_l, "TFLOPS": flops / ms_l / 1e9}
        out[f"grouped_identical_to_looped_{key}"] = all(bool(torch.equal(a, b)) for a, b in zip(C_batched, Cs))
        if fast == 0:
            C_full = C_batched
    h.fastMode = 0

    def plain():
        for i in range(len(probs)):
            ozb.dgemm(h, "n", "n", ms[i], ns[i], ks[i], 1.0, As[i], ms[i], Bs[i], ks[i], 0.0, Cs[i], ms[i])

    ms_p = timed_ms(torch, plain, 1)
    out["plain_fp64_slices_looped"] = {"ms": ms_p, "TFLOPS": flops / ms_p / 1e9}
    C_fsum = [c.clone() for c in Cs]
    # checker: 16 x 16 sampled entries per problem against the exact product
    orc = Restatement()
    acc = {}
    g = np.random.default_rng(9)
    for i, (m, n, k, _, A_h, B_h) in enumerate(probs):
        rows = np.sort(g.choice(m, size=min(16, m), replace=False))
        cols = np.sort(g.choice(n, size=min(16, n), replace=False))
        Arows = np.ascontiguousarray(A_h[:, rows].T)
        Bcols = np.ascontiguousarray(B_h[cols, :])
        ri, ci = torch.as_tensor(rows, device="cuda"), torch.as_tensor(cols, device="cuda")
        blocks = {name: X[i][ci][:, ri].contiguous().cpu().numpy()
                  for name, X in (("int8_grouped_full", C_full), ("plain_fsum", C_fsum))}
        merge_errors(acc, exact_errors(orc, Arows, Bcols, blocks))
    acc["method"] = "exact accumulator of the C restatement, 16 x 16 sampled entries per problem"
    out["accuracy_vs_exact"] = acc
    out["speedup_grouped_full_vs_plain_looped"] = ms_p / out["int8_grouped_full"]["ms"]
    if cpu:
        ref = _reference()
        if ref is not None:
            ref.set_flags(sumMode=0, fastMode=0, nSplitMax=0, reproMode=1)
            t, fl = 0.0, 0.0
            for m, n, k, _, A_h, B_h in probs[:16]:
                Cz = np.zeros((n, m))
                ref.dgemm("n", "n", m, n, k, 1.0, A_h, m, B_h, k, 0.0, Cz, m)  # warm-up
                t0 = time.perf_counter()
                ref.dgemm("n", "n", m, n, k, 1.0, A_h, m, B_h, k, 0.0, Cz, m)
                t += time.perf_counter() - t0
                fl += 2.0 * m * n * k
            out["cpu_baseline"] = {"value": fl / t / 1e12, "unit": "TFLOPS", "cores": ref.threads(),
                                   "kind": "reference", "cpu_model": _cpu_model(),
                                   "sample": f"reference ozblasRgemm (plain, sumMode 0) looped over problems 0..15 "
                                             f"({fl / 1e9:.1f} GFLOP effective, {t:.2f} s, each after a warm-up)"}
            ref.close()
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


def stencil7(g3):
    """7-point stencil CSR on a g3^3 grid, natural order, sorted columns (32-bit): (rowptr, colind)."""
    import numpy as np

    m = g3 ** 3
    idx = np.arange(m, dtype=np.int64)
    xi, yi, zi = idx % g3, (idx // g3) % g3, idx // (g3 * g3)
    offs = [(-g3 * g3, zi > 0), (-g3, yi > 0), (-1, xi > 0), (0, np.ones(m, bool)), (1, xi < g3 - 1),
            (g3, yi < g3 - 1), (g3 * g3, zi < g3 - 1)]
    C7 = np.stack([idx + o for o, _ in offs], 1)
    M7 = np.stack([k for _, k in offs], 1)
    colind = C7[M7].astype(np.int32)
    rowptr = np.zeros(m + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(M7.sum(1))
    return rowptr.astype(np.int32), colind, M7


def hbm_roofline(nbytes, ms, traffic=None, what="whole call"):
    peaks, kind = measured_peaks()
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "timed": what, "peak_source": kind,
            "algorithmic_bytes": nbytes}


def span_ms(h, fn, reps=3):
    """Minimum device span (ms) of a call's kernels over `reps` calls, from the exec info's t_comp (CUDA events
    the library records on its stream before the call's first kernel and after its last)."""
    ts = []
    for _ in range(max(reps, 1)):
        fn()
        ts.append(float(h.t_comp) * 1e3)
    return min(ts)


def mem_record(h, fn, nb, ms, traffic, reps, **kw):
    """A memory-bound call's record: whole-call GB/s (CUDA events around the API call, host work included) and
    the HBM roofline of the call's kernels (algorithmic bytes over their device span)."""
    kms = span_ms(h, fn, reps)
    rec = {"GBps": nb / ms / 1e6, "ms": ms, "kernel_ms": kms, "slices": [h.nSplitA, h.nSplitB], **kw}
    if kms > 0:
        rec["roofline"] = hbm_roofline(nb, kms, traffic, what="device span of the call's kernels")
    rec["roofline_whole_call"] = hbm_roofline(nb, ms, None)
    return rec


def ncu_traffic(key):
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            return json.load(f).get(key)
    return None


def cpu_mean(fn, reps):
    """Mean wall time (s) of `fn` over `reps` calls after one warm-up call, and the last result."""
    r = fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = fn()
        ts.append(time.perf_counter() - t0)
    return statistics.mean(ts), r


def memory_extras(ozb, h, torch, reps=3, cg_iters=2000, cpu=True):
    """Config 2 (DOT / NRM2 n = 2^24 phi = 2, GEMV 8192^2 phi = 1, CSRMV on the 128^3 7-point stencil, both sum
    modes) and config 4 (CG on 100^3, 2000 iterations), through the public API on host-generated inputs.  Each
    carries its HBM roofline (algorithmic bytes over the device span of the call's kernels; roofline_whole_call: over
    the call's CUDA-event time, host work included) and, with cpu, the reference CPU
    library's time on the same inputs (mean of `cpu reps` calls after a warm-up) and whether the bits agree."""
    import numpy as np

    out = {}
    ref = _reference() if cpu else None

    def cpu_leg(rec, name, fn, nbytes, reps_cpu, gpu_value):
        if ref is None:
            return
        t, r = cpu_mean(fn, reps_cpu)
        rec["cpu_baseline"] = {"value": nbytes / t / 1e9, "unit": "GB/s", "ms": t * 1e3, "cores": ref.threads(),
                               "kind": "reference", "cpu_model": _cpu_model(),
                               "sample": f"reference {name} on the same inputs, mean of {reps_cpu} after 1 warm-up"}
        a, b = np.asarray(gpu_value, dtype=np.float64), np.asarray(r, dtype=np.float64)
        rec["bit_exact_vs_reference"] = bool(np.array_equal(a.view(np.int64), b.view(np.int64)))

    # DOT / NRM2, n = 2^24, phi = 2 (seeds 1, 2)
    nv = 1 << 24
    x_h = phi_matrix(nv, 1, 2.0, 1).ravel()
    y_h = phi_matrix(nv, 1, 2.0, 2).ravel()
    x, y = torch.from_numpy(x_h).cuda(), torch.from_numpy(y_h).cuda()
    for sm in (0, 1):
        h.sumMode = sm
        if ref is not None:
            ref.set_flags(sumMode=sm)
        res = []
        ms = timed_ms(torch, lambda: res.append(ozb.ddot(h, nv, x, y)), reps=reps)
        nb = 16.0 * nv
        rec = mem_record(h, lambda: ozb.ddot(h, nv, x, y), nb, ms, ncu_traffic(f"ddot_2p24_sum{sm}"), reps)
        cpu_leg(rec, "ozblasRdot", lambda: ref.ddot(x_h, y_h), nb, 10, res[-1])
        out[f"ddot_2p24_sum{sm}"] = rec
        res = []
        ms = timed_ms(torch, lambda: res.append(ozb.dnrm2(h, nv, x)), reps=reps)
        nb = 8.0 * nv
        rec = mem_record(h, lambda: ozb.dnrm2(h, nv, x), nb, ms, ncu_traffic(f"dnrm2_2p24_sum{sm}"), reps)
        cpu_leg(rec, "ozblasRnrm2", lambda: ref.dnrm2(x_h), nb, 10, res[-1])
        out[f"dnrm2_2p24_sum{sm}"] = rec
    del x, y, x_h, y_h
    # GEMV 8192^2, phi = 1, y = A x, beta = 0 (seeds 1, 2): algorithmic bytes 8 (mn + n + m)
    mg = 8192
    A_h = phi_matrix(mg, mg, 1.0, 1)
    xg_h = phi_matrix(mg, 1, 1.0, 2).ravel()
    Ag, xg = torch.from_numpy(A_h).cuda(), torch.from_numpy(xg_h).cuda()
    yg = torch.zeros(mg, dtype=torch.float64, device="cuda")
    for sm in (0, 1):
        h.sumMode = sm
        if ref is not None:
            ref.set_flags(sumMode=sm)
        gv = lambda: ozb.dgemv(h, "n", mg, mg, 1.0, Ag, mg, xg, 0.0, yg)
        ms = timed_ms(torch, gv, reps=reps)
        nb = 8.0 * (mg * mg + 2 * mg)
        rec = mem_record(h, gv, nb, ms, ncu_traffic(f"dgemv_8192_sum{sm}"), reps)
        cpu_leg(rec, "ozblasRgemv", lambda: ref.dgemv("n", mg, mg, 1.0, A_h, mg, xg_h, 0.0, np.zeros(mg)), nb, 3,
                yg.cpu().numpy())
        out[f"dgemv_8192_sum{sm}"] = rec
    del Ag, xg, yg, A_h
    torch.cuda.empty_cache()
    # CSRMV: 7-point stencil on 128^3, values phi = 1 (seed 3), x phi = 1 (seed 4), beta = 0
    rp_h, ci_h, _ = stencil7(128)
    m = len(rp_h) - 1
    nnz = len(ci_h)
    val_h = phi_matrix(nnz, 1, 1.0, 3).ravel()
    xv_h = phi_matrix(m, 1, 1.0, 4).ravel()
    val, colind, rowptr = (torch.from_numpy(a).cuda() for a in (val_h, ci_h, rp_h))
    xv = torch.from_numpy(xv_h).cuda()
    yv = torch.zeros(m, dtype=torch.float64, device="cuda")
    nbytes = 12.0 * nnz + 4.0 * (m + 1) + 8.0 * m + 8.0 * m
    for sm in (0, 1):
        h.sumMode = sm
        if ref is not None:
            ref.set_flags(sumMode=sm)
        cv = lambda: ozb.dcsrmv(h, "n", m, m, nnz, 1.0, val, colind, rowptr, xv, 0.0, yv)
        ms = timed_ms(torch, cv, reps=reps)
        rec = mem_record(h, cv, nbytes, ms, ncu_traffic(f"dcsrmv_stencil128_sum{sm}"), reps, nnz=nnz)
        cpu_leg(rec, "ozblasRcsrmv", lambda: ref.dcsrmv(m, m, 1.0, val_h, ci_h, rp_h, xv_h, 0.0, np.zeros(m)),
                nbytes, 3, yv.cpu().numpy())
        out[f"dcsrmv_stencil128_sum{sm}"] = rec
    del val, colind, rowptr, xv, yv, val_h, xv_h
    torch.cuda.empty_cache()
    # CG: 7-point Poisson on 100^3 plus 0.01 U(0,1) on the diagonal (seed 5), b = A x_true (x_true ~ N(0,1),
    # seed 6, row sums on the host), x0 = 0, NearSum, tol = 0, history every iteration (verbose = 1)
    g3 = 100
    rp_h, ci_h, M7 = stencil7(g3)
    m = len(rp_h) - 1
    V7 = np.full((m, 7), -1.0)
    V7[:, 3] = 6.0 + 0.01 * np.random.default_rng(5).random(m)
    val_h = V7[M7]
    xt = np.random.default_rng(6).standard_normal(m)
    b_h = np.zeros(m)
    rows_of = np.repeat(np.arange(m), np.diff(rp_h))
    np.add.at(b_h, rows_of, val_h * xt[ci_h])
    nnz = len(ci_h)
    val, colind, rowptr, b = (torch.from_numpy(a).cuda() for a in (val_h, ci_h, rp_h, b_h))
    xs = torch.zeros(m, dtype=torch.float64, device="cuda")
    iters = cg_iters
    h1 = np.zeros(iters + 1)
    h2 = np.zeros(iters + 1)
    h.sumMode, h.verbose = 1, 1
    ms = timed_ms(torch, lambda: (xs.zero_(), ozb.dcg(h, "n", m, nnz, val, colind, rowptr, b, xs, iters, 0.0, h1, h2)),
                  reps=min(reps, 2))
    l0 = h.launch_count()
    xs.zero_()
    ozb.dcg(h, "n", m, nnz, val, colind, rowptr, b, xs, iters, 0.0, h1, h2)
    per_iter_bytes = 12.0 * nnz + 4.0 * (m + 1) + 116.0 * m
    rec = {"ms": ms, "ms_per_iter": ms / iters, "GBps": per_iter_bytes * iters / ms / 1e6,
           "iterations": h.cg_numiter, "nnz": nnz, "final_rel_res": float(h1[iters]),
           "launches_per_iter": (h.launch_count() - l0) / iters, "bytes_per_iter": per_iter_bytes,
           "roofline": hbm_roofline(per_iter_bytes * iters, ms, None, "whole solve (2000 iterations)")}
    if ref is not None:
        # bounded sample: the reference CG at 10 and 20 iterations (same flags); per iteration = the difference
        ref.set_flags(sumMode=1, verbose=1)
        t0 = time.perf_counter()
        _, hist10 = ref.dcg(val_h, ci_h, rp_h, b_h, np.zeros(m), 10, 0.0)
        t10 = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.dcg(val_h, ci_h, rp_h, b_h, np.zeros(m), 20, 0.0)
        t20 = time.perf_counter() - t0
        per = max(t20 - t10, 1e-9) / 10
        rec["cpu_baseline"] = {"value": per_iter_bytes / per / 1e9, "unit": "GB/s", "ms_per_iter": per * 1e3,
                               "cores": ref.threads(), "kind": "reference", "cpu_model": _cpu_model(),
                               "sample": f"reference ozblasRcg (NearSum, verbose 1) at 10 and 20 iterations "
                                         f"({t10:.2f} s, {t20:.2f} s, SplitA included in both); per iteration = "
                                         "the difference / 10"}
        g = h1[: len(hist10)]
        rec["history_first_10_bit_exact_vs_reference"] = bool(
            np.array_equal(np.asarray(g).view(np.int64), np.asarray(hist10, dtype=np.float64).view(np.int64)))
    out[f"dcg_100cube_{iters}it"] = rec
    h.sumMode, h.verbose = 0, 0
    if ref is not None:
        ref.close()
    return out


if __name__ == "__main__":
    sys.exit(main())
