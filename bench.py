#!/usr/bin/env python
"""Headline benchmark: Poisson solves/s to 1e-10 relative residual.

Workload (one "step"): one full MG solve of the level-11 Q1 Poisson system
(2049 x 2049 nodes, 4,198,401 unknowns, ELL FP64; the largest single-GPU
configuration, whose mixed-precision comparison is reported beside it), V(4,4)
with damped Jacobi (omega 0.7), bilinear prolongation / transposed restriction,
coarsest level 3 solved by CG (iteration cap 100, the reference's own MG test
setting), stop at ||r|| < 1e-10 ||r0||; b = A u*, u* ~ U[-1,1] (splitmix64,
seed 42 + rank), x0 = 0.  Inputs are resident in HBM when a timed step starts;
L2 is flushed before every step (256 MiB written, then 256 MiB read, so that no
dirty line of the flush is written back inside the step) and the flush is
outside the step's events.  --level 10 runs the level-10 solve (1,050,625 unknowns).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (torchrun): every rank solves its own independent system (weak scaling,
no data-path collective); the step time is the max over ranks.
--impl reference: the reference's own CPU MG solver (compiled from its sources
into oracle/_ref/) on this host's cores, same workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Poisson solves/s & HBM GB/s to 1e-10 rel. residual, mixed vs FP64; p99 latency"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "honei_ref")
MIN_LEVEL = 3
COARSE_CAP = 100
MIXED_LEVEL = 11
DEFAULT_LEVEL = 11
SERVING_RATES = (50.0, 100.0, 200.0, 500.0, 1000.0, 2000.0)
SUB_MAX_ROWS = 20000    # levels up to this many rows run in the fused small-level kernels


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--level", type=int, default=DEFAULT_LEVEL)
    ap.add_argument("--serving-duration", type=float, default=10.0, help="seconds per serving rate")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-next", action="store_true", help="skip the CSR / Krylov / legacy-multigrid timings")
    return ap.parse_args()


def mg_solve_bytes(level: int, cycles: int, row_bytes, min_level: int = MIN_LEVEL, n_pre: int = 4, n_post: int = 4,
                   s: int = 8) -> int:
    """Algorithmic HBM bytes of one MG solve (each vector / matrix entry touched once per pass).

    row_bytes(l, which) = matrix bytes per row of the layout the level-l operator
    ("A"), its restriction ("R", rows = level l-1) or prolongation ("P") runs on
    (plain FP64: 9 x 12 = 108; compressed: 3 per slot; row patterns: 1; transfers
    applied by the Q1 transfer kernels: 0).
    Jacobi sweep rb + 4s per row; defect rb + 3s; restriction rb(R) + 2s per
    coarse row + the fine input; prolongation-add rb(P) + 2s per fine row + the
    coarse input; convergence defect once per cycle plus the initial one; the
    coarse solve is counted once (it runs in registers)."""
    total = 0
    for l in range(min_level + 1, level + 1):
        nf = ((1 << l) + 1) ** 2
        nc = ((1 << (l - 1)) + 1) ** 2
        total += (n_pre + n_post) * nf * (row_bytes(l, "A") + 4 * s)
        total += nf * (row_bytes(l, "A") + 3 * s)
        total += nc * (row_bytes(l, "R") + 2 * s) + nf * s
        total += nf * (row_bytes(l, "P") + 2 * s) + nc * s
    n0 = ((1 << min_level) + 1) ** 2
    total += n0 * (row_bytes(min_level, "A") + 2 * s)
    nF = ((1 << level) + 1) ** 2
    total += nF * (row_bytes(level, "A") + 3 * s)      # convergence defect + norm
    return cycles * total + nF * (row_bytes(level, "A") + 3 * s)


def layout_row_bytes(hb, dtype, levels):
    """row_bytes(l, which) for mg_solve_bytes, from matrices of the same shapes as the
    hierarchy's (the layout choice is made once per shape and process)."""
    import torch
    # levels above SUB_MAX_ROWS rows apply their transfers with the Q1 transfer kernels,
    # which read no matrix (unless HB2_Q1_TRANSFER=0); the fused small levels read them
    q1t = os.environ.get("HB2_Q1_TRANSFER", "1") != "0"
    table = {}
    for l in levels:
        table[(l, "A")] = hb.SparseMatrixELL.poisson_q1(l, dtype).layout()[2]
        if l > min(levels):
            P, R = hb.SparseMatrixELL.transfer(l, dtype)
            table[(l, "P")], table[(l, "R")] = P.layout()[2], R.layout()[2]
            if q1t and ((1 << l) + 1) ** 2 > SUB_MAX_ROWS:
                table[(l, "P")] = table[(l, "R")] = 0
    return lambda l, which: table[(l, which)]


JACOBI_BYTES_PER_ROW = 9 * (8 + 4) + 4 * 8     # FP64 values, int32 columns: 140 B
KERNEL_OF_LAYOUT = {0: "ell_kernel", 1: "ell_compact_kernel", 2: "ell_pattern_kernel"}


def layout_text(kind, table_size, bytes_per_row):
    if kind == 2:
        return "row patterns: 1-byte pattern id per row (%d patterns), %d B/row" % (table_size, bytes_per_row)
    if kind == 1:
        return "1-byte value codes (table of %d) + int16 column offsets, %d B/row" % (table_size, bytes_per_row)
    return "FP64 values + int32 columns, %d B/row" % bytes_per_row


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reference_cpu(level: int, reps: int, warmup: int, tag: str, threads: int, env=None):
    """Run the reference's own MG solver (oracle/_ref/honei_ref) and parse its RESULT line."""
    env = dict(os.environ, **(env or {}))
    with tempfile.NamedTemporaryFile("w", suffix=".honeirc", delete=False) as f:
        f.write(f"mc::num_threads = {threads}\nlog::categories = none\nlog::output = /dev/null\n")
        env["HONEI_CONFIG"] = f.name
    env["HONEI_COARSE_CAP"] = str(COARSE_CAP)
    out = subprocess.run([REF_BIN, "bench", "mg", tag, str(level), str(reps), str(warmup)], capture_output=True,
                         text=True, env=env, timeout=1800)
    os.unlink(env["HONEI_CONFIG"])
    for line in out.stdout.splitlines():
        if line.startswith("RESULT "):
            return json.loads(line[len("RESULT "):])
    raise RuntimeError("reference run failed: " + out.stderr[-500:])


def oracle_port_cpu(level: int, reps: int):
    """Fallback CPU baseline: the oracle's C restatement (single thread)."""
    from honei_b200.inputs import uniform
    from oracle import oracle as o
    A = o.q1_ell(level)
    b = o.ell_spmv(A, uniform(A.rows, 42))
    import numpy as np
    t = []
    for _ in range(reps):
        t0 = time.perf_counter()
        x, it, _ = o.mg_q1(level, b, max_iters_coarse=COARSE_CAP)
        t.append(time.perf_counter() - t0)
    relres = float(np.linalg.norm(b - o.ell_spmv(A, x)) / np.linalg.norm(b))
    return {"seconds_per_solve": sum(t) / len(t), "iters": it, "tag": "oracle-port", "x": x, "relres": relres}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    res = None
    kind = "reference"
    try:
        res = reference_cpu(args.level, args.steps, min(args.warmup, 1), "mc", threads)
    except Exception:
        res = oracle_port_cpu(args.level, max(1, args.steps))
        kind, threads = "port", 1
    v = 1.0 / res["seconds_per_solve"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * res["seconds_per_solve"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: b = A u*, u* ~ U[-1,1] (splitmix64 seed 42)",
            "config": workload_config(args, world),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": kind,
                             "sample": f"{args.steps} MG solves at level {args.level} "
                                       f"(tags::CPU::MultiCore::SSE, {threads} threads)",
                             "iters": res.get("iters")},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, world):
    return {"workload": f"mg-v44-fp64-q1-level{args.level}", "level": args.level,
            "unknowns": ((1 << args.level) + 1) ** 2, "matrix": "SparseMatrixELL (9 slots, int32 columns on device)",
            "coarse_level": MIN_LEVEL, "coarse_solver": f"CG, cap {COARSE_CAP}, tree-ordered dots", "smoother": "Jacobi omega 0.7, 4+4",
            "tol": 1e-10, "l2": "flushed before every step (256 MiB written, then 256 MiB read), flush outside the step "
                                "events; the level's vectors alone exceed L2 at level 11",
            "parallelism": f"{world} independent systems (one per GPU)" if world > 1 else "single system"}


ROW_BYTES = {"jacobi": 4, "spmv": 2, "defect": 3}   # vector accesses per row (8 B each in FP64)


def kernel_roofline(hb, kind, A, level, peak, dev, reps=12, label=None, dtype=None, key_suffix=""):
    """One ELL kernel of the level-`level` operator on the layout A runs on, timed in
    its steady state: 40 launches captured in one CUDA graph, rotating over sets of
    input and output vectors of more than 2x L2 in all (every launch reads its vectors
    from DRAM), CUDA events around each replay on the launching stream, the mean
    launch time the median over replays.  achieved = algorithmic bytes per launch
    (matrix bytes per row of the layout + the vector accesses) / that time."""
    import numpy as np
    import torch
    from honei_b200.kernel_bench import graph_time
    dtype = dtype or torch.float64
    es = 8 if dtype == torch.float64 else 4
    n = A.rows()
    P = hb.RISmoother.jacobi_precon(A, 0.7)
    ms = graph_time(kind, A, P, n, dtype, np.float64 if es == 8 else np.float32, dev, reps)
    kind_l, table_size, rb = A.layout()
    vk, vr, vw = A.layout_variant(1 if kind == "defect" else 0)
    variant = variant_name(vk, vr, vw)
    nbytes = n * (rb + es * ROW_BYTES[kind])
    achieved = nbytes / (ms * 1e-3) / 1e9
    key = f"{variant}:{kind}:L{level}{key_suffix}"
    return {"bound": "hbm", "kernel": label or f"{kind} on {variant}", "variant": variant, "level": level,
            "layout": layout_text(kind_l, table_size, rb), "achieved": achieved, "peak": peak[0], "unit": "GB/s",
            "frac": achieved / peak[0], "peak_source": peak[1], "traffic": load_traffic(key), "traffic_key": key,
            "algorithmic_bytes": nbytes, "bytes_per_row": rb + es * ROW_BYTES[kind], "launch_us": 1000 * ms,
            "launch_shape": list(A.launch_shape(1 if kind == "defect" else 0)),
            "timing": "CUDA graph of 40 launches over rotating vector sets (> 2x L2), events around each replay"}


def time_solves(hb, data, b, x, flush, steps, warmup, stream):
    """CUDA-event times of `steps` MG solves (x = 0 each time), L2 flushed before each"""
    import torch
    ts = []
    for i in range(warmup + steps):
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hb.fill(x, 0.0)
        hb.MGSolver.value(data, b, x)
        e1.record(stream)
        e1.synchronize()
        if i >= warmup:
            ts.append(e0.elapsed_time(e1))
    return ts


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        rc = run_reference_arm(args, rank, world)
        barrier(world)
        return rc

    import torch

    import honei_b200 as hb
    from honei_b200.inputs import uniform
    from honei_b200.kernel_bench import L2Flush

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    L = args.level
    n = ((1 << L) + 1) ** 2

    params = hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-10, coarse_exact=False)
    data = hb.MGData.poisson_q1(MIN_LEVEL, L, params=params)
    A = hb.SparseMatrixELL.poisson_q1(L)
    u = hb.DenseVector(torch.from_numpy(uniform(n, 42 + rank)).to(dev))
    b = hb.DenseVector(torch.zeros(n, dtype=torch.float64, device=dev))
    hb.Product.value(b, A, u)
    x = hb.DenseVector(torch.zeros(n, dtype=torch.float64, device=dev))
    flush = L2Flush(dev)

    def one_solve():
        hb.fill(x, 0.0)
        hb.MGSolver.value(data, b, x)

    for _ in range(args.warmup):
        one_solve()
    torch.cuda.synchronize()

    # ---------------------------------------------------------------- timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    launches0 = hb.launch_count()
    cycles = []
    with Clocks(local) as clk:
        t_wall0 = time.perf_counter()
        for i in range(args.steps):
            flush()
            ev[i][0].record(stream)
            one_solve()
            ev[i][1].record(stream)
            cycles.append(data.used_iters)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall0
    barrier(world)
    gpu_launches = hb.launch_count() - launches0     # this library's kernels (graph nodes included)
    step_ms = [a.elapsed_time(b_) for a, b_ in ev]
    mean_ms = statistics.mean(step_ms)
    mean_ms_max = max_over_ranks(mean_ms, world, dev)
    value = world * 1000.0 / mean_ms_max

    # correctness of the timed solve (relative residual, on the device)
    r = hb.DenseVector(torch.zeros(n, dtype=torch.float64, device=dev))
    hb.Defect.value(r, b, A, x)
    relres = hb.Norm.value(r) / hb.Norm.value(b)

    # ---------------------------------------------------------------- end to end
    hb_pinned = torch.from_numpy(uniform(n, 42 + rank)).pin_memory()
    b_host = torch.empty(n, dtype=torch.float64).pin_memory()
    bd = torch.zeros(n, dtype=torch.float64, device=dev)
    ud = hb_pinned.to(dev, non_blocking=True)
    hb.Product.value(hb.DenseVector(bd), A, hb.DenseVector(ud))
    b_host.copy_(bd.cpu())
    x_host = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b_dev = b_host.to(dev, non_blocking=True)
        x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
        hb.MGSolver.value(data, hb.DenseVector(b_dev), hb.DenseVector(x_dev))
        x_host.copy_(x_dev, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_mean = max_over_ranks(statistics.mean(e2e_ms), world, dev)

    # ---------------------------------------------------------------- dominant kernel
    peaks = load_peaks()
    roof = kernel_roofline(hb, "jacobi", A, L, peaks, dev,
                           label=f"fused Jacobi sweep x' = x + P (b - A x), level {L}, FP64")
    solve_bytes = mg_solve_bytes(L, int(statistics.median(cycles)),
                                 layout_row_bytes(hb, torch.float64, range(MIN_LEVEL, L + 1)))
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: b = A u*, u* ~ U[-1,1] (splitmix64 seed 42+rank)",
        "config": workload_config(args, world),
        "hbm_gbs": solve_bytes / (mean_ms_max * 1e-3) / 1e9,
        "latency_ms": {"p50": percentile(step_ms, 50), "p99": percentile(step_ms, 99), "max": max(step_ms)},
        "cycles": int(statistics.median(cycles)), "relres": relres,
        "wall_ms_per_step_incl_flush": 1000 * t_wall / args.steps,
        "roofline": roof,
        "e2e": {"value": world * 1000.0 / e2e_mean, "unit": "solves/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": gpu_launches,
        "clocks": clk.summary(),
    }
    # the single-GPU characterisation beside the headline (replica runs skip it)
    keep = {}
    if world == 1:
        line["roofline_extra"] = roofline_extra(hb, A, L, peaks, dev)
        if L != 10:
            line["level10_solve"] = level10_solve(hb, dev, flush, args, stream)
        if not args.no_mixed:
            line["mixed_vs_fp64"] = mixed_vs_fp64(hb, dev, flush, MIXED_LEVEL, min(args.steps, 5),
                                                  min(args.warmup, 2), rank, keep=keep)
            line["mixed_vs_fp64"]["anisotropic"] = anisotropic_probe(hb, dev, flush, MIXED_LEVEL, rank)
            line["mixed_vs_fp64"]["bf16_inner"] = bf16_variant(hb, dev, flush, MIXED_LEVEL, peaks, rank)
        if not args.no_batch:
            line["batched"] = batched_solves(hb, dev, flush, min(args.steps, 3), min(args.warmup, 1), rank)
        if not args.no_serving:
            line["serving"] = serving_loop(rank, duration=args.serving_duration)
        if not args.no_next:
            line["next_rows"] = next_rows(hb, dev, flush, rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(L, keep if L == MIXED_LEVEL else None)
        errors = line["cpu_baseline"].pop("errors", None)
        if errors and "mixed_vs_fp64" in line:
            line["mixed_vs_fp64"].update(errors)
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def roofline_extra(hb, A, L, peaks, dev):
    """The other kernels' steady-state rooflines: the SpMV and the fused defect + norm
    on the tuned layout at level L; the level-10 sweep on its tuned layout; and, on the
    plain ELL arrays (FP64 values + int32 columns read with 128-bit loads: 124 / 132
    B/row), the SpMV and defect at level L."""
    out = [kernel_roofline(hb, "spmv", A, L, peaks, dev, label=f"y = A x, level {L}, tuned layout"),
           kernel_roofline(hb, "defect", A, L, peaks, dev, label=f"r = b - A x with ||r||^2, level {L}, tuned layout")]
    if L != 10:
        A10 = hb.SparseMatrixELL.poisson_q1(10)
        out.append(kernel_roofline(hb, "jacobi", A10, 10, peaks, dev, label="fused Jacobi sweep, level 10, tuned layout"))
        del A10
    # the same sweep with the L2 prefetch option (half a wave of rows ahead; off in the
    # solvers, where it cost 1-4 %: a level's vectors partly stay in L2 between passes)
    old_pf = os.environ.get("HB2_Q1_PREFETCH")
    os.environ["HB2_Q1_PREFETCH"] = "0.5"
    try:
        e = kernel_roofline(hb, "jacobi", A, L, peaks, dev,
                            label=f"fused Jacobi sweep, level {L}, tuned layout, L2 prefetch option (HB2_Q1_PREFETCH=0.5)")
    finally:
        if old_pf is None:
            del os.environ["HB2_Q1_PREFETCH"]
        else:
            os.environ["HB2_Q1_PREFETCH"] = old_pf
    e["traffic"], e["traffic_key"] = None, None
    out.append(e)
    old = os.environ.get("HB2_ELL_COMPACT")
    os.environ["HB2_ELL_COMPACT"] = "0"        # the plain layout (read when a matrix is created)
    try:
        Ap = hb.SparseMatrixELL.poisson_q1(L)
    finally:
        if old is None:
            del os.environ["HB2_ELL_COMPACT"]
        else:
            os.environ["HB2_ELL_COMPACT"] = old
    out.append(kernel_roofline(hb, "spmv", Ap, L, peaks, dev, label=f"y = A x, level {L}, plain ELL"))
    out.append(kernel_roofline(hb, "defect", Ap, L, peaks, dev, label=f"r = b - A x with ||r||^2, level {L}, plain ELL"))
    return out


def level10_solve(hb, dev, flush, args, stream):
    """The level-10 MG solve (1,050,625 unknowns), same parameters and timing."""
    import torch
    from honei_b200.inputs import uniform
    L = 10
    n = ((1 << L) + 1) ** 2
    A = hb.SparseMatrixELL.poisson_q1(L)
    data = hb.MGData.poisson_q1(MIN_LEVEL, L, params=hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-10,
                                                                    coarse_exact=False))
    b = hb.DenseVector(n)
    hb.Product.value(b, A, hb.DenseVector(torch.from_numpy(uniform(n, 42)).to(dev)))
    x = hb.DenseVector(n)
    ts = time_solves(hb, data, b, x, flush, args.steps, args.warmup, stream)
    r = hb.DenseVector(n)
    hb.Defect.value(r, b, A, x)
    return {"level": L, "unknowns": n, "ms_per_solve": statistics.mean(ts), "solves_per_s": 1000.0 / statistics.mean(ts),
            "p99_ms": percentile(ts, 99), "cycles": data.used_iters, "relres": hb.Norm.value(r) / hb.Norm.value(b)}


def next_rows(hb, dev, flush, rank, reps=3):
    """Device timings of the paths beside the MG solve (CUDA events on the launching
    stream, L2 flushed before each timed call): SparseMatrixCSR Product on the level-11
    Q1 operator, CGSolver VAR and BiCGStabSolver VAR per iteration (level 10, Jacobi
    vector P, 200 iterations), the legacy banded Multigrid (levels 1-10, V(2,2), to 1e-8;
    FIXED in FP64 and MIXED with FP32 levels)."""
    import torch
    from honei_b200 import _lib
    from honei_b200.inputs import uniform
    stream = torch.cuda.current_stream()
    s_ptr = ctypes_stream(stream)
    peak = load_peaks()[0]

    def timed(fn):
        fn()
        ts = []
        for _ in range(reps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), r

    out = {}
    # CSR
    L = 11
    n = ((1 << L) + 1) ** 2
    E = hb.SparseMatrixELL.poisson_q1(L)
    C = hb.SparseMatrixCSR.from_ell(E)
    del E
    x = hb.DenseVector(torch.from_numpy(uniform(n, 1)).to(dev))
    y = hb.DenseVector(n)
    ms, _ = timed(lambda: _lib.call("hb2_product_csr", C.handle, x.ptr, y.ptr, s_ptr))
    nbytes = (n + 1) * 4 + C.used_blocks() * 12 + 16 * n
    out["csr_spmv"] = {"workload": "Q1 level 11, %d rows, %d entries, FP64" % (n, C.used_blocks()),
                       "launch_us": 1000 * ms, "algorithmic_bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9,
                       "frac": nbytes / (ms * 1e-3) / 1e9 / peak}
    del C, x, y
    # Krylov
    L = 10
    n = ((1 << L) + 1) ** 2
    A = hb.SparseMatrixELL.poisson_q1(L)
    d = hb.DenseVector(n)
    _lib.call("hb2_jacobi_precon", A.handle, 1.0, d.ptr, s_ptr)
    b = hb.DenseVector(n)
    hb.Product.value(b, A, hb.DenseVector(torch.from_numpy(uniform(n, 42)).to(dev)))
    for name, method in (("cg_var", hb.HB2_CG_VAR), ("bicgstab", hb.HB2_BICGSTAB_VAR)):
        K = hb.KrylovSolver(method, A, d, 200, 0.0)
        x0 = hb.DenseVector(n)
        ms, r = timed(lambda: K.solve(b, x0))
        its = r[1] - 1 if method == hb.HB2_BICGSTAB_VAR else r[1]
        out[name] = {"workload": "Q1 level 10, Jacobi vector P, %d iterations" % its, "solve_ms": ms,
                     "us_per_iteration": 1000 * ms / its}
        del K
    # legacy banded multigrid
    A64 = [hb.BandedMatrixQx.poisson_q1(l) for l in range(1, L + 1)]
    A32 = [hb.BandedMatrixQx.poisson_q1(l, torch.float32) for l in range(1, L + 1)]
    bq = hb.DenseVector(n)
    hb.Product.value(bq, A64[-1], hb.DenseVector(torch.from_numpy(uniform(n, 42)).to(dev)))
    mg = hb.Multigrid(A64, 1, hb.mg_info(n_max_iter=100, tolerance=1e-8))
    ms, r = timed(lambda: mg.value(bq, hb.DenseVector(n)))
    out["legacy_mg_fixed"] = {"workload": "banded Q1 levels 1-10, V(2,2), FP64, to 1e-8", "solve_ms": ms,
                              "cycles": r[1]}
    mg32 = hb.Multigrid(A32, 1, hb.mg_info(n_max_iter=2, tolerance=1e-8, adaptive=True))
    ms, r = timed(lambda: mg32.value_mixed(A64[-1], bq, hb.DenseVector(n)))
    out["legacy_mg_mixed"] = {"workload": "FP32 banded levels 1-10 under FP64 defect correction, to 1e-8",
                              "solve_ms": ms, "outer_steps": r[1], "inner_cycles": r[2]}
    return out


def finite_or_text(v):
    """A float for the JSON line; inf / nan (a diverged solve) as text, which strict
    JSON parsers accept."""
    import math
    return v if math.isfinite(v) else str(v)


def mixed_vs_fp64(hb, dev, flush, level, steps, warmup, rank, aniso=1.0, max_cycles=100, max_outer=100, keep=None):
    """Level-11 Q1 Poisson (4,198,401 unknowns) to 1e-10 relative residual,
    plain FP64 MG vs iterative refinement (FP64 defect / update / norm around an FP32
    MG V(4,4) inner solve to 1e-3, restarted from zero each outer step, its coarse CG
    (FP64 arithmetic) cap 100 at the same eps 1e-3, the reference's one eps_relative
    for both).  The whole IR solve is one CUDA graph.  Times are CUDA-event times per
    solve, L2 flushed before each.  aniso scales the x-coupling of every level's
    operator (the anisotropic variant); max_cycles caps the MG cycles of both solvers,
    max_outer the IR steps.  keep (dict): receives host copies of both solutions, for
    the error against the reference's FP64 solution (cpu_baseline)."""
    import statistics

    import torch

    from honei_b200.inputs import uniform
    n = ((1 << level) + 1) ** 2
    A = hb.SparseMatrixELL.poisson_q1(level, aniso=aniso)
    u = hb.DenseVector(torch.from_numpy(uniform(n, 42 + rank)).to(dev))
    b = hb.DenseVector(n)
    hb.Product.value(b, A, u)
    fp64 = hb.MGData.poisson_q1(MIN_LEVEL, level, aniso=aniso,
                                params=hb.mg_params(max_iters=max_cycles, max_iters_coarse=COARSE_CAP, eps=1e-10,
                                                    coarse_exact=False))
    # the inner MG's coarse CG stops at the inner eps, as the reference's one
    # eps_relative does for both (math/mg.hh:585-594)
    inner = hb.MGData.poisson_q1(MIN_LEVEL, level, dtype=torch.float32, aniso=aniso,
                                 params=hb.mg_params(max_iters=max_cycles, max_iters_coarse=COARSE_CAP, eps=1e-3,
                                                     coarse_eps=1e-3, coarse_exact=False, coarse_fp64=True))
    x64 = hb.DenseVector(n)
    xir = hb.DenseVector(n)

    def timed(fn):
        ts = []
        for i in range(warmup + steps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            if i >= warmup:
                ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts)

    info = {}

    # a diverging solve (the anisotropic variant) ends with a NaN / Inf defect norm,
    # which the solvers report as NotFinite after their last cycle
    def run64():
        hb.fill(x64, 0.0)
        try:
            hb.MGSolver.value(fp64, b, x64)
        except hb.NotFinite:
            info["fp64_not_finite"] = True

    def runir():
        hb.fill(xir, 0.0)
        info["outer"], info["inner"] = None, None
        try:
            _, it, st = hb.IRSolver.value(A, b, xir, inner, eps=1e-10, max_iters=max_outer, reset_inner=True)
            info["outer"], info["inner"] = it, int(st[3])
        except hb.NotFinite as e:
            info["mixed_not_finite"] = True
            info["outer"], info["inner"] = int(e.stats[0]), int(e.stats[3])

    t64 = timed(run64)
    tir = timed(runir)
    r = hb.DenseVector(n)
    nb = hb.Norm.value(b)
    hb.Defect.value(r, b, A, x64)
    rel64 = hb.Norm.value(r) / nb
    hb.Defect.value(r, b, A, xir)
    relir = hb.Norm.value(r) / nb
    d = hb.DenseVector(x64.elements - xir.elements)
    err = hb.Norm.value(d) / hb.Norm.value(x64)
    res = {"level": level, "unknowns": n, "fp64_mg_ms": t64, "fp64_cycles": fp64.used_iters,
           "fp64_relres": finite_or_text(rel64), "mixed_ir_ms": tir, "ir_outer_iters": info["outer"],
           "ir_inner_fp32_cycles": info["inner"], "mixed_relres": finite_or_text(relir),
           "mixed_rel_error_vs_fp64_gpu": finite_or_text(err), "speedup_mixed_over_fp64": t64 / tir,
           "inner": "FP32 ELL MG V(4,4) to 1e-3 (restart from zero), FP64 coarse CG cap 100 / eps 1e-3"}
    if keep is not None:
        keep["x64"], keep["xir"] = x64.elements.cpu().numpy(), xir.elements.cpu().numpy()
        keep["b"] = b.elements.cpu().numpy()
        keep["relres_mixed"], keep["relres_fp64"] = relir, rel64
    if aniso != 1.0:
        res["x_coupling"] = aniso
        res["cycle_cap"], res["outer_cap"] = max_cycles, max_outer
        res["fp64_converged"] = bool(rel64 <= 1e-10)
        res["mixed_converged"] = bool(relir <= 1e-10)
        res["fp64_not_finite"] = info.get("fp64_not_finite", False)
        res["mixed_not_finite"] = info.get("mixed_not_finite", False)
    return res


def bf16_variant(hb, dev, flush, level, peaks, rank):
    """The BF16-stored inner matrices (hb2_ell_create_bf16) against FP32-stored ones in
    the mixed-precision refinement at `level`, on two operators:
    * "q1": the level-11 Q1 Poisson operator.  s = 3 makes 8/3, -1/3 and 1 exact in BF16.
      The tuned FP32 levels run the Q1 stencil kernel (one byte per row); the BF16
      ones run the BF16 layout.
    * "coefficients": the Q1 finite-element operator with per-cell coefficients of
      contrast 4 (seeded), rediscretised on the coarse levels.  No two rows repeat,
      so every FP32 level runs on the plain layout; BF16 pure and with row-sum
      compensated diagonals.
    Per operator: IRSolver.choose_inner over the candidates (FP32 first), i.e. each
    IR solve to 1e-10 with its outer steps, inner cycles, best-of-2 time and `kept`
    (converged with inner cycles within 10 % of the FP32-stored solve's -- the rule
    for keeping a BF16 variant) and the choice; each solution's true relative
    residual and its error against the FP64 MG solution of the same system; and the
    level's Jacobi sweep on each inner matrix (graph-timed, algorithmic bytes)."""
    import numpy as np
    import torch

    from honei_b200 import inputs
    n = ((1 << level) + 1) ** 2
    out = {"level": level, "unknowns": n,
           "rule": "kept when converged with inner MG cycles <= 1.1 x the FP32-stored inner solve's"}
    inner_prm = hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-3, coarse_eps=1e-3, coarse_exact=False,
                             coarse_fp64=True)
    u = torch.from_numpy(inputs.uniform(n, 42 + rank)).to(dev)
    for op in ("q1", "coefficients"):
        k = np.ones((1 << level, 1 << level)) if op == "q1" else inputs.element_coefficients(level, 7)
        if op == "q1":
            A64 = hb.SparseMatrixELL.poisson_q1(level)
            fp64 = hb.MGData.poisson_q1(MIN_LEVEL, level, params=hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-10,
                                                                                 coarse_exact=False))
            cands = {"fp32": hb.MGData.poisson_q1(MIN_LEVEL, level, dtype=torch.float32, params=inner_prm),
                     "bf16": hb.MGData.q1_coefficient(k, MIN_LEVEL, torch.float32, params=inner_prm, bf16="pure")}
        else:
            A64 = hb.SparseMatrixELL.from_arrays(*inputs.q1_coefficient_operator(k))
            fp64 = hb.MGData.q1_coefficient(k, MIN_LEVEL, torch.float64,
                                           params=hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-10,
                                                               coarse_exact=False))
            cands = {"fp32": hb.MGData.q1_coefficient(k, MIN_LEVEL, torch.float32, params=inner_prm),
                     "bf16_compensated": hb.MGData.q1_coefficient(k, MIN_LEVEL, torch.float32, params=inner_prm,
                                                                  bf16="compensated"),
                     "bf16_pure": hb.MGData.q1_coefficient(k, MIN_LEVEL, torch.float32, params=inner_prm,
                                                           bf16="pure")}
        b = hb.DenseVector(n)
        hb.Product.value(b, A64, hb.DenseVector(u))
        x64 = hb.DenseVector(n)
        hb.MGSolver.value(fp64, b, x64)
        xr = x64.numpy().copy()
        nb = float(torch.linalg.norm(b.elements))
        choice, rep = hb.IRSolver.choose_inner(A64, b, cands)
        x = hb.DenseVector(n)
        r = hb.DenseVector(n)
        for name, inner in cands.items():
            if not rep[name]["converged"]:
                continue
            hb.fill(x, 0.0)
            hb.IRSolver.value(A64, b, x, inner, eps=1e-10, reset_inner=True)
            hb.Defect.value(r, b, A64, x)
            rep[name]["relres"] = float(torch.linalg.norm(r.elements)) / nb
            rep[name]["rel_error_vs_fp64_mg"] = float(np.linalg.norm(x.numpy() - xr) / np.linalg.norm(xr))
        # the finest level's inner matrix of each candidate: its Jacobi sweep
        finest = {"fp32": hb.SparseMatrixELL.poisson_q1(level, torch.float32) if op == "q1" else
                  hb.SparseMatrixELL.from_arrays(*inputs.q1_coefficient_operator(k, np.float32))}
        if op == "q1":
            finest["bf16"] = hb.SparseMatrixELL.from_arrays(*inputs.q1_coefficient_operator(k, np.float32)).to_bf16()
        else:
            finest["bf16_compensated"] = finest["fp32"].to_bf16(compensate=True)
            finest["bf16_pure"] = finest["fp32"].to_bf16()
        for name, M in finest.items():
            kr = kernel_roofline(hb, "jacobi", M, level, peaks, dev, dtype=torch.float32,
                                 label=f"fused Jacobi sweep, level {level}, {op} operator, {name} inner matrix",
                                 key_suffix="" if op == "q1" else
                                 ":coefficients" + ("" if name == "fp32" else "-" + name.split("_")[1]))
            rep[name]["sweep"] = {key: kr[key] for key in ("variant", "launch_shape", "bytes_per_row", "launch_us",
                                                           "achieved", "frac", "traffic", "traffic_key")}
            if hasattr(M, "scale"):
                rep[name]["scale"], rep[name]["max_rel_rounding_error"] = M.scale, M.max_rel_error
        rep["fp64_mg_cycles"] = fp64.used_iters
        rep["choice"] = choice
        out[op] = rep
        del cands, fp64, finest, A64
        torch.cuda.synchronize()
    return out


def anisotropic_probe(hb, dev, flush, level, rank):
    """The level-11 system's anisotropic variant: every level's x-coupling (DL/DU) scaled by a
    factor, the diagonal raised to keep zero interior row sums.  The reference's
    method (V(4,4) damped Jacobi on rediscretised coarse operators, coarse CG)
    diverges for the factor 100 -- in FP64, and on the CPU oracle as well -- and
    converges up to a factor of about 10.  The factor 100 runs for a bounded number of
    cycles and is reported with the defect it reached; the factor 10 is solved to
    1e-10 in FP64 and in mixed precision like the isotropic case."""
    return {"x_coupling_100": mixed_vs_fp64(hb, dev, flush, level, 1, 0, rank, aniso=100.0, max_cycles=10,
                                            max_outer=3),
            "x_coupling_10": mixed_vs_fp64(hb, dev, flush, level, 2, 1, rank, aniso=10.0, max_cycles=300,
                                           max_outer=30)}


def batch_workload(seed, nsys=512, lo=4, hi=9, multi_frac=0.25, multi_rhs=8):
    """The batched workload: levels uniform in lo..hi, exactly multi_frac of the systems with multi_rhs RHS."""
    import numpy as np
    rng = np.random.default_rng(seed)
    levels = rng.integers(lo, hi + 1, nsys)
    nrhs = np.ones(nsys, dtype=np.int64)
    nrhs[rng.permutation(nsys)[:int(round(multi_frac * nsys))]] = multi_rhs
    return [(int(l), int(k)) for l, k in zip(levels, nrhs)]


def batched_solves(hb, dev, flush, steps, warmup, rank):
    """The batched workload: 512 Q1 systems (levels U{4..9}, 25 % with 8 RHS, RHS ~ U[-1,1]) solved
    together by the batched mixed-precision MG-preconditioned CG to 1e-8, against
    looping the single-system FP64 MG solver (V(4,4), coarse CG cap 100) to 1e-8 over
    the same right-hand sides.  Device time per batch solve with CUDA events (L2
    flushed before each; the batch's vectors exceed L2); end to end adds the pinned
    host->device copies of every RHS and the device->host copies of every solution."""
    import statistics

    import numpy as np
    import torch

    from honei_b200.inputs import uniform
    systems = batch_workload(2024 + rank)
    B = hb.BatchedPoissonSolver(systems)
    info = B.info()
    host_b, host_x, dev_b = [], [], []
    for s, (level, k) in enumerate(systems):
        n = B.unknowns(level)
        hbuf = torch.from_numpy(np.stack([uniform(n, 7919 * s + j + 1) for j in range(k)])).pin_memory()
        host_b.append(hbuf)
        host_x.append(torch.empty_like(hbuf).pin_memory())
        dev_b.append(hbuf.to(dev))
    nvec = sum(k for _, k in systems)

    def load_rhs(src):
        for s in range(len(systems)):
            B.set_rhs(s, src[s])

    def timed(fn):
        ts = []
        for i in range(warmup + steps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            if i >= warmup:
                ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts)

    load_rhs(dev_b)
    l0 = hb.launch_count()
    t_dev = timed(lambda: B.solve())
    launches = (hb.launch_count() - l0) // (warmup + steps)
    iters = [B.result(s, j)[0] for s, (_, k) in enumerate(systems) for j in range(k)]
    rels = [B.result(s, j)[1] for s, (_, k) in enumerate(systems) for j in range(k)]

    def e2e():
        load_rhs(host_b)
        B.solve()
        for s in range(len(systems)):
            B.solution(s, out=host_x[s])

    t_e2e = timed(e2e)
    # true residual of a sample of solutions, FP64 on the device
    worst = 0.0
    for s in range(0, len(systems), 37):
        level, k = systems[s]
        A = hb.SparseMatrixELL.poisson_q1(level)
        x = B.solution(s)
        for j in range(k):
            r = hb.DenseVector(B.unknowns(level))
            bj = hb.DenseVector(dev_b[s][j].clone())
            hb.Defect.value(r, bj, A, hb.DenseVector(x[j].clone()))
            worst = max(worst, hb.Norm.value(r) / hb.Norm.value(bj))
    # the loop of the single-system solver over every right-hand side of the batch:
    # one FP64 MG hierarchy per level (built before the loop), each RHS solved from
    # x = 0 in turn, the whole loop between two CUDA events (L2 flushed before it)
    params = hb.mg_params(max_iters_coarse=COARSE_CAP, eps=1e-8, coarse_exact=False)
    hier = {level: hb.MGData.poisson_q1(MIN_LEVEL, level, params=params) for level in sorted({l for l, _ in systems})}
    xs = {level: hb.DenseVector(B.unknowns(level)) for level in hier}
    loop_cycles = []

    def loop():
        for s, (level, k) in enumerate(systems):
            for j in range(k):
                hb.fill(xs[level], 0.0)
                hb.MGSolver.value(hier[level], hb.DenseVector(dev_b[s][j]), xs[level])
                loop_cycles.append(hier[level].used_iters)
    for level in hier:                              # warm-up: one solve per level
        s0 = next(i for i, (l, _) in enumerate(systems) if l == level)
        hb.fill(xs[level], 0.0)
        hb.MGSolver.value(hier[level], hb.DenseVector(dev_b[s0][0]), xs[level])
    flush()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    loop()
    e1.record()
    e1.synchronize()
    t_loop = e0.elapsed_time(e1)
    del hier
    return {"systems": len(systems), "rhs": nvec, "levels": "U{4..9}", "multi_rhs_systems": sum(k > 1 for _, k in systems),
            "device_ms": t_dev, "rhs_per_s": nvec * 1000.0 / t_dev,
            "e2e_ms": t_e2e, "e2e_rhs_per_s": nvec * 1000.0 / t_e2e,
            "h2d_bytes": 8 * sum(B.unknowns(l) * k for l, k in systems),
            "pcg_steps": B.steps, "max_iters": max(iters), "mean_iters": statistics.mean(iters),
            "max_rel_defect": max(rels), "worst_true_relres_sampled": worst,
            "launches_per_step": info["launches_per_step"], "launches_per_solve": launches,
            "device_bytes": info["device_bytes"],
            "loop_fp64_mg_ms": t_loop, "loop_solves": nvec, "loop_mean_cycles": statistics.mean(loop_cycles),
            "loop": "the level-10 single-system FP64 MG solver (V(4,4), coarse CG cap 100) to 1e-8 over all "
                    f"{nvec} right-hand sides in turn, one resident hierarchy per level, timed as one loop",
            "speedup_vs_loop": t_loop / t_dev,
            "method": "CG VAR (FP64) + one FP32 MG V(4,4) preconditioner, FP64 coarse CG cap 100; tol 1e-8"}


def serving_loop(rank, rates=SERVING_RATES, duration=10.0, fp64_max_rate=200.0):
    """The serving workload: Poisson arrivals for `duration` s per rate (50 ... 2000 req/s), levels
    log-uniform in 5..11, tolerance 1e-8 / 1e-10 50/50, seeded U[-1,1] RHS; slot pool
    sized under a 120 GB budget.  Latency = host clock from arrival to the solution in
    pinned host memory.  Three servers on the same arrivals: the hybrid one (FP64 MG
    when idle, continuous batching otherwise), the batched engine alone, and FP64 MG one
    request at a time (up to fp64_max_rate: above its ~380 req/s capacity its queue
    only grows).  python -m honei_b200.serving runs the same sweep for 60 s per rate."""
    from honei_b200 import serving
    keys = ("rate_req_s", "arrived", "finished", "solves_per_s", "p50_ms", "p99_ms", "max_rel_defect_1e-8",
            "max_rel_defect_1e-10")
    pool = serving.RhsPool(seed=rank)
    srv = serving.PoissonServer(budget_bytes=120e9)
    seq = serving.FP64SequentialServer()
    hyb = serving.HybridServer(srv, seq)
    serving.run(srv, 200, 1.0, pool, seed=99)
    serving.run(hyb, 50, 1.0, pool, seed=99)
    out = {"budget_bytes": 120e9, "device_bytes": srv.device_bytes, "slots": srv.slots, "duration_s": duration,
           "hybrid": [], "batched_mixed": [], "fp64_sequential": []}
    for rate in rates:
        hyb.routed.clear()
        s, _ = serving.run(hyb, rate, duration, pool, seed=rank)
        out["hybrid"].append(dict({k: s[k] for k in keys}, routed=dict(hyb.routed)))
        s, _ = serving.run(srv, rate, duration, pool, seed=rank)
        out["batched_mixed"].append({k: s[k] for k in keys})
        if rate <= fp64_max_rate:
            s, _ = serving.run(seq, rate, duration, pool, seed=rank)
            out["fp64_sequential"].append({k: s[k] for k in keys})
    return out


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def percentile(vals, p):
    s = sorted(vals)
    k = min(len(s) - 1, max(0, int(round((p / 100.0) * (len(s) - 1)))))
    return s[k]


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def variant_name(kind, rows_per_thread, kernel):
    """Name of an ELL kernel variant as HB2_ELL_COMPACT spells it (plain, forceR,
    patternR, patternwinR, q1stencilR, q1gatherR, q1pair, q1stripR, bf16rR)."""
    if kind == 3:
        return "bf16r%d" % rows_per_thread
    if kind == 2:
        if int(kernel) == 4:
            return "q1pair"
        return ({1: "patternwin%d", 2: "q1stencil%d", 3: "q1gather%d", 5: "q1strip%d"}.get(int(kernel), "pattern%d")
                % rows_per_thread)
    if kind == 1:
        return "force%d" % rows_per_thread
    return "plain"


def load_traffic(key):
    """DRAM bytes (read + write) per launch of a kernel, from the committed ncu
    summaries: a line `traffic_bytes_per_launch[<variant>:<kernel>:L<level>]: <bytes>`
    in any file under profiles/ (None when that kernel was not captured)."""
    import glob
    tag = "traffic_bytes_per_launch[%s]:" % key
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            for line in open(path):
                if line.startswith(tag):
                    return float(line[len(tag):])
        except Exception:
            pass
    return None


def q1_lambda_min(level):
    """smallest eigenvalue of the Q1 stencil (8/3 centre, -1/3 neighbours) on the
    interior nodes of the (2^L + 1)^2 grid: 1 / ||A^-1|| for the error bound"""
    import math
    c = math.cos(math.pi / (1 << level))
    return (8.0 - 4.0 * c - 4.0 * c * c) / 3.0


def solution_errors(level, keep, x_ref, ref_relres, ref_what):
    """The GPU solutions (FP64 MG and mixed IR) against the reference's own FP64 CPU
    solution of the same system, with the bound the two residuals allow:
    ||x - x_ref|| <= ||A^-1|| (||r|| + ||r_ref||)."""
    import numpy as np
    nx = float(np.linalg.norm(x_ref))
    bound = (keep["relres_mixed"] + ref_relres) * float(np.linalg.norm(keep["b"])) / (q1_lambda_min(level) * nx)
    return {"mixed_rel_error_vs_reference_fp64": float(np.linalg.norm(keep["xir"] - x_ref)) / nx,
            "fp64_gpu_rel_error_vs_reference_fp64": float(np.linalg.norm(keep["x64"] - x_ref)) / nx,
            "mixed_error_bound_from_residuals": bound, "reference_fp64_relres": ref_relres,
            "reference_fp64_solution": ref_what}


def cpu_baseline(level, keep=None):
    """The reference's own tags::CPU::SSE MG solver on one host core (oracle/_ref), one
    solve of the headline's system; when `keep` holds the GPU solutions (level 11),
    the reference's solution is dumped and the GPU results' errors are stated
    against it."""
    import numpy as np
    reps = 1
    dump = os.path.join(tempfile.gettempdir(), "hb2_ref_x_%d.bin" % os.getpid())
    try:
        res = reference_cpu(level, reps, 0, "sse", 1, env={"HONEI_DUMP_X": dump} if keep else None)
        out = {"value": 1.0 / res["seconds_per_solve"], "unit": "solves/s", "cores": 1, "kind": "reference",
               "sample": f"{reps} MG solve at level {level} (reference tags::CPU::SSE, 1 thread)",
               "iters": res["iters"]}
        if keep and os.path.exists(dump):
            x_ref = np.fromfile(dump, dtype=np.float64)
            os.unlink(dump)
            if x_ref.size == keep["xir"].size:
                out["errors"] = solution_errors(level, keep, x_ref, float(res["relres"]),
                                                "reference tags::CPU::SSE MGSolver (oracle/_ref)")
        return out
    except Exception as e:  # binary absent: the oracle port
        res = oracle_port_cpu(level, 1)
        out = {"value": 1.0 / res["seconds_per_solve"], "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"1 MG solve at level {level} (oracle C port; reference binary unavailable: {e})"}
        if keep and "x" in res:
            out["errors"] = solution_errors(level, keep, res["x"], res["relres"], "oracle port of the MGSolver")
        return out


if __name__ == "__main__":
    sys.exit(main())
