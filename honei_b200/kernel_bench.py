"""Per-kernel timing of the hot kernels on one Q1 level.

    python -m honei_b200.kernel_bench [--kernel all|jacobi|spmv|defect|q1|restrict|prolong|csr_spmv|csr_defect|
                                                cgvar|bicgstab|coarse_cg|solves]
                                      [--level 10] [--iters 20] [--dtype f64|f32]
                                      [--operator q1|coefficients] [--storage native|bf16|bf16c]

Each launch is preceded by an L2 flush (256 MiB written, then 256 MiB read, so
that no dirty line of the flush is written back during the launch; --flush write
keeps only the write) and timed alone with CUDA
events on the launching stream; the line reports the mean launch time and the
algorithmic bandwidth (bytes per row as in the design notes) against the
measured HBM peak.  The first launch of each kernel is a warm-up.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics

import torch

from . import _lib
from .inputs import uniform
from .la import BandedMatrixQx, DenseVector, SparseMatrixELL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def peak_gbs() -> float:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


class L2Flush:
    """Evicts L2 (126 MB on B200) before a timed launch: writes a 256 MiB buffer,
    then (clean=True) reads another 256 MiB, so that the launch finds neither its
    inputs in L2 nor dirty lines of the flush whose write-back it would pay for
    during its own reads."""

    def __init__(self, device, clean: bool = True):
        self.w = torch.empty(64 << 20, dtype=torch.float32, device=device)
        self.r = torch.ones(64 << 20, dtype=torch.float32, device=device) if clean else None
        self.out = torch.empty((), dtype=torch.float32, device=device)

    def __call__(self):
        self.w.zero_()
        if self.r is not None:
            torch.sum(self.r, dim=0, out=self.out)


def graph_time(name, A, P, n, dt, npdt, dev, reps, launches=40):
    """Mean time of one launch of `name` (jacobi / spmv / defect / copy) inside a CUDA
    graph of `launches` back-to-back launches that rotate over sets of input and
    output vectors (more than 2x L2 in all, so each launch reads its vectors from
    DRAM while the TLBs stay warm); CUDA events around each replay."""
    import numpy as np
    s = 8 if dt == torch.float64 else 4
    set_bytes = 4 * n * s
    nsets = max(3, -(-(2 * 126 * 2 ** 20 + set_bytes) // set_bytes))
    sets = []
    for j in range(nsets):
        x = torch.from_numpy(uniform(n, 100 + j, dtype=npdt)).to(dev)
        sets.append((x, torch.empty_like(x), torch.from_numpy(uniform(n, 200 + j, dtype=npdt)).to(dev),
                     P.elements.clone()))
    nrm = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()

    def call(j):
        x, y, b, pj = sets[j % nsets]
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        if name == "jacobi":
            _lib.call("hb2_jacobi_sweep_ell", A.handle, ctypes.c_void_p(pj.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                      ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), st)
        elif name == "spmv":
            _lib.call("hb2_product_ell", A.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), st)
        elif name == "defect":
            _lib.call("hb2_defect_ell", A.handle, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                      ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(nrm.data_ptr()), st)
        elif name == "prolong":
            # A = the prolongation: b (fine) += A x[:coarse]
            _lib.call("hb2_product_add_ell", A.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(b.data_ptr()), st)
        elif name == "restrict":
            # A = the restriction: y[:coarse] = A x (fine)
            _lib.call("hb2_product_ell", A.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), st)
        else:
            y.copy_(x)

    with torch.cuda.stream(stream):
        for j in range(nsets):      # warm-up (and the stream's reduction workspace) outside the capture
            call(j)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        for j in range(launches):
            call(j)
    g.replay()
    torch.cuda.synchronize()
    ts = []
    for _ in range(max(3, reps // 4)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            g.replay()
            e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / launches)
    del g
    return statistics.median(ts)


def solves(level: int, runs: int) -> int:
    """--kernel solves: the two solves the benchmark times at `level` -- FP64 MG
    (V(4,4), coarse level 3, coarse CG cap 100 with tree-ordered dots) to 1e-10, then
    IR to 1e-10 around an FP32 inner MG to 1e-3 whose FP64 coarse CG stops at 1e-3 --
    of b = A u, u ~ U[-1,1] (seed 42), each `runs` times from x = 0 (no L2 flush).
    Prints the last run's times (CUDA events) and its launch counts: under a profiler,
    the launch list of one solve of each kind (HB2_MG_LOOP=host HB2_IR_LOOP=host turn
    the device-side loops into plain launches)."""
    import honei_b200 as hb
    dev = torch.device("cuda")
    n = ((1 << level) + 1) ** 2
    A = SparseMatrixELL.poisson_q1(level)
    b = DenseVector(n)
    hb.Product.value(b, A, DenseVector(torch.from_numpy(uniform(n, 42)).to(dev)))
    fp64 = hb.MGData.poisson_q1(3, level, params=hb.mg_params(max_iters_coarse=100, eps=1e-10, coarse_exact=False))
    inner = hb.MGData.poisson_q1(3, level, dtype=torch.float32,
                                 params=hb.mg_params(max_iters_coarse=100, eps=1e-3, coarse_eps=1e-3,
                                                     coarse_exact=False, coarse_fp64=True))
    x = DenseVector(n)
    out = {"kernel": "solves", "level": level, "runs": runs}
    ir = {}

    def run_ir():
        _, ir["outer"], st = hb.IRSolver.value(A, b, x, inner, eps=1e-10, reset_inner=True)
        ir["inner"] = int(st[3])

    for name, fn in (("fp64_mg", lambda: hb.MGSolver.value(fp64, b, x)), ("mixed_ir", run_ir)):
        for _ in range(runs):
            hb.fill(x, 0.0)
            torch.cuda.synchronize()
            c0 = hb.launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            out[name + "_ms"] = e0.elapsed_time(e1)
            out[name + "_launches"] = hb.launch_count() - c0
    out.update(fp64_cycles=fp64.used_iters, ir_outer=ir["outer"], ir_inner_cycles=ir["inner"])
    print(json.dumps(out))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="all")
    ap.add_argument("--level", type=int, default=10)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--operator", default="q1", choices=["q1", "coefficients"],
                    help="q1: the Q1 Poisson operator; coefficients: the Q1 finite-element operator with per-cell "
                         "coefficients of contrast 4 (seed 7), no two rows alike")
    ap.add_argument("--storage", default="native", choices=["native", "bf16", "bf16c"],
                    help="bf16 / bf16c: the matrix stored in BF16 (pure / row-sum compensated), FP32 vectors")
    ap.add_argument("--flush", default="clean", choices=["clean", "write", "none", "graph"],
                    help="clean: write then read 256 MiB before each launch; write: the write only; none: "
                         "bursts of 8 back-to-back launches, no flush (warm L2), time per launch; graph: "
                         "40 launches in one CUDA graph rotating over vector sets of more than 2x L2 in all "
                         "(every launch reads its vectors from DRAM), time per launch")
    a = ap.parse_args(argv)
    if a.kernel == "solves":
        return solves(a.level, max(1, a.iters))
    dt = torch.float64 if a.dtype == "f64" else torch.float32
    s = 8 if a.dtype == "f64" else 4
    import numpy as np
    npdt = np.float64 if a.dtype == "f64" else np.float32
    dev = torch.device("cuda")
    L = a.level
    n = ((1 << L) + 1) ** 2
    nc = ((1 << (L - 1)) + 1) ** 2
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    flush = L2Flush(dev, clean=a.flush == "clean") if a.flush in ("clean", "write") else None

    def vec(m, seed):
        return DenseVector(torch.from_numpy(uniform(m, seed, dtype=npdt)).to(dev))

    if a.storage != "native" and a.dtype != "f32":
        ap.error("--storage bf16 / bf16c needs --dtype f32")
    if a.operator == "q1":
        A = SparseMatrixELL.poisson_q1(L, dt)
    else:
        from .inputs import element_coefficients, q1_coefficient_operator
        A = SparseMatrixELL.from_arrays(*q1_coefficient_operator(element_coefficients(L, 7), npdt))
    if a.storage != "native":
        A = A.to_bf16(compensate=a.storage == "bf16c")
    rb = A.layout()[2]              # matrix bytes per row of the layout in use
    x, b, y, y2 = vec(n, 1), vec(n, 2), vec(n, 3), vec(n, 4)
    _lib.call("hb2_product_ell", A.handle, x.ptr, b.ptr, stream)        # b = A x (setup)
    P = DenseVector(n, dtype=dt)
    _lib.call("hb2_jacobi_precon", A.handle, 0.7, P.ptr, stream)
    nrm = torch.zeros(1, dtype=torch.float64, device=dev)
    xc = torch.empty(n, dtype=dt, device=dev)
    kernels = {
        # the floor for streaming this many bytes: torch's device copy of one vector
        # (read n, write n elements), timed the same way
        "copy": (lambda: xc.copy_(x.elements), 2 * n * s),
        "jacobi": (lambda: _lib.call("hb2_jacobi_sweep_ell", A.handle, P.ptr, b.ptr, x.ptr, y.ptr, stream),
                   n * (rb + 4 * s)),
        "spmv": (lambda: _lib.call("hb2_product_ell", A.handle, x.ptr, y.ptr, stream), n * (rb + 2 * s)),
        "defect": (lambda: _lib.call("hb2_defect_ell", A.handle, b.ptr, x.ptr, y.ptr,
                                     ctypes.c_void_p(nrm.data_ptr()), stream), n * (rb + 3 * s)),
    }
    if a.kernel in ("all", "q1"):
        Q = BandedMatrixQx.poisson_q1(L, dt)
        kernels["q1"] = (lambda: _lib.call("hb2_product_q1", Q.handle, x.ptr, y.ptr, stream), n * (9 * s + 2 * s))
    if a.kernel in ("all", "restrict", "prolong"):
        Pm, Rm = SparseMatrixELL.transfer(L, dt)
        c = vec(nc, 5)
        # the Q1 transfer kernels read no matrix (HB2_Q1_TRANSFER=0: the stored layout)
        if os.environ.get("HB2_Q1_TRANSFER", "1") != "0":
            rbr, rbp = 0, 0
        else:
            rbr, rbp = Rm.layout()[2], Pm.layout()[2]
        kernels["restrict"] = (lambda: _lib.call("hb2_product_ell", Rm.handle, x.ptr, c.ptr, stream),
                               nc * (rbr + s) + n * s)
        kernels["prolong"] = (lambda: _lib.call("hb2_product_add_ell", Pm.handle, c.ptr, y2.ptr, stream),
                              n * (rbp + 2 * s) + nc * s)
    if a.kernel in ("all", "csr_spmv", "csr_defect"):
        from .la import SparseMatrixCSR
        C = SparseMatrixCSR.from_ell(A)
        # algorithmic: the CSR arrays (uint32 row offsets, per block a 4-byte
        # column and its values), x and y (and rhs); the device layout reads
        # slots (incl. padding) and a 4-byte row index per row instead
        cb = (n + 1) * 4 + C.used_blocks() * (4 + s * C.blocksize())
        slots, long_rows, long_entries, unroll = C.layout()
        print(json.dumps({"csr_layout": {"slots": slots, "padding": slots - C.used_blocks() * C.blocksize() + long_entries,
                                         "long_rows": long_rows, "unroll": unroll,
                                         "device_bytes_per_launch": slots * (4 + s) + 4 * n + long_entries * (4 + s) + 2 * n * s}}),
              flush=True)
        kernels["csr_spmv"] = (lambda: _lib.call("hb2_product_csr", C.handle, x.ptr, y.ptr, stream), cb + 2 * n * s)
        kernels["csr_defect"] = (lambda: _lib.call("hb2_defect_csr", C.handle, b.ptr, x.ptr, y.ptr, stream),
                                 cb + 3 * n * s)
    if a.kernel == "coarse_cg":
        # the MG's coarsest-level solve: CG on the level-3 operator (81 unknowns) for
        # 100 iterations (the cap of the bench; eps 0 never stops early), which runs
        # as one warp with the operator and vectors in registers
        from .solvers import CGSolver
        A3 = SparseMatrixELL.poisson_q1(3, dt)
        n3 = A3.rows()
        b3 = vec(n3, 9)
        x3 = DenseVector(n3, dtype=dt)
        ts = []
        used = 0
        for i in range(a.iters + 1):
            x3.elements.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, used, _ = CGSolver.value(A3, None, b3, x3, 100, 0.0)
            e1.record()
            e1.synchronize()
            if i > 0:
                ts.append(1000 * e0.elapsed_time(e1))
        us = statistics.median(ts)
        print(json.dumps({"kernel": "coarse_cg", "level": 3, "rows": n3, "iterations": used, "solve_us": us,
                          "us_per_iteration": us / max(used, 1)}), flush=True)
        return 0
    if a.kernel in ("cgvar", "bicgstab") and a.dtype == "f64":
        from .solvers import HB2_BICGSTAB_VAR, HB2_CG_VAR, KrylovSolver
        # Jacobi vector preconditioner; a fixed number of iterations (eps = 0)
        dvec = torch.empty(n, dtype=dt, device=dev)
        _lib.call("hb2_jacobi_precon", A.handle, 1.0, ctypes.c_void_p(dvec.data_ptr()), stream)
        iters = 200
        K = KrylovSolver(HB2_CG_VAR if a.kernel == "cgvar" else HB2_BICGSTAB_VAR, A, DenseVector(dvec), iters, 0.0)
        x0 = DenseVector(n, dtype=dt)
        K.solve(b, DenseVector(n, dtype=dt))        # warm-up
        ts = []
        for _ in range(3):
            x0.elements.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, used, _ = K.solve(b, x0)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = statistics.median(ts)
        its = used - 1 if a.kernel == "bicgstab" else used
        # algorithmic bytes per iteration: the SpMV(s) (matrix bytes + x + y) and the
        # vector passes (CG VAR: update with z = d (.) r and its dot 56, direction 32
        # bytes per row; BiCGStab: 2 Jacobi products 2*24, s 40, t dots 16, update 56,
        # r~ 32, direction 32 bytes per row)
        per_row = (rb + 16 + 88) if a.kernel == "cgvar" else (2 * (rb + 16) + 48 + 40 + 16 + 56 + 32 + 32)
        nbytes = n * per_row
        us_it = 1000 * ms / its
        print(json.dumps({"kernel": a.kernel, "level": L, "rows": n, "iterations": its, "solve_ms": ms,
                          "us_per_iteration": us_it, "algorithmic_bytes_per_iteration": nbytes,
                          "gbs": nbytes / (us_it * 1e-6) / 1e9, "frac_of_measured_peak": nbytes / (us_it * 1e-6) / 1e9 / peak_gbs()}),
              flush=True)
        return 0
    names = list(kernels) if a.kernel == "all" else [a.kernel]
    peak = peak_gbs()
    if a.flush == "graph":
        for name in names:
            if name not in ("jacobi", "spmv", "defect", "copy", "prolong", "restrict"):
                continue
            M = A if name not in ("prolong", "restrict") else (Pm if name == "prolong" else Rm)
            ms = graph_time(name, M, P, n, dt, npdt, dev, a.iters)
            nbytes = kernels[name][1]
            gbs = nbytes / (ms * 1e-3) / 1e9
            print(json.dumps({"kernel": name, "level": L, "dtype": a.dtype, "operator": a.operator,
                              "storage": a.storage, "rows": n, "layout": M.layout()[0],
                              "variant": list(M.layout_variant(0 if name != "defect" else 1)) if name != "copy" else None,
                              "launch_shape": list(M.launch_shape(0 if name != "defect" else 1)),
                              "flush": "graph", "matrix_bytes_per_row": rb, "launch_us": 1000 * ms,
                              "algorithmic_bytes": nbytes, "gbs": gbs, "frac_of_measured_peak": gbs / peak}), flush=True)
        return 0
    for name in names:
        fn, nbytes = kernels[name]
        times = []
        for i in range(a.iters + 1):
            if a.flush != "none":
                flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(1 if a.flush != "none" else 8):
                fn()
            e1.record()
            e1.synchronize()
            if i > 0:
                times.append(e0.elapsed_time(e1) / (1 if a.flush != "none" else 8))
        ms = statistics.mean(times)
        gbs = nbytes / (ms * 1e-3) / 1e9
        print(json.dumps({"kernel": name, "level": L, "dtype": a.dtype, "rows": n, "layout": A.layout()[0],
                          "variant": list(A.layout_variant(0 if name != "defect" else 1)) if name != "copy" else None,
                          "flush": a.flush,
                          "matrix_bytes_per_row": rb,
                          "launch_us": 1000 * ms,
                          "algorithmic_bytes": nbytes, "gbs": gbs, "frac_of_measured_peak": gbs / peak}),
              flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
