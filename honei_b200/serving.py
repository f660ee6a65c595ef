"""Serving loop: Poisson solve requests admitted as they arrive, solved with continuous batching.

A request asks for the Q1 Poisson system of one grid level with its own right-hand
side and relative tolerance.  The server keeps one batched solver resident on the
device (``BatchedPoissonSolver``: per-level operators and MG hierarchies built once,
a fixed pool of request slots per level) and runs a loop:

  1. admit: every queued request whose level has a free slot gets it -- its RHS is
     copied host -> device (pinned, asynchronous) and the slot is started with the
     request's tolerance; requests without a free slot wait in a FIFO per level;
  2. step: one PCG step of everything in flight (a single CUDA graph launch: every
     stage of the step is one launch over the work items of all in-flight requests,
     whatever their level or arrival time);
  3. retire: finished slots are copied device -> host (pinned) and freed.

Requests that arrive while others are on the GPU join at the next step, and each
result is bit-identical to the same request solved alone: a request's iterates
depend only on its own data (per-request reductions in a fixed order).

Admission is under a device-memory budget: the slot pool is sized so that the
solver's device memory (vectors, hierarchies, scratch) stays within it, and a
request is admitted only into a free slot.

``FP64SequentialServer`` is the comparison point: resident FP64 MG hierarchies per
level (the single-system solver), requests served one at a time in arrival order.

``HybridServer`` routes a request that arrives at an idle server to the FP64 MG
hierarchy and batches the rest.

    python -m honei_b200.serving --rates 50,200,1000,2000 --duration 60 [--hybrid] [--fp64]
"""
from __future__ import annotations

import argparse
import collections
import dataclasses
import json
import math
import time

import numpy as np
import torch

from .inputs import uniform
from .solvers import BatchedPoissonSolver, MGData, MGSolver, batch_params, mg_params

LEVELS = tuple(range(5, 12))


@dataclasses.dataclass
class Request:
    rid: int
    level: int
    tol: float
    rhs: torch.Tensor                 # (1, n) FP64, pinned host memory
    arrival: float = 0.0              # seconds on the loop's clock
    done: float = math.nan
    iters: int = 0
    rel_defect: float = math.nan
    x: torch.Tensor | None = None     # (1, n) FP64 host result


def unknowns(level):
    return ((1 << level) + 1) ** 2


def sample_level(rng, lo=5, hi=11):
    """log n uniform in [log (2^lo+1)^2, log (2^hi+1)^2], rounded to the nearest level."""
    m = math.exp(rng.uniform(math.log((1 << lo) + 1), math.log((1 << hi) + 1)))
    return int(min(hi, max(lo, round(math.log2(max(m - 1.0, 1.0))))))


class RhsPool:
    """Seeded U[-1,1] right-hand sides, a few per level, in pinned host memory
    (generated before the loop starts: a server receives its data, it does not make it)."""

    def __init__(self, levels=LEVELS, per_level=4, seed=0):
        self.pool = {L: [torch.from_numpy(uniform(unknowns(L), seed * 1000 + 17 * L + k)).reshape(1, -1).pin_memory()
                         for k in range(per_level)] for L in levels}

    def get(self, level, k):
        p = self.pool[level]
        return p[k % len(p)]


def poisson_arrivals(rate, duration, rng):
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def slot_bytes(level, coarse_level=3):
    """Device bytes one slot of `level` needs: five FP64 outer vectors and four FP32
    vectors per level of its hierarchy, padded to 64 elements."""
    pad = lambda n: max(64, (n + 63) // 64 * 64)
    return 5 * 8 * pad(unknowns(level)) + sum(4 * 4 * pad(unknowns(l)) for l in range(coarse_level, level + 1))


def default_slots(budget_bytes, levels=LEVELS, base=32, coarse_level=3):
    """`base` slots per level, fewer for the largest levels, scaled down to fit the budget."""
    slots = {L: base if L <= 9 else max(4, base // (2 if L == 10 else 4)) for L in levels}
    need = sum(slot_bytes(L, coarse_level) * k for L, k in slots.items())
    if need > 0.8 * budget_bytes:       # headroom for operators, hierarchies, scratch
        f = 0.8 * budget_bytes / need
        slots = {L: max(1, int(k * f)) for L, k in slots.items()}
    return slots


class PoissonServer:
    """keep_results: hand each finished request a host copy of its solution (req.x);
    otherwise the solution is copied to the slot's pinned host buffer and left there
    until the slot's next request (a long run at a high rate would fill host memory)."""

    def __init__(self, slots=None, budget_bytes=120e9, coarse_level=3, params=None, stream=None, keep_results=False):
        self.keep_results = keep_results
        self.slots = slots or default_slots(budget_bytes, coarse_level=coarse_level)
        self.levels = sorted(self.slots)
        estimate = sum(slot_bytes(L, coarse_level) * k for L, k in self.slots.items())
        if estimate > budget_bytes:
            raise MemoryError(f"slot pool needs about {estimate} B > budget {budget_bytes:.0f} B")
        self.systems = [(L, 1) for L in self.levels for _ in range(self.slots[L])]
        self.solver = BatchedPoissonSolver(self.systems, coarse_level=coarse_level,
                                           params=params or batch_params(max_iters=200), stream=stream)
        info = self.solver.info()
        self.device_bytes = info["device_bytes"]
        if self.device_bytes > budget_bytes:
            raise MemoryError(f"slot pool needs {self.device_bytes} B > budget {budget_bytes:.0f} B")
        self.budget_bytes = budget_bytes
        self.free = {L: collections.deque(i for i, (l, _) in enumerate(self.systems) if l == L) for L in self.levels}
        self.queue = {L: collections.deque() for L in self.levels}
        self.active = {}              # system index -> Request
        self.out = {i: torch.empty((1, unknowns(L)), dtype=torch.float64).pin_memory()
                    for i, (L, _) in enumerate(self.systems)}
        self.steps = 0

    def submit(self, req: Request):
        self.queue[req.level].append(req)

    def pending(self):
        return len(self.active) + sum(len(q) for q in self.queue.values())

    def _admit(self):
        for L in self.levels:
            q, free = self.queue[L], self.free[L]
            while q and free:
                req, slot = q.popleft(), free.popleft()
                self.solver.set_rhs(slot, req.rhs)
                self.solver.start(slot, eps=req.tol, zero_guess=True)
                self.active[slot] = req

    def poll(self, clock, steps=1):
        """admit, run `steps` PCG steps of everything in flight, retire; returns the finished requests"""
        self._admit()
        if not self.active:
            return []
        done = self.solver.step(steps)
        self.steps += steps
        finished = []
        for slot in done:
            req = self.active.pop(slot, None)
            if req is None:
                continue
            self.solver.solution(slot, out=self.out[slot])
            req.iters, req.rel_defect = self.solver.result(slot)
            finished.append((slot, req))
        if finished:
            torch.cuda.current_stream().synchronize()
            now = clock()
            for slot, req in finished:
                req.x = self.out[slot].clone() if self.keep_results else None
                req.done = now
                self.free[req.level].append(slot)
        return [req for _, req in finished]


class FP64SequentialServer:
    """Resident FP64 MG hierarchies per level (levels 3..L, V(4,4), coarse CG cap 100);
    requests solved one at a time in arrival order."""

    def __init__(self, levels=LEVELS, coarse_level=3, keep_results=False):
        self.keep_results = keep_results
        self.data = {}
        self.vec = {}
        for L in levels:
            self.data[L] = {tol: MGData.poisson_q1(coarse_level, L, params=mg_params(max_iters_coarse=100, eps=tol,
                                                                                      coarse_eps=1e-10, coarse_exact=False))
                            for tol in (1e-8, 1e-10)}
            self.vec[L] = (torch.empty(unknowns(L), dtype=torch.float64, device="cuda"),
                           torch.empty(unknowns(L), dtype=torch.float64, device="cuda"),
                           torch.empty(unknowns(L), dtype=torch.float64).pin_memory())
        self.queue = collections.deque()

    def submit(self, req):
        self.queue.append(req)

    def pending(self):
        return len(self.queue)

    def poll(self, clock, steps=1):
        if not self.queue:
            return []
        req = self.queue.popleft()
        b, x, out = self.vec[req.level]
        b.copy_(req.rhs.reshape(-1), non_blocking=True)
        x.zero_()
        data = self.data[req.level][req.tol]
        MGSolver.value(data, b, x)
        out.copy_(x, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        req.iters = data.used_iters
        req.rel_defect = data.rnorm_final / data.rnorm_initial
        req.x = out.reshape(1, -1).clone() if self.keep_results else None
        req.done = clock()
        return [req]


class HybridServer:
    """Continuous batching with a fast path for an idle server.  A request that
    arrives while nothing is in flight or waiting is solved at once by the resident
    FP64 MG hierarchy of its level (one graph launch: at low load a single MG solve
    has the lower latency, while a batched PCG step costs a fixed ~0.5 ms and a
    request needs several); requests that find others in flight or waiting join the
    batched mixed-precision engine.  Either way a result meets its tolerance; which
    path served it depends on the load (``routed`` counts them)."""

    def __init__(self, batched: PoissonServer, direct: FP64SequentialServer):
        self.batched, self.direct = batched, direct
        self.waiting = collections.deque()
        self.routed = collections.Counter()

    def submit(self, req):
        self.waiting.append(req)

    def pending(self):
        return len(self.waiting) + self.batched.pending() + self.direct.pending()

    def poll(self, clock, steps=1):
        idle = not self.batched.active and not any(self.batched.queue.values())
        if idle and len(self.waiting) == 1:
            req = self.waiting.popleft()
            self.direct.submit(req)
            self.routed["fp64_mg"] += 1
            return self.direct.poll(clock)
        while self.waiting:
            self.batched.submit(self.waiting.popleft())
            self.routed["batched"] += 1
        return self.batched.poll(clock, steps)


def run(server, rate, duration, pool, seed=0, drain_limit=60.0):
    """Drive `server` with Poisson arrivals at `rate` req/s for `duration` s (host clock);
    returns the latency / throughput summary and the finished requests."""
    rng = np.random.default_rng(seed)
    times = poisson_arrivals(rate, duration, rng)
    reqs = []
    for i, t in enumerate(times):
        L = sample_level(rng)
        tol = 1e-8 if rng.random() < 0.5 else 1e-10
        reqs.append(Request(i, L, tol, pool.get(L, i), arrival=t))
    t0 = time.perf_counter()
    clock = lambda: time.perf_counter() - t0
    nxt, finished = 0, []
    while True:
        now = clock()
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            server.submit(reqs[nxt])
            nxt += 1
        if server.pending():
            finished += server.poll(clock)
        elif nxt < len(reqs):
            time.sleep(max(0.0, min(reqs[nxt].arrival - clock(), 0.001)))
        else:
            break
        if now > duration + drain_limit:
            break
    lat = sorted(1000.0 * (r.done - r.arrival) for r in finished)
    span = max((r.done for r in finished), default=duration)
    pct = lambda p: lat[min(len(lat) - 1, int(round(p / 100.0 * (len(lat) - 1))))] if lat else math.nan
    by_level = collections.Counter(r.level for r in finished)
    return {"rate_req_s": rate, "duration_s": duration, "arrived": len(reqs), "finished": len(finished),
            "solves_per_s": len(finished) / span if span > 0 else math.nan,
            "p50_ms": pct(50), "p99_ms": pct(99), "max_ms": lat[-1] if lat else math.nan,
            "max_rel_defect_1e-8": max((r.rel_defect for r in finished if r.tol == 1e-8), default=math.nan),
            "max_rel_defect_1e-10": max((r.rel_defect for r in finished if r.tol == 1e-10), default=math.nan),
            "levels": dict(sorted(by_level.items()))}, finished


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="50,100,200,500,1000,2000")
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--fp64", action="store_true", help="also run the FP64 sequential server")
    ap.add_argument("--hybrid", action="store_true", help="also run the hybrid server (FP64 MG when idle)")
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    pool = RhsPool(seed=a.seed)
    server = PoissonServer(budget_bytes=a.budget_gb * 1e9)
    print(json.dumps({"slots": server.slots, "device_bytes": server.device_bytes,
                      "budget_bytes": server.budget_bytes}), flush=True)
    run(server, 200, 1.0, pool, seed=a.seed + 99)      # warm-up
    for rate in [float(r) for r in a.rates.split(",")]:
        summary, _ = run(server, rate, a.duration, pool, seed=a.seed)
        summary["server"] = "batched mixed-precision PCG (continuous batching)"
        print(json.dumps(summary), flush=True)
    if a.hybrid:
        hyb = HybridServer(server, FP64SequentialServer())
        run(hyb, 50, 1.0, pool, seed=a.seed + 99)
        for rate in [float(r) for r in a.rates.split(",")]:
            hyb.routed.clear()
            summary, _ = run(hyb, rate, a.duration, pool, seed=a.seed)
            summary["server"] = "hybrid: FP64 MG when idle, else batched mixed-precision PCG"
            summary["routed"] = dict(hyb.routed)
            print(json.dumps(summary), flush=True)
    if a.fp64:
        seq = FP64SequentialServer()
        run(seq, 50, 1.0, pool, seed=a.seed + 99)
        for rate in [float(r) for r in a.rates.split(",")]:
            summary, _ = run(seq, rate, a.duration, pool, seed=a.seed)
            summary["server"] = "FP64 MG, one request at a time"
            print(json.dumps(summary), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
