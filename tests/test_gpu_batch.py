"""Batched MG-preconditioned CG (hb2_batch_*): many Q1 systems of different levels
with several right-hand sides each, solved together.

Checked against the oracle on the CPU: the true residual of every solution
(FP64 ELL product of the oracle), agreement with the oracle's FP64 MG solution,
and -- the property continuous batching rests on -- that every right-hand side's
result is bit-identical whether it is solved alone, in a large mix, or started
while other systems are already in flight.
"""
import numpy as np
import pytest
import torch

import honei_b200 as hb
from honei_b200 import _lib
from honei_b200.inputs import uniform

pytestmark = pytest.mark.gpu

MIX = [(4, 1), (6, 3), (5, 1), (3, 1), (7, 2), (4, 8), (6, 1), (5, 2)]


def rhs_for(system, level, k):
    n = hb.BatchedPoissonSolver.unknowns(level)
    return np.stack([uniform(n, 1000 * system + 17 * j + 3) for j in range(k)])


def solve_mix(systems, seeds=None, **kw):
    B = hb.BatchedPoissonSolver(systems, **kw)
    for s, (level, k) in enumerate(systems):
        sid = seeds[s] if seeds else s
        B.set_rhs(s, torch.from_numpy(rhs_for(sid, level, k)).cuda())
    B.solve()
    torch.cuda.synchronize()
    return B, [B.solution(s).cpu().numpy() for s in range(len(systems))]


def test_batch_true_residual(oracle):
    B, xs = solve_mix(MIX)
    assert B.info()["vectors"] == sum(k for _, k in MIX)
    for s, (level, k) in enumerate(MIX):
        A = oracle.q1_ell(level)
        b = rhs_for(s, level, k)
        for j in range(k):
            it, rel = B.result(s, j)
            assert rel < 1e-8 and 0 < it < 100, (s, j, it, rel)
            r = b[j] - oracle.ell_spmv(A, xs[s][j])
            # the recursive residual tracks the true one closely in FP64
            assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(b[j]), (s, j)


def test_every_rhs_of_the_512_system_batch_converges():
    """The batched workload (512 systems, levels 4..9, a quarter with 8 right-hand
    sides: 1,408 in all): every right-hand side reaches 1e-8 within a few PCG steps.
    (A coarse solve whose recurrence differs from the standard one between calls once
    left some of them short of the tolerance after 100 steps.)"""
    import bench
    systems = bench.batch_workload(2024)
    B, _ = solve_mix(systems)
    worst, most = 0.0, 0
    for s, (level, k) in enumerate(systems):
        for j in range(k):
            it, rel = B.result(s, j)
            worst, most = max(worst, rel), max(most, it)
    assert worst < 1e-8 and most <= 20, (worst, most)


def test_batch_agrees_with_oracle_mg(oracle):
    systems = [(5, 1), (6, 2)]
    B, xs = solve_mix(systems)
    for s, (level, k) in enumerate(systems):
        b = rhs_for(s, level, k)
        for j in range(k):
            x_ref, _, _ = oracle.mg_q1(level, b[j], eps=1e-12)
            err = np.linalg.norm(xs[s][j] - x_ref) / np.linalg.norm(x_ref)
            assert err < 1e-6, (s, j, err)


def test_alone_and_in_the_mix_are_bit_identical():
    _, xs_mix = solve_mix(MIX)
    for s in (0, 4, 5):
        level, k = MIX[s]
        _, xs_alone = solve_mix([(level, k)], seeds=[s])
        assert np.array_equal(xs_alone[0].view(np.uint64), xs_mix[s].view(np.uint64)), s


def test_staggered_starts_match_the_batch_solve():
    """Systems started while others are in flight (serving-style stepping) give
    the same bits as the all-at-once solve."""
    _, xs_ref = solve_mix(MIX)
    B = hb.BatchedPoissonSolver(MIX)
    for s, (level, k) in enumerate(MIX):
        B.set_rhs(s, torch.from_numpy(rhs_for(s, level, k)).cuda())
    pending = list(range(len(MIX)))
    done = set()
    steps = 0
    while len(done) < len(MIX):
        if pending:
            B.start(pending.pop(0))          # one new system per step
        done |= set(B.step(1))
        done -= set(pending)                 # never-started systems report idle
        steps += 1
        assert steps < 400
    for s in range(len(MIX)):
        x = B.solution(s).cpu().numpy()
        assert np.array_equal(x.view(np.uint64), xs_ref[s].view(np.uint64)), s


def test_zero_rhs_and_iteration_cap():
    B = hb.BatchedPoissonSolver([(4, 1), (5, 1)], params=hb.batch_params(max_iters=2))
    B.set_rhs(0, torch.zeros((1, hb.BatchedPoissonSolver.unknowns(4)), dtype=torch.float64, device="cuda"))
    B.set_rhs(1, torch.from_numpy(rhs_for(1, 5, 1)).cuda())
    B.solve()
    assert B.result(0) == (0, 0.0)
    assert not B.solution(0).any()
    it, rel = B.result(1)
    assert it == 2 and rel > 1e-8


def test_bad_levels_are_rejected():
    with pytest.raises(_lib.HoneiError):
        hb.BatchedPoissonSolver([(4, 1)], coarse_level=4)
    with pytest.raises(_lib.HoneiError):
        hb.BatchedPoissonSolver([(2, 1)], coarse_level=3)
