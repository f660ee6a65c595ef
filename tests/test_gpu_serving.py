"""Serving loop on the device: requests admitted while others are in flight, their
iterations batched into shared launches -- and each result bit-identical to the same
request served alone; every result meets its own tolerance (checked against the
oracle's FP64 operator on the CPU)."""
import numpy as np
import pytest
import torch

from honei_b200 import serving

pytestmark = pytest.mark.gpu

SLOTS = {5: 3, 6: 2, 7: 2}


def make(rid, level, tol):
    rhs = torch.from_numpy(serving.uniform(serving.unknowns(level), 100 + rid)).reshape(1, -1).pin_memory()
    return serving.Request(rid, level, tol, rhs)


def serve(server, batches):
    """batches: lists of requests submitted one poll apart; polls until all are done"""
    finished = {}
    tick = [0.0]
    clock = lambda: tick[0]
    for reqs in batches:
        for r in reqs:
            server.submit(r)
        for r in server.poll(clock):
            finished[r.rid] = r
        tick[0] += 1.0
    while server.pending():
        for r in server.poll(clock):
            finished[r.rid] = r
        tick[0] += 1.0
        assert tick[0] < 2000
    return finished


def test_results_are_the_same_alone_and_in_the_mix(oracle):
    mix = [[make(0, 7, 1e-10), make(1, 5, 1e-8)], [make(2, 6, 1e-8)], [], [make(3, 5, 1e-10), make(4, 7, 1e-8)],
           [make(5, 6, 1e-10), make(6, 5, 1e-8), make(7, 5, 1e-8)]]   # 3 level-5 slots: one waits in the queue
    server = serving.PoissonServer(slots=SLOTS, budget_bytes=4e9, keep_results=True)
    got = serve(server, mix)
    assert sorted(got) == list(range(8))
    for reqs in mix:
        for r in reqs:
            alone = serve(serving.PoissonServer(slots=SLOTS, budget_bytes=4e9, keep_results=True), [[make(r.rid, r.level, r.tol)]])
            a, m = alone[r.rid], got[r.rid]
            assert np.array_equal(a.x.numpy().view(np.uint64), m.x.numpy().view(np.uint64)), r.rid
            assert a.iters == m.iters
            assert m.rel_defect < r.tol
            A = oracle.q1_ell(r.level)
            b = r.rhs.numpy()[0]
            res = b - oracle.ell_spmv(A, m.x.numpy()[0])
            assert np.linalg.norm(res) <= 1.05 * r.tol * np.linalg.norm(b), r.rid


def test_admission_respects_the_device_memory_budget():
    server = serving.PoissonServer(slots=SLOTS, budget_bytes=4e9, keep_results=True)
    assert server.device_bytes <= 4e9
    with pytest.raises(MemoryError):
        serving.PoissonServer(slots={7: 64}, budget_bytes=50e6)


def test_queue_waits_for_a_free_slot():
    server = serving.PoissonServer(slots={5: 1}, budget_bytes=1e9, keep_results=True)
    reqs = [make(i, 5, 1e-8) for i in range(3)]
    got = serve(server, [reqs])
    # one slot: requests finish strictly one after another, in arrival order
    done = [got[i].done for i in range(3)]
    assert done[0] < done[1] < done[2]


def test_hybrid_server_routes_by_load(oracle):
    """An idle server solves a lone request on the FP64 MG hierarchy; requests that find
    others waiting go to the batched engine.  Every result meets its tolerance on the
    oracle's FP64 operator, whichever path served it."""
    hyb = serving.HybridServer(serving.PoissonServer(slots=SLOTS, budget_bytes=4e9, keep_results=True),
                               serving.FP64SequentialServer(levels=(5, 6, 7), keep_results=True))
    got = serve(hyb, [[make(0, 6, 1e-8)], [], [make(1, 7, 1e-10), make(2, 5, 1e-8), make(3, 6, 1e-10)]])
    assert sorted(got) == [0, 1, 2, 3]
    assert hyb.routed["fp64_mg"] == 1 and hyb.routed["batched"] == 3
    for r in got.values():
        A = oracle.q1_ell(r.level)
        b = r.rhs.numpy()[0]
        res = b - oracle.ell_spmv(A, r.x.numpy()[0])
        assert np.linalg.norm(res) <= 1.05 * r.tol * np.linalg.norm(b), r.rid
