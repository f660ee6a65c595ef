"""Host-side logic of the serving loop (no GPU): arrivals, level sampling, slot sizing."""
import collections

import numpy as np

from honei_b200 import serving


def test_poisson_arrivals_rate():
    rng = np.random.default_rng(1)
    t = serving.poisson_arrivals(500.0, 20.0, rng)
    assert abs(len(t) - 10000) < 400
    assert all(b > a for a, b in zip(t, t[1:])) and t[-1] < 20.0


def test_levels_log_uniform_over_5_to_11():
    rng = np.random.default_rng(2)
    c = collections.Counter(serving.sample_level(rng) for _ in range(20000))
    assert set(c) == set(range(5, 12))
    # log-uniform in the grid width: interior levels about equally likely, the ends half as likely
    inner = [c[L] / 20000 for L in range(6, 11)]
    assert max(inner) - min(inner) < 0.03
    assert abs(c[5] / 20000 - 0.5 * np.mean(inner)) < 0.03 and abs(c[11] / 20000 - 0.5 * np.mean(inner)) < 0.03


def test_slot_pool_fits_the_budget():
    for budget in (120e9, 8e9, 1e9):
        slots = serving.default_slots(budget)
        need = sum(serving.slot_bytes(L) * k for L, k in slots.items())
        assert need <= 0.8 * budget or all(k == 1 for k in slots.values())
        assert set(slots) == set(range(5, 12))
    assert serving.default_slots(120e9)[5] == 32


class _FakeBatched:
    def __init__(self):
        self.active, self.queue, self.got = {}, {5: collections.deque()}, []

    def submit(self, r):
        self.got.append(r)

    def pending(self):
        return 0

    def poll(self, clock, steps=1):
        return []


class _FakeDirect(_FakeBatched):
    def poll(self, clock, steps=1):
        return [self.got.pop()] if self.got else []


def test_hybrid_routing_rule():
    """a lone request at an idle server goes to the FP64 MG path, a burst to the batch"""
    b, d = _FakeBatched(), _FakeDirect()
    hyb = serving.HybridServer(b, d)
    hyb.submit("a")
    assert hyb.poll(lambda: 0.0) == ["a"] and hyb.routed["fp64_mg"] == 1
    for r in ("b", "c"):
        hyb.submit(r)
    hyb.poll(lambda: 0.0)
    assert b.got == ["b", "c"] and hyb.routed["batched"] == 2
    b.active = {0: "b"}          # something in flight: even a lone request is batched
    hyb.submit("d")
    hyb.poll(lambda: 0.0)
    assert b.got[-1] == "d" and hyb.routed["fp64_mg"] == 1
