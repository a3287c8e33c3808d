"""Serving form, host side (no GPU): the request stream, the scheduler's
admission and retirement logic against a fake engine, and the CPU
restatement of the two request kinds."""

import math

import numpy as np
import pytest

from oracle import serving_oracle as so
from ops_b200 import serving


def test_stream_is_seeded_and_follows_the_mix():
    a = serving.make_stream(2000, 50.0, seed=6)
    b = serving.make_stream(2000, 50.0, seed=6)
    assert [(r.kind, r.n, r.arrival) for r in a] == [(r.kind, r.n, r.arrival) for r in b]
    adi = sum(r.kind == serving.ADI3D for r in a) / len(a)
    assert 0.26 < adi < 0.34
    assert all(64 <= r.n <= 2048 for r in a if r.kind == serving.POISSON2D)
    assert all(32 <= r.n <= 192 for r in a if r.kind == serving.ADI3D)
    # Poisson process: mean inter-arrival 1/rate
    gaps = np.diff([r.arrival for r in a])
    assert abs(gaps.mean() - 0.02) < 0.003
    # log-uniform sizes: median near the geometric mean of the range
    pn = sorted(r.n for r in a if r.kind == serving.POISSON2D)
    assert 250 < pn[len(pn) // 2] < 470


class FakeEngine:
    """Finishes a request after `cost` runs; records the active set."""

    def __init__(self, slots=4):
        self.mode = serving.MIXED
        self.slots = slots
        self.active_sets = []
        self.live = {}
        self.next = 0
        self._launches = 0

    def request_bytes(self, kind, n):
        return n * 1000

    def submit(self, kind, n, seed, steps=10):
        assert len(self.live) < self.slots
        rid = self.next
        self.next += 1
        self.live[rid] = [n, 1 + n % 3]
        return rid

    def run(self, iters):
        self.active_sets.append(sorted(self.live))
        self._launches += iters
        done = []
        for rid, v in self.live.items():
            v[1] -= 1
            if v[1] <= 0:
                done.append(rid)
        return done

    def result(self, rid):
        r = serving.Result()
        r.done, r.iterations, r.rel_residual = 1, 7, 1e-9
        return r

    def fetch(self, rid, count):
        return np.zeros(count)

    def release(self, rid):
        del self.live[rid]

    def launches(self):
        return self._launches


def test_scheduler_admits_by_budget_and_retires_continuously():
    eng = FakeEngine()
    stream = [serving.Request(k, serving.POISSON2D, 100 + k, k, 0.0) for k in range(12)]
    st = serving.serve(eng, stream, budget_bytes=350 * 1000, iters=1, max_active=3)
    assert st["requests"] == 12
    # never more than 3 active, never more than the budget (350 KB here)
    assert max(len(s) for s in eng.active_sets) <= 3
    for s in eng.active_sets:
        assert sum(100 + k for k in s) * 1000 <= 350 * 1000
    # continuous batching: some run sees a request that joined after the first run
    assert len(eng.active_sets) > 1 and eng.active_sets[0] != eng.active_sets[-1]
    assert all(r.finish >= r.arrival for r in st["done"])
    assert st["p99_s"] >= st["p50_s"]


def test_thomas_restatement_solves_the_system():
    n = 37
    d = np.random.default_rng(0).standard_normal(n)
    d[0] = d[-1] = 0.0
    x = so.thomas_along(d.reshape(n, 1), 0, 1.0).ravel()
    a, b, c = -0.5, 2.0, -0.5
    r = np.empty(n)
    r[0], r[-1] = x[0] - d[0], x[-1] - d[-1]
    r[1:-1] = a * x[:-2] + b * x[1:-1] + c * x[2:] - d[1:-1]
    assert np.max(np.abs(r)) < 1e-14


def test_adi_restatement_decays_and_keeps_the_boundary():
    u0 = so.adi_init(12, 5)
    u = so.adi_steps(12, 5, 3)
    assert np.array_equal(u[0], u0[0]) and np.array_equal(u[:, :, -1], u0[:, :, -1])
    inner = lambda v: v[1:-1, 1:-1, 1:-1]
    assert np.abs(inner(u)).max() < np.abs(inner(u0)).max()


def test_poisson_rhs_and_residual():
    n = 20
    b = so.poisson_rhs(n, 3)
    assert b.shape == (n, n) and abs(b).max() <= (1.0 / 21) ** 2
    A = np.zeros((n * n, n * n))
    for j in range(n):
        for i in range(n):
            e = np.zeros((n, n))
            e[j, i] = 1.0
            A[:, j * n + i] = so.poisson_apply(e).ravel()
    x = np.linalg.solve(A, b.ravel()).reshape(n, n)
    assert so.relative_residual(x, 3) < 1e-13
