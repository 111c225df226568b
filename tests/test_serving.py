"""Request loop: admission against an HBM budget in arrival order, concurrency and the latency summary
(CPU, with a stand-in solver); on the GPU, each solve is bit-identical alone and in a mix."""
import threading
import time

import numpy as np
import pytest

from common import pkg

S = pkg.serving


def _req(rid, arrival, n=8, G=3):
    prob = pkg.problems.random_small(100 + rid, n, n, G, "S8")
    return S.Request(rid, arrival, prob, steps=2, maxit=2)


def test_config3_stream_shape():
    reqs = S.config3_requests(rate=200.0, duration=2.0, seed=3)
    assert 300 < len(reqs) < 500                       # ~ rate * duration
    t = [r.arrival_s for r in reqs]
    assert t == sorted(t) and t[-1] < 2.0
    assert all(32 <= r.prob.nx <= 384 and 17 <= r.prob.ng <= 64 and r.prob.quad in ("S8", "S16") for r in reqs)
    assert [r.prob.nx for r in S.config3_requests(200.0, 2.0, 3)] == [r.prob.nx for r in reqs]   # seeded


def test_admission_respects_budget_and_order():
    sizes = {0: 60, 1: 50, 2: 30, 3: 30, 4: 100}
    running, peak = [0], [0]
    lock = threading.Lock()
    order = []

    def fake_solve(r, t0):
        with lock:
            running[0] += sizes[r.rid]
            peak[0] = max(peak[0], running[0])
            order.append(r.rid)
        time.sleep(0.05)
        with lock:
            running[0] -= sizes[r.rid]
        return S.Result(r.rid, r.arrival_s, 0.0, time.perf_counter() - t0, sizes[r.rid], 10, [1.0], [1])

    srv = S.Server(hbm_budget=100, max_active=8, solver=fake_solve, sizer=lambda r: sizes[r.rid])
    res, log = srv.run([_req(k, 0.0) for k in range(5)], realtime=False)
    assert [r.rid for r in res] == [0, 1, 2, 3, 4]
    assert peak[0] <= 100                               # never over budget
    assert order == [0, 1, 2, 3, 4]                     # strict arrival order (head-of-line blocking)
    assert [e[1] for e in log] == [0, 1, 2, 3, 4]
    assert all(e[2] <= 100 for e in log)


def test_oversized_request_is_refused():
    srv = S.Server(hbm_budget=10, solver=lambda r, t0: None, sizer=lambda r: 11)
    with pytest.raises(ValueError):
        srv.run([_req(0, 0.0)], realtime=False)


def test_realtime_admission_waits_for_arrival():
    def fake_solve(r, t0):
        now = time.perf_counter() - t0
        return S.Result(r.rid, r.arrival_s, now, now, 1, 1, [1.0], [1])

    srv = S.Server(hbm_budget=10, solver=fake_solve, sizer=lambda r: 1)
    res, log = srv.run([_req(0, 0.0), _req(1, 0.15)], realtime=True)
    assert log[1][0] >= 0.15 - 1e-3                      # not admitted before it arrived
    summ = S.latency_summary(res)
    assert summ["requests"] == 2 and summ["failed"] == 0


@pytest.mark.gpu
def test_solve_is_identical_alone_and_in_a_mix():
    reqs = [_req(k, 0.0, n=12 + 4 * k, G=2 + k % 2) for k in range(4)]
    alone, _ = S.Server(hbm_budget=1 << 40, max_active=1).run(reqs, realtime=False)
    mixed, log = S.Server(hbm_budget=1 << 40, max_active=4).run(reqs, realtime=False)
    assert all(not r.error for r in alone + mixed), [r.error for r in alone + mixed]
    for a, b in zip(alone, mixed):
        assert np.array_equal(a.T, b.T)
        assert a.its == b.its
    assert max(e[2] for e in log) >= sum(S.required_bytes(r) for r in reqs[:2])   # several ran at once


@pytest.mark.gpu
def test_budget_limits_concurrency_on_device():
    reqs = [_req(k, 0.0, n=16) for k in range(4)]
    one = max(S.required_bytes(r) for r in reqs)
    res, log = S.Server(hbm_budget=2 * one + 1, max_active=8).run(reqs, realtime=False)
    assert all(not r.error for r in res), [r.error for r in res]
    assert max(e[2] for e in log) <= 2 * one + 1


@pytest.mark.gpu
def test_batched_server_matches_solves_alone():
    """Continuous batching: requests of different sizes, quadratures and precisions, arriving while
    others run, give the same temperatures as each solved on its own."""
    reqs = [_req(k, 0.02 * k, n=10 + 3 * k, G=2 + k % 2) for k in range(5)]
    reqs[1].precision = "fp64"
    reqs[3].prob = pkg.problems.random_small(203, 9, 11, 2, "S12")
    alone, _ = S.Server(hbm_budget=1 << 40, max_active=1).run(reqs, realtime=False)
    batched, log = S.BatchedServer(hbm_budget=1 << 40).run(reqs, realtime=True)
    assert all(not r.error for r in alone + batched), [r.error for r in alone + batched]
    for a, b in zip(alone, batched):
        assert np.array_equal(a.T, b.T)
        assert a.its == b.its
    assert len(log) == 5
