"""Serving loop host logic on the CPU: the request stream and the admission
controller (with a stand-in for the GPU work)."""
import threading
import time

import numpy as np
import pytest

from dgquest_b200 import serving as S


def test_request_stream_shape():
    reqs = S.make_requests(2000, rate=200.0, single=True)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    # mean gap 1/rate within a few percent over 2000 draws
    assert abs(arr[-1] / len(reqs) - 1 / 200.0) < 0.1 / 200.0
    ns = np.array([r.n for r in reqs])
    assert ns.min() == 16 and ns.max() == 33
    kinds = [r.kind for r in reqs]
    frac = {k: kinds.count(k) / len(kinds) for k in ("random", "ghzqft", "bv")}
    assert abs(frac["random"] - 0.4) < 0.05 and abs(frac["ghzqft"] - 0.3) < 0.05
    for r in reqs[:200]:
        assert len(set(r.zq)) == 4 and all(0 <= q < r.n for q in r.zq)
        if r.kind == "random":
            assert 8 <= r.depth <= 24
    f64 = S.make_requests(500, single=False)
    assert max(r.n for r in f64) == 32
    # the stream is a pure function of its seed
    again = S.make_requests(2000, rate=200.0, single=True)
    assert [(r.n, r.kind, r.zq, r.arrival) for r in again] == [(r.n, r.kind, r.zq, r.arrival) for r in reqs]


def test_admission_respects_budget_and_finishes_everything():
    reqs = S.make_requests(60, rate=5000.0, single=False, n_range=(16, 20))
    budget = 3 * (16 << 20)  # room for three 20-qubit states at most
    lock = threading.Lock()
    live = {"bytes": 0, "peak": 0}

    def fake(r):
        with lock:
            live["bytes"] += S.state_bytes(r)
            live["peak"] = max(live["peak"], live["bytes"])
        time.sleep(0.002 * (1 + (r.n - 16)))
        with lock:
            live["bytes"] -= S.state_bytes(r)
        return np.zeros(4, dtype=np.uint64), np.zeros(4)

    srv = S.Server(env=None, hbm_budget=budget, workers=8, runner=fake)
    out = srv.serve(reqs, realtime=True)
    assert [r.rid for r in out] == list(range(60))
    assert live["peak"] <= budget and srv.peak_in_use <= budget
    assert srv.peak_in_flight > 1  # requests overlapped
    st = S.summarize(out)
    assert st["requests"] == 60 and st["p99_ms"] >= st["p50_ms"] > 0


def test_head_of_line_request_is_not_starved():
    # one big request followed by a stream of small ones: the big one must run
    big = S.Request(0, "bv", 20, 0, 1, 0.0, (0, 1, 2, 3), 1, False)
    small = [S.Request(i, "bv", 16, 0, 1, 0.0001 * i, (0, 1, 2, 3), 1, False) for i in range(1, 40)]
    budget = S.state_bytes(big) + S.state_bytes(small[0])

    def fake(r):
        time.sleep(0.003)
        return np.zeros(1, dtype=np.uint64), np.zeros(1)

    srv = S.Server(env=None, hbm_budget=budget, workers=4, max_bypass=3, runner=fake)
    out = srv.serve([big] + small, realtime=False)
    assert len(out) == 40
    admitted_order = sorted(out, key=lambda r: r.admitted)
    assert [r.rid for r in admitted_order].index(0) <= 3 + 1


def test_idle_registers_reused_and_evicted_largest_first():
    """Resident registers: a request reuses an idle register of its size and
    precision; a request that needs a new register evicts idle ones, largest
    first, until the new one fits beside them (host logic only)."""
    budget = (16 << 20) + (16 << 18) + (8 << 18)
    srv = S.Server(env=None, hbm_budget=budget, workers=2, runner=lambda r: (None, None))
    mk = lambda n, single: S.Request(0, "bv", n, 0, 1, 0.0, (0,), 2, single)  # noqa: E731
    srv.idle[(20, False)].append("reg20")
    srv.idle[(18, False)].append("reg18")
    srv.idle[(18, True)].append("reg18f")
    srv.idle_bytes = (16 << 20) + (16 << 18) + (8 << 18)
    q, ev = srv._take(mk(18, False), in_use=16 << 18)
    assert q == "reg18" and ev == [] and srv.reused == 1
    # a new 19-qubit complex128 register: the 20-qubit idle one goes first
    q, ev = srv._take(mk(19, False), in_use=(16 << 18) + (16 << 19))
    assert q is None and ev == ["reg20"]
    assert srv.idle_bytes == 8 << 18


def test_register_creation_retried_when_memory_is_short():
    """Device memory short although the byte count admitted the request
    (the pool's free memory split among blocks of other sizes; here a fake
    device that holds less than the admission budget): the idle registers
    are destroyed and the creation retried; after a second failure the
    server drains the requests in flight and retries once more (host logic
    only, with fake register operations)."""
    from dgquest_b200 import quest as Q
    lock = threading.Lock()
    live, destroyed, failures = {}, [], [0]
    capacity = 40 << 20  # the admission budget below is 64 MiB

    def create(r):
        with lock:
            if sum(live.values()) + S.state_bytes(r) > capacity:
                failures[0] += 1
                raise Q.QuESTError(103, "QuEST Error in function createQureg: CUDA runtime error. (out of memory)")
            q = ("reg", r.rid)
            live[q] = S.state_bytes(r)
            return q

    def destroy(q):
        with lock:
            destroyed.append(q)
            del live[q]

    def runner(r, q):
        time.sleep(0.002)
        return [r.rid], None

    reqs = [S.Request(i, "bv", 16 + (i % 5), 0, 1, 0.001 * i, (0,), 2, bool(i % 2)) for i in range(80)]
    srv = S.Server(env=None, hbm_budget=64 << 20, workers=4, runner=runner, register_ops=(create, destroy))
    res = srv.serve(reqs, realtime=False)
    assert [x.rid for x in res] == list(range(80))
    assert all(x.samples == [x.rid] for x in res)
    assert failures[0] > 0 and destroyed  # memory ran short, idle registers were handed back
    srv.close()
    assert not live

    def broken(r):
        raise Q.QuESTError(104, "Invalid argument.")

    srv = S.Server(env=None, hbm_budget=64 << 20, workers=2, runner=runner, register_ops=(broken, destroy))
    with pytest.raises(Q.QuESTError):
        srv.serve(reqs[:4], realtime=False)
