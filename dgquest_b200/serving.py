"""Serving loop: circuits arriving as a Poisson stream, admitted by state bytes
against free HBM, run concurrently (continuous batching).

Every admitted request gets its own register, and so its own CUDA stream and
its own stream-ordered allocation: requests that arrive while others are on
the GPU start as soon as a worker slot and enough memory are free, and their
kernels overlap on the device with the ones already running. A request's
result depends only on the request (its circuit, its sample seed), never on
what else is in flight, which is what the mix-invariance test checks.

Request i of a stream (seeded MT19937, published algorithm):
  arrival gap -ln(1 - u) / rate; n uniform in [16, 33] (complex64) or
  [16, 32] (complex128); kind 40 % random layers (depth uniform in [8, 24]),
  30 % GHZ+QFT, 30 % Bernstein-Vazirani; 4 distinct qubits for <Z>.
Each request returns 1024 sampled bitstrings and <Z_q> on its 4 qubits.

No counterpart in dgQuEST, which runs one circuit per process."""
import collections
import math
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import circuits as C
from . import quest as Q

SAMPLES = 1024


@dataclass
class Request:
    rid: int
    kind: str       # "random" | "ghzqft" | "bv"
    n: int
    depth: int      # random-layer depth (0 for the other kinds)
    seed: int       # circuit seed
    arrival: float  # seconds after the stream starts
    zq: tuple       # qubits whose <Z> is returned
    sample_seed: int
    single: bool    # complex64 register


@dataclass
class Result:
    rid: int
    samples: np.ndarray
    expz: np.ndarray
    arrival: float
    admitted: float
    done: float

    @property
    def latency(self):
        return self.done - self.arrival


def make_requests(count, rate=200.0, single=False, seed=None, n_range=None, first_id=0):
    """Request stream: `seed` drives arrivals, sizes and kinds; circuit and
    sample seeds follow the request ids first_id, first_id + 1, ..."""
    rng = C.Mt19937(C.config_seed(5) if seed is None else seed)
    lo, hi = n_range or ((16, 33) if single else (16, 32))
    t = 0.0
    out = []
    for i in range(count):
        t += -math.log(1.0 - rng.uniform()) / rate
        n = lo + rng.below(hi - lo + 1)
        u = rng.uniform()
        kind = "random" if u < 0.4 else ("ghzqft" if u < 0.7 else "bv")
        depth = 8 + rng.below(17) if kind == "random" else 0
        zq = []
        while len(zq) < min(4, n):
            q = rng.below(n)
            if q not in zq:
                zq.append(q)
        rid = first_id + i
        out.append(Request(rid, kind, n, depth, C.config_seed(5, rid), t, tuple(zq), C.config_seed(5, 100000 + rid),
                           single))
    return out


def request_ops(r):
    if r.kind == "random":
        return C.random_layers(r.n, r.depth, r.seed)
    if r.kind == "ghzqft":
        return C.ghz_qft(r.n)
    return C.bernstein_vazirani(r.n, r.seed, measure=False)


def state_bytes(r):
    return (8 if r.single else 16) << max(r.n, 9)


def run_request(r, env, ops=None, q=None):
    """One request: samples and <Z> (2 P(q=0) - 1). With q (a register of the
    request's size and precision, lent by the server) the register is reset
    to |0...0> and kept; otherwise the request creates and destroys its own."""
    own = q is None
    if own:
        q = Q.dgq_createQuregF32(r.n, env) if r.single else Q.createQureg(r.n, env)
    try:
        Q.initZeroState(q)
        Q.apply_circuit(q, request_ops(r) if ops is None else ops)
        samples = Q.sample(q, SAMPLES, r.sample_seed)
        expz = np.array([2.0 * Q.calcProbOfOutcome(q, k, 0) - 1.0 for k in r.zq])
    finally:
        if own:
            Q.destroyQureg(q, env)
    return samples, expz


class Server:
    """Admission by state bytes, `workers` requests in flight at most.

    A waiting request is admitted when its state fits in the budget next to
    the states in flight; requests behind one that does not fit may go first
    (first fit in arrival order) until it has been passed over `max_bypass`
    times, after which nothing else is admitted before it.

    States stay resident: a finished request's register goes back to an idle
    set and the next request of the same size and precision reuses it (reset
    to |0...0>), so requests do not pay for creating and destroying device
    state under load. Idle registers are destroyed, largest first, when a new
    register would not fit in the budget beside them."""

    def __init__(self, env, hbm_budget=None, workers=6, max_bypass=8, runner=None, cached_kernels_only=True,
                 keep_resident=False, spec_policy=1, register_ops=None):
        self.env = env
        # one-off circuit structures run the interpreting kernel instead of
        # waiting for a kernel compile; their kernels compile in the background
        self.cached_kernels_only = cached_kernels_only and runner is None
        # 1: kernels of new structures compile in the background for later
        # requests; 2: nothing is compiled (structures that never repeat)
        self.spec_policy = spec_policy
        # register_ops = (create(r) -> register, destroy(register)): the
        # register path with a caller's runner(r, register) (host-only tests)
        self.custom_runner = runner if register_ops is None else None
        self.runner = runner or (lambda r, q=None: run_request(r, env, q=q))
        if register_ops is None:
            register_ops = (lambda r: Q.dgq_createQuregF32(r.n, env) if r.single else Q.createQureg(r.n, env),
                            lambda q: Q.destroyQureg(q, env))
        self._create_reg, self._destroy_reg = register_ops
        self.idle = collections.defaultdict(list)  # (n, single) -> registers
        self.idle_bytes = 0
        self.reused = 0
        # keep_resident: idle registers outlive serve() (until close())
        self.keep_resident = keep_resident
        self.peak_in_use = 0
        self.peak_in_flight = 0
        if hbm_budget is None:
            # free HBM (with the register pool's spare memory), less a margin
            # for the per-request scratch, the specialised kernels and the
            # pool's fragmentation
            hbm_budget = int(Q.dgq_getAvailableMemory() * 0.85)
        self.budget = int(hbm_budget)
        self.workers = int(workers)
        self.max_bypass = int(max_bypass)

    def prewarm(self, single=False):
        """Grows the register memory pool to the budget once (registers are
        stream-ordered allocations from a pool that keeps freed memory), so
        that the first requests do not pay for mapping fresh device memory.
        Returns the bytes touched."""
        regs, used = [], 0
        n = 33 if single else 32
        try:
            while n >= 16:
                b = (8 if single else 16) << n
                if used + b > self.budget:
                    n -= 1
                    continue
                q = Q.dgq_createQuregF32(n, self.env) if single else Q.createQureg(n, self.env)
                regs.append(q)
                used += b
        finally:
            for q in regs:
                Q.destroyQureg(q, self.env)
        return used

    def prespecialise(self, single=False, n_range=None, background=True):
        """Queues the compiles of the specialised kernels of the circuit
        structures that recur in the stream: GHZ+QFT of every size from the
        JIT threshold (22 qubits) up (random-layer and Bernstein-Vazirani
        structures depend on each request's seed). Returns the kernels queued."""
        from . import ir
        lo, hi = n_range or ((16, 33) if single else (16, 32))
        total = 0
        for n in range(max(lo, 22), hi + 1):
            total += ir.specialise(C.ghz_qft(n), n, 1 if single else 2, background=background)
        return total

    def _take(self, r, in_use):
        """With the lock held: an idle register for r (or None: create one),
        and the idle registers to destroy so that a new one fits."""
        key = (r.n, r.single)
        if self.idle[key]:
            self.idle_bytes -= state_bytes(r)
            self.reused += 1
            return self.idle[key].pop(), []
        evict = []
        # in_use already counts r: keep idle + in_use within the budget
        order = sorted(((n, single) for (n, single), regs in self.idle.items() if regs),
                       key=lambda k: -((8 if k[1] else 16) << max(k[0], 9)))
        for k in order:
            while self.idle[k] and self.idle_bytes + in_use > self.budget:
                evict.append(self.idle[k].pop())
                self.idle_bytes -= (8 if k[1] else 16) << max(k[0], 9)
        return None, evict

    def close(self):
        """Destroys the idle registers."""
        for regs in self.idle.values():
            for q in regs:
                self._destroy_reg(q)
        self.idle.clear()
        self.idle_bytes = 0

    def _create(self, r, cond, state):
        """A new register for admitted request r. The byte count admitted r,
        but device memory can still be short where the pool's free memory
        is split among blocks of other sizes: on an out-of-memory error the
        idle registers are destroyed and the creation retried; on a second
        one, no further request is admitted until the others in flight have
        finished, and the creation is retried then (with the lock held)."""
        def short(exc):
            return isinstance(exc, Q.QuESTError) and exc.code in (101, 103)

        for attempt in range(2):
            try:
                return self._create_reg(r)
            except Exception as exc:  # noqa: BLE001
                if not short(exc):
                    raise
            with cond:
                if attempt == 0:
                    self.close()
                    continue
                state["draining"] += 1
                try:
                    # (requests whose creation waits here too count as finished)
                    while state["in_flight"] > state["draining"] and state["error"] is None:
                        cond.wait(0.05)
                    self.close()
                    return self._create_reg(r)
                finally:
                    state["draining"] -= 1
                    cond.notify_all()

    def serve(self, requests, realtime=True):
        """Runs the stream; returns results in request order. With realtime,
        request i becomes visible at its arrival time, else all at once."""
        requests = sorted(requests, key=lambda r: r.arrival)
        for r in requests:
            if state_bytes(r) > self.budget:
                raise ValueError(f"request {r.rid}: {state_bytes(r)} state bytes exceed the budget {self.budget}")
        cond = threading.Condition()
        waiting = collections.deque()
        bypassed = collections.Counter()
        state = {"in_use": 0, "in_flight": 0, "arrived": 0, "finished": 0, "error": None, "draining": 0}
        results = {}
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        def arrivals():
            for r in requests:
                if realtime:
                    dt = r.arrival - now()
                    if dt > 0:
                        time.sleep(dt)
                with cond:
                    waiting.append(r)
                    state["arrived"] += 1
                    cond.notify_all()

        def pick():
            # called with the lock held: first fit, head reserved once bypassed enough
            if state["draining"]:
                return None
            for i, r in enumerate(waiting):
                if state["in_use"] + state_bytes(r) <= self.budget:
                    for j in range(i):
                        bypassed[waiting[j].rid] += 1
                    del waiting[i]
                    return r
                if bypassed[r.rid] >= self.max_bypass:
                    return None
            return None

        def worker():
            while True:
                with cond:
                    while True:
                        if state["error"] is not None:
                            return
                        r = pick()
                        if r is not None:
                            break
                        if state["arrived"] == len(requests) and not waiting:
                            return
                        cond.wait(0.05)
                    state["in_use"] += state_bytes(r)
                    state["in_flight"] += 1
                    self.peak_in_use = max(self.peak_in_use, state["in_use"])
                    self.peak_in_flight = max(self.peak_in_flight, state["in_flight"])
                    admitted = now()
                    q = None
                    if self.custom_runner is None:
                        q, evict = self._take(r, state["in_use"])
                        # destroyed before the lock is released, so that no
                        # other worker counts on memory that is not free yet
                        for e in evict:
                            self._destroy_reg(e)
                try:
                    if self.custom_runner is not None:
                        samples, expz = self.runner(r)
                    else:
                        if q is None:
                            q = self._create(r, cond, state)
                        samples, expz = self.runner(r, q)
                except Exception as exc:  # noqa: BLE001
                    if q is not None:
                        self._destroy_reg(q)
                    with cond:
                        state["error"] = exc
                        cond.notify_all()
                    return
                with cond:
                    if q is not None:
                        self.idle[(r.n, r.single)].append(q)
                        self.idle_bytes += state_bytes(r)
                    state["in_use"] -= state_bytes(r)
                    state["in_flight"] -= 1
                    state["finished"] += 1
                    results[r.rid] = Result(r.rid, samples, expz, r.arrival, admitted, now())
                    cond.notify_all()

        prev_policy = Q.dgq_setSpecialisationPolicy(self.spec_policy) if self.cached_kernels_only else None
        feeder = threading.Thread(target=arrivals, daemon=True)
        pool = [threading.Thread(target=worker, daemon=True) for _ in range(self.workers)]
        feeder.start()
        for t in pool:
            t.start()
        feeder.join()
        for t in pool:
            t.join()
        if prev_policy is not None:
            Q.dgq_setSpecialisationPolicy(prev_policy)
        if not self.keep_resident:
            self.close()
        if state["error"] is not None:
            raise state["error"]
        return [results[r.rid] for r in sorted(requests, key=lambda r: r.rid)]


def summarize(results):
    lat = np.array([r.latency for r in results]) * 1e3
    first = min(r.arrival for r in results)
    last = max(r.done for r in results)
    return {"requests": len(results), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "circuits_per_s": len(results) / (last - first) if last > first else float("nan"),
            "wall_s": last - first}
