"""Seeded synthetic circuits and the op-list record shared by every path.

An op list is a numpy structured array of OP_DTYPE; one record is one QuEST
API call (kinds below). The same list is replayed through this library's
QuEST API (``replay``), applied by the CPU oracle, and fed to the reference
build, so all three see identical calls.

Randomness: MT19937 seeded with ``init_genrand(seed)`` (``Mt19937`` below,
the generator the reference links, src/mt19937ar.c:61-74), drawn as
  u32()          = genrand_int32
  uniform()      = 53-bit (a >> 5, b >> 6) construction on [0, 1)
  below(k)       = u32() % k
Seeds follow the plan's convention seed = 20261203 + 1000 * config + request.

Workloads (the reference's benchmark circuits have no public suite; these
are seeded stand-ins with the shapes its headline configurations name):
  ghz_qft(n)                    GHZ chain then QFT with controlledPhaseShift
                                and a final swap network
  random_layers(n, depth, seed) per layer Rx/Ry/Rz with U[0, 2pi) angles on
                                every qubit, then CZ on a Fisher-Yates
                                perfect matching
  bernstein_vazirani(n, seed)   hidden (n-1)-bit string, optional measurement
  grid_sqrt(rows, cols, depth)  sqrt(X)/sqrt(Y)/sqrt(W) layers and CZ on four
                                alternating grid-edge patterns
  hea(n, depth, seed)           Ry, Rz on every qubit then a CNOT ladder
"""
import math

import numpy as np

OP_DTYPE = np.dtype([("kind", "<i4"), ("q0", "<i4"), ("q1", "<i4"), ("q2", "<i4"), ("p", "<f8", (8,))])
assert OP_DTYPE.itemsize == 80

H, X, Y, Z, S, T, RX, RY, RZ, PHASE = range(10)
CNOT, CZ, CPHASE, CRX, CRY, CRZ, COMPACT, CCOMPACT, UNITARY, CUNITARY = range(10, 20)
SQX, SQY, SQW, SWAP, MEASURE, CY = range(20, 26)

KIND_NAMES = {
    H: "hadamard", X: "pauliX", Y: "pauliY", Z: "pauliZ", S: "sGate", T: "tGate", RX: "rotateX", RY: "rotateY",
    RZ: "rotateZ", PHASE: "phaseShift", CNOT: "controlledNot", CZ: "controlledPhaseFlip",
    CPHASE: "controlledPhaseShift", CRX: "controlledRotateX", CRY: "controlledRotateY", CRZ: "controlledRotateZ",
    COMPACT: "compactUnitary", CCOMPACT: "controlledCompactUnitary", UNITARY: "unitary",
    CUNITARY: "controlledUnitary", SQX: "SqX", SQY: "SqY", SQW: "SqW", SWAP: "swapGate", MEASURE: "measure",
    CY: "controlledPauliY",
}

CONFIG_SEED_BASE = 20261203


def config_seed(config, request=0):
    return CONFIG_SEED_BASE + 1000 * config + request


class Mt19937:
    """MT19937 with init_genrand seeding (published algorithm)."""

    N, M = 624, 397

    def __init__(self, seed):
        mt = [0] * self.N
        mt[0] = seed & 0xFFFFFFFF
        for i in range(1, self.N):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mt = mt
        self.idx = self.N

    def _twist(self):
        mt, N, M = self.mt, self.N, self.M
        for k in range(N):
            y = (mt[k] & 0x80000000) | (mt[(k + 1) % N] & 0x7FFFFFFF)
            mt[k] = mt[(k + M) % N] ^ (y >> 1) ^ (0x9908B0DF if (y & 1) else 0)
        self.idx = 0

    def u32(self):
        if self.idx >= self.N:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF

    def uniform(self):
        a = self.u32() >> 5
        b = self.u32() >> 6
        return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0)

    def below(self, k):
        return self.u32() % k


class OpList:
    """Builder for op lists."""

    def __init__(self):
        self.rows = []

    def add(self, kind, q0=0, q1=0, q2=0, p=()):
        pp = [0.0] * 8
        for i, v in enumerate(p):
            pp[i] = float(v)
        self.rows.append((int(kind), int(q0), int(q1), int(q2), pp))
        return self

    def array(self):
        arr = np.zeros(len(self.rows), dtype=OP_DTYPE)
        for i, (k, a, b, c, p) in enumerate(self.rows):
            arr[i]["kind"] = k
            arr[i]["q0"] = a
            arr[i]["q1"] = b
            arr[i]["q2"] = c
            arr[i]["p"] = p
        return arr


# ---------------------------------------------------------------- workloads
def ghz_qft(n, swaps=True):
    """H(0); CNOT(i, i+1); for t = n-1..0: H(t), CPHASE(c, t, pi/2^(t-c)) for c < t; swaps (i, n-1-i)."""
    b = OpList()
    b.add(H, 0)
    for i in range(n - 1):
        b.add(CNOT, i, i + 1)
    for t in range(n - 1, -1, -1):
        b.add(H, t)
        for c in range(t - 1, -1, -1):
            b.add(CPHASE, c, t, p=(math.pi / (2 ** (t - c)),))
    if swaps:
        for i in range(n // 2):
            b.add(SWAP, i, n - 1 - i)
    return b.array()


def perfect_matching(rng, n):
    perm = list(range(n))
    for i in range(n - 1, 0, -1):
        j = rng.below(i + 1)
        perm[i], perm[j] = perm[j], perm[i]
    return [(perm[2 * k], perm[2 * k + 1]) for k in range(n // 2)]


def random_layers(n, depth, seed):
    """Per layer: Rx/Ry/Rz (uniform choice) with U[0, 2pi) angle on each qubit, then CZ on a random matching."""
    rng = Mt19937(seed)
    b = OpList()
    kinds = (RX, RY, RZ)
    for _ in range(depth):
        for q in range(n):
            k = kinds[rng.below(3)]
            b.add(k, q, p=(2.0 * math.pi * rng.uniform(),))
        for (a, c) in perfect_matching(rng, n):
            b.add(CZ, a, c)
    return b.array()


def bv_secret(n, seed):
    rng = Mt19937(seed)
    return [rng.below(2) for _ in range(n - 1)]


def bernstein_vazirani(n, seed, measure=True):
    """Hidden string s on qubits 0..n-2, ancilla n-1: H layer, X+H ancilla, CNOT(i, n-1) for s_i, H layer."""
    s = bv_secret(n, seed)
    b = OpList()
    for q in range(n - 1):
        b.add(H, q)
    b.add(X, n - 1)
    b.add(H, n - 1)
    for q in range(n - 1):
        if s[q]:
            b.add(CNOT, q, n - 1)
    for q in range(n - 1):
        b.add(H, q)
    if measure:
        for q in range(n):
            b.add(MEASURE, q)
    return b.array()


def grid_edges(rows, cols, pattern):
    """Four alternating edge patterns: 0/1 horizontal even/odd columns, 2/3 vertical even/odd rows."""
    edges = []
    if pattern in (0, 1):
        for r in range(rows):
            for c in range(pattern, cols - 1, 2):
                edges.append((r * cols + c, r * cols + c + 1))
    else:
        for r in range(pattern - 2, rows - 1, 2):
            for c in range(cols):
                edges.append((r * cols + c, (r + 1) * cols + c))
    return edges


def grid_sqrt(rows, cols, depth, seed):
    """Per cycle: sqrt(X)/sqrt(Y)/sqrt(W), never the previous gate on that qubit; then CZ on pattern cycle % 4."""
    rng = Mt19937(seed)
    n = rows * cols
    b = OpList()
    prev = [-1] * n
    choices = (SQX, SQY, SQW)
    for cycle in range(depth):
        for q in range(n):
            while True:
                g = choices[rng.below(3)]
                if g != prev[q]:
                    break
            prev[q] = g
            b.add(g, q)
        for (a, c) in grid_edges(rows, cols, cycle % 4):
            b.add(CZ, a, c)
    return b.array()


def hea(n, depth, seed):
    """Hardware-efficient ansatz: per layer Ry(theta), Rz(phi) on each qubit, then CNOT(i, i+1).

    Angles are 2 pi x the MT19937 (init_genrand(seed)) 53-bit uniforms in
    gate order; numpy's RandomState draws the same sequence (two 32-bit
    outputs per double, a >> 5 and b >> 6), which keeps this vectorised."""
    per = 2 * n + (n - 1)
    arr = np.zeros(depth * per, dtype=OP_DTYPE)
    if depth == 0 or n == 0:
        return arr
    ang = 2.0 * math.pi * np.random.RandomState(seed & 0xFFFFFFFF).random_sample(2 * n * depth)
    layer = np.zeros(per, dtype=OP_DTYPE)
    layer["kind"][0:2 * n:2] = RY
    layer["kind"][1:2 * n:2] = RZ
    layer["q0"][0:2 * n] = np.repeat(np.arange(n), 2)
    layer["kind"][2 * n:] = CNOT
    layer["q0"][2 * n:] = np.arange(n - 1)
    layer["q1"][2 * n:] = np.arange(1, n)
    for d in range(depth):
        blk = arr[d * per:(d + 1) * per]
        blk[:] = layer
        blk["p"][:2 * n, 0] = ang[d * 2 * n:(d + 1) * 2 * n]
    return arr


def batch_workload(count, seed=None):
    """The batched workload: `count` hardware-efficient ansatz circuits with
    qubit counts uniform in [10, 22] and depths uniform in [4, 32]; sizes are
    drawn from MT19937(seed) (n = 10 + u32 % 13, depth = 4 + u32 % 29) and
    circuit i uses angle seed config_seed(4, i). Returns [(n, depth, ops)]."""
    rng = Mt19937(config_seed(4) if seed is None else seed)
    out = []
    for i in range(count):
        n = 10 + rng.below(13)
        d = 4 + rng.below(29)
        out.append((n, d, hea(n, d, config_seed(4, i))))
    return out


def replay(q, ops, quest=None):
    """Replays an op list through the QuEST API of libdgq; returns measurement outcomes."""
    if quest is None:
        from . import quest as quest_mod
        quest = quest_mod
    outcomes = []
    for rec in ops:
        k = int(rec["kind"])
        a, b = int(rec["q0"]), int(rec["q1"])
        p = rec["p"]
        if k == H:
            quest.hadamard(q, a)
        elif k == X:
            quest.pauliX(q, a)
        elif k == Y:
            quest.pauliY(q, a)
        elif k == Z:
            quest.pauliZ(q, a)
        elif k == S:
            quest.sGate(q, a)
        elif k == T:
            quest.tGate(q, a)
        elif k == RX:
            quest.rotateX(q, a, float(p[0]))
        elif k == RY:
            quest.rotateY(q, a, float(p[0]))
        elif k == RZ:
            quest.rotateZ(q, a, float(p[0]))
        elif k == PHASE:
            quest.phaseShift(q, a, float(p[0]))
        elif k == CNOT:
            quest.controlledNot(q, a, b)
        elif k == CY:
            quest.controlledPauliY(q, a, b)
        elif k == CZ:
            quest.controlledPhaseFlip(q, a, b)
        elif k == CPHASE:
            quest.controlledPhaseShift(q, a, b, float(p[0]))
        elif k == CRX:
            quest.controlledRotateX(q, a, b, float(p[0]))
        elif k == CRY:
            quest.controlledRotateY(q, a, b, float(p[0]))
        elif k == CRZ:
            quest.controlledRotateZ(q, a, b, float(p[0]))
        elif k == COMPACT:
            quest.compactUnitary(q, a, quest.Complex(p[0], p[1]), quest.Complex(p[2], p[3]))
        elif k == CCOMPACT:
            quest.controlledCompactUnitary(q, a, b, quest.Complex(p[0], p[1]), quest.Complex(p[2], p[3]))
        elif k in (UNITARY, CUNITARY):
            m = quest.ComplexMatrix2(quest.Complex(p[0], p[1]), quest.Complex(p[2], p[3]),
                                     quest.Complex(p[4], p[5]), quest.Complex(p[6], p[7]))
            if k == UNITARY:
                quest.unitary(q, a, m)
            else:
                quest.controlledUnitary(q, a, b, m)
        elif k == SQX:
            quest.SqX(q, a)
        elif k == SQY:
            quest.SqY(q, a)
        elif k == SQW:
            quest.SqW(q, a)
        elif k == SWAP:
            quest.swapGate(q, a, b)
        elif k == MEASURE:
            outcomes.append(int(quest.measure(q, a)))
        else:
            raise ValueError(f"unknown op kind {k}")
    return outcomes


def random_unitary(rng_np, dim):
    """Haar-ish random unitary via QR of a complex Gaussian matrix (numpy Generator)."""
    z = rng_np.standard_normal((dim, dim)) + 1j * rng_np.standard_normal((dim, dim))
    qm, r = np.linalg.qr(z)
    d = np.diag(r)
    return qm * (d / np.abs(d))


def mixed_ops(n, count, seed, kinds=None, with_measure=False):
    """A seeded mix of every single- and two-qubit API call (parity coverage)."""
    rng = Mt19937(seed)
    gen = np.random.default_rng(seed)
    b = OpList()
    all_kinds = [H, X, Y, Z, S, T, RX, RY, RZ, PHASE, CNOT, CZ, CPHASE, CRX, CRY, CRZ, COMPACT, CCOMPACT, UNITARY,
                 CUNITARY, SQX, SQY, SQW, SWAP, CY]
    if with_measure:
        all_kinds.append(MEASURE)
    kinds = kinds or all_kinds
    for _ in range(count):
        k = kinds[rng.below(len(kinds))]
        a = rng.below(n)
        c = rng.below(n - 1)
        if c >= a:
            c += 1
        ang = 2.0 * math.pi * rng.uniform() - math.pi
        if k in (COMPACT, CCOMPACT):
            u = random_unitary(gen, 2)
            ph = np.exp(-0.5j * np.angle(np.linalg.det(u)))
            u = u * ph  # SU(2): [[alpha, -conj(beta)], [beta, conj(alpha)]]
            alpha, beta = u[0, 0], u[1, 0]
            norm = math.sqrt(abs(alpha) ** 2 + abs(beta) ** 2)
            alpha, beta = alpha / norm, beta / norm
            b.add(k, a, c, p=(alpha.real, alpha.imag, beta.real, beta.imag))
        elif k in (UNITARY, CUNITARY):
            u = random_unitary(gen, 2)
            b.add(k, a, c, p=(u[0, 0].real, u[0, 0].imag, u[0, 1].real, u[0, 1].imag,
                              u[1, 0].real, u[1, 0].imag, u[1, 1].real, u[1, 1].imag))
        else:
            b.add(k, a, c, p=(ang,))
    return b.array()
