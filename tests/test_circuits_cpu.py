"""Workload generators: the vectorised ansatz equals its gate-by-gate
definition, and the batched workload has the stated size ranges."""
import math

import numpy as np

from dgquest_b200 import circuits as C


def hea_by_gate(n, depth, seed):
    rng = C.Mt19937(seed)
    b = C.OpList()
    for _ in range(depth):
        for q in range(n):
            b.add(C.RY, q, p=(2.0 * math.pi * rng.uniform(),))
            b.add(C.RZ, q, p=(2.0 * math.pi * rng.uniform(),))
        for q in range(n - 1):
            b.add(C.CNOT, q, q + 1)
    return b.array()


def test_hea_matches_gate_by_gate_definition():
    for n, d, s in [(10, 4, 5), (13, 7, C.config_seed(4, 3)), (22, 2, 99), (1, 3, 7)]:
        assert C.hea(n, d, s).tobytes() == hea_by_gate(n, d, s).tobytes()


def test_batch_workload_ranges():
    w = C.batch_workload(300)
    ns = np.array([n for n, _, _ in w])
    ds = np.array([d for _, d, _ in w])
    assert ns.min() >= 10 and ns.max() <= 22 and ds.min() >= 4 and ds.max() <= 32
    assert len(set(ns.tolist())) == 13
    n, d, ops = w[0]
    assert len(ops) == d * (3 * n - 1)
    assert np.array_equal(ops, C.hea(n, d, C.config_seed(4, 0)))
