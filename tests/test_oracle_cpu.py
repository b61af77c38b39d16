"""CPU tests: the oracle against an independent dense numpy simulator, the
MT19937 known answers, the measurement rule, and the seeded generators."""
import math

import numpy as np
import pytest

import dense_ref
import oracle
from dgquest_b200 import circuits as C


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6, 9])
def test_oracle_matches_dense_numpy(n):
    if n == 1:
        ops = (C.OpList().add(C.H, 0).add(C.RX, 0, p=(0.3,)).add(C.T, 0).add(C.SQW, 0).add(C.RZ, 0, p=(1.1,))
               .add(C.S, 0).add(C.SQX, 0).add(C.PHASE, 0, p=(-0.7,)).add(C.Y, 0).add(C.SQY, 0).array())
    else:
        ops = C.mixed_ops(n, 300, 100 + n)
    a, p0, _ = oracle.run(n, ops)
    b = dense_ref.run(n, ops)
    assert np.abs(a - b).max() <= 1e-13
    assert np.abs(p0 - dense_ref.prob_zero_all(b, n)).max() <= 1e-13
    assert abs(np.vdot(a, a).real - 1) <= 1e-13


def test_oracle_multi_qubit_unitary_matches_dense():
    n = 6
    gen = np.random.default_rng(3)
    ops = C.mixed_ops(n, 40, 9)
    for targs in ([2, 0], [5, 1, 3], [0, 4, 2, 1]):
        u = C.random_unitary(gen, 1 << len(targs))
        o = oracle.Oracle(n)
        o.apply(ops)
        o.multi_qubit_unitary(targs, u)
        psi = dense_ref.run(n, ops)
        dense_ref.apply_multi(psi, n, targs, u)
        assert np.abs(o.amps() - psi).max() <= 1e-13


def test_mt19937_known_answers():
    # published reference outputs of mt19937ar (Matsumoto & Nishimura):
    # init_genrand(5489) starts 3499211612; init_by_array({0x123, 0x234,
    # 0x345, 0x456}) starts 1067595299 955945823 477289528 4107218783 4228976476
    assert oracle.mt_outputs_by_seed(5489, 1) == [3499211612]
    assert oracle.mt_outputs_by_array([0x123, 0x234, 0x345, 0x456], 5) == [
        1067595299, 955945823, 477289528, 4107218783, 4228976476]
    py = C.Mt19937(5489)
    assert [py.u32() for _ in range(3)] == oracle.mt_outputs_by_seed(5489, 3)


def test_measurement_rule_and_collapse():
    # outcome = real1() > P0 (src/QuEST_common.c:97-115); P0 within REAL_EPS of 0 or 1 draws nothing
    n = 5
    o = oracle.Oracle(n)
    o.seed([12345, 67890])
    o.apply(C.OpList().add(C.H, 0).add(C.RY, 1, p=(1.0,)).add(C.X, 2).array())
    draws = oracle.mt_outputs_by_array([12345, 67890], 2)
    u0 = draws[0] / 4294967295.0
    p0 = math.cos(0.5) ** 2
    out1, prob1 = o.measure(1)
    assert out1 == int(u0 > p0)
    assert prob1 == pytest.approx(p0 if out1 == 0 else 1 - p0, abs=1e-14)
    out2, prob2 = o.measure(2)  # deterministic: |1>, no draw consumed
    assert (out2, prob2) == (1, pytest.approx(1.0, abs=1e-14))
    u1 = draws[1] / 4294967295.0
    out0, _ = o.measure(0)
    assert out0 == int(u1 > 0.5)
    assert abs(o.total_prob() - 1) <= 1e-13


def test_bv_oracle_recovers_secret():
    n = 10
    ops = C.bernstein_vazirani(n, 42, measure=True)
    _, _, out = oracle.run(n, ops, seed_keys=[1, 2])
    assert out[:n - 1] == C.bv_secret(n, 42)
    assert out[n - 1] == 1


def test_generators_are_deterministic_and_shaped():
    a = C.random_layers(30, 20, C.config_seed(2))
    b = C.random_layers(30, 20, C.config_seed(2))
    assert np.array_equal(a, b)
    assert len(a) == 20 * (30 + 15)
    assert set(np.unique(a["kind"])) <= {C.RX, C.RY, C.RZ, C.CZ}
    g = C.ghz_qft(20)
    assert len(g) == 1 + 19 + 20 + 190 + 10
    s = C.grid_sqrt(4, 8, 16, C.config_seed(3))
    kinds = s["kind"]
    assert set(np.unique(kinds)) == {C.SQX, C.SQY, C.SQW, C.CZ}
    # never the same square-root gate twice in a row on a qubit
    last = {}
    for r in s:
        if r["kind"] == C.CZ:
            continue
        assert last.get(int(r["q0"])) != int(r["kind"])
        last[int(r["q0"])] = int(r["kind"])
    h = C.hea(10, 3, 1)
    assert len(h) == 3 * (20 + 9)
