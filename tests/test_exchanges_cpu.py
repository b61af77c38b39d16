"""Qubit exchanges of the host tier and of sharded registers, planned on the
host (no GPU): how many exchange passes a circuit needs when its state is
cut into pages or shards of 2^local amplitudes.

The host tier moves one qubit per pass; a sharded register moves every qubit
of a segment boundary in one pass, bringing in the shard-index qubits that
are needed again before the shard qubits they replace (as dgQuEST's section
boundaries reorder several qubits at once)."""
import numpy as np
import pytest

from dgquest_b200 import circuits as C
from dgquest_b200 import ir


def hadamard_all(n):
    b = C.OpList()
    for q in range(n):
        b.add(C.H, q)
    return b.array()


def test_local_gates_need_no_exchange():
    n, local = 20, 16
    b = C.OpList()
    for q in range(local):
        b.add(C.RX, q, p=[0.3]).add(C.CNOT, q, (q + 1) % local)
    for q in range(local, n):  # diagonal gates and controls above the page stay where they are
        b.add(C.RZ, q, p=[0.2]).add(C.CZ, q, 0).add(C.CNOT, q, 1)
    for batch in (False, True):
        assert ir.plan_exchanges(b.array(), n, local, batch) == (1, 0, 0)


@pytest.mark.parametrize("n,local", [(20, 16), (18, 14), (24, 21)])
def test_one_pass_per_qubit_or_per_boundary(n, local):
    ops = hadamard_all(n)
    # host tier: one pass for each qubit above the page
    assert ir.plan_exchanges(ops, n, local, False) == (1 + n - local, n - local, n - local)
    # sharded: the first gate above the shard brings in all the others at once
    assert ir.plan_exchanges(ops, n, local, True) == (2, 1, n - local)


def test_batching_never_adds_passes_on_random_circuits():
    for seed in range(6):
        n = 20
        ops = C.random_layers(n, 12, C.config_seed(2, 800 + seed))
        for local in (15, 17, 19):
            seg0, ex0, moved0 = ir.plan_exchanges(ops, n, local, False)
            seg1, ex1, moved1 = ir.plan_exchanges(ops, n, local, True)
            assert ex0 == moved0 and seg0 <= ex0 + 1
            assert ex1 <= ex0
            assert ex1 <= moved1 <= ex1 * (n - local)
            assert seg1 == ex1 + 1


def test_benchmark_workload_exchange_counts():
    """The benchmark's cases: the 30-qubit depth-20 random circuit in 8
    shards takes 9 passes moving 23 qubits (18 passes one qubit at a time);
    the 28-qubit depth-8 circuit in the host tier's 2^25-amplitude pages
    takes 7."""
    ops = C.random_layers(30, 20, C.config_seed(2))
    assert ir.plan_exchanges(ops, 30, 27, True) == (10, 9, 23)
    assert ir.plan_exchanges(ops, 30, 27, False) == (19, 18, 18)
    ops = C.random_layers(28, 8, C.config_seed(2, 500))
    assert ir.plan_exchanges(ops, 28, 25, False) == (8, 7, 7)


def test_bad_arguments():
    from dgquest_b200 import quest as Q
    ops = hadamard_all(4)
    with pytest.raises(Q.QuESTError):
        ir.plan_exchanges(ops, 4, 5, True)
    with pytest.raises(Q.QuESTError):
        ir.plan_exchanges(ops, 4, 0, True)


def test_two_qubits_above_the_page_needed_one_after_the_other():
    """A controlled rotation whose target is above the page, then a rotation
    of its control (also above the page): the host tier moves each qubit in
    a pass of its own, a sharded register moves both in one."""
    n, local = 18, 16
    b = C.OpList()
    for q in range(local):
        b.add(C.H, q)
    b.add(C.CRX, n - 2, n - 1, p=(0.3,)).add(C.SWAP, 0, 1)  # only the target must be inside the page
    b.add(C.RX, n - 2, p=(0.2,))
    ops = b.array()
    seg0, ex0, moved0 = ir.plan_exchanges(ops, n, local, False)
    seg1, ex1, moved1 = ir.plan_exchanges(ops, n, local, True)
    assert (ex0, moved0) == (2, 2)
    assert (ex1, moved1) == (1, 2)


def test_sharded_register_arguments_checked_before_any_device_call():
    from dgquest_b200 import quest as Q
    env = Q.QuESTEnv()  # never used: the checks come first
    for n, sb in [(16, 0), (16, 5), (15, 2), (0, 1)]:
        with pytest.raises(Q.QuESTError):
            Q.create_sharded(n, env, sb)
