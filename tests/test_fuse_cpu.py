"""CPU tests of the dense-block form's host side: gates fused into dense
K-qubit unitaries (composed in FP64) must give the oracle's state to 1e-12
per amplitude when applied, for every gate kind the API records, and gates
wider than K qubits must pass through unchanged."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C
from dgquest_b200 import ir

NO_SWAP = [C.H, C.X, C.Y, C.Z, C.S, C.T, C.RX, C.RY, C.RZ, C.PHASE, C.CNOT, C.CZ, C.CPHASE, C.CRX, C.CRY, C.CRZ,
           C.COMPACT, C.CCOMPACT, C.UNITARY, C.CUNITARY, C.SQX, C.SQY, C.SQW, C.CY]


def zero_state(n):
    a = np.zeros(1 << n, dtype=np.complex128)
    a[0] = 1.0
    return a


@pytest.mark.parametrize("k", [5, 6, 7])
@pytest.mark.parametrize("kind", ["random", "ghzqft", "grid", "mixed"])
def test_fused_blocks_match_oracle(k, kind):
    n = 10
    ops = {"random": lambda: C.random_layers(n, 10, C.config_seed(2, 50 + k)),
           "ghzqft": lambda: C.ghz_qft(n, swaps=False),
           "grid": lambda: C.grid_sqrt(2, 5, 8, C.config_seed(3, 50 + k)),
           "mixed": lambda: C.mixed_ops(n, 300, 60 + k, kinds=NO_SWAP)}[kind]()
    t, tm, cm, o = ir.ops_to_ir(ops, n)
    got, blocks = ir.fuse_apply_host(n, k, t, tm, cm, o, zero_state(n))
    ref = oracle.run(n, ops)[0]
    assert blocks >= 1
    assert np.abs(got - ref).max() <= 1e-12
    assert abs(np.vdot(got, got).real - 1.0) <= 1e-12


def _apply_ref(a, n, t, target, controls, op0):
    """numpy reference of the IR gates used below (H, X, Z phase flip, Rz)."""
    idx = np.arange(1 << n)
    cmask = sum(1 << c for c in controls)
    on = (idx & cmask) == cmask
    a = a.copy()
    if t == ir.OP_Z:
        a[on] *= -1
    elif t == ir.OP_RZ:
        bit = (idx >> target) & 1
        a[on] *= np.exp(1j * op0 * np.where(bit[on] == 1, 1.0, -1.0))
    elif t in (ir.OP_H, ir.OP_X):
        lo = on & (((idx >> target) & 1) == 0)
        i0 = idx[lo]
        i1 = i0 | (1 << target)
        x, y = a[i0].copy(), a[i1].copy()
        if t == ir.OP_H:
            s = 1 / np.sqrt(2)
            a[i0], a[i1] = s * (x + y), s * (x - y)
        else:
            a[i0], a[i1] = y, x
    return a


def test_gates_wider_than_the_block_pass_through():
    n, k = 10, 5
    gates = []  # (type, target, controls, operand)
    for q in range(n):
        gates.append((ir.OP_H, q, [], 0.0))
    gates.append((ir.OP_Z, 0, [0, 1, 2, 3, 4, 5, 6, 7], 0.0))   # phase flip on 8 qubits
    gates.append((ir.OP_RZ, 3, [1], 0.37))
    gates.append((ir.OP_X, 9, [0, 2, 4, 6, 8], 0.0))            # 5 controls + target = 6 qubits
    for q in range(0, n, 2):
        gates.append((ir.OP_H, q, [], 0.0))
    gates.append((ir.OP_RZ, 8, [], -1.1))
    t = np.array([g[0] for g in gates], dtype=np.int32)
    tm = np.array([0 if g[0] == ir.OP_Z else 1 << g[1] for g in gates], dtype=np.uint64)
    cm = np.array([sum(1 << c for c in g[2]) for g in gates], dtype=np.uint64)
    o = np.zeros((len(gates), 8))
    o[:, 0] = [g[3] for g in gates]
    ref = zero_state(n)
    for g in gates:
        ref = _apply_ref(ref, n, g[0], g[1], g[2], g[3])
    got, blocks = ir.fuse_apply_host(n, k, t, tm, cm, o, zero_state(n))
    assert blocks >= 2
    assert np.abs(got - ref).max() <= 1e-12
