"""Op list -> dgQuEST gate IR, for the host-only planner entry point.

Mirrors the encoding the C API applies when a gate is recorded
(src/cpp/QuEST_distributed.cpp:118-364): rotations carry angle/2, diagonal
gates carry their qubits in the control mask, controlledNot is Pauli-X with
a control, swapGate relabels logical qubits.
"""
import ctypes
import math

import numpy as np

from . import circuits as C

OP_ONE, OP_T, OP_S, OP_Z = 0, 1, 2, 4
OP_PHASE, OP_RZ, OP_X, OP_Y, OP_H, OP_RX, OP_RY, OP_COMPACT, OP_UNITARY = 8, 10, 11, 12, 14, 15, 16, 17, 18

R = 1 / math.sqrt(2)
SQ = {C.SQX: (R, 0, 0, -R, 0, -R, R, 0), C.SQY: (R, 0, -R, 0, R, 0, R, 0), C.SQW: (R, 0, -0.5, -0.5, 0.5, -0.5, R, 0)}


def ops_to_ir(ops, n):
    l2v = list(range(n))
    types, tm, cm, opnd = [], [], [], []

    def add(t, targets, controls, operand=()):
        types.append(t)
        tm.append(sum(1 << l2v[x] for x in targets))
        cm.append(sum(1 << l2v[x] for x in controls))
        o = [0.0] * 8
        for i, v in enumerate(operand):
            o[i] = float(v)
        opnd.append(o)

    for r in ops:
        k, a, b, p = int(r["kind"]), int(r["q0"]), int(r["q1"]), r["p"]
        if k == C.H: add(OP_H, [a], [])
        elif k == C.X: add(OP_X, [a], [])
        elif k == C.Y: add(OP_Y, [a], [])
        elif k == C.Z: add(OP_Z, [], [a])
        elif k == C.S: add(OP_S, [], [a])
        elif k == C.T: add(OP_T, [], [a])
        elif k == C.RX: add(OP_RX, [a], [], [p[0] * 0.5])
        elif k == C.RY: add(OP_RY, [a], [], [p[0] * 0.5])
        elif k == C.RZ: add(OP_RZ, [a], [], [p[0] * 0.5])
        elif k == C.PHASE: add(OP_PHASE, [], [a], [p[0]])
        elif k == C.CNOT: add(OP_X, [b], [a])
        elif k == C.CY: add(OP_Y, [b], [a])
        elif k == C.CZ: add(OP_Z, [], [a, b])
        elif k == C.CPHASE: add(OP_PHASE, [], [a, b], [p[0]])
        elif k == C.CRX: add(OP_RX, [b], [a], [p[0] * 0.5])
        elif k == C.CRY: add(OP_RY, [b], [a], [p[0] * 0.5])
        elif k == C.CRZ: add(OP_RZ, [b], [a], [p[0] * 0.5])
        elif k == C.COMPACT: add(OP_COMPACT, [a], [], p[:4])
        elif k == C.CCOMPACT: add(OP_COMPACT, [b], [a], p[:4])
        elif k == C.UNITARY: add(OP_UNITARY, [a], [], p)
        elif k == C.CUNITARY: add(OP_UNITARY, [b], [a], p)
        elif k in SQ: add(OP_UNITARY, [a], [], SQ[k])
        elif k == C.SWAP: l2v[a], l2v[b] = l2v[b], l2v[a]
        elif k == C.MEASURE: raise ValueError("measure has no gate encoding")
        else: raise ValueError(k)
    return (np.array(types, dtype=np.int32), np.array(tm, dtype=np.uint64), np.array(cm, dtype=np.uint64),
            np.array(opnd, dtype=np.float64).reshape(-1, 8))


def fuse_apply_host(n, k, types, tm, cm, opnd, amps):
    """The dense-block form on the host: gates (IR arrays) fused into blocks
    of k qubits and applied in FP64 to amps (length 2^n); returns (new amps,
    number of blocks)."""
    from .quest import _check, _library
    P = ctypes.POINTER
    re = np.ascontiguousarray(amps.real, dtype=np.float64).copy()
    im = np.ascontiguousarray(amps.imag, dtype=np.float64).copy()
    t = np.ascontiguousarray(types, dtype=np.int32)
    tm = np.ascontiguousarray(tm, dtype=np.uint64)
    cm = np.ascontiguousarray(cm, dtype=np.uint64)
    o = np.ascontiguousarray(opnd, dtype=np.float64).reshape(-1, 8)
    nb = _library().dgq_fuseApplyHost(n, k, len(t), t.ctypes.data_as(P(ctypes.c_int32)),
                                      tm.ctypes.data_as(P(ctypes.c_uint64)), cm.ctypes.data_as(P(ctypes.c_uint64)),
                                      o.ctypes.data_as(P(ctypes.c_double)), re.ctypes.data_as(P(ctypes.c_double)),
                                      im.ctypes.data_as(P(ctypes.c_double)))
    _check()
    return re + 1j * im, nb


def plan_exchanges(ops, n, local_qubits, batch):
    """Host-only: (segments, exchange passes, qubits moved) of an op list on
    a register whose pages (batch=False, host tier) or shards (batch=True)
    hold 2^local_qubits amplitudes (no GPU needed)."""
    from .quest import _check, _library
    fn = _library().dgq_planExchanges
    P = ctypes.POINTER
    t, tm, _, _ = ops_to_ir(ops, n)
    seg, ex, moved = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
    fn(n, local_qubits, 1 if batch else 0, len(t), t.ctypes.data_as(P(ctypes.c_int32)),
       tm.ctypes.data_as(P(ctypes.c_uint64)), ctypes.byref(seg), ctypes.byref(ex), ctypes.byref(moved))
    _check()
    return seg.value, ex.value, moved.value


def plan(ops, n, tile_bits=0, want_merged=False):
    """Host-only plan statistics of an op list (no GPU needed)."""
    from .quest import PlanStats, _check, _library
    fn = _library().dgq_planGates
    P = ctypes.POINTER
    t, tm, cm, o = ops_to_ir(ops, n)
    st = PlanStats()
    merged = np.zeros(max(1, len(t)), dtype=np.int32)
    nm = ctypes.c_int32(0)
    fn(n, tile_bits, len(t), t.ctypes.data_as(P(ctypes.c_int32)), tm.ctypes.data_as(P(ctypes.c_uint64)),
       cm.ctypes.data_as(P(ctypes.c_uint64)), o.ctypes.data_as(P(ctypes.c_double)), ctypes.byref(st),
       merged.ctypes.data_as(P(ctypes.c_int32)) if want_merged else None, ctypes.byref(nm))
    _check()
    if want_merged:
        return st, merged[:nm.value].tolist()
    return st


def specialise(ops, n, precision, background=True):
    """Compiles ahead of time the specialised sweep kernels a register of n
    qubits (precision 1 complex64, 2 complex128) would use for the op list
    after initZeroState; returns the number of kernels."""
    from .quest import _check, _library
    P = ctypes.POINTER
    t, tm, cm, o = ops_to_ir(ops, n)
    r = _library().dgq_specialiseGates(n, precision, len(t), t.ctypes.data_as(P(ctypes.c_int32)),
                                       tm.ctypes.data_as(P(ctypes.c_uint64)), cm.ctypes.data_as(P(ctypes.c_uint64)),
                                       o.ctypes.data_as(P(ctypes.c_double)), 1 if background else 0)
    _check()
    return r
