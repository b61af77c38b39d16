"""Independent dense numpy statevector simulator (test helper).

Textbook QuEST gate definitions (Rx(t) = exp(-i t X / 2) etc.), written
without reference to either dgQuEST's kernel formulas or this project's
kernels: a third opinion for the oracle on small registers.
"""
import math

import numpy as np

from dgquest_b200 import circuits as C

R2 = 1 / math.sqrt(2)
I2 = np.eye(2, dtype=complex)
MX = np.array([[0, 1], [1, 0]], dtype=complex)
MY = np.array([[0, -1j], [1j, 0]], dtype=complex)
MZ = np.diag([1, -1]).astype(complex)
MH = R2 * np.array([[1, 1], [1, -1]], dtype=complex)
MS = np.diag([1, 1j])
MT = np.diag([1, np.exp(1j * math.pi / 4)])
SQX = R2 * np.array([[1, -1j], [-1j, 1]])
SQY = R2 * np.array([[1, -1], [1, 1]], dtype=complex)
SQW = np.array([[R2, -0.5 - 0.5j], [0.5 - 0.5j, R2]])


def rx(t):
    return np.array([[math.cos(t / 2), -1j * math.sin(t / 2)], [-1j * math.sin(t / 2), math.cos(t / 2)]])


def ry(t):
    return np.array([[math.cos(t / 2), -math.sin(t / 2)], [math.sin(t / 2), math.cos(t / 2)]], dtype=complex)


def rz(t):
    return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])


def phase(t):
    return np.diag([1, np.exp(1j * t)])


def apply1(psi, n, t, u, controls=()):
    idx = np.arange(1 << n, dtype=np.int64)
    sel = ((idx >> t) & 1) == 0
    for c in controls:
        sel &= ((idx >> c) & 1) == 1
    i0 = idx[sel]
    i1 = i0 | (1 << t)
    a0, a1 = psi[i0].copy(), psi[i1].copy()
    psi[i0] = u[0, 0] * a0 + u[0, 1] * a1
    psi[i1] = u[1, 0] * a0 + u[1, 1] * a1


def apply_multi(psi, n, targs, u):
    k = len(targs)
    idx = np.arange(1 << n, dtype=np.int64)
    tmask = sum(1 << t for t in targs)
    base = idx[(idx & tmask) == 0]
    cols = []
    for m in range(1 << k):
        off = sum(((m >> j) & 1) << targs[j] for j in range(k))
        cols.append(base | off)
    V = np.stack([psi[c] for c in cols], axis=0)
    W = u @ V
    for m in range(1 << k):
        psi[cols[m]] = W[m]


def run(n, ops):
    psi = np.zeros(1 << n, dtype=complex)
    psi[0] = 1
    for rec in ops:
        k, a, b, p = int(rec["kind"]), int(rec["q0"]), int(rec["q1"]), rec["p"]
        if k == C.H: apply1(psi, n, a, MH)
        elif k == C.X: apply1(psi, n, a, MX)
        elif k == C.Y: apply1(psi, n, a, MY)
        elif k == C.Z: apply1(psi, n, a, MZ)
        elif k == C.S: apply1(psi, n, a, MS)
        elif k == C.T: apply1(psi, n, a, MT)
        elif k == C.RX: apply1(psi, n, a, rx(p[0]))
        elif k == C.RY: apply1(psi, n, a, ry(p[0]))
        elif k == C.RZ: apply1(psi, n, a, rz(p[0]))
        elif k == C.PHASE: apply1(psi, n, a, phase(p[0]))
        elif k == C.CNOT: apply1(psi, n, b, MX, (a,))
        elif k == C.CY: apply1(psi, n, b, MY, (a,))
        elif k == C.CZ: apply1(psi, n, b, MZ, (a,))
        elif k == C.CPHASE: apply1(psi, n, b, phase(p[0]), (a,))
        elif k == C.CRX: apply1(psi, n, b, rx(p[0]), (a,))
        elif k == C.CRY: apply1(psi, n, b, ry(p[0]), (a,))
        elif k == C.CRZ: apply1(psi, n, b, rz(p[0]), (a,))
        elif k in (C.COMPACT, C.CCOMPACT):
            al, be = complex(p[0], p[1]), complex(p[2], p[3])
            u = np.array([[al, -be.conjugate()], [be, al.conjugate()]])
            if k == C.COMPACT: apply1(psi, n, a, u)
            else: apply1(psi, n, b, u, (a,))
        elif k in (C.UNITARY, C.CUNITARY):
            u = np.array([[complex(p[0], p[1]), complex(p[2], p[3])], [complex(p[4], p[5]), complex(p[6], p[7])]])
            if k == C.UNITARY: apply1(psi, n, a, u)
            else: apply1(psi, n, b, u, (a,))
        elif k == C.SQX: apply1(psi, n, a, SQX)
        elif k == C.SQY: apply1(psi, n, a, SQY)
        elif k == C.SQW: apply1(psi, n, a, SQW)
        elif k == C.SWAP:
            idx = np.arange(1 << n, dtype=np.int64)
            sel = (((idx >> a) & 1) == 1) & (((idx >> b) & 1) == 0)
            i = idx[sel]
            j = (i & ~(1 << a)) | (1 << b)
            psi[i], psi[j] = psi[j].copy(), psi[i].copy()
        else:
            raise ValueError(k)
    return psi


def prob_zero_all(psi, n):
    idx = np.arange(len(psi), dtype=np.int64)
    p = np.abs(psi) ** 2
    return np.array([p[((idx >> q) & 1) == 0].sum() for q in range(n)])
