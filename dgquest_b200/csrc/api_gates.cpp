// api_gates.cpp -- the gate calls of the QuEST C API (src/QuEST.c:30-458
// and src/cpp/QuEST_distributed.cpp:118-364): validation, then one recorded
// Gate in dgQuEST's IR encoding per call (rotations carry angle / 2,
// diagonal gates their qubits in the control mask).
#include "api_internal.h"

using dgq::Gate;

extern "C" {
// ---------------------------------------------------------------- gates
// Encodings: src/cpp/QuEST_distributed.cpp:118-364 (rotations store angle/2).
void hadamard(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_HADAMARD, bit(t), 0, nullptr, 0);
}
void pauliX(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_PAULI_X, bit(t), 0, nullptr, 0);
}
void pauliY(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_PAULI_Y, bit(t), 0, nullptr, 0);
}
void pauliZ(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_PAULI_Z, 0, bit(t), nullptr, 0);
}
void sGate(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_S_GATE, 0, bit(t), nullptr, 0);
}
void tGate(Qureg q, const int t) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_T_GATE, 0, bit(t), nullptr, 0);
}
void phaseShift(Qureg q, const int t, qreal angle) {
    if (!vTarget(q, t, __func__)) return;
    record(q, dgq::OP_PHASE_SHIFT, 0, bit(t), &angle, 1);
}
void rotateX(Qureg q, const int t, qreal angle) {
    if (!vTarget(q, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_X, bit(t), 0, &a, 1);
}
void rotateY(Qureg q, const int t, qreal angle) {
    if (!vTarget(q, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_Y, bit(t), 0, &a, 1);
}
void rotateZ(Qureg q, const int t, qreal angle) {
    if (!vTarget(q, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_Z, bit(t), 0, &a, 1);
}
void controlledRotateX(Qureg q, const int c, const int t, qreal angle) {
    if (!vControlTarget(q, c, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_X, bit(t), bit(c), &a, 1);
}
void controlledRotateY(Qureg q, const int c, const int t, qreal angle) {
    if (!vControlTarget(q, c, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_Y, bit(t), bit(c), &a, 1);
}
void controlledRotateZ(Qureg q, const int c, const int t, qreal angle) {
    if (!vControlTarget(q, c, t, __func__)) return;
    const double a = angle * 0.5;
    record(q, dgq::OP_ROTATE_Z, bit(t), bit(c), &a, 1);
}
// src/QuEST_common.c:56-63 and :154-183
static void pairFromRotation(qreal angle, Vector axis, Complex *alpha, Complex *beta) {
    const double mag = std::sqrt(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
    const double ux = axis.x / mag, uy = axis.y / mag, uz = axis.z / mag;
    alpha->real = std::cos(angle / 2.0);
    alpha->imag = -std::sin(angle / 2.0) * uz;
    beta->real = std::sin(angle / 2.0) * uy;
    beta->imag = -std::sin(angle / 2.0) * ux;
}
void rotateAroundAxis(Qureg q, const int t, qreal angle, Vector axis) {
    if (!vTarget(q, t, __func__)) return;
    if (axis.x == 0 && axis.y == 0 && axis.z == 0) {
        raise(E_ZERO_VECTOR, __func__);
        return;
    }
    Complex a, b;
    pairFromRotation(angle, axis, &a, &b);
    const double op[4] = {a.real, a.imag, b.real, b.imag};
    record(q, dgq::OP_COMPACT_UNITARY, bit(t), 0, op, 4);
}
void controlledRotateAroundAxis(Qureg q, const int c, const int t, qreal angle, Vector axis) {
    if (!vControlTarget(q, c, t, __func__)) return;
    if (axis.x == 0 && axis.y == 0 && axis.z == 0) {
        raise(E_ZERO_VECTOR, __func__);
        return;
    }
    Complex a, b;
    pairFromRotation(angle, axis, &a, &b);
    const double op[4] = {a.real, a.imag, b.real, b.imag};
    record(q, dgq::OP_COMPACT_UNITARY, bit(t), bit(c), op, 4);
}
void compactUnitary(Qureg q, const int t, Complex alpha, Complex beta) {
    if (!vTarget(q, t, __func__)) return;
    if (!isPairUnitary(alpha, beta)) {
        raise(E_NON_UNITARY_COMPLEX_PAIR, __func__);
        return;
    }
    const double op[4] = {alpha.real, alpha.imag, beta.real, beta.imag};
    record(q, dgq::OP_COMPACT_UNITARY, bit(t), 0, op, 4);
}
void controlledCompactUnitary(Qureg q, const int c, const int t, Complex alpha, Complex beta) {
    if (!vControlTarget(q, c, t, __func__)) return;
    if (!isPairUnitary(alpha, beta)) {
        raise(E_NON_UNITARY_COMPLEX_PAIR, __func__);
        return;
    }
    const double op[4] = {alpha.real, alpha.imag, beta.real, beta.imag};
    record(q, dgq::OP_COMPACT_UNITARY, bit(t), bit(c), op, 4);
}
void unitary(Qureg q, const int t, ComplexMatrix2 u) {
    if (!vTarget(q, t, __func__)) return;
    if (!isMatrix2Unitary(u)) {
        raise(E_NON_UNITARY_MATRIX, __func__);
        return;
    }
    recordMatrix(q, bit(t), 0, u);
}
void controlledUnitary(Qureg q, const int c, const int t, ComplexMatrix2 u) {
    if (!vControlTarget(q, c, t, __func__)) return;
    if (!isMatrix2Unitary(u)) {
        raise(E_NON_UNITARY_MATRIX, __func__);
        return;
    }
    recordMatrix(q, bit(t), bit(c), u);
}
void multiControlledUnitary(Qureg q, int *cs, const int nc, const int t, ComplexMatrix2 u) {
    if (!vTarget(q, t, __func__) || !vMultiControls(q, cs, nc, __func__)) return;
    u64 cm = 0;
    for (int i = 0; i < nc; i++) {
        if (cs[i] == t) {
            raise(E_TARGET_IN_CONTROLS, __func__);
            return;
        }
        cm |= bit(cs[i]);
    }
    if (!isMatrix2Unitary(u)) {
        raise(E_NON_UNITARY_MATRIX, __func__);
        return;
    }
    recordMatrix(q, bit(t), cm, u);
}
void controlledNot(Qureg q, const int c, const int t) {
    if (!vControlTarget(q, c, t, __func__)) return;
    record(q, dgq::OP_PAULI_X, bit(t), bit(c), nullptr, 0);
}
void controlledPauliY(Qureg q, const int c, const int t) {
    if (!vControlTarget(q, c, t, __func__)) return;
    record(q, dgq::OP_PAULI_Y, bit(t), bit(c), nullptr, 0);
}
void controlledPhaseFlip(Qureg q, const int a, const int b) {
    if (!vControlTarget(q, a, b, __func__)) return;
    record(q, dgq::OP_PAULI_Z, 0, bit(a) | bit(b), nullptr, 0);
}
void multiControlledPhaseFlip(Qureg q, int *cs, int nc) {
    if (!vMultiControls(q, cs, nc, __func__)) return;
    u64 cm = 0;
    for (int i = 0; i < nc; i++) cm |= bit(cs[i]);
    record(q, dgq::OP_PAULI_Z, 0, cm, nullptr, 0);
}
void controlledPhaseShift(Qureg q, const int a, const int b, qreal angle) {
    if (!vControlTarget(q, a, b, __func__)) return;
    record(q, dgq::OP_PHASE_SHIFT, 0, bit(a) | bit(b), &angle, 1);
}
void multiControlledPhaseShift(Qureg q, int *cs, int nc, qreal angle) {
    if (!vMultiControls(q, cs, nc, __func__)) return;
    u64 cm = 0;
    for (int i = 0; i < nc; i++) cm |= bit(cs[i]);
    record(q, dgq::OP_PHASE_SHIFT, 0, cm, &angle, 1);
}
void swapGate(Qureg q, int a, int b) {
    if (!vUniqueTargets(q, a, b, __func__)) return;
    // relabel logical qubits instead of moving amplitudes: later gates and
    // read-outs translate through l2v
    QuregState &s = *stateOf(q);
    for (int k = 0; k < (s.densityQubits ? 2 : 1); k++) {
        // density registers: the row qubits and the column qubits
        const int x = a + k * s.densityQubits, y = b + k * s.densityQubits;
        std::swap(s.l2v[x], s.l2v[y]);
        s.v2l[s.l2v[x]] = x;
        s.v2l[s.l2v[y]] = y;
    }
}
// src/QuEST.c:320-416 (u1/u2/u3 and the square-root gates are 2x2 unitaries)
void u1Gate(Qureg q, int t, qreal lambda) {
    ComplexMatrix2 u{{1.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {std::cos(lambda), std::sin(lambda)}};
    unitary(q, t, u);
}
void u2Gate(Qureg q, int t, qreal phi, qreal lambda) {
    const double r = 1 / std::sqrt(2);
    ComplexMatrix2 u{{r, 0.0},
                     {-std::cos(lambda) * r, -std::sin(lambda) * r},
                     {std::cos(phi) * r, std::sin(phi) * r},
                     {std::cos(phi + lambda) * r, std::sin(phi + lambda) * r}};
    unitary(q, t, u);
}
void u3Gate(Qureg q, int t, qreal theta, qreal phi, qreal lambda) {
    const double ct = std::cos(theta / 2), st = std::sin(theta / 2);
    ComplexMatrix2 u{{ct, 0.0},
                     {-std::cos(lambda) * st, -std::sin(lambda) * st},
                     {std::cos(phi) * st, std::sin(phi) * st},
                     {std::cos(phi + lambda) * ct, std::sin(phi + lambda) * ct}};
    unitary(q, t, u);
}
void SqX(Qureg q, int t) {
    const double r = 1 / std::sqrt(2);
    ComplexMatrix2 u{{r, 0.0}, {0.0, -r}, {0.0, -r}, {r, 0.0}};
    unitary(q, t, u);
}
void SqY(Qureg q, int t) {
    const double r = 1 / std::sqrt(2);
    ComplexMatrix2 u{{r, 0.0}, {-r, 0.0}, {r, 0.0}, {r, 0.0}};
    unitary(q, t, u);
}
void SqW(Qureg q, int t) {
    const double r = 1 / std::sqrt(2);
    ComplexMatrix2 u{{r, 0.0}, {-0.5, -0.5}, {0.5, -0.5}, {r, 0.0}};
    unitary(q, t, u);
}
void fSim(Qureg q, int t1, int t2, qreal theta, qreal phi) {
    controlledPhaseShift(q, t1, t2, -phi);
    controlledNot(q, t1, t2);
    controlledRotateX(q, t2, t1, theta * 2);
    controlledNot(q, t1, t2);
}

ComplexMatrixN createComplexMatrixN(int numQubits) {
    ComplexMatrixN m;
    m.numQubits = numQubits;
    m.real = nullptr;
    m.imag = nullptr;
    if (numQubits < 1 || numQubits > 12) {
        raise(E_INVALID_NUM_TARGETS, __func__);
        return m;
    }
    const int d = 1 << numQubits;
    m.real = (qreal **) malloc(sizeof(qreal *) * (size_t) d);
    m.imag = (qreal **) malloc(sizeof(qreal *) * (size_t) d);
    for (int r = 0; r < d; r++) {
        m.real[r] = (qreal *) calloc((size_t) d, sizeof(qreal));
        m.imag[r] = (qreal *) calloc((size_t) d, sizeof(qreal));
    }
    return m;
}

void destroyComplexMatrixN(ComplexMatrixN m) {
    if (!m.real) return;
    const int d = 1 << m.numQubits;
    for (int r = 0; r < d; r++) {
        free(m.real[r]);
        free(m.imag[r]);
    }
    free(m.real);
    free(m.imag);
}

void multiQubitUnitary(Qureg q, int *targs, int numTargs, ComplexMatrixN u) {
    if (!vQureg(q, __func__)) return;
    if (!targs || numTargs < 1 || numTargs > (int) q.numQubitsRepresented || u.numQubits != numTargs || !u.real ||
        !u.imag) {
        raise(E_INVALID_NUM_TARGETS, __func__);
        return;
    }
    u64 tm = 0;
    for (int i = 0; i < numTargs; i++) {
        if (targs[i] < 0 || targs[i] >= (int) q.numQubitsRepresented) {
            raise(E_INVALID_TARGET_QUBIT, __func__);
            return;
        }
        if (tm & bit(targs[i])) {
            raise(E_INVALID_NUM_TARGETS, __func__);
            return;
        }
        tm |= bit(targs[i]);
    }
    const int d = 1 << numTargs;
    // unitarity: U^dagger U = 1 within the tolerance QuEST uses for 2x2
    for (int r = 0; r < d; r++) {
        for (int c = 0; c < d; c++) {
            double re = 0.0, im = 0.0;
            for (int k = 0; k < d; k++) {
                re += u.real[k][r] * u.real[k][c] + u.imag[k][r] * u.imag[k][c];
                im += u.real[k][r] * u.imag[k][c] - u.imag[k][r] * u.real[k][c];
            }
            if (std::fabs(re - (r == c ? 1.0 : 0.0)) > 1e3 * REAL_EPS || std::fabs(im) > 1e3 * REAL_EPS) {
                raise(E_NON_UNITARY_MATRIX, __func__);
                return;
            }
        }
    }
    if (numTargs == 1) {
        ComplexMatrix2 m2{{u.real[0][0], u.imag[0][0]},
                          {u.real[0][1], u.imag[0][1]},
                          {u.real[1][0], u.imag[1][0]},
                          {u.real[1][1], u.imag[1][1]}};
        recordMatrix(q, tm, 0, m2);
        return;
    }
    if (numTargs > dgq::kMaxDenseTargets) {
        raise(E_UNSUPPORTED, __func__, "multiQubitUnitary supports at most 7 targets");
        return;
    }
    QuregState &s = *stateOf(q);
    std::vector<double> m((size_t) 2 * d * d);
    for (int r = 0; r < d; r++)
        for (int c = 0; c < d; c++) {
            m[(size_t) 2 * (r * d + c)] = u.real[r][c];
            m[(size_t) 2 * (r * d + c) + 1] = u.imag[r][c];
        }
    for (int k = 0; k < (s.densityQubits ? 2 : 1); k++) {
        // density registers: conj(U) on the column qubits as well
        const int shift = k * s.densityQubits;
        Gate g;
        g.type = dgq::OP_MULTI_UNITARY;
        g.targetMask = toVirtualMask(s, tm << shift);
        g.controlMask = 0;
        g.numMultiTargets = numTargs;
        for (int i = 0; i < numTargs; i++) g.multiTargets[i] = s.l2v[targs[i] + shift];
        g.multiIndex = (int32_t) s.pool.mats.size();
        std::vector<double> mk = m;
        if (k == 1)
            for (size_t i = 1; i < mk.size(); i += 2) mk[i] = -mk[i];
        s.pool.mats.push_back(std::move(mk));
        s.pending.push_back(g);
    }
    s.probsValid = false;
}

}  // extern "C"
