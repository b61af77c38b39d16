// ir.h -- gate IR recorded by the QuEST API and consumed by the planner.
//
// The numbering of GateType and the (type, targetMask, controlMask, operand)
// encoding follow dgQuEST's IR (src/cpp/QuEST_backend.h:89-114,160-178) on
// purpose: the peephole merge rules depend on it (phase powers 0..7 add
// mod 8, DAG.cpp:165-171), and diagonal gates (type < OP_PAULI_X) carry
// their qubits in controlMask with targetMask = 0, except Rz which keeps its
// target but still costs no tile qubit (DAG.cpp:224-228).
// Masks here are in VIRTUAL address bits (the logical->virtual relabelling
// done by swapGate is applied when a gate is recorded).
#pragma once

#include <cstdint>
#include <cstring>

namespace dgq {

typedef uint64_t u64;
typedef uint32_t u32;

enum GateType : int {
    // phase powers e^{i pi t/4} on amplitudes whose control bits are all 1
    OP_ONE = 0,
    OP_T_GATE = 1,
    OP_S_GATE = 2,
    OP_T_GATE_CONJ_NEG = 3,
    OP_PAULI_Z = 4,
    OP_T_GATE_NEG = 5,
    OP_S_GATE_CONJ = 6,
    OP_T_GATE_CONJ = 7,
    OP_PHASE_SHIFT = 8,   // e^{i angle} on control match
    OP_RESERVED_9 = 9,    // (kernel-only in dgQuEST; unused here)
    OP_ROTATE_Z = 10,     // diag(e^{-i a}, e^{+i a}) on target, a = angle/2 stored
    OP_PAULI_X = 11,
    OP_PAULI_Y = 12,
    OP_PAULI_Y_CONJ = 13,
    OP_HADAMARD = 14,
    OP_ROTATE_X = 15,
    OP_ROTATE_Y = 16,
    OP_COMPACT_UNITARY = 17,
    OP_UNITARY = 18,
    // extensions (no dgQuEST counterpart)
    OP_MULTI_UNITARY = 19,  // dense 2^k x 2^k on targetMask, matrix in a side pool
};

static inline bool isDiagonalType(int t) { return t < OP_PAULI_X; }

struct Gate {
    GateType type = OP_ONE;
    u64 targetMask = 0;
    u64 controlMask = 0;
    // operand: angle (rotations store angle/2; phase shifts store the angle),
    // compact (alpha.re, alpha.im, beta.re, beta.im), or a 2x2 matrix
    // row-major (r0c0.re, r0c0.im, r0c1.re, r0c1.im, r1c0..., r1c1...).
    double op[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int32_t multiIndex = -1;  // OP_MULTI_UNITARY: index into the matrix pool
    int32_t multiTargets[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // OP_MULTI_UNITARY target order
    int32_t numMultiTargets = 0;

    double angle() const { return op[0]; }
    void setAngle(double a) { op[0] = a; }
};

static inline int popcount64(u64 x) { return __builtin_popcountll(x); }

// 2x2 complex matrix of a non-diagonal gate type, row-major re/im pairs
// (the canonical matrices of dgQuEST getUnitaryMatrix, QuEST_backend.h:480-530).
void gateMatrix(const Gate &g, double m[8]);

}  // namespace dgq
