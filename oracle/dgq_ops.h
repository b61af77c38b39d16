/*
 * dgq_ops.h -- the op-list record shared by the test infrastructure.
 *
 * TEST INFRASTRUCTURE ONLY. This header belongs to the oracle: it is used by
 * the CPU oracle (dgq_oracle.c) and by the harness that drives the reference
 * build (ref_harness.cpp). The product library never includes it.
 *
 * One record = one QuEST API call. The same op list drives every path:
 *   - the product, replayed call by call through the QuEST C API,
 *   - the CPU oracle (dgq_oracle.c), which applies each call's gate math,
 *   - the reference build (ref_harness.cpp), replayed through the
 *     reference's own QuEST API (include/QuEST.h of the reference).
 * The Python mirror of this record is dgquest_b200/circuits.py::OP_DTYPE.
 */
#ifndef DGQ_OPS_H
#define DGQ_OPS_H

#include <stdint.h>

enum dgq_op_kind {
    DGQ_OP_H = 0,        /* hadamard(q0)                                   */
    DGQ_OP_X = 1,        /* pauliX(q0)                                     */
    DGQ_OP_Y = 2,        /* pauliY(q0)                                     */
    DGQ_OP_Z = 3,        /* pauliZ(q0)                                     */
    DGQ_OP_S = 4,        /* sGate(q0)                                      */
    DGQ_OP_T = 5,        /* tGate(q0)                                      */
    DGQ_OP_RX = 6,       /* rotateX(q0, p0)                                */
    DGQ_OP_RY = 7,       /* rotateY(q0, p0)                                */
    DGQ_OP_RZ = 8,       /* rotateZ(q0, p0)                                */
    DGQ_OP_PHASE = 9,    /* phaseShift(q0, p0)                             */
    DGQ_OP_CNOT = 10,    /* controlledNot(q0 = control, q1 = target)       */
    DGQ_OP_CZ = 11,      /* controlledPhaseFlip(q0, q1)                    */
    DGQ_OP_CPHASE = 12,  /* controlledPhaseShift(q0, q1, p0)               */
    DGQ_OP_CRX = 13,     /* controlledRotateX(q0, q1, p0)                  */
    DGQ_OP_CRY = 14,     /* controlledRotateY(q0, q1, p0)                  */
    DGQ_OP_CRZ = 15,     /* controlledRotateZ(q0, q1, p0)                  */
    DGQ_OP_COMPACT = 16, /* compactUnitary(q0, alpha=(p0,p1), beta=(p2,p3)) */
    DGQ_OP_CCOMPACT = 17,/* controlledCompactUnitary(q0, q1, alpha, beta)  */
    DGQ_OP_UNITARY = 18, /* unitary(q0, u = p0..p7, row-major re/im)       */
    DGQ_OP_CUNITARY = 19,/* controlledUnitary(q0, q1, u)                   */
    DGQ_OP_SQX = 20,     /* SqX(q0)                                        */
    DGQ_OP_SQY = 21,     /* SqY(q0)                                        */
    DGQ_OP_SQW = 22,     /* SqW(q0)                                        */
    DGQ_OP_SWAP = 23,    /* swapGate(q0, q1)                               */
    DGQ_OP_MEASURE = 24, /* measure(q0)                                    */
    DGQ_OP_CY = 25,      /* controlledPauliY(q0, q1)                       */
    DGQ_OP_KIND_COUNT = 26
};

typedef struct dgq_op {
    int32_t kind;
    int32_t q0, q1, q2;
    double p[8];
} dgq_op;

#endif /* DGQ_OPS_H */
