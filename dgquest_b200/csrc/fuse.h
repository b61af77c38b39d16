// fuse.h -- the dense-block form: recorded gates fused into dense unitaries
// on K qubits, each applied as one dense sweep (a complex GEMM over the
// state: on the tensor cores for complex64 registers and K = 6, the SIMT
// dense kernel otherwise).
//
// Blocks are chosen with dgQuEST's greedy rule (DAG.cpp:219-259: take every
// gate whose qubits fit the budget, in dependency order), with a block's
// qubits being every qubit its gates touch (targets, controls and the
// qubits of diagonal gates), grown one runnable-next gate at a time by the
// addition that lets the most gates in. The block unitary is composed in
// FP64 on the host by applying each gate to the columns of the identity.
#pragma once

#include <vector>

#include "ir.h"
#include "planner.h"

namespace dgq {

// The gates as dense OP_MULTI_UNITARY gates on exactly K qubits (matrices
// appended to pool, row-major (re, im)); a gate that touches more than K
// qubits passes through unchanged, with the gates that the same greedy step
// takes beside it. *blocks (if given) counts the dense gates made.
// Requires 1 <= K <= 7 and K <= numBits.
// maxBlocks > 0 stops after that many blocks (the rest of the gates are
// dropped; *stopped, if given, is set): a cost estimate that only needs to
// know whether the form stays below a bound.
std::vector<Gate> fuseDenseBlocks(const std::vector<Gate> &gates, int numBits, int K, MatrixPool &pool,
                                  int *blocks = nullptr, int maxBlocks = 0, bool *stopped = nullptr);

// Applies one recorded gate to the 2^K-amplitude vectors v[c * 2^K ..] for
// c < numVectors, where local[b] is the vector index bit of address bit b
// (every qubit the gate touches must have one).
void applyGateLocal(const Gate &g, const MatrixPool &pool, const int local[64], int K, double *v, int numVectors);

}  // namespace dgq
