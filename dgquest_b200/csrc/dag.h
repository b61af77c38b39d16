// dag.h -- dependency DAG over recorded gates, with peephole merging and the
// greedy "fits in a qubit budget" block selection.
//
// Behaviour follows dgQuEST's DAG (src/cpp/DAG.cpp):
//   * a gate depends on the latest gate touching any of its target/control
//     qubits (per-qubit barrier stacks, DAG.cpp:199-216);
//   * a new gate merges into the latest gate when both have identical
//     target and control masks and the latest gate has no successors
//     (DAG.cpp:155-195): phase powers add mod 8, phase shifts add angles,
//     2x2 unitaries multiply, self-inverse X/Y/Y*/H cancel, rotations add
//     angles or cancel;
//   * block selection visits the DAG depth-first from its front nodes and
//     takes every gate whose non-diagonal target union still fits the budget
//     (DAG.cpp:219-259); the rest becomes the residual DAG.
// The data structure is this project's own: nodes live in a vector in
// insertion order (a valid topological order), edges are index lists, and
// the depth-first walk is iterative.
#pragma once

#include <vector>

#include "ir.h"

namespace dgq {

class GateDag {
public:
    explicit GateDag(int numQubits, bool mergeGates = true);

    void add(const Gate &g);
    bool empty() const { return alive_ == 0; }
    size_t size() const { return alive_; }

    // Removes and returns (in dependency order) the greedy block whose
    // non-diagonal targets, OR-ed into `mask`, have at most `budget` bits;
    // at most maxGates gates are taken. `mask` returns the block's target
    // union (including the seed bits it came in with).
    std::vector<Gate> takeBlock(int budget, u64 &mask, size_t maxGates);

    std::vector<Gate> gatesInOrder() const;

    // Gates of the largest dependency-closed set whose non-diagonal targets
    // all lie in `allowed` (count only / remove and return them).
    size_t countAllowed(u64 allowed) const;
    std::vector<Gate> takeAllowed(u64 allowed);
    // Non-diagonal target bits of the gates that could run next if their
    // targets were allowed (frontier of the allowed-closed set).
    u64 frontierTargets(u64 allowed) const;
    // The distinct sets of missing target bits of those next gates.
    std::vector<u64> frontierSets(u64 allowed) const;
    // With touchCost, the queries above count every qubit a gate touches
    // (targets, controls, diagonal gates' qubits) instead of its
    // non-diagonal targets: the selection of gates that a dense unitary on
    // the allowed qubits can absorb.
    void setTouchCost(bool on) {
        touchCost_ = on;
        flatValid_ = false;
    }

private:
    // Alive nodes in insertion order as (touched qubits, non-diagonal
    // targets): a gate can run inside `allowed` exactly when its targets lie
    // in `allowed` and no earlier gate on one of its qubits was held back,
    // because its predecessors are the latest earlier gates on its qubits.
    // The scans below run over this flat copy, rebuilt after a change.
    void refreshFlat() const;
    mutable bool flatValid_ = false;
    bool touchCost_ = false;
    mutable std::vector<u64> flatTouch_, flatCost_;

    struct Node {
        Gate g;
        std::vector<int> prev;
        std::vector<int> next;
        bool alive = true;
    };
    bool tryMerge(int top, const Gate &g);
    void unlinkDeleted(int idx);

    int numQubits_;
    bool merge_;
    size_t alive_ = 0;
    std::vector<Node> nodes_;
    std::vector<std::vector<int>> qubitStack_;
    std::vector<int> front_;
};

// Product of two 2x2 complex matrices (row-major re/im): c = a * b.
void matMul2(const double a[8], const double b[8], double c[8]);

}  // namespace dgq
