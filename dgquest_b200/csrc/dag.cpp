// dag.cpp -- see dag.h for the behaviour and its dgQuEST citations.
#include "dag.h"

#include <algorithm>
#include <cmath>

namespace dgq {

static const double kPiOn4 = 0.78539816339744830961566084581987572;
static const double kRsqrt2 = 0.7071067811865475244008443621;

void matMul2(const double a[8], const double b[8], double c[8]) {
    // element (r, k) lives at [4r + 2k] (re) and [4r + 2k + 1] (im)
    for (int r = 0; r < 2; r++) {
        for (int k = 0; k < 2; k++) {
            double re = 0.0, im = 0.0;
            for (int m = 0; m < 2; m++) {
                const double xr = a[4 * r + 2 * m], xi = a[4 * r + 2 * m + 1];
                const double yr = b[4 * m + 2 * k], yi = b[4 * m + 2 * k + 1];
                re += xr * yr - xi * yi;
                im += xr * yi + xi * yr;
            }
            c[4 * r + 2 * k] = re;
            c[4 * r + 2 * k + 1] = im;
        }
    }
}

void gateMatrix(const Gate &g, double m[8]) {
    for (int i = 0; i < 8; i++) m[i] = 0.0;
    const double a = g.op[0];
    switch (g.type) {
        case OP_ROTATE_Z:
            m[0] = std::cos(a); m[1] = -std::sin(a);
            m[6] = std::cos(a); m[7] = std::sin(a);
            break;
        case OP_PAULI_X: m[2] = 1.0; m[4] = 1.0; break;
        case OP_PAULI_Y: m[3] = -1.0; m[5] = 1.0; break;
        case OP_PAULI_Y_CONJ: m[3] = 1.0; m[5] = -1.0; break;
        case OP_HADAMARD: m[0] = kRsqrt2; m[2] = kRsqrt2; m[4] = kRsqrt2; m[6] = -kRsqrt2; break;
        case OP_ROTATE_X:
            m[0] = std::cos(a); m[3] = -std::sin(a);
            m[5] = -std::sin(a); m[6] = std::cos(a);
            break;
        case OP_ROTATE_Y:
            m[0] = std::cos(a); m[2] = -std::sin(a);
            m[4] = std::sin(a); m[6] = std::cos(a);
            break;
        case OP_COMPACT_UNITARY:  // [[alpha, -conj(beta)], [beta, conj(alpha)]]
            m[0] = g.op[0]; m[1] = g.op[1];
            m[2] = -g.op[2]; m[3] = g.op[3];
            m[4] = g.op[2]; m[5] = g.op[3];
            m[6] = g.op[0]; m[7] = -g.op[1];
            break;
        case OP_UNITARY:
            for (int i = 0; i < 8; i++) m[i] = g.op[i];
            break;
        default:
            break;
    }
}

GateDag::GateDag(int numQubits, bool mergeGates)
    : numQubits_(numQubits), merge_(mergeGates), qubitStack_((size_t) numQubits) {}

// Merge the new gate g into node `top` (identical masks, no successors).
// Returns true when g was absorbed (top updated or deleted).
bool GateDag::tryMerge(int top, const Gate &g) {
    Node &t = nodes_[(size_t) top];
    if (t.g.targetMask != g.targetMask || t.g.controlMask != g.controlMask) return false;
    // lower type first; on equal types the later gate (g) plays "first"
    const bool newIsHigher = g.type > t.g.type;
    const Gate &lo = newIsHigher ? t.g : g;
    const Gate &hi = newIsHigher ? g : t.g;
    auto removeTop = [&]() {
        unlinkDeleted(top);
        return true;
    };
    if ((int) hi.type < 8) {
        const int sum = ((int) lo.type + (int) hi.type) % 8;
        if (sum == 0) return removeTop();
        t.g.type = (GateType) sum;
        return true;
    }
    if (hi.type == OP_PHASE_SHIFT) {
        Gate merged = hi;
        merged.op[0] = hi.op[0] + (lo.type == OP_PHASE_SHIFT ? lo.op[0] : kPiOn4 * (int) lo.type);
        t.g = merged;
        return true;
    }
    if (hi.type == OP_UNITARY) {
        // time order: t (earlier) then g (later): result = later * earlier
        double mLater[8], mEarlier[8], prod[8];
        if (g.type == OP_UNITARY) {
            for (int i = 0; i < 8; i++) mLater[i] = g.op[i];
        } else {
            gateMatrix(g, mLater);
        }
        if (t.g.type == OP_UNITARY) {
            for (int i = 0; i < 8; i++) mEarlier[i] = t.g.op[i];
        } else {
            gateMatrix(t.g, mEarlier);
        }
        matMul2(mLater, mEarlier, prod);
        Gate merged = hi;
        merged.type = OP_UNITARY;
        for (int i = 0; i < 8; i++) merged.op[i] = prod[i];
        t.g = merged;
        return true;
    }
    if (lo.type == hi.type) {
        if (lo.type >= OP_PAULI_X && lo.type <= OP_HADAMARD) return removeTop();
        if (lo.type == OP_ROTATE_X || lo.type == OP_ROTATE_Y || lo.type == OP_ROTATE_Z) {
            if (lo.op[0] == -hi.op[0]) return removeTop();
            t.g.op[0] = lo.op[0] + hi.op[0];
            return true;
        }
    }
    return false;
}

void GateDag::unlinkDeleted(int idx) {
    flatValid_ = false;
    Node &d = nodes_[(size_t) idx];
    for (auto &st : qubitStack_) {
        if (!st.empty() && st.back() == idx) st.pop_back();
    }
    if (d.prev.empty()) {
        front_.erase(std::remove(front_.begin(), front_.end(), idx), front_.end());
    } else {
        for (int p : d.prev) {
            auto &nx = nodes_[(size_t) p].next;
            nx.erase(std::remove(nx.begin(), nx.end(), idx), nx.end());
        }
    }
    d.alive = false;
    d.prev.clear();
    d.next.clear();
    alive_--;
}

void GateDag::add(const Gate &g) {
    flatValid_ = false;
    const u64 barrier = g.targetMask | g.controlMask;
    const int idx = (int) nodes_.size();
    Node node;
    node.g = g;
    bool linked = false;
    for (int q = 0; q < numQubits_; q++) {
        if (!((barrier >> q) & 1ULL)) continue;
        auto &st = qubitStack_[(size_t) q];
        if (!st.empty()) {
            const int top = st.back();
            if (merge_ && !linked && nodes_[(size_t) top].next.empty() && tryMerge(top, g)) {
                // absorbed; the stacks pushed so far for this gate must be undone
                for (int q2 = 0; q2 < q; q2++) {
                    if (!((barrier >> q2) & 1ULL)) continue;
                    auto &s2 = qubitStack_[(size_t) q2];
                    if (!s2.empty() && s2.back() == idx) s2.pop_back();
                }
                for (int p : node.prev) {
                    auto &nx = nodes_[(size_t) p].next;
                    nx.erase(std::remove(nx.begin(), nx.end(), idx), nx.end());
                }
                return;
            }
            if (std::find(node.prev.begin(), node.prev.end(), top) == node.prev.end()) {
                node.prev.push_back(top);
                nodes_[(size_t) top].next.push_back(idx);
            }
            linked = true;
        }
        st.push_back(idx);
    }
    if (node.prev.empty()) front_.push_back(idx);
    nodes_.push_back(std::move(node));
    alive_++;
}

std::vector<Gate> GateDag::takeBlock(int budget, u64 &mask, size_t maxGates) {
    const size_t N = nodes_.size();
    std::vector<u64> cost(N, 0);
    std::vector<size_t> remain(N, 0);
    std::vector<char> visited(N, 0), selected(N, 0);
    for (size_t i = 0; i < N; i++) {
        if (!nodes_[i].alive) continue;
        cost[i] = isDiagonalType(nodes_[i].g.type) ? 0 : nodes_[i].g.targetMask;
        remain[i] = nodes_[i].prev.size();
    }
    // iterative depth-first walk: (node, next child position)
    std::vector<std::pair<int, size_t>> stack;
    auto enter = [&](int v) {
        visited[(size_t) v] = 1;
        if (popcount64(mask | cost[(size_t) v]) <= budget) {
            selected[(size_t) v] = 1;
            mask |= cost[(size_t) v];
            stack.emplace_back(v, 0);
        }
    };
    const std::vector<int> fronts = front_;
    for (int f : fronts) {
        if (visited[(size_t) f]) continue;
        enter(f);
        while (!stack.empty()) {
            auto &top = stack.back();
            const auto &nx = nodes_[(size_t) top.first].next;
            if (top.second >= nx.size()) {
                stack.pop_back();
                continue;
            }
            const int c = nx[top.second++];
            if (!visited[(size_t) c] && --remain[(size_t) c] == 0) enter(c);
        }
    }
    std::vector<Gate> taken, rest;
    for (size_t i = 0; i < N; i++) {
        if (!nodes_[i].alive) continue;
        if (selected[i] && taken.size() < maxGates)
            taken.push_back(nodes_[i].g);
        else
            rest.push_back(nodes_[i].g);
    }
    // rebuild the residual DAG (with merging, as a fresh DAG)
    nodes_.clear();
    flatValid_ = false;
    front_.clear();
    alive_ = 0;
    for (auto &st : qubitStack_) st.clear();
    for (const Gate &g : rest) add(g);
    return taken;
}

void GateDag::refreshFlat() const {
    if (flatValid_) return;
    flatTouch_.clear();
    flatCost_.clear();
    for (const Node &nd : nodes_) {
        if (!nd.alive) continue;
        const u64 touch = nd.g.targetMask | nd.g.controlMask;
        flatTouch_.push_back(touch);
        flatCost_.push_back(touchCost_ ? touch : isDiagonalType(nd.g.type) ? 0 : nd.g.targetMask);
    }
    flatValid_ = true;
}

// Insertion order is a topological order, so one forward pass decides
// which gates are reachable inside `allowed`: a gate held back holds back
// every later gate on its qubits.
size_t GateDag::countAllowed(u64 allowed) const {
    refreshFlat();
    const size_t n = flatTouch_.size();
    const u64 *touch = flatTouch_.data(), *cost = flatCost_.data();
    const u64 all = numQubits_ >= 64 ? ~0ULL : ((1ULL << numQubits_) - 1);
    u64 blocked = 0;
    size_t count = 0;
    for (size_t i = 0; i < n && blocked != all; i++) {
        if ((touch[i] & blocked) || (cost[i] & ~allowed)) {
            blocked |= touch[i];
            continue;
        }
        count++;
    }
    return count;
}

u64 GateDag::frontierTargets(u64 allowed) const {
    u64 frontier = 0;
    for (u64 m : frontierSets(allowed)) frontier |= m;
    return frontier;
}

std::vector<u64> GateDag::frontierSets(u64 allowed) const {
    refreshFlat();
    const size_t n = flatTouch_.size();
    const u64 *touch = flatTouch_.data(), *cost = flatCost_.data();
    const u64 all = numQubits_ >= 64 ? ~0ULL : ((1ULL << numQubits_) - 1);
    std::vector<u64> sets;
    u64 blocked = 0;
    for (size_t i = 0; i < n && blocked != all; i++) {
        if (touch[i] & blocked) {
            blocked |= touch[i];
            continue;
        }
        const u64 missing = cost[i] & ~allowed;
        if (missing) {
            if (std::find(sets.begin(), sets.end(), missing) == sets.end()) sets.push_back(missing);
            blocked |= touch[i];
        }
    }
    return sets;
}

std::vector<Gate> GateDag::takeAllowed(u64 allowed) {
    std::vector<char> ok(nodes_.size(), 0);
    std::vector<Gate> taken, rest;
    for (size_t i = 0; i < nodes_.size(); i++) {
        const Node &nd = nodes_[i];
        if (!nd.alive) continue;
        const u64 cost = touchCost_ ? (nd.g.targetMask | nd.g.controlMask)
                                    : isDiagonalType(nd.g.type) ? 0 : nd.g.targetMask;
        bool all = (cost & ~allowed) == 0;
        for (int p : nd.prev)
            if (all && !ok[(size_t) p]) all = false;
        if (all) {
            ok[i] = 1;
            taken.push_back(nd.g);
        } else {
            rest.push_back(nd.g);
        }
    }
    nodes_.clear();
    flatValid_ = false;
    front_.clear();
    alive_ = 0;
    for (auto &st : qubitStack_) st.clear();
    for (const Gate &g : rest) add(g);
    return taken;
}

std::vector<Gate> GateDag::gatesInOrder() const {
    std::vector<Gate> out;
    for (const auto &n : nodes_)
        if (n.alive) out.push_back(n.g);
    return out;
}

}  // namespace dgq
