// fuse.cpp -- see fuse.h.
#include "fuse.h"

#include <cmath>
#include <cstring>

#include "dag.h"

namespace dgq {

namespace {

constexpr double kPiOn4 = 0.78539816339744830961566084581987572;

uint32_t localMask(u64 m, const int local[64]) {
    uint32_t r = 0;
    for (int b = 0; b < 64 && m; b++) {
        if (!((m >> b) & 1ULL)) continue;
        m &= ~(1ULL << b);
        r |= 1u << local[b];
    }
    return r;
}

// v[i] *= (cr + i ci) where (i & ctrl) == ctrl (and, with sel, (i & sel) selects)
void phaseWhere(double *v, int D, uint32_t ctrl, double cr, double ci) {
    for (int i = 0; i < D; i++) {
        if ((uint32_t) (i & ctrl) != ctrl) continue;
        const double re = v[2 * i], im = v[2 * i + 1];
        v[2 * i] = re * cr - im * ci;
        v[2 * i + 1] = re * ci + im * cr;
    }
}

}  // namespace

void applyGateLocal(const Gate &g, const MatrixPool &pool, const int local[64], int K, double *v, int numVectors) {
    const int D = 1 << K;
    const uint32_t ctrl = localMask(g.controlMask, local);
    for (int c = 0; c < numVectors; c++) {
        double *x = v + (size_t) 2 * D * c;
        if (g.type < OP_PHASE_SHIFT) {
            // e^{i pi t / 4} where every control bit is 1
            const double a = kPiOn4 * (int) g.type;
            if (g.type != OP_ONE) phaseWhere(x, D, ctrl, std::cos(a), std::sin(a));
        } else if (g.type == OP_PHASE_SHIFT) {
            phaseWhere(x, D, ctrl, std::cos(g.op[0]), std::sin(g.op[0]));
        } else if (g.type == OP_ROTATE_Z) {
            // diag(e^{-i a}, e^{+i a}) on the target where the controls match
            const uint32_t t = localMask(g.targetMask, local);
            const double cs = std::cos(g.op[0]), sn = std::sin(g.op[0]);
            for (int i = 0; i < D; i++) {
                if ((uint32_t) (i & ctrl) != ctrl) continue;
                const double s = (i & t) ? sn : -sn;
                const double re = x[2 * i], im = x[2 * i + 1];
                x[2 * i] = re * cs - im * s;
                x[2 * i + 1] = re * s + im * cs;
            }
        } else if (g.type == OP_MULTI_UNITARY) {
            const int k = g.numMultiTargets;
            const int d = 1 << k;
            const std::vector<double> &m = pool.mats[(size_t) g.multiIndex];
            int tl[8];
            uint32_t tmask = 0;
            for (int i = 0; i < k; i++) {
                tl[i] = local[g.multiTargets[i]];
                tmask |= 1u << tl[i];
            }
            double in[2 * 128], out[2 * 128];
            for (int base = 0; base < D; base++) {
                if (base & (int) tmask) continue;
                if ((uint32_t) (base & ctrl) != ctrl) continue;
                auto idx = [&](int j) {
                    int r = base;
                    for (int i = 0; i < k; i++)
                        if ((j >> i) & 1) r |= 1 << tl[i];
                    return r;
                };
                for (int j = 0; j < d; j++) {
                    in[2 * j] = x[2 * idx(j)];
                    in[2 * j + 1] = x[2 * idx(j) + 1];
                }
                for (int r = 0; r < d; r++) {
                    double re = 0.0, im = 0.0;
                    for (int j = 0; j < d; j++) {
                        const double mr = m[2 * ((size_t) r * d + j)], mi = m[2 * ((size_t) r * d + j) + 1];
                        re += mr * in[2 * j] - mi * in[2 * j + 1];
                        im += mr * in[2 * j + 1] + mi * in[2 * j];
                    }
                    out[2 * r] = re;
                    out[2 * r + 1] = im;
                }
                for (int j = 0; j < d; j++) {
                    x[2 * idx(j)] = out[2 * j];
                    x[2 * idx(j) + 1] = out[2 * j + 1];
                }
            }
        } else {
            // a 2x2 on each target bit where the controls match
            double m[8];
            gateMatrix(g, m);
            for (u64 tm = g.targetMask; tm; tm &= tm - 1) {
                const int bit = 1 << local[__builtin_ctzll(tm)];
                for (int i0 = 0; i0 < D; i0++) {
                    if (i0 & bit) continue;
                    if ((uint32_t) (i0 & ctrl) != ctrl) continue;
                    const int i1 = i0 | bit;
                    const double ar = x[2 * i0], ai = x[2 * i0 + 1], br = x[2 * i1], bi = x[2 * i1 + 1];
                    x[2 * i0] = m[0] * ar - m[1] * ai + m[2] * br - m[3] * bi;
                    x[2 * i0 + 1] = m[0] * ai + m[1] * ar + m[2] * bi + m[3] * br;
                    x[2 * i1] = m[4] * ar - m[5] * ai + m[6] * br - m[7] * bi;
                    x[2 * i1 + 1] = m[4] * ai + m[5] * ar + m[6] * bi + m[7] * br;
                }
            }
        }
    }
}

std::vector<Gate> fuseDenseBlocks(const std::vector<Gate> &gates, int numBits, int K, MatrixPool &pool,
                                  int *blocks, int maxBlocks, bool *stopped) {
    std::vector<Gate> out;
    if (blocks) *blocks = 0;
    if (stopped) *stopped = false;
    int made = 0;
    if (K < 1 || K > 7 || K > numBits) return gates;
    GateDag dag(numBits, true);
    dag.setTouchCost(true);
    for (const Gate &g : gates) dag.add(g);
    const int D = 1 << K;
    std::vector<double> u((size_t) 2 * D * D);
    while (!dag.empty()) {
        if (maxBlocks > 0 && made >= maxBlocks) {
            if (stopped) *stopped = true;
            break;
        }
        u64 mask = 0;
        for (;;) {
            size_t best = 0;
            u64 bestAdd = 0;
            for (u64 add : dag.frontierSets(mask)) {
                if (__builtin_popcountll(mask | add) > K) continue;
                const size_t c = dag.countAllowed(mask | add);
                if (c > best || (c == best && bestAdd && __builtin_popcountll(add) < __builtin_popcountll(bestAdd))) {
                    best = c;
                    bestAdd = add;
                }
            }
            if (!bestAdd) break;
            mask |= bestAdd;
        }
        std::vector<Gate> gs = mask ? dag.takeAllowed(mask) : std::vector<Gate>();
        if (gs.empty()) {
            // the next runnable gate touches more than K qubits: it (and what
            // fits beside it in its qubits) passes through unchanged
            const std::vector<u64> next = dag.frontierSets(0);
            if (next.empty()) break;
            gs = dag.takeAllowed(next.front());
            if (gs.empty()) break;
            out.insert(out.end(), gs.begin(), gs.end());
            continue;
        }
        // pad the block to K qubits with the lowest unused address bits
        for (int b = 0; __builtin_popcountll(mask) < K && b < numBits; b++) mask |= 1ULL << b;
        int local[64];
        Gate f;
        f.type = OP_MULTI_UNITARY;
        f.targetMask = mask;
        f.controlMask = 0;
        f.numMultiTargets = K;
        int n = 0;
        for (int b = 0; b < 64; b++) {
            local[b] = -1;
            if ((mask >> b) & 1ULL) {
                local[b] = n;
                f.multiTargets[n++] = b;
            }
        }
        // columns of the identity, then every gate of the block in order
        std::fill(u.begin(), u.end(), 0.0);
        for (int c = 0; c < D; c++) u[(size_t) 2 * (c * D + c)] = 1.0;
        for (const Gate &g : gs) applyGateLocal(g, pool, local, K, u.data(), D);
        // row-major (re, im): entry (r, c) is amplitude r of column c
        std::vector<double> m((size_t) 2 * D * D);
        for (int r = 0; r < D; r++)
            for (int c = 0; c < D; c++) {
                m[(size_t) 2 * (r * D + c)] = u[(size_t) 2 * (c * D + r)];
                m[(size_t) 2 * (r * D + c) + 1] = u[(size_t) 2 * (c * D + r) + 1];
            }
        f.multiIndex = (int32_t) pool.mats.size();
        pool.mats.push_back(std::move(m));
        out.push_back(f);
        made++;
        if (blocks) (*blocks)++;
    }
    return out;
}

}  // namespace dgq
