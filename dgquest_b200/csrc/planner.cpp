// planner.cpp -- see planner.h.
#include "planner.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "dag.h"

namespace dgq {

static const double kRsqrt2 = 0.7071067811865475244008443621;

// Block selection. dgQuEST's rule (DAG.cpp:219-259) walks the DAG depth
// first and admits gates while the target union fits; the tile bits then
// follow from the order of the walk. Here the tile's free bits are chosen
// first: starting from the 5 coalesced bits, add one at a time the bit that
// lets the most gates run (dependency-closed, non-diagonal targets inside
// the tile), considering only bits some runnable-next gate targets, then
// take every gate that fits. Phases inside a block use the same rule with
// the 4 register bits.
// Grows `mask` up to `budget` bits: each step adds the missing target bits
// of one runnable-next gate, choosing the addition that lets the most gates
// run (ties: fewer new bits; with preferHigh, bits above the 5 coalesced).
// Registers of at least this many address bits choose tile bits with a
// one-step lookahead unless told otherwise (measured on the 30-qubit random
// circuit of depth 20: 17 instead of 19 sweeps for 3x the planning time).
static int lookaheadMinBits() {
    static const int v = []() {
        const char *e = getenv("DGQ_PLAN_LOOKAHEAD_BITS");
        return e ? atoi(e) : 24;
    }();
    return v;
}

bool lookaheadBySize(int numBits) { return numBits >= lookaheadMinBits(); }

// lookahead: score each candidate addition by the best follow-up addition too
static void growMask(const GateDag &dag, u64 &mask, int budget, bool preferHigh, bool lookahead = false) {
    const u64 low = (1ULL << kCoalescedBits) - 1;
    const bool look = lookahead;
    while (popcount64(mask) < budget) {
        const std::vector<u64> cands = dag.frontierSets(mask);
        size_t best = 0;
        u64 bestAdd = 0;
        for (u64 add : cands) {
            if (popcount64(mask | add) > budget) continue;
            size_t c = dag.countAllowed(mask | add);
            if (look && popcount64(mask | add) < budget) {
                // score a candidate by the best follow-up addition as well
                for (u64 add2 : dag.frontierSets(mask | add)) {
                    if (popcount64(mask | add | add2) > budget) continue;
                    c = std::max(c, dag.countAllowed(mask | add | add2));
                }
            }
            bool better = c > best;
            if (!better && c == best && bestAdd) {
                const int pa = popcount64(add), pb = popcount64(bestAdd);
                if (pa < pb)
                    better = true;
                else if (pa == pb && preferHigh && (bestAdd & low) && !(add & low))
                    better = true;
            }
            if (better) {
                best = c;
                bestAdd = add;
            }
        }
        if (!bestAdd) break;
        mask |= bestAdd;
    }
}

bool planBlocksEach(const std::vector<Gate> &gates, int numBits, int tileBits, int seedBits,
                    const std::function<bool(BlockPlan &)> &onBlock, int lookahead) {
    GateDag dag(numBits, true);
    for (const Gate &g : gates) dag.add(g);
    const u64 seed = (1ULL << seedBits) - 1;
    const u64 all = numBits >= 64 ? ~0ULL : ((1ULL << numBits) - 1);
    const bool look = lookahead < 0 ? lookaheadBySize(numBits) : lookahead > 0;
    while (!dag.empty()) {
        BlockPlan b;
        u64 mask = seed & all;
        growMask(dag, mask, tileBits, false, look);
        // pad to tileBits with the lowest unused bits above the seed
        for (int bit = seedBits; popcount64(mask) < tileBits && bit < numBits; bit++) mask |= 1ULL << bit;
        b.tileMask = mask & all;
        b.gates = dag.takeAllowed(b.tileMask);
        // only a gate wider than the tile is left: not plannable here
        if (b.gates.empty()) return false;
        if (!onBlock(b)) return true;
    }
    return true;
}

std::vector<BlockPlan> planBlocks(const std::vector<Gate> &gates, int numBits, int tileBits, bool *complete,
                                  int seedBits, int lookahead) {
    std::vector<BlockPlan> blocks;
    const bool ok = planBlocksEach(
        gates, numBits, tileBits, seedBits,
        [&](BlockPlan &b) {
            blocks.push_back(std::move(b));
            return true;
        },
        lookahead);
    if (complete) *complete = ok;
    return blocks;
}

namespace {

struct TileMap {
    int local[64];   // address bit -> tile-local bit, -1 if not in tile
    int ctaIdx[64];  // address bit -> blockIdx bit, -1 if in tile
    int tilePos[kMaxTileBits];
};

TileMap makeTileMap(u64 tileMask, int numBits) {
    TileMap m;
    int nl = 0, nc = 0;
    for (int b = 0; b < 64; b++) {
        m.local[b] = -1;
        m.ctaIdx[b] = -1;
    }
    for (int b = 0; b < numBits; b++) {
        if ((tileMask >> b) & 1ULL) {
            m.tilePos[nl] = b;
            m.local[b] = nl++;
        } else {
            m.ctaIdx[b] = nc++;
        }
    }
    return m;
}

struct Split {
    uint32_t tileLocal = 0;  // tile-local mask
    uint32_t cta = 0;        // blockIdx-space mask
};

Split splitMask(u64 m, const TileMap &tm) {
    Split s;
    for (int b = 0; b < 64 && m; b++) {
        if (!((m >> b) & 1ULL)) continue;
        m &= ~(1ULL << b);
        if (tm.local[b] >= 0)
            s.tileLocal |= 1u << tm.local[b];
        else
            s.cta |= 1u << tm.ctaIdx[b];
    }
    return s;
}

struct PhaseLayout {
    int regPos[kRegBits];
    int thrPos[kMaxThreadBits];
    uint32_t regLocalMask = 0;
    bool direct = false;
};

// Register bits: `front` first (dense-gate target order), then the other
// targets, then padding from the top tile bit down. Thread bits: three bits
// of distinct (position mod 3) first, so that each quarter-warp touches 8
// distinct swizzled bank groups, then the rest in increasing order.
PhaseLayout makeLayout(const std::vector<int> &front, uint32_t targetsLocal, int tileBits, bool paired = false) {
    PhaseLayout L;
    int nr = 0;
    // paired form: tile-local bit 0 is the pair inside a slot, never a
    // register or thread bit
    uint32_t used = paired ? 1u : 0u;
    if (paired) targetsLocal &= ~1u;
    for (int p : front) {
        L.regPos[nr++] = p;
        used |= 1u << p;
    }
    for (int p = 0; p < tileBits && nr < kRegBits; p++) {
        if (((targetsLocal >> p) & 1u) && !((used >> p) & 1u)) {
            L.regPos[nr++] = p;
            used |= 1u << p;
        }
    }
    for (int p = tileBits - 1; p >= 0 && nr < kRegBits; p--) {
        if (!((used >> p) & 1u)) {
            L.regPos[nr++] = p;
            used |= 1u << p;
        }
    }
    if (paired) used &= ~1u;
    L.regLocalMask = used;
    std::vector<int> thr;
    for (int p = paired ? 1 : 0; p < tileBits; p++)
        if (!((used >> p) & 1u)) thr.push_back(p);
    // slots (16 B) are indexed by tile-local bits 1.. in the paired form
    const int sh = paired ? 1 : 0;
    L.direct = ((used >> sh) & ((1u << kCoalescedBits) - 1)) == 0;
    if (L.direct) {
        // lanes on tile bits 0..4 (address bits 0..4): the phase can read and
        // write HBM directly in 512-byte runs; bits 0..2 have distinct
        // classes mod 3, so its shared-memory accesses stay conflict-free
        int i = 0;
        for (int p : thr) L.thrPos[i++] = p;
        return L;
    }
    std::vector<int> lanes, rest;
    int classes = 0;
    for (int p : thr) {
        const int q = p - sh;
        if ((int) lanes.size() < 3 && !((classes >> (q % 3)) & 1)) {
            lanes.push_back(p);
            classes |= 1 << (q % 3);
        } else {
            rest.push_back(p);
        }
    }
    int i = 0;
    for (int p : lanes) L.thrPos[i++] = p;
    for (int p : rest) L.thrPos[i++] = p;
    return L;
}

uint8_t regSpace(uint32_t tileLocal, const PhaseLayout &L) {
    uint8_t r = 0;
    for (int b = 0; b < kRegBits; b++)
        if ((tileLocal >> L.regPos[b]) & 1u) r |= (uint8_t) (1u << b);
    return r;
}

bool isZero(double x) { return x == 0.0; }

}  // namespace

double opFlopsPerAmp(const KOp &op) {
    double f = 0.0;
    switch (op.kind) {
        case KOP_M2R:
        case KOP_M2I:
        case KOP_PH:
        case KOP_Z2: f = 6.0; break;
        case KOP_M2C: f = 14.0; break;
        case KOP_DENSE: f = 8.0 * (double) (1 << op.k) - 2.0; break;
        case KOP_RY1:
        case KOP_RY2:
        case KOP_RX1:
        case KOP_RX2: f = 4.0; break;   // one FMA per output component
        case KOP_H1: f = 2.0; break;    // one add per output component
        case KOP_PH1: f = 3.0; break;   // a complex multiply on half of the amplitudes
        case KOP_RN1: f = 8.0; break;   // x + p y: two complex FMAs per amplitude
        default: f = 0.0; break;
    }
    const int c = __builtin_popcount(op.ctrlReg) + __builtin_popcount(op.ctrlLoc) + __builtin_popcount(op.ctrlCta);
    return f / (double) (1u << c);
}

void encodeHeaderOnly(int numBits, int numReal, int tileBits, const SweepHeader &hdr, TileProgram &out,
                      bool paired) {
    std::memset(&out, 0, sizeof(out));
    out.paired = paired ? 1 : 0;
    out.globalRe = 1.0;
    out.numBits = numBits;
    out.numReal = numReal;
    out.initKind = hdr.initKind;
    out.initIndex = hdr.initIndex;
    out.initAmp = hdr.initAmp;
    out.hasRestrict = hdr.hasRestrict ? 1 : 0;
    out.restrictMask = hdr.restrictMask;
    out.restrictValue = hdr.restrictValue;
    out.restrictScale = hdr.restrictScale;
    // tile = the lowest tileBits bits
    for (int i = 0; i < tileBits - kCoalescedBits; i++) out.highPos[i] = (uint8_t) (kCoalescedBits + i);
    for (int i = 0; i < numBits - tileBits; i++) out.ctaPos[i] = (uint8_t) (tileBits + i);
}

bool encodeBlock(const BlockPlan &block, int numBits, int numReal, int tileBits, const MatrixPool &pool,
                 const SweepHeader &first, std::vector<TileProgram> &out, PlanStats *stats, std::string *err,
                 bool paired) {
    const TileMap tm = makeTileMap(block.tileMask, numBits);

    // ---- phases: greedy DAG selection with the register budget
    struct Phase {
        std::vector<Gate> gates;
        std::vector<int> front;  // dense-gate target order (tile-local)
        uint32_t targetsLocal = 0;
    };
    std::vector<Phase> phases;
    {
        GateDag dag(numBits, false);
        for (const Gate &g : block.gates) dag.add(g);
        while (!dag.empty()) {
            // paired form: address bit 0 is always inside the thread
            u64 mask = paired ? 1ULL : 0ULL;
            growMask(dag, mask, kRegBits + (paired ? 1 : 0), true, true);
            std::vector<Gate> gs = dag.takeAllowed(mask);
            if (gs.empty()) {
                // a multi-target gate wider than the register bits
                u64 m2 = 0;
                gs = dag.takeBlock(kRegBits, m2, 1u << 20);
            }
            if (gs.empty()) {
                if (err) *err = "a gate has more non-diagonal targets than the register tile holds";
                return false;
            }
            // a dense multi-qubit gate fixes the register order: give it its own phase
            Phase cur;
            auto flush = [&]() {
                if (!cur.gates.empty()) phases.push_back(cur);
                cur = Phase();
            };
            for (const Gate &g : gs) {
                if (g.type == OP_MULTI_UNITARY) {
                    if (paired && (g.targetMask & 1ULL)) {
                        if (err) *err = "paired form: a multi-qubit unitary targets address bit 0";
                        return false;
                    }
                    flush();
                    Phase d;
                    d.gates.push_back(g);
                    for (int i = 0; i < g.numMultiTargets; i++) d.front.push_back(tm.local[g.multiTargets[i]]);
                    d.targetsLocal = splitMask(g.targetMask, tm).tileLocal;
                    phases.push_back(d);
                    continue;
                }
                cur.gates.push_back(g);
                if (!isDiagonalType(g.type)) cur.targetsLocal |= splitMask(g.targetMask, tm).tileLocal;
            }
            flush();
        }
    }

    // ---- programs
    auto newProgram = [&](bool isFirst) {
        out.emplace_back();
        TileProgram &p = out.back();
        std::memset(&p, 0, sizeof(p));
        p.numBits = numBits;
        p.numReal = numReal;
        p.globalRe = 1.0;
        p.globalIm = 0.0;
        p.hasGlobal = 0;
        p.paired = paired ? 1 : 0;
        if (isFirst) {
            p.initKind = first.initKind;
            p.initIndex = first.initIndex;
            p.initAmp = first.initAmp;
            p.hasRestrict = first.hasRestrict ? 1 : 0;
            p.restrictMask = first.restrictMask;
            p.restrictValue = first.restrictValue;
            p.restrictScale = first.restrictScale;
        } else {
            p.initKind = INIT_NONE;
        }
        for (int i = 0; i < tileBits - kCoalescedBits; i++) p.highPos[i] = (uint8_t) tm.tilePos[kCoalescedBits + i];
        for (int b = 0; b < numBits; b++)
            if (tm.ctaIdx[b] >= 0) p.ctaPos[tm.ctaIdx[b]] = (uint8_t) b;
        if (stats) stats->sweeps++;
        return &out.back();
    };
    TileProgram *prog = newProgram(true);
    int numCoef = 0;

    for (const Phase &ph : phases) {
        const PhaseLayout L = makeLayout(ph.front, ph.targetsLocal, tileBits, paired);
        // encode the phase's ops into a scratch list first; uncontrolled
        // rotations leave their scalar factor in (phRe, phIm)
        std::vector<KOp> ops;
        std::vector<double> coef;
        double phRe = 1.0, phIm = 0.0;
        auto scaleBy = [&](double fr, double fi) {
            const double r = phRe * fr - phIm * fi, i = phRe * fi + phIm * fr;
            phRe = r;
            phIm = i;
        };
        for (const Gate &g : ph.gates) {
            KOp op;
            std::memset(&op, 0, sizeof(op));
            op.selCta = -1;
            const Split c = splitMask(g.controlMask, tm);
            op.ctrlReg = regSpace(c.tileLocal, L);
            op.ctrlLoc = (uint16_t) (c.tileLocal & ~L.regLocalMask);
            op.ctrlCta = c.cta;
            op.coef = (uint16_t) coef.size();  // phase-relative, rebased when copied
            auto targetReg = [&](u64 tmask) -> int {
                const Split t = splitMask(tmask, tm);
                if (paired && t.tileLocal == 1u) return 4;  // the pair inside a slot
                for (int b = 0; b < kRegBits; b++)
                    if (t.tileLocal == (1u << L.regPos[b])) return b;
                return -1;
            };
            bool emit = true;
            bool selIsReg = false;
            const int t = (int) g.type;
            if (t < 8) {
                switch (t) {
                    case OP_ONE: emit = false; break;
                    case OP_S_GATE: op.kind = KOP_MULI; break;
                    case OP_PAULI_Z: op.kind = KOP_NEG; break;
                    case OP_S_GATE_CONJ: op.kind = KOP_MULNI; break;
                    default: {
                        // odd powers: e^{i pi t / 4} with (+-1 +- i)/sqrt(2)
                        op.kind = KOP_PH;
                        const double c0 = (t == 1 || t == 7) ? kRsqrt2 : -kRsqrt2;
                        const double s0 = (t == 1 || t == 3) ? kRsqrt2 : -kRsqrt2;
                        coef.push_back(c0);
                        coef.push_back(s0);
                        break;
                    }
                }
            } else if (g.type == OP_PHASE_SHIFT) {
                op.kind = KOP_PH;
                coef.push_back(std::cos(g.op[0]));
                coef.push_back(std::sin(g.op[0]));
            } else if (g.type == OP_ROTATE_Z && g.controlMask == 0) {
                // diag(e^{-ia}, e^{ia}) = e^{-ia} diag(1, e^{2ia})
                op.kind = KOP_PH1;
                coef.push_back(std::cos(2.0 * g.op[0]));
                coef.push_back(std::sin(2.0 * g.op[0]));
                scaleBy(std::cos(g.op[0]), -std::sin(g.op[0]));
                const Split s = splitMask(g.targetMask, tm);
                if (s.tileLocal) {
                    const uint8_t r = regSpace(s.tileLocal, L);
                    if (r) {
                        op.k = (uint8_t) __builtin_ctz(r);
                        selIsReg = true;
                    } else {
                        op.selLoc = (uint16_t) s.tileLocal;
                    }
                } else {
                    op.selCta = (int8_t) __builtin_ctz(s.cta);
                }
            } else if (g.type == OP_ROTATE_Z) {
                op.kind = KOP_Z2;
                coef.push_back(std::cos(g.op[0]));
                coef.push_back(std::sin(g.op[0]));
                const Split s = splitMask(g.targetMask, tm);
                if (s.tileLocal) {
                    const uint8_t r = regSpace(s.tileLocal, L);
                    if (r) {
                        op.k = (uint8_t) __builtin_ctz(r);
                        selIsReg = true;
                    } else {
                        op.selLoc = (uint16_t) s.tileLocal;
                    }
                } else {
                    op.selCta = (int8_t) __builtin_ctz(s.cta);
                }
            } else if (g.type == OP_MULTI_UNITARY) {
                op.kind = KOP_DENSE;
                op.k = (uint8_t) g.numMultiTargets;
                const auto &m = pool.mats[(size_t) g.multiIndex];
                coef.insert(coef.end(), m.begin(), m.end());
            } else {
                const int k = targetReg(g.targetMask);
                if (k < 0) {
                    if (err) *err = "internal: pair-gate target is not a register bit";
                    return false;
                }
                op.k = (uint8_t) k;
                const bool free = g.controlMask == 0;
                switch (g.type) {
                    case OP_HADAMARD:
                        if (!free) {
                            op.kind = KOP_M2R;
                            coef.insert(coef.end(), {kRsqrt2, kRsqrt2, kRsqrt2, -kRsqrt2});
                        } else {
                            op.kind = KOP_H1;
                            scaleBy(kRsqrt2, 0.0);
                        }
                        break;
                    case OP_ROTATE_Y:
                    case OP_ROTATE_X: {
                        const double cs = std::cos(g.op[0]), sn = std::sin(g.op[0]);
                        const bool isY = g.type == OP_ROTATE_Y;
                        if (!free) {
                            op.kind = isY ? KOP_M2R : KOP_M2I;
                            if (isY)
                                coef.insert(coef.end(), {cs, -sn, sn, cs});
                            else
                                coef.insert(coef.end(), {cs, -sn, -sn, cs});
                        } else if (std::fabs(cs) >= std::fabs(sn)) {
                            op.kind = isY ? KOP_RY1 : KOP_RX1;
                            coef.push_back(sn / cs);
                            scaleBy(cs, 0.0);
                        } else {
                            op.kind = isY ? KOP_RY2 : KOP_RX2;
                            coef.push_back(cs / sn);
                            scaleBy(sn, 0.0);
                        }
                        break;
                    }
                    case OP_PAULI_X: op.kind = KOP_X; break;
                    case OP_PAULI_Y: op.kind = KOP_Y; break;
                    case OP_PAULI_Y_CONJ: op.kind = KOP_YC; break;
                    default: {
                        double m[8];
                        gateMatrix(g, m);
                        // uncontrolled rotation about an axis in the XY plane:
                        // U = d [[1, p], [-conj(p), 1]] with d = U00 = U11,
                        // |p| <= 1; d goes to the sweep's global factor
                        const double d2 = m[0] * m[0] + m[1] * m[1];
                        const double o2 = m[2] * m[2] + m[3] * m[3];
                        const double tol = 1e-15 * std::sqrt(d2 + o2);
                        if (free && d2 > 0.0 && o2 <= d2 * (1.0 + 1e-12) && std::fabs(m[6] - m[0]) <= tol &&
                            std::fabs(m[7] - m[1]) <= tol) {
                            // p = U01 / U00, q = U10 / U00 must equal -conj(p)
                            const double pr = (m[2] * m[0] + m[3] * m[1]) / d2, pi = (m[3] * m[0] - m[2] * m[1]) / d2;
                            const double qr = (m[4] * m[0] + m[5] * m[1]) / d2, qi = (m[5] * m[0] - m[4] * m[1]) / d2;
                            if (std::fabs(qr + pr) <= 1e-14 && std::fabs(qi - pi) <= 1e-14) {
                                scaleBy(m[0], m[1]);
                                if (std::fabs(pi) <= 1e-16) {
                                    op.kind = KOP_RY1;  // p = -t
                                    coef.push_back(-pr);
                                } else if (std::fabs(pr) <= 1e-16) {
                                    op.kind = KOP_RX1;  // p = -i t
                                    coef.push_back(-pi);
                                } else {
                                    op.kind = KOP_RN1;
                                    coef.push_back(pr);
                                    coef.push_back(pi);
                                }
                                break;
                            }
                        }
                        if (isZero(m[1]) && isZero(m[3]) && isZero(m[5]) && isZero(m[7])) {
                            op.kind = KOP_M2R;
                            coef.insert(coef.end(), {m[0], m[2], m[4], m[6]});
                        } else if (isZero(m[1]) && isZero(m[2]) && isZero(m[4]) && isZero(m[7])) {
                            op.kind = KOP_M2I;
                            coef.insert(coef.end(), {m[0], m[3], m[5], m[6]});
                        } else {
                            op.kind = KOP_M2C;
                            coef.insert(coef.end(), m, m + 8);
                        }
                        break;
                    }
                }
            }
            if (emit) {
                const int rc = op.ctrlReg ? 1 : 0;
                const uint8_t kSaved = op.k;
                if (op.k == 4 && op.kind != KOP_DENSE) op.k = 0;  // codes index k < 4; paired ops keep k = 4
                op.thrCtl = (op.ctrlLoc || op.ctrlCta) ? 1 : 0;
                switch (op.kind) {
                    case KOP_M2R: op.code = (uint8_t) (KC_M2R + op.k + 4 * rc); break;
                    case KOP_M2I: op.code = (uint8_t) (KC_M2I + op.k + 4 * rc); break;
                    case KOP_M2C: op.code = (uint8_t) (KC_M2C + op.k + 4 * rc); break;
                    case KOP_X: op.code = (uint8_t) (KC_X + op.k + 4 * rc); break;
                    case KOP_Y: op.code = (uint8_t) (KC_Y + op.k + 4 * rc); break;
                    case KOP_YC: op.code = (uint8_t) (KC_YC + op.k + 4 * rc); break;
                    case KOP_Z2: op.code = (uint8_t) (selIsReg ? KC_Z2R + op.k + 4 * rc : KC_Z2T + rc); break;
                    case KOP_PH: op.code = (uint8_t) (KC_PH + rc); break;
                    case KOP_NEG: op.code = (uint8_t) (KC_NEG + rc); break;
                    case KOP_MULI: op.code = (uint8_t) (KC_MULI + rc); break;
                    case KOP_MULNI: op.code = (uint8_t) (KC_MULNI + rc); break;
                    case KOP_DENSE: op.code = (uint8_t) (KC_DENSE + op.k - 1); break;
                    case KOP_RY1: op.code = (uint8_t) (KC_RY1 + op.k); break;
                    case KOP_RY2: op.code = (uint8_t) (KC_RY2 + op.k); break;
                    case KOP_RX1: op.code = (uint8_t) (KC_RX1 + op.k); break;
                    case KOP_RX2: op.code = (uint8_t) (KC_RX2 + op.k); break;
                    case KOP_H1: op.code = (uint8_t) (KC_H1 + op.k); break;
                    case KOP_PH1: op.code = (uint8_t) (selIsReg ? KC_PH1R + op.k : KC_PH1T); break;
                    case KOP_RN1: op.code = (uint8_t) (KC_RN1 + op.k); break;
                    default: break;
                }
                op.k = kSaved;
                ops.push_back(op);
            }
        }
        if (ops.size() > (size_t) kMaxOps || coef.size() > (size_t) kMaxCoef) {
            if (err) *err = "a single register phase exceeds the tile program capacity";
            return false;
        }
        // start a new program (one more sweep over the same tile) when full
        if (prog->numPhases + 1 > kMaxPhases || prog->numOps + (int) ops.size() > kMaxOps ||
            numCoef + (int) coef.size() > kMaxCoef) {
            prog = newProgram(false);
            numCoef = 0;
        }
        if (phRe != 1.0 || phIm != 0.0) {
            const double gr = prog->globalRe, gi = prog->globalIm;
            prog->globalRe = gr * phRe - gi * phIm;
            prog->globalIm = gr * phIm + gi * phRe;
            prog->hasGlobal = 1;
        }
        KPhase &kp = prog->phases[prog->numPhases++];
        std::memset(&kp, 0, sizeof(kp));
        for (int i = 0; i < tileBits - kRegBits - (paired ? 1 : 0); i++) kp.thrPos[i] = (uint8_t) L.thrPos[i];
        for (int b = 0; b < kRegBits; b++) kp.regPos[b] = (uint8_t) L.regPos[b];
        kp.direct = L.direct ? 1 : 0;
        kp.opBegin = (uint16_t) prog->numOps;
        for (KOp o : ops) {
            o.coef = (uint16_t) (o.coef + numCoef);
            prog->ops[prog->numOps++] = o;
            if (stats) {
                stats->ops++;
                stats->flopsPerAmp += opFlopsPerAmp(o);
            }
        }
        kp.opEnd = (uint16_t) prog->numOps;
        for (int j = 0; j < kRegs; j++) {
            uint32_t loc = 0;
            for (int b = 0; b < kRegBits; b++)
                if ((j >> b) & 1) loc |= 1u << L.regPos[b];
            kp.regOff[j] = (uint16_t) tileSwizzle(paired ? loc >> 1 : loc);
        }
        for (double c : coef) prog->coef[numCoef++] = c;
        prog->numCoef = (uint16_t) numCoef;
        if (stats) stats->phases++;
    }
    if (stats) stats->gates += (int) block.gates.size();
    return true;
}

}  // namespace dgq
