// jit.cpp -- see jit.h.
#include "jit.h"

#include <nvrtc.h>

#include <atomic>
#include <condition_variable>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

namespace dgq {

// Embedded texts of tile_program.h and jit_prelude.cuh (generated at build
// time into jit_sources.inc as kTileProgramSource / kJitPreludeSource).
#include "jit_sources.inc"

namespace {

const char *kernelKindName(int code) {
    if (code < KC_M2I) return "jM2R";
    if (code < KC_M2C) return "jM2I";
    if (code < KC_X) return "jM2C";
    if (code < KC_Y) return "jX";
    if (code < KC_YC) return "jY";
    if (code < KC_Z2R) return "jYC";
    return "jZ2R";
}

void emitOp(std::ostringstream &o, const KOp &op) {
    const unsigned cr = op.ctrlReg;
    const int off = op.coef;
    std::ostringstream body;
    if (op.code < KC_Z2T) {
        const int base = (op.code / 8) * 8;
        const int kk = op.code - base;
        const int k = kk & 3;
        const bool ctrl = kk >= 4;
        const char *fn = kernelKindName(op.code);
        const bool coef = !(op.code >= KC_X && op.code < KC_Z2R);
        body << "dgq::" << fn << "<" << k << ", " << (ctrl ? "true" : "false") << ", " << cr << "u>(a"
             << (coef ? ", prog.coef + " + std::to_string(off) : std::string()) << ");";
    } else if (op.code == KC_Z2T || op.code == KC_Z2T + 1) {
        const bool ctrl = op.code == KC_Z2T + 1;
        std::ostringstream sel;
        bool any = false;
        if (op.selLoc) {
            sel << "((loc & " << op.selLoc << "u) != 0u)";
            any = true;
        }
        if (op.selCta >= 0) {
            sel << (any ? " || " : "") << "(((cta >> " << (int) op.selCta << ") & 1u) != 0u)";
            any = true;
        }
        if (!any) sel << "false";
        body << "{ const bool b_ = " << sel.str() << "; dgq::jPH<" << (ctrl ? "true" : "false") << ", " << cr
             << "u>(a, prog.coef[" << off << "], b_ ? prog.coef[" << off + 1 << "] : -prog.coef[" << off + 1
             << "]); }";
    } else if (op.code == KC_PH || op.code == KC_PH + 1) {
        body << "dgq::jPH<" << (op.code == KC_PH + 1 ? "true" : "false") << ", " << cr << "u>(a, prog.coef[" << off
             << "], prog.coef[" << off + 1 << "]);";
    } else if (op.code == KC_NEG || op.code == KC_NEG + 1) {
        body << "dgq::jNEG<" << (op.code == KC_NEG + 1 ? "true" : "false") << ", " << cr << "u>(a);";
    } else if (op.code == KC_MULI || op.code == KC_MULI + 1) {
        body << "dgq::jMULI<" << (op.code == KC_MULI + 1 ? "true" : "false") << ", " << cr << "u>(a);";
    } else if (op.code == KC_MULNI || op.code == KC_MULNI + 1) {
        body << "dgq::jMULNI<" << (op.code == KC_MULNI + 1 ? "true" : "false") << ", " << cr << "u>(a);";
    } else if (op.code >= KC_DENSE && op.code < KC_DENSE + 4) {
        body << "dgq::jDense<" << (op.code - KC_DENSE + 1) << ", " << cr << "u>(a, prog.coef + " << off << ");";
    } else if (op.code >= KC_RY1 && op.code < KC_H1) {
        static const char *names[4] = {"jRY1", "jRY2", "jRX1", "jRX2"};
        body << "dgq::" << names[(op.code - KC_RY1) / 4] << "<" << (op.code - KC_RY1) % 4 << ">(a, prog.coef + " << off
             << ");";
    } else if (op.code >= KC_RN1 && op.code < KC_RN1 + 4) {
        body << "dgq::jRN1<" << op.code - KC_RN1 << ">(a, prog.coef + " << off << ");";
    } else if (op.code >= KC_H1 && op.code < KC_H1 + 4) {
        body << "dgq::jH1<" << op.code - KC_H1 << ">(a);";
    } else if (op.code >= KC_PH1R && op.code < KC_PH1R + 4) {
        body << "dgq::jPH1R<" << op.code - KC_PH1R << ">(a, prog.coef + " << off << ");";
    } else if (op.code == KC_PH1T) {
        std::ostringstream sel;
        bool any = false;
        if (op.selLoc) {
            sel << "((loc & " << op.selLoc << "u) != 0u)";
            any = true;
        }
        if (op.selCta >= 0) {
            sel << (any ? " || " : "") << "(((cta >> " << (int) op.selCta << ") & 1u) != 0u)";
            any = true;
        }
        body << "if (" << (any ? sel.str() : std::string("false")) << ") dgq::jPH<false, 0u>(a, prog.coef[" << off
             << "], prog.coef[" << off + 1 << "]);";
    }
    if (op.thrCtl) {
        std::ostringstream cond;
        bool any = false;
        if (op.ctrlLoc) {
            cond << "((loc & " << op.ctrlLoc << "u) == " << op.ctrlLoc << "u)";
            any = true;
        }
        if (op.ctrlCta) {
            cond << (any ? " && " : "") << "((cta & " << op.ctrlCta << "u) == " << op.ctrlCta << "u)";
            any = true;
        }
        o << "    if (" << (any ? cond.str() : std::string("true")) << ") { " << body.str() << " }\n";
    } else {
        o << "    " << body.str() << "\n";
    }
}

// Thread/CTA condition of an op (its controls among non-register bits), or "".
std::string thrCond(const KOp &op) {
    if (!op.thrCtl) return std::string();
    std::ostringstream cond;
    bool any = false;
    if (op.ctrlLoc) {
        cond << "((loc & " << op.ctrlLoc << "u) == " << op.ctrlLoc << "u)";
        any = true;
    }
    if (op.ctrlCta) {
        cond << (any ? " && " : "") << "((cta & " << op.ctrlCta << "u) == " << op.ctrlCta << "u)";
        any = true;
    }
    return any ? cond.str() : std::string("true");
}

// Selector of KC_Z2T / KC_PH1T (a thread or CTA bit) as a condition.
std::string selCond(const KOp &op) {
    std::ostringstream sel;
    bool any = false;
    if (op.selLoc) {
        sel << "((loc & " << op.selLoc << "u) != 0u)";
        any = true;
    }
    if (op.selCta >= 0) {
        sel << (any ? " || " : "") << "(((cta >> " << (int) op.selCta << ") & 1u) != 0u)";
        any = true;
    }
    return any ? sel.str() : std::string("false");
}

// 1: the op multiplies every amplitude of a thread by one phase factor
// that depends only on thread and CTA bits; 2: by -1 or +-i (integer sign
// flips when applied on their own); 0: neither.
int scalarKind(const KOp &op) {
    const bool allAmps = op.ctrlReg == 0;
    if (op.code == KC_PH1T) return 1;
    if ((op.code == KC_Z2T || op.code == KC_PH) || ((op.code == KC_Z2T + 1 || op.code == KC_PH + 1) && allAmps))
        return 1;
    if ((op.code == KC_NEG || op.code == KC_MULI || op.code == KC_MULNI) ||
        ((op.code == KC_NEG + 1 || op.code == KC_MULI + 1 || op.code == KC_MULNI + 1) && allAmps))
        return 2;
    return 0;
}

// A scalar op (scalarKind != 0) multiplied into the phase factor acc_.
void emitScalarAcc(std::ostringstream &o, const KOp &op) {
    const std::string tc = thrCond(op);
    const std::string on = tc.empty() ? std::string("true") : tc;
    const int off = op.coef;
    const int base = op.code & ~1;
    if (op.code == KC_PH1T) {
        o << "    dgq::jAccPhase(acc_, (" << on << ") && (" << selCond(op) << "), prog.coef[" << off << "], prog.coef["
          << off + 1 << "]);\n";
    } else if (base == KC_Z2T) {
        o << "    dgq::jAccPhase(acc_, " << on << ", prog.coef[" << off << "], (" << selCond(op) << ") ? prog.coef["
          << off + 1 << "] : -prog.coef[" << off + 1 << "]);\n";
    } else if (base == KC_PH) {
        o << "    dgq::jAccPhase(acc_, " << on << ", prog.coef[" << off << "], prog.coef[" << off + 1 << "]);\n";
    } else if (base == KC_NEG) {
        o << "    dgq::jAccNeg(acc_, " << on << ");\n";
    } else {
        o << "    dgq::jAccMulI(acc_, " << on << ", " << (base == KC_MULI ? "1.0" : "-1.0") << ");\n";
    }
}

// Whether the scalar ops of ops [b, e) go into one factor: when at least two
// of them are phase factors, or one is and there are sign flips besides
// (a lone sign flip stays on the integer pipe).
bool foldScalars(const TileProgram &prog, int b, int e) {
    int nPhase = 0, nSign = 0;
    for (int k = b; k < e; k++) {
        const int kind = scalarKind(prog.ops[k]);
        nPhase += kind == 1;
        nSign += kind == 2;
    }
    return nPhase >= 2 || (nPhase >= 1 && nSign >= 1);
}

}  // namespace

namespace {

// Address bit of tile-local bit l, as a CUDA expression.
std::string addrBitExpr(int l) {
    if (l < kCoalescedBits) return std::to_string(l);
    return "prog.highPos[" + std::to_string(l - kCoalescedBits) + "]";
}

// Address bits of this thread's element 0 and of the 4 register bits in
// the layout of phase ph (any layout).
void emitLayoutAddressing(std::ostringstream &o, const KPhase &ph, int W, const char *ctaExpr, const char *gt,
                          const char *rb) {
    o << "    const uint64_t " << gt << " = dgq::jCtaBase(prog, " << ctaExpr << ", W)";
    for (int i = 0; i < W - kRegBits; i++)
        o << " | ((uint64_t) ((tid >> " << i << ") & 1u) << " << addrBitExpr(ph.thrPos[i]) << ")";
    o << ";\n";
    o << "    const uint64_t " << rb << "[4] = {";
    for (int b = 0; b < kRegBits; b++) o << (b ? ", " : "") << "1ULL << " << addrBitExpr(ph.regPos[b]);
    o << "};\n";
}

// Address of thread `tid`'s element 0 and of the 4 register bits in a
// direct phase layout (thread bits 0..4 = address bits 0..4).
void emitDirectAddressing(std::ostringstream &o, const KPhase &ph, int W, const char *gt, const char *rb) {
    o << "    const uint64_t " << gt << " = dgq::jCtaBase(prog, cta, W) | (uint64_t) (tid & 31u)";
    for (int i = kCoalescedBits; i < W - kRegBits; i++)
        o << " | ((uint64_t) ((tid >> " << i << ") & 1u) << prog.highPos[" << (int) ph.thrPos[i] - kCoalescedBits << "])";
    o << ";\n";
    o << "    const uint64_t " << rb << "[4] = {";
    for (int b = 0; b < kRegBits; b++)
        o << (b ? ", " : "") << "1ULL << prog.highPos[" << (int) ph.regPos[b] - kCoalescedBits << "]";
    o << "};\n";
}

}  // namespace

// CTAs per SM the kernel is compiled for: 16 warps per SM at 128 registers
// a thread by default; DGQ_JIT_CTAS_PER_SM overrides (register cap
// 65536 / (threads x CTAs)).
static int ctasPerSm(int T, bool single) {
    static int env = -2;
    if (env == -2) {
        const char *e = getenv("DGQ_JIT_CTAS_PER_SM");
        env = e ? atoi(e) : -1;
    }
    if (env > 0) return env;
    // complex64 amplitudes need half the registers: 3 x 256-thread CTAs per SM
    const int regs = single ? 85 : 128;
    return 65536 / (regs * T) > 0 ? 65536 / (regs * T) : 1;
}

// ------------------------------------------------------------ paired form
namespace {

std::string cf(int off) { return "(float) prog.coef[" + std::to_string(off) + "]"; }

// In-slot 2x2 (target address bit 0) as 8 float expressions (row-major re, im).
bool inSlotMatrix(const KOp &op, std::string m[8]) {
    const int off = op.coef;
    const char *z = "0.0f", *one = "1.0f", *mone = "-1.0f";
    auto set = [&](std::initializer_list<std::string> v) {
        int i = 0;
        for (const auto &x : v) m[i++] = x;
    };
    switch (op.kind) {
        case KOP_M2R: set({cf(off), z, cf(off + 1), z, cf(off + 2), z, cf(off + 3), z}); return true;
        case KOP_M2I: set({cf(off), z, z, cf(off + 1), z, cf(off + 2), cf(off + 3), z}); return true;
        case KOP_M2C:
            set({cf(off), cf(off + 1), cf(off + 2), cf(off + 3), cf(off + 4), cf(off + 5), cf(off + 6), cf(off + 7)});
            return true;
        case KOP_X: set({z, z, one, z, one, z, z, z}); return true;
        case KOP_Y: set({z, z, z, mone, z, one, z, z}); return true;
        case KOP_YC: set({z, z, z, one, z, mone, z, z}); return true;
        case KOP_RY1: set({one, z, "-" + cf(off), z, cf(off), z, one, z}); return true;
        case KOP_RY2: set({cf(off), z, mone, z, one, z, cf(off), z}); return true;
        case KOP_RX1: set({one, z, z, "-" + cf(off), z, "-" + cf(off), one, z}); return true;
        case KOP_RX2: set({cf(off), z, z, mone, z, mone, cf(off), z}); return true;
        case KOP_H1: set({one, z, one, z, one, z, mone, z}); return true;
        case KOP_RN1: set({one, z, cf(off), cf(off + 1), "-" + cf(off), cf(off + 1), one, z}); return true;
        default: return false;
    }
}

std::string selExpr(const KOp &op) {
    std::ostringstream sel;
    bool any = false;
    const unsigned sl = op.selLoc & ~1u;
    if (sl) {
        sel << "((loc & " << sl << "u) != 0u)";
        any = true;
    }
    if (op.selCta >= 0) {
        sel << (any ? " || " : "") << "(((cta >> " << (int) op.selCta << ") & 1u) != 0u)";
        any = true;
    }
    return any ? sel.str() : std::string("false");
}

// Compile-time signs of the paired form. Bit j of negR (negI) is set when
// slot j's stored real (imaginary) pair holds the negated values. The
// negations inside gates (CZ and the other sign flips, the -1 entries of
// the factored Rx / Ry / H forms, the component swaps of Y and of the
// factors +-i) become changes of these masks or the choice of a
// coefficient's sign, so no instruction carries them. Round-to-nearest is
// symmetric, so every stored value equals the untracked computation's up
// to its sign. A phase's closing factor absorbs the masks (or sign flips
// on the integer pipe restore the values, when the phase has none), so
// values leave the registers with their true signs.
struct PairedSigns {
    uint32_t negR = 0, negI = 0;
    // component c of the pair (j0, j1): 0 R[j0], 1 I[j0], 2 R[j1], 3 I[j1]
    int sign(int c, int j0, int j1) const {
        const int j = c < 2 ? j0 : j1;
        const uint32_t m = (c & 1) ? negI : negR;
        return ((m >> j) & 1u) ? -1 : 1;
    }
    void set(int c, int j0, int j1, int s) {
        const int j = c < 2 ? j0 : j1;
        uint32_t &m = (c & 1) ? negI : negR;
        m = s < 0 ? (m | (1u << j)) : (m & ~(1u << j));
    }
};

// template argument of a mask
std::string hexu(uint32_t m) {
    char b[16];
    snprintf(b, sizeof b, "0x%xu", m);
    return b;
}

void flushSigns(std::ostringstream &o, PairedSigns &sg) {
    if (sg.negR | sg.negI) o << "    dgq::pFlushS<" << hexu(sg.negR) << ", " << hexu(sg.negI) << ">(R, I);\n";
    sg.negR = sg.negI = 0;
}

// f(p, j0, j1) for the pairs of register bit K whose j0 matches cr, p the
// pair's index among all 8 (the index the prelude's masks use)
template <class F>
void forPairsHost(int K, uint32_t cr, F f) {
    for (int p = 0; p < kRegs / 2; p++) {
        const int j0 = ((p >> K) << (K + 1)) | (p & ((1 << K) - 1));
        const int j1 = j0 | (1 << K);
        if ((j0 & (int) cr) != (int) cr) continue;
        f(p, j0, j1);
    }
}

// Output o of a factored pair gate, in true values: u * in[b] + k * coef * in[a]
// (u, k = +-1; coef is the op's coefficient, or 1 for H). The prelude's
// p*s templates fix b and a per kind; these tables give the signs.
struct LinearOut {
    int b, u, a, k;
};

// Coefficient-sign mask of a factored pair gate on bit K: output o is
// stored as fma2(+-coef, in[a], in[b]) with the sign of u * (sign of in[b]),
// so no negation is computed.
uint32_t linearMask(PairedSigns &sg, int K, const LinearOut (&outs)[4]) {
    uint32_t cs = 0;
    forPairsHost(K, 0u, [&](int p, int j0, int j1) {
        int ns[4];
        for (int c = 0; c < 4; c++) {
            const LinearOut &L = outs[c];
            const int sB = sg.sign(L.b, j0, j1), sA = sg.sign(L.a, j0, j1);
            ns[c] = L.u * sB;
            if (L.k * sA * L.u * sB < 0) cs |= 1u << (4 * p + c);
        }
        for (int c = 0; c < 4; c++) sg.set(c, j0, j1, ns[c]);
    });
    return cs;
}

// Output o of a pair permutation (X, Y, Y*), in true values: m * in[src].
struct PermOut {
    int src, m;
};

// Flip mask of a pair permutation; keep = true (the op runs under a
// condition known only at run time): the outputs keep their slots' signs,
// with a flip where the two differ; otherwise the signs move with the values.
uint32_t permMask(PairedSigns &sg, int K, uint32_t cr, const PermOut (&outs)[4], bool keep) {
    uint32_t fm = 0;
    forPairsHost(K, cr, [&](int p, int j0, int j1) {
        int ns[4];
        for (int c = 0; c < 4; c++) {
            const int trueSign = outs[c].m * sg.sign(outs[c].src, j0, j1);
            if (keep) {
                if (trueSign * sg.sign(c, j0, j1) < 0) fm |= 1u << (4 * p + c);
                ns[c] = sg.sign(c, j0, j1);
            } else {
                ns[c] = trueSign;
            }
        }
        for (int c = 0; c < 4; c++) sg.set(c, j0, j1, ns[c]);
    });
    return fm;
}

// (c + i s) on the slots in `slots` ((c - i s) on those in `sw`), keeping
// their signs; c / s / ns are float2 expressions (ns = -s)
void emitPhaseSlots(std::ostringstream &o, const PairedSigns &sg, uint32_t slots, uint32_t sw, const std::string &c,
                    const std::string &s, const std::string &ns) {
    if (!slots) return;
    o << "    dgq::pPhaseS<" << hexu(slots) << ", " << hexu((sg.negR ^ sg.negI) & slots) << ", " << hexu(sw & slots)
      << ">(R, I, " << c << ", " << s << ", " << ns << ");\n";
}

// Every slot times (gr + i gi), absorbing the signs (the values leave with
// their true signs); gr / gi are double expressions.
void emitGlobalAbsorb(std::ostringstream &o, PairedSigns &sg, const std::string &gr, const std::string &gi) {
    o << "    dgq::pGlobalS<" << hexu(sg.negR) << ", " << hexu(sg.negI) << ">(R, I, " << gr << ", " << gi << ");\n";
    sg.negR = sg.negI = 0;
}

// The sign-aware form of an op, written to `body`; false when the op has
// none (the caller flushes the signs and emits the plain form). keep: the
// op runs under a run-time condition, so it must leave the signs as they
// are (phases and flips do by construction).
bool emitSignedPaired(std::ostringstream &body, const KOp &op, PairedSigns &sg, bool keep) {
    const uint32_t cr = op.ctrlReg;
    const int k = op.k, off = op.coef;
    const std::string c0 = cf(off), c1 = cf(off + 1);
    auto slotsOf = [&](uint32_t need, uint32_t sel) {
        uint32_t m = 0;
        for (int j = 0; j < kRegs; j++)
            if ((j & (int) need) == (int) need && (!sel || (j & (int) sel))) m |= 1u << j;
        return m;
    };
    const bool slotKind = op.kind == KOP_NEG || op.kind == KOP_MULI || op.kind == KOP_MULNI || op.kind == KOP_PH ||
                          op.kind == KOP_Z2 || op.kind == KOP_PH1;
    if (k == 4 && !slotKind) return false;  // a gate inside the slot
    switch (op.kind) {
        case KOP_RY1:
        case KOP_RY2:
        case KOP_RX1:
        case KOP_RX2:
        case KOP_H1: {
            if (keep) return false;
            static const LinearOut ry1[4] = {{0, 1, 2, -1}, {1, 1, 3, -1}, {2, 1, 0, 1}, {3, 1, 1, 1}};
            static const LinearOut ry2[4] = {{2, -1, 0, 1}, {3, -1, 1, 1}, {0, 1, 2, 1}, {1, 1, 3, 1}};
            static const LinearOut rx1[4] = {{0, 1, 3, 1}, {1, 1, 2, -1}, {2, 1, 1, 1}, {3, 1, 0, -1}};
            static const LinearOut rx2[4] = {{3, 1, 0, 1}, {2, -1, 1, 1}, {1, 1, 2, 1}, {0, -1, 3, 1}};
            static const LinearOut h1[4] = {{0, 1, 2, 1}, {1, 1, 3, 1}, {0, 1, 2, -1}, {1, 1, 3, -1}};
            const LinearOut(&t)[4] = op.kind == KOP_RY1   ? ry1
                                     : op.kind == KOP_RY2 ? ry2
                                     : op.kind == KOP_RX1 ? rx1
                                     : op.kind == KOP_RX2 ? rx2
                                                          : h1;
            const char *name = op.kind == KOP_RY1   ? "pRY1s"
                               : op.kind == KOP_RY2 ? "pRY2s"
                               : op.kind == KOP_RX1 ? "pRX1s"
                               : op.kind == KOP_RX2 ? "pRX2s"
                                                    : "pH1s";
            const uint32_t cs = linearMask(sg, k, t);
            body << "    dgq::" << name << "<" << k << ", " << hexu(cs) << ">(R, I"
                 << (op.kind == KOP_H1 ? std::string() : ", prog.coef + " + std::to_string(off)) << ");\n";
            return true;
        }
        case KOP_X:
        case KOP_Y:
        case KOP_YC: {
            static const PermOut px[4] = {{2, 1}, {3, 1}, {0, 1}, {1, 1}};
            static const PermOut py[4] = {{3, 1}, {2, -1}, {1, -1}, {0, 1}};
            static const PermOut pyc[4] = {{3, -1}, {2, 1}, {1, 1}, {0, -1}};
            const uint32_t fm = permMask(sg, k, cr, op.kind == KOP_X ? px : op.kind == KOP_Y ? py : pyc, keep);
            body << "    dgq::" << (op.kind == KOP_X ? "pXs" : "pYs") << "<" << k << ", " << cr << "u, " << hexu(fm)
                 << ">(R, I);\n";
            return true;
        }
        case KOP_NEG:
            if (keep) {
                // flips the stored values: right whatever their signs
                body << "    dgq::pNEG<" << (cr ? "true" : "false") << ", " << cr << "u, false>(R, I);\n";
            } else {
                const uint32_t m = slotsOf(cr, 0u);
                sg.negR ^= m;
                sg.negI ^= m;
            }
            return true;
        case KOP_MULI:
        case KOP_MULNI: {
            // +i: (r, i) -> (-i, r); -i: (r, i) -> (i, -r)
            const int mr = op.kind == KOP_MULI ? -1 : 1, mi = -mr;
            const uint32_t slots = slotsOf(cr, 0u);
            uint32_t fm = 0;
            for (int j = 0; j < kRegs; j++) {
                if (!((slots >> j) & 1u)) continue;
                const int sR = ((sg.negR >> j) & 1u) ? -1 : 1, sI = ((sg.negI >> j) & 1u) ? -1 : 1;
                const int tR = mr * sI, tI = mi * sR;  // signs of the swapped stored values
                if (keep) {
                    if (tR * sR < 0) fm |= 1u << (2 * j);
                    if (tI * sI < 0) fm |= 1u << (2 * j + 1);
                } else {
                    sg.negR = tR < 0 ? (sg.negR | (1u << j)) : (sg.negR & ~(1u << j));
                    sg.negI = tI < 0 ? (sg.negI | (1u << j)) : (sg.negI & ~(1u << j));
                }
            }
            body << "    dgq::pSwapRIs<" << cr << "u, " << hexu(fm) << ">(R, I);\n";
            return true;
        }
        case KOP_PH:
            emitPhaseSlots(body, sg, slotsOf(cr, 0u), 0u, "dgq::b2(" + c0 + ")", "dgq::b2(" + c1 + ")",
                           "dgq::b2(-" + c1 + ")");
            return true;
        case KOP_Z2:
            if (op.code < KC_Z2T) {
                // (c + i s) where register bit k is 1, (c - i s) where it is 0
                const uint32_t slots = slotsOf(cr, 0u);
                emitPhaseSlots(body, sg, slots, slots & ~slotsOf(0u, 1u << k), "dgq::b2(" + c0 + ")",
                               "dgq::b2(" + c1 + ")", "dgq::b2(-" + c1 + ")");
            } else if (op.selLoc == 1u) {
                emitPhaseSlots(body, sg, slotsOf(cr, 0u), 0u, "dgq::b2(" + c0 + ")",
                               "make_float2(-" + c1 + ", " + c1 + ")", "make_float2(" + c1 + ", -" + c1 + ")");
            } else {
                body << "    { const bool b_ = " << selExpr(op) << ";\n";
                emitPhaseSlots(body, sg, slotsOf(cr, 0u), 0u, "dgq::b2(" + c0 + ")",
                               "dgq::b2(b_ ? " + c1 + " : -" + c1 + ")", "dgq::b2(b_ ? -" + c1 + " : " + c1 + ")");
                body << "    }\n";
            }
            return true;
        case KOP_PH1:
            if (op.code < KC_PH1T) {
                emitPhaseSlots(body, sg, slotsOf(0u, 1u << k), 0u, "dgq::b2(" + c0 + ")", "dgq::b2(" + c1 + ")",
                               "dgq::b2(-" + c1 + ")");
            } else if (op.selLoc == 1u) {
                emitPhaseSlots(body, sg, 0xFFFFu, 0u, "make_float2(1.0f, " + c0 + ")", "make_float2(0.0f, " + c1 + ")",
                               "make_float2(-0.0f, -" + c1 + ")");
            } else {
                body << "    if (" << selExpr(op) << ") {\n";
                emitPhaseSlots(body, sg, 0xFFFFu, 0u, "dgq::b2(" + c0 + ")", "dgq::b2(" + c1 + ")",
                               "dgq::b2(-" + c1 + ")");
                body << "    }\n";
            }
            return true;
        default:
            return false;
    }
}

void emitOpPaired(std::ostringstream &o, const KOp &op, PairedSigns &sg) {
    const unsigned cr = op.ctrlReg;
    const bool ctrl = cr != 0;
    const bool hi = (op.ctrlLoc & 1u) != 0;  // controlled on address bit 0
    const int off = op.coef;
    const int k = op.k;
    const unsigned clr = op.ctrlLoc & ~1u;
    const bool runtimeCond = clr || op.ctrlCta;
    auto condExpr = [&]() {
        std::ostringstream cond;
        bool any = false;
        if (clr) {
            cond << "((loc & " << clr << "u) == " << clr << "u)";
            any = true;
        }
        if (op.ctrlCta) cond << (any ? " && " : "") << "((cta & " << op.ctrlCta << "u) == " << op.ctrlCta << "u)";
        return cond.str();
    };
    if (hi && op.kind == KOP_NEG) {
        // -1 on the high amplitude of each (controlled) slot: flipping the
        // stored high halves is right whatever their tracked signs
        std::ostringstream body;
        body << "    dgq::pNEG<" << (cr ? "true" : "false") << ", " << cr << "u, true>(R, I);\n";
        if (runtimeCond)
            o << "    if (" << condExpr() << ") {\n" << body.str() << "    }\n";
        else
            o << body.str();
        return;
    }
    if (!hi) {
        std::ostringstream sbody;
        PairedSigns trial = sg;
        if (emitSignedPaired(sbody, op, trial, runtimeCond)) {
            sg = trial;
            if (runtimeCond) {
                o << "    if (" << condExpr() << ") {\n" << sbody.str() << "    }\n";
            } else {
                o << sbody.str();
            }
            return;
        }
    }
    flushSigns(o, sg);
    const std::string tpl3 = std::string(ctrl ? "true" : "false") + ", " + std::to_string(cr) + "u, " + (hi ? "true" : "false");
    std::ostringstream body;
    const bool pairKind = op.kind == KOP_M2R || op.kind == KOP_M2I || op.kind == KOP_M2C || op.kind == KOP_X ||
                          op.kind == KOP_Y || op.kind == KOP_YC || op.kind == KOP_RY1 || op.kind == KOP_RY2 ||
                          op.kind == KOP_RX1 || op.kind == KOP_RX2 || op.kind == KOP_H1 || op.kind == KOP_RN1;
    if (pairKind && k == 4) {
        std::string m[8];
        inSlotMatrix(op, m);
        body << "dgq::pInSlot<" << (ctrl ? "true" : "false") << ", " << cr << "u>(R, I";
        for (int i = 0; i < 8; i++) body << ", " << m[i];
        body << ");";
    } else {
        switch (op.kind) {
            case KOP_M2R: body << "dgq::pM2R<" << k << ", " << tpl3 << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_M2I: body << "dgq::pM2I<" << k << ", " << tpl3 << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_M2C: body << "dgq::pM2C<" << k << ", " << tpl3 << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_X: body << "dgq::pX<" << k << ", " << tpl3 << ">(R, I);"; break;
            case KOP_Y: body << "dgq::pY<" << k << ", " << tpl3 << ">(R, I);"; break;
            case KOP_YC: body << "dgq::pYC<" << k << ", " << tpl3 << ">(R, I);"; break;
            case KOP_RY1: body << "dgq::pRY1<" << k << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_RY2: body << "dgq::pRY2<" << k << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_RX1: body << "dgq::pRX1<" << k << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_RX2: body << "dgq::pRX2<" << k << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_H1: body << "dgq::pH1<" << k << ">(R, I);"; break;
            case KOP_RN1: body << "dgq::pRN1<" << k << ">(R, I, prog.coef + " << off << ");"; break;
            case KOP_NEG: body << "dgq::pNEG<" << tpl3 << ">(R, I);"; break;
            case KOP_MULI: body << "dgq::pMULI<" << tpl3 << ">(R, I);"; break;
            case KOP_MULNI: body << "dgq::pMULNI<" << tpl3 << ">(R, I);"; break;
            case KOP_PH:
                body << "dgq::pPH<" << tpl3 << ">(R, I, dgq::b2(" << cf(off) << "), dgq::b2(" << cf(off + 1) << "));";
                break;
            case KOP_Z2:
                if (op.code < KC_Z2T) {
                    body << "dgq::pZ2R<" << k << ", " << tpl3 << ">(R, I, prog.coef + " << off << ");";
                } else if (op.selLoc == 1u) {
                    body << "dgq::pPH<" << tpl3 << ">(R, I, dgq::b2(" << cf(off) << "), make_float2(-" << cf(off + 1)
                         << ", " << cf(off + 1) << "));";
                } else {
                    body << "{ const bool b_ = " << selExpr(op) << "; dgq::pPH<" << tpl3 << ">(R, I, dgq::b2(" << cf(off)
                         << "), dgq::b2(b_ ? " << cf(off + 1) << " : -" << cf(off + 1) << ")); }";
                }
                break;
            case KOP_PH1:
                if (op.code < KC_PH1T) {
                    body << "dgq::pPH1R<" << k << ">(R, I, prog.coef + " << off << ");";
                } else if (op.selLoc == 1u) {
                    body << "dgq::pPH<false, 0u, false>(R, I, make_float2(1.0f, " << cf(off) << "), make_float2(0.0f, "
                         << cf(off + 1) << "));";
                } else {
                    body << "if (" << selExpr(op) << ") dgq::pPH<false, 0u, false>(R, I, dgq::b2(" << cf(off)
                         << "), dgq::b2(" << cf(off + 1) << "));";
                }
                break;
            case KOP_DENSE: body << "dgq::pDense<" << k << ", " << cr << "u>(R, I, prog.coef + " << off << ");"; break;
            default: break;
        }
    }
    const unsigned cl = op.ctrlLoc & ~1u;
    if (cl || op.ctrlCta) {
        std::ostringstream cond;
        bool any = false;
        if (cl) {
            cond << "((loc & " << cl << "u) == " << cl << "u)";
            any = true;
        }
        if (op.ctrlCta) cond << (any ? " && " : "") << "((cta & " << op.ctrlCta << "u) == " << op.ctrlCta << "u)";
        o << "    if (" << cond.str() << ") { " << body.str() << " }\n";
    } else {
        o << "    " << body.str() << "\n";
    }
}

// scalarKind for the paired form: conditions on address bit 0 (the pair
// inside a slot) select one amplitude of each slot, so those ops are not
// scalars of the thread.
int scalarKindPaired(const KOp &op) {
    if ((op.ctrlLoc & 1u) != 0 || op.ctrlReg != 0) return 0;
    switch (op.kind) {
        case KOP_PH: return 1;
        case KOP_Z2: return op.code >= KC_Z2T && op.selLoc != 1u ? 1 : 0;
        case KOP_PH1: return op.code >= KC_PH1T && op.selLoc != 1u ? 1 : 0;
        case KOP_NEG:
        case KOP_MULI:
        case KOP_MULNI: return 2;
        default: return 0;
    }
}

void emitScalarAccPaired(std::ostringstream &o, const KOp &op) {
    const unsigned cl = op.ctrlLoc & ~1u;
    std::ostringstream cond;
    bool any = false;
    if (cl) {
        cond << "((loc & " << cl << "u) == " << cl << "u)";
        any = true;
    }
    if (op.ctrlCta) {
        cond << (any ? " && " : "") << "((cta & " << op.ctrlCta << "u) == " << op.ctrlCta << "u)";
        any = true;
    }
    const std::string on = any ? cond.str() : std::string("true");
    const int off = op.coef;
    switch (op.kind) {
        case KOP_PH:
            o << "    dgq::jAccPhase(acc_, " << on << ", prog.coef[" << off << "], prog.coef[" << off + 1 << "]);\n";
            break;
        case KOP_Z2:
            o << "    dgq::jAccPhase(acc_, " << on << ", prog.coef[" << off << "], (" << selExpr(op) << ") ? prog.coef["
              << off + 1 << "] : -prog.coef[" << off + 1 << "]);\n";
            break;
        case KOP_PH1:
            o << "    dgq::jAccPhase(acc_, (" << on << ") && (" << selExpr(op) << "), prog.coef[" << off
              << "], prog.coef[" << off + 1 << "]);\n";
            break;
        case KOP_NEG: o << "    dgq::jAccNeg(acc_, " << on << ");\n"; break;
        case KOP_MULI: o << "    dgq::jAccMulI(acc_, " << on << ", 1.0);\n"; break;
        default: o << "    dgq::jAccMulI(acc_, " << on << ", -1.0);\n"; break;
    }
}

// Address bit of tile-local bit l of a paired tile (bits 0..5 are address bits 0..5).
std::string pairedAddr(int l) {
    if (l < kCoalescedBits) return std::to_string(l);
    return "prog.highPos[" + std::to_string(l - kCoalescedBits) + "]";
}

// slot loop helpers: address of this thread's slot j in a layout (gt | rb bits)
void emitPairedLayoutAddressing(std::ostringstream &o, const KPhase &ph, int W, const char *gt, const char *rb) {
    o << "    const uint64_t " << gt << " = cb";
    for (int i = 0; i < W - kRegBits - 1; i++)
        o << " | ((uint64_t) ((tid >> " << i << ") & 1u) << " << pairedAddr(ph.thrPos[i]) << ")";
    o << ";\n    const uint64_t " << rb << "[4] = {";
    for (int b = 0; b < kRegBits; b++) o << (b ? ", " : "") << "1ULL << " << pairedAddr(ph.regPos[b]);
    o << "};\n";
}

}  // namespace

std::string generatePairedSource(const TileProgram &prog, int W) {
    const int T = 1 << (W - kRegBits - 1);
    const int minBlocks = ctasPerSm(T, false);
    std::ostringstream o;
    o << "#include \"jit_prelude.cuh\"\n";
    o << "extern \"C\" __global__ void __launch_bounds__(" << T << ", " << minBlocks
      << ") dgq_sweep(float2 *__restrict__ st, const __grid_constant__ dgq::TileProgram prog) {\n";
    o << "    constexpr int W = " << W << ";\n";
    o << "    constexpr uint32_t T = " << T << "u;\n";
    o << "    extern __shared__ float4 sm[];\n";
    o << "    const uint32_t tid = threadIdx.x, cta = blockIdx.x + prog.ctaOffset;\n";
    o << "    (void) cta;\n    (void) T;\n";
    o << "    float2 R[dgq::kRegs], I[dgq::kRegs];\n";
    o << "    const uint64_t cb = dgq::jCtaBase(prog, cta, W);\n";
    const int np = prog.numPhases;
    const bool firstDirect = np > 0 && prog.phases[0].direct;
    const bool lastDirect = np > 0 && prog.phases[np - 1].direct;
    const std::string fix = "dgq::pFixSlot<" + std::to_string(prog.initKind) + ", " +
                            (prog.hasRestrict ? "true" : "false") + ">(prog, g_, R[j], I[j]);";
    const bool needFix = prog.initKind != INIT_NONE || prog.hasRestrict;
    const std::string load = prog.initKind == INIT_NONE ? "dgq::pLoadSlot(st, g_, R[j], I[j]); " : "";
    // scalar diagonal ops fold into one factor per phase, as in the unpaired
    // form; the sweep's global factor starts the first such phase's factor
    int nPhaseOps[kMaxPhases] = {0}, nSignOps[kMaxPhases] = {0};
    int gPhase = -1;
    for (int p = 0; p < np; p++) {
        for (int k = prog.phases[p].opBegin; k < prog.phases[p].opEnd; k++) {
            const int kind = scalarKindPaired(prog.ops[k]);
            nPhaseOps[p] += kind == 1;
            nSignOps[p] += kind == 2;
        }
        if (gPhase < 0 && nPhaseOps[p] > 0 && (prog.renormIn || prog.hasGlobal)) gPhase = p;
    }
    if (firstDirect) {
        emitPairedLayoutAddressing(o, prog.phases[0], W, "gIn", "rbIn");
        o << "#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) { const uint64_t g_ = dgq::jIdx(gIn, rbIn, j); "
          << load << (needFix ? fix : "") << " }\n";
    } else {
        // canonical layout: slot tid + T * j (lanes on address bits 1..5)
        o << "    const uint64_t gC = cb | ((uint64_t) (tid & 31u) << 1)";
        for (int i = 0; i < W - 10; i++) o << " | ((uint64_t) ((tid >> " << 5 + i << ") & 1u) << prog.highPos[" << 1 + i << "])";
        o << ";\n    const uint64_t rbC[4] = {";
        for (int b = 0; b < kRegBits; b++) o << (b ? ", " : "") << "1ULL << prog.highPos[" << W - 9 + b << "]";
        o << "};\n";
        o << "#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) { const uint64_t g_ = dgq::jIdx(gC, rbC, j); "
          << load << (needFix ? fix : "") << " }\n";
        if (np > 0)
            o << "#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) sm[dgq::swz(tid + T * (uint32_t) j)] = "
                 "make_float4(R[j].x, R[j].y, I[j].x, I[j].y);\n    __syncthreads();\n";
    }
    for (int p = 0; p < np; p++) {
        const KPhase &ph = prog.phases[p];
        const bool readSmem = !(p == 0 && firstDirect);
        const bool writeSmem = !(p == np - 1 && lastDirect);
        o << "  {\n    const uint32_t loc = 0u";
        for (int i = 0; i < W - kRegBits - 1; i++) o << " | (((tid >> " << i << ") & 1u) << " << (int) ph.thrPos[i] << ")";
        o << ";\n    (void) loc;\n    const uint32_t sb = dgq::swz(loc >> 1);\n    (void) sb;\n";
        if (readSmem)
            for (int j = 0; j < kRegs; j++)
                o << "    { const float4 q_ = sm[sb ^ " << ph.regOff[j] << "u]; R[" << j << "] = make_float2(q_.x, q_.y); I["
                  << j << "] = make_float2(q_.z, q_.w); }\n";
        const bool fold = p == gPhase || nPhaseOps[p] >= 2 || (nPhaseOps[p] >= 1 && nSignOps[p] >= 1);
        if (p == gPhase && prog.renormIn)
            o << "    double2 acc_;\n    { const double sc_ = rsqrt(*prog.normIn); acc_ = make_double2(prog.globalRe * "
                 "sc_, prog.globalIm * sc_); }\n";
        else if (p == gPhase)
            o << "    double2 acc_ = make_double2(prog.globalRe, prog.globalIm);\n";
        else if (fold)
            o << "    double2 acc_ = make_double2(1.0, 0.0);\n";
        PairedSigns sg;
        for (int k = ph.opBegin; k < ph.opEnd; k++) {
            if (fold && scalarKindPaired(prog.ops[k]))
                emitScalarAccPaired(o, prog.ops[k]);
            else
                emitOpPaired(o, prog.ops[k], sg);
        }
        if (fold)
            emitGlobalAbsorb(o, sg, "acc_.x", "acc_.y");
        else
            flushSigns(o, sg);
        if (writeSmem) {
            for (int j = 0; j < kRegs; j++)
                o << "    sm[sb ^ " << ph.regOff[j] << "u] = make_float4(R[" << j << "].x, R[" << j << "].y, I[" << j
                  << "].x, I[" << j << "].y);\n";
            o << "    __syncthreads();\n";
        }
        o << "  }\n";
    }
    if (np > 0 && !lastDirect)
        o << "#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) { const float4 q_ = sm[dgq::swz(tid + T * "
             "(uint32_t) j)]; R[j] = make_float2(q_.x, q_.y); I[j] = make_float2(q_.z, q_.w); }\n";
    if (gPhase >= 0) {
        // applied with the factor of phase gPhase
    } else if (prog.renormIn) {
        o << "    { const double sc_ = rsqrt(*prog.normIn); dgq::pGlobal(R, I, prog.globalRe * sc_, prog.globalIm * sc_); }\n";
    } else if (prog.hasGlobal) {
        o << "    dgq::pGlobal(R, I, prog.globalRe, prog.globalIm);\n";
    }
    if (prog.renormOut) o << "    dgq::pNormAccumulate(R, I, prog.normOut);\n";
    if (lastDirect) {
        emitPairedLayoutAddressing(o, prog.phases[np - 1], W, "gOut", "rbOut");
        o << "#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) dgq::pStoreSlot(st, dgq::jIdx(gOut, rbOut, j), R[j], I[j]);\n}\n";
    } else {
        o << "    const uint64_t gS = cb | ((uint64_t) (tid & 31u) << 1)";
        for (int i = 0; i < W - 10; i++)
            o << " | ((uint64_t) ((tid >> " << 5 + i << ") & 1u) << prog.highPos[" << 1 + i << "])";
        o << ";\n    const uint64_t rbS[4] = {";
        for (int b = 0; b < kRegBits; b++) o << (b ? ", " : "") << "1ULL << prog.highPos[" << W - 9 + b << "]";
        o << "};\n#pragma unroll\n    for (int j = 0; j < dgq::kRegs; j++) dgq::pStoreSlot(st, dgq::jIdx(gS, rbS, j), R[j], I[j]);\n}\n";
    }
    return o.str();
}

std::string generateSweepSource(const TileProgram &prog, int W) {
    if (prog.denseK) return std::string();  // dense sweeps run the dense kernel (dense.cu)
    if (prog.paired) return generatePairedSource(prog, W);
    const int T = 1 << (W - kRegBits);
    const int minBlocks = ctasPerSm(T, prog.isSingle != 0);
    std::ostringstream o;
    o << "#include \"jit_prelude.cuh\"\n";
    o << "typedef " << (prog.isSingle ? "float2" : "double2") << " V;\n";
    o << "extern \"C\" __global__ void __launch_bounds__(" << T << ", " << minBlocks
      << ") dgq_sweep(V *__restrict__ st, const __grid_constant__ dgq::TileProgram prog) {\n";
    o << "    constexpr int W = " << W << ";\n";
    o << "    extern __shared__ V sm[];\n";
    o << "    const uint32_t tid = threadIdx.x, cta = blockIdx.x + prog.ctaOffset;\n";
    o << "    (void) cta;\n";
    o << "    V a[dgq::kRegs];\n";
    const int np = prog.numPhases;
    const bool firstDirect = np > 0 && prog.phases[0].direct;
    const bool lastDirect = np > 0 && prog.phases[np - 1].direct;
    // the sweep's global factor (and renormalisation) is one number for all
    // amplitudes: it starts the factor of the first phase with a scalar
    // phase op instead of costing a multiply of its own at the end
    int gPhase = -1;
    if (prog.renormIn || prog.hasGlobal)
        for (int p = 0; p < np && gPhase < 0; p++)
            for (int k = prog.phases[p].opBegin; k < prog.phases[p].opEnd; k++)
                if (scalarKind(prog.ops[k]) == 1) {
                    gPhase = p;
                    break;
                }
    if (firstDirect) {
        emitDirectAddressing(o, prog.phases[0], W, "gIn", "rbIn");
        o << "    dgq::jLoadDirect<" << prog.initKind << ", " << (prog.hasRestrict ? "true" : "false")
          << ">(st, prog, gIn, rbIn, a);\n";
    } else {
        o << "    dgq::jLoad<W, " << prog.initKind << ", " << (prog.hasRestrict ? "true" : "false")
          << ">(st, prog, tid, cta, a);\n";
        if (np > 0) o << "    dgq::jToSmem<W>(sm, tid, a);\n    __syncthreads();\n";
    }
    for (int p = 0; p < np; p++) {
        const KPhase &ph = prog.phases[p];
        const bool readSmem = !(p == 0 && firstDirect);
        const bool writeSmem = !(p == np - 1 && lastDirect);
        o << "  {\n    const uint32_t loc = 0u";
        for (int i = 0; i < W - kRegBits; i++) o << " | (((tid >> " << i << ") & 1u) << " << (int) ph.thrPos[i] << ")";
        o << ";\n    (void) loc;\n    const uint32_t sb = dgq::swz(loc);\n    (void) sb;\n";
        if (readSmem)
            for (int j = 0; j < kRegs; j++) o << "    a[" << j << "] = sm[sb ^ " << ph.regOff[j] << "u];\n";
        const bool fold = p == gPhase || foldScalars(prog, ph.opBegin, ph.opEnd);
        if (p == gPhase && prog.renormIn)
            o << "    double2 acc_;\n    { const double sc_ = rsqrt(*prog.normIn); acc_ = make_double2(prog.globalRe * "
                 "sc_, prog.globalIm * sc_); }\n";
        else if (p == gPhase)
            o << "    double2 acc_ = make_double2(prog.globalRe, prog.globalIm);\n";
        else if (fold)
            o << "    double2 acc_ = make_double2(1.0, 0.0);\n";
        for (int k = ph.opBegin; k < ph.opEnd; k++) {
            if (fold && scalarKind(prog.ops[k]))
                emitScalarAcc(o, prog.ops[k]);
            else
                emitOp(o, prog.ops[k]);
        }
        if (fold) o << "    dgq::jGlobal(a, acc_.x, acc_.y);\n";
        if (writeSmem) {
            for (int j = 0; j < kRegs; j++) o << "    sm[sb ^ " << ph.regOff[j] << "u] = a[" << j << "];\n";
            o << "    __syncthreads();\n";
        }
        o << "  }\n";
    }
    if (np > 0 && !lastDirect) o << "    dgq::jFromSmem<W>(sm, tid, a);\n";
    if (gPhase >= 0) {
        // applied with the factor of phase gPhase
    } else if (prog.renormIn) {
        o << "    { const double sc_ = rsqrt(*prog.normIn); dgq::jGlobal(a, prog.globalRe * sc_, prog.globalIm * sc_); }\n";
    } else if (prog.hasGlobal) {
        o << "    dgq::jGlobal(a, prog.globalRe, prog.globalIm);\n";
    }
    if (prog.renormOut) o << "    dgq::jNormAccumulate(a, prog.normOut);\n";
    if (lastDirect) {
        emitDirectAddressing(o, prog.phases[np - 1], W, "gOut", "rbOut");
        o << "    dgq::jStoreDirect(st, gOut, rbOut, a);\n}\n";
    } else {
        o << "    dgq::jStore<W>(st, prog, tid, cta, a);\n}\n";
    }
    return o.str();
}

bool jitEnabled() {
    static int enabled = -1;
    if (enabled < 0) {
        const char *e = getenv("DGQ_JIT");
        enabled = (e && e[0] == '0') ? 0 : 1;
    }
    return enabled == 1;
}

namespace {

// Driver entry points through the runtime (no link-time dependency on the
// driver library, so the library also loads on hosts without a GPU).
struct Driver {
    CUresult (*moduleLoadData)(CUmodule *, const void *) = nullptr;
    CUresult (*moduleGetFunction)(CUfunction *, CUmodule, const char *) = nullptr;
    CUresult (*funcSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
    CUresult (*launchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                             CUstream, void **, void **) = nullptr;
    CUresult (*getErrorString)(CUresult, const char **) = nullptr;
    bool ok = false;
};

const Driver &driver() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, []() {
        auto get = [](const char *name, void **fn) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *fn != nullptr;
        };
        d.ok = get("cuModuleLoadData", (void **) &d.moduleLoadData) &&
               get("cuModuleGetFunction", (void **) &d.moduleGetFunction) &&
               get("cuFuncSetAttribute", (void **) &d.funcSetAttribute) &&
               get("cuLaunchKernel", (void **) &d.launchKernel) &&
               get("cuGetErrorString", (void **) &d.getErrorString);
    });
    return d;
}

// Driver calls act on the calling thread's current context. A host thread
// whose first CUDA work in this library is a module load or a launch of a
// specialised kernel (a serving worker reusing a register, say) has none
// yet: bind the runtime's primary context of the current device first
// (cudaSetDevice makes it current), once per thread.
bool ensureContext() {
    thread_local bool bound = false;
    if (bound) return true;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return false;
    bound = true;
    return true;
}

// Loaded kernels, per source and device: a function belongs to the context
// of the device it was loaded on (a sharded register on several devices
// loads each source once per device).
struct CacheEntry {
    std::string source;
    int device;
    CUmodule module;
    CUfunction fn;
};

int currentDevice() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    return dev;
}

std::mutex g_cacheMutex;
std::unordered_map<size_t, std::vector<CacheEntry>> g_cache;

CUfunction cacheFind(const std::string &src) {
    std::lock_guard<std::mutex> lk(g_cacheMutex);
    const int dev = currentDevice();
    auto it = g_cache.find(std::hash<std::string>()(src));
    if (it == g_cache.end()) return nullptr;
    for (const auto &e : it->second)
        if (e.device == dev && e.source == src) return e.fn;
    return nullptr;
}

bool compileOne(const std::string &src, std::vector<char> &cubin, std::string &log) {
    nvrtcProgram prog;
    const char *headers[2] = {kTileProgramSource, kJitPreludeSource};
    const char *names[2] = {"tile_program.h", "jit_prelude.cuh"};
    if (nvrtcCreateProgram(&prog, src.c_str(), "dgq_sweep.cu", 2, headers, names) != NVRTC_SUCCESS) {
        log = "nvrtcCreateProgram failed";
        return false;
    }
    const char *opts[] = {"-arch=sm_100a", "--std=c++17", "-default-device", "-lineinfo"};
    const nvrtcResult r = nvrtcCompileProgram(prog, 4, opts);
    size_t logSize = 0;
    nvrtcGetProgramLogSize(prog, &logSize);
    if (logSize > 1) {
        log.resize(logSize);
        nvrtcGetProgramLog(prog, &log[0]);
    }
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return false;
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin.resize(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    return true;
}

}  // namespace

namespace {

// Compiled but not yet loaded kernels (from background compiles), and the
// background compile queue. Heap-allocated and never destroyed, so a
// compile still running at process exit touches no destroyed object.
// Background compiles run on a pool of worker threads that wait for work on
// a condition variable; at process exit the pool is stopped and JOINED, so
// no worker is inside NVRTC, or still tearing down its thread state, while
// the process destroys NVRTC's and the CUDA runtime's globals.
struct CubinCache {
    std::mutex mu;
    std::condition_variable work;
    std::unordered_map<size_t, std::vector<std::pair<std::string, std::vector<char>>>> cubins;
    std::vector<std::string> queue;
    std::unordered_map<size_t, int> queued;  // source hash -> pending count
    std::vector<std::thread> pool;
    int alive = 0;  // workers that have not returned
    std::condition_variable gone;
    bool stopping = false;
};
CubinCache &cubinCache() {
    static CubinCache *c = new CubinCache();
    return *c;
}

bool cubinFind(const std::string &src, std::vector<char> *out) {
    CubinCache &c = cubinCache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.cubins.find(std::hash<std::string>()(src));
    if (it == c.cubins.end()) return false;
    for (const auto &e : it->second)
        if (e.first == src) {
            if (out) *out = e.second;
            return true;
        }
    return false;
}

void backgroundWorker() {
    CubinCache &c = cubinCache();
    for (;;) {
        std::string src;
        {
            std::unique_lock<std::mutex> lk(c.mu);
            c.work.wait(lk, [&]() { return c.stopping || !c.queue.empty(); });
            if (c.stopping) {
                c.alive--;
                c.gone.notify_all();
                return;
            }
            src = std::move(c.queue.back());
            c.queue.pop_back();
        }
        std::vector<char> cubin;
        std::string log;
        const bool ok = compileOne(src, cubin, log);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t h = std::hash<std::string>()(src);
        if (ok) c.cubins[h].emplace_back(src, std::move(cubin));
        if (--c.queued[h] <= 0) c.queued.erase(h);
    }
}

}  // namespace

CUfunction jitFindLoaded(const std::string &source) { return cacheFind(source); }

bool jitAllReady(const std::vector<std::string> &sources) {
    for (const auto &src : sources)
        if (!cacheFind(src) && !cubinFind(src, nullptr)) return false;
    return true;
}

// Drops the queue, lets compiles in progress finish (30 s at most) and joins
// the workers. Called by dgq_shutdown (the Python binding calls it from its
// exit hook, while NVRTC and the CUDA runtime are still intact) and, as a
// fallback, from a C atexit handler.
void jitStopBackground() {
    CubinCache &c = cubinCache();
    std::vector<std::thread> pool;
    bool all = false;
    {
        std::unique_lock<std::mutex> lk(c.mu);
        c.stopping = true;
        c.queue.clear();
        c.work.notify_all();
        all = c.gone.wait_for(lk, std::chrono::seconds(30), [&]() { return c.alive == 0; });
        pool.swap(c.pool);
    }
    for (auto &t : pool) {
        if (!t.joinable()) continue;
        if (all)
            t.join();
        else
            t.detach();
    }
}

static void stopBackgroundCompiles() { jitStopBackground(); }

void jitCompileInBackground(const std::vector<std::string> &sources) {
    static std::once_flag registered;
    std::call_once(registered, []() { std::atexit(stopBackgroundCompiles); });
    CubinCache &c = cubinCache();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.stopping) return;
    for (const auto &src : sources) {
        if (cacheFind(src)) continue;
        const size_t h = std::hash<std::string>()(src);
        bool have = false;
        auto it = c.cubins.find(h);
        if (it != c.cubins.end())
            for (const auto &e : it->second) have = have || e.first == src;
        if (have || c.queued.count(h)) continue;
        c.queued[h]++;
        c.queue.push_back(src);
    }
    unsigned hw = std::thread::hardware_concurrency();
    const size_t maxWorkers = std::max(1u, std::min(8u, hw / 2));
    while (c.pool.size() < maxWorkers && c.queue.size() > c.pool.size()) {
        c.alive++;
        c.pool.emplace_back(backgroundWorker);
    }
    c.work.notify_all();
}

bool jitCompileOnly(const std::string &src, std::vector<char> &cubin, std::string &log) {
    return compileOne(src, cubin, log);
}

bool jitGetKernels(const std::vector<std::string> &sources, std::vector<CUfunction> &out, JitStats *stats,
                   std::string *err) {
    const auto t0 = std::chrono::steady_clock::now();
    out.assign(sources.size(), nullptr);
    std::vector<size_t> todo;
    // identical sources in one batch compile once
    std::unordered_map<std::string, size_t> firstOf;
    std::vector<size_t> dupOf(sources.size(), (size_t) -1);
    int reused = 0;
    for (size_t i = 0; i < sources.size(); i++) {
        out[i] = cacheFind(sources[i]);
        if (out[i]) {
            reused++;
            continue;
        }
        auto it = firstOf.find(sources[i]);
        if (it != firstOf.end()) {
            dupOf[i] = it->second;
            continue;
        }
        firstOf[sources[i]] = i;
        todo.push_back(i);
    }
    std::vector<std::vector<char>> cubins(sources.size());
    std::vector<std::string> logs(sources.size());
    std::vector<char> ok(sources.size(), 0);
    std::atomic<int> fromBackground{0};
    if (!todo.empty()) {
        unsigned hw = std::thread::hardware_concurrency();
        if (hw == 0) hw = 4;
        const unsigned nthreads = std::min<unsigned>(hw, (unsigned) todo.size());
        std::atomic<size_t> next{0};
        auto worker = [&]() {
            for (size_t t; (t = next.fetch_add(1)) < todo.size();) {
                const size_t i = todo[t];
                if (cubinFind(sources[i], &cubins[i])) {
                    ok[i] = 1;
                    fromBackground++;
                    continue;
                }
                ok[i] = compileOne(sources[i], cubins[i], logs[i]) ? 1 : 0;
            }
        };
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nthreads; t++) pool.emplace_back(worker);
        worker();
        for (auto &th : pool) th.join();
    }
    bool allOk = true;
    const Driver &drv = driver();
    if (!todo.empty() && !drv.ok) {
        if (err) *err = "CUDA driver entry points unavailable";
        return false;
    }
    if (!todo.empty() && !ensureContext()) {
        if (err) *err = "no CUDA device context for this thread";
        return false;
    }
    for (size_t i : todo) {
        if (!ok[i]) {
            if (err) *err = "NVRTC compile failed: " + logs[i].substr(0, 2000);
            allOk = false;
            continue;
        }
        CUmodule mod = nullptr;
        CUfunction fn = nullptr;
        CUresult r = drv.moduleLoadData(&mod, cubins[i].data());
        if (r == CUDA_SUCCESS) r = drv.moduleGetFunction(&fn, mod, "dgq_sweep");
        if (r != CUDA_SUCCESS) {
            const char *msg = nullptr;
            drv.getErrorString(r, &msg);
            if (err) *err = std::string("loading a specialised kernel failed: ") + (msg ? msg : "?");
            allOk = false;
            continue;
        }
        out[i] = fn;
        std::lock_guard<std::mutex> lk(g_cacheMutex);
        g_cache[std::hash<std::string>()(sources[i])].push_back({sources[i], currentDevice(), mod, fn});
    }
    for (size_t i = 0; i < sources.size(); i++)
        if (dupOf[i] != (size_t) -1) out[i] = out[dupOf[i]];
    if (stats) {
        // kernels compiled in the background and only loaded here count as reused
        stats->compiled = (int) todo.size() - fromBackground.load();
        stats->reused = reused + fromBackground.load();
        stats->compileMillis = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return allOk;
}

cudaError_t launchJitSweep(CUfunction fn, void *st, int W, const TileProgram &prog, cudaStream_t s) {
    // paired complex64 form: 16 slots of 2 amplitudes per thread
    const int T = 1 << (W - kRegBits - (prog.paired ? 1 : 0));
    const unsigned smem = (unsigned) ((prog.isSingle ? sizeof(float2) : sizeof(double2)) << W);
    // one attribute call per function: cheap and idempotent
    const Driver &drv = driver();
    if (!drv.ok) return cudaErrorNotSupported;
    if (!ensureContext()) return cudaErrorInvalidDevice;
    CUresult r = drv.funcSetAttribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int) smem);
    if (r != CUDA_SUCCESS) return cudaErrorLaunchFailure;
    const unsigned grid = prog.ctaCount ? prog.ctaCount : 1u << (prog.numBits - W);
    void *args[2] = {(void *) &st, (void *) &prog};
    r = drv.launchKernel(fn, grid, 1, 1, (unsigned) T, 1, 1, smem, (CUstream) s, args, nullptr);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

}  // namespace dgq
