// api.cpp -- the QuEST C API of libdgq and the per-register engine behind it.
//
// Front end (validation, API -> gate encoding) follows dgQuEST's
// src/QuEST.c:30-458, src/QuEST_validation.c and
// src/cpp/QuEST_distributed.cpp:106-364. The engine replaces dgQuEST's
// orchestrator (src/cpp/QuEST_backend_distributed.cpp): the state is
// resident in HBM, so there are no tasks, pages or MPI exchanges; pending
// gates are planned into tile sweeps and launched on the register's stream
// when a read-out needs them (QuEST_distributed.cpp:106-116).
#include <sys/time.h>
#include <unistd.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "QuEST.h"
#include "dgq.h"
#include "dag.h"
#include "fuse.h"
#include "ir.h"
#include "jit.h"
#include "kernels.h"
#include "planner.h"
#include "qureg_state.h"
#include "rng.h"

using dgq::Gate;


// ====================================================================
// errors (codes and messages of src/QuEST_validation.c:19-80)
// ====================================================================
namespace {

enum ErrorCode {
    E_SUCCESS = 0,
    E_INVALID_NUM_QUBITS,
    E_INVALID_TARGET_QUBIT,
    E_INVALID_CONTROL_QUBIT,
    E_INVALID_STATE_INDEX,
    E_INVALID_NUM_AMPS,
    E_INVALID_OFFSET_NUM_AMPS,
    E_TARGET_IS_CONTROL,
    E_TARGET_IN_CONTROLS,
    E_TARGETS_NOT_UNIQUE,
    E_INVALID_NUM_CONTROLS,
    E_NON_UNITARY_MATRIX,
    E_NON_UNITARY_COMPLEX_PAIR,
    E_ZERO_VECTOR,
    E_SYS_TOO_BIG_TO_PRINT,
    E_COLLAPSE_STATE_ZERO_PROB,
    E_INVALID_QUBIT_OUTCOME,
    E_CANNOT_OPEN_FILE,
    E_SECOND_ARG_MUST_BE_STATEVEC,
    E_MISMATCHING_QUREG_DIMENSIONS,
    E_MISMATCHING_QUREG_TYPES,
    E_DEFINED_ONLY_FOR_STATEVECS,
    E_DEFINED_ONLY_FOR_DENSMATRS,
    E_INVALID_PROB,
    E_UNNORM_PROBS,
    E_INVALID_ONE_QUBIT_DEPHASE_PROB,
    E_INVALID_TWO_QUBIT_DEPHASE_PROB,
    E_INVALID_ONE_QUBIT_DEPOL_PROB,
    E_INVALID_TWO_QUBIT_DEPOL_PROB,
    // codes of this library (no counterpart in dgQuEST)
    E_INVALID_NUM_TARGETS = 100,
    E_SYS_TOO_BIG_FOR_DEVICE = 101,
    E_UNSUPPORTED = 102,
    E_CUDA = 103,
    E_INVALID_ARGUMENT = 104,
};

const char *errorMessage(int code) {
    switch (code) {
        case E_INVALID_NUM_QUBITS: return "Invalid number of qubits. Must create >0.";
        case E_INVALID_TARGET_QUBIT: return "Invalid target qubit. Note qubits are zero indexed.";
        case E_INVALID_CONTROL_QUBIT: return "Invalid control qubit. Note qubits are zero indexed.";
        case E_INVALID_STATE_INDEX: return "Invalid state index. Must be >=0 and <2^numQubits.";
        case E_INVALID_NUM_AMPS: return "Invalid number of amplitudes. Must be >=0 and <=2^numQubits.";
        case E_INVALID_OFFSET_NUM_AMPS: return "More amplitudes given than exist in the statevector from the given starting index.";
        case E_TARGET_IS_CONTROL: return "Control qubit cannot equal target qubit.";
        case E_TARGET_IN_CONTROLS: return "Control qubits cannot include target qubit.";
        case E_TARGETS_NOT_UNIQUE: return "The two target qubits must be unique.";
        case E_INVALID_NUM_CONTROLS: return "Invalid number of control qubits. Must be >0 and <numQubits.";
        case E_NON_UNITARY_MATRIX: return "Matrix is not unitary.";
        case E_NON_UNITARY_COMPLEX_PAIR: return "Compact matrix formed by given complex numbers is not unitary.";
        case E_ZERO_VECTOR: return "Invalid axis vector. Must be non-zero.";
        case E_COLLAPSE_STATE_ZERO_PROB: return "Can't collapse to state with zero probability.";
        case E_INVALID_QUBIT_OUTCOME: return "Invalid measurement outcome -- must be either 0 or 1.";
        case E_DEFINED_ONLY_FOR_STATEVECS: return "Operation valid only for state-vectors.";
        case E_DEFINED_ONLY_FOR_DENSMATRS: return "Operation valid only for density matrices.";
        case E_INVALID_PROB: return "Probabilities must be in [0, 1].";
        case E_INVALID_ONE_QUBIT_DEPHASE_PROB:
            return "The probability of a single qubit dephase error cannot exceed 1/2, which maximally mixes.";
        case E_INVALID_TWO_QUBIT_DEPHASE_PROB:
            return "The probability of a two-qubit qubit dephase error cannot exceed 3/4, which maximally mixes.";
        case E_INVALID_ONE_QUBIT_DEPOL_PROB:
            return "The probability of a single qubit depolarising error cannot exceed 3/4, which maximally mixes.";
        case E_INVALID_TWO_QUBIT_DEPOL_PROB:
            return "The probability of a two-qubit depolarising error cannot exceed 15/16, which maximally mixes.";
        case E_MISMATCHING_QUREG_DIMENSIONS: return "Dimensions of the qubit registers don't match.";
        case E_MISMATCHING_QUREG_TYPES:
            return "Registers must both be state-vectors or both be density matrices.";
        case E_SECOND_ARG_MUST_BE_STATEVEC: return "Second argument must be a state-vector.";
        case E_INVALID_NUM_TARGETS: return "Invalid number of target qubits. Must be >0 and <=numQubits, and unique.";
        case E_SYS_TOO_BIG_FOR_DEVICE: return "The state-vector does not fit in free GPU memory.";
        case E_UNSUPPORTED: return "Operation not supported by this library.";
        case E_CUDA: return "CUDA runtime error.";
        case E_INVALID_ARGUMENT: return "Invalid argument.";
        default: return "Unknown error.";
    }
}

std::atomic<int> g_errMode{DGQ_ERRORS_EXIT};
// the last recorded error is per thread: registers driven from several host
// threads (the serving loop) each see the errors of their own calls
thread_local int g_lastError = 0;
thread_local std::string g_lastMessage;
thread_local int64_t g_errorCount = 0;  // errors raised in record mode by this thread
std::atomic<int64_t> g_launches{0};
dgq::Mt19937 g_rng;

// Raises an error: exits (default) or records it. Always returns false so
// that callers can write `if (!ok) return ...`.
bool raise(int code, const char *func, const char *detail = nullptr) {
    std::string msg = std::string("QuEST Error in function ") + func + ": " + errorMessage(code);
    if (detail && *detail) msg += std::string(" (") + detail + ")";
    if (g_errMode == DGQ_ERRORS_EXIT) {
        printf("!!!\n%s\n!!!\nexiting..\n", msg.c_str());
        fflush(stdout);
        exit(code);
    }
    g_lastError = code;
    g_errorCount++;
    g_lastMessage = msg;
    return false;
}

bool cudaOk(cudaError_t e, const char *func) {
    if (e == cudaSuccess) return true;
    return raise(E_CUDA, func, cudaGetErrorString(e));
}

double nowMillis() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

namespace dgq {
// Error reporting for entry points defined in other translation units:
// follows the library's error mode (exit with QuEST's message, or record).
bool raiseExternal(int code, const char *func, const char *detail) { return raise(code, func, detail); }
}  // namespace dgq

// ====================================================================
// environment and register state
// ====================================================================
struct QuESTEnvValue {
    int device = 0;
};


namespace {

QuregState *stateOf(const Qureg &q) { return q.state; }

size_t ampBytes(const QuregState &s) { return s.single ? sizeof(float2) : sizeof(double2); }

void resetMapping(QuregState &s) {
    for (int i = 0; i < 64; i++) {
        s.l2v[i] = i;
        s.v2l[i] = i;
    }
}

u64 toVirtualMask(const QuregState &s, u64 logicalMask) {
    u64 v = 0;
    for (int b = 0; b < s.numQubits; b++)
        if ((logicalMask >> b) & 1ULL) v |= 1ULL << s.l2v[b];
    return v;
}

uint64_t toVirtualIndex(const QuregState &s, uint64_t logical) {
    uint64_t v = 0;
    for (int b = 0; b < s.numQubits; b++) v |= ((logical >> b) & 1ULL) << s.l2v[b];
    return v;
}

// ---------------------------------------------------------------- cost model
// Recast of dgQuEST's time predictor (src/cpp/time_predictor.cpp:201-395):
// dgQuEST predicts T(K) = sum over sections of the calculation time
// (processTime + sum of per-gate times per fused gate) plus transfers, with
// per-gate times measured on its GPU, and takes the argmin over K. Here the
// state stays in HBM and the argmin is over the tile width W; a plan's time
// is a cost per sweep (one pass of the state through HBM) plus a cost per
// register phase (one pass of the tile through shared memory and the FP64
// pipes), both per amplitude. The two rates are fitted to sweep-kernel times
// measured on B200 (complex128, 2^28 and 2^30 amplitudes; random layers of
// depth 8 and 20, a 4-row sqrt-gate grid, GHZ+QFT and a hardware-efficient
// ansatz, each at W = 10, 11, 12): 2.6 ms per sweep and 1.8 ms per phase
// for 2^30 amplitudes. For circuits of equal gates the FP64 work is the same
// at every W, so it lives in those two rates.
// The rates can be replaced by a calibration of this GPU
// (dgquest_b200/calibrate.py measures them; dgq_setCostModel installs them,
// dgq_loadCostModel or DGQ_COST_FILE reads the file it writes).
// The predictor also chooses the form of a plan (dgq_setDenseFusion(q, -1),
// the default): register-phase tiles, or the gates fused into dense blocks of
// K = 5, 6 or 7 qubits, each block one dense sweep. A dense sweep costs a
// fixed time per block per amplitude (denseMs, ms per block per 2^30
// amplitudes) for three variants: complex128 SIMT, complex64 SIMT and
// complex64 on the tensor cores (K = 6 only). Built-in: the K = 6 figures
// measured on B200 at 30 qubits (58.1, 37.4 and 14.8 ms), K = 5 and 7 scaled
// by 2^K (the SIMT dense kernel is compute-bound, 8 x 2^K flops per
// amplitude). Tiles on a complex64 register (the paired form) cost
// c64TileFactor times the complex128 prediction (measured: 77 of 140 ms on
// the 30-qubit circuit). A dense form is taken when its prediction is below
// denseMargin times the tile form's.
enum DenseVariant { DV_F64 = 0, DV_C64 = 1, DV_C64_TC = 2 };
// complex64 dense 6-qubit sweeps on the tensor cores (dgq_setTensorCores)
std::atomic<int> g_tensorCores{1};
struct CostModel {
    double sweepSecondsPerAmp = 2.6e-3 / 1073741824.0;
    double phaseSecondsPerAmp = 1.8e-3 / 1073741824.0;
    double launchSeconds = 3e-6;
    double denseMs[3][3] = {{29.05, 58.1, 116.2}, {18.7, 37.4, 74.8}, {0.0, 14.8, 0.0}};  // [variant][K - 5]
    double c64TileFactor = 0.55;
    double denseMargin = 0.8;
};

std::mutex g_costMutex;
CostModel g_cost;
bool g_costFileTried = false;

const char *kDenseVariantName[3] = {"f64", "c64", "c64tc"};

// Optional lines of a cost file: "dense_ms_per_2p30_<f64|c64|c64tc>_k<K> <ms>"
// and "c64_tile_factor <x>"; applied to `cm` (other keys are ignored).
void readCostFileExtras(const char *path, CostModel &cm) {
    FILE *f = fopen(path, "r");
    if (!f) return;
    char line[256];
    while (fgets(line, sizeof(line), f)) {
        char key[64];
        double v = 0.0;
        if (line[0] == '#' || sscanf(line, "%63s %lf", key, &v) != 2 || !std::isfinite(v) || v < 0.0) continue;
        if (!strcmp(key, "c64_tile_factor") && v > 0.0) cm.c64TileFactor = v;
        for (int var = 0; var < 3; var++)
            for (int K = 5; K <= 7; K++) {
                char name[64];
                snprintf(name, sizeof name, "dense_ms_per_2p30_%s_k%d", kDenseVariantName[var], K);
                if (!strcmp(key, name)) cm.denseMs[var][K - 5] = v;
            }
    }
    fclose(f);
}

// "dgq_cost 1" then "sweep_ms_per_2p30 <x>" and "phase_ms_per_2p30 <y>"
// lines (any order, '#' comments); returns false on a malformed file.
bool readCostFile(const char *path, double &sweepMs, double &phaseMs) {
    FILE *f = fopen(path, "r");
    if (!f) return false;
    char line[256];
    bool header = false, haveS = false, haveP = false;
    while (fgets(line, sizeof(line), f)) {
        char key[64];
        double v = 0.0;
        if (line[0] == '#' || line[0] == '\n') continue;
        if (sscanf(line, "%63s %lf", key, &v) != 2) continue;
        if (!strcmp(key, "dgq_cost") && v == 1.0) header = true;
        if (!strcmp(key, "sweep_ms_per_2p30")) {
            sweepMs = v;
            haveS = true;
        }
        if (!strcmp(key, "phase_ms_per_2p30")) {
            phaseMs = v;
            haveP = true;
        }
    }
    fclose(f);
    return header && haveS && haveP && sweepMs > 0.0 && phaseMs >= 0.0 && std::isfinite(sweepMs) &&
           std::isfinite(phaseMs);
}

CostModel costModel() {
    std::lock_guard<std::mutex> lk(g_costMutex);
    if (!g_costFileTried) {
        g_costFileTried = true;
        const char *path = getenv("DGQ_COST_FILE");
        double sw = 0.0, ph = 0.0;
        if (path && readCostFile(path, sw, ph)) {
            g_cost.sweepSecondsPerAmp = sw * 1e-3 / 1073741824.0;
            g_cost.phaseSecondsPerAmp = ph * 1e-3 / 1073741824.0;
            readCostFileExtras(path, g_cost);
        }
    }
    return g_cost;
}

double predictPlanSeconds(const std::vector<Gate> &gates, int numBits, int W, const dgq::MatrixPool &pool,
                          int lookahead) {
    const CostModel cm = costModel();
    std::vector<dgq::BlockPlan> blocks = dgq::planBlocks(gates, numBits, W, nullptr, dgq::kCoalescedBits, lookahead);
    const double amps = std::ldexp(1.0, numBits);
    std::vector<dgq::TileProgram> progs;
    dgq::PlanStats st;
    dgq::SweepHeader h;
    std::string err;
    for (const auto &b : blocks) {
        progs.clear();
        if (!dgq::encodeBlock(b, numBits, numBits, W, pool, h, progs, &st, &err)) return 1e30;
    }
    return st.sweeps * (amps * cm.sweepSecondsPerAmp + cm.launchSeconds) + st.phases * amps * cm.phaseSecondsPerAmp;
}

int chooseTileBits(QuregState &s) {
    // complex64 tiles could reach 2^13 amplitudes in 64 KiB, but at 16
    // amplitudes a thread that is one 512-thread CTA per SM, which hides no
    // latency; 2^12 keeps three CTAs per SM (override: dgq_setTileBits(13))
    // a set width of 13 is honoured in either precision (complex128: 128 KiB
    // of shared memory, one 512-thread CTA per SM, specialised kernels only)
    const int hi = std::min(s.tileBitsSetting >= dgq::kMaxTileBitsC64 ? dgq::kMaxTileBitsC64 : dgq::kMaxTileBitsF64,
                            s.numBits);
    const int lo = dgq::kMinTileBits;
    s.planLookahead = -1;
    if (s.tileBitsSetting > 0) return std::max(lo, std::min(hi, s.tileBitsSetting));
    if (const char *env = getenv("DGQ_TILE_BITS")) {
        const int w = atoi(env);
        if (w > 0) return std::max(lo, std::min(hi, w));
    }
    // candidates: every width, with and without lookahead block selection on
    // registers large enough for it; planned concurrently, one host thread each
    struct Cand {
        int W, lookahead;
        double t;
    };
    std::vector<Cand> cands;
    for (int W = lo; W <= hi; W++) {
        if (dgq::lookaheadBySize(s.numBits)) cands.push_back({W, 1, 1e300});
        cands.push_back({W, 0, 1e300});
    }
    {
        std::vector<std::thread> th;
        for (size_t i = 1; i < cands.size(); i++)
            th.emplace_back([&, i]() {
                cands[i].t = predictPlanSeconds(s.pending, s.numBits, cands[i].W, s.pool, cands[i].lookahead);
            });
        cands[0].t = predictPlanSeconds(s.pending, s.numBits, cands[0].W, s.pool, cands[0].lookahead);
        for (auto &x : th) x.join();
    }
    // the smaller tile, then lookahead, on ties
    int best = std::min(hi, 12);
    double bestT = 1e300;
    s.planLookahead = -1;
    for (const Cand &c : cands) {
        if (c.t < bestT) {
            bestT = c.t;
            best = c.W;
            s.planLookahead = c.lookahead;
        }
    }
    s.predictedTileSeconds = bestT;
    return best;
}

// Predicted time of the dense-block form with K-qubit blocks: the blocks'
// dense sweeps plus the tile sweeps of the gates that touch more than K
// qubits and pass through. *blocksOut: the number of blocks.
// bound > 0: stop counting blocks once they cost more than bound seconds
// (*stopped is set and the result is the cost of the blocks counted).
double predictDenseSeconds(const QuregState &s, int K, int *blocksOut, double bound, bool *stopped) {
    const CostModel cm = costModel();
    const int var = !s.single ? DV_F64 : (K == 6 && g_tensorCores.load() ? DV_C64_TC : DV_C64);
    const double rate = cm.denseMs[var][K - 5] > 0.0 ? cm.denseMs[var][K - 5] : cm.denseMs[DV_C64][K - 5];
    const double amps = std::ldexp(1.0, s.numBits);
    const double perBlock = rate * 1e-3 * amps / 1073741824.0 + cm.launchSeconds;
    const int maxBlocks = bound > 0.0 ? (int) std::min(1e6, std::floor(bound / perBlock)) + 1 : 0;
    dgq::MatrixPool pool = s.pool;
    int blocks = 0;
    bool cut = false;
    const std::vector<Gate> fused = dgq::fuseDenseBlocks(s.pending, s.numBits, K, pool, &blocks, maxBlocks, &cut);
    if (blocksOut) *blocksOut = blocks;
    if (stopped) *stopped = cut;
    double t = blocks * perBlock;
    if (cut) return t;
    std::vector<Gate> rest;
    for (const Gate &g : fused)
        if (!(g.type == dgq::OP_MULTI_UNITARY && g.numMultiTargets > dgq::kRegBits)) rest.push_back(g);
    if (!rest.empty()) {
        const double tt = predictPlanSeconds(rest, s.numBits, std::min(12, s.numBits), pool, -1);
        t += s.single ? tt * cm.c64TileFactor : tt;
    }
    return t;
}

// The predictor's choice of form for the pending gates (dgq_setDenseFusion
// -1): 0 for register-phase tiles, else the dense block width K. Fills the
// plan statistics' predictions (ms) for every candidate.
int chooseForm(QuregState &s) {
    const CostModel cm = costModel();
    // the tile form first: its prediction bounds the dense estimates, whose
    // block counting stops as soon as they cannot win
    s.formTileBits = chooseTileBits(s);
    s.formLookahead = s.planLookahead;
    double tile = s.predictedTileSeconds;
    if (s.single) tile *= cm.c64TileFactor;
    s.stats.predictedTileMs = tile * 1e3;
    double dense[3] = {0.0, 0.0, 0.0};
    int blocks[3] = {0, 0, 0};
    bool cut[3] = {false, false, false};
    {
        std::vector<std::thread> th;
        for (int K = 5; K <= 7; K++)
            if (s.numBits >= K + 2)
                th.emplace_back([&, K]() {
                    dense[K - 5] = predictDenseSeconds(s, K, &blocks[K - 5], tile * cm.denseMargin, &cut[K - 5]);
                });
        for (auto &x : th) x.join();
    }
    s.stats.denseBound = 0;
    int best = 0;
    double bestT = tile * cm.denseMargin;
    for (int K = 5; K <= 7; K++) {
        s.stats.predictedDenseMs[K - 5] = dense[K - 5] * 1e3;
        if (cut[K - 5]) s.stats.denseBound |= 1 << (K - 5);
        if (s.numBits >= K + 2 && blocks[K - 5] > 0 && !cut[K - 5] && dense[K - 5] < bestT) {
            bestT = dense[K - 5];
            best = K;
        }
    }
    return best;
}

// ---------------------------------------------------------------- execution
// Registers with at least this many address bits get runtime-specialised
// sweep kernels (DGQ_JIT_MIN_BITS overrides): below it a sweep takes
// microseconds and the generic tile kernel beats a compile.
std::atomic<int> g_jitMinBits{-1};

// The complex64 paired form (DGQ_F32_PAIRED=0 turns it off).
bool pairedEnabled() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("DGQ_F32_PAIRED");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// Tile bits of the paired form, the in-slot bit included: 2^12 slots of two
// amplitudes (64 KiB of shared memory, 256 threads), or a set width 10..14.
int pairedTileBits(const QuregState &s) {
    int W = (s.tileBitsSetting >= 10 && s.tileBitsSetting <= dgq::kMaxTileBits) ? s.tileBitsSetting : 13;
    return std::min(W, s.numBits);
}

int jitMinBits() {
    int v = g_jitMinBits.load();
    if (v < 0) {
        const char *e = getenv("DGQ_JIT_MIN_BITS");
        v = e ? atoi(e) : 22;
        g_jitMinBits.store(v);
    }
    return v;
}

}  // namespace

namespace dgq {

int buildPrograms(QuregState &s, int W, std::vector<TileProgram> &out, PlanStats &st, std::string &err,
                  bool paired, const std::function<bool(size_t)> &emit) {
    // hands the programs from index `from` on to emit
    auto emitted = [&](size_t from) -> bool {
        if (!emit) return true;
        for (size_t i = from; i < out.size(); i++)
            if (!emit(i)) return false;
        return true;
    };
    out.clear();
    SweepHeader h;
    if (s.initPending) {
        h.initKind = s.initKind;
        h.initIndex = s.initIndex;
        h.initAmp = s.initAmp;
    } else if (s.restrictActive) {
        h.hasRestrict = true;
        h.restrictMask = s.rMask;
        h.restrictValue = s.rValue;
        h.restrictScale = s.rScale;
    }
    // unitaries wider than a register phase are sweeps of their own: plan
    // the gates between them as usual
    s.denseHost.clear();
    bool first = true;
    std::vector<Gate> seg;
    auto planSegment = [&]() -> int {
        if (seg.empty()) return 0;
        int code = 0;
        const bool complete = planBlocksEach(seg, s.numBits, W, paired ? kCoalescedBits + 1 : kCoalescedBits,
                                             [&](BlockPlan &b) {
                                                 SweepHeader hb = first ? h : SweepHeader();
                                                 const size_t from = out.size();
                                                 if (!encodeBlock(b, s.numBits, s.numQubits, W, s.pool, hb, out, &st,
                                                                  &err, paired)) {
                                                     code = E_UNSUPPORTED;
                                                     return false;
                                                 }
                                                 first = false;
                                                 if (!emitted(from)) {
                                                     code = -1;
                                                     return false;
                                                 }
                                                 return true;
                                             },
                                             s.planLookahead);
        if (code) return code;
        if (!complete) {
            err = "a multi-qubit gate is wider than the register tile";
            return E_UNSUPPORTED;
        }
        seg.clear();
        return 0;
    };
    for (const Gate &g : s.pending) {
        if (g.type != OP_MULTI_UNITARY || g.numMultiTargets <= kRegBits) {
            seg.push_back(g);
            continue;
        }
        if (int code = planSegment()) return code;
        if (first) {
            // the initialisation / collapse runs before the dense sweep
            out.emplace_back();
            encodeHeaderOnly(s.numBits, s.numQubits, W, h, out.back(), paired);
            st.sweeps++;
            first = false;
            if (!emitted(out.size() - 1)) return -1;
        }
        TileProgram &p = out.emplace_back();
        std::memset(&p, 0, sizeof(p));
        p.numBits = s.numBits;
        p.numReal = s.numQubits;
        p.globalRe = 1.0;
        p.denseK = g.numMultiTargets;
        p.denseOff = (uint32_t) s.denseHost.size();
        for (int i = 0; i < g.numMultiTargets; i++) p.denseTargets[i] = (uint8_t) g.multiTargets[i];
        const auto &m = s.pool.mats[(size_t) g.multiIndex];
        s.denseHost.insert(s.denseHost.end(), m.begin(), m.end());
        if (s.single && tcBlockSupported(s.numBits, g.numMultiTargets)) {
            // the pipelined tensor-core operand ([Whi | Wlo], FP16) in the doubles buffer
            const size_t nf = tcBlockMatrixFloats(g.numMultiTargets);
            p.denseTcOff = (uint32_t) s.denseHost.size();
            s.denseHost.resize(s.denseHost.size() + (nf + 1) / 2, 0.0);
            packTcBlockMatrix(g.numMultiTargets, m.data(), p.denseTargets,
                              reinterpret_cast<float *>(s.denseHost.data() + p.denseTcOff));
        } else if (s.single && g.numMultiTargets == 6 && s.numBits >= 12) {
            // the tensor-core operand of 4096-amplitude registers: 2 x 128 x 128 floats
            const size_t nf = tcDenseMatrixFloats();
            p.denseTcOff = (uint32_t) s.denseHost.size();
            s.denseHost.resize(s.denseHost.size() + (nf + 1) / 2, 0.0);
            packTcDenseMatrix(m.data(), reinterpret_cast<float *>(s.denseHost.data() + p.denseTcOff));
        }
        st.sweeps++;
        st.flopsPerAmp += 8.0 * (double) (1 << g.numMultiTargets);
        if (!emitted(out.size() - 1)) return -1;
    }
    if (int code = planSegment()) return code;
    if (s.single && !out.empty() && out.back().denseTcOff) {
        // a tensor-core sweep rounds its FP32 sums toward zero: end with a
        // pass that renormalises its output (wired by the renormalisation
        // schedule, which puts a measurement on the sweep before the last)
        out.emplace_back();
        encodeHeaderOnly(s.numBits, s.numQubits, W, SweepHeader(), out.back(), paired);
        st.sweeps++;
        if (!emitted(out.size() - 1)) return -1;
    }
    if (out.empty()) {
        out.emplace_back();
        encodeHeaderOnly(s.numBits, s.numQubits, W, h, out.back(), paired);
        st.sweeps = 1;
        if (!emitted(0)) return -1;
    }
    return 0;
}

void consumePending(QuregState &s) {
    s.pending.clear();
    s.pool.mats.clear();
    s.initPending = false;
    s.restrictActive = false;
    s.rMask = s.rValue = 0;
    s.rScale = 1.0;
    s.probsValid = false;
}

}  // namespace dgq

namespace {

cudaError_t allocOn(void **ptr, size_t bytes, cudaStream_t st);
void freeOn(void *ptr, cudaStream_t st);

// Dense 6-target unitaries on complex64 registers run on the tensor cores
// (dgq_setTensorCores(0): the SIMT dense kernel instead).

// 0: compile specialised kernels when a plan needs them; 1: specialise only
// plans whose kernels are compiled already, interpret the others while
// their kernels compile on background host threads (serving: a one-off
// circuit structure should not wait for NVRTC).
std::atomic<int> g_specPolicy{0};

bool launchProgram(QuregState &s, size_t i, const char *func) {
    const CUfunction fn = i < s.plannedFns.size() ? s.plannedFns[i] : nullptr;
    const dgq::TileProgram &p = s.planned[i];
    if (p.renormOut && !cudaOk(cudaMemsetAsync(p.normOut, 0, sizeof(double), s.stream), func)) return false;
    cudaError_t e;
    if (p.denseK) {
        dgq::DenseArgs da;
        if (!dgq::denseArgs(s.numBits, p.denseK, p.denseTargets, da))
            return raise(E_UNSUPPORTED, func, "dense unitary does not fit the register");
        if (p.renormIn) da.normIn = p.normIn;
        if (p.renormOut) da.normOut = p.normOut;
        if (p.denseTcOff && g_tensorCores.load()) {
            static uint32_t *errWord = dgq::tcDenseErrorWord();
            const float *op = reinterpret_cast<const float *>(s.dDense + p.denseTcOff);
            e = dgq::tcBlockSupported(s.numBits, p.denseK)
                    ? dgq::launchTcBlock((float2 *) s.dState, p.denseK, da, op, errWord, s.stream)
                    : dgq::launchTcDense((float2 *) s.dState, da, op, errWord, s.stream);
        } else {
            e = dgq::launchDense(s.dState, s.single, p.denseK, da, s.dDense + p.denseOff, s.stream);
        }
    } else {
        e = fn ? dgq::launchJitSweep(fn, s.dState, s.plannedTileBits, p, s.stream)
               : dgq::launchTile(s.dState, s.single, s.plannedTileBits, p, s.stream);
    }
    if (!cudaOk(e, func)) return false;
    g_launches++;
    return true;
}

// Programs from index `from` on.
bool launchPlanned(QuregState &s, const char *func, size_t from = 0) {
    for (size_t i = from; i < s.planned.size(); i++)
        if (!launchProgram(s, i, func)) return false;
    return true;
}

// complex64: sweep i < last adds up the norm of its output when i % 4 == 3
// or it is the sweep before the last, and the next sweep divides by its
// square root, so FP32 rounding drift never accumulates over more than 4
// sweeps and the final sweep starts from a renormalised state (the
// per-sweep global factor already restores the scale of the factored
// rotations exactly). `last` is unknown (SIZE_MAX) while a sweep two or
// more places before the last is launched as the plan is being made.
void setRenorm(QuregState &s, size_t i, size_t last, int &event) {
    dgq::TileProgram &p = s.planned[i];
    p.isSingle = s.single ? 1 : 0;
    // (a register in host memory or in shards runs each sweep page by page:
    // no sweep sees the whole output's norm before the next one starts)
    if (!s.single || s.hostTier || s.sharded) return;
    const dgq::TileProgram *prev = i > 0 ? &s.planned[i - 1] : nullptr;
    if (prev && prev->renormOut) {
        p.renormIn = 1;
        p.normIn = prev->normOut;
    }
    if (i < last && (i % 4 == 3 || i + 1 == last)) {
        p.renormOut = 1;
        p.normOut = s.dNorm + (event++ & 1);
    }
}

// Plans the pending gates into s.planned (dgq_sweepSource: specialise =
// false plans as for specialisation but compiles nothing). With launch, the
// sweeps are issued too: when their kernels are compiled already, each sweep
// is launched as soon as the two after it are planned, so planning the rest
// of the circuit overlaps the GPU's work on the first sweeps.
bool planPending(QuregState &s, const char *func, bool specialise = true, bool launch = false) {
    s.planned.clear();
    s.plannedFns.clear();
    if (s.pending.empty() && !s.initPending) return true;
    const double t0 = nowMillis();
    int denseBlocks = 0;
    int formK = s.denseFusion > 0 ? s.denseFusion : 0;
    s.stats.formAuto = 0;
    s.formTileBits = 0;
    s.stats.predictedTileMs = 0.0;
    for (double &x : s.stats.predictedDenseMs) x = 0.0;
    if (s.denseFusion < 0 && !s.pending.empty()) {
        formK = chooseForm(s);
        s.stats.formAuto = 1;
    }
    s.stats.formK = formK;
    if (formK > 0 && s.numBits >= formK + 2 && !s.pending.empty())
        s.pending = dgq::fuseDenseBlocks(s.pending, s.numBits, formK, s.pool, &denseBlocks);
    const bool jitOn = dgq::jitEnabled();
    const bool wantJit = jitOn && (!specialise || s.numBits >= jitMinBits());
    // complex64 registers of >= 2^10 amplitudes run the paired form (two
    // amplitudes per slot, packed FP32 arithmetic) when specialised, unless a
    // sweep cannot be encoded that way (a multi-qubit unitary on address bit 0)
    const bool pairedOk = wantJit && s.single && s.allowPaired && pairedEnabled() && s.numBits >= 10;
    // policies 1 and 2 compile first only for registers of >= 2^32
    // amplitudes: below that the interpreting kernel, 2-3x slower than
    // specialised code, finishes a one-off circuit before its kernels would
    // have compiled while several requests compile at once (measured in the
    // serving loop: compiling first from 2^28 amplitudes on, complex64
    // requests of 28..33 qubits took 2.8 s on average); at 2^32 and above
    // the interpreted sweeps themselves take seconds
    const int policy = g_specPolicy.load();
    const bool cachedOnly = specialise && wantJit && policy >= 1 && s.numBits < 32;
    // launching while planning: not when the plan may be redone (policy 1
    // falls back to the interpreting kernel when a kernel is missing; the
    // paired form falls back on a multi-qubit unitary on bit 0) nor with dense
    // sweeps, whose matrices are uploaded once the plan is complete
    bool stream = launch && specialise && !cachedOnly;
    for (const Gate &g : s.pending)
        if (g.type == dgq::OP_MULTI_UNITARY && (g.numMultiTargets > dgq::kRegBits || (pairedOk && (g.targetMask & 1ULL))))
            stream = false;
    dgq::PlanStats st;
    std::string err;
    int W = 0;
    bool paired = false;
    size_t launched = 0;  // programs issued while planning
    bool missing = false;  // a sweep's kernel is not loaded: the rest wait for the plan
    int event = 0;
    int reused = 0;
    std::function<bool(size_t)> emit;
    if (stream) {
        emit = [&](size_t k) -> bool {
            while (!missing && launched + 2 <= k) {
                const size_t i = launched;
                setRenorm(s, i, SIZE_MAX, event);
                CUfunction fn = nullptr;
                if (wantJit && !s.planned[i].denseK) {
                    fn = dgq::jitFindLoaded(dgq::generateSweepSource(s.planned[i], W));
                    if (!fn) {
                        missing = true;
                        break;
                    }
                    reused++;
                }
                s.plannedFns.resize(i + 1, nullptr);
                s.plannedFns[i] = fn;
                s.plannedTileBits = W;
                if (!launchProgram(s, i, func)) return false;
                launched++;
            }
            return true;
        };
    }
    // interpret: the programs are for the interpreting kernel (W <= 12, unpaired)
    auto build = [&](bool pairedForm, bool interpret) -> int {
        paired = pairedForm;
        s.planLookahead = -1;
        if (paired) {
            W = pairedTileBits(s);
        } else if (s.formTileBits > 0 && formK == 0) {
            // the form choice planned the tile widths already
            W = s.formTileBits;
            s.planLookahead = s.formLookahead;
        } else {
            W = chooseTileBits(s);
        }
        if (interpret) W = std::min(W, dgq::kMaxTileBitsF64);
        st = dgq::PlanStats();
        err.clear();
        event = 0;
        int code = dgq::buildPrograms(s, W, s.planned, st, err, paired, emit);
        if (code) return code;
        const size_t last = s.planned.size() - 1;
        for (size_t i = launched; i <= last; i++) setRenorm(s, i, last, event);
        return 0;
    };
    int code = build(pairedOk, !wantJit);
    if (code == -1) return false;
    if (code && pairedOk && launched == 0) code = build(false, !wantJit);
    if (code == -1) return false;
    if (code) return raise(code, func, err.c_str());
    s.plannedFns.resize(s.planned.size(), nullptr);
    s.stats.jitCompiled = 0;
    s.stats.jitReused = reused;
    s.stats.jitMillis = 0.0;
    if (specialise && wantJit) {
        std::vector<std::string> sources;
        std::vector<size_t> which;  // tile programs (dense sweeps have their own kernel)
        for (size_t i = launched; i < s.planned.size(); i++)
            if (!s.planned[i].denseK) {
                sources.push_back(dgq::generateSweepSource(s.planned[i], W));
                which.push_back(i);
            }
        if (cachedOnly && !dgq::jitAllReady(sources)) {
            if (policy == 1) dgq::jitCompileInBackground(sources);
            if (paired || W > dgq::kMaxTileBitsF64) {
                // the interpreting kernel runs unpaired programs of W <= 12
                code = build(false, true);
                if (code) return raise(code, func, err.c_str());
                s.plannedFns.assign(s.planned.size(), nullptr);
            }
        } else {
            dgq::JitStats js;
            std::string jerr;
            std::vector<CUfunction> fns;
            if (!dgq::jitGetKernels(sources, fns, &js, &jerr)) return raise(E_UNSUPPORTED, func, jerr.c_str());
            for (size_t k = 0; k < which.size(); k++) s.plannedFns[which[k]] = fns[k];
            s.stats.jitCompiled = js.compiled;
            s.stats.jitReused += js.reused;
            s.stats.jitMillis = js.compileMillis;
        }
    }
    if (!s.denseHost.empty() && specialise) {
        // a new buffer per plan, freed in stream order after earlier launches
        // (the host-only planner entry points, specialise = false, upload nothing)
        freeOn(s.dDense, s.stream);
        s.dDense = nullptr;
        if (!cudaOk(allocOn((void **) &s.dDense, s.denseHost.size() * sizeof(double), s.stream), func) ||
            !cudaOk(cudaMemcpyAsync(s.dDense, s.denseHost.data(), s.denseHost.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, s.stream),
                    func) ||
            !cudaOk(cudaStreamSynchronize(s.stream), func))
            return false;
    }
    s.plannedPaired = paired;
    s.plannedTileBits = W;
    s.stats.sweeps = st.sweeps;
    s.stats.phases = st.phases;
    s.stats.ops = st.ops;
    s.stats.gates = st.gates;
    s.stats.tileBits = W;
    s.stats.numBits = s.numBits;
    s.stats.flopsPerAmp = st.flopsPerAmp;
    s.stats.launchBytes = (int64_t) st.sweeps * (int64_t) sizeof(dgq::TileProgram);
    s.stats.planMillis = nowMillis() - t0;
    s.stats.streamedSweeps = (int) launched;
    s.stats.denseBlocks = denseBlocks;
    dgq::consumePending(s);
    return !launch || launchPlanned(s, func, launched);
}

// Register memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// register's stream, from the device's default pool with no release
// threshold): creating or destroying one register neither waits for nor
// serialises kernels that other registers run on their own streams, and
// freed states are reused by later registers without returning to the driver.
cudaMemPool_t registerPool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPool_t p = nullptr;
        if (cudaDeviceGetDefaultMemPool(&p, dev) != cudaSuccess) return nullptr;
        uint64_t keep = ~0ULL;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}

// Bytes the pool holds but no register uses.
size_t poolSpare() {
    cudaMemPool_t p = registerPool();
    if (!p) return 0;
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &used);
    return reserved > used ? (size_t) (reserved - used) : 0;
}

cudaError_t allocOn(void **ptr, size_t bytes, cudaStream_t st) {
    *ptr = nullptr;
    cudaError_t e = cudaMallocAsync(ptr, bytes, st);
    if (e == cudaErrorMemoryAllocation) {
        // pool blocks of other sizes may hold the memory: hand them back, retry
        cudaGetLastError();
        if (cudaMemPool_t p = registerPool()) {
            cudaStreamSynchronize(st);
            cudaMemPoolTrimTo(p, 0);
        }
        e = cudaMallocAsync(ptr, bytes, st);
    }
    return e;
}

void freeOn(void *ptr, cudaStream_t st) {
    if (ptr) cudaFreeAsync(ptr, st);
}

bool flush(QuregState &s, const char *func) {
    if (s.pending.empty() && !s.initPending) return true;
    if (s.hostTier || s.sharded) return dgq::hostTierFlush(s, func);
    return planPending(s, func, true, true);
}

// Entry points that need the state in HBM.
bool vDeviceResident(const QuregState &s, const char *func) {
    if (s.sharded) return raise(E_UNSUPPORTED, func, "not available for a sharded register");
    if (!s.hostTier) return true;
    return raise(E_UNSUPPORTED, func, "not available for a register held in host memory (larger than the device budget)");
}

bool readLogicalFor(QuregState &s, double *re, double *im, const char *func);

// The diagonal of a device-resident density register, rho(i, i) = entry
// i (2^n + 1) of the vectorisation, gathered on the device: 2^n complex
// values cross to the host instead of 4^n.
bool densityDiagonal(QuregState &s, std::vector<double> &diag, const char *func) {
    const int n = s.densityQubits;
    const uint64_t dim = 1ULL << n;
    double2 *dOut = nullptr;
    if (!cudaOk(cudaMallocAsync((void **) &dOut, dim * sizeof(double2), s.stream), func)) return false;
    dgq::GatherArgs ga;
    std::memset(&ga, 0, sizeof(ga));
    ga.begin = 0;
    ga.count = dim;
    ga.stride = dim + 1;
    ga.numReal = s.numQubits;
    ga.hasRestrict = s.restrictActive ? 1 : 0;
    ga.restrictMask = s.rMask;
    ga.restrictValue = s.rValue;
    ga.restrictScale = s.rScale;
    for (int b = 0; b < s.numQubits; b++) ga.l2v[b] = (uint8_t) s.l2v[b];
    std::vector<double2> host((size_t) dim);
    const bool ok = cudaOk(dgq::launchGather(s.dState, s.single, ga, dOut, s.stream), func) &&
                    cudaOk(cudaMemcpyAsync(host.data(), dOut, dim * sizeof(double2), cudaMemcpyDeviceToHost, s.stream),
                           func);
    g_launches++;
    cudaFreeAsync(dOut, s.stream);
    if (!ok || !cudaOk(cudaStreamSynchronize(s.stream), func)) return false;
    diag.resize((size_t) dim);
    for (uint64_t i = 0; i < dim; i++) diag[(size_t) i] = host[(size_t) i].x;
    return true;
}

// Density registers: P(row qubit t = 0) and the trace from the diagonal
// (gathered on the device; a register in host memory reads its whole
// vectorisation, 16 x 4^n bytes).
bool densityProbs(QuregState &s, const char *func) {
    const int n = s.densityQubits;
    const uint64_t dim = 1ULL << n;
    std::vector<double> diag;
    if (s.hostTier || s.sharded) {
        std::vector<double> re(dim * dim), im(dim * dim);
        if (!readLogicalFor(s, re.data(), im.data(), func)) return false;
        diag.resize((size_t) dim);
        for (uint64_t i = 0; i < dim; i++) diag[(size_t) i] = re[i + (i << n)];
    } else if (!densityDiagonal(s, diag, func)) {
        return false;
    }
    std::vector<double> p0((size_t) n, 0.0);
    double total = 0.0;
    for (uint64_t i = 0; i < dim; i++) {
        const double d = diag[(size_t) i];
        total += d;
        for (int t = 0; t < n; t++)
            if (!((i >> t) & 1ULL)) p0[(size_t) t] += d;
    }
    s.p0.assign((size_t) s.numBits, 0.0);
    for (int t = 0; t < n; t++) s.p0[(size_t) s.l2v[t]] = p0[(size_t) t];
    s.totalProb = total;
    s.probsValid = true;
    return true;
}

bool ensureProbs(QuregState &s, const char *func) {
    if (s.probsValid) return true;
    if (!flush(s, func)) return false;
    if (s.densityQubits) return densityProbs(s, func);
    if (s.hostTier || s.sharded) {
        std::vector<double> p0;
        double total = 0.0;
        if (!dgq::hostTierProbs(s, p0, total, func)) return false;
        const double sc2 = s.restrictActive ? s.rScale * s.rScale : 1.0;
        s.totalProb = total * sc2;
        s.p0.assign((size_t) s.numBits, 0.0);
        for (int b = 0; b < s.numBits; b++) s.p0[(size_t) b] = p0[(size_t) b] * sc2;
        if (s.restrictActive)
            for (int b = 0; b < s.numBits; b++)
                if ((s.rMask >> b) & 1ULL) s.p0[(size_t) b] = ((s.rValue >> b) & 1ULL) ? 0.0 : s.totalProb;
        s.probsValid = true;
        return true;
    }
    dgq::ProbArgs a;
    std::memset(&a, 0, sizeof(a));
    int nf = 0;
    for (int b = 0; b < s.numBits; b++) {
        if (s.restrictActive && ((s.rMask >> b) & 1ULL)) continue;
        a.freePos[nf++] = (uint8_t) b;
    }
    a.nFree = nf;
    a.kappa = std::min(4, std::max(0, nf - 12));
    a.rValue = s.restrictActive ? s.rValue : 0;
    const size_t need = (size_t) dgq::probNumCtas(a) * 17;
    if (need > s.partialCap) {
        freeOn(s.dPartial, s.stream);
        s.dPartial = nullptr;
        if (!cudaOk(allocOn((void **) &s.dPartial, need * sizeof(double), s.stream), func)) return false;
        s.partialCap = need;
    }
    if (!cudaOk(dgq::launchProb(s.dState, s.single, a, s.dPartial, s.dProbOut, s.stream), func)) return false;
    g_launches += 2;
    std::vector<double> out((size_t) nf + 1);
    if (!cudaOk(cudaMemcpyAsync(out.data(), s.dProbOut, out.size() * sizeof(double), cudaMemcpyDeviceToHost, s.stream),
                func))
        return false;
    if (!cudaOk(cudaStreamSynchronize(s.stream), func)) return false;
    const double sc2 = s.restrictActive ? s.rScale * s.rScale : 1.0;
    s.p0.assign((size_t) s.numBits, 0.0);
    s.totalProb = out[(size_t) nf] * sc2;
    for (int i = 0; i < nf; i++) s.p0[a.freePos[i]] = out[(size_t) i] * sc2;
    if (s.restrictActive) {
        for (int b = 0; b < s.numBits; b++) {
            if (!((s.rMask >> b) & 1ULL)) continue;
            s.p0[(size_t) b] = ((s.rValue >> b) & 1ULL) ? 0.0 : s.totalProb;
        }
    }
    s.probsValid = true;
    return true;
}

// ---------------------------------------------------------------- validation
bool vQureg(const Qureg &q, const char *func) {
    if (!q.state) return raise(E_INVALID_ARGUMENT, func, "destroyed or uninitialised Qureg");
    return true;
}
bool vTarget(const Qureg &q, int t, const char *func) {
    if (!vQureg(q, func)) return false;
    if (t < 0 || t >= (int) q.numQubitsRepresented) return raise(E_INVALID_TARGET_QUBIT, func);
    return true;
}
bool vControlTarget(const Qureg &q, int c, int t, const char *func) {
    if (!vTarget(q, t, func)) return false;
    if (c < 0 || c >= (int) q.numQubitsRepresented) return raise(E_INVALID_CONTROL_QUBIT, func);
    if (c == t) return raise(E_TARGET_IS_CONTROL, func);
    return true;
}
bool vUniqueTargets(const Qureg &q, int a, int b, const char *func) {
    if (!vTarget(q, a, func) || !vTarget(q, b, func)) return false;
    if (a == b) return raise(E_TARGETS_NOT_UNIQUE, func);
    return true;
}
bool vMultiControls(const Qureg &q, const int *c, int n, const char *func) {
    if (!vQureg(q, func)) return false;
    if (n < 1 || n > (int) q.numQubitsRepresented || !c) return raise(E_INVALID_NUM_CONTROLS, func);
    for (int i = 0; i < n; i++)
        if (c[i] < 0 || c[i] >= (int) q.numQubitsRepresented) return raise(E_INVALID_CONTROL_QUBIT, func);
    return true;
}
bool vStateIndex(const Qureg &q, long long idx, const char *func) {
    if (!vQureg(q, func)) return false;
    const long long maxIdx = 1LL << q.numQubitsRepresented;
    if (idx < 0 || idx >= maxIdx) return raise(E_INVALID_STATE_INDEX, func);
    return true;
}
bool vStateVec(const Qureg &q, const char *func) {
    if (!vQureg(q, func)) return false;
    if (q.isDensityMatrix) return raise(E_DEFINED_ONLY_FOR_STATEVECS, func);
    return true;
}
bool vDensity(const Qureg &q, const char *func) {
    if (!vQureg(q, func)) return false;
    if (!q.isDensityMatrix) return raise(E_DEFINED_ONLY_FOR_DENSMATRS, func);
    return true;
}
bool vOutcome(int o, const char *func) {
    if (o != 0 && o != 1) return raise(E_INVALID_QUBIT_OUTCOME, func);
    return true;
}
// src/QuEST_validation.c:103-128
bool isPairUnitary(Complex a, Complex b) {
    return std::fabs(-1 + a.real * a.real + a.imag * a.imag + b.real * b.real + b.imag * b.imag) < REAL_EPS;
}
bool isMatrix2Unitary(const ComplexMatrix2 &u) {
    if (std::fabs(u.r0c0.real * u.r0c0.real + u.r0c0.imag * u.r0c0.imag + u.r1c0.real * u.r1c0.real +
                  u.r1c0.imag * u.r1c0.imag - 1) > REAL_EPS)
        return false;
    if (std::fabs(u.r0c1.real * u.r0c1.real + u.r0c1.imag * u.r0c1.imag + u.r1c1.real * u.r1c1.real +
                  u.r1c1.imag * u.r1c1.imag - 1) > REAL_EPS)
        return false;
    if (std::fabs(u.r0c0.real * u.r0c1.real + u.r0c0.imag * u.r0c1.imag + u.r1c0.real * u.r1c1.real +
                  u.r1c0.imag * u.r1c1.imag) > REAL_EPS)
        return false;
    if (std::fabs(u.r0c1.real * u.r0c0.imag - u.r0c0.real * u.r0c1.imag + u.r1c1.real * u.r1c0.imag -
                  u.r1c0.real * u.r1c1.imag) > REAL_EPS)
        return false;
    return true;
}

// ---------------------------------------------------------------- recording
void push(QuregState &s, dgq::GateType type, u64 logicalTargets, u64 logicalControls, const double *op, int nop) {
    Gate g;
    g.type = type;
    g.targetMask = toVirtualMask(s, logicalTargets);
    g.controlMask = toVirtualMask(s, logicalControls);
    for (int i = 0; i < nop; i++) g.op[i] = op[i];
    s.pending.push_back(g);
    s.probsValid = false;
}

// The complex conjugate of a gate in the same encoding: phase powers
// e^{i pi k/4} become k -> 8 - k, angles change sign (phase shift, Rz and Rx
// store -angle; Ry is real), Y and its conjugate trade types, and the
// imaginary parts of compact pairs and 2x2 matrices change sign.
dgq::GateType conjugateGate(dgq::GateType type, const double *op, int nop, double *out) {
    for (int i = 0; i < nop; i++) out[i] = op[i];
    if (type <= dgq::OP_T_GATE_CONJ) return (dgq::GateType) ((8 - (int) type) % 8);
    switch (type) {
        case dgq::OP_PHASE_SHIFT:
        case dgq::OP_ROTATE_Z:
        case dgq::OP_ROTATE_X: out[0] = -op[0]; break;
        case dgq::OP_PAULI_Y: return dgq::OP_PAULI_Y_CONJ;
        case dgq::OP_PAULI_Y_CONJ: return dgq::OP_PAULI_Y;
        case dgq::OP_COMPACT_UNITARY:
            out[1] = -op[1];
            out[3] = -op[3];
            break;
        case dgq::OP_UNITARY:
            for (int i = 1; i < 8; i += 2) out[i] = -op[i];
            break;
        default: break;  // X, H, Ry: real
    }
    return type;
}

// Density registers apply rho -> U rho U^dagger as U on the row qubits
// 0..n-1 and conj(U) on the column qubits n..2n-1 of the vectorisation
// (upstream QuEST's representation of createDensityQureg, QuEST.h:139).
void record(const Qureg &q, dgq::GateType type, u64 logicalTargets, u64 logicalControls, const double *op, int nop) {
    QuregState &s = *stateOf(q);
    push(s, type, logicalTargets, logicalControls, op, nop);
    if (const int n = s.densityQubits) {
        double c[8];
        const dgq::GateType ct = conjugateGate(type, op, nop, c);
        push(s, ct, logicalTargets << n, logicalControls << n, c, nop);
    }
}

void recordMatrix(const Qureg &q, u64 targets, u64 controls, const ComplexMatrix2 &u) {
    const double m[8] = {u.r0c0.real, u.r0c0.imag, u.r0c1.real, u.r0c1.imag,
                         u.r1c0.real, u.r1c0.imag, u.r1c1.real, u.r1c1.imag};
    record(q, dgq::OP_UNITARY, targets, controls, m, 8);
}

u64 bit(int q) { return 1ULL << q; }

// Runs the pending work, applies a pending collapse to the amplitudes, and
// moves amplitudes so that virtual bit = logical qubit (swapGate relabels
// undone in HBM by swapBitsKernel, disjoint bit pairs per pass): afterwards
// the buffer is the state in logical order, as dgQuEST's reorder at a
// section boundary leaves it (QuEST_gpu_kernel.cu:589-654).
bool normaliseLayout(QuregState &s, const char *func) {
    if (s.restrictActive && s.pending.empty() && !s.initPending) {
        // an empty program carries the collapse header into one sweep
        dgq::Gate g;
        g.type = dgq::OP_ONE;
        s.pending.push_back(g);
    }
    if (!flush(s, func)) return false;
    if (s.hostTier || s.sharded) return true;  // read through the map, page by page
    for (;;) {
        dgq::SwapArgs a;
        std::memset(&a, 0, sizeof(a));
        a.numBits = s.numBits;
        uint64_t used = 0;
        for (int q = 0; q < s.numQubits && a.numPairs < 32; q++) {
            const int v = s.l2v[q];
            if (v == q || ((used >> q) & 1ULL) || ((used >> v) & 1ULL)) continue;
            a.a[a.numPairs] = (uint8_t) q;
            a.b[a.numPairs] = (uint8_t) v;
            a.numPairs++;
            used |= (1ULL << q) | (1ULL << v);
        }
        if (a.numPairs == 0) break;
        if (!cudaOk(dgq::launchSwapBits(s.dState, s.single, a, s.stream), func)) return false;
        g_launches++;
        for (int k = 0; k < a.numPairs; k++) {
            // the qubits at virtual bits a[k] and b[k] trade places
            const int qa = s.v2l[a.a[k]], qb = s.v2l[a.b[k]];
            s.v2l[a.a[k]] = qb;
            s.v2l[a.b[k]] = qa;
            s.l2v[qa] = a.b[k];
            s.l2v[qb] = a.a[k];
        }
    }
    return cudaOk(cudaStreamSynchronize(s.stream), func);
}

// Device budget for new registers (dgq_setDeviceBudget; 0: free HBM):
// larger states go to the host tier.
std::atomic<int64_t> g_deviceBudget{0};

}  // namespace

namespace dgq {
bool planForPages(QuregState &s, const char *func) { return planPending(s, func, true, false); }
}  // namespace dgq

// ====================================================================
// C API
// ====================================================================
extern "C" {

int dgq_setErrorMode(int mode) {
    const int prev = g_errMode;
    g_errMode = mode == DGQ_ERRORS_RECORD ? DGQ_ERRORS_RECORD : DGQ_ERRORS_EXIT;
    return prev;
}

int dgq_applyCircuit(Qureg q, const dgq_gate_record *r, int count, int *outcomes) {
    if (!vQureg(q, __func__)) return -1;
    if (count < 0 || (count > 0 && !r)) return raise(E_INVALID_ARGUMENT, __func__, "null records") ? 0 : -1;
    int m = 0;
    for (int i = 0; i < count; i++) {
        const int64_t before = g_errorCount;
        const dgq_gate_record &g = r[i];
        const int a = g.q0, b = g.q1;
        const double *p = g.p;
        switch (g.kind) {
            case 0: hadamard(q, a); break;
            case 1: pauliX(q, a); break;
            case 2: pauliY(q, a); break;
            case 3: pauliZ(q, a); break;
            case 4: sGate(q, a); break;
            case 5: tGate(q, a); break;
            case 6: rotateX(q, a, p[0]); break;
            case 7: rotateY(q, a, p[0]); break;
            case 8: rotateZ(q, a, p[0]); break;
            case 9: phaseShift(q, a, p[0]); break;
            case 10: controlledNot(q, a, b); break;
            case 11: controlledPhaseFlip(q, a, b); break;
            case 12: controlledPhaseShift(q, a, b, p[0]); break;
            case 13: controlledRotateX(q, a, b, p[0]); break;
            case 14: controlledRotateY(q, a, b, p[0]); break;
            case 15: controlledRotateZ(q, a, b, p[0]); break;
            case 16: compactUnitary(q, a, Complex{p[0], p[1]}, Complex{p[2], p[3]}); break;
            case 17: controlledCompactUnitary(q, a, b, Complex{p[0], p[1]}, Complex{p[2], p[3]}); break;
            case 18:
            case 19: {
                ComplexMatrix2 u;
                u.r0c0 = Complex{p[0], p[1]};
                u.r0c1 = Complex{p[2], p[3]};
                u.r1c0 = Complex{p[4], p[5]};
                u.r1c1 = Complex{p[6], p[7]};
                if (g.kind == 18)
                    unitary(q, a, u);
                else
                    controlledUnitary(q, a, b, u);
                break;
            }
            case 20: SqX(q, a); break;
            case 21: SqY(q, a); break;
            case 22: SqW(q, a); break;
            case 23: swapGate(q, a, b); break;
            case 24: {
                const int o = measure(q, a);
                if (outcomes && g_errorCount == before) outcomes[m] = o;
                m++;
                break;
            }
            case 25: controlledPauliY(q, a, b); break;
            default: {
                char msg[64];
                snprintf(msg, sizeof msg, "record %d has unknown kind %d", i, g.kind);
                raise(E_INVALID_ARGUMENT, __func__, msg);
                return -1;
            }
        }
        if (g_errorCount != before) return -1;
    }
    return count;
}

int dgq_sampleOutcomes(Qureg q, int numSamples, uint32_t seed, uint64_t *outcomes) {
    if (!vStateVec(q, __func__)) return -1;
    if (numSamples < 0 || (numSamples > 0 && !outcomes))
        return raise(E_INVALID_ARGUMENT, __func__, "numSamples < 0 or null output") ? 0 : -1;
    QuregState &s = *stateOf(q);
    if (!vDeviceResident(s, __func__)) return -1;
    if (!flush(s, __func__)) return -1;
    if (numSamples == 0) return 0;
    dgq::Mt19937 rng;
    rng.seed(seed);
    std::vector<double> u((size_t) numSamples);
    for (double &x : u) x = rng.res53();
    dgq::SampleArgs a;
    a.numAmps = 1ULL << s.numBits;
    a.restrictMask = s.restrictActive ? s.rMask : 0;
    a.restrictValue = s.restrictActive ? s.rValue : 0;
    a.restrictScale2 = s.restrictActive ? s.rScale * s.rScale : 1.0;
    const size_t runs = (size_t) dgq::sampleScratchCount(a.numAmps);
    void *scratch = nullptr;
    const size_t bytes = runs * sizeof(double) + (size_t) numSamples * (sizeof(double) + sizeof(uint64_t));
    if (!cudaOk(allocOn(&scratch, bytes, s.stream), __func__)) return -1;
    double *dSums = (double *) scratch;
    double *dU = dSums + runs;
    uint64_t *dOut = (uint64_t *) (dU + numSamples);
    std::vector<uint64_t> v((size_t) numSamples);
    bool ok = cudaOk(cudaMemcpyAsync(dU, u.data(), u.size() * sizeof(double), cudaMemcpyHostToDevice, s.stream),
                     __func__) &&
              cudaOk(dgq::launchSample(s.dState, s.single, a, dSums, dU, numSamples, dOut, s.stream), __func__) &&
              cudaOk(cudaMemcpyAsync(v.data(), dOut, v.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost, s.stream),
                     __func__);
    freeOn(scratch, s.stream);
    ok = ok && cudaOk(cudaStreamSynchronize(s.stream), __func__);
    if (!ok) return -1;
    g_launches += 3;
    for (int k = 0; k < numSamples; k++) {
        uint64_t logical = 0;
        for (int b = 0; b < s.numQubits; b++)
            if ((v[(size_t) k] >> s.l2v[b]) & 1ULL) logical |= 1ULL << b;
        outcomes[k] = logical;
    }
    return 0;
}

int dgq_setSpecialisationPolicy(int policy) {
    if (policy < 0 || policy > 2) {
        raise(E_INVALID_ARGUMENT, __func__, "policy must be 0, 1 or 2");
        return -1;
    }
    return g_specPolicy.exchange(policy);
}

int dgq_setTensorCores(int enable) { return g_tensorCores.exchange(enable ? 1 : 0); }

int dgq_getDeviceErrors(void) {
    uint32_t *w = dgq::tcDenseErrorWord();
    uint32_t v = 0;
    if (!w || cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return (int) v;
}

int64_t dgq_getAvailableMemory(void) {
    size_t freeB = 0, totalB = 0;
    if (!cudaOk(cudaMemGetInfo(&freeB, &totalB), __func__)) return -1;
    return (int64_t) (freeB + poolSpare());
}

int dgq_getLastError(char *msg, int len) {
    const int code = g_lastError;
    if (msg && len > 0) {
        std::strncpy(msg, g_lastMessage.c_str(), (size_t) len - 1);
        msg[len - 1] = '\0';
    }
    g_lastError = 0;
    g_lastMessage.clear();
    return code;
}

int64_t dgq_getLaunchCount(void) { return g_launches.load(); }

// ---------------------------------------------------------------- env
void seedQuESTDefault(void) {
    // src/QuEST_common.c:127-142: milliseconds since the epoch and the pid
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    const double ms = (double) tv.tv_sec * 1000 + (double) (tv.tv_usec / 1000);
    unsigned long key[2] = {(unsigned long) ms, (unsigned long) getpid()};
    g_rng.seedArray(key, 2);
}

void seedQuEST(unsigned long int *seedArray, int numSeeds) {
    if (!seedArray || numSeeds < 1) {
        raise(E_INVALID_ARGUMENT, __func__, "need at least one seed");
        return;
    }
    g_rng.seedArray(seedArray, numSeeds);
}

QuESTEnv createQuESTEnv(void) {
    seedQuESTDefault();
    QuESTEnv env;
    env.value = new QuESTEnvValue();
    env.rank = 0;
    int dev = 0;
    if (!cudaOk(cudaGetDevice(&dev), __func__)) return env;
    env.value->device = dev;
    return env;
}

void destroyQuESTEnv(QuESTEnv env) { delete env.value; }

int getQuEST_PREC(void) { return (int) (sizeof(qreal) / 4); }

// ---------------------------------------------------------------- registers
}  // extern "C"

static Qureg createQuregWith(int numQubits, QuESTEnv env, bool single, const char *func, int shardBits = 0,
                             const int *shardDevices = nullptr) {
    Qureg q;
    std::memset(&q, 0, sizeof(q));
    if (numQubits <= 0) {
        raise(E_INVALID_NUM_QUBITS, func);
        return q;
    }
    if (numQubits > dgq::kMaxStateBits - 2) {
        raise(E_SYS_TOO_BIG_FOR_DEVICE, func);
        return q;
    }
    auto *s = new QuregState();
    s->numQubits = numQubits;
    s->numBits = std::max(numQubits, dgq::kMinTileBits);
    s->single = single;
    resetMapping(*s);
    const size_t bytes = ampBytes(*s) << s->numBits;
    size_t freeB = 0, totalB = 0;
    if (!cudaOk(cudaMemGetInfo(&freeB, &totalB), func)) {
        delete s;
        return q;
    }
    const size_t avail = freeB + poolSpare() > (64u << 20) ? freeB + poolSpare() - (64u << 20) : 0;
    const int64_t setBudget = g_deviceBudget.load();
    // the host tier serves states beyond a set budget, or beyond what the
    // device could hold at all; a state that only does not fit next to the
    // registers alive now is an error (E_SYS_TOO_BIG_FOR_DEVICE), as before
    const size_t never = totalB > (1ull << 30) ? totalB - (1ull << 30) : totalB;
    const bool hostTier =
        shardBits == 0 && (setBudget > 0 ? bytes > std::min<size_t>(avail, (size_t) setBudget) : bytes > never);
    if (shardBits > 0) {
        // shards of 2^(n - shardBits) amplitudes on the given devices
        std::string err;
        int code = E_UNSUPPORTED;
        s->pageBits = s->numBits - shardBits;
        if (!dgq::shardAttach(*s, shardBits, shardDevices, code, err)) {
            delete s;
            raise(code, func, err.c_str());
            return q;
        }
    } else if (hostTier) {
        // the host tier: the state in pinned host memory, paged through HBM
        const size_t budget = setBudget > 0 ? std::min<size_t>(avail, (size_t) setBudget) : avail;
        std::string err;
        if (!dgq::hostTierAttach(*s, budget, err)) {
            delete s;
            raise(E_SYS_TOO_BIG_FOR_DEVICE, func, err.c_str());
            return q;
        }
    } else if (bytes > avail) {
        delete s;
        raise(E_SYS_TOO_BIG_FOR_DEVICE, func);
        return q;
    }
    if (!cudaOk(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), func)) {
        dgq::hostTierRelease(*s);
        dgq::shardRelease(*s);
        delete s;
        return q;
    }
    if (!registerPool() || (!s->hostTier && !s->sharded && !cudaOk(allocOn(&s->dState, bytes, s->stream), func)) ||
        !cudaOk(allocOn((void **) &s->dProbOut, sizeof(double) * (dgq::kMaxStateBits + 1), s->stream), func) ||
        !cudaOk(allocOn((void **) &s->dNorm, sizeof(double) * 2, s->stream), func) ||
        !cudaOk(cudaStreamSynchronize(s->stream), func)) {
        freeOn(s->dState, s->stream);
        freeOn(s->dProbOut, s->stream);
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
        dgq::hostTierRelease(*s);
        dgq::shardRelease(*s);
        delete s;
        return q;
    }
    q.isDensityMatrix = 0;
    q.numQubitsRepresented = (u64) numQubits;
    q.numQubitsInStateVec = (u64) numQubits;
    q.numAmpsTotal = 1ULL << numQubits;
    q.env = env;
    q.state = s;
    initZeroState(q);
    return q;
}

extern "C" {

Qureg createQureg(int numQubits, QuESTEnv env) { return createQuregWith(numQubits, env, false, __func__); }

Qureg dgq_createQuregF32(int numQubits, QuESTEnv env) { return createQuregWith(numQubits, env, true, __func__); }

// include/QuEST.h:139 (declared only in dgQuEST): an n-qubit density matrix
// in |0><0|, held as the 2n-qubit vectorisation (row qubits 0..n-1, column
// qubits n..2n-1), complex128
Qureg createDensityQureg(int numQubits, QuESTEnv env) {
    Qureg q;
    std::memset(&q, 0, sizeof(q));
    if (numQubits <= 0) {
        raise(E_INVALID_NUM_QUBITS, __func__);
        return q;
    }
    if (2 * numQubits > dgq::kMaxStateBits - 2) {
        raise(E_SYS_TOO_BIG_FOR_DEVICE, __func__);
        return q;
    }
    q = createQuregWith(2 * numQubits, env, false, __func__);
    if (!q.state) return q;
    q.state->densityQubits = numQubits;
    q.isDensityMatrix = 1;
    q.numQubitsRepresented = (u64) numQubits;
    return q;
}

Qureg dgq_createShardedQureg(int numQubits, QuESTEnv env, int shardBits, const int *devices, int single) {
    if (shardBits < 1 || shardBits > 4 || numQubits - shardBits < DGQ_MIN_SHARD_QUBITS) {
        Qureg q;
        std::memset(&q, 0, sizeof(q));
        raise(numQubits <= 0 ? E_INVALID_NUM_QUBITS : E_INVALID_ARGUMENT, __func__,
              "shardBits must be 1..4 with at least 14 qubits in each shard");
        return q;
    }
    return createQuregWith(numQubits, env, single != 0, __func__, shardBits, devices);
}

int dgq_getPrecision(Qureg qureg) {
    if (!vQureg(qureg, __func__)) return 0;
    return stateOf(qureg)->single ? 1 : 2;
}

void searchQuregTaskPartitions(Qureg qureg, QuESTEnv env) {
    (void) env;
    if (!vQureg(qureg, __func__)) return;
    // dgQuEST picks its partition K here (QuEST_backend_distributed.cpp:86-121);
    // the recast picks the tile width for the gates recorded so far.
    QuregState &s = *stateOf(qureg);
    if (s.tileBitsSetting == 0 && !s.pending.empty()) s.tileBitsSetting = chooseTileBits(s);
}

void destroyQureg(Qureg qureg, QuESTEnv env) {
    (void) env;
    QuregState *s = qureg.state;
    if (!s) return;
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        freeOn(s->dState, s->stream);
        freeOn(s->dPartial, s->stream);
        freeOn(s->dProbOut, s->stream);
        freeOn(s->dNorm, s->stream);
        freeOn(s->dDense, s->stream);
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    dgq::hostTierRelease(*s);
    dgq::shardRelease(*s);
    delete s;
}

int getNumQubits(Qureg qureg) { return (int) qureg.numQubitsRepresented; }
int getNumAmps(Qureg qureg) { return (int) qureg.numAmpsTotal; }

// ---------------------------------------------------------------- init
static void setInit(Qureg q, int32_t kind, uint64_t index, double amp) {
    QuregState &s = *stateOf(q);
    s.pending.clear();
    s.pool.mats.clear();
    resetMapping(s);
    s.restrictActive = false;
    s.rMask = s.rValue = 0;
    s.rScale = 1.0;
    s.initPending = true;
    s.initKind = kind;
    s.initIndex = index;
    s.initAmp = amp;
    s.probsValid = false;
}

void initZeroState(Qureg qureg) {
    if (!vQureg(qureg, __func__)) return;
    setInit(qureg, dgq::INIT_CLASSICAL, 0, 0.0);
}

void initPlusState(Qureg qureg) {
    if (!vQureg(qureg, __func__)) return;
    // density registers: |+><+| has every element 1/2^n
    const double dim = (double) (1LL << qureg.numQubitsRepresented);
    setInit(qureg, dgq::INIT_PLUS, 0, qureg.isDensityMatrix ? 1.0 / dim : 1.0 / std::sqrt(dim));
}

void initClassicalState(Qureg qureg, long long int stateInd) {
    if (!vStateIndex(qureg, stateInd, __func__)) return;
    // density registers: |k><k| is element (k, k)
    const uint64_t k = (uint64_t) stateInd;
    setInit(qureg, dgq::INIT_CLASSICAL, qureg.isDensityMatrix ? k + (k << qureg.numQubitsRepresented) : k, 0.0);
}

// Replaces the register's vector by (reals, imags), 2^numQubits entries in
// logical order (a density register's vectorisation).
static void loadAmps(QuregState &s, const double *reals, const double *imags, const char *func) {
    s.pending.clear();
    s.pool.mats.clear();
    s.initPending = false;
    resetMapping(s);
    s.restrictActive = false;
    s.rMask = s.rValue = 0;
    s.rScale = 1.0;
    s.probsValid = false;
    const uint64_t n = 1ULL << s.numQubits;
    const uint64_t total = 1ULL << s.numBits;
    if (s.hostTier || s.sharded) {
        if (s.hostTier) cudaOk(dgq::hostTierSync(s, func) ? cudaSuccess : cudaErrorUnknown, func);
        // shards: the amplitudes in storage type on the host, then one copy per shard
        std::vector<char> staged(s.sharded ? ampBytes(s) << s.numBits : 0);
        void *dst = s.sharded ? (void *) staged.data() : s.hState;
        for (uint64_t i = 0; i < total; i++) {
            const double r = i < n ? reals[i] : 0.0, m = i < n ? imags[i] : 0.0;
            if (s.single)
                reinterpret_cast<float2 *>(dst)[i] = make_float2((float) r, (float) m);
            else
                reinterpret_cast<double2 *>(dst)[i] = make_double2(r, m);
        }
        if (s.sharded) dgq::shardWriteVirtual(s, 0, total, staged.data(), func);
        return;
    }
    // stage re and im in chunks, interleave on the GPU
    const uint64_t chunk = std::min<uint64_t>(n, 1ULL << 24);
    double *dRe = nullptr, *dIm = nullptr;
    if (!cudaOk(cudaMalloc(&dRe, chunk * sizeof(double)), func)) return;
    if (!cudaOk(cudaMalloc(&dIm, chunk * sizeof(double)), func)) {
        cudaFree(dRe);
        return;
    }
    if (total > n) {
        cudaOk(cudaMemsetAsync((char *) s.dState + n * ampBytes(s), 0, (total - n) * ampBytes(s), s.stream), func);
    }
    for (uint64_t off = 0; off < n; off += chunk) {
        const uint64_t c = std::min(chunk, n - off);
        cudaOk(cudaMemcpyAsync(dRe, reals + off, c * sizeof(double), cudaMemcpyHostToDevice, s.stream), func);
        cudaOk(cudaMemcpyAsync(dIm, imags + off, c * sizeof(double), cudaMemcpyHostToDevice, s.stream), func);
        cudaOk(dgq::launchInterleave(dRe, dIm, c, c, (char *) s.dState + off * ampBytes(s), s.single, s.stream), func);
        g_launches++;
    }
    cudaOk(cudaStreamSynchronize(s.stream), func);
    cudaFree(dRe);
    cudaFree(dIm);
}

void initStateFromAmps(Qureg qureg, qreal *reals, qreal *imags) {
    if (!vStateVec(qureg, __func__)) return;
    if (!reals || !imags) {
        raise(E_INVALID_ARGUMENT, __func__, "null amplitude array");
        return;
    }
    loadAmps(*stateOf(qureg), reals, imags, __func__);
}

// include/QuEST.h:257 (declared only in dgQuEST): amplitudes [startInd,
// startInd + numAmps) in logical order, the others kept
void setAmps(Qureg qureg, long long int startInd, qreal *reals, qreal *imags, long long int numAmps) {
    if (!vStateVec(qureg, __func__) || !vStateIndex(qureg, startInd, __func__)) return;
    QuregState &s = *stateOf(qureg);
    if (numAmps < 0 || numAmps > (1LL << s.numQubits)) {
        raise(E_INVALID_NUM_AMPS, __func__);
        return;
    }
    if (startInd + numAmps > (1LL << s.numQubits)) {
        raise(E_INVALID_OFFSET_NUM_AMPS, __func__);
        return;
    }
    if (numAmps > 0 && (!reals || !imags)) {
        raise(E_INVALID_ARGUMENT, __func__, "null amplitude array");
        return;
    }
    if (!normaliseLayout(s, __func__)) return;
    s.probsValid = false;
    if (s.hostTier || s.sharded) {
        // shards: read, change and write back the whole state (virtual order)
        std::vector<char> staged(s.sharded ? ampBytes(s) << s.numBits : 0);
        if (s.sharded && !dgq::shardReadVirtual(s, 0, 1ULL << s.numBits, staged.data(), __func__)) return;
        void *dst = s.sharded ? (void *) staged.data() : s.hState;
        for (long long k = 0; k < numAmps; k++) {
            const uint64_t v = toVirtualIndex(s, (uint64_t) (startInd + k));
            if (s.single)
                reinterpret_cast<float2 *>(dst)[v] = make_float2((float) reals[k], (float) imags[k]);
            else
                reinterpret_cast<double2 *>(dst)[v] = make_double2(reals[k], imags[k]);
        }
        if (s.sharded) dgq::shardWriteVirtual(s, 0, 1ULL << s.numBits, staged.data(), __func__);
        return;
    }
    const uint64_t chunk = std::min<uint64_t>((uint64_t) std::max<long long>(numAmps, 1), 1ULL << 24);
    double *dRe = nullptr, *dIm = nullptr;
    if (!cudaOk(cudaMalloc(&dRe, chunk * sizeof(double)), __func__)) return;
    if (!cudaOk(cudaMalloc(&dIm, chunk * sizeof(double)), __func__)) {
        cudaFree(dRe);
        return;
    }
    for (uint64_t off = 0; off < (uint64_t) numAmps; off += chunk) {
        const uint64_t c = std::min(chunk, (uint64_t) numAmps - off);
        char *dst = (char *) s.dState + ((uint64_t) startInd + off) * ampBytes(s);
        if (!cudaOk(cudaMemcpyAsync(dRe, reals + off, c * sizeof(double), cudaMemcpyHostToDevice, s.stream), __func__) ||
            !cudaOk(cudaMemcpyAsync(dIm, imags + off, c * sizeof(double), cudaMemcpyHostToDevice, s.stream), __func__) ||
            !cudaOk(dgq::launchInterleave(dRe, dIm, c, c, dst, s.single, s.stream), __func__))
            break;
        g_launches++;
    }
    cudaOk(cudaStreamSynchronize(s.stream), __func__);
    cudaFree(dRe);
    cudaFree(dIm);
}

// include/QuEST.h:267 (declared only in dgQuEST): targetQureg := copyQureg
// (same qubit count and precision); the copy's pending work runs first
void cloneQureg(Qureg targetQureg, Qureg copyQureg) {
    if (!vQureg(targetQureg, __func__) || !vQureg(copyQureg, __func__)) return;
    QuregState &t = *stateOf(targetQureg);
    QuregState &c = *stateOf(copyQureg);
    if (t.numQubits != c.numQubits) {
        raise(E_MISMATCHING_QUREG_DIMENSIONS, __func__);
        return;
    }
    bool sameShards = t.sharded == c.sharded && t.shardBits == c.shardBits;
    for (int k = 0; sameShards && t.sharded && k < (1 << t.shardBits); k++) sameShards = t.shardDev[k] == c.shardDev[k];
    if (t.single != c.single || t.hostTier != c.hostTier || !sameShards || t.densityQubits != c.densityQubits) {
        raise(E_MISMATCHING_QUREG_TYPES, __func__);
        return;
    }
    if (&t == &c) return;
    if (!flush(c, __func__) || !cudaOk(cudaStreamSynchronize(c.stream), __func__)) return;
    // the target's own pending work is dropped: its state is replaced
    t.pending.clear();
    t.pool.mats.clear();
    t.initPending = false;
    if (t.hostTier) {
        if (!dgq::hostTierSync(t, __func__)) return;
        std::memcpy(t.hState, c.hState, ampBytes(t) << t.numBits);
    } else if (t.sharded) {
        if (!dgq::shardSync(t, __func__) || !dgq::shardCopy(t, c, __func__)) return;
    } else if (!cudaOk(cudaMemcpyAsync(t.dState, c.dState, ampBytes(t) << t.numBits, cudaMemcpyDeviceToDevice,
                                       t.stream),
                       __func__) ||
               !cudaOk(cudaStreamSynchronize(t.stream), __func__)) {
        return;
    }
    std::memcpy(t.l2v, c.l2v, sizeof(t.l2v));
    std::memcpy(t.v2l, c.v2l, sizeof(t.v2l));
    t.restrictActive = c.restrictActive;
    t.rMask = c.rMask;
    t.rValue = c.rValue;
    t.rScale = c.rScale;
    t.probsValid = false;
}

// include/QuEST.h:229: for state-vectors, the pure state's amplitudes
void initPureState(Qureg qureg, Qureg pure) {
    if (!vQureg(qureg, __func__) || !vQureg(pure, __func__)) return;
    if (!qureg.isDensityMatrix) {
        cloneQureg(qureg, pure);
        return;
    }
    // density register: rho = |psi><psi|, built on the host
    if (pure.isDensityMatrix) {
        raise(E_SECOND_ARG_MUST_BE_STATEVEC, __func__);
        return;
    }
    if (pure.numQubitsRepresented != qureg.numQubitsRepresented) {
        raise(E_MISMATCHING_QUREG_DIMENSIONS, __func__);
        return;
    }
    QuregState &s = *stateOf(qureg);
    const int n = s.densityQubits;
    const uint64_t dim = 1ULL << n;
    std::vector<double> pr(dim), pi(dim), re(dim * dim), im(dim * dim);
    if (!readLogicalFor(*stateOf(pure), pr.data(), pi.data(), __func__)) return;
    for (uint64_t c = 0; c < dim; c++)
        for (uint64_t r = 0; r < dim; r++) {
            re[r + (c << n)] = pr[r] * pr[c] + pi[r] * pi[c];
            im[r + (c << n)] = pi[r] * pr[c] - pr[r] * pi[c];
        }
    loadAmps(s, re.data(), im.data(), __func__);
}

// include/QuEST.h:183
void reportQuregParams(Qureg qureg) {
    if (!vQureg(qureg, __func__)) return;
    const QuregState &s = *stateOf(qureg);
    printf("QUBITS:\n");
    printf("Number of qubits is %d.\n", s.numQubits);
    printf("Number of amps is %llu.\n", 1ULL << s.numQubits);
    printf("Precision: %s, state in %s.\n", s.single ? "complex64" : "complex128",
           s.hostTier ? "pinned host memory (host tier)" : s.sharded ? "HBM shards" : "HBM");
}

// include/QuEST.h:177: every amplitude, for small registers
void reportStateToScreen(Qureg qureg, QuESTEnv env, int reportRank) {
    (void) env;
    (void) reportRank;
    if (!vQureg(qureg, __func__)) return;
    QuregState &s = *stateOf(qureg);
    if (s.numQubits > 5) {
        printf("Error: reportStateToScreen will not print output for systems of more than 5 qubits.\n");
        return;
    }
    const uint64_t n = 1ULL << s.numQubits;
    std::vector<double> re(n), im(n);
    if (dgq_getStateVector(qureg, re.data(), im.data()) != 0) return;
    printf("Reporting state from rank 0 [\n");
    printf("real, imag\n");
    for (uint64_t i = 0; i < n; i++) printf("%.14f, %.14f\n", re[i], im[i]);
    printf("]\n");
}

// include/QuEST.h:538
void getEnvironmentString(QuESTEnv env, Qureg qureg, char str[200]) {
    (void) env;
    if (!str) return;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    snprintf(str, 200, "CUDA=1 OpenMP=0 MPI=0 threads=%d ranks=1 device=%d SMs=%d qubits=%d", 1, dev, sms,
             qureg.state ? qureg.state->numQubits : 0);
}

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

// ---------------------------------------------------------------- noise
// Density registers: a channel rho -> sum_K K rho K^dagger on k = 1 or 2
// qubits is one dense op on the row qubits and the column qubits together
// (targets qs[0..k), qs[0..k) + n; matrix index bits in that order), the
// superoperator S[(r', c')][(r, c)] = sum_K K[r'][r] conj(K[c'][c]).
using Kraus = std::vector<std::complex<double>>;  // d x d, row-major

static void recordChannel(Qureg q, const int *qs, int k, const std::vector<Kraus> &kraus) {
    QuregState &s = *stateOf(q);
    const int n = s.densityQubits, d = 1 << k, D = d * d;
    std::vector<double> m((size_t) 2 * D * D, 0.0);
    for (const Kraus &K : kraus)
        for (int rp = 0; rp < d; rp++)
            for (int cp = 0; cp < d; cp++)
                for (int r = 0; r < d; r++)
                    for (int c = 0; c < d; c++) {
                        const std::complex<double> v = K[(size_t) (rp * d + r)] * std::conj(K[(size_t) (cp * d + c)]);
                        const size_t at = (size_t) 2 * ((rp + cp * d) * D + (r + c * d));
                        m[at] += v.real();
                        m[at + 1] += v.imag();
                    }
    Gate g;
    g.type = dgq::OP_MULTI_UNITARY;
    u64 tm = 0;
    for (int i = 0; i < k; i++) tm |= bit(qs[i]) | bit(qs[i] + n);
    g.targetMask = toVirtualMask(s, tm);
    g.controlMask = 0;
    g.numMultiTargets = 2 * k;
    for (int i = 0; i < k; i++) {
        g.multiTargets[i] = s.l2v[qs[i]];
        g.multiTargets[k + i] = s.l2v[qs[i] + n];
    }
    g.multiIndex = (int32_t) s.pool.mats.size();
    s.pool.mats.push_back(std::move(m));
    s.pending.push_back(g);
    s.probsValid = false;
}

static const std::complex<double> kI(0.0, 1.0);

static Kraus pauli(int p) {  // 0 I, 1 X, 2 Y, 3 Z
    switch (p) {
        case 1: return {0.0, 1.0, 1.0, 0.0};
        case 2: return {0.0, -kI, kI, 0.0};
        case 3: return {1.0, 0.0, 0.0, -1.0};
        default: return {1.0, 0.0, 0.0, 1.0};
    }
}

// P_a (x) P_b on two qubits, a the low bit of the 4 x 4 index
static Kraus pauli2(int pa, int pb, double w) {
    const Kraus A = pauli(pa), B = pauli(pb);
    Kraus K(16);
    for (int rb = 0; rb < 2; rb++)
        for (int ra = 0; ra < 2; ra++)
            for (int cb = 0; cb < 2; cb++)
                for (int ca = 0; ca < 2; ca++)
                    K[(size_t) ((ra + 2 * rb) * 4 + (ca + 2 * cb))] = w * A[(size_t) (ra * 2 + ca)] * B[(size_t) (rb * 2 + cb)];
    return K;
}

static bool vNoise(Qureg q, int t, double prob, double maxProb, int code, const char *func) {
    if (!vDensity(q, func) || !vTarget(q, t, func)) return false;
    if (!(prob >= 0.0 && prob <= 1.0)) return raise(E_INVALID_PROB, func);
    if (prob > maxProb) return raise(code, func);
    return true;
}

// include/QuEST.h:1373: (1 - p) rho + p Z rho Z
void applyOneQubitDephaseError(Qureg q, const int targetQubit, qreal prob) {
    if (!vNoise(q, targetQubit, prob, 0.5, E_INVALID_ONE_QUBIT_DEPHASE_PROB, __func__)) return;
    const double a = std::sqrt(1.0 - prob), b = std::sqrt(prob);
    Kraus K0 = pauli(0), K1 = pauli(3);
    for (auto &x : K0) x *= a;
    for (auto &x : K1) x *= b;
    recordChannel(q, &targetQubit, 1, {K0, K1});
}

// include/QuEST.h:1399: (1 - p) rho + p/3 (Za rho Za + Zb rho Zb + ZaZb rho ZaZb)
void applyTwoQubitDephaseError(Qureg q, const int qubit1, const int qubit2, qreal prob) {
    if (!vNoise(q, qubit1, prob, 0.75, E_INVALID_TWO_QUBIT_DEPHASE_PROB, __func__) ||
        !vUniqueTargets(q, qubit1, qubit2, __func__))
        return;
    const int qs[2] = {qubit1, qubit2};
    const double w = std::sqrt(prob / 3.0);
    recordChannel(q, qs, 2,
                  {pauli2(0, 0, std::sqrt(1.0 - prob)), pauli2(3, 0, w), pauli2(0, 3, w), pauli2(3, 3, w)});
}

// include/QuEST.h:1423: (1 - p) rho + p/3 (X rho X + Y rho Y + Z rho Z)
void applyOneQubitDepolariseError(Qureg q, const int targetQubit, qreal prob) {
    if (!vNoise(q, targetQubit, prob, 0.75, E_INVALID_ONE_QUBIT_DEPOL_PROB, __func__)) return;
    std::vector<Kraus> ks;
    for (int p = 0; p < 4; p++) {
        Kraus K = pauli(p);
        const double w = p == 0 ? std::sqrt(1.0 - prob) : std::sqrt(prob / 3.0);
        for (auto &x : K) x *= w;
        ks.push_back(K);
    }
    recordChannel(q, &targetQubit, 1, ks);
}

// include/QuEST.h:1445: amplitude damping (decay to |0>) with probability p:
// Kraus operators [[1, 0], [0, sqrt(1 - p)]] and [[0, sqrt(p)], [0, 0]]
void applyOneQubitDampingError(Qureg q, const int targetQubit, qreal prob) {
    // any probability in [0, 1] is valid; vNoise reports the rest as E_INVALID_PROB
    if (!vNoise(q, targetQubit, prob, 1.0, E_INVALID_PROB, __func__)) return;
    const Kraus K0 = {1.0, 0.0, 0.0, std::sqrt(1.0 - prob)};
    const Kraus K1 = {0.0, std::sqrt(prob), 0.0, 0.0};
    recordChannel(q, &targetQubit, 1, {K0, K1});
}

// include/QuEST.h:1494: (1 - p) rho + p/15 (sum of the 15 non-identity
// two-qubit Paulis P rho P)
void applyTwoQubitDepolariseError(Qureg q, const int qubit1, const int qubit2, qreal prob) {
    if (!vNoise(q, qubit1, prob, 15.0 / 16.0, E_INVALID_TWO_QUBIT_DEPOL_PROB, __func__) ||
        !vUniqueTargets(q, qubit1, qubit2, __func__))
        return;
    const int qs[2] = {qubit1, qubit2};
    std::vector<Kraus> ks;
    for (int pa = 0; pa < 4; pa++)
        for (int pb = 0; pb < 4; pb++)
            ks.push_back(pauli2(pa, pb, pa == 0 && pb == 0 ? std::sqrt(1.0 - prob) : std::sqrt(prob / 15.0)));
    recordChannel(q, qs, 2, ks);
}

// include/QuEST.h:1507: combineQureg := (1 - prob) combineQureg + prob
// otherQureg (equal-size density matrices; on the host)
void addDensityMatrix(Qureg combineQureg, qreal prob, Qureg otherQureg) {
    if (!vDensity(combineQureg, __func__) || !vDensity(otherQureg, __func__)) return;
    if (combineQureg.numQubitsRepresented != otherQureg.numQubitsRepresented) {
        raise(E_MISMATCHING_QUREG_DIMENSIONS, __func__);
        return;
    }
    if (!(prob >= 0.0 && prob <= 1.0)) {
        raise(E_INVALID_PROB, __func__);
        return;
    }
    QuregState &a = *stateOf(combineQureg);
    QuregState &b = *stateOf(otherQureg);
    const size_t len = (size_t) 1 << a.numQubits;
    std::vector<double> ar(len), ai(len), br(len), bi(len);
    if (!readLogicalFor(a, ar.data(), ai.data(), __func__) || !readLogicalFor(b, br.data(), bi.data(), __func__))
        return;
    for (size_t i = 0; i < len; i++) {
        ar[i] = (1.0 - prob) * ar[i] + prob * br[i];
        ai[i] = (1.0 - prob) * ai[i] + prob * bi[i];
    }
    loadAmps(a, ar.data(), ai.data(), __func__);
}

// include/QuEST.h:1524: Tr(rho^2) = the sum of |rho_rc|^2 over all elements
qreal calcPurity(Qureg q) {
    if (!vDensity(q, __func__)) return 0.0;
    QuregState &s = *stateOf(q);
    const size_t len = (size_t) 1 << s.numQubits;
    std::vector<double> re(len), im(len);
    if (!readLogicalFor(s, re.data(), im.data(), __func__)) return 0.0;
    double t = 0.0;
    for (size_t i = 0; i < len; i++) t += re[i] * re[i] + im[i] * im[i];
    return t;
}

// ---------------------------------------------------------------- read-outs
// Amplitude `index` of the register's vector (logical order; a density
// register's vectorisation).
static Complex ampAt(QuregState &s, uint64_t index, const char *func) {
    Complex out{0.0, 0.0};
    if (!flush(s, func)) return out;
    const uint64_t v = toVirtualIndex(s, index);
    if (s.restrictActive && (v & s.rMask) != s.rValue) {
        if (!cudaOk(cudaStreamSynchronize(s.stream), func)) return out;
        return out;
    }
    double2 a;
    if (s.sharded) {
        // one amplitude from the shard that holds it
        if (s.single) {
            float2 f;
            if (!dgq::shardReadVirtual(s, v, 1, &f, func)) return out;
            a = make_double2(f.x, f.y);
        } else if (!dgq::shardReadVirtual(s, v, 1, &a, func)) {
            return out;
        }
    } else if (s.hostTier) {
        // the flushed state is in pinned host memory
        if (s.single) {
            const float2 f = reinterpret_cast<const float2 *>(s.hState)[v];
            a = make_double2(f.x, f.y);
        } else {
            a = reinterpret_cast<const double2 *>(s.hState)[v];
        }
    } else if (s.single) {
        float2 f;
        if (!cudaOk(cudaMemcpyAsync(&f, (const float2 *) s.dState + v, sizeof(f), cudaMemcpyDeviceToHost, s.stream),
                    func))
            return out;
        if (!cudaOk(cudaStreamSynchronize(s.stream), func)) return out;
        a = make_double2(f.x, f.y);
    } else {
        if (!cudaOk(cudaMemcpyAsync(&a, (const double2 *) s.dState + v, sizeof(a), cudaMemcpyDeviceToHost, s.stream),
                    func))
            return out;
        if (!cudaOk(cudaStreamSynchronize(s.stream), func)) return out;
    }
    const double sc = s.restrictActive ? s.rScale : 1.0;
    out.real = a.x * sc;
    out.imag = a.y * sc;
    return out;
}

Complex getAmp(Qureg q, long long int index) {
    if (!vStateVec(q, __func__) || !vStateIndex(q, index, __func__)) return Complex{0.0, 0.0};
    return ampAt(*stateOf(q), (uint64_t) index, __func__);
}

// include/QuEST.h:591 (declared only in dgQuEST): element (row, col) of a
// density matrix
Complex getDensityAmp(Qureg q, long long int row, long long int col) {
    if (!vDensity(q, __func__) || !vStateIndex(q, row, __func__) || !vStateIndex(q, col, __func__))
        return Complex{0.0, 0.0};
    QuregState &s = *stateOf(q);
    return ampAt(s, (uint64_t) row + ((uint64_t) col << s.densityQubits), __func__);
}
qreal getRealAmp(Qureg q, long long int index) { return getAmp(q, index).real; }
qreal getImagAmp(Qureg q, long long int index) { return getAmp(q, index).imag; }
qreal getProbAmp(Qureg q, long long int index) {
    const Complex a = getAmp(q, index);
    return a.real * a.real + a.imag * a.imag;
}

qreal calcProbOfOutcome(Qureg q, const int measureQubit, int outcome) {
    if (!vTarget(q, measureQubit, __func__) || !vOutcome(outcome, __func__)) return 0.0;
    QuregState &s = *stateOf(q);
    if (!ensureProbs(s, __func__)) return 0.0;
    const double p0 = s.p0[(size_t) s.l2v[measureQubit]];
    return outcome == 1 ? 1.0 - p0 : p0;
}

qreal calcTotalProb(Qureg q) {
    if (!vQureg(q, __func__)) return 0.0;
    QuregState &s = *stateOf(q);
    if (!ensureProbs(s, __func__)) return 0.0;
    return s.totalProb;
}

static void applyCollapse(QuregState &s, int v, int outcome, double prob) {
    if ((s.rMask >> v) & 1ULL) return;  // already fixed by an earlier collapse
    s.rMask |= 1ULL << v;
    if (outcome) s.rValue |= 1ULL << v;
    s.rScale /= std::sqrt(prob);
    s.restrictActive = true;
    s.probsValid = false;
}

qreal collapseToOutcome(Qureg q, const int measureQubit, int outcome) {
    if (!vTarget(q, measureQubit, __func__) || !vOutcome(outcome, __func__)) return 0.0;
    QuregState &s = *stateOf(q);
    if (!ensureProbs(s, __func__)) return 0.0;
    const int v = s.l2v[measureQubit];
    const double p0 = s.p0[(size_t) v];
    const double prob = outcome == 1 ? 1.0 - p0 : p0;
    if (prob < REAL_EPS) {
        raise(E_COLLAPSE_STATE_ZERO_PROB, __func__);
        return 0.0;
    }
    applyCollapse(s, v, outcome, prob);
    // density registers: the column qubit too (P rho P / prob)
    if (s.densityQubits) applyCollapse(s, s.l2v[measureQubit + s.densityQubits], outcome, prob);
    return prob;
}

// src/QuEST_common.c:97-115 (outcome rule) with QuEST's collapse semantics
int measureWithStats(Qureg q, int measureQubit, qreal *outcomeProb) {
    if (!vTarget(q, measureQubit, __func__)) return 0;
    QuregState &s = *stateOf(q);
    if (!ensureProbs(s, __func__)) return 0;
    const int v = s.l2v[measureQubit];
    const double zeroProb = s.p0[(size_t) v];
    // QuEST's REAL_EPS for the register's precision (1e-13 double, 1e-5 single)
    const double eps = s.single ? 1e-5 : REAL_EPS;
    int outcome;
    if (zeroProb < eps)
        outcome = 1;
    else if (1 - zeroProb < eps)
        outcome = 0;
    else
        outcome = (g_rng.real1() > zeroProb);
    const double prob = outcome == 0 ? zeroProb : 1 - zeroProb;
    if (outcomeProb) *outcomeProb = prob;
    applyCollapse(s, v, outcome, prob);
    if (s.densityQubits) applyCollapse(s, s.l2v[measureQubit + s.densityQubits], outcome, prob);
    return outcome;
}

int measure(Qureg q, int measureQubit) { return measureWithStats(q, measureQubit, nullptr); }

// ---------------------------------------------------------------- extensions
int dgq_setTileBits(Qureg q, int tileBits) {
    if (!vQureg(q, __func__)) return -1;
    QuregState &s = *stateOf(q);
    const int prev = s.tileBitsSetting;
    if (tileBits != 0 && (tileBits < dgq::kMinTileBits || tileBits > dgq::kMaxTileBits)) {
        raise(E_INVALID_ARGUMENT, __func__, "tile bits must be 0 or in [9, 14] (14: paired complex64 only)");
        return prev;
    }
    s.tileBitsSetting = tileBits;
    return prev;
}

int dgq_getPlanStats(Qureg q, dgq_plan_stats *out) {
    if (!vQureg(q, __func__) || !out) return -1;
    *out = stateOf(q)->stats;
    return 0;
}

int dgq_setDenseFusion(Qureg q, int qubits) {
    if (!vQureg(q, __func__)) return -1;
    if (qubits != 0 && qubits != -1 && (qubits < dgq::kMinDenseTargets || qubits > dgq::kMaxDenseTargets)) {
        raise(E_INVALID_ARGUMENT, __func__, "dense fusion takes -1 (the predictor chooses), 0 or 5..7 qubits");
        return -2;
    }
    QuregState &s = *stateOf(q);
    const int prev = s.denseFusion;
    s.denseFusion = qubits;
    return prev;
}

int dgq_setCostModel(double sweepMsPer2p30, double phaseMsPer2p30) {
    if (!(sweepMsPer2p30 > 0.0) || !(phaseMsPer2p30 >= 0.0) || !std::isfinite(sweepMsPer2p30) ||
        !std::isfinite(phaseMsPer2p30))
        return raise(E_INVALID_ARGUMENT, __func__, "rates must be finite, sweep > 0, phase >= 0") ? 0 : -1;
    std::lock_guard<std::mutex> lk(g_costMutex);
    g_costFileTried = true;
    g_cost.sweepSecondsPerAmp = sweepMsPer2p30 * 1e-3 / 1073741824.0;
    g_cost.phaseSecondsPerAmp = phaseMsPer2p30 * 1e-3 / 1073741824.0;
    return 0;
}

int dgq_loadCostModel(const char *path) {
    double sw = 0.0, ph = 0.0;
    if (!path || !readCostFile(path, sw, ph))
        return raise(E_INVALID_ARGUMENT, __func__, "missing or malformed cost file") ? 0 : -1;
    if (dgq_setCostModel(sw, ph) != 0) return -1;
    std::lock_guard<std::mutex> lk(g_costMutex);
    readCostFileExtras(path, g_cost);
    return 0;
}

int dgq_setDenseCost(int variant, int K, double msPer2p30) {
    if (variant < 0 || variant > 2 || K < 5 || K > 7 || !(msPer2p30 >= 0.0) || !std::isfinite(msPer2p30))
        return raise(E_INVALID_ARGUMENT, __func__, "variant 0..2, K 5..7, a finite rate >= 0") ? 0 : -1;
    costModel();  // a DGQ_COST_FILE is read first, so this call is not overwritten by it
    std::lock_guard<std::mutex> lk(g_costMutex);
    g_cost.denseMs[variant][K - 5] = msPer2p30;
    return 0;
}

double dgq_getDenseCost(int variant, int K) {
    if (variant < 0 || variant > 2 || K < 5 || K > 7) return -1.0;
    return costModel().denseMs[variant][K - 5];
}

int dgq_getCostModel(double *sweepMsPer2p30, double *phaseMsPer2p30) {
    const CostModel cm = costModel();
    if (sweepMsPer2p30) *sweepMsPer2p30 = cm.sweepSecondsPerAmp * 1073741824.0 * 1e3;
    if (phaseMsPer2p30) *phaseMsPer2p30 = cm.phaseSecondsPerAmp * 1073741824.0 * 1e3;
    return 0;
}

void dgq_shutdown(void) { dgq::jitStopBackground(); }

int64_t dgq_setDeviceBudget(int64_t bytes) { return g_deviceBudget.exchange(bytes > 0 ? bytes : 0); }

int dgq_getShardStats(Qureg q, int *shardBits, int64_t *passes, int64_t *exchanges, int64_t *bytesExchanged) {
    if (!vQureg(q, __func__)) return -1;
    const QuregState &s = *stateOf(q);
    if (shardBits) *shardBits = s.sharded ? s.shardBits : 0;
    if (passes) *passes = s.sharded ? s.hostTierPasses : 0;
    if (exchanges) *exchanges = s.sharded ? s.hostTierSwaps : 0;
    if (bytesExchanged) *bytesExchanged = s.sharded ? s.hostTierBytes : 0;
    return s.sharded ? 1 : 0;
}

int dgq_getHostTierStats(Qureg q, int *pageBits, int64_t *passes, int64_t *exchanges, int64_t *bytesMoved) {
    if (!vQureg(q, __func__)) return -1;
    const QuregState &s = *stateOf(q);
    if (pageBits) *pageBits = s.hostTier ? s.pageBits : 0;
    if (passes) *passes = s.hostTierPasses;
    if (exchanges) *exchanges = s.hostTierSwaps;
    if (bytesMoved) *bytesMoved = s.hostTierBytes;
    return s.hostTier ? 1 : 0;
}

int dgq_planPending(Qureg q) {
    if (!vQureg(q, __func__) || !vDeviceResident(*stateOf(q), __func__)) return -1;
    return planPending(*stateOf(q), __func__) ? 0 : -1;
}

int dgq_launchPlanned(Qureg q) {
    if (!vQureg(q, __func__)) return -1;
    QuregState &s = *stateOf(q);
    if (!vDeviceResident(s, __func__)) return -1;
    if (!launchPlanned(s, __func__)) return -1;
    s.probsValid = false;
    return 0;
}

int dgq_sync(Qureg q) {
    if (!vQureg(q, __func__)) return -1;
    QuregState &s = *stateOf(q);
    if (!flush(s, __func__)) return -1;
    return cudaOk(cudaStreamSynchronize(s.stream), __func__) ? 0 : -1;
}

void *dgq_getStream(Qureg q) {
    if (!vQureg(q, __func__)) return nullptr;
    return (void *) stateOf(q)->stream;
}

void *dgq_getDeviceState(Qureg q, int *numBits) {
    if (!vQureg(q, __func__)) return nullptr;
    if (!vDeviceResident(*stateOf(q), __func__)) return nullptr;
    if (!normaliseLayout(*stateOf(q), __func__)) return nullptr;
    if (numBits) *numBits = stateOf(q)->numBits;
    return (void *) stateOf(q)->dState;
}

// The register's vector in logical order (collapse applied) into re/im
// (2^numQubits entries; a density register's vectorisation).
static bool readLogical(QuregState &s, double *re, double *im, const char *func) {
    if (!flush(s, func)) return false;
    const uint64_t n = 1ULL << s.numQubits;
    if (s.hostTier || s.sharded) {
        // logical order through the map, from pinned host memory (shards:
        // from a host copy of the shards)
        std::vector<char> staged(s.sharded ? ampBytes(s) << s.numBits : 0);
        if (s.sharded && !dgq::shardReadVirtual(s, 0, 1ULL << s.numBits, staged.data(), func)) return false;
        const void *src = s.sharded ? (const void *) staged.data() : s.hState;
        const double sc = s.restrictActive ? s.rScale : 1.0;
        for (uint64_t i = 0; i < n; i++) {
            const uint64_t v = toVirtualIndex(s, i);
            double2 a;
            if (s.single) {
                const float2 f = reinterpret_cast<const float2 *>(src)[v];
                a = make_double2(f.x, f.y);
            } else {
                a = reinterpret_cast<const double2 *>(src)[v];
            }
            const bool keep = !s.restrictActive || (v & s.rMask) == s.rValue;
            re[i] = keep ? a.x * sc : 0.0;
            im[i] = keep ? a.y * sc : 0.0;
        }
        return true;
    }
    const uint64_t chunk = std::min<uint64_t>(n, 1ULL << 22);
    double2 *dOut = nullptr;
    if (!cudaOk(cudaMalloc(&dOut, chunk * sizeof(double2)), func)) return false;
    std::vector<double2> host((size_t) chunk);
    dgq::GatherArgs ga;
    std::memset(&ga, 0, sizeof(ga));
    ga.numReal = s.numQubits;
    ga.hasRestrict = s.restrictActive ? 1 : 0;
    ga.restrictMask = s.rMask;
    ga.restrictValue = s.rValue;
    ga.restrictScale = s.rScale;
    for (int b = 0; b < s.numQubits; b++) ga.l2v[b] = (uint8_t) s.l2v[b];
    bool ok = true;
    for (uint64_t off = 0; off < n && ok; off += chunk) {
        ga.begin = off;
        ga.count = std::min(chunk, n - off);
        ok = cudaOk(dgq::launchGather(s.dState, s.single, ga, dOut, s.stream), func) &&
             cudaOk(cudaMemcpyAsync(host.data(), dOut, ga.count * sizeof(double2), cudaMemcpyDeviceToHost, s.stream),
                    func) &&
             cudaOk(cudaStreamSynchronize(s.stream), func);
        g_launches++;
        for (uint64_t i = 0; ok && i < ga.count; i++) {
            re[off + i] = host[(size_t) i].x;
            im[off + i] = host[(size_t) i].y;
        }
    }
    cudaFree(dOut);
    return ok;
}

int dgq_getStateVector(Qureg q, qreal *re, qreal *im) {
    if (!vQureg(q, __func__) || !re || !im) return -1;
    return readLogical(*stateOf(q), re, im, __func__) ? 0 : -1;
}

}  // extern "C"

namespace {
bool readLogicalFor(QuregState &s, double *re, double *im, const char *func) { return readLogical(s, re, im, func); }
}  // namespace

extern "C" {


int dgq_calcProbOfAllZero(Qureg q, qreal *probs) {
    if (!vQureg(q, __func__) || !probs) return -1;
    QuregState &s = *stateOf(q);
    if (!ensureProbs(s, __func__)) return -1;
    // density registers: the represented qubits (the row qubits)
    const int count = s.densityQubits ? s.densityQubits : s.numQubits;
    for (int i = 0; i < count; i++) probs[i] = s.p0[(size_t) s.l2v[i]];
    return 0;
}

int dgq_measureFp64Peak(double *tflops) {
    if (!tflops) return -1;
    int dev = 0, sms = 0;
    if (!cudaOk(cudaGetDevice(&dev), __func__) ||
        !cudaOk(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), __func__))
        return -1;
    const int blocks = sms * 8, iters = 4096;
    double *out = nullptr;
    cudaEvent_t e0, e1;
    if (!cudaOk(cudaMalloc(&out, sizeof(double) * (size_t) blocks * 256), __func__)) return -1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    bool ok = cudaOk(dgq::launchFp64Peak(out, blocks, iters / 4, 0), __func__);  // warm-up
    float best = 1e30f;
    for (int r = 0; ok && r < 3; r++) {
        cudaEventRecord(e0, 0);
        ok = cudaOk(dgq::launchFp64Peak(out, blocks, iters, 0), __func__);
        cudaEventRecord(e1, 0);
        ok = ok && cudaOk(cudaEventSynchronize(e1), __func__);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
        g_launches++;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (!ok) return -1;
    const double fmas = (double) blocks * 256.0 * iters * 16.0 * 8.0;
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
    return 0;
}

int dgq_fuseApplyHost(int numQubits, int K, int count, const int32_t *types, const uint64_t *targetMasks,
                      const uint64_t *controlMasks, const double *operands, double *re, double *im) {
    if (numQubits < 1 || numQubits > 20 || K < 1 || K > 7 || K > numQubits || count < 0 ||
        (count > 0 && (!types || !targetMasks || !controlMasks || !operands)) || !re || !im) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    const u64 all = (1ULL << numQubits) - 1;
    std::vector<Gate> gates;
    for (int i = 0; i < count; i++) {
        Gate g;
        g.type = (dgq::GateType) types[i];
        g.targetMask = targetMasks[i];
        g.controlMask = controlMasks[i];
        if ((g.targetMask | g.controlMask) & ~all || g.type < 0 || g.type >= dgq::OP_MULTI_UNITARY) {
            raise(E_INVALID_ARGUMENT, __func__);
            return -1;
        }
        for (int k = 0; k < 8; k++) g.op[k] = operands[8 * i + k];
        gates.push_back(g);
    }
    dgq::MatrixPool pool;
    int blocks = 0;
    const std::vector<Gate> fused = dgq::fuseDenseBlocks(gates, numQubits, K, pool, &blocks);
    const size_t D = (size_t) 1 << numQubits;
    std::vector<double> v(2 * D);
    for (size_t i = 0; i < D; i++) {
        v[2 * i] = re[i];
        v[2 * i + 1] = im[i];
    }
    int local[64];
    for (int b = 0; b < 64; b++) local[b] = b < numQubits ? b : -1;
    for (const Gate &g : fused) dgq::applyGateLocal(g, pool, local, numQubits, v.data(), 1);
    for (size_t i = 0; i < D; i++) {
        re[i] = v[2 * i];
        im[i] = v[2 * i + 1];
    }
    return blocks;
}

// Gates given in dgQuEST's IR encoding through the host-only entry points
// (dgq_planGates, dgq_sweepSource), checked before the planner sees them:
// types 0..18 except the unused 9 (the multi-qubit unitary needs a matrix
// pool these calls do not take), masks inside the register, disjoint target
// and control masks, one target bit for Rz and the non-diagonal types, and
// no target but at least one qubit for the diagonal phase types.
static bool gatesFromArrays(int numQubits, int count, const int32_t *types, const uint64_t *targetMasks,
                            const uint64_t *controlMasks, const double *operands, std::vector<Gate> &out,
                            const char *func) {
    const u64 all = numQubits >= 64 ? ~0ULL : (1ULL << numQubits) - 1;
    out.clear();
    out.reserve((size_t) count);
    for (int i = 0; i < count; i++) {
        const int t = types[i];
        const u64 tm = targetMasks[i], cm = controlMasks[i];
        bool ok = t >= 0 && t <= dgq::OP_UNITARY && t != dgq::OP_RESERVED_9 && !((tm | cm) & ~all) && !(tm & cm);
        if (ok && t >= dgq::OP_ROTATE_Z) ok = tm != 0 && (tm & (tm - 1)) == 0;
        if (ok && t < dgq::OP_ROTATE_Z) ok = tm == 0 && cm != 0;
        if (!ok) {
            char msg[160];
            snprintf(msg, sizeof msg, "gate %d: type %d, target mask 0x%llx, control mask 0x%llx is not a valid gate", i,
                     t, (unsigned long long) tm, (unsigned long long) cm);
            raise(E_INVALID_ARGUMENT, func, msg);
            return false;
        }
        Gate g;
        g.type = (dgq::GateType) t;
        g.targetMask = tm;
        g.controlMask = cm;
        for (int k = 0; k < 8; k++) g.op[k] = operands[8 * i + k];
        out.push_back(g);
    }
    return true;
}

int dgq_planGates(int numQubits, int tileBits, int count, const int32_t *types, const uint64_t *targetMasks,
                  const uint64_t *controlMasks, const double *operands, dgq_plan_stats *out, int32_t *mergedTypes,
                  int32_t *numMerged) {
    if (numQubits < 1 || numQubits > dgq::kMaxStateBits - 2 || count < 0 || (count > 0 && (!types || !targetMasks ||
        !controlMasks || !operands)) || !out) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    QuregState s;
    s.numQubits = numQubits;
    s.numBits = std::max(numQubits, dgq::kMinTileBits);
    resetMapping(s);
    s.tileBitsSetting = tileBits;
    if (!gatesFromArrays(numQubits, count, types, targetMasks, controlMasks, operands, s.pending, __func__)) return -1;
    if (mergedTypes || numMerged) {
        dgq::GateDag dag(s.numBits, true);
        for (const Gate &g : s.pending) dag.add(g);
        const std::vector<Gate> merged = dag.gatesInOrder();
        if (numMerged) *numMerged = (int32_t) merged.size();
        if (mergedTypes)
            for (size_t i = 0; i < merged.size(); i++) mergedTypes[i] = (int32_t) merged[i].type;
    }
    s.initPending = true;
    s.initKind = dgq::INIT_CLASSICAL;
    if (!planPending(s, __func__, false)) return -1;
    *out = s.stats;
    return 0;
}

int dgq_planExchanges(int numQubits, int localQubits, int batch, int count, const int32_t *types,
                      const uint64_t *targetMasks, int32_t *segments, int32_t *exchanges, int32_t *qubitsMoved) {
    if (numQubits < 1 || numQubits > dgq::kMaxStateBits - 2 || localQubits < 1 || localQubits > numQubits ||
        count < 0 || (count > 0 && (!types || !targetMasks))) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    std::vector<Gate> gates((size_t) count);
    const uint64_t all = numQubits >= 64 ? ~0ULL : (1ULL << numQubits) - 1;
    for (int i = 0; i < count; i++) {
        if (types[i] < 0 || types[i] > dgq::OP_MULTI_UNITARY || (targetMasks[i] & ~all)) {
            raise(E_INVALID_ARGUMENT, __func__, "a gate type or target outside the register");
            return -1;
        }
        gates[(size_t) i].type = (dgq::GateType) types[i];
        gates[(size_t) i].targetMask = targetMasks[i];
    }
    int seg = 0, ex = 0, moved = 0;
    dgq::planExchanges(gates, localQubits, numQubits, batch != 0, seg, ex, moved);
    if (segments) *segments = seg;
    if (exchanges) *exchanges = ex;
    if (qubitsMoved) *qubitsMoved = moved;
    return 0;
}

int dgq_setSpecialisationMinBits(int minBits) {
    const int prev = jitMinBits();
    g_jitMinBits.store(minBits < 0 ? 22 : minBits);
    return prev;
}

int dgq_sweepSource(int numQubits, int tileBits, int count, const int32_t *types, const uint64_t *targetMasks,
                    const uint64_t *controlMasks, const double *operands, int sweep, int precision, char *buf,
                    int len) {
    if (numQubits < 1 || numQubits > dgq::kMaxStateBits - 2 || count < 0 || !buf || len <= 0) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    QuregState s;
    s.numQubits = numQubits;
    s.numBits = std::max(numQubits, dgq::kMinTileBits);
    s.single = precision == 1 || precision == 3;
    s.allowPaired = precision == 1;
    resetMapping(s);
    s.tileBitsSetting = tileBits;
    if (count > 0 && (!types || !targetMasks || !controlMasks || !operands)) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    if (!gatesFromArrays(numQubits, count, types, targetMasks, controlMasks, operands, s.pending, __func__)) return -1;
    s.initPending = true;
    s.initKind = dgq::INIT_CLASSICAL;
    const bool ok = planPending(s, __func__, false);
    for (auto &p : s.planned) p.isSingle = s.single ? 1 : 0;
    if (!ok) return -1;
    if (sweep < 0 || sweep >= (int) s.planned.size()) return (int) s.planned.size();
    const std::string src = dgq::generateSweepSource(s.planned[(size_t) sweep], s.plannedTileBits);
    std::strncpy(buf, src.c_str(), (size_t) len - 1);
    buf[len - 1] = '\0';
    return (int) src.size() < len ? (int) s.planned.size() : -2;
}

int dgq_compileSweepSource(const char *source, char *log, int len) {
    if (!source) return -1;
    std::vector<char> cubin;
    std::string lg;
    const bool ok = dgq::jitCompileOnly(source, cubin, lg);
    if (log && len > 0) {
        std::strncpy(log, lg.c_str(), (size_t) len - 1);
        log[len - 1] = '\0';
    }
    return ok ? (int) cubin.size() : -1;
}

// src/QuEST.h:1306 (declared, no body in dgQuEST): <bra|ket> for state-vectors
Complex calcInnerProduct(Qureg bra, Qureg ket) {
    Complex out{0.0, 0.0};
    if (!vStateVec(bra, __func__) || !vStateVec(ket, __func__)) return out;
    QuregState &b = *stateOf(bra);
    QuregState &k = *stateOf(ket);
    if (b.numQubits != k.numQubits) {
        raise(E_MISMATCHING_QUREG_DIMENSIONS, __func__);
        return out;
    }
    if (!vDeviceResident(b, __func__) || !vDeviceResident(k, __func__)) return out;
    if (!flush(b, __func__) || !flush(k, __func__)) return out;
    if (!cudaOk(cudaStreamSynchronize(b.stream), __func__) || !cudaOk(cudaStreamSynchronize(k.stream), __func__))
        return out;
    dgq::InnerArgs a;
    std::memset(&a, 0, sizeof(a));
    a.numReal = b.numQubits;
    a.identity = 1;
    for (int i = 0; i < b.numQubits; i++) {
        a.l2vBra[i] = (uint8_t) b.l2v[i];
        a.l2vKet[i] = (uint8_t) k.l2v[i];
        if (b.l2v[i] != i || k.l2v[i] != i) a.identity = 0;
    }
    a.braRestrict = b.restrictActive;
    a.braMask = b.rMask;
    a.braValue = b.rValue;
    a.braScale = b.rScale;
    a.ketRestrict = k.restrictActive;
    a.ketMask = k.rMask;
    a.ketValue = k.rValue;
    a.ketScale = k.rScale;
    double2 *dPart = nullptr, *dOut = nullptr;
    if (!cudaOk(cudaMalloc(&dPart, sizeof(double2) * (size_t) (dgq::innerNumCtas() + 1)), __func__)) return out;
    dOut = dPart + dgq::innerNumCtas();
    double2 h{0.0, 0.0};
    const bool ok = cudaOk(dgq::launchInner(b.dState, b.single, k.dState, k.single, a, dPart, dOut, b.stream), __func__) &&
                    cudaOk(cudaMemcpyAsync(&h, dOut, sizeof(h), cudaMemcpyDeviceToHost, b.stream), __func__) &&
                    cudaOk(cudaStreamSynchronize(b.stream), __func__);
    g_launches += 2;
    cudaFree(dPart);
    if (!ok) return out;
    out.real = h.x;
    out.imag = h.y;
    return out;
}

// src/QuEST.h:1539 (declared, no body in dgQuEST): |<pure|qureg>|^2 for state-vectors
qreal calcFidelity(Qureg qureg, Qureg pureState) {
    if (!vQureg(qureg, __func__) || !vQureg(pureState, __func__)) return 0.0;
    if (qureg.isDensityMatrix) {
        // <psi| rho |psi> on the host (include/QuEST.h:1539)
        if (pureState.isDensityMatrix) return raise(E_SECOND_ARG_MUST_BE_STATEVEC, __func__), 0.0;
        if (pureState.numQubitsRepresented != qureg.numQubitsRepresented)
            return raise(E_MISMATCHING_QUREG_DIMENSIONS, __func__), 0.0;
        QuregState &s = *stateOf(qureg);
        const int n = s.densityQubits;
        const uint64_t dim = 1ULL << n;
        std::vector<double> re(dim * dim), im(dim * dim), pr(dim), pi(dim);
        if (!readLogicalFor(s, re.data(), im.data(), __func__) ||
            !readLogicalFor(*stateOf(pureState), pr.data(), pi.data(), __func__))
            return 0.0;
        std::complex<double> f = 0.0;
        for (uint64_t c = 0; c < dim; c++) {
            std::complex<double> row = 0.0;  // (rho psi)_r summed against conj(psi_r) below
            for (uint64_t r = 0; r < dim; r++)
                row += std::conj(std::complex<double>(pr[r], pi[r])) *
                       std::complex<double>(re[r + (c << n)], im[r + (c << n)]);
            f += row * std::complex<double>(pr[c], pi[c]);
        }
        return f.real();
    }
    const Complex ip = calcInnerProduct(qureg, pureState);
    return ip.real * ip.real + ip.imag * ip.imag;
}

}  // extern "C"
