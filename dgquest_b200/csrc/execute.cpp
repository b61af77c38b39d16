// execute.cpp -- from recorded gates to kernel launches: the cost model and
// its choice of tile width and form (the recast of dgQuEST's time predictor,
// src/cpp/time_predictor.cpp:201-395), planning pending gates into sweep
// programs (dense sweeps included), the complex64 renormalisation schedule,
// launches on the register's stream, and the register memory pool.
#include "api_internal.h"

#include <unordered_map>

using dgq::Gate;

namespace dgq_api {
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
// complex64 dense 5- and 6-qubit sweeps on the tensor cores (dgq_setTensorCores)
std::atomic<int> g_tensorCores{1};

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
// The form choice of a gate-list structure, kept for later plans of the same
// structure (a circuit run again with the same gates on the same register
// shape): the choice depends on the gates' types, qubits and target orders,
// the register's shape and settings and the cost model, not on angles
// (except through merges that cancel gates, which only makes a kept choice
// less than optimal, never wrong). It saves the candidate planning, about
// 6 ms of a 30-qubit circuit's 10 ms of planning.
struct FormChoice {
    int formK = 0, tileBits = 0, lookahead = -1;
    double tileSeconds = 0.0;
    dgq_plan_stats stats{};
};
std::mutex g_formMutex;
std::unordered_map<uint64_t, FormChoice> g_formCache;

uint64_t formKey(const QuregState &s, const CostModel &cm) {
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&](const void *p, size_t n) {
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ULL;
    };
    const int32_t shape[5] = {s.numBits, s.single ? 1 : 0, s.tileBitsSetting, g_tensorCores.load(),
                              (int32_t) s.pending.size()};
    mix(shape, sizeof(shape));
    mix(&cm, sizeof(cm));
    for (const Gate &g : s.pending) {
        const int32_t t = (int32_t) g.type;
        mix(&t, sizeof(t));
        mix(&g.targetMask, sizeof(g.targetMask));
        mix(&g.controlMask, sizeof(g.controlMask));
        if (g.type == dgq::OP_MULTI_UNITARY) mix(g.multiTargets, sizeof(int32_t) * (size_t) g.numMultiTargets);
    }
    return h;
}

int chooseForm(QuregState &s) {
    const CostModel cm = costModel();
    const uint64_t key = formKey(s, cm);
    {
        std::lock_guard<std::mutex> lk(g_formMutex);
        auto it = g_formCache.find(key);
        if (it != g_formCache.end()) {
            const FormChoice &f = it->second;
            s.formTileBits = f.tileBits;
            s.formLookahead = f.lookahead;
            s.planLookahead = f.lookahead;
            s.predictedTileSeconds = f.tileSeconds;
            s.stats.predictedTileMs = f.stats.predictedTileMs;
            for (int i = 0; i < 3; i++) s.stats.predictedDenseMs[i] = f.stats.predictedDenseMs[i];
            s.stats.denseBound = f.stats.denseBound;
            return f.formK;
        }
    }
    const int formK = chooseFormUncached(s, cm);
    FormChoice f;
    f.formK = formK;
    f.tileBits = s.formTileBits;
    f.lookahead = s.formLookahead;
    f.tileSeconds = s.predictedTileSeconds;
    f.stats = s.stats;
    std::lock_guard<std::mutex> lk(g_formMutex);
    if (g_formCache.size() >= 256) g_formCache.clear();
    g_formCache[key] = f;
    return formK;
}

int chooseFormUncached(QuregState &s, const CostModel &cm) {
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

}  // namespace dgq_api

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

namespace dgq_api {

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
bool launchPlanned(QuregState &s, const char *func, size_t from) {
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
bool planPending(QuregState &s, const char *func, bool specialise, bool launch) {
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

}  // namespace dgq_api
