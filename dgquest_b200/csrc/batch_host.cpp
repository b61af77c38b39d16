// batch_host.cpp -- the batched form: many registers, one persistent launch.
//
// dgq_batchCreate plans the pending gates of every register (host threads,
// one register at a time per thread), packs the sweep programs into flat
// device arrays, orders the work list (batch.h) and captures
//   memset(counters) -> memset(expectation sums) -> persistent kernel
// into a CUDA graph on the batch's own stream; dgq_batchLaunch replays it.
// The tile width and the number of registers interleaved sweep by sweep
// come from an autotuner that times the candidates on a sample of the batch
// (or from an explicit dgq_batch_config).
//
// There is no counterpart in dgQuEST, which simulates one register at a
// time; each register's sweeps are the same programs its own single-register
// launch would run, so the batched result equals the single-register one.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "batch.h"
#include "dgq.h"
#include "qureg_state.h"

namespace dgq {
bool raiseExternal(int code, const char *func, const char *detail);
}

namespace {

using dgq::BatchCircuit;
using dgq::BatchSweep;
using dgq::KOp;
using dgq::KPhase;
using dgq::TileProgram;

constexpr int E_SYS_TOO_BIG_FOR_DEVICE = 101;
constexpr int E_UNSUPPORTED = 102;
constexpr int E_CUDA = 103;
constexpr int E_INVALID_ARGUMENT = 104;

double nowMs() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One register's programs in compact form (offsets relative to the register).
struct RegPlan {
    int tileBits = 0;
    std::vector<BatchSweep> sweeps;
    std::vector<KPhase> phases;
    std::vector<KOp> ops;
    std::vector<double> coef;
    double flopsPerAmp = 0.0;
    int err = 0;
    std::string errMsg;
};

void compact(const std::vector<TileProgram> &progs, int W, RegPlan &out) {
    out.tileBits = W;
    for (const TileProgram &p : progs) {
        BatchSweep h;
        std::memset(&h, 0, sizeof(h));
        h.numPhases = p.numPhases;
        h.numOps = p.numOps;
        h.numBits = p.numBits;
        h.numReal = p.numReal;
        h.initKind = p.initKind;
        h.hasRestrict = p.hasRestrict;
        h.hasGlobal = p.hasGlobal;
        h.tileBits = W;
        h.globalRe = p.globalRe;
        h.globalIm = p.globalIm;
        h.initIndex = p.initIndex;
        h.initAmp = p.initAmp;
        h.restrictMask = p.restrictMask;
        h.restrictValue = p.restrictValue;
        h.restrictScale = p.restrictScale;
        h.phaseOff = (uint32_t) out.phases.size();
        h.opOff = (uint32_t) out.ops.size();
        h.coefOff = (uint32_t) out.coef.size();
        std::memcpy(h.highPos, p.highPos, sizeof(h.highPos));
        std::memcpy(h.ctaPos, p.ctaPos, sizeof(h.ctaPos));
        out.sweeps.push_back(h);
        out.phases.insert(out.phases.end(), p.phases, p.phases + p.numPhases);
        out.ops.insert(out.ops.end(), p.ops, p.ops + p.numOps);
        out.coef.insert(out.coef.end(), p.coef, p.coef + p.numCoef);
    }
}

int tileBitsFor(const QuregState &s, int maxTileBits) {
    return std::max(dgq::kMinTileBits, std::min(maxTileBits, s.numBits));
}

// Plans the registers `which` at tile width min(W, numBits), in parallel.
void planAll(const std::vector<QuregState *> &regs, const std::vector<int> &which, int W, std::vector<RegPlan> &plans) {
    plans.assign(which.size(), RegPlan());
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 4;
    nt = std::min<unsigned>(nt, 32u);
    nt = std::min<unsigned>(nt, (unsigned) std::max<size_t>(1, which.size()));
    std::atomic<size_t> next{0};
    auto work = [&]() {
        std::vector<TileProgram> progs;
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= which.size()) break;
            QuregState &s = *regs[which[i]];
            const int w = tileBitsFor(s, W);
            dgq::PlanStats st;
            std::string err;
            const int code = dgq::buildPrograms(s, w, progs, st, err);
            if (code) {
                plans[i].err = code;
                plans[i].errMsg = err;
                continue;
            }
            bool dense = false;
            for (const auto &pg : progs) dense = dense || pg.denseK;
            if (dense) {
                plans[i].err = E_UNSUPPORTED;
                plans[i].errMsg = "a batch register uses a multi-qubit unitary of more than 4 targets";
                continue;
            }
            compact(progs, w, plans[i]);
            plans[i].flopsPerAmp = st.flopsPerAmp;
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
}

struct DeviceBatch {
    BatchCircuit *circ = nullptr;
    BatchSweep *sweeps = nullptr;
    KPhase *phases = nullptr;
    KOp *ops = nullptr;
    double2 *leanCoef = nullptr;
    double *coef = nullptr;
    uint64_t *items = nullptr;
    uint32_t *counters = nullptr;  // ticket, then the done counters
    double *zsum = nullptr;
    uint32_t *error = nullptr;
    size_t numCounters = 0, numZ = 0, numItems = 0;
    int64_t programBytes = 0;
    int maxTileBits = 0, grid = 0, ctasPerSm = 0;
    int numSweeps = 0, whole = 0;
    std::vector<uint32_t> zOff;  // per register of the batch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        void *ptrs[] = {circ, sweeps, phases, ops, leanCoef, coef, items, counters, zsum, error};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        *this = DeviceBatch();
    }
};

template <class T>
cudaError_t upload(T **dst, const std::vector<T> &src, int64_t *bytes) {
    const size_t n = std::max<size_t>(1, src.size()) * sizeof(T);
    cudaError_t e = cudaMalloc((void **) dst, n);
    if (e != cudaSuccess) return e;
    if (bytes) *bytes += (int64_t) (src.size() * sizeof(T));
    if (src.empty()) return cudaSuccess;
    return cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// Builds the device arrays, the work list and the graph for the registers
// `which` (indices into regs) planned as `plans`.
cudaError_t buildDevice(const std::vector<QuregState *> &regs, const std::vector<int> &which,
                        const std::vector<RegPlan> &plans, bool single, int maxTileBits, int groupFactor,
                        int ctasPerSm, cudaStream_t stream, DeviceBatch &d) {
    d.release();
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int maxCtas = dgq::batchCtasPerSm(single, maxTileBits);
    if (maxCtas < 1) return cudaErrorInvalidConfiguration;
    d.ctasPerSm = ctasPerSm > 0 ? std::min(ctasPerSm, maxCtas) : maxCtas;
    d.grid = sms * d.ctasPerSm;
    d.maxTileBits = maxTileBits;

    std::vector<BatchCircuit> circ(which.size());
    std::vector<BatchSweep> sweeps;
    std::vector<KPhase> phases;
    std::vector<KOp> ops;
    std::vector<double> coef;
    d.zOff.assign(which.size(), 0);
    uint32_t doneOff = 1;  // counters[0] is the ticket
    uint32_t zOff = 0;
    for (size_t i = 0; i < which.size(); i++) {
        const QuregState &s = *regs[which[i]];
        const RegPlan &p = plans[i];
        BatchCircuit &c = circ[i];
        std::memset(&c, 0, sizeof(c));
        c.state = s.dState;
        c.numBits = (uint32_t) s.numBits;
        c.tileBits = (uint32_t) p.tileBits;
        c.numSweeps = (uint32_t) p.sweeps.size();
        c.firstSweep = (uint32_t) sweeps.size();
        c.zOff = zOff;
        c.doneOff = doneOff;
        c.tilesPerSweep = 1u << (s.numBits - p.tileBits);
        d.zOff[i] = zOff;
        zOff += (uint32_t) s.numBits + 1;
        doneOff += c.numSweeps;
        for (BatchSweep h : p.sweeps) {
            h.phaseOff += (uint32_t) phases.size();
            h.opOff += (uint32_t) ops.size();
            h.coefOff += (uint32_t) coef.size();
            sweeps.push_back(h);
        }
        phases.insert(phases.end(), p.phases.begin(), p.phases.end());
        ops.insert(ops.end(), p.ops.begin(), p.ops.end());
        coef.insert(coef.end(), p.coef.begin(), p.coef.end());
    }
    d.numSweeps = (int) sweeps.size();
    d.numCounters = doneOff;
    bool dense = false, lean = true;
    for (const KOp &op : ops) {
        dense = dense || op.kind == dgq::KOP_DENSE;
        lean = lean && ((dgq::kLeanKinds >> op.kind) & 1u);
    }
    const int form = dense ? dgq::kBatchFormDense : lean ? dgq::kBatchFormLean : dgq::kBatchFormGeneral;
    // the lean form reads each op's (at most two) coefficients beside its record
    std::vector<double2> leanCoef;
    if (form == dgq::kBatchFormLean) {
        leanCoef.assign(ops.size(), make_double2(0.0, 0.0));
        for (const BatchSweep &h : sweeps)
            for (int o = 0; o < h.numOps; o++) {
                const size_t c = (size_t) h.coefOff + ops[h.opOff + o].coef;
                if (c < coef.size()) leanCoef[h.opOff + o].x = coef[c];
                if (c + 1 < coef.size()) leanCoef[h.opOff + o].y = coef[c + 1];
            }
    }
    d.numZ = std::max<uint32_t>(1, zOff);

    // work list: largest registers first; registers of several tiles in
    // groups of about groupFactor x grid tiles, sweep by sweep inside a group;
    // single-tile registers (whole-register items) last
    std::vector<size_t> order(which.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return circ[a].numBits > circ[b].numBits; });
    std::vector<uint64_t> items;
    const uint64_t budget = (uint64_t) std::max(1, groupFactor) * (uint64_t) d.grid;
    size_t k = 0;
    while (k < order.size() && circ[order[k]].tilesPerSweep > 1) {
        std::vector<size_t> group;
        uint64_t tiles = 0;
        while (k < order.size() && circ[order[k]].tilesPerSweep > 1 && (group.empty() || tiles < budget)) {
            group.push_back(order[k]);
            tiles += circ[order[k]].tilesPerSweep;
            k++;
        }
        uint32_t maxS = 0;
        for (size_t g : group) maxS = std::max(maxS, circ[g].numSweeps);
        for (uint32_t sw = 0; sw < maxS; sw++)
            for (size_t g : group)
                if (sw < circ[g].numSweeps)
                    for (uint32_t t = 0; t < circ[g].tilesPerSweep; t++)
                        items.push_back(dgq::batchItem((uint32_t) g, sw, t));
    }
    d.whole = 0;
    for (; k < order.size(); k++) {
        if (circ[order[k]].numSweeps == 0) continue;
        items.push_back(dgq::batchItem((uint32_t) order[k], dgq::kBatchWhole, 0));
        d.whole++;
    }
    d.numItems = items.size();

    d.programBytes = 0;
    if ((e = upload(&d.circ, circ, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.sweeps, sweeps, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.phases, phases, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.ops, ops, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.leanCoef, leanCoef, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.coef, coef, &d.programBytes)) != cudaSuccess) return e;
    if ((e = upload(&d.items, items, &d.programBytes)) != cudaSuccess) return e;
    if ((e = cudaMalloc((void **) &d.counters, d.numCounters * sizeof(uint32_t))) != cudaSuccess) return e;
    if ((e = cudaMalloc((void **) &d.zsum, d.numZ * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc((void **) &d.error, sizeof(uint32_t))) != cudaSuccess) return e;

    dgq::BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.circ = d.circ;
    a.sweeps = d.sweeps;
    a.phases = d.phases;
    a.ops = d.ops;
    a.leanCoef = d.leanCoef;
    a.coef = d.coef;
    a.items = d.items;
    a.numItems = (uint32_t) d.numItems;
    a.spinLimit = 1u << 22;  // polls of >= 256 ns each: a second or more
    a.ticket = d.counters;
    a.done = d.counters;
    a.zsum = d.zsum;
    a.error = d.error;

    e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t e1 = cudaMemsetAsync(d.counters, 0, d.numCounters * sizeof(uint32_t), stream);
    if (e1 == cudaSuccess) e1 = cudaMemsetAsync(d.zsum, 0, d.numZ * sizeof(double), stream);
    if (e1 == cudaSuccess) e1 = cudaMemsetAsync(d.error, 0, sizeof(uint32_t), stream);
    if (e1 == cudaSuccess && d.numItems > 0) e1 = dgq::launchBatch(a, single, maxTileBits, d.grid, form, stream);
    e = cudaStreamEndCapture(stream, &d.graph);
    if (e1 != cudaSuccess) return e1;
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&d.exec, d.graph, 0);
}

struct TunedConfig {
    int maxTileBits, groupFactor, ctasPerSm;
};
std::mutex g_tuneMutex;
std::map<std::string, TunedConfig> g_tuned;

// precision, and how many registers have each address width
std::string signature(const std::vector<QuregState *> &regs, bool single) {
    int hist[dgq::kMaxStateBits + 1] = {0};
    for (const QuregState *s : regs) hist[s->numBits]++;
    std::string k = single ? "c64:" : "c128:";
    for (int b = 0; b <= dgq::kMaxStateBits; b++)
        if (hist[b]) k += std::to_string(b) + "x" + std::to_string(hist[b]) + ",";
    return k;
}

bool fail(int code, const char *func, const char *detail) { return dgq::raiseExternal(code, func, detail); }

bool cudaCheck(cudaError_t e, const char *func) {
    if (e == cudaSuccess) return true;
    return fail(E_CUDA, func, cudaGetErrorString(e));
}

// Times one configuration on a sample: ms per launch (the best of two after
// a warm-up launch); failed or timed-out configurations rank last.
double timeConfig(const std::vector<QuregState *> &regs, const std::vector<int> &sample,
                  const std::vector<RegPlan> &plans, bool single, const TunedConfig &c, cudaStream_t stream) {
    DeviceBatch d;
    if (buildDevice(regs, sample, plans, single, c.maxTileBits, c.groupFactor, c.ctasPerSm, stream, d) !=
        cudaSuccess) {
        d.release();
        cudaGetLastError();
        return 1e30;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e30;
    cudaGraphLaunch(d.exec, stream);
    for (int r = 0; r < 2; r++) {
        cudaEventRecord(e0, stream);
        cudaGraphLaunch(d.exec, stream);
        cudaEventRecord(e1, stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, (double) ms);
    }
    uint32_t err = 0;
    cudaMemcpy(&err, d.error, sizeof(err), cudaMemcpyDeviceToHost);
    if (err) best = 1e30;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    d.release();
    return best;
}

}  // namespace

struct dgq_batch_s {
    std::vector<QuregState *> regs;
    bool single = false;
    cudaStream_t stream = nullptr;
    DeviceBatch d;
    dgq_batch_stats stats{};
    bool launched = false;
};

extern "C" {

dgq_batch dgq_batchCreate(const Qureg *quregs, int count, const dgq_batch_config *cfg) {
    const char *fn = "dgq_batchCreate";
    if (!quregs || count < 1) {
        fail(E_INVALID_ARGUMENT, fn, "no registers");
        return nullptr;
    }
    const double t0 = nowMs();
    dgq_batch b = new dgq_batch_s();
    b->regs.resize(count);
    bool allInit = true;
    int maxBits = 0;
    auto abandon = [&](int code, const char *detail) -> dgq_batch {
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        fail(code, fn, detail);
        return nullptr;
    };
    for (int i = 0; i < count; i++) {
        QuregState *s = quregs[i].state;
        if (!s) return abandon(E_INVALID_ARGUMENT, "a register handle is not initialised");
        if (s->hostTier) return abandon(E_UNSUPPORTED, "a register held in host memory");
        if (s->sharded) return abandon(E_UNSUPPORTED, "a sharded register");
        if (s->densityQubits) return abandon(E_UNSUPPORTED, "a density matrix");
        b->regs[i] = s;
        if (i == 0) b->single = s->single;
        if (s->single != b->single) return abandon(E_UNSUPPORTED, "a batch holds registers of one precision");
        if (!s->initPending) allInit = false;
        maxBits = std::max(maxBits, s->numBits);
    }
    // work items carry the register in 20 bits, the sweep in 16 and the tile in 28
    if (count > (1 << 20)) return abandon(E_INVALID_ARGUMENT, "more than 2^20 registers");
    if (maxBits - dgq::kMinTileBits > 28) return abandon(E_UNSUPPORTED, "a register wider than 37 qubits");
    {
        std::vector<QuregState *> sorted = b->regs;
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            return abandon(E_INVALID_ARGUMENT, "a register appears twice in the batch");
    }
    // the registers' earlier work must be done before the batch stream runs
    for (QuregState *s : b->regs)
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) return abandon(E_CUDA, "register stream failed");
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return abandon(E_CUDA, "cudaStreamCreate failed");
    std::vector<int> all(count);
    for (int i = 0; i < count; i++) all[i] = i;

    TunedConfig chosen{std::min(dgq::kBatchMaxTileBits, std::max(dgq::kMinTileBits, maxBits)), 2, 0};
    bool tune = !cfg || cfg->tune;
    if (cfg && cfg->tileBits) chosen.maxTileBits = cfg->tileBits;
    if (cfg && cfg->groupFactor) chosen.groupFactor = cfg->groupFactor;
    if (cfg && cfg->ctasPerSm) chosen.ctasPerSm = cfg->ctasPerSm;
    if (chosen.maxTileBits < dgq::kMinTileBits || chosen.maxTileBits > dgq::kBatchMaxTileBits)
        return abandon(E_INVALID_ARGUMENT, "tileBits must be 9..12");
    const char *envTune = getenv("DGQ_BATCH_TUNE");
    if (envTune && atoi(envTune) == 0) tune = false;
    // tuning launches overwrite the states: only when every register restarts
    // from an initialisation (which every launch recomputes)
    if (!allInit) tune = false;
    double tuneMs = 0.0;
    const std::string sig = signature(b->regs, b->single);
    if (tune) {
        std::lock_guard<std::mutex> lk(g_tuneMutex);
        auto it = g_tuned.find(sig);
        if (it != g_tuned.end()) {
            chosen = it->second;
            tune = false;
        }
    }
    if (tune) {
        const double tt = nowMs();
        // sample: every 8th register of the size-sorted list (about 1/8 of the work)
        std::vector<int> bySize = all;
        std::stable_sort(bySize.begin(), bySize.end(),
                         [&](int x, int y) { return b->regs[x]->numBits > b->regs[y]->numBits; });
        const int stride = count >= 64 ? 8 : 1;
        std::vector<int> sample;
        for (int i = 0; i < count; i += stride) sample.push_back(bySize[i]);
        std::vector<int> widths;
        for (int w = dgq::kMinTileBits + 1; w <= dgq::kBatchMaxTileBits; w++)
            if (w <= std::max(dgq::kMinTileBits, maxBits)) widths.push_back(w);
        if (widths.empty()) widths.push_back(dgq::kMinTileBits);
        double best = 1e30;
        for (int w : widths) {
            std::vector<RegPlan> sp;
            planAll(b->regs, sample, w, sp);
            bool ok = true;
            for (const auto &p : sp) ok = ok && p.err == 0;
            if (!ok) continue;
            for (int gf : {1, 2, 4}) {
                const TunedConfig c{w, gf, 0};
                const double ms = timeConfig(b->regs, sample, sp, b->single, c, b->stream);
                if (ms < best) {
                    best = ms;
                    chosen = c;
                }
            }
        }
        tuneMs = nowMs() - tt;
        std::lock_guard<std::mutex> lk(g_tuneMutex);
        g_tuned[sig] = chosen;
    }
    std::vector<RegPlan> plans;
    planAll(b->regs, all, chosen.maxTileBits, plans);
    double flops = 0.0;
    int64_t gates = 0;
    for (int i = 0; i < count; i++) {
        if (!plans[i].err && plans[i].sweeps.size() >= dgq::kBatchWhole) {
            plans[i].err = E_UNSUPPORTED;
            plans[i].errMsg = "a register needs 65535 or more sweeps";
        }
        if (plans[i].err) {
            const std::string msg = plans[i].errMsg;
            return abandon(plans[i].err, msg.c_str());
        }
        flops += plans[i].flopsPerAmp * (double) (1ULL << b->regs[i]->numBits);
        gates += (int64_t) b->regs[i]->pending.size();
    }
    const double planMs = nowMs() - t0 - tuneMs;
    cudaError_t e = buildDevice(b->regs, all, plans, b->single, chosen.maxTileBits, chosen.groupFactor,
                                chosen.ctasPerSm, b->stream, b->d);
    if (e != cudaSuccess) {
        b->d.release();
        return abandon(e == cudaErrorMemoryAllocation ? E_SYS_TOO_BIG_FOR_DEVICE : E_CUDA, cudaGetErrorString(e));
    }
    for (QuregState *s : b->regs) dgq::consumePending(*s);

    dgq_batch_stats &st = b->stats;
    st.registers = count;
    st.wholeRegisters = b->d.whole;
    st.sweeps = b->d.numSweeps;
    st.tileBits = chosen.maxTileBits;
    st.groupFactor = chosen.groupFactor;
    st.grid = b->d.grid;
    st.ctasPerSm = b->d.ctasPerSm;
    st.tuned = tuneMs > 0.0 ? 1 : 0;
    st.items = (int64_t) b->d.numItems;
    st.gates = gates;
    st.programBytes = b->d.programBytes;
    int64_t stateBytes = 0, sweepBytes = 0;
    for (int i = 0; i < count; i++) {
        const int64_t bytes = (int64_t) (b->single ? 8 : 16) << b->regs[i]->numBits;
        stateBytes += bytes;
        sweepBytes += 2 * bytes * (int64_t) plans[i].sweeps.size();
    }
    st.stateBytes = stateBytes;
    st.sweepBytes = sweepBytes;
    st.planMillis = planMs;
    st.tuneMillis = tuneMs;
    st.flopsPerLaunch = flops;
    return b;
}

int dgq_batchLaunch(dgq_batch b) {
    if (!b || !b->d.exec) return fail(E_INVALID_ARGUMENT, "dgq_batchLaunch", "null batch") ? 0 : -1;
    if (!cudaCheck(cudaGraphLaunch(b->d.exec, b->stream), "dgq_batchLaunch")) return -1;
    for (QuregState *s : b->regs) s->probsValid = false;
    b->launched = true;
    return 0;
}

int dgq_batchWait(dgq_batch b) {
    const char *fn = "dgq_batchWait";
    if (!b) return fail(E_INVALID_ARGUMENT, fn, "null batch") ? 0 : -1;
    if (!cudaCheck(cudaStreamSynchronize(b->stream), fn)) return -1;
    uint32_t err = 0;
    if (!cudaCheck(cudaMemcpy(&err, b->d.error, sizeof(err), cudaMemcpyDeviceToHost), fn)) return -1;
    if (err) return fail(E_CUDA, fn, "a sweep of the batch waited too long for the previous sweep") ? 0 : -1;
    return 0;
}

int dgq_batchExpectationZ(dgq_batch b, double *out) {
    const char *fn = "dgq_batchExpectationZ";
    if (!b || !out) return fail(E_INVALID_ARGUMENT, fn, "null batch or output") ? 0 : -1;
    if (!b->launched) return fail(E_INVALID_ARGUMENT, fn, "the batch has not been launched") ? 0 : -1;
    if (dgq_batchWait(b) != 0) return -1;
    std::vector<double> z(b->d.numZ);
    if (!cudaCheck(cudaMemcpy(z.data(), b->d.zsum, z.size() * sizeof(double), cudaMemcpyDeviceToHost), fn))
        return -1;
    size_t o = 0;
    for (size_t i = 0; i < b->regs.size(); i++) {
        const QuregState &s = *b->regs[i];
        const double *zs = z.data() + b->d.zOff[i];
        const double tot = zs[s.numBits];
        for (int q = 0; q < s.numQubits; q++) {
            const double one = zs[s.l2v[q]];
            out[o++] = tot > 0.0 ? (tot - 2.0 * one) / tot : 0.0;
        }
    }
    return 0;
}

int dgq_batchGetStats(dgq_batch b, dgq_batch_stats *out) {
    if (!b || !out) return fail(E_INVALID_ARGUMENT, "dgq_batchGetStats", "null batch or output") ? 0 : -1;
    *out = b->stats;
    return 0;
}

void *dgq_batchGetStream(dgq_batch b) { return b ? (void *) b->stream : nullptr; }

void dgq_batchDestroy(dgq_batch b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->d.release();
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
