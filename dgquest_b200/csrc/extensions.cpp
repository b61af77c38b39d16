// extensions.cpp -- entry points of include/dgq.h that have no dgQuEST
// counterpart: error mode, op-list recording, sampling, plan statistics and
// the plan/launch split, cost-model settings, device state access, the
// host-only planner and kernel-source calls, the FP64 peak probe.
#include "api_internal.h"

using dgq::Gate;

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

}  // extern "C"

extern "C" {
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

}  // extern "C"

extern "C" {
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

int dgq_specialiseGates(int numQubits, int precision, int count, const int32_t *types, const uint64_t *targetMasks,
                        const uint64_t *controlMasks, const double *operands, int background) {
    if (numQubits < 1 || numQubits > dgq::kMaxStateBits - 2 || count < 0 || precision < 1 || precision > 3 ||
        (count > 0 && (!types || !targetMasks || !controlMasks || !operands))) {
        raise(E_INVALID_ARGUMENT, __func__);
        return -1;
    }
    if (!dgq::jitEnabled()) return 0;
    // the plan a register of this size and precision makes for these gates
    // after initZeroState (the same planning as dgq_sweepSource)
    QuregState s;
    s.numQubits = numQubits;
    s.numBits = std::max(numQubits, dgq::kMinTileBits);
    s.single = precision == 1 || precision == 3;
    s.allowPaired = precision == 1;
    resetMapping(s);
    if (!gatesFromArrays(numQubits, count, types, targetMasks, controlMasks, operands, s.pending, __func__)) return -1;
    s.initPending = true;
    s.initKind = dgq::INIT_CLASSICAL;
    if (!planPending(s, __func__, false)) return -1;
    std::vector<std::string> sources;
    for (auto &p : s.planned) {
        p.isSingle = s.single ? 1 : 0;
        if (!p.denseK) sources.push_back(dgq::generateSweepSource(p, s.plannedTileBits));
    }
    if (background) {
        dgq::jitCompileInBackground(sources);
        return (int) sources.size();
    }
    std::vector<CUfunction> fns;
    std::string err;
    if (!dgq::jitGetKernels(sources, fns, nullptr, &err)) {
        raise(E_UNSUPPORTED, __func__, err.c_str());
        return -1;
    }
    return (int) sources.size();
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

}  // extern "C"
