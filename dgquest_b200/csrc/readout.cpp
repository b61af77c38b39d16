// readout.cpp -- read-outs of the QuEST C API: P(q = 0) for every qubit in
// one pass (src/cpp/QuEST_gpu_kernel.cu:656-840), getAmp
// (src/cpp/QuEST_backend_distributed.cpp:649-663), collapse and
// measurement with MT19937 (src/QuEST_common.c:97-152), the state in
// logical order, inner products and fidelity; density registers read their
// diagonal on the device.
#include "api_internal.h"

using dgq::Gate;

namespace dgq_api {

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

}  // namespace dgq_api

extern "C" {
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
        // the flushed state is in pinned host memory (an all-zero page is not read)
        if (dgq::hostTierPageZero(s, v)) {
            a = make_double2(0.0, 0.0);
        } else if (s.single) {
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

}  // extern "C"

extern "C" {
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
            const bool keep = (!s.restrictActive || (v & s.rMask) == s.rValue) && !dgq::hostTierPageZero(s, v);
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

namespace dgq_api {
bool readLogicalFor(QuregState &s, double *re, double *im, const char *func) { return readLogical(s, re, im, func); }
}  // namespace dgq_api

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

}  // extern "C"

extern "C" {
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

