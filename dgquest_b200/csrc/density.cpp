// density.cpp -- density-matrix calls declared in dgQuEST's header without
// bodies (include/QuEST.h:1373-1539), with upstream QuEST's semantics: the
// five noise channels as superoperators on the row and column qubits of the
// vectorised matrix, mixing and purity.
#include "api_internal.h"

using dgq::Gate;

extern "C" {
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

}  // extern "C"
