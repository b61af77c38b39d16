// api.cpp -- the QuEST C API of libdgq: errors and validation (codes and
// messages of src/QuEST_validation.c:19-80), the environment, register
// creation and destruction, the logical->virtual qubit map, gate recording
// (src/cpp/QuEST_distributed.cpp:118-364) and the state initialisers.
// Gates record lazily; a read-out plans and runs what is pending
// (QuEST_distributed.cpp:106-116). The engine behind the API: execute.cpp
// (planning and launches), readout.cpp, api_gates.cpp, density.cpp,
// extensions.cpp; shared declarations in api_internal.h.
#include "api_internal.h"

using dgq::Gate;

// ====================================================================
// errors (codes and messages of src/QuEST_validation.c:19-80)
// ====================================================================
namespace dgq_api {

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
bool raise(int code, const char *func, const char *detail) {
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

}  // namespace dgq_api

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

namespace dgq_api {

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

}  // namespace dgq_api

namespace dgq_api {
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

}  // namespace dgq_api

namespace dgq {
bool planForPages(QuregState &s, const char *func) { return planPending(s, func, true, false); }
}  // namespace dgq

extern "C" {
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

}  // extern "C"

// Replaces the register's vector by (reals, imags), 2^numQubits entries in
// logical order (a density register's vectorisation).
void loadAmps(QuregState &s, const double *reals, const double *imags, const char *func) {
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
        // every page is written below: none is all-zero any more
        if (s.hostTier) s.pageZero.assign(s.pageZero.size(), 0);
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

extern "C" {

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
        // shards: read, change and write back the whole state (virtual order);
        // host tier: all-zero pages get their zeros first
        dgq::hostTierMaterialise(s);
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
        t.pageZero = c.pageZero;
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

}  // extern "C"
