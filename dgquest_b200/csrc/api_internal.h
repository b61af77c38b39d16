// api_internal.h -- declarations shared by the translation units of the C API
// (api.cpp, api_gates.cpp, execute.cpp, readout.cpp, density.cpp,
// extensions.cpp): error reporting, register state access, validation,
// gate recording, planning and launch, memory, read-out helpers.
#pragma once

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

namespace dgq_api {

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

// The predictor also chooses the form of a plan (dgq_setDenseFusion(q, -1),
// the default): register-phase tiles, or the gates fused into dense blocks of
// K = 5, 6 or 7 qubits, each block one dense sweep. A dense sweep costs a
// fixed time per block per amplitude (denseMs, ms per block per 2^30
// amplitudes) for three variants: complex128 SIMT, complex64 SIMT and
// complex64 on the tensor cores (K = 5 and 6). Built-in: figures measured on
// B200 at 30 qubits (K = 6: 58.1, 37.4 and 5.5 ms; K = 5 on the tensor
// cores 5.24 ms), the SIMT K = 5 and 7 scaled by 2^K (the SIMT dense kernel
// is compute-bound, 8 x 2^K flops per amplitude). Tiles on a complex64
// register (the paired form) cost c64TileFactor times the complex128
// prediction (measured: 77 of 140 ms on the 30-qubit circuit). A dense form
// is taken when its prediction is below denseMargin times the tile form's.
enum DenseVariant { DV_F64 = 0, DV_C64 = 1, DV_C64_TC = 2 };

struct CostModel {
    double sweepSecondsPerAmp = 2.6e-3 / 1073741824.0;
    double phaseSecondsPerAmp = 1.8e-3 / 1073741824.0;
    double launchSeconds = 3e-6;
    double denseMs[3][3] = {{29.05, 58.1, 116.2}, {18.7, 37.4, 74.8}, {5.24, 5.5, 0.0}};  // [variant][K - 5]
    double c64TileFactor = 0.55;
    double denseMargin = 0.8;
};

const char *errorMessage(int code);
extern std::atomic<int> g_errMode;
extern thread_local int g_lastError;
extern thread_local std::string g_lastMessage;
extern thread_local int64_t g_errorCount;
extern std::atomic<int64_t> g_launches;
extern dgq::Mt19937 g_rng;
bool raise(int code, const char *func, const char *detail = nullptr);
bool cudaOk(cudaError_t e, const char *func);
double nowMillis();
QuregState *stateOf(const Qureg &q);
size_t ampBytes(const QuregState &s);
void resetMapping(QuregState &s);
u64 toVirtualMask(const QuregState &s, u64 logicalMask);
uint64_t toVirtualIndex(const QuregState &s, uint64_t logical);
bool vQureg(const Qureg &q, const char *func);
bool vTarget(const Qureg &q, int t, const char *func);
bool vControlTarget(const Qureg &q, int c, int t, const char *func);
bool vUniqueTargets(const Qureg &q, int a, int b, const char *func);
bool vMultiControls(const Qureg &q, const int *c, int n, const char *func);
bool vStateIndex(const Qureg &q, long long idx, const char *func);
bool vStateVec(const Qureg &q, const char *func);
bool vDensity(const Qureg &q, const char *func);
bool vOutcome(int o, const char *func);
bool isPairUnitary(Complex a, Complex b);
bool isMatrix2Unitary(const ComplexMatrix2 &u);
void push(QuregState &s, dgq::GateType type, u64 logicalTargets, u64 logicalControls, const double *op, int nop);
dgq::GateType conjugateGate(dgq::GateType type, const double *op, int nop, double *out);
void record(const Qureg &q, dgq::GateType type, u64 logicalTargets, u64 logicalControls, const double *op, int nop);
void recordMatrix(const Qureg &q, u64 targets, u64 controls, const ComplexMatrix2 &u);
u64 bit(int q);
bool normaliseLayout(QuregState &s, const char *func);
extern std::atomic<int64_t> g_deviceBudget;
extern std::atomic<int> g_tensorCores;
extern std::mutex g_costMutex;
extern CostModel g_cost;
extern bool g_costFileTried;
extern const char *kDenseVariantName[3];
void readCostFileExtras(const char *path, CostModel &cm);
bool readCostFile(const char *path, double &sweepMs, double &phaseMs);
CostModel costModel();
double predictPlanSeconds(const std::vector<Gate> &gates, int numBits, int W, const dgq::MatrixPool &pool,
                          int lookahead);
int chooseTileBits(QuregState &s);
double predictDenseSeconds(const QuregState &s, int K, int *blocksOut, double bound, bool *stopped);
int chooseForm(QuregState &s);
int chooseFormUncached(QuregState &s, const CostModel &cm);
extern std::atomic<int> g_jitMinBits;
bool pairedEnabled();
int pairedTileBits(const QuregState &s);
int jitMinBits();
extern std::atomic<int> g_specPolicy;
bool launchProgram(QuregState &s, size_t i, const char *func);
bool launchPlanned(QuregState &s, const char *func, size_t from = 0);
void setRenorm(QuregState &s, size_t i, size_t last, int &event);
bool planPending(QuregState &s, const char *func, bool specialise = true, bool launch = false);
cudaMemPool_t registerPool();
size_t poolSpare();
cudaError_t allocOn(void **ptr, size_t bytes, cudaStream_t st);
void freeOn(void *ptr, cudaStream_t st);
bool flush(QuregState &s, const char *func);
bool vDeviceResident(const QuregState &s, const char *func);
bool densityDiagonal(QuregState &s, std::vector<double> &diag, const char *func);
bool densityProbs(QuregState &s, const char *func);
bool ensureProbs(QuregState &s, const char *func);
bool readLogicalFor(QuregState &s, double *re, double *im, const char *func);

}  // namespace dgq_api

using namespace dgq_api;

// Replaces the register's state by (reals, imags) in logical order (api.cpp).
void loadAmps(QuregState &s, const double *reals, const double *imags, const char *func);
