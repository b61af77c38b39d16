// qureg_state.h -- the engine state behind a Qureg handle (shared by the
// register API in api.cpp and the batched form in batch_host.cpp).
#pragma once

#include <functional>

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "QuEST.h"
#include "dgq.h"
#include "ir.h"
#include "planner.h"
#include "tile_program.h"

struct QuregState {
    int numQubits = 0;  // user-visible qubits (density registers: 2 x densityQubits)
    // density matrix of densityQubits qubits (0: a state vector), held as the
    // state vector of its 2 x densityQubits-qubit vectorisation: element
    // (row r, column c) at index r + (c << densityQubits)
    int densityQubits = 0;
    int numBits = 0;    // address bits of the buffer (>= numQubits, >= kMinTileBits)
    bool single = false;  // complex64 amplitudes (float2) instead of complex128
    void *dState = nullptr;
    cudaStream_t stream = nullptr;

    // recorded, not yet executed
    std::vector<dgq::Gate> pending;
    dgq::MatrixPool pool;
    bool initPending = false;
    int32_t initKind = dgq::INIT_NONE;
    uint64_t initIndex = 0;
    double initAmp = 0.0;

    // lazy measurement collapse applied to the state in HBM
    bool restrictActive = false;
    uint64_t rMask = 0, rValue = 0;
    double rScale = 1.0;

    // logical qubit -> address bit (swapGate relabels instead of moving data)
    int l2v[64];
    int v2l[64];

    // P(bit = 0) per address bit, of the (collapsed, normalised) state
    bool probsValid = false;
    std::vector<double> p0;
    double totalProb = 1.0;
    double *dPartial = nullptr;
    size_t partialCap = 0;
    double *dProbOut = nullptr;
    double *dNorm = nullptr;  // complex64 renormalisation: two running sums of |a|^2

    int tileBitsSetting = 0;  // 0 = cost model
    int planLookahead = -1;   // block selection with lookahead (the cost model's choice; -1: by size)
    bool allowPaired = true;  // complex64: the paired form where it applies
    int denseFusion = -1;     // > 0: gates fused into dense blocks of this many qubits;
                              // -1: the predictor chooses tiles or dense blocks per plan
    double predictedTileSeconds = 0.0;  // the tile-width choice's predicted plan time
    int formTileBits = 0;   // the form choice's tile width for the plan being made (0: none)
    int formLookahead = -1;
    // matrices of the planned dense sweeps (host copy and device buffer)
    std::vector<double> denseHost;
    double *dDense = nullptr;
    bool plannedPaired = false;
    std::vector<dgq::TileProgram> planned;
    std::vector<CUfunction> plannedFns;  // runtime-specialised kernel per program (or null)
    int plannedTileBits = 0;
    dgq_plan_stats stats{};

    // host tier (states larger than the device budget): the state lives in
    // pinned host memory in pages of 2^pageBits amplitudes (address bits
    // below pageBits); every pass streams the pages through device buffers,
    // one CUDA stream per buffer, and gates on page-index bits are first
    // brought into the page by a page-pair exchange of two address bits
    bool hostTier = false;
    void *hState = nullptr;
    // pageZero[p] = 1: page p holds only zeros and its host memory is stale
    // (never read: passes skip it or clear its device buffer, read-outs see
    // zeros); the counterpart of dgQuEST's all-zero pages (OPTIMIZE_ZERO,
    // src/cpp/QuEST_backend_distributed.cpp:17,343-347)
    std::vector<uint8_t> pageZero;
    int pageBits = 0;
    static constexpr int kPageBufs = 4;
    void *dPage[kPageBufs] = {};
    cudaStream_t pageStream[kPageBufs] = {};
    double *dPagePartial[kPageBufs] = {};
    double *dPageOut[kPageBufs] = {};
    size_t pagePartialCap = 0;
    // sharded register: 2^shardBits shards of 2^pageBits amplitudes, shard
    // k holding global indices [k << pageBits, (k + 1) << pageBits) in HBM of
    // device shardDev[k] (shards may share a device); a gate on a
    // shard-index bit first exchanges it (with any other shard-index bits
    // needed soon) for shard bits, in one pass over blocks of shard pairs
    bool sharded = false;
    int shardBits = 0;
    int homeDevice = 0;  // the device of `stream` and of the read-out buffers
    static constexpr int kMaxShards = 16;
    void *dShard[kMaxShards] = {};
    int shardDev[kMaxShards] = {};
    cudaStream_t shardStream[kMaxShards] = {};
    double *dShardPartial[kMaxShards] = {};
    double *dShardOut[kMaxShards] = {};
    size_t shardPartialCap = 0;

    // counters of the host tier and of sharded registers
    int64_t hostTierSwaps = 0;   // page-pair (shard-pair) exchange passes run so far
    int64_t hostTierPasses = 0;  // page (shard) passes: sweep segments and read-outs
    int64_t hostTierBytes = 0;   // host tier: bytes copied between host and device;
                                 // shards: bytes that crossed between shards
};

namespace dgq {

// Plans the register's pending gates (and pending initialisation or
// collapse) into sweep programs of tile width W. Returns 0, or the QuEST
// error code with err set. The register is not changed.
// paired: the complex64 paired form (TileProgram::paired; W counts the
// in-slot bit, so W - 1 tile bits index 16-byte slots).
// emit (if set) is called with the index of each program as soon as it is
// complete, in order; when it returns false, planning stops and
// buildPrograms returns -1 (the callback has reported its own error).
int buildPrograms(QuregState &s, int W, std::vector<TileProgram> &out, PlanStats &st, std::string &err,
                  bool paired = false, const std::function<bool(size_t)> &emit = nullptr);
// Drops the pending work that buildPrograms planned (after it has been
// launched or kept for launching).
void consumePending(QuregState &s);

// Plans the register's pending gates (and pending initialisation or
// collapse) into s.planned / s.plannedFns, compiling kernels as needed,
// without launching (api.cpp).
bool planForPages(QuregState &s, const char *func);

// host tier (host_tier.cpp). attach: allocates the pinned state and the
// page buffers for a device budget of budgetBytes (false with err set when
// they cannot be had); flush: runs the pending work over the pages;
// probs: P(bit = 0) for every address bit and the total probability of the
// (collapsed, unscaled) state.
bool hostTierAttach(QuregState &s, size_t budgetBytes, std::string &err);
void hostTierRelease(QuregState &s);
bool hostTierFlush(QuregState &s, const char *func);
bool hostTierProbs(QuregState &s, std::vector<double> &p0, double &total, const char *func);
// Writes zeros into the host memory of the all-zero pages (before the host
// copy of the state is read or written as a whole) and clears their flags.
void hostTierMaterialise(QuregState &s);
// Whether the amplitude at virtual index `index` lies in an all-zero page.
bool hostTierPageZero(const QuregState &s, uint64_t index);
bool hostTierSync(QuregState &s, const char *func);

// sharded registers (host_tier.cpp). attach: 2^shardBits shards on the
// given devices (nullptr: all on the current device), peer access enabled
// between the devices used; flush (hostTierFlush) runs the pending work
// shard by shard; probs as for the host tier; readVirtual/writeVirtual copy
// amplitudes [begin, begin + count) in virtual order (storage type) between
// the shards and host memory.
bool shardAttach(QuregState &s, int shardBits, const int *devices, int &code, std::string &err);
void shardRelease(QuregState &s);
bool shardSync(QuregState &s, const char *func);
bool shardReadVirtual(QuregState &s, uint64_t begin, uint64_t count, void *host, const char *func);
bool shardWriteVirtual(QuregState &s, uint64_t begin, uint64_t count, const void *host, const char *func);
bool shardCopy(QuregState &t, const QuregState &c, const char *func);
// How the host tier (batch = false) or a sharded register (batch = true)
// with 2^localBits amplitudes per page cuts `gates`: segments, exchange
// passes and qubits moved (host only).
void planExchanges(const std::vector<Gate> &gates, int localBits, int numBits, bool batch, int &segments,
                   int &exchanges, int &qubitsMoved);

}  // namespace dgq
