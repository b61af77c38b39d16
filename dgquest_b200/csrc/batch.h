// batch.h -- many independent registers swept by one persistent launch.
//
// Every register of a batch has its own list of sweep programs (the same
// programs the single-register path launches one by one). The batch keeps
// them in four flat device arrays (sweep headers, phases, ops,
// coefficients) and a work list of items:
//   (register c, sweep s, tile t)   one tile of one sweep, or
//   (register c, kBatchWhole, 0)    every sweep of a register whose state is
//                                   a single tile, run back to back by one CTA.
// CTAs take items in list order from a ticket counter. An item waits (on
// the host-zeroed done counter of sweep s-1 of its register) until every
// tile of the previous sweep has been written. The list puts every item
// after the items it waits on, and a CTA only waits after it has taken its
// ticket, so the CTAs holding earlier tickets are running and the wait
// always ends; each wait is still bounded and reports a timeout through
// the error word instead of spinning for ever.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tile_program.h"

namespace dgq {

constexpr uint32_t kBatchWhole = 0xFFFFu;
constexpr int kBatchMaxTileBits = 12;

// Sweep header: TileProgram without its arrays; the arrays live at the
// given offsets of the batch's phase / op / coefficient arrays.
struct BatchSweep {
    int32_t numPhases;
    int32_t numOps;
    int32_t numBits;
    int32_t numReal;
    int32_t initKind;
    int32_t hasRestrict;
    int32_t hasGlobal;
    int32_t tileBits;
    double globalRe, globalIm;
    uint64_t initIndex;
    double initAmp;
    uint64_t restrictMask, restrictValue;
    double restrictScale;
    uint32_t phaseOff, opOff, coefOff, pad;
    uint8_t highPos[kMaxTileBits - kCoalescedBits];
    uint8_t ctaPos[kMaxStateBits];
};

struct BatchCircuit {
    void *state;             // double2 or float2 amplitudes
    uint32_t numBits;        // address bits of the state
    uint32_t tileBits;       // W of this register's sweeps
    uint32_t numSweeps;
    uint32_t firstSweep;     // index into the sweep headers
    uint32_t zOff;           // numBits + 1 sums in the expectation array
    uint32_t doneOff;        // numSweeps done counters
    uint32_t tilesPerSweep;  // 2^(numBits - tileBits)
    uint32_t pad;
};

struct BatchArgs {
    const BatchCircuit *circ;
    const BatchSweep *sweeps;
    const KPhase *phases;
    const KOp *ops;
    const double2 *leanCoef;  // lean form: the first two coefficients of each op, by op index
    const double *coef;
    const uint64_t *items;  // c | s << 20 | t << 36
    uint32_t numItems;
    uint32_t spinLimit;     // polls of a done counter before giving up
    uint32_t *ticket;       // zeroed before the launch
    uint32_t *done;         // zeroed before the launch
    double *zsum;           // zeroed before the launch: per register, sum |a|^2 over
                            // amplitudes with address bit b set (b < numBits), then the total
    uint32_t *error;        // 0, or 1 when a wait timed out
};

inline uint64_t batchItem(uint32_t c, uint32_t s, uint32_t t) {
    return (uint64_t) c | ((uint64_t) s << 20) | ((uint64_t) t << 36);
}

// One launch of the persistent batch kernel: grid CTAs of 2^(maxTileBits-4)
// threads with 2^maxTileBits amplitudes of shared memory.
// Kernel forms: with the dense-op case (a program holds a dense op), the
// general form, and the lean form (every op kind is a rotation, CNOT, CZ or
// phase kind).
constexpr int kBatchFormDense = 0, kBatchFormGeneral = 1, kBatchFormLean = 2;
cudaError_t launchBatch(const BatchArgs &a, bool single, int maxTileBits, int grid, int form, cudaStream_t s);
// CTAs of that kernel resident per SM (0 on error). Also sets the kernel's
// shared-memory limit: call it before the first launch (and before a launch
// is recorded into a graph).
int batchCtasPerSm(bool single, int maxTileBits);

}  // namespace dgq
