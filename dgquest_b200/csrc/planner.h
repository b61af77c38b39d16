// planner.h -- cuts a recorded gate list into state sweeps ("fused blocks")
// and encodes each sweep as a TileProgram for the tile kernel.
//
// dgQuEST cuts its circuit twice with the same greedy DAG selection
// (src/cpp/QuEST_backend.cpp:118-141,152-182): into sections that fit a task
// and into 11-qubit fused gates seeded with the 5 coalesced low bits, then
// re-DAGs each fused gate with budget 1 to group gates by target
// (src/cpp/QuEST_gpu_kernel.cu:529-562). On one GPU with the state resident
// in HBM there are no sections: the planner takes blocks of W tile bits
// (seeded with the 5 low bits, padded from bit 5 upward like
// QuEST_gpu_kernel.cu:504-509), then phases of 4 register bits.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "ir.h"
#include "tile_program.h"

namespace dgq {

struct BlockPlan {
    u64 tileMask = 0;         // W address bits, bits 0..4 always included
    std::vector<Gate> gates;  // dependency order
};

struct PlanStats {
    int sweeps = 0;     // kernel launches (state read+write passes)
    int phases = 0;     // register layouts summed over sweeps
    int ops = 0;        // kernel ops summed over sweeps
    int gates = 0;      // gates after merging
    double flopsPerAmp = 0;  // algorithmic FP64 flops per amplitude, summed over ops
};

// Multi-qubit unitary matrices referenced by OP_MULTI_UNITARY gates.
struct MatrixPool {
    std::vector<std::vector<double>> mats;  // row-major 2^k x 2^k, (re, im) interleaved
};

// `complete` (if given) is set to false when gates are left that no tile
// can hold (a gate with more non-diagonal targets than the tile width).
// seedBits: the lowest address bits every tile holds (5: the coalesced bits
// of complex128 tiles; 6 for the complex64 paired form, whose tile-local
// bit 0 is the pair inside a slot and bits 1..5 the coalesced slot bits).
// lookahead: 1 scores each candidate addition of tile bits by the best
// follow-up addition as well (fewer sweeps on deep circuits, 3x the
// planning time), 0 does not, -1 uses it for registers of >= 24 address bits
// (DGQ_PLAN_LOOKAHEAD_BITS overrides the 24).
std::vector<BlockPlan> planBlocks(const std::vector<Gate> &gates, int numBits, int tileBits, bool *complete = nullptr,
                                  int seedBits = kCoalescedBits, int lookahead = -1);
// The same blocks, handed to `onBlock` one at a time as they are chosen
// (a caller can encode and launch a sweep while the next one is planned);
// stops early when onBlock returns false. Returns false when gates are left
// that no tile can hold.
bool planBlocksEach(const std::vector<Gate> &gates, int numBits, int tileBits, int seedBits,
                    const std::function<bool(BlockPlan &)> &onBlock, int lookahead = -1);
// Whether lookahead -1 means lookahead for a register of numBits bits.
bool lookaheadBySize(int numBits);

// Encodes one block. The gate list may not fit one TileProgram; then the
// block is emitted as several programs over the same tile (each one more
// sweep). Only the first program carries `first` (init / lazy collapse).
struct SweepHeader {
    int32_t initKind = INIT_NONE;
    uint64_t initIndex = 0;
    double initAmp = 0.0;
    bool hasRestrict = false;
    uint64_t restrictMask = 0, restrictValue = 0;
    double restrictScale = 1.0;
};

// paired: encode for the complex64 paired form (TileProgram::paired); fails
// (with *err set) on a multi-qubit unitary that targets address bit 0.
bool encodeBlock(const BlockPlan &block, int numBits, int numReal, int tileBits, const MatrixPool &pool,
                 const SweepHeader &first, std::vector<TileProgram> &out, PlanStats *stats, std::string *err,
                 bool paired = false);

// A program that only applies the header (init and/or lazy collapse).
void encodeHeaderOnly(int numBits, int numReal, int tileBits, const SweepHeader &hdr, TileProgram &out,
                      bool paired = false);

// Algorithmic FP64 flops per amplitude of one kernel op (formulas of
// QuEST_gpu_kernel.cu:17-170 counted as multiplies + adds per amplitude,
// averaged over the amplitudes it touches when uncontrolled).
double opFlopsPerAmp(const KOp &op);

}  // namespace dgq
