// jit.h -- runtime specialisation of sweep programs (NVRTC, sm_100a).
//
// codegen turns the structure of a TileProgram (tile width, phase layouts,
// the op sequence with target bits and control masks, coefficient offsets)
// into the source of one straight-line kernel; JitCache compiles sources in
// parallel host threads, loads the cubins and keeps the functions keyed by
// source, so every later plan with the same structure (any angles, any
// tile placement) reuses them.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "tile_program.h"

namespace dgq {

std::string generateSweepSource(const TileProgram &prog, int tileBits);

struct JitStats {
    int compiled = 0;       // kernels compiled by the last call
    int reused = 0;         // kernels found in the cache by the last call
    double compileMillis = 0.0;
};

// Returns one CUfunction per source (nullptr entries on failure, with *err).
bool jitGetKernels(const std::vector<std::string> &sources, std::vector<CUfunction> &out, JitStats *stats,
                   std::string *err);

cudaError_t launchJitSweep(CUfunction fn, void *st, int tileBits, const TileProgram &prog, cudaStream_t s);

// The loaded kernel of `source`, or nullptr when it is not loaded yet
// (compiles nothing).
CUfunction jitFindLoaded(const std::string &source);

// Whether every source is compiled already (loaded, or compiled in the
// background and waiting to be loaded).
bool jitAllReady(const std::vector<std::string> &sources);
// Queues the sources that are neither loaded nor compiled for NVRTC
// compilation on background host threads (no GPU work); later
// jitGetKernels calls load the results instead of compiling.
void jitCompileInBackground(const std::vector<std::string> &sources);

// Stops the background compiles: drops the queue, waits for compiles in
// progress (30 s at most) and joins the worker threads.
void jitStopBackground();

// NVRTC compile only (no GPU needed).
bool jitCompileOnly(const std::string &src, std::vector<char> &cubin, std::string &log);

// Whether runtime specialisation is enabled (DGQ_JIT=0 disables it).
bool jitEnabled();

}  // namespace dgq
