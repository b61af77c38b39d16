// kernels.h -- host-side launch interface of kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tile_program.h"

#include <atomic>

namespace dgq {

// Dynamic shared memory above 48 KiB must be opted into per kernel and per
// device (cudaFuncSetAttribute applies to the current device). `done` holds
// one bit per device ordinal (< 64) for which the opt-in has been made;
// concurrent callers may both set the attribute, which is harmless.
inline cudaError_t ensureSmemOptIn(const void *func, int bytes, std::atomic<uint64_t> &done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev < 64 ? (1ULL << dev) : 0ULL;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    if (bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return cudaSuccess;
}

}  // namespace dgq

namespace dgq {

struct ProbArgs {
    int32_t nFree;     // address bits not fixed by the lazy collapse
    int32_t kappa;     // log2 of 4096-amplitude units per CTA (0..4)
    uint64_t rValue;   // fixed bits' values
    uint8_t freePos[kMaxStateBits];  // address bit of sub-index bit i
};

struct SwapArgs {
    int32_t numBits;
    int32_t numPairs;  // exchange bit a[i] with bit b[i]
    uint8_t a[32];
    uint8_t b[32];
};

struct GatherArgs {
    uint64_t begin, count;
    uint64_t stride;  // logical index of entry i: begin + i * stride (0 means 1)
    int32_t numReal;
    int32_t hasRestrict;
    uint64_t restrictMask, restrictValue;
    double restrictScale;
    uint8_t l2v[kMaxStateBits];
};

struct InnerArgs {
    int32_t numReal;
    int32_t identity;  // both maps are the identity
    int32_t braRestrict, ketRestrict;
    uint64_t braMask, braValue, ketMask, ketValue;
    double braScale, ketScale;
    uint8_t l2vBra[kMaxStateBits];
    uint8_t l2vKet[kMaxStateBits];
};

// Dense multi-target unitaries (csrc/dense.cu): 5..7 targets.
constexpr int kMinDenseTargets = 5;
constexpr int kMaxDenseTargets = 7;
struct DenseArgs {
    int32_t numBits = 0;
    int32_t tileBits = 0;       // min(12, numBits): targets + lowest other bits
    int32_t hasRestrict = 0;
    uint64_t restrictMask = 0, restrictValue = 0;
    double restrictScale = 1.0;
    uint8_t tilePos[12] = {0};  // address bit of tile bit b (ascending)
    int8_t rowBit[12] = {0};    // matrix-index bit of tile bit b, or -1
    int8_t colBit[12] = {0};    // column-index bit of tile bit b, or -1
    uint8_t ctaPos[kMaxStateBits] = {0};
    // complex64 renormalisation: scale the input by 1/sqrt(*normIn), add the
    // output's sum of |a|^2 to *normOut (null: off)
    const double *normIn = nullptr;
    double *normOut = nullptr;
};
// Fills the tile map for K targets (targets[i] = address bit of matrix bit i).
bool denseArgs(int numBits, int K, const uint8_t *targets, DenseArgs &a);
// U: 2^K x 2^K row-major, (re, im) interleaved FP64, in device memory.
cudaError_t launchDense(void *st, bool single, int K, const DenseArgs &a, const double *U, cudaStream_t s);

// Tensor-core form for complex64 and 6 targets (tc_dense.cu): the matrix is
// packed on the host (packTcDenseMatrix, tcDenseMatrixFloats floats).
void packTcDenseMatrix(const double *U, float *out);
size_t tcDenseMatrixFloats();
// Device word set to 1 when a tensor-core sweep gave up waiting for its MMAs.
uint32_t *tcDenseErrorWord();
cudaError_t launchTcDense(float2 *st, const DenseArgs &a, const float *Apacked, uint32_t *error, cudaStream_t s);

// Pipelined tensor-core form (tc_block.cu): complex64, K = 5 or 6 targets,
// split FP16 on tcgen05 kind::f16, for registers of at least K + 7 address
// bits (tcBlockSupported). Its operand is packed on the host
// (packTcBlockMatrix, tcBlockMatrixFloats(K) floats).
bool tcBlockSupported(int numBits, int K);
size_t tcBlockMatrixFloats(int K);
// targets: address bit of matrix bit i (the kernel's pattern order is
// ascending by address; the packing permutes U to it)
void packTcBlockMatrix(int K, const double *U, const uint8_t *targets, float *out);
cudaError_t launchTcBlock(float2 *st, int K, const DenseArgs &a, const float *Wpacked, uint32_t *error,
                          cudaStream_t s);

struct SampleArgs {
    uint64_t numAmps;
    uint64_t restrictMask, restrictValue;  // lazy collapse (mask 0: none)
    double restrictScale2;                 // its scale squared
};

// Samples: `count` addresses drawn from |amp|^2 by the uniforms in [0, 1);
// sums holds sampleScratchCount(numAmps) doubles of scratch.
cudaError_t launchSample(const void *st, bool single, const SampleArgs &a, double *sums, const double *uniforms,
                         int count, uint64_t *out, cudaStream_t s);
uint64_t sampleScratchCount(uint64_t numAmps);

cudaError_t launchInner(const void *bra, bool braSingle, const void *ket, bool ketSingle, const InnerArgs &args,
                        double2 *partial, double2 *out, cudaStream_t s);
int innerNumCtas();

// The interpreting sweep kernel (complex128 or unpaired complex64 programs, W 9..12).
cudaError_t launchTile(void *st, bool single, int tileBits, const TileProgram &prog, cudaStream_t s);
cudaError_t launchProb(const void *st, bool single, const ProbArgs &args, double *partial, double *out,
                       cudaStream_t s);
int probNumCtas(const ProbArgs &args);
// Exchanges address bits a[k] <-> b[k] (disjoint pairs) of the whole state, in place.
cudaError_t launchSwapBits(void *st, bool single, const SwapArgs &args, cudaStream_t s);
// Host tier: exchanges local bit `bit` with the page-index bit in which the
// pages a and b (2^pageBits amplitudes each) differ.
cudaError_t launchPageSwap(void *a, void *b, bool single, int pageBits, int bit, cudaStream_t s);
// Sharded registers: x[o | patX] <-> y[o | patY] for every offset o of a
// 2^pageBits-amplitude shard whose bits at pos[0..m) (ascending) are 0.
struct BlockSwapArgs {
    int pageBits;
    int m;
    int pos[4];
    uint64_t patX;
    uint64_t patY;
};
cudaError_t launchBlockSwap(void *x, void *y, bool single, const BlockSwapArgs &args, cudaStream_t s);
cudaError_t launchGather(const void *st, bool single, const GatherArgs &args, double2 *out, cudaStream_t s);
cudaError_t launchFp64Peak(double *out, int blocks, int iters, cudaStream_t s);
cudaError_t launchInterleave(const double *re, const double *im, uint64_t count, uint64_t total, void *out,
                             bool single, cudaStream_t s);

}  // namespace dgq
