// tc_block.cu -- dense K-target unitary (K = 5 or 6) on a complex64 state
// with the 5th generation tensor cores, as a pipelined persistent sweep.
//
// The complex product Y = U X runs as one real GEMM per tile:
//   D[m][n] = sum_k X[m][k] W[k][n]
// with m a column of the tile (a pattern of 7 non-target address bits), k =
// 2 s + ri the input real index (target pattern s, real / imaginary part)
// and n = 2 s' + ri' the output real index: W[2s+0][2s'+0] = Ur[s'][s],
// W[2s+1][2s'+0] = -Ui[s'][s], W[2s+0][2s'+1] = Ui[s'][s], W[2s+1][2s'+1] =
// Ur[s'][s]. So the tile is 128 columns x 2^K amplitudes (M = 128, K_mma =
// KR = 2^(K+1), N = KR outputs).
//
// Precision: split FP16 ("FP16x3"). Every operand value is split into an
// FP16 head and an FP16 tail (x = hi + lo to about 22 bits) and
//   D = Xhi Whi + Xhi Wlo + Xlo Whi
// accumulates in FP32 in tensor memory. W is scaled by 2^8 on the host, and
// each column of X by a power of two chosen from its largest magnitude (so
// FP16's range never truncates it); the epilogue divides both out exactly.
// The first two products run as ONE MMA of width 2 KR on the concatenated
// operand [Whi | Wlo] (the A operand is read once for both), the third as an
// MMA of width KR on Whi; the epilogue adds the two halves of D.
//
// Pipeline (one CTA per SM, persistent over tiles, 25 warps):
//   warps 0-15  producer: four threads per column m of tile i (lanes c,
//               c + 8, c + 16, c + 24 of a warp, a quarter of the column's
//               2^K amplitudes each; eight consecutive columns per quarter
//               warp, contiguous when the lowest non-target bits are the
//               lowest address bits) load the tile (before waiting for the
//               buffer), agree on the column's scale through shuffles,
//               split, and store into X
//               buffer i % 2 (16-byte stores, K-major operand layout);
//   warp 24     issuer: one thread issues the MMAs of tile i into tensor
//               memory buffer i % 2 and commits them to two mbarriers (the X
//               buffer is free again; the accumulator is ready);
//   warps 16-23 consumer: row m of the accumulator (TMEM lane m; warps
//               16 + j and 20 + j reach lanes 32 j .. 32 j + 31) is read by
//               two threads, each half of the outputs; they release it and
//               write column m's 2^K outputs back to global memory.
// So the loads of tile i + 1, the MMAs of tile i and the stores of tile
// i - 1 overlap. All waits poll an mbarrier a bounded number of times; on a
// timeout the CTA raises the error word, every role stops at its next wait,
// and the issuer drains its MMAs (one more bounded wait) before tensor
// memory is released.
//
// Operand layout (no swizzle, K-major): 8-row x 16-byte core matrices; row r
// of a core matrix at 16 r bytes; core matrix (row group g, K chunk c of 8
// FP16 values) at (c * groups + g) * 128 bytes: SBO = 128 B (next row
// group), LBO = groups * 128 B (next K chunk); one MMA (K = 16) covers two K
// chunks. Descriptor and instruction-descriptor fields follow CUTLASS's
// UMMA definitions (cute/arch/mma_sm100_desc.hpp).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "kernels.h"

namespace dgq {

namespace {

constexpr int kTbCols = 128;         // M: tile columns
constexpr int kTbColBits = 7;
constexpr int kTbQuarters = 4;       // producer threads per column
constexpr int kTbProducerWarps = 16;
constexpr int kTbProducers = 32 * kTbProducerWarps;  // warps 0-15: four threads per column
constexpr int kTbConsumerWarps = 8;                  // warps 16-23: two per TMEM lane quarter
constexpr int kTbIssuerWarp = kTbProducerWarps + kTbConsumerWarps;
constexpr int kTbThreads = 32 * (kTbIssuerWarp + 1);
constexpr float kTbWScale = 256.0f;  // W carries 2^8

template <int K>
struct TbShape {
    static constexpr int D = 1 << K;        // target patterns
    static constexpr int KR = 2 * D;        // real inputs = real outputs
    static constexpr int XBytes = kTbCols * KR * 2;      // one FP16 part of a tile
    static constexpr int WBytes = KR * 2 * KR * 2;       // [Whi | Wlo]: 2 KR rows of KR FP16
    static constexpr int TmemCols = 2 * KR;              // one accumulator (both halves)
    static constexpr int TmemAlloc = 2 * TmemCols;       // double-buffered
    static constexpr int Smem = WBytes + 4 * XBytes + 4 * kTbCols * 4 + 8 * 16 + 1024;
};

struct TbArgs {
    int32_t numBits;
    int32_t hasRestrict;
    uint64_t restrictMask, restrictValue;
    float restrictScale;
    uint8_t tgtPos[6];    // address bit of target-pattern bit i
    uint8_t colPos[kTbColBits];
    uint8_t nCta;
    uint8_t ctaPos[kMaxStateBits];
    const double *normIn;  // complex64 renormalisation (null: off)
    double *normOut;
};

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t tbDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t) ((addr >> 4) & 0x3FFFu);
    d |= (uint64_t) ((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t) ((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t) 1 << 46;  // descriptor version (sm100); base offset 0, no swizzle
    return d;
}

// f16 x f16 -> f32, A and B K-major, M = 128
__host__ __device__ constexpr uint32_t tbIdesc(int N) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (kTbCols >> 4) << 24);
}

__device__ __forceinline__ void tbMma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void tbCommit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tbArrive(uint32_t mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool tbTryWait(uint32_t mbar, uint32_t parity) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for phase `parity` of the mbarrier; gives up after `limit` polls or
// when another role has raised *abort (returns false).
__device__ __forceinline__ bool tbWait(uint32_t mbar, uint32_t parity, volatile uint32_t *abort, uint32_t limit) {
    for (uint32_t n = 0; n < limit; n++) {
        if (tbTryWait(mbar, parity)) return true;
        if (*abort) return false;
        if (n > 64) __nanosleep(128);
    }
    return false;
}

constexpr uint32_t kTbPollLimit = 1u << 22;

// byte offset of operand element (row, k) in a K-major no-swizzle FP16
// operand with `groups` 8-row groups
__host__ __device__ __forceinline__ uint32_t tbOffset(uint32_t row, uint32_t k, uint32_t groups) {
    return (((k >> 3) * groups + (row >> 3)) << 7) + ((row & 7u) << 4) + ((k & 7u) << 1);
}

__device__ __forceinline__ uint32_t h2bits(__half2 h) { return *reinterpret_cast<uint32_t *>(&h); }

// Address offset of target pattern s, from the offsets of its bits.
template <int NB>
__device__ __forceinline__ uint64_t tbPattern(uint32_t s, const uint64_t (&bit)[NB]) {
    uint64_t o = 0;
#pragma unroll
    for (int i = 0; i < NB; i++) o |= (s >> i) & 1u ? bit[i] : 0ULL;
    return o;
}

// VA: amplitudes moved per global access (1, 2 or 4): 2^L when the L lowest
// address bits are the lowest targets (adjacent patterns are adjacent
// amplitudes, so 16- or 32-byte accesses fill whole sectors).
template <int VA>
__device__ __forceinline__ void tbLoadRun(const float2 *p, float2 *dst) {
    if (VA == 1) {
        dst[0] = __ldg(p);
    } else {
        const float4 f = __ldg(reinterpret_cast<const float4 *>(p));
        dst[0] = make_float2(f.x, f.y);
        dst[1] = make_float2(f.z, f.w);
        if (VA == 4) {
            const float4 g = __ldg(reinterpret_cast<const float4 *>(p) + 1);
            dst[2] = make_float2(g.x, g.y);
            dst[3] = make_float2(g.z, g.w);
        }
    }
}
template <int VA>
__device__ __forceinline__ void tbStoreRun(float2 *p, const float2 *src) {
    if (VA == 1) {
        p[0] = src[0];
    } else {
        reinterpret_cast<float4 *>(p)[0] = make_float4(src[0].x, src[0].y, src[1].x, src[1].y);
        if (VA == 4) reinterpret_cast<float4 *>(p)[1] = make_float4(src[2].x, src[2].y, src[3].x, src[3].y);
    }
}

template <int K, int VA>
__global__ void __launch_bounds__(kTbThreads, 1)
    tcBlockKernel(float2 *__restrict__ st, const __grid_constant__ TbArgs a, const uint4 *__restrict__ Wpacked,
                  uint32_t *__restrict__ error) {
    typedef TbShape<K> S;
    // when the lowest targets are address bits 0 and 1, each column is one
    // run in memory: the consumers stage the tile in its X buffer and write
    // whole columns per warp instruction (X is then released by them)
    constexpr bool STAGE = VA == 4;
    constexpr int P = S::D / kTbQuarters;  // amplitudes a producer thread holds per tile
    constexpr int PB = K - 2;              // their pattern bits (the low bits of s)
    extern __shared__ __align__(1024) unsigned char smRaw[];
    unsigned char *base = smRaw + ((1024u - (smemAddr(smRaw) & 1023u)) & 1023u);
    unsigned char *W = base;
    unsigned char *X = base + S::WBytes;  // [buffer][hi, lo]
    float *colInv = reinterpret_cast<float *>(X + 4 * S::XBytes);  // [tile & 3][column]
    uint64_t *bars = reinterpret_cast<uint64_t *>(colInv + 4 * kTbCols);  // xFull[2] xEmpty[2] dFull[2] dEmpty[2] drain
    __shared__ uint32_t tmemBase;
    __shared__ volatile uint32_t abortFlag;
    __shared__ double red[kTbConsumerWarps];

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t numTiles = 1u << (a.numBits - K - kTbColBits);
    const uint32_t barXFull = smemAddr(bars), barXEmpty = barXFull + 16, barDFull = barXFull + 32,
                   barDEmpty = barXFull + 48, barDrain = barXFull + 64;

    // resident W, already in the operand layout
    for (uint32_t i = tid; i < (uint32_t) S::WBytes / 16u; i += kTbThreads)
        reinterpret_cast<uint4 *>(W)[i] = __ldg(Wpacked + i);
    if (tid == 0) {
        abortFlag = 0;
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barXFull + 8 * b), "r"(kTbProducers)
                         : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barXEmpty + 8 * b),
                         "r"(STAGE ? 32u * kTbConsumerWarps : 1u)
                         : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barDFull + 8 * b) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barDEmpty + 8 * b), "r"(32 * kTbConsumerWarps)
                         : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barDrain) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kTbIssuerWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(&tmemBase)),
                     "r"((uint32_t) S::TmemAlloc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmemBase;

    auto tileBase = [&](uint32_t tile) {
        uint64_t b = 0;
        for (int i = 0; i < a.nCta; i++) b |= (uint64_t) ((tile >> i) & 1u) << a.ctaPos[i];
        return b;
    };
    const uint32_t myTiles = blockIdx.x < numTiles ? (numTiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp < kTbProducerWarps) {
        // ------------------------------------------------------- producer
        // lane = quarter * 8 + c: column m = 8 warp + c, patterns quarter * P + j
        const uint32_t c8 = lane & 7u, qd = lane >> 3, m = warp * 8u + c8;
        uint64_t colAddr = 0;
        for (int j = 0; j < kTbColBits; j++) colAddr |= (uint64_t) ((m >> j) & 1u) << a.colPos[j];
        uint64_t lowBit[PB];
        for (int i = 0; i < PB; i++) lowBit[i] = 1ULL << a.tgtPos[i];
        const uint64_t qOff = (uint64_t) (qd & 1u) << a.tgtPos[PB] | (uint64_t) (qd >> 1) << a.tgtPos[PB + 1];
        const float inScale = a.normIn ? (float) rsqrt(*a.normIn) : 1.0f;
        float2 v[P];
        for (uint32_t i = 0; i < myTiles; i++) {
            const uint32_t b = i & 1u, u = i >> 1;
            // the tile's loads go out before the wait for the buffer: their
            // latency overlaps the MMAs still reading it
            {
                const uint64_t tb = tileBase(blockIdx.x + i * gridDim.x) | colAddr | qOff;
#pragma unroll
                for (int j = 0; j < P; j += VA) tbLoadRun<VA>(st + (tb | tbPattern<PB>((uint32_t) j, lowBit)), v + j);
            }
            if (u > 0 && !tbWait(barXEmpty + 8 * b, (u - 1) & 1u, &abortFlag, kTbPollLimit)) {
                if (!abortFlag) atomicOr(error, 2u);
                abortFlag = 1;
                break;
            }
            if (a.hasRestrict) {
                const uint64_t tb = tileBase(blockIdx.x + i * gridDim.x) | colAddr | qOff;
#pragma unroll
                for (int j = 0; j < P; j++) {
                    const bool keep = ((tb | tbPattern<PB>((uint32_t) j, lowBit)) & a.restrictMask) == a.restrictValue;
                    const float k = keep ? a.restrictScale : 0.0f;
                    v[j] = make_float2(v[j].x * k, v[j].y * k);
                }
            }
            float mx = 0.0f;
#pragma unroll
            for (int j = 0; j < P; j++) mx = fmaxf(mx, fmaxf(fabsf(v[j].x), fabsf(v[j].y)));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
            // power of two taking the column's largest magnitude to [2^13, 2^14)
            int e = 0;
            if (mx > 0.0f) e = (int) ((__float_as_uint(mx) >> 23) & 0xFFu) - 127;
            const int sh = min(max(13 - e, -100), 100);
            const float scale = ldexpf(1.0f, sh);
            if (qd == 0) colInv[(i & 3u) * kTbCols + m] = ldexpf(1.0f, -sh) * inScale * (1.0f / kTbWScale);
            unsigned char *xh = X + b * 2 * S::XBytes;
            unsigned char *xl = xh + S::XBytes;
#pragma unroll
            for (int c = 0; c < P / 4; c++) {
                uint32_t hi[4], lo[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float xr = v[4 * c + q].x * scale, xi = v[4 * c + q].y * scale;
                    const __half2 hh = __floats2half2_rn(xr, xi);
                    const float2 hf = __half22float2(hh);
                    hi[q] = h2bits(hh);
                    lo[q] = h2bits(__floats2half2_rn(xr - hf.x, xi - hf.y));
                }
                // patterns qd P + 4 c .. + 3: K elements 2 (qd P + 4 c) .. + 7
                const uint32_t off = tbOffset(m, 2u * (qd * (uint32_t) P + 4u * (uint32_t) c), kTbCols / 8);
                *reinterpret_cast<uint4 *>(xh + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<uint4 *>(xl + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tbArrive(barXFull + 8 * b);
        }
    } else if (warp < kTbIssuerWarp) {
        // ------------------------------------------------------- consumer
        // warp % 4 == j reaches TMEM lanes 32 j ..; the two warps of a lane
        // quarter take the first and the second half of the outputs
        const uint32_t j = (warp - kTbProducerWarps) & 3u, half = (warp - kTbProducerWarps) >> 2;
        const uint32_t m = 32u * j + lane;
        uint64_t colAddr = 0;
        for (int q = 0; q < kTbColBits; q++) colAddr |= (uint64_t) ((m >> q) & 1u) << a.colPos[q];
        uint64_t tBit[K];
        for (int q = 0; q < K; q++) tBit[q] = 1ULL << a.tgtPos[q];
        double norm = 0.0;
        for (uint32_t i = 0; i < myTiles; i++) {
            const uint32_t d = i & 1u, v2 = i >> 1;
            if (!tbWait(barDFull + 8 * d, v2 & 1u, &abortFlag, kTbPollLimit)) {
                if (!abortFlag) atomicOr(error, 4u);
                abortFlag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const float inv = colInv[(i & 3u) * kTbCols + m];
            const uint64_t tb = tileBase(blockIdx.x + i * gridDim.x) | colAddr;
            const uint32_t tbase = tmem + ((32u * j) << 16) + d * (uint32_t) S::TmemCols;
            // 16 output reals (8 amplitudes) per chunk, written back as they come
#pragma unroll
            for (int cc = 0; cc < S::KR / 32; cc++) {
                const int c = (int) half * (S::KR / 32) + cc;
                uint32_t r0[16], r1[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(r0[0]), "=r"(r0[1]), "=r"(r0[2]), "=r"(r0[3]), "=r"(r0[4]), "=r"(r0[5]), "=r"(r0[6]),
                      "=r"(r0[7]), "=r"(r0[8]), "=r"(r0[9]), "=r"(r0[10]), "=r"(r0[11]), "=r"(r0[12]), "=r"(r0[13]),
                      "=r"(r0[14]), "=r"(r0[15])
                    : "r"(tbase + 16u * (uint32_t) c)
                    : "memory");
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(r1[0]), "=r"(r1[1]), "=r"(r1[2]), "=r"(r1[3]), "=r"(r1[4]), "=r"(r1[5]), "=r"(r1[6]),
                      "=r"(r1[7]), "=r"(r1[8]), "=r"(r1[9]), "=r"(r1[10]), "=r"(r1[11]), "=r"(r1[12]), "=r"(r1[13]),
                      "=r"(r1[14]), "=r"(r1[15])
                    : "r"(tbase + (uint32_t) S::KR + 16u * (uint32_t) c)
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float2 y[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    y[q] = make_float2((__uint_as_float(r0[2 * q]) + __uint_as_float(r1[2 * q])) * inv,
                                       (__uint_as_float(r0[2 * q + 1]) + __uint_as_float(r1[2 * q + 1])) * inv);
                    if (a.normOut) norm += (double) (y[q].x * y[q].x + y[q].y * y[q].y);
                }
                if constexpr (STAGE) {
                    // into the tile's X buffer (its MMAs are complete), column m
                    // at m D amplitudes, 16-byte chunks rotated by m against
                    // bank conflicts
                    float4 *col = reinterpret_cast<float4 *>(X + (i & 1u) * 2 * S::XBytes) + m * (S::D / 2);
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        col[((uint32_t) (4 * c + q)) ^ (m & (S::D / 2 - 1u))] =
                            make_float4(y[2 * q].x, y[2 * q].y, y[2 * q + 1].x, y[2 * q + 1].y);
                } else {
#pragma unroll
                    for (int q = 0; q < 8; q += VA)
                        tbStoreRun<VA>(st + (tb | tbPattern<K>((uint32_t) (8 * c + q), tBit)), y + q);
                }
            }
            // every value of the accumulator is read: hand the buffer back
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            tbArrive(barDEmpty + 8 * d);
            if constexpr (STAGE) {
                // each warp writes 16 whole columns back, a column's adjacent
                // amplitude pairs on adjacent lanes (one contiguous run per
                // column when the targets are the lowest address bits)
                asm volatile("bar.sync 2, %0;" ::"r"(32 * kTbConsumerWarps) : "memory");
                const float4 *stage = reinterpret_cast<const float4 *>(X + (i & 1u) * 2 * S::XBytes);
                constexpr uint32_t CPI = 64u / S::D;  // columns per warp instruction (32 lanes x 2 amplitudes)
                const uint32_t wq = warp - kTbProducerWarps;
                const uint64_t tbase0 = tileBase(blockIdx.x + i * gridDim.x);
#pragma unroll 1
                for (uint32_t k = 0; k < kTbCols / kTbConsumerWarps; k += CPI) {
                    const uint32_t mc = wq * (kTbCols / kTbConsumerWarps) + k + lane / (S::D / 2);
                    const uint32_t ch = lane % (S::D / 2);
                    uint64_t ca = 0;
                    for (int q = 0; q < kTbColBits; q++) ca |= (uint64_t) ((mc >> q) & 1u) << a.colPos[q];
                    const float4 v = stage[mc * (S::D / 2) + (ch ^ (mc & (S::D / 2 - 1u)))];
                    *reinterpret_cast<float4 *>(st + (tbase0 | ca | tbPattern<K>(2u * ch, tBit))) = v;
                }
                tbArrive(barXEmpty + 8 * (i & 1u));
            }
        }
        if (a.normOut) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) norm += __shfl_xor_sync(0xffffffffu, norm, o);
            if (lane == 0) red[warp - kTbProducerWarps] = norm;
        }
    } else if (lane == 0) {
        // ------------------------------------------------------- issuer
        const uint32_t lboX = (kTbCols / 8) * 128, lboW = (2 * S::KR / 8) * 128;
        const uint32_t wAddr = smemAddr(W), xAddr = smemAddr(X);
        for (uint32_t i = 0; i < myTiles; i++) {
            const uint32_t b = i & 1u, u = i >> 1, d = i & 1u, v2 = i >> 1;
            if (!tbWait(barXFull + 8 * b, u & 1u, &abortFlag, kTbPollLimit) ||
                (v2 > 0 && !tbWait(barDEmpty + 8 * d, (v2 - 1) & 1u, &abortFlag, kTbPollLimit))) {
                if (!abortFlag) atomicOr(error, 8u);
                abortFlag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + d * (uint32_t) S::TmemCols;
            const uint32_t xh = xAddr + b * 2 * (uint32_t) S::XBytes, xl = xh + (uint32_t) S::XBytes;
            // Xhi [Whi | Wlo] over N = 2 KR, then Xlo Whi over N = KR
#pragma unroll 1
            for (int ks = 0; ks < S::KR / 16; ks++)
                tbMma(acc, tbDesc(xh + (uint32_t) ks * 2 * lboX, lboX, 128), tbDesc(wAddr + (uint32_t) ks * 2 * lboW, lboW, 128),
                      tbIdesc(2 * S::KR), ks > 0 ? 1u : 0u);
#pragma unroll 1
            for (int ks = 0; ks < S::KR / 16; ks++)
                tbMma(acc, tbDesc(xl + (uint32_t) ks * 2 * lboX, lboX, 128), tbDesc(wAddr + (uint32_t) ks * 2 * lboW, lboW, 128),
                      tbIdesc(S::KR), 1u);
            if (!STAGE) tbCommit(barXEmpty + 8 * b);  // staged: the consumers release X
            tbCommit(barDFull + 8 * d);
        }
        // every MMA issued here has completed before tensor memory is released
        // (a bounded wait that an abort does not cut short)
        tbCommit(barDrain);
        bool drained = false;
        for (uint32_t n = 0; n < 2 * kTbPollLimit && !drained; n++) {
            drained = tbTryWait(barDrain, 0);
            if (!drained && n > 64) __nanosleep(128);
        }
        if (!drained) atomicOr(error, 16u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (a.normOut && tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kTbConsumerWarps; w++) t += red[w];
        atomicAdd(a.normOut, t);
    }
    if (warp == kTbIssuerWarp) {
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t) S::TmemAlloc)
                     : "memory");
    }
}

}  // namespace

size_t tcBlockMatrixFloats(int K) { return K == 5 ? TbShape<5>::WBytes / 4 : TbShape<6>::WBytes / 4; }

// The kernel takes the targets in ascending address order (pattern bit i =
// the i-th lowest target), so that the lowest targets, when they are the
// lowest address bits, make adjacent patterns adjacent amplitudes. perm[s]:
// the matrix index (bit j = target j as given) of the ascending-order
// pattern s.
static void ascendingPatterns(int K, const uint8_t *targets, int *perm) {
    int order[8];
    for (int i = 0; i < K; i++) order[i] = i;
    std::sort(order, order + K, [&](int x, int y) { return targets[x] < targets[y]; });
    for (int s = 0; s < (1 << K); s++) {
        int m = 0;
        for (int i = 0; i < K; i++)
            if ((s >> i) & 1) m |= 1 << order[i];
        perm[s] = m;
    }
}

// [Whi | Wlo] in the K-major FP16 operand layout: row n < KR is output real
// index n of Whi, row KR + n the same of Wlo; both scaled by 2^8; patterns in
// ascending target order.
void packTcBlockMatrix(int K, const double *Uin, const uint8_t *targets, float *out) {
    const int D = 1 << K, KR = 2 * D;
    int perm[64];
    ascendingPatterns(K, targets, perm);
    std::vector<double> U((size_t) 2 * D * D);
    for (int r = 0; r < D; r++)
        for (int c = 0; c < D; c++) {
            U[(size_t) 2 * (r * D + c)] = Uin[2 * (perm[r] * D + perm[c])];
            U[(size_t) 2 * (r * D + c) + 1] = Uin[2 * (perm[r] * D + perm[c]) + 1];
        }
    const uint32_t groups = (uint32_t) (2 * KR / 8);
    unsigned char *bytes = reinterpret_cast<unsigned char *>(out);
    std::memset(bytes, 0, (size_t) KR * 2 * KR * 2);
    for (int n = 0; n < KR; n++)
        for (int k = 0; k < KR; k++) {
            const int so = n >> 1, ro = n & 1, si = k >> 1, ri = k & 1;
            const double ur = U[2 * (so * D + si)], ui = U[2 * (so * D + si) + 1];
            double w;
            if (ro == 0)
                w = ri == 0 ? ur : -ui;
            else
                w = ri == 0 ? ui : ur;
            w *= (double) kTbWScale;
            const __half hi = __double2half((double) w);
            const __half lo = __double2half(w - (double) __half2float(hi));
            std::memcpy(bytes + tbOffset((uint32_t) n, (uint32_t) k, groups), &hi, 2);
            std::memcpy(bytes + tbOffset((uint32_t) (KR + n), (uint32_t) k, groups), &lo, 2);
        }
}

template <int K, int VA>
static cudaError_t launchTcBlockKV(float2 *st, const TbArgs &a, const uint4 *w, uint32_t *error, unsigned grid,
                                   cudaStream_t s) {
    static std::atomic<uint64_t> optIn{0};
    cudaError_t e = ensureSmemOptIn((const void *) tcBlockKernel<K, VA>, TbShape<K>::Smem, optIn);
    if (e != cudaSuccess) return e;
    tcBlockKernel<K, VA><<<grid, kTbThreads, TbShape<K>::Smem, s>>>(st, a, w, error);
    return cudaGetLastError();
}

bool tcBlockSupported(int numBits, int K) { return (K == 5 || K == 6) && numBits >= K + kTbColBits; }

cudaError_t launchTcBlock(float2 *st, int K, const DenseArgs &da, const float *Wpacked, uint32_t *error,
                          cudaStream_t s) {
    if (!tcBlockSupported(da.numBits, K) || !error) return cudaErrorInvalidValue;
    TbArgs a;
    std::memset(&a, 0, sizeof(a));
    a.numBits = da.numBits;
    a.hasRestrict = da.hasRestrict;
    a.restrictMask = da.restrictMask;
    a.restrictValue = da.restrictValue;
    a.restrictScale = (float) da.restrictScale;
    a.normIn = da.normIn;
    a.normOut = da.normOut;
    // targets in ascending address order (the operand was packed in that
    // order); columns: the 7 lowest other bits; the rest index tiles
    uint64_t tmask = 0;
    for (int b = 0; b < da.tileBits; b++)
        if (da.rowBit[b] >= 0) tmask |= 1ULL << da.tilePos[b];
    int nt0 = 0;
    for (int b = 0; b < da.numBits; b++)
        if ((tmask >> b) & 1ULL) a.tgtPos[nt0++] = (uint8_t) b;
    int low = 0;  // targets that are the lowest address bits 0, 1, ...
    while (low < nt0 && a.tgtPos[low] == low) low++;
    int nc = 0, nt = 0;
    for (int b = 0; b < da.numBits; b++) {
        if ((tmask >> b) & 1ULL) continue;
        if (nc < kTbColBits)
            a.colPos[nc++] = (uint8_t) b;
        else
            a.ctaPos[nt++] = (uint8_t) b;
    }
    a.nCta = (uint8_t) nt;
    if (nc != kTbColBits || __builtin_popcountll(tmask) != K) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t tiles = 1u << (a.numBits - K - kTbColBits);
    const unsigned grid = (unsigned) (tiles < (uint32_t) sms ? tiles : (uint32_t) sms);
    const int va = low >= 2 ? 4 : (low == 1 ? 2 : 1);
    const uint4 *w = reinterpret_cast<const uint4 *>(Wpacked);
    if (K == 5) {
        if (va == 4) return launchTcBlockKV<5, 4>(st, a, w, error, grid, s);
        if (va == 2) return launchTcBlockKV<5, 2>(st, a, w, error, grid, s);
        return launchTcBlockKV<5, 1>(st, a, w, error, grid, s);
    }
    if (va == 4) return launchTcBlockKV<6, 4>(st, a, w, error, grid, s);
    if (va == 2) return launchTcBlockKV<6, 2>(st, a, w, error, grid, s);
    return launchTcBlockKV<6, 1>(st, a, w, error, grid, s);
}

}  // namespace dgq
