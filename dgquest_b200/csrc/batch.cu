// batch.cu -- the persistent kernel of the batched form (batch.h).
//
// One CTA works one item at a time. A tile item is the interpreting tile
// kernel of kernels.cu with the tile width taken at run time (a register of
// 2^10 amplitudes runs 2^10-amplitude tiles on the first 64 threads of the
// CTA, synchronised by a named barrier), the state read through L2 only
// (ld.global.cg: another SM wrote it in the previous sweep) and, on a
// register's last sweep, the sums that give <Z_q> for every qubit added to
// the register's expectation slots with one atomic per address bit per CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "batch.h"
#include "interp.cuh"
#include "tile_program.h"

namespace dgq {

namespace {

__device__ __forceinline__ uint32_t swzB(uint32_t x) { return x ^ (((x >> 3) ^ (x >> 6) ^ (x >> 9) ^ (x >> 12)) & 7u); }

__device__ __forceinline__ void groupBarrier(uint32_t threads) {
    asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

__device__ __forceinline__ uint32_t loadAcquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <class V>
__device__ __forceinline__ V loadCg(const V *p);
template <>
__device__ __forceinline__ double2 loadCg<double2>(const double2 *p) {
    return __ldcg(p);
}
template <>
__device__ __forceinline__ float2 loadCg<float2>(const float2 *p) {
    return __ldcg(p);
}

// Adds the tile's contribution to the register's expectation sums: for each
// address bit b, the sum of |a|^2 over amplitudes with bit b set, and the
// tile's total. Lanes cover address bits 0..4, warps the tile's next bits,
// registers its top 4 bits and the tile index the remaining bits.
// tot: the thread's sum of |a|^2; rs[k]: the part of it whose register bit k is 1.
__device__ __noinline__ void addExpectationSums(double tot, const double (&rs)[4], const BatchSweep &h, uint32_t tid,
                                                uint32_t threads, int W, uint32_t tile, double *zs) {
    __shared__ double red[16][10];
    double v[10];
    v[0] = tot;
#pragma unroll
    for (int i = 0; i < 5; i++) v[1 + i] = ((tid >> i) & 1u) ? tot : 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) v[6 + k] = rs[k];
#pragma unroll
    for (int k = 0; k < 10; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    const uint32_t warp = tid >> 5;
    if ((tid & 31u) == 0) {
#pragma unroll
        for (int k = 0; k < 10; k++) red[warp][k] = v[k];
    }
    groupBarrier(threads);
    if (tid == 0) {
        const uint32_t warps = threads >> 5;
        double ctaTot = 0.0, lane[5] = {0, 0, 0, 0, 0}, reg[4] = {0, 0, 0, 0};
        for (uint32_t w = 0; w < warps; w++) {
            ctaTot += red[w][0];
            for (int i = 0; i < 5; i++) lane[i] += red[w][1 + i];
            for (int k = 0; k < 4; k++) reg[k] += red[w][6 + k];
        }
        for (int i = 0; i < 5; i++)
            if (lane[i] != 0.0) atomicAdd(zs + i, lane[i]);
        for (int i = 0; i < W - 9; i++) {
            double s = 0.0;
            for (uint32_t w = 0; w < warps; w++)
                if ((w >> i) & 1u) s += red[w][0];
            if (s != 0.0) atomicAdd(zs + h.highPos[i], s);
        }
        for (int k = 0; k < 4; k++)
            if (reg[k] != 0.0) atomicAdd(zs + h.highPos[W - 9 + k], reg[k]);
        for (int i = 0; i < h.numBits - W; i++)
            if (((tile >> i) & 1u) && ctaTot != 0.0) atomicAdd(zs + h.ctaPos[i], ctaTot);
        atomicAdd(zs + h.numBits, ctaTot);
    }
}

// One tile of one sweep, run by the first 2^(W-4) threads of the CTA; h is
// the sweep header staged in shared memory.
template <class V, int W, bool DENSE, bool LEAN>
__device__ __forceinline__ void sweepTile(const BatchArgs &args, const BatchSweep &h, V *__restrict__ st, uint32_t tile,
                                          V *sm, double *zs) {
    constexpr uint32_t T = 1u << (W - kRegBits);
    const uint32_t tid = threadIdx.x;

    uint64_t tpart = tid & 31u;
    for (int i = 0; i < h.numBits - W; i++) tpart |= (uint64_t) ((tile >> i) & 1u) << h.ctaPos[i];
#pragma unroll
    for (int i = 0; i < W - 9; i++) tpart |= (uint64_t) ((tid >> (5 + i)) & 1u) << h.highPos[i];
    const uint64_t jb0 = 1ULL << h.highPos[W - 9];
    const uint64_t jb1 = 1ULL << h.highPos[W - 8];
    const uint64_t jb2 = 1ULL << h.highPos[W - 7];
    const uint64_t jb3 = 1ULL << h.highPos[W - 6];
    auto gidx = [&](int j) -> uint64_t {
        return tpart | ((j & 1) ? jb0 : 0ULL) | ((j & 2) ? jb1 : 0ULL) | ((j & 4) ? jb2 : 0ULL) | ((j & 8) ? jb3 : 0ULL);
    };

    V a[kRegs];
    if (h.initKind == INIT_NONE) {
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = loadCg(st + gidx(j));
    } else {
        const uint64_t ci = h.initIndex;
        const double pa = h.initAmp;
        const int kind = h.initKind;
        const int nr = h.numReal;
#pragma unroll
        for (int j = 0; j < kRegs; j++) {
            const uint64_t g = gidx(j);
            double re = 0.0;
            if (kind == INIT_CLASSICAL)
                re = (g == ci) ? 1.0 : 0.0;
            else if (kind == INIT_PLUS)
                re = ((g >> nr) == 0ULL) ? pa : 0.0;
            a[j] = mk<V>((typename Real<V>::T) re, 0);
        }
    }
    if (h.hasRestrict) {
        const uint64_t rm = h.restrictMask, rv = h.restrictValue;
        const typename Real<V>::T sc = (typename Real<V>::T) h.restrictScale;
#pragma unroll
        for (int j = 0; j < kRegs; j++) {
            const bool keep = (gidx(j) & rm) == rv;
            a[j] = keep ? mk<V>(a[j].x * sc, a[j].y * sc) : mk<V>(0, 0);
        }
    }

    const KPhase *phases = args.phases + h.phaseOff;
    const KOp *__restrict__ ops = args.ops + h.opOff;
    const double *__restrict__ coef = args.coef + h.coefOff;
    if (h.numPhases > 0) {
#pragma unroll
        for (int j = 0; j < kRegs; j++) sm[swzB(tid + T * (uint32_t) j)] = a[j];
        groupBarrier(T);
        for (int p = 0; p < h.numPhases; p++) {
            const KPhase &ph = phases[p];
            uint32_t loc = 0;
#pragma unroll
            for (int i = 0; i < W - kRegBits; i++) loc |= ((tid >> i) & 1u) << ph.thrPos[i];
            const uint32_t sb = swzB(loc);
#pragma unroll
            for (int j = 0; j < kRegs; j++) a[j] = sm[sb ^ ph.regOff[j]];
            const int e = ph.opEnd;
            for (int o = ph.opBegin; o < e; o++) {
                // the 16-byte op record in one read-only load
                const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(ops + o));
                KOp op;
                memcpy(&op, &raw, sizeof(op));
                if constexpr (LEAN) {
                    // the lean kinds' two coefficients, loaded beside the
                    // record instead of after it
                    const double2 cc = __ldg(args.leanCoef + h.opOff + o);
                    const double cv[2] = {cc.x, cc.y};
                    applyOpAt<V, DENSE, LEAN>(op, cv, a, loc, tile);
                } else {
                    applyOp<V, DENSE, LEAN>(op, coef, a, loc, tile);
                }
            }
#pragma unroll
            for (int j = 0; j < kRegs; j++) sm[sb ^ ph.regOff[j]] = a[j];
            groupBarrier(T);
        }
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = sm[swzB(tid + T * (uint32_t) j)];
    }
    if (h.hasGlobal) {
        const typename Real<V>::T gr = (typename Real<V>::T) h.globalRe, gi = (typename Real<V>::T) h.globalIm;
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = mk<V>(gr * a[j].x - gi * a[j].y, gr * a[j].y + gi * a[j].x);
    }
    // store addresses rebuilt here (nothing address-related stays live across the phases)
    uint64_t tp2 = tid & 31u;
    for (int i = 0; i < h.numBits - W; i++) tp2 |= (uint64_t) ((tile >> i) & 1u) << h.ctaPos[i];
#pragma unroll
    for (int i = 0; i < W - 9; i++) tp2 |= (uint64_t) ((tid >> (5 + i)) & 1u) << h.highPos[i];
    const uint64_t kb0 = 1ULL << h.highPos[W - 9];
    const uint64_t kb1 = 1ULL << h.highPos[W - 8];
    const uint64_t kb2 = 1ULL << h.highPos[W - 7];
    const uint64_t kb3 = 1ULL << h.highPos[W - 6];
    auto sidx = [&](int j) -> uint64_t {
        return tp2 | ((j & 1) ? kb0 : 0ULL) | ((j & 2) ? kb1 : 0ULL) | ((j & 4) ? kb2 : 0ULL) | ((j & 8) ? kb3 : 0ULL);
    };
    double tot = 0.0, rs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        __stcg(st + sidx(j), a[j]);
        if (zs) {
            const double p = (double) a[j].x * (double) a[j].x + (double) a[j].y * (double) a[j].y;
            tot += p;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if ((j >> k) & 1) rs[k] += p;
        }
    }
    if (zs) addExpectationSums(tot, rs, h, tid, T, W, tile, zs);
    // the next sweep of a whole-register item reads what other threads wrote
    // and overwrites the shared exchange buffer
    groupBarrier(T);
}

// Sweeps [w0, w1) of one register on tile `tile` (one sweep for a tile
// item, all of them for a whole-register item); each header is copied to
// shared memory first, so the phase loop holds no header registers.
template <class V, int W, bool DENSE, bool LEAN>
__device__ __forceinline__ void runSweeps(const BatchArgs &args, const BatchCircuit &C, uint32_t w0, uint32_t w1,
                                       uint32_t tile, V *sm, BatchSweep *hs) {
    constexpr uint32_t T = 1u << (W - kRegBits);
    V *st = reinterpret_cast<V *>(C.state);
    for (uint32_t w = w0; w < w1; w++) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(args.sweeps + C.firstSweep + w);
        uint32_t *dst = reinterpret_cast<uint32_t *>(hs);
        for (uint32_t i = threadIdx.x; i < sizeof(BatchSweep) / 4; i += T) dst[i] = __ldg(src + i);
        groupBarrier(T);
        sweepTile<V, W, DENSE, LEAN>(args, *hs, st, tile, sm, w + 1 == C.numSweeps ? args.zsum + C.zOff : nullptr);
    }
}

// DENSE: the batch's programs hold dense ops (multi-qubit unitaries of up to
// 4 targets inside a register phase); without them the kernel is compiled
// without that case (FP64: no spills instead of 1.3 KB of spill stores).
// LEAN: every op kind is one of kLeanKinds (rotations, CNOT, CZ, phases).
template <class V, bool DENSE, bool LEAN>
__global__ void __launch_bounds__(1 << (kBatchMaxTileBits - kRegBits), 2)
    batchKernel(const __grid_constant__ BatchArgs args) {
    extern __shared__ __align__(16) unsigned char smRaw[];
    V *sm = reinterpret_cast<V *>(smRaw);
    __shared__ uint64_t sItem;
    __shared__ uint32_t sAbort;
    __shared__ BatchSweep sHead;
    const uint32_t tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const uint32_t k = atomicAdd(args.ticket, 1u);
            sItem = k < args.numItems ? args.items[k] : ~0ULL;
            sAbort = 0;
        }
        __syncthreads();
        const uint64_t it = sItem;
        if (it == ~0ULL) break;
        const uint32_t c = (uint32_t) (it & 0xFFFFFu);
        const uint32_t s = (uint32_t) ((it >> 20) & 0xFFFFu);
        const uint32_t t = (uint32_t) (it >> 36);
        const BatchCircuit C = args.circ[c];
        if (tid == 0 && s != kBatchWhole && s > 0) {
            const uint32_t *d = args.done + C.doneOff + s - 1;
            uint32_t polls = 0;
            while (loadAcquire(d) < C.tilesPerSweep) {
                if (++polls > args.spinLimit) {
                    atomicOr(args.error, 1u);
                    sAbort = 1;
                    break;
                }
                __nanosleep(256);
            }
        }
        __syncthreads();
        if (sAbort) break;
        const uint32_t T = 1u << (C.tileBits - kRegBits);
        if (tid < T) {
            const uint32_t w0 = s == kBatchWhole ? 0u : s, w1 = s == kBatchWhole ? C.numSweeps : s + 1;
            const uint32_t tile = s == kBatchWhole ? 0u : t;
            switch (C.tileBits) {
                case 9: runSweeps<V, 9, DENSE, LEAN>(args, C, w0, w1, tile, sm, &sHead); break;
                case 10: runSweeps<V, 10, DENSE, LEAN>(args, C, w0, w1, tile, sm, &sHead); break;
                case 11: runSweeps<V, 11, DENSE, LEAN>(args, C, w0, w1, tile, sm, &sHead); break;
                default: runSweeps<V, 12, DENSE, LEAN>(args, C, w0, w1, tile, sm, &sHead); break;
            }
            __threadfence();
        }
        __syncthreads();
        if (tid == 0 && s != kBatchWhole) atomicAdd(args.done + C.doneOff + s, 1u);
    }
}

// The kernel's dynamic shared-memory limit is set once, to the widest tile,
// by ctasPerSmV (called before any launch is recorded), so that launches
// recorded in graphs stay valid whatever tile width later batches use.
template <class V>
cudaError_t launchBatchV(const BatchArgs &a, int maxTileBits, int grid, int form, cudaStream_t s) {
    const size_t smem = sizeof(V) << maxTileBits;
    const int T = 1 << (maxTileBits - kRegBits);
    if (form == kBatchFormDense)
        batchKernel<V, true, false><<<grid, T, smem, s>>>(a);
    else if (form == kBatchFormLean)
        batchKernel<V, false, true><<<grid, T, smem, s>>>(a);
    else
        batchKernel<V, false, false><<<grid, T, smem, s>>>(a);
    return cudaGetLastError();
}

// All forms have the same launch bounds and shared memory; the occupancy
// is the smallest of them.
template <class V, bool DENSE, bool LEAN>
int ctasPerSmForm(int maxTileBits) {
    const size_t smem = sizeof(V) << maxTileBits;
    if (cudaFuncSetAttribute(batchKernel<V, DENSE, LEAN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int) (sizeof(V) << kBatchMaxTileBits)) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batchKernel<V, DENSE, LEAN>, 1 << (maxTileBits - kRegBits),
                                                      smem) != cudaSuccess)
        return 0;
    return n;
}

template <class V>
int ctasPerSmV(int maxTileBits) {
    const int a = ctasPerSmForm<V, true, false>(maxTileBits), b = ctasPerSmForm<V, false, false>(maxTileBits),
              c = ctasPerSmForm<V, false, true>(maxTileBits);
    return std::min(a, std::min(b, c));
}

}  // namespace

cudaError_t launchBatch(const BatchArgs &a, bool single, int maxTileBits, int grid, int form, cudaStream_t s) {
    if (maxTileBits < kMinTileBits || maxTileBits > kBatchMaxTileBits || grid < 1) return cudaErrorInvalidValue;
    return single ? launchBatchV<float2>(a, maxTileBits, grid, form, s)
                  : launchBatchV<double2>(a, maxTileBits, grid, form, s);
}

int batchCtasPerSm(bool single, int maxTileBits) {
    if (maxTileBits < kMinTileBits || maxTileBits > kBatchMaxTileBits) return 0;
    return single ? ctasPerSmV<float2>(maxTileBits) : ctasPerSmV<double2>(maxTileBits);
}

}  // namespace dgq
