// kernels.cu -- the sm_100a kernels of the FP64 state-vector path.
//
//   tileKernel<W,V,LEAN> one sweep of the state applying a fused block
//                    (dgQuEST statevec_fusedKernel, QuEST_gpu_kernel.cu:175-359)
//   probKernel       P(bit = 0) for every address bit in one read pass
//   probFinalize     (statevec_findProbabilityOfZeroKernel + reducePingpong,
//                    QuEST_gpu_kernel.cu:656-840)
//   swapBitsKernel   in-HBM exchange of address-bit pairs (the successor of
//                    reorder_data_kernel, QuEST_gpu_kernel.cu:589-654)
//   gatherKernel     logical-order copy-out of the state through the
//                    logical->virtual map
//
// The state is 2^numBits double2 (re, im) amplitudes in HBM, in place.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "interp.cuh"
#include "kernels.h"
#include "tile_program.h"

namespace dgq {

__device__ __forceinline__ uint32_t swz(uint32_t x) { return x ^ (((x >> 3) ^ (x >> 6) ^ (x >> 9) ^ (x >> 12)) & 7u); }

// ------------------------------------------------------------ tile kernel
// 128 registers per thread: 16 warps per SM at every tile width. V is
// double2 (complex128) or float2 (complex64, with the per-sweep
// renormalisation of the complex64 form: scale by 1/sqrt(*normIn) with the
// global factor, add the output's sum of |a|^2 to *normOut).
template <int W, class V, bool LEAN>
__global__ void __launch_bounds__(1 << (W - kRegBits), 65536 / (128 << (W - kRegBits)))
    tileKernel(V *__restrict__ st, const __grid_constant__ TileProgram prog) {
    typedef typename Real<V>::T R;
    constexpr int T = 1 << (W - kRegBits);
    extern __shared__ __align__(16) unsigned char smRaw[];
    V *sm = reinterpret_cast<V *>(smRaw);
    const uint32_t tid = threadIdx.x;
    const uint32_t cta = blockIdx.x + prog.ctaOffset;

    // address of canonical element (tid, j): base | lane bits | thread high bits | j bits
    uint64_t tpart = tid & 31u;
    const int nCta = prog.numBits - W;
    for (int i = 0; i < nCta; i++) tpart |= (uint64_t) ((cta >> i) & 1u) << prog.ctaPos[i];
#pragma unroll
    for (int i = 0; i < W - 9; i++) tpart |= (uint64_t) ((tid >> (5 + i)) & 1u) << prog.highPos[i];
    const uint64_t jb0 = 1ULL << prog.highPos[W - 9];
    const uint64_t jb1 = 1ULL << prog.highPos[W - 8];
    const uint64_t jb2 = 1ULL << prog.highPos[W - 7];
    const uint64_t jb3 = 1ULL << prog.highPos[W - 6];
    auto gidx = [&](int j) -> uint64_t {
        return tpart | ((j & 1) ? jb0 : 0ULL) | ((j & 2) ? jb1 : 0ULL) | ((j & 4) ? jb2 : 0ULL) | ((j & 8) ? jb3 : 0ULL);
    };

    V a[kRegs];
    if (prog.initKind == INIT_NONE) {
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = st[gidx(j)];
    } else {
        const uint64_t ci = prog.initIndex;
        const double pa = prog.initAmp;
        const int kind = prog.initKind;
        const int nr = prog.numReal;
#pragma unroll
        for (int j = 0; j < kRegs; j++) {
            const uint64_t g = gidx(j);
            double re = 0.0;
            if (kind == INIT_CLASSICAL)
                re = (g == ci) ? 1.0 : 0.0;
            else if (kind == INIT_PLUS)
                re = ((g >> nr) == 0ULL) ? pa : 0.0;
            a[j] = mk<V>((R) re, (R) 0);
        }
    }
    if (prog.hasRestrict) {
        const uint64_t rm = prog.restrictMask, rv = prog.restrictValue;
        const R sc = (R) prog.restrictScale;
#pragma unroll
        for (int j = 0; j < kRegs; j++) {
            const bool keep = (gidx(j) & rm) == rv;
            a[j] = keep ? mk<V>(a[j].x * sc, a[j].y * sc) : mk<V>((R) 0, (R) 0);
        }
    }

    const int numPhases = prog.numPhases;
    if (numPhases > 0) {
#pragma unroll
        for (int j = 0; j < kRegs; j++) sm[swz(tid + (uint32_t) (T * j))] = a[j];
        __syncthreads();
        for (int p = 0; p < numPhases; p++) {
            const KPhase &ph = prog.phases[p];
            uint32_t loc = 0;
#pragma unroll
            for (int i = 0; i < W - kRegBits; i++) loc |= ((tid >> i) & 1u) << ph.thrPos[i];
            const uint32_t sb = swz(loc);
#pragma unroll
            for (int j = 0; j < kRegs; j++) a[j] = sm[sb ^ ph.regOff[j]];
            const int e = ph.opEnd;
            for (int o = ph.opBegin; o < e; o++) applyOp<V, !LEAN, LEAN>(prog.ops[o], prog.coef, a, loc, cta);
#pragma unroll
            for (int j = 0; j < kRegs; j++) sm[sb ^ ph.regOff[j]] = a[j];
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = sm[swz(tid + (uint32_t) (T * j))];
    }
    if (prog.hasGlobal || prog.renormIn) {
        double grd = prog.globalRe, gid = prog.globalIm;
        if (prog.renormIn) {
            const double sc = rsqrt(*prog.normIn);
            grd *= sc;
            gid *= sc;
        }
        const R gr = (R) grd, gi = (R) gid;
#pragma unroll
        for (int j = 0; j < kRegs; j++) a[j] = mk<V>(gr * a[j].x - gi * a[j].y, gr * a[j].y + gi * a[j].x);
    }
    if (prog.renormOut) {
        __shared__ double red[32];
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < kRegs; j++) acc += (double) a[j].x * (double) a[j].x + (double) a[j].y * (double) a[j].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((tid & 31u) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < T / 32; w++) t += red[w];
            atomicAdd(prog.normOut, t);
        }
    }
#pragma unroll
    for (int j = 0; j < kRegs; j++) st[gidx(j)] = a[j];
}

template <int W, class V, bool LEAN>
static cudaError_t launchTileWL(V *st, const TileProgram &prog, cudaStream_t s) {
    static std::atomic<uint64_t> optIn{0};
    const size_t smem = sizeof(V) << W;
    cudaError_t e = ensureSmemOptIn((const void *) tileKernel<W, V, LEAN>, (int) smem, optIn);
    if (e != cudaSuccess) return e;
    const unsigned grid = prog.ctaCount ? prog.ctaCount : 1u << (prog.numBits - W);
    tileKernel<W, V, LEAN><<<grid, 1 << (W - kRegBits), smem, s>>>(st, prog);
    return cudaGetLastError();
}

// The lean form when every op of the program is a lean kind (rotations,
// CNOT, CZ, phases): measured 10-11 % faster on a 28-qubit random circuit.
template <int W, class V>
static cudaError_t launchTileW(V *st, const TileProgram &prog, cudaStream_t s) {
    bool lean = true;
    for (int i = 0; i < prog.numOps && lean; i++) lean = (kLeanKinds >> prog.ops[i].kind) & 1u;
    return lean ? launchTileWL<W, V, true>(st, prog, s) : launchTileWL<W, V, false>(st, prog, s);
}

template <class V>
static cudaError_t launchTileV(V *st, int tileBits, const TileProgram &prog, cudaStream_t s) {
    switch (tileBits) {
        case 9: return launchTileW<9>(st, prog, s);
        case 10: return launchTileW<10>(st, prog, s);
        case 11: return launchTileW<11>(st, prog, s);
        case 12: return launchTileW<12>(st, prog, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchTile(void *st, bool single, int tileBits, const TileProgram &prog, cudaStream_t s) {
    if (prog.paired) return cudaErrorInvalidValue;  // the paired form is runtime-specialised only
    return single ? launchTileV((float2 *) st, tileBits, prog, s) : launchTileV((double2 *) st, tileBits, prog, s);
}

// ------------------------------------------------------- probabilities
// Sub-index s enumerates the amplitudes allowed by the lazy collapse
// (address bits outside `restrict` mask): address = rValue | deposit(s).
// s bits 0..7 = thread, 8..11 = register j, 12..12+kappa-1 = unit within
// the CTA, the rest = blockIdx. Each CTA writes 17 partial sums:
// [0..7] zero-sums of the thread bits, [8..11] of the j bits,
// [12..15] of the unit bits, [16] the CTA total.
template <class V>
__global__ void __launch_bounds__(256) probKernel(const V *__restrict__ st, const __grid_constant__ ProbArgs args, double *partial) {
    const uint32_t tid = threadIdx.x;
    const uint32_t cta = blockIdx.x;
    const int nFree = args.nFree;
    const int kappa = args.kappa;
    auto bitOf = [&](int i) -> uint64_t { return i < nFree ? (1ULL << args.freePos[i]) : 0ULL; };
    uint64_t dTid = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((tid >> i) & 1u) dTid |= bitOf(i);
    uint64_t dCta = 0;
    for (int i = 0; 12 + kappa + i < nFree; i++)
        if ((cta >> i) & 1u) dCta |= bitOf(12 + kappa + i);
    const uint64_t j0 = bitOf(8), j1 = bitOf(9), j2 = bitOf(10), j3 = bitOf(11);
    const uint64_t limit = nFree >= 63 ? ~0ULL : (1ULL << nFree);

    double tot = 0.0, zj0 = 0.0, zj1 = 0.0, zj2 = 0.0, zj3 = 0.0;
    double zu[4] = {0.0, 0.0, 0.0, 0.0};
    const int units = 1 << kappa;
    for (int u = 0; u < units; u++) {
        uint64_t dU = 0;
        for (int b = 0; b < kappa; b++)
            if ((u >> b) & 1) dU |= bitOf(12 + b);
        const uint64_t gbase = args.rValue | dCta | dU | dTid;
        const uint64_t sbase = ((((uint64_t) cta << kappa) | (uint64_t) u) << 12) | tid;
        double ut = 0.0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint64_t s = sbase | ((uint64_t) j << 8);
            const uint64_t g = gbase | ((j & 1) ? j0 : 0ULL) | ((j & 2) ? j1 : 0ULL) | ((j & 4) ? j2 : 0ULL) | ((j & 8) ? j3 : 0ULL);
            double p = 0.0;
            if (s < limit) {
                const V v = st[g];
                const double re = (double) v.x, im = (double) v.y;
                p = re * re + im * im;
            }
            ut += p;
            if (!(j & 1)) zj0 += p;
            if (!(j & 2)) zj1 += p;
            if (!(j & 4)) zj2 += p;
            if (!(j & 8)) zj3 += p;
        }
        tot += ut;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if (b < kappa && !((u >> b) & 1)) zu[b] += ut;
    }
    double v[17];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = ((tid >> i) & 1u) ? 0.0 : tot;
    v[8] = zj0;
    v[9] = zj1;
    v[10] = zj2;
    v[11] = zj3;
#pragma unroll
    for (int b = 0; b < 4; b++) v[12 + b] = zu[b];
    v[16] = tot;
    __shared__ double red[8][17];
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int i = 0; i < 17; i++) {
        double x = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][i] = x;
    }
    __syncthreads();
    if (tid < 17) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < 8; w++) x += red[w][tid];
        partial[(size_t) cta * 17 + tid] = x;
    }
}

// out[b] for sub-index bit b < nFree, out[nFree] = total.
__global__ void __launch_bounds__(256) probFinalize(const double *__restrict__ partial, int numCtas, int nFree,
                                                   int kappa, double *out) {
    const int b = blockIdx.x;  // 0..nFree
    double x = 0.0;
    const int local = 12 + kappa;
    for (int c = threadIdx.x; c < numCtas; c += blockDim.x) {
        if (b == nFree) {
            x += partial[(size_t) c * 17 + 16];
        } else if (b < local) {
            x += partial[(size_t) c * 17 + b];
        } else if (!((c >> (b - local)) & 1)) {
            x += partial[(size_t) c * 17 + 16];
        }
    }
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int) (blockDim.x >> 5); w++) t += red[w];
        out[b] = t;
    }
}

cudaError_t launchProb(const void *st, bool single, const ProbArgs &args, double *partial, double *out,
                       cudaStream_t s) {
    const int grid = args.nFree > 12 + args.kappa ? (1 << (args.nFree - 12 - args.kappa)) : 1;
    if (single)
        probKernel<float2><<<grid, 256, 0, s>>>((const float2 *) st, args, partial);
    else
        probKernel<double2><<<grid, 256, 0, s>>>((const double2 *) st, args, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    probFinalize<<<args.nFree + 1, 256, 0, s>>>(partial, grid, args.nFree, args.kappa, out);
    return cudaGetLastError();
}

int probNumCtas(const ProbArgs &args) {
    return args.nFree > 12 + args.kappa ? (1 << (args.nFree - 12 - args.kappa)) : 1;
}

// Page-pair exchange of the host tier: pages a and b differ only in the
// page-index bit that is being exchanged with local bit `bit`; every
// amplitude of a whose local index has `bit` = 1 trades places with the
// amplitude of b at the same index with `bit` = 0 (the two halves that the
// exchange of the two address bits moves).
template <class V>
__global__ void pageSwapKernel(V *__restrict__ a, V *__restrict__ b, int pageBits, int bit) {
    const uint64_t half = 1ULL << (pageBits - 1);
    const uint64_t lo = (1ULL << bit) - 1;
    for (uint64_t k = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; k < half;
         k += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t i = ((k & ~lo) << 1) | (1ULL << bit) | (k & lo);
        const uint64_t j = i ^ (1ULL << bit);
        const V x = a[i];
        a[i] = b[j];
        b[j] = x;
    }
}

// --------------------------------------------------- bit-pair exchange
// For every index whose bits at a[i] read pattern p and at b[i] read q with
// p > q (as integers over the k pairs), exchange it with the index whose
// patterns are swapped. Every orbit has length 1 or 2, so this is in place.
template <class V>
__global__ void swapBitsKernel(V *__restrict__ st, const __grid_constant__ SwapArgs args) {
    const uint64_t numAmps = 1ULL << args.numBits;
    for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < numAmps;
         i += (uint64_t) gridDim.x * blockDim.x) {
        uint32_t p = 0, q = 0;
        for (int k = 0; k < args.numPairs; k++) {
            p |= (uint32_t) ((i >> args.a[k]) & 1ULL) << k;
            q |= (uint32_t) ((i >> args.b[k]) & 1ULL) << k;
        }
        if (p <= q) continue;
        uint64_t j = i;
        for (int k = 0; k < args.numPairs; k++) {
            j &= ~((1ULL << args.a[k]) | (1ULL << args.b[k]));
            j |= (uint64_t) ((q >> k) & 1u) << args.a[k];
            j |= (uint64_t) ((p >> k) & 1u) << args.b[k];
        }
        const V x = st[i];
        const V y = st[j];
        st[i] = y;
        st[j] = x;
    }
}

cudaError_t launchPageSwap(void *a, void *b, bool single, int pageBits, int bit, cudaStream_t s) {
    if (pageBits < 1 || bit < 0 || bit >= pageBits) return cudaErrorInvalidValue;
    const uint64_t half = 1ULL << (pageBits - 1);
    const unsigned grid = (unsigned) std::min<uint64_t>((half + 255) / 256, 148u * 16u);
    if (single)
        pageSwapKernel<float2><<<grid, 256, 0, s>>>((float2 *) a, (float2 *) b, pageBits, bit);
    else
        pageSwapKernel<double2><<<grid, 256, 0, s>>>((double2 *) a, (double2 *) b, pageBits, bit);
    return cudaGetLastError();
}

// Block exchange between two shards (sharded registers, several qubits at
// once): for every offset o whose bits at the m positions pos[] are 0,
// x[o | patX] trades places with y[o | patY] (patX, patY: patterns over those
// positions). k enumerates the offsets; inserting a 0 at each position in
// ascending order turns k into o, so consecutive threads touch consecutive
// amplitudes except across the inserted bits.
template <class V>
__global__ void blockSwapKernel(V *__restrict__ x, V *__restrict__ y, const __grid_constant__ BlockSwapArgs args) {
    const uint64_t count = 1ULL << (args.pageBits - args.m);
    for (uint64_t k = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (uint64_t) gridDim.x * blockDim.x) {
        uint64_t o = k;
        for (int t = 0; t < args.m; t++) {
            const int b = args.pos[t];
            o = ((o >> b) << (b + 1)) | (o & ((1ULL << b) - 1));
        }
        const V v = x[o | args.patX];
        x[o | args.patX] = y[o | args.patY];
        y[o | args.patY] = v;
    }
}

cudaError_t launchBlockSwap(void *x, void *y, bool single, const BlockSwapArgs &args, cudaStream_t s) {
    // positions ascending, inside the shard, patterns on them only
    if (args.m < 1 || args.m > 4 || args.pageBits <= args.m || args.pageBits > 40) return cudaErrorInvalidValue;
    uint64_t mask = 0;
    for (int t = 0; t < args.m; t++) {
        if (args.pos[t] < 0 || args.pos[t] >= args.pageBits || (t > 0 && args.pos[t] <= args.pos[t - 1]))
            return cudaErrorInvalidValue;
        mask |= 1ULL << args.pos[t];
    }
    if ((args.patX & ~mask) || (args.patY & ~mask)) return cudaErrorInvalidValue;
    const uint64_t count = 1ULL << (args.pageBits - args.m);
    const unsigned grid = (unsigned) std::min<uint64_t>((count + 255) / 256, 148u * 16u);
    if (single)
        blockSwapKernel<float2><<<grid, 256, 0, s>>>((float2 *) x, (float2 *) y, args);
    else
        blockSwapKernel<double2><<<grid, 256, 0, s>>>((double2 *) x, (double2 *) y, args);
    return cudaGetLastError();
}

cudaError_t launchSwapBits(void *st, bool single, const SwapArgs &args, cudaStream_t s) {
    const uint64_t numAmps = 1ULL << args.numBits;
    uint64_t blocks = (numAmps + 255) / 256;
    if (blocks > 148ULL * 64) blocks = 148ULL * 64;
    if (single)
        swapBitsKernel<float2><<<(unsigned) blocks, 256, 0, s>>>((float2 *) st, args);
    else
        swapBitsKernel<double2><<<(unsigned) blocks, 256, 0, s>>>((double2 *) st, args);
    return cudaGetLastError();
}

// ------------------------------------------------------------ gather
// out[l] = st[virt(l)] for logical indices l in [begin, begin + count),
// with virt() the logical->virtual bit map and the lazy collapse applied.
template <class V>
__global__ void gatherKernel(const V *__restrict__ st, const __grid_constant__ GatherArgs args, double2 *__restrict__ out) {
    for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < args.count;
         i += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t l = args.begin + i * (args.stride ? args.stride : 1ULL);
        uint64_t v = 0;
        for (int b = 0; b < args.numReal; b++) v |= ((l >> b) & 1ULL) << args.l2v[b];
        double2 x = make_double2((double) st[v].x, (double) st[v].y);
        if (args.hasRestrict) {
            if ((v & args.restrictMask) != args.restrictValue)
                x = make_double2(0.0, 0.0);
            else
                x = make_double2(x.x * args.restrictScale, x.y * args.restrictScale);
        }
        out[i] = x;
    }
}

cudaError_t launchGather(const void *st, bool single, const GatherArgs &args, double2 *out, cudaStream_t s) {
    uint64_t blocks = (args.count + 255) / 256;
    if (blocks > 148ULL * 32) blocks = 148ULL * 32;
    if (blocks == 0) blocks = 1;
    if (single)
        gatherKernel<float2><<<(unsigned) blocks, 256, 0, s>>>((const float2 *) st, args, out);
    else
        gatherKernel<double2><<<(unsigned) blocks, 256, 0, s>>>((const double2 *) st, args, out);
    return cudaGetLastError();
}

}  // namespace dgq

namespace dgq {

// ------------------------------------------------- amplitude upload
// out[i] = (re[i], im[i]) for i < count, zero for count <= i < total.
template <class V>
__global__ void interleaveKernel(const double *__restrict__ re, const double *__restrict__ im, uint64_t count,
                                 uint64_t total, V *__restrict__ out) {
    for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t) gridDim.x * blockDim.x) {
        V v;
        v.x = i < count ? re[i] : 0.0;
        v.y = i < count ? im[i] : 0.0;
        out[i] = v;
    }
}

cudaError_t launchInterleave(const double *re, const double *im, uint64_t count, uint64_t total, void *out,
                             bool single, cudaStream_t s) {
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ULL * 32) blocks = 148ULL * 32;
    if (single)
        interleaveKernel<float2><<<(unsigned) blocks, 256, 0, s>>>(re, im, count, total, (float2 *) out);
    else
        interleaveKernel<double2><<<(unsigned) blocks, 256, 0, s>>>(re, im, count, total, (double2 *) out);
    return cudaGetLastError();
}

}  // namespace dgq

namespace dgq {

// ------------------------------------------------ FP64 pipe microbenchmark
// Eight independent DFMA chains per thread; the result is written so the
// work cannot be removed. Used to state the FP64 roofline next to HBM.
__global__ void __launch_bounds__(256) fp64PeakKernel(double *out, int iters, double seed) {
    double x0 = seed + threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
           x7 = x0 + 7;
    const double m = 0.999999, c = 1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fma(x0, m, c);
            x1 = fma(x1, m, c);
            x2 = fma(x2, m, c);
            x3 = fma(x3, m, c);
            x4 = fma(x4, m, c);
            x5 = fma(x5, m, c);
            x6 = fma(x6, m, c);
            x7 = fma(x7, m, c);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

cudaError_t launchFp64Peak(double *out, int blocks, int iters, cudaStream_t s) {
    fp64PeakKernel<<<blocks, 256, 0, s>>>(out, iters, 1.0);
    return cudaGetLastError();
}

}  // namespace dgq

namespace dgq {

// ------------------------------------------------------ inner product
// sum over logical indices of conj(bra) * ket, both registers read through
// their own logical->virtual maps and lazy collapses; FP64 accumulation,
// fixed reduction order (partials per CTA, then one finalise CTA).
template <class VB, class VK>
__global__ void __launch_bounds__(256) innerKernel(const VB *__restrict__ bra, const VK *__restrict__ ket,
                                                   const __grid_constant__ InnerArgs args, double2 *partial) {
    double re = 0.0, im = 0.0;
    const uint64_t n = 1ULL << args.numReal;
    for (uint64_t l = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (uint64_t) gridDim.x * blockDim.x) {
        uint64_t vb = l, vk = l;
        if (!args.identity) {
            vb = 0;
            vk = 0;
            for (int b = 0; b < args.numReal; b++) {
                const uint64_t bit = (l >> b) & 1ULL;
                vb |= bit << args.l2vBra[b];
                vk |= bit << args.l2vKet[b];
            }
        }
        double br = (double) bra[vb].x, bi = (double) bra[vb].y;
        double kr = (double) ket[vk].x, ki = (double) ket[vk].y;
        if (args.braRestrict) {
            const bool keep = (vb & args.braMask) == args.braValue;
            br = keep ? br * args.braScale : 0.0;
            bi = keep ? bi * args.braScale : 0.0;
        }
        if (args.ketRestrict) {
            const bool keep = (vk & args.ketMask) == args.ketValue;
            kr = keep ? kr * args.ketScale : 0.0;
            ki = keep ? ki * args.ketScale : 0.0;
        }
        re += br * kr + bi * ki;
        im += br * ki - bi * kr;
    }
    __shared__ double sre[8], sim[8];
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sre[threadIdx.x >> 5] = re;
        sim[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; w++) {
            a += sre[w];
            b += sim[w];
        }
        partial[blockIdx.x] = make_double2(a, b);
    }
}

__global__ void innerFinalize(const double2 *__restrict__ partial, int n, double2 *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int i = 0; i < n; i++) {
        a += partial[i].x;
        b += partial[i].y;
    }
    *out = make_double2(a, b);
}

int innerNumCtas() { return 148 * 8; }

cudaError_t launchInner(const void *bra, bool braSingle, const void *ket, bool ketSingle, const InnerArgs &args,
                        double2 *partial, double2 *out, cudaStream_t s) {
    const int grid = innerNumCtas();
    if (braSingle && ketSingle)
        innerKernel<float2, float2><<<grid, 256, 0, s>>>((const float2 *) bra, (const float2 *) ket, args, partial);
    else if (braSingle)
        innerKernel<float2, double2><<<grid, 256, 0, s>>>((const float2 *) bra, (const double2 *) ket, args, partial);
    else if (ketSingle)
        innerKernel<double2, float2><<<grid, 256, 0, s>>>((const double2 *) bra, (const float2 *) ket, args, partial);
    else
        innerKernel<double2, double2><<<grid, 256, 0, s>>>((const double2 *) bra, (const double2 *) ket, args, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    innerFinalize<<<1, 32, 0, s>>>(partial, grid, out);
    return cudaGetLastError();
}

}  // namespace dgq
