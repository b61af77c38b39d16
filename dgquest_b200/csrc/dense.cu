// dense.cu -- one sweep applying a dense 2^K x 2^K unitary on K target bits
// (multiQubitUnitary with more targets than a register phase holds).
//
// A CTA owns a tile of 2^TB amplitudes (TB = min(12, numBits)) spanning the
// K target bits and the TB - K lowest other address bits ("columns"); the
// remaining bits come from blockIdx. The tile is loaded in address order
// (coalesced), laid out in shared memory as X[row][column] (row = matrix
// index over the targets, targs[0] its least significant bit), and every
// thread accumulates a 4 x 4 block of Y = U X over 16-column chunks of U
// staged in shared memory. Y goes back through shared memory and is stored
// in address order. The matrix stays in FP64 in global memory (L2 resident)
// and is rounded to the state's precision when staged.
#include <cuda_runtime.h>

#include <cstdint>

#include "interp.cuh"
#include "kernels.h"

namespace dgq {

namespace {

constexpr int kDenseTileBits = 12;
constexpr int kDenseChunk = 16;

template <class V, int K>
__global__ void __launch_bounds__(256, 2) denseKernel(V *__restrict__ st, const __grid_constant__ DenseArgs a,
                                                     const double *__restrict__ U) {
    typedef typename Real<V>::T R;
    constexpr int D = 1 << K;
    const int TB = a.tileBits;
    const int C = TB - K;
    const int G = 1 << C;              // columns (groups) in the tile
    const int T = (1 << TB) >> 4;      // threads doing work: 16 outputs each
    const int RB = D / 4;              // row blocks
    extern __shared__ __align__(16) unsigned char smRaw[];
    V *Xs = reinterpret_cast<V *>(smRaw);                 // [D][G]
    V *Us = Xs + (1 << TB);                               // [kDenseChunk][D]
    const uint32_t tid = threadIdx.x;
    const uint32_t cta = blockIdx.x;

    uint64_t base = 0;
    for (int i = 0; i < a.numBits - TB; i++) base |= (uint64_t) ((cta >> i) & 1u) << a.ctaPos[i];

    // address-ordered tile index i = tid + T j -> (address, row, column): the
    // bits of tid and of j are disjoint, so their parts OR together; the 16
    // j parts sit in a table
    __shared__ uint64_t jAddr[16];
    __shared__ uint32_t jRow[16], jCol[16];
    const int tb = TB - 4;  // bits of tid
    auto part = [&](uint32_t bits, int from, int to, uint64_t &addr, uint32_t &row, uint32_t &col) {
        addr = 0;
        row = 0;
        col = 0;
        for (int b = from; b < to; b++) {
            if (!((bits >> (b - from)) & 1u)) continue;
            addr |= 1ULL << a.tilePos[b];
            const int r = a.rowBit[b];
            if (r >= 0)
                row |= 1u << r;
            else
                col |= 1u << a.colBit[b];
        }
    };
    if (tid < 16) {
        uint64_t ad;
        uint32_t r, c;
        part(tid, tb, TB, ad, r, c);
        jAddr[tid] = ad;
        jRow[tid] = r;
        jCol[tid] = c;
    }
    uint64_t tAddr;
    uint32_t tRow, tCol;
    part(tid, 0, tb, tAddr, tRow, tCol);
    tAddr |= base;
    __syncthreads();

    R inScale = (R) 1;
    if (a.normIn) inScale = (R) rsqrt(*a.normIn);
    if ((int) tid < T) {
        for (int j = 0; j < 16; j++) {
            const uint64_t addr = tAddr | jAddr[j];
            V v = st[addr];
            R sc = inScale;
            if (a.hasRestrict && (addr & a.restrictMask) != a.restrictValue) sc = (R) 0;
            else if (a.hasRestrict) sc *= (R) a.restrictScale;
            v = mk<V>(v.x * sc, v.y * sc);
            Xs[(tRow | jRow[j]) * G + (tCol | jCol[j])] = v;
        }
    }
    __syncthreads();

    const int rb = (int) tid % RB, cb = (int) tid / RB;
    R accR[4][4], accI[4][4];
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            accR[p][q] = 0;
            accI[p][q] = 0;
        }
    for (int c0 = 0; c0 < D; c0 += kDenseChunk) {
        // stage U[:, c0 .. c0 + 16) as Us[cc][r]
        for (int e = (int) tid; e < kDenseChunk * D; e += (int) blockDim.x) {
            const int cc = e / D, r = e % D;
            const double *m = U + 2 * ((size_t) r * D + (size_t) (c0 + cc));
            Us[cc * D + r] = mk<V>((R) m[0], (R) m[1]);
        }
        __syncthreads();
        if ((int) tid < T) {
#pragma unroll 4
            for (int cc = 0; cc < kDenseChunk; cc++) {
                V u[4], x[4];
#pragma unroll
                for (int p = 0; p < 4; p++) u[p] = Us[cc * D + rb * 4 + p];
#pragma unroll
                for (int q = 0; q < 4; q++) x[q] = Xs[(c0 + cc) * G + cb * 4 + q];
#pragma unroll
                for (int p = 0; p < 4; p++)
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        accR[p][q] = fma(u[p].x, x[q].x, fma(-u[p].y, x[q].y, accR[p][q]));
                        accI[p][q] = fma(u[p].x, x[q].y, fma(u[p].y, x[q].x, accI[p][q]));
                    }
            }
        }
        __syncthreads();
    }
    // Y into the tile buffer (every read of X is done), then out in address order
    if ((int) tid < T) {
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) Xs[(rb * 4 + p) * G + cb * 4 + q] = mk<V>(accR[p][q], accI[p][q]);
    }
    __syncthreads();
    double norm = 0.0;
    if ((int) tid < T) {
        for (int j = 0; j < 16; j++) {
            const V y = Xs[(tRow | jRow[j]) * G + (tCol | jCol[j])];
            st[tAddr | jAddr[j]] = y;
            norm += (double) y.x * (double) y.x + (double) y.y * (double) y.y;
        }
    }
    if (a.normOut) {
        __shared__ double red[8];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) norm += __shfl_xor_sync(0xffffffffu, norm, o);
        if ((tid & 31u) == 0) red[tid >> 5] = norm;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < 8; w++) t += red[w];
            atomicAdd(a.normOut, t);
        }
    }
}

template <class V, int K>
cudaError_t launchDenseVK(V *st, const DenseArgs &a, const double *U, cudaStream_t s) {
    const size_t smem = (sizeof(V) << a.tileBits) + sizeof(V) * kDenseChunk * (1u << K);
    static std::atomic<uint64_t> optIn{0};
    cudaError_t e = ensureSmemOptIn((const void *) denseKernel<V, K>,
                                    (int) ((sizeof(V) << kDenseTileBits) + sizeof(V) * kDenseChunk * (1u << 7)), optIn);
    if (e != cudaSuccess) return e;
    const unsigned grid = 1u << (a.numBits - a.tileBits);
    denseKernel<V, K><<<grid, 256, smem, s>>>(st, a, U);
    return cudaGetLastError();
}

template <class V>
cudaError_t launchDenseV(V *st, int K, const DenseArgs &a, const double *U, cudaStream_t s) {
    switch (K) {
        case 5: return launchDenseVK<V, 5>(st, a, U, s);
        case 6: return launchDenseVK<V, 6>(st, a, U, s);
        case 7: return launchDenseVK<V, 7>(st, a, U, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool denseArgs(int numBits, int K, const uint8_t *targets, DenseArgs &a) {
    if (K < kMinDenseTargets || K > kMaxDenseTargets) return false;
    const int TB = numBits < kDenseTileBits ? numBits : kDenseTileBits;
    if (TB - K < 2) return false;  // 4 x 4 blocks need >= 4 columns
    a = DenseArgs();
    a.numBits = numBits;
    a.tileBits = TB;
    uint64_t tmask = 0;
    for (int i = 0; i < K; i++) tmask |= 1ULL << targets[i];
    // columns: the lowest non-target bits
    int cols = 0;
    uint64_t cmask = 0;
    for (int b = 0; b < numBits && cols < TB - K; b++)
        if (!((tmask >> b) & 1ULL)) {
            cmask |= 1ULL << b;
            cols++;
        }
    const uint64_t tile = tmask | cmask;
    int nt = 0, nc = 0, colRank = 0;
    for (int b = 0; b < numBits; b++) {
        if ((tile >> b) & 1ULL) {
            a.tilePos[nt] = (uint8_t) b;
            a.rowBit[nt] = -1;
            a.colBit[nt] = -1;
            if ((tmask >> b) & 1ULL) {
                for (int i = 0; i < K; i++)
                    if (targets[i] == b) a.rowBit[nt] = (int8_t) i;
            } else {
                a.colBit[nt] = (int8_t) colRank++;
            }
            nt++;
        } else {
            a.ctaPos[nc++] = (uint8_t) b;
        }
    }
    return nt == TB;
}

cudaError_t launchDense(void *st, bool single, int K, const DenseArgs &a, const double *U, cudaStream_t s) {
    return single ? launchDenseV((float2 *) st, K, a, U, s) : launchDenseV((double2 *) st, K, a, U, s);
}

}  // namespace dgq
