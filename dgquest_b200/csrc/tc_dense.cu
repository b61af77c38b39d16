// tc_dense.cu -- dense 6-target unitary on a complex64 state with the 5th
// generation tensor cores (tcgen05, kind::tf32), split precision 3xTF32.
//
// Complex Y = U X is the real product [Yr; Yi] = [[Ur, -Ui], [Ui, Ur]] [Xr; Xi]:
// M = 128 output rows, K = 128, N = 64 columns (groups of 64 amplitudes that
// differ in the 6 target bits). Each operand is split into a TF32 head and
// an FP32 tail (x = hi + lo, hi = x with the 13 low mantissa bits cleared),
// and D = Ahi Bhi + Ahi Blo + Alo Bhi accumulates in FP32 in tensor memory,
// which keeps the product to FP32 accuracy. The real matrix A (head and
// tail, 2 x 64 KiB, prepared on the host) stays in shared memory for the
// whole persistent CTA; per tile of 4096 amplitudes the CTA loads the
// columns, splits them into the B operands, issues 16 K-steps x 3 MMAs from
// one thread, waits on an mbarrier (bounded), reads D with tcgen05.ld and
// writes the tile back through shared memory in address order.
//
// Operand layout (K-major, no swizzle): 8-row x 16-byte core matrices; row
// r of a core matrix at 16 r bytes, core matrix (row group g, K chunk c of 4
// elements) at ((c * groups) + g) * 128 bytes, so SBO = 128 B (next row
// group) and LBO = groups * 128 B (next K chunk); one MMA (K = 8) covers two
// K chunks. The encodings follow the UMMA descriptor definitions of CUTLASS
// (cute/arch/mma_sm100_desc.hpp).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "kernels.h"

namespace dgq {

namespace {

constexpr int kTcK = 6;               // targets
constexpr int kTcD = 1 << kTcK;       // 64 complex rows
constexpr int kTcM = 2 * kTcD;        // 128 real rows (A rows, D lanes)
constexpr int kTcKdim = 2 * kTcD;     // 128 real inputs
constexpr int kTcN = 64;              // columns per tile (tile = 4096 amplitudes)
constexpr int kTcThreads = 128;
constexpr uint32_t kABytes = kTcM * kTcKdim * 4;   // 64 KiB per A part
constexpr uint32_t kBBytes = kTcN * kTcKdim * 4;   // 32 KiB per B part
constexpr uint32_t kXBytes = 4096 * 8;                // tile staging: X[column][row], later Y
constexpr uint32_t kTcSmem = 2 * kABytes + 2 * kBBytes + kXBytes + 1024;
// eight accumulators (K eighths, all 512 TMEM columns), summed in FP32 with
// round-to-nearest in the epilogue: each sums 6 MMAs instead of 48, which
// keeps the tensor core's FP32 accumulation from biasing the norm
constexpr int kTcAcc = 8;
constexpr uint32_t kTmemCols = kTcN * kTcAcc;

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

// byte offset of element (row, k) in a K-major no-swizzle operand with `groups` row groups
__device__ __forceinline__ uint32_t kmajorOffset(uint32_t row, uint32_t k, uint32_t groups) {
    return (((k >> 2) * groups + (row >> 3)) << 7) + ((row & 7u) << 4) + ((k & 3u) << 2);
}

__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t) ((addr >> 4) & 0x3FFFu);
    d |= (uint64_t) ((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t) ((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t) 1 << 46;  // descriptor version for sm100
    // base offset 0, LBO mode 0, layout type 0 (no swizzle)
    return d;
}

// tf32 x tf32 -> f32, both K-major, M = 128, N = 64
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t) (kTcN >> 3) << 17) |
                            ((uint32_t) (kTcM >> 4) << 24);

__device__ __forceinline__ void mmaTf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ float tf32Head(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// Polls the mbarrier phase `parity`; false after `limit` polls.
__device__ __forceinline__ bool waitParity(uint32_t mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t n = 0; n < limit; n++) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

__global__ void __launch_bounds__(kTcThreads, 1)
    tcDenseKernel(float2 *__restrict__ st, const __grid_constant__ DenseArgs a, const float *__restrict__ Apacked,
                  uint32_t *__restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smRaw[];
    unsigned char *base = smRaw + ((1024u - (smemAddr(smRaw) & 1023u)) & 1023u);
    unsigned char *aHi = base;
    unsigned char *aLo = base + kABytes;
    unsigned char *bHi = base + 2 * kABytes;
    unsigned char *bLo = bHi + kBBytes;
    // tile staging: X in as [row][column], Y out as [column][row]
    float2 *xs = reinterpret_cast<float2 *>(bLo + kBBytes);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmemBase;
    __shared__ uint32_t abort;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const int TB = a.tileBits;  // 12: 6 targets + 6 column bits
    const uint32_t numTiles = 1u << (a.numBits - TB);

    // resident A (head and tail), already in the operand layout
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(Apacked);
        uint4 *dst = reinterpret_cast<uint4 *>(aHi);
        for (uint32_t i = tid; i < 2 * kABytes / 16; i += kTcThreads) dst[i] = __ldg(src + i);
    }
    if (tid == 0) {
        abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(&tmemBase)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmemBase;
    const uint32_t mbarAddr = smemAddr(&mbar);
    uint32_t parity = 0;

    // address-ordered tile index i = tid + 128 j: the parts of tid (7 bits)
    // and of j (5 bits) OR together; the 32 j parts sit in a table
    __shared__ uint64_t jAddr[32];
    __shared__ uint32_t jRow[32], jCol[32];
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
    if (tid < 32) {
        uint64_t ad;
        uint32_t r, c;
        part(tid, 7, TB, ad, r, c);
        jAddr[tid] = ad;
        jRow[tid] = r;
        jCol[tid] = c;
    }
    uint64_t tAddr;
    uint32_t tRow, tCol;
    part(tid, 0, 7, tAddr, tRow, tCol);
    float inScale = 1.0f;
    if (a.normIn) inScale = (float) rsqrt(*a.normIn);
    double norm = 0.0;
    __syncthreads();

    constexpr int kPer = 4096 / kTcThreads;  // amplitudes per thread and tile
    auto tileBaseOf = [&](uint32_t tile) {
        uint64_t b = 0;
        for (int i = 0; i < a.numBits - TB; i++) b |= (uint64_t) ((tile >> i) & 1u) << a.ctaPos[i];
        return b;
    };
    // the next tile's amplitudes are loaded into registers while the current
    // tile's MMAs and epilogue run
    float2 next[kPer];
    if (blockIdx.x < numTiles) {
        const uint64_t nb = tileBaseOf(blockIdx.x);
#pragma unroll
        for (int j = 0; j < kPer; j++) next[j] = st[nb | tAddr | jAddr[j]];
    }
    for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x) {
        const uint64_t tileBase = tileBaseOf(tile);
        // columns -> B head / tail: B[n][k] = Re X[k][n] (k < 64), Im X[k - 64][n]
#pragma unroll
        for (int j = 0; j < kPer; j++) {
            const uint64_t addr = tileBase | tAddr | jAddr[j];
            const uint32_t row = tRow | jRow[j], col = tCol | jCol[j];
            float2 v = next[j];
            float sc = inScale;
            if (a.hasRestrict) sc = (addr & a.restrictMask) == a.restrictValue ? sc * (float) a.restrictScale : 0.0f;
            xs[row * kTcN + col] = make_float2(v.x * sc, v.y * sc);
        }
        __syncthreads();
        // B head / tail in 16-byte pieces: column n, K chunk c (4 rows of X)
        // (consecutive threads: consecutive columns, so both the 8-byte reads
        // and the 16-byte writes are contiguous across a warp)
        for (uint32_t p = tid; p < kTcN * (kTcKdim / 4); p += kTcThreads) {
            const uint32_t n = p % kTcN, c = p / kTcN;  // c < 16: real parts, c >= 16: imaginary parts
            const uint32_t r0 = (c & 15u) * 4u;
            const float2 x0 = xs[(r0 + 0) * kTcN + n], x1 = xs[(r0 + 1) * kTcN + n];
            const float2 x2 = xs[(r0 + 2) * kTcN + n], x3 = xs[(r0 + 3) * kTcN + n];
            float4 v = c < 16 ? make_float4(x0.x, x1.x, x2.x, x3.x) : make_float4(x0.y, x1.y, x2.y, x3.y);
            const float4 h = make_float4(tf32Head(v.x), tf32Head(v.y), tf32Head(v.z), tf32Head(v.w));
            const uint32_t off = kmajorOffset(n, c * 4u, kTcN / 8);
            *reinterpret_cast<float4 *>(bHi + off) = h;
            *reinterpret_cast<float4 *>(bLo + off) = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t aLbo = (kTcM / 8) * 128, bLbo = (kTcN / 8) * 128;
            for (int s = 0; s < kTcKdim / 8; s++) {
                const uint64_t dAh = smemDesc(smemAddr(aHi) + (uint32_t) s * 2 * aLbo, aLbo, 128);
                const uint64_t dAl = smemDesc(smemAddr(aLo) + (uint32_t) s * 2 * aLbo, aLbo, 128);
                const uint64_t dBh = smemDesc(smemAddr(bHi) + (uint32_t) s * 2 * bLbo, bLbo, 128);
                const uint64_t dBl = smemDesc(smemAddr(bLo) + (uint32_t) s * 2 * bLbo, bLbo, 128);
                // K quarter q = s / 4 accumulates in TMEM columns [64 q, 64 q + 64)
                const uint32_t acc = tmem + (uint32_t) (s / (kTcKdim / 8 / kTcAcc)) * kTcN;
                mmaTf32(acc, dAh, dBh, (s % (kTcKdim / 8 / kTcAcc)) != 0 ? 1u : 0u);
                mmaTf32(acc, dAh, dBl, 1u);
                mmaTf32(acc, dAl, dBh, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbarAddr)
                         : "memory");
        }
        if (tile + gridDim.x < numTiles) {
            const uint64_t nb = tileBaseOf(tile + gridDim.x);
#pragma unroll
            for (int j = 0; j < kPer; j++) next[j] = st[nb | tAddr | jAddr[j]];
        }
        if (!waitParity(mbarAddr, parity, 1u << 22)) {
            atomicOr(error, 1u);
            abort = 1;
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (abort) {
            // the committed MMAs may still be writing tensor memory: before it
            // is released below, wait once more (bounded) for their commit
            // (the phase just waited on), and skip this tile's epilogue
            waitParity(mbarAddr, parity ^ 1u, 1u << 24);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            break;
        }
        // D row (lane) 32 w + t: Re Y[row] for rows < 64, Im Y[row - 64] above
        const uint32_t m = warp * 32 + lane;
        float *ysf = reinterpret_cast<float *>(xs);
#pragma unroll 1
        for (int chunk = 0; chunk < kTcN / 16; chunk++) {
            float y[16];
#pragma unroll
            for (int q = 0; q < 16; q++) y[q] = 0.0f;
#pragma unroll
            for (int acc = 0; acc < kTcAcc; acc++) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((warp * 32u) << 16) + (uint32_t) (acc * kTcN + chunk * 16);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr)
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int q = 0; q < 16; q++) y[q] += __uint_as_float(r[q]);
            }
            const uint32_t row = m & (kTcD - 1), half = m >> kTcK;
#pragma unroll
            for (int q = 0; q < 16; q++) ysf[2 * ((uint32_t) (chunk * 16 + q) * kTcD + row) + half] = y[q];
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        for (uint32_t j = 0; j < (1u << TB) / kTcThreads; j++) {
            const float2 y = xs[(tCol | jCol[j]) * kTcD + (tRow | jRow[j])];
            st[tileBase | tAddr | jAddr[j]] = y;
            norm += (double) y.x * (double) y.x + (double) y.y * (double) y.y;
        }
        __syncthreads();
    }
    if (a.normOut) {
        __shared__ double red[kTcThreads / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) norm += __shfl_xor_sync(0xffffffffu, norm, o);
        if (lane == 0) red[warp] = norm;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < kTcThreads / 32; w++) t += red[w];
            atomicAdd(a.normOut, t);
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

__device__ uint32_t g_tcDenseError;

}  // namespace

// A = [[Ur, -Ui], [Ui, Ur]] in FP32, split into TF32 head and FP32 tail, both
// in the K-major operand layout: 2 x 128 x 128 floats.
void packTcDenseMatrix(const double *U, float *out) {
    float *hi = out, *lo = out + kTcM * kTcKdim;
    for (int m = 0; m < kTcM; m++)
        for (int k = 0; k < kTcKdim; k++) {
            const int r = m & (kTcD - 1), c = k & (kTcD - 1);
            const double ur = U[2 * (r * kTcD + c)], ui = U[2 * (r * kTcD + c) + 1];
            double v;
            if (m < kTcD)
                v = k < kTcD ? ur : -ui;
            else
                v = k < kTcD ? ui : ur;
            const float f = (float) v;
            uint32_t bits;
            std::memcpy(&bits, &f, 4);
            bits &= 0xFFFFE000u;
            float h;
            std::memcpy(&h, &bits, 4);
            const uint32_t off = ((((uint32_t) k >> 2) * (kTcM / 8) + ((uint32_t) m >> 3)) << 7) +
                                 (((uint32_t) m & 7u) << 4) + (((uint32_t) k & 3u) << 2);
            hi[off / 4] = h;
            lo[off / 4] = f - h;
        }
}

size_t tcDenseMatrixFloats() { return 2 * (size_t) kTcM * kTcKdim; }

uint32_t *tcDenseErrorWord() {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tcDenseError) != cudaSuccess) return nullptr;
    return (uint32_t *) p;
}

cudaError_t launchTcDense(float2 *st, const DenseArgs &a, const float *Apacked, uint32_t *error, cudaStream_t s) {
    if (a.tileBits != 12 || !error) return cudaErrorInvalidValue;
    static std::atomic<uint64_t> optIn{0};
    cudaError_t e = ensureSmemOptIn((const void *) tcDenseKernel, (int) kTcSmem, optIn);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t tiles = 1u << (a.numBits - a.tileBits);
    const unsigned grid = (unsigned) (tiles < (uint32_t) sms ? tiles : (uint32_t) sms);
    tcDenseKernel<<<grid, kTcThreads, kTcSmem, s>>>(st, a, Apacked, error);
    return cudaGetLastError();
}

}  // namespace dgq
