// jit_prelude.cuh -- device code shared by the runtime-specialised sweep
// kernels (codegen.cpp writes one kernel per sweep program and NVRTC
// compiles it for sm_100a together with this header and tile_program.h).
//
// The generated kernel is the tile kernel of kernels.cu with everything
// that is fixed by the plan turned into compile-time constants: the phase
// layouts (register and thread bits, shared-memory offsets), the sequence
// of operations with their target register bits and control masks, and the
// positions of their coefficients in the parameter block. The amplitudes
// then flow from one operation to the next as plain SSA values, with no
// dispatch and no merge points, and the coefficients are read straight from
// the constant bank. Only values that change between runs of the same
// structure (coefficients, address-bit positions, initial index, collapse
// mask) stay in the TileProgram parameter.
#pragma once

#include "tile_program.h"

namespace dgq {

// V is double2 (complex128 state) or float2 (complex64 state); R its scalar.
template <class V>
struct VecOf;
template <>
struct VecOf<double2> {
    typedef double R;
    static __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct VecOf<float2> {
    typedef float R;
    static __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
};
#define DGQJ_R typename VecOf<V>::R
#define DGQJ_MK(x, y) VecOf<V>::make((x), (y))

__device__ __forceinline__ uint32_t swz(uint32_t x) { return x ^ (((x >> 3) ^ (x >> 6) ^ (x >> 9) ^ (x >> 12)) & 7u); }

// ---------------------------------------------------------------- operations
#define DGQJ_PAIR_LOOP(K, CTRL, cr, ...)                                        \
    _Pragma("unroll") for (int p_ = 0; p_ < kRegs / 2; p_++) {                  \
        const int j0 = ((p_ >> (K)) << ((K) + 1)) | (p_ & ((1 << (K)) - 1));    \
        const int j1 = j0 | (1 << (K));                                         \
        if ((CTRL) && (j0 & (cr)) != (cr)) continue;                            \
        V &x = a[j0];                                                           \
        V &y = a[j1];                                                           \
        __VA_ARGS__                                                             \
    }

#define DGQJ_AMP_LOOP(CTRL, cr, ...)                                            \
    _Pragma("unroll") for (int j = 0; j < kRegs; j++) {                         \
        if ((CTRL) && (j & (cr)) != (cr)) continue;                             \
        V &x = a[j];                                                            \
        __VA_ARGS__                                                             \
    }

// [[m0, m1], [m2, m3]] real
template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jM2R(V (&a)[kRegs], const double *c) {
    const DGQJ_R m0 = (DGQJ_R) c[0], m1 = (DGQJ_R) c[1], m2 = (DGQJ_R) c[2], m3 = (DGQJ_R) c[3];
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const DGQJ_R t0 = m2 * x.x, t1 = m2 * x.y, u0 = m1 * y.x, u1 = m1 * y.y;
        x.x = fma(m0, x.x, u0);
        x.y = fma(m0, x.y, u1);
        y.x = fma(m3, y.x, t0);
        y.y = fma(m3, y.y, t1);
    })
}

// [[m0, i m1], [i m2, m3]] with m real
template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jM2I(V (&a)[kRegs], const double *c) {
    const DGQJ_R m0 = (DGQJ_R) c[0], m1 = (DGQJ_R) c[1], m2 = (DGQJ_R) c[2], m3 = (DGQJ_R) c[3];
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const DGQJ_R t0 = m2 * x.y, t1 = m2 * x.x, u0 = m1 * y.y, u1 = m1 * y.x;
        x.x = fma(m0, x.x, -u0);
        x.y = fma(m0, x.y, u1);
        y.x = fma(m3, y.x, -t0);
        y.y = fma(m3, y.y, t1);
    })
}

// general complex 2x2, row-major (re, im)
template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jM2C(V (&a)[kRegs], const double *c) {
    const DGQJ_R u0 = (DGQJ_R) c[0], u1 = (DGQJ_R) c[1], u2 = (DGQJ_R) c[2], u3 = (DGQJ_R) c[3], u4 = (DGQJ_R) c[4],
                 u5 = (DGQJ_R) c[5], u6 = (DGQJ_R) c[6], u7 = (DGQJ_R) c[7];
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        DGQJ_R xr = u0 * x.x;
        xr = fma(-u1, x.y, xr);
        xr = fma(u2, y.x, xr);
        xr = fma(-u3, y.y, xr);
        DGQJ_R xi = u0 * x.y;
        xi = fma(u1, x.x, xi);
        xi = fma(u2, y.y, xi);
        xi = fma(u3, y.x, xi);
        DGQJ_R yr = u4 * x.x;
        yr = fma(-u5, x.y, yr);
        yr = fma(u6, y.x, yr);
        yr = fma(-u7, y.y, yr);
        DGQJ_R yi = u4 * x.y;
        yi = fma(u5, x.x, yi);
        yi = fma(u6, y.y, yi);
        yi = fma(u7, y.x, yi);
        x = DGQJ_MK(xr, xi);
        y = DGQJ_MK(yr, yi);
    })
}

template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jX(V (&a)[kRegs]) {
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const V t = x;
        x = y;
        y = t;
    })
}

template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jY(V (&a)[kRegs]) {
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const V t = x;
        x = DGQJ_MK(y.y, -y.x);
        y = DGQJ_MK(-t.y, t.x);
    })
}

template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jYC(V (&a)[kRegs]) {
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const V t = x;
        x = DGQJ_MK(-y.y, y.x);
        y = DGQJ_MK(t.y, -t.x);
    })
}

template <class V>
__device__ __forceinline__ void jPhaseMul(V &x, double csd, double snd) {
    const DGQJ_R cs = (DGQJ_R) csd, sn = (DGQJ_R) snd;
    const DGQJ_R t = sn * x.y, u = sn * x.x;
    x.x = fma(cs, x.x, -t);
    x.y = fma(cs, x.y, u);
}

// diag(c - i s, c + i s) selected by register bit K
template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jZ2R(V (&a)[kRegs], const double *c) {
    const double cs = c[0], sn = c[1];
    DGQJ_AMP_LOOP(CTRL, CR, { jPhaseMul(x, cs, ((j >> K) & 1) ? sn : -sn); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jPH(V (&a)[kRegs], double cs, double sn) {
    DGQJ_AMP_LOOP(CTRL, CR, { jPhaseMul(x, cs, sn); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jNEG(V (&a)[kRegs]) {
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(-x.x, -x.y); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jMULI(V (&a)[kRegs]) {
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(-x.y, x.x); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jMULNI(V (&a)[kRegs]) {
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(x.y, -x.x); })
}

// Factored uncontrolled gates (the scalar factor is applied once per sweep)
template <int K, class V>
__device__ __forceinline__ void jRY1(V (&a)[kRegs], const double *c) {
    const DGQJ_R t = (DGQJ_R) c[0];
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(fma(-t, y.x, x0.x), fma(-t, y.y, x0.y));
        y = DGQJ_MK(fma(t, x0.x, y.x), fma(t, x0.y, y.y));
    })
}
template <int K, class V>
__device__ __forceinline__ void jRY2(V (&a)[kRegs], const double *c) {
    const DGQJ_R u = (DGQJ_R) c[0];
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(fma(u, x0.x, -y.x), fma(u, x0.y, -y.y));
        y = DGQJ_MK(fma(u, y.x, x0.x), fma(u, y.y, x0.y));
    })
}
template <int K, class V>
__device__ __forceinline__ void jRX1(V (&a)[kRegs], const double *c) {
    const DGQJ_R t = (DGQJ_R) c[0];
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(fma(t, y.y, x0.x), fma(-t, y.x, x0.y));
        y = DGQJ_MK(fma(t, x0.y, y.x), fma(-t, x0.x, y.y));
    })
}
template <int K, class V>
__device__ __forceinline__ void jRX2(V (&a)[kRegs], const double *c) {
    const DGQJ_R u = (DGQJ_R) c[0];
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(fma(u, x0.x, y.y), fma(u, x0.y, -y.x));
        y = DGQJ_MK(fma(u, y.x, x0.y), fma(u, y.y, -x0.x));
    })
}
template <int K, class V>
__device__ __forceinline__ void jH1(V (&a)[kRegs]) {
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(x0.x + y.x, x0.y + y.y);
        y = DGQJ_MK(x0.x - y.x, x0.y - y.y);
    })
}
// phase (cs + i sn) on the amplitudes whose register bit K is 1
template <int K, class V>
__device__ __forceinline__ void jPH1R(V (&a)[kRegs], const double *c) {
    const double cs = c[0], sn = c[1];
#pragma unroll
    for (int j = 0; j < kRegs; j++)
        if ((j >> K) & 1) jPhaseMul(a[j], cs, sn);
}
template <class V>
__device__ __forceinline__ void jGlobal(V (&a)[kRegs], double grd, double gid) {
    const DGQJ_R gr = (DGQJ_R) grd, gi = (DGQJ_R) gid;
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const V x = a[j];
        a[j] = DGQJ_MK(fma(gr, x.x, -gi * x.y), fma(gr, x.y, gi * x.x));
    }
}

template <int KK, uint32_t CR, class V>
__device__ __forceinline__ void jDense(V (&a)[kRegs], const double *m) {
    constexpr int D = 1 << KK;
#pragma unroll
    for (int g = 0; g < (kRegs >> KK); g++) {
        const int base = g << KK;
        if ((base & CR) != CR) continue;
        V v[D];
#pragma unroll
        for (int c = 0; c < D; c++) v[c] = a[base + c];
#pragma unroll
        for (int r = 0; r < D; r++) {
            DGQJ_R re = 0, im = 0;
#pragma unroll
            for (int c = 0; c < D; c++) {
                const DGQJ_R mr = (DGQJ_R) m[2 * (r * D + c)], mi = (DGQJ_R) m[2 * (r * D + c) + 1];
                re = fma(mr, v[c].x, re);
                re = fma(-mi, v[c].y, re);
                im = fma(mr, v[c].y, im);
                im = fma(mi, v[c].x, im);
            }
            a[base + r] = DGQJ_MK(re, im);
        }
    }
}

// ---------------------------------------------------------------- tile I/O
// Canonical element (tid, j) of the tile sits at tile-local index
// tid + T * j: lanes cover the 5 lowest address bits, j the top 4 tile bits.
template <int W>
__device__ __forceinline__ uint64_t jBase(const TileProgram &prog, uint32_t tid, uint32_t cta) {
    uint64_t t = tid & 31u;
    const int nCta = prog.numBits - W;
    for (int i = 0; i < nCta; i++) t |= (uint64_t) ((cta >> i) & 1u) << prog.ctaPos[i];
#pragma unroll
    for (int i = 0; i < W - 9; i++) t |= (uint64_t) ((tid >> (5 + i)) & 1u) << prog.highPos[i];
    return t;
}

template <int W>
__device__ __forceinline__ uint64_t jIndex(const TileProgram &prog, uint64_t base, int j) {
    uint64_t g = base;
    if (j & 1) g |= 1ULL << prog.highPos[W - 9];
    if (j & 2) g |= 1ULL << prog.highPos[W - 8];
    if (j & 4) g |= 1ULL << prog.highPos[W - 7];
    if (j & 8) g |= 1ULL << prog.highPos[W - 6];
    return g;
}

template <int W, int INIT, bool RESTRICT, class V>
__device__ __forceinline__ void jLoad(const V *__restrict__ st, const TileProgram &prog, uint32_t tid,
                                      uint32_t cta, V (&a)[kRegs]) {
    const uint64_t base = jBase<W>(prog, tid, cta);
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const uint64_t g = jIndex<W>(prog, base, j);
        V v;
        if (INIT == INIT_NONE) {
            v = st[g];
        } else if (INIT == INIT_CLASSICAL) {
            v = DGQJ_MK((DGQJ_R) (g == prog.initIndex ? 1.0 : 0.0), (DGQJ_R) 0);
        } else if (INIT == INIT_PLUS) {
            v = DGQJ_MK((DGQJ_R) ((g >> prog.numReal) == 0ULL ? prog.initAmp : 0.0), (DGQJ_R) 0);
        } else {
            v = DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        if (RESTRICT) {
            const bool keep = (g & prog.restrictMask) == prog.restrictValue;
            const DGQJ_R sc = (DGQJ_R) prog.restrictScale;
            v = keep ? DGQJ_MK(v.x * sc, v.y * sc) : DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        a[j] = v;
    }
}

template <int W, class V>
__device__ __forceinline__ void jStore(V *__restrict__ st, const TileProgram &prog, uint32_t tid, uint32_t cta,
                                       const V (&a)[kRegs]) {
    const uint64_t base = jBase<W>(prog, tid, cta);
#pragma unroll
    for (int j = 0; j < kRegs; j++) st[jIndex<W>(prog, base, j)] = a[j];
}

// Adds the CTA's sum of |a|^2 (FP64) to *out: one atomic per CTA.
template <class V>
__device__ __forceinline__ void jNormAccumulate(const V (&a)[kRegs], double *out) {
    __shared__ double red[32];
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kRegs; j++) acc += (double) a[j].x * (double) a[j].x + (double) a[j].y * (double) a[j].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int) (blockDim.x >> 5); w++) t += red[w];
        atomicAdd(out, t);
    }
}

// Direct layouts: thread bits 0..4 are address bits 0..4; the other
// thread bits and the 4 register bits are given as address-bit values.
template <int INIT, bool RESTRICT, class V>
__device__ __forceinline__ void jLoadDirect(const V *__restrict__ st, const TileProgram &prog, uint64_t gt,
                                            const uint64_t (&rb)[kRegBits], V (&a)[kRegs]) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const uint64_t g = gt | ((j & 1) ? rb[0] : 0ULL) | ((j & 2) ? rb[1] : 0ULL) | ((j & 4) ? rb[2] : 0ULL) |
                           ((j & 8) ? rb[3] : 0ULL);
        V v;
        if (INIT == INIT_NONE) {
            v = st[g];
        } else if (INIT == INIT_CLASSICAL) {
            v = DGQJ_MK((DGQJ_R) (g == prog.initIndex ? 1.0 : 0.0), (DGQJ_R) 0);
        } else if (INIT == INIT_PLUS) {
            v = DGQJ_MK((DGQJ_R) ((g >> prog.numReal) == 0ULL ? prog.initAmp : 0.0), (DGQJ_R) 0);
        } else {
            v = DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        if (RESTRICT) {
            const bool keep = (g & prog.restrictMask) == prog.restrictValue;
            const DGQJ_R sc = (DGQJ_R) prog.restrictScale;
            v = keep ? DGQJ_MK(v.x * sc, v.y * sc) : DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        a[j] = v;
    }
}

template <class V>
__device__ __forceinline__ void jStoreDirect(V *__restrict__ st, uint64_t gt, const uint64_t (&rb)[kRegBits],
                                             const V (&a)[kRegs]) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const uint64_t g = gt | ((j & 1) ? rb[0] : 0ULL) | ((j & 2) ? rb[1] : 0ULL) | ((j & 4) ? rb[2] : 0ULL) |
                           ((j & 8) ? rb[3] : 0ULL);
        st[g] = a[j];
    }
}

__device__ __forceinline__ uint64_t jCtaBase(const TileProgram &prog, uint32_t cta, int W) {
    uint64_t t = 0;
    const int nCta = prog.numBits - W;
    for (int i = 0; i < nCta; i++) t |= (uint64_t) ((cta >> i) & 1u) << prog.ctaPos[i];
    return t;
}

// Global index of element j for a thread whose own address bits are gt and
// whose register bits have the address-bit values rb (any layout).
__device__ __forceinline__ uint64_t jIdx(uint64_t gt, const uint64_t (&rb)[kRegBits], int j) {
    return gt | ((j & 1) ? rb[0] : 0ULL) | ((j & 2) ? rb[1] : 0ULL) | ((j & 4) ? rb[2] : 0ULL) | ((j & 8) ? rb[3] : 0ULL);
}

// In-register initial state / lazy collapse for elements whose global
// indices are given by (gt, rb).
template <int INIT, bool RESTRICT, class V>
__device__ __forceinline__ void jFixup(const TileProgram &prog, uint64_t gt, const uint64_t (&rb)[kRegBits],
                                       V (&a)[kRegs]) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const uint64_t g = jIdx(gt, rb, j);
        V v = a[j];
        if (INIT == INIT_CLASSICAL) {
            v = DGQJ_MK((DGQJ_R) (g == prog.initIndex ? 1.0 : 0.0), (DGQJ_R) 0);
        } else if (INIT == INIT_PLUS) {
            v = DGQJ_MK((DGQJ_R) ((g >> prog.numReal) == 0ULL ? prog.initAmp : 0.0), (DGQJ_R) 0);
        } else if (INIT == INIT_BLANK) {
            v = DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        if (RESTRICT) {
            const bool keep = (g & prog.restrictMask) == prog.restrictValue;
            const DGQJ_R sc = (DGQJ_R) prog.restrictScale;
            v = keep ? DGQJ_MK(v.x * sc, v.y * sc) : DGQJ_MK((DGQJ_R) 0, (DGQJ_R) 0);
        }
        a[j] = v;
    }
}

__device__ __forceinline__ void jCpAsync16(void *smemPtr, const void *gptr) {
    const uint32_t s = (uint32_t) __cvta_generic_to_shared(smemPtr);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gptr) : "memory");
}
__device__ __forceinline__ void jCpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void jCpAsyncWait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void jCpAsyncWait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// cp.async of tile `cta`'s canonical elements into buffer buf
template <int W, class V>
__device__ __forceinline__ void jPrefetch(const V *__restrict__ st, const TileProgram &prog, uint32_t tid,
                                          uint32_t cta, V *buf) {
    constexpr uint32_t T = 1u << (W - kRegBits);
    const uint64_t base = jBase<W>(prog, tid, cta);
#pragma unroll
    for (int j = 0; j < kRegs; j++) jCpAsync16(&buf[swz(tid + T * (uint32_t) j)], st + jIndex<W>(prog, base, j));
}

template <int W, class V>
__device__ __forceinline__ void jToSmem(V *sm, uint32_t tid, const V (&a)[kRegs]) {
    constexpr uint32_t T = 1u << (W - kRegBits);
#pragma unroll
    for (int j = 0; j < kRegs; j++) sm[swz(tid + T * (uint32_t) j)] = a[j];
}

template <int W, class V>
__device__ __forceinline__ void jFromSmem(const V *sm, uint32_t tid, V (&a)[kRegs]) {
    constexpr uint32_t T = 1u << (W - kRegBits);
#pragma unroll
    for (int j = 0; j < kRegs; j++) a[j] = sm[swz(tid + T * (uint32_t) j)];
}

}  // namespace dgq
