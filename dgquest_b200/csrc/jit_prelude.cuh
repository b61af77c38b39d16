// jit_prelude.cuh -- device code shared by the runtime-specialised sweep
// kernels (jit.cpp writes one kernel per sweep program and NVRTC
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

// Sign flips on the integer pipe (standalone negations of CZ, S, Y and
// their conjugates), keeping the FP pipes for the gate arithmetic.
__device__ __forceinline__ double jFlip(double x) {
    return __longlong_as_double(__double_as_longlong(x) ^ (long long) 0x8000000000000000ULL);
}
__device__ __forceinline__ float jFlip(float x) { return __int_as_float(__float_as_int(x) ^ (int) 0x80000000); }

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
        x = DGQJ_MK(y.y, jFlip(y.x));
        y = DGQJ_MK(jFlip(t.y), t.x);
    })
}

template <int K, bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jYC(V (&a)[kRegs]) {
    DGQJ_PAIR_LOOP(K, CTRL, CR, {
        const V t = x;
        x = DGQJ_MK(jFlip(y.y), y.x);
        y = DGQJ_MK(t.y, jFlip(t.x));
    })
}

template <class V>
__device__ __forceinline__ void jPhaseMul(V &x, double csd, double snd) {
    const DGQJ_R cs = (DGQJ_R) csd, sn = (DGQJ_R) snd;
    const DGQJ_R t = sn * x.y, u = sn * x.x;
    x.x = fma(cs, x.x, -t);
    x.y = fma(cs, x.y, u);
}

// Per-thread factor of a register phase: diagonal ops whose condition
// involves only thread and CTA bits multiply every amplitude the thread
// holds by the same number, and they commute with every other op of the
// phase (those act on register bits); they are multiplied into one factor
// (a few scalar operations each) that is applied once, at the end.
__device__ __forceinline__ void jAccPhase(double2 &acc, bool on, double cs, double sn) {
    const double r = fma(acc.x, cs, -acc.y * sn), i = fma(acc.x, sn, acc.y * cs);
    acc.x = on ? r : acc.x;
    acc.y = on ? i : acc.y;
}
__device__ __forceinline__ void jAccNeg(double2 &acc, bool on) {
    acc.x = on ? -acc.x : acc.x;
    acc.y = on ? -acc.y : acc.y;
}
// times i (sign +1) or -i (sign -1)
__device__ __forceinline__ void jAccMulI(double2 &acc, bool on, double sign) {
    const double r = -sign * acc.y, i = sign * acc.x;
    acc.x = on ? r : acc.x;
    acc.y = on ? i : acc.y;
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
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(jFlip(x.x), jFlip(x.y)); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jMULI(V (&a)[kRegs]) {
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(jFlip(x.y), x.x); })
}

template <bool CTRL, uint32_t CR, class V>
__device__ __forceinline__ void jMULNI(V (&a)[kRegs]) {
    DGQJ_AMP_LOOP(CTRL, CR, { x = DGQJ_MK(x.y, jFlip(x.x)); })
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
// [[1, p], [-conj(p), 1]]
template <int K, class V>
__device__ __forceinline__ void jRN1(V (&a)[kRegs], const double *c) {
    const DGQJ_R pr = (DGQJ_R) c[0], pi = (DGQJ_R) c[1];
    DGQJ_PAIR_LOOP(K, false, 0u, {
        const V x0 = x;
        x = DGQJ_MK(fma(pr, y.x, fma(-pi, y.y, x0.x)), fma(pr, y.y, fma(pi, y.x, x0.y)));
        y = DGQJ_MK(fma(-pr, x0.x, fma(-pi, x0.y, y.x)), fma(-pr, x0.y, fma(pi, x0.x, y.y)));
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

// ============================================================ paired form
// complex64 state, address bit 0 kept inside the thread: slot j of a thread
// holds two amplitudes (address bit 0 = 0 "lo" and 1 "hi") as packed pairs
// R[j] = (re_lo, re_hi), I[j] = (im_lo, im_hi). Every op below applies the
// same arithmetic to both halves with one packed FP32 instruction
// (__ffma2_rn / __fmul2_rn / __fadd2_rn), so a thread updates 32
// amplitudes with the instruction count the complex128 kernel spends on 16.
// HI: the op is controlled on address bit 0 (only the hi halves change).
__device__ __forceinline__ float2 b2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return __fmul2_rn(a, make_float2(-1.0f, -1.0f)); }
// sign flip on the integer pipe (standalone negations: CZ, S, Y), leaving
// the FMA pipe to the arithmetic
__device__ __forceinline__ float2 flip2(float2 a) {
    return make_float2(__int_as_float(__float_as_int(a.x) ^ (int) 0x80000000),
                       __int_as_float(__float_as_int(a.y) ^ (int) 0x80000000));
}
template <bool HI>
__device__ __forceinline__ float2 keepLo(float2 old, float2 nw) {
    return HI ? make_float2(old.x, nw.y) : nw;
}

#define DGQP_PAIR_LOOP(K, CTRL, cr, ...)                                        \
    _Pragma("unroll") for (int p_ = 0; p_ < kRegs / 2; p_++) {                  \
        const int j0 = ((p_ >> (K)) << ((K) + 1)) | (p_ & ((1 << (K)) - 1));    \
        const int j1 = j0 | (1 << (K));                                         \
        if ((CTRL) && (j0 & (cr)) != (cr)) continue;                            \
        const float2 rx = R[j0], ix = I[j0], ry = R[j1], iy = I[j1];            \
        float2 nrx, nix, nry, niy;                                              \
        __VA_ARGS__                                                             \
        R[j0] = keepLo<HI>(rx, nrx);                                            \
        I[j0] = keepLo<HI>(ix, nix);                                            \
        R[j1] = keepLo<HI>(ry, nry);                                            \
        I[j1] = keepLo<HI>(iy, niy);                                            \
    }

#define DGQP_SLOT_LOOP(CTRL, cr, ...)                                           \
    _Pragma("unroll") for (int j = 0; j < kRegs; j++) {                         \
        if ((CTRL) && (j & (cr)) != (cr)) continue;                             \
        const float2 r = R[j], i = I[j];                                        \
        float2 nr, ni;                                                          \
        __VA_ARGS__                                                             \
        R[j] = keepLo<HI>(r, nr);                                               \
        I[j] = keepLo<HI>(i, ni);                                               \
    }

typedef float2 PRegs[kRegs];

// [[m0, m1], [m2, m3]] real
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pM2R(PRegs &R, PRegs &I, const double *c) {
    const float2 m0 = b2((float) c[0]), m1 = b2((float) c[1]), m2 = b2((float) c[2]), m3 = b2((float) c[3]);
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = fma2(m0, rx, mul2(m1, ry));
        nix = fma2(m0, ix, mul2(m1, iy));
        nry = fma2(m3, ry, mul2(m2, rx));
        niy = fma2(m3, iy, mul2(m2, ix));
    })
}
// [[m0, i m1], [i m2, m3]]
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pM2I(PRegs &R, PRegs &I, const double *c) {
    const float2 m0 = b2((float) c[0]), m1 = b2((float) c[1]), m2 = b2((float) c[2]), m3 = b2((float) c[3]);
    const float2 n1 = b2(-(float) c[1]), n2 = b2(-(float) c[2]);
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = fma2(m0, rx, mul2(n1, iy));
        nix = fma2(m0, ix, mul2(m1, ry));
        nry = fma2(m3, ry, mul2(n2, ix));
        niy = fma2(m3, iy, mul2(m2, rx));
    })
}
// general complex 2x2, row-major (re, im)
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pM2C(PRegs &R, PRegs &I, const double *c) {
    const float2 u0 = b2((float) c[0]), u1 = b2((float) c[1]), u2 = b2((float) c[2]), u3 = b2((float) c[3]);
    const float2 u4 = b2((float) c[4]), u5 = b2((float) c[5]), u6 = b2((float) c[6]), u7 = b2((float) c[7]);
    const float2 v1 = b2(-(float) c[1]), v3 = b2(-(float) c[3]), v5 = b2(-(float) c[5]), v7 = b2(-(float) c[7]);
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = fma2(v3, iy, fma2(u2, ry, fma2(v1, ix, mul2(u0, rx))));
        nix = fma2(u3, ry, fma2(u2, iy, fma2(u1, rx, mul2(u0, ix))));
        nry = fma2(v7, iy, fma2(u6, ry, fma2(v5, ix, mul2(u4, rx))));
        niy = fma2(u7, ry, fma2(u6, iy, fma2(u5, rx, mul2(u4, ix))));
    })
}
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pX(PRegs &R, PRegs &I) {
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = ry;
        nix = iy;
        nry = rx;
        niy = ix;
    })
}
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pY(PRegs &R, PRegs &I) {
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = iy;
        nix = flip2(ry);
        nry = flip2(ix);
        niy = rx;
    })
}
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pYC(PRegs &R, PRegs &I) {
    DGQP_PAIR_LOOP(K, CTRL, CR, {
        nrx = flip2(iy);
        nix = ry;
        nry = ix;
        niy = flip2(rx);
    })
}
// slot-wise phase (c + i s), c / s / -s given as packed pairs
__device__ __forceinline__ void pMulPhase(float2 &r, float2 &i, float2 c, float2 s, float2 ns) {
    const float2 r0 = r;
    r = fma2(c, r0, mul2(ns, i));
    i = fma2(c, i, mul2(s, r0));
}
// diag(c - i s, c + i s) selected by slot register bit K
template <int K, bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pZ2R(PRegs &R, PRegs &I, const double *cf) {
    const float2 c = b2((float) cf[0]), s = b2((float) cf[1]), ns = b2(-(float) cf[1]);
    DGQP_SLOT_LOOP(CTRL, CR, {
        nr = r;
        ni = i;
        if ((j >> K) & 1)
            pMulPhase(nr, ni, c, s, ns);
        else
            pMulPhase(nr, ni, c, ns, s);
    })
}
// phase (c + i s) on every (controlled) slot; c, s packed per half
template <bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pPH(PRegs &R, PRegs &I, float2 c, float2 s) {
    const float2 ns = mul2(s, make_float2(-1.0f, -1.0f));
    DGQP_SLOT_LOOP(CTRL, CR, {
        nr = r;
        ni = i;
        pMulPhase(nr, ni, c, s, ns);
    })
}
template <bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pNEG(PRegs &R, PRegs &I) {
    DGQP_SLOT_LOOP(CTRL, CR, {
        nr = flip2(r);
        ni = flip2(i);
    })
}
template <bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pMULI(PRegs &R, PRegs &I) {
    DGQP_SLOT_LOOP(CTRL, CR, {
        nr = flip2(i);
        ni = r;
    })
}
template <bool CTRL, uint32_t CR, bool HI>
__device__ __forceinline__ void pMULNI(PRegs &R, PRegs &I) {
    DGQP_SLOT_LOOP(CTRL, CR, {
        nr = i;
        ni = flip2(r);
    })
}
// factored uncontrolled rotations on a slot register bit
template <int K>
__device__ __forceinline__ void pRY1(PRegs &R, PRegs &I, const double *c) {
    constexpr bool HI = false;
    const float2 t = b2((float) c[0]), nt = b2(-(float) c[0]);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = fma2(nt, ry, rx);
        nix = fma2(nt, iy, ix);
        nry = fma2(t, rx, ry);
        niy = fma2(t, ix, iy);
    })
}
template <int K>
__device__ __forceinline__ void pRY2(PRegs &R, PRegs &I, const double *c) {
    constexpr bool HI = false;
    const float2 u = b2((float) c[0]);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = fma2(u, rx, neg2(ry));
        nix = fma2(u, ix, neg2(iy));
        nry = fma2(u, ry, rx);
        niy = fma2(u, iy, ix);
    })
}
template <int K>
__device__ __forceinline__ void pRX1(PRegs &R, PRegs &I, const double *c) {
    constexpr bool HI = false;
    const float2 t = b2((float) c[0]), nt = b2(-(float) c[0]);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = fma2(t, iy, rx);
        nix = fma2(nt, ry, ix);
        nry = fma2(t, ix, ry);
        niy = fma2(nt, rx, iy);
    })
}
template <int K>
__device__ __forceinline__ void pRX2(PRegs &R, PRegs &I, const double *c) {
    constexpr bool HI = false;
    const float2 u = b2((float) c[0]);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = fma2(u, rx, iy);
        nix = fma2(u, ix, neg2(ry));
        nry = fma2(u, ry, ix);
        niy = fma2(u, iy, neg2(rx));
    })
}
template <int K>
__device__ __forceinline__ void pRN1(PRegs &R, PRegs &I, const double *c) {
    constexpr bool HI = false;
    const float2 pr = b2((float) c[0]), pi = b2((float) c[1]), npr = b2(-(float) c[0]), npi = b2(-(float) c[1]);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = fma2(pr, ry, fma2(npi, iy, rx));
        nix = fma2(pr, iy, fma2(pi, ry, ix));
        nry = fma2(npr, rx, fma2(npi, ix, ry));
        niy = fma2(npr, ix, fma2(pi, rx, iy));
    })
}
template <int K>
__device__ __forceinline__ void pH1(PRegs &R, PRegs &I) {
    constexpr bool HI = false;
    const float2 m1 = make_float2(-1.0f, -1.0f);
    DGQP_PAIR_LOOP(K, false, 0u, {
        nrx = add2(rx, ry);
        nix = add2(ix, iy);
        nry = fma2(m1, ry, rx);
        niy = fma2(m1, iy, ix);
    })
}
// phase (c + i s) on the slots whose register bit K is 1
template <int K>
__device__ __forceinline__ void pPH1R(PRegs &R, PRegs &I, const double *cf) {
    const float2 c = b2((float) cf[0]), s = b2((float) cf[1]), ns = b2(-(float) cf[1]);
#pragma unroll
    for (int j = 0; j < kRegs; j++)
        if ((j >> K) & 1) pMulPhase(R[j], I[j], c, s, ns);
}
// general complex 2x2 acting inside each (controlled) slot: (lo, hi) -> M (lo, hi)
template <bool CTRL, uint32_t CR>
__device__ __forceinline__ void pInSlot(PRegs &R, PRegs &I, float m0r, float m0i, float m1r, float m1i, float m2r,
                                        float m2i, float m3r, float m3i) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        if (CTRL && (j & CR) != CR) continue;
        const float2 r = R[j], i = I[j];
        R[j] = make_float2(m0r * r.x - m0i * i.x + m1r * r.y - m1i * i.y, m2r * r.x - m2i * i.x + m3r * r.y - m3i * i.y);
        I[j] = make_float2(m0r * i.x + m0i * r.x + m1r * i.y + m1i * r.y, m2r * i.x + m2i * r.x + m3r * i.y + m3i * r.y);
    }
}
template <int KK, uint32_t CR>
__device__ __forceinline__ void pDense(PRegs &R, PRegs &I, const double *m) {
    constexpr int D = 1 << KK;
#pragma unroll
    for (int g = 0; g < (kRegs >> KK); g++) {
        const int base = g << KK;
        if ((base & CR) != CR) continue;
        float2 vr[D], vi[D];
#pragma unroll
        for (int c = 0; c < D; c++) {
            vr[c] = R[base + c];
            vi[c] = I[base + c];
        }
#pragma unroll
        for (int r = 0; r < D; r++) {
            float2 ar = b2(0.0f), ai = b2(0.0f);
#pragma unroll
            for (int c = 0; c < D; c++) {
                const float mr = (float) m[2 * (r * D + c)], mi = (float) m[2 * (r * D + c) + 1];
                ar = fma2(b2(mr), vr[c], ar);
                ar = fma2(b2(-mi), vi[c], ar);
                ai = fma2(b2(mr), vi[c], ai);
                ai = fma2(b2(mi), vr[c], ai);
            }
            R[base + r] = ar;
            I[base + r] = ai;
        }
    }
}
__device__ __forceinline__ void pGlobal(PRegs &R, PRegs &I, double grd, double gid) {
    const float2 c = b2((float) grd), s = b2((float) gid), ns = b2(-(float) gid);
#pragma unroll
    for (int j = 0; j < kRegs; j++) pMulPhase(R[j], I[j], c, s, ns);
}

// ------------------------------------------- sign-tracked paired forms
// The generator tracks which stored pairs hold negated values and passes
// its decisions as masks: CS bit 4 p + o set means output o of pair p
// (o: 0 R[j0], 1 I[j0], 2 R[j1], 3 I[j1]; pairs in register order) takes
// the coefficient's negation, FM bit 4 p + o set means that output is
// stored flipped; slot masks have bit j for slot j. The arithmetic of an
// output is fma2(+-coef, A, B) with A and B fixed per kind.
#define DGQS_PAIRS(K, CR, ...)                                                  \
    _Pragma("unroll") for (int p_ = 0; p_ < kRegs / 2; p_++) {                  \
        const int j0 = ((p_ >> (K)) << ((K) + 1)) | (p_ & ((1 << (K)) - 1));    \
        const int j1 = j0 | (1 << (K));                                         \
        if ((j0 & (CR)) != (CR)) continue;                                      \
        const float2 rx = R[j0], ix = I[j0], ry = R[j1], iy = I[j1];            \
        __VA_ARGS__                                                             \
    }
#define DGQS_C(o) ((CS >> (4 * p_ + (o))) & 1u ? n_ : c_)
#define DGQS_F(o, v) ((FM >> (4 * p_ + (o))) & 1u ? flip2(v) : (v))
template <int K, uint32_t CS>
__device__ __forceinline__ void pRY1s(PRegs &R, PRegs &I, const double *c) {
    const float2 c_ = b2((float) c[0]), n_ = b2(-(float) c[0]);
    DGQS_PAIRS(K, 0, R[j0] = fma2(DGQS_C(0), ry, rx); I[j0] = fma2(DGQS_C(1), iy, ix);
               R[j1] = fma2(DGQS_C(2), rx, ry); I[j1] = fma2(DGQS_C(3), ix, iy);)
}
template <int K, uint32_t CS>
__device__ __forceinline__ void pRY2s(PRegs &R, PRegs &I, const double *c) {
    const float2 c_ = b2((float) c[0]), n_ = b2(-(float) c[0]);
    DGQS_PAIRS(K, 0, R[j0] = fma2(DGQS_C(0), rx, ry); I[j0] = fma2(DGQS_C(1), ix, iy);
               R[j1] = fma2(DGQS_C(2), ry, rx); I[j1] = fma2(DGQS_C(3), iy, ix);)
}
template <int K, uint32_t CS>
__device__ __forceinline__ void pRX1s(PRegs &R, PRegs &I, const double *c) {
    const float2 c_ = b2((float) c[0]), n_ = b2(-(float) c[0]);
    DGQS_PAIRS(K, 0, R[j0] = fma2(DGQS_C(0), iy, rx); I[j0] = fma2(DGQS_C(1), ry, ix);
               R[j1] = fma2(DGQS_C(2), ix, ry); I[j1] = fma2(DGQS_C(3), rx, iy);)
}
template <int K, uint32_t CS>
__device__ __forceinline__ void pRX2s(PRegs &R, PRegs &I, const double *c) {
    const float2 c_ = b2((float) c[0]), n_ = b2(-(float) c[0]);
    DGQS_PAIRS(K, 0, R[j0] = fma2(DGQS_C(0), rx, iy); I[j0] = fma2(DGQS_C(1), ix, ry);
               R[j1] = fma2(DGQS_C(2), ry, ix); I[j1] = fma2(DGQS_C(3), iy, rx);)
}
// H without its 1/sqrt 2: a set CS bit subtracts A instead of adding it
template <int K, uint32_t CS>
__device__ __forceinline__ void pH1s(PRegs &R, PRegs &I) {
    const float2 m1 = b2(-1.0f);
#define DGQS_H(o, a, b) ((CS >> (4 * p_ + (o))) & 1u ? fma2(m1, (a), (b)) : add2((b), (a)))
    DGQS_PAIRS(K, 0, R[j0] = DGQS_H(0, ry, rx); I[j0] = DGQS_H(1, iy, ix);
               R[j1] = DGQS_H(2, ry, rx); I[j1] = DGQS_H(3, iy, ix);)
#undef DGQS_H
}
// pair permutations: X swaps the slots; Y and Y* also swap the components
template <int K, uint32_t CR, uint32_t FM>
__device__ __forceinline__ void pXs(PRegs &R, PRegs &I) {
    DGQS_PAIRS(K, CR, R[j0] = DGQS_F(0, ry); I[j0] = DGQS_F(1, iy); R[j1] = DGQS_F(2, rx); I[j1] = DGQS_F(3, ix);)
}
template <int K, uint32_t CR, uint32_t FM>
__device__ __forceinline__ void pYs(PRegs &R, PRegs &I) {
    DGQS_PAIRS(K, CR, R[j0] = DGQS_F(0, iy); I[j0] = DGQS_F(1, ry); R[j1] = DGQS_F(2, ix); I[j1] = DGQS_F(3, rx);)
}
// times +-i: the components swap (slot masks; FM bit 2 j + o, o: 0 R, 1 I)
template <uint32_t NEED, uint32_t FM>
__device__ __forceinline__ void pSwapRIs(PRegs &R, PRegs &I) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        if ((j & NEED) != NEED) continue;
        const float2 r = R[j], i = I[j];
        R[j] = (FM >> (2 * j)) & 1u ? flip2(i) : i;
        I[j] = (FM >> (2 * j + 1)) & 1u ? flip2(r) : r;
    }
}
// (c + i s) on the slots in SLOTS; DIFF: slots whose two pairs carry
// different signs (the cross terms take the other sign); SW: slots that
// take (c - i s) instead
template <uint32_t SLOTS, uint32_t DIFF, uint32_t SW>
__device__ __forceinline__ void pPhaseS(PRegs &R, PRegs &I, float2 c, float2 s, float2 ns) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        if (!((SLOTS >> j) & 1u)) continue;
        const bool d = (((DIFF ^ SW) >> j) & 1u) != 0;
        const float2 r = R[j];
        R[j] = fma2(c, r, mul2(d ? s : ns, I[j]));
        I[j] = fma2(c, I[j], mul2(d ? ns : s, r));
    }
}
// every slot times (gr + i gi), leaving the values with their true signs
template <uint32_t NR, uint32_t NI>
__device__ __forceinline__ void pGlobalS(PRegs &R, PRegs &I, double grd, double gid) {
    const float2 c = b2((float) grd), nc = b2(-(float) grd), s = b2((float) gid), ns = b2(-(float) gid);
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        const bool nr = (NR >> j) & 1u, ni = (NI >> j) & 1u;
        const float2 r = R[j];
        R[j] = fma2(nr ? nc : c, r, mul2(ni ? s : ns, I[j]));
        I[j] = fma2(ni ? nc : c, I[j], mul2(nr ? ns : s, r));
    }
}
// restores the true signs (integer-pipe flips)
template <uint32_t NR, uint32_t NI>
__device__ __forceinline__ void pFlushS(PRegs &R, PRegs &I) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        if ((NR >> j) & 1u) R[j] = flip2(R[j]);
        if ((NI >> j) & 1u) I[j] = flip2(I[j]);
    }
}
#undef DGQS_F
#undef DGQS_C
#undef DGQS_PAIRS
// Adds the CTA's sum of |a|^2 to *out (FP32 per thread, FP64 across threads).
__device__ __forceinline__ void pNormAccumulate(const PRegs &R, const PRegs &I, double *out) {
    __shared__ double red[32];
    float2 acc = b2(0.0f);
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        acc = fma2(R[j], R[j], acc);
        acc = fma2(I[j], I[j], acc);
    }
    double t = (double) acc.x + (double) acc.y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double u = 0.0;
        for (int w = 0; w < (int) (blockDim.x >> 5); w++) u += red[w];
        atomicAdd(out, u);
    }
}
// global I/O of one slot: amplitudes g (bit 0 clear) and g | 1 are adjacent
__device__ __forceinline__ void pLoadSlot(const float2 *__restrict__ st, uint64_t g, float2 &r, float2 &i) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(st + g));
    r = make_float2(v.x, v.z);
    i = make_float2(v.y, v.w);
}
__device__ __forceinline__ void pStoreSlot(float2 *__restrict__ st, uint64_t g, float2 r, float2 i) {
    *reinterpret_cast<float4 *>(st + g) = make_float4(r.x, i.x, r.y, i.y);
}
// initial state / lazy collapse of a slot at address g (bit 0 clear)
template <int INIT, bool RESTRICT>
__device__ __forceinline__ void pFixSlot(const TileProgram &prog, uint64_t g, float2 &r, float2 &i) {
    if (INIT == INIT_CLASSICAL) {
        r = make_float2(g == prog.initIndex ? 1.0f : 0.0f, (g | 1ULL) == prog.initIndex ? 1.0f : 0.0f);
        i = b2(0.0f);
    } else if (INIT == INIT_PLUS) {
        const float a = (float) prog.initAmp;
        r = make_float2((g >> prog.numReal) == 0ULL ? a : 0.0f, ((g | 1ULL) >> prog.numReal) == 0ULL ? a : 0.0f);
        i = b2(0.0f);
    } else if (INIT == INIT_BLANK) {
        r = b2(0.0f);
        i = b2(0.0f);
    }
    if (RESTRICT) {
        const float sc = (float) prog.restrictScale;
        const float2 k = make_float2((g & prog.restrictMask) == prog.restrictValue ? sc : 0.0f,
                                     ((g | 1ULL) & prog.restrictMask) == prog.restrictValue ? sc : 0.0f);
        r = mul2(r, k);
        i = mul2(i, k);
    }
}

}  // namespace dgq
