// interp.cuh -- the gate operations of the interpreting tile kernels.
//
// One KOp (tile_program.h) acts on the 16 amplitudes a thread holds in
// registers; the register bit it pairs on, its control masks and the
// offset of its coefficients come from the op record, so one compiled
// kernel runs any sweep program. Shared by the single-register tile kernel
// (kernels.cu) and the batched persistent kernel (batch.cu); V is double2
// (complex128 state) or float2 (complex64 state), coefficients are FP64 in
// the program and rounded to V's scalar type where they are used.
// Gate math follows dgQuEST's per-gate kernels (QuEST_gpu_kernel.cu:17-170).
#pragma once

#include <cuda_runtime.h>

#include "tile_program.h"

namespace dgq {

template <class V>
struct Real;
template <>
struct Real<double2> {
    typedef double T;
};
template <>
struct Real<float2> {
    typedef float T;
};
template <class V>
__device__ __forceinline__ V mk(typename Real<V>::T x, typename Real<V>::T y) {
    V v;
    v.x = x;
    v.y = y;
    return v;
}

template <int K, class V, class F>
__device__ __forceinline__ void forPairs(V (&a)[kRegs], uint32_t ctrlReg, F f) {
#pragma unroll
    for (int p = 0; p < kRegs / 2; p++) {
        const int j0 = ((p >> K) << (K + 1)) | (p & ((1 << K) - 1));
        const int j1 = j0 | (1 << K);
        if ((j0 & ctrlReg) == ctrlReg) f(a[j0], a[j1]);
    }
}

template <class V, class F>
__device__ __forceinline__ void forAll(V (&a)[kRegs], uint32_t ctrlReg, F f) {
#pragma unroll
    for (int j = 0; j < kRegs; j++) {
        if ((j & ctrlReg) == ctrlReg) f(a[j], j);
    }
}

#define DGQ_DISPATCH_K(kval, ...)       \
    switch (kval) {                     \
        case 0: {                       \
            constexpr int K = 0;        \
            __VA_ARGS__;                \
        } break;                        \
        case 1: {                       \
            constexpr int K = 1;        \
            __VA_ARGS__;                \
        } break;                        \
        case 2: {                       \
            constexpr int K = 2;        \
            __VA_ARGS__;                \
        } break;                        \
        default: {                      \
            constexpr int K = 3;        \
            __VA_ARGS__;                \
        } break;                        \
    }

template <int KK, class V>
__device__ __forceinline__ void denseApply(V (&a)[kRegs], uint32_t ctrlReg, const double *m) {
    typedef typename Real<V>::T R;
    constexpr int D = 1 << KK;
#pragma unroll
    for (int g = 0; g < (kRegs >> KK); g++) {
        const int base = g << KK;
        if ((base & ctrlReg) != ctrlReg) continue;
        V v[D];
#pragma unroll
        for (int c = 0; c < D; c++) v[c] = a[base + c];
#pragma unroll
        for (int r = 0; r < D; r++) {
            R re = 0, im = 0;
#pragma unroll
            for (int c = 0; c < D; c++) {
                const R mr = (R) m[2 * (r * D + c)], mi = (R) m[2 * (r * D + c) + 1];
                re = fma(mr, v[c].x, re);
                re = fma(-mi, v[c].y, re);
                im = fma(mr, v[c].y, im);
                im = fma(mi, v[c].x, im);
            }
            a[base + r] = mk<V>(re, im);
        }
    }
}

// DENSE = false drops the dense-op case (KOP_DENSE), whose 2^k-amplitude
// temporaries otherwise set the register budget of every other op: callers
// that know their programs hold no dense op compile without it.
// LEAN = true keeps only the kinds of rotation / CNOT / CZ circuits
// (kLeanKinds, tile_program.h): every case is a path that updates the thread's amplitudes in
// place, and fewer paths leave the compiler fewer register moves to
// reconcile after the switch.
// c: the op's own coefficients (coef + op.coef of its program).
template <class V, bool DENSE = true, bool LEAN = false>
__device__ __forceinline__ void applyOpAt(const KOp &op, const double *c, V (&a)[kRegs], uint32_t loc,
                                          uint32_t cta) {
    typedef typename Real<V>::T R;
    if ((cta & op.ctrlCta) != op.ctrlCta || (loc & op.ctrlLoc) != op.ctrlLoc) return;
    const uint32_t cr = op.ctrlReg;
    switch (op.kind) {
        case KOP_M2R:
            if constexpr (LEAN) break; {
            const R m0 = (R) c[0], m1 = (R) c[1], m2 = (R) c[2], m3 = (R) c[3];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V nx = mk<V>(m0 * x.x + m1 * y.x, m0 * x.y + m1 * y.y);
                const V ny = mk<V>(m2 * x.x + m3 * y.x, m2 * x.y + m3 * y.y);
                x = nx;
                y = ny;
            }));
            break;
        }
        case KOP_M2I:
            if constexpr (LEAN) break; {
            // [[a, i b], [i c, d]]
            const R m0 = (R) c[0], m1 = (R) c[1], m2 = (R) c[2], m3 = (R) c[3];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V nx = mk<V>(m0 * x.x - m1 * y.y, m0 * x.y + m1 * y.x);
                const V ny = mk<V>(m3 * y.x - m2 * x.y, m3 * y.y + m2 * x.x);
                x = nx;
                y = ny;
            }));
            break;
        }
        case KOP_M2C:
            if constexpr (LEAN) break; {
            const R u0 = (R) c[0], u1 = (R) c[1], u2 = (R) c[2], u3 = (R) c[3], u4 = (R) c[4], u5 = (R) c[5], u6 = (R) c[6], u7 = (R) c[7];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V nx = mk<V>(u0 * x.x - u1 * x.y + u2 * y.x - u3 * y.y,
                                                u0 * x.y + u1 * x.x + u2 * y.y + u3 * y.x);
                const V ny = mk<V>(u4 * x.x - u5 * x.y + u6 * y.x - u7 * y.y,
                                                u4 * x.y + u5 * x.x + u6 * y.y + u7 * y.x);
                x = nx;
                y = ny;
            }));
            break;
        }
        case KOP_X:
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V t = x;
                x = y;
                y = t;
            }));
            break;
        case KOP_Y:
            if constexpr (LEAN) break;
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V t = x;
                x = mk<V>(y.y, -y.x);
                y = mk<V>(-t.y, t.x);
            }));
            break;
        case KOP_YC:
            if constexpr (LEAN) break;
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, cr, [&](V &x, V &y) {
                const V t = x;
                x = mk<V>(-y.y, y.x);
                y = mk<V>(t.y, -t.x);
            }));
            break;
        case KOP_NEG:
            forAll(a, cr, [&](V &x, int) { x = mk<V>(-x.x, -x.y); });
            break;
        case KOP_MULI:
            if constexpr (LEAN) break;
            forAll(a, cr, [&](V &x, int) { x = mk<V>(-x.y, x.x); });
            break;
        case KOP_MULNI:
            if constexpr (LEAN) break;
            forAll(a, cr, [&](V &x, int) { x = mk<V>(x.y, -x.x); });
            break;
        case KOP_PH: {
            const R cs = (R) c[0], sn = (R) c[1];
            forAll(a, cr, [&](V &x, int) { x = mk<V>(cs * x.x - sn * x.y, cs * x.y + sn * x.x); });
            break;
        }
        case KOP_Z2: {
            const R cs = (R) c[0], sn = (R) c[1];
            const bool regSel = op.code < KC_Z2T;
            const uint32_t sr = regSel ? (1u << op.k) : 0u;
            const bool thrBit = ((loc & op.selLoc) != 0u) || (op.selCta >= 0 && ((cta >> op.selCta) & 1u));
            forAll(a, cr, [&](V &x, int j) {
                const bool bit = sr ? ((j & sr) != 0u) : thrBit;
                const R s = bit ? sn : -sn;
                x = mk<V>(cs * x.x - s * x.y, cs * x.y + s * x.x);
            });
            break;
        }
        case KOP_RY1: {
            const R t = (R) c[0];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(fma(-t, y.x, x0.x), fma(-t, y.y, x0.y));
                y = mk<V>(fma(t, x0.x, y.x), fma(t, x0.y, y.y));
            }));
            break;
        }
        case KOP_RY2: {
            const R u = (R) c[0];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(fma(u, x0.x, -y.x), fma(u, x0.y, -y.y));
                y = mk<V>(fma(u, y.x, x0.x), fma(u, y.y, x0.y));
            }));
            break;
        }
        case KOP_RX1: {
            const R t = (R) c[0];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(fma(t, y.y, x0.x), fma(-t, y.x, x0.y));
                y = mk<V>(fma(t, x0.y, y.x), fma(-t, x0.x, y.y));
            }));
            break;
        }
        case KOP_RX2: {
            const R u = (R) c[0];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(fma(u, x0.x, y.y), fma(u, x0.y, -y.x));
                y = mk<V>(fma(u, y.x, x0.y), fma(u, y.y, -x0.x));
            }));
            break;
        }
        case KOP_H1:
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(x0.x + y.x, x0.y + y.y);
                y = mk<V>(x0.x - y.x, x0.y - y.y);
            }));
            break;
        case KOP_PH1: {
            const R cs = (R) c[0], sn = (R) c[1];
            if (op.code == KC_PH1T) {
                const bool bit = ((loc & op.selLoc) != 0u) || (op.selCta >= 0 && ((cta >> op.selCta) & 1u));
                if (bit) forAll(a, 0u, [&](V &x, int) { x = mk<V>(cs * x.x - sn * x.y, cs * x.y + sn * x.x); });
            } else {
                // the selector bit as a compile-time mask: 8 amplitudes, no predicates
                DGQ_DISPATCH_K(op.k, forAll(a, 1u << K, [&](V &x, int) {
                    x = mk<V>(cs * x.x - sn * x.y, cs * x.y + sn * x.x);
                }));
            }
            break;
        }
        case KOP_RN1:
            if constexpr (LEAN) break; {
            const R pr = (R) c[0], pi = (R) c[1];
            DGQ_DISPATCH_K(op.k, forPairs<K>(a, 0u, [&](V &x, V &y) {
                const V x0 = x;
                x = mk<V>(fma(pr, y.x, fma(-pi, y.y, x0.x)), fma(pr, y.y, fma(pi, y.x, x0.y)));
                y = mk<V>(fma(-pr, x0.x, fma(-pi, x0.y, y.x)), fma(-pr, x0.y, fma(pi, x0.x, y.y)));
            }));
            break;
        }
        case KOP_DENSE:
            if constexpr (DENSE) {
                switch (op.k) {
                    case 1: denseApply<1>(a, cr, c); break;
                    case 2: denseApply<2>(a, cr, c); break;
                    case 3: denseApply<3>(a, cr, c); break;
                    default: denseApply<4>(a, cr, c); break;
                }
            }
            break;
        default:
            break;
    }
}

template <class V, bool DENSE = true, bool LEAN = false>
__device__ __forceinline__ void applyOp(const KOp &op, const double *coef, V (&a)[kRegs], uint32_t loc,
                                        uint32_t cta) {
    applyOpAt<V, DENSE, LEAN>(op, coef + op.coef, a, loc, cta);
}

}  // namespace dgq
