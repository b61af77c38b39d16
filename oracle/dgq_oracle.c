/*
 * dgq_oracle.c -- CPU restatement of dgQuEST's state-vector gate semantics.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle: tests/, the smoke check
 * and the CPU-baseline leg of bench.py use it as the checker or as the timed
 * CPU baseline. The product library never links, loads or calls it.
 *
 * What it restates (citations are into the dgQuEST sources):
 *   - API call -> gate encoding: src/cpp/QuEST_distributed.cpp:118-364
 *     (rotations store angle*0.5 at :172,:213,:222,:267,:300,:309; diagonal
 *     gates carry their qubits in the control mask; controlledNot is Pauli-X
 *     with a control, :271-277).
 *   - per-gate register math of the fused kernel:
 *     src/cpp/QuEST_gpu_kernel.cu:17-170 (one function below per formula),
 *     with sin/cos of the stored angle taken on the host as at :461-468.
 *   - the Sq{X,Y,W} matrices: src/QuEST.c:373-416 (Inv_sqrt2 = 1/sqrt(2)).
 *   - the measurement rule: src/QuEST_common.c:97-115 (outcome = real1 > P0,
 *     short-circuited within REAL_EPS = 1e-13 of 0 or 1), seeding
 *     src/QuEST_common.c:147-152, and MT19937 (init_genrand, init_by_array,
 *     genrand_int32, genrand_real1) as used by src/mt19937ar.c:61-154.
 *     measure/collapse itself has no body in dgQuEST (QuEST.h:1289 is only a
 *     prototype); the collapse follows QuEST's documented semantics: zero the
 *     other outcome and rescale by 1/sqrt(P(outcome)).
 *   - multiQubitUnitary is not declared in dgQuEST; it follows QuEST's
 *     documented semantics (targs[0] is the least significant matrix bit).
 *
 * The oracle applies gates one at a time in call order. dgQuEST's DAG merges
 * (src/cpp/DAG.cpp:155-195) change results only at rounding level, so the
 * oracle does not merge. OpenMP parallelises the amplitude loops; results do
 * not depend on the thread count except in the probability sums.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dgq_ops.h"

#define ORC_RSQRT2 0.7071067811865475244008443621
#define ORC_REAL_EPS 1e-13

/* ---------------------------------------------------------------------- */
/* MT19937 (Matsumoto & Nishimura 1998, init_by_array revision 2002).      */
/* Restated from the published algorithm; state is per oracle instance.    */
/* ---------------------------------------------------------------------- */
#define MT_N 624
#define MT_M 397

typedef struct {
    uint32_t mt[MT_N];
    int mti;
} orc_mt;

static void mt_seed(orc_mt *g, uint32_t s) {
    g->mt[0] = s;
    for (int i = 1; i < MT_N; i++) {
        uint32_t prev = g->mt[i - 1];
        g->mt[i] = 1812433253u * (prev ^ (prev >> 30)) + (uint32_t) i;
    }
    g->mti = MT_N;
}

static void mt_seed_array(orc_mt *g, const unsigned long *key, int len) {
    mt_seed(g, 19650218u);
    int i = 1, j = 0;
    for (int k = (MT_N > len ? MT_N : len); k > 0; k--) {
        uint32_t prev = g->mt[i - 1];
        g->mt[i] = (g->mt[i] ^ ((prev ^ (prev >> 30)) * 1664525u)) + (uint32_t) key[j] + (uint32_t) j;
        i++;
        j++;
        if (i >= MT_N) {
            g->mt[0] = g->mt[MT_N - 1];
            i = 1;
        }
        if (j >= len) j = 0;
    }
    for (int k = MT_N - 1; k > 0; k--) {
        uint32_t prev = g->mt[i - 1];
        g->mt[i] = (g->mt[i] ^ ((prev ^ (prev >> 30)) * 1566083941u)) - (uint32_t) i;
        i++;
        if (i >= MT_N) {
            g->mt[0] = g->mt[MT_N - 1];
            i = 1;
        }
    }
    g->mt[0] = 0x80000000u;
}

static uint32_t mt_next(orc_mt *g) {
    if (g->mti >= MT_N) {
        for (int k = 0; k < MT_N; k++) {
            uint32_t y = (g->mt[k] & 0x80000000u) | (g->mt[(k + 1) % MT_N] & 0x7fffffffu);
            g->mt[k] = g->mt[(k + MT_M) % MT_N] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->mti = 0;
    }
    uint32_t y = g->mt[g->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* uniform on the closed interval [0,1]: the 32-bit draw divided by 2^32-1 */
static double mt_real1(orc_mt *g) {
    return (double) mt_next(g) * (1.0 / 4294967295.0);
}

/* ---------------------------------------------------------------------- */
/* State                                                                   */
/* ---------------------------------------------------------------------- */
typedef struct orc_state {
    int n;
    uint64_t numAmps;
    double *amp; /* interleaved (re, im), numAmps pairs */
    orc_mt rng;
} orc_state;

orc_state *orc_create(int numQubits) {
    if (numQubits <= 0 || numQubits > 40) return NULL;
    orc_state *s = (orc_state *) calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->n = numQubits;
    s->numAmps = 1ULL << numQubits;
    s->amp = (double *) malloc(sizeof(double) * 2 * s->numAmps);
    if (!s->amp) {
        free(s);
        return NULL;
    }
    mt_seed(&s->rng, 5489u);
    return s;
}

void orc_destroy(orc_state *s) {
    if (!s) return;
    free(s->amp);
    free(s);
}

int orc_num_qubits(const orc_state *s) { return s->n; }
double *orc_amps(orc_state *s) { return s->amp; }

void orc_init_zero(orc_state *s) {
    const int64_t N = (int64_t) s->numAmps;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        s->amp[2 * i] = 0.0;
        s->amp[2 * i + 1] = 0.0;
    }
    s->amp[0] = 1.0;
}

void orc_init_classical(orc_state *s, uint64_t index) {
    orc_init_zero(s);
    s->amp[0] = 0.0;
    s->amp[2 * index] = 1.0;
}

void orc_init_plus(orc_state *s) {
    const int64_t N = (int64_t) s->numAmps;
    const double f = 1.0 / sqrt((double) N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        s->amp[2 * i] = f;
        s->amp[2 * i + 1] = 0.0;
    }
}

void orc_set_amps(orc_state *s, const double *re, const double *im) {
    const int64_t N = (int64_t) s->numAmps;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        s->amp[2 * i] = re[i];
        s->amp[2 * i + 1] = im[i];
    }
}

void orc_seed(orc_state *s, const unsigned long *keys, int numKeys) {
    mt_seed_array(&s->rng, keys, numKeys);
}

/* ---------------------------------------------------------------------- */
/* Gate math (QuEST_gpu_kernel.cu:17-170)                                  */
/* ---------------------------------------------------------------------- */
enum {
    K_Z, K_S, K_SCONJ, K_T, K_TCONJ, K_PHASE,    /* diagonal, on control match */
    K_RZ, K_X, K_Y, K_YCONJ, K_H, K_RX, K_RY,    /* pair ops                   */
    K_COMPACT, K_UNITARY
};

typedef struct {
    double c, s;          /* cos/sin of the stored angle */
    double ar, ai, br, bi; /* compact pair                */
    double u[8];          /* 2x2 row-major re/im          */
} gate_par;

static inline void diag_apply(int kind, double *re, double *im, const gate_par *p) {
    const double r = *re, i = *im;
    switch (kind) {
        case K_Z: *re = -r; *im = -i; break;                                 /* :17-22  */
        case K_S: *re = -i; *im = r; break;                                  /* :24-29  */
        case K_SCONJ: *re = i; *im = -r; break;                              /* :31-36  */
        case K_T: *re = ORC_RSQRT2 * (r - i); *im = ORC_RSQRT2 * (i + r); break;  /* :38-43 */
        case K_TCONJ: *re = ORC_RSQRT2 * (r + i); *im = ORC_RSQRT2 * (i - r); break; /* :45-50 */
        case K_PHASE: *re = p->c * r - p->s * i; *im = p->c * i + p->s * r; break;   /* :66-71 */
        default: break;
    }
}

static inline void pair_apply(int kind, double *r0, double *i0, double *r1, double *i1, const gate_par *p) {
    const double a = *r0, b = *i0, c = *r1, d = *i1;
    switch (kind) {
        case K_RZ: /* :73-82 */
            *r0 = p->c * a + p->s * b;
            *i0 = p->c * b - p->s * a;
            *r1 = p->c * c - p->s * d;
            *i1 = p->c * d + p->s * c;
            break;
        case K_X: /* :84-93 */
            *r0 = c; *i0 = d; *r1 = a; *i1 = b;
            break;
        case K_Y: /* :95-104 */
            *r0 = d; *i0 = -c; *r1 = -b; *i1 = a;
            break;
        case K_YCONJ: /* :106-115 */
            *r0 = -d; *i0 = c; *r1 = b; *i1 = -a;
            break;
        case K_H: /* :117-126 */
            *r0 = ORC_RSQRT2 * (a + c);
            *i0 = ORC_RSQRT2 * (b + d);
            *r1 = ORC_RSQRT2 * (a - c);
            *i1 = ORC_RSQRT2 * (b - d);
            break;
        case K_RX: /* :128-137 */
            *r0 = p->c * a + p->s * d;
            *i0 = p->c * b - p->s * c;
            *r1 = p->c * c + p->s * b;
            *i1 = p->c * d - p->s * a;
            break;
        case K_RY: /* :139-148 */
            *r0 = p->c * a - p->s * c;
            *i0 = p->c * b - p->s * d;
            *r1 = p->s * a + p->c * c;
            *i1 = p->s * b + p->c * d;
            break;
        case K_COMPACT: /* :150-159 */
            *r0 = p->ar * a - p->ai * b - p->br * c - p->bi * d;
            *i0 = p->ar * b + p->ai * a - p->br * d + p->bi * c;
            *r1 = p->br * a - p->bi * b + p->ar * c + p->ai * d;
            *i1 = p->br * b + p->bi * a + p->ar * d - p->ai * c;
            break;
        case K_UNITARY: { /* :161-170 */
            const double *u = p->u;
            *r0 = u[0] * a - u[1] * b + u[2] * c - u[3] * d;
            *i0 = u[0] * b + u[1] * a + u[2] * d + u[3] * c;
            *r1 = u[4] * a - u[5] * b + u[6] * c - u[7] * d;
            *i1 = u[4] * b + u[5] * a + u[6] * d + u[7] * c;
            break;
        }
        default: break;
    }
}

/* diagonal gate on every amplitude whose index has all bits of ctrl set */
static void apply_diag(orc_state *s, int kind, uint64_t ctrl, const gate_par *p) {
    const int64_t N = (int64_t) s->numAmps;
    double *A = s->amp;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        if (((uint64_t) i & ctrl) == ctrl) diag_apply(kind, &A[2 * i], &A[2 * i + 1], p);
    }
}

/* pair gate on target t for every pair whose index has all bits of ctrl set */
static void apply_pair(orc_state *s, int kind, int t, uint64_t ctrl, const gate_par *p) {
    const int64_t half = (int64_t) (s->numAmps >> 1);
    const uint64_t tm = 1ULL << t;
    double *A = s->amp;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < half; k++) {
        const uint64_t i0 = (((uint64_t) k & ~(tm - 1)) << 1) | ((uint64_t) k & (tm - 1));
        if ((i0 & ctrl) != ctrl) continue;
        const uint64_t i1 = i0 | tm;
        pair_apply(kind, &A[2 * i0], &A[2 * i0 + 1], &A[2 * i1], &A[2 * i1 + 1], p);
    }
}

static void set_angle(gate_par *p, double storedAngle) {
    p->c = cos(storedAngle);
    p->s = sin(storedAngle);
}

static void set_unitary(gate_par *p, const double *u8) {
    memcpy(p->u, u8, sizeof(double) * 8);
}

/* ---------------------------------------------------------------------- */
/* Probabilities and measurement                                           */
/* ---------------------------------------------------------------------- */
double orc_prob_zero(const orc_state *s, int q) {
    const int64_t N = (int64_t) s->numAmps;
    const uint64_t m = 1ULL << q;
    const double *A = s->amp;
    double sum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sum)
    for (int64_t i = 0; i < N; i++) {
        if (((uint64_t) i & m) == 0) sum += A[2 * i] * A[2 * i] + A[2 * i + 1] * A[2 * i + 1];
    }
    return sum;
}

void orc_prob_zero_all(const orc_state *s, double *out) {
    for (int q = 0; q < s->n; q++) out[q] = orc_prob_zero(s, q);
}

double orc_total_prob(const orc_state *s) {
    const int64_t N = (int64_t) s->numAmps;
    const double *A = s->amp;
    double sum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sum)
    for (int64_t i = 0; i < N; i++) sum += A[2 * i] * A[2 * i] + A[2 * i + 1] * A[2 * i + 1];
    return sum;
}

/* QuEST_common.c:97-115 */
static int outcome_from_prob(orc_state *s, double zeroProb, double *outcomeProb) {
    int outcome;
    if (zeroProb < ORC_REAL_EPS)
        outcome = 1;
    else if (1 - zeroProb < ORC_REAL_EPS)
        outcome = 0;
    else
        outcome = (mt_real1(&s->rng) > zeroProb);
    *outcomeProb = outcome == 0 ? zeroProb : 1 - zeroProb;
    return outcome;
}

void orc_collapse(orc_state *s, int q, int outcome, double outcomeProb) {
    const int64_t N = (int64_t) s->numAmps;
    const uint64_t m = 1ULL << q;
    const uint64_t want = outcome ? m : 0;
    const double f = 1.0 / sqrt(outcomeProb);
    double *A = s->amp;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        if (((uint64_t) i & m) == want) {
            A[2 * i] *= f;
            A[2 * i + 1] *= f;
        } else {
            A[2 * i] = 0.0;
            A[2 * i + 1] = 0.0;
        }
    }
}

int orc_measure(orc_state *s, int q, double *outcomeProbOut) {
    double p0 = orc_prob_zero(s, q);
    double op;
    int outcome = outcome_from_prob(s, p0, &op);
    orc_collapse(s, q, outcome, op);
    if (outcomeProbOut) *outcomeProbOut = op;
    return outcome;
}

/* ---------------------------------------------------------------------- */
/* multiQubitUnitary (QuEST semantics; no dgQuEST counterpart)             */
/* u is row-major 2^k x 2^k, re and im separate                           */
/* ---------------------------------------------------------------------- */
void orc_multi_qubit_unitary(orc_state *s, const int *targs, int k, const double *ure, const double *uim) {
    const int64_t dim = 1LL << k;
    uint64_t tmask = 0;
    for (int j = 0; j < k; j++) tmask |= 1ULL << targs[j];
    const int64_t groups = (int64_t) (s->numAmps >> k);
    double *A = s->amp;
#pragma omp parallel
    {
        double *vr = (double *) malloc(sizeof(double) * dim);
        double *vi = (double *) malloc(sizeof(double) * dim);
        uint64_t *idx = (uint64_t *) malloc(sizeof(uint64_t) * dim);
#pragma omp for schedule(static)
        for (int64_t g = 0; g < groups; g++) {
            /* deposit g into the non-target bits */
            uint64_t base = 0, rem = (uint64_t) g;
            for (int b = 0; b < s->n; b++) {
                if (tmask & (1ULL << b)) continue;
                base |= (rem & 1ULL) << b;
                rem >>= 1;
            }
            for (int64_t r = 0; r < dim; r++) {
                uint64_t ii = base;
                for (int j = 0; j < k; j++) ii |= (((uint64_t) r >> j) & 1ULL) << targs[j];
                idx[r] = ii;
                vr[r] = A[2 * ii];
                vi[r] = A[2 * ii + 1];
            }
            for (int64_t r = 0; r < dim; r++) {
                double sr = 0.0, si = 0.0;
                for (int64_t c = 0; c < dim; c++) {
                    const double mr = ure[r * dim + c], mi = uim[r * dim + c];
                    sr += mr * vr[c] - mi * vi[c];
                    si += mr * vi[c] + mi * vr[c];
                }
                A[2 * idx[r]] = sr;
                A[2 * idx[r] + 1] = si;
            }
        }
        free(vr);
        free(vi);
        free(idx);
    }
}

/* ---------------------------------------------------------------------- */
/* One API call (QuEST_distributed.cpp:118-364; QuEST.c:93-423)             */
/* Returns the measurement outcome for DGQ_OP_MEASURE, else 0; -1 if the    */
/* op kind is unknown.                                                      */
/* ---------------------------------------------------------------------- */
int orc_apply_op(orc_state *s, const dgq_op *op) {
    gate_par p;
    memset(&p, 0, sizeof(p));
    const uint64_t m0 = 1ULL << op->q0;
    const uint64_t m1 = 1ULL << op->q1;
    const double inv_sqrt2 = 1 / sqrt(2); /* QuEST.c:376 */
    switch (op->kind) {
        case DGQ_OP_H: apply_pair(s, K_H, op->q0, 0, &p); break;
        case DGQ_OP_X: apply_pair(s, K_X, op->q0, 0, &p); break;
        case DGQ_OP_Y: apply_pair(s, K_Y, op->q0, 0, &p); break;
        case DGQ_OP_Z: apply_diag(s, K_Z, m0, &p); break;
        case DGQ_OP_S: apply_diag(s, K_S, m0, &p); break;
        case DGQ_OP_T: apply_diag(s, K_T, m0, &p); break;
        case DGQ_OP_RX: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RX, op->q0, 0, &p); break;
        case DGQ_OP_RY: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RY, op->q0, 0, &p); break;
        case DGQ_OP_RZ: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RZ, op->q0, 0, &p); break;
        case DGQ_OP_PHASE: set_angle(&p, op->p[0]); apply_diag(s, K_PHASE, m0, &p); break;
        case DGQ_OP_CNOT: apply_pair(s, K_X, op->q1, m0, &p); break;
        case DGQ_OP_CY: apply_pair(s, K_Y, op->q1, m0, &p); break;
        case DGQ_OP_CZ: apply_diag(s, K_Z, m0 | m1, &p); break;
        case DGQ_OP_CPHASE: set_angle(&p, op->p[0]); apply_diag(s, K_PHASE, m0 | m1, &p); break;
        case DGQ_OP_CRX: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RX, op->q1, m0, &p); break;
        case DGQ_OP_CRY: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RY, op->q1, m0, &p); break;
        case DGQ_OP_CRZ: set_angle(&p, op->p[0] * 0.5); apply_pair(s, K_RZ, op->q1, m0, &p); break;
        case DGQ_OP_COMPACT:
            p.ar = op->p[0]; p.ai = op->p[1]; p.br = op->p[2]; p.bi = op->p[3];
            apply_pair(s, K_COMPACT, op->q0, 0, &p);
            break;
        case DGQ_OP_CCOMPACT:
            p.ar = op->p[0]; p.ai = op->p[1]; p.br = op->p[2]; p.bi = op->p[3];
            apply_pair(s, K_COMPACT, op->q1, m0, &p);
            break;
        case DGQ_OP_UNITARY: set_unitary(&p, op->p); apply_pair(s, K_UNITARY, op->q0, 0, &p); break;
        case DGQ_OP_CUNITARY: set_unitary(&p, op->p); apply_pair(s, K_UNITARY, op->q1, m0, &p); break;
        case DGQ_OP_SQX: { /* QuEST.c:373-386 */
            const double u[8] = {inv_sqrt2, 0.0, 0.0, -inv_sqrt2, 0.0, -inv_sqrt2, inv_sqrt2, 0.0};
            set_unitary(&p, u);
            apply_pair(s, K_UNITARY, op->q0, 0, &p);
            break;
        }
        case DGQ_OP_SQY: { /* QuEST.c:388-401 */
            const double u[8] = {inv_sqrt2, 0.0, -inv_sqrt2, 0.0, inv_sqrt2, 0.0, inv_sqrt2, 0.0};
            set_unitary(&p, u);
            apply_pair(s, K_UNITARY, op->q0, 0, &p);
            break;
        }
        case DGQ_OP_SQW: { /* QuEST.c:403-416 */
            const double u[8] = {inv_sqrt2, 0.0, -0.5, -0.5, 0.5, -0.5, inv_sqrt2, 0.0};
            set_unitary(&p, u);
            apply_pair(s, K_UNITARY, op->q0, 0, &p);
            break;
        }
        case DGQ_OP_SWAP: {
            /* exchange |..1_a..0_b..> and |..0_a..1_b..>; the reference has
             * no swapGate, its harness feeds it three CNOTs, which permute the
             * same amplitudes exactly. */
            if (op->q0 == op->q1) break;
            const int64_t N = (int64_t) s->numAmps;
            double *A = s->amp;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; i++) {
                const uint64_t u = (uint64_t) i;
                if ((u & m0) && !(u & m1)) {
                    const uint64_t j = (u & ~m0) | m1;
                    const double tr = A[2 * u], ti = A[2 * u + 1];
                    A[2 * u] = A[2 * j];
                    A[2 * u + 1] = A[2 * j + 1];
                    A[2 * j] = tr;
                    A[2 * j + 1] = ti;
                }
            }
            break;
        }
        case DGQ_OP_MEASURE: return orc_measure(s, op->q0, NULL);
        default: return -1;
    }
    return 0;
}

/* Applies a whole op list; measurement outcomes go to outcomes[] in order
 * (may be NULL). Returns the number of ops applied, or -(i+1) on a bad op i. */
int64_t orc_apply_ops(orc_state *s, const dgq_op *ops, int64_t count, int *outcomes) {
    int64_t nm = 0;
    for (int64_t i = 0; i < count; i++) {
        int r = orc_apply_op(s, &ops[i]);
        if (r < 0) return -(i + 1);
        if (ops[i].kind == DGQ_OP_MEASURE && outcomes) outcomes[nm++] = r;
    }
    return count;
}

/* MT19937 helpers exposed for the tests (known-answer sequence). */
void orc_mt_first_outputs(const unsigned long *keys, int numKeys, uint32_t *out, int count) {
    orc_mt g;
    mt_seed_array(&g, keys, numKeys);
    for (int i = 0; i < count; i++) out[i] = mt_next(&g);
}

void orc_mt_first_outputs_seed(uint32_t seed, uint32_t *out, int count) {
    orc_mt g;
    mt_seed(&g, seed);
    for (int i = 0; i < count; i++) out[i] = mt_next(&g);
}

/* Threads the OpenMP loops use from now on (the CPU baseline times the
 * oracle on all host cores and on one). */
void orc_set_threads(int n) {
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    if (n > 0) omp_set_num_threads(n);
#else
    (void) n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
