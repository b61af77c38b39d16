/* A plain C caller of the QuEST API, built against include/QuEST.h and
 * linked with libdgq.so only (no Python, no extensions): the drop-in check
 * for programs written against dgQuEST's header.
 *
 *   quest_dropin ghzqft N   GHZ + QFT on N qubits (H(0); CNOT(i, i+1); for
 *                           t = N-1..0: H(t), controlledPhaseShift(c, t,
 *                           pi / 2^(t-c)) for c < t; swapGate(i, N-1-i)),
 *                           then P(q=0) for every qubit and all amplitudes
 *   quest_dropin mixed N    rotations, compactUnitary, controlled gates, a
 *                           multiQubitUnitary and measure() under a fixed
 *                           seed; prints outcomes, then P(q=0) and amplitudes
 *   quest_dropin sharded N  GHZ + QFT as above on a register split into 4
 *                           shards (dgq_createShardedQureg from dgq.h, all on
 *                           the current device); the calls are unchanged
 *
 * Output: lines "p0 q value", "amp i re im", "outcome q value". */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "QuEST.h"
#include "dgq.h"

static const double kPi = 3.14159265358979323846;

static void ghz_qft(Qureg q, int n) {
    hadamard(q, 0);
    for (int i = 0; i < n - 1; i++) controlledNot(q, i, i + 1);
    for (int t = n - 1; t >= 0; t--) {
        hadamard(q, t);
        for (int c = t - 1; c >= 0; c--) controlledPhaseShift(q, c, t, kPi / pow(2.0, t - c));
    }
    for (int i = 0; i < n / 2; i++) swapGate(q, i, n - 1 - i);
}

static void mixed(Qureg q, int n) {
    for (int k = 0; k < n; k++) {
        rotateX(q, k, 0.1 + 0.37 * k);
        rotateY(q, (k + 1) % n, -0.2 + 0.11 * k);
        rotateZ(q, (k + 2) % n, 0.3 * k);
    }
    Complex a = {cos(0.4) * cos(0.9), cos(0.4) * sin(0.9)}, b = {sin(0.4) * cos(-0.3), sin(0.4) * sin(-0.3)};
    compactUnitary(q, 1, a, b);
    controlledNot(q, 0, n - 1);
    controlledPhaseShift(q, 2, 3, 0.77);
    controlledPhaseFlip(q, 1, 4);
    pauliX(q, 5);
    pauliZ(q, 6);
    /* a 3-qubit unitary: the 8 x 8 discrete Fourier matrix / sqrt 8 */
    int targs[3] = {2, 5, 7};
    ComplexMatrixN m = createComplexMatrixN(3);
    for (int r = 0; r < 8; r++)
        for (int c = 0; c < 8; c++) {
            m.real[r][c] = cos(2 * kPi * r * c / 8.0) / sqrt(8.0);
            m.imag[r][c] = sin(2 * kPi * r * c / 8.0) / sqrt(8.0);
        }
    multiQubitUnitary(q, targs, 3, m);
    destroyComplexMatrixN(m);
    for (int k = 0; k < n; k++) hadamard(q, k);
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s ghzqft|mixed N\n", argv[0]);
        return 2;
    }
    const int n = atoi(argv[2]);
    QuESTEnv env = createQuESTEnv();
    unsigned long seeds[2] = {12345, 67890};
    seedQuEST(seeds, 2);
    const int sharded = !strcmp(argv[1], "sharded");
    Qureg q = sharded ? dgq_createShardedQureg(n, env, 2, NULL, 0) : createQureg(n, env);
    initZeroState(q);
    if (!strcmp(argv[1], "ghzqft") || sharded) {
        ghz_qft(q, n);
    } else {
        mixed(q, n);
        searchQuregTaskPartitions(q, env);
        for (int k = 0; k < 3; k++) printf("outcome %d %d\n", k, measure(q, k));
        rotateY(q, 4, 0.5);
    }
    for (int k = 0; k < n; k++) printf("p0 %d %.17g\n", k, calcProbOfOutcome(q, k, 0));
    for (long long i = 0; i < (1LL << n); i++) {
        const Complex c = getAmp(q, i);
        printf("amp %lld %.17g %.17g\n", i, c.real, c.imag);
    }
    destroyQureg(q, env);
    destroyQuESTEnv(env);
    return 0;
}
