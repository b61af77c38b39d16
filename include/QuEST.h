/*
 * QuEST.h -- the C ABI of libdgq (dgquest_b200), a B200-native state-vector
 * simulator that is a drop-in for dgQuEST's gate-application path.
 *
 * Type layouts and function signatures match dgQuEST's include/QuEST.h so
 * that programs written against it (e.g. the C programs in its testcases directory) compile and link
 * unchanged; each declaration cites the dgQuEST prototype it replaces.
 * Note that Qureg carries u64 qubit counts, as dgQuEST's header does
 * (include/QuEST.h:88-104), not int as in upstream QuEST.
 *
 * Precision: qreal is double (dgQuEST supports only QuEST_PREC 2,
 * include/QuEST_precision.h:41). The complex64 tensor-core form is an
 * extension declared in dgq.h.
 *
 * Execution model (as in dgQuEST): gate calls only record; getAmp,
 * calcProbOfOutcome, measure and the other read-outs run everything that is
 * pending on the GPU. Invalid arguments print QuEST's message and exit with
 * its error code (src/QuEST_validation.c:82-91) unless dgq_setErrorMode()
 * selects status recording (dgq.h).
 */
#ifndef DGQ_QUEST_H
#define DGQ_QUEST_H

#ifdef __cplusplus
extern "C" {
#endif

#define QuEST_PREC 2
typedef double qreal;
#define REAL_EPS 1e-13

typedef unsigned long long u64;

/* include/QuEST.h:58-62 */
typedef struct Complex {
    qreal real;
    qreal imag;
} Complex;

/* include/QuEST.h:66-72 */
typedef struct ComplexMatrix2 {
    Complex r0c0, r0c1;
    Complex r1c0, r1c1;
} ComplexMatrix2;

/* include/QuEST.h:76-80 */
typedef struct Vector {
    qreal x, y, z;
} Vector;

/* include/QuEST.h:79-82 */
typedef struct {
    struct QuESTEnvValue *value;
    int rank;
} QuESTEnv;

/* include/QuEST.h:88-104 */
typedef struct Qureg {
    int isDensityMatrix;
    u64 numQubitsRepresented;
    u64 numQubitsInStateVec;
    u64 numAmpsTotal;
    QuESTEnv env;
    struct QuregState *state;
} Qureg;

/* Extension (upstream QuEST's shape; dgQuEST declares no multi-qubit
 * unitary): a 2^numQubits x 2^numQubits matrix, real[r][c] + i imag[r][c]. */
typedef struct ComplexMatrixN {
    int numQubits;
    qreal **real;
    qreal **imag;
} ComplexMatrixN;

/* ---- environment ---------------------------------------------------- */
QuESTEnv createQuESTEnv(void);                       /* include/QuEST.h:528 */
void destroyQuESTEnv(QuESTEnv env);                   /* include/QuEST.h:536 */
void seedQuESTDefault(void);                          /* include/QuEST.h:1317 */
void seedQuEST(unsigned long int *seedArray, int numSeeds); /* include/QuEST.h:1332 */
int getQuEST_PREC(void);                              /* src/QuEST.c:456-458 */

/* ---- registers -------------------------------------------------------- */
Qureg createQureg(int numQubits, QuESTEnv env);       /* include/QuEST.h:125 */
/* declared only in dgQuEST; upstream QuEST's representation: an n-qubit
 * density matrix held as the 2n-qubit vector of its elements, element
 * (row r, column c) at index r + (c << n); gates act as U rho U^dagger */
Qureg createDensityQureg(int numQubits, QuESTEnv env); /* include/QuEST.h:139 */
void searchQuregTaskPartitions(Qureg qureg, QuESTEnv env); /* include/QuEST.h:127 */
void destroyQureg(Qureg qureg, QuESTEnv env);         /* include/QuEST.h:148 */
int getNumQubits(Qureg qureg);                        /* include/QuEST.h:187 */
int getNumAmps(Qureg qureg);                          /* include/QuEST.h:191 */

/* ---- initialisation --------------------------------------------------- */
void initZeroState(Qureg qureg);                      /* include/QuEST.h:199 */
void initPlusState(Qureg qureg);                      /* include/QuEST.h:210 */
void initClassicalState(Qureg qureg, long long int stateInd); /* include/QuEST.h:220 */
void initStateFromAmps(Qureg qureg, qreal *reals, qreal *imags); /* include/QuEST.h:242 */
/* declared only in dgQuEST (no body there); state-vector semantics of upstream QuEST */
void initPureState(Qureg qureg, Qureg pure);           /* include/QuEST.h:229 */
void setAmps(Qureg qureg, long long int startInd, qreal *reals, qreal *imags, long long int numAmps); /* :257 */
void cloneQureg(Qureg targetQureg, Qureg copyQureg);  /* include/QuEST.h:267 */
void reportQuregParams(Qureg qureg);                  /* include/QuEST.h:183 */
void reportStateToScreen(Qureg qureg, QuESTEnv env, int reportRank); /* include/QuEST.h:177 */
void getEnvironmentString(QuESTEnv env, Qureg qureg, char str[200]); /* include/QuEST.h:538 */

/* ---- gates -------------------------------------------------------------- */
void phaseShift(Qureg qureg, const int targetQubit, qreal angle);                       /* :299 */
void controlledPhaseShift(Qureg qureg, const int idQubit1, const int idQubit2, qreal angle); /* :340 */
void multiControlledPhaseShift(Qureg qureg, int *controlQubits, int numControlQubits, qreal angle); /* :380 */
void controlledPhaseFlip(Qureg qureg, const int idQubit1, const int idQubit2);          /* :416 */
void multiControlledPhaseFlip(Qureg qureg, int *controlQubits, int numControlQubits);    /* :460 */
void sGate(Qureg qureg, const int targetQubit);                                          /* :489 */
void tGate(Qureg qureg, const int targetQubit);                                          /* :518 */
void compactUnitary(Qureg qureg, const int targetQubit, Complex alpha, Complex beta);     /* :638 */
void unitary(Qureg qureg, const int targetQubit, ComplexMatrix2 u);                      /* :664 */
void rotateX(Qureg qureg, const int rotQubit, qreal angle);                              /* :695 */
void rotateY(Qureg qureg, const int rotQubit, qreal angle);                              /* :726 */
void rotateZ(Qureg qureg, const int rotQubit, qreal angle);                              /* :757 */
void rotateAroundAxis(Qureg qureg, const int rotQubit, qreal angle, Vector axis);        /* :773 */
void controlledRotateX(Qureg qureg, const int controlQubit, const int targetQubit, qreal angle); /* :805 */
void controlledRotateY(Qureg qureg, const int controlQubit, const int targetQubit, qreal angle); /* :836 */
void controlledRotateZ(Qureg qureg, const int controlQubit, const int targetQubit, qreal angle); /* :867 */
void controlledRotateAroundAxis(Qureg qureg, const int controlQubit, const int targetQubit, qreal angle, Vector axis); /* :903 */
void controlledCompactUnitary(Qureg qureg, const int controlQubit, const int targetQubit, Complex alpha, Complex beta); /* :947 */
void controlledUnitary(Qureg qureg, const int controlQubit, const int targetQubit, ComplexMatrix2 u); /* :989 */
void multiControlledUnitary(Qureg qureg, int *controlQubits, const int numControlQubits, const int targetQubit, ComplexMatrix2 u); /* :1045 */
void pauliX(Qureg qureg, const int targetQubit);                                         /* :1074 */
void pauliY(Qureg qureg, const int targetQubit);                                         /* :1104 */
void pauliZ(Qureg qureg, const int targetQubit);                                         /* :1134 */
void hadamard(Qureg qureg, const int targetQubit);                                       /* :1166 */
void controlledNot(Qureg qureg, const int controlQubit, const int targetQubit);          /* :1205 */
void controlledPauliY(Qureg qureg, const int controlQubit, const int targetQubit);       /* :1246 */
void swapGate(Qureg qureg, int qb1, int qb2);                                            /* :1541 (declared only in dgQuEST) */
void u1Gate(Qureg qureg, int targetQubit, qreal lambda);                                 /* :1543, body src/QuEST.c:320-334 */
void u2Gate(Qureg qureg, int targetQubit, qreal phi, qreal lambda);                      /* :1544, body src/QuEST.c:336-352 */
void u3Gate(Qureg qureg, int targetQubit, qreal theta, qreal phi, qreal lambda);         /* :1545, body src/QuEST.c:354-371 */
void SqX(Qureg qureg, int targetQubit);                                                  /* :1546, body src/QuEST.c:373-386 */
void SqY(Qureg qureg, int targetQubit);                                                  /* :1547, body src/QuEST.c:388-401 */
void SqW(Qureg qureg, int targetQubit);                                                  /* :1548, body src/QuEST.c:403-416 */
void fSim(Qureg qureg, int targetQubit1, int targetQubit2, qreal theta, qreal phi);      /* :1549, body src/QuEST.c:418-423 */

/* Extension: dense unitary on numTargs qubits, targs[0] the least
 * significant bit of the matrix index (upstream QuEST semantics). */
void multiQubitUnitary(Qureg qureg, int *targs, int numTargs, ComplexMatrixN u);
ComplexMatrixN createComplexMatrixN(int numQubits);
void destroyComplexMatrixN(ComplexMatrixN matr);

/* ---- read-outs and measurement ----------------------------------------- */
Complex getAmp(Qureg qureg, long long int index);             /* include/QuEST.h:548 */
qreal getRealAmp(Qureg qureg, long long int index);           /* include/QuEST.h:559 */
qreal getImagAmp(Qureg qureg, long long int index);           /* include/QuEST.h:570 */
qreal getProbAmp(Qureg qureg, long long int index);           /* include/QuEST.h:580 */
qreal calcTotalProb(Qureg qureg);                             /* include/QuEST.h:602 */
qreal calcProbOfOutcome(Qureg qureg, const int measureQubit, int outcome); /* include/QuEST.h:1259 */
qreal collapseToOutcome(Qureg qureg, const int measureQubit, int outcome); /* include/QuEST.h:1277 */
int measure(Qureg qureg, int measureQubit);                   /* include/QuEST.h:1289 */
int measureWithStats(Qureg qureg, int measureQubit, qreal *outcomeProb); /* include/QuEST.h:1303 */
Complex calcInnerProduct(Qureg bra, Qureg ket);                 /* include/QuEST.h:1306 (declared only in dgQuEST) */
qreal calcFidelity(Qureg qureg, Qureg pureState);               /* include/QuEST.h:1539 (declared only in dgQuEST) */

/* ---- density matrices (declared only in dgQuEST) ------------------------ */
Complex getDensityAmp(Qureg qureg, long long int row, long long int col); /* include/QuEST.h:591 */
qreal calcPurity(Qureg qureg);                                  /* include/QuEST.h:1524 */
void applyOneQubitDephaseError(Qureg qureg, const int targetQubit, qreal prob); /* include/QuEST.h:1373 */
void applyTwoQubitDephaseError(Qureg qureg, const int qubit1, const int qubit2, qreal prob); /* :1399 */
void applyOneQubitDepolariseError(Qureg qureg, const int targetQubit, qreal prob); /* include/QuEST.h:1423 */
void applyOneQubitDampingError(Qureg qureg, const int targetQubit, qreal prob); /* include/QuEST.h:1445 */
void applyTwoQubitDepolariseError(Qureg qureg, const int qubit1, const int qubit2, qreal prob); /* :1494 */
void addDensityMatrix(Qureg combineQureg, qreal prob, Qureg otherQureg); /* include/QuEST.h:1507 */

#ifdef __cplusplus
}
#endif

#endif /* DGQ_QUEST_H */
