/*
 * ref_harness.cpp -- drives the reference (dgQuEST) built from its own
 * sources, to produce golden outputs for the oracle and the tests.
 *
 * TEST INFRASTRUCTURE ONLY. Built by `make -C oracle ref` (oracle/Makefile) into oracle/_ref/
 * and run on a GPU host; its outputs are committed as fixtures under
 * tests/golden/ by tests/golden/make_golden.py.
 *
 * Usage: ref_harness <ops.bin> <numQubits> <out.bin> full
 *        ref_harness <ops.bin> <numQubits> <out.bin> sample <indices.bin>
 * The working directory must hold QuEST.conf ("minK maxK designatedK") and a
 * predict_data.txt (may be empty when K is designated): the reference reads
 * both from the CWD (src/cpp/QuEST_distributed.cpp:42-56,
 * src/cpp/QuEST_backend_distributed.cpp:90).
 *
 * It replays the op list through the reference's QuEST API (include/QuEST.h),
 * calls searchQuregTaskPartitions and then getAmp(q, 0), which runs every
 * section as the reference's testcases do (testcases/GHZ_QFT-30.c:43-46),
 * and times that call. swapGate has no reference body, so a swap is fed as
 * three controlledNot calls; measure has no reference body either, so op
 * lists with measurements are rejected here.
 *
 * Output (little endian): "DGQR", int32 version=1, int32 n, int64 numAmps,
 * double seconds(getAmp), double seconds(all calcProbOfOutcome),
 * double P(q=0)[n], then for "sample" int64 index[numAmps], then
 * double (re,im)[numAmps] in the logical index order.
 * Amplitudes are read from the reference's host page table through the
 * logical->virtual mapping exactly as statevec_getAmp does
 * (src/cpp/QuEST_backend_distributed.cpp:649-663), with a page that was
 * never allocated (all-zero, OPTIMIZE_ZERO) read as zeros.
 */
#include <sys/time.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "QuEST.h"
#include "QuEST_backend.h"
#include "dgq_ops.h"

static double wall() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double) tv.tv_sec + 1e-6 * (double) tv.tv_usec;
}

static ComplexMatrix2 mat_from(const double *p) {
    ComplexMatrix2 u;
    u.r0c0 = {p[0], p[1]};
    u.r0c1 = {p[2], p[3]};
    u.r1c0 = {p[4], p[5]};
    u.r1c1 = {p[6], p[7]};
    return u;
}

static void replay(Qureg q, const dgq_op &op) {
    switch (op.kind) {
        case DGQ_OP_H: hadamard(q, op.q0); break;
        case DGQ_OP_X: pauliX(q, op.q0); break;
        case DGQ_OP_Y: pauliY(q, op.q0); break;
        case DGQ_OP_Z: pauliZ(q, op.q0); break;
        case DGQ_OP_S: sGate(q, op.q0); break;
        case DGQ_OP_T: tGate(q, op.q0); break;
        case DGQ_OP_RX: rotateX(q, op.q0, op.p[0]); break;
        case DGQ_OP_RY: rotateY(q, op.q0, op.p[0]); break;
        case DGQ_OP_RZ: rotateZ(q, op.q0, op.p[0]); break;
        case DGQ_OP_PHASE: phaseShift(q, op.q0, op.p[0]); break;
        case DGQ_OP_CNOT: controlledNot(q, op.q0, op.q1); break;
        case DGQ_OP_CY: controlledPauliY(q, op.q0, op.q1); break;
        case DGQ_OP_CZ: controlledPhaseFlip(q, op.q0, op.q1); break;
        case DGQ_OP_CPHASE: controlledPhaseShift(q, op.q0, op.q1, op.p[0]); break;
        case DGQ_OP_CRX: controlledRotateX(q, op.q0, op.q1, op.p[0]); break;
        case DGQ_OP_CRY: controlledRotateY(q, op.q0, op.q1, op.p[0]); break;
        case DGQ_OP_CRZ: controlledRotateZ(q, op.q0, op.q1, op.p[0]); break;
        case DGQ_OP_COMPACT:
            compactUnitary(q, op.q0, Complex{op.p[0], op.p[1]}, Complex{op.p[2], op.p[3]});
            break;
        case DGQ_OP_CCOMPACT:
            controlledCompactUnitary(q, op.q0, op.q1, Complex{op.p[0], op.p[1]}, Complex{op.p[2], op.p[3]});
            break;
        case DGQ_OP_UNITARY: unitary(q, op.q0, mat_from(op.p)); break;
        case DGQ_OP_CUNITARY: controlledUnitary(q, op.q0, op.q1, mat_from(op.p)); break;
        case DGQ_OP_SQX: SqX(q, op.q0); break;
        case DGQ_OP_SQY: SqY(q, op.q0); break;
        case DGQ_OP_SQW: SqW(q, op.q0); break;
        case DGQ_OP_SWAP:
            controlledNot(q, op.q0, op.q1);
            controlledNot(q, op.q1, op.q0);
            controlledNot(q, op.q0, op.q1);
            break;
        default:
            fprintf(stderr, "ref_harness: op kind %d has no reference implementation\n", op.kind);
            exit(3);
    }
}

int main(int argc, char **argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: %s ops.bin n out.bin full|sample [indices.bin]\n", argv[0]);
        return 2;
    }
    const int n = atoi(argv[2]);
    std::vector<dgq_op> ops;
    {
        FILE *f = fopen(argv[1], "rb");
        if (!f) {
            perror("ops");
            return 2;
        }
        dgq_op op;
        while (fread(&op, sizeof(op), 1, f) == 1) ops.push_back(op);
        fclose(f);
    }
    const bool full = strcmp(argv[4], "full") == 0;
    std::vector<int64_t> indices;
    if (!full) {
        if (argc < 6) return 2;
        FILE *f = fopen(argv[5], "rb");
        if (!f) {
            perror("indices");
            return 2;
        }
        int64_t v;
        while (fread(&v, sizeof(v), 1, f) == 1) indices.push_back(v);
        fclose(f);
    }

    QuESTEnv env = createQuESTEnv();
    Qureg q = createQureg(n, env);
    for (const auto &op : ops) replay(q, op);
    searchQuregTaskPartitions(q, env);

    const double t0 = wall();
    getAmp(q, 0);
    const double t1 = wall();
    std::vector<double> p0(n);
    for (int k = 0; k < n; k++) p0[k] = calcProbOfOutcome(q, k, 0);
    const double t2 = wall();

    auto *state = dynamic_cast<QuregStateDistributed *>(q.state);
    const uint64_t pageMask = state->numAmpsPerPage - 1;
    auto read_amp = [&](uint64_t logical, double &re, double &im) {
        const uint64_t v = translateIndex(logical, state->mapping[0].l2v, n);
        const qComplex *page = state->pageTable[0][v >> state->numQubitsPerPage];
        if (!page) {
            re = 0.0;
            im = 0.0;
            return;
        }
        re = page[v & pageMask].x;
        im = page[v & pageMask].y;
    };

    FILE *out = fopen(argv[3], "wb");
    if (!out) {
        perror("out");
        return 2;
    }
    const int32_t version = 1, nn = n;
    const int64_t numAmps = full ? (int64_t) (1ULL << n) : (int64_t) indices.size();
    const double tg = t1 - t0, tp = t2 - t1;
    fwrite("DGQR", 1, 4, out);
    fwrite(&version, 4, 1, out);
    fwrite(&nn, 4, 1, out);
    fwrite(&numAmps, 8, 1, out);
    fwrite(&tg, 8, 1, out);
    fwrite(&tp, 8, 1, out);
    fwrite(p0.data(), 8, (size_t) n, out);
    if (!full) fwrite(indices.data(), 8, indices.size(), out);
    std::vector<double> buf;
    buf.reserve(2 * 65536);
    for (int64_t i = 0; i < numAmps; i++) {
        double re, im;
        read_amp(full ? (uint64_t) i : (uint64_t) indices[i], re, im);
        buf.push_back(re);
        buf.push_back(im);
        if (buf.size() >= 2 * 65536) {
            fwrite(buf.data(), 8, buf.size(), out);
            buf.clear();
        }
    }
    fwrite(buf.data(), 8, buf.size(), out);
    fclose(out);
    fprintf(stderr, "ref_harness: n=%d getAmp %.6f s, probs %.6f s\n", n, tg, tp);
    destroyQureg(q, env);
    destroyQuESTEnv(env);
    return 0;
}
