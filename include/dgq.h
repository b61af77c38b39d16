/*
 * dgq.h -- libdgq extensions beyond the QuEST C API (include/QuEST.h).
 *
 * None of these has a counterpart in dgQuEST unless a citation says so.
 * They cover: error-status mode, tile-width (block width) choice, the plan
 * and launch split used for device timing, plan statistics, bulk state
 * read-out, and kernel launch accounting.
 */
#ifndef DGQ_EXT_H
#define DGQ_EXT_H

#include <stdint.h>

#include "QuEST.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Precision form: a register whose 2^n amplitudes are complex64 (two
 * floats, 8 bytes each) with FP32 gate arithmetic; every QuEST call accepts
 * it. Read-outs return doubles; probabilities are accumulated in FP64.
 * Its sweeps always run runtime-specialised kernels and may use tiles of
 * 2^13 amplitudes. dgq_getPrecision returns 1 (complex64) or 2. */
Qureg dgq_createQuregF32(int numQubits, QuESTEnv env);
int dgq_getPrecision(Qureg qureg);

/* Error handling. Mode 0 (default) prints QuEST's message and exits with
 * its code, as dgQuEST does (src/QuEST_validation.c:82-91). Mode 1 records
 * the error instead: the failing call returns without effect (a zero or
 * default value where it returns one) and dgq_getLastError() reports it. */
#define DGQ_ERRORS_EXIT 0
#define DGQ_ERRORS_RECORD 1
int dgq_setErrorMode(int mode);
/* Returns the calling thread's last error code (0 = none) and clears it;
 * copies the message into msg (if msg != NULL and len > 0). Errors are
 * recorded per host thread. */
int dgq_getLastError(char *msg, int len);

/* Tile width W (address bits per CTA tile, 9..12) used for this register.
 * 0 selects it with the cost model (the recast of dgQuEST's time predictor,
 * src/cpp/time_predictor.cpp:343-395). Returns the previous setting. */
int dgq_setTileBits(Qureg qureg, int tileBits);

/* Plan statistics of the most recent execution of pending gates. */
typedef struct dgq_plan_stats {
    int32_t sweeps;        /* tile-kernel launches (state read + write passes) */
    int32_t phases;        /* register layouts over all sweeps */
    int32_t ops;           /* kernel ops over all sweeps */
    int32_t gates;         /* gates after peephole merging */
    int32_t tileBits;      /* W used */
    int32_t numBits;       /* address bits of the state buffer */
    double flopsPerAmp;    /* algorithmic FP64 flops per amplitude, whole plan */
    double planMillis;     /* host planning time (including kernel specialisation) */
    int32_t jitCompiled;   /* sweep kernels compiled for this plan */
    int32_t jitReused;     /* sweep kernels found already compiled */
    double jitMillis;      /* time spent specialising kernels */
    int64_t launchBytes;   /* host->device bytes per launch of the whole plan
                              (one sweep program per kernel parameter block) */
    int32_t streamedSweeps; /* sweeps launched while the rest of the plan was
                               still being made (their kernels were compiled) */
    int32_t denseBlocks;    /* dense fused blocks (dgq_setDenseFusion) */
    int32_t formK;          /* form of the plan: 0 register-phase tiles, K dense K-qubit blocks */
    int32_t formAuto;       /* 1 when the predictor chose the form (dgq_setDenseFusion -1) */
    double predictedTileMs; /* predictions of the form choice (0 when not made): the tile form */
    double predictedDenseMs[3]; /* and the dense-block forms with K = 5, 6, 7 */
    int32_t denseBound;     /* bit K - 5 set: the K estimate stopped counting blocks once they
                               cost more than the tile form, and is that lower bound */
} dgq_plan_stats;
int dgq_getPlanStats(Qureg qureg, dgq_plan_stats *out);

/* Stops the library's background kernel compiles (specialisation policy 1)
 * and joins their threads. Call it before the process exits (the Python
 * binding does, from its exit hook): process teardown destroys NVRTC's
 * state in an order a compile still running on another thread cannot
 * survive. Registers stay usable; later plans compile in the foreground. */
void dgq_shutdown(void);

/* Cost model of the tile-width choice (the recast of dgQuEST's time
 * predictor and its predict_data.txt calibration, time_predictor.cpp:397-476):
 * a plan costs sweepMs per sweep plus phaseMs per register phase, per 2^30
 * amplitudes. Built-in rates were fitted on B200 (2.6 and 1.8 ms);
 * dgquest_b200/calibrate.py measures them on the GPU at hand and writes a
 * cost file ("dgq_cost 1", "sweep_ms_per_2p30 x", "phase_ms_per_2p30 y"),
 * read by dgq_loadCostModel or, at the first plan, from DGQ_COST_FILE.
 * Return 0, or -1 on a bad argument or file. */
int dgq_setCostModel(double sweepMsPer2p30, double phaseMsPer2p30);
int dgq_loadCostModel(const char *path);
int dgq_getCostModel(double *sweepMsPer2p30, double *phaseMsPer2p30);
/* Rates of the dense-block forms in the form choice: ms per dense block per
 * 2^30 amplitudes for variant 0 (complex128, SIMT), 1 (complex64, SIMT) or
 * 2 (complex64, tensor cores; K = 6), K = 5..7. A cost file may carry them
 * as "dense_ms_per_2p30_<f64|c64|c64tc>_k<K> <ms>", and the complex64 tile
 * factor as "c64_tile_factor <x>". Set returns 0 or -1; get returns the
 * rate, or -1 on a bad argument. */
int dgq_setDenseCost(int variant, int K, double msPer2p30);
double dgq_getDenseCost(int variant, int K);

/* Host tier. A register whose state is larger than the device's memory (or
 * than the budget set here for registers created later, capped by free
 * HBM; 0 restores the default) keeps its state in pinned host memory in pages of
 * 2^pageBits amplitudes and streams the pages through four device buffers
 * (copy in, sweeps, copy out, overlapped on four streams). A gate on a qubit
 * outside the page first exchanges that qubit with a page qubit in a pass
 * over page pairs. Gates, read-outs and measurement work as in HBM; dense
 * sweeps (multi-qubit unitaries of more than 4 targets), sampling, inner
 * products, batches and the plan/launch split report E_UNSUPPORTED for
 * such registers. Returns the previous budget. */
int64_t dgq_setDeviceBudget(int64_t bytes);
/* 1 for a host-tier register (with its page width, page passes, qubit
 * exchanges and host<->device bytes so far; an exchange that also runs the
 * next segment counts as a pass too), 0 for a register in HBM, -1 on error. */
int dgq_getHostTierStats(Qureg qureg, int *pageBits, int64_t *passes, int64_t *exchanges, int64_t *bytesMoved);

/* Sharded registers: dgQuEST's multi-GPU state (each GPU holds a slice and an
 * MPI page exchange moves qubits between slices,
 * src/cpp/QuEST_backend_distributed.cpp:403-601) in one process. The state is
 * split into 2^shardBits shards of 2^(numQubits - shardBits) amplitudes, shard
 * k holding amplitudes [k << (numQubits - shardBits), (k + 1) << ...) in the
 * HBM of device devices[k] (NULL: every shard on the current device; several
 * shards may share a device; distinct devices need peer access, which is
 * enabled here). Pending gates run segment by segment, each segment's
 * sweeps on every shard in place; a gate on a shard-index qubit first
 * exchanges it with a qubit inside the shards, one kernel per shard pair
 * swapping half-shards through peer memory (NVLink) when the pair spans two
 * devices. Gates (multi-qubit unitaries of at most 4 targets), read-outs,
 * measurement, setAmps, initStateFromAmps and cloneQureg (between registers
 * of the same shard layout) work as in HBM; dense sweeps, sampling, inner
 * products, batches, dgq_getDeviceState and the plan/launch split report
 * E_UNSUPPORTED. single != 0 makes a complex64 register. shardBits is 1..4
 * and every shard holds at least DGQ_MIN_SHARD_QUBITS qubits. */
#define DGQ_MIN_SHARD_QUBITS 14
Qureg dgq_createShardedQureg(int numQubits, QuESTEnv env, int shardBits, const int *devices, int single);
/* 1 for a sharded register (with its shard-index bits, shard passes, qubit
 * exchanges and bytes moved between shards so far), 0 otherwise, -1 on
 * error. */
int dgq_getShardStats(Qureg qureg, int *shardBits, int64_t *passes, int64_t *exchanges, int64_t *bytesExchanged);

/* Form of a register's plans (the recast of dgQuEST's time predictor,
 * time_predictor.cpp:343-395, which takes the argmin over its block width).
 * qubits = 5, 6 or 7: the register's gates are fused into dense unitaries
 * on that many qubits (dgQuEST's greedy block rule, DAG.cpp:219-259, with
 * every qubit a gate touches counted), composed in FP64 on the host and
 * applied one per sweep as a complex GEMM over the state: on the tensor
 * cores (tcgen05, 3xTF32) for complex64 registers and 6 qubits, the SIMT
 * dense kernel otherwise. 0 runs gates in register-phase sweeps. -1 (the
 * default) lets the cost model choose per plan between the register-phase
 * tiles (and their width) and dense blocks of 5, 6 or 7 qubits; the plan
 * statistics report the choice (formK) and every prediction. Registers of
 * fewer than qubits + 2 address bits are not fused. Returns the previous
 * setting, or -2 on a bad argument. */
int dgq_setDenseFusion(Qureg qureg, int qubits);

/* Plans the pending gates (and pending initialisation / collapse) into
 * sweep programs and keeps them; dgq_launchPlanned launches them on the
 * register's stream without waiting. A kept plan can be launched again:
 * every launch recomputes the whole plan from its initial state, so it is
 * only meaningful for plans that start from an initialisation. */
int dgq_planPending(Qureg qureg);
int dgq_launchPlanned(Qureg qureg);
/* Runs everything pending and waits for the GPU. */
int dgq_sync(Qureg qureg);

/* The CUDA stream (cudaStream_t) all of this register's kernels run on. */
void *dgq_getStream(Qureg qureg);
/* Device pointer of the state buffer (interleaved re/im doubles, or floats
 * for complex64 registers) and its number of address bits (>= numQubits;
 * extra bits are always |0>). Pending gates run first, a pending collapse
 * is applied and swapGate relabels are undone in HBM, so the buffer holds
 * the state in logical index order until the next gate call. */
void *dgq_getDeviceState(Qureg qureg, int *numBits);

/* Copies all 2^n amplitudes, in logical index order, into re[] and im[]. */
int dgq_getStateVector(Qureg qureg, qreal *re, qreal *im);

/* Kernel launches issued by this library since the process started. */
int64_t dgq_getLaunchCount(void);

/* P(qubit = 0) for every qubit in one pass (the reduction behind
 * calcProbOfOutcome, src/cpp/QuEST_gpu_kernel.cu:769-807). */
int dgq_calcProbOfAllZero(Qureg qureg, qreal *probs);

/* Measures the FP64 FMA throughput of the current device (TFLOP/s, an FMA
 * counted as two flops) with a register-resident DFMA loop over all SMs. */
int dgq_measureFp64Peak(double *tflops);

/* P(address bit = 0) for every bit of a state the caller owns, computed
 * without allocating any GPU memory. No counterpart in dgQuEST: it serves
 * callers that cannot call cudaMalloc while they call this library (hosts
 * that manage all device memory themselves, such as a framework's caching
 * allocator or a server with a fixed HBM budget, where an allocation behind
 * their back can fail or fragment their pool; latency-bound loops where an
 * allocation would synchronise the device). deviceState: 2^numBits
 * interleaved complex128 amplitudes in device memory; deviceProbs:
 * numBits + 1 doubles in device memory, receiving P(bit b = 0) for
 * b < numBits and the total probability last. Both must be memory of the
 * device that is current at the call (checked; another GPU's memory is
 * rejected). stream: a cudaStream_t (NULL = default stream); results are
 * ready when the stream reaches them. The partial sums go to a static
 * device array of 16384 x 17 doubles (2.125 MiB, resident on every GPU that
 * loads the library until the process exits), so numBits is limited to
 * 1..30; larger states are rejected. The first call on each device looks up
 * that array's device address (make that first call before any stream
 * capture). Calls share the array: calls that overlap on the GPU race.
 * Returns 0, or -1 (invalid argument / too large) or -2 (CUDA error),
 * reported like every other error of this library. */
int dgq_calcProbOfAllZeroNoAlloc(const void *deviceState, int numBits, double *deviceProbs, void *stream);

/* Host-only planning (no GPU call): plans `count` gates given in dgQuEST's
 * IR encoding (type numbers of src/cpp/QuEST_backend.h:89-114, target and
 * control bit masks, operand[8] per gate with rotations carrying angle/2)
 * on a register of numQubits with tile width tileBits (0 = cost model), and
 * reports the plan. Merged gates are returned through mergedTypes (may be
 * NULL, else room for `count` entries) with *numMerged set. */
int dgq_planGates(int numQubits, int tileBits, int count, const int32_t *types, const uint64_t *targetMasks,
                  const uint64_t *controlMasks, const double *operands, dgq_plan_stats *out, int32_t *mergedTypes,
                  int32_t *numMerged);

/* Host-only view of the qubit exchanges (no GPU call): how the gates
 * (dgq_planGates encoding; only types and target masks matter) are cut into
 * segments whose non-diagonal targets lie below localQubits, by the host tier
 * (batch = 0: pages of 2^localQubits amplitudes, one exchange pass per qubit)
 * or by a sharded register (batch = 1: shards of 2^localQubits amplitudes,
 * every qubit of a boundary in one pass). Reports the segments, the exchange
 * passes and the qubits moved; returns 0, or -1 on a bad argument. */
int dgq_planExchanges(int numQubits, int localQubits, int batch, int count, const int32_t *types,
                      const uint64_t *targetMasks, int32_t *segments, int32_t *exchanges, int32_t *qubitsMoved);

/* Host-only view of the dense-block form (no GPU call): fuses the gates
 * (dgq_planGates encoding) into dense blocks of K = 1..7 qubits as
 * dgq_setDenseFusion does and applies the fused gates in FP64 on the host
 * to the state (re, im) of numQubits <= 20 qubits, in place. Returns the
 * number of dense blocks, or -1 on a bad argument. For tests of the
 * fusion; the product path applies the blocks on the GPU. */
int dgq_fuseApplyHost(int numQubits, int K, int count, const int32_t *types, const uint64_t *targetMasks,
                      const uint64_t *controlMasks, const double *operands, double *re, double *im);

/* Registers with at least minBits address bits run runtime-specialised
 * sweep kernels (default 22, or DGQ_JIT_MIN_BITS; DGQ_JIT=0 disables
 * specialisation). Negative restores the default. Returns the previous value. */
int dgq_setSpecialisationMinBits(int minBits);
/* 0 (default): plans that need specialised kernels compile them before
 * running. 1: a plan runs specialised only if its kernels are compiled
 * already; otherwise it runs the interpreting kernel while its kernels
 * compile on background host threads for later plans of the same structure
 * (for serving one-off circuits); registers of >= 32 address bits still
 * compile first. 2: as 1 without the background compiles (a stream of
 * circuits whose structures do not repeat). Returns the previous policy. */
int dgq_setSpecialisationPolicy(int policy);
/* multiQubitUnitary with 6 targets on a complex64 register of >= 12 qubits
 * runs on the tensor cores (tcgen05, 3xTF32 split, FP32 accumulation) when
 * enabled (default 1); 0 selects the SIMT dense kernel. Returns the previous
 * setting. */
int dgq_setTensorCores(int enable);
/* Nonzero when a tensor-core sweep stopped waiting for its MMAs (bounded
 * wait); its output is then invalid. Waits for the device. */
int dgq_getDeviceErrors(void);

/* Host-only view of the runtime specialisation: the CUDA source generated
 * for sweep `sweep` of the plan of the given gates (same encoding as
 * dgq_planGates; precision 1 = complex64 (the paired form where it applies),
 * 2 = complex128, 3 = complex64 in the unpaired form; returns the number
 * of sweeps, -2 if buf is too small), and
 * an NVRTC compile of such a source for sm_100a (returns the cubin size, or
 * -1 with the compiler log in `log`). Neither needs a GPU. */
int dgq_sweepSource(int numQubits, int tileBits, int count, const int32_t *types, const uint64_t *targetMasks,
                    const uint64_t *controlMasks, const double *operands, int sweep, int precision, char *buf,
                    int len);
int dgq_compileSweepSource(const char *source, char *log, int len);

/* Compiles ahead of time the specialised sweep kernels that a register of
 * numQubits and `precision` (1 complex64, 2 complex128, 3 complex64 without
 * the paired form) would use for these gates after initZeroState, so that
 * a later run of the same circuit structure finds them compiled. With
 * background = 1 the compiles are queued on the library's compile threads
 * and the call returns at once (no GPU work); with 0 they are compiled and
 * loaded for the current device before it returns. Returns the number of
 * kernels, or -1 on error. No counterpart in dgQuEST (the serving loop uses
 * it for circuit structures that recur, such as GHZ+QFT of each size). */
int dgq_specialiseGates(int numQubits, int precision, int count, const int32_t *types, const uint64_t *targetMasks,
                        const uint64_t *controlMasks, const double *operands, int background);

/* Circuit records: one 80-byte record per API call, applied in order
 * through the entry points of QuEST.h (same validation, same lazy
 * recording). kind: 0 hadamard, 1 pauliX, 2 pauliY, 3 pauliZ, 4 sGate,
 * 5 tGate, 6 rotateX, 7 rotateY, 8 rotateZ, 9 phaseShift (angle p[0]),
 * 10 controlledNot, 11 controlledPhaseFlip, 12 controlledPhaseShift,
 * 13 controlledRotateX, 14 controlledRotateY, 15 controlledRotateZ
 * (control q0, target q1, angle p[0]), 16 compactUnitary (alpha p[0..1],
 * beta p[2..3]), 17 controlledCompactUnitary (control q0, target q1),
 * 18 unitary (ComplexMatrix2 as r0c0 r0c1 r1c0 r1c1 re/im pairs in p),
 * 19 controlledUnitary, 20 SqX, 21 SqY, 22 SqW, 23 swapGate (q0, q1),
 * 24 measure (outcome appended to outcomes), 25 controlledPauliY.
 * No counterpart in dgQuEST (its callers make one API call per gate).
 * Returns the number of records applied, or -1 at the first record the
 * API rejected (error mode "record") or with an unknown kind. */
typedef struct dgq_gate_record {
    int32_t kind;
    int32_t q0, q1, q2;
    double p[8];
} dgq_gate_record;
int dgq_applyCircuit(Qureg qureg, const dgq_gate_record *records, int count, int *outcomes);

/* Draws numSamples basis states from |amp|^2 of the register (after its
 * pending gates run) and writes them as logical indices (bit q = qubit q).
 * Sample k uses the k-th 53-bit uniform u of MT19937 seeded with
 * init_genrand(seed) ((a >> 5) * 2^26 + (b >> 6) over 2^53) and is the
 * smallest address of the state buffer whose cumulative probability
 * exceeds u x total; registers without swapGate calls keep addresses in
 * logical order. The state is not changed. Deterministic for a given state
 * and seed. No counterpart in dgQuEST (its measure is single-shot and
 * unimplemented). */
int dgq_sampleOutcomes(Qureg qureg, int numSamples, uint32_t seed, uint64_t *outcomes);

/* Device bytes new registers can use on the current device: free memory
 * plus what the registers' stream-ordered pool holds unused (register
 * memory is allocated and freed in stream order, so destroyed registers'
 * states are kept for reuse instead of being returned). */
int64_t dgq_getAvailableMemory(void);

/* ---------------------------------------------------------------- batches
 * Batched form (no counterpart in dgQuEST, which runs one register at a
 * time). The pending gates of many registers -- recorded through the usual
 * API calls, one precision per batch -- are planned together and run by ONE
 * persistent kernel launch, captured in a CUDA graph with the resets it
 * needs. CTAs take (register, sweep, tile) work items in order and wait, on
 * device counters, for the previous sweep of the same register.
 * Each launch recomputes every register from its recorded initialisation,
 * so a batch can be launched repeatedly when every register starts with
 * initZeroState / initPlusState / initClassicalState; the states hold the
 * final amplitudes after each launch (getAmp etc. work as usual). */
typedef struct dgq_batch_s *dgq_batch;
typedef struct dgq_batch_config {
    int32_t tileBits;     /* widest tile, 9..12 (registers narrower than it use their width); 0 = choose */
    int32_t groupFactor;  /* registers interleaved sweep by sweep: about groupFactor x grid tiles; 0 = choose */
    int32_t ctasPerSm;    /* persistent CTAs per SM; 0 = as many as fit */
    int32_t tune;         /* 1: time candidate tile widths and group factors on a sample of the batch */
} dgq_batch_config;
typedef struct dgq_batch_stats {
    int32_t registers;
    int32_t wholeRegisters;  /* registers that fit one tile: one item runs all their sweeps */
    int32_t sweeps;          /* sweep programs over all registers */
    int32_t tileBits;
    int32_t groupFactor;
    int32_t grid;            /* persistent CTAs */
    int32_t ctasPerSm;
    int32_t tuned;           /* 1 when the autotuner ran for this batch */
    int64_t items;           /* work items per launch */
    int64_t gates;           /* recorded gates (before merging) */
    int64_t programBytes;    /* device bytes of programs and work list (uploaded once) */
    int64_t stateBytes;      /* amplitude bytes of all registers */
    int64_t sweepBytes;      /* algorithmic HBM bytes of one launch: sum over sweeps of 2 x state bytes */
    double planMillis;       /* host planning and packing */
    double tuneMillis;       /* autotuning (0 when a cached choice was used) */
    double flopsPerLaunch;   /* algorithmic flops of one launch */
} dgq_batch_stats;
/* cfg NULL: autotuned (the choice is cached per precision and register-size
 * histogram; DGQ_BATCH_TUNE=0 disables tuning). Returns NULL on error. */
dgq_batch dgq_batchCreate(const Qureg *quregs, int count, const dgq_batch_config *cfg);
int dgq_batchLaunch(dgq_batch batch);   /* replays the graph; does not wait */
int dgq_batchWait(dgq_batch batch);     /* waits and checks the kernel's wait-timeout flag */
/* Waits, then writes <Z_q> = P(q=0) - P(q=1) of every register's qubits,
 * register by register (sum of numQubits values). */
int dgq_batchExpectationZ(dgq_batch batch, double *out);
int dgq_batchGetStats(dgq_batch batch, dgq_batch_stats *out);
void *dgq_batchGetStream(dgq_batch batch);
void dgq_batchDestroy(dgq_batch batch);

#ifdef __cplusplus
}
#endif

#endif /* DGQ_EXT_H */
