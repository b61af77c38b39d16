// tile_program.h -- the per-launch program of the fused tile kernel.
//
// One launch = one sweep of the state: every CTA owns one tile of 2^W
// amplitudes whose indices range over W "tile" address bits (always
// including the 5 lowest bits, so each warp moves 512-byte runs) with the
// other bits fixed by blockIdx. Inside the CTA each thread keeps 16
// amplitudes in registers. The gate list of the fused block is cut into
// phases; in a phase the 4 register bits cover every non-diagonal target,
// so all of the phase's gates run in registers, and phases change layout
// through shared memory. Diagonal gates need no register placement (they
// read the index bits), which is dgQuEST's treatment of diagonal gates and
// of Rz on a non-local target (QuEST_gpu_kernel.cu:300-311).
//
// The program is passed by value as a __grid_constant__ kernel parameter
// (constant bank; uniform loads), so no per-launch host-to-device copy is
// needed and the launch can be captured in a CUDA graph as is.
#pragma once

#include <cstdint>

namespace dgq {

constexpr int kRegBits = 4;
constexpr int kRegs = 1 << kRegBits;
constexpr int kCoalescedBits = 5;
constexpr int kMinTileBits = 9;   // >= 32 threads (one full warp)
constexpr int kMaxTileBits = 14;      // paired complex64 form: 2^13 slots of 16 B (128 KiB)
constexpr int kMaxTileBitsF64 = 12;   // complex128: 2^12 x 16 B (64 KiB)
constexpr int kMaxTileBitsC64 = 13;   // unpaired complex64: 2^13 x 8 B (64 KiB)
constexpr int kMaxThreadBits = kMaxTileBits - kRegBits - 1;  // 512 threads
constexpr int kMaxStateBits = 40;
constexpr int kMaxPhases = 56;
constexpr int kMaxOps = 640;
constexpr int kMaxCoef = 1500;

enum KOpKind : uint8_t {
    KOP_M2R = 0,   // real 2x2 [[a, b], [c, d]] on a register pair
    KOP_M2I = 1,   // [[a, i b], [i c, d]] (a, b, c, d real): the Rx family
    KOP_M2C = 2,   // general complex 2x2 (8 coefficients, row-major re/im)
    KOP_X = 3,     // swap
    KOP_Y = 4,     // Pauli-Y
    KOP_YC = 5,    // conjugated Pauli-Y
    KOP_NEG = 6,   // multiply by -1
    KOP_MULI = 7,  // multiply by +i
    KOP_MULNI = 8, // multiply by -i
    KOP_PH = 9,    // multiply by (c + i s)
    KOP_Z2 = 10,   // multiply by (c - i s) when the selector bit is 0, (c + i s) when 1
    KOP_DENSE = 11, // dense 2^k x 2^k on register bits 0..k-1 (k = op.k), coefficients re/im
    // Uncontrolled gates with their scalar factor moved into the sweep's
    // global factor (TileProgram::globalRe/Im), leaving unit entries:
    KOP_RY1 = 12,  // [[1, -t], [t, 1]]        (Ry with |cos| >= |sin|, t = tan)
    KOP_RY2 = 13,  // [[u, -1], [1, u]]        (Ry with |sin| > |cos|, u = cot)
    KOP_RX1 = 14,  // [[1, -i t], [-i t, 1]]   (Rx, t = tan)
    KOP_RX2 = 15,  // [[u, -i], [-i, u]]       (Rx, u = cot)
    KOP_H1 = 16,   // [[1, 1], [1, -1]]        (Hadamard without 1/sqrt 2)
    KOP_PH1 = 17,  // multiply by (c + i s) where the selector bit is 1 (Rz without e^{-i a})
    KOP_RN1 = 18   // [[1, p], [-conj(p), 1]], p complex: rotations about an axis in the XY plane
                   // (sqrt X, sqrt Y, sqrt W, ...) divided by their equal diagonal entry
};

// The op kinds of rotation / CNOT / CZ / phase circuits (the interpreting
// kernels' lean form handles these only).
constexpr uint32_t kLeanKinds = (1u << KOP_X) | (1u << KOP_NEG) | (1u << KOP_PH) | (1u << KOP_Z2) |
                                (1u << KOP_RY1) | (1u << KOP_RY2) | (1u << KOP_RX1) | (1u << KOP_RX2) |
                                (1u << KOP_H1) | (1u << KOP_PH1);

// Dispatch codes of the tile kernel: one straight-line case per
// (operation, target register bit, register-control present). Pair
// operations: base + k (+4 when some control bit is a register bit).
enum KCode : uint8_t {
    KC_M2R = 0,
    KC_M2I = 8,
    KC_M2C = 16,
    KC_X = 24,
    KC_Y = 32,
    KC_YC = 40,
    KC_Z2R = 48,   // Rz-like, selector = register bit k (+4 controlled)
    KC_Z2T = 56,   // selector is a thread/CTA bit (+1 controlled)
    KC_PH = 58,    // +1 controlled
    KC_NEG = 60,   // +1 controlled
    KC_MULI = 62,  // +1 controlled
    KC_MULNI = 64, // +1 controlled
    KC_DENSE = 66, // + (k - 1), k = 1..4
    KC_RY1 = 70,   // + k; never controlled
    KC_RY2 = 74,
    KC_RX1 = 78,
    KC_RX2 = 82,
    KC_H1 = 86,
    KC_PH1R = 90,  // + k: selector = register bit k
    KC_PH1T = 94,  // selector is a thread/CTA bit
    KC_RN1 = 95,   // + k; never controlled
    KC_COUNT = 99
};

// 16 bytes; every field is read uniformly by all threads of the CTA.
struct KOp {
    uint8_t kind;      // KOpKind (accounting)
    uint8_t code;      // KCode (dispatch)
    uint8_t thrCtl;    // 1 when ctrlLoc or ctrlCta is non-zero
    uint8_t ctrlReg;   // control bits in register-index space
    uint16_t ctrlLoc;  // control bits among the thread (non-register) tile bits
    uint16_t selLoc;   // KC_Z2T selector when it is a thread tile bit
    uint32_t ctrlCta;  // control bits in blockIdx space (non-tile address bits)
    uint16_t coef;     // offset into TileProgram::coef
    int8_t selCta;     // KC_Z2T selector bit index in blockIdx space, -1 if none
    uint8_t k;         // target register bit (pair ops), selector register bit (KC_Z2R), k (dense)
};

struct KPhase {
    uint8_t thrPos[kMaxThreadBits];  // tile-local bit of thread-index bit i
    uint8_t direct;                  // 1: thread bits 0..4 are tile bits 0..4 (coalesced global I/O)
    uint8_t regPos[kRegBits];        // tile-local bit of register bit b
    uint8_t pad[2];
    uint16_t opBegin, opEnd;
    uint16_t regOff[kRegs];  // swizzled shared-memory offset of register j
};

enum InitKind : int32_t {
    INIT_NONE = 0,       // read the state
    INIT_CLASSICAL = 1,  // |initIndex>
    INIT_PLUS = 2,       // initAmp on every index below 2^numReal
    INIT_BLANK = 3,      // all zero
};

struct TileProgram {
    int32_t numPhases;
    int32_t numOps;
    int32_t numBits;   // address bits of the state buffer
    int32_t numReal;   // qubits the user sees (<= numBits)
    int32_t initKind;
    int32_t hasRestrict;
    int32_t hasGlobal;       // multiply every amplitude by (globalRe + i globalIm) before the store
    int32_t isSingle;        // 1: complex64 state (float2), 0: complex128 (double2)
    double globalRe, globalIm;
    // complex64 renormalisation (runtime-specialised kernels only): the
    // sweep scales by 1/sqrt(*normIn) and adds its output's sum of |a|^2
    // to *normOut (zeroed before the launch)
    int32_t renormIn, renormOut;
    const double *normIn;
    double *normOut;
    uint64_t initIndex;
    double initAmp;
    uint64_t restrictMask;   // lazy measurement collapse applied at load:
    uint64_t restrictValue;  //   amp = (idx & mask) == value ? amp * scale : 0
    double restrictScale;
    uint8_t highPos[kMaxTileBits - kCoalescedBits];  // address bit of tile-local bit 5 + i
    uint8_t ctaPos[kMaxStateBits];                   // address bit of blockIdx bit i
    uint16_t numCoef;  // coefficients used (coef[0 .. numCoef))
    // 1: complex64 paired form. Address bit 0 stays inside each thread: a
    // thread holds 16 slots of two amplitudes (address bit 0 = 0 and 1), as
    // packed (re_lo, re_hi) and (im_lo, im_hi) pairs; phases place 4 slot
    // bits in registers, the other W - 5 tile bits on threads, and ops with
    // op.k == 4 act on the pair inside a slot (target address bit 0).
    uint8_t paired;
    uint8_t pad0[1];
    // the launch covers CTAs ctaOffset .. ctaOffset + ctaCount (0: all): a
    // sweep over one page of a state held in host memory, whose page-index
    // bits are the top blockIdx bits
    uint32_t ctaOffset, ctaCount;
    // > 0: not a tile sweep but a dense 2^denseK x 2^denseK unitary on the
    // address bits denseTargets[0..denseK) (bit 0 of the matrix index first);
    // its matrix is at denseOff doubles into the register's matrix buffer
    int32_t denseK;
    uint32_t denseOff;
    uint32_t denseTcOff;  // complex64, 6 targets: packed tensor-core operand (0: none)
    uint8_t denseTargets[8];
    KPhase phases[kMaxPhases];
    KOp ops[kMaxOps];
    double coef[kMaxCoef];
};

static_assert(sizeof(KOp) == 16, "KOp layout");
static_assert(sizeof(TileProgram) <= 32000, "TileProgram must fit the kernel parameter space");

// Shared-memory swizzle of a tile-local index: the low 3 bits (the 16-byte
// bank group) are XOR-ed with the higher bit triples. Linear over GF(2),
// so swz(a | b) = swz(a) ^ swz(b) for disjoint a, b.
static inline constexpr uint32_t tileSwizzle(uint32_t x) {
    return x ^ (((x >> 3) ^ (x >> 6) ^ (x >> 9) ^ (x >> 12)) & 7u);
}

}  // namespace dgq
