"""Python mirror of the QuEST C API exported by libdgq.so.

Names, argument order and meaning follow dgQuEST's include/QuEST.h (each
C declaration in include/QuEST.h cites its dgQuEST prototype). Structures
are passed by value exactly as in C. The C library's default on invalid
input is QuEST's: print and exit(code) (src/QuEST_validation.c:82-91).
This mirror switches the library to status recording and raises
``QuESTError(code, message)`` instead, so a Python process survives bad
input; ``code`` is QuEST's error code.
"""
import atexit
import ctypes
from ctypes import POINTER, Structure, c_double, c_int, c_int64, c_longlong, c_ulong, c_ulonglong, c_void_p

import numpy as np

from . import load_library

qreal = c_double


class Complex(Structure):
    _fields_ = [("real", qreal), ("imag", qreal)]


class ComplexMatrix2(Structure):
    _fields_ = [("r0c0", Complex), ("r0c1", Complex), ("r1c0", Complex), ("r1c1", Complex)]


class Vector(Structure):
    _fields_ = [("x", qreal), ("y", qreal), ("z", qreal)]


class QuESTEnv(Structure):
    _fields_ = [("value", c_void_p), ("rank", c_int)]


class Qureg(Structure):
    _fields_ = [
        ("isDensityMatrix", c_int),
        ("numQubitsRepresented", c_ulonglong),
        ("numQubitsInStateVec", c_ulonglong),
        ("numAmpsTotal", c_ulonglong),
        ("env", QuESTEnv),
        ("state", c_void_p),
    ]


class ComplexMatrixN(Structure):
    _fields_ = [("numQubits", c_int), ("real", POINTER(POINTER(qreal))), ("imag", POINTER(POINTER(qreal)))]


class PlanStats(Structure):
    _fields_ = [
        ("sweeps", ctypes.c_int32),
        ("phases", ctypes.c_int32),
        ("ops", ctypes.c_int32),
        ("gates", ctypes.c_int32),
        ("tileBits", ctypes.c_int32),
        ("numBits", ctypes.c_int32),
        ("flopsPerAmp", c_double),
        ("planMillis", c_double),
        ("jitCompiled", ctypes.c_int32),
        ("jitReused", ctypes.c_int32),
        ("jitMillis", c_double),
        ("launchBytes", ctypes.c_int64),
        ("streamedSweeps", ctypes.c_int32),
        ("denseBlocks", ctypes.c_int32),
        ("formK", ctypes.c_int32),
        ("formAuto", ctypes.c_int32),
        ("predictedTileMs", c_double),
        ("predictedDenseMs", c_double * 3),
        ("denseBound", ctypes.c_int32),
    ]


class BatchConfig(Structure):
    _fields_ = [("tileBits", ctypes.c_int32), ("groupFactor", ctypes.c_int32), ("ctasPerSm", ctypes.c_int32),
                ("tune", ctypes.c_int32)]


class BatchStats(Structure):
    _fields_ = [
        ("registers", ctypes.c_int32),
        ("wholeRegisters", ctypes.c_int32),
        ("sweeps", ctypes.c_int32),
        ("tileBits", ctypes.c_int32),
        ("groupFactor", ctypes.c_int32),
        ("grid", ctypes.c_int32),
        ("ctasPerSm", ctypes.c_int32),
        ("tuned", ctypes.c_int32),
        ("items", ctypes.c_int64),
        ("gates", ctypes.c_int64),
        ("programBytes", ctypes.c_int64),
        ("stateBytes", ctypes.c_int64),
        ("sweepBytes", ctypes.c_int64),
        ("planMillis", c_double),
        ("tuneMillis", c_double),
        ("flopsPerLaunch", c_double),
    ]


class QuESTError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


I, D, Q, E, P = c_int, c_double, Qureg, QuESTEnv, POINTER
_SIGS = {
    # name: (restype, argtypes)
    "createQuESTEnv": (QuESTEnv, []),
    "destroyQuESTEnv": (None, [E]),
    "seedQuESTDefault": (None, []),
    "seedQuEST": (None, [P(c_ulong), I]),
    "getQuEST_PREC": (I, []),
    "createQureg": (Qureg, [I, E]),
    "searchQuregTaskPartitions": (None, [Q, E]),
    "destroyQureg": (None, [Q, E]),
    "getNumQubits": (I, [Q]),
    "getNumAmps": (I, [Q]),
    "initZeroState": (None, [Q]),
    "initPlusState": (None, [Q]),
    "initClassicalState": (None, [Q, c_longlong]),
    "initStateFromAmps": (None, [Q, P(D), P(D)]),
    "initPureState": (None, [Q, Q]),
    "setAmps": (None, [Q, c_longlong, P(D), P(D), c_longlong]),
    "cloneQureg": (None, [Q, Q]),
    "reportQuregParams": (None, [Q]),
    "reportStateToScreen": (None, [Q, QuESTEnv, I]),
    "getEnvironmentString": (None, [QuESTEnv, Q, ctypes.c_char_p]),
    "phaseShift": (None, [Q, I, D]),
    "controlledPhaseShift": (None, [Q, I, I, D]),
    "multiControlledPhaseShift": (None, [Q, P(I), I, D]),
    "controlledPhaseFlip": (None, [Q, I, I]),
    "multiControlledPhaseFlip": (None, [Q, P(I), I]),
    "sGate": (None, [Q, I]),
    "tGate": (None, [Q, I]),
    "compactUnitary": (None, [Q, I, Complex, Complex]),
    "unitary": (None, [Q, I, ComplexMatrix2]),
    "rotateX": (None, [Q, I, D]),
    "rotateY": (None, [Q, I, D]),
    "rotateZ": (None, [Q, I, D]),
    "rotateAroundAxis": (None, [Q, I, D, Vector]),
    "controlledRotateX": (None, [Q, I, I, D]),
    "controlledRotateY": (None, [Q, I, I, D]),
    "controlledRotateZ": (None, [Q, I, I, D]),
    "controlledRotateAroundAxis": (None, [Q, I, I, D, Vector]),
    "controlledCompactUnitary": (None, [Q, I, I, Complex, Complex]),
    "controlledUnitary": (None, [Q, I, I, ComplexMatrix2]),
    "multiControlledUnitary": (None, [Q, P(I), I, I, ComplexMatrix2]),
    "pauliX": (None, [Q, I]),
    "pauliY": (None, [Q, I]),
    "pauliZ": (None, [Q, I]),
    "hadamard": (None, [Q, I]),
    "controlledNot": (None, [Q, I, I]),
    "controlledPauliY": (None, [Q, I, I]),
    "swapGate": (None, [Q, I, I]),
    "u1Gate": (None, [Q, I, D]),
    "u2Gate": (None, [Q, I, D, D]),
    "u3Gate": (None, [Q, I, D, D, D]),
    "SqX": (None, [Q, I]),
    "SqY": (None, [Q, I]),
    "SqW": (None, [Q, I]),
    "fSim": (None, [Q, I, I, D, D]),
    "multiQubitUnitary": (None, [Q, P(I), I, ComplexMatrixN]),
    "createComplexMatrixN": (ComplexMatrixN, [I]),
    "destroyComplexMatrixN": (None, [ComplexMatrixN]),
    "getAmp": (Complex, [Q, c_longlong]),
    "getRealAmp": (D, [Q, c_longlong]),
    "getImagAmp": (D, [Q, c_longlong]),
    "getProbAmp": (D, [Q, c_longlong]),
    "calcTotalProb": (D, [Q]),
    "calcProbOfOutcome": (D, [Q, I, I]),
    "collapseToOutcome": (D, [Q, I, I]),
    "measure": (I, [Q, I]),
    "measureWithStats": (I, [Q, I, P(D)]),
    "calcInnerProduct": (Complex, [Q, Q]),
    "calcFidelity": (D, [Q, Q]),
    # extensions (include/dgq.h)
    "dgq_setErrorMode": (I, [I]),
    "dgq_getLastError": (I, [ctypes.c_char_p, I]),
    "dgq_setTileBits": (I, [Q, I]),
    "dgq_getPlanStats": (I, [Q, P(PlanStats)]),
    "dgq_planPending": (I, [Q]),
    "dgq_setDenseFusion": (I, [Q, I]),
    "dgq_setDeviceBudget": (ctypes.c_int64, [ctypes.c_int64]),
    "dgq_shutdown": (None, []),
    "dgq_setCostModel": (I, [D, D]),
    "dgq_loadCostModel": (I, [ctypes.c_char_p]),
    "dgq_getCostModel": (I, [P(D), P(D)]),
    "dgq_setDenseCost": (I, [I, I, D]),
    "dgq_getDenseCost": (D, [I, I]),
    "dgq_getHostTierStats": (I, [Q, P(I), P(ctypes.c_int64), P(ctypes.c_int64), P(ctypes.c_int64)]),
    "dgq_createShardedQureg": (Qureg, [I, E, I, P(I), I]),
    "dgq_getShardStats": (I, [Q, P(I), P(ctypes.c_int64), P(ctypes.c_int64), P(ctypes.c_int64)]),
    "dgq_launchPlanned": (I, [Q]),
    "dgq_sync": (I, [Q]),
    "dgq_getStream": (c_void_p, [Q]),
    "dgq_getDeviceState": (c_void_p, [Q, P(I)]),
    "dgq_getStateVector": (I, [Q, P(D), P(D)]),
    "dgq_getLaunchCount": (c_int64, []),
    "dgq_calcProbOfAllZero": (I, [Q, P(D)]),
    "dgq_measureFp64Peak": (I, [P(D)]),
    "dgq_createQuregF32": (Qureg, [I, E]),
    "createDensityQureg": (Qureg, [I, E]),
    "getDensityAmp": (Complex, [Q, ctypes.c_longlong, ctypes.c_longlong]),
    "calcPurity": (D, [Q]),
    "applyOneQubitDephaseError": (None, [Q, I, D]),
    "applyTwoQubitDephaseError": (None, [Q, I, I, D]),
    "applyOneQubitDepolariseError": (None, [Q, I, D]),
    "applyOneQubitDampingError": (None, [Q, I, D]),
    "applyTwoQubitDepolariseError": (None, [Q, I, I, D]),
    "addDensityMatrix": (None, [Q, D, Q]),
    "dgq_getPrecision": (I, [Q]),
    "dgq_sweepSource": (I, [I, I, I, P(ctypes.c_int32), P(ctypes.c_uint64), P(ctypes.c_uint64), P(D), I, I,
                            ctypes.c_char_p, I]),
    "dgq_compileSweepSource": (I, [ctypes.c_char_p, ctypes.c_char_p, I]),
    "dgq_specialiseGates": (I, [I, I, I, P(ctypes.c_int32), P(ctypes.c_uint64), P(ctypes.c_uint64), P(D), I]),
    "dgq_setSpecialisationMinBits": (I, [I]),
    "dgq_setSpecialisationPolicy": (I, [I]),
    "dgq_setTensorCores": (I, [I]),
    "dgq_getDeviceErrors": (I, []),
    "dgq_calcProbOfAllZeroNoAlloc": (I, [c_void_p, I, c_void_p, c_void_p]),
    "dgq_fuseApplyHost": (I, [I, I, I, P(ctypes.c_int32), P(ctypes.c_uint64), P(ctypes.c_uint64), P(D), P(D), P(D)]),
    "dgq_planExchanges": (I, [I, I, I, I, P(ctypes.c_int32), P(ctypes.c_uint64), P(ctypes.c_int32),
                              P(ctypes.c_int32), P(ctypes.c_int32)]),
    "dgq_planGates": (I, [I, I, I, P(ctypes.c_int32), P(ctypes.c_uint64), P(ctypes.c_uint64), P(D), P(PlanStats),
                          P(ctypes.c_int32), P(ctypes.c_int32)]),
    "dgq_applyCircuit": (I, [Q, c_void_p, I, P(I)]),
    "dgq_sampleOutcomes": (I, [Q, I, ctypes.c_uint32, P(ctypes.c_uint64)]),
    "dgq_getAvailableMemory": (c_int64, []),
    "dgq_batchCreate": (c_void_p, [P(Qureg), I, P(BatchConfig)]),
    "dgq_batchLaunch": (I, [c_void_p]),
    "dgq_batchWait": (I, [c_void_p]),
    "dgq_batchExpectationZ": (I, [c_void_p, P(D)]),
    "dgq_batchGetStats": (I, [c_void_p, P(BatchStats)]),
    "dgq_batchGetStream": (c_void_p, [c_void_p]),
    "dgq_batchDestroy": (None, [c_void_p]),
}

_lib = None


def _library():
    global _lib
    if _lib is None:
        lib = load_library()
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        lib.dgq_setErrorMode(1)
        _lib = lib
    return _lib


def _check():
    lib = _library()
    buf = ctypes.create_string_buffer(512)
    code = lib.dgq_getLastError(buf, 512)
    if code:
        raise QuESTError(code, buf.value.decode(errors="replace"))


def _wrap(name):
    def call(*args):
        out = getattr(_library(), name)(*args)
        _check()
        return out

    call.__name__ = name
    call.__doc__ = f"QuEST API `{name}` (see include/QuEST.h)."
    return call


for _name in _SIGS:
    globals()[_name] = _wrap(_name)


def _shutdown():
    # runs at interpreter exit, before C-level teardown: stop and join the
    # library's background compile threads while NVRTC is intact
    if _lib is not None:
        _lib.dgq_shutdown()


atexit.register(_shutdown)


# ---------------------------------------------------------------- helpers
def mat2(m):
    """ComplexMatrix2 from a 2x2 array-like of complex numbers."""
    m = np.asarray(m, dtype=np.complex128)
    return ComplexMatrix2(*(Complex(float(m[r, c].real), float(m[r, c].imag)) for r in range(2) for c in range(2)))


def int_array(values):
    arr = (c_int * len(values))(*[int(v) for v in values])
    return arr


def matrixN(u):
    """ComplexMatrixN (library-allocated) filled from a square complex array."""
    u = np.asarray(u, dtype=np.complex128)
    k = int(round(np.log2(u.shape[0])))
    m = createComplexMatrixN(k)
    for r in range(u.shape[0]):
        for c in range(u.shape[1]):
            m.real[r][c] = float(u[r, c].real)
            m.imag[r][c] = float(u[r, c].imag)
    return m


def state_vector(q):
    """All amplitudes of q in logical order, as a complex128 numpy array (a
    density register: its 4^n elements, element (r, c) at r + c * 2^n)."""
    n = int(q.numQubitsInStateVec)
    re = np.empty(1 << n, dtype=np.float64)
    im = np.empty(1 << n, dtype=np.float64)
    dgq_getStateVector(q, re.ctypes.data_as(POINTER(c_double)), im.ctypes.data_as(POINTER(c_double)))
    return re + 1j * im


def density_matrix(q):
    """The density matrix of a density register as a 2^n x 2^n array."""
    dim = 1 << int(q.numQubitsRepresented)
    return state_vector(q).reshape(dim, dim).T


def prob_all_zero(q):
    n = int(q.numQubitsRepresented)
    out = np.empty(n, dtype=np.float64)
    dgq_calcProbOfAllZero(q, out.ctypes.data_as(POINTER(c_double)))
    return out


def plan_stats(q):
    st = PlanStats()
    dgq_getPlanStats(q, ctypes.byref(st))
    return st


def host_tier_stats(q):
    """(page bits, page passes, qubit exchanges, host<->device bytes) of a
    host-tier register, or None for a register in HBM."""
    pb = ctypes.c_int(0)
    passes = ctypes.c_int64(0)
    ex = ctypes.c_int64(0)
    moved = ctypes.c_int64(0)
    r = dgq_getHostTierStats(q, ctypes.byref(pb), ctypes.byref(passes), ctypes.byref(ex), ctypes.byref(moved))
    return (pb.value, passes.value, ex.value, moved.value) if r == 1 else None


def create_sharded(n, env, shard_bits, devices=None, single=False):
    """A register of n qubits in 2^shard_bits shards; devices[k] is the CUDA
    device of shard k (None: all on the current device)."""
    arr = None
    if devices is not None:
        assert len(devices) == 1 << shard_bits
        arr = (I * len(devices))(*[int(d) for d in devices])
    return dgq_createShardedQureg(n, env, shard_bits, arr, 1 if single else 0)


def shard_stats(q):
    """(shard bits, shard passes, qubit exchanges, bytes moved between
    shards) of a sharded register, or None for any other register."""
    sb = ctypes.c_int(0)
    passes = ctypes.c_int64(0)
    ex = ctypes.c_int64(0)
    moved = ctypes.c_int64(0)
    r = dgq_getShardStats(q, ctypes.byref(sb), ctypes.byref(passes), ctypes.byref(ex), ctypes.byref(moved))
    return (sb.value, passes.value, ex.value, moved.value) if r == 1 else None


def seed(keys):
    arr = (c_ulong * len(keys))(*[int(k) for k in keys])
    seedQuEST(arr, len(keys))


def apply_circuit(q, ops):
    """Records an op list (circuits.OP_DTYPE records, the dgq_gate_record
    layout) through dgq_applyCircuit in one call; returns measurement outcomes."""
    ops = np.ascontiguousarray(ops)
    assert ops.dtype.itemsize == 80
    n_meas = int((ops["kind"] == 24).sum()) if len(ops) else 0
    out = (c_int * max(1, n_meas))()
    dgq_applyCircuit(q, ops.ctypes.data if len(ops) else None, len(ops), out)
    return [int(out[i]) for i in range(n_meas)]


def sample(q, count, seed):
    """dgq_sampleOutcomes: `count` logical basis-state indices drawn from |amp|^2."""
    out = np.empty(max(1, count), dtype=np.uint64)
    dgq_sampleOutcomes(q, count, seed & 0xFFFFFFFF, out.ctypes.data_as(POINTER(ctypes.c_uint64)))
    return out[:count]


def init_from_amps(q, amps):
    amps = np.ascontiguousarray(amps, dtype=np.complex128)
    re = np.ascontiguousarray(amps.real)
    im = np.ascontiguousarray(amps.imag)
    initStateFromAmps(q, re.ctypes.data_as(POINTER(c_double)), im.ctypes.data_as(POINTER(c_double)))


class Batch:
    """A dgq_batch over registers whose gates are already recorded.

    config: None (autotuned) or a dict with tileBits / groupFactor / ctasPerSm / tune."""

    def __init__(self, quregs, config=None):
        self.quregs = list(quregs)
        self.handle = None
        arr = (Qureg * len(self.quregs))(*self.quregs)
        cfg = None
        if config is not None:
            cfg = BatchConfig(int(config.get("tileBits", 0)), int(config.get("groupFactor", 0)),
                              int(config.get("ctasPerSm", 0)), int(config.get("tune", 0)))
        self.handle = dgq_batchCreate(arr, len(self.quregs), ctypes.byref(cfg) if cfg is not None else None)
        if not self.handle:
            raise QuESTError(-1, "dgq_batchCreate returned NULL")
        self.num_values = sum(int(q.numQubitsRepresented) for q in self.quregs)

    def launch(self):
        dgq_batchLaunch(self.handle)

    def wait(self):
        dgq_batchWait(self.handle)

    def expectation_z(self):
        out = np.empty(self.num_values, dtype=np.float64)
        dgq_batchExpectationZ(self.handle, out.ctypes.data_as(POINTER(c_double)))
        return out

    def stats(self):
        st = BatchStats()
        dgq_batchGetStats(self.handle, ctypes.byref(st))
        return st

    def stream(self):
        return dgq_batchGetStream(self.handle)

    def close(self):
        if self.handle:
            dgq_batchDestroy(self.handle)
            self.handle = None

