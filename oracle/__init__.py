"""The oracle: CPU restatement of dgQuEST's gate semantics (dgq_oracle.c).

TEST INFRASTRUCTURE ONLY. tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py use it as the checker or as the timed CPU
baseline; the product (dgquest_b200/libdgq.so) never loads it.

Pinned against the reference: tests/golden/ holds outputs of the reference
itself (built from its sources by oracle/Makefile `ref` into oracle/_ref and
run on a B200 by tests/golden/make_golden.py); tests/test_oracle.py checks
the oracle against them and against dense numpy matrices.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int64, c_uint32, c_ulong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")

_lib = None


def build():
    """Compiles liboracle.so (gcc + OpenMP) if it is missing or stale."""
    src = os.path.join(HERE, "dgq_oracle.c")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = c_void_p
        L.orc_create.argtypes = [c_int]
        L.orc_destroy.argtypes = [c_void_p]
        L.orc_amps.restype = POINTER(c_double)
        L.orc_amps.argtypes = [c_void_p]
        L.orc_init_zero.argtypes = [c_void_p]
        L.orc_init_plus.argtypes = [c_void_p]
        L.orc_init_classical.argtypes = [c_void_p, ctypes.c_uint64]
        L.orc_set_amps.argtypes = [c_void_p, POINTER(c_double), POINTER(c_double)]
        L.orc_seed.argtypes = [c_void_p, POINTER(c_ulong), c_int]
        L.orc_apply_ops.restype = c_int64
        L.orc_apply_ops.argtypes = [c_void_p, c_void_p, c_int64, POINTER(c_int)]
        L.orc_prob_zero.restype = c_double
        L.orc_prob_zero.argtypes = [c_void_p, c_int]
        L.orc_prob_zero_all.argtypes = [c_void_p, POINTER(c_double)]
        L.orc_total_prob.restype = c_double
        L.orc_total_prob.argtypes = [c_void_p]
        L.orc_collapse.argtypes = [c_void_p, c_int, c_int, c_double]
        L.orc_measure.restype = c_int
        L.orc_measure.argtypes = [c_void_p, c_int, POINTER(c_double)]
        L.orc_multi_qubit_unitary.argtypes = [c_void_p, POINTER(c_int), c_int, POINTER(c_double), POINTER(c_double)]
        L.orc_mt_first_outputs.argtypes = [POINTER(c_ulong), c_int, POINTER(c_uint32), c_int]
        L.orc_mt_first_outputs_seed.argtypes = [c_uint32, POINTER(c_uint32), c_int]
        L.orc_max_threads.restype = c_int
        L.orc_set_threads.argtypes = [c_int]
        _lib = L
    return _lib


class Oracle:
    """One state vector of n qubits held by the CPU oracle."""

    def __init__(self, n):
        self.n = n
        self.ptr = lib().orc_create(n)
        if not self.ptr:
            raise MemoryError(f"oracle cannot allocate {n} qubits")
        lib().orc_init_zero(self.ptr)

    def close(self):
        if self.ptr:
            lib().orc_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()

    def init_zero(self):
        lib().orc_init_zero(self.ptr)

    def init_plus(self):
        lib().orc_init_plus(self.ptr)

    def init_classical(self, index):
        lib().orc_init_classical(self.ptr, index)

    def set_amps(self, amps):
        amps = np.ascontiguousarray(amps, dtype=np.complex128)
        re = np.ascontiguousarray(amps.real)
        im = np.ascontiguousarray(amps.imag)
        lib().orc_set_amps(self.ptr, re.ctypes.data_as(POINTER(c_double)), im.ctypes.data_as(POINTER(c_double)))

    def seed(self, keys):
        arr = (c_ulong * len(keys))(*keys)
        lib().orc_seed(self.ptr, arr, len(keys))

    def apply(self, ops):
        ops = np.ascontiguousarray(ops)
        nmeas = int(np.sum(ops["kind"] == 24))
        outcomes = (c_int * max(1, nmeas))()
        r = lib().orc_apply_ops(self.ptr, ops.ctypes.data_as(c_void_p), len(ops), outcomes)
        if r < 0:
            raise ValueError(f"oracle rejected op {-r - 1}")
        return [outcomes[i] for i in range(nmeas)]

    def amps(self):
        p = lib().orc_amps(self.ptr)
        flat = np.ctypeslib.as_array(p, shape=(2 << self.n,))
        return (flat[0::2] + 1j * flat[1::2]).copy()

    def prob_zero_all(self):
        out = np.empty(self.n, dtype=np.float64)
        lib().orc_prob_zero_all(self.ptr, out.ctypes.data_as(POINTER(c_double)))
        return out

    def total_prob(self):
        return lib().orc_total_prob(self.ptr)

    def collapse(self, q, outcome):
        """collapseToOutcome: keep the amplitudes with bit q == outcome, renormalised."""
        p0 = lib().orc_prob_zero(self.ptr, q)
        lib().orc_collapse(self.ptr, q, outcome, p0 if outcome == 0 else 1.0 - p0)

    def measure(self, q):
        p = c_double()
        return lib().orc_measure(self.ptr, q, ctypes.byref(p)), p.value

    def multi_qubit_unitary(self, targs, u):
        u = np.asarray(u, dtype=np.complex128)
        re = np.ascontiguousarray(u.real)
        im = np.ascontiguousarray(u.imag)
        t = (c_int * len(targs))(*targs)
        lib().orc_multi_qubit_unitary(self.ptr, t, len(targs), re.ctypes.data_as(POINTER(c_double)),
                                      im.ctypes.data_as(POINTER(c_double)))


def mt_outputs_by_array(keys, count):
    out = (c_uint32 * count)()
    arr = (c_ulong * len(keys))(*keys)
    lib().orc_mt_first_outputs(arr, len(keys), out, count)
    return list(out)


def mt_outputs_by_seed(seed, count):
    out = (c_uint32 * count)()
    lib().orc_mt_first_outputs_seed(seed, out, count)
    return list(out)


def run(n, ops, seed_keys=None):
    """Applies ops to |0..0> and returns (amplitudes, P(q=0) per qubit, measurement outcomes)."""
    o = Oracle(n)
    if seed_keys is not None:
        o.seed(seed_keys)
    outcomes = o.apply(ops)
    amps = o.amps()
    p0 = o.prob_zero_all()
    o.close()
    return amps, p0, outcomes


def max_threads():
    return lib().orc_max_threads()


def set_threads(n):
    """Threads of the oracle's OpenMP loops from now on."""
    lib().orc_set_threads(int(n))
