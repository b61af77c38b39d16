"""CPU tests of the host planner and the runtime specialisation: plans for
the headline circuits, DAG merge rules, and NVRTC compiles of generated
sweep kernels for sm_100a (no GPU is used)."""
import ctypes

import numpy as np
import pytest

from dgquest_b200 import circuits as C
from dgquest_b200 import ir
from dgquest_b200 import quest as Q

P = ctypes.POINTER


def test_random_circuit_plan_shape():
    ops = C.random_layers(30, 20, C.config_seed(2))
    prev = None
    for w in (9, 10, 11, 12):
        st = ir.plan(ops, 30, w)
        assert st.tileBits == w and st.numBits == 30
        assert st.gates == 900
        if prev is not None:
            assert st.sweeps <= prev  # wider tiles never need more sweeps here
        prev = st.sweeps
    assert 15 <= prev <= 30


def test_merge_rules():
    # T T -> S ; S S -> Z ; Z Z -> nothing ; Rx(a) Rx(b) -> Rx(a+b) ; H H -> nothing ; X then U -> U
    b = C.OpList()
    b.add(C.T, 0).add(C.T, 0)            # -> S (type 2)
    b.add(C.H, 1).add(C.H, 1)            # cancel
    b.add(C.RX, 2, p=(0.3,)).add(C.RX, 2, p=(0.4,))  # one Rx
    b.add(C.Z, 3).add(C.Z, 3)            # cancel
    b.add(C.PHASE, 4, p=(0.2,)).add(C.T, 4)  # one phase shift
    st, merged = ir.plan(b.array(), 10, 9, want_merged=True)
    assert sorted(merged) == sorted([2, 15, 8])


def _sources(ops, n, w, precision=2):
    t, tm, cm, o = ir.ops_to_ir(ops, n)
    buf = ctypes.create_string_buffer(1 << 20)
    args = (n, w, len(t), t.ctypes.data_as(P(ctypes.c_int32)), tm.ctypes.data_as(P(ctypes.c_uint64)),
            cm.ctypes.data_as(P(ctypes.c_uint64)), o.ctypes.data_as(P(ctypes.c_double)))
    count = Q.dgq_sweepSource(*args, 0, precision, buf, len(buf))
    out = []
    for s in range(count):
        Q.dgq_sweepSource(*args, s, precision, buf, len(buf))
        out.append(buf.value)
    return out


@pytest.mark.parametrize("w,precision", [(9, 2), (12, 2), (13, 1), (11, 1), (12, 3)])
def test_generated_sweeps_compile(w, precision):
    ops = np.concatenate([C.mixed_ops(14, 150, 3, kinds=[k for k in range(26) if k != C.MEASURE]),
                          C.random_layers(14, 2, 5)])
    srcs = _sources(ops, 14, w, precision)
    assert len(srcs) >= 1
    log = ctypes.create_string_buffer(1 << 16)
    for s in srcs[:3]:
        size = Q.dgq_compileSweepSource(s, log, len(log))
        assert size > 0, log.value.decode()
    # precision 1 selects the paired complex64 form (float4 slots)
    assert all((b"float4 sm[]" in s) == (precision == 1) for s in srcs)


def test_paired_sources_carry_signs_at_compile_time():
    """The paired complex64 generator writes no negation into a kernel: CZ,
    Y, S and the -1 entries of the factored rotations become compile-time
    signs (template masks) that a phase's closing factor or a flip restores;
    the kernels still compile."""
    n = 14
    kinds = [C.CZ, C.Y, C.S, C.CY, C.CNOT, C.H, C.RX, C.RY, C.RZ]
    ops = np.concatenate([C.mixed_ops(n, 200, 21, kinds=kinds), C.random_layers(n, 2, 9)])
    srcs = _sources(ops, n, 13, 1)
    assert srcs and all(b"float4 sm[]" in s for s in srcs)
    joined = b"".join(srcs)
    assert b"neg2(" not in joined
    assert b"dgq::pRY2s<" in joined or b"dgq::pRX2s<" in joined
    assert b"dgq::pFlushS<" in joined or b"dgq::pGlobalS<" in joined
    log = ctypes.create_string_buffer(1 << 16)
    assert Q.dgq_compileSweepSource(srcs[0], log, len(log)) > 0, log.value.decode()


@pytest.mark.parametrize("bad", ["multi_unitary_type", "type_out_of_range", "mask_beyond_register",
                                 "empty_target", "target_is_control"])
def test_plan_gates_rejects_invalid_gates(bad):
    # the host-only planner takes raw IR arrays: a gate it cannot encode is an
    # E_INVALID_ARGUMENT error, not undefined behaviour in the planner
    n = 12
    t, tm, cm, o = ir.ops_to_ir(C.random_layers(n, 2, 3), n)
    i = 5
    assert t[i] in (ir.OP_RX, ir.OP_RY, ir.OP_RZ)
    if bad == "multi_unitary_type":
        t[i] = 19
    elif bad == "type_out_of_range":
        t[i] = 27
    elif bad == "mask_beyond_register":
        tm[i] = np.uint64(1 << n)
    elif bad == "empty_target":
        tm[i] = np.uint64(0)
    else:
        cm[i] = tm[i]
    st = Q.PlanStats()
    with pytest.raises(Q.QuESTError):
        Q.dgq_planGates(n, 0, len(t), t.ctypes.data_as(P(ctypes.c_int32)), tm.ctypes.data_as(P(ctypes.c_uint64)),
                        cm.ctypes.data_as(P(ctypes.c_uint64)), o.ctypes.data_as(P(ctypes.c_double)),
                        ctypes.byref(st), None, None)
    buf = ctypes.create_string_buffer(1 << 16)
    with pytest.raises(Q.QuESTError):
        Q.dgq_sweepSource(n, 0, len(t), t.ctypes.data_as(P(ctypes.c_int32)), tm.ctypes.data_as(P(ctypes.c_uint64)),
                          cm.ctypes.data_as(P(ctypes.c_uint64)), o.ctypes.data_as(P(ctypes.c_double)), 0, 2, buf,
                          len(buf))


def test_specialise_ahead_counts_the_plans_kernels():
    # host-only: the number of kernels equals the number of sweeps the plan
    # of the same gates would launch (GHZ+QFT has no dense sweeps)
    n = 24
    ops = C.ghz_qft(n)
    count = ir.specialise(ops, n, 2, background=True)
    assert count == ir.plan(ops, n, 0).sweeps
    with pytest.raises(Q.QuESTError):
        Q.dgq_specialiseGates(n, 4, 0, None, None, None, None, 1)
