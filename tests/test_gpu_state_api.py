"""State-vector calls declared (without bodies) in dgQuEST's header:
setAmps, cloneQureg, initPureState, the report helpers, and the device
buffer in logical order after swapGate relabels (dgq_getDeviceState, which
undoes the relabels in HBM with the bit-swap kernel). Exact comparisons:
these calls move amplitudes without arithmetic."""
import ctypes

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def with_swaps(n, seed):
    b = C.OpList()
    for q in range(n):
        b.add(C.H, q)
    b.add(C.SWAP, 0, n - 1).add(C.SWAP, 2, 5).add(C.SWAP, 5, 7)
    ops = np.concatenate([b.array(), C.random_layers(n, 3, seed)])
    return ops


@pytest.mark.parametrize("single", [False, True])
def test_set_amps_in_logical_order(quest, env, single):
    n = 12
    ops = with_swaps(n, 301)
    q = quest.dgq_createQuregF32(n, env) if single else quest.createQureg(n, env)
    try:
        C.replay(q, ops)
        before = oracle.run(n, ops)[0]
        rng = np.random.default_rng(3)
        start, count = 100, 700
        vals = rng.normal(size=count) + 1j * rng.normal(size=count)
        re = np.ascontiguousarray(vals.real)
        im = np.ascontiguousarray(vals.imag)
        D = ctypes.POINTER(ctypes.c_double)
        quest.setAmps(q, start, re.ctypes.data_as(D), im.ctypes.data_as(D), count)
        got = quest.state_vector(q)
    finally:
        quest.destroyQureg(q, env)
    want = before.copy()
    want[start:start + count] = vals
    tol = 2e-6 if single else 1e-12
    assert np.abs(got - want).max() <= tol
    with pytest.raises(quest.QuESTError):
        q2 = quest.createQureg(4, env)
        try:
            quest.setAmps(q2, 10, re.ctypes.data_as(D), im.ctypes.data_as(D), 10)
        finally:
            quest.destroyQureg(q2, env)


def test_clone_and_init_pure_state(quest, env):
    n = 14
    ops = with_swaps(n, 302)
    a = quest.createQureg(n, env)
    b = quest.createQureg(n, env)
    c = quest.createQureg(n, env)
    try:
        C.replay(a, ops)
        quest.collapseToOutcome(a, 3, 1)  # a pending collapse travels with the copy
        quest.cloneQureg(b, a)
        quest.initPureState(c, a)
        sa, sb, sc = quest.state_vector(a), quest.state_vector(b), quest.state_vector(c)
        assert np.array_equal(sa, sb) and np.array_equal(sa, sc)
        quest.hadamard(b, 4)  # b is independent of a afterwards
        assert np.array_equal(quest.state_vector(a), sa)
        assert not np.array_equal(quest.state_vector(b), sa)
        odd = quest.createQureg(n - 1, env)
        with pytest.raises(quest.QuESTError):
            quest.cloneQureg(odd, a)
        quest.destroyQureg(odd, env)
    finally:
        for q in (a, b, c):
            quest.destroyQureg(q, env)


def test_device_state_in_logical_order(quest, env):
    from cuda.bindings import runtime as cudart
    n = 13
    ops = with_swaps(n, 303)
    q = quest.createQureg(n, env)
    try:
        C.replay(q, ops)
        quest.collapseToOutcome(q, 1, 0)
        want = quest.state_vector(q)
        nb = ctypes.c_int(0)
        ptr = quest.dgq_getDeviceState(q, ctypes.byref(nb))
        assert nb.value == n
        host = np.empty(1 << n, dtype=np.complex128)
        err, = cudart.cudaMemcpy(host.ctypes.data, ptr, host.nbytes, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == cudart.cudaError_t.cudaSuccess
        assert np.array_equal(host, want)
        # gates after the relabels were undone still act on the right qubits
        quest.hadamard(q, 0)
        ref = oracle.Oracle(n)
        ref.apply(ops)
        ref.collapse(1, 0)
        ref.apply(np.concatenate([C.OpList().add(C.H, 0).array()]))
        assert np.abs(quest.state_vector(q) - ref.amps()).max() <= 1e-12
        ref.close()
    finally:
        quest.destroyQureg(q, env)


def test_report_helpers(quest, env, capfd):
    q = quest.createQureg(3, env)
    try:
        quest.hadamard(q, 0)
        quest.reportQuregParams(q)
        quest.reportStateToScreen(q, env, 0)
        buf = ctypes.create_string_buffer(200)
        quest.getEnvironmentString(env, q, buf)
    finally:
        quest.destroyQureg(q, env)
    out = capfd.readouterr().out
    assert "Number of qubits is 3." in out
    assert "0.70710678118655, 0.00000000000000" in out
    assert b"qubits=3" in buf.value
