"""Dense 5- and 6-target unitaries on complex64 registers through the tensor
cores: the pipelined split-FP16 sweep (registers of >= K + 7 address bits)
and the 3xTF32 sweep of 12-bit registers (6 targets), against the oracle
(fidelity >= 1 - 1e-6, max amplitude error <= 2e-6) and against the SIMT
dense kernel (<= 2e-6), with no MMA wait timing out."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def run(Q, env, n, targs, u, pre, post):
    q = Q.dgq_createQuregF32(n, env)
    C.replay(q, pre)
    m = Q.matrixN(u)
    Q.multiQubitUnitary(q, Q.int_array(targs), len(targs), m)
    Q.destroyComplexMatrixN(m)
    C.replay(q, post)
    amps = Q.state_vector(q)
    Q.destroyQureg(q, env)
    return amps


@pytest.mark.parametrize("n,targs", [(12, [0, 1, 2, 3, 4, 5]), (12, [11, 3, 7, 0, 9, 5]), (16, [15, 2, 9, 4, 12, 0]),
                                     (20, [6, 19, 1, 13, 8, 3]), (13, [12, 6, 7, 8, 9, 10]),
                                     (14, [0, 1, 2, 3, 4, 5]), (12, [3, 11, 0, 6, 9]), (17, [16, 8, 1, 4, 12]),
                                     (21, [20, 19, 18, 17, 16]), (13, [0, 1, 2, 7, 12]),
                                     (16, [1, 0, 9, 12, 4, 15])])
def test_tensor_core_dense(quest, env, n, targs):
    Q = quest
    u = C.random_unitary(np.random.default_rng(n + targs[0]), 1 << len(targs))
    pre = C.random_layers(n, 2, C.config_seed(3, n))
    post = C.random_layers(n, 1, C.config_seed(3, 100 + n))
    prev = Q.dgq_setTensorCores(1)
    try:
        a_tc = run(Q, env, n, targs, u, pre, post)
        assert Q.dgq_getDeviceErrors() == 0
        Q.dgq_setTensorCores(0)
        a_simt = run(Q, env, n, targs, u, pre, post)
    finally:
        Q.dgq_setTensorCores(prev)
    o = oracle.Oracle(n)
    o.apply(pre)
    o.multi_qubit_unitary(targs, u)
    o.apply(post)
    ref = o.amps()
    o.close()
    assert abs(np.vdot(ref, a_tc)) ** 2 >= 1 - 1e-6
    assert np.abs(a_tc - ref).max() <= 2e-6
    assert np.abs(a_tc - a_simt).max() <= 2e-6


def test_tensor_core_dense_after_collapse(quest, env):
    # a collapse still pending when the dense sweep runs (applied as the
    # sweep loads its tiles), then more gates; the oracle collapses at once
    Q = quest
    n, targs = 18, [2, 17, 9, 5, 13, 0]
    u = C.random_unitary(np.random.default_rng(99), 64)
    pre = C.random_layers(n, 2, C.config_seed(3, 300))
    post = C.random_layers(n, 1, C.config_seed(3, 301))
    q = Q.dgq_createQuregF32(n, env)
    C.replay(q, pre)
    p = Q.collapseToOutcome(q, 7, 1)
    m = Q.matrixN(u)
    Q.multiQubitUnitary(q, Q.int_array(targs), 6, m)
    Q.destroyComplexMatrixN(m)
    C.replay(q, post)
    a = Q.state_vector(q)
    Q.destroyQureg(q, env)
    assert Q.dgq_getDeviceErrors() == 0
    o = oracle.Oracle(n)
    o.apply(pre)
    po = 1.0 - o.prob_zero_all()[7]
    o.collapse(7, 1)
    o.multi_qubit_unitary(targs, u)
    o.apply(post)
    ref = o.amps()
    o.close()
    assert abs(p - po) <= 1e-6
    assert abs(np.vdot(ref, a)) ** 2 >= 1 - 1e-6
    assert np.abs(a - ref).max() <= 2e-6
