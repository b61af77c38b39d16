"""multiQubitUnitary with 5..7 targets: the dense sweep kernel against the
oracle (1e-12 per amplitude for complex128, fidelity >= 1 - 1e-6 for
complex64), between other gates, right after initialisation and after a
measurement collapse; registers from 9 to 16 qubits."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def apply_dense(Q, q, targs, u):
    m = Q.matrixN(u)
    Q.multiQubitUnitary(q, Q.int_array(targs), len(targs), m)
    Q.destroyComplexMatrixN(m)


@pytest.mark.parametrize("n,targs,single", [
    (9, [0, 1, 2, 3, 4], False),
    (10, [7, 2, 9, 0, 4], False),
    (12, [11, 0, 5, 3, 8, 1], False),
    (14, [13, 12, 11, 10, 9, 8, 7], False),
    (16, [2, 15, 6, 0, 9, 12], False),
    (9, [8, 6, 4, 2, 0, 1, 3], False),
    (13, [0, 3, 6, 9, 12], True),
    (16, [15, 1, 7, 4, 10, 13, 0], True),
])
def test_dense_unitary_matches_oracle(quest, env, n, targs, single):
    Q = quest
    gen = np.random.default_rng(n * 31 + len(targs))
    u = C.random_unitary(gen, 1 << len(targs))
    pre = C.mixed_ops(n, 80, 11 + n)
    post = C.mixed_ops(n, 80, 12 + n)
    q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
    C.replay(q, pre)
    apply_dense(Q, q, targs, u)
    C.replay(q, post)
    apply_dense(Q, q, list(reversed(targs)), u.conj().T)
    amps = Q.state_vector(q)
    Q.destroyQureg(q, env)
    o = oracle.Oracle(n)
    o.apply(pre)
    o.multi_qubit_unitary(targs, u)
    o.apply(post)
    o.multi_qubit_unitary(list(reversed(targs)), u.conj().T)
    ref = o.amps()
    o.close()
    if single:
        assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
    else:
        assert np.abs(amps - ref).max() <= 1e-12


def test_dense_first_and_after_collapse(quest, env):
    Q = quest
    n = 11
    targs = [3, 9, 0, 6, 1]
    u = C.random_unitary(np.random.default_rng(5), 32)
    q = Q.createQureg(n, env)
    Q.initPlusState(q)
    apply_dense(Q, q, targs, u)          # the dense sweep is the first work after the init
    Q.collapseToOutcome(q, 4, 1)
    apply_dense(Q, q, targs, u.conj().T)  # and right after a lazy collapse
    amps = Q.state_vector(q)
    Q.destroyQureg(q, env)
    o = oracle.Oracle(n)
    o.init_plus()
    o.multi_qubit_unitary(targs, u)
    o.collapse(4, 1)
    o.multi_qubit_unitary(targs, u.conj().T)
    assert np.abs(amps - o.amps()).max() <= 1e-12
    o.close()


def test_dense_rejects_eight_targets(quest, env):
    Q = quest
    q = Q.createQureg(10, env)
    u = np.eye(256, dtype=complex)
    with pytest.raises(Q.QuESTError):
        apply_dense(Q, q, list(range(8)), u)
    Q.destroyQureg(q, env)
