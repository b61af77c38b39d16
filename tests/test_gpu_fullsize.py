"""Full-size checks (the benchmark's 30-qubit registers) through properties
that need no oracle run at that size:

* round trip: the depth-20 random circuit followed by its inverse returns
  |0...0> (complex128: |<0|psi>| = 1 and total probability 1 within 1e-12;
  complex64 paired form: |<0|psi>|^2 >= 1 - 1e-6);
* Bernstein-Vazirani on 30 qubits: measuring qubits 0..28 returns the hidden
  string exactly (a basis state: every outcome is certain)."""
import numpy as np
import pytest

from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu

SELF_INVERSE = {C.H, C.X, C.Y, C.Z, C.CNOT, C.CZ, C.CY, C.SWAP}
ANGLE = {C.RX, C.RY, C.RZ, C.PHASE, C.CPHASE, C.CRX, C.CRY, C.CRZ}


def inverse(ops):
    inv = ops[::-1].copy()
    kinds = inv["kind"]
    assert np.isin(kinds, list(ANGLE | SELF_INVERSE)).all()
    ang = np.isin(kinds, list(ANGLE))
    inv["p"][ang, 0] *= -1.0
    return inv


@pytest.mark.parametrize("single", [False, True])
def test_random_circuit_round_trip_30_qubits(quest, env, single):
    n = 30
    ops = C.random_layers(n, 20, C.config_seed(2))
    q = quest.dgq_createQuregF32(n, env) if single else quest.createQureg(n, env)
    try:
        quest.initZeroState(q)
        quest.apply_circuit(q, ops)
        mid = quest.getAmp(q, 0)  # runs the circuit; the inverse is a plan of its own
        quest.apply_circuit(q, inverse(ops))
        a0 = quest.getAmp(q, 0)
        total = quest.calcTotalProb(q)
        st = quest.plan_stats(q)
    finally:
        quest.destroyQureg(q, env)
    p = a0.real ** 2 + a0.imag ** 2
    assert st.gates == 900 and st.sweeps >= 10  # the inverse ran as a full plan
    assert mid.real ** 2 + mid.imag ** 2 < 1e-3  # and the state in between was far from |0...0>
    if single:
        assert p >= 1 - 1e-6
        assert abs(total - 1.0) <= 1e-5
    else:
        assert abs(p - 1.0) <= 1e-12
        assert abs(total - 1.0) <= 1e-12


def test_bernstein_vazirani_30_qubits(quest, env):
    n = 30
    seed = C.config_seed(2, 1)
    ops = C.bernstein_vazirani(n, seed, measure=True)
    quest.seed([12345, 67890])
    q = quest.createQureg(n, env)
    try:
        out = quest.apply_circuit(q, ops)
    finally:
        quest.destroyQureg(q, env)
    assert out[: n - 1] == [int(b) for b in C.bv_secret(n, seed)]
