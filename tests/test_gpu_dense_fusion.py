"""The dense-block form on the GPU (dgq_setDenseFusion): gates fused into
dense K-qubit unitaries, each one dense sweep. complex128 runs the SIMT
dense kernel (max amplitude error <= 1e-12 against the oracle, |1 - norm|
<= 1e-12); complex64 with K = 6 runs the tensor-core sweep (fidelity >=
1 - 1e-6, amplitudes within 2e-6)."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def run(quest, env, n, ops, k, single):
    q = quest.dgq_createQuregF32(n, env) if single else quest.createQureg(n, env)
    try:
        assert quest.dgq_setDenseFusion(q, k) == -1  # the default: the predictor chooses
        quest.initZeroState(q)
        C.replay(q, ops)
        amps = quest.state_vector(q)
        st = quest.plan_stats(q)
        norm = quest.calcTotalProb(q)
    finally:
        quest.destroyQureg(q, env)
    return amps, st, norm


@pytest.mark.parametrize("k", [5, 6, 7])
def test_complex128_dense_blocks(quest, env, k):
    n = 16
    ops = C.random_layers(n, 10, C.config_seed(2, 70 + k))
    amps, st, norm = run(quest, env, n, ops, k, False)
    ref = oracle.run(n, ops)[0]
    assert st.denseBlocks >= 1 and st.sweeps == st.denseBlocks + 1  # + the pass that initialises |0...0>
    assert np.abs(amps - ref).max() <= 1e-12
    assert abs(norm - 1.0) <= 1e-12


@pytest.mark.parametrize("kind", ["random", "grid"])
def test_complex64_tensor_core_blocks(quest, env, kind):
    n = 16
    ops = (C.random_layers(n, 12, C.config_seed(2, 80)) if kind == "random"
           else C.grid_sqrt(4, 4, 10, C.config_seed(3, 80)))
    amps, st, norm = run(quest, env, n, ops, 6, True)
    ref = oracle.run(n, ops)[0]
    assert st.denseBlocks >= 4
    # + the pass that initialises |0...0> and the closing renormalisation pass
    assert st.sweeps == st.denseBlocks + 2
    assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6
    assert abs(norm - 1.0) <= 1e-5
    assert quest.dgq_getDeviceErrors() == 0


def test_dense_fusion_argument_checks(quest, env):
    q = quest.createQureg(12, env)
    try:
        with pytest.raises(quest.QuESTError):
            quest.dgq_setDenseFusion(q, 4)
        assert quest.dgq_setDenseFusion(q, 6) == -1
        assert quest.dgq_setDenseFusion(q, 0) == 6
        assert quest.dgq_setDenseFusion(q, -1) == 0
    finally:
        quest.destroyQureg(q, env)


def test_form_choice_takes_dense_blocks_when_cheaper(quest, env):
    """With dense rates that make 6-qubit blocks cheap, the default form
    choice fuses the circuit into dense blocks: the same result as forcing
    that form, and the oracle's amplitudes (complex128, 1e-12)."""
    Q = quest
    keys = [(v, k) for v in range(3) for k in (5, 6, 7)]
    prev = {key: Q.dgq_getDenseCost(*key) for key in keys}
    n = 22  # large enough that a block's launch overhead (3 us) does not decide
    ops = C.random_layers(n, 6, C.config_seed(2, 777))
    try:
        for k in (5, 7):
            Q.dgq_setDenseCost(0, k, 1e3)
        Q.dgq_setDenseCost(0, 6, 1e-3)
        out = {}
        for name, fusion in (("auto", -1), ("forced", 6)):
            q = Q.createQureg(n, env)
            Q.dgq_setDenseFusion(q, fusion)
            C.replay(q, ops)
            Q.dgq_planPending(q)
            st = Q.plan_stats(q)
            Q.dgq_launchPlanned(q)
            out[name] = (Q.state_vector(q), st.formK, st.formAuto, st.denseBlocks)
            Q.destroyQureg(q, env)
        assert out["auto"][1:] == (6, 1, out["forced"][3]) and out["forced"][3] > 0
        assert np.abs(out["auto"][0] - out["forced"][0]).max() == 0.0
        ref, _, _ = oracle.run(n, ops)
        assert np.abs(out["auto"][0] - ref).max() <= 1e-12
    finally:
        for key, r in prev.items():
            Q.dgq_setDenseCost(*key, r)
