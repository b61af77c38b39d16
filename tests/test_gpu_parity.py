"""GPU parity: the product (libdgq.so through the QuEST C API) against the
oracle on the same op lists and seeds. Tolerance: 1e-12 max abs error per
amplitude and per P(q=0); measurement outcomes bit-exact."""
import math

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_product(Q, env, n, ops, seed_keys=None, tile_bits=0):
    q = Q.createQureg(n, env)
    if tile_bits:
        Q.dgq_setTileBits(q, tile_bits)
    if seed_keys is not None:
        Q.seed(seed_keys)
    out = C.replay(q, ops)
    amps = Q.state_vector(q)
    p0 = Q.prob_all_zero(q)
    stats = Q.plan_stats(q)
    Q.destroyQureg(q, env)
    return amps, p0, out, stats


def check(amps, p0, ref_amps, ref_p0):
    assert np.abs(amps - ref_amps).max() <= TOL
    assert np.abs(p0 - ref_p0).max() <= TOL


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 9, 10, 12, 14])
def test_mixed_ops_every_call(quest, env, n):
    ops = C.mixed_ops(max(n, 2), 400, 1000 + n) if n > 1 else C.OpList().add(C.H, 0).add(C.RX, 0, p=(0.3,)).add(
        C.T, 0).add(C.SQW, 0).add(C.RZ, 0, p=(1.1,)).array()
    if n == 1:
        pass
    amps, p0, _, _ = run_product(quest, env, n, ops)
    ref_amps, ref_p0, _ = oracle.run(n, ops)
    check(amps, p0, ref_amps, ref_p0)


@pytest.mark.parametrize("tile_bits", [9, 10, 11, 12])
def test_random_layers_every_tile_width(quest, env, tile_bits):
    n = 16
    ops = C.random_layers(n, 10, C.config_seed(2, tile_bits))
    amps, p0, _, st = run_product(quest, env, n, ops, tile_bits=tile_bits)
    assert st.tileBits == tile_bits
    ref_amps, ref_p0, _ = oracle.run(n, ops)
    check(amps, p0, ref_amps, ref_p0)


def test_ghz_qft_with_swap_network(quest, env):
    n = 14
    ops = C.ghz_qft(n)
    amps, p0, _, _ = run_product(quest, env, n, ops)
    ref_amps, ref_p0, _ = oracle.run(n, ops)
    check(amps, p0, ref_amps, ref_p0)


def test_bv_measurement_is_bit_exact(quest, env):
    n = 13
    ops = C.bernstein_vazirani(n, C.config_seed(2, 7), measure=True)
    amps, p0, out, _ = run_product(quest, env, n, ops, seed_keys=[12345, 67890])
    ref_amps, ref_p0, ref_out = oracle.run(n, ops, seed_keys=[12345, 67890])
    assert out == ref_out
    assert out[:n - 1] == C.bv_secret(n, C.config_seed(2, 7))
    check(amps, p0, ref_amps, ref_p0)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_measurements_match_oracle(quest, env, seed):
    n = 11
    ops = np.concatenate([C.mixed_ops(n, 150, seed), C.OpList().add(C.MEASURE, 4).add(C.MEASURE, 0).array(),
                          C.mixed_ops(n, 80, seed + 50),
                          C.OpList().add(C.MEASURE, 10).add(C.MEASURE, 4).add(C.MEASURE, 7).array()])
    keys = [seed, 777]
    amps, p0, out, _ = run_product(quest, env, n, ops, seed_keys=keys)
    ref_amps, ref_p0, ref_out = oracle.run(n, ops, seed_keys=keys)
    assert out == ref_out
    check(amps, p0, ref_amps, ref_p0)


@pytest.mark.parametrize("targs", [[3, 0], [1, 6, 4], [0, 9, 2, 5], [10, 11, 12, 13]])
def test_multi_qubit_unitary(quest, env, targs):
    n = 14
    gen = np.random.default_rng(len(targs))
    u = C.random_unitary(gen, 1 << len(targs))
    pre = C.mixed_ops(n, 60, 3)
    post = C.mixed_ops(n, 60, 4)
    q = quest.createQureg(n, env)
    C.replay(q, pre)
    m = quest.matrixN(u)
    quest.multiQubitUnitary(q, quest.int_array(targs), len(targs), m)
    quest.destroyComplexMatrixN(m)
    C.replay(q, post)
    amps = quest.state_vector(q)
    quest.destroyQureg(q, env)
    o = oracle.Oracle(n)
    o.apply(pre)
    o.multi_qubit_unitary(targs, u)
    o.apply(post)
    assert np.abs(amps - o.amps()).max() <= TOL


def test_init_variants_and_readouts(quest, env):
    n = 12
    ops = C.mixed_ops(n, 100, 21)
    gen = np.random.default_rng(5)
    psi = gen.standard_normal(1 << n) + 1j * gen.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    q = quest.createQureg(n, env)
    for mode in ("plus", "classical", "amps"):
        o = oracle.Oracle(n)
        if mode == "plus":
            quest.initPlusState(q)
            o.init_plus()
        elif mode == "classical":
            quest.initClassicalState(q, 1234)
            o.init_classical(1234)
        else:
            quest.init_from_amps(q, psi)
            o.set_amps(psi)
        C.replay(q, ops)
        o.apply(ops)
        ref = o.amps()
        assert np.abs(quest.state_vector(q) - ref).max() <= TOL
        for idx in (0, 1, 77, (1 << n) - 1):
            a = quest.getAmp(q, idx)
            assert abs(complex(a.real, a.imag) - ref[idx]) <= TOL
            assert quest.getProbAmp(q, idx) == pytest.approx(abs(ref[idx]) ** 2, abs=TOL)
        assert quest.calcTotalProb(q) == pytest.approx(1.0, abs=TOL)
        for k in range(n):
            assert quest.calcProbOfOutcome(q, k, 1) == pytest.approx(1 - o.prob_zero_all()[k], abs=TOL)
    quest.destroyQureg(q, env)


def test_collapse_to_outcome(quest, env):
    n = 10
    ops = C.mixed_ops(n, 120, 8)
    q = quest.createQureg(n, env)
    C.replay(q, ops)
    o = oracle.Oracle(n)
    o.apply(ops)
    p1 = 1 - o.prob_zero_all()[3]
    got = quest.collapseToOutcome(q, 3, 1)
    assert got == pytest.approx(p1, abs=TOL)
    oracle.lib().orc_collapse(o.ptr, 3, 1, p1)
    assert np.abs(quest.state_vector(q) - o.amps()).max() <= TOL
    # gates after the collapse see the collapsed state
    more = C.mixed_ops(n, 50, 9)
    C.replay(q, more)
    o.apply(more)
    assert np.abs(quest.state_vector(q) - o.amps()).max() <= TOL
    quest.destroyQureg(q, env)


def test_invalid_input_raises_quest_error(quest, env):
    q = quest.createQureg(5, env)
    with pytest.raises(quest.QuESTError) as ei:
        quest.hadamard(q, 5)
    assert ei.value.code == 2  # E_INVALID_TARGET_QUBIT
    with pytest.raises(quest.QuESTError) as ei:
        quest.controlledNot(q, 1, 1)
    assert ei.value.code == 7  # E_TARGET_IS_CONTROL
    with pytest.raises(quest.QuESTError) as ei:
        quest.unitary(q, 0, quest.mat2([[1, 1], [0, 1]]))
    assert ei.value.code == 11  # E_NON_UNITARY_MATRIX
    with pytest.raises(quest.QuESTError):
        quest.getAmp(q, 32)
    with pytest.raises(quest.QuESTError):
        quest.calcProbOfOutcome(q, 0, 2)
    quest.destroyQureg(q, env)


def test_plan_fuses_and_counts(quest, env):
    n = 20
    ops = C.random_layers(n, 6, 3)
    q = quest.createQureg(n, env)
    C.replay(q, ops)
    quest.dgq_sync(q)
    st = quest.plan_stats(q)
    assert 1 <= st.sweeps < 6 * n
    assert st.gates <= len(ops)
    assert st.numBits == n
    quest.destroyQureg(q, env)


@pytest.fixture
def specialised(quest):
    prev = quest.dgq_setSpecialisationMinBits(1)
    yield
    quest.dgq_setSpecialisationMinBits(prev)


@pytest.mark.parametrize("tile_bits", [9, 10, 11, 12])
def test_specialised_kernels_match_oracle(quest, env, specialised, tile_bits):
    n = 15
    ops = np.concatenate([C.mixed_ops(n, 250, 500 + tile_bits), C.random_layers(n, 4, 7)])
    amps, p0, _, st = run_product(quest, env, n, ops, tile_bits=tile_bits)
    assert st.jitCompiled + st.jitReused == st.sweeps
    ref_amps, ref_p0, _ = oracle.run(n, ops)
    check(amps, p0, ref_amps, ref_p0)


def test_specialised_dense_and_measure(quest, env, specialised):
    n = 13
    gen = np.random.default_rng(11)
    u = C.random_unitary(gen, 16)
    pre = C.mixed_ops(n, 80, 12)
    post = np.concatenate([C.mixed_ops(n, 80, 13), C.OpList().add(C.MEASURE, 2).add(C.MEASURE, 9).array()])
    q = quest.createQureg(n, env)
    quest.seed([5, 6])
    C.replay(q, pre)
    m = quest.matrixN(u)
    quest.multiQubitUnitary(q, quest.int_array([1, 7, 3, 12]), 4, m)
    quest.destroyComplexMatrixN(m)
    out = C.replay(q, post)
    amps = quest.state_vector(q)
    st = quest.plan_stats(q)
    quest.destroyQureg(q, env)
    o = oracle.Oracle(n)
    o.seed([5, 6])
    o.apply(pre)
    o.multi_qubit_unitary([1, 7, 3, 12], u)
    ref_out = o.apply(post)
    assert out == ref_out
    assert np.abs(amps - o.amps()).max() <= TOL
