"""The batched form (one persistent launch over many registers) against the
oracle and against the same registers run one by one.

Tolerances: complex128 batches match the oracle to 1e-12 per amplitude and
in <Z_q> (FP64 sums); complex64 batches keep fidelity >= 1 - 1e-6 against
the oracle and <Z_q> within 2e-5. The batched and single-register paths run
the same sweep programs, so their complex128 amplitudes agree to 1e-13."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def exp_z(amps, n):
    p = np.abs(amps) ** 2
    idx = np.arange(len(amps))
    return np.array([p[(idx >> q) & 1 == 0].sum() - p[(idx >> q) & 1 == 1].sum() for q in range(n)])


def make_regs(Q, env, sizes, depths, single=False, seed0=0):
    regs, ops_list = [], []
    for i, (n, d) in enumerate(zip(sizes, depths)):
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        Q.initZeroState(q)
        ops = C.hea(n, d, C.config_seed(4, seed0 + i))
        C.replay(q, ops)
        regs.append(q)
        ops_list.append(ops)
    return regs, ops_list


def destroy(Q, env, regs):
    for q in regs:
        Q.destroyQureg(q, env)


SIZES = [9, 10, 12, 13, 14, 16, 11, 15, 10, 13, 12, 17, 9, 14]
DEPTHS = [3, 5, 8, 4, 6, 3, 7, 5, 2, 9, 4, 3, 6, 5]


@pytest.mark.parametrize("config", [None, {"tileBits": 12, "groupFactor": 1},
                                    {"tileBits": 10, "groupFactor": 4}, {"tileBits": 11, "ctasPerSm": 1},
                                    {"tileBits": 9, "groupFactor": 2}])
def test_batch_f64_matches_oracle(quest, env, config):
    Q = quest
    regs, ops_list = make_regs(Q, env, SIZES, DEPTHS, seed0=10)
    b = Q.Batch(regs, config)
    b.launch()
    z = b.expectation_z()
    st = b.stats()
    assert st.registers == len(regs)
    o = 0
    for q, n, ops in zip(regs, SIZES, ops_list):
        ref, ref_p0, _ = oracle.run(n, ops)
        amps = Q.state_vector(q)
        assert np.abs(amps - ref).max() <= 1e-12
        assert np.abs(z[o:o + n] - exp_z(ref, n)).max() <= 1e-12
        # the register API reads the batched result
        assert np.abs(Q.prob_all_zero(q) - ref_p0).max() <= 1e-12
        o += n
    b.close()
    destroy(Q, env, regs)


def test_batch_equals_single_register_runs(quest, env):
    Q = quest
    sizes = [18, 13, 12, 20, 10]
    depths = [6, 9, 12, 4, 30]
    regs, ops_list = make_regs(Q, env, sizes, depths, seed0=40)
    b = Q.Batch(regs, {"tileBits": 12, "groupFactor": 2})
    b.launch()
    b.wait()
    for q, n, ops in zip(regs, sizes, ops_list):
        single = Q.createQureg(n, env)
        Q.initZeroState(single)
        C.replay(single, ops)
        a1 = Q.state_vector(single)
        a2 = Q.state_vector(q)
        assert np.abs(a1 - a2).max() <= 1e-13
        Q.destroyQureg(single, env)
    b.close()
    destroy(Q, env, regs)


def test_batch_relaunch_is_idempotent(quest, env):
    Q = quest
    regs, ops_list = make_regs(Q, env, SIZES[:8], DEPTHS[:8], seed0=70)
    b = Q.Batch(regs, {"tileBits": 11, "groupFactor": 1})
    b.launch()
    z1 = b.expectation_z()
    amps1 = [Q.state_vector(q) for q in regs]
    for _ in range(3):
        b.launch()
    z2 = b.expectation_z()
    # amplitudes repeat bit for bit; <Z> sums are accumulated by atomics in
    # whatever order the CTAs finish, so they repeat to rounding
    assert np.abs(z1 - z2).max() <= 1e-14
    for q, a in zip(regs, amps1):
        assert np.array_equal(Q.state_vector(q), a)
    b.close()
    destroy(Q, env, regs)


def test_batch_f32_fidelity(quest, env):
    Q = quest
    sizes = [10, 12, 14, 16, 13, 11]
    depths = [8, 12, 6, 10, 16, 20]
    regs, ops_list = make_regs(Q, env, sizes, depths, single=True, seed0=90)
    b = Q.Batch(regs)  # autotuned
    b.launch()
    z = b.expectation_z()
    o = 0
    for q, n, ops in zip(regs, sizes, ops_list):
        ref, _, _ = oracle.run(n, ops)
        amps = Q.state_vector(q)
        fid = abs(np.vdot(ref, amps)) ** 2 / np.vdot(amps, amps).real
        assert fid >= 1 - 1e-6
        assert np.abs(z[o:o + n] - exp_z(ref, n)).max() <= 2e-5
        o += n
    b.close()
    destroy(Q, env, regs)


def test_batch_mixed_gates_and_init(quest, env):
    """Every gate kind the op list carries (no measurement), plus |+> and
    classical initial states, through the batch."""
    Q = quest
    regs, refs, sizes = [], [], [11, 13, 14]
    for i, n in enumerate(sizes):
        q = Q.createQureg(n, env)
        ops = C.mixed_ops(n, 200, 500 + i, with_measure=False)
        o = oracle.Oracle(n)
        if i == 0:
            Q.initPlusState(q)
            o.init_plus()
        elif i == 1:
            Q.initClassicalState(q, 4321)
            o.init_classical(4321)
        else:
            Q.initZeroState(q)
            o.init_zero()
        C.replay(q, ops)
        o.apply(ops)
        refs.append(o.amps())
        o.close()
        regs.append(q)
    b = Q.Batch(regs, {"tileBits": 12})
    b.launch()
    z = b.expectation_z()
    off = 0
    for q, n, ref in zip(regs, sizes, refs):
        assert np.abs(Q.state_vector(q) - ref).max() <= 1e-12
        assert np.abs(z[off:off + n] - exp_z(ref, n)).max() <= 1e-12
        off += n
    b.close()
    destroy(Q, env, regs)


def test_batch_rejects_mixed_precision(quest, env):
    Q = quest
    a = Q.createQureg(10, env)
    c = Q.dgq_createQuregF32(10, env)
    with pytest.raises(Q.QuESTError):
        Q.Batch([a, c])
    Q.destroyQureg(a, env)
    Q.destroyQureg(c, env)


def test_apply_circuit_matches_replay(quest, env):
    """dgq_applyCircuit (one call for an op list) records the same calls as
    replaying the list call by call, measurements included."""
    Q = quest
    n = 12
    ops = C.mixed_ops(n, 300, 7, with_measure=True)
    Q.seed([3, 4])
    q1 = Q.createQureg(n, env)
    out1 = C.replay(q1, ops)
    a1 = Q.state_vector(q1)
    Q.seed([3, 4])
    q2 = Q.createQureg(n, env)
    out2 = Q.apply_circuit(q2, ops)
    a2 = Q.state_vector(q2)
    assert out1 == out2
    assert np.array_equal(a1, a2)
    bad = np.zeros(1, dtype=C.OP_DTYPE)
    bad[0]["kind"] = 99
    with pytest.raises(Q.QuESTError):
        Q.apply_circuit(q2, bad)
    Q.destroyQureg(q1, env)
    Q.destroyQureg(q2, env)


@pytest.mark.parametrize("single", [False, True])
def test_batch_with_register_phase_dense_ops(quest, env, single):
    """Registers with multi-qubit unitaries of 2..4 targets (dense ops inside
    a register phase) select the batch kernel form that handles them."""
    Q = quest
    sizes = [10, 13, 12, 15]
    gen = np.random.default_rng(21)
    regs, refs = [], []
    for i, n in enumerate(sizes):
        targs = [[1, 4], [0, 7, 3], [11, 2, 5, 8], [14, 6, 9][: 2 + i % 2]][i]
        u = C.random_unitary(gen, 1 << len(targs))
        pre = C.hea(n, 3, C.config_seed(4, 40 + i))
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        Q.initZeroState(q)
        C.replay(q, pre)
        m = Q.matrixN(u)
        Q.multiQubitUnitary(q, Q.int_array(targs), len(targs), m)
        Q.destroyComplexMatrixN(m)
        post = C.hea(n, 2, C.config_seed(4, 50 + i))
        C.replay(q, post)
        o = oracle.Oracle(n)
        o.apply(pre)
        o.multi_qubit_unitary(targs, u)
        o.apply(post)
        refs.append(o.amps())
        o.close()
        regs.append(q)
    b = Q.Batch(regs)
    b.launch()
    b.wait()
    for q, ref in zip(regs, refs):
        amps = Q.state_vector(q)
        if single:
            assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
        else:
            assert np.abs(amps - ref).max() <= 1e-12
    b.close()
    destroy(Q, env, regs)
