"""Sharded registers: the state split into 2^shardBits shards held in HBM
(here all on the one device of the test box, so the exchanges run through
local memory; on several devices the same kernels use peer memory).

Gates on the shard-index qubits need shard-pair exchanges. Tolerances as in
HBM: complex128 amplitudes within 1e-12 of the oracle, P(q = 0) within
1e-12, measurement outcomes bit-exact for a fixed seed; complex64 fidelity
>= 1 - 1e-6."""
import ctypes

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["interpreted", "specialised"])
def kernels(request, quest):
    prev = quest.dgq_setSpecialisationMinBits(14 if request.param == "specialised" else 40)
    yield request.param
    quest.dgq_setSpecialisationMinBits(prev)


@pytest.mark.parametrize("shard_bits", [1, 2, 3])
@pytest.mark.parametrize("kind", ["random", "ghzqft", "mixed"])
def test_shards_match_oracle(quest, env, kernels, kind, shard_bits):
    n = 19 if kind != "mixed" else 17
    ops = {"random": lambda: C.random_layers(n, 8, C.config_seed(2, 120)),
           "ghzqft": lambda: C.ghz_qft(n),
           "mixed": lambda: C.mixed_ops(n, 400, 121)}[kind]()
    q = quest.create_sharded(n, env, shard_bits)
    try:
        sb, _, _, _ = quest.shard_stats(q)
        assert sb == shard_bits
        C.replay(q, ops)
        amps = quest.state_vector(q)
        p0 = quest.prob_all_zero(q)
        total = quest.calcTotalProb(q)
        _, passes, exchanges, moved = quest.shard_stats(q)
    finally:
        quest.destroyQureg(q, env)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
    assert abs(total - 1.0) <= 1e-12
    assert passes >= 1
    # an exchange of m qubits moves 1 - 2^-m of the state between shards
    state = 16 << n
    assert exchanges * state // 2 <= moved <= exchanges * state
    if kind != "ghzqft":
        assert exchanges >= 1  # gates on the shard-index qubits


def test_shards_agree_with_hbm_register(quest, env):
    """A 24-qubit random circuit in 8 shards against the same circuit in one
    HBM buffer (both on the GPU; different sweep groupings round apart)."""
    n = 24
    ops = C.random_layers(n, 12, C.config_seed(2, 122))
    a = quest.createQureg(n, env)
    b = quest.create_sharded(n, env, 3)
    try:
        for q in (a, b):
            C.replay(q, ops)
        va, vb = quest.state_vector(a), quest.state_vector(b)
        pa, pb = quest.prob_all_zero(a), quest.prob_all_zero(b)
        _, _, exchanges, moved = quest.shard_stats(b)
    finally:
        quest.destroyQureg(a, env)
        quest.destroyQureg(b, env)
    assert np.abs(va - vb).max() <= 1e-12
    assert np.abs(pa - pb).max() <= 1e-12
    state = 16 << n
    assert exchanges >= 1 and exchanges * state // 2 <= moved <= exchanges * state


def test_shards_measurement_bit_exact(quest, env):
    n = 17
    ops = C.bernstein_vazirani(n, C.config_seed(2, 123), measure=True)
    quest.seed([12345, 67890])
    q = quest.create_sharded(n, env, 2)
    try:
        out = C.replay(q, ops)
        amp = quest.getAmp(q, sum(int(b) << k for k, b in enumerate(out)))
    finally:
        quest.destroyQureg(q, env)
    _, _, ref_out = oracle.run(n, ops, seed_keys=[12345, 67890])
    assert out == ref_out
    secret = C.bv_secret(n, C.config_seed(2, 123))
    assert out[: n - 1] == [int(b) for b in secret[: n - 1]]
    assert abs(abs(complex(amp.real, amp.imag)) - 1.0) <= 1e-12


def test_shards_measurement_mid_circuit(quest, env):
    n = 18
    kinds = [k for k in range(C.CY + 1) if k not in (C.SWAP,)]
    ops = C.mixed_ops(n, 260, 124, kinds=kinds, with_measure=True)
    quest.seed([7, 8])
    q = quest.create_sharded(n, env, 3)
    try:
        out = C.replay(q, ops)
        amps = quest.state_vector(q)
        p0 = quest.prob_all_zero(q)
        _, _, exchanges, _ = quest.shard_stats(q)
    finally:
        quest.destroyQureg(q, env)
    ref, ref_p0, ref_out = oracle.run(n, ops, seed_keys=[7, 8])
    assert out == ref_out
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
    assert exchanges >= 1


def test_shards_collapse_before_exchange(quest, env):
    """A measurement followed at once by a gate on a shard-index qubit: the
    pending collapse is applied in the address bits it was recorded in,
    before the exchange moves them."""
    n = 17
    page = n - 2  # qubits below this one are in the page; the highest of them is the first to leave
    b = C.OpList()
    for k in range(page):
        b.add(C.H, k)
    b.add(C.RY, page - 1, p=[0.7]).add(C.CNOT, page - 1, 2)
    # the measurement runs the gates above without an exchange; the next gate
    # then exchanges qubit n - 1 with the measured qubit's bit
    b.add(C.MEASURE, page - 1).add(C.H, n - 1).add(C.RX, n - 2, p=[0.4]).add(C.MEASURE, n - 1).add(C.H, n - 1)
    ops = b.array()
    quest.seed([3, 4])
    q = quest.create_sharded(n, env, 2)
    try:
        out = C.replay(q, ops)
        amps = quest.state_vector(q)
        _, _, exchanges, _ = quest.shard_stats(q)
    finally:
        quest.destroyQureg(q, env)
    ref, _, ref_out = oracle.run(n, ops, seed_keys=[3, 4])
    assert out == ref_out
    assert np.abs(amps - ref).max() <= 1e-12
    assert exchanges >= 1


def test_shards_complex64(quest, env):
    n = 18
    ops = C.random_layers(n, 10, C.config_seed(2, 125))
    quest.dgq_setSpecialisationMinBits(14)
    try:
        q = quest.create_sharded(n, env, 2, single=True)
        assert quest.dgq_getPrecision(q) == 1
        C.replay(q, ops)
        amps = quest.state_vector(q)
        quest.destroyQureg(q, env)
    finally:
        quest.dgq_setSpecialisationMinBits(-1)
    ref = oracle.run(n, ops)[0]
    assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6


def test_shards_state_calls(quest, env):
    """initStateFromAmps, setAmps (after swapGate relabels and exchanges),
    getAmp and cloneQureg on sharded registers; exact: no arithmetic."""
    n = 16
    rng = np.random.default_rng(5)
    vals = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    vals /= np.linalg.norm(vals)
    D = ctypes.POINTER(ctypes.c_double)
    re, im = np.ascontiguousarray(vals.real), np.ascontiguousarray(vals.imag)
    a = quest.create_sharded(n, env, 2)
    b = quest.create_sharded(n, env, 2)
    try:
        quest.initStateFromAmps(a, re.ctypes.data_as(D), im.ctypes.data_as(D))
        assert np.array_equal(quest.state_vector(a), vals)
        quest.swapGate(a, 0, n - 1)  # a relabel, then an exchange moves qubit 15 into the shard
        quest.hadamard(a, 0)
        quest.hadamard(a, 0)
        got = quest.state_vector(a)
        want = vals.reshape([2] * n)
        want = np.swapaxes(want, 0, n - 1).reshape(-1)  # axis 0 is qubit n - 1
        assert np.abs(got - want).max() <= 1e-15
        start, count = 1000, 5000
        sub = rng.normal(size=count) + 1j * rng.normal(size=count)
        sre, sim = np.ascontiguousarray(sub.real), np.ascontiguousarray(sub.imag)
        quest.setAmps(a, start, sre.ctypes.data_as(D), sim.ctypes.data_as(D), count)
        want = got.copy()
        want[start:start + count] = sub
        assert np.array_equal(quest.state_vector(a), want)
        c = quest.getAmp(a, 40000)
        assert complex(c.real, c.imag) == want[40000]
        quest.cloneQureg(b, a)
        assert np.array_equal(quest.state_vector(b), want)
        other = quest.create_sharded(n, env, 1)
        with pytest.raises(quest.QuESTError):
            quest.cloneQureg(other, a)
        quest.destroyQureg(other, env)
    finally:
        quest.destroyQureg(a, env)
        quest.destroyQureg(b, env)


def test_shards_unsupported_and_invalid(quest, env):
    q = quest.create_sharded(16, env, 1)
    try:
        quest.hadamard(q, 15)
        with pytest.raises(quest.QuESTError):
            quest.sample(q, 4, 1)
        with pytest.raises(quest.QuESTError):
            quest.Batch([q])
        with pytest.raises(quest.QuESTError):
            quest.dgq_getDeviceState(q, None)
        assert abs(quest.calcProbOfOutcome(q, 15, 0) - 0.5) <= 1e-12
    finally:
        quest.destroyQureg(q, env)
    for n, sb in [(16, 0), (16, 5), (15, 2)]:  # shard bits 1..4, >= 14 qubits a shard
        with pytest.raises(quest.QuESTError):
            quest.create_sharded(n, env, sb)
    with pytest.raises(quest.QuESTError):
        quest.create_sharded(16, env, 1, devices=[0, 4096])
    plain = quest.createQureg(16, env)
    assert quest.shard_stats(plain) is None
    quest.destroyQureg(plain, env)
