"""The host tier: registers larger than the device budget keep their state
in pinned host memory and stream it through the GPU a page at a time.

A small device budget (1 MiB: four page buffers of 2^14 complex128
amplitudes) puts registers of 16..20 qubits in the host tier, so gates on
the qubits above the page need page-pair exchanges. Tolerances as in HBM:
complex128 amplitudes within 1e-12 of the oracle, P(q = 0) within 1e-12,
measurement outcomes bit-exact for a fixed seed; complex64 fidelity
>= 1 - 1e-6."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu

BUDGET = 1 << 20


@pytest.fixture
def small_budget(quest):
    prev = quest.dgq_setDeviceBudget(BUDGET)
    yield
    quest.dgq_setDeviceBudget(prev)


@pytest.fixture(params=["interpreted", "specialised"])
def kernels(request, quest):
    prev = quest.dgq_setSpecialisationMinBits(14 if request.param == "specialised" else 40)
    yield request.param
    quest.dgq_setSpecialisationMinBits(prev)


@pytest.mark.parametrize("kind", ["random", "ghzqft", "mixed"])
def test_host_tier_matches_oracle(quest, env, small_budget, kernels, kind):
    n = 20 if kind != "mixed" else 17
    ops = {"random": lambda: C.random_layers(n, 8, C.config_seed(2, 90)),
           "ghzqft": lambda: C.ghz_qft(n),
           "mixed": lambda: C.mixed_ops(n, 400, 91)}[kind]()
    q = quest.createQureg(n, env)
    try:
        pb, _, _, _ = quest.host_tier_stats(q)
        assert pb == 14
        quest.initZeroState(q)
        C.replay(q, ops)
        amps = quest.state_vector(q)
        p0 = quest.prob_all_zero(q)
        total = quest.calcTotalProb(q)
        _, passes, exchanges, moved = quest.host_tier_stats(q)
    finally:
        quest.destroyQureg(q, env)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
    assert abs(total - 1.0) <= 1e-12
    assert passes >= 2 and moved > 0
    if kind != "ghzqft":
        assert exchanges >= 1  # gates on the qubits above the page


def test_host_tier_measurement_bit_exact(quest, env, small_budget):
    n = 17
    ops = C.bernstein_vazirani(n, C.config_seed(2, 92), measure=True)
    quest.seed([12345, 67890])
    q = quest.createQureg(n, env)
    try:
        assert quest.host_tier_stats(q) is not None
        out = C.replay(q, ops)
        # the collapsed state is the measured basis state
        amp = quest.getAmp(q, sum(int(b) << k for k, b in enumerate(out)))
    finally:
        quest.destroyQureg(q, env)
    _, _, ref_out = oracle.run(n, ops, seed_keys=[12345, 67890])
    assert out == ref_out
    secret = C.bv_secret(n, C.config_seed(2, 92))
    assert out[: n - 1] == [int(b) for b in secret[: n - 1]]
    assert abs(abs(complex(amp.real, amp.imag)) - 1.0) <= 1e-12


def test_host_tier_complex64(quest, env, small_budget):
    n = 18
    ops = C.random_layers(n, 10, C.config_seed(2, 93))
    quest.dgq_setSpecialisationMinBits(14)
    try:
        q = quest.dgq_createQuregF32(n, env)
        assert quest.host_tier_stats(q) is not None
        quest.initZeroState(q)
        C.replay(q, ops)
        amps = quest.state_vector(q)
        quest.destroyQureg(q, env)
    finally:
        quest.dgq_setSpecialisationMinBits(-1)
    ref = oracle.run(n, ops)[0]
    assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6


def test_host_tier_unsupported_calls(quest, env, small_budget):
    q = quest.createQureg(17, env)
    try:
        assert quest.host_tier_stats(q) is not None
        quest.hadamard(q, 16)
        with pytest.raises(quest.QuESTError):
            quest.sample(q, 4, 1)
        with pytest.raises(quest.QuESTError):
            quest.Batch([q])
        assert abs(quest.calcProbOfOutcome(q, 16, 0) - 0.5) <= 1e-12
    finally:
        quest.destroyQureg(q, env)
    # registers within the budget stay in HBM
    small = quest.createQureg(16, env)
    assert quest.host_tier_stats(small) is None
    quest.destroyQureg(small, env)


def test_host_tier_measurement_mid_circuit(quest, env, small_budget):
    """Measurements between gate batches: each collapse stays lazy until the
    next pass, which applies it before any qubit exchange; probabilities of
    qubits above the page read the collapsed pages only."""
    n = 18
    kinds = [k for k in range(C.CY + 1) if k not in (C.SWAP,)]
    ops = C.mixed_ops(n, 260, 95, kinds=kinds, with_measure=True)
    quest.seed([7, 8])
    q = quest.createQureg(n, env)
    try:
        out = C.replay(q, ops)
        amps = quest.state_vector(q)
        p0 = quest.prob_all_zero(q)
        _, _, exchanges, _ = quest.host_tier_stats(q)
    finally:
        quest.destroyQureg(q, env)
    ref, ref_p0, ref_out = oracle.run(n, ops, seed_keys=[7, 8])
    assert out == ref_out
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
    assert exchanges >= 1


def test_host_tier_collapse_before_exchange(quest, env, small_budget):
    """A measurement followed at once by a gate on a page-index qubit: the
    pending collapse is applied before the page exchange moves its bit."""
    n = 17
    page = 14  # qubits below this one are in the page; the highest of them is the first to leave
    b = C.OpList()
    for k in range(page):
        b.add(C.H, k)
    b.add(C.RY, page - 1, p=[0.7]).add(C.CNOT, page - 1, 2)
    # the measurement runs the gates above without an exchange; the next gate
    # then exchanges qubit n - 1 with the measured qubit's bit
    b.add(C.MEASURE, page - 1).add(C.H, n - 1).add(C.RX, n - 2, p=[0.4]).add(C.MEASURE, n - 1).add(C.H, n - 1)
    ops = b.array()
    quest.seed([3, 4])
    q = quest.createQureg(n, env)
    try:
        assert quest.host_tier_stats(q) is not None
        out = C.replay(q, ops)
        amps = quest.state_vector(q)
    finally:
        quest.destroyQureg(q, env)
    ref, _, ref_out = oracle.run(n, ops, seed_keys=[3, 4])
    assert out == ref_out
    assert np.abs(amps - ref).max() <= 1e-12


def test_host_tier_skips_all_zero_pages(quest, env, small_budget):
    """After initZeroState only page 0 holds amplitudes; gates inside the
    page keep the other pages all-zero, so the pass moves page 0 alone, an
    exchange brings in only the non-zero page of each pair, and the
    read-outs see zeros in the pages never written (dgQuEST's all-zero
    pages, OPTIMIZE_ZERO). Amplitudes within 1e-12 of the oracle."""
    n, page = 18, 14
    b = C.OpList()
    for k in range(page):
        b.add(C.H, k)
    b.add(C.CNOT, 0, 5).add(C.RY, 3, p=[0.3])
    ops1 = b.array()
    ops2 = C.OpList().add(C.H, n - 1).add(C.CNOT, n - 1, 2).array()  # one exchange, then more gates
    q = quest.createQureg(n, env)
    try:
        pb, _, _, _ = quest.host_tier_stats(q)
        assert pb == page
        page_bytes = 16 << page
        quest.initZeroState(q)
        C.replay(q, ops1)
        quest.getAmp(q, 0)  # runs the first pass
        _, _, _, moved1 = quest.host_tier_stats(q)
        assert moved1 == page_bytes  # page 0 copied out; the other 15 pages skipped
        a_far = quest.getAmp(q, (1 << n) - 1)
        assert a_far.real == 0.0 and a_far.imag == 0.0
        C.replay(q, ops2)
        amps = quest.state_vector(q)
        p0 = quest.prob_all_zero(q)
        _, _, exchanges, moved2 = quest.host_tier_stats(q)
    finally:
        quest.destroyQureg(q, env)
    assert exchanges >= 1
    # the exchange brought in one non-zero page per non-zero pair, not every page
    assert moved2 - moved1 < 2 * (16 << n)
    ops = np.concatenate([ops1, ops2])
    ref, ref_p0, _ = oracle.run(n, ops)
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
