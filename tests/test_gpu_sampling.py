"""dgq_sampleOutcomes against the oracle's probabilities.

A sample with uniform u must be the first index whose cumulative
probability exceeds u x total: checked against the oracle's exact
cumulative sums with a slack of 1e-12 (complex128) or 2e-6 (complex64) for
registers in logical order (no swapGate). Registers with relabelled qubits
and collapsed registers are checked for support and frequencies."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def uniforms(seed, count):
    # MT19937 init_genrand(seed), 53-bit draws: numpy's RandomState yields the same sequence
    return np.random.RandomState(seed).random_sample(count)


def check_cdf(samples, probs, u, slack):
    cdf = np.cumsum(probs)
    t = u * cdf[-1]
    for i, tk in zip(samples.astype(np.int64), t):
        lo = cdf[i - 1] if i > 0 else 0.0
        assert lo <= tk + slack and cdf[i] >= tk - slack and probs[i] > 0


@pytest.mark.parametrize("n,single", [(9, False), (12, False), (15, False), (13, True), (16, True)])
def test_samples_follow_exact_cdf(quest, env, n, single):
    Q = quest
    ops = C.random_layers(n, 6, C.config_seed(5, 700 + n))
    q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
    Q.apply_circuit(q, ops)
    s1 = Q.sample(q, 1024, 1234 + n)
    s2 = Q.sample(q, 1024, 1234 + n)
    assert np.array_equal(s1, s2)  # deterministic for a state and a seed
    ref, _, _ = oracle.run(n, ops)
    check_cdf(s1, np.abs(ref) ** 2, uniforms(1234 + n, 1024), 2e-6 if single else 1e-12)
    Q.destroyQureg(q, env)


def test_samples_with_relabelled_qubits(quest, env):
    """GHZ+QFT ends with swaps (relabelled, not moved): outcomes are logical
    indices with the right support and frequencies."""
    Q = quest
    n = 10
    ops = C.ghz_qft(n)
    q = Q.createQureg(n, env)
    Q.apply_circuit(q, ops)
    s = Q.sample(q, 4096, 99)
    ref, _, _ = oracle.run(n, ops)
    p = np.abs(ref) ** 2
    assert np.all(p[s.astype(np.int64)] > 1e-15)
    freq = np.bincount(s.astype(np.int64), minlength=1 << n) / len(s)
    assert np.abs(freq - p).max() < 0.03
    Q.destroyQureg(q, env)


def test_samples_after_collapse(quest, env):
    Q = quest
    n = 12
    q = Q.createQureg(n, env)
    Q.apply_circuit(q, C.random_layers(n, 4, 5))
    Q.collapseToOutcome(q, 3, 1)
    s = Q.sample(q, 512, 7)
    assert np.all((s >> np.uint64(3)) & np.uint64(1) == 1)
    Q.destroyQureg(q, env)


def test_bv_samples_are_the_secret(quest, env):
    Q = quest
    for n, single in [(20, False), (22, True)]:
        ops = C.bernstein_vazirani(n, C.config_seed(5, 3), measure=False)
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        Q.apply_circuit(q, ops)
        s = Q.sample(q, 64, 1)
        bits = C.bv_secret(n, C.config_seed(5, 3))
        secret = sum(b << i for i, b in enumerate(bits))
        mask = (1 << (n - 1)) - 1
        assert np.all((s.astype(np.int64) & mask) == secret)
        Q.destroyQureg(q, env)
