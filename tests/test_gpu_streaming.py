"""Sweeps launched while the rest of the circuit is still being planned.

When every sweep kernel of a plan is compiled already, executing pending
gates launches sweep i as soon as sweeps i+1 and i+2 are planned. The
launched programs are the ones a complete plan holds, so the streamed run
must equal a replay of the complete plan bit for bit, and the oracle within
the usual tolerances (complex128: 1e-12 per amplitude; complex64: fidelity
>= 1 - 1e-6, amplitudes within 2e-6)."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


@pytest.fixture
def specialise_small(quest):
    prev = quest.dgq_setSpecialisationMinBits(14)
    yield
    quest.dgq_setSpecialisationMinBits(prev)


@pytest.mark.parametrize("single", [False, True])
def test_streamed_run_equals_plan_replay_and_oracle(quest, env, specialise_small, single):
    n = 18
    ops = C.random_layers(n, 16, C.config_seed(2, 880 + int(single)))
    q = quest.dgq_createQuregF32(n, env) if single else quest.createQureg(n, env)
    try:
        quest.initZeroState(q)
        C.replay(q, ops)
        quest.getAmp(q, 0)  # first run: the sweep kernels are compiled
        quest.initZeroState(q)
        C.replay(q, ops)
        streamed = quest.state_vector(q)
        st = quest.plan_stats(q)
        assert st.sweeps >= 4
        assert st.streamedSweeps == st.sweeps - 2
        # the same gates planned completely first, then launched
        quest.initZeroState(q)
        C.replay(q, ops)
        assert quest.dgq_planPending(q) == 0
        assert quest.plan_stats(q).streamedSweeps == 0
        assert quest.dgq_launchPlanned(q) == 0
        replayed = quest.state_vector(q)
        assert np.array_equal(streamed, replayed)
    finally:
        quest.destroyQureg(q, env)
    ref = oracle.run(n, ops)[0]
    if single:
        assert abs(np.vdot(ref, streamed)) ** 2 >= 1 - 1e-6
        assert np.abs(streamed - ref).max() <= 2e-6
    else:
        assert np.abs(streamed - ref).max() <= 1e-12


def test_uncompiled_structure_waits_for_the_plan(quest, env, specialise_small):
    """From the first sweep whose kernel is not compiled yet, nothing more is
    launched while planning: the missing kernels are compiled together once
    the plan is complete, then the remaining sweeps run."""
    n = 17
    ops = C.random_layers(n, 10, C.config_seed(2, 890))
    q = quest.createQureg(n, env)
    try:
        C.replay(q, ops)
        amps = quest.state_vector(q)
        st = quest.plan_stats(q)
        assert st.jitCompiled > 0
        assert st.streamedSweeps <= st.sweeps - 2
    finally:
        quest.destroyQureg(q, env)
    ref = oracle.run(n, ops)[0]
    assert np.abs(amps - ref).max() <= 1e-12


def test_first_cuda_work_of_a_thread_is_a_specialised_launch(quest, env, specialise_small):
    """A host thread whose first CUDA work is loading and launching a
    specialised kernel (a register created on another thread) gets the
    device's primary context bound before the driver calls."""
    import threading
    n = 16
    ops = C.random_layers(n, 6, C.config_seed(2, 886))
    q = quest.createQureg(n, env)
    result = {}

    def run():
        try:
            C.replay(q, ops)
            result["amps"] = quest.state_vector(q)
        except Exception as exc:  # noqa: BLE001
            result["error"] = exc

    try:
        t = threading.Thread(target=run)
        t.start()
        t.join()
    finally:
        quest.destroyQureg(q, env)
    assert "error" not in result, result.get("error")
    ref = oracle.run(n, ops)[0]
    assert np.abs(result["amps"] - ref).max() <= 1e-12
