"""Specialisation policy 1 (serving): a plan whose kernels are not compiled
runs the interpreting kernel at once and compiles in the background; a later
plan of the same structure runs specialised. Both give the oracle's result
(1e-12 complex128; complex64 fidelity >= 1 - 1e-6)."""
import time

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("single", [False, True])
def test_cached_only_policy(quest, env, single):
    Q = quest
    prev_bits = Q.dgq_setSpecialisationMinBits(1)
    prev = Q.dgq_setSpecialisationPolicy(1)
    try:
        n = 15
        # a circuit structure no other test plans
        ops = C.random_layers(n, 5, C.config_seed(2, 4242 + int(single)))
        ref, _, _ = oracle.run(n, ops)

        def run():
            q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
            C.replay(q, ops)
            Q.dgq_planPending(q)
            st = Q.plan_stats(q)
            Q.dgq_launchPlanned(q)
            amps = Q.state_vector(q)
            Q.destroyQureg(q, env)
            return st, amps

        st1, a1 = run()
        assert st1.jitCompiled == 0 and st1.jitReused == 0  # interpreted, nothing compiled in the call
        deadline = time.time() + 120
        while True:
            st2, a2 = run()
            if st2.jitReused + st2.jitCompiled == st2.sweeps or time.time() > deadline:
                break
            time.sleep(0.5)
        assert st2.jitReused + st2.jitCompiled == st2.sweeps
        assert st2.jitCompiled == 0  # loaded from the background compiles
        for a in (a1, a2):
            if single:
                assert abs(np.vdot(ref, a)) ** 2 >= 1 - 1e-6
            else:
                assert np.abs(a - ref).max() <= 1e-12
    finally:
        Q.dgq_setSpecialisationPolicy(prev)
        Q.dgq_setSpecialisationMinBits(-1 if prev_bits == 22 else prev_bits)


def test_exit_with_background_compiles_in_flight(quest):
    """A process that exits while background compiles are still queued or
    running (specialisation policy 1) ends cleanly: the binding's exit hook
    stops and joins the compile threads before process teardown."""
    import subprocess
    import sys
    code = """
import sys
sys.path.insert(0, %r)
from dgquest_b200 import quest as Q, circuits as C
env = Q.createQuESTEnv()
Q.dgq_setSpecialisationPolicy(1)
for i in range(6):
    q = Q.createQureg(23, env)
    C.replay(q, C.random_layers(23, 6, 4000 + i))
    Q.getAmp(q, 0)
    Q.destroyQureg(q, env)
print("ok")
""" % (str(__import__("pathlib").Path(__file__).resolve().parents[1]),)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().endswith("ok")


@pytest.mark.parametrize("single", [False, True])
def test_specialise_ahead_of_time(quest, env, single):
    """dgq_specialiseGates (foreground) compiles and loads the kernels a
    register's plan of the same gates uses: the plan then compiles nothing
    and reuses every kernel, with the oracle's result."""
    from dgquest_b200 import ir
    Q = quest
    prev_bits = Q.dgq_setSpecialisationMinBits(1)
    try:
        n = 16
        ops = C.random_layers(n, 4, C.config_seed(2, 5150 + int(single)))  # a structure no other test plans
        count = ir.specialise(ops, n, 1 if single else 2, background=False)
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        C.replay(q, ops)
        Q.dgq_planPending(q)
        st = Q.plan_stats(q)
        Q.dgq_launchPlanned(q)
        amps = Q.state_vector(q)
        Q.destroyQureg(q, env)
        assert count == st.sweeps
        assert st.jitCompiled == 0 and st.jitReused == st.sweeps
        ref, _, _ = oracle.run(n, ops)
        if single:
            assert abs(np.vdot(ref, amps)) ** 2 >= 1 - 1e-6
        else:
            assert np.abs(amps - ref).max() <= 1e-12
    finally:
        Q.dgq_setSpecialisationMinBits(-1 if prev_bits == 22 else prev_bits)
