"""Density registers (createDensityQureg and the density-matrix calls that
dgQuEST's header declares): an n-qubit density matrix held as the 2n-qubit
vector of its elements, gates applied as U rho U^dagger, noise channels as
Kraus maps. Checked against numpy on 5 qubits: unitary circuits against
|psi><psi| from the oracle, channels against explicit Kraus sums,
probabilities, collapse and purity against the numpy matrix (1e-12), and
measurement outcomes against the oracle's state-vector measurement under the
same seed (bit-exact). These calls have no body in dgQuEST, so the
semantics follow upstream QuEST's documentation in the header."""
import ctypes

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu

N = 5
TOL = 1e-12
PAULI = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0])]


def op_on(k, qubits, n):
    """The 2^n x 2^n operator of a 2^m x 2^m matrix k on `qubits` (the first
    qubit is the low bit of k's index)."""
    dim = 1 << n
    m = len(qubits)
    full = np.zeros((dim, dim), dtype=complex)
    for col in range(dim):
        sub_c = sum(((col >> q) & 1) << i for i, q in enumerate(qubits))
        rest = col & ~sum(1 << q for q in qubits)
        for sub_r in range(1 << m):
            row = rest | sum(((sub_r >> i) & 1) << q for i, q in enumerate(qubits))
            full[row, col] += k[sub_r, sub_c]
    return full


def channel(rho, kraus, qubits, n):
    out = np.zeros_like(rho)
    for k in kraus:
        K = op_on(k, qubits, n)
        out += K @ rho @ K.conj().T
    return out


def unitary_ops(seed):
    kinds = [k for k in range(C.CY + 1) if k != C.MEASURE]
    return np.concatenate([C.mixed_ops(N, 160, seed, kinds=kinds), C.random_layers(N, 3, seed + 1)])


def test_unitary_circuit_is_psi_psi_dagger(quest, env):
    ops = unitary_ops(401)
    q = quest.createDensityQureg(N, env)
    try:
        assert q.isDensityMatrix == 1 and q.numQubitsRepresented == N and q.numQubitsInStateVec == 2 * N
        C.replay(q, ops)
        rho = quest.density_matrix(q)
        p0 = quest.prob_all_zero(q)
        total = quest.calcTotalProb(q)
        purity = quest.calcPurity(q)
        amp = quest.getDensityAmp(q, 3, 17)
    finally:
        quest.destroyQureg(q, env)
    psi = oracle.run(N, ops)[0]
    want = np.outer(psi, psi.conj())
    assert np.abs(rho - want).max() <= TOL
    diag = np.real(np.diag(want))
    assert np.abs(p0 - [diag[[i for i in range(1 << N) if not (i >> t) & 1]].sum() for t in range(N)]).max() <= TOL
    assert abs(total - 1.0) <= TOL and abs(purity - 1.0) <= TOL
    assert abs(complex(amp.real, amp.imag) - want[3, 17]) <= TOL


def test_noise_channels_match_kraus_sums(quest, env):
    ops = unitary_ops(402)
    psi = oracle.run(N, ops)[0]
    rho = np.outer(psi, psi.conj())
    q = quest.createDensityQureg(N, env)
    try:
        C.replay(q, ops)
        p = 0.2
        quest.applyOneQubitDephaseError(q, 1, p)
        rho = channel(rho, [np.sqrt(1 - p) * PAULI[0], np.sqrt(p) * PAULI[3]], [1], N)
        quest.applyOneQubitDepolariseError(q, 3, 0.3)
        rho = channel(rho, [np.sqrt(0.7) * PAULI[0]] + [np.sqrt(0.1) * PAULI[i] for i in (1, 2, 3)], [3], N)
        quest.applyOneQubitDampingError(q, 0, 0.4)
        rho = channel(rho, [np.array([[1, 0], [0, np.sqrt(0.6)]]), np.array([[0, np.sqrt(0.4)], [0, 0]])], [0], N)
        quest.hadamard(q, 2)
        rho = channel(rho, [np.array([[1, 1], [1, -1]]) / np.sqrt(2)], [2], N)
        quest.applyTwoQubitDephaseError(q, 4, 2, 0.25)
        zz = [np.kron(PAULI[b], PAULI[a]) for a, b in ((0, 0), (3, 0), (0, 3), (3, 3))]  # qubit 4 = low bit
        rho = channel(rho, [np.sqrt(0.75) * zz[0]] + [np.sqrt(0.25 / 3) * m for m in zz[1:]], [4, 2], N)
        quest.applyTwoQubitDepolariseError(q, 0, 3, 0.5)
        ks = []
        for a in range(4):
            for b in range(4):
                w = np.sqrt(0.5) if a == b == 0 else np.sqrt(0.5 / 15)
                ks.append(w * np.kron(PAULI[b], PAULI[a]))  # qubit 0 = low bit
        rho = channel(rho, ks, [0, 3], N)
        quest.controlledRotateY(q, 1, 4, 0.9)
        cry = np.eye(4, dtype=complex)
        c, s = np.cos(0.45), np.sin(0.45)
        cry[np.ix_([1, 3], [1, 3])] = [[c, -s], [s, c]]  # control qubit 1 = low bit
        rho = channel(rho, [cry], [1, 4], N)
        got = quest.density_matrix(q)
        purity = quest.calcPurity(q)
        total = quest.calcTotalProb(q)
        p0 = quest.calcProbOfOutcome(q, 2, 0)
    finally:
        quest.destroyQureg(q, env)
    assert np.abs(got - rho).max() <= TOL
    assert abs(purity - np.real(np.trace(rho @ rho))) <= TOL
    assert abs(total - 1.0) <= TOL
    diag = np.real(np.diag(rho))
    assert abs(p0 - diag[[i for i in range(1 << N) if not (i >> 2) & 1]].sum()) <= TOL
    assert purity < 0.9  # the channels mixed the state


def test_collapse_and_measurement(quest, env):
    ops = unitary_ops(403)
    q = quest.createDensityQureg(N, env)
    try:
        C.replay(q, ops)
        quest.applyOneQubitDephaseError(q, 0, 0.1)
        rho = quest.density_matrix(q)
        prob = quest.collapseToOutcome(q, 2, 1)
        got = quest.density_matrix(q)
    finally:
        quest.destroyQureg(q, env)
    P = op_on(np.diag([0.0, 1.0]), [2], N)
    want = P @ rho @ P
    assert abs(prob - np.real(np.trace(want))) <= TOL
    assert np.abs(got - want / prob).max() <= TOL
    # measurement outcomes: the same draws as the oracle's state-vector run
    # (P(0) of a pure |psi><psi| equals the state's)
    meas = np.concatenate([ops, C.OpList().add(C.MEASURE, 1).add(C.MEASURE, 3).add(C.H, 0).add(C.MEASURE, 0).array()])
    quest.seed([12345, 67890])
    q = quest.createDensityQureg(N, env)
    try:
        out = C.replay(q, meas)
        rho = quest.density_matrix(q)
    finally:
        quest.destroyQureg(q, env)
    psi, _, ref_out = oracle.run(N, meas, seed_keys=[12345, 67890])
    assert out == ref_out
    assert np.abs(rho - np.outer(psi, psi.conj())).max() <= TOL


def test_initial_states_mixing_and_fidelity(quest, env):
    q = quest.createDensityQureg(N, env)
    other = quest.createDensityQureg(N, env)
    pure = quest.createQureg(N, env)
    dim = 1 << N
    try:
        quest.initPlusState(q)
        assert np.abs(quest.density_matrix(q) - np.full((dim, dim), 1.0 / dim)).max() <= TOL
        quest.initClassicalState(q, 11)
        want = np.zeros((dim, dim))
        want[11, 11] = 1.0
        assert np.abs(quest.density_matrix(q) - want).max() <= TOL
        C.replay(pure, unitary_ops(404))
        psi = quest.state_vector(pure)
        quest.initPureState(q, pure)
        assert np.abs(quest.density_matrix(q) - np.outer(psi, psi.conj())).max() <= TOL
        quest.initPlusState(other)
        quest.addDensityMatrix(q, 0.25, other)
        mixed = 0.75 * np.outer(psi, psi.conj()) + 0.25 * np.full((dim, dim), 1.0 / dim)
        assert np.abs(quest.density_matrix(q) - mixed).max() <= TOL
        fid = quest.calcFidelity(q, pure)
        assert abs(fid - np.real(psi.conj() @ mixed @ psi)) <= TOL
    finally:
        for r in (q, other, pure):
            quest.destroyQureg(r, env)


def test_density_only_and_state_vector_only_calls(quest, env):
    q = quest.createDensityQureg(3, env)
    v = quest.createQureg(3, env)
    try:
        with pytest.raises(quest.QuESTError):
            quest.applyOneQubitDephaseError(v, 0, 0.1)  # defined only for density matrices
        with pytest.raises(quest.QuESTError):
            quest.getAmp(q, 0)  # defined only for state vectors
        with pytest.raises(quest.QuESTError):
            quest.calcInnerProduct(q, v)
        with pytest.raises(quest.QuESTError):
            quest.applyOneQubitDephaseError(q, 0, 0.6)  # above 1/2
        with pytest.raises(quest.QuESTError):
            quest.applyOneQubitDepolariseError(q, 0, 0.8)  # above 3/4
        with pytest.raises(quest.QuESTError):
            quest.applyTwoQubitDepolariseError(q, 0, 0, 0.1)  # same qubit twice
        six = quest.createQureg(6, env)  # as many amplitudes as q, but a state vector
        try:
            with pytest.raises(quest.QuESTError):
                quest.cloneQureg(six, q)
        finally:
            quest.destroyQureg(six, env)
        D = ctypes.POINTER(ctypes.c_double)
        buf = np.zeros(8)
        with pytest.raises(quest.QuESTError):
            quest.initStateFromAmps(q, buf.ctypes.data_as(D), buf.ctypes.data_as(D))
    finally:
        quest.destroyQureg(q, env)
        quest.destroyQureg(v, env)


def test_noise_channel_probability_errors(quest, env):
    # each channel's own limit raises its own QuEST message; a probability
    # outside [0, 1] raises the generic one (QuEST_validation.c messages)
    q = quest.createDensityQureg(3, env)
    generic = "Probabilities must be in [0, 1]."
    cases = [
        (lambda p: quest.applyOneQubitDephaseError(q, 0, p), 0.6, "single qubit dephase"),
        (lambda p: quest.applyTwoQubitDephaseError(q, 0, 1, p), 0.8, "two-qubit qubit dephase"),
        (lambda p: quest.applyOneQubitDepolariseError(q, 0, p), 0.8, "single qubit depolarising"),
        (lambda p: quest.applyTwoQubitDepolariseError(q, 0, 1, p), 0.95, "two-qubit depolarising"),
        (lambda p: quest.applyOneQubitDampingError(q, 0, p), None, None),
    ]
    try:
        for call, above, words in cases:
            if above is not None:
                with pytest.raises(quest.QuESTError) as ei:
                    call(above)
                assert words in ei.value.message, ei.value.message
            for bad in (-0.1, 1.5):
                with pytest.raises(quest.QuESTError) as ei:
                    call(bad)
                assert ei.value.message.endswith(generic), ei.value.message
        quest.applyOneQubitDampingError(q, 0, 1.0)  # full decay is a valid channel
        assert abs(quest.calcTotalProb(q) - 1.0) <= TOL
    finally:
        quest.destroyQureg(q, env)
