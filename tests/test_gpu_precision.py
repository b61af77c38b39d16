"""The complex64 precision form against the FP64 oracle.

Tolerances (stated, FP32 arithmetic on unit-norm states): fidelity
|<psi64|psi32>|^2 >= 1 - 1e-6, max |amplitude error| <= 2e-6 for n <= 16,
|1 - norm| <= 1e-5, P(q=0) within 1e-5; measurement outcomes equal where
the outcome is decided with margin (BV: deterministic)."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu


def run_f32(Q, env, n, ops, tile_bits=0, seed_keys=None):
    q = Q.dgq_createQuregF32(n, env)
    assert Q.dgq_getPrecision(q) == 1
    if tile_bits:
        Q.dgq_setTileBits(q, tile_bits)
    if seed_keys is not None:
        Q.seed(seed_keys)
    out = C.replay(q, ops)
    amps = Q.state_vector(q)
    p0 = Q.prob_all_zero(q)
    norm = Q.calcTotalProb(q)
    Q.destroyQureg(q, env)
    return amps, p0, norm, out


def fidelity(a, b):
    return abs(np.vdot(a, b)) ** 2


@pytest.mark.parametrize("tile_bits", [9, 11, 12, 13])
def test_f32_random_layers(quest, env, tile_bits):
    n = 16
    ops = C.random_layers(n, 12, C.config_seed(2, 300 + tile_bits))
    amps, p0, norm, _ = run_f32(quest, env, n, ops, tile_bits)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert fidelity(ref, amps) >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6
    assert abs(norm - 1) <= 1e-5
    assert np.abs(p0 - ref_p0).max() <= 1e-5


def test_f32_every_call_and_grid(quest, env):
    n = 14
    ops = np.concatenate([C.mixed_ops(n, 300, 41), C.grid_sqrt(2, 7, 6, C.config_seed(3, 14))])
    amps, p0, norm, _ = run_f32(quest, env, n, ops)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert fidelity(ref, amps) >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6


def test_f32_bv_measurement(quest, env):
    n = 15
    ops = C.bernstein_vazirani(n, C.config_seed(2, 9), measure=True)
    _, _, _, out = run_f32(quest, env, n, ops, seed_keys=[1, 2])
    _, _, ref_out = oracle.run(n, ops, seed_keys=[1, 2])
    assert out == ref_out


def test_inner_product_and_fidelity_across_precisions(quest, env):
    n = 15
    ops = C.random_layers(n, 10, 77)
    q64 = quest.createQureg(n, env)
    q32 = quest.dgq_createQuregF32(n, env)
    C.replay(q64, ops)
    C.replay(q32, ops)
    ip = quest.calcInnerProduct(q64, q32)
    ref = oracle.run(n, ops)[0]
    a32 = quest.state_vector(q32)
    assert abs(complex(ip.real, ip.imag) - np.vdot(ref, a32)) <= 1e-6
    assert quest.calcFidelity(q64, q32) >= 1 - 1e-6
    assert quest.calcFidelity(q64, q64) == pytest.approx(1.0, abs=1e-12)
    quest.destroyQureg(q64, env)
    quest.destroyQureg(q32, env)


@pytest.fixture
def specialise_all(quest):
    """Runtime-specialised kernels for every register size (the complex64
    paired form needs them); restores the default afterwards."""
    prev = quest.dgq_setSpecialisationMinBits(1)
    yield
    quest.dgq_setSpecialisationMinBits(-1 if prev == 22 else prev)


@pytest.mark.parametrize("n,tile_bits", [(16, 13), (14, 10), (15, 12), (13, 13), (12, 0)])
def test_f32_paired_form(quest, env, specialise_all, n, tile_bits):
    """The paired form (two amplitudes per slot, packed FP32) on every kind of
    call: random layers, the API call mix (multi-qubit unitaries on address
    bit 0 fall back to the unpaired form), BV measurement."""
    Q = quest
    ops = np.concatenate([C.random_layers(n, 6, C.config_seed(2, 900 + n)), C.mixed_ops(n, 250, 60 + n)])
    amps, p0, norm, _ = run_f32(Q, env, n, ops, tile_bits)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert fidelity(ref, amps) >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6
    assert abs(norm - 1) <= 1e-5
    assert np.abs(p0 - ref_p0).max() <= 1e-5


@pytest.mark.parametrize("n,tile_bits", [(15, 13), (14, 11)])
def test_f32_paired_sign_heavy(quest, env, specialise_all, n, tile_bits):
    """Gates whose negations the paired generator carries as compile-time
    signs (CZ, Y, S, controlled Y, X on a control, H and Rx / Ry at angles
    of every quadrant), on every qubit including address bit 0, so signs
    pass through rotations, swaps, phases, controls known only at run time
    and the phase-end restore."""
    Q = quest
    kinds = [C.CZ, C.Y, C.S, C.CY, C.CNOT, C.H, C.RX, C.RY, C.RZ, C.Z, C.SWAP]
    ops = np.concatenate([C.mixed_ops(n, 400, 700 + n, kinds=kinds), C.random_layers(n, 3, 11 + n)])
    amps, p0, norm, _ = run_f32(Q, env, n, ops, tile_bits)
    ref, ref_p0, _ = oracle.run(n, ops)
    assert fidelity(ref, amps) >= 1 - 1e-6
    assert np.abs(amps - ref).max() <= 2e-6
    assert abs(norm - 1) <= 1e-5
    assert np.abs(p0 - ref_p0).max() <= 1e-5



def test_f32_paired_is_selected(quest, env, specialise_all):
    Q = quest
    n = 16
    q = Q.dgq_createQuregF32(n, env)
    C.replay(q, C.random_layers(n, 4, 3))
    Q.dgq_planPending(q)
    st = Q.plan_stats(q)
    # the paired form uses 2^13-amplitude tiles by default and is specialised
    assert st.tileBits == 13 and st.jitCompiled + st.jitReused == st.sweeps
    Q.destroyQureg(q, env)
