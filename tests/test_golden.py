"""Golden vectors produced by the reference itself (dgQuEST built from its
sources for sm_100a, run on a B200 by tests/golden/make_golden.py): the
oracle must reproduce them (CPU), and so must the product (GPU)."""
import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    d = np.load(path)
    return int(d["n"]), d["ops"], d["p0"], d["amps"], d["indices"]


def test_golden_fixtures_present():
    names = {os.path.basename(p) for p in GOLDEN}
    for required in ("mixed_n14.npz", "random_n14_d20.npz", "ghzqft_n14.npz", "ghzqft_n20.npz", "bv_n14.npz"):
        assert required in names


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference(path):
    n, ops, p0, amps, idx = load(path)
    if n > 24:
        pytest.skip("full-size golden case: checked on the GPU")
    got, got_p0, _ = oracle.run(n, ops)
    if len(idx):
        got = got[idx]
    assert np.abs(got - amps).max() <= 1e-13
    assert np.abs(got_p0 - p0).max() <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_product_reproduces_reference(quest, env, path):
    from dgquest_b200 import circuits as C
    n, ops, p0, amps, idx = load(path)
    q = quest.createQureg(n, env)
    C.replay(q, ops)
    if len(idx):
        got = np.array([complex(a.real, a.imag) for a in (quest.getAmp(q, int(i)) for i in idx)])
    else:
        got = quest.state_vector(q)
    got_p0 = quest.prob_all_zero(q)
    quest.destroyQureg(q, env)
    assert np.abs(got - amps).max() <= 1e-12
    assert np.abs(got_p0 - p0).max() <= 1e-12
