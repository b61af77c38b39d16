"""The serving loop on the GPU: results are the same alone and in the mix,
and match the oracle.

Tolerances: samples are compared exactly (a request's sampler sees the same
state and seed alone and in the mix); <Z> to 1e-12 (complex128) and 1e-6
(complex64) between the two runs, and to 1e-10 / 2e-5 against the oracle."""
import numpy as np
import pytest

import oracle
from dgquest_b200 import serving as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("single", [False, True])
def test_results_same_alone_and_in_the_mix(quest, env, single):
    reqs = S.make_requests(24, rate=2000.0, single=single, n_range=(10, 17))
    alone = {r.rid: S.run_request(r, env) for r in reqs}
    srv = S.Server(env, workers=6)
    mixed = srv.serve(reqs, realtime=True)
    assert srv.peak_in_flight > 1
    tol = 1e-6 if single else 1e-12
    for res in mixed:
        s0, z0 = alone[res.rid]
        assert np.array_equal(res.samples, s0)
        assert np.abs(res.expz - z0).max() <= tol
    st = S.summarize(mixed)
    assert st["requests"] == 24 and st["p99_ms"] >= st["p50_ms"]


def test_results_match_oracle(quest, env):
    reqs = S.make_requests(9, rate=1000.0, single=False, n_range=(10, 14))
    out = S.Server(env, workers=3).serve(reqs, realtime=False)
    for r, res in zip(reqs, out):
        amps, p0, _ = oracle.run(r.n, S.request_ops(r))
        expz = np.array([2 * p0[q] - 1 for q in r.zq])
        assert np.abs(res.expz - expz).max() <= 1e-10
        p = np.abs(amps) ** 2
        assert np.all(p[res.samples.astype(np.int64)] > 0)
