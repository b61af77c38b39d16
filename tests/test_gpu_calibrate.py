"""Cost-model calibration on the GPU (dgquest_b200.calibrate): a short
measurement gives finite, non-negative rates that the planner then uses and
that round-trip through the cost file."""
import math

import pytest

from dgquest_b200 import calibrate as CAL

pytestmark = pytest.mark.gpu


def test_calibration_measures_and_installs(quest, env, tmp_path):
    prev = CAL.current()
    path = tmp_path / "cost.txt"
    try:
        sweep_ms, phase_ms, rows = CAL.calibrate(22, str(path), widths=(11, 12), repeats=2,
                                                 names=["random8", "ghzqft", "hea6"])
        assert len(rows) == 6 and all(r["ms"] > 0 for r in rows)
        assert sweep_ms > 0 and phase_ms >= 0 and math.isfinite(sweep_ms) and math.isfinite(phase_ms)
        assert CAL.current() == pytest.approx((sweep_ms, phase_ms), rel=1e-6)
        quest.dgq_setCostModel(*prev)
        assert quest.dgq_loadCostModel(str(path).encode()) == 0
        assert CAL.current() == pytest.approx((sweep_ms, phase_ms), rel=1e-5)
    finally:
        quest.dgq_setCostModel(*prev)


def test_dense_rate_calibration(quest, env, tmp_path):
    # the form choice's dense-block rates: measured per variant and width,
    # positive and finite, and
    # written to / read back from the cost file
    prev_rates = CAL.current()
    keys = [(v, k) for v in range(3) for k in (5, 6, 7)]
    prev = {key: quest.dgq_getDenseCost(*key) for key in keys}
    path = tmp_path / "cost.txt"
    try:
        dense = CAL.measure_dense(22, Ks=(5, 6), repeats=2)
        assert set(dense) == {("f64", 5), ("f64", 6), ("c64", 5), ("c64", 6), ("c64tc", 6)}
        assert all(ms > 0 and math.isfinite(ms) for ms in dense.values())
        CAL.write(str(path), *prev_rates, dense=dense)
        assert quest.dgq_loadCostModel(str(path).encode()) == 0
        assert quest.dgq_getDenseCost(0, 6) == pytest.approx(dense[("f64", 6)], rel=1e-5)
        assert quest.dgq_getDenseCost(2, 6) == pytest.approx(dense[("c64tc", 6)], rel=1e-5)
    finally:
        quest.dgq_setCostModel(*prev_rates)
        for key, r in prev.items():
            quest.dgq_setDenseCost(*key, r)
