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
