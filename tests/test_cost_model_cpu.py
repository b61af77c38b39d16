"""The tile-width cost model and its calibration file (host only): the
file format is read and checked, and the planner's width choice is the
argmin of sweeps x sweep_ms + phases x phase_ms (+ 3 us per launch) over the
widths, for whichever rates are installed."""
import ctypes

import pytest

from dgquest_b200 import calibrate as CAL
from dgquest_b200 import circuits as C
from dgquest_b200 import ir
from dgquest_b200 import quest as Q


@pytest.fixture
def restore_rates():
    prev = CAL.current()
    yield
    Q.dgq_setCostModel(*prev)


def predicted(st, n, sweep_ms, phase_ms):
    amps = float(1 << n)
    return st.sweeps * (amps * sweep_ms * 1e-3 / 2**30 + 3e-6) + st.phases * amps * phase_ms * 1e-3 / 2**30


@pytest.mark.parametrize("rates", [(2.6, 1.8), (10.0, 0.01), (0.01, 10.0)])
def test_width_choice_is_the_model_argmin(rates, restore_rates):
    n = 20  # below the lookahead threshold: one candidate per width
    Q.dgq_setCostModel(*rates)
    for ops in (C.random_layers(n, 12, C.config_seed(2, 710)), C.grid_sqrt(4, 5, 10, C.config_seed(3, 711))):
        cands = {w: ir.plan(ops, n, w) for w in (9, 10, 11, 12)}
        best = min(cands, key=lambda w: (predicted(cands[w], n, *rates), w))
        assert ir.plan(ops, n, 0).tileBits == best


def test_cost_file_round_trip(tmp_path, restore_rates):
    path = tmp_path / "cost.txt"
    CAL.write(str(path), 3.25, 0.75, note="test")
    assert Q.dgq_loadCostModel(str(path).encode()) == 0
    s, p = CAL.current()
    assert abs(s - 3.25) < 1e-9 and abs(p - 0.75) < 1e-9
    bad = tmp_path / "bad.txt"
    bad.write_text("sweep_ms_per_2p30 1.0\n")  # no header, no phase rate
    with pytest.raises(Q.QuESTError):
        Q.dgq_loadCostModel(str(bad).encode())
    with pytest.raises(Q.QuESTError):
        Q.dgq_setCostModel(-1.0, 1.0)
    assert CAL.current() == pytest.approx((3.25, 0.75))


def test_fit_recovers_rates():
    rows = []
    for s, p in [(17, 52), (19, 55), (21, 57), (8, 23), (14, 44), (20, 49)]:
        rows.append({"sweeps": s, "phases": p, "ms": (s * 2.5 + p * 1.5) / 16.0})  # n = 26
    sweep_ms, phase_ms = CAL.fit(rows, 26)
    assert abs(sweep_ms - 2.5) < 1e-9 and abs(phase_ms - 1.5) < 1e-9
    assert ctypes.sizeof(ctypes.c_double) == 8


def test_errors_are_recorded_per_thread(restore_rates):
    """An error raised on one host thread is reported to that thread only."""
    import threading
    lib = Q._library()
    seen = {}

    def fail():
        lib.dgq_setCostModel(-1.0, 1.0)  # raw call: the error stays recorded
        seen["other"] = lib.dgq_getLastError(None, 0)

    t = threading.Thread(target=fail)
    t.start()
    t.join()
    assert seen["other"] != 0
    assert lib.dgq_getLastError(None, 0) == 0


@pytest.fixture
def restore_dense():
    prev = {(v, k): Q.dgq_getDenseCost(v, k) for v in range(3) for k in (5, 6, 7)}
    yield
    for (v, k), r in prev.items():
        Q.dgq_setDenseCost(v, k, r)


def test_form_choice_defaults_to_tiles_for_gate_circuits(restore_rates, restore_dense):
    # built-in rates: a dense block sweep costs far more than a register-phase
    # sweep covers, so rotation circuits stay in the tile form
    n = 24
    st = ir.plan(C.random_layers(n, 12, C.config_seed(2, 712)), n, 0)
    assert st.formAuto == 1 and st.formK == 0 and st.denseBlocks == 0
    assert st.predictedTileMs > 0
    # every dense estimate stopped early at a bound above the tile form's
    assert st.denseBound == 0b111
    assert min(st.predictedDenseMs) > 0.8 * st.predictedTileMs


@pytest.mark.parametrize("rates,expect", [((5.0, 0.001, 5.0), 6), ((0.001, 5.0, 5.0), 5), ((5.0, 5.0, 0.0005), 7)])
def test_form_choice_is_the_cheapest_dense_width(rates, expect, restore_rates, restore_dense):
    n = 26  # large enough that a block's launch overhead (3 us) does not decide
    for k, r in zip((5, 6, 7), rates):
        assert Q.dgq_setDenseCost(0, k, r) == 0
    st = ir.plan(C.random_layers(n, 12, C.config_seed(2, 713)), n, 0)
    assert st.formAuto == 1 and st.formK == expect and st.denseBlocks > 0
    pred = list(st.predictedDenseMs)
    assert not (st.denseBound >> (expect - 5)) & 1
    assert pred[expect - 5] < 0.8 * st.predictedTileMs
    # the chosen width's prediction is the smallest of the complete ones
    full = [p for i, p in enumerate(pred) if not (st.denseBound >> i) & 1]
    assert pred[expect - 5] == min(full)


def test_dense_rates_from_a_cost_file(tmp_path, restore_rates, restore_dense):
    path = tmp_path / "cost.txt"
    path.write_text("dgq_cost 1\nsweep_ms_per_2p30 2.6\nphase_ms_per_2p30 1.8\n"
                    "dense_ms_per_2p30_f64_k6 0.002\ndense_ms_per_2p30_c64tc_k6 1.5\nc64_tile_factor 0.5\n")
    assert Q.dgq_loadCostModel(str(path).encode()) == 0
    assert Q.dgq_getDenseCost(0, 6) == pytest.approx(0.002)
    assert Q.dgq_getDenseCost(2, 6) == pytest.approx(1.5)
    n = 26
    st = ir.plan(C.random_layers(n, 12, C.config_seed(2, 714)), n, 0)
    assert st.formK == 6
    with pytest.raises(Q.QuESTError):
        Q.dgq_setDenseCost(3, 6, 1.0)
    with pytest.raises(Q.QuESTError):
        Q.dgq_setDenseCost(0, 8, 1.0)


def test_form_choice_is_kept_per_structure(restore_rates, restore_dense):
    # a second plan of the same gate structure (other angles) reuses the
    # choice: same width, form and predictions
    n = 26
    a = ir.plan(C.random_layers(n, 10, C.config_seed(2, 715)), n, 0)
    ops = C.random_layers(n, 10, C.config_seed(2, 715)).copy()
    ops["p"][:, 0] += 0.125  # same structure, other angles
    b = ir.plan(ops, n, 0)
    assert (a.tileBits, a.sweeps, a.formK) == (b.tileBits, b.sweeps, b.formK)
    assert a.predictedTileMs == b.predictedTileMs
    # a different cost model is a different key: the choice is made again
    Q.dgq_setCostModel(100.0, 0.01)
    c = ir.plan(ops, n, 0)
    assert c.predictedTileMs != b.predictedTileMs
