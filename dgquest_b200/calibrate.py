"""Cost-model calibration on the GPU at hand (the counterpart of dgQuEST's
`sampler` binary, which times gates and writes predict_data.txt for its time
predictor, time_predictor.cpp:397-476).

The tile-width choice predicts a plan's time as
    sweeps x sweep_ms + phases x phase_ms        (per 2^30 amplitudes),
and the form choice a dense-block plan's as blocks x dense_ms (per variant
and block width K; --dense measures those too).
This module plans a set of seeded circuits at several tile widths, times
every plan with CUDA events on the register's stream, fits the two rates by
least squares (non-negative), writes them to a cost file and installs them:

    python -m dgquest_b200.calibrate --qubits 28 --out dgq_cost.txt
    DGQ_COST_FILE=dgq_cost.txt python my_program.py
"""
import argparse
import ctypes
import json

import numpy as np

from . import circuits as C
from . import quest as Q

HEADER = "dgq_cost 1"


def circuits(n):
    """The calibration set: random layers of depth 8 and 20, a 4-row grid of
    sqrt gates, GHZ+QFT and a hardware-efficient ansatz (seeded)."""
    return {
        "random8": C.random_layers(n, 8, C.config_seed(2, 700)),
        "random20": C.random_layers(n, 20, C.config_seed(2, 701)),
        "grid16": C.grid_sqrt(4, n // 4, 16, C.config_seed(3, 702)),
        "ghzqft": C.ghz_qft(n),
        "hea6": C.hea(n, 6, C.config_seed(4, 703)),
    }


def measure(n=26, widths=(10, 11, 12), repeats=3, names=None):
    """Rows (circuit, W, sweeps, phases, ms) for one complex128 register of n
    qubits; ms is the median of `repeats` timed launches of the plan."""
    import torch
    env = Q.createQuESTEnv()
    q = Q.createQureg(n, env)
    stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
    rows = []
    try:
        for name, ops in circuits(n).items():
            if names and name not in names:
                continue
            for w in widths:
                Q.dgq_setTileBits(q, w)
                Q.initZeroState(q)
                Q.apply_circuit(q, ops)
                Q.dgq_planPending(q)
                st = Q.plan_stats(q)
                Q.dgq_launchPlanned(q)
                torch.cuda.synchronize()
                ts = []
                for _ in range(repeats):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    Q.dgq_launchPlanned(q)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ts.append(e0.elapsed_time(e1))
                rows.append({"circuit": name, "W": w, "sweeps": int(st.sweeps), "phases": int(st.phases),
                             "ms": float(np.median(ts))})
    finally:
        Q.dgq_setTileBits(q, 0)
        Q.destroyQureg(q, env)
        Q.destroyQuESTEnv(env)
    return rows


DENSE_VARIANTS = (("f64", False, 0), ("c64", True, 0), ("c64tc", True, 1))


def measure_dense(n=26, Ks=(5, 6, 7), repeats=3):
    """ms per dense block per 2^30 amplitudes, {(variant, K): ms}, for the
    form choice: two random K-qubit unitaries (multiQubitUnitary) on an
    n-qubit register, the plan timed with CUDA events (the init pass
    included, so the figure is a slight over-estimate per block)."""
    import torch
    gen = np.random.default_rng(11)
    env = Q.createQuESTEnv()
    out = {}
    try:
        for name, single, tc in DENSE_VARIANTS:
            for K in Ks:
                if name == "c64tc" and K != 6:
                    continue
                prev = Q.dgq_setTensorCores(tc)
                q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
                try:
                    Q.initPlusState(q)
                    for t in (list(range(K)), list(range(n - K, n))):
                        m = Q.matrixN(C.random_unitary(gen, 1 << K))
                        Q.multiQubitUnitary(q, Q.int_array(t), K, m)
                        Q.destroyComplexMatrixN(m)
                    Q.dgq_planPending(q)
                    stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
                    Q.dgq_launchPlanned(q)
                    torch.cuda.synchronize()
                    ts = []
                    for _ in range(repeats):
                        e0 = torch.cuda.Event(enable_timing=True)
                        e1 = torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        Q.dgq_launchPlanned(q)
                        e1.record(stream)
                        torch.cuda.synchronize()
                        ts.append(e0.elapsed_time(e1))
                    out[(name, K)] = float(np.median(ts)) / 2 * 2.0 ** (30 - n)
                finally:
                    Q.destroyQureg(q, env)
                    Q.dgq_setTensorCores(prev)
    finally:
        Q.destroyQuESTEnv(env)
    return out


def fit(rows, n):
    """Non-negative least squares for (sweep_ms, phase_ms) per 2^30 amplitudes."""
    scale = 2.0 ** (30 - n)
    A = np.array([[r["sweeps"], r["phases"]] for r in rows], dtype=np.float64)
    y = np.array([r["ms"] * scale for r in rows], dtype=np.float64)
    x, *_ = np.linalg.lstsq(A, y, rcond=None)
    if x[1] < 0:  # phases cost nothing measurable: sweeps alone
        x = np.array([float(np.dot(A[:, 0], y) / np.dot(A[:, 0], A[:, 0])), 0.0])
    if x[0] <= 0:
        x = np.array([float(np.dot(A.sum(1), y) / np.dot(A.sum(1), A.sum(1)))] * 2)
    return float(x[0]), float(x[1])


def write(path, sweep_ms, phase_ms, note="", dense=None):
    with open(path, "w") as f:
        f.write(f"{HEADER}\n")
        if note:
            f.write(f"# {note}\n")
        f.write(f"sweep_ms_per_2p30 {sweep_ms:.6f}\n")
        f.write(f"phase_ms_per_2p30 {phase_ms:.6f}\n")
        for (name, K), ms in sorted((dense or {}).items()):
            f.write(f"dense_ms_per_2p30_{name}_k{K} {ms:.6f}\n")


def install_dense(dense):
    """Installs measured dense rates (dgq_setDenseCost)."""
    index = {name: i for i, (name, _, _) in enumerate(DENSE_VARIANTS)}
    for (name, K), ms in dense.items():
        Q.dgq_setDenseCost(index[name], K, ms)


def calibrate(n=26, out=None, widths=(10, 11, 12), repeats=3, names=None, dense=False):
    """Measures, fits, installs (dgq_setCostModel, and with dense=True the
    dense-block rates, dgq_setDenseCost) and optionally writes the rates;
    returns (sweep_ms, phase_ms, rows)."""
    rows = measure(n, widths, repeats, names)
    sweep_ms, phase_ms = fit(rows, n)
    Q.dgq_setCostModel(sweep_ms, phase_ms)
    drates = measure_dense(n, repeats=repeats) if dense else None
    if drates:
        install_dense(drates)
    if out:
        write(out, sweep_ms, phase_ms, note=f"fitted on {len(rows)} plans at n={n}", dense=drates)
    return sweep_ms, phase_ms, rows


def current():
    s, p = ctypes.c_double(0.0), ctypes.c_double(0.0)
    Q.dgq_getCostModel(ctypes.byref(s), ctypes.byref(p))
    return s.value, p.value


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--qubits", type=int, default=26)
    ap.add_argument("--out", default="dgq_cost.txt")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--dense", action="store_true", help="also measure the dense-block rates of the form choice")
    args = ap.parse_args()
    sweep_ms, phase_ms, rows = calibrate(args.qubits, args.out, repeats=args.repeats, dense=args.dense)
    print(json.dumps({"sweep_ms_per_2p30": sweep_ms, "phase_ms_per_2p30": phase_ms, "plans": len(rows),
                      "file": args.out}))


if __name__ == "__main__":
    main()
