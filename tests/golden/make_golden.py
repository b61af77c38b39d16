"""Generates the golden fixtures in tests/golden/ by running the reference.

The reference (dgQuEST) is compiled from its own sources by
`make -C oracle ref` into oracle/_ref/ref_harness (sm_100a); this script runs
that binary on a GPU host for each case below and stores, per case, an .npz
with the op list, the reference's P(q=0) for every qubit, its amplitudes
(all of them, or at seeded sample indices), and the reference's own
getAmp time. Usage (on a GPU host, from the repository root):

    python tests/golden/make_golden.py --out <dir> [--big]

Reference settings: QuEST.conf = "K K K" (designated K, the reference reads
it from the working directory, src/cpp/QuEST_distributed.cpp:42-56) with
K = min(5, n - 12) (the reference needs n - K >= 12 and K <= 5 keeps its
reorder launch within 1024 threads, src/cpp/QuEST_gpu_kernel.cu:646-653),
and an empty predict_data.txt (K is designated, so no calibration is used).
Swaps reach the reference as three controlledNot calls; measurement has no
reference body, so golden cases carry no measurements.
"""
import argparse
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dgquest_b200 import circuits as C  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def cases(big):
    out = [
        ("mixed_n14", 14, C.mixed_ops(14, 500, 4242, kinds=[k for k in range(26) if k not in (C.MEASURE,)]), "full"),
        ("random_n14_d20", 14, C.random_layers(14, 20, C.config_seed(2, 14)), "full"),
        ("ghzqft_n14", 14, C.ghz_qft(14), "full"),
        ("bv_n14", 14, C.bernstein_vazirani(14, C.config_seed(2, 1), measure=False), "full"),
        ("grid_n16_d8", 16, C.grid_sqrt(4, 4, 8, C.config_seed(3, 16)), "full"),
        ("ghzqft_n20", 20, C.ghz_qft(20), "sample"),
        ("random_n22_d20", 22, C.random_layers(22, 20, C.config_seed(2, 22)), "sample"),
    ]
    if big:
        out += [
            ("random_n30_d20", 30, C.random_layers(30, 20, C.config_seed(2)), "sample"),
            ("bv_n30", 30, C.bernstein_vazirani(30, C.config_seed(2, 1), measure=False), "sample"),
        ]
    return out


def sample_indices(n, seed=7, count=4096):
    rng = np.random.default_rng(seed + n)
    idx = rng.choice(1 << n, size=min(count, 1 << n), replace=False).astype(np.int64)
    idx = np.unique(np.concatenate([idx, np.array([0, (1 << n) - 1], dtype=np.int64)]))
    return idx


def read_output(path, n, full):
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == b"DGQR"
    version, nn = np.frombuffer(data[4:12], dtype="<i4")
    assert version == 1 and nn == n
    num = int(np.frombuffer(data[12:20], dtype="<i8")[0])
    t_get, t_prob = np.frombuffer(data[20:36], dtype="<f8")
    off = 36
    p0 = np.frombuffer(data[off:off + 8 * n], dtype="<f8").copy()
    off += 8 * n
    idx = None
    if not full:
        idx = np.frombuffer(data[off:off + 8 * num], dtype="<i8").copy()
        off += 8 * num
    ri = np.frombuffer(data[off:off + 16 * num], dtype="<f8")
    amps = ri[0::2] + 1j * ri[1::2]
    return p0, idx, amps, float(t_get), float(t_prob)


def run_case(name, n, ops, mode, outdir):
    k = min(5, n - 12)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "QuEST.conf"), "w") as f:
            f.write(f"{k} {k} {k}\n")
        open(os.path.join(d, "predict_data.txt"), "w").close()
        ops_path = os.path.join(d, "ops.bin")
        np.ascontiguousarray(ops).tofile(ops_path)
        out_path = os.path.join(d, "out.bin")
        cmd = [HARNESS, ops_path, str(n), out_path, "full" if mode == "full" else "sample"]
        if mode != "full":
            idx_path = os.path.join(d, "idx.bin")
            sample_indices(n).tofile(idx_path)
            cmd.append(idx_path)
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0"))
        t0 = time.time()
        r = subprocess.run(cmd, cwd=d, env=env, capture_output=True, text=True, timeout=1200)
        wall = time.time() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        p0, idx, amps, t_get, t_prob = read_output(out_path, n, mode == "full")
    path = os.path.join(outdir, f"{name}.npz")
    np.savez_compressed(path, n=n, k=k, ops=ops, p0=p0, amps=amps,
                        indices=idx if idx is not None else np.zeros(0, dtype=np.int64),
                        ref_getamp_seconds=t_get, ref_probs_seconds=t_prob, ref_wall_seconds=wall)
    print(f"{name}: n={n} K={k} amps={len(amps)} getAmp {t_get:.3f}s probs {t_prob:.3f}s wall {wall:.1f}s",
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--big", action="store_true", help="also the 30-qubit cases")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    if not os.path.exists(HARNESS):
        sys.exit(f"reference harness missing: build it with `make -C oracle ref` ({HARNESS})")
    os.makedirs(a.out, exist_ok=True)
    for name, n, ops, mode in cases(a.big):
        if a.only and name not in a.only.split(","):
            continue
        run_case(name, n, ops, mode, a.out)


if __name__ == "__main__":
    main()
