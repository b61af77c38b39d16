"""Benchmark: 30-qubit depth-20 random circuit, FP64, through libdgq.

One step = one full circuit on the resident 2^30-amplitude complex128 state
(16 GiB in HBM): initialise |0...0> and apply every planned sweep. Workload
(the reference's headline configuration for this path): per layer a random
Rx/Ry/Rz with angle U[0, 2pi) on each of the 30 qubits, then CZ on a seeded
perfect matching; 20 layers; seed 20261203 + 2000; MT19937 draws.

  value   circuits/s over all ranks, kernels only, state resident in HBM
          (CUDA events on the library's stream around K steps)
  e2e     the same metric through the public QuEST API each step: record
          every gate call, getAmp(q, 0) (plans + runs), calcProbOfOutcome
          for every qubit; kernel programs travel host->device as kernel
          parameters, the amplitude and probabilities come back
  roofline  the tile kernel (the only kernel of a step) against the measured
          HBM copy bandwidth; algorithmic bytes per step = (2 x sweeps - 1)
          x 2^30 x 16 B (the first sweep writes |0...0> without reading),
          per launch their average over the step's sweeps

Inputs are larger than L2 (16 GiB state vs 126 MB L2), so no flush is needed.
With --gpus N (torchrun), each rank runs an independent replica (the path
does not shard on one GPU); the time is the max over ranks.
`--impl reference` times the reference's algorithm on the host cores instead
(the CPU oracle, OpenMP on all cores, one complete layer of the circuit per
step; the circuit time is the mean layer time x 20). The default run also
times dgQuEST's own GPU path on the same circuit (`reference_gpu`: the
reference built from its sources, oracle/_ref/ref_harness) and the CPU
oracle on one layer with all cores and one (`cpu_baseline`).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q circuit time & HBM GB/s FP64 vs FP32-TC @fidelity≥1−1e-6; serving p99 ms"
N_QUBITS = 30
DEPTH = 20


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, nm in enumerate(names):
                if s[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        loaded = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": float(np.median(loaded)) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup(gpus, backend=None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo for host-only runs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- CPU legs
def layer_of(ops, n, layer):
    """The ops of one layer of the random circuit: n rotations, then n/2 CZ."""
    per = n + n // 2
    return ops[layer * per:(layer + 1) * per]


def cpu_time_ops(n, samples, threads):
    """Times the oracle (OpenMP, `threads` threads) applying each op list of
    `samples` in turn to one n-qubit state; returns the seconds of each."""
    import oracle
    oracle.set_threads(threads)
    o = oracle.Oracle(n)
    out = []
    for sample in samples:
        t0 = time.perf_counter()
        o.apply(sample)
        out.append(time.perf_counter() - t0)
    o.close()
    return out


def cpu_one_core_layer(ops, n):
    """One-core estimate of a layer's time: one op of each kind the layer
    holds (Rx, Ry, Rz, CZ; qubits from the middle of the register) timed on
    one thread, weighted by the kind counts of layer 0. Returns (seconds per
    layer, description)."""
    from dgquest_b200 import circuits as C
    layer = layer_of(ops, n, 0)
    kinds = [int(k) for k in layer["kind"]]
    counts = {k: kinds.count(k) for k in set(kinds)}
    reps = []
    for k in sorted(counts):
        idx = [i for i, kk in enumerate(kinds) if kk == k]
        reps.append(layer[idx[len(idx) // 2]:idx[len(idx) // 2] + 1])
    times = cpu_time_ops(n, reps, 1)
    per_kind = dict(zip(sorted(counts), times))
    t_layer = sum(counts[k] * per_kind[k] for k in counts)
    names = {C.RX: "Rx", C.RY: "Ry", C.RZ: "Rz", C.CZ: "CZ"}
    desc = ("1 thread: one op of each kind of layer 0 timed (" +
            ", ".join(f"{names.get(k, k)} {per_kind[k]:.2f} s x {counts[k]}" for k in sorted(counts)) +
            f"), weighted by the layer's kind counts; x {len(ops) // len(layer)} layers")
    return t_layer, desc


def run_reference_arm(args, world, rank):
    """The reference's algorithm on the host cores: dgQuEST has no CPU
    executor for this path, so the oracle port (plain C + OpenMP, all host
    threads) applies the circuit gate by gate. Each step applies one
    complete layer of the 30-qubit circuit (30 rotations + 15 CZ, layers in
    turn); circuits/s = 1 / (mean layer time x 20 layers)."""
    from dgquest_b200 import circuits as C
    if rank != 0:
        return
    import oracle
    ops = C.random_layers(N_QUBITS, DEPTH, C.config_seed(2))
    cores = oracle.max_threads()
    warm = [ops[:2]] * max(0, args.warmup)  # warm-up: two gates each (pages the state in)
    samples = warm + [layer_of(ops, N_QUBITS, i % DEPTH) for i in range(args.steps)]
    times = cpu_time_ops(N_QUBITS, samples, cores)[len(warm):]
    t_layer = float(np.mean(times))
    circuit_s = t_layer * DEPTH
    circuits_per_s = 1.0 / circuit_s
    sample = (f"{args.steps} complete layers (30 rotations + 15 CZ each) of the 30-qubit circuit, one per step; "
              f"circuit time = mean layer time x {DEPTH}")
    line = {"metric": METRIC, "value": circuits_per_s, "unit": "circuits/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_layer * 1000.0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded MT19937 random circuit)", "impl": "reference",
            "config": {"workload": "random circuit n=30 depth=20 (Rx/Ry/Rz + CZ matching), complex128",
                       "qubits": N_QUBITS, "depth": DEPTH, "parallelism": "host cores"},
            "extrapolated": True, "fraction_of_circuit_timed": args.steps / DEPTH,
            "layer_seconds": times,
            "cpu_baseline": {"value": circuits_per_s, "unit": "circuits/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": circuits_per_s, "unit": "circuits/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, n=None, ops=None):
    """dgQuEST's own GPU path, built from the reference's sources for sm_100a
    (oracle/_ref/ref_harness, `make -C oracle ref`), on the same circuit and
    GPU (by default the 30-qubit depth-20 random circuit): its QuEST calls,
    searchQuregTaskPartitions and getAmp(q, 0) with K = 5 (QuEST.conf
    "5 5 5"), timed by the harness around getAmp. Also reads 64 sampled
    amplitudes for a comparison with this library's."""
    import tempfile
    from dgquest_b200 import circuits as C
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"unavailable": "oracle/_ref/ref_harness not built (make -C oracle ref needs the reference sources)"}
    if n is None:
        n = N_QUBITS
        ops = C.random_layers(n, DEPTH, C.config_seed(2))
    idx = np.unique(np.random.RandomState(11).randint(0, 1 << n, size=64).astype(np.int64))
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "QuEST.conf"), "w") as f:
            f.write("5 5 5\n")
        open(os.path.join(d, "predict_data.txt"), "w").close()
        np.ascontiguousarray(ops).tofile(os.path.join(d, "ops.bin"))
        idx.tofile(os.path.join(d, "idx.bin"))
        clocks = ClockSampler(0)
        clocks.start()
        t0 = time.perf_counter()
        r = subprocess.run([harness, "ops.bin", str(n), "out.bin", "sample", "idx.bin"], cwd=d,
                           capture_output=True, text=True, timeout=600)
        wall = time.perf_counter() - t0
        clk = clocks.stop()
        if r.returncode != 0:
            return {"unavailable": f"ref_harness exited {r.returncode}: {(r.stderr or r.stdout)[-300:]}"}
        with open(os.path.join(d, "out.bin"), "rb") as f:
            data = f.read()
    num = int(np.frombuffer(data[12:20], dtype="<i8")[0])
    t_get, t_prob = np.frombuffer(data[20:36], dtype="<f8")
    off = 36 + 8 * n + 8 * num
    ri = np.frombuffer(data[off:off + 16 * num], dtype="<f8")
    return {"impl": "dgQuEST built from its sources for sm_100a (ref_harness), K = 5",
            "getamp_s": float(t_get), "probs_s": float(t_prob), "wall_s": wall,
            "circuits_per_s": 1.0 / float(t_get), "clocks": clk,
            "sample_indices": idx.tolist(), "sample_amps": (ri[0::2] + 1j * ri[1::2]),
            "note": "getamp_s is the reference's own timing of getAmp(q, 0), which runs the whole circuit"}


# ---------------------------------------------------------------- GPU leg
def form_report(st, measured):
    """The predictor's form choice of a plan (plan statistics) beside the
    measured times (ms) of the forms that were run."""
    pred = {"tiles": round(st.predictedTileMs, 2)}
    for i, k in enumerate((5, 6, 7)):
        v = round(st.predictedDenseMs[i], 2)
        pred[f"dense_k{k}"] = f">{v}" if (st.denseBound >> i) & 1 else v
    chosen = f"tiles W={st.tileBits}" if st.formK == 0 else f"dense K={st.formK}"
    return {"chosen": chosen, "by_predictor": bool(st.formAuto), "predicted_ms": pred,
            "measured_ms": {k: round(v, 2) for k, v in measured.items()},
            "note": "'>x': the estimate stopped counting blocks once they cost more than the tile form"}


def time_dense_form(n, ops, single, K, runs=1):
    """One warm-up and `runs` timed launches (ms, CUDA events) of the circuit
    fused into dense K-qubit blocks (dgq_setDenseFusion(q, K))."""
    import torch

    from dgquest_b200 import quest as Q
    env = Q.createQuESTEnv()
    q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
    Q.dgq_setDenseFusion(q, K)
    Q.initZeroState(q)
    Q.apply_circuit(q, ops)
    Q.dgq_planPending(q)
    blocks = Q.plan_stats(q).denseBlocks
    stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
    Q.dgq_launchPlanned(q)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(runs):
        Q.dgq_launchPlanned(q)
    e1.record(stream)
    torch.cuda.synchronize()
    Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)
    return e0.elapsed_time(e1) / runs, int(blocks)


def run_gpu(args, world, rank, local, ref_gpu=None):
    import torch

    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q

    torch.cuda.set_device(local)
    n, depth = args.qubits, args.depth
    ops = C.random_layers(n, depth, C.config_seed(2))
    env = Q.createQuESTEnv()
    q = Q.createQureg(n, env)
    if args.tile_bits:
        Q.dgq_setTileBits(q, args.tile_bits)
    stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))

    # plan once (host), then every step relaunches the full plan from |0...0>
    Q.initZeroState(q)
    C.replay(q, ops)
    Q.dgq_planPending(q)
    st = Q.plan_stats(q)
    for _ in range(args.warmup):
        Q.dgq_launchPlanned(q)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    l0 = Q.dgq_getLaunchCount()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        Q.dgq_launchPlanned(q)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = Q.dgq_getLaunchCount() - l0
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1000.0)

    # numerics of the timed plan: norm must stay 1
    norm = Q.calcTotalProb(q)

    # e2e through the public API
    e2e_times = []
    record_times = []
    for i in range(args.e2e_steps + 1):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Q.initZeroState(q)
        C.replay(q, ops)
        t1 = time.perf_counter()
        a = Q.getAmp(q, 0)
        probs = [Q.calcProbOfOutcome(q, k, 0) for k in range(n)]
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_times.append(dt)
            record_times.append(t1 - t0)
    e2e_t = max_over_ranks(float(np.mean(e2e_times)), world)
    if ref_gpu and "sample_amps" in ref_gpu:
        # the register holds the circuit's final state (last e2e run)
        amps = [Q.getAmp(q, int(i)) for i in ref_gpu.pop("sample_indices")]
        ours = np.array([complex(a.real, a.imag) for a in amps])
        ref_gpu["max_abs_err_vs_this_library"] = float(np.abs(ours - ref_gpu.pop("sample_amps")).max())
        ref_gpu["amplitudes_compared"] = len(ours)
    st2 = Q.plan_stats(q)
    h2d = int(st2.launchBytes)  # one sweep program per kernel parameter block
    d2h = 16 + (n + 1) * 8

    hbm, hbm_kind = peaks()
    # algorithmic bytes: every sweep reads and writes the state once, except
    # the first, which initialises |0...0> in the kernel and only writes
    state_bytes = float(1 << n) * 16
    bytes_per_step = (2.0 * st.sweeps - 1.0) * state_bytes
    bytes_per_launch = bytes_per_step / st.sweeps  # average over the step's launches
    avg_launch_s = (ms_step / 1000.0) / st.sweeps
    achieved = bytes_per_launch / avg_launch_s / 1e9
    flops = st.flopsPerAmp * (1 << n)
    pk = ctypes.c_double(0.0)
    Q.dgq_measureFp64Peak(ctypes.byref(pk))
    fp64_peak = pk.value
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("tile_kernel_bytes_per_launch_n30")
    # precision form: the same circuit on a complex64 register (8 GiB)
    fp32 = None
    if not args.no_fp32:
        q32 = Q.dgq_createQuregF32(n, env)
        s32 = torch.cuda.ExternalStream(Q.dgq_getStream(q32))
        Q.initZeroState(q32)
        C.replay(q32, ops)
        Q.dgq_planPending(q32)
        st32 = Q.plan_stats(q32)
        for _ in range(args.warmup):
            Q.dgq_launchPlanned(q32)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(s32)
        for _ in range(args.steps):
            Q.dgq_launchPlanned(q32)
        f1.record(s32)
        torch.cuda.synchronize()
        ms32 = max_over_ranks(f0.elapsed_time(f1), world) / args.steps
        # both registers now hold the circuit's final state (fresh run of the FP64 plan)
        Q.initZeroState(q)
        C.replay(q, ops)
        fid = Q.calcFidelity(q, q32)
        form32 = {"tiles": ms32}
        if not args.no_dense:
            form32["dense_k6_tensor_cores"], _ = time_dense_form(n, ops, True, 6)
        fp32 = {"ms_per_step": ms32, "circuits_per_s": world * 1000.0 / ms32, "speedup_vs_fp64": ms_step / ms32,
                "form_choice": form_report(st32, form32),
                "fidelity_vs_fp64": fid, "dtype": "complex64 amplitudes, FP32 arithmetic (SIMT)",
                "tile_bits": st32.tileBits, "sweeps": st32.sweeps,
                "hbm_gbs": 2.0 * (1 << n) * 8 * st32.sweeps / (ms32 / 1000.0) / 1e9}
        Q.destroyQureg(q32, env)
    Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)
    form64 = {"tiles": ms_step}
    if not args.no_dense:
        form64["dense_k6_simt"], _ = time_dense_form(n, ops, False, 6)
    form64 = form_report(st, form64)

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "circuits/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded MT19937 random circuit)",
                "config": {"workload": "random circuit n=30 depth=20 (Rx/Ry/Rz + CZ matching), complex128",
                           "qubits": n, "depth": depth, "tile_bits": st.tileBits, "sweeps": st.sweeps,
                           "phases": st.phases, "gates_after_merge": st.gates,
                           "l2": "inputs larger than L2 (16 GiB state)", "parallelism": f"replicas x{world}"},
                "gate_layers_per_s": depth / (ms_step / 1000.0),
                "hbm_gbs_step": bytes_per_step / (ms_step / 1000.0) / 1e9,
                "fp64_tflops_algorithmic": flops / (ms_step / 1000.0) / 1e12,
                "norm_error": abs(norm - 1.0),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic,
                             "peak_source": hbm_kind,
                             "kernel": (f"dgq_sweep (runtime-specialised tile kernel, W={st.tileBits})"
                                        if st.jitCompiled + st.jitReused else f"tileKernel<{st.tileBits}>")},
                "fp64_roofline": {"achieved_tflops": flops / (ms_step / 1000.0) / 1e12,
                                  "peak_tflops": fp64_peak, "frac": flops / (ms_step / 1000.0) / 1e12 / fp64_peak,
                                  "peak_source": "measured live (DFMA loop, dgq_measureFp64Peak)",
                                  "circuit_floor_ms": max(flops / (fp64_peak * 1e12),
                                                          bytes_per_step / (hbm * 1e9)) * 1e3},
                "e2e": {"value": world / e2e_t, "unit": "circuits/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_t * 1000.0,
                        "record_ms": float(np.mean(record_times)) * 1000.0,
                        "plan_ms": st2.planMillis,
                        "streamed_sweeps": int(st2.streamedSweeps),
                        "cold_specialisation_ms": st.jitMillis,
                        "note": "steady state: the sweep kernels specialised for this circuit's structure are "
                                "compiled once (cold_specialisation_ms, first planning) and reused; sweeps "
                                "launch while the rest of the circuit is planned (streamed_sweeps)"},
                "gpu_launches": int(launches), "clocks": clk, "fp32_form": fp32, "form_choice": form64}
        if ref_gpu is not None:
            if "getamp_s" in ref_gpu:
                ref_gpu["e2e_speedup_of_this_library"] = ref_gpu["getamp_s"] / e2e_t
            line["reference_gpu"] = ref_gpu
    return line


def run_ncu_case(args):
    """One plan of the random circuit on a small register, run twice (ncu: -s skips the first);
    with --batch-case K, the first K circuits of the batched workload as one batch, launched twice."""
    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    env = Q.createQuESTEnv()
    if args.dense_case:
        # two dense 6-qubit unitaries on a complex64 register (tensor cores), plan launched twice
        gen = np.random.default_rng(7)
        q = Q.dgq_createQuregF32(args.qubits, env)
        Q.initPlusState(q)
        for t in ([0, 1, 2, 3, 4, 5], [args.qubits - 1, 7, 15, 3, 11, 9]):
            m = Q.matrixN(C.random_unitary(gen, 64))
            Q.multiQubitUnitary(q, Q.int_array(t), 6, m)
            Q.destroyComplexMatrixN(m)
        Q.dgq_planPending(q)
        for _ in range(2):
            Q.dgq_launchPlanned(q)
        Q.dgq_sync(q)
        print(json.dumps({"case": "dense", "qubits": args.qubits, "sweeps": Q.plan_stats(q).sweeps,
                          "norm": Q.calcTotalProb(q), "device_errors": Q.dgq_getDeviceErrors()}))
        Q.destroyQureg(q, env)
        Q.destroyQuESTEnv(env)
        return
    if args.batch_case:
        single = args.precision == 1
        regs = []
        for n, d, ops in C.batch_workload(args.batch_case):
            q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
            Q.initZeroState(q)
            Q.apply_circuit(q, ops)
            regs.append(q)
        b = Q.Batch(regs, {"tileBits": args.tile_bits or 12, "groupFactor": 2})
        for _ in range(2):
            b.launch()
        z = b.expectation_z()
        st = b.stats()
        print(json.dumps({"case": "batch", "circuits": len(regs), "items": int(st.items), "sweeps": st.sweeps,
                          "sweep_bytes": int(st.sweepBytes), "z_abs_max": float(np.abs(z).max())}))
        b.close()
        for q in regs:
            Q.destroyQureg(q, env)
        Q.destroyQuESTEnv(env)
        return
    q = Q.dgq_createQuregF32(args.qubits, env) if args.precision == 1 else Q.createQureg(args.qubits, env)
    if args.tile_bits:
        Q.dgq_setTileBits(q, args.tile_bits)
    Q.dgq_setSpecialisationMinBits(1)
    for _ in range(2):
        Q.initZeroState(q)
        C.replay(q, C.random_layers(args.qubits, args.depth, C.config_seed(2)))
        Q.dgq_sync(q)
    st = Q.plan_stats(q)
    print(json.dumps({"case": "random", "qubits": args.qubits, "depth": args.depth, "tile_bits": st.tileBits,
                      "sweeps": st.sweeps, "norm": Q.calcTotalProb(q)}))
    Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)


def run_host_tier_form(args, world):
    """Host tier: the random circuit (28 qubits, depth 8, complex128: 4 GiB)
    on a register held in pinned host memory under a 2 GiB device budget
    (pages of 2^25 amplitudes through four device buffers), against the same
    circuit in HBM; host<->device traffic is every pass's pages both ways."""
    import torch

    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    n, depth, budget = 28, 8, 2 << 30
    ops = C.random_layers(n, depth, C.config_seed(2, 500))
    env = Q.createQuESTEnv()
    out = {"workload": f"random circuit n={n} depth={depth}, complex128, device budget {budget >> 30} GiB",
           "qubits": n, "depth": depth}
    # reference run in HBM
    q = Q.createQureg(n, env)
    Q.initZeroState(q)
    C.replay(q, ops)
    Q.getAmp(q, 0)
    t0 = time.perf_counter()
    Q.initZeroState(q)
    C.replay(q, ops)
    Q.getAmp(q, 0)
    out["hbm_ms"] = (time.perf_counter() - t0) * 1e3
    idx = np.random.RandomState(5).randint(0, 1 << n, size=1024)
    ref = [Q.getAmp(q, int(i)) for i in idx]
    Q.destroyQureg(q, env)
    prev = Q.dgq_setDeviceBudget(budget)
    try:
        q = Q.createQureg(n, env)
    finally:
        Q.dgq_setDeviceBudget(prev)
    st = Q.host_tier_stats(q)
    out["page_bits"] = st[0]
    for rep in range(2):
        p0 = Q.host_tier_stats(q)
        t0 = time.perf_counter()
        Q.initZeroState(q)
        C.replay(q, ops)
        Q.getAmp(q, 0)
        dt = time.perf_counter() - t0
    p1 = Q.host_tier_stats(q)
    passes, exchanges, moved = p1[1] - p0[1], p1[2] - p0[2], p1[3] - p0[3]
    out.update({"ms_per_circuit": dt * 1e3, "page_passes": int(passes), "qubit_exchanges": int(exchanges),
                "host_device_bytes": int(moved), "host_device_gbs": moved / dt / 1e9,
                "vs_hbm": dt * 1e3 / out["hbm_ms"]})
    err = 0.0
    for i, a in zip(idx, ref):
        b = Q.getAmp(q, int(i))
        err = max(err, abs(complex(a.real, a.imag) - complex(b.real, b.imag)))
    out["max_abs_err_vs_hbm_sampled"] = err
    Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)
    return out


def run_sharded_form(args, world):
    """Sharded register: the 30-qubit depth-20 random circuit (complex128) in
    8 shards of 2 GiB, all on this GPU (on several GPUs the exchange kernels
    reach the partner shard through peer memory instead), against the same
    circuit in one HBM buffer. Wall time of initZeroState + gates + getAmp;
    exchange bytes are half of every shard in each direction per exchange."""
    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    n, depth, shard_bits = 30, 20, 3
    ops = C.random_layers(n, depth, C.config_seed(2))
    env = Q.createQuESTEnv()
    out = {"workload": f"random circuit n={n} depth={depth}, complex128, {1 << shard_bits} shards on one GPU",
           "qubits": n, "depth": depth, "shards": 1 << shard_bits}
    idx = np.random.RandomState(6).randint(0, 1 << n, size=1024)

    def timed(q):
        for _ in range(2):
            t0 = time.perf_counter()
            Q.initZeroState(q)
            C.replay(q, ops)
            Q.getAmp(q, 0)
            dt = time.perf_counter() - t0
        return dt

    q = Q.createQureg(n, env)
    out["hbm_ms"] = timed(q) * 1e3
    ref = [Q.getAmp(q, int(i)) for i in idx]
    Q.destroyQureg(q, env)
    q = Q.create_sharded(n, env, shard_bits)
    p0 = Q.shard_stats(q)
    dt = timed(q)
    p1 = Q.shard_stats(q)
    # the second of the two timed runs
    passes, exchanges, moved = [(b - a) // 2 for a, b in zip(p0[1:], p1[1:])]
    out.update({"ms_per_circuit": dt * 1e3, "shard_passes": int(passes), "qubit_exchanges": int(exchanges),
                "bytes_between_shards": int(moved), "vs_hbm": dt * 1e3 / out["hbm_ms"]})
    err = 0.0
    for i, a in zip(idx, ref):
        b = Q.getAmp(q, int(i))
        err = max(err, abs(complex(a.real, a.imag) - complex(b.real, b.imag)))
    out["max_abs_err_vs_hbm_sampled"] = err
    Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)
    return out


def run_dense_form(args, world):
    """Dense 6-qubit blocks: multiQubitUnitary with 6 targets on a 30-qubit
    register, complex64 on the tensor cores (tcgen05, split FP16) and on the
    SIMT dense kernel, complex128 on the SIMT dense kernel. Time per dense
    sweep (the plan's time over its blocks), and for the tensor cores the
    time of one block alone (5 and 6 targets) from plans of 4 and 8 blocks."""
    import torch

    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    n = args.dense_qubits
    gen = np.random.default_rng(7)
    blocks = [([0, 1, 2, 3, 4, 5], C.random_unitary(gen, 64)), ([29, 7, 15, 22, 3, 11], C.random_unitary(gen, 64)),
              ([6, 12, 18, 24, 28, 1], C.random_unitary(gen, 64)), ([10, 27, 5, 20, 14, 26], C.random_unitary(gen, 64))]
    blocks = [(t, u) for t, u in blocks if max(t) < n]
    env = Q.createQuESTEnv()
    out = {"workload": f"{len(blocks)} dense 6-qubit unitaries (64x64) on {n} qubits", "qubits": n}
    runs = (("complex64_tensor_cores", True, 1), ("complex64_simt", True, 0), ("complex128_simt", False, 0))
    states = {}
    for name, single, tc in runs:
        prev = Q.dgq_setTensorCores(tc)
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        Q.initPlusState(q)
        for t, u in blocks:
            m = Q.matrixN(u)
            Q.multiQubitUnitary(q, Q.int_array(t), 6, m)
            Q.destroyComplexMatrixN(m)
        Q.dgq_planPending(q)
        st = Q.plan_stats(q)
        stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
        for _ in range(args.warmup):
            Q.dgq_launchPlanned(q)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        steps = max(1, min(args.steps, 5))
        e0.record(stream)
        for _ in range(steps):
            Q.dgq_launchPlanned(q)
        e1.record(stream)
        torch.cuda.synchronize()
        Q.dgq_setTensorCores(prev)
        ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
        # per dense block: the plan's time over its blocks (the init pass and, on
        # complex64 tensor cores, the final renormalisation pass included)
        per = ms / max(1, len(blocks))
        amp = 8 if single else 16
        flops = 8.0 * 64 * (1 << n)  # complex MACs x 8 per dense sweep (algorithmic)
        out[name] = {"ms_per_plan": ms, "sweeps": st.sweeps, "ms_per_block": per,
                     "tflops_algorithmic": flops / (per / 1e3) / 1e12,
                     "hbm_gbs": 2.0 * (1 << n) * amp / (per / 1e3) / 1e9,
                     "device_errors": Q.dgq_getDeviceErrors()}
        states[name] = q
    # one tensor-core block alone: plans of 4 and of 8 gates differ by the
    # sweeps they plan (the initialisation and final renormalisation passes
    # cancel; gates that commute onto the same targets share one block)
    hbm = peaks()[0]
    marginal = {}
    for K in (5, 6):
        t_plan, n_blocks = [], []
        for reps in (1, 2):
            q = Q.dgq_createQuregF32(n, env)
            Q.initPlusState(q)
            g2 = np.random.default_rng(11)
            for _ in range(reps):
                for t, _u in blocks:
                    m = Q.matrixN(C.random_unitary(g2, 1 << K))
                    Q.multiQubitUnitary(q, Q.int_array(t[:K]), K, m)
                    Q.destroyComplexMatrixN(m)
            Q.dgq_planPending(q)
            n_blocks.append(Q.plan_stats(q).sweeps)
            stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
            Q.dgq_launchPlanned(q)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(3):
                Q.dgq_launchPlanned(q)
            e1.record(stream)
            torch.cuda.synchronize()
            t_plan.append(e0.elapsed_time(e1) / 3)
            Q.destroyQureg(q, env)
        per = (t_plan[1] - t_plan[0]) / max(1, n_blocks[1] - n_blocks[0])
        marginal[f"k{K}"] = {"ms_per_block": per, "hbm_frac": 2.0 * (1 << n) * 8 / (per / 1e3) / 1e9 / hbm,
                             "sweeps_planned": n_blocks}
    out["complex64_tensor_cores"]["marginal_per_block"] = marginal
    out["fidelity_tc_vs_complex128"] = Q.calcFidelity(states["complex128_simt"], states["complex64_tensor_cores"])
    out["fidelity_simt_complex64_vs_complex128"] = Q.calcFidelity(states["complex128_simt"],
                                                                  states["complex64_simt"])
    out["speedup_tc_vs_simt_complex64"] = (out["complex64_simt"]["ms_per_block"] /
                                           out["complex64_tensor_cores"]["ms_per_block"])
    for q in states.values():
        Q.destroyQureg(q, env)
    Q.destroyQuESTEnv(env)
    return out


def run_precision_form(args, world):
    """Precision form on its own workload: the 4x8 grid circuit of depth 16
    (sqrt X / sqrt Y / sqrt W, never the same gate twice in a row on a qubit,
    CZ on the 4 alternating edge patterns) on 32 qubits, complex64 (32 GiB)
    against complex128 (64 GiB) of the same seed."""
    import torch

    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    n, depth = 32, 16
    ops = C.grid_sqrt(4, 8, depth, C.config_seed(3))
    # dgQuEST's own GPU path on the same circuit first (its process needs the
    # 64 GiB of a complex128 state while this one holds none)
    ref = run_reference_gpu(args, n, ops) if not args.no_ref_gpu and world == 1 else None
    env = Q.createQuESTEnv()
    out = {"workload": "4x8 grid, depth 16, sqrt-X/Y/W + CZ patterns, 32 qubits", "qubits": n, "depth": depth}
    regs = {}
    for name, single in (("complex128", False), ("complex64", True)):
        q = Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env)
        Q.initZeroState(q)
        Q.apply_circuit(q, ops)
        Q.dgq_planPending(q)
        st = Q.plan_stats(q)
        stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
        for _ in range(args.warmup):
            Q.dgq_launchPlanned(q)
        torch.cuda.synchronize()
        steps = max(1, min(args.steps, 3))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            Q.dgq_launchPlanned(q)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
        amp = 8 if single else 16
        out[name] = {"ms_per_circuit": ms, "sweeps": st.sweeps, "tile_bits": st.tileBits, "plan_stats": st,
                     "hbm_gbs": 2.0 * (1 << n) * amp * st.sweeps / (ms / 1e3) / 1e9,
                     "gate_layers_per_s": depth / (ms / 1e3)}
        regs[name] = q
    q64, q32 = regs["complex128"], regs["complex64"]
    out["fidelity"] = Q.calcFidelity(q64, q32)
    idx = np.random.RandomState(3).randint(0, 1 << n, size=2048)
    err = 0.0
    for i in idx:
        a = Q.getAmp(q64, int(i))
        b = Q.getAmp(q32, int(i))
        err = max(err, abs(complex(a.real, a.imag) - complex(b.real, b.imag)))
    out["max_abs_err_sampled"] = err
    out["amplitudes_sampled"] = len(idx)
    if ref is not None and "sample_amps" in ref:
        # both precisions against the reference's own amplitudes
        ridx = ref.pop("sample_indices")
        ramps = ref.pop("sample_amps")
        for name in ("complex128", "complex64"):
            amps = [Q.getAmp(regs[name], int(i)) for i in ridx]
            ours = np.array([complex(a.real, a.imag) for a in amps])
            ref[f"max_abs_err_{name}_vs_reference"] = float(np.abs(ours - ramps).max())
        ref["amplitudes_compared"] = len(ridx)
    if ref is not None:
        out["reference_gpu"] = ref
    out["speedup_complex64"] = out["complex128"]["ms_per_circuit"] / out["complex64"]["ms_per_circuit"]
    out["arithmetic"] = "complex64 paired form (packed FP32 SIMT register phases)"
    for name in ("complex128", "complex64"):
        st_ = out[name].pop("plan_stats")
        out[name]["form_choice"] = form_report(st_, {"tiles": out[name]["ms_per_circuit"]})
    Q.destroyQureg(q32, env)
    if not args.no_tc_blocks:
        # the same circuit fused into dense 6-qubit blocks, each a split-FP16 GEMM
        # on the tensor cores (one warm-up and one timed run: seconds each)
        q = Q.dgq_createQuregF32(n, env)
        Q.dgq_setDenseFusion(q, 6)
        Q.initZeroState(q)
        Q.apply_circuit(q, ops)
        Q.dgq_planPending(q)
        st = Q.plan_stats(q)
        stream = torch.cuda.ExternalStream(Q.dgq_getStream(q))
        Q.dgq_launchPlanned(q)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Q.dgq_launchPlanned(q)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        err = 0.0
        for i in idx:
            a = Q.getAmp(q64, int(i))
            b = Q.getAmp(q, int(i))
            err = max(err, abs(complex(a.real, a.imag) - complex(b.real, b.imag)))
        out["complex64"]["form_choice"]["measured_ms"]["dense_k6_tensor_cores"] = round(ms, 2)
        out["complex64_tensor_core_blocks"] = {
            "ms_per_circuit": ms, "dense_blocks": int(st.denseBlocks), "sweeps": st.sweeps,
            "tensor_tflops_algorithmic": st.denseBlocks * (1 << n) * 1536.0 / (ms / 1e3) / 1e12,
            "fidelity": Q.calcFidelity(q64, q), "max_abs_err_sampled": err,
            "device_errors": int(Q.dgq_getDeviceErrors()),
            "vs_paired_form": ms / out["complex64"]["ms_per_circuit"],
            "note": "gates fused into dense 6-qubit unitaries (FP64 composition), one tcgen05 kind::f16 "
                    "split-FP16 GEMM sweep per block; warm-up 1, timed 1"}
        Q.destroyQureg(q, env)
    Q.destroyQureg(q64, env)
    Q.destroyQuESTEnv(env)
    return out


def l2_read_gbs():
    """Read bandwidth of a 48 MiB buffer that stays in L2 (FP32 sums, best of
    5 runs of 100, CUDA events): the yardstick of work whose data lives in
    L2, like a batch of small registers."""
    import torch
    x = torch.ones(12 << 20, dtype=torch.float32, device="cuda")
    out = torch.empty((), dtype=torch.float32, device="cuda")
    for _ in range(3):
        torch.sum(x, dim=0, out=out)
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(100):
            torch.sum(x, dim=0, out=out)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 4.0 * x.numel() * 100 / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def run_batch_form(args, world):
    """Batched form: 4096 ansatz circuits (n in [10, 22], depth in [4, 32]) in
    one persistent launch per step, complex128 and complex64; tile width and
    grouping from the autotuner, the launch replayed from a CUDA graph."""
    import torch

    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    wl = C.batch_workload(args.batch_circuits)
    env = Q.createQuESTEnv()
    out = {"workload": f"{len(wl)} hardware-efficient ansatz circuits, n~U[10,22], depth~U[4,32], <Z_q> of every qubit",
           "circuits": len(wl), "gates": int(sum(len(o) for _, _, o in wl))}
    steps = max(1, min(args.steps, 5))
    l2 = l2_read_gbs()
    pk = ctypes.c_double(0.0)
    Q.dgq_measureFp64Peak(ctypes.byref(pk))
    out["l2_read_gbs_measured"] = l2
    out["fp64_peak_tflops_measured"] = pk.value
    for name, single in (("complex128", False), ("complex64", True)):
        regs = [Q.dgq_createQuregF32(n, env) if single else Q.createQureg(n, env) for n, _, _ in wl]
        t0 = time.perf_counter()
        for q, (n, d, ops) in zip(regs, wl):
            Q.initZeroState(q)
            Q.apply_circuit(q, ops)
        record_ms = (time.perf_counter() - t0) * 1e3
        b = Q.Batch(regs)
        st = b.stats()
        stream = torch.cuda.ExternalStream(b.stream())
        for _ in range(args.warmup):
            b.launch()
        b.wait()
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.launch()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
        z = b.expectation_z()
        b.close()
        # end to end through the API: record every circuit, plan (tuning
        # cached), upload, launch, read <Z> back
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for q, (n, d, ops) in zip(regs, wl):
            Q.initZeroState(q)
            Q.apply_circuit(q, ops)
        b2 = Q.Batch(regs)
        b2.launch()
        z2 = b2.expectation_z()
        e2e_ms = (time.perf_counter() - t0) * 1e3
        st2 = b2.stats()
        b2.close()
        for q in regs:
            Q.destroyQureg(q, env)
        hbm = peaks()[0]
        out[name] = {"ms_per_launch": ms, "circuits_per_s": world * len(wl) / (ms / 1e3),
                     "hbm_gbs_algorithmic": st.sweepBytes / (ms / 1e3) / 1e9,
                     "roofline_frac": st.sweepBytes / (ms / 1e3) / 1e9 / hbm,
                     "l2_frac": st.sweepBytes / (ms / 1e3) / 1e9 / l2,
                     "flop_tflops_algorithmic": st.flopsPerLaunch / (ms / 1e3) / 1e12,
                     "fp64_frac": (st.flopsPerLaunch / (ms / 1e3) / 1e12 / pk.value) if not single else None,
                     "bound_note": "registers of <= 2^22 amplitudes stay in L2: against HBM, the measured L2 "
                                   "read bandwidth and (complex128) the FP64 peak",
                     "sweep_bytes": int(st.sweepBytes), "state_bytes": int(st.stateBytes),
                     "tile_bits": st.tileBits, "group_factor": st.groupFactor, "grid": st.grid,
                     "ctas_per_sm": st.ctasPerSm, "items": int(st.items), "sweeps": st.sweeps,
                     "whole_register_items": st.wholeRegisters, "tuned": bool(st.tuned),
                     "tune_ms": st.tuneMillis, "plan_ms": st.planMillis, "record_ms": record_ms,
                     "e2e_ms": e2e_ms, "e2e_plan_ms": st2.planMillis,
                     "e2e_h2d_bytes": int(st2.programBytes), "e2e_d2h_bytes": int(8 * len(z2)),
                     "z_abs_max": float(np.abs(z).max()), "z_repeat_max_diff": float(np.abs(z - z2).max())}
    Q.destroyQuESTEnv(env)
    return out


def run_serving_form(args, world):
    """Serving loop: Poisson arrivals at 200 requests/s, n uniform in [16, 33]
    (complex64) or [16, 32] (complex128), 40/30/30 random / GHZ+QFT / BV,
    1024 samples and <Z> on 4 qubits per request; the first --serve-requests
    requests of the stream, admitted by state bytes against free HBM."""
    from dgquest_b200 import circuits as C
    from dgquest_b200 import quest as Q
    from dgquest_b200 import serving as S
    env = Q.createQuESTEnv()
    out = {"workload": "Poisson arrivals 200/s; random(depth 8-24)/GHZ+QFT/BV 40/30/30; 1024 samples + <Z> on 4 qubits",
           "requests_per_precision": args.serve_requests, "warmup_requests": args.serve_warmup}
    for name, single in (("complex64", True), ("complex128", False)):
        reqs = S.make_requests(args.serve_requests, rate=200.0, single=single)
        srv = S.Server(env, workers=args.serve_workers, keep_resident=True, spec_policy=args.serve_policy)
        # a running server: memory pool grown, then a warm-up stream of other
        # requests (same distribution, another seed) before the measured one
        srv.prewarm(single)
        specialised = srv.prespecialise(single)
        warm = S.make_requests(args.serve_warmup, rate=200.0, single=single, seed=C.config_seed(5, 900000),
                               first_id=200000)
        cold = S.summarize(srv.serve(warm, realtime=True)) if warm else None
        res = srv.serve(reqs, realtime=True)
        st = S.summarize(res)
        # the same server at lower offered rates: where latency stops being
        # queueing (service time = done - admitted, queueing = admitted - arrival)
        sweep = []
        for k, rate in enumerate(float(x) for x in args.serve_rates.split(",") if x):
            low = S.make_requests(args.serve_rate_requests, rate=rate, single=single,
                                  seed=C.config_seed(5, 910000 + k), first_id=300000 + 1000 * k)
            rs = srv.serve(low, realtime=True)
            lo = S.summarize(rs)
            svc = np.array([r.done - r.admitted for r in rs]) * 1e3
            que = np.array([r.admitted - r.arrival for r in rs]) * 1e3
            big = [r.latency * 1e3 for r, q in zip(rs, low) if q.n >= 31]
            small = [r.latency * 1e3 for r, q in zip(rs, low) if q.n <= 28]
            sweep.append({"offered_rate": rate, "requests": lo["requests"], "p50_ms": lo["p50_ms"],
                          "p99_ms": lo["p99_ms"], "circuits_per_s": lo["circuits_per_s"],
                          "service_p50_ms": float(np.percentile(svc, 50)), "service_p99_ms": float(np.percentile(svc, 99)),
                          "queue_p99_ms": float(np.percentile(que, 99)),
                          "p99_ms_n_le_28": float(np.percentile(small, 99)) if small else None,
                          "p50_ms_n_ge_31": float(np.percentile(big, 50)) if big else None})
        st["rate_sweep"] = sweep
        st["registers_reused"] = srv.reused
        st["prespecialised_kernels"] = specialised
        srv.close()
        if cold:
            st["warmup_stream"] = {"requests": cold["requests"], "p50_ms": cold["p50_ms"], "p99_ms": cold["p99_ms"],
                                   "circuits_per_s": cold["circuits_per_s"]}
        st.update({"peak_in_flight": srv.peak_in_flight, "peak_state_gb": srv.peak_in_use / 1e9,
                   "budget_gb": srv.budget / 1e9, "offered_rate": 200.0,
                   "offered_state_gb_per_s": sum(S.state_bytes(r) for r in reqs) / reqs[-1].arrival / 1e9,
                   "n_range": [min(r.n for r in reqs), max(r.n for r in reqs)]})
        out[name] = st
    Q.destroyQuESTEnv(env)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dgq", choices=["dgq", "reference"])
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--tile-bits", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the run of dgQuEST's own GPU path (oracle/_ref/ref_harness)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-grid32", action="store_true")
    ap.add_argument("--serve-warmup", type=int, default=60, help="requests of the serving warm-up stream")
    ap.add_argument("--serve-rates", default="4,8,12",
                    help="offered rates (req/s) of the serving rate sweep on the same server ('' to skip)")
    ap.add_argument("--serve-rate-requests", type=int, default=60, help="requests per rate of the sweep")
    ap.add_argument("--serve-policy", type=int, default=1, choices=[1, 2],
                    help="specialisation policy of the serving loop (2: no background compiles)")
    ap.add_argument("--no-host-tier", action="store_true", help="skip the host-tier (pinned host memory) run")
    ap.add_argument("--no-shards", action="store_true", help="skip the sharded-register run")
    ap.add_argument("--no-tc-blocks", action="store_true", help="skip the dense-block tensor-core run of the grid circuit")
    ap.add_argument("--no-dense", action="store_true")
    ap.add_argument("--dense-qubits", type=int, default=30)
    ap.add_argument("--batch-circuits", type=int, default=4096)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--batch-case", type=int, default=0, help="--ncu-case: a batch of this many workload circuits")
    ap.add_argument("--dense-case", action="store_true", help="--ncu-case: dense 6-qubit unitaries, complex64")
    ap.add_argument("--serve-requests", type=int, default=120)
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--precision", type=int, default=2, choices=[1, 2], help="--ncu-case register precision")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run one small case once (for ncu captures): --qubits/--depth/--tile-bits, specialised kernels")
    args = ap.parse_args()
    if args.ncu_case:
        run_ncu_case(args)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "dgq" else args.warmup

    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu and args.qubits == N_QUBITS and args.depth == DEPTH:
        # first, while this process holds no device memory of its own
        ref_gpu = run_reference_gpu(args)
    line = run_gpu(args, world, rank, local, ref_gpu)
    if not args.no_dense:
        dense = run_dense_form(args, world)
        if rank == 0:
            line["dense_blocks"] = dense
    if not args.no_host_tier and rank == 0 and world == 1:
        line["host_tier"] = run_host_tier_form(args, world)
    if not args.no_shards and rank == 0 and world == 1:
        line["sharded"] = run_sharded_form(args, world)
    if not args.no_grid32:
        grid = run_precision_form(args, world)
        if rank == 0:
            line["precision_form_grid32"] = grid
    if not args.no_batch:
        batch = run_batch_form(args, world)
        if rank == 0:
            line["batched_form"] = batch
    if not args.no_serve and rank == 0:
        line["serving"] = run_serving_form(args, world)
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle
        from dgquest_b200 import circuits as C
        ops = C.random_layers(N_QUBITS, DEPTH, C.config_seed(2))
        cores = oracle.max_threads()
        t_all = cpu_time_ops(N_QUBITS, [ops[:2], layer_of(ops, N_QUBITS, 0)], cores)[1]
        t_one, one_desc = cpu_one_core_layer(ops, N_QUBITS)
        oracle.set_threads(cores)
        line["cpu_baseline"] = {"value": 1.0 / (t_all * DEPTH), "unit": "circuits/s", "cores": cores,
                                "kind": "port", "extrapolated": True,
                                "sample": f"oracle (OpenMP, {cores} threads) on layer 0 of the 30-qubit circuit "
                                          f"(30 rotations + 15 CZ, {t_all:.2f} s), x {DEPTH} layers",
                                "one_core": {"value": 1.0 / (t_one * DEPTH), "unit": "circuits/s", "cores": 1,
                                             "sample": one_desc}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
