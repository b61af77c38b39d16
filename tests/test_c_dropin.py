"""A plain C program written against include/QuEST.h (tests/c/quest_dropin.c)
builds and links with libdgq.so alone (CPU), and on the GPU prints the
oracle's amplitudes (1e-12), P(q=0) (1e-12) and measurement outcomes
(bit-exact, seeded) for GHZ+QFT (also on a sharded register) and for a
mixed circuit with a multi-qubit unitary."""
import math
import os
import subprocess

import numpy as np
import pytest

import oracle
from dgquest_b200 import circuits as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "quest_dropin.c")
LIBDIR = os.path.join(ROOT, "dgquest_b200")


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("c") / "quest_dropin")
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR,
           "-ldgq", "-Wl,-rpath," + LIBDIR, "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_builds_against_the_header(dropin):
    assert os.path.exists(dropin)


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p0, amps, outcomes = {}, {}, {}
    for line in r.stdout.splitlines():
        f = line.split()
        if f[0] == "p0":
            p0[int(f[1])] = float(f[2])
        elif f[0] == "amp":
            amps[int(f[1])] = complex(float(f[2]), float(f[3]))
        elif f[0] == "outcome":
            outcomes[int(f[1])] = int(f[2])
    n = len(p0)
    return (np.array([p0[k] for k in range(n)]), np.array([amps[i] for i in range(1 << n)]),
            [outcomes[k] for k in sorted(outcomes)])


def mixed_ops(n):
    b = C.OpList()
    for k in range(n):
        b.add(C.RX, k, p=(0.1 + 0.37 * k,))
        b.add(C.RY, (k + 1) % n, p=(-0.2 + 0.11 * k,))
        b.add(C.RZ, (k + 2) % n, p=(0.3 * k,))
    a = complex(math.cos(0.4) * math.cos(0.9), math.cos(0.4) * math.sin(0.9))
    bb = complex(math.sin(0.4) * math.cos(-0.3), math.sin(0.4) * math.sin(-0.3))
    b.add(C.COMPACT, 1, p=(a.real, a.imag, bb.real, bb.imag))
    b.add(C.CNOT, 0, n - 1)
    b.add(C.CPHASE, 2, 3, p=(0.77,))
    b.add(C.CZ, 1, 4)
    b.add(C.X, 5)
    b.add(C.Z, 6)
    post = C.OpList()
    for k in range(n):
        post.add(C.H, k)
    for k in range(3):
        post.add(C.MEASURE, k)
    post.add(C.RY, 4, p=(0.5,))
    dft = np.array([[np.exp(2j * np.pi * r * c / 8) for c in range(8)] for r in range(8)]) / math.sqrt(8)
    return b.array(), dft, post.array()


@pytest.mark.gpu
def test_c_program_ghz_qft_matches_oracle(quest, dropin):
    n = 16
    p0, amps, _ = run(dropin, "ghzqft", n)
    ref, ref_p0, _ = oracle.run(n, C.ghz_qft(n))
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12


@pytest.mark.gpu
def test_c_program_sharded_register_matches_oracle(quest, dropin):
    """The same calls on a register in 4 shards (2 qubits above each shard,
    so the QFT's gates on them go through qubit exchanges)."""
    n = 16
    p0, amps, _ = run(dropin, "sharded", n)
    ref, ref_p0, _ = oracle.run(n, C.ghz_qft(n))
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12


@pytest.mark.gpu
def test_c_program_mixed_matches_oracle(quest, dropin):
    n = 14
    p0, amps, outcomes = run(dropin, "mixed", n)
    pre, dft, post = mixed_ops(n)
    o = oracle.Oracle(n)
    o.seed([12345, 67890])
    o.apply(pre)
    o.multi_qubit_unitary([2, 5, 7], dft)
    ref_out = o.apply(post)
    ref = o.amps()
    ref_p0 = o.prob_zero_all()
    o.close()
    assert outcomes == ref_out
    assert np.abs(amps - ref).max() <= 1e-12
    assert np.abs(p0 - ref_p0).max() <= 1e-12
