"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks, as
torchrun would start them (RANK / WORLD_SIZE / MASTER_ADDR on 127.0.0.1).
Checks the max-over-ranks timing, the barrier, and that only rank 0 runs
and prints the reference arm."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(world, backend="gloo")
    bench.barrier(w)
    mx = bench.max_over_ranks(1.5 + r, w)
    # the reference arm: rank 0 alone times and prints (here on a tiny sample)
    buf = io.StringIO()

    class Args:
        gpus, steps, warmup, ref_gates = world, 1, 0, 1
    if r != 0:
        with redirect_stdout(buf):
            bench.run_reference_arm(Args, w, r)
    bench.barrier(w)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"world": w, "rank": r, "max": mx, "printed": buf.getvalue()}, f)
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [x["rank"] for x in res] == [0, 1]
    assert all(x["world"] == 2 for x in res)
    assert all(x["max"] == pytest.approx(2.5) for x in res)
    assert res[1]["printed"] == ""  # non-zero ranks run no reference work and print nothing
