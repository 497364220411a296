"""The multi-rank plumbing of bench.py on CPU (gloo, two ranks): the step time
every rank reports is the largest over the ranks, barriers pass, and the
reference arm runs on rank 0 only (other ranks exit at once with nothing
printed).  On GPUs the same functions run over NCCL, one process per GPU,
each rank stepping its own replica of the workload."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local = bench.ranks()
    assert (r, w, local) == (rank, world, rank)
    bench.init_ranks(w, "gloo")
    bench.barrier(w)
    ms = 10.0 + 7.5 * r  # this rank's step time
    got = bench.max_over_ranks(ms, w, "cpu")
    bench.barrier(w)
    bench.close_ranks(w)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(repr(got))


def test_max_over_ranks_gloo(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    vals = [float((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    assert vals == [17.5, 17.5]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25
    bench.barrier(1)
    bench.init_ranks(1)
    bench.close_ranks(1)


@pytest.mark.parametrize("impl", ["reference"])
def test_reference_arm_other_ranks_exit(impl):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", impl, "--gpus", "2", "--n", "64",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, timeout=300, env=env,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
