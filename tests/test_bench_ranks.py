"""The multi-process side of bench.py, on the CPU with gloo ranks.

A system of this solver does not shard: with N GPUs bench.py runs N independent
replicas, one process per GPU, each factoring and solving its own seeded system
with no collective on the data path.  The only cross-rank steps are the barrier
before the timed region and the maximum of the per-rank times, from which rank 0
reports the whole job's unknowns/s.  These tests run those steps with two gloo
ranks; the reference arm's rule (rank 0 alone works and prints, the others exit
0) runs through torch.distributed.run with two processes."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _replica_rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = 1.0 + 0.5 * rank          # rank 1 is the slowest
        worst = bench.max_over_ranks(dist, ms, "cpu")
        e2e = bench.max_over_ranks(dist, 10.0 - rank, "cpu")   # rank 0 is the slowest here
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"worst": worst, "e2e": e2e, "seeds": bench.replica_seeds(rank)}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_replica_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # every rank sees the same maxima, in the order the collectives were issued
    assert [r["worst"] for r in res] == [1.5, 1.5]
    assert [r["e2e"] for r in res] == [10.0, 10.0]
    # each replica solves its own system
    assert len({tuple(r["seeds"]) for r in res}) == world


def test_whole_job_value_counts_every_replica():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25
    assert bench.whole_job_value(1, 1000, 0.5) == 2000.0
    assert bench.whole_job_value(4, 1000, 0.5) == 8000.0


def test_reference_arm_under_torchrun_prints_once(tmp_path):
    """`bench.py --impl reference` launched like the GPU arm with two ranks:
    rank 0 times the reference on the host cores and prints one JSON line, the
    other rank exits 0 without work."""
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as po
    if not po.ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["steps"] == 1
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
