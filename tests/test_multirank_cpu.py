"""Multi-rank paths of bench.py on CPU (gloo, world size 2, 127.0.0.1).

FDK reconstructions do not shard: N GPUs run N independent replicas of the workload with no
collective on the data path. What the N > 1 run adds is host logic: every rank's time is reduced
to the maximum over ranks before rates are formed, the rate counts the units of all ranks, and
the reference arm prints its line on rank 0 only while the other ranks exit without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch
    sys.path.insert(0, str(REPO))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 1 + 0.5 r seconds; the job's time is the slowest rank's
        t = bench.max_over_ranks(1.0 + 0.5 * rank, "cpu")
        rate = bench.replica_rate(1000.0, world, 3, t)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"t": t, "rate": rate}, f)
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    for r in res:
        assert r["t"] == pytest.approx(1.5)
        # 1000 units per rank per step, 3 steps, 2 ranks, over the slowest rank's 1.5 s
        assert r["rate"] == pytest.approx(1000.0 * 2 * 3 / 1.5)


def test_max_over_ranks_single_process():
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.max_over_ranks(2.25, "cpu") == 2.25
    assert bench.replica_rate(10.0, 1, 4, 2.0) == pytest.approx(20.0)


def test_reference_arm_two_ranks_rank0_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(REPO / "bench.py"), "--impl", "reference", "--config", "fan256", "--gpus", "2",
           "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=str(REPO), capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2
    assert line["value"] > 0 and line["unit"] == "GUPS"
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
