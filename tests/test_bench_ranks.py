"""Host logic of bench.py's multi-process path, on CPU with gloo.

bench.py --gpus N runs one process per GPU (the sharded grid, one block of
subdomains per rank, weak scaling): every rank times its own steps and the
job reports the slowest rank's time; the reference arm runs on rank 0 only.
Both are checked here with two gloo ranks and no GPU.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        mine = 1.0 + 1.5 * rank
        slowest = bench.max_over_ranks(mine, world)
        single = bench.max_over_ranks(mine, 1)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"slowest": slowest, "single": single}, f)
    finally:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def test_slowest_rank_over_gloo(tmp_path):
    world = 2
    mp.start_processes(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn")
    for r in range(world):
        got = json.load(open(tmp_path / f"rank{r}.json"))
        assert got["slowest"] == 2.5          # every rank sees rank 1's time
        assert got["single"] == 1.0 + 1.5 * r  # one rank: its own


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
