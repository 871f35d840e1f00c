"""Host logic of bench.py, on CPU (no GPU).

bench.py --gpus N runs one process per GPU (the sharded grid, one block of
subdomains per rank, weak scaling): every rank times its own steps and the
job reports the slowest rank's time; the reference arm runs on rank 0 only
and prints the contract's line.  Both are checked here, the first with two
gloo ranks.  The clock sampler that fills the line's `clocks` runs against an
nvidia-smi stand-in.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
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


def test_reference_arm_line():
    """Rank 0 of the reference arm prints one JSON line with the contract's
    keys: the reference Host path's rate as value, cpu_baseline and e2e
    describing the same run, no host-device bytes (one-rank workload, a
    second of CPU work)."""
    import oracle
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "drop_in_1rank", "--steps", "1", "--warmup", "1"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = p.stdout.strip().splitlines()
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    if not oracle.available("ref"):
        assert "unavailable" in line
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["workload"] == "drop_in_1rank"
    base = line["cpu_baseline"]
    assert base["kind"] == "reference" and base["value"] == line["value"] and base["cores"] == 1
    assert base["unit"] == line["unit"] and base["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # the same config object as the GPU arm prints, and the declared step counts
    sys.path.insert(0, ROOT)
    import bench
    w = bench.load_workloads().WORKLOADS["drop_in_1rank"]
    assert line["config"] == bench.workload_config(w, 1, (1, 1, 1))
    assert line["steps"] == 1 and line["warmup"] == 1 and line["ms_per_step"] > 0
    assert "1 timed steps after 1 warm-up" in base["sample"]


def test_reference_arm_loads_nothing_of_the_product():
    """The reference arm runs the reference build alone: no module of the
    product package is imported and no library of it is mapped."""
    import oracle
    if not oracle.available("ref"):
        pytest.skip("reference build not present")
    probe = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'clustered_64',\n"
        "            '--steps', '1', '--warmup', '1', '--particles', '20000']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "mods = sorted(m for m in sys.modules if m.startswith('dsdecompx_b200'))\n"
        "maps = sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')})\n"
        "print('PROBE', mods, [m for m in maps if 'dsdecompx_b200' in m], file=sys.stderr)\n")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    p = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert "PROBE [] []" in p.stderr, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["config"]["subdomains"] == 64 and line["config"]["grid"] == [4, 4, 4]


def test_shard_factors_cover_the_rank_count():
    """bench.py's weak-scaling layout: N ranks as (a, b, c) blocks of the
    workload, a * b * c = N, the prime factors spread over the axes."""
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_factors(1) == (1, 1, 1)
    assert bench.shard_factors(2) == (2, 1, 1)
    assert bench.shard_factors(4) == (2, 2, 1)
    assert bench.shard_factors(8) == (2, 2, 2)
    for n in range(1, 33):
        a, b, c = bench.shard_factors(n)
        assert a * b * c == n and max(a, b, c) <= n


def test_sharded_process_grids_are_blocks_of_the_workload():
    """For the default workload at 2, 3, 4 and 8 ranks the planner's process
    grid of the grown box is the workload's grid times the block counts, so
    every rank owns exactly one block (bench.py refuses to run otherwise)."""
    sys.path.insert(0, ROOT)
    import bench
    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    w = W.WORKLOADS["clustered_64"]
    block, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    for n in (2, 3, 4, 8):
        fa = bench.shard_factors(n)
        upper = tuple(u * k for u, k in zip(w.upper, fa))
        dims, _ = dsx.plan_topology(w.nranks * n, 0, (0, 0, 0), w.policy, w.lower, upper)
        assert tuple(dims) == tuple(d * k for d, k in zip(block, fa)), (n, dims)


def _fake_nvidia_smi(tmp_path, row):
    """An nvidia-smi stand-in on PATH that prints `row` every 10 ms."""
    tool = tmp_path / "nvidia-smi"
    tool.write_text("#!/bin/sh\nwhile true; do echo '%s'; sleep 0.01; done\n" % row)
    tool.chmod(0o755)
    return dict(os.environ, PATH=str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))


def _sample(env):
    import time
    sys.path.insert(0, ROOT)
    import bench
    old = os.environ["PATH"]
    os.environ["PATH"] = env["PATH"]
    try:
        with bench.ClockSampler(0) as clocks:
            time.sleep(0.2)
        return clocks.summary()
    finally:
        os.environ["PATH"] = old


def test_clock_sampler_reads_clocks_and_reasons(tmp_path):
    """The sampler behind the bench line's `clocks`: the median SM clock, the
    maximum, and every throttle reason seen active during the region."""
    capped = _sample(_fake_nvidia_smi(
        tmp_path, "0, 1965, 1965, 990.10, 0x4, Not Active, Not Active, Not Active, Active"))
    assert capped["sm_mhz"] == 1965.0 and capped["sm_max_mhz"] == 1965.0
    assert capped["reasons"] == ["sw_power_cap"] and capped["samples"] >= 1
    slowed = _sample(_fake_nvidia_smi(
        tmp_path, "0, 1200, 1965, 500.00, 0x8, Active, Active, Not Active, Not Active"))
    assert slowed["sm_mhz"] == 1200.0
    assert slowed["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]


def test_clock_sampler_without_nvidia_smi(tmp_path):
    env = dict(os.environ, PATH=str(tmp_path))   # no nvidia-smi anywhere on PATH
    assert _sample(env)["reasons"] == ["unavailable"]
