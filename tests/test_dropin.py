"""The single-rank drop-in: the C++ API program (tests/cpp/dropin_sanity.cpp,
built against include/dsdecompx.hpp and libdsx.so) and the C-ABI migrate,
checked against the oracle's 1-rank migrate bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from helpers import same
from oracle import Grid

pytestmark = pytest.mark.gpu


def oracle_wrap(x, y, z, lower, upper):
    g = Grid("port", 1, (1, 1, 1), "manual", lower, upper)
    g.set_owned(0, dict(x=x, y=y, z=z, global_id=np.arange(len(x), dtype=np.int32)))
    res = g.migrate()
    assert res[0, 5] == len(x)
    return g.read(0, "x"), g.read(0, "y"), g.read(0, "z")


def test_cpp_dropin_sanity(cuda, tmp_path):
    import dsdecompx_b200 as dsx
    exe = os.path.join(os.path.dirname(dsx.library_path()), "dropin_sanity")
    assert os.path.exists(exe), "tests/cpp programs are built by __graft_entry__.build()"
    out = tmp_path / "positions.bin"
    proc = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=120)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "dropin_sanity: ok" in proc.stdout
    data = np.fromfile(out, dtype=np.float64).reshape(6, -1)
    want = oracle_wrap(data[0], data[1], data[2], (0.0, 0.0, 0.0), (10.0, 10.0, 10.0))
    for a in range(3):
        assert same(data[3 + a], want[a]), a


def test_cpp_grid_sanity(cuda):
    """The virtual grid's C++ face (include/dsx_grid.hpp) in a C++ program:
    id conservation, sum of reverse == #ghosts per call and per captured
    step, split-phase misuse and bad cuts raise the reference's types."""
    import dsdecompx_b200 as dsx
    exe = os.path.join(os.path.dirname(dsx.library_path()), "grid_sanity")
    assert os.path.exists(exe), "tests/cpp programs are built by __graft_entry__.build()"
    proc = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "grid_sanity: ok" in proc.stdout


@pytest.mark.gpu
def test_cpp_shard_sanity(cuda):
    """The native sharded grid (include/dsx_shard.h) in a C++ program: shards
    as threads on one GPU with a barrier-and-copy transport, every array of
    every subdomain equal to one grid's after migrate, halo build, reverse
    sums, field exchanges and refresh (Manual over 4 shards, Dynamic over 2)."""
    import dsdecompx_b200 as dsx
    exe = os.path.join(os.path.dirname(dsx.library_path()), "shard_sanity")
    assert os.path.exists(exe), "tests/cpp programs are built by __graft_entry__.build()"
    proc = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "shard_sanity: ok" in proc.stdout


@pytest.mark.parametrize("lower,upper", [((0.0, 0.0, 0.0), (100.0, 100.0, 100.0)),
                                         ((-3.7, 1e-3, 1e6), (5.1, 0.3, 1e6 + 7.25))])
def test_rank_migrate_matches_oracle(cuda, lower, upper):
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(31)
    n = 200_000
    lo, hi = np.asarray(lower), np.asarray(upper)
    ext = hi - lo
    pos = lo + ext * rng.uniform(-2.5, 3.5, size=(n, 3))
    # edge values: faces, just outside, signed zero relative to the lower face,
    # far away, and values whose wrap rounds onto the upper face
    edge = np.array([lo, hi, lo - 1e-17, hi + 1e-12, lo + 0.0, lo * 1.0 - 5e-324,
                     lo + 1e9 * ext, lo - 3e7 * ext, np.nextafter(hi, -np.inf), np.nextafter(lo, -np.inf)])
    pos[:len(edge)] = edge
    x, y, z = (torch.tensor(pos[:, a].copy(), device="cuda") for a in range(3))
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    res = dsx.rank_migrate(x, y, z, n, lower, upper, stream=stream)
    stream.synchronize()
    assert res["new_owned_count"] == n and res["sent_count"] == 0
    want = oracle_wrap(pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), lower, upper)
    for t, w in zip((x, y, z), want):
        assert same(t.cpu().numpy(), w)


def test_rank_migrate_requires_a_stream(cuda):
    import torch

    import dsdecompx_b200 as dsx
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="explicit communication stream"):
        dsx.rank_migrate(x, x, x, 4, (0, 0, 0), (1, 1, 1), stream=0)
