"""Sharded virtual grid on the device: R shards (each a CUDA grid of all P
subdomains holding only its own block) run in lockstep on one GPU, their
exchanges served as device buffers, and every array of every subdomain is
compared bit for bit with one CUDA grid that holds all P subdomains (itself
checked against the oracle by test_gpu_parity.py).  The segment copies and
the assembly of the owned particles are also checked directly.
"""
import numpy as np
import pytest

from helpers import ALL_FIELDS, same
from oracle import Grid
from shard_scenario import Scenario, initial, lockstep_drive

pytestmark = pytest.mark.gpu

TYPE_INDEX = {"int32": 0, "int64": 1, "uint32": 2, "uint64": 3, "float32": 4, "float64": 5}

CASES = {
    "4x4x4-R8": dict(nranks=64, dims=(4, 4, 4), policy="manual", upper=(16.0, 16.0, 16.0),
                     halo_width=1.0, N=120_000, R=8, fields=ALL_FIELDS[:3]),
    "2x2x2-R2-all-fields": dict(nranks=8, dims=(2, 2, 2), policy="manual", upper=(10.0, 10.0, 10.0),
                                halo_width=1.0, N=20_000, R=2, fields=ALL_FIELDS),
    "3x1x4-R3-open": dict(nranks=12, dims=(3, 1, 4), policy="manual", upper=(9.0, 5.0, 12.0),
                          periodic=(True, False, False), halo_width=0.8, N=20_000, R=3,
                          fields=ALL_FIELDS[:2]),
    "dynamic-4x4x2-R4": dict(nranks=32, dims=(4, 4, 2), policy="dynamic", upper=(24.0, 24.0, 12.0),
                             halo_width=0.9, dynamic=(1.0, 1.05, 0.5, 0.1), N=60_000, R=4,
                             fields=ALL_FIELDS[:2]),
}


def grid_kw(kw):
    return dict(nranks=kw["nranks"], dims=kw["dims"], policy=kw["policy"], lower=(0.0, 0.0, 0.0),
                upper=kw["upper"], periodic=kw.get("periodic", (True, True, True)),
                halo_width=kw["halo_width"], dynamic=kw.get("dynamic"), fields=kw["fields"])


@pytest.mark.parametrize("case", list(CASES))
def test_lockstep_shards_match_one_grid(cuda, case):
    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    kw = CASES[case]
    P, R, N = kw["nranks"], kw["R"], kw["N"]
    owner = Grid("port", P, kw["dims"], kw["policy"], (0, 0, 0), kw["upper"],
                 kw.get("periodic", (True, True, True)), kw["halo_width"], True, kw.get("dynamic"),
                 [(n, TYPE_INDEX[t], c) for n, t, c in kw["fields"]])
    per = initial(owner, P, kw["upper"], N, 41, kw["fields"])
    owner.close()
    ref = dsx.VirtualGrid(**grid_kw(kw), particles=N, ghost_capacity=2 * N)
    ref.upload(per)
    shards = []
    for s in range(R):
        e = shd.DeviceEngine(**grid_kw(kw), particles=2 * N // R + 4096, ghost_capacity=N // R)
        shards.append(shd.ShardedGrid(e, s, R))
    try:
        for sh in shards:
            sh.upload({int(t): per[t] for t in sh.mine})
        Scenario(shards, lockstep_drive(shards), ref, P, kw["fields"]).run(steps=3, sigma=0.8)
        if kw["policy"] == "dynamic":
            for a, b in zip(ref.cuts(), shards[-1].E.grid.cuts()):
                assert same(a, b)
    finally:
        ref.close()
        for sh in shards:
            sh.E.close()


def test_copy_segments_any_alignment(cuda):
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(8)
    src = torch.randint(0, 256, (3 << 20,), dtype=torch.uint8, device="cuda")
    dst = torch.zeros(3 << 20, dtype=torch.uint8, device="cuda")
    want = dst.clone()
    rows = []
    at = 0
    for k in range(400):
        n = int(rng.choice([1, 3, 8, 17, 64, 1000, 4099, 300_000]))
        s0 = int(rng.integers(0, src.numel() - n))
        if at + n > dst.numel():
            break
        d0 = at + int(rng.integers(0, 16))
        if d0 + n > dst.numel():
            break
        rows.append((s0, d0, n))
        want[d0:d0 + n] = src[s0:s0 + n]
        at = d0 + n
    c = np.zeros(len(rows), dtype=dsx.COPY_DTYPE)
    for i, (s0, d0, n) in enumerate(rows):
        c[i] = (src.data_ptr() + s0, dst.data_ptr() + d0, n)
    dsx.copy_segments(c)
    torch.cuda.synchronize()
    assert torch.equal(dst, want)


def test_assemble_checks_its_segments(cuda):
    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(2)
    from helpers import split_by_owner, uniform_particles
    g = dsx.VirtualGrid(8, (2, 2, 2), "manual", (0, 0, 0), (10, 10, 10), halo_width=1.0,
                        particles=4000, ghost_capacity=4000)
    try:
        data = uniform_particles(rng, 1000, (0, 0, 0), (10, 10, 10))
        g.upload(split_by_owner(np.arange(1000) % 8, data, 8))
        before = {r: g.snapshot(r) for r in range(8)}
        # reverse the subdomain order: subdomain r gets what 7 - r held
        counts = np.array([g.counts(7 - r)[0] for r in range(8)], dtype=np.int64)
        o, _ = g.all_counts()
        ob = np.concatenate([[0], np.cumsum(o)])
        seg = np.zeros(8, dtype=dsx.SEGMENT_DTYPE)
        for r in range(8):
            seg[r] = (-1, ob[7 - r], r, 0, counts[r])
        g.assemble(counts, [], seg)
        for r in range(8):
            got = g.snapshot(r)
            for k in dsx.ARRAYS:
                assert same(got[k], before[7 - r][k]), (r, k)
        bad = seg.copy()
        bad[0]["count"] += 1
        with pytest.raises(ValueError):
            g.assemble(counts, [], bad)
        bad = seg.copy()
        bad[0]["source"] = 3
        with pytest.raises(ValueError):
            g.assemble(counts, [], bad)
        with pytest.raises(MemoryError):
            g.assemble(counts * 10, [], seg[:0])
    finally:
        g.close()


def test_one_shard_over_nccl(cuda):
    """The distributed driver over a one-rank NCCL group (its all-reduces on
    device tensors; a single shard has no peers): the sharded step of one
    shard equals the grid's own calls."""
    import datetime
    import os
    import socket

    import torch.distributed as dist

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    from shard_scenario import distributed_drive
    kw = CASES["dynamic-4x4x2-R4"]
    P, N = kw["nranks"], 30_000
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    owner = Grid("port", P, kw["dims"], kw["policy"], (0, 0, 0), kw["upper"], (True, True, True),
                 kw["halo_width"], True, kw["dynamic"], [(n, TYPE_INDEX[t], c) for n, t, c in kw["fields"]])
    per = initial(owner, P, kw["upper"], N, 43, kw["fields"])
    owner.close()
    ref = dsx.VirtualGrid(**grid_kw(kw), particles=N, ghost_capacity=2 * N)
    ref.upload(per)
    e = shd.DeviceEngine(**grid_kw(kw), particles=N + 4096, ghost_capacity=N)
    sh = shd.ShardedGrid(e, 0, 1)
    try:
        sh.upload({t: per[t] for t in range(P)})
        Scenario([sh], distributed_drive(sh), ref, P, kw["fields"]).run(steps=2, sigma=0.8)
    finally:
        ref.close()
        e.close()
        dist.destroy_process_group()


def test_native_shard_over_nccl(cuda):
    """The native sharded grid (dsx_shard_*) through its torch.distributed
    transport on a one-rank NCCL group: every call equals the grid's own."""
    import datetime
    import os
    import socket

    import torch.distributed as dist

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    from shard_scenario import distributed_drive
    kw = CASES["dynamic-4x4x2-R4"]
    P, N = kw["nranks"], 30_000
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    owner = Grid("port", P, kw["dims"], kw["policy"], (0, 0, 0), kw["upper"], (True, True, True),
                 kw["halo_width"], True, kw["dynamic"], [(n, TYPE_INDEX[t], c) for n, t, c in kw["fields"]])
    per = initial(owner, P, kw["upper"], N, 47, kw["fields"])
    owner.close()
    ref = dsx.VirtualGrid(**grid_kw(kw), particles=N, ghost_capacity=2 * N)
    ref.upload(per)
    sh = shd.NativeShardedGrid(**grid_kw(kw), particles=N + 4096, ghost_capacity=N)
    try:
        names = dsx.ARRAYS + [f[0] for f in kw["fields"]]
        counts = np.array([len(d["x"]) for d in per], dtype=np.int64)
        host = []
        for name in names:
            dt = np.dtype(ref.dtype_of(name))
            host.append(np.ascontiguousarray(np.concatenate([np.asarray(d[name], dtype=dt).reshape(-1)
                                                             for d in per])))
        sh.upload_flat(counts, [h.ctypes.data for h in host])
        Scenario([sh], distributed_drive(sh), ref, P, kw["fields"]).run(steps=2, sigma=0.8)
    finally:
        ref.close()
        sh.close()
        dist.destroy_process_group()


def test_native_fused_step_over_nccl(cuda):
    """The native shard's fused step (dsx_shard_step) through its
    torch.distributed transport on a one-rank NCCL group equals the grid's
    own batched step: every owned array (forces summed back included) and
    every ghost array, step after step, Dynamic cuts."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    kw = CASES["dynamic-4x4x2-R4"]
    P, N = kw["nranks"], 30_000
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    owner = Grid("port", P, kw["dims"], kw["policy"], (0, 0, 0), kw["upper"], (True, True, True),
                 kw["halo_width"], True, kw["dynamic"], [(n, TYPE_INDEX[t], c) for n, t, c in kw["fields"]])
    per = initial(owner, P, kw["upper"], N, 53, kw["fields"])
    owner.close()
    ref = dsx.VirtualGrid(**grid_kw(kw), particles=N, ghost_capacity=2 * N)
    ref.upload(per)
    sh = shd.NativeShardedGrid(**grid_kw(kw), particles=N + 4096, ghost_capacity=N)

    def region(view, a, offset, count, dtype):
        size = np.dtype(dtype).itemsize
        return torch.as_tensor(_Bytes(view.base[a] + size * int(offset), size * count),
                               device="cuda").view(torch.float64 if dtype == np.float64 else torch.int32)

    side = torch.cuda.Stream()
    calls = []
    seen = []

    def forces(view, stream):
        # every ghost slot of the view: a force from the ghost's own
        # position and id (equal ghosts get equal forces in any slot)
        seen.append(stream)
        cap = int(view.ghost_capacity)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            x = region(view, 0, view.ghost_offset, cap, np.float64)
            y = region(view, 1, view.ghost_offset, cap, np.float64)
            gid = region(view, 12, view.ghost_offset, cap, np.int32)
            a = torch.remainder(gid, 1009).double().mul(1e-3)
            region(view, 6, view.ghost_offset, cap, np.float64).copy_(x.mul(0.5).add(a))
            region(view, 7, view.ghost_offset, cap, np.float64).copy_(y.mul(0.25).sub(a))
            region(view, 8, view.ghost_offset, cap, np.float64).copy_(a.mul(a).add(1.0))

    try:
        names = dsx.ARRAYS + [f[0] for f in kw["fields"]]
        counts = np.array([len(d["x"]) for d in per], dtype=np.int64)
        host = []
        for name in names:
            dt = np.dtype(ref.dtype_of(name))
            host.append(np.ascontiguousarray(np.concatenate([np.asarray(d[name], dtype=dt).reshape(-1)
                                                             for d in per])))
        sh.upload_flat(counts, [h.ctypes.data for h in host])
        rng = np.random.default_rng(9)
        for step in range(3):
            # the same displacement on both, keyed by the owned order (equal)
            v = ref.view()
            n = int(v.particles)
            d = torch.from_numpy(rng.normal(0.0, 0.6, size=(3, n))).cuda()
            for k, view in enumerate((v, sh.owned_view())):
                for a in range(3):
                    region(view, a, view.owned_offset, n, np.float64).add_(d[a])
            torch.cuda.synchronize()
            with torch.cuda.stream(side):
                assert ref.step(forces, capture=False) == 0
                assert sh.step_fused(forces) == 0
            torch.cuda.synchronize()
            calls.append(step)
            vr, vs = ref.view(), sh.owned_view()
            assert int(vr.particles) == int(vs.particles) == n
            o_ref, g_ref = ref.all_counts()
            o_sh, g_sh = sh.all_counts()
            assert (o_ref == o_sh).all() and (g_ref == g_sh).all(), step
            G = int(g_ref.sum())
            for a, name in enumerate(names):
                dt = np.dtype(ref.dtype_of(name))
                width = dt.itemsize * ref.components(name)
                for off_r, off_s, count in ((vr.owned_offset, vs.owned_offset, n),
                                            (vr.ghost_offset, vs.ghost_offset, G)):
                    got = torch.as_tensor(_Bytes(vs.base[a] + width * int(off_s), width * count),
                                          device="cuda")
                    want = torch.as_tensor(_Bytes(vr.base[a] + width * int(off_r), width * count),
                                           device="cuda")
                    assert torch.equal(got, want), (step, name)
            assert G > 0
        # both callbacks ran on every step, on the step's stream
        assert calls == [0, 1, 2] and len(seen) == 6 and all(s == side.cuda_stream for s in seen)
    finally:
        ref.close()
        sh.close()
        dist.destroy_process_group()


class _Bytes:
    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = dict(shape=(int(nbytes),), typestr="|u1",
                                             data=(int(ptr), False), version=3, strides=None)
