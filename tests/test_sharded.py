"""Sharded virtual grid: the host side on CPU.

The planning helpers are checked directly; the protocol (migrate, halo build
and refresh, reverse_halo, field exchanges, Dynamic rebalance) runs with
shard engines over the oracle, R shards in lockstep in one process and two
shards as gloo ranks, and every array of every subdomain is compared bit for
bit with one oracle grid holding all subdomains.
"""
import datetime
import itertools
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import ALL_FIELDS
from oracle import Grid
from shard_oracle import OracleEngine
from shard_scenario import Scenario, distributed_drive, initial, lockstep_drive

from dsdecompx_b200 import sharded as shd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIELDS3 = [(n, t, c) for n, t, c in ALL_FIELDS[:3]]
TYPE_INDEX = {"int32": 0, "int64": 1, "uint32": 2, "uint64": 3, "float32": 4, "float64": 5}


def oracle_fields(fields):
    return [(n, TYPE_INDEX[t], c) for n, t, c in fields]


# ------------------------------------------------------------ planning

@pytest.mark.parametrize("dims,R,blocks", [
    ((4, 4, 4), 8, True), ((4, 4, 4), 2, True), ((2, 2, 2), 4, True), ((3, 1, 4), 2, True),
    ((3, 3, 3), 4, False), ((8, 8, 4), 8, True),
    # shard counts with no factorisation that divides the grid: runs of ranks
    ((4, 4, 4), 5, False), ((8, 8, 4), 7, False), ((4, 4, 4), 3, False),
    # prime or composite counts that still divide one or two axes
    ((5, 2, 2), 5, True), ((6, 4, 4), 6, True), ((3, 3, 3), 9, True)])
def test_block_owners(dims, R, blocks):
    owners = shd.block_owners(dims, R)
    P = int(np.prod(dims))
    assert owners.shape == (P,) and set(owners) == set(range(R))
    counts = np.bincount(owners, minlength=R)
    assert counts.max() - counts.min() <= 1
    if not blocks:
        # no exact block split: contiguous runs of ranks
        assert (np.diff(owners) >= 0).all()
    else:
        # blocks: each shard's subdomains form a box of the process grid
        for s in range(R):
            c = np.array([shd.subdomain_coords(t, dims) for t in np.flatnonzero(owners == s)])
            span = c.max(axis=0) - c.min(axis=0) + 1
            assert np.prod(span) == len(c)


def test_native_plan_matches_block_owners():
    """The library's default owners (dsx_shard_plan_owners, host only) are
    block_owners' on every grid of up to 6 per axis and every shard count,
    and it refuses what block_owners refuses."""
    for dims in itertools.product(range(1, 7), repeat=3):
        P = int(np.prod(dims))
        for R in range(1, min(P, 12) + 1):
            assert (shd.plan_owners(dims, R) == shd.block_owners(dims, R)).all(), (dims, R)
    for dims, R in (((2, 2, 2), 9), ((2, 2, 2), 0), ((0, 2, 2), 1)):
        with pytest.raises(Exception):
            shd.plan_owners(dims, R)


def test_block_owners_prefers_the_smallest_cut():
    # 8 x 8 x 4 over 4 shards: 2 x 2 x 1 cuts 2 * 32 faces, 4 x 1 x 1 cuts 3 * 32
    owners = shd.block_owners((8, 8, 4), 4)
    coords = np.array([shd.subdomain_coords(t, (8, 8, 4)) for t in range(256)])
    assert len({tuple(c) for c in coords[owners == 0][:, :2] // 4}) == 1
    assert set(coords[owners == 0][:, 2]) == {0, 1, 2, 3}


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 1, 4), (4, 4, 4)])
def test_halo_tables_point_back(dims):
    from dsdecompx_b200 import plan_topology
    P = int(np.prod(dims))
    topo = [plan_topology(P, t, dims, "manual", (0, 0, 0), (1, 1, 1), (True, False, True))[1]
            for t in range(P)]
    nn, sender_of = shd.halo_tables(topo)
    for t in range(P):
        for m in range(nn[t]):
            e = sender_of[t, m]
            if topo[t][m]["rank"] < 0:
                assert e == -1
                continue
            q, n = divmod(int(e), 26)
            assert q == topo[t][m]["rank"]
            assert topo[q][n]["rank"] == t
            assert tuple(topo[q][n]["direction"]) == tuple(-d for d in topo[t][m]["direction"])


def test_ghost_plans_agree_between_shards():
    """What shard a sends shard b (lists and their order) is what b expects."""
    from dsdecompx_b200 import plan_topology
    dims, R = (4, 2, 3), 3
    P = int(np.prod(dims))
    topo = [plan_topology(P, t, dims)[1] for t in range(P)]
    nn, sender_of = shd.halo_tables(topo)
    owners = shd.block_owners(dims, R)
    rng = np.random.default_rng(5)
    length = np.zeros(P * 26, np.int64)
    for t in range(P):
        for n in range(nn[t]):
            length[t * 26 + n] = rng.integers(0, 9)
    first = np.concatenate([[0], np.cumsum(length)])[:-1]   # any local layout
    plans = [shd.GhostPlan(s, owners, nn, sender_of, length, first) for s in range(R)]
    # identity of every local ghost slot: (list e, position k in the list)
    ident = np.full(int(length.sum()), -1, np.int64)
    for e in range(P * 26):
        ident[first[e]:first[e] + length[e]] = e * 10_000 + np.arange(length[e])

    def expand(rows):
        if not len(rows):
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        src = np.concatenate([np.arange(r[0], r[0] + r[2]) for r in rows])
        dst = np.concatenate([np.arange(r[1], r[1] + r[2]) for r in rows])
        return src, dst

    for s in range(R):
        p = plans[s]
        # what each assembled slot must hold: blocks in (receiver, neighbor) order
        want = []
        for t in np.flatnonzero(owners == s):
            for m in range(nn[t]):
                e = sender_of[t, m]
                if e >= 0:
                    want.extend(e * 10_000 + np.arange(length[e]))
        got = np.full(p.total, -1, np.int64)
        src, dst = expand(p.local)
        got[dst] = ident[src]
        for q, rows in p.recv.items():
            # shard q's buffer for s: its engine slots in q's send rows
            bsrc, boff = expand(plans[q].send[s])
            buf = np.full(plans[q].send_n[s], -1, np.int64)
            buf[boff] = ident[bsrc]
            off, dst = expand(rows)
            got[dst] = buf[off]
            assert p.recv_n[q] == plans[q].send_n[s]
        assert p.total == len(want) and np.array_equal(got, np.array(want, np.int64))
        assert p.g.sum() == p.total


def test_packed_sections_are_aligned():
    b = [8, 4, 12, 1]
    offs = shd.section_offsets(5, b)
    assert offs == [0, 48, 80, 144] and all(o % 16 == 0 for o in offs)
    assert shd.packed_bytes(5, b) == 160


# ------------------------------------------------------------ protocol

def make_ref(kw, fields):
    return Grid("port", kw["nranks"], kw["dims"], kw["policy"], (0, 0, 0), kw["upper"],
                kw.get("periodic", (True, True, True)), kw["halo_width"], True, kw.get("dynamic"),
                oracle_fields(fields))


def make_shards(kw, fields, R, run=None):
    shards = []
    for s in range(R):
        e = OracleEngine(kw["nranks"], kw["dims"], kw["policy"], (0, 0, 0), kw["upper"],
                         kw.get("periodic", (True, True, True)), kw["halo_width"], True,
                         kw.get("dynamic"), oracle_fields(fields))
        shards.append(shd.ShardedGrid(e, s, R, run=run))
    return shards


CASES = {
    "2x2x2-R2": dict(nranks=8, dims=(2, 2, 2), policy="manual", upper=(10.0, 10.0, 10.0),
                     halo_width=1.0, N=3000),
    "3x1x4-R3-open": dict(nranks=12, dims=(3, 1, 4), policy="manual", upper=(9.0, 5.0, 12.0),
                          periodic=(True, False, False), halo_width=0.8, N=3000),
    "dynamic-R4": dict(nranks=8, dims=(2, 2, 2), policy="dynamic", upper=(12.0, 12.0, 12.0),
                       halo_width=0.9, dynamic=(1.0, 1.05, 0.5, 0.1), N=3000),
    "3x3x3-R4-runs": dict(nranks=27, dims=(3, 3, 3), policy="manual", upper=(9.0, 9.0, 9.0),
                          halo_width=0.7, N=4000),
}


@pytest.mark.parametrize("case,R", [("2x2x2-R2", 2), ("3x1x4-R3-open", 3), ("dynamic-R4", 4),
                                    ("3x3x3-R4-runs", 4)])
def test_lockstep_shards_match_one_grid(case, R):
    kw = CASES[case]
    fields = FIELDS3
    ref = make_ref(kw, fields)
    shards = make_shards(kw, fields, R)
    per = initial(ref, kw["nranks"], kw["upper"], kw["N"], 17, fields)
    for t in range(kw["nranks"]):
        ref.set_owned(t, per[t])
    for sh in shards:
        sh.upload({t: per[t] for t in sh.mine})
    Scenario(shards, lockstep_drive(shards), ref, kw["nranks"], fields).run(steps=3, sigma=0.8)
    if kw["policy"] == "dynamic":
        assert not np.allclose(ref.cuts()[0], np.linspace(0, 12, 3))
    sent = {k: sum(sh.sent_bytes[k] for sh in shards) for k in shards[0].sent_bytes}
    assert sent["migrants"] > 0 and sent["ghost lists"] > 0 and sent["returned values"] > 0, sent


def test_lockstep_rebalance_with_work():
    kw = CASES["dynamic-R4"]
    fields = []
    ref = make_ref(kw, fields)
    shards = make_shards(kw, fields, 2)
    per = initial(ref, 8, kw["upper"], kw["N"], 3, fields)
    for t in range(8):
        ref.set_owned(t, per[t])
    for sh in shards:
        sh.upload({t: per[t] for t in sh.mine})
    work = np.linspace(1.0, 4.0, 8) * 100.0
    flags, imb = ref.rebalance(work, force=True)
    outs = shd.run_lockstep([sh.rebalance_steps(work, True) for sh in shards])
    for sh, (out, imbalance) in zip(shards, outs):
        assert imbalance == imb[0]
        for t, row in out.items():
            assert row == tuple(int(v) for v in flags[t])
    for a, b in zip(ref.cuts(), shards[0].E.g.cuts()):
        assert np.array_equal(a, b)
    Scenario(shards, lockstep_drive(shards), ref, 8, fields).compare("after rebalance")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def gloo_rank(rank, world, port, case):
    import torch
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        kw = CASES[case]
        fields = FIELDS3
        ref = make_ref(kw, fields)
        e = OracleEngine(kw["nranks"], kw["dims"], kw["policy"], (0, 0, 0), kw["upper"],
                         kw.get("periodic", (True, True, True)), kw["halo_width"], True,
                         kw.get("dynamic"), oracle_fields(fields))
        sh = shd.ShardedGrid(e, rank, world, run=lambda g: shd.run_distributed(g, device="cpu"))
        per = initial(ref, kw["nranks"], kw["upper"], kw["N"], 23, fields)
        for t in range(kw["nranks"]):
            ref.set_owned(t, per[t])
        sh.upload({t: per[t] for t in sh.mine})
        Scenario([sh], distributed_drive(sh), ref, kw["nranks"], fields).run(steps=2, sigma=0.8)
    finally:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


@pytest.mark.parametrize("case", ["2x2x2-R2", "dynamic-R4"])
def test_two_gloo_ranks_match_one_grid(case):
    mp.start_processes(gloo_rank, args=(2, free_port(), case), nprocs=2, start_method="spawn")


def test_row_and_segment_merging():
    assert list(shd.group_exclusive(np.array([0, 0, 1, 1, 1]), np.array([1, 2, 3, 4, 5]))) == [0, 1, 0, 3, 7]
    rows = np.array([(0, 10, 5), (5, 15, 3), (9, 18, 1), (10, 19, 2)])
    assert shd.merge_rows(rows).tolist() == [[0, 10, 8], [9, 18, 3]]
    rng = np.random.default_rng(3)
    from dsdecompx_b200 import SEGMENT_DTYPE
    for _ in range(20):
        k = 40
        seg = np.zeros(k, dtype=SEGMENT_DTYPE)
        seg["source"] = rng.integers(-1, 2, k)
        seg["dst_rank"] = rng.integers(0, 3, k)
        seg["count"] = rng.integers(1, 4, k)
        # contiguous destinations per subdomain, sources often continuing
        for r in range(3):
            sel = np.flatnonzero(seg["dst_rank"] == r)
            seg["dst_index"][sel] = np.cumsum(seg["count"][sel]) - seg["count"][sel]
            seg["src_index"][sel] = seg["dst_index"][sel] + 100 * r + rng.integers(0, 2, len(sel))
        merged = shd.merge_segments(seg)
        assert len(merged) <= len(seg)

        def expand(s):
            return sorted((int(x["dst_rank"]), int(x["dst_index"]) + i, int(x["source"]),
                           int(x["src_index"]) + i) for x in s for i in range(int(x["count"])))
        assert expand(seg) == expand(merged)


# ------------------------------------------------------- failures

def drive_until_failure(gens):
    """Serves the shards' requests (all-reduces only) until they stop;
    returns what each raised (None: it finished)."""
    replies = [None] * len(gens)
    outcome = [None] * len(gens)
    live = list(range(len(gens)))
    while live:
        reqs = {}
        for i in list(live):
            try:
                reqs[i] = gens[i].send(replies[i])
            except StopIteration:
                live.remove(i)
            except Exception as exc:   # noqa: BLE001 - recorded for the assertions
                outcome[i] = exc
                live.remove(i)
        if not reqs:
            break
        assert len(reqs) == len(gens), "a shard stopped while another waits in a collective"
        assert all(isinstance(r, shd.AllReduce) for r in reqs.values())
        total = sum(r.values for r in reqs.values())
        replies = [total.copy() for _ in gens]
    return outcome


@pytest.mark.parametrize("case", ["2x2x2-R2", "dynamic-R4"])
def test_shards_agree_on_a_storage_shortfall(case):
    """One shard's storage is too small for its subdomains after migration:
    every shard raises the same error at the same collective (the reference's
    error agreement), before any particle moves between shards."""
    kw = CASES[case]
    ref = make_ref(kw, [])
    shards = make_shards(kw, [], 2)
    per = initial(ref, kw["nranks"], kw["upper"], kw["N"], 19, [])
    for sh in shards:
        sh.upload({t: per[t] for t in sh.mine})
    shards[1].E.capacity = 10
    outcome = drive_until_failure([sh.migrate_steps() for sh in shards])
    assert all(isinstance(e, MemoryError) for e in outcome), outcome
    assert all("shard(s) [1]" in str(e) for e in outcome)


def gloo_failure_rank(rank, world, port, out_dir, mode):
    import torch
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=20))
    kw = CASES["2x2x2-R2"]
    ref = make_ref(kw, [])
    e = OracleEngine(kw["nranks"], kw["dims"], kw["policy"], (0, 0, 0), kw["upper"],
                     (True, True, True), kw["halo_width"], True, None, [])
    sh = shd.ShardedGrid(e, rank, world, run=lambda g: shd.run_distributed(g, device="cpu"))
    per = initial(ref, kw["nranks"], kw["upper"], kw["N"], 29, [])
    sh.upload({t: per[t] for t in sh.mine})
    if mode == "storage" and rank == 0:
        e.capacity = 10
    result = "finished"
    try:
        sh.migrate()
        sh.exchange_halo(rebuild=True)
        if mode == "peer_leaves":
            if rank == 1:
                os._exit(0)   # leaves between steps, none of its work in flight
            sh.migrate()      # the next collective must fail, not wait for ever
    except MemoryError as exc:
        result = "MemoryError: " + str(exc)
    except RuntimeError as exc:
        result = "RuntimeError: " + str(exc)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(result)
    if mode == "storage":
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_agree_on_a_storage_shortfall(tmp_path):
    mp.start_processes(gloo_failure_rank, args=(2, free_port(), str(tmp_path), "storage"), nprocs=2,
                       start_method="spawn")
    for r in range(2):
        got = open(tmp_path / f"rank{r}.txt").read()
        assert got.startswith("MemoryError") and "shard(s) [0]" in got, (r, got)


def test_a_rank_that_leaves_is_detected_by_the_next_collective(tmp_path):
    mp.start_processes(gloo_failure_rank, args=(2, free_port(), str(tmp_path), "peer_leaves"),
                       nprocs=2, start_method="spawn")
    got = open(tmp_path / "rank0.txt").read()
    assert got.startswith("RuntimeError"), got


@pytest.mark.parametrize("case,R,start", [
    ("2x2x2-R2", 2, "one-subdomain"),
    ("wide-halo-R3", 3, "placed"),
])
def test_lockstep_edge_cases(case, R, start):
    """Every particle starting in subdomain 0 (the other shards start
    empty, the first migrate sends almost everything across shards); a halo
    wider than half a cell (every particle has many images)."""
    kw = dict(CASES.get(case, {}))
    if case == "wide-halo-R3":
        kw = dict(nranks=27, dims=(3, 3, 3), policy="manual", upper=(6.0, 6.0, 6.0),
                  halo_width=1.1, N=1500)
    fields = FIELDS3[:2]
    ref = make_ref(kw, fields)
    shards = make_shards(kw, fields, R)
    per = initial(ref, kw["nranks"], kw["upper"], kw["N"], 71, fields)
    if start == "one-subdomain":
        everything = {k: np.concatenate([p[k] for p in per]) for k in per[0]}
        per = [everything] + [{k: v[:0] for k, v in everything.items()} for _ in per[1:]]
    for t in range(kw["nranks"]):
        ref.set_owned(t, per[t])
    for sh in shards:
        sh.upload({t: per[t] for t in sh.mine})
    Scenario(shards, lockstep_drive(shards), ref, kw["nranks"], fields).run(steps=2, sigma=0.5)


def gloo_transport_rank(rank, world, port, out_dir):
    import ctypes as C

    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=20))
    tr = shd.TorchTransport(device="cpu")
    lines = []
    # the callbacks as the library calls them: through the struct's pointers
    v = (C.c_longlong * 4)(1, -2, 3 + rank, 1 << 40)
    lines.append(str(tr.struct.allreduce_i64(None, v, 4)) + " " + " ".join(str(x) for x in v))
    d = (C.c_double * 3)(0.5, -1.25 * (rank + 1), 1e300)
    lines.append(str(tr.struct.allreduce_f64(None, d, 3)) + " " + " ".join(repr(x) for x in d))
    torch.distributed.destroy_process_group()
    # without a process group the call fails: a status, not an exception
    # through the C frames, and the cause kept for the caller
    status = tr.struct.allreduce_i64(None, v, 4)
    lines.append(f"{status} {type(tr.error).__name__ if tr.error is not None else None}")
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write("\n".join(lines))


def test_torch_transport_sums_over_gloo_ranks(tmp_path):
    """The native shard's torch.distributed transport: its C callbacks sum
    int64 and float64 vectors over every rank in place, and report a failed
    collective as DSX_E_RUNTIME with the exception kept for the caller."""
    mp.start_processes(gloo_transport_rank, args=(2, free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn")
    for rank in range(2):
        i64, f64, fail = open(os.path.join(tmp_path, f"rank{rank}.txt")).read().split("\n")
        assert i64.split() == ["0", "2", "-4", "7", str(2 << 40)]
        assert f64.split() == ["0", "1.0", "-3.75", "2e+300"]
        assert fail.split()[0] == "-3" and fail.split()[1] != "None"


# ---------------------------------------------------------------------------
# The fused sharded step's host plan (dsx_shard_plan_step) over gloo ranks

PLAN_P, PLAN_DIMS, PLAN_UPPER = 32, (4, 4, 2), (16.0, 16.0, 8.0)


def plan_contribution(rank, world, seed):
    """This rank's part of the fused step's all-reduce, in its order: the
    export of its own subdomains, the immigrant counters and emigrant pairs
    of its own sources, its storage."""
    import dsdecompx_b200 as dsx
    P, E = PLAN_P, 26
    owners = shd.plan_owners(PLAN_DIMS, world)
    rng = np.random.default_rng(seed + rank)
    stays, bret, iret = np.zeros(P, np.int64), np.zeros(P, np.int64), np.zeros(P, np.int64)
    lret = np.zeros((P, E), np.int64)
    imm_total, imm_bnd, imm_img = np.zeros(P, np.int64), np.zeros(P, np.int64), np.zeros(P, np.int64)
    imm_list = np.zeros((P, E), np.int64)
    pairs = np.zeros((P, P), np.int64)
    for q in range(P):
        if owners[q] != rank:
            continue
        _, nbrs = dsx.plan_topology(P, q, PLAN_DIMS, "manual", (0, 0, 0), PLAN_UPPER)
        stays[q] = rng.integers(500, 2000)
        bret[q] = rng.integers(0, stays[q] // 2)
        iret[q] = bret[q] + rng.integers(0, bret[q] + 1)
        for n, nb in enumerate(nbrs):
            if nb["rank"] >= 0:
                lret[q, n] = rng.integers(0, stays[q] // 8)
            if nb["rank"] >= 0 and nb["rank"] != q:
                t = nb["rank"]
                c = int(rng.integers(0, 40))
                pairs[t, q] += c
                imm_total[t] += c
                b = int(rng.integers(0, c + 1))
                imm_bnd[t] += b
                imm_img[t] += b + int(rng.integers(0, b + 1))
    # the receivers' lists gain the immigrants' images: spread each
    # destination's images over its active lists
    for t in range(P):
        if imm_img[t]:
            _, nbrs = dsx.plan_topology(P, t, PLAN_DIMS, "manual", (0, 0, 0), PLAN_UPPER)
            active = [n for n, nb in enumerate(nbrs) if nb["rank"] >= 0]
            for k in range(int(imm_img[t])):
                imm_list[t, active[k % len(active)]] += 1
    storage = np.zeros(world, np.int64)
    storage[rank] = 1 << 30
    return owners, np.concatenate([stays, bret, iret, lret.ravel(), imm_total, imm_list.ravel(),
                                   imm_bnd, imm_img, pairs.ravel(), storage])


def plan_step(owners, shard, world, sums):
    import ctypes as C

    import dsdecompx_b200 as dsx
    desc = dsx._grid_desc(PLAN_P, PLAN_DIMS, "manual", (0, 0, 0), PLAN_UPPER, (True,) * 3, 1.0,
                          True, None)
    fn = dsx.lib().dsx_shard_plan_step
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_longlong, C.c_void_p]
    own = np.ascontiguousarray(owners, dtype=np.int32)
    s = np.ascontiguousarray(sums, dtype=np.int64)
    out = np.zeros(6 + 4 * world, dtype=np.int64)
    dsx._check(fn(C.byref(desc), own.ctypes.data, shard, world, s.ctypes.data, len(s),
                  out.ctypes.data))
    return out


def gloo_plan_rank(rank, world, port, out_dir):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=20))
    owners, mine = plan_contribution(rank, world, 71)
    total = torch.from_numpy(mine.copy())
    torch.distributed.all_reduce(total)
    out = plan_step(owners, rank, world, total.numpy())
    np.save(os.path.join(out_dir, f"sums{rank}.npy"), total.numpy())
    np.save(os.path.join(out_dir, f"plan{rank}.npy"), out)
    torch.distributed.destroy_process_group()


def test_fused_step_plans_agree_over_gloo_ranks(tmp_path):
    """Two gloo ranks sum their counts as the fused sharded step does and
    each plans its layout (dsx_shard_plan_step, no GPU): every message one
    rank plans to send is the size the other plans to receive, the owned and
    ghost totals add up to the summed counts, and one shard alone plans the
    same totals with nothing to send."""
    world = 2
    mp.start_processes(gloo_plan_rank, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn")
    P, E = PLAN_P, 26
    sums = [np.load(os.path.join(tmp_path, f"sums{r}.npy")) for r in range(world)]
    assert np.array_equal(sums[0], sums[1])
    s = sums[0]
    stays, bret, iret = s[:P], s[P:2 * P], s[2 * P:3 * P]
    lret = s[3 * P:3 * P + P * E]
    imm_total = s[29 * P:30 * P]
    imm_list = s[30 * P:30 * P + P * E]
    imm_bnd, imm_img = s[56 * P:57 * P], s[57 * P:58 * P]
    plans = [np.load(os.path.join(tmp_path, f"plan{r}.npy")) for r in range(world)]
    owners = shd.plan_owners(PLAN_DIMS, world)
    per_peer = [p[6:].reshape(world, 4) for p in plans]
    for a in range(world):
        for b in range(world):
            if a != b:
                assert per_peer[a][b, 0] == per_peer[b][a, 1]   # emigrants a -> b
                assert per_peer[a][b, 2] == per_peer[b][a, 3]   # ghost lists a -> b
        mine = owners == a
        assert plans[a][0] == (stays + imm_total)[mine].sum()
        assert plans[a][1] == per_peer[a][:, 0].sum()
        assert plans[a][2] == plans[a][3] + per_peer[a][:, 2].sum()
        assert plans[a][4] == (bret + imm_bnd)[mine].sum()
        assert plans[a][5] == (iret + imm_img)[mine].sum()
    every_list = int((lret + imm_list).sum())
    assert sum(p[3] for p in plans) == every_list
    alone = plan_step(np.zeros(P, dtype=np.int64), 0, 1,
                      np.concatenate([s[:58 * P + P * P], [1 << 31]]))
    assert alone[0] == (stays + imm_total).sum() and alone[1] == 0
    assert alone[2] == alone[3] == every_list
