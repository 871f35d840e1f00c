"""The CUDA path against the reference's own Host path (oracle/_ref: the
dsDecompX sources built unmodified, one thread per subdomain) at the full
sizes of the benchmark configurations, on the same seeded inputs:

* clustered_64 (16M particles, 4x4x4 Dynamic, 80% in 32 Gaussian blobs, an
  int64 id field) and large_256 (27.2M particles, 8x8x4, five fields) through
  the graph-captured batched step (dsx_grid_step);
* virtual_2x2x2 (8M particles, 2x2x2, a float64 and a float32 x 3 field) with
  forward_exchange and reverse_exchange(sum) of both fields inside the step's
  callback, as the benchmark runs it;
* drop_in_1rank (1M particles, one rank) through dsx_rank_migrate.

Each step: the same N(0, drift) displacement (keyed by global id) goes to
both sides; the GPU runs its whole step, with the benchmark's ghost-force
kernel in the callback; the reference runs migrate, exchange_halo(rebuild),
receives the GPU's ghost forces in its own ghost slots, then
reverse_exchange / reverse_halo.  Then every owned and every ghost array of
every subdomain, the counts and the Dynamic cut planes are compared bit for
bit (src/migration.cpp:395-591 order, src/halo.cpp:164-238,609-649 ghost
plan and receive order, src/halo.cpp:1476-1531 reverse order,
src/runtime.cpp:345-447 cuts).
"""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

FIELD_TYPES = ["int32", "int64", "uint32", "uint64", "float32", "float64"]


class DeviceBytes:
    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = dict(shape=(int(nbytes),), typestr="|u1",
                                             data=(int(ptr), False), version=3, strides=None)


def reference_grid(w, field_capacity=0):
    """The reference's grid of the workload; without a field capacity it
    carries no fields (a probe for the process grid)."""
    dims = w.dims if w.policy == "manual" else (0, 0, 0)
    fields = [(n, FIELD_TYPES.index(t), c) for n, t, c in w.fields] if field_capacity else []
    return oracle.Grid("ref", w.nranks, dims, w.policy, w.lower, w.upper, (True,) * 3, w.halo,
                       fields=fields, field_capacity=field_capacity)


def array_info(grid, a):
    """(dtype, components) of array id a: 13 core arrays, then the fields (a
    field may share its name with a core array, e.g. "charge")."""
    import dsdecompx_b200 as dsx
    if a < 13:
        return np.dtype(dsx.CORE_DTYPES[a]), 1
    _, t, c = grid.fields[a - 13]
    return np.dtype(dsx.FIELD_DTYPES[t]), c


def gpu_state(grid, names):
    """Host copies of every array's owned and ghost regions (rank order, by
    array id), the per-rank counts and their prefixes."""
    import torch
    v = grid.view()
    o, g = grid.all_counts()
    N, G = int(o.sum()), int(g.sum())
    state = {}
    for a, name in enumerate(names):
        dtype, comps = array_info(grid, a)
        size = dtype.itemsize * comps

        def region(offset, count):
            if count == 0:
                return np.zeros(0, dtype=dtype)
            t = torch.as_tensor(DeviceBytes(v.base[a] + size * int(offset), size * count),
                                device="cuda")
            return t.cpu().numpy().view(dtype)
        state[a] = (region(v.owned_offset, N), region(v.ghost_offset, G))
    ob = np.concatenate([[0], np.cumsum(o)])
    gb = np.concatenate([[0], np.cumsum(g)])
    return state, o, g, ob, gb


def rank_arrays(grid, state, ob, gb, r, a):
    comps = array_info(grid, a)[1]
    owned, ghosts = state[a]
    got = np.concatenate([owned[ob[r] * comps:ob[r + 1] * comps],
                          ghosts[gb[r] * comps:gb[r + 1] * comps]])
    return got.reshape(-1, comps) if comps > 1 else got


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def drift_both(ref, grid, P, rng, sigma, N):
    """x += N(0, sigma) keyed by global id, the same values on both sides
    (the two owned layouts are equal: the previous step compared them)."""
    d = rng.normal(0.0, sigma, size=(N, 3))
    for r in range(P):
        o, _ = ref.counts(r)
        if not o:
            continue
        gid = ref.read(r, "global_id", 0, o)
        for a, name in enumerate("xyz"):
            v = ref.read(r, name, 0, o) + d[gid, a]
            ref.write(r, name, 0, v)
            grid.write(r, name, 0, v)


def run_config(cuda, workload, steps, seed=2024):
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    w = W.WORKLOADS[workload]
    assert oracle.available("ref"), "the reference build oracle/_ref is required"
    with reference_grid(w) as probe:
        dims = probe.topology(0)[0]
    data = W.generate(w, seed=seed)
    owner = W.initial_owner(w, dims, data["x"], data["y"], data["z"])
    counts, grouped = W.group_by_owner(data, owner, w.nranks)
    del data, owner
    N = int(counts.sum())
    P = w.nranks
    names = dsx.ARRAYS + [f[0] for f in w.fields]
    cap = int(2 * counts.max() + 65536)
    ref = reference_grid(w, field_capacity=cap)
    grid = dsx.VirtualGrid(P, w.dims, w.policy, w.lower, w.upper, halo_width=w.halo,
                           fields=w.fields, particles=N, ghost_capacity=int(0.9 * N))
    try:
        assert tuple(grid.topology(0)[0]) == tuple(dims)
        host = [np.ascontiguousarray(grouped[n]) if n in grouped else None for n in names]
        grid.upload_flat(counts, [h.ctypes.data if h is not None else None for h in host])
        starts = np.concatenate([[0], np.cumsum(counts)])
        for r in range(P):
            ref.set_owned(r, {k: v[starts[r]:starts[r + 1]] for k, v in grouped.items()})
        del grouped, host
        wl = W.harness()
        field_names = [f[0] for f in w.fields] if w.field_exchange else []
        stream = torch.cuda.Stream()

        def callback(view, s):
            wl.dsxw_ghost_forces(C.byref(view), seed, 0, s)
            if field_names:
                grid.forward_exchange(field_names, stream=s)
                grid.reverse_exchange([(n, "sum") for n in field_names], stream=s)

        rng = np.random.default_rng(seed + 1)
        for step in range(steps):
            drift_both(ref, grid, P, rng, w.drift, N)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                status = grid.step(callback, capture=step > 0)
            stream.synchronize()
            assert status == 0, (workload, step, status)

            ref.migrate()
            ref.exchange_halo(rebuild=True)
            state, o, g, ob, gb = gpu_state(grid, names)
            for r in range(P):
                assert ref.counts(r) == (o[r], g[r]), (workload, step, r, ref.counts(r), o[r], g[r])
            # the reference receives the GPU's ghost forces in its own slots
            for r in range(P):
                if g[r]:
                    for a, name in ((6, "fx"), (7, "fy"), (8, "fz")):
                        ref.write(r, name, int(o[r]), state[a][1][gb[r]:gb[r + 1]])
            if field_names:
                ref.reverse_exchange([(n, "sum") for n in field_names])
            ref.reverse_halo()
            for r in range(P):
                for a, name in enumerate(names):
                    want = ref.read(r, name) if a < 13 else ref.read_field(r, name)
                    got = rank_arrays(grid, state, ob, gb, r, a)
                    assert got.shape == want.shape, (workload, step, r, name)
                    if not np.array_equal(bits(got), bits(want)):
                        bad = np.flatnonzero((got != want).reshape(len(got), -1).any(axis=1))
                        raise AssertionError(f"{workload} step {step} rank {r} {name}: "
                                             f"{len(bad)} rows differ, first at {bad[:5]} "
                                             f"(owned {o[r]})")
            for a, (cg, cr) in enumerate(zip(grid.cuts(), ref.cuts())):
                assert np.array_equal(bits(cg), bits(cr)), (workload, step, a, cg, cr)
        return int(g.sum())
    finally:
        grid.close()
        ref.close()


def test_clustered_64_matches_reference(cuda):
    ghosts = run_config(cuda, "clustered_64", steps=3)
    assert ghosts > 1_000_000


def test_virtual_2x2x2_with_field_exchanges_matches_reference(cuda):
    ghosts = run_config(cuda, "virtual_2x2x2", steps=2)
    assert ghosts > 1_000_000


def test_large_256_matches_reference(cuda):
    ghosts = run_config(cuda, "large_256", steps=2)
    assert ghosts > 5_000_000


def test_drop_in_1rank_matches_reference(cuda):
    """One rank (config C1): the reference makes no ghosts and only wraps
    (src/halo.cpp:325-350, src/migration.cpp:102-128); dsx_rank_migrate must
    leave the same positions bit for bit, step after step."""
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    w = W.WORKLOADS["drop_in_1rank"]
    data = W.generate(w, seed=2024)
    N = w.particles
    ref = oracle.Grid("ref", 1, (1, 1, 1), "manual", w.lower, w.upper, (True,) * 3, w.halo)
    try:
        ref.set_owned(0, data)
        dev = [torch.from_numpy(data[k].copy()).cuda() for k in "xyz"]
        stream = torch.cuda.Stream()
        rng = np.random.default_rng(2025)
        for step in range(3):
            d = rng.normal(0.0, 1.5, size=(N, 3))     # wider than the config's 0.1: more wraps
            for a, name in enumerate("xyz"):
                v = ref.read(0, name) + d[:, a]
                ref.write(0, name, 0, v)
                dev[a].copy_(torch.from_numpy(v))
            torch.cuda.synchronize()
            res = dsx.rank_migrate(dev[0], dev[1], dev[2], N, w.lower, w.upper, stream=stream)
            stream.synchronize()
            out = ref.migrate()
            assert res["new_owned_count"] == N == out[0, 5]
            halo = ref.exchange_halo(rebuild=True)
            assert halo[0, 0] == 0                    # no ghosts at one rank
            ref.reverse_halo()
            for a, name in enumerate("xyz"):
                got = dev[a].cpu().numpy()
                assert np.array_equal(bits(got), bits(ref.read(0, name))), (step, name)
            assert np.array_equal(ref.read(0, "global_id"), np.arange(N, dtype=np.int32))
    finally:
        ref.close()
