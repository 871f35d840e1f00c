"""The allocation-free migrate (dsx_migrate_noalloc) against the grid's
migrate (dsx_grid_migrate), through the C ABI.

dsx_migrate_noalloc exists for callers that cannot allocate device memory --
a solver whose framework owns every GPU byte through its own pool, or a
latency-critical loop that cannot afford an allocation's implicit device
synchronization.  Its scratch lives in one fixed device array inside the
library, so the checks here are: the same result as the existing entry point
(bit for bit, as every parity test in this suite), on two calls in a row (the
second call sees the scratch the first one left behind), and no change in the
device's free memory across the second call, with uniform cuts and with
explicit non-uniform cuts (the latter against a grid given the same cuts).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P, DIMS, L, N = 8, (2, 2, 2), 10.0, 60000


def noalloc_fn():
    import dsdecompx_b200 as dsx
    fn = dsx.lib().dsx_migrate_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(dsx._GridDesc), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                   C.POINTER(C.c_void_p), C.POINTER(C.c_longlong), C.POINTER(C.c_void_p),
                   C.POINTER(C.c_longlong), C.c_void_p, C.c_char_p, C.c_int]
    return fn


def make_desc(nranks=P, dims=DIMS):
    import dsdecompx_b200 as dsx
    return dsx._grid_desc(nranks, dims, "manual", (0, 0, 0), (L, L, L), (True, True, True),
                          1.0, True, None)


# non-uniform cuts (3 per axis: lower, one interior plane, upper)
CUTS = np.array([0.0, 3.5, 10.0, 0.0, 6.25, 10.0, 0.0, 4.0, 10.0])


@pytest.mark.parametrize("cuts", [None, CUTS], ids=["uniform", "explicit_cuts"])
def test_noalloc_migrate_matches_grid_migrate(cuda, cuts):
    import torch

    import dsdecompx_b200 as dsx
    from oracle import Grid

    rng = np.random.default_rng(77)
    pos = rng.uniform(0, L, size=(N, 3))
    shape = Grid("port", P, DIMS, "manual", (0, 0, 0), (L, L, L))
    if cuts is not None:
        shape.set_cuts(np.split(cuts, 3))
    owner = shape.owner_rank(pos)
    order = np.argsort(owner, kind="stable")
    counts = np.bincount(owner, minlength=P).astype(np.int64)
    host = {"x": pos[order, 0], "y": pos[order, 1], "z": pos[order, 2]}
    for name in ("vx", "vy", "vz", "fx", "fy", "fz", "charge"):
        host[name] = rng.normal(size=N)
    host["mass"] = np.ones(N)
    host["type"] = rng.integers(0, 8, N).astype(np.int32)
    host["global_id"] = order.astype(np.int32)

    grid = dsx.VirtualGrid(P, DIMS, "manual", (0, 0, 0), (L, L, L), halo_width=1.0, particles=N)
    if cuts is not None:
        grid.set_cuts(np.split(cuts, 3))
    cut_arg = None if cuts is None else np.ascontiguousarray(cuts).ctypes.data_as(
        C.POINTER(C.c_double))
    starts = np.concatenate([[0], np.cumsum(counts)])
    grid.upload([{k: v[starts[r]:starts[r + 1]] for k, v in host.items()} for r in range(P)])

    dev_in = [torch.from_numpy(np.ascontiguousarray(host[name])).cuda() for name in dsx.ARRAYS]
    dev_out = [torch.empty_like(t) for t in dev_in]
    fn = noalloc_fn()
    desc = make_desc()
    stream = torch.cuda.current_stream().cuda_stream
    counts_in = counts.copy()
    err = C.create_string_buffer(256)
    for call in range(2):
        # the same displacement for both paths, in rank order
        delta = rng.normal(0.0, 0.8, size=(N, 3))
        for a, name in enumerate("xyz"):
            dev_in[a] += torch.from_numpy(delta[:, a]).cuda()
        o = np.concatenate([[0], np.cumsum(counts_in)])
        for r in range(P):
            for a, name in enumerate("xyz"):
                grid.write(r, name, 0, dev_in[a][o[r]:o[r + 1]].cpu().numpy())
        expect = grid.migrate()
        torch.cuda.synchronize()

        counts_out = np.zeros(P, dtype=np.int64)
        results = np.zeros((P, 6), dtype=np.int64)
        ins = (C.c_void_p * 13)(*[t.data_ptr() for t in dev_in])
        outs = (C.c_void_p * 13)(*[t.data_ptr() for t in dev_out])
        # the free-memory window covers the entry point alone
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status = fn(C.byref(desc), cut_arg, counts_in.ctypes.data_as(C.POINTER(C.c_longlong)),
                    ins, counts_out.ctypes.data_as(C.POINTER(C.c_longlong)), outs,
                    results.ctypes.data_as(C.POINTER(C.c_longlong)), stream, err, 256)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert status == 0, err.value
        if call == 1:
            # the first call may load the library's device code (and with it
            # the scratch array); the second must leave free memory unchanged
            assert free_after == free_before, "the call allocated device memory"

        assert (results == expect).all(), (results, expect)
        assert (counts_out == expect[:, 5]).all()
        want = [np.zeros(N, dtype=np.float64) for _ in range(11)] + \
               [np.zeros(N, dtype=np.int32) for _ in range(2)]
        grid.download_flat([w.ctypes.data for w in want])
        for a, name in enumerate(dsx.ARRAYS):
            got = dev_out[a].cpu().numpy()
            assert np.array_equal(got.view(np.uint8), want[a].view(np.uint8)), (call, name)
        dev_in, dev_out = dev_out, dev_in
        counts_in = counts_out
    grid.close()


def test_noalloc_rejects_sizes_beyond_its_limit(cuda):
    fn = noalloc_fn()
    desc = make_desc()
    counts = np.full(P, 40000, dtype=np.int64)          # 320000 > 262144
    out = np.zeros(P, dtype=np.int64)
    arrays = (C.c_void_p * 13)()
    err = C.create_string_buffer(256)
    status = fn(C.byref(desc), None, counts.ctypes.data_as(C.POINTER(C.c_longlong)), arrays,
                out.ctypes.data_as(C.POINTER(C.c_longlong)), arrays, None, None, err, 256)
    assert status == -4
    assert b"at most 262144 particles" in err.value
    many = make_desc(nranks=128, dims=(8, 4, 4))
    status = fn(C.byref(many), None, np.zeros(128, dtype=np.int64).ctypes.data_as(
        C.POINTER(C.c_longlong)), arrays, np.zeros(128, dtype=np.int64).ctypes.data_as(
        C.POINTER(C.c_longlong)), arrays, None, None, err, 256)
    assert status == -4 and b"64 subdomains" in err.value
