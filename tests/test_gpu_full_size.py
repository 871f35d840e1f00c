"""The batched step at the benchmark workloads' full sizes, through
properties that hold at any size (these complement the element-by-element
comparison with the reference's Host path at the same sizes in
test_gpu_config_parity.py, over more drifted steps and after a rebuild):

* ids are conserved: after every step the owned global ids are a
  permutation of 0..N-1;
* every owned particle lies in its own subdomain (out_of_domain is clear
  after the step's migrate);
* the reverse sum adds exactly what the ghosts hold: every ghost carries the
  force (1, 2, 3), so the owned force sums grow by (G, 2G, 3G) exactly
  (small integers add exactly in FP64 in any order);
* the step's ghosts are the per-call path's: a rebuild of the plan on the
  same owned particles gives bit-identical ghost positions and ids.

Workloads: clustered_64 (16M particles, Dynamic 4x4x4, 80% in 32 Gaussian
blobs) and large_256 (27.2M particles, 8x8x4, five fields), drifted between
steps by the benchmark harness.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class DeviceArray:
    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = dict(shape=(n,), typestr=typestr, data=(ptr, False),
                                             version=3, strides=None)


@pytest.mark.parametrize("workload", ["clustered_64", "large_256"])
def test_full_size_step_properties(cuda, workload):
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    w = W.WORKLOADS[workload]
    dims, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    data = W.generate(w, seed=11)
    data["fx"] = np.zeros(w.particles)
    data["fy"] = np.zeros(w.particles)
    data["fz"] = np.zeros(w.particles)
    owner = W.initial_owner(w, dims, data["x"], data["y"], data["z"])
    counts, grouped = W.group_by_owner(data, owner, w.nranks)
    del data, owner
    N = int(counts.sum())
    names = dsx.ARRAYS + [f[0] for f in w.fields]
    host = [np.ascontiguousarray(grouped[n]) if n in grouped else None for n in names]
    del grouped
    grid = dsx.VirtualGrid(w.nranks, w.dims, w.policy, w.lower, w.upper, halo_width=w.halo,
                           fields=w.fields, particles=N, ghost_capacity=int(0.9 * N))
    wl = W.harness()
    stream = torch.cuda.Stream()
    try:
        grid.upload_flat(counts, [h.ctypes.data if h is not None else None for h in host])
        del host

        def owned(a, typestr="<f8", size=8):
            v = grid.view()
            return torch.as_tensor(DeviceArray(v.base[a] + size * int(v.owned_offset), N, typestr),
                                   device="cuda")

        def fill(view, s):
            cap = int(view.ghost_capacity)
            with torch.cuda.stream(torch.cuda.ExternalStream(s)):
                for k, value in ((6, 1.0), (7, 2.0), (8, 3.0)):
                    torch.as_tensor(DeviceArray(view.base[k] + 8 * int(view.ghost_offset), cap, "<f8"),
                                    device="cuda").fill_(value)

        ids = torch.arange(N, dtype=torch.int32, device="cuda")
        for step in range(4):
            with torch.cuda.stream(stream):
                v = grid.view()
                wl.dsxw_drift(C.byref(v), 5, step, w.drift, stream.cuda_stream)
                wl.dsxw_advance(stream.cuda_stream)
            stream.synchronize()
            before = [float(owned(a).sum().item()) for a in (6, 7, 8)]
            with torch.cuda.stream(stream):
                status = grid.step(fill, capture=step > 0)
            stream.synchronize()
            assert status == 0, (step, status)
            G = grid.totals(stream=stream)["ghosts"]
            assert G > 0
            after = [float(owned(a).sum().item()) for a in (6, 7, 8)]
            for k, scale in enumerate((1.0, 2.0, 3.0)):
                assert after[k] - before[k] == scale * G, (step, k, after[k] - before[k], G)
            assert torch.equal(torch.sort(owned(12, "<i4", 4)).values, ids), step
            flags, anyv = grid.out_of_domain(stream=stream)
            assert not anyv, (step, np.flatnonzero(flags))
        # the step's ghosts equal a per-call rebuild on the same particles
        v = grid.view()
        step_ghosts = [torch.as_tensor(DeviceArray(v.base[a] + b * int(v.ghost_offset), G, t),
                                       device="cuda").clone()
                       for a, b, t in ((0, 8, "<f8"), (1, 8, "<f8"), (2, 8, "<f8"), (12, 4, "<i4"))]
        counts_step = grid.all_counts(stream=stream)[1]
        grid.exchange_halo(rebuild=True, stream=stream)
        stream.synchronize()
        assert (grid.all_counts(stream=stream)[1] == counts_step).all()
        v = grid.view()
        for (a, b, t), want in zip(((0, 8, "<f8"), (1, 8, "<f8"), (2, 8, "<f8"), (12, 4, "<i4")),
                                   step_ghosts):
            got = torch.as_tensor(DeviceArray(v.base[a] + b * int(v.ghost_offset), G, t), device="cuda")
            assert torch.equal(got.view(torch.int32) if t == "<i4" else got.view(torch.int64),
                               want.view(torch.int32) if t == "<i4" else want.view(torch.int64)), a
    finally:
        grid.close()


def test_full_size_two_shards_match_one_grid(cuda):
    """clustered_64 (16M particles, Dynamic cuts) split over two shards in
    lockstep on one GPU against one grid holding all 64 subdomains: after
    each drifted migrate, halo build and reverse sum every owned and every
    ghost array of every subdomain is bit-identical (compared on the
    device)."""
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    from dsdecompx_b200 import workloads as W
    w = W.WORKLOADS["clustered_64"]
    dims, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    data = W.generate(w, seed=13)
    owner = W.initial_owner(w, dims, data["x"], data["y"], data["z"])
    counts, grouped = W.group_by_owner(data, owner, w.nranks)
    del data, owner
    N, P = int(counts.sum()), w.nranks
    names = dsx.ARRAYS + [f[0] for f in w.fields]
    ob = np.concatenate([[0], np.cumsum(counts)])
    kw = dict(halo_width=w.halo, fields=w.fields)
    ref = dsx.VirtualGrid(P, w.dims, w.policy, w.lower, w.upper, particles=N,
                          ghost_capacity=int(0.9 * N), **kw)
    host = [np.ascontiguousarray(grouped[n]) if n in grouped else None for n in names]
    ref.upload_flat(counts, [h.ctypes.data if h is not None else None for h in host])
    shards = []
    for r in range(2):
        e = shd.DeviceEngine(P, w.dims, w.policy, w.lower, w.upper, particles=N, ghost_capacity=N // 2, **kw)
        sh = shd.ShardedGrid(e, r, 2)
        c = np.where(sh.owners == r, counts, 0)
        part = [np.ascontiguousarray(np.concatenate([h[ob[t]:ob[t + 1]] for t in sh.mine]))
                if h is not None else None for h in host]
        sh.upload_flat(c, [p.ctypes.data if p is not None else None for p in part])
        shards.append(sh)
    del host, grouped
    wl = W.harness()
    sizes = [8] * 11 + [4, 4] + [8]   # bytes per record of every array (one int64 field)

    def region(base, offset, start, n, a):
        t = "<i4" if sizes[a] == 4 else "<i8"
        return torch.as_tensor(DeviceArray(base + sizes[a] * (offset + start), n, t), device="cuda")

    def compare(what, ghosts):
        rv = ref.view()
        ro_, rg = ref.all_counts()
        rob = np.concatenate([[0], np.cumsum(ro_)])
        rgb = np.concatenate([[0], np.cumsum(rg)])
        for sh in shards:
            sv = sh.E.grid.view()
            so = sh.E.owned_counts()
            sob = np.concatenate([[0], np.cumsum(so)])
            for t in sh.mine:
                assert so[t] == ro_[t], (what, t)
                for a in range(len(sizes)):
                    assert torch.equal(region(rv.base[a], int(rv.owned_offset), int(rob[t]), int(ro_[t]), a),
                                       region(sv.base[a], int(sv.owned_offset), int(sob[t]), int(so[t]), a)), \
                        (what, t, a)
                if ghosts:
                    g = int(sh.plan.g[t])
                    assert g == rg[t], (what, t)
                    for a in range(len(sizes)):
                        mine_g = region(sh.E.asm[a].data_ptr(), 0, int(sh.plan.gbase[t]), g, a)
                        want = region(rv.base[a], int(rv.ghost_offset), int(rgb[t]), g, a)
                        assert torch.equal(want, mine_g), (what, t, a)

    def ghost_forces(base, offset, gid_base, gid_offset, n):
        gid = torch.as_tensor(DeviceArray(gid_base + 4 * gid_offset, n, "<i4"), device="cuda")
        for k, a in enumerate((6, 7, 8)):
            f = torch.as_tensor(DeviceArray(base[a] + 8 * offset, n, "<f8"), device="cuda")
            f.copy_(torch.sin(gid.double() * 0.37 + k))

    try:
        for step in range(2):
            for g in [ref] + [sh.E.grid for sh in shards]:
                v = g.view()
                wl.dsxw_drift(C.byref(v), 9, step, 0.3, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            ref.migrate()
            shd.run_lockstep([sh.migrate_steps() for sh in shards])
            compare(f"migrate {step}", False)
            ref.exchange_halo(rebuild=True)
            shd.run_lockstep([sh.exchange_halo_steps(True, False) for sh in shards])
            compare(f"halo {step}", True)
            rv = ref.view()
            G = int(ref.totals()["ghosts"])
            ghost_forces(list(rv.base), int(rv.ghost_offset), rv.base[12], int(rv.ghost_offset), G)
            for sh in shards:
                asm = [t.data_ptr() for t in sh.E.asm]
                ghost_forces(asm, 0, asm[12], 0, int(sh.plan.total))
            torch.cuda.synchronize()
            ref.reverse_halo()
            shd.run_lockstep([sh.reverse_halo_steps() for sh in shards])
            compare(f"reverse {step}", False)
    finally:
        ref.close()
        for sh in shards:
            sh.E.close()
