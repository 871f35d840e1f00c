"""The batched step at the benchmark workloads' full sizes, through
properties that hold at any size (the oracle finishes only small cases):

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
