"""CUDA path vs the oracle (the reference's Host algorithm), bit for bit.

Every case drives the virtual grid through the C ABI (dsdecompx_b200 ->
libdsx.so) and the C restatement through the same seeded calls, then compares
every array of every subdomain: ids, positions (with the periodic shift),
velocities, forces, mass, charge, type and all registered fields.
"""
import numpy as np
import pytest

from helpers import ALL_FIELDS, Pair, same, split_by_owner, uniform_particles
from oracle import Grid

pytestmark = pytest.mark.gpu


def run_scenario(cuda, *, P, dims, L, halo, N, steps, seed, fields=ALL_FIELDS, sigma=0.3,
                 periodic=(True, True, True), edges=True, policy="manual", dynamic=None,
                 lower=(0.0, 0.0, 0.0), ghost_capacity=0, data_fn=None, plain=False):
    rng = np.random.default_rng(seed)
    upper = tuple(lo + l for lo, l in zip(lower, L))
    pair = Pair(P, dims, policy, lower, upper, periodic, halo, edges, dynamic, fields,
                particles=N, ghost_capacity=ghost_capacity)
    if plain:
        pair.gpu.set_plain(True)
    try:
        data = data_fn(rng, N, lower, upper) if data_fn else uniform_particles(rng, N, lower, upper, fields)
        owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
        pair.upload(split_by_owner(owner, data, P))
        pair.compare("upload")
        names = [f[0] for f in fields]
        for step in range(steps):
            pair.displace(rng, sigma)
            mg, mr = pair.gpu.migrate(), pair.ref.migrate()
            assert (mg == mr).all(), (step, mg, mr)
            if policy == "dynamic":
                for a, b in zip(pair.gpu.cuts(), pair.ref.cuts()):
                    assert same(a, b), (step, a, b)
            pair.compare(f"migrate {step}")
            hg, hr = pair.gpu.exchange_halo(rebuild=step % 2 == 0), pair.ref.exchange_halo(rebuild=step % 2 == 0)
            assert (hg[:, :2] == hr[:, :2]).all(), (step, hg, hr)
            pair.compare(f"halo build {step}")
            pair.set_ghost(rng, ["fx", "fy", "fz"])
            pair.gpu.reverse_halo()
            pair.ref.reverse_halo()
            pair.compare(f"reverse_halo {step}")
            if names:
                ops = ["sum", "min", "max", "replace"]
                spec = [(n, ops[(i + step) % 4]) for i, n in enumerate(names)]
                pair.set_ghost(rng, names)
                pair.gpu.reverse_exchange(spec)
                pair.ref.reverse_exchange(spec)
                pair.compare(f"reverse_exchange {step}")
                pair.gpu.forward_exchange(names[::-1])
                pair.ref.forward_exchange(names[::-1])
                pair.compare(f"forward_exchange {step}")
            # refresh along the plan after a small move
            pair.displace(rng, sigma * 0.1)
            hg, hr = pair.gpu.exchange_halo(), pair.ref.exchange_halo()
            assert (hg[:, 0] == hr[:, 0]).all()
            assert P == 1 or hg[:, 3].all(), hg
            pair.compare(f"refresh {step}")
        return pair
    except Exception:
        pair.close()
        raise


def test_two_by_two_by_two_all_field_types(cuda):
    run_scenario(cuda, P=8, dims=(2, 2, 2), L=(10.0, 10.0, 10.0), halo=1.0, N=6000, steps=3,
                 seed=1).close()


def test_single_rank_has_no_ghosts(cuda):
    pair = run_scenario(cuda, P=1, dims=(1, 1, 1), L=(10.0, 10.0, 10.0), halo=2.0, N=3000,
                        steps=2, seed=2, sigma=3.0)
    assert pair.gpu.counts(0)[1] == 0
    pair.close()


def test_uneven_grid_non_periodic_faces_only(cuda):
    run_scenario(cuda, P=12, dims=(3, 1, 4), L=(9.0, 5.0, 12.0), halo=0.8, N=8000, steps=3,
                 seed=3, periodic=(True, False, False), edges=False,
                 lower=(-4.5, 1.0, 100.0)).close()


def test_many_subdomains_with_long_jumps(cuda):
    # particles jump several cells: direct routing to any rank
    run_scenario(cuda, P=64, dims=(4, 4, 4), L=(16.0, 16.0, 16.0), halo=1.2, N=20000, steps=2,
                 seed=4, sigma=3.0, fields=ALL_FIELDS[:3]).close()


def test_balanced_policy_picks_the_reference_grid(cuda):
    pair = run_scenario(cuda, P=6, dims=(0, 0, 0), L=(12.0, 8.0, 4.0), halo=0.5, N=3000,
                        steps=1, seed=5, policy="balanced", fields=())
    assert pair.gpu.topology(0)[0] == pair.ref.topology(0)[0]
    pair.close()


def test_dynamic_boundaries_follow_the_reference(cuda):
    def clustered(rng, n, lower, upper):
        lower, upper = np.asarray(lower), np.asarray(upper)
        d = uniform_particles(rng, n, lower, upper, ALL_FIELDS[:2])
        k = int(0.8 * n)
        centre = rng.uniform(lower, upper, size=(4, 3))
        pick = rng.integers(0, 4, k)
        pos = centre[pick] + rng.normal(0, 1.5, size=(k, 3))
        pos = lower + np.mod(pos - lower, upper - lower)
        d["x"][:k], d["y"][:k], d["z"][:k] = pos[:, 0], pos[:, 1], pos[:, 2]
        return d

    pair = run_scenario(cuda, P=8, dims=(0, 0, 0), L=(24.0, 24.0, 24.0), halo=1.0, N=12000,
                        steps=4, seed=6, policy="dynamic", fields=ALL_FIELDS[:2],
                        dynamic=(1.0, 1.10, 0.5, 0.10), data_fn=clustered)
    # the boundaries moved
    assert not np.allclose(pair.gpu.cuts()[0], np.linspace(0, 24, 3))
    pair.close()


def test_largest_grid_with_dynamic_boundaries(cuda):
    """The engine's largest grid (1024 subdomains, 16x8x8 here): the layout
    runs one thread per subdomain, and the Dynamic rebalance has 32 slab sums,
    more than one pass of its lanes.  Clustered particles so that the cut
    planes move; every call compared with the oracle."""
    def clustered(rng, n, lower, upper):
        lower, upper = np.asarray(lower), np.asarray(upper)
        d = uniform_particles(rng, n, lower, upper, ALL_FIELDS[:1])
        k = int(0.7 * n)
        centre = rng.uniform(lower, upper, size=(6, 3))
        pos = centre[rng.integers(0, 6, k)] + rng.normal(0, 3.0, size=(k, 3))
        pos = lower + np.mod(pos - lower, upper - lower)
        d["x"][:k], d["y"][:k], d["z"][:k] = pos[:, 0], pos[:, 1], pos[:, 2]
        return d

    pair = run_scenario(cuda, P=1024, dims=(0, 0, 0), L=(96.0, 48.0, 48.0), halo=0.7, N=60000,
                        steps=3, seed=77, policy="dynamic", fields=ALL_FIELDS[:1],
                        dynamic=(1.0, 1.05, 0.5, 0.10), data_fn=clustered)
    try:
        dims = pair.gpu.topology(0)[0]
        assert sum(dims) > 31, dims
        assert not np.allclose(pair.gpu.cuts()[0], np.linspace(0, 96, dims[0] + 1))
    finally:
        pair.close()


def test_ghost_overflow_grows_and_rebuilds(cuda):
    # a deliberately tiny ghost capacity: the build must detect the overflow,
    # grow the ghost region and rebuild, with results identical to the oracle
    run_scenario(cuda, P=8, dims=(2, 2, 2), L=(8.0, 8.0, 8.0), halo=1.5, N=4000, steps=2,
                 seed=7, ghost_capacity=64, fields=ALL_FIELDS[:2]).close()


def test_all_particles_start_on_one_rank(cuda):
    rng = np.random.default_rng(8)
    pair = Pair(8, (2, 2, 2), "manual", (0, 0, 0), (6, 6, 6), halo_width=0.7,
                fields=ALL_FIELDS[:3], particles=5000)
    data = uniform_particles(rng, 5000, (0, 0, 0), (6, 6, 6), ALL_FIELDS[:3])
    per = [data] + [{k: v[:0] for k, v in data.items()} for _ in range(7)]
    pair.upload(per)
    assert (pair.gpu.migrate() == pair.ref.migrate()).all()
    pair.compare("scatter from rank 0")
    assert (pair.gpu.exchange_halo(True)[:, 0] == pair.ref.exchange_halo(True)[:, 0]).all()
    pair.compare("halo")
    pair.close()


def test_rebalance_api(cuda):
    rng = np.random.default_rng(9)
    pair = Pair(8, (0, 0, 0), "dynamic", (0, 0, 0), (8, 8, 8), halo_width=0.25,
                dynamic=(0.0, 1.10, 1.0, 0.10), particles=3000)
    data = uniform_particles(rng, 3000, (0, 0, 0), (8, 8, 8))
    owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    pair.upload(split_by_owner(owner, data, 8))
    work = [100.0] + [1.0] * 7
    rg, ig = pair.gpu.rebalance(work, force=True)
    rr, ir = pair.ref.rebalance(work, force=True)
    assert (rg == rr).all() and same(ig, ir), (rg, rr, ig, ir)
    for a, b in zip(pair.gpu.cuts(), pair.ref.cuts()):
        assert same(a, b)
    pair.compare("after rebalance")
    pair.close()


@pytest.mark.parametrize("kind", ["owners", "ghosts", "tiles", "auto"])
def test_refresh_kinds_follow_the_reference(cuda, kind):
    """Full refreshes along the plan (every field type, a halo wider than
    half a cell so that owners have many images) walked owner by owner,
    ghost by ghost and tile by tile give the oracle's ghosts."""
    rng = np.random.default_rng(41)
    pair = run_scenario(cuda, P=12, dims=(3, 2, 2), L=(9.0, 7.0, 6.0), halo=1.9, N=6000,
                        steps=1, seed=40)
    try:
        pair.gpu.set_refresh_kind(kind)
        for k in range(3):
            pair.displace(rng, 0.05)
            hg, hr = pair.gpu.exchange_halo(), pair.ref.exchange_halo()
            assert hg[:, 3].all() and (hg[:, 0] == hr[:, 0]).all()
            pair.compare(f"refresh {k}")
    finally:
        pair.close()


@pytest.mark.parametrize("kind", ["owners", "ghosts", "tiles"])
def test_positions_only_refresh(cuda, kind):
    pair = run_scenario(cuda, P=8, dims=(2, 2, 2), L=(10.0, 10.0, 10.0), halo=1.0, N=5000,
                        steps=1, seed=10, fields=ALL_FIELDS[:2])
    pair.gpu.set_refresh_kind(kind)
    rng = np.random.default_rng(11)
    before = [pair.gpu.snapshot(r) for r in range(8)]
    pair.displace(rng, 0.05)
    h = pair.gpu.exchange_halo(positions_only=True)
    pair.ref.exchange_halo()
    assert h[:, 3].all() and not h[:, 1].any()
    for r in range(8):
        a, b = pair.gpu.snapshot(r), pair.ref.snapshot(r)
        o = a["owned"]
        for k in ("x", "y", "z", "fx", "fy", "fz"):
            assert same(a[k][o:], b[k][o:]), k
        for k in ("vx", "mass", "global_id", "q"):
            assert same(a[k][o:], before[r][k][o:]), k
    pair.close()


class DeviceArray:
    """Wraps a raw device pointer for torch.as_tensor (CUDA array interface)."""

    def __init__(self, ptr, n, typestr="<f8"):
        self.__cuda_array_interface__ = dict(shape=(n,), typestr=typestr, data=(ptr, False),
                                             version=3, strides=None)


def ghost_force_filler(torch, capacity):
    """Step callback: every slot of the ghost region gets a force that depends
    only on its slot, copied on the step's stream from tensors made up front
    (nothing is allocated while a graph is being captured)."""
    slots = torch.arange(capacity, device="cuda", dtype=torch.float64)
    values = [torch.sin(slots * (j + 1)) for j in range(3)]

    def fill(view, stream):
        assert int(view.ghost_capacity) == capacity
        s = torch.cuda.ExternalStream(stream)
        with torch.cuda.stream(s):
            for j, k in enumerate((6, 7, 8)):
                t = torch.as_tensor(DeviceArray(view.base[k] + 8 * int(view.ghost_offset), capacity),
                                    device="cuda")
                t.copy_(values[j])
    return fill


def growing_force_filler(torch, most):
    """Like ghost_force_filler for a ghost region that may grow: slot k gets
    sin((j + 1) k), written from tensors made up front for up to `most` slots."""
    slots = torch.arange(most, device="cuda", dtype=torch.float64)
    values = [torch.sin(slots * (j + 1)) for j in range(3)]

    def fill(view, stream):
        capacity = int(view.ghost_capacity)
        assert capacity <= most
        s = torch.cuda.ExternalStream(stream)
        with torch.cuda.stream(s):
            for j, k in enumerate((6, 7, 8)):
                t = torch.as_tensor(DeviceArray(view.base[k] + 8 * int(view.ghost_offset), capacity),
                                    device="cuda")
                t.copy_(values[j][:capacity])
    return fill


def test_batched_step_ghost_overflow_redo(cuda):
    """A step whose ghost region overflows (capacity 64) grows it and redoes
    the halo build, the callback and the reverse sum; the result equals the
    per-call path, which grows the same way."""
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(17)
    fields = ALL_FIELDS[:2]
    kw = dict(nranks=8, dims=(2, 2, 2), lower=(0, 0, 0), upper=(12, 12, 12), halo_width=0.6,
              fields=fields, particles=8000, ghost_capacity=64)
    data = uniform_particles(rng, 8000, (0, 0, 0), (12, 12, 12), fields)
    a = Pair(**kw)
    owner = a.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 8)
    a.upload(per)
    b = dsx.VirtualGrid(**kw)
    b.upload(per)
    fill = growing_force_filler(torch, 1 << 18)
    side = torch.cuda.Stream()
    try:
        for step in range(3):
            a.displace(rng, 0.3)
            for r in range(8):
                o = b.counts(r)[0]
                for name in "xyz":
                    b.write(r, name, 0, a.gpu.read(r, name, 0, o))
            a.gpu.migrate()
            a.ref.migrate()
            a.gpu.exchange_halo(rebuild=True)
            a.ref.exchange_halo(rebuild=True)
            fill(a.gpu.view(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            for r in range(8):
                o, g = a.ref.counts(r)
                for name in ("fx", "fy", "fz"):
                    a.ref.write(r, name, o, a.gpu.read(r, name, o, g))
            a.gpu.reverse_halo()
            a.ref.reverse_halo()
            a.compare(f"calls {step}")
            torch.cuda.synchronize()
            before = int(b.view().ghost_capacity)
            with torch.cuda.stream(side):
                st = b.step(fill, capture=step > 0)
            side.synchronize()
            assert st == 0
            if step == 0:
                assert int(b.view().ghost_capacity) > before == 64
            for r in range(8):
                x, y = a.gpu.snapshot(r), b.snapshot(r)
                for k in x:
                    assert same(x[k], y[k]), (step, r, k)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("tuned", [False, True], ids=["default", "autotuned"])
def test_batched_step_matches_calls(cuda, tuned):
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(12)
    fields = ALL_FIELDS[:2]
    kw = dict(nranks=8, dims=(2, 2, 2), lower=(0, 0, 0), upper=(12, 12, 12), halo_width=0.6,
              fields=fields, particles=8000, ghost_capacity=12000)
    data = uniform_particles(rng, 8000, (0, 0, 0), (12, 12, 12), fields)
    a = Pair(**kw)
    owner = a.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 8)
    a.upload(per)
    b = dsx.VirtualGrid(**kw)
    b.upload(per)
    fill = ghost_force_filler(torch, 12000)
    side = torch.cuda.Stream()
    for step in range(4):
        if tuned and step in (0, 2):
            # tuning reads the particles and replaces the launch shapes
            rep = b.autotune()
            assert rep["classify_threads"] in (64, 128, 256)
            assert rep["reverse_ctas_per_sm"] in (4, 8, 16, 32)
            assert rep["ghost_capacity"] >= 12000
            assert min(rep["classify_ms"].values()) > 0
            assert min(rep["classify_combined_ms"].values()) > 0
        a.displace(rng, 0.3)
        for r in range(8):
            o = b.counts(r)[0]
            for name in "xyz":
                b.write(r, name, 0, a.gpu.read(r, name, 0, o))
        a.gpu.migrate()
        a.ref.migrate()
        a.gpu.exchange_halo(rebuild=True)
        a.ref.exchange_halo(rebuild=True)
        fill(a.gpu.view(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for r in range(8):
            o, g = a.ref.counts(r)
            for name in ("fx", "fy", "fz"):
                a.ref.write(r, name, o, a.gpu.read(r, name, o, g))
        a.gpu.reverse_halo()
        a.ref.reverse_halo()
        a.compare(f"calls {step}")
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            st = b.step(fill, capture=step > 0)
        side.synchronize()
        assert st == 0
        for r in range(8):
            x, y = a.gpu.snapshot(r), b.snapshot(r)
            for k in x:
                assert same(x[k], y[k]), (step, r, k)
    a.close()
    b.close()


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 2, 2)], ids=["2x2x2", "3x2x2"])
def test_plain_launches_follow_the_reference(cuda, dims):
    """One launch per subdomain (the comparison mode) gives the same arrays."""
    P = int(np.prod(dims))
    run_scenario(cuda, P=P, dims=dims, L=(12.0, 10.0, 9.0), halo=1.0, N=20000, steps=3,
                 seed=31, fields=ALL_FIELDS[:3], plain=True).close()


def test_halo_backward_is_reverse_halo(cuda):
    import torch
    pair = run_scenario(cuda, P=8, dims=(2, 2, 2), L=(10.0, 10.0, 10.0), halo=1.2, N=5000,
                        steps=1, seed=13, fields=())
    v = pair.gpu.view()
    G = int(pair.gpu.all_counts()[1].sum())
    N = int(v.particles)
    cot = torch.randn(3, G, dtype=torch.float64, device="cuda")
    grad = torch.randn(3, N, dtype=torch.float64, device="cuda")
    expect = grad.clone()
    pair.gpu.halo_backward(cot, grad)
    # reverse_halo on the same cotangents stored as ghost forces
    for j, k in enumerate((6, 7, 8)):
        gt = torch.as_tensor(DeviceArray(v.base[k] + 8 * int(v.ghost_offset), G), device="cuda")
        gt.copy_(cot[j])
        ot = torch.as_tensor(DeviceArray(v.base[k] + 8 * int(v.owned_offset), N), device="cuda")
        ot.copy_(expect[j])
    pair.gpu.reverse_halo()
    torch.cuda.synchronize()
    for j, k in enumerate((6, 7, 8)):
        ot = torch.as_tensor(DeviceArray(v.base[k] + 8 * int(v.owned_offset), N), device="cuda")
        assert torch.equal(ot, grad[j])
    pair.close()


def test_halo_backward_is_the_references_reverse_halo(cuda):
    """The adjoint of the ghost copy (dsx_grid_halo_backward) equals the
    reference's own reverse_halo (oracle/_ref, src/halo.cpp:1288-1347) on
    identical cotangents written as ghost forces, bit for bit."""
    import torch

    import oracle
    assert oracle.available("ref"), "the reference build oracle/_ref is required"
    lower, upper, halo = (0.0, 0.0, 0.0), (10.0, 10.0, 10.0), 1.2
    pair = run_scenario(cuda, P=8, dims=(2, 2, 2), L=(10.0, 10.0, 10.0), halo=halo, N=5000,
                        steps=1, seed=17, fields=())
    gpu = pair.gpu
    try:
        gpu.exchange_halo(rebuild=True)
        o, g = gpu.all_counts()
        ob = np.concatenate([[0], np.cumsum(o)])
        gb = np.concatenate([[0], np.cumsum(g)])
        N, G = int(o.sum()), int(g.sum())
        with oracle.Grid("ref", 8, (2, 2, 2), "manual", lower, upper, (True,) * 3, halo) as ref:
            for r in range(8):
                snap = gpu.snapshot(r)
                ref.set_owned(r, {k: np.asarray(snap[k])[:o[r]]
                                  for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz",
                                            "mass", "charge", "type", "global_id")})
            ref.exchange_halo(rebuild=True)
            for r in range(8):
                assert ref.counts(r) == (o[r], g[r])
                snap = gpu.snapshot(r)
                for k in ("x", "y", "z", "global_id"):
                    assert same(ref.read(r, k), snap[k]), (r, k)
            gen = torch.Generator(device="cuda").manual_seed(5)
            cot = torch.randn(3, G, dtype=torch.float64, device="cuda", generator=gen)
            grad0 = torch.randn(3, N, dtype=torch.float64, device="cuda", generator=gen)
            grad = grad0.clone()
            gpu.halo_backward(cot, grad)
            torch.cuda.synchronize()
            cot_h, grad0_h, grad_h = cot.cpu().numpy(), grad0.cpu().numpy(), grad.cpu().numpy()
            for r in range(8):
                for j, name in enumerate(("fx", "fy", "fz")):
                    ref.write(r, name, 0, grad0_h[j, ob[r]:ob[r + 1]])
                    ref.write(r, name, int(o[r]), cot_h[j, gb[r]:gb[r + 1]])
            ref.reverse_halo()
            for r in range(8):
                for j, name in enumerate(("fx", "fy", "fz")):
                    assert same(ref.read(r, name, 0, int(o[r])), grad_h[j, ob[r]:ob[r + 1]]), \
                        (r, name)
    finally:
        pair.close()


@pytest.mark.parametrize("fields,particles,box,halo", [
    (ALL_FIELDS[:1], 300_000, 12.0, 0.6),
    (ALL_FIELDS[:2], 300_000, 12.0, 0.6),
    (ALL_FIELDS, 40_000, 12.0, 0.6),
    (ALL_FIELDS[:2], 20_000, 6.0, 1.1)],
    ids=["record-104B", "record-116B", "record-204B", "wide-halo"])
def test_batched_step_many_tiles(cuda, fields, particles, box, halo):
    """The batched step against the per-call path and the oracle with far
    more 512-particle tiles than SMs: records the move stages in one pass
    (104 B and 116 B per particle), a record too wide for one pass (204 B:
    two passes of at most 56 KB per tile), and a halo wider than half a cell
    (every particle has 26 images, more than a tile stages: they are written
    from the hitting lanes)."""
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(29)
    capacity = 2 * particles if halo < 1.0 else 30 * particles
    kw = dict(nranks=27, dims=(3, 3, 3), lower=(0, 0, 0), upper=(box, box, box), halo_width=halo,
              fields=fields, particles=particles, ghost_capacity=capacity)
    data = uniform_particles(rng, particles, (0, 0, 0), (box, box, box), fields)
    a = Pair(**kw)
    owner = a.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 27)
    a.upload(per)
    b = dsx.VirtualGrid(**kw)
    b.upload(per)
    fill = ghost_force_filler(torch, capacity)
    side = torch.cuda.Stream()
    try:
        for step in range(3):
            a.displace(rng, 0.4)
            for r in range(27):
                o = b.counts(r)[0]
                for name in "xyz":
                    b.write(r, name, 0, a.gpu.read(r, name, 0, o))
            a.gpu.migrate()
            a.ref.migrate()
            a.gpu.exchange_halo(rebuild=True)
            a.ref.exchange_halo(rebuild=True)
            fill(a.gpu.view(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            for r in range(27):
                o, g = a.ref.counts(r)
                for name in ("fx", "fy", "fz"):
                    a.ref.write(r, name, o, a.gpu.read(r, name, o, g))
            a.gpu.reverse_halo()
            a.ref.reverse_halo()
            a.compare(f"calls {step}")
            torch.cuda.synchronize()
            with torch.cuda.stream(side):
                st = b.step(fill, capture=step > 0)
            side.synchronize()
            assert st == 0
            for r in range(27):
                x, y = a.gpu.snapshot(r), b.snapshot(r)
                for k in x:
                    assert same(x[k], y[k]), (step, r, k)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("fields,particles", [(ALL_FIELDS[:2], 200_000), (ALL_FIELDS, 60_000)],
                         ids=["record-116B", "record-204B"])
def test_every_tuning_gives_the_same_step(cuda, fields, particles):
    """The batched step with each move kind forced (staged in one pass,
    direct reads, staged in passes, staged without the force arrays) and each
    classify shape, with and without the immigrant counters combined per
    warp, and reverse grid: particles, ghosts and sums identical to
    the per-call path (itself checked against the oracle here).  At 204 B per
    particle one staged pass does not fit and kind 1 falls back to passes,
    while the stage without forces (about 92 KB a tile) fits."""
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(31)
    capacity = 2 * particles
    kw = dict(nranks=27, dims=(3, 3, 3), lower=(0, 0, 0), upper=(12.0, 12.0, 12.0),
              halo_width=0.6, fields=fields, particles=particles, ghost_capacity=capacity)
    data = uniform_particles(rng, particles, (0, 0, 0), (12.0, 12.0, 12.0), fields)
    a = Pair(**kw)
    owner = a.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 27)
    a.upload(per)
    tunings = [(128, "staged", 0), (64, "direct", 4), (256, "staged passes", 32),
               (128, "staged direct forces", 8), (128, "staged", 0, True), (64, "staged", 8, True),
               (256, "direct", 4, True)]
    grids = []
    for t in tunings:
        g = dsx.VirtualGrid(**kw)
        g.upload(per)
        g.set_tuning(*t)
        grids.append(g)
    with pytest.raises(ValueError):
        grids[0].set_tuning(96, "staged", 0)
    fill = ghost_force_filler(torch, capacity)
    side = torch.cuda.Stream()
    try:
        for step in range(3):
            a.displace(rng, 0.4)
            for g in grids:
                for r in range(27):
                    o = g.counts(r)[0]
                    for name in "xyz":
                        g.write(r, name, 0, a.gpu.read(r, name, 0, o))
            a.gpu.migrate()
            a.ref.migrate()
            a.gpu.exchange_halo(rebuild=True)
            a.ref.exchange_halo(rebuild=True)
            fill(a.gpu.view(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            for r in range(27):
                o, gh = a.ref.counts(r)
                for name in ("fx", "fy", "fz"):
                    a.ref.write(r, name, o, a.gpu.read(r, name, o, gh))
            a.gpu.reverse_halo()
            a.ref.reverse_halo()
            a.compare(f"calls {step}")
            torch.cuda.synchronize()
            for t, g in zip(tunings, grids):
                with torch.cuda.stream(side):
                    st = g.step(fill, capture=step > 0)
                side.synchronize()
                assert st == 0, t
                for r in range(27):
                    x, y = a.gpu.snapshot(r), g.snapshot(r)
                    for k in x:
                        assert same(x[k], y[k]), (t, step, r, k)
    finally:
        a.close()
        for g in grids:
            g.close()


def nan_equal(a, b) -> bool:
    """Bitwise equality, except that every NaN counts as the same value (a
    NaN made by inf - inf has the platform's own bits)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        if not np.array_equal(na, nb):
            return False
        a, b = np.where(na, 0.0, a), np.where(nb, 0.0, b)
    return same(a, b)


def test_boundary_values_follow_the_reference(cuda):
    """Positions on the cut planes, on the box faces, on the halo thresholds,
    signed zeros, denormals, values far outside the box, infinities and NaN:
    owners, wrapped positions, ghosts and sums as the reference's Host path
    makes them."""
    rng = np.random.default_rng(77)
    L, h = 10.0, 1.0
    special = np.array([0.0, -0.0, 5.0, 10.0, h, 5.0 - h, 5.0 + h, 10.0 - h, np.nextafter(5.0, 0),
                        np.nextafter(5.0, 10), np.nextafter(10.0, 0), np.nextafter(h, 0),
                        np.nextafter(10.0 - h, 10), -1e-300, 1e-320, 1e300, -1e300, 23.0, -7.5,
                        np.inf, -np.inf, np.nan])
    N = 3000
    data = uniform_particles(rng, N, (0, 0, 0), (L, L, L))
    for k in "xyz":
        pick = rng.random(N) < 0.5
        data[k][pick] = rng.choice(special, pick.sum())
    empty = {k: v[:0] for k, v in data.items()}
    pair = Pair(8, (2, 2, 2), "manual", (0, 0, 0), (L, L, L), (True, True, True), h, True, None,
                (), particles=N)
    try:
        pair.upload([data] + [empty] * 7)
        for step in range(2):
            pair.gpu.migrate()
            pair.ref.migrate()
            pair.gpu.exchange_halo(rebuild=True)
            pair.ref.exchange_halo(rebuild=True)
            pair.set_ghost(rng, ["fx", "fy", "fz"])
            pair.gpu.reverse_halo()
            pair.ref.reverse_halo()
            for r in range(8):
                a, b = pair.gpu.snapshot(r), pair.ref.snapshot(r)
                assert (a["owned"], a["ghosts"]) == (b["owned"], b["ghosts"]), (step, r)
                for k in b:
                    if k not in ("owned", "ghosts"):
                        assert nan_equal(a[k], b[k]), (step, r, k)
    finally:
        pair.close()


def test_empty_grid(cuda):
    """No particles at all: every call and the batched step run and stay empty."""
    import torch

    import dsdecompx_b200 as dsx
    kw = dict(nranks=8, dims=(2, 2, 2), lower=(0, 0, 0), upper=(10, 10, 10), halo_width=1.0,
              particles=0)
    pair = Pair(**kw)
    g = dsx.VirtualGrid(**kw)
    try:
        empty = uniform_particles(np.random.default_rng(1), 0, (0, 0, 0), (10, 10, 10))
        pair.upload([empty] * 8)
        g.upload([empty] * 8)
        assert (pair.gpu.migrate() == pair.ref.migrate()).all()
        pair.gpu.exchange_halo(rebuild=True)
        pair.ref.exchange_halo(rebuild=True)
        pair.gpu.reverse_halo()
        pair.ref.reverse_halo()
        pair.compare("empty")
        assert g.autotune()["ghost_capacity"] >= 0
        side = torch.cuda.Stream()
        for capture in (False, True, True):
            with torch.cuda.stream(side):
                assert g.step(None, capture=capture, stream=side.cuda_stream) == 0
            side.synchronize()
        with pytest.raises(ValueError, match="created stream"):
            g.step(None, capture=True)
        o, gh = g.all_counts()
        assert o.sum() == 0 and gh.sum() == 0
    finally:
        pair.close()
        g.close()


def test_set_cuts_follows_the_reference(cuda):
    """Explicit cut planes (the cuts a Dynamic rebalance would set): owners,
    ghosts and sums as the oracle makes them; bad cuts are refused."""
    rng = np.random.default_rng(41)
    L = (12.0, 10.0, 9.0)
    pair = Pair(8, (2, 2, 2), "manual", (0, 0, 0), L, (True, True, True), 0.7, True, None,
                ALL_FIELDS[:2], particles=6000)
    try:
        data = uniform_particles(rng, 6000, (0, 0, 0), L, ALL_FIELDS[:2])
        owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
        pair.upload(split_by_owner(owner, data, 8))
        for step, cuts in enumerate([([0, 4.5, 12.0], [0, 6.25, 10.0], [0, 3.0, 9.0]),
                                     ([0, 7.5, 12.0], [0, 2.0, 10.0], [0, 5.5, 9.0])]):
            pair.gpu.set_cuts(cuts)
            pair.ref.set_cuts(cuts)
            for a, b in zip(pair.gpu.cuts(), pair.ref.cuts()):
                assert same(a, b)
            pair.displace(rng, 0.2)
            assert (pair.gpu.migrate() == pair.ref.migrate()).all()
            pair.gpu.exchange_halo(rebuild=True)
            pair.ref.exchange_halo(rebuild=True)
            pair.set_ghost(rng, ["fx", "fy", "fz"])
            pair.gpu.reverse_halo()
            pair.ref.reverse_halo()
            pair.compare(f"cuts {step}")
        for bad in ([[0, 6.0, 11.0], [0, 5, 10], [0, 4, 9]],     # does not reach the upper face
                    [[0, 12.0, 12.0], [0, 5, 10], [0, 4, 9]],    # not strictly increasing
                    [[0.5, 6.0, 12.0], [0, 5, 10], [0, 4, 9]]):  # does not start at the lower face
            with pytest.raises(ValueError):
                pair.gpu.set_cuts(bad)
    finally:
        pair.close()


def test_rescale_and_update_domain_follow_the_reference(cuda):
    """A changing box (NPT-like): rescale_domain keeps the halo plan and a
    refresh moves ghosts with the new periodic shifts, update_domain
    invalidates the plan; cut planes keep their fractions.  The batched step
    on a second grid (its captured graphs re-made for the new box) gives the
    same arrays as the per-call path."""
    import torch

    import dsdecompx_b200 as dsx
    rng = np.random.default_rng(6)
    N = 8000
    L = np.array([12.0, 10.0, 9.0])
    kw = dict(nranks=27, dims=(3, 3, 3), lower=(0, 0, 0), upper=tuple(L), halo_width=0.8,
              fields=ALL_FIELDS[:2], particles=N, ghost_capacity=4 * N)
    pair = Pair(**kw)
    twin = dsx.VirtualGrid(**kw)
    fill = growing_force_filler(torch, 1 << 16)
    side = torch.cuda.Stream()
    try:
        data = uniform_particles(rng, N, (0, 0, 0), tuple(L), ALL_FIELDS[:2])
        owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
        per = split_by_owner(owner, data, 27)
        pair.upload(per)
        twin.upload(per)
        box = L.copy()
        for step, (factor, update) in enumerate([(1.02, False), (0.97, True), (1.01, False)]):
            # per-call path and oracle
            assert (pair.gpu.migrate() == pair.ref.migrate()).all()
            pair.gpu.exchange_halo(rebuild=True)
            pair.ref.exchange_halo(rebuild=True)
            fill(pair.gpu.view(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            for r in range(27):
                o, g = pair.ref.counts(r)
                for name in ("fx", "fy", "fz"):
                    pair.ref.write(r, name, o, pair.gpu.read(r, name, o, g))
            pair.gpu.reverse_halo()
            pair.ref.reverse_halo()
            pair.compare(f"calls {step}")
            # the same step batched on the twin
            with torch.cuda.stream(side):
                assert twin.step(fill, capture=True) == 0
            side.synchronize()
            for r in range(27):
                x, y = pair.gpu.snapshot(r), twin.snapshot(r)
                for k in x:
                    assert same(x[k], y[k]), (step, r, k)
            # new box on all three, positions scaled by the caller
            new = box * factor
            pair.gpu.rescale_domain((0, 0, 0), tuple(new), update=update)
            pair.ref.rescale_domain((0, 0, 0), tuple(new), update=update)
            twin.rescale_domain((0, 0, 0), tuple(new), update=update)
            box = new
            for g_ in (pair.gpu, pair.ref, twin):
                for r in range(27):
                    o = g_.counts(r)[0]
                    for name in "xyz":
                        g_.write(r, name, 0, g_.read(r, name, 0, o) * factor)
            for a, b in zip(pair.gpu.cuts(), pair.ref.cuts()):
                assert same(a, b), step
            hg, hr = pair.gpu.exchange_halo(), pair.ref.exchange_halo()
            assert (hg[:, 0] == hr[:, 0]).all()
            # rescale kept the plan (refreshed in place), update rebuilt it
            assert (hg[:, 3] == (0 if update else 1)).all()
            pair.compare(f"{'update' if update else 'rescale'} {step}")
    finally:
        pair.close()
        twin.close()


def test_owner_rank_and_out_of_domain(cuda):
    """owner_rank of arbitrary positions (faces, cut planes, far values,
    infinities, NaN) and the per-subdomain out-of-domain flags, against the
    oracle's owner rule, before and after a migrate."""
    import torch
    rng = np.random.default_rng(9)
    L = (12.0, 10.0, 9.0)
    pair = Pair(12, (3, 2, 2), "manual", (0, 0, 0), L, (True, True, False), 0.7, True, None,
                (), particles=5000)
    try:
        data = uniform_particles(rng, 5000, (0, 0, 0), L)
        owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
        pair.upload(split_by_owner(owner, data, 12))
        flags, anyv = pair.gpu.out_of_domain()
        assert not anyv and not flags.any()
        pair.displace(rng, 0.5)
        expect = np.zeros(12, dtype=np.int32)
        for r in range(12):
            o, _ = pair.ref.counts(r)
            pos = np.stack([pair.ref.read(r, k, 0, o) for k in "xyz"], 1)
            expect[r] = int((pair.ref.owner_rank(pos) != r).any()) if o else 0
        flags, anyv = pair.gpu.out_of_domain()
        assert (flags == expect).all() and anyv == bool(expect.any())
        pair.gpu.migrate()
        pair.ref.migrate()
        flags, anyv = pair.gpu.out_of_domain()
        assert not anyv
        special = np.array([0.0, -0.0, 4.0, 8.0, 12.0, 5.0, 10.0, 9.0, np.nextafter(4.0, 0),
                            -1e-300, 1e300, -37.5, np.inf, -np.inf, np.nan])
        pos = rng.uniform(-20, 30, size=(4000, 3))
        pick = rng.random(pos.shape) < 0.3
        pos[pick] = rng.choice(special, pick.sum())
        dev = [torch.as_tensor(np.ascontiguousarray(pos[:, a]), device="cuda") for a in range(3)]
        out = torch.empty(len(pos), dtype=torch.int32, device="cuda")
        pair.gpu.owner_rank(*dev, out)
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == pair.ref.owner_rank(pos)).all()
        # raw addresses need the count; lengths must agree (checked on the host)
        out.zero_()
        pair.gpu.owner_rank(*[t.data_ptr() for t in dev], out.data_ptr(), n=len(pos))
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == pair.ref.owner_rank(pos)).all()
        with pytest.raises(ValueError):
            pair.gpu.owner_rank(*[t.data_ptr() for t in dev], out.data_ptr())
        with pytest.raises(ValueError):
            pair.gpu.owner_rank(dev[0], dev[1], dev[2][:10], out)
    finally:
        pair.close()


@pytest.mark.parametrize("mode", ["default_stream", "graphs", "graphs_lean"])
def test_split_phase_halo_exchange(cuda, mode):
    """begin/end halo exchange with other GPU work in between: the same
    ghosts as the oracle's exchange_halo (builds, refreshes and a build that
    overflows and is redone in end); misuse is refused.  On the default
    stream the two halves are plain launches; on an explicit stream they are
    the captured graph segments, replayed over both owned halves, with the
    refresh on every resident CTA or on 2 CTAs per SM ("lean")."""
    import contextlib

    import torch
    rng = np.random.default_rng(23)
    L = (12.0, 10.0, 9.0)
    pair = Pair(12, (3, 2, 2), "manual", (0, 0, 0), L, (True, True, True), 0.8, True, None,
                ALL_FIELDS[:2], particles=8000, ghost_capacity=128)
    if mode == "graphs_lean":
        pair.gpu.set_split_share(2)
    other = torch.cuda.Stream()
    busy = torch.empty(1 << 24, device="cuda")
    scope = contextlib.nullcontext() if mode == "default_stream" else \
        torch.cuda.stream(torch.cuda.Stream())
    try:
        with scope:
            split_phase_steps(pair, rng, other, busy, L)
    finally:
        torch.cuda.synchronize()
        pair.close()


def split_phase_steps(pair, rng, other, busy, L):
    import torch
    data = uniform_particles(rng, 8000, (0, 0, 0), L, ALL_FIELDS[:2])
    owner = pair.ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    pair.upload(split_by_owner(owner, data, 12))
    for step in range(8):
        pair.displace(rng, 0.3 if step % 2 == 0 else 0.02)
        if step % 2 == 0:
            pair.gpu.migrate()
            pair.ref.migrate()
        rebuild = step % 2 == 0
        pair.gpu.begin_halo_exchange(rebuild=rebuild)
        with torch.cuda.stream(other):     # "interior" work meanwhile
            busy.normal_()
        hg = pair.gpu.end_halo_exchange()
        hr = pair.ref.exchange_halo(rebuild=rebuild)
        assert (hg[:, 0] == hr[:, 0]).all(), step
        assert (hg[:, 3] == (0 if rebuild else 1)).all(), step
        pair.compare(f"split {step}")
        pair.set_ghost(rng, ["fx", "fy", "fz"])
        pair.gpu.reverse_halo()
        pair.ref.reverse_halo()
        pair.compare(f"reverse {step}")
    pair.gpu.begin_halo_exchange()
    with pytest.raises(RuntimeError, match="in progress"):
        pair.gpu.begin_halo_exchange()
    with pytest.raises(RuntimeError, match="in progress"):
        pair.gpu.migrate()
    with pytest.raises(RuntimeError, match="in progress"):
        pair.gpu.rescale_domain((0, 0, 0), L)
    with pytest.raises(RuntimeError, match="in progress"):
        pair.gpu.autotune()
    with pytest.raises(RuntimeError, match="in progress"):
        pair.gpu.set_split_share(1)
    pair.gpu.end_halo_exchange()
    with pytest.raises(RuntimeError, match="without begin"):
        pair.gpu.end_halo_exchange()


@pytest.mark.parametrize("dims", [(3, 2, 2), (10, 1, 2)], ids=["counted", "bisected"])
def test_owner_rank_with_uneven_cuts(cuda, dims):
    """owner_rank where the cut planes are not uniform (the cell guessed from
    uniform cuts is then often wrong and the exact search must decide):
    random positions, the cut values themselves and their neighbors, faces,
    NaN and infinities, against the oracle; axes short enough to be counted
    and long enough to be bisected."""
    import torch
    rng = np.random.default_rng(19)
    L = (12.0, 10.0, 9.0)
    P = int(np.prod(dims))
    pair = Pair(P, dims, "manual", (0, 0, 0), L, (True, False, True), 0.5, True, None, (),
                particles=100)
    try:
        cuts = []
        for a in range(3):
            inner = np.sort(rng.uniform(0.05, 0.95, dims[a] - 1)) * L[a]
            cuts.append(np.concatenate([[0.0], inner, [L[a]]]))
        pair.gpu.set_cuts(cuts)
        pair.ref.set_cuts(cuts)
        special = np.concatenate([np.concatenate(cuts), np.nextafter(np.concatenate(cuts), -np.inf),
                                  np.nextafter(np.concatenate(cuts), np.inf),
                                  [-0.0, -1e-300, 1e300, -37.5, np.inf, -np.inf, np.nan]])
        pos = rng.uniform(-15, 25, size=(20000, 3))
        pick = rng.random(pos.shape) < 0.4
        pos[pick] = rng.choice(special, pick.sum())
        dev = [torch.as_tensor(np.ascontiguousarray(pos[:, a]), device="cuda") for a in range(3)]
        out = torch.empty(len(pos), dtype=torch.int32, device="cuda")
        pair.gpu.owner_rank(*dev, out)
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == pair.ref.owner_rank(pos)).all()
    finally:
        pair.close()


def test_step_callback_exception_reaches_the_caller(cuda):
    """An exception raised by the step's callback cannot cross the C frames;
    the Python call that ran the step raises it afterwards."""
    pair = run_scenario(cuda, P=8, dims=(2, 2, 2), L=(10.0, 10.0, 10.0), halo=1.0, N=3000,
                        steps=1, seed=61, fields=())
    try:
        def broken(view, stream):
            raise ValueError("from the callback")
        with pytest.raises(RuntimeError, match="from the callback"):
            pair.gpu.step(broken, capture=False)
        assert pair.gpu.step(None, capture=False) == 0   # the grid goes on
    finally:
        pair.close()


@pytest.mark.parametrize("ghost_capacity", [30000, 500], ids=["ample", "overflow"])
def test_async_steps_match_synchronous_steps(cuda, ghost_capacity):
    """dsx_grid_step_async queues each step before the previous one has
    finished (it checks that one's build at its event) and dsx_grid_step_wait
    completes them; the arrays, counts and cut planes must equal those of the
    same steps run one at a time by dsx_grid_step, bit for bit.  The tiny
    ghost capacity makes the first steps overflow, so the redo (grow, build,
    callback, reverse sum) runs on the queued path too.  The callback draws
    the drift and the ghost forces from the harness's device step counter,
    reset before each grid, so both grids see the same draws."""
    import ctypes as C

    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    wl = W.harness()
    rng = np.random.default_rng(31)
    n = 20000
    kw = dict(nranks=8, dims=(0, 0, 0), policy="dynamic", lower=(0, 0, 0), upper=(16, 16, 16),
              halo_width=0.8, fields=ALL_FIELDS[:2], particles=n,
              ghost_capacity=ghost_capacity, dynamic=(1.0, 1.05, 0.5, 0.10))
    data = uniform_particles(rng, n, (0, 0, 0), (16, 16, 16), ALL_FIELDS[:2])
    grids = [dsx.VirtualGrid(**kw) for _ in range(2)]
    with Grid("port", 8, (0, 0, 0), "dynamic", (0, 0, 0), (16, 16, 16), (True,) * 3, 0.8,
              dynamic=kw["dynamic"]) as probe:
        owner = probe.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 8)
    for g in grids:
        g.upload(per)
    stream = torch.cuda.Stream()

    def work(view, s):
        assert wl.dsxw_step_work(C.byref(view), 7, 0.25, s) == 0

    steps = 6
    torch.cuda.synchronize()
    wl.dsxw_set_step(0, stream.cuda_stream)
    for _ in range(steps):
        assert grids[0].step(work, capture=True, stream=stream) == 0
    stream.synchronize()
    wl.dsxw_set_step(0, stream.cuda_stream)
    for _ in range(steps):
        grids[1].step_async(work, stream=stream)
    assert grids[1].step_wait() == 0
    stream.synchronize()
    for r in range(8):
        a, b = grids[0].snapshot(r), grids[1].snapshot(r)
        for k in a:
            assert same(a[k], b[k]), (ghost_capacity, r, k)
    for ca, cb in zip(grids[0].cuts(), grids[1].cuts()):
        assert same(ca, cb)
    for g in grids:
        g.close()


def test_calls_between_queued_steps_complete_them(cuda):
    """A per-call operation after dsx_grid_step_async first completes the
    queued step (its build checked, its graph finished): the same sequence
    of steps and calls, queued on one grid and one call at a time on the
    other, leaves the same arrays, counts and cut planes."""
    import ctypes as C

    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W
    wl = W.harness()
    rng = np.random.default_rng(33)
    n = 12000
    kw = dict(nranks=8, dims=(2, 2, 2), policy="dynamic", lower=(0, 0, 0), upper=(12, 12, 12),
              halo_width=0.8, fields=ALL_FIELDS[:1], particles=n, ghost_capacity=20000,
              dynamic=(1.0, 1.05, 0.5, 0.10))
    data = uniform_particles(rng, n, (0, 0, 0), (12, 12, 12), ALL_FIELDS[:1])
    grids = [dsx.VirtualGrid(**kw) for _ in range(2)]
    with Grid("port", 8, (2, 2, 2), "dynamic", (0, 0, 0), (12, 12, 12), (True,) * 3, 0.8,
              dynamic=kw["dynamic"]) as probe:
        owner = probe.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    per = split_by_owner(owner, data, 8)
    for g in grids:
        g.upload(per)
    stream = torch.cuda.Stream()

    def work(view, s):
        assert wl.dsxw_step_work(C.byref(view), 5, 0.2, s) == 0

    torch.cuda.synchronize()
    for k, g in enumerate(grids):
        wl.dsxw_set_step(0, stream.cuda_stream)
        for _ in range(2):
            if k == 0:
                assert g.step(work, capture=True, stream=stream) == 0
            else:
                g.step_async(work, stream=stream)
        g.migrate(stream=stream)                     # completes a queued step first
        g.exchange_halo(rebuild=True, stream=stream)
        g.reverse_halo(stream=stream)
        for _ in range(2):
            if k == 0:
                assert g.step(work, capture=True, stream=stream) == 0
            else:
                g.step_async(work, stream=stream)
        if k == 1:
            assert g.step_wait() == 0
        stream.synchronize()
    for r in range(8):
        a, b = grids[0].snapshot(r), grids[1].snapshot(r)
        for key in a:
            assert same(a[key], b[key]), (r, key)
    for ca, cb in zip(grids[0].cuts(), grids[1].cuts()):
        assert same(ca, cb)
    for g in grids:
        g.close()
