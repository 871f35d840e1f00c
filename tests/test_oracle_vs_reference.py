"""Pins the oracle: the C restatement (oracle/dsx_oracle.c) against the
reference's own Host path built from its sources (oracle/_ref), bit for bit,
on seeded scenarios covering migrate, halo build and refresh, reverse_halo,
reverse_exchange with every op and field type, rebalance and the Dynamic
policy.  CPU only."""
import numpy as np
import pytest

import oracle
from helpers import ALL_FIELDS, FIELD_TYPE_NAMES, same, split_by_owner, uniform_particles

needs_ref = pytest.mark.skipif(not oracle.available("ref_debug"),
                               reason="reference build (oracle/_ref) not present")


def make_pair(kind_a, kind_b, **kw):
    fields = [(n, FIELD_TYPE_NAMES.index(t), c) for n, t, c in kw.pop("fields")]
    cap = kw.pop("field_capacity")
    a = oracle.Grid(kind_a, fields=fields, field_capacity=cap, **kw)
    b = oracle.Grid(kind_b, fields=fields, field_capacity=cap, **kw)
    return a, b


def compare(a, b, P, what):
    for r in range(P):
        x, y = a.snapshot(r), b.snapshot(r)
        assert x["owned"] == y["owned"] and x["ghosts"] == y["ghosts"], (what, r)
        for k in x:
            assert same(x[k], y[k]), (what, r, k)


def scenario(P, dims, L, halo, N, steps, seed, fields=ALL_FIELDS, sigma=0.3, policy="manual",
             periodic=(True, True, True), edges=True, dynamic=None, lower=(0.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    upper = tuple(lo + l for lo, l in zip(lower, L))
    # The reference's debug invariants reject particles that drift out of the
    # box through a non-periodic face (src/migration.cpp:558-577); its release
    # build clamps them into the edge cell, which is what the port follows.
    kind = "ref_debug" if all(periodic) else "ref"
    a, b = make_pair("port", kind, nranks=P, dims=dims, policy=policy, lower=lower,
                     upper=upper, periodic=periodic, halo_width=halo, edges_and_corners=edges,
                     dynamic=dynamic, fields=fields, field_capacity=4 * N + 64)
    data = uniform_particles(rng, N, lower, upper, fields)
    owner = b.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    assert (owner == a.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))).all()
    for r, d in enumerate(split_by_owner(owner, data, P)):
        a.set_owned(r, d)
        b.set_owned(r, d)
    names = [f[0] for f in fields]
    for step in range(steps):
        for r in range(P):
            o, _ = a.counts(r)
            dx = rng.normal(0, sigma, size=(o, 3))
            for k, name in enumerate("xyz"):
                v = a.read(r, name, 0, o) + dx[:, k]
                a.write(r, name, 0, v)
                b.write(r, name, 0, v)
        ma, mb = a.migrate(), b.migrate()
        assert (ma == mb).all(), (step, ma, mb)
        for x, y in zip(a.cuts(), b.cuts()):
            assert same(x, y)
        compare(a, b, P, f"migrate {step}")
        ha, hb = a.exchange_halo(step % 2 == 0), b.exchange_halo(step % 2 == 0)
        assert (ha[:, :2] == hb[:, :2]).all(), (ha, hb)
        compare(a, b, P, f"halo {step}")
        for r in range(P):
            o, g = a.counts(r)
            for name in ["fx", "fy", "fz"] + names:
                comps = a.components(name)
                t = next((ft for fn, ft, _ in fields if fn == name), "float64")
                from helpers import field_values
                v = field_values(rng, name, t, comps, g)
                a.write(r, name, o, v)
                b.write(r, name, o, v)
        a.reverse_halo()
        b.reverse_halo()
        compare(a, b, P, f"reverse_halo {step}")
        if names:
            ops = ["sum", "min", "max", "replace"]
            spec = [(n, ops[(i + step) % 4]) for i, n in enumerate(names)]
            a.reverse_exchange(spec)
            b.reverse_exchange(spec)
            compare(a, b, P, f"reverse_exchange {step}")
        for r in range(P):
            o, _ = a.counts(r)
            dx = rng.normal(0, sigma * 0.1, size=(o, 3))
            for k, name in enumerate("xyz"):
                v = a.read(r, name, 0, o) + dx[:, k]
                a.write(r, name, 0, v)
                b.write(r, name, 0, v)
        ha, hb = a.exchange_halo(False), b.exchange_halo(False)
        assert (ha[:, :2] == hb[:, :2]).all(), (ha, hb)
        compare(a, b, P, f"refresh {step}")
    a.close()
    b.close()


@needs_ref
@pytest.mark.parametrize("P,dims,L,halo,kw", [
    (1, (1, 1, 1), (10.0, 10.0, 10.0), 2.0, dict(sigma=3.0)),
    (2, (2, 1, 1), (10.0, 10.0, 10.0), 1.0, {}),
    (8, (2, 2, 2), (10.0, 10.0, 10.0), 1.0, {}),
    (12, (3, 1, 4), (9.0, 5.0, 12.0), 0.8,
     dict(periodic=(True, False, False), edges=False, lower=(-4.5, 1.0, 100.0))),
    (27, (3, 3, 3), (9.0, 9.0, 9.0), 0.9, dict(sigma=2.5, fields=ALL_FIELDS[:3])),
    (6, (0, 0, 0), (12.0, 8.0, 4.0), 0.5, dict(policy="balanced")),
    # a halo wider than half a cell: one particle reaches the same receiver
    # as its -x and its +x image (two blocks of one sender)
    (2, (2, 1, 1), (10.0, 10.0, 10.0), 3.0, dict(sigma=1.0)),
    (3, (3, 1, 1), (9.0, 4.0, 4.0), 2.5, dict(fields=ALL_FIELDS[:2])),
    # every axis periodic with the box off the origin: no shortcut wrap
    (8, (2, 2, 2), (10.0, 10.0, 10.0), 1.0, dict(lower=(-5.0, -5.0, -5.0), sigma=2.0)),
])
def test_port_matches_reference(P, dims, L, halo, kw):
    scenario(P, dims, L, halo, N=1500 * max(1, P // 4), steps=3, seed=P, **kw)


@needs_ref
def test_port_matches_reference_dynamic():
    scenario(8, (0, 0, 0), (16.0, 16.0, 16.0), 1.0, N=3000, steps=4, seed=21,
             policy="dynamic", dynamic=(1.0, 1.01, 0.5, 0.1), fields=ALL_FIELDS[:2], sigma=1.0)


@needs_ref
def test_port_matches_reference_rebalance():
    rng = np.random.default_rng(5)
    a, b = make_pair("port", "ref_debug", nranks=8, dims=(0, 0, 0), policy="dynamic",
                     lower=(0, 0, 0), upper=(8, 8, 8), periodic=(True,) * 3, halo_width=0.25,
                     edges_and_corners=True, dynamic=(0.0, 1.10, 1.0, 0.10), fields=[],
                     field_capacity=0)
    data = uniform_particles(rng, 2000, (0, 0, 0), (8, 8, 8))
    owner = a.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
    for r, d in enumerate(split_by_owner(owner, data, 8)):
        a.set_owned(r, d)
        b.set_owned(r, d)
    for work, force in [([100.0] + [1.0] * 7, True), (None, False), ([5.0] * 8, False),
                        ([1, 2, 3, 4, 5, 6, 7, 8.0], True)]:
        ra, ia = a.rebalance(work, force)
        rb, ib = b.rebalance(work, force)
        assert (ra == rb).all() and same(ia, ib)
        for x, y in zip(a.cuts(), b.cuts()):
            assert same(x, y)
        compare(a, b, 8, "rebalance")
    a.close()
    b.close()


def boundary_data(rng, N, L, h):
    """Uniform particles whose coordinates are, half of the time, one of the
    delicate values: cut planes, box faces, halo thresholds and their
    neighbours in FP64, signed zeros, denormals, far-away values, infinities
    and NaN."""
    special = np.array([0.0, -0.0, L / 2, L, h, L / 2 - h, L / 2 + h, L - h,
                        np.nextafter(L / 2, 0), np.nextafter(L / 2, L), np.nextafter(L, 0),
                        np.nextafter(h, 0), np.nextafter(L - h, L), -1e-300, 1e-320, 1e300,
                        -1e300, 2.3 * L, -0.75 * L, np.inf, -np.inf, np.nan])
    data = uniform_particles(rng, N, (0, 0, 0), (L, L, L))
    for k in "xyz":
        pick = rng.random(N) < 0.5
        data[k][pick] = rng.choice(special, pick.sum())
    return data


def nan_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        if not np.array_equal(na, nb):
            return False
        a, b = np.where(na, 0.0, a), np.where(nb, 0.0, b)
    return same(a, b)


@needs_ref
def test_boundary_values_port_vs_reference():
    """The restatement and the reference agree on the delicate inputs too
    (the reference's release build: its debug invariants stop on particles
    that belong to no subdomain, such as NaN positions)."""
    rng = np.random.default_rng(77)
    L, h, N, P = 10.0, 1.0, 3000, 8
    a, b = make_pair("port", "ref", nranks=P, dims=(2, 2, 2), policy="manual", lower=(0, 0, 0),
                     upper=(L, L, L), periodic=(True, True, True), halo_width=h,
                     edges_and_corners=True, dynamic=None, fields=[], field_capacity=4 * N + 64)
    try:
        data = boundary_data(rng, N, L, h)
        empty = {k: v[:0] for k, v in data.items()}
        for g in (a, b):
            g.set_owned(0, data)
            for r in range(1, P):
                g.set_owned(r, empty)
        for step in range(2):
            assert (a.migrate() == b.migrate()).all()
            a.exchange_halo(rebuild=True)
            b.exchange_halo(rebuild=True)
            for r in range(P):
                o, g_ = a.counts(r)
                f = rng.normal(size=g_)
                for name in ("fx", "fy", "fz"):
                    a.write(r, name, o, f)
                    b.write(r, name, o, f)
            a.reverse_halo()
            b.reverse_halo()
            for r in range(P):
                x, y = a.snapshot(r), b.snapshot(r)
                assert (x["owned"], x["ghosts"]) == (y["owned"], y["ghosts"]), (step, r)
                for k in x:
                    if k not in ("owned", "ghosts"):
                        assert nan_equal(x[k], y[k]), (step, r, k)
    finally:
        a.close()
        b.close()


@needs_ref
@pytest.mark.parametrize("policy,P,dims", [("manual", 8, (2, 2, 2)), ("dynamic", 27, (3, 3, 3))])
def test_rescale_and_update_domain(policy, P, dims):
    """Box changes (NPT-like): rescale_domain keeps the halo plan and refreshes
    ghosts with the new periodic shifts, update_domain invalidates it; cut
    planes keep their fractions of the extent.  Port vs reference."""
    rng = np.random.default_rng(5)
    N = 6000
    L = (12.0, 10.0, 9.0)
    dyn = (1.0, 1.01, 0.5, 0.1) if policy == "dynamic" else None
    a, b = make_pair("port", "ref", nranks=P, dims=dims, policy=policy, lower=(0, 0, 0),
                     upper=L, periodic=(True, True, True), halo_width=0.8,
                     edges_and_corners=True, dynamic=dyn, fields=ALL_FIELDS[:2],
                     field_capacity=4 * N + 64)
    try:
        data = uniform_particles(rng, N, (0, 0, 0), L, ALL_FIELDS[:2])
        owner = b.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1))
        for r, d in enumerate(split_by_owner(owner, data, P)):
            a.set_owned(r, d)
            b.set_owned(r, d)
        box = np.array(L)
        for step, (factor, update) in enumerate([(1.02, False), (0.97, True), (1.01, False)]):
            assert (a.migrate() == b.migrate()).all()
            a.exchange_halo(rebuild=True)
            b.exchange_halo(rebuild=True)
            compare(a, b, P, f"build {step}")
            new = box * factor
            for g in (a, b):
                g.rescale_domain((0.0, 0.0, 0.0), tuple(new), update=update)
                for r in range(P):
                    o, _ = g.counts(r)
                    for k, name in enumerate("xyz"):
                        g.write(r, name, 0, g.read(r, name, 0, o) * factor)
            box = new
            for x, y in zip(a.cuts(), b.cuts()):
                assert same(x, y), step
            ha, hb = a.exchange_halo(), b.exchange_halo()
            assert (ha[:, 0] == hb[:, 0]).all()
            compare(a, b, P, f"after {'update' if update else 'rescale'} {step}")
    finally:
        a.close()
        b.close()
