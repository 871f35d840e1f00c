"""Shared scenario builder for the parity tests: the same seeded inputs and
the same sequence of calls go to the CUDA grid and to the oracle, and every
array of every subdomain is compared bit for bit."""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

from oracle import FIELD_DTYPES, Grid

FIELD_TYPE_NAMES = ["int32", "int64", "uint32", "uint64", "float32", "float64"]

ALL_FIELDS = [("q", "float64", 1), ("vec3f", "float32", 3), ("tag", "int32", 1),
              ("big", "int64", 2), ("u", "uint32", 1), ("uu", "uint64", 1),
              ("wide", "float64", 7)]


def field_values(rng, name: str, t: str, comps: int, n: int) -> np.ndarray:
    dtype = FIELD_DTYPES[FIELD_TYPE_NAMES.index(t)]
    if t.startswith("float"):
        v = rng.normal(size=(n, comps))
    elif t.startswith("uint"):
        v = rng.integers(0, 1 << 30, size=(n, comps))
    else:
        v = rng.integers(-(1 << 30), 1 << 30, size=(n, comps))
    v = v.astype(dtype)
    return v.reshape(n) if comps == 1 else v


def bits(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    return a.view(np.uint8) if a.dtype.kind == "f" else a


def same(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


def uniform_particles(rng, n: int, lower, upper, fields=()) -> Dict[str, np.ndarray]:
    lower, upper = np.asarray(lower, float), np.asarray(upper, float)
    pos = rng.uniform(lower, upper, size=(n, 3))
    d = dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
             vx=rng.normal(size=n), vy=rng.normal(size=n), vz=rng.normal(size=n),
             fx=rng.normal(size=n), fy=rng.normal(size=n), fz=rng.normal(size=n),
             mass=np.ones(n), charge=rng.uniform(-1, 1, n),
             type=rng.integers(0, 8, n).astype(np.int32),
             global_id=np.arange(n, dtype=np.int32))
    for name, t, c in fields:
        d[name] = field_values(rng, name, t, c, n)
    return d


def split_by_owner(owner: np.ndarray, data: Dict[str, np.ndarray], nranks: int):
    out = []
    for r in range(nranks):
        m = owner == r
        out.append({k: np.asarray(v)[m] for k, v in data.items()})
    return out


class Pair:
    """A CUDA VirtualGrid and the oracle port driven in lockstep."""

    def __init__(self, nranks, dims=(0, 0, 0), policy="manual", lower=(0, 0, 0),
                 upper=(1, 1, 1), periodic=(True, True, True), halo_width=0.0,
                 edges_and_corners=True, dynamic=None, fields=(), particles=0,
                 ghost_capacity=0, oracle_kind="port"):
        import dsdecompx_b200 as dsx
        self.fields = list(fields)
        self.P = nranks
        kw = dict(nranks=nranks, dims=dims, policy=policy, lower=lower, upper=upper,
                  periodic=periodic, halo_width=halo_width,
                  edges_and_corners=edges_and_corners, dynamic=dynamic)
        self.gpu = dsx.VirtualGrid(fields=self.fields, particles=particles,
                                   ghost_capacity=ghost_capacity, **kw)
        self.ref = Grid(oracle_kind, fields=[(n, FIELD_TYPE_NAMES.index(t), c)
                                             for n, t, c in self.fields],
                        field_capacity=4 * max(particles, 16), **kw)

    def upload(self, per_rank: List[Dict[str, np.ndarray]]):
        self.gpu.upload(per_rank)
        for r, d in enumerate(per_rank):
            self.ref.set_owned(r, d)

    def displace(self, rng, sigma: float):
        for r in range(self.P):
            o, _ = self.ref.counts(r)
            dx = rng.normal(0.0, sigma, size=(o, 3))
            for a, name in enumerate("xyz"):
                v = self.ref.read(r, name, 0, o) + dx[:, a]
                self.ref.write(r, name, 0, v)
                self.gpu.write(r, name, 0, v)

    def set_ghost(self, rng, names: Sequence[str]):
        for r in range(self.P):
            o, g = self.ref.counts(r)
            for name in names:
                comps = self.ref.components(name)
                t = None
                for fn, ft, fc in self.fields:
                    if fn == name:
                        t = ft
                v = field_values(rng, name, t, comps, g) if t else rng.normal(size=g)
                self.ref.write(r, name, o, v)
                self.gpu.write(r, name, o, v)

    def compare(self, what: str = ""):
        for r in range(self.P):
            a, b = self.gpu.snapshot(r), self.ref.snapshot(r)
            assert a["owned"] == b["owned"] and a["ghosts"] == b["ghosts"], \
                (what, r, a["owned"], b["owned"], a["ghosts"], b["ghosts"])
            for k in b:
                if k in ("owned", "ghosts"):
                    continue
                assert same(a[k], b[k]), (what, r, k)

    def close(self):
        self.gpu.close()
        self.ref.close()
