"""One seeded scenario for sharded grids against a grid that holds every
subdomain (the oracle, or the CUDA grid of one process).

Every draw depends only on (step, subdomain) and every ghost value only on
(ghost id, receiver), so that each shard can make its own without a shared
random stream; when the orders agree the arrays agree bit for bit.
"""
import numpy as np

from helpers import ALL_FIELDS, FIELD_TYPE_NAMES, same, split_by_owner, uniform_particles
from oracle import ARRAYS, FIELD_DTYPES

OPS = ["sum", "min", "max", "replace"]


def initial(ref, P, upper, N, seed, fields):
    rng = np.random.default_rng(seed)
    data = uniform_particles(rng, N, (0.0, 0.0, 0.0), upper, fields)
    owner = ref.owner_rank(np.stack([data["x"], data["y"], data["z"]], 1)) if hasattr(ref, "owner_rank") \
        else None
    return split_by_owner(owner, data, P)


def displacement(step, t, n, sigma):
    return np.random.default_rng(100_003 * step + 7 * t + 11).normal(0.0, sigma, size=(n, 3))


def ghost_value(name, t, gids, fields):
    types = {n: (FIELD_DTYPES[FIELD_TYPE_NAMES.index(ty)], c) for n, ty, c in fields}
    if name in ARRAYS:
        dtype, comps = np.float64, 1
    else:
        dtype, comps = types[name]
    k = np.arange(comps)
    if np.dtype(dtype).kind == "f":
        v = np.sin(gids.astype(np.float64)[:, None] * 0.37 + t + 1.3 * k)
    else:
        v = (gids.astype(np.int64)[:, None] * 2654435761 + 97 * t + k) % (1 << 28)
    v = v.astype(dtype)
    return v.reshape(-1) if comps == 1 else v


class Scenario:
    """shards: the ShardedGrid objects of this process; drive(name, *args)
    runs that collective call on all of them and returns their results (one
    per shard); ref: a grid of all P subdomains with the same calls."""

    def __init__(self, shards, drive, ref, P, fields):
        self.shards, self.drive, self.ref, self.P = shards, drive, ref, P
        self.fields = list(fields)
        self.names = list(ARRAYS) + [f[0] for f in self.fields]

    def displace(self, step, sigma):
        for t in range(self.P):
            o = self.ref.counts(t)[0]
            d = displacement(step, t, o, sigma)
            for a, name in enumerate("xyz"):
                self.ref.write(t, name, 0, self.ref.read(t, name, 0, o) + d[:, a])
        for sh in self.shards:
            for t in sh.mine:
                o = sh.counts(t)[0]
                d = displacement(step, t, o, sigma)
                for a, name in enumerate("xyz"):
                    sh.write_owned(t, name, 0, sh.read_owned(t, name) + d[:, a])

    def compare(self, what, names=None, ghosts=True):
        for sh in self.shards:
            for t in sh.mine:
                o, g = self.ref.counts(t)
                so, sg = sh.counts(t)
                assert so == o, (what, t, so, o)
                if ghosts:
                    assert sg == g, (what, t, sg, g)
                for name in names or self.names:
                    want = self.ref.read(t, name, 0, o + (g if ghosts else 0))
                    got = sh.read(t, name) if ghosts else sh.read_owned(t, name)
                    assert same(want, got), (what, t, name)

    def set_ghosts(self, names):
        for t in range(self.P):
            o, g = self.ref.counts(t)
            gid = self.ref.read(t, "global_id", o, g)
            for name in names:
                self.ref.write(t, name, o, ghost_value(name, t, gid, self.fields))
        for sh in self.shards:
            for t in sh.mine:
                o, g = sh.counts(t)
                gid = sh.read(t, "global_id")[o:]
                for name in names:
                    sh.write_ghosts(t, name, ghost_value(name, t, gid, self.fields))

    def run(self, steps, sigma):
        for step in range(steps):
            self.displace(step, sigma)
            mr = self.ref.migrate()
            for out in self.drive("migrate"):
                for t, row in out.items():
                    assert tuple(int(v) for v in mr[t]) == row, (step, t, mr[t], row)
            self.compare(f"migrate {step}")
            hr = self.ref.exchange_halo(rebuild=True)
            for out in self.drive("exchange_halo", True, False):
                for t, row in out.items():
                    assert (int(hr[t][0]), int(hr[t][1])) == row[:2], (step, t, hr[t], row)
            self.compare(f"halo build {step}")
            self.set_ghosts(["fx", "fy", "fz"])
            self.ref.reverse_halo()
            self.drive("reverse_halo")
            self.compare(f"reverse_halo {step}")
            fnames = [f[0] for f in self.fields]
            if fnames:
                spec = [(n, OPS[(i + step) % 4]) for i, n in enumerate(fnames)]
                self.set_ghosts(fnames)
                self.ref.reverse_exchange(spec)
                self.drive("reverse_exchange", spec)
                self.compare(f"reverse_exchange {step}")
                self.ref.forward_exchange(fnames[::-1])
                self.drive("forward_exchange", fnames[::-1])
                self.compare(f"forward_exchange {step}")
            # refresh along the plan after a small move
            self.displace(step + 1000, sigma * 0.1)
            hr = self.ref.exchange_halo()
            for out in self.drive("exchange_halo", False, False):
                for t, row in out.items():
                    assert (int(hr[t][0]), int(hr[t][1])) == row[:2], (step, t, hr[t], row)
            self.compare(f"refresh {step}")
            # positions-only refresh: the ghosts' positions follow, the rest
            # of their records stays (compared on the positions)
            self.displace(step + 2000, sigma * 0.1)
            self.ref.exchange_halo()
            for out in self.drive("exchange_halo", False, True):
                for t, row in out.items():
                    assert row[0] == int(self.ref.counts(t)[1]) and row[3] == 1, (step, t, row)
            self.compare(f"positions refresh {step}", names=["x", "y", "z", "global_id"])


def lockstep_drive(shards):
    from dsdecompx_b200.sharded import run_lockstep

    def drive(name, *args):
        return run_lockstep([getattr(s, name + "_steps")(*args) for s in shards])
    return drive


def distributed_drive(shard):
    def drive(name, *args):
        return [getattr(shard, name)(*args)]
    return drive


__all__ = ["ALL_FIELDS", "Scenario", "initial", "lockstep_drive", "distributed_drive"]
