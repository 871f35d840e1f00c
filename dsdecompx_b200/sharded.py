"""Sharded virtual grid: the P subdomains of one box split over R processes.

The reference runs one MPI rank per subdomain; here one process per GPU owns
a block of subdomains (contiguous Cartesian blocks of the process grid, so
that the surface between processes is small) and keeps a grid of all P
subdomains that holds particles only in its own.  Every collective call runs
the local call of that grid, then ONE exchange step with the processes that
own the receiving subdomains, then assembles its own subdomains in the
reference's order (dsDecompX src/migration.cpp:147-389, src/halo.cpp:609-649,
src/halo.cpp:956-1040):

* migrate: subdomain t holds its retained particles, then the immigrants of
  every source subdomain q in ascending q, whichever process q lives on.  The
  local migrate already places particles bound for another process's
  subdomain t into the local copy of t, grouped by source in ascending order;
  those groups are sent to t's owner.  The (destination, source) counts are
  summed over all processes first, so every receiver knows where each group
  goes and how many bytes each peer sends.
* exchange_halo: receiver t's ghosts are its neighbors' send lists in t's
  own neighbor-block order.  The local build writes the lists of local
  senders (to every receiver); lists for another process's receiver are sent
  there, and every process assembles its receivers' blocks into a separate
  ghost region (the one its callers read and write).
* reverse_halo: the forces of every assembled ghost go back to the process
  that owns its sender, into the local grid's slot of the same list, and the
  local reverse_halo sums each owner's images in the reference's order.
* forward_exchange / reverse_exchange of registered fields follow the
  refresh and the reverse.

The protocol is written once, as generator steps that yield communication
requests (:class:`AllReduce` of a small vector, :class:`Exchange` of byte
buffers with peers).  :func:`run_distributed` serves them with
torch.distributed (NCCL between GPUs, gloo on CPU: grouped point-to-point
sends and receives per peer), :func:`run_lockstep` serves several shards of
one process in lockstep (a received buffer is the sender's own).  Engines
(the device engine here, or any object with the same methods) do the local
work; a shard never reads another shard's memory except through a request.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import ARRAYS, COPY_DTYPE, SEGMENT_DTYPE, VirtualGrid, copy_segments

KMAX = 26           # neighbor entries per subdomain
XYZ = [0, 1, 2]     # array ids of the positions
FORCES = [6, 7, 8]  # array ids of the forces


# ------------------------------------------------------------ requests

class AllReduce:
    """Sum of a numeric vector over all shards (every shard gets the sum)."""

    def __init__(self, values: np.ndarray):
        self.values = np.ascontiguousarray(values)


class Exchange:
    """Point-to-point exchange: sends[p] goes to shard p; recv_bytes[p] is the
    size of what shard p sends here (both sides derive the sizes from the
    same all-reduced counts; empty messages are not sent)."""

    def __init__(self, sends: Dict[int, object], recv_bytes: Dict[int, int]):
        self.sends = sends
        self.recv_bytes = recv_bytes


def run_distributed(gen, device="cuda", group=None):
    """Runs one shard's protocol steps over torch.distributed (this process is
    the shard with the process group's rank)."""
    import torch
    import torch.distributed as dist
    reply = None
    while True:
        try:
            req = gen.send(reply)
        except StopIteration as stop:
            return stop.value
        if isinstance(req, AllReduce):
            t = torch.from_numpy(req.values.copy()).to(device)
            dist.all_reduce(t, group=group)
            reply = t.cpu().numpy()
        elif isinstance(req, Exchange):
            ops, recv = [], {}
            for p in sorted(req.recv_bytes):
                n = int(req.recv_bytes[p])
                if n:
                    buf = torch.empty(n, dtype=torch.uint8, device=device)
                    recv[p] = buf
                    ops.append(dist.P2POp(dist.irecv, buf, p, group))
            for p in sorted(req.sends):
                buf = req.sends[p]
                if buf is not None and buf.numel():
                    ops.append(dist.P2POp(dist.isend, buf, p, group))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            reply = recv
        else:
            raise TypeError(f"unknown request {req!r}")


def run_lockstep(gens: Sequence):
    """Runs the protocol steps of several shards of this process together:
    shard i's generator is gens[i]; every shard must make the same requests in
    the same order."""
    R = len(gens)
    replies: List[object] = [None] * R
    while True:
        reqs, done = [], []
        for i, g in enumerate(gens):
            try:
                reqs.append(g.send(replies[i]))
            except StopIteration as stop:
                done.append(stop.value)
        if done:
            if len(done) != R:
                raise RuntimeError("shards left the protocol at different steps")
            return done
        kinds = {type(r) for r in reqs}
        if len(kinds) != 1:
            raise RuntimeError("shards made different requests")
        if isinstance(reqs[0], AllReduce):
            total = reqs[0].values.copy()
            for r in reqs[1:]:
                total = total + r.values
            replies = [total.copy() for _ in range(R)]
        else:
            replies = []
            for i in range(R):
                got = {}
                for p, n in reqs[i].recv_bytes.items():
                    if not n:
                        continue
                    buf = reqs[p].sends.get(i)
                    if buf is None or int(buf.numel()) != int(n):
                        raise RuntimeError(f"shard {p} sends {0 if buf is None else buf.numel()} "
                                           f"bytes to shard {i}, which expects {n}")
                    got[p] = buf
                replies.append(got)


# ------------------------------------------------------- host planning

def subdomain_coords(rank: int, dims) -> Tuple[int, int, int]:
    """Row-major process-grid coordinates (z fastest), as the reference's
    Cartesian communicator numbers its ranks."""
    return rank // (dims[1] * dims[2]), (rank // dims[2]) % dims[1], rank % dims[2]


def block_owners(dims, nshards: int) -> np.ndarray:
    """Shard of every subdomain: contiguous Cartesian blocks when some
    (a, b, c), a * b * c = nshards, divides dims (the one with the least cut
    area between blocks; ties: the first in (a, b, c) order), else
    contiguous runs of subdomain ranks."""
    P = int(np.prod(dims))
    if nshards < 1 or nshards > P:
        raise ValueError("shards must be in 1..P")
    best = None
    for a in range(1, nshards + 1):
        if nshards % a or dims[0] % a:
            continue
        for b in range(1, nshards // a + 1):
            if (nshards // a) % b or dims[1] % b:
                continue
            c = nshards // a // b
            if dims[2] % c:
                continue
            cut = (a - 1) * dims[1] * dims[2] + (b - 1) * dims[0] * dims[2] + (c - 1) * dims[0] * dims[1]
            if best is None or cut < best[0]:
                best = (cut, a, b, c)
    owners = np.zeros(P, dtype=np.int64)
    if best is None:
        for t in range(P):
            owners[t] = t * nshards // P
        return owners
    _, a, b, c = best
    bx, by, bz = dims[0] // a, dims[1] // b, dims[2] // c
    for t in range(P):
        x, y, z = subdomain_coords(t, dims)
        owners[t] = ((x // bx) * b + y // by) * c + z // bz
    return owners


def plan_owners(dims, nshards: int) -> np.ndarray:
    """block_owners as the native library plans it (dsx_shard_plan_owners,
    host only): the owners a NativeShardedGrid created without them gets."""
    import ctypes as C

    from . import _check, lib
    d = np.ascontiguousarray([int(v) for v in dims], dtype=np.int32)
    out = np.zeros(int(np.prod(d, dtype=np.int64)), dtype=np.int32)
    _check(lib().dsx_shard_plan_owners(d.ctypes.data_as(C.POINTER(C.c_int)), int(nshards),
                                       out.ctypes.data_as(C.POINTER(C.c_int))))
    return out.astype(np.int64)


def halo_tables(topology):
    """(nn[P], sender_of[P, 26]) from every subdomain's neighbor list:
    receiver t's block m holds the list of its neighbor q toward -d_m, entry
    q * 26 + n (-1: no sender), the matching rule of the reference's receives
    (src/halo.cpp:609-649)."""
    P = len(topology)
    nn = np.array([len(t) for t in topology], dtype=np.int64)
    sender_of = np.full((P, KMAX), -1, dtype=np.int64)
    for t in range(P):
        for m, nb in enumerate(topology[t]):
            q = nb["rank"]
            if q < 0:
                continue
            want = tuple(-d for d in nb["direction"])
            for n, back in enumerate(topology[q]):
                if tuple(back["direction"]) == want:
                    sender_of[t, m] = q * KMAX + n
                    break
    return nn, sender_of


def packed_bytes(n: int, elem_bytes: Sequence[int]) -> int:
    """Size of a packed buffer of n records: one section per array, each
    starting on a 16-byte boundary."""
    return int(sum((n * b + 15) // 16 * 16 for b in elem_bytes))


def section_offsets(n: int, elem_bytes: Sequence[int]) -> List[int]:
    out, at = [], 0
    for b in elem_bytes:
        out.append(at)
        at += (n * b + 15) // 16 * 16
    return out


def group_exclusive(keys: np.ndarray, values: np.ndarray) -> np.ndarray:
    """Exclusive running sum of values within runs of equal consecutive keys."""
    if not len(values):
        return values.copy()
    before = np.cumsum(values) - values
    start = np.ones(len(keys), dtype=bool)
    start[1:] = keys[1:] != keys[:-1]
    first = np.maximum.accumulate(np.where(start, np.arange(len(keys)), 0))
    return before - before[first]


def merge_rows(rows: np.ndarray) -> np.ndarray:
    """(source, destination, count) rows with the runs that continue each
    other in both source and destination merged into one row."""
    rows = np.asarray(rows, dtype=np.int64).reshape(-1, 3)
    if len(rows) < 2:
        return rows
    s, d, n = rows[:, 0], rows[:, 1], rows[:, 2]
    start = np.ones(len(rows), dtype=bool)
    start[1:] = (s[1:] != s[:-1] + n[:-1]) | (d[1:] != d[:-1] + n[:-1])
    at = np.flatnonzero(start)
    return np.stack([s[at], d[at], np.add.reduceat(n, at)], axis=1)


class GhostPlan:
    """Where every block of this shard's receivers comes from and where the
    lists of its senders go: (k, 3) rows of (source index, destination index,
    count) -- local: engine ghost slot -> assembled slot; recv[p]: offset in
    shard p's buffer -> assembled slot; send[p]: engine ghost slot -> offset
    in the buffer for shard p."""

    def __init__(self, shard, owners, nn, sender_of, length, first):
        P = len(owners)
        owners = np.asarray(owners)
        length = np.asarray(length, dtype=np.int64)
        first = np.asarray(first, dtype=np.int64)
        blocks = np.arange(KMAX)[None, :] < np.asarray(nn)[:, None]      # [P, 26]
        sender_shard = np.where(sender_of >= 0, owners[np.maximum(sender_of, 0) // KMAX], -1)
        live = blocks & (sender_of >= 0)
        live &= np.where(live, length[np.maximum(sender_of, 0)], 0) > 0
        # receivers of this shard, blocks in (t, m) order
        mine = owners == shard
        t_idx, m_idx = np.nonzero(live & mine[:, None])
        e = sender_of[t_idx, m_idx]
        n = length[e]
        at = np.cumsum(n) - n
        self.total = int(n.sum())
        self.g = np.bincount(t_idx, weights=n, minlength=P).astype(np.int64)
        self.gbase = np.zeros(P, dtype=np.int64)
        order = np.flatnonzero(mine)
        self.gbase[order] = np.cumsum(self.g[order]) - self.g[order]
        p = sender_shard[t_idx, m_idx]
        loc = p == shard
        self.local = merge_rows(np.stack([first[e[loc]], at[loc], n[loc]], axis=1))
        self.recv: Dict[int, np.ndarray] = {}
        self.recv_n: Dict[int, int] = {}
        for q in np.unique(p[~loc]):
            sel = p == q
            off = np.cumsum(n[sel]) - n[sel]
            self.recv[int(q)] = merge_rows(np.stack([off, at[sel], n[sel]], axis=1))
            self.recv_n[int(q)] = int(n[sel].sum())
        # lists of this shard's senders to other shards' receivers, in the
        # receivers' (t, m) order
        t_idx, m_idx = np.nonzero(live & ~mine[:, None] & (sender_shard == shard))
        e = sender_of[t_idx, m_idx]
        n = length[e]
        p = owners[t_idx]
        self.send: Dict[int, np.ndarray] = {}
        self.send_n: Dict[int, int] = {}
        for q in np.unique(p):
            sel = p == q
            off = np.cumsum(n[sel]) - n[sel]
            self.send[int(q)] = merge_rows(np.stack([first[e[sel]], off, n[sel]], axis=1))
            self.send_n[int(q)] = int(n[sel].sum())


def merge_segments(seg: np.ndarray) -> np.ndarray:
    """Assembly segments in (destination subdomain, position) order, with
    the ones that continue each other (same source and subdomain, contiguous
    source and destination) merged."""
    seg = seg[np.lexsort((seg["dst_index"], seg["dst_rank"]))]
    if len(seg) < 2:
        return seg
    cont = np.zeros(len(seg), dtype=bool)
    cont[1:] = ((seg["source"][1:] == seg["source"][:-1]) & (seg["dst_rank"][1:] == seg["dst_rank"][:-1]) &
                (seg["src_index"][1:] == seg["src_index"][:-1] + seg["count"][:-1]) &
                (seg["dst_index"][1:] == seg["dst_index"][:-1] + seg["count"][:-1]))
    at = np.flatnonzero(~cont)
    out = seg[at].copy()
    out["count"] = np.add.reduceat(seg["count"], at)
    return out


def _rows(ranges) -> np.ndarray:
    return np.asarray(ranges, dtype=np.int64).reshape(-1, 3)


def _swap(ranges) -> np.ndarray:
    r = _rows(ranges)
    return r[:, [1, 0, 2]]


# --------------------------------------------------------- the grid

class ShardedGrid:
    """One shard of a sharded virtual grid.

    engine: the local engine (a :class:`DeviceEngine` for the device path);
    shard, nshards: this shard's index and the number of shards; owners:
    shard of every subdomain (default :func:`block_owners`); run: how the
    protocol's requests are served when a method is called directly
    (default :func:`run_distributed`).  The ``*_steps`` methods return the
    protocol generators themselves, for :func:`run_lockstep`.
    """

    def __init__(self, engine, shard: int, nshards: int, owners=None, run=None):
        self.E = engine
        self.P = engine.P
        self.shard, self.nshards = int(shard), int(nshards)
        self.owners = (np.asarray(owners, dtype=np.int64) if owners is not None
                       else block_owners(engine.dims, nshards))
        if self.owners.shape != (self.P,) or self.owners.min() < 0 or self.owners.max() >= nshards:
            raise ValueError("owners must give a shard in 0..nshards-1 for every subdomain")
        self.mine = np.flatnonzero(self.owners == self.shard)
        self.nn, self.sender_of = halo_tables(engine.topology)
        self.plan: Optional[GhostPlan] = None
        self.run = run or (lambda gen: run_distributed(gen, device=engine.device))
        # bytes this shard sent to other shards, per kind of message
        self.sent_bytes = {"migrants": 0, "ghost lists": 0, "returned values": 0}

    # ---- particles
    def upload(self, per_subdomain: Dict[int, Dict[str, np.ndarray]]):
        """Particles of this shard's subdomains (dicts of host arrays keyed by
        subdomain; missing subdomains are empty)."""
        for t in per_subdomain:
            if self.owners[t] != self.shard:
                raise ValueError(f"subdomain {t} belongs to shard {self.owners[t]}")
        self.E.upload(per_subdomain)
        self.plan = None

    def upload_flat(self, counts, arrays: List[Optional[int]]):
        """Particles from raw host or device pointers (arrays[13 + nfields],
        subdomains concatenated in rank order; counts[P] zero outside this
        shard's subdomains)."""
        c = np.asarray(counts, dtype=np.int64)
        if c.shape != (self.P,) or (c[self.owners != self.shard] != 0).any():
            raise ValueError("particles outside this shard's subdomains")
        self.E.grid.upload_flat(c, arrays)
        self.plan = None

    def download_flat(self, arrays: List[Optional[int]]) -> np.ndarray:
        return self.E.grid.download_flat(arrays)

    def ghost_view(self, totals):
        """A dsx_grid_view whose ghost region is this shard's assembled ghosts
        (for device code written against the grid view): totals is a device
        int32 tensor whose element 0 this call sets to the ghost count."""
        from . import GridView
        plan = self.plan
        v = self.E.grid.view()
        g = GridView()
        for a in range(len(self.E.names)):
            g.base[a] = self.E.asm[a].data_ptr() if self.E.asm else None
        g.owned_offset = 0
        g.ghost_offset = 0
        g.particles = 0
        g.ghost_capacity = self.E.asm_cap
        g.nranks = self.P
        totals.fill_(int(plan.total) if plan is not None else 0)
        g.halo_totals = totals.data_ptr()
        return g

    def counts(self, t: int) -> Tuple[int, int]:
        self._check_mine(t)
        g = int(self.plan.g[t]) if self.plan is not None else 0
        return int(self.E.owned_counts()[t]), g

    def read(self, t: int, name: str) -> np.ndarray:
        """Owned records then assembled ghosts of subdomain t (array `name`)."""
        self._check_mine(t)
        owned = self.E.read_owned(t, name)
        if self.plan is None or not self.plan.g[t]:
            return owned
        ghosts = self.E.read_assembled(int(self.plan.gbase[t]), int(self.plan.g[t]), name)
        return np.concatenate([owned, ghosts])

    def read_owned(self, t: int, name: str) -> np.ndarray:
        self._check_mine(t)
        return self.E.read_owned(t, name)

    def write_ghosts(self, t: int, name: str, values):
        """Values of the assembled ghosts of subdomain t (array `name`)."""
        self._check_mine(t)
        if self.plan is None:
            raise RuntimeError("no halo plan: call exchange_halo first")
        n = int(self.plan.g[t])
        v = np.asarray(values)
        if v.shape[0] != n:
            raise ValueError(f"subdomain {t} has {n} ghosts")
        self.E.write_assembled(int(self.plan.gbase[t]), name, v)

    def write_owned(self, t: int, name: str, start: int, values):
        self._check_mine(t)
        self.E.write_owned(t, name, start, values)

    def snapshot(self, t: int) -> Dict[str, np.ndarray]:
        out = {name: self.read(t, name) for name in self.E.names}
        out["owned"], out["ghosts"] = self.counts(t)
        return out

    def _check_mine(self, t: int):
        if self.owners[t] != self.shard:
            raise ValueError(f"subdomain {t} belongs to shard {self.owners[t]}")

    # ---- collective calls (every shard calls them in the same order)
    def migrate(self):
        return self.run(self.migrate_steps())

    def rebalance(self, work=None, force: bool = False):
        return self.run(self.rebalance_steps(work, force))

    def exchange_halo(self, rebuild: bool = False, positions_only: bool = False):
        return self.run(self.exchange_halo_steps(rebuild, positions_only))

    def reverse_halo(self):
        return self.run(self.reverse_halo_steps())

    def forward_exchange(self, names: Sequence[str]):
        return self.run(self.forward_exchange_steps(names))

    def reverse_exchange(self, fields: Sequence[Tuple[str, str]]):
        return self.run(self.reverse_exchange_steps(fields))

    def step(self, callback=None):
        """migrate -> exchange_halo(rebuild) -> callback(self) -> reverse_halo."""
        return self.run(self.step_steps(callback))

    # ---- protocol steps
    def step_steps(self, callback=None):
        mig = yield from self.migrate_steps()
        halo = yield from self.exchange_halo_steps(True, False)
        if callback is not None:
            callback(self)
        yield from self.reverse_halo_steps()
        return mig, halo

    def migrate_steps(self):
        E = self.E
        if E.dynamic:
            # the automatic rebalance sees every shard's counts
            total = yield AllReduce(E.owned_counts().astype(np.float64))
            E.set_rebalance_work(total)
        res = E.migrate_local()
        return (yield from self._redistribute(res))

    def rebalance_steps(self, work=None, force: bool = False):
        E = self.E
        local = np.zeros(self.P, dtype=np.float64)
        if work is None:
            local[self.mine] = E.owned_counts()[self.mine]
        else:
            w = np.asarray(work, dtype=np.float64)
            local[self.mine] = w[self.mine] if w.shape == (self.P,) else w
        total = yield AllReduce(local)
        flags, imbalance = E.rebalance_local(total, force)
        res = E.last_migration()
        mig = yield from self._redistribute(res)
        out = {t: (int(flags[t, 0]), int(flags[t, 1]), int(mig[t][5])) for t in self.mine}
        return out, float(imbalance)

    def _redistribute(self, res):
        """Sends every particle the local migrate placed into another shard's
        subdomain to that shard and assembles this shard's subdomains."""
        E, P, me, owners = self.E, self.P, self.shard, self.owners
        M = E.migration_pairs()
        # one all-reduce carries the (destination, source) counts, every
        # subdomain's retained particles and every shard's storage, so that
        # all shards see any shard's shortfall before data moves and fail
        # together (the reference agrees on errors the same way,
        # src/runtime.cpp:214-230)
        retained_mine = np.zeros(P, dtype=np.int64)
        retained_mine[self.mine] = res[self.mine, 2]
        capacity = np.zeros(self.nshards, dtype=np.int64)
        capacity[me] = E.capacity
        red = yield AllReduce(np.concatenate([M.reshape(-1).astype(np.int64), retained_mine, capacity]))
        Mg = red[:P * P].reshape(P, P)
        need = np.bincount(owners, weights=red[P * P:P * P + P] + Mg.sum(axis=1),
                           minlength=self.nshards).astype(np.int64)
        short = np.flatnonzero(need > red[P * P + P:])
        if len(short):
            self.plan = None
            raise MemoryError(f"dsDecompX: particle storage of shard(s) {short.tolist()} is smaller "
                              f"than their subdomains' particles after migration "
                              f"({need[short].tolist()} > {red[P * P + P:][short].tolist()})")
        local_n = res[:, 5].astype(np.int64)
        obase = np.concatenate([[0], np.cumsum(local_n)])
        allb = E.elem_bytes_all
        sends = {}
        for p in range(self.nshards):
            ts = np.flatnonzero((owners == p) & (local_n > 0))
            if p == me or not len(ts):
                continue
            cnt = local_n[ts]
            n = int(cnt.sum())
            rows = np.stack([obase[ts], np.cumsum(cnt) - cnt, cnt], axis=1)
            buf = E.new_buffer(packed_bytes(n, allb))
            E.copy(("buffer", buf, n, E.all_arrays), ("owned",), rows, E.all_arrays)
            sends[p] = buf
            self.sent_bytes["migrants"] += packed_bytes(n, allb)
        # what each peer sends: its sources' groups for my subdomains
        mine = self.mine
        sub = Mg[mine]                                               # [my subdomains, sources]
        from_peer = {p: int(sub[:, owners == p].sum()) for p in range(self.nshards) if p != me}
        recv = yield Exchange(sends, {p: packed_bytes(n, allb) for p, n in from_peer.items()})
        # new layout of t: retained, then the groups of its sources in
        # ascending source order, from this shard or from the source's shard
        peers = sorted(recv)
        retained = res[mine, 2].astype(np.int64)
        received = sub.sum(axis=1)
        new_counts = np.zeros(P, dtype=np.int64)
        new_counts[mine] = retained + received
        ti, q = np.nonzero(sub)
        c = sub[ti, q]
        p = owners[q]
        source = np.full(len(c), -1, dtype=np.int64)
        src = np.zeros(len(c), dtype=np.int64)
        loc = p == me
        src[loc] = obase[mine[ti[loc]]] + retained[ti[loc]] + group_exclusive(ti[loc], c[loc])
        for k, pp in enumerate(peers):
            sel = p == pp
            src[sel] = np.cumsum(c[sel]) - c[sel]
            source[sel] = k
        sent = res[mine, 3].astype(np.int64)
        out = {int(t): (int(sent[i] != 0 or received[i] != 0), int(res[t, 1]), int(retained[i]),
                        int(sent[i]), int(received[i]), int(new_counts[t]))
               for i, t in enumerate(mine)}
        self.plan = None
        if not peers and not local_n[owners != me].any():
            # nothing came in and nothing left: the local layout is final
            return out
        keep = retained > 0
        nk = int(keep.sum())
        seg = np.zeros(nk + len(c), dtype=SEGMENT_DTYPE)
        seg["source"][:nk] = -1
        seg["src_index"][:nk] = obase[mine[keep]]
        seg["dst_rank"][:nk] = mine[keep]
        seg["dst_index"][:nk] = 0
        seg["count"][:nk] = retained[keep]
        seg["source"][nk:] = source
        seg["src_index"][nk:] = src
        seg["dst_rank"][nk:] = mine[ti]
        seg["dst_index"][nk:] = retained[ti] + group_exclusive(ti, c)
        seg["count"][nk:] = c
        seg = merge_segments(seg)
        E.assemble_owned(new_counts, [(recv[pp], from_peer[pp]) for pp in peers], seg)
        return out

    def exchange_halo_steps(self, rebuild: bool = False, positions_only: bool = False):
        E = self.E
        build = rebuild or self.plan is None
        E.halo_local(build, positions_only and not build)
        if build:
            length, first = E.send_lists()
            total = yield AllReduce(length.astype(np.int64))
            length = total.astype(np.int64)
            prev = self.plan
            self.plan = GhostPlan(self.shard, self.owners, self.nn, self.sender_of, length, first)
            grew = E.ensure_assembled(self.plan.total)
        else:
            prev, grew = self.plan, False
        arrays = XYZ if (positions_only and not build) else E.all_arrays
        yield from self._ship_lists(arrays)
        plan = self.plan
        out = {}
        for t in self.mine:
            # layout_changed (src/runtime.cpp:966-980): a requested rebuild,
            # or another ghost count than before (none since a migrate); a
            # build is only ever forced by a missing plan, so the ghost ids of
            # an unrequested rebuild never need comparing
            g = int(plan.g[t])
            if rebuild:
                changed = 1
            elif prev is None:
                changed = int(g != 0)
            else:
                changed = int(int(prev.g[t]) != g)
            out[int(t)] = (g, changed, int(grew), int(not build))
        return out

    def _ship_lists(self, arrays):
        """Lists of local senders: into the assembled region (own receivers)
        or to the receivers' shards; lists of other shards' senders into the
        assembled region."""
        E, plan = self.E, self.plan
        b = [E.elem_bytes[a] for a in arrays]
        sends = {}
        for p, rows in plan.send.items():
            n = plan.send_n[p]
            buf = E.new_buffer(packed_bytes(n, b))
            E.copy(("buffer", buf, n, arrays), ("ghost",), _rows(rows), arrays)
            sends[p] = buf
            self.sent_bytes["ghost lists"] += packed_bytes(n, b)
        recv_bytes = {p: packed_bytes(n, b) for p, n in plan.recv_n.items()}
        recv = yield Exchange(sends, recv_bytes)
        if len(plan.local):
            E.copy(("assembled",), ("ghost",), _rows(plan.local), arrays)
        for p, rows in plan.recv.items():
            E.copy(("assembled",), ("buffer", recv[p], plan.recv_n[p], arrays), _rows(rows), arrays)

    def _return_lists(self, arrays):
        """The inverse of _ship_lists: assembled values back into the local
        engine's ghost slots of the same lists (own senders) or to the
        senders' shards."""
        E, plan = self.E, self.plan
        b = [E.elem_bytes[a] for a in arrays]
        if len(plan.local):
            E.copy(("ghost",), ("assembled",), _swap(plan.local), arrays)
        sends = {}
        for p, rows in plan.recv.items():
            n = plan.recv_n[p]
            buf = E.new_buffer(packed_bytes(n, b))
            E.copy(("buffer", buf, n, arrays), ("assembled",), _swap(rows), arrays)
            sends[p] = buf
            self.sent_bytes["returned values"] += packed_bytes(n, b)
        recv_bytes = {p: packed_bytes(n, b) for p, n in plan.send_n.items()}
        recv = yield Exchange(sends, recv_bytes)
        for p, rows in plan.send.items():
            E.copy(("ghost",), ("buffer", recv[p], plan.send_n[p], arrays), _swap(rows), arrays)

    def reverse_halo_steps(self):
        if self.plan is None:
            raise RuntimeError("reverse_halo without a halo plan")
        yield from self._return_lists(FORCES)
        self.E.reverse_local()

    def forward_exchange_steps(self, names: Sequence[str]):
        if self.plan is None:
            raise RuntimeError("forward_exchange without a halo plan")
        self.E.forward_local(list(names))
        yield from self._ship_lists([self.E.array_id(n) for n in names])

    def reverse_exchange_steps(self, fields: Sequence[Tuple[str, str]]):
        if self.plan is None:
            raise RuntimeError("reverse_exchange without a halo plan")
        yield from self._return_lists([self.E.array_id(n) for n, _ in fields])
        self.E.reverse_exchange_local(list(fields))


# ----------------------------------------------------- device engine

class DeviceEngine:
    """The local engine of a shard on this process's GPU: a VirtualGrid of
    all P subdomains, the assembled ghost region (device tensors), and the
    copies between them as dsx_copy_segments calls on the current stream."""

    device = "cuda"

    def __init__(self, nranks: int, dims=(0, 0, 0), policy: str = "manual",
                 lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), periodic=(True, True, True),
                 halo_width: float = 0.0, edges_and_corners: bool = True, dynamic=None,
                 fields: Sequence[Tuple[str, object, int]] = (), particles: int = 0,
                 ghost_capacity: int = 0):
        import torch
        self.torch = torch
        self.grid = VirtualGrid(nranks, dims, policy, lower, upper, periodic, halo_width,
                                edges_and_corners, dynamic, fields, particles, ghost_capacity)
        self.P = nranks
        self.dims = self.grid.topology(0)[0]
        self.topology = [self.grid.neighbors(t) for t in range(nranks)]
        self.dynamic = policy == "dynamic"
        self.names = ARRAYS + [f[0] for f in self.grid.fields]
        self.all_arrays = list(range(len(self.names)))
        self.elem_bytes = [np.dtype(self.grid.dtype_of(n)).itemsize * self.grid.components(n)
                           for n in self.names]
        self.elem_bytes_all = list(self.elem_bytes)
        self.asm_cap = 0
        self.asm: List = []
        self._last_migration = None
        self.capacity = int(particles)   # owned particles this shard can hold
        self.launches = 0   # kernels of this library launched through this engine

    def close(self):
        self.grid.close()

    def array_id(self, name: str) -> int:
        return self.names.index(name)

    # ---- local calls
    def owned_counts(self) -> np.ndarray:
        return self.grid.all_counts()[0]

    def set_rebalance_work(self, work):
        self.grid.set_rebalance_work(work)

    def migrate_local(self):
        # classify, scan, layout, move, emigrant histogram / column scan /
        # placement, and the rebalance kernel of a Dynamic grid
        self.launches += 7 + (1 if self.dynamic else 0)
        return self.grid.migrate()

    def rebalance_local(self, work, force):
        # Decomp::rebalance: explicit rebalance, then a migrate without the
        # automatic one; its per-subdomain counts follow from the layout
        before = self.owned_counts()
        flags, imbalance = self.grid.rebalance(work, force)
        self._last_migration = before
        return flags, imbalance[0] if len(imbalance) else 1.0

    def last_migration(self):
        """Per-subdomain results of the migrate inside the last rebalance, in
        migrate's format (previous from before, the rest from the pairs)."""
        before = self._last_migration
        pairs = self.grid.migration_pairs()
        now = self.owned_counts()
        sent = pairs.sum(axis=0)
        received = pairs.sum(axis=1)
        res = np.zeros((self.P, 6), dtype=np.int64)
        res[:, 1] = before
        res[:, 2] = before - sent
        res[:, 3] = sent
        res[:, 4] = received
        res[:, 5] = now
        res[:, 0] = (sent != 0) | (received != 0)
        return res

    def migration_pairs(self):
        self.launches += 1
        return self.grid.migration_pairs()

    def halo_local(self, build: bool, positions_only: bool):
        # build: classify, scan, layout, scatter; refresh: one kernel
        self.launches += 4 if build else 1
        return self.grid.exchange_halo(rebuild=build, positions_only=positions_only)

    def send_lists(self):
        return self.grid.send_lists()

    def reverse_local(self):
        self.launches += 1
        self.grid.reverse_halo()

    def forward_local(self, names):
        self.grid.forward_exchange(names)

    def reverse_exchange_local(self, fields):
        self.grid.reverse_exchange(fields)

    def upload(self, per_subdomain):
        empty = {n: np.zeros((0,) + ((self.grid.components(n),) if self.grid.components(n) > 1 else ()),
                             dtype=self.grid.dtype_of(n)) for n in self.names}
        self.grid.upload([per_subdomain.get(t, empty) for t in range(self.P)])

    # ---- memory
    def new_buffer(self, nbytes: int):
        return self.torch.empty(int(nbytes), dtype=self.torch.uint8, device="cuda")

    def ensure_assembled(self, n: int) -> bool:
        if n <= self.asm_cap:
            return False
        cap = max(int(n * 1.25), 1024)
        new = [self.torch.empty(cap * b, dtype=self.torch.uint8, device="cuda") for b in self.elem_bytes]
        if self.asm:
            for a, b in enumerate(self.elem_bytes):
                new[a][:self.asm_cap * b].copy_(self.asm[a])
        self.asm, self.asm_cap = new, cap
        return True

    def _bases(self, place, arrays):
        kind = place[0]
        v = self.grid.view()
        if kind == "owned":
            return [v.base[a] + int(v.owned_offset) * self.elem_bytes[a] for a in arrays]
        if kind == "ghost":
            return [v.base[a] + int(v.ghost_offset) * self.elem_bytes[a] for a in arrays]
        if kind == "assembled":
            return [self.asm[a].data_ptr() for a in arrays]
        if kind == "buffer":
            _, buf, n, sections = place
            offs = section_offsets(n, [self.elem_bytes[a] for a in sections])
            at = {a: o for a, o in zip(sections, offs)}
            return [buf.data_ptr() + at[a] for a in arrays]
        raise ValueError(kind)

    def copy(self, dst, src, rows: np.ndarray, arrays):
        """rows: (source index, destination index, count) per range; every
        array of `arrays` is copied."""
        if not len(rows):
            return
        sb, db = self._bases(src, arrays), self._bases(dst, arrays)
        out = np.zeros(len(rows) * len(arrays), dtype=COPY_DTYPE)
        for j, a in enumerate(arrays):
            b = self.elem_bytes[a]
            part = out[j * len(rows):(j + 1) * len(rows)]
            part["src"] = (sb[j] + rows[:, 0] * b).astype(np.uint64)
            part["dst"] = (db[j] + rows[:, 1] * b).astype(np.uint64)
            part["bytes"] = rows[:, 2] * b
        out = out[out["bytes"] > 0]
        if out.size:
            self.launches += 1
            copy_segments(out, self.torch.cuda.current_stream().cuda_stream)

    def assemble_owned(self, counts, buffers, segments):
        sources = []
        for buf, n in buffers:
            sources.append(self._bases(("buffer", buf, n, self.all_arrays), self.all_arrays))
        self.launches += 2   # the copies and the new layout
        self.grid.assemble(counts, sources, segments)

    # ---- host reads
    def read_owned(self, t: int, name: str) -> np.ndarray:
        return self.grid.read(t, name, 0, self.grid.counts(t)[0])

    def write_owned(self, t: int, name: str, start: int, values):
        self.grid.write(t, name, start, values)

    def read_assembled(self, lo: int, n: int, name: str) -> np.ndarray:
        a = self.array_id(name)
        b = self.elem_bytes[a]
        raw = self.asm[a][lo * b:(lo + n) * b].cpu().numpy()
        dt = np.dtype(self.grid.dtype_of(name))
        comps = self.grid.components(name)
        out = raw.view(dt)
        return out.reshape(n, comps) if comps > 1 else out

    def write_assembled(self, lo: int, name: str, values):
        a = self.array_id(name)
        b = self.elem_bytes[a]
        arr = np.ascontiguousarray(values, dtype=self.grid.dtype_of(name)).reshape(-1)
        raw = self.torch.from_numpy(arr.view(np.uint8).copy())
        self.asm[a][lo * b:lo * b + raw.numel()].copy_(raw)


# ------------------------------------------------- the native protocol

import ctypes as _C

_ALLREDUCE_I64 = _C.CFUNCTYPE(_C.c_int, _C.c_void_p, _C.POINTER(_C.c_longlong), _C.c_longlong)
_ALLREDUCE_F64 = _C.CFUNCTYPE(_C.c_int, _C.c_void_p, _C.POINTER(_C.c_double), _C.c_longlong)
_EXCHANGE = _C.CFUNCTYPE(_C.c_int, _C.c_void_p, _C.c_int, _C.POINTER(_C.c_int),
                         _C.POINTER(_C.c_void_p), _C.POINTER(_C.c_longlong), _C.c_int,
                         _C.POINTER(_C.c_int), _C.POINTER(_C.c_void_p), _C.POINTER(_C.c_longlong),
                         _C.c_void_p)


class _Transport(_C.Structure):
    _fields_ = [("user", _C.c_void_p), ("allreduce_i64", _ALLREDUCE_I64),
                ("allreduce_f64", _ALLREDUCE_F64), ("exchange", _EXCHANGE)]


class _DeviceBytes:
    """n device bytes at a raw address, as a CUDA-array-interface object."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = dict(shape=(int(n),), typestr="|u1", data=(int(ptr), False),
                                             version=3, strides=None)


class TorchTransport:
    """The native shard's transport over torch.distributed (NCCL between
    GPUs): sums through all_reduce, messages through grouped isend / irecv
    per peer on the caller's stream.  Exceptions become DSX_E_RUNTIME."""

    def __init__(self, device="cuda", group=None):
        self.device, self.group = device, group
        self.error: Optional[BaseException] = None
        self._i64 = _ALLREDUCE_I64(self._allreduce_i64)
        self._f64 = _ALLREDUCE_F64(self._allreduce_f64)
        self._ex = _EXCHANGE(self._exchange)
        self.struct = _Transport(None, self._i64, self._f64, self._ex)

    def _allreduce(self, ptr, n, dtype):
        import torch
        import torch.distributed as dist
        if dist.get_world_size(self.group) == 1:
            return   # the sum over one shard is its own values
        host = np.ctypeslib.as_array(ptr, shape=(int(n),))
        t = torch.from_numpy(host.astype(dtype)).to(self.device)
        dist.all_reduce(t, group=self.group)
        host[:] = t.cpu().numpy()

    def _allreduce_i64(self, user, ptr, n):
        try:
            self._allreduce(ptr, n, np.int64)
            return 0
        except BaseException as exc:   # never through the C frames
            self.error = exc
            return -3

    def _allreduce_f64(self, user, ptr, n):
        try:
            self._allreduce(ptr, n, np.float64)
            return 0
        except BaseException as exc:
            self.error = exc
            return -3

    def _exchange(self, user, nsend, to, send, send_bytes, nrecv, frm, recv, recv_bytes, stream):
        try:
            import torch
            import torch.distributed as dist
            ops = []
            as_tensor = lambda p, n: torch.as_tensor(_DeviceBytes(p, n), device=self.device)
            for k in range(nrecv):
                ops.append(dist.P2POp(dist.irecv, as_tensor(recv[k], recv_bytes[k]), int(frm[k]), self.group))
            for k in range(nsend):
                ops.append(dist.P2POp(dist.isend, as_tensor(send[k], send_bytes[k]), int(to[k]), self.group))
            if ops:
                with torch.cuda.stream(torch.cuda.ExternalStream(stream or 0)):
                    for w in dist.batch_isend_irecv(ops):
                        w.wait()
            return 0
        except BaseException as exc:
            self.error = exc
            return -3


class NativeShardedGrid:
    """One shard of the native sharded grid (dsx_shard_*): the same protocol
    as ShardedGrid, run by the library, with a transport (default: this
    process's torch.distributed group)."""

    def __init__(self, nranks: int, dims=(0, 0, 0), policy: str = "manual", lower=(0.0, 0.0, 0.0),
                 upper=(1.0, 1.0, 1.0), periodic=(True, True, True), halo_width: float = 0.0,
                 edges_and_corners: bool = True, dynamic=None,
                 fields: Sequence[Tuple[str, object, int]] = (), particles: int = 0,
                 ghost_capacity: int = 0, shard: Optional[int] = None, nshards: Optional[int] = None,
                 owners=None, transport: Optional[TorchTransport] = None, device="cuda"):
        from . import FIELD_TYPES, _check, _FieldDesc, _grid_desc, lib
        import torch.distributed as dist
        self.L = lib()
        self._check = _check
        self.P = nranks
        self.shard = dist.get_rank() if shard is None else int(shard)
        self.nshards = dist.get_world_size() if nshards is None else int(nshards)
        self.transport = transport or TorchTransport(device)
        d = _grid_desc(nranks, dims, policy, lower, upper, periodic, halo_width, edges_and_corners, dynamic)
        self.fields = [(str(n), FIELD_TYPES[t] if isinstance(t, str) else int(t), int(c))
                       for n, t, c in fields]
        self._names = [n.encode() for n, _, _ in self.fields]
        fd = (_FieldDesc * max(len(self.fields), 1))(
            *[_FieldDesc(self._names[i], t, c) for i, (_, t, c) in enumerate(self.fields)])
        own = None
        if owners is not None:
            self._owners_arg = np.ascontiguousarray(owners, dtype=np.int32)
            own = self._owners_arg.ctypes.data_as(_C.POINTER(_C.c_int))
        h = _C.c_void_p()
        self._call(self.L.dsx_shard_create(_C.byref(d), fd, len(self.fields), int(particles),
                                           int(ghost_capacity), self.shard, self.nshards, own,
                                           _C.byref(self.transport.struct), _C.byref(h)))
        self.h = h
        out = np.zeros(nranks, dtype=np.int32)
        self._call(self.L.dsx_shard_owners(self.h, out.ctypes.data_as(_C.POINTER(_C.c_int))))
        self.owners = out.astype(np.int64)
        self.mine = np.flatnonzero(self.owners == self.shard)

    def _call(self, status):
        err, self.transport.error = self.transport.error, None
        if status != 0 and err is not None:
            raise RuntimeError(f"transport failed: {err!r}") from err
        self._check(status)

    def close(self):
        if getattr(self, "h", None):
            self.L.dsx_shard_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self, stream):
        from . import _stream
        return _stream(stream)

    def upload_flat(self, counts, arrays: List[Optional[int]], stream=None):
        c = np.ascontiguousarray(counts, dtype=np.int64)
        ptrs = (_C.c_void_p * (13 + len(self.fields)))(*[a or None for a in arrays])
        self._call(self.L.dsx_shard_upload(self.h, c.ctypes.data_as(_C.POINTER(_C.c_longlong)), ptrs,
                                           self._stream(stream)))

    def migrate(self, stream=None):
        res = np.zeros((self.P, 6), dtype=np.int64)
        self._call(self.L.dsx_shard_migrate(self.h, self._stream(stream),
                                            res.ctypes.data_as(_C.POINTER(_C.c_longlong))))
        return {int(t): tuple(int(v) for v in res[t]) for t in self.mine}

    def rebalance(self, work=None, force: bool = False, stream=None):
        res = np.zeros((self.P, 3), dtype=np.int64)
        imb = _C.c_double()
        w = None if work is None else np.ascontiguousarray(work, dtype=np.float64)
        self._call(self.L.dsx_shard_rebalance(
            self.h, None if w is None else w.ctypes.data_as(_C.POINTER(_C.c_double)), 1 if force else 0,
            self._stream(stream), res.ctypes.data_as(_C.POINTER(_C.c_longlong)), _C.byref(imb)))
        return {int(t): tuple(int(v) for v in res[t]) for t in self.mine}, imb.value

    def exchange_halo(self, rebuild: bool = False, positions_only: bool = False, stream=None):
        res = np.zeros((self.P, 4), dtype=np.int64)
        self._call(self.L.dsx_shard_exchange_halo(self.h, 1 if rebuild else 0, 1 if positions_only else 0,
                                                  self._stream(stream),
                                                  res.ctypes.data_as(_C.POINTER(_C.c_longlong))))
        return {int(t): tuple(int(v) for v in res[t]) for t in self.mine}

    def reverse_halo(self, stream=None):
        self._call(self.L.dsx_shard_reverse_halo(self.h, self._stream(stream)))

    def _field_ids(self, names):
        index = {n: i for i, (n, _, _) in enumerate(self.fields)}
        return (_C.c_int * max(len(names), 1))(*[index[n] for n in names])

    def forward_exchange(self, names: Sequence[str], stream=None):
        self._call(self.L.dsx_shard_forward_exchange(self.h, len(names), self._field_ids(names),
                                                     self._stream(stream)))

    def reverse_exchange(self, fields: Sequence[Tuple[str, str]], stream=None):
        from . import OPS
        ops = (_C.c_int * max(len(fields), 1))(*[OPS[o] for _, o in fields])
        self._call(self.L.dsx_shard_reverse_exchange(self.h, len(fields),
                                                     self._field_ids([n for n, _ in fields]), ops,
                                                     self._stream(stream)))

    def step(self, callback=None, stream=None):
        """migrate -> exchange_halo(rebuild) -> callback(self) -> reverse_halo."""
        mig = self.migrate(stream)
        halo = self.exchange_halo(True, False, stream)
        if callback is not None:
            callback(self)
        self.reverse_halo(stream)
        return mig, halo

    def step_fused(self, callback=None, stream=None) -> int:
        """One fused step (dsx_shard_step): migrate, halo build,
        callback(view, stream), reverse_halo, planned from every shard's
        counts.  The view holds this shard's owned particles and its own
        receivers' ghosts.  Returns the device status bits (0 == ok)."""
        from . import STEP_CALLBACK, _raise_callback_error, _trampoline
        cache = self.__dict__.setdefault("_fused_cb", {})
        key = id(callback)
        if key not in cache:
            if callback is None:
                cache[key] = (None, STEP_CALLBACK())
            else:
                cache[key] = (callback, STEP_CALLBACK(_trampoline(callback, self)))
        st = _C.c_uint()
        fn = self.L.dsx_shard_step
        fn.argtypes = [_C.c_void_p, STEP_CALLBACK, _C.c_void_p, _C.c_void_p, _C.POINTER(_C.c_uint)]
        self._callback_error = None
        status = fn(self.h, cache[key][1], None, self._stream(stream), _C.byref(st))
        _raise_callback_error(self)
        self._call(status)
        return st.value

    def owned_view(self):
        from . import GridView
        v = GridView()
        self._call(self.L.dsx_shard_owned_view(self.h, _C.byref(v)))
        return v

    def totals(self, stream=None) -> Dict[str, int]:
        """The local grid's totals (owned, emigrants of the last migrate,
        ghosts of its own lists, boundary owners)."""
        out = np.zeros(4, dtype=np.int64)
        self._call(self.L.dsx_shard_totals(self.h, out.ctypes.data_as(_C.POINTER(_C.c_longlong)),
                                           self._stream(stream)))
        return dict(particles=int(out[0]), emigrants=int(out[1]), ghosts=int(out[2]),
                    boundary=int(out[3]))

    @property
    def launches(self) -> int:
        n = _C.c_longlong()
        self._call(self.L.dsx_shard_launches(self.h, _C.byref(n)))
        return n.value

    def ghost_view(self):
        from . import GridView
        v = GridView()
        self._call(self.L.dsx_shard_ghost_view(self.h, _C.byref(v)))
        return v

    def all_counts(self, stream=None):
        o = np.zeros(self.P, dtype=np.int64)
        g = np.zeros(self.P, dtype=np.int64)
        self._call(self.L.dsx_shard_counts(self.h, o.ctypes.data_as(_C.POINTER(_C.c_longlong)),
                                           g.ctypes.data_as(_C.POINTER(_C.c_longlong)),
                                           self._stream(stream)))
        return o, g

    def download_flat(self, arrays: List[Optional[int]], stream=None):
        """This shard's owned particles into host or device arrays (the
        subdomains concatenated in rank order); returns the counts."""
        c = np.zeros(self.P, dtype=np.int64)
        ptrs = (_C.c_void_p * (13 + len(self.fields)))(*[a or None for a in arrays])
        self._call(self.L.dsx_shard_download(self.h, c.ctypes.data_as(_C.POINTER(_C.c_longlong)), ptrs,
                                             self._stream(stream)))
        return c

    def counts(self, t: int) -> Tuple[int, int]:
        o, g = self.all_counts()
        return int(o[t]), int(g[t])

    def read_owned(self, t: int, name: str) -> np.ndarray:
        return self.read(t, name)[:self.counts(t)[0]]

    def _array(self, name: str):
        """(array id, element dtype, components) of a core array or field."""
        from . import ARRAYS, CORE_DTYPES, FIELD_DTYPES
        if name in ARRAYS:
            return ARRAYS.index(name), np.dtype(CORE_DTYPES[ARRAYS.index(name)]), 1
        k = [f[0] for f in self.fields].index(name)
        return 13 + k, np.dtype(FIELD_DTYPES[self.fields[k][1]]), self.fields[k][2]

    def read(self, t: int, name: str) -> np.ndarray:
        """Owned records then assembled ghosts of subdomain t (host)."""
        o, g = self.all_counts()
        a, dt, comps = self._array(name)
        b = dt.itemsize * comps
        out = np.zeros((int(o[t]) + int(g[t])) * b, dtype=np.uint8)
        v = self.owned_view()
        _device_to_host(out[:int(o[t]) * b], v.base[a] + b * (int(v.owned_offset) + int(o[:t].sum())))
        if g[t]:
            _device_to_host(out[int(o[t]) * b:], self.ghost_view().base[a] + b * int(g[:t].sum()))
        arr = out.view(dt)
        return arr.reshape(-1, comps) if comps > 1 else arr

    def write_owned(self, t: int, name: str, start: int, values):
        o, _ = self.all_counts()
        a, dt, comps = self._array(name)
        raw = np.ascontiguousarray(values, dtype=dt).reshape(-1).view(np.uint8)
        v = self.owned_view()
        b = dt.itemsize * comps
        _host_to_device(v.base[a] + b * (int(v.owned_offset) + int(o[:t].sum()) + int(start)), raw)

    def write_ghosts(self, t: int, name: str, values):
        _, g = self.all_counts()
        a, dt, comps = self._array(name)
        raw = np.ascontiguousarray(values, dtype=dt).reshape(-1).view(np.uint8)
        if raw.size != int(g[t]) * dt.itemsize * comps:
            raise ValueError(f"subdomain {t} has {int(g[t])} ghosts")
        _host_to_device(self.ghost_view().base[a] + dt.itemsize * comps * int(g[:t].sum()), raw)


def _device_to_host(dst: np.ndarray, src_ptr: int):
    if dst.size:
        import torch
        dst[:] = torch.as_tensor(_DeviceBytes(src_ptr, dst.size), device="cuda").cpu().numpy()


def _host_to_device(dst_ptr: int, src: np.ndarray):
    if src.size:
        import torch
        torch.as_tensor(_DeviceBytes(dst_ptr, src.size), device="cuda").copy_(torch.from_numpy(src.copy()))
