"""A shard engine over the oracle (test infrastructure).

It has the methods of dsdecompx_b200.sharded.DeviceEngine, backed by an
oracle grid of all P subdomains (the C restatement of the reference's Host
path) and numpy buffers, so that the sharded protocol -- its plans, its
ordering and its exchanges over torch.distributed -- runs on CPU and can be
checked against one oracle grid that holds every subdomain.
"""
import os
import sys
from typing import Dict

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from dsdecompx_b200.sharded import halo_tables, section_offsets  # noqa: E402

ARRAYS = orc.ARRAYS


class OracleEngine:
    device = "cpu"

    def __init__(self, nranks, dims=(0, 0, 0), policy="manual", lower=(0, 0, 0), upper=(1, 1, 1),
                 periodic=(True, True, True), halo_width=0.0, edges_and_corners=True, dynamic=None,
                 fields=()):
        import torch
        self.torch = torch
        self.g = orc.Grid("port", nranks, dims, policy, lower, upper, periodic, halo_width,
                          edges_and_corners, dynamic, fields)
        self.P = nranks
        self.dims = self.g.topology(0)[0]
        self.topology = [self.g.neighbors(t) for t in range(nranks)]
        self.nn, self.sender_of = halo_tables(self.topology)
        self.dynamic = policy == "dynamic"
        self.names = list(ARRAYS) + [f[0] for f in self.g.fields]
        self.all_arrays = list(range(len(self.names)))
        self.elem_bytes = [np.dtype(self.g.dtype_of(n)).itemsize * self.g.components(n)
                           for n in self.names]
        self.elem_bytes_all = list(self.elem_bytes)
        self.asm = [np.zeros(0, np.uint8) for _ in self.names]
        self.capacity = 1 << 40   # owned particles this shard can hold (the oracle grows)
        self.asm_cap = 0
        self._before = None
        self._last_res = None

    def close(self):
        self.g.close()

    def array_id(self, name):
        return self.names.index(name)

    # ---- raw views
    def _typed(self, name, raw, n):
        comps = self.g.components(name)
        v = raw.view(self.g.dtype_of(name))
        return v.reshape(n, comps) if comps > 1 else v

    def _owned_bytes(self, a):
        name = self.names[a]
        parts = [np.ascontiguousarray(self.g.read(t, name, 0, self.g.counts(t)[0])).reshape(-1).view(np.uint8)
                 for t in range(self.P)]
        return np.concatenate(parts) if parts else np.zeros(0, np.uint8)

    def _ghost_bytes(self, a):
        name = self.names[a]
        parts = []
        for t in range(self.P):
            o, g = self.g.counts(t)
            parts.append(np.ascontiguousarray(self.g.read(t, name, o, g)).reshape(-1).view(np.uint8))
        return np.concatenate(parts)

    def _write_ghost_bytes(self, a, raw):
        name = self.names[a]
        b = self.elem_bytes[a]
        at = 0
        for t in range(self.P):
            o, g = self.g.counts(t)
            if g:
                self.g.write(t, name, o, self._typed(name, raw[at * b:(at + g) * b].copy(), g))
            at += g

    def _view(self, place, a, writable=False):
        kind = place[0]
        if kind == "owned":
            return self._owned_bytes(a)
        if kind == "ghost":
            return self._ghost_bytes(a)
        if kind == "assembled":
            return self.asm[a]
        if kind == "buffer":
            _, buf, n, sections = place
            offs = section_offsets(n, [self.elem_bytes[s] for s in sections])
            j = sections.index(a)
            arr = buf.numpy()
            return arr[offs[j]:offs[j] + n * self.elem_bytes[a]]
        raise ValueError(kind)

    def copy(self, dst, src, rows, arrays):
        if not len(rows):
            return
        for a in arrays:
            b = self.elem_bytes[a]
            s = self._view(src, a)
            d = self._view(dst, a, True)
            for si, di, c in rows:
                d[di * b:(di + c) * b] = s[si * b:(si + c) * b]
            if dst[0] == "ghost":
                self._write_ghost_bytes(a, d)

    # ---- local calls
    def owned_counts(self):
        return np.array([self.g.counts(t)[0] for t in range(self.P)], dtype=np.int64)

    def set_rebalance_work(self, work):
        self.g.set_rebalance_work(work)

    def _remember_sources(self):
        gids, src = [], []
        for t in range(self.P):
            o = self.g.counts(t)[0]
            gids.append(self.g.read(t, "global_id", 0, o))
            src.append(np.full(o, t, np.int64))
        self._before = (np.concatenate(gids), np.concatenate(src), self.owned_counts())

    def migrate_local(self):
        self._remember_sources()
        res = self.g.migrate()
        self._last_res = res
        return res

    def rebalance_local(self, work, force):
        self._remember_sources()
        flags, imb = self.g.rebalance(work, force)
        return flags, float(imb[0]) if len(imb) else 1.0

    def migration_pairs(self):
        gids, src, before = self._before
        order = np.argsort(gids)
        pairs = np.zeros((self.P, self.P), dtype=np.int64)
        now = self.owned_counts()
        for t in range(self.P):
            ids = self.g.read(t, "global_id", 0, now[t])
            where = order[np.searchsorted(gids[order], ids)]
            came = src[where]
            moved = came != t
            np.add.at(pairs[t], came[moved], 1)
        return pairs

    def last_migration(self):
        before = self._before[2]
        pairs = self.migration_pairs()
        now = self.owned_counts()
        sent, received = pairs.sum(axis=0), pairs.sum(axis=1)
        res = np.zeros((self.P, 6), dtype=np.int64)
        res[:, 1] = before
        res[:, 2] = before - sent
        res[:, 3] = sent
        res[:, 4] = received
        res[:, 5] = now
        res[:, 0] = (sent != 0) | (received != 0)
        return res

    def halo_local(self, build, positions_only):
        return self.g.exchange_halo(rebuild=build)

    def send_lists(self):
        length = np.zeros(self.P * 26, dtype=np.int64)
        first = np.zeros(self.P * 26, dtype=np.int64)
        at = 0
        for t in range(self.P):
            blocks = self.g.halo_blocks(t)
            for m, n in enumerate(blocks):
                e = self.sender_of[t, m]
                if e >= 0:
                    length[e] = n
                    first[e] = at
                at += int(n)
        return length, first

    def reverse_local(self):
        self.g.reverse_halo()

    def forward_local(self, names):
        self.g.forward_exchange(names)

    def reverse_exchange_local(self, fields):
        self.g.reverse_exchange(fields)

    def upload(self, per_subdomain: Dict[int, Dict[str, np.ndarray]]):
        for t in range(self.P):
            d = per_subdomain.get(t)
            self.g.set_owned(t, d if d is not None else {"x": np.zeros(0)})

    # ---- memory
    def new_buffer(self, nbytes):
        return self.torch.zeros(int(nbytes), dtype=self.torch.uint8)

    def ensure_assembled(self, n):
        if n <= self.asm_cap:
            return False
        cap = max(int(n * 1.25), 16)
        for a, b in enumerate(self.elem_bytes):
            new = np.zeros(cap * b, np.uint8)
            new[:self.asm_cap * b] = self.asm[a][:self.asm_cap * b]
            self.asm[a] = new
        self.asm_cap = cap
        return True

    def assemble_owned(self, counts, buffers, segments):
        counts = np.asarray(counts, dtype=np.int64)
        ob = np.concatenate([[0], np.cumsum(counts)])
        data = [dict() for _ in range(self.P)]
        for a, name in enumerate(self.names):
            b = self.elem_bytes[a]
            cur = self._owned_bytes(a)
            new = np.zeros(int(ob[-1]) * b, np.uint8)
            for s in segments:
                src = cur if s["source"] < 0 else self._view(
                    ("buffer", buffers[s["source"]][0], buffers[s["source"]][1], self.all_arrays), a)
                d0 = (int(ob[s["dst_rank"]]) + int(s["dst_index"])) * b
                s0 = int(s["src_index"]) * b
                new[d0:d0 + int(s["count"]) * b] = src[s0:s0 + int(s["count"]) * b]
            for t in range(self.P):
                n = int(counts[t])
                data[t][name] = self._typed(name, new[int(ob[t]) * b:int(ob[t + 1]) * b].copy(), n)
        for t in range(self.P):
            self.g.set_owned(t, data[t])

    def read_owned(self, t, name):
        return self.g.read(t, name, 0, self.g.counts(t)[0])

    def write_owned(self, t, name, start, values):
        self.g.write(t, name, start, values)

    def read_assembled(self, lo, n, name):
        a = self.array_id(name)
        b = self.elem_bytes[a]
        return self._typed(name, self.asm[a][lo * b:(lo + n) * b].copy(), n)

    def write_assembled(self, lo, name, values):
        a = self.array_id(name)
        b = self.elem_bytes[a]
        raw = np.ascontiguousarray(values, dtype=self.g.dtype_of(name)).reshape(-1).view(np.uint8)
        self.asm[a][lo * b:lo * b + raw.size] = raw
