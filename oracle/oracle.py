"""ctypes front end shared by the C restatement and the reference build.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Array ids shared by the oracle, the reference driver and the CUDA C-ABI.
ARRAYS = ["x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "mass", "charge",
          "type", "global_id"]
CORE_DTYPES = [np.float64] * 11 + [np.int32, np.int32]
# dsdecompx::FieldType order (include/field.hpp:22-29)
FIELD_DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float32, np.float64]
# dsdecompx::ReduceOp order (include/field.hpp:31-36)
OPS = {"sum": 0, "min": 1, "max": 2, "replace": 3}
# dsdecompx::GridPolicy order (include/grid.hpp:26-33)
POLICIES = {"manual": 0, "balanced": 1, "topology_aware": 2, "dynamic": 3}

_LIBS = {
    "port": os.path.join(HERE, "_build", "libdsx_oracle.so"),
    "ref": os.path.join(HERE, "_ref", "libdsx_ref.so"),
    "ref_debug": os.path.join(HERE, "_ref", "libdsx_ref_debug.so"),
}
_loaded: Dict[str, C.CDLL] = {}


def library_path(kind: str) -> str:
    return _LIBS[kind]


def available(kind: str) -> bool:
    return os.path.exists(_LIBS[kind])


def _lib(kind: str) -> C.CDLL:
    if kind not in _loaded:
        path = _LIBS[kind]
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library {path} is not built (run __graft_entry__.build())")
        lib = C.CDLL(path)
        prefix = "orc_" if kind == "port" else "ref_"
        vp, ip, dp, llp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong)
        getattr(lib, prefix + "last_error").restype = C.c_char_p
        getattr(lib, prefix + "last_error").argtypes = [vp]
        create = getattr(lib, prefix + "create")
        create.restype = vp
        for name, args in [
            ("destroy", [vp]), ("size", [vp]),
            ("topology", [vp, C.c_int, ip, ip, dp]),
            ("neighbors", [vp, C.c_int, ip, ip, dp]),
            ("cuts", [vp, dp]),
            ("owner_rank", [vp, C.c_longlong, dp, ip]),
            ("set_owned", [vp, C.c_int, C.c_longlong, C.POINTER(C.c_void_p), C.c_void_p,
                           C.c_void_p, C.POINTER(C.c_void_p)]),
            ("counts", [vp, C.c_int, llp, llp]),
            ("read", [vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p]),
            ("write", [vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p]),
            ("migrate", [vp, llp]),
            ("exchange_halo", [vp, C.c_int, llp]),
            ("reverse_halo", [vp]),
            ("rebalance", [vp, dp, C.c_int, llp, dp]),
            ("set_halo_width", [vp, C.c_double]),
            ("invalidate_halo", [vp]),
            ("rescale_domain", [vp, dp, dp, C.c_int]),
        ]:
            fn = getattr(lib, prefix + name)
            fn.restype = C.c_int
            fn.argtypes = args
        if kind == "port":
            lib.orc_set_cuts.restype = C.c_int
            lib.orc_set_cuts.argtypes = [vp, dp]
            lib.orc_reverse_exchange.argtypes = [vp, C.c_int, ip, ip]
            lib.orc_forward_exchange.argtypes = [vp, C.c_int, ip]
        else:
            lib.ref_reverse_exchange.argtypes = [vp, C.c_int, C.c_char_p, ip]
            lib.ref_timed.argtypes = [vp, C.c_int, dp]
        _loaded[kind] = lib
    return _loaded[kind]


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    pass


class Grid:
    """P virtual subdomains of one periodic (or not) box.

    ``fields`` is a list of ``(name, field_type, components)`` with
    ``field_type`` an index into :data:`FIELD_DTYPES`.
    """

    def __init__(self, kind: str, nranks: int, dims: Sequence[int] = (0, 0, 0),
                 policy: str = "manual", lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0),
                 periodic=(True, True, True), halo_width: float = 0.0,
                 edges_and_corners: bool = True,
                 dynamic: Optional[Tuple[float, float, float, float]] = None,
                 fields: Sequence[Tuple[str, int, int]] = (),
                 field_capacity: int = 0):
        self.kind = kind
        self.lib = _lib(kind)
        self.pre = "orc_" if kind == "port" else "ref_"
        self.nranks = nranks
        self.fields = [(str(n), int(t), int(c)) for n, t, c in fields]
        self.field_index = {n: i for i, (n, _, _) in enumerate(self.fields)}
        dims_a = (C.c_int * 3)(*dims)
        lo = (C.c_double * 3)(*lower)
        hi = (C.c_double * 3)(*upper)
        per = (C.c_int * 3)(*[1 if p else 0 for p in periodic])
        dyn = (C.c_double * 4)(*dynamic) if dynamic is not None else None
        nf = len(self.fields)
        types = (C.c_int * max(nf, 1))(*[t for _, t, _ in self.fields])
        comps = (C.c_longlong * max(nf, 1))(*[c for _, _, c in self.fields])
        err = C.create_string_buffer(512)
        create = getattr(self.lib, self.pre + "create")
        if kind == "port":
            create.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_double, C.c_int,
                               C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int),
                               C.POINTER(C.c_longlong), C.c_char_p, C.c_int]
            self.h = create(nranks, dims_a, POLICIES[policy], lo, hi, per, halo_width,
                            1 if edges_and_corners else 0, dyn, nf, types, comps, err, 512)
        else:
            create.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_double, C.c_int,
                               C.POINTER(C.c_double), C.c_int, C.c_char_p, C.POINTER(C.c_int),
                               C.POINTER(C.c_longlong), C.c_longlong, C.c_char_p, C.c_int]
            names = "\n".join(n for n, _, _ in self.fields).encode()
            self.h = create(nranks, dims_a, POLICIES[policy], lo, hi, per, halo_width,
                            1 if edges_and_corners else 0, dyn, nf, names, types, comps,
                            int(field_capacity), err, 512)
        if not self.h:
            raise OracleError(err.value.decode())

    # ---------------------------------------------------------------- helpers
    def _call(self, name, *args):
        status = getattr(self.lib, self.pre + name)(self.h, *args)
        if status != 0:
            raise OracleError(getattr(self.lib, self.pre + "last_error")(self.h).decode())
        return status

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, self.pre + "destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def dtype_of(self, name: str):
        if name in ARRAYS:
            return CORE_DTYPES[ARRAYS.index(name)]
        return FIELD_DTYPES[self.fields[self.field_index[name]][1]]

    def array_id(self, name: str) -> int:
        if name in ARRAYS:
            return ARRAYS.index(name)
        return 13 + self.field_index[name]

    def components(self, name: str) -> int:
        if name in ARRAYS:
            return 1
        return self.fields[self.field_index[name]][2]

    # -------------------------------------------------------------- topology
    def topology(self, rank: int):
        dims = (C.c_int * 3)()
        coords = (C.c_int * 3)()
        local = (C.c_double * 6)()
        self._call("topology", rank, dims, coords, local)
        return tuple(dims), tuple(coords), (tuple(local[:3]), tuple(local[3:]))

    def neighbors(self, rank: int):
        count = C.c_int()
        info = (C.c_int * (26 * 5))()
        shifts = (C.c_double * (26 * 3))()
        self._call("neighbors", rank, C.byref(count), info, shifts)
        out = []
        for n in range(count.value):
            out.append(dict(rank=info[5 * n], direction=tuple(info[5 * n + 1:5 * n + 4]),
                            slot=info[5 * n + 4], shift=tuple(shifts[3 * n:3 * n + 3])))
        return out

    def cuts(self):
        dims = self.topology(0)[0]
        out = (C.c_double * (sum(dims) + 3))()
        self._call("cuts", out)
        flat = list(out)
        res, k = [], 0
        for d in dims:
            res.append(np.array(flat[k:k + d + 1]))
            k += d + 1
        return res

    def owner_rank(self, positions: np.ndarray) -> np.ndarray:
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(len(pos), dtype=np.int32)
        self._call("owner_rank", len(pos), pos.ctypes.data_as(C.POINTER(C.c_double)),
                   out.ctypes.data_as(C.POINTER(C.c_int)))
        return out

    # ------------------------------------------------------------- particles
    def set_owned(self, rank: int, data: Dict[str, np.ndarray]):
        n = len(data["x"])
        keep = []
        core = (C.c_void_p * 11)()
        for a, name in enumerate(ARRAYS[:11]):
            if name in data:
                arr = np.ascontiguousarray(data[name], dtype=np.float64)
                keep.append(arr)
                core[a] = arr.ctypes.data
        typ = gid = None
        if "type" in data:
            typ = np.ascontiguousarray(data["type"], dtype=np.int32); keep.append(typ)
        if "global_id" in data:
            gid = np.ascontiguousarray(data["global_id"], dtype=np.int32); keep.append(gid)
        fptrs = (C.c_void_p * max(len(self.fields), 1))()
        for f, (name, t, c) in enumerate(self.fields):
            if name in data:
                arr = np.ascontiguousarray(data[name], dtype=FIELD_DTYPES[t]).reshape(-1)
                assert arr.size == n * c, (name, arr.size, n, c)
                keep.append(arr)
                fptrs[f] = arr.ctypes.data
        self._call("set_owned", rank, n, core, _ptr(typ), _ptr(gid), fptrs)

    def set_rebalance_work(self, work=None):
        """Work per rank for the next migrate's automatic rebalance."""
        if self.kind != "port":
            raise OracleError("set_rebalance_work is a call of the restatement")
        w = None if work is None else np.ascontiguousarray(work, dtype=np.float64)
        self._call("set_rebalance_work", None if w is None else w.ctypes.data_as(C.POINTER(C.c_double)))

    def halo_blocks(self, rank: int) -> np.ndarray:
        """Ghosts of `rank` per receive block (its neighbor order)."""
        if self.kind != "port":
            raise OracleError("halo_blocks is a query of the restatement")
        n = C.c_int()
        out = np.zeros(26, dtype=np.int64)
        self._call("halo_blocks", rank, C.byref(n), out.ctypes.data_as(C.POINTER(C.c_longlong)))
        return out[:n.value]

    def counts(self, rank: int) -> Tuple[int, int]:
        o, g = C.c_longlong(), C.c_longlong()
        self._call("counts", rank, C.byref(o), C.byref(g))
        return o.value, g.value

    def read(self, rank: int, name: str, start: int = 0, count: Optional[int] = None) -> np.ndarray:
        owned, ghosts = self.counts(rank)
        if count is None:
            count = owned + ghosts - start
        comps = self.components(name)
        out = np.zeros(count * comps, dtype=self.dtype_of(name))
        self._call("read", rank, self.array_id(name), start, count, _ptr(out))
        return out.reshape(count, comps) if comps > 1 else out

    def read_field(self, rank: int, field: str) -> np.ndarray:
        """Owned + ghost values of a registered field (by field name, even
        where it shares a name with a core array)."""
        f = self.field_index[field]
        _, t, comps = self.fields[f]
        owned, ghosts = self.counts(rank)
        out = np.zeros((owned + ghosts) * comps, dtype=FIELD_DTYPES[t])
        self._call("read", rank, 13 + f, 0, owned + ghosts, _ptr(out))
        return out.reshape(-1, comps) if comps > 1 else out

    def write(self, rank: int, name: str, start: int, values: np.ndarray):
        comps = self.components(name)
        arr = np.ascontiguousarray(values, dtype=self.dtype_of(name)).reshape(-1)
        count = arr.size // comps
        self._call("write", rank, self.array_id(name), start, count, _ptr(arr))

    def snapshot(self, rank: int) -> Dict[str, np.ndarray]:
        out = {name: self.read(rank, name) for name in ARRAYS}
        for name, _, _ in self.fields:
            out[name] = self.read(rank, name)
        out["owned"], out["ghosts"] = self.counts(rank)
        return out

    # ------------------------------------------------------------ operations
    def migrate(self) -> np.ndarray:
        res = np.zeros((self.nranks, 6), dtype=np.int64)
        self._call("migrate", res.ctypes.data_as(C.POINTER(C.c_longlong)))
        return res

    def exchange_halo(self, rebuild: bool = False) -> np.ndarray:
        res = np.zeros((self.nranks, 4), dtype=np.int64)
        self._call("exchange_halo", 1 if rebuild else 0,
                   res.ctypes.data_as(C.POINTER(C.c_longlong)))
        return res

    def reverse_halo(self):
        self._call("reverse_halo")

    def reverse_exchange(self, fields: List[Tuple[str, str]]):
        ops = (C.c_int * max(len(fields), 1))(*[OPS[o] for _, o in fields])
        if self.kind == "port":
            ids = (C.c_int * max(len(fields), 1))(*[self.field_index[n] for n, _ in fields])
            self._call("reverse_exchange", len(fields), ids, ops)
        else:
            names = "\n".join(n for n, _ in fields).encode()
            self._call("reverse_exchange", len(fields), names, ops)

    def forward_exchange(self, names: List[str]):
        if self.kind != "port":
            raise OracleError("the reference Host path has no forward_exchange")
        ids = (C.c_int * max(len(names), 1))(*[self.field_index[n] for n in names])
        self._call("forward_exchange", len(names), ids)

    def rebalance(self, work: Optional[Sequence[float]] = None, force: bool = False):
        res = np.zeros((self.nranks, 3), dtype=np.int64)
        imb = np.zeros(self.nranks, dtype=np.float64)
        w = None
        if work is not None:
            w = np.ascontiguousarray(work, dtype=np.float64)
        self._call("rebalance", None if w is None else w.ctypes.data_as(C.POINTER(C.c_double)),
                   1 if force else 0, res.ctypes.data_as(C.POINTER(C.c_longlong)),
                   imb.ctypes.data_as(C.POINTER(C.c_double)))
        return res, imb

    def set_halo_width(self, width: float):
        self._call("set_halo_width", float(width))

    def invalidate_halo(self):
        self._call("invalidate_halo")

    def set_cuts(self, cuts: Sequence[Sequence[float]]):
        """Replaces the cut planes (three increasing arrays spanning the
        domain); the halo plan becomes invalid.  Port only: the reference has
        no public call for it (it sets cuts inside its rebalance)."""
        if self.kind != "port":
            raise OracleError("set_cuts: the reference has no public call for it")
        flat = np.ascontiguousarray(np.concatenate([np.asarray(c, float) for c in cuts]))
        self._call("set_cuts", flat.ctypes.data_as(C.POINTER(C.c_double)))

    def rescale_domain(self, lower, upper, update: bool = False):
        """Decomp::rescale_domain (update=False: the halo plan is kept) or
        Decomp::update_domain (update=True: the plan is invalidated)."""
        lo = (C.c_double * 3)(*lower)
        hi = (C.c_double * 3)(*upper)
        self._call("rescale_domain", lo, hi, 1 if update else 0)

    def timed(self, op: str) -> float:
        """Slowest rank's wall time of one collective call (reference only)."""
        ops = {"migrate": 0, "halo_rebuild": 1, "halo_refresh": 2, "reverse_halo": 3}
        sec = C.c_double()
        self._call("timed", ops[op], C.byref(sec))
        return sec.value
