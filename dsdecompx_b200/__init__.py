"""B200-native particle bookkeeping for dsDecompX-style domain decomposition.

The compute path is the in-tree native library ``_lib/libdsx.so`` (hand-written
sm_100a CUDA behind the C ABI of ``include/dsx.h``).  This module is a thin
ctypes front end over that ABI for Python callers (tests, benchmarks, and
torch users); there is no Python or CPU fallback: if the library is missing,
importing :func:`lib` raises.

* :func:`rank_migrate` -- the single-rank drop-in migrate on device arrays.
* :class:`VirtualGrid` -- P subdomains of one box on one GPU: ``migrate``,
  ``exchange_halo``, ``reverse_halo``, ``reverse_exchange``,
  ``forward_exchange``, ``rebalance``, ``halo_backward`` and the batched,
  graph-captured ``step``.
* :mod:`dsdecompx_b200.sharded` -- the P subdomains split over several
  processes (one GPU each): ``NativeShardedGrid`` (the library's
  ``dsx_shard_*`` with a torch.distributed transport) and ``ShardedGrid``
  (the same protocol in Python, with engines that can be swapped).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _build

ARRAYS = ["x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "mass", "charge", "type",
          "global_id"]
CORE_DTYPES = [np.float64] * 11 + [np.int32, np.int32]
FIELD_DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float32, np.float64]
FIELD_TYPES = {"int32": 0, "int64": 1, "uint32": 2, "uint64": 3, "float32": 4, "float64": 5}
OPS = {"sum": 0, "min": 1, "max": 2, "replace": 3}
POLICIES = {"manual": 0, "balanced": 1, "topology_aware": 2, "dynamic": 3}

DSX_OK = 0
ERRORS = {-1: ValueError, -2: RuntimeError, -3: RuntimeError, -4: MemoryError, -5: OverflowError}


class DsxError(RuntimeError):
    pass


class _Domain(C.Structure):
    _fields_ = [("lower", C.c_double * 3), ("upper", C.c_double * 3), ("periodic", C.c_int * 3)]


class _MigrationResult(C.Structure):
    _fields_ = [("ownership_changed", C.c_int), ("previous_owned_count", C.c_longlong),
                ("retained_count", C.c_longlong), ("sent_count", C.c_longlong),
                ("received_count", C.c_longlong), ("new_owned_count", C.c_longlong)]


class _GridDesc(C.Structure):
    _fields_ = [("nranks", C.c_int), ("dims", C.c_int * 3), ("policy", C.c_int),
                ("lower", C.c_double * 3), ("upper", C.c_double * 3), ("periodic", C.c_int * 3),
                ("halo_width", C.c_double), ("edges_and_corners", C.c_int),
                ("dyn_interval", C.c_double), ("dyn_threshold", C.c_double),
                ("dyn_relaxation", C.c_double), ("dyn_min_fraction", C.c_double)]


class _FieldDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_int), ("components", C.c_int)]


# dsx_tune_report.move_staged values
MOVE_KINDS = {0: "direct", 1: "staged", 2: "staged passes", 3: "staged direct forces"}


class TuneReport(C.Structure):
    _fields_ = [("classify_threads", C.c_int), ("move_staged", C.c_int),
                ("reverse_ctas_per_sm", C.c_int), ("ghost_capacity", C.c_longlong),
                ("classify_ms", C.c_float * 3), ("move_ms", C.c_float * 4),
                ("reverse_ms", C.c_float * 4), ("classify_combine", C.c_int),
                ("classify_combined_ms", C.c_float * 3)]


class GridView(C.Structure):
    _fields_ = [("base", C.c_void_p * 32), ("owned_offset", C.c_longlong),
                ("ghost_offset", C.c_longlong), ("n", C.c_void_p), ("obase", C.c_void_p),
                ("g", C.c_void_p), ("gbase", C.c_void_p), ("halo_totals", C.c_void_p),
                ("particles", C.c_longlong), ("ghost_capacity", C.c_longlong),
                ("nranks", C.c_int)]


STEP_CALLBACK = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.POINTER(GridView))

_LIB: Optional[C.CDLL] = None


def library_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """The native library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not os.path.exists(path):
            raise DsxError(f"{path} is missing: run __graft_entry__.build() (there is no CPU fallback)")
        L = C.CDLL(path)
        vp, ip, dp, llp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong)
        L.dsx_last_error.restype = C.c_char_p
        L.dsx_version.restype = C.c_char_p
        sig = {
            "dsx_rank_migrate": [vp, vp, vp, C.c_longlong, C.POINTER(_Domain), vp,
                                 C.POINTER(_MigrationResult)],
            "dsx_plan_topology": [C.POINTER(_GridDesc), C.c_int, ip, ip, ip, dp],
            "dsx_grid_create": [C.POINTER(_GridDesc), C.POINTER(_FieldDesc), C.c_int, C.c_longlong,
                                C.c_longlong, C.POINTER(vp)],
            "dsx_grid_destroy": [vp],
            "dsx_grid_topology": [vp, C.c_int, ip, ip, dp],
            "dsx_grid_neighbors": [vp, C.c_int, ip, ip, dp],
            "dsx_grid_cuts": [vp, dp, vp],
            "dsx_grid_upload": [vp, llp, C.POINTER(vp), vp],
            "dsx_grid_counts": [vp, llp, llp, vp],
            "dsx_grid_download": [vp, llp, C.POINTER(vp), vp],
            "dsx_grid_totals": [vp, llp, vp],
            "dsx_grid_read": [vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, vp, vp],
            "dsx_grid_write": [vp, C.c_int, C.c_int, C.c_longlong, C.c_longlong, vp, vp],
            "dsx_grid_view_get": [vp, C.POINTER(GridView)],
            "dsx_grid_migrate": [vp, vp, llp],
            "dsx_grid_exchange_halo": [vp, C.c_int, C.c_int, vp, llp],
            "dsx_grid_reverse_halo": [vp, vp],
            "dsx_grid_reverse_exchange": [vp, C.c_int, ip, ip, vp],
            "dsx_grid_forward_exchange": [vp, C.c_int, ip, vp],
            "dsx_grid_rebalance": [vp, dp, C.c_int, vp, llp, dp],
            "dsx_grid_set_halo_width": [vp, C.c_double],
            "dsx_grid_invalidate_halo": [vp],
            "dsx_grid_halo_backward": [vp, vp, vp, vp, vp, vp, vp, vp],
            "dsx_grid_step": [vp, STEP_CALLBACK, vp, C.c_int, vp, C.POINTER(C.c_uint)],
            "dsx_grid_step_async": [vp, STEP_CALLBACK, vp, vp],
            "dsx_grid_step_wait": [vp, C.POINTER(C.c_uint)],
            "dsx_grid_step_kernel_count": [vp],
            "dsx_grid_profile": [vp, C.c_int],
            "dsx_grid_set_plain": [vp, C.c_int],
            "dsx_grid_set_tuning": [vp, C.c_int, C.c_int, C.c_int, C.c_int],
            "dsx_grid_set_cuts": [vp, C.POINTER(C.c_double), vp],
            "dsx_grid_owner_rank": [vp, vp, vp, vp, C.c_longlong, vp, vp],
            "dsx_grid_begin_halo_exchange": [vp, C.c_int, C.c_int, vp],
            "dsx_grid_set_split_share": [vp, C.c_int],
            "dsx_grid_set_refresh_kind": [vp, C.c_int],
            "dsx_grid_end_halo_exchange": [vp, vp, C.POINTER(C.c_longlong)],
            "dsx_grid_out_of_domain": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), vp],
            "dsx_grid_rescale_domain": [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, vp],
            "dsx_grid_autotune": [vp, vp, vp],
            "dsx_grid_migration_pairs": [vp, llp, vp],
            "dsx_grid_send_lists": [vp, ip, ip, vp],
            "dsx_grid_assemble": [vp, llp, C.c_int, C.POINTER(vp), C.c_longlong, vp, vp],
            "dsx_grid_set_rebalance_work": [vp, dp],
            "dsx_copy_segments": [vp, C.c_longlong, vp],
            "dsx_shard_create": [C.POINTER(_GridDesc), C.POINTER(_FieldDesc), C.c_int, C.c_longlong,
                                 C.c_longlong, C.c_int, C.c_int, ip, vp, C.POINTER(vp)],
            "dsx_shard_destroy": [vp],
            "dsx_shard_owners": [vp, ip],
            "dsx_shard_plan_owners": [ip, C.c_int, ip],
            "dsx_shard_upload": [vp, llp, C.POINTER(vp), vp],
            "dsx_shard_download": [vp, llp, C.POINTER(vp), vp],
            "dsx_shard_migrate": [vp, vp, llp],
            "dsx_shard_rebalance": [vp, dp, C.c_int, vp, llp, dp],
            "dsx_shard_exchange_halo": [vp, C.c_int, C.c_int, vp, llp],
            "dsx_shard_reverse_halo": [vp, vp],
            "dsx_shard_forward_exchange": [vp, C.c_int, ip, vp],
            "dsx_shard_reverse_exchange": [vp, C.c_int, ip, ip, vp],
            "dsx_shard_owned_view": [vp, C.POINTER(GridView)],
            "dsx_shard_ghost_view": [vp, C.POINTER(GridView)],
            "dsx_shard_counts": [vp, llp, llp, vp],
            "dsx_shard_launches": [vp, llp],
            "dsx_shard_totals": [vp, llp, vp],
            "dsx_grid_kernel_times": [vp, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_float)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _LIB = L
    return _LIB


# dsx_segment and dsx_copy as numpy record types (C layout, natural alignment)
SEGMENT_DTYPE = np.dtype([("source", np.int32), ("src_index", np.int64), ("dst_rank", np.int32),
                          ("dst_index", np.int64), ("count", np.int64)], align=True)
COPY_DTYPE = np.dtype([("src", np.uint64), ("dst", np.uint64), ("bytes", np.int64)], align=True)


def copy_segments(copies: np.ndarray, stream=None):
    """Device-to-device copies (a COPY_DTYPE array), all in one kernel."""
    c = np.ascontiguousarray(copies, dtype=COPY_DTYPE)
    if c.size:
        _check(lib().dsx_copy_segments(c.ctypes.data, c.size, _stream(stream)))


def _trampoline(callback, owner):
    """A step callback for the C ABI: callback(view, stream).  An exception
    cannot cross the C frames, so it is kept on `owner` and raised by the
    Python call that ran the step (_raise_callback_error)."""
    def trampoline(user, s, view_ptr):
        try:
            callback(view_ptr.contents, s or 0)   # the default stream arrives as None
        except BaseException as exc:
            if getattr(owner, "_callback_error", None) is None:
                owner._callback_error = exc
    return trampoline


def _raise_callback_error(owner):
    exc = getattr(owner, "_callback_error", None)
    if exc is not None:
        owner._callback_error = None
        raise RuntimeError(f"the step callback raised {type(exc).__name__}: {exc}") from exc


def _check(status: int):
    if status != DSX_OK:
        msg = lib().dsx_last_error().decode()
        raise ERRORS.get(status, DsxError)(msg)


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def rank_migrate(x, y, z, owned: int, lower, upper, periodic=(True, True, True), stream=None):
    """Single-rank drop-in migrate on device arrays (torch tensors or raw
    device pointers): wraps positions into the periodic box in place and
    returns the MigrationResult fields as a dict."""
    dom = _Domain((C.c_double * 3)(*lower), (C.c_double * 3)(*upper),
                  (C.c_int * 3)(*[1 if p else 0 for p in periodic]))
    res = _MigrationResult()
    ptr = lambda t: t if isinstance(t, int) else t.data_ptr()
    _check(lib().dsx_rank_migrate(ptr(x), ptr(y), ptr(z), owned, C.byref(dom), _stream(stream),
                                  C.byref(res)))
    return {k: getattr(res, k) for k, _ in _MigrationResult._fields_}


def _grid_desc(nranks, dims, policy, lower, upper, periodic, halo_width, edges_and_corners,
               dynamic) -> _GridDesc:
    dyn = dynamic if dynamic is not None else (1.0, 1.10, 0.5, 0.10)
    return _GridDesc(nranks, (C.c_int * 3)(*dims), POLICIES[policy], (C.c_double * 3)(*lower),
                     (C.c_double * 3)(*upper), (C.c_int * 3)(*[1 if p else 0 for p in periodic]),
                     float(halo_width), 1 if edges_and_corners else 0, *[float(v) for v in dyn])


def plan_topology(nranks: int, rank: int, dims=(0, 0, 0), policy: str = "manual",
                  lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), periodic=(True, True, True),
                  edges_and_corners: bool = True):
    """Host-only topology of one virtual rank: (dims, neighbor list)."""
    d = _grid_desc(nranks, dims, policy, lower, upper, periodic, 0.0, edges_and_corners, None)
    out_dims = (C.c_int * 3)()
    count = C.c_int()
    info = (C.c_int * (26 * 5))()
    shifts = (C.c_double * (26 * 3))()
    _check(lib().dsx_plan_topology(C.byref(d), rank, out_dims, C.byref(count), info, shifts))
    return tuple(out_dims), [dict(rank=info[5 * n], direction=tuple(info[5 * n + 1:5 * n + 4]),
                                  slot=info[5 * n + 4], shift=tuple(shifts[3 * n:3 * n + 3]))
                             for n in range(count.value)]


class VirtualGrid:
    """P subdomains of one box on one GPU (the reference's P MPI ranks).

    ``fields`` lists ``(name, type, components)`` with ``type`` a key of
    :data:`FIELD_TYPES` or its index.
    """

    def __init__(self, nranks: int, dims=(0, 0, 0), policy: str = "manual",
                 lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), periodic=(True, True, True),
                 halo_width: float = 0.0, edges_and_corners: bool = True,
                 dynamic: Optional[Tuple[float, float, float, float]] = None,
                 fields: Sequence[Tuple[str, object, int]] = (), particles: int = 0,
                 ghost_capacity: int = 0):
        self.L = lib()
        d = _grid_desc(nranks, dims, policy, lower, upper, periodic, halo_width,
                       edges_and_corners, dynamic)
        self.fields = []
        for name, t, comps in fields:
            t = FIELD_TYPES[t] if isinstance(t, str) else int(t)
            self.fields.append((str(name), t, int(comps)))
        self.field_index = {n: i for i, (n, _, _) in enumerate(self.fields)}
        self._names = [n.encode() for n, _, _ in self.fields]
        fd = (_FieldDesc * max(len(self.fields), 1))(
            *[_FieldDesc(self._names[i], t, c) for i, (_, t, c) in enumerate(self.fields)])
        h = C.c_void_p()
        _check(self.L.dsx_grid_create(C.byref(d), fd, len(self.fields), int(particles),
                                      int(ghost_capacity), C.byref(h)))
        self.h = h
        self.nranks = nranks
        self.particles = int(particles)
        self._callbacks = []

    def close(self):
        if getattr(self, "h", None):
            self.L.dsx_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------- metadata
    def dtype_of(self, name: str):
        if name in ARRAYS:
            return CORE_DTYPES[ARRAYS.index(name)]
        return FIELD_DTYPES[self.fields[self.field_index[name]][1]]

    def components(self, name: str) -> int:
        return 1 if name in ARRAYS else self.fields[self.field_index[name]][2]

    def array_id(self, name: str) -> int:
        return ARRAYS.index(name) if name in ARRAYS else 13 + self.field_index[name]

    def topology(self, rank: int):
        dims = (C.c_int * 3)()
        coords = (C.c_int * 3)()
        local = (C.c_double * 6)()
        _check(self.L.dsx_grid_topology(self.h, rank, dims, coords, local))
        return tuple(dims), tuple(coords), (tuple(local[:3]), tuple(local[3:]))

    def neighbors(self, rank: int):
        count = C.c_int()
        info = (C.c_int * (26 * 5))()
        shifts = (C.c_double * (26 * 3))()
        _check(self.L.dsx_grid_neighbors(self.h, rank, C.byref(count), info, shifts))
        return [dict(rank=info[5 * n], direction=tuple(info[5 * n + 1:5 * n + 4]),
                     slot=info[5 * n + 4], shift=tuple(shifts[3 * n:3 * n + 3]))
                for n in range(count.value)]

    def cuts(self, stream=None):
        dims = self.topology(0)[0]
        out = (C.c_double * (sum(dims) + 3))()
        _check(self.L.dsx_grid_cuts(self.h, out, _stream(stream)))
        flat, res, k = list(out), [], 0
        for dd in dims:
            res.append(np.array(flat[k:k + dd + 1]))
            k += dd + 1
        return res

    # -------------------------------------------------------- particles
    def upload(self, per_rank: List[Dict[str, np.ndarray]], stream=None):
        """per_rank[r]: dict of host arrays of rank r's owned particles."""
        counts = np.array([len(d["x"]) for d in per_rank], dtype=np.int64)
        keep = []
        ptrs = (C.c_void_p * (13 + len(self.fields)))()
        for a, name in enumerate(ARRAYS):
            if all(name in d for d in per_rank):
                arr = np.ascontiguousarray(np.concatenate([np.asarray(d[name]) for d in per_rank]),
                                           dtype=CORE_DTYPES[a])
                keep.append(arr)
                ptrs[a] = arr.ctypes.data
        for f, (name, t, c) in enumerate(self.fields):
            if all(name in d for d in per_rank):
                arr = np.ascontiguousarray(
                    np.concatenate([np.asarray(d[name]).reshape(-1) for d in per_rank]),
                    dtype=FIELD_DTYPES[t])
                keep.append(arr)
                ptrs[13 + f] = arr.ctypes.data
        _check(self.L.dsx_grid_upload(self.h, counts.ctypes.data_as(C.POINTER(C.c_longlong)), ptrs,
                                      _stream(stream)))

    def upload_flat(self, counts, arrays: List[Optional[int]], stream=None):
        """Upload from raw host/device pointers (arrays[13 + nfields], None
        entries zero-filled), owned particles concatenated in rank order."""
        c = np.ascontiguousarray(counts, dtype=np.int64)
        ptrs = (C.c_void_p * (13 + len(self.fields)))(*[a or None for a in arrays])
        _check(self.L.dsx_grid_upload(self.h, c.ctypes.data_as(C.POINTER(C.c_longlong)), ptrs,
                                      _stream(stream)))

    def download_flat(self, arrays: List[Optional[int]], stream=None) -> np.ndarray:
        """Inverse of upload_flat; returns the per-rank owned counts."""
        c = np.zeros(self.nranks, dtype=np.int64)
        ptrs = (C.c_void_p * (13 + len(self.fields)))(*[a or None for a in arrays])
        _check(self.L.dsx_grid_download(self.h, c.ctypes.data_as(C.POINTER(C.c_longlong)), ptrs,
                                        _stream(stream)))
        return c

    def totals(self, stream=None) -> Dict[str, int]:
        out = np.zeros(4, dtype=np.int64)
        _check(self.L.dsx_grid_totals(self.h, out.ctypes.data_as(C.POINTER(C.c_longlong)),
                                      _stream(stream)))
        return dict(particles=int(out[0]), emigrants=int(out[1]), ghosts=int(out[2]),
                    boundary=int(out[3]))

    def all_counts(self, stream=None):
        o = np.zeros(self.nranks, dtype=np.int64)
        g = np.zeros(self.nranks, dtype=np.int64)
        _check(self.L.dsx_grid_counts(self.h, o.ctypes.data_as(C.POINTER(C.c_longlong)),
                                      g.ctypes.data_as(C.POINTER(C.c_longlong)), _stream(stream)))
        return o, g

    def counts(self, rank: int, stream=None) -> Tuple[int, int]:
        o, g = self.all_counts(stream)
        return int(o[rank]), int(g[rank])

    def read(self, rank: int, name: str, start: int = 0, count: Optional[int] = None, stream=None):
        owned, ghosts = self.counts(rank, stream)
        if count is None:
            count = owned + ghosts - start
        comps = self.components(name)
        out = np.zeros(count * comps, dtype=self.dtype_of(name))
        _check(self.L.dsx_grid_read(self.h, rank, self.array_id(name), start, count,
                                    out.ctypes.data, _stream(stream)))
        return out.reshape(count, comps) if comps > 1 else out

    def write(self, rank: int, name: str, start: int, values, stream=None):
        comps = self.components(name)
        arr = np.ascontiguousarray(values, dtype=self.dtype_of(name)).reshape(-1)
        _check(self.L.dsx_grid_write(self.h, rank, self.array_id(name), start, arr.size // comps,
                                     arr.ctypes.data, _stream(stream)))

    def snapshot(self, rank: int, stream=None) -> Dict[str, np.ndarray]:
        out = {name: self.read(rank, name, stream=stream) for name in ARRAYS}
        for name, _, _ in self.fields:
            out[name] = self.read(rank, name, stream=stream)
        out["owned"], out["ghosts"] = self.counts(rank, stream)
        return out

    def view(self) -> GridView:
        v = GridView()
        _check(self.L.dsx_grid_view_get(self.h, C.byref(v)))
        return v

    # ------------------------------------------------------- operations
    def migrate(self, stream=None, results: bool = True):
        res = np.zeros((self.nranks, 6), dtype=np.int64) if results else None
        _check(self.L.dsx_grid_migrate(self.h, _stream(stream),
                                       None if res is None else res.ctypes.data_as(C.POINTER(C.c_longlong))))
        return res

    def exchange_halo(self, rebuild: bool = False, positions_only: bool = False, stream=None,
                      results: bool = True):
        res = np.zeros((self.nranks, 4), dtype=np.int64) if results else None
        _check(self.L.dsx_grid_exchange_halo(
            self.h, 1 if rebuild else 0, 1 if positions_only else 0, _stream(stream),
            None if res is None else res.ctypes.data_as(C.POINTER(C.c_longlong))))
        return res

    def reverse_halo(self, stream=None):
        _check(self.L.dsx_grid_reverse_halo(self.h, _stream(stream)))

    def reverse_exchange(self, fields: List[Tuple[str, str]], stream=None):
        n = len(fields)
        ids = (C.c_int * max(n, 1))(*[self.field_index[f] if f in self.field_index else -1
                                      for f, _ in fields])
        ops = (C.c_int * max(n, 1))(*[OPS[o] for _, o in fields])
        _check(self.L.dsx_grid_reverse_exchange(self.h, n, ids, ops, _stream(stream)))

    def forward_exchange(self, names: List[str], stream=None):
        n = len(names)
        ids = (C.c_int * max(n, 1))(*[self.field_index.get(f, -1) for f in names])
        _check(self.L.dsx_grid_forward_exchange(self.h, n, ids, _stream(stream)))

    def rebalance(self, work=None, force: bool = False, stream=None):
        res = np.zeros((self.nranks, 3), dtype=np.int64)
        imb = np.zeros(self.nranks, dtype=np.float64)
        w = None if work is None else np.ascontiguousarray(work, dtype=np.float64)
        _check(self.L.dsx_grid_rebalance(
            self.h, None if w is None else w.ctypes.data_as(C.POINTER(C.c_double)),
            1 if force else 0, _stream(stream), res.ctypes.data_as(C.POINTER(C.c_longlong)),
            imb.ctypes.data_as(C.POINTER(C.c_double))))
        return res, imb

    def set_halo_width(self, width: float):
        _check(self.L.dsx_grid_set_halo_width(self.h, float(width)))

    def invalidate_halo(self):
        _check(self.L.dsx_grid_invalidate_halo(self.h))

    def halo_backward(self, ghost_cot, owner_grad, stream=None):
        """owner_grad[:, i] += sum of ghost_cot[:, slot] over the ghost images
        of owned particle i (device tensors of shape (3, n))."""
        _check(self.L.dsx_grid_halo_backward(
            self.h, ghost_cot[0].data_ptr(), ghost_cot[1].data_ptr(), ghost_cot[2].data_ptr(),
            owner_grad[0].data_ptr(), owner_grad[1].data_ptr(), owner_grad[2].data_ptr(),
            _stream(stream)))

    def _step_callback(self, callback):
        # one C function pointer per Python callback: the engine keeps its
        # captured graphs only while the callback pointer stays the same
        cache = self.__dict__.setdefault("_cb_cache", {})
        key = id(callback)
        if key not in cache:
            if callback is None:
                cache[key] = (None, STEP_CALLBACK())
            else:
                cache[key] = (callback, STEP_CALLBACK(_trampoline(callback, self)))
        return cache[key][1]

    def step_async(self, callback=None, stream=None) -> None:
        """Queues one captured batched step (dsx_grid_step_async) and returns:
        the previous queued step's build is checked (and an overflow redone)
        before this one is queued.  step_wait() completes the queue."""
        cb = self._step_callback(callback)
        self._callback_error = None
        status = self.L.dsx_grid_step_async(self.h, cb, None, _stream(stream))
        _raise_callback_error(self)
        _check(status)

    def step_wait(self) -> int:
        """Completes the queued steps; the OR of their status bits."""
        st = C.c_uint()
        self._callback_error = None
        status = self.L.dsx_grid_step_wait(self.h, C.byref(st))
        _raise_callback_error(self)
        _check(status)
        return st.value

    def step(self, callback=None, capture: bool = False, stream=None) -> int:
        """One batched step: migrate -> halo build -> callback(view, stream)
        -> reverse_halo.  Returns the device status bits (0 == ok)."""
        cb = self._step_callback(callback)
        st = C.c_uint()
        self._callback_error = None
        status = self.L.dsx_grid_step(self.h, cb, None, 1 if capture else 0, _stream(stream),
                                      C.byref(st))
        _raise_callback_error(self)
        _check(status)
        return st.value

    def autotune(self, stream=None) -> Dict[str, object]:
        """Times the batched step's launch-shape candidates on the current
        particles, keeps the fastest and sizes the ghost region; returns the
        choices and the measured milliseconds per launch."""
        r = TuneReport()
        _check(self.L.dsx_grid_autotune(self.h, _stream(stream), C.byref(r)))
        kinds = MOVE_KINDS
        return {"classify_threads": r.classify_threads,
                "classify_combine": bool(r.classify_combine),
                "move": kinds.get(r.move_staged, "?"),
                "reverse_ctas_per_sm": r.reverse_ctas_per_sm,
                "ghost_capacity": int(r.ghost_capacity),
                "classify_ms": {n: round(float(v), 4) for n, v in zip((64, 128, 256), r.classify_ms)},
                "classify_combined_ms": {n: round(float(v), 4)
                                         for n, v in zip((64, 128, 256), r.classify_combined_ms)},
                "move_ms": {"staged": round(float(r.move_ms[0]), 4),
                            "direct": round(float(r.move_ms[1]), 4),
                            "staged passes": round(float(r.move_ms[2]), 4),
                            "staged direct forces": round(float(r.move_ms[3]), 4)},
                "reverse_ms": {n: round(float(v), 4) for n, v in zip((4, 8, 16, 32), r.reverse_ms)}}

    def begin_halo_exchange(self, rebuild: bool = False, positions_only: bool = False, stream=None):
        """Enqueues the halo refresh or build and returns at once."""
        _check(self.L.dsx_grid_begin_halo_exchange(self.h, 1 if rebuild else 0,
                                                   1 if positions_only else 0, _stream(stream)))

    def end_halo_exchange(self, stream=None):
        """Waits for the exchange begun before; results as exchange_halo's."""
        res = np.zeros((self.nranks, 4), dtype=np.int64)
        _check(self.L.dsx_grid_end_halo_exchange(self.h, _stream(stream),
                                                 res.ctypes.data_as(C.POINTER(C.c_longlong))))
        return res

    REFRESH_KINDS = {"ghosts": 0, "owners": 1, "tiles": 2, "auto": 3}

    def set_refresh_kind(self, kind="auto"):
        """Refresh walk: "ghosts" (each ghost's owner gathered), "owners"
        (each boundary owner once), "tiles" (each tile's owners staged whole)
        or "auto" (the default: tiles for a full refresh of nine arrays or
        more, else ghosts); True / False stand for "owners" / "ghosts"."""
        if isinstance(kind, bool):
            kind = "owners" if kind else "ghosts"
        _check(self.L.dsx_grid_set_refresh_kind(self.h, self.REFRESH_KINDS[kind]))

    def set_split_share(self, ctas_per_sm: int = 0):
        """CTAs per SM the split-phase refresh may occupy (0: all resident)."""
        _check(self.L.dsx_grid_set_split_share(self.h, int(ctas_per_sm)))

    def owner_rank(self, x, y, z, out, n: Optional[int] = None, stream=None):
        """Owning subdomain of n device positions into the int32 device array
        `out`: torch tensors (n defaults to their common length, which every
        one must have), or raw device addresses with n given."""
        arrays = (x, y, z, out)
        if all(isinstance(t, int) for t in arrays):
            if n is None:
                raise ValueError("owner_rank on raw addresses needs the particle count n")
            ptrs = arrays
        elif any(isinstance(t, int) for t in arrays):
            raise ValueError("owner_rank takes four tensors or four addresses")
        else:
            sizes = {int(t.numel()) for t in arrays}
            if len(sizes) != 1 or (n is not None and n > min(sizes)):
                raise ValueError("owner_rank: x, y, z and out must hold n elements each")
            n = min(sizes) if n is None else n
            if x.dtype != y.dtype or str(x.dtype) != "torch.float64" or str(out.dtype) != "torch.int32":
                raise ValueError("owner_rank: float64 positions, int32 out")
            ptrs = tuple(t.data_ptr() for t in arrays)
        _check(self.L.dsx_grid_owner_rank(self.h, ptrs[0], ptrs[1], ptrs[2], int(n), ptrs[3],
                                          _stream(stream)))

    def out_of_domain(self, stream=None):
        """(per-subdomain flags, any): owned particles that belong elsewhere."""
        flags = np.zeros(self.nranks, dtype=np.int32)
        anyv = C.c_int()
        _check(self.L.dsx_grid_out_of_domain(self.h, flags.ctypes.data_as(C.POINTER(C.c_int)),
                                             C.byref(anyv), _stream(stream)))
        return flags, bool(anyv.value)

    def set_cuts(self, cuts: Sequence[Sequence[float]], stream=None):
        """Replaces the cut planes (three increasing arrays spanning the box,
        dims[a] + 1 values each); the halo plan becomes invalid."""
        flat = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float64) for c in cuts]))
        _check(self.L.dsx_grid_set_cuts(self.h, flat.ctypes.data_as(C.POINTER(C.c_double)),
                                        _stream(stream)))

    def rescale_domain(self, lower, upper, update: bool = False, stream=None):
        """New box: cut planes keep their fractions, periodic shifts follow.
        update=False (Decomp::rescale_domain) keeps the halo plan;
        update=True (Decomp::update_domain) invalidates it."""
        lo = (C.c_double * 3)(*lower)
        hi = (C.c_double * 3)(*upper)
        _check(self.L.dsx_grid_rescale_domain(self.h, lo, hi, 1 if update else 0, _stream(stream)))

    def set_tuning(self, classify_threads: int = 128, move: str = "staged",
                   reverse_ctas_per_sm: int = 0, classify_combine: bool = False):
        """Sets the batched step's launch shapes (the choices autotune reports)."""
        kind = {v: k for k, v in MOVE_KINDS.items()}[move]
        _check(self.L.dsx_grid_set_tuning(self.h, classify_threads, kind, reverse_ctas_per_sm,
                                          1 if classify_combine else 0))

    # ----------------------------------------------- sharded grids
    def migration_pairs(self, stream=None) -> np.ndarray:
        """Emigrants of the last migration per (destination, source): (P, P)."""
        out = np.zeros((self.nranks, self.nranks), dtype=np.int64)
        _check(self.L.dsx_grid_migration_pairs(self.h, out.ctypes.data_as(C.POINTER(C.c_longlong)),
                                               _stream(stream)))
        return out

    def send_lists(self, stream=None):
        """(length, first ghost slot) of every send list, 26 per sender."""
        n = self.nranks * 26
        length = np.zeros(n, dtype=np.int32)
        first = np.zeros(n, dtype=np.int32)
        _check(self.L.dsx_grid_send_lists(self.h, length.ctypes.data_as(C.POINTER(C.c_int)),
                                          first.ctypes.data_as(C.POINTER(C.c_int)), _stream(stream)))
        return length.astype(np.int64), first.astype(np.int64)

    def assemble(self, counts, sources: Sequence[Sequence[int]], segments: np.ndarray, stream=None):
        """New owned particles from segments (a SEGMENT_DTYPE array) of the
        current ones (source -1) and of device buffers: sources[k][a] is the
        address of array a's element 0 in buffer k."""
        c = np.ascontiguousarray(counts, dtype=np.int64)
        table = (C.c_void_p * max(32 * len(sources), 1))()
        for k, ptrs in enumerate(sources):
            for a, p in enumerate(ptrs):
                table[32 * k + a] = p
        seg = np.ascontiguousarray(segments, dtype=SEGMENT_DTYPE)
        _check(self.L.dsx_grid_assemble(self.h, c.ctypes.data_as(C.POINTER(C.c_longlong)),
                                        len(sources), table, seg.size,
                                        seg.ctypes.data if seg.size else None, _stream(stream)))

    def set_rebalance_work(self, work=None):
        """Work per subdomain for the next migrate's automatic rebalance."""
        if work is None:
            _check(self.L.dsx_grid_set_rebalance_work(self.h, None))
            return
        w = np.ascontiguousarray(work, dtype=np.float64)
        _check(self.L.dsx_grid_set_rebalance_work(self.h, w.ctypes.data_as(C.POINTER(C.c_double))))

    def set_plain(self, plain: bool = True):
        """Per-call operations launch their tile kernels once per subdomain
        (comparison runs; results are unchanged)."""
        _check(self.L.dsx_grid_set_plain(self.h, 1 if plain else 0))

    def profile(self, enable: bool = True):
        _check(self.L.dsx_grid_profile(self.h, 1 if enable else 0))

    def kernel_times(self) -> List[Tuple[str, float]]:
        """(name, ms) of every kernel interval of the last profiled step."""
        names = (C.c_char_p * 64)()
        ms = (C.c_float * 64)()
        n = self.L.dsx_grid_kernel_times(self.h, 64, names, ms)
        if n < 0:
            _check(n)
        return [(names[i].decode(), float(ms[i])) for i in range(n)]

    def step_kernel_count(self) -> int:
        return self.L.dsx_grid_step_kernel_count(self.h)
