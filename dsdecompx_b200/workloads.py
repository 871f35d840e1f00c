"""Seeded synthetic workloads with the shapes of the benchmark configurations.

There is no public dataset behind these runs: each configuration fixes the
box, process grid, halo width, particle count and value distributions, and
the particles are drawn here with numpy's PCG64 generator from a fixed seed.
The per-step drift and ghost forces are drawn on the device by the harness
kernels of ``workload/workload.cu`` (counter-based, keyed by particle id).

The module needs only numpy until :func:`harness` is called, so a CPU-only
caller (the reference timing in ``bench.py``) can load it from its file
without importing the package or its native library.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np


@dataclass
class Workload:
    name: str
    nranks: int
    dims: Tuple[int, int, int]
    policy: str
    upper: Tuple[float, float, float]
    particles: int
    halo: float
    drift: float
    fields: List[Tuple[str, str, int]] = field(default_factory=list)
    blobs: int = 0               # Gaussian blobs (clustered configuration)
    blob_sigma: float = 0.0
    blob_fraction: float = 0.0
    field_exchange: bool = False  # forward/reverse_exchange of the fields each step
    description: str = ""

    @property
    def lower(self):
        return (0.0, 0.0, 0.0)

    def record_bytes(self) -> int:
        sizes = {"int32": 4, "int64": 8, "uint32": 4, "uint64": 8, "float32": 4, "float64": 8}
        return 96 + sum(sizes[t] * c for _, t, c in self.fields)


WORKLOADS: Dict[str, Workload] = {
    "drop_in_1rank": Workload(
        "drop_in_1rank", 1, (1, 1, 1), "manual", (100.0, 100.0, 100.0), 1_000_000, 2.8, 0.1,
        description="1 rank, periodic cube L=100, 1M uniform particles, halo 2.8, N(0,0.1) drift"),
    "virtual_2x2x2": Workload(
        "virtual_2x2x2", 8, (2, 2, 2), "manual", (200.0, 200.0, 200.0), 8_000_000, 2.8, 0.5,
        fields=[("charge", "float64", 1), ("vec", "float32", 3)], field_exchange=True,
        description="2x2x2 virtual grid, L=200, 8M uniform particles, halo 2.8, f64 + f32x3 "
                    "fields with forward/reverse_exchange, N(0,0.5) drift"),
    "clustered_64": Workload(
        "clustered_64", 64, (0, 0, 0), "dynamic", (256.0, 256.0, 256.0), 16_000_000, 2.8, 0.1,
        fields=[("id64", "int64", 1)], blobs=32, blob_sigma=8.0, blob_fraction=0.8,
        description="4x4x4 virtual grid with Dynamic boundaries, L=256, 16M particles (80% in 32 "
                    "Gaussian blobs sigma=8, 20% uniform), halo 2.8, int64 ids, N(0,0.1) drift"),
    "large_256": Workload(
        "large_256", 256, (8, 8, 4), "manual", (400.0, 400.0, 200.0), 27_200_000, 2.8, 0.05,
        fields=[("energy", "float64", 1), ("pressure", "float64", 1), ("dipole", "float64", 3),
                ("species", "int32", 1), ("id64", "int64", 1)],
        description="8x8x4 virtual grid, box 400x400x200 at density 0.85 (27.2M particles), "
                    "halo 2.8, fields 2x f64, f64x3, int32 type 0..7, int64 ids, N(0,0.05) drift"),
}


def generate(w: Workload, seed: int = 2024, particles: int = 0) -> Dict[str, np.ndarray]:
    """Host arrays of the workload's particles (positions inside the box)."""
    n = particles or w.particles
    rng = np.random.default_rng(seed)
    lower, upper = np.asarray(w.lower), np.asarray(w.upper)
    extent = upper - lower
    pos = rng.uniform(lower, upper, size=(n, 3))
    if w.blobs:
        k = int(w.blob_fraction * n)
        centres = rng.uniform(lower, upper, size=(w.blobs, 3))
        pick = rng.integers(0, w.blobs, k)
        blob = centres[pick] + rng.normal(0.0, w.blob_sigma, size=(k, 3))
        pos[:k] = lower + np.mod(blob - lower, extent)
        pos = pos[rng.permutation(n)]
    d = dict(x=np.ascontiguousarray(pos[:, 0]), y=np.ascontiguousarray(pos[:, 1]),
             z=np.ascontiguousarray(pos[:, 2]))
    d["vx"], d["vy"], d["vz"] = (rng.normal(size=n) for _ in range(3))
    d["mass"] = np.ones(n)
    d["global_id"] = np.arange(n, dtype=np.int32)
    for name, t, c in w.fields:
        if name == "id64":
            d[name] = np.arange(n, dtype=np.int64)
        elif name == "charge":
            d[name] = rng.uniform(-1.0, 1.0, n)
        elif name == "species":
            d[name] = rng.integers(0, 8, n).astype(np.int32)
        elif t == "float32":
            d[name] = rng.normal(size=(n, c)).astype(np.float32)
        else:
            d[name] = rng.normal(size=(n, c)) if c > 1 else rng.normal(size=n)
    return d


def initial_owner(w: Workload, dims, x, y, z) -> np.ndarray:
    """Owner under uniform cuts (the grid's initial geometry)."""
    c = []
    for a, v in enumerate((x, y, z)):
        rel = (v - w.lower[a]) / (w.upper[a] - w.lower[a]) * dims[a]
        c.append(np.clip(np.floor(rel).astype(np.int64), 0, dims[a] - 1))
    return ((c[0] * dims[1] + c[1]) * dims[2] + c[2]).astype(np.int64)


def group_by_owner(data: Dict[str, np.ndarray], owner: np.ndarray, nranks: int):
    """(counts, arrays) with the particles of each rank contiguous, in rank order."""
    order = np.argsort(owner, kind="stable")
    counts = np.bincount(owner, minlength=nranks).astype(np.int64)
    return counts, {k: np.ascontiguousarray(v[order]) for k, v in data.items()}


_WL = None


def harness() -> C.CDLL:
    """The synthetic drift / ghost-force kernels."""
    global _WL
    if _WL is None:
        from . import _build
        path = _build.WORKLOAD_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build()")
        _WL = C.CDLL(path)
        _WL.dsxw_drift.argtypes = [C.c_void_p, C.c_ulonglong, C.c_longlong, C.c_double, C.c_void_p]
        _WL.dsxw_ghost_forces.argtypes = [C.c_void_p, C.c_ulonglong, C.c_longlong, C.c_void_p]
        _WL.dsxw_advance.argtypes = [C.c_void_p]
        _WL.dsxw_set_step.argtypes = [C.c_ulonglong, C.c_void_p]
        _WL.dsxw_interior.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        _WL.dsxw_step_work.argtypes = [C.c_void_p, C.c_ulonglong, C.c_double, C.c_void_p]
        _WL.dsxw_drift_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_longlong, C.c_ulonglong, C.c_longlong, C.c_double,
                                          C.c_void_p]
    return _WL
