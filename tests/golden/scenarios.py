"""Golden scenarios: seeded inputs, the calls made, and a SHA-1 digest of
every array of every subdomain after each call (and of every input drawn).
``make_golden.py`` records them from the reference's own Host path
(oracle/_ref, built from the reference sources) into <scenario>.json; the
tests regenerate the same inputs from the stored seed (their digests must
match too), replay the calls on the C restatement (CPU) and on the CUDA grid
(GPU) and compare every digest, i.e. bit for bit.  Test infrastructure only."""
from __future__ import annotations

import hashlib

import numpy as np

FIELD_TYPE_NAMES = ["int32", "int64", "uint32", "uint64", "float32", "float64"]
ARRAYS = ["x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "mass", "charge", "type",
          "global_id"]

FIELDS_A = [("q", "float64", 1), ("vec3f", "float32", 3), ("tag", "int32", 1), ("big", "int64", 2)]
FIELDS_B = [("u", "uint32", 1), ("uu", "uint64", 1), ("wide", "float64", 5)]

SCENARIOS = {
    "single_rank": dict(P=1, dims=(1, 1, 1), policy="manual", lower=(0.0, 0.0, 0.0),
                        upper=(8.0, 8.0, 8.0), periodic=(True, True, True), halo=1.0, edges=True,
                        dynamic=None, fields=FIELDS_A[:2], N=600, steps=2, sigma=2.5),
    "grid_2x2x2": dict(P=8, dims=(2, 2, 2), policy="manual", lower=(0.0, 0.0, 0.0),
                       upper=(10.0, 10.0, 10.0), periodic=(True, True, True), halo=1.0,
                       edges=True, dynamic=None, fields=FIELDS_A, N=1600, steps=2, sigma=0.4),
    "grid_3x1x4_open_faces": dict(P=12, dims=(3, 1, 4), policy="manual", lower=(-4.5, 1.0, 100.0),
                                  upper=(4.5, 6.0, 112.0), periodic=(True, True, True), halo=0.8,
                                  edges=False, dynamic=None, fields=FIELDS_B, N=2000, steps=2,
                                  sigma=0.5),
    "dynamic_8": dict(P=8, dims=(0, 0, 0), policy="dynamic", lower=(0.0, 0.0, 0.0),
                      upper=(16.0, 16.0, 16.0), periodic=(True, True, True), halo=1.0, edges=True,
                      dynamic=(1.0, 1.01, 0.5, 0.1), fields=FIELDS_A[:1], N=2400, steps=3,
                      sigma=0.8, clustered=True),
}


def initial_particles(rng, spec):
    n = spec["N"]
    lo, hi = np.asarray(spec["lower"]), np.asarray(spec["upper"])
    pos = rng.uniform(lo, hi, size=(n, 3))
    if spec.get("clustered"):
        k = int(0.8 * n)
        centre = rng.uniform(lo, hi, size=(3, 3))
        pos[:k] = lo + np.mod(centre[rng.integers(0, 3, k)] + rng.normal(0, 1.2, (k, 3)) - lo, hi - lo)
    d = {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy()}
    for name in ("vx", "vy", "vz", "fx", "fy", "fz"):
        d[name] = rng.normal(size=n)
    d["mass"] = rng.uniform(0.5, 2.0, n)
    d["charge"] = rng.uniform(-1, 1, n)
    d["type"] = rng.integers(0, 8, n).astype(np.int32)
    d["global_id"] = rng.permutation(n).astype(np.int32)
    for name, t, c in spec["fields"]:
        d[name] = values(rng, t, c, n)
    return d


def values(rng, t, c, n):
    dtype = np.dtype(["int32", "int64", "uint32", "uint64", "float32", "float64"].index(t) and
                     {"int32": np.int32, "int64": np.int64, "uint32": np.uint32,
                      "uint64": np.uint64, "float32": np.float32, "float64": np.float64}[t]
                     or np.int32)
    if t.startswith("float"):
        v = rng.normal(size=(n, c))
    elif t.startswith("uint"):
        v = rng.integers(0, 1 << 30, size=(n, c))
    else:
        v = rng.integers(-(1 << 30), 1 << 30, size=(n, c))
    v = v.astype(dtype)
    return v.reshape(n) if c == 1 else v


def digest(a) -> str:
    a = np.ascontiguousarray(a)
    h = hashlib.sha1()
    h.update(f"{a.dtype.str}{a.shape}".encode())
    h.update(a.tobytes())
    return h.hexdigest()


def run(grid, spec, record=None, replay=None, seed=0):
    """Drives `grid` (an oracle.Grid or a dsdecompx_b200.VirtualGrid) through
    the scenario, drawing its inputs from `seed`; `record` (if given) gets the
    digest of every input.  Returns the digests of the outputs (every snapshot
    and call result)."""
    rng = np.random.default_rng(seed)
    P = spec["P"]
    out = {}
    names = [f[0] for f in spec["fields"]]

    def take(key, make):
        v = make()
        if record is not None:
            record[key] = digest(v)
        return v

    def snap(tag):
        for r in range(P):
            s = grid.snapshot(r)
            out[f"{tag}/r{r}/counts"] = digest(np.array([s["owned"], s["ghosts"]], dtype=np.int64))
            for k in ARRAYS + names:
                out[f"{tag}/r{r}/{k}"] = digest(np.asarray(s[k]))

    init = initial_particles(rng, spec)
    if record is not None:
        for k, v in init.items():
            record[f"in/init/{k}"] = digest(v)
    owner = grid.owner_rank(np.stack([init["x"], init["y"], init["z"]], 1))
    per = [{k: v[owner == r] for k, v in init.items()} for r in range(P)]
    grid.upload(per) if hasattr(grid, "upload") else [grid.set_owned(r, d) for r, d in enumerate(per)]
    snap("upload")
    ops = ["sum", "min", "max", "replace"]
    for step in range(spec["steps"]):
        for r in range(P):
            o, _ = grid.counts(r)
            d = take(f"in/s{step}/move/r{r}", lambda: rng.normal(0.0, spec["sigma"], size=(o, 3)))
            for a, name in enumerate("xyz"):
                grid.write(r, name, 0, grid.read(r, name, 0, o) + d[:, a])
        out[f"s{step}/migrate/result"] = digest(np.asarray(grid.migrate(), dtype=np.int64))
        snap(f"s{step}/migrate")
        out[f"s{step}/cuts"] = digest(np.concatenate(grid.cuts()))
        out[f"s{step}/halo/result"] = digest(np.asarray(grid.exchange_halo(rebuild=step % 2 == 0)[:, :2], dtype=np.int64))
        snap(f"s{step}/halo")
        for r in range(P):
            o, g = grid.counts(r)
            f = take(f"in/s{step}/ghostf/r{r}", lambda: rng.normal(size=(g, 3)))
            for a, name in enumerate(("fx", "fy", "fz")):
                grid.write(r, name, o, f[:, a])
            for fname, t, c in spec["fields"]:
                v = take(f"in/s{step}/ghost_{fname}/r{r}", lambda: values(rng, t, c, g))
                grid.write(r, fname, o, v)
        grid.reverse_halo()
        snap(f"s{step}/reverse_halo")
        if names:
            grid.reverse_exchange([(n, ops[(i + step) % 4]) for i, n in enumerate(names)])
            snap(f"s{step}/reverse_exchange")
        for r in range(P):
            o, _ = grid.counts(r)
            d = take(f"in/s{step}/nudge/r{r}", lambda: rng.normal(0.0, 0.05, size=(o, 3)))
            for a, name in enumerate("xyz"):
                grid.write(r, name, 0, grid.read(r, name, 0, o) + d[:, a])
        out[f"s{step}/refresh/result"] = digest(np.asarray(grid.exchange_halo(rebuild=False)[:, :2], dtype=np.int64))
        snap(f"s{step}/refresh")
    return out


def make_oracle(kind, spec):
    import oracle
    return oracle.Grid(kind, spec["P"], spec["dims"], spec["policy"], spec["lower"], spec["upper"],
                       spec["periodic"], spec["halo"], spec["edges"], spec["dynamic"],
                       [(n, FIELD_TYPE_NAMES.index(t), c) for n, t, c in spec["fields"]],
                       field_capacity=6 * spec["N"] + 64)
