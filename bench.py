#!/usr/bin/env python
"""Throughput of the particle-bookkeeping step on B200.

One step = migrate (with the Dynamic rebalance when the workload has it) ->
exchange_halo (plan build) -> the synthetic "user" work (ghost forces N(0,1),
field exchanges when the workload names them, the next N(0,sigma) drift) ->
reverse_halo, run as the batched, CUDA-graph-captured step of the virtual grid
(dsx_grid_step).  Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                  [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): the sharded virtual grid.  The
global grid is N copies of the workload's block (the box and the particle
count grow with N: weak scaling); each rank owns one block of subdomains and
every step exchanges migrants, ghost lists and ghost forces with the ranks
that own the neighboring blocks over NCCL (grouped send/recv per peer).  The
timed region is the max over ranks.  --sharded runs the same path on one GPU
(one shard).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "M particles/s per migrate+halo+reverse step"
DEFAULT_WORKLOAD = "clustered_64"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (no dsx_grid_autotune before timing)")
    ap.add_argument("--particles", type=int, default=0,
                    help="override the workload's particle count (small profiling cases)")
    ap.add_argument("--no-aux", action="store_true",
                    help="skip the timings of the calls around the step (owner queries, "
                         "refreshes, split-phase overlap, rebalance, box changes)")
    ap.add_argument("--sharded", action="store_true",
                    help="the sharded grid's step (the multi-GPU path) also at one GPU")
    ap.add_argument("--exchange-volume", type=int, default=0, metavar="R",
                    help="bytes the sharded protocol sends per step with R shards (R = a^3 blocks "
                         "of the workload), the shards run in lockstep on one GPU")
    ap.add_argument("--sharded-impl", default="native", choices=["native", "python"],
                    help="the library's sharded protocol (dsx_shard_*) or the Python one")
    ap.add_argument("--sharded-step", default="fused", choices=["fused", "calls"],
                    help="native sharded grid: the fused step (dsx_shard_step) or the per-call "
                         "operations")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None
        self.skip = 0

    def _lines(self):
        self.file.flush()
        with open(self.file.name) as f:
            return sum(1 for line in f if line.count(",") >= 8)

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={CLOCK_QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "20"], stdout=self.file,
                stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: the timed region begins
            # once it samples, and only the samples after that count
            t0 = time.time()
            while self._lines() == 0 and time.time() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.skip = self._lines()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.file:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if len(rows) > self.skip:
            rows = rows[self.skip:]
        elif rows:
            rows = rows[-1:]   # the region ended before the next sample: the last one before it
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def algorithmic_bytes(S, N, E, G, B):
    """Bytes each kernel must move at minimum (reads + writes) for one step
    of N owned particles (E emigrants), G ghosts and B boundary owners, with
    S bytes per particle record (96 core + registered fields)."""
    R = N - E
    return {
        "mig_classify": 24 * N,                               # positions
        "mig_move": 24 * N + (S - 24) * R + S * R + 8 * E,    # read all, write retained, list emigrants
        "emig_place": E * (8 + 2 * S),
        "halo_classify": 24 * N + 4 * N,                      # positions in, mask out
        "halo_scatter": 4 * N + S * B + (S + 12) * G + 8 * B,  # masks, owners, ghosts + maps
        "reverse_sum": 8 * B + 4 * G + 24 * G + 48 * B,       # CSR, ghost forces, owner RMW
        # fused step (migrate + plan build in one pipeline)
        "step_classify": 24 * N + 6 * N,                      # positions in; destination + mask out
        "step_move": 6 * N + S * R + S * R + 8 * E + (S + 12) * G + 8 * B,
        "immigrant_halo": E * (24 + 4),
    }


def host_link(stream, copy, pieces, moved, device):
    """The host link alone, for scale beside e2e: the owned state down
    (device -> pinned host), up (into a device scratch of the same size, so
    the grid's state is left as it is) and both at once on two streams.  The
    downloads rewrite the host copy with the bytes it already holds, so the
    concurrent uploads read the same values either way."""
    import torch
    scratch = torch.empty(max(int(d.numel()) for d, _ in pieces), dtype=torch.uint8,
                          device=f"cuda:{device}")

    def timed(down, up):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a.record(stream)
        copy.wait_stream(stream)
        for d, h in pieces:
            if down:
                with torch.cuda.stream(stream):
                    h.copy_(d, non_blocking=True)
            if up:
                with torch.cuda.stream(copy):
                    scratch[:h.numel()].copy_(h, non_blocking=True)
        stream.wait_stream(copy)
        b.record(stream)
        torch.cuda.synchronize(device)
        return a.elapsed_time(b)

    timed(True, True)   # warm-up
    d2h, h2d, both = timed(True, False), timed(False, True), timed(True, True)
    gbs = lambda ms, n: round(n / (ms / 1e3) / 1e9, 1)
    return {"d2h_gbs": gbs(d2h, moved), "h2d_gbs": gbs(h2d, moved),
            "both_ms": round(both, 3), "both_gbs": gbs(both, 2 * moved)}


def harness_bytes(w, N, G, B):
    """Least bytes of the benchmark's step callback (the stand-in for the
    user's integrator and force loop): the drift reads each owned particle's
    id and position and writes the position back (52 B), the ghost forces
    write 24 B per ghost; workloads with field exchanges add the library's
    forward_exchange (2b G + 4 G) and reverse_exchange sum (b G + 4 G + 2b B)
    of every field of b bytes per particle."""
    sizes = {"int32": 4, "int64": 8, "uint32": 4, "uint64": 8, "float32": 4, "float64": 8}
    total = 52 * N + 24 * G
    if w.field_exchange:
        for _, t, c in w.fields:
            b = sizes[t] * c
            total += (2 * b * G + 4 * G) + (b * G + 4 * G + 2 * b * B)
    return int(total)


def step_accounting(step_bytes, harness, ms_per_step, kernels_ms, peak):
    """The step's roofline under one stated accounting: every byte the timed
    step must move (the library's kernels and the callback inside the step)
    over the device-timed wall time of the step."""
    whole = step_bytes + harness
    gbs = whole / (ms_per_step / 1e3) / 1e9
    return {"accounting": "library kernels' algorithmic bytes + the step callback's "
                          "(drift 52 B/particle, ghost forces 24 B/ghost, field exchanges) "
                          "over the timed ms_per_step",
            "bytes": int(whole), "library_bytes": int(step_bytes), "callback_bytes": int(harness),
            "ms_per_step": round(ms_per_step, 4), "achieved_gbs": round(gbs, 1),
            "frac_of_peak": round(gbs / peak, 4),
            "library_bytes_over_wall_frac": round(step_bytes / (ms_per_step / 1e3) / 1e9 / peak, 4),
            "library_kernels_ms": round(kernels_ms, 4)}


# ------------------------------------------------------------------- our arm

class DeviceBytes:
    """A device address range as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = dict(shape=(int(nbytes),), typestr="|u1",
                                             data=(int(ptr), False), version=3, strides=None)


def max_over_ranks(value, world, device=None):
    """The slowest rank's figure: an all-reduce MAX over the process group
    (a CUDA tensor on `device` for NCCL, a CPU tensor for gloo)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=f"cuda:{device}" if device is not None else "cpu")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world, device):
    import numpy as np
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W

    w = W.WORKLOADS[args.workload]
    if args.particles:
        import dataclasses
        w = dataclasses.replace(w, particles=args.particles)
    wl = W.harness()
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device)
    if w.nranks == 1:
        return run_drop_in(args, w, wl, stream, rank, world)

    dims, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    data = W.generate(w, seed=args.seed)
    owner = W.initial_owner(w, dims, data["x"], data["y"], data["z"])
    counts, grouped = W.group_by_owner(data, owner, w.nranks)
    del data, owner
    N = int(counts.sum())
    S = w.record_bytes()
    names = dsx.ARRAYS + [f[0] for f in w.fields]
    # pinned host copies of the state (the e2e leg copies them every step)
    pinned = []
    for name in names:
        if name in grouped:
            t = torch.from_numpy(np.ascontiguousarray(grouped[name])).pin_memory()
        else:
            t = torch.zeros(N, dtype=torch.float64).pin_memory()
        pinned.append(t)
    del grouped
    grid = dsx.VirtualGrid(w.nranks, w.dims, w.policy, w.lower, w.upper, halo_width=w.halo,
                           fields=w.fields, particles=N, ghost_capacity=int(0.9 * N))
    ptrs = [t.data_ptr() for t in pinned]
    with torch.cuda.stream(stream):
        grid.upload_flat(counts, ptrs)
    field_ids = list(range(len(w.fields))) if w.field_exchange else []
    seed = args.seed + 1000 * rank

    def user_work(view, s):
        # the user's integrator and force loop: ghost forces and the drift of
        # the owned particles (one launch), field exchanges where the
        # workload has them
        wl.dsxw_step_work(C.byref(view), seed, w.drift, s)
        if field_ids:
            grid.forward_exchange([w.fields[i][0] for i in field_ids], stream=s)
            grid.reverse_exchange([(w.fields[i][0], "sum") for i in field_ids], stream=s)

    harness_kernels = 1 + (0 if not field_ids else 2)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    tune = None
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            status = grid.step(user_work, capture=True)
            assert status == 0, status
        if not args.no_autotune:
            # launch shapes picked on this workload's particles, then the
            # step is re-captured with them
            tune = grid.autotune(stream=stream)
            for _ in range(2):
                status = grid.step(user_work, capture=True)
                assert status == 0, status
    stream.synchronize()

    # timed: the step calls alone (each returns its device status), no timing
    # marks inside the graphs and no count reads between steps
    # The steps are queued back to back (dsx_grid_step_async): each one is
    # queued once the previous step's build status has been read at its
    # event, and the wait completes the last one and returns the OR of every
    # step's status bits.  The same steps one call at a time (dsx_grid_step,
    # which waits for each) are timed after them for comparison.
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clocks:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                grid.step_async(user_work, stream=stream)
            status = grid.step_wait()
            end.record(stream)
            assert status == 0, status
        torch.cuda.synchronize(device)
    elapsed_ms = start.elapsed_time(end)
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s0.record(stream)
        for _ in range(args.steps):
            status = grid.step(user_work, capture=True)
            assert status == 0, status
        s1.record(stream)
    torch.cuda.synchronize(device)
    sync_ms = max_over_ranks(s0.elapsed_time(s1) / args.steps, world, device)
    clock = clocks.summary()
    kernels_per_step = grid.step_kernel_count()
    launches = args.steps * (kernels_per_step + harness_kernels)
    elapsed_ms = max_over_ranks(elapsed_ms, world, device)
    ms_per_step = elapsed_ms / args.steps
    value = world * N / (ms_per_step / 1e3) / 1e6

    # per-kernel CUDA-event times and the step's counts, from separate steps
    # that carry timing marks (graphs re-captured with the marks)
    per_kernel = {}
    totals_acc = {"particles": 0, "emigrants": 0, "ghosts": 0, "boundary": 0}
    profiled = max(4, min(args.steps, 20))
    with torch.cuda.stream(stream):
        grid.profile(True)
        grid.step(user_work, capture=True)
        grid.step(user_work, capture=True)
        for _ in range(profiled):
            status = grid.step(user_work, capture=True)
            assert status == 0, status
            for name, ms in grid.kernel_times():
                per_kernel.setdefault(name, []).append(ms)
            for k, v in grid.totals(stream=stream).items():
                totals_acc[k] += v
        grid.profile(False)
        grid.step(user_work, capture=True)   # graphs without the marks again
        grid.step(user_work, capture=True)
    stream.synchronize()

    avg = {k: sum(v) / len(v) for k, v in per_kernel.items()}
    mean_tot = {k: v / profiled for k, v in totals_acc.items()}
    alg = algorithmic_bytes(S, N, mean_tot["emigrants"], mean_tot["ghosts"], mean_tot["boundary"])
    ours = {k: v for k, v in avg.items() if k not in ("callback",)}
    dominant = max(ours, key=ours.get)
    peak, peak_kind = peaks()
    step_bytes = sum(v for k, v in alg.items() if k in ours)
    ours_ms = sum(ours.values())
    harness = harness_bytes(w, mean_tot["particles"] or N, mean_tot["ghosts"],
                            mean_tot["boundary"])
    roof = None
    if dominant in alg:
        achieved = alg[dominant] / (avg[dominant] / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": int(alg[dominant]),
                "avg_launch_ms": round(avg[dominant], 4),
                "traffic": traffic_from_profiles(w.name, dominant, N)}

    # e2e: the same step with the whole owned state in pinned host memory.
    # Every step's input crosses host -> device before it and its result
    # device -> host after it, one cudaMemcpyAsync per piece (an array, or a
    # 64 MB part of one) through the grid's view (dsx_grid_view_get): piece
    # p's download runs on the step's stream while the upload of the pieces
    # before it (the next step's input, each depending only on its own
    # download) runs on a second stream, so the two directions of the host
    # link overlap and only the last piece's upload trails the downloads.
    e2e = None
    if args.e2e_steps > 0:
        copy = torch.cuda.Stream(device)
        nbytes = [N * np.dtype(grid.dtype_of(n)).itemsize * grid.components(n) for n in names]
        host_bytes = [t.view(-1).view(torch.uint8)[:nb] for t, nb in zip(pinned, nbytes)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        piece = 64 << 20

        def owned_pieces():
            """(device, host) byte tensors of every piece of the owned state."""
            v = grid.view()
            out = []
            for a, nb in enumerate(nbytes):
                d = torch.as_tensor(DeviceBytes(int(v.base[a]) + (nb // N) * int(v.owned_offset),
                                                nb), device=f"cuda:{device}")
                for o in range(0, nb, piece):
                    out.append((d[o:o + piece], host_bytes[a][o:o + piece]))
            return out

        with torch.cuda.stream(stream):
            grid.download_flat(ptrs)
            barrier()
            e0.record(stream)
            for d, h in owned_pieces():                     # the first step's input
                d.copy_(h, non_blocking=True)
            for k in range(args.e2e_steps):
                status = grid.step(user_work, capture=True)
                assert status == 0, status
                last = k == args.e2e_steps - 1
                for d, h in owned_pieces():
                    h.copy_(d, non_blocking=True)           # this step's result (step stream)
                    if not last:
                        done = torch.cuda.Event()
                        done.record(stream)
                        copy.wait_event(done)
                        with torch.cuda.stream(copy):       # the next step's input
                            d.copy_(h, non_blocking=True)
                if not last:
                    stream.wait_stream(copy)
            e1.record(stream)
        torch.cuda.synchronize(device)
        e_ms = e0.elapsed_time(e1) / args.e2e_steps
        e_ms = max_over_ranks(e_ms, world, device)
        moved = int(sum(nbytes))
        e2e = {"value": round(world * N / (e_ms / 1e3) / 1e6, 3), "unit": "M particles/s",
               "h2d_bytes_per_step": moved, "d2h_bytes_per_step": moved,
               "ms_per_step": round(e_ms, 3), "steps": args.e2e_steps,
               "path": "pinned host -> owned state (64 MB pieces) -> dsx_grid_step -> pinned host "
                       "(each piece's download overlaps the earlier pieces' uploads)",
               "link": host_link(stream, copy, owned_pieces(), moved, device)}

    # per-call path (every call returns its counts synchronously, no graph);
    # events between the calls give each call's share (host time between
    # them included)
    plain = None
    plain_parts = None
    if args.plain_steps > 0:
        parts = ["migrate", "exchange_halo", "callback", "reverse_halo", "counts"]
        marks = [[torch.cuda.Event(enable_timing=True) for _ in range(len(parts) + 1)]
                 for _ in range(args.plain_steps)]
        grid.profile(False)
        with torch.cuda.stream(stream):
            for ev in marks:
                ev[0].record(stream)
                grid.migrate(stream=stream)
                ev[1].record(stream)
                grid.exchange_halo(rebuild=True, stream=stream)
                ev[2].record(stream)
                user_work(grid.view(), stream.cuda_stream)
                ev[3].record(stream)
                grid.reverse_halo(stream=stream)
                ev[4].record(stream)
                grid.all_counts(stream=stream)
                ev[5].record(stream)
        torch.cuda.synchronize(device)
        plain = round(marks[0][0].elapsed_time(marks[-1][-1]) / args.plain_steps, 3)
        plain_parts = {name: round(sum(ev[k].elapsed_time(ev[k + 1]) for ev in marks)
                                   / args.plain_steps, 4) for k, name in enumerate(parts)}

    # plain launches: the same per-call operations, every tile kernel launched
    # once per subdomain (the launch pattern of one process per subdomain)
    per_subdomain = None
    if args.plain_steps > 0:
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        grid.set_plain(True)
        with torch.cuda.stream(stream):
            q0.record(stream)
            for _ in range(args.plain_steps):
                grid.migrate(stream=stream)
                grid.exchange_halo(rebuild=True, stream=stream)
                user_work(grid.view(), stream.cuda_stream)
                grid.reverse_halo(stream=stream)
                grid.all_counts(stream=stream)
            q1.record(stream)
        torch.cuda.synchronize(device)
        grid.set_plain(False)
        per_subdomain = round(q0.elapsed_time(q1) / args.plain_steps, 3)

    aux = None
    if not args.no_aux:
        try:
            aux = measure_calls(grid, w, N, S, stream, device)
        except Exception as exc:   # reported, not fatal: the step's line stands
            aux = {"error": f"{type(exc).__name__}: {exc}"}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "M particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy PCG64 + counter-based device deviates)",
        "config": workload_config(w, world, dims),
        "step": "graph-captured batched steps queued back to back (dsx_grid_step_async)",
        "sync_ms_per_step": round(sync_ms, 4),
        "autotune": tune,
        "roofline": roof,
        "step_roofline": step_accounting(step_bytes, harness, ms_per_step, ours_ms, peak),
        "kernel_ms": {k: round(v, 4) for k, v in avg.items()},
        "totals_per_step": {k: int(v) for k, v in mean_tot.items()},
        "per_call_ms_per_step": plain, "per_call_parts_ms": plain_parts,
        "plain_ms_per_step": per_subdomain,
        "batched_vs_plain": round(per_subdomain / ms_per_step, 3) if per_subdomain else None,
        "clocks": clock,
        "e2e": e2e,
        "gpu_launches": launches,
        "aux": aux,
    }
    return line


def measure_calls(grid, w, N, S, stream, device, reps=10):
    """CUDA-event timings of the calls around the step, on the step's
    particles: owner queries and the out-of-domain check over every owned
    particle, halo refreshes (positions only, full) along the current plan,
    the split-phase refresh with independent work on another stream between
    begin and end, an explicit rebalance (with its migrate), and box / cut
    changes.  Bytes are each call's least traffic; fractions are of the
    measured copy bandwidth."""
    import numpy as np
    import torch
    peak, _ = peaks()

    def timed(fn, n=reps):
        fn()
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize(device)
        return a.elapsed_time(b) / n

    def row(ms, nbytes):
        gbs = nbytes / (ms / 1e3) / 1e9
        return {"ms": round(ms, 4), "bytes": int(nbytes), "achieved_gbs": round(gbs, 1),
                "frac": round(gbs / peak, 4)}

    out = {}
    with torch.cuda.stream(stream):
        grid.exchange_halo(rebuild=True, stream=stream, results=False)
        v = grid.view()
        G = int(grid.totals(stream=stream)["ghosts"])
        o = int(v.owned_offset)
        pos = [v.base[a] + 8 * o for a in range(3)]
        owner = torch.empty(N, dtype=torch.int32, device=device)
        out["owner_rank"] = row(timed(lambda: grid.owner_rank(
            pos[0], pos[1], pos[2], owner.data_ptr(), n=N, stream=stream)), 28 * N)
        out["out_of_domain"] = row(timed(lambda: grid.out_of_domain(stream=stream)), 24 * N)
        # per ghost: owner index and list entry, the owner's positions in,
        # positions and zeroed forces out (full: velocities and fields too)
        fb = S - 96
        out["refresh_positions"] = row(timed(lambda: grid.exchange_halo(
            positions_only=True, stream=stream, results=False)), 80 * G)
        out["refresh_full"] = row(timed(lambda: grid.exchange_halo(
            stream=stream, results=False)), (128 + 2 * fb) * G)
        # the same refreshes walked by each kind (the default picks ghosts or
        # tiles by what the refresh copies)
        for kind in ("owners", "ghosts", "tiles"):
            grid.set_refresh_kind(kind)
            out[f"refresh_positions_by_{kind[:-1]}"] = row(timed(lambda: grid.exchange_halo(
                positions_only=True, stream=stream, results=False)), 80 * G)
            out[f"refresh_full_by_{kind[:-1]}"] = row(timed(lambda: grid.exchange_halo(
                stream=stream, results=False)), (128 + 2 * fb) * G)
        grid.set_refresh_kind("auto")
        # split phase: begin launches the refresh (one captured graph) and
        # returns; interior work that needs the SMs, not HBM (the harness's
        # FP64 multiply-add stand-in over the owned positions), runs on
        # another stream until end.  Its length is matched to the refresh's.
        side = torch.cuda.Stream(device)
        from dsdecompx_b200 import workloads as W
        wl = W.harness()
        scratch = torch.empty(N, dtype=torch.float64, device=device)

        def interior_fn(rounds):
            def run():
                v = grid.view()
                wl.dsxw_interior(C.byref(v), rounds, scratch.data_ptr(), side.cuda_stream)
            return run

        def alone(rounds):
            def fn():
                side.wait_stream(stream)
                interior_fn(rounds)()
                stream.wait_stream(side)
            return fn

        t_refresh = out["refresh_positions"]["ms"]
        rounds = 64
        for _ in range(6):       # interior about as long as the refresh
            t_work = timed(alone(rounds))
            if abs(t_work - t_refresh) < 0.15 * t_refresh:
                break
            rounds = max(1, int(rounds * t_refresh / max(t_work, 1e-4)))
        t_work = timed(alone(rounds))
        work = interior_fn(rounds)

        def split():
            side.wait_stream(stream)   # before begin: the two then run side by side
            grid.begin_halo_exchange(positions_only=True, stream=stream)
            work()
            grid.end_halo_exchange(stream=stream)
            stream.wait_stream(side)

        shares = {}
        for share in (0, 4, 2, 1):
            grid.set_split_share(share)
            t_ref_share = timed(lambda: (grid.begin_halo_exchange(positions_only=True,
                                                                  stream=stream),
                                         grid.end_halo_exchange(stream=stream)))
            t_split = timed(split)
            shares[str(share)] = {
                "refresh_ms": round(t_ref_share, 4), "begin_work_end_ms": round(t_split, 4),
                "hidden_fraction": round((t_ref_share + t_work - t_split) /
                                         min(t_ref_share, t_work), 3)}
        best = max(shares, key=lambda k: shares[k]["hidden_fraction"])
        grid.set_split_share(0)
        torch.cuda.synchronize(device)
        h0 = time.perf_counter()
        grid.begin_halo_exchange(positions_only=True, stream=stream)
        h1 = time.perf_counter()
        grid.end_halo_exchange(stream=stream)
        h2 = time.perf_counter()
        grid.exchange_halo(positions_only=True, stream=stream, results=True)
        h3 = time.perf_counter()
        out["split_phase"] = {"interior_ms": round(t_work, 4),
                              "interior": f"FP64 multiply-add stand-in, {rounds} rounds x 4 "
                                          "chains per owned particle, 32 B of HBM traffic each, "
                                          "on another stream",
                              "by_ctas_per_sm": shares, "best_ctas_per_sm": int(best),
                              "hidden_fraction": shares[best]["hidden_fraction"],
                              "begin_host_us": round((h1 - h0) * 1e6, 1),
                              "end_host_us": round((h2 - h1) * 1e6, 1),
                              "blocking_call_host_us": round((h3 - h2) * 1e6, 1)}
        counts = grid.all_counts(stream=stream)[0].astype(np.float64)
        out["rebalance_with_work_ms"] = round(timed(lambda: grid.rebalance(
            counts, force=True, stream=stream), 3), 3)
        lo, up = w.lower, w.upper
        bigger = tuple(u * 1.0001 for u in up)

        def rescale():
            grid.rescale_domain(lo, bigger, stream=stream)
            grid.rescale_domain(lo, up, stream=stream)
        out["rescale_domain_pair_ms"] = round(timed(rescale, 3), 3)
        out["set_cuts_ms"] = round(timed(lambda: grid.set_cuts(grid.cuts(stream=stream),
                                                               stream=stream), 3), 3)
    out["particles"], out["ghosts"] = N, G
    return out


def exchange_volume(args):
    """Bytes each shard sends per step (migrants, ghost lists, returned
    forces) with R shards, each one block of the workload: R instances of
    the Python protocol run in lockstep on one GPU and count what they send.
    With the measured peer bandwidth this is the NVLink part of a step."""
    import ctypes as Cc

    import numpy as np
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    from dsdecompx_b200 import workloads as W
    R = args.exchange_volume
    w = W.WORKLOADS[args.workload]
    per = args.particles or w.particles
    fa = shard_factors(R)
    bdims, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    dims = tuple(d * k for d, k in zip(bdims, fa))
    P = int(np.prod(dims))
    upper = tuple(u * k for u, k in zip(w.upper, fa))
    coords = np.array([shd.subdomain_coords(t, dims) for t in range(P)])
    owners = ((coords[:, 0] // bdims[0]) * fa[1] + coords[:, 1] // bdims[1]) * fa[2] + coords[:, 2] // bdims[2]
    shards = []
    for r in range(R):
        b = (r // (fa[1] * fa[2]), (r // fa[2]) % fa[1], r % fa[2])
        d = W.generate(w, seed=args.seed + 7919 * r, particles=per)
        for a, name in enumerate("xyz"):
            d[name] = d[name] + b[a] * w.upper[a]
        d["global_id"] = (d["global_id"] + r * per).astype(np.int32)
        if "id64" in d:
            d["id64"] = d["id64"] + r * per
        cell = []
        for a, name in enumerate("xyz"):
            rel = np.floor((d[name] - w.lower[a]) / (upper[a] - w.lower[a]) * dims[a]).astype(np.int64)
            cell.append(np.clip(rel, b[a] * bdims[a], (b[a] + 1) * bdims[a] - 1))
        own = (cell[0] * dims[1] + cell[1]) * dims[2] + cell[2]
        engine = shd.DeviceEngine(P, dims if w.policy == "manual" else (0, 0, 0), w.policy, w.lower, upper,
                                  halo_width=w.halo, fields=w.fields, particles=int(1.5 * per) + 65536,
                                  ghost_capacity=per)
        sh = shd.ShardedGrid(engine, r, R, owners=owners)
        sh.upload({int(t): {k: v[own == t] for k, v in d.items()} for t in np.flatnonzero(owners == r)})
        shards.append(sh)
    wl = W.harness()
    steps = max(args.steps, 1)
    for step in range(args.warmup + steps):
        if step == args.warmup:
            for sh in shards:
                sh.sent_bytes = {k: 0 for k in sh.sent_bytes}
        for r, sh in enumerate(shards):
            v = sh.E.grid.view()
            wl.dsxw_drift(Cc.byref(v), args.seed + r, step, w.drift, torch.cuda.current_stream().cuda_stream)
        shd.run_lockstep([sh.step_steps() for sh in shards])
    torch.cuda.synchronize()
    sent = [{k: v / steps for k, v in sh.sent_bytes.items()} for sh in shards]
    most = max(sum(s.values()) for s in sent)
    link = 770.0   # measured NVLink peer copy, GB/s per direction
    return {"metric": "bytes sent per shard per step", "value": int(most), "unit": "B",
            "higher_is_better": False, "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "emulated_shards": R, "data": "synthetic",
            "config": {"workload": w.name, "particles_per_shard": per, "blocks": list(fa),
                       "subdomains": P, "grid": list(dims)},
            "per_kind_max_bytes": {k: int(max(s[k] for s in sent)) for k in sent[0]},
            "per_kind_mean_bytes": {k: int(np.mean([s[k] for s in sent])) for k in sent[0]},
            "nvlink_us_per_step_at_770_gbs": round(most / (link * 1e9) * 1e6, 1),
            "assembled_ghosts_per_shard": [int(sh.plan.total) for sh in shards]}


def shard_factors(world):
    """(a, b, c), a * b * c = world: the block counts along x, y, z (prime
    factors go to the axis with the fewest blocks so far)."""
    f, n, p = [1, 1, 1], world, 2
    while n > 1:
        while n % p == 0:
            f[f.index(min(f))] *= p
            n //= p
        p += 1
    return tuple(f)


def run_sharded(args, rank, world, device):
    """The step of the sharded grid: migrate -> halo build -> ghost forces and
    drift -> reverse_halo, every call one exchange step with the neighboring
    blocks' ranks."""
    import numpy as np
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import sharded as shd
    from dsdecompx_b200 import workloads as W

    w = W.WORKLOADS[args.workload]
    if args.particles:
        import dataclasses
        w = dataclasses.replace(w, particles=args.particles)
    if w.nranks == 1:
        raise SystemExit("the sharded grid needs a workload of several subdomains")
    wl = W.harness()
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device)
    fa = shard_factors(world)
    bdims, _ = dsx.plan_topology(w.nranks, 0, w.dims, w.policy, w.lower, w.upper)
    upper = tuple(u * k for u, k in zip(w.upper, fa))
    P = w.nranks * world
    dims, _ = dsx.plan_topology(P, 0, w.dims if w.policy == "manual" else (0, 0, 0), w.policy,
                                w.lower, upper) if w.policy != "manual" else \
        (tuple(d * k for d, k in zip(bdims, fa)), None)
    if tuple(dims) != tuple(d * k for d, k in zip(bdims, fa)):
        raise SystemExit(f"process grid {dims} is not {fa} blocks of {bdims}")
    # rank (bx, by, bz) owns the block of subdomains at those block coordinates
    bx, by, bz = rank // (fa[1] * fa[2]), (rank // fa[2]) % fa[1], rank % fa[2]
    coords = np.array([shd.subdomain_coords(t, dims) for t in range(P)])
    owners = ((coords[:, 0] // bdims[0]) * fa[1] + coords[:, 1] // bdims[1]) * fa[2] + coords[:, 2] // bdims[2]
    # this block's particles: the workload's distribution in the block's box
    data = W.generate(w, seed=args.seed + 7919 * rank)
    n = len(data["x"])
    for a, (name, k) in enumerate(zip("xyz", (bx, by, bz))):
        data[name] = data[name] + k * w.upper[a]
    data["global_id"] = (data["global_id"] + rank * n).astype(np.int32)
    if "id64" in data:
        data["id64"] = data["id64"] + rank * n
    cell = []
    for a, (name, k) in enumerate(zip("xyz", (bx, by, bz))):
        rel = np.floor((data[name] - w.lower[a]) / (upper[a] - w.lower[a]) * dims[a]).astype(np.int64)
        cell.append(np.clip(rel, k * bdims[a], (k + 1) * bdims[a] - 1))
    owner = (cell[0] * dims[1] + cell[1]) * dims[2] + cell[2]
    counts, grouped = W.group_by_owner(data, owner, P)
    del data, owner, cell
    N = int(counts.sum())
    S = w.record_bytes()
    names = dsx.ARRAYS + [f[0] for f in w.fields]
    # pinned host copies sized for the shard's storage: after migration a
    # rank may hold more particles than it started with
    capacity = int(1.5 * N) + 65536
    pinned = []
    for name in names:
        src = np.ascontiguousarray(grouped[name]) if name in grouped else np.zeros(N)
        t = torch.zeros((capacity,) + src.shape[1:], dtype=torch.from_numpy(src[:0]).dtype).pin_memory()
        t[:N].copy_(torch.from_numpy(src))
        pinned.append(t)
    del grouped
    ptrs = [t.data_ptr() for t in pinned]
    native = args.sharded_impl == "native"
    grid_args = (P, dims if w.policy == "manual" else (0, 0, 0), w.policy, w.lower, upper)
    grid_kw = dict(halo_width=w.halo, fields=w.fields, particles=capacity,
                   ghost_capacity=int(0.9 * N))
    if native:
        sh = shd.NativeShardedGrid(*grid_args, **grid_kw, shard=rank, nshards=world, owners=owners,
                                   device=f"cuda:{device}")
        engine = None
    else:
        engine = shd.DeviceEngine(*grid_args, **grid_kw)
        sh = shd.ShardedGrid(engine, rank, world, owners=owners,
                             run=lambda g: shd.run_distributed(g, device=f"cuda:{device}"))
    totals = torch.zeros(4, dtype=torch.int32, device=device)
    seed = args.seed + 1000 * rank

    def user_work(shard):
        s = stream.cuda_stream
        gv = shard.ghost_view() if native else shard.ghost_view(totals)
        wl.dsxw_ghost_forces(C.byref(gv), seed, 0, s)
        v = shard.owned_view() if native else shard.E.grid.view()
        wl.dsxw_drift(C.byref(v), seed, 0, w.drift, s)
        wl.dsxw_advance(s)

    def launched():
        return sh.launches if native else engine.launches

    fused = native and args.sharded_step == "fused"

    def fused_work(view, s):
        wl.dsxw_step_work(C.byref(view), seed, w.drift, s)

    def one_step():
        if fused:
            status = sh.step_fused(fused_work, stream=stream)
            assert status == 0, status
        else:
            sh.step(user_work)

    with torch.cuda.stream(stream):
        sh.upload_flat(counts, ptrs)
        for _ in range(args.warmup):
            one_step()
    stream.synchronize()
    torch.distributed.barrier()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = launched()
    with ClockSampler(device) as clocks:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                one_step()
            end.record(stream)
        torch.cuda.synchronize(device)
    launches = launched() - launches0 + 3 * args.steps
    elapsed_ms = max_over_ranks(start.elapsed_time(end), world, device)
    torch.distributed.barrier()
    clock = clocks.summary()
    ms_per_step = elapsed_ms / args.steps
    everyone = torch.tensor([float(N)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(everyone)
    Ntot = int(everyone.item())
    value = Ntot / (ms_per_step / 1e3) / 1e6
    # the step's least traffic (this rank): what the fused step's kernels move
    tot = sh.totals(stream=stream) if native else engine.grid.totals(stream=stream)
    alg = algorithmic_bytes(S, tot["particles"], tot["emigrants"], tot["ghosts"], tot["boundary"])
    step_bytes = sum(alg[k] for k in ("step_classify", "step_move", "emig_place", "immigrant_halo",
                                      "reverse_sum"))
    peak, peak_kind = peaks()
    achieved = step_bytes / (ms_per_step / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "whole sharded step (fused: planned kernels + exchanges)"
            if fused else "whole sharded step (per-call path + exchanges)",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6.65 TB/s",
            "algorithmic_bytes_per_launch": int(step_bytes), "avg_launch_ms": round(ms_per_step, 4),
            "traffic": None}
    e2e = None
    if args.e2e_steps > 0:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            cnt = sh.download_flat(ptrs)
            torch.distributed.barrier()
            e0.record(stream)
            for _ in range(args.e2e_steps):
                sh.upload_flat(cnt, ptrs)
                one_step()
                cnt = sh.download_flat(ptrs)
            e1.record(stream)
        torch.cuda.synchronize(device)
        e_ms = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, world, device)
        nb = int(cnt.sum()) * S + 8 * P
        e2e = {"value": round(Ntot / (e_ms / 1e3) / 1e6, 3), "unit": "M particles/s",
               "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb, "ms_per_step": round(e_ms, 3),
               "path": f"{type(sh).__name__}.upload_flat (pinned host) -> step -> download_flat"}
    (sh if native else engine).close()
    return {
        "metric": METRIC, "value": round(value, 3), "unit": "M particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy PCG64 + counter-based device deviates)",
        "config": workload_config(w, world, dims),
        "step": ("native sharded grid, fused step (dsx_shard_step: layout planned from every "
                 "shard's counts, one all-reduce, three NCCL exchanges)" if fused else
                 ("native sharded grid (dsx_shard_*" if native else "sharded grid (ShardedGrid") +
                 ": per-call operations, one NCCL exchange step per call)"),
        "roofline": roof,
        "clocks": clock,
        "e2e": e2e,
        "gpu_launches": launches,
    }


def traffic_from_profiles(workload, kernel, N):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of
    this workload (profiles/traffic.json), scaled to this launch's particle
    count; None when no capture of this workload and kernel is committed."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            data = json.load(f)
        entry = data[workload][kernel]
        return int(entry["dram_bytes_per_particle"] * N)
    except Exception:
        return None


def run_drop_in(args, w, wl, stream, rank, world):
    """Single-rank drop-in: drift + dsx_rank_migrate in place (no ghosts at
    one rank, so exchange_halo and reverse_halo do no work)."""
    import numpy as np
    import torch

    import dsdecompx_b200 as dsx
    from dsdecompx_b200 import workloads as W

    data = W.generate(w, seed=args.seed)
    N = w.particles
    dev = torch.device("cuda", torch.cuda.current_device())
    x, y, z = (torch.from_numpy(data[k]).to(dev) for k in "xyz")
    gid = torch.from_numpy(data["global_id"]).to(dev)
    seed = args.seed + 1000 * rank

    def step():
        wl.dsxw_drift_arrays(x.data_ptr(), y.data_ptr(), z.data_ptr(), gid.data_ptr(), N, seed, 0,
                             w.drift, stream.cuda_stream)
        wl.dsxw_advance(stream.cuda_stream)
        dsx.rank_migrate(x, y, z, N, w.lower, w.upper, stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # the positions (24 MB at 1M particles) fit in L2: a 256 MB write between
    # timed steps evicts them, and only the steps are timed
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    marks = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(args.steps)]
    with ClockSampler(torch.cuda.current_device()) as clocks:
        with torch.cuda.stream(stream):
            for a, b in marks:
                flush.zero_()
                a.record(stream)
                step()
                b.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    device = torch.cuda.current_device()
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in marks), world, device) / args.steps

    # the migrate alone (its wrap reads 24 B per particle and writes only the
    # coordinates that change), for the roofline
    # (a 1 GB flush keeps the GPU busy while the host enqueues the next
    # launch, so the interval holds the kernel, not the host's call overhead)
    reps = max(args.steps, 10)
    big = torch.empty(1 << 30, dtype=torch.uint8, device=dev)
    mig = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(reps)]
    with torch.cuda.stream(stream):
        for m0, m1 in mig:
            big.zero_()
            m0.record(stream)
            dsx.rank_migrate(x, y, z, N, w.lower, w.upper, stream=stream)
            m1.record(stream)
    torch.cuda.synchronize()
    mig_ms = sum(m0.elapsed_time(m1) for m0, m1 in mig) / reps
    del big
    peak, peak_kind = peaks()
    achieved = 24 * N / (mig_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "rank_migrate (k_wrap_inplace)", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6.65 TB/s",
            "algorithmic_bytes_per_launch": 24 * N, "avg_launch_ms": round(mig_ms, 4),
            "traffic": None}

    # e2e: positions in from pinned host memory, the step, positions back out
    e2e = None
    if args.e2e_steps > 0:
        host = [t.cpu().pin_memory() for t in (x, y, z)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.e2e_steps):
                for d, h in zip((x, y, z), host):
                    d.copy_(h, non_blocking=True)
                step()
                for d, h in zip((x, y, z), host):
                    h.copy_(d, non_blocking=True)
            e1.record(stream)
        torch.cuda.synchronize()
        e_ms = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, world, device)
        e2e = {"value": round(world * N / (e_ms / 1e3) / 1e6, 3), "unit": "M particles/s",
               "h2d_bytes_per_step": 24 * N, "d2h_bytes_per_step": 24 * N,
               "ms_per_step": round(e_ms, 3),
               "path": "pinned host x,y,z -> drift + dsx_rank_migrate -> pinned host"}
    return {"metric": METRIC, "value": round(world * N / (ms / 1e3) / 1e6, 3),
            "unit": "M particles/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, world, (1, 1, 1)),
            "step": "drift + dsx_rank_migrate (one rank: no ghosts, as in the reference)",
            "clocks": clocks.summary(), "gpu_launches": 3 * args.steps, "roofline": roof,
            "e2e": e2e}


# --------------------------------------------------------- reference (CPU)

def load_workloads():
    """The workload definitions (numpy only), loaded from their file: the
    reference arm imports nothing of the product package or its library."""
    import importlib.util
    name = "dsx_bench_workloads"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "dsdecompx_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload_config(w, world, dims):
    """The `config` object of the bench line: the workload alone (box, grid,
    particles, record), identical for both arms at the same N."""
    S = w.record_bytes()
    fa = shard_factors(world)
    cfg = {"workload": w.name, "description": w.description, "subdomains": w.nranks * world,
           "grid": [int(d) for d in dims], "particles": w.particles * world, "record_bytes": S}
    if world > 1:
        cfg["description"] += f"; one block per GPU, {fa[0]}x{fa[1]}x{fa[2]} blocks"
    if w.nranks == 1:
        cfg["l2"] = "L2 flushed (256 MB write) before every timed step"
    else:
        cfg["l2"] = "inputs larger than L2 (%.2f GB of owned records per GPU)" % (
            w.particles * S / 1e9)
    cfg["parallelism"] = "1 GPU" if world == 1 else f"subdomain blocks x{world}"
    return cfg


def reference_sample(W, w, world, seed, per_block):
    """Host arrays and initial owners of `per_block` particles per GPU block
    of the workload grown to `world` blocks (world 1: the workload itself),
    drawn as the GPU arm draws them."""
    import numpy as np
    fa = shard_factors(world)
    upper = tuple(u * k for u, k in zip(w.upper, fa))
    parts = []
    for rank in range(world):
        d = W.generate(w, seed=seed + 7919 * rank if world > 1 else seed, particles=per_block)
        k3 = (rank // (fa[1] * fa[2]), (rank // fa[2]) % fa[1], rank % fa[2])
        for a, name in enumerate("xyz"):
            d[name] = d[name] + k3[a] * w.upper[a]
        d["global_id"] = (d["global_id"] + rank * per_block).astype(np.int32)
        if "id64" in d:
            d["id64"] = d["id64"] + rank * per_block
        d["_block"] = np.full(per_block, rank, dtype=np.int64)
        parts.append(d)
    data = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    return data, upper


def reference_rate(w, world, seed, steps, warmup, budget_s=150.0):
    """The reference's own Host path (oracle/_ref, built from its sources)
    with one thread per subdomain: M particles/s of migrate + exchange_halo
    (rebuild) + reverse_halo, timed like its communication_test (slowest rank
    per call), `steps` timed steps after `warmup`, on a sample of the workload
    sized so that all of them fit `budget_s`.  Returns (cpu_baseline, dims,
    seconds per step) or (None, reason, None)."""
    import numpy as np

    import oracle

    if not oracle.available("ref"):
        return None, "reference build oracle/_ref/libdsx_ref.so is missing", None
    W = load_workloads()
    P = w.nranks * world
    fa = shard_factors(world)
    fields = [(n, ["int32", "int64", "uint32", "uint64", "float32", "float64"].index(t), c)
              for n, t, c in w.fields]
    manual_dims = tuple(d * k for d, k in zip(w.dims, fa)) if w.policy == "manual" else (0, 0, 0)

    def run(per_block, nsteps, nwarm):
        data, upper = reference_sample(W, w, world, seed, per_block)
        n_sample = len(data["x"])
        block = data.pop("_block")
        # the process grid first (the reference's own planner), then the
        # owners, then the grid with field storage sized by the largest rank
        with oracle.Grid("ref", P, manual_dims, w.policy, w.lower, upper) as probe_grid:
            dims = probe_grid.topology(0)[0]
        bdims = [d // k for d, k in zip(dims, fa)]
        k3 = np.stack([block // (fa[1] * fa[2]), (block // fa[2]) % fa[1], block % fa[2]])
        cell = []
        for a, name in enumerate("xyz"):
            rel = np.floor((data[name] - w.lower[a]) / (upper[a] - w.lower[a]) * dims[a])
            cell.append(np.clip(rel.astype(np.int64), k3[a] * bdims[a],
                                (k3[a] + 1) * bdims[a] - 1))
        owner = (cell[0] * dims[1] + cell[1]) * dims[2] + cell[2]
        order = np.argsort(owner, kind="stable")
        bounds = np.searchsorted(owner[order], np.arange(P + 1))
        cap = int(max(4 * np.diff(bounds).max(), 3 * n_sample // P) + 4096)
        g = oracle.Grid("ref", P, manual_dims, w.policy, w.lower, upper, (True,) * 3, w.halo,
                        fields=fields, field_capacity=cap)
        for r in range(P):
            idx = order[bounds[r]:bounds[r + 1]]
            g.set_owned(r, {k: v[idx] for k, v in data.items()})
        del data, owner, order
        rng = np.random.default_rng(seed + 1)
        times = []
        for step in range(nwarm + nsteps):
            for r in range(P):              # drift (harness, not timed)
                o, _ = g.counts(r)
                if o:
                    for name in "xyz":
                        g.write(r, name, 0, g.read(r, name, 0, o) + rng.normal(0, w.drift, o))
            t = g.timed("migrate") + g.timed("halo_rebuild")
            for r in range(P):              # ghost forces (harness, not timed)
                o, gh = g.counts(r)
                for name in ("fx", "fy", "fz"):
                    g.write(r, name, o, rng.normal(size=gh))
            t += g.timed("reverse_halo")
            if step >= nwarm:
                times.append(t)
        g.close()
        return n_sample, n_sample / statistics.mean(times) / 1e6, statistics.mean(times), dims

    probe = min(w.particles, max(1, 1_000_000 // world))
    _, rate, _, _ = run(probe, 1, 1)
    # size the sample so that (steps + warmup) steps fit the budget
    per_particle = 1.0 / (rate * 1e6)
    per_block = int(min(w.particles,
                        max(probe, budget_s / max(1, steps + warmup) / per_particle / world)))
    n_sample, rate, step_s, dims = run(per_block, steps, warmup)
    sample = (f"{n_sample} of the {w.particles * world}-particle {w.name} workload (same box, "
              f"grid, halo and distributions), {steps} timed steps after {warmup} warm-up; "
              f"{P} thread-ranks on {os.cpu_count()} host CPUs; {step_s:.3f} s per step")
    return ({"value": round(rate, 4), "unit": "M particles/s", "cores": P,
             "kind": "reference", "sample": sample}, dims, step_s)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # the reference's Host path on the host cores, on this arm's config
        # (the workload grown to --gpus blocks); rank 0 alone runs it
        if rank != 0:
            return
        W = load_workloads()
        w = W.WORKLOADS[args.workload]
        if args.particles:
            import dataclasses
            w = dataclasses.replace(w, particles=args.particles)
        base, dims, step_s = reference_rate(w, args.gpus, args.seed, args.steps, args.warmup)
        if base is None:
            print(json.dumps({"impl": "reference", "unavailable": dims}))
            return
        line = {"metric": METRIC, "value": base["value"], "unit": base["unit"],
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(step_s * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded numpy PCG64)", "impl": "reference",
                "config": workload_config(w, args.gpus, dims),
                "step": "reference Host path (oracle/_ref): migrate + exchange_halo(rebuild) + "
                        "reverse_halo, one thread per subdomain",
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": base["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if args.exchange_volume:
        print(json.dumps(exchange_volume(args)))
        return
    sharded = world > 1 or args.sharded
    if sharded:
        import datetime
        # NCCL's own log lines (its version banner) go to stderr: stdout
        # carries only the JSON line
        os.environ.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
        torch.cuda.set_device(local)
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", str(29500 + os.getpid() % 1000))
        torch.distributed.init_process_group("nccl", rank=rank, world_size=world,
                                             timeout=datetime.timedelta(seconds=120))
        line = run_sharded(args, rank, world, local)
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            W = load_workloads()
            w = W.WORKLOADS[args.workload]
            if args.particles:
                import dataclasses
                w = dataclasses.replace(w, particles=args.particles)
            base, why, _ = reference_rate(w, 1, args.seed, 2, 1, budget_s=25.0)
            line["cpu_baseline"] = base if base else {"unavailable": why}
        print(json.dumps(line))


if __name__ == "__main__":
    main()
