#!/usr/bin/env python
"""Headline benchmark: PSSM-profile Smith-Waterman-Gotoh GCUPS, batched vs plain, on B200.

Workload (one "step"): the PSSM configuration of the reference's benchmark
set — 4,000 int8 PSSM queries of length 50-2,000 (log-uniform), each built
from a synthetic 50-member family MSA (40-90% identity), against a 2.6 M-residue
synthetic database, top 300 targets per query (1.2 M uneven pairs), gap
costs 44/4.  One step scores every pair once through the captured CUDA graph
of persistent kernels (batched form).  GCUPS = sum of m*n over pairs (the
reference's gapped_cells) / step time.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--scale S]

Under torchrun (N > 1) the batch is split by target shards (residue-balanced
contiguous shards of the database, profiles replicated): each rank scores the
pairs whose target it holds, and every step ends with the exchange that
gathers the scores to rank 0 in pair order (strong scaling; the step time is
the max over ranks).  Rank 0 prints one JSON line.

On one GPU the line also carries the other rows, each with its own CPU
baseline and parity check: `calibration` (per-profile calibration of config-3
PSSMs), `ungapped` (config 2, 2x10^7 hits), `gate` (evidence / chain / gate on
2x10^7 seed hits), `search` (config 5 whole searches and their serving sweep)
and `serving` (config-4 scoring requests).  Each has a flag to skip it.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SW-Gotoh GCUPS (bit-exact), batched, PSSM queries"
UNIT = "GCUPS"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the 4,000 queries (quick runs)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--autotune", action="store_true",
                    help="measure the tile-class rates on this workload instead of the built-in B200 rates")
    ap.add_argument("--no-autotune", action="store_true", help="(default) use the built-in or loaded rates")
    ap.add_argument("--tuning-in", default=None, help="load a saved tile-class table and rates (JSON) before planning")
    ap.add_argument("--tuning-out", default=None, help="save the tile-class table and rates used (JSON)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--plain-pairs", type=int, default=2000)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--serving-pairs", type=int, default=20000, help="config-4 requests for the serving measurement (0: skip)")
    ap.add_argument("--ungapped-hits", type=int, default=20_000_000, help="config-2 hits for the ungapped measurement (0: skip)")
    ap.add_argument("--serving-seconds", type=float, default=2.0, help="arrival window per swept rate")
    ap.add_argument("--calib-profiles", type=int, default=1000,
                    help="config-3 profiles for the per-profile calibration measurement (0: skip)")
    ap.add_argument("--search-queries", type=int, default=1000,
                    help="config-5 queries for the whole-search measurement (0: skip)")
    ap.add_argument("--search-targets", type=int, default=1_000_000, help="config-5 database sequences")
    ap.add_argument("--exhaustive-queries", type=int, default=200,
                    help="config-1 queries against its 20,000 targets (0: skip)")
    ap.add_argument("--long-pairs", type=int, default=50_000, help="config-4 pairs, both halves (0: skip)")
    ap.add_argument("--gate-hits", type=int, default=20_000_000,
                    help="seed hits for the evidence / chain / gate measurement (0: skip)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def combine_ranks(ms, cells, device):
    """Whole-job step time and work across ranks: the slowest rank's step time (every rank scores its own
    instance of the workload, so the job ends with the slowest) and the sum of the ranks' cells."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells)], device=device, dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def make_workload(args, rank):
    from synth import workloads as W
    nq = max(8, int(round(4000 * args.scale)))
    db = max(50_000, int(round(2_600_000 * args.scale)))
    return W.config3(seed=args.seed + rank, n_queries=nq, db_residues=db)


def rows_upload_bytes(rows):
    """Bytes the library sends to the device for these int32 profile rows: one per score for a profile whose
    scores all fit int8 (it uploads those as int8), four otherwise."""
    return sum(r.size * (1 if r.size == 0 or (int(r.min()) >= -128 and int(r.max()) <= 127) else 4) for r in rows)


def config_of(args, w, world):
    return {"workload": "PSSM-profile SW-Gotoh (config 3: 4,000 int8 PSSM queries of length 50-2,000 from "
                        "50-member family MSAs vs a 2.6M-residue DB, top 300 targets per query, gaps 44/4)",
            "queries": w.info["queries"], "pairs": int(w.n_pairs), "db_residues": w.info["db_residues"],
            "db_seqs": w.info["db_seqs"], "cells_per_step": int(w.cells()), "gap_open": 44, "gap_extend": 4,
            "scale": args.scale, "seed": args.seed, "ranks": world,
            "parallelism": f"dp{world} (independent workload per GPU)",
            "l2": "flushed (256 MiB write) before every timed step"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def read_traffic(name="sw16_pssm_config3.md"):
    """Per-launch DRAM traffic of a kernel from its committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return int(ln.split(":")[1].strip())
            except ValueError:
                return None
    return None


def cpu_baseline(w, gpu_scores, seconds, seed=0):
    """The reference's CPU path restated (AVX2 u8 -> i16 striped -> exact scalar, queries in parallel over all
    host cores) timed on the whole workload, repeated until about `seconds` of CPU time have passed."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    ar = O.Arena(w.rows, w.targets())
    cells = w.cells()
    times, ref, kinds = [], None, None
    t_all = time.perf_counter()
    while not times or (time.perf_counter() - t_all < seconds and len(times) < 5):
        t0 = time.perf_counter()
        ref, kinds = O.striped_pairs(ar, w.pair_q, w.pair_t, w.gap_open, w.gap_extend, threads=cores,
                                     with_kinds=True)
        times.append(time.perf_counter() - t0)
    dt = float(np.median(times))
    out = {"value": round(cells / dt / 1e9, 3), "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"the whole workload ({w.n_pairs:,} pairs, {cells:,} cells), median of {len(times)} runs "
                     f"({dt:.2f} s each): the reference's default AVX2 path (u8 striped, i16 striped with lazy-F, "
                     f"exact scalar) restated in C, queries in parallel over {cores} threads",
           "kernel_mix": {"u8": int((kinds == 1).sum()), "i16": int((kinds == 2).sum()),
                          "scalar": int((kinds == 3).sum())}}
    if gpu_scores is not None:
        out["matches_gpu"] = bool(np.array_equal(ref, gpu_scores))
    return out


def repo_libraries_mapped():
    """Shared libraries of this repository mapped into the process (from /proc/self/maps)."""
    out = set()
    try:
        for ln in open("/proc/self/maps"):
            f = ln.split()
            if len(f) >= 6 and f[-1].endswith(".so") and os.path.realpath(f[-1]).startswith(os.path.realpath(ROOT)):
                out.add(os.path.relpath(os.path.realpath(f[-1]), os.path.realpath(ROOT)))
    except OSError:
        pass
    return sorted(out)


def run_reference(args):
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return 0
    w = make_workload(args, 0)
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    ar = O.Arena(w.rows, w.targets())
    cells = w.cells()
    for _ in range(args.warmup):
        O.striped_pairs(ar, w.pair_q, w.pair_t, w.gap_open, w.gap_extend, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.striped_pairs(ar, w.pair_q, w.pair_t, w.gap_open, w.gap_extend, threads=cores)
        times.append(time.perf_counter() - t0)
    v = round(cells / float(np.median(times)) / 1e9, 3)
    cb = {"cores": cores, "sample": f"the whole workload per step ({w.n_pairs:,} pairs, {cells:,} cells): the "
                                    f"reference's default AVX2 path (u8 -> i16 striped -> scalar) restated in C, "
                                    f"queries in parallel over {cores} threads"}
    mapped = repo_libraries_mapped()
    if any(os.path.basename(x) == "libsabertooth_b200.so" for x in mapped):
        raise RuntimeError("the reference arm mapped the product library: " + ", ".join(mapped))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config_of(args, w, 1),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                             "sample": "per step: " + cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "libraries_mapped": mapped,
            "note": "the reference (Rust) cannot be built here (no cargo, crates not vendored); its AVX2 "
                    "scoring path restated in C runs on all host cores; the inputs come from synth/ (the PSSM "
                    "builder in synth/libsynth.so), and no product code is loaded"}
    print(json.dumps(line), flush=True)
    return 0


def run_sharded(args, rank, world, local):
    """N > 1: the config-3 batch split by target shards (src/shard.rs:69-97 balance; queries and profiles
    replicated).  Every rank builds the same workload, uploads only its shard of the database, and scores
    the pairs whose target it holds through a captured plan; one step = that plan + the exchange: an NCCL
    all-gather of (global pair index, score) records, placed in global pair order on rank 0 by one
    index_copy (padding records point at a sink slot past the last pair).  Total work is fixed: strong
    scaling.  Step time = the slowest rank's, value = all pairs' cells / that time."""
    import torch
    import torch.distributed as dist
    from sabertooth_b200 import Context, GapCosts
    from sabertooth_b200._lib import PAIR_DTYPE
    from sabertooth_b200.shard import ShardMap
    dev = torch.device("cuda", local)
    t_gen = time.perf_counter()
    w = make_workload(args, 0)
    t_gen = time.perf_counter() - t_gen
    gaps = GapCosts(w.gap_open, w.gap_extend)
    n = w.n_pairs
    smap = ShardMap.of(w.db_offsets, world)
    res, offs = smap.shard_db(w.db_residues, w.db_offsets, rank)
    ctx = Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_db(res, offs)
    ids = ctx.create_profiles(w.rows)
    gpairs = np.zeros(n, dtype=PAIR_DTYPE)
    gpairs["profile"] = ids[w.pair_q]
    gpairs["target"] = w.pair_t
    gpairs["band_radius"] = -1
    idx, pairs = smap.route(gpairs, rank)
    k = len(idx)
    qlen = np.array([len(r) for r in w.rows], dtype=np.int64)
    tlen = np.diff(w.db_offsets.astype(np.int64))
    my_cells = int((qlen[w.pair_q[idx]] * tlen[w.pair_t[idx]]).sum())
    width_t = torch.tensor([k], dtype=torch.int64, device=dev)
    dist.all_reduce(width_t, op=dist.ReduceOp.MAX)
    width = max(int(width_t.item()), 1)
    d_scores = torch.zeros(max(k, 1), dtype=torch.int32, device=dev)
    rec = torch.zeros((width, 2), dtype=torch.int64, device=dev)
    rec[:, 0] = n  # padding records land in the sink slot
    if k:
        rec[:k, 0] = torch.from_numpy(idx).to(dev)
    gbuf = torch.zeros((world * width, 2), dtype=torch.int64, device=dev)
    merged = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    plan = ctx.plan(pairs, gaps, d_scores.data_ptr()) if k else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        if plan is not None:
            plan.run()
            rec[:k, 1].copy_(d_scores[:k])
        dist.all_gather_into_tensor(gbuf, rec)
        if rank == 0:
            merged.index_copy_(0, gbuf[:, 0], gbuf[:, 1])

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        launches0 = ctx.launch_count()
        clk = ClockSampler(local)
        clk.start()
        for s in range(args.steps):
            flush.zero_()
            starts[s].record(stream)
            step()
            ends[s].record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        clocks = clk.stop()
        launches = ctx.launch_count() - launches0
    ms_rank = float(np.mean([a.elapsed_time(b) for a, b in zip(starts, ends)]))
    ms, _ = combine_ranks(ms_rank, my_cells, dev)
    cells = w.cells()
    gcups = cells / (ms * 1e-3) / 1e9

    # end to end through the public API with host buffers, every step on every rank: profiles from pinned
    # int32 rows, this rank's pairs up, scores down, the host (index, score) records gathered to rank 0 and
    # placed there; timed per rank between barriers, the slowest rank's time
    nrows = np.array([len(r) for r in w.rows], dtype=np.uint64)
    row_offs = np.zeros(len(w.rows) + 1, dtype=np.uint64)
    row_offs[1:] = np.cumsum(nrows)
    rows_pin = torch.empty((int(row_offs[-1]), 21), dtype=torch.int32, pin_memory=True).numpy()
    for q, r in enumerate(w.rows):
        rows_pin[int(row_offs[q]):int(row_offs[q + 1])] = r
    from sabertooth_b200.shard import gather_scores
    e2e_ms, e2e_ok = [], True
    dev_scores = merged[:n].to(torch.int32).cpu().numpy() if rank == 0 else None
    for _ in range(max(args.e2e_steps, 3)):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eids = ctx.create_profiles_arena(rows_pin, row_offs)
        lp = pairs.copy()
        lp["profile"] = eids[w.pair_q[idx]]
        sc = ctx.sw_score_pairs(lp, gaps) if k else np.zeros(0, np.int32)
        got = gather_scores(idx, sc, n, device=dev)
        ctx.free_profiles(eids)
        t_rank = time.perf_counter() - t0
        tmax, _ = combine_ranks(t_rank * 1e3, 0, dev)
        e2e_ms.append(tmax)
        if rank == 0:
            e2e_ok &= bool(np.array_equal(got, dev_scores))
    e2e_t = float(np.median(e2e_ms))
    if plan is not None:
        plan.close()
    ctx.free_profiles(ids)
    if rank != 0:
        return None
    # parity sample on rank 0: the merged scores of 2,000 random pairs against the oracle
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    sel = rng.choice(n, size=min(2000, n), replace=False)
    ar = O.Arena(w.rows, w.targets())
    sample_ok = bool(np.array_equal(O.sw_pairs(ar, w.pair_q[sel], w.pair_t[sel], w.gap_open, w.gap_extend),
                                    dev_scores[sel]))
    cfg = config_of(args, w, world)
    cfg["parallelism"] = f"target shards x{world} (residue-balanced contiguous, profiles replicated), " \
                         "scores gathered to rank 0 (NCCL all-gather) inside every step"
    return {"metric": METRIC, "value": round(gcups, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int16x2 (packed DPX) + int32 rescore", "data": "synthetic",
            "config": cfg, "clocks": clocks, "gpu_launches": int(launches),
            "e2e": {"value": round(cells / (e2e_t * 1e-3) / 1e9, 2), "unit": UNIT,
                    "h2d_bytes_per_step": int(rows_upload_bytes(w.rows) + k * PAIR_DTYPE.itemsize),
                    "d2h_bytes_per_step": int(k * 4), "ms_per_step": round(e2e_t, 2),
                    "matches_device_run": bool(e2e_ok),
                    "includes": "per step on every rank: profile build from pinned int32 rows, this rank's pairs "
                                "up, plan, launches, scores down, host records gathered to rank 0 and placed; "
                                "rank 0's host-to-device bytes stated"},
            "shards": [{"targets": int(b - a), "residues": int(w.db_offsets[b] - w.db_offsets[a])}
                       for a, b in smap.ranges],
            "matches_oracle_sample": sample_ok, "setup_s": {"generate": round(t_gen, 1)}}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        result = run_sharded(args, rank, world, local)
        if rank == 0:
            print(json.dumps(result), flush=True)
        dist.barrier()
        dist.destroy_process_group()
        return 0
    from sabertooth_b200 import Context, GapCosts
    from sabertooth_b200._lib import PAIR_DTYPE

    t_gen = time.perf_counter()
    w = make_workload(args, rank)
    t_gen = time.perf_counter() - t_gen
    gaps = GapCosts(w.gap_open, w.gap_extend)
    cells = w.cells()

    ctx = Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
    pairs["profile"] = ids[w.pair_q]
    pairs["target"] = w.pair_t
    pairs["band_radius"] = -1

    t_tune = time.perf_counter()
    if args.tuning_in:
        saved_tuning = json.load(open(args.tuning_in))
        ctx.set_tuning_table(np.array(saved_tuning["table"], dtype=np.int32))
        if "rates" in saved_tuning:
            ctx.set_tuning_rates(np.array(saved_tuning["rates"], dtype=np.float32))
    tuned = ctx.autotune(pairs, gaps, max_pairs=400_000) if args.autotune and not args.no_autotune else 0
    t_tune = time.perf_counter() - t_tune
    if args.tuning_out and rank == 0:
        with open(args.tuning_out, "w") as f:
            json.dump({"table": ctx.tuning_table().tolist(), "rates": ctx.tuning_rates().tolist()}, f)

    d_scores = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    d_kern = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    t_plan = time.perf_counter()
    plan = ctx.plan(pairs, gaps, d_scores.data_ptr(), d_kern.data_ptr())
    t_plan = time.perf_counter() - t_plan
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            plan.run()
        stream.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        launches0 = ctx.launch_count()
        clk = ClockSampler(local)
        clk.start()
        for s in range(args.steps):
            flush.zero_()
            starts[s].record(stream)
            plan.run()
            ends[s].record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        clocks = clk.stop()
        launches = ctx.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    ms = float(np.mean(step_ms))
    if world > 1:
        ms, total_cells = combine_ranks(ms, cells, "cuda")
    else:
        total_cells = float(cells)
    gcups = total_cells / (ms * 1e-3) / 1e9
    stats = plan.stats()
    launch_profile = [{"tile": (f"G{sh[0]}xR{sh[1]}xC{sh[2]}" if isinstance(sh, tuple) else sh), "cells": c, "ms": round(t, 3),
                       "gcups": round(c / (t * 1e-3) / 1e9, 1) if t > 0 else None}
                      for sh, c, t in plan.profile()] if rank == 0 else None
    scores = d_scores.cpu().numpy()
    kern = d_kern.cpu().numpy()

    result = None
    if rank == 0:
        # roofline: packed s16x2 DPX add-max throughput measured now on this GPU; 6 DPX ops per packed cell pair
        dpx = ctx.probe_dpx()
        peak_gcups = 2.0 * dpx / 6.0 / 1e9
        per_gpu_gcups = cells / (float(np.mean(step_ms)) * 1e-3) / 1e9
        # plain per-call path (the drop-in): one st_sw_score per pair, host target, blocking
        from sabertooth_b200 import QueryProfile
        rng = np.random.default_rng(1)
        sample = rng.choice(w.n_pairs, size=min(args.plain_pairs, w.n_pairs), replace=False)
        qps = {}
        targets = [w.db_residues[int(a):int(b)] for a, b in zip(w.db_offsets[:-1], w.db_offsets[1:])]
        pc = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        from sabertooth_b200._lib import check, lib
        import ctypes as C
        sc, kk = C.c_int32(), C.c_uint32()
        plain_ok = True
        for p in sample:
            q = int(w.pair_q[p])
            t = targets[int(w.pair_t[p])]
            check(lib.st_sw_score(ctx.handle, int(ids[q]), t.ctypes.data, t.size, gaps.open, gaps.extend,
                                  C.byref(sc), C.byref(kk)))
            plain_ok &= sc.value == int(scores[p])
            pc += len(w.rows[q]) * t.size
        plain_s = time.perf_counter() - t0
        plain_gcups = pc / plain_s / 1e9
        del qps
        # the same drop-in under concurrent callers, as the reference's rayon workers call sw_score_with
        # (src/search.rs:552-556): one host thread per core, each calling st_sw_score on its share
        n_thr = os.cpu_count() or 1
        csample = rng.choice(w.n_pairs, size=min(args.plain_pairs * 8, w.n_pairs), replace=False)
        cres = np.zeros(len(csample), dtype=np.int64)
        c_cells = int(sum(len(w.rows[int(w.pair_q[p])]) * targets[int(w.pair_t[p])].size for p in csample))

        def plain_worker(k):
            s_, k_ = C.c_int32(), C.c_uint32()
            for i in range(k, len(csample), n_thr):
                p_ = int(csample[i])
                t_ = targets[int(w.pair_t[p_])]
                check(lib.st_sw_score(ctx.handle, int(ids[int(w.pair_q[p_])]), t_.ctypes.data, t_.size, gaps.open,
                                      gaps.extend, C.byref(s_), C.byref(k_)))
                cres[i] = s_.value

        def conc_round():
            ths = [threading.Thread(target=plain_worker, args=(k,)) for k in range(n_thr)]
            t0 = time.perf_counter()
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            return time.perf_counter() - t0

        conc_round()  # untimed: every thread's call slot (stream, pinned block, buffers) is created here
        conc_ok = bool(np.array_equal(cres, scores[csample]))
        conc_runs = []
        for _ in range(3):
            cres[:] = -1
            conc_runs.append(conc_round())
            conc_ok &= bool(np.array_equal(cres, scores[csample]))
        conc_s = float(np.median(conc_runs))
        plain_conc = {"value": round(c_cells / conc_s / 1e9, 3), "unit": UNIT, "pairs": int(len(csample)),
                      "threads": n_thr, "matches_batched": conc_ok,
                      "runs_gcups": [round(c_cells / t / 1e9, 3) for t in conc_runs],
                      "how": "one host thread per core, each calling st_sw_score (host target, blocking) on its "
                             "share of the sample; calls run side by side on per-call streams; median of three "
                             "rounds after an untimed one"}

        # end to end through the C ABI with host buffers, the database resident (uploaded once, as an index
        # is): every step uploads the query profiles' int32 rows and the pairs from pinned host memory, plans,
        # runs and reads the scores and kernel tags back, then frees the profiles
        nrows = np.array([len(r) for r in w.rows], dtype=np.uint64)
        row_offs = np.zeros(len(w.rows) + 1, dtype=np.uint64)
        row_offs[1:] = np.cumsum(nrows)
        rows_pin = torch.empty((int(row_offs[-1]), 21), dtype=torch.int32, pin_memory=True).numpy()
        for q, r in enumerate(w.rows):
            rows_pin[int(row_offs[q]):int(row_offs[q + 1])] = r
        pairs_pin = torch.empty(w.n_pairs * PAIR_DTYPE.itemsize, dtype=torch.uint8,
                                pin_memory=True).numpy().view(PAIR_DTYPE)
        pairs_pin[:] = pairs
        local_q = w.pair_q.astype(np.int64)
        h2d = int(rows_upload_bytes(w.rows) + pairs_pin.nbytes)
        d2h = int(w.n_pairs * 8)
        e2e_times, e2e_ok, parts = [], True, []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eids = ctx.create_profiles_arena(rows_pin, row_offs)
            t1 = time.perf_counter()
            pairs_pin["profile"] = eids[local_q]
            t2 = time.perf_counter()
            es, ek = ctx.sw_score_pairs(pairs_pin, gaps, with_kernels=True)
            t3 = time.perf_counter()
            ctx.free_profiles(eids)
            t4 = time.perf_counter()
            e2e_times.append(t4 - t0)
            parts.append([t1 - t0, t2 - t1, t3 - t2, t4 - t3])
            e2e_ok &= bool(np.array_equal(es, scores))
        e2e_parts = {k: [round(1e3 * float(p[i]), 2) for p in parts]
                     for i, k in enumerate(["profiles", "pair_ids", "score_pairs", "free"])}
        e2e_seq_gcups = cells / float(np.median(e2e_times)) / 1e9

        # the same steps back to back as a serving loop runs them: step s+1's profiles are built
        # and its pairs filled and launched while step s runs on the GPU (st_sw_score_pairs_async);
        # every step still uploads its rows and pairs and reads its scores and kernel tags back
        outs = [torch.empty(w.n_pairs, dtype=torch.int32, pin_memory=True).numpy() for _ in range(2)]
        kouts = [torch.empty(w.n_pairs, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
                 for _ in range(2)]
        steps_ov = max(24, args.e2e_steps)  # a run of back-to-back steps pays the pipeline fill once
        t_runs = []
        for _ in range(3):  # three runs of steps_ov steps; the median run is reported
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            prev = None
            for s_ in range(steps_ov):
                eids = ctx.create_profiles_arena(rows_pin, row_offs)
                pairs_pin["profile"] = eids[local_q]
                bt = ctx.sw_score_pairs_async(pairs_pin, gaps, scores=outs[s_ % 2], kernels=kouts[s_ % 2])
                if prev is not None:
                    es, _ = prev[0].wait()
                    e2e_ok &= bool(np.array_equal(es, scores))
                    ctx.free_profiles(prev[1])
                prev = (bt, eids)
            es, _ = prev[0].wait()
            e2e_ok &= bool(np.array_equal(es, scores))
            ctx.free_profiles(prev[1])
            t_runs.append(time.perf_counter() - t0)
        t_ov = float(np.median(t_runs))
        e2e_gcups = cells * steps_ov / t_ov / 1e9

        cb = cpu_baseline(w, scores, args.cpu_seconds)
        traffic = read_traffic()
        result = {
            "metric": METRIC, "value": round(gcups, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int16x2 (packed DPX) + int32 rescore", "data": "synthetic",
            "config": config_of(args, w, world),
            "roofline": {"bound": "dpx", "achieved": round(per_gpu_gcups, 2), "peak": round(peak_gcups, 2),
                         "unit": UNIT, "frac": round(per_gpu_gcups / peak_gcups, 4), "traffic": traffic,
                         "peak_source": f"measured live: __viaddmax_s16x2 {dpx / 1e12:.2f} Tops/s device-wide; "
                                        "peak cells/s = 2 * ops/s / 6 (6 DPX ops per packed pair of cells)"},
            "cpu_baseline": cb,
            "e2e": {"value": round(e2e_gcups, 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": steps_ov, "matches_device_run": bool(e2e_ok),
                    "ms_per_step": round(1e3 * t_ov / steps_ov, 2),
                    "runs_ms_per_step": [round(1e3 * t / steps_ov, 2) for t in t_runs],
                    "includes": "per step: profile build from int32 rows (pinned; the library uploads the rows "
                                "of a profile whose scores fit int8 as int8, which h2d counts), profile ids into "
                                "the pairs, "
                                "pair upload, plan, kernel launches, scores + kernel tags download, profile "
                                "free; target database resident; step s+1 is prepared while step s runs; "
                                "each timed run (median of 3) is `steps` steps back to back and includes "
                                "the first step's preparation, when the device is idle",
                    "sequential": {"value": round(e2e_seq_gcups, 2), "steps": args.e2e_steps,
                                   "ms_per_step": round(1e3 * float(np.median(e2e_times)), 2),
                                   "ms_parts": e2e_parts}},
            "plain": {"value": round(plain_gcups, 3), "unit": UNIT, "pairs": int(len(sample)),
                      "matches_batched": bool(plain_ok),
                      "how": "one st_sw_score call per pair (host target, 2 launches, blocking)"},
            "plain_concurrent": plain_conc,
            "batched_vs_plain": round(gcups / world / plain_gcups, 1),
            "clocks": clocks,
            "gpu_launches": int(launches),
            "kernels_per_step": int(launches // max(args.steps, 1)),
            "rescored_pairs": int(stats["rescored_pairs"]),
            "gpu32_pairs": int((kern == 2).sum()),
            "launch_classes": int(stats["launch_classes"]),
            "launch_profile": launch_profile,
            "autotuned_classes": int(tuned),
            "class_rates_tcells_per_s": [round(float(r), 3) for r in ctx.tuning_rates()],
            "setup_s": {"generate": round(t_gen, 1), "autotune": round(t_tune, 1), "plan": round(t_plan, 2)},
            "step_ms_min_max": [round(min(step_ms), 3), round(max(step_ms), 3)],
        }
    plan.close()
    # the other rows are single-GPU measurements: taken on one GPU runs only (the other ranks would wait)
    extra = result is not None and world == 1
    if extra and args.calib_profiles > 0:
        result["calibration"] = calibration_measure(ctx, args, w, ids, gaps)
    # the config-3 profiles are done with; kernels that stage a query's rows size them by the live profiles
    ctx.free_profiles(ids)
    if extra and args.ungapped_hits > 0:
        result["ungapped"] = ungapped_measure(ctx, args)
    if extra and args.gate_hits > 0:
        result["gate"] = gate_measure(ctx, args)
    if extra and args.search_queries > 0:
        result["search"] = search_measure(ctx, args)
    if extra and args.exhaustive_queries > 0:
        result["exhaustive"] = exhaustive_measure(ctx, args)
    if extra and args.long_pairs > 0:
        result["long_mix"] = long_mix_measure(ctx, args)
    if extra and args.serving_pairs > 0:
        result["serving"] = serving_measure(ctx, args)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    ctx.close()
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0


def ungapped_measure(ctx, args):
    """Row (U): ungapped diagonal scoring of prefilter seed hits (config 2: 1,000 queries, 374,000 targets,
    68 M residues, 2x10^7 hits, 30% on planted-homolog diagonals). Hits resident on the device; per step one
    st_ungapped_hits_device call (per-hit best + per-(query, target) best). Roofline: algorithmic bytes
    (window residues + 12 B hit + 4 B output per hit) / time against the measured HBM copy bandwidth."""
    import torch
    from oracle import oracle as O
    from synth import workloads as W
    t0 = time.perf_counter()
    w = W.config2(seed=args.seed, n_hits=args.ungapped_hits)
    t_gen = time.perf_counter() - t0
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    hits = w.hits.copy()
    hits["query"] = ids[hits["query"]]
    n = len(hits)
    st = torch.cuda.Stream()
    ctx.set_stream(st.cuda_stream)
    d_hits = torch.from_numpy(hits.view(np.uint8)).cuda()
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_pb = torch.empty(n, dtype=torch.int32, device="cuda")
    d_pq = torch.empty(n, dtype=torch.int32, device="cuda")
    d_pt = torch.empty(n, dtype=torch.int32, device="cuda")
    d_np = torch.zeros(1, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ab = w.algorithmic_bytes()
    with torch.cuda.stream(st):
        for _ in range(3):
            ctx.ungapped_hits_device(d_hits.data_ptr(), n, d_out.data_ptr(), d_pb.data_ptr(), d_pq.data_ptr(),
                                     d_pt.data_ptr(), d_np.data_ptr())
        ts = []
        for _ in range(max(3, args.steps)):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            ctx.ungapped_hits_device(d_hits.data_ptr(), n, d_out.data_ptr(), d_pb.data_ptr(), d_pq.data_ptr(),
                                     d_pt.data_ptr(), d_np.data_ptr())
            b.record(st)
            st.synchronize()
            ts.append(a.elapsed_time(b))
    ctx.set_stream(0)
    ms = float(np.median(ts))
    got = d_out.cpu().numpy()
    n_runs = int(d_np.item())
    # CPU baseline: the reference's AVX2 batched Kadane restated in C over the whole workload, all host
    # cores (median of three runs); its results are the parity check of the GPU's
    targets = [w.db_residues[int(a_):int(b_)] for a_, b_ in zip(w.db_offsets[:-1], w.db_offsets[1:])]
    arena = O.Arena(w.rows, targets)
    t_runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        want = O.ungapped_hits_avx2(arena, w.hits["query"], w.hits["target"], w.hits["diag"])
        t_runs.append(time.perf_counter() - t0)
    t_cpu = float(np.median(t_runs))
    rng = np.random.default_rng(args.seed)
    sel = np.sort(rng.choice(n, min(n, 200_000), replace=False))
    scalar_ok = bool(np.array_equal(O.ungapped_hits(arena, w.hits["query"][sel], w.hits["target"][sel],
                                                    w.hits["diag"][sel]), want[sel]))
    # the per-(query, target) runs against the same runs reduced from the CPU baseline's scores
    key = w.hits["query"].astype(np.int64) * (1 << 32) + w.hits["target"]
    heads = np.ones(n, dtype=bool)
    heads[1:] = key[1:] != key[:-1]
    idx = np.nonzero(heads)[0]
    pairs_ok = (n_runs == len(idx)
                and np.array_equal(d_pb[:n_runs].cpu().numpy(), np.maximum.reduceat(want, idx))
                and np.array_equal(d_pq[:n_runs].cpu().numpy().view(np.uint32), hits["query"][idx])
                and np.array_equal(d_pt[:n_runs].cpu().numpy().view(np.uint32), hits["target"][idx]))
    peak = hbm_peak_gbs()
    gbs = ab / (ms * 1e-3) / 1e9
    ctx.free_profiles(ids)
    return {"workload": f"config 2: {len(w.rows)} queries, {len(w.db_offsets) - 1} targets "
                        f"({int(w.db_offsets[-1]) / 1e6:.1f} M residues), {n} hits (30% homolog diagonals)",
            "ms_per_step": round(ms, 3), "mhits_per_s": round(n / ms / 1e3, 1),
            "algorithmic_bytes": int(ab), "runs": n_runs,
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "traffic": read_traffic("ungapped_config2.md"),
                         "peak_source": hbm_peak()[1]},
            "matches_cpu_baseline": bool(np.array_equal(got, want)), "pairs_match_cpu_baseline": bool(pairs_ok),
            "cpu_baseline_matches_scalar_sample": scalar_ok,
            "cpu_baseline": {"value": round(n / t_cpu / 1e6, 2), "unit": "Mhits/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": f"the whole workload ({n} hits), median of 3 runs: the "
                                                       "reference's AVX2 batched Kadane (biased u8 tables, 32 lanes, "
                                                       "window-start order, exact rescore) restated in C, queries in "
                                                       "parallel over all host threads"},
            "setup_s": round(t_gen, 1)}


def search_measure(ctx, args):
    """Config 5 as whole searches: a 10^6-sequence database (~265 M residues) and 1,000 sequence queries, each
    with 5 planted homologs; the reference's sequence defaults (spaced seed 111001101, k-mer score 22, 512 k-mers
    per window, exact seeds, 4 diagonals, window 48) with the gate moved to the database size
    (size_adjusted_gate, src/prefilter.rs:253-257); gaps 11/1.  One step = st_prefilter_queries for the whole
    batch (host residues in, ranked candidates out: seeds -> hits -> evidence -> chains -> gate) then
    st_sw_score_pairs over every candidate (host pairs in, scores out)."""
    from oracle import oracle as O
    from sabertooth_b200 import GapCosts, PrefilterParams
    from sabertooth_b200._lib import PAIR_DTYPE
    from synth import workloads as W
    t0 = time.perf_counter()
    w = W.config5(seed=args.seed, n_queries=args.search_queries, n_targets=args.search_targets)
    t_gen = time.perf_counter() - t0
    n_res = int(w.db_offsets[-1])
    ctx.upload_db(w.db_residues, w.db_offsets)
    t0 = time.perf_counter()
    ctx.seed_index_build("111001101")
    t_index = time.perf_counter() - t0
    ids = ctx.create_profiles(w.rows)
    gate = W.size_adjusted_gate(42, n_res)
    params = PrefilterParams(min_diag_score=gate, span=9)
    gaps = GapCosts.sequence_default()
    ctx.prefilter_queries(ids[:16], w.queries[:16], params, gaps)  # warm-up
    qlen = np.array([len(q) for q in w.queries], dtype=np.int64)
    tlen = np.diff(w.db_offsets.astype(np.int64))
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        cands, st, sst = ctx.prefilter_queries(ids, w.queries, params, gaps)
        t1 = time.perf_counter()
        pairs = np.zeros(len(cands), dtype=PAIR_DTYPE)
        pairs["profile"] = cands["query"]
        pairs["target"] = cands["target"]
        pairs["band_radius"] = -1
        scores = ctx.sw_score_pairs(pairs, gaps)
        t2 = time.perf_counter()
        runs.append((t1 - t0, t2 - t1))
    t_pre = float(np.median([r[0] for r in runs]))
    t_sw = float(np.median([r[1] for r in runs]))
    inv = np.zeros(int(ids.max()) + 1, dtype=np.int64)
    inv[ids] = np.arange(len(ids))
    cq = inv[cands["query"]]
    cells = int((qlen[cq] * tlen[cands["target"]]).sum())
    # CPU baseline: the restated seed stage (best-first similar k-mers over a direct-table index) + evidence +
    # gate, then the reference's AVX2 striped SW over the candidates, for a sample of queries on all host threads
    t0 = time.perf_counter()
    di = O.DirectSeedIndex(w.db_residues, w.db_offsets, "111001101")
    t_cpu_index = time.perf_counter() - t0
    k = min(48, len(ids))
    sp = {"kmer_score": params.kmer_score, "max_kmers_per_pos": params.max_kmers_per_pos, "exact_seeds": 1,
          "max_seed_occ": 0}
    gp = {"min_hits": params.min_hits, "diag_hits": params.diag_hits, "max_diagonals": params.max_diagonals,
          "diag_window": params.diag_window, "span": 9, "min_diag_score": gate, "gap_open": gaps.open,
          "gap_ext": gaps.extend, "max_candidates": params.max_candidates, "regions": 0}
    t0 = time.perf_counter()
    cc, nc, nh = O.prefilter_search(w.rows[:k], w.queries[:k], di, sp, gp, cap_per_query=1 << 15)
    t_cpu_pre = time.perf_counter() - t0
    same = True
    for q in range(k):
        g = cands[cq == q].copy()
        g["query"] = q
        same &= bool(np.array_equal(g, cc[q]))
    sample = np.concatenate([cc[q] for q in range(k)]) if k else np.zeros(0, dtype=O.CANDIDATE_DTYPE)
    targets_s = np.unique(sample["target"]) if len(sample) else np.zeros(0, np.uint32)
    remap = {int(t): i for i, t in enumerate(targets_s)}
    arena = O.Arena(w.rows[:k], [w.db_residues[int(w.db_offsets[t]):int(w.db_offsets[t + 1])] for t in targets_s])
    t0 = time.perf_counter()
    cpu_scores = O.striped_pairs(arena, sample["query"], np.array([remap[int(t)] for t in sample["target"]],
                                                                  dtype=np.uint32), gaps.open, gaps.extend)
    t_cpu_sw = time.perf_counter() - t0
    gpu_s = np.concatenate([scores[cq == q] for q in range(k)]) if k else np.zeros(0, np.int32)
    same_scores = bool(same and np.array_equal(cpu_scores, gpu_s))
    ctx.free_profiles(ids)
    nq = len(ids)
    serving = search_serving(ctx, w, params, gaps, rates=(100, 500, 1000, 2000, 3000, 5000, 6500),
                             seconds=args.serving_seconds,
                             seed=args.seed, batched_qps=nq / (t_pre + t_sw))
    return {"workload": f"config 5 searches: {nq} sequence queries against {len(tlen)} targets ({n_res / 1e6:.0f} M "
                        f"residues), 5 planted homologs per query; seed 111001101, k-mer score 22, cap 512, exact "
                        f"seeds, gate {gate} (size-adjusted 42), gaps 11/1",
            "index_build_s": round(t_index, 3),
            "prefilter_ms": round(t_pre * 1e3, 1), "sw_ms": round(t_sw * 1e3, 1),
            "queries_per_s": round(nq / (t_pre + t_sw), 1), "prefilter_queries_per_s": round(nq / t_pre, 1),
            "hits": int(sst["postings_visited"]), "ghits_per_s": round(sst["postings_visited"] / t_pre / 1e9, 2),
            "candidates": int(len(cands)), "sw_cells": cells, "sw_gcups": round(cells / t_sw / 1e9, 1),
            "seed_stats": {k_: int(v) for k_, v in sst.items()},
            "gate_stats": {k_: int(v) for k_, v in st.items()},
            "matches_cpu_baseline": same, "sw_scores_match_cpu_baseline": same_scores,
            "cpu_baseline": {"value": round(k / (t_cpu_pre + t_cpu_sw), 2), "unit": "queries/s",
                             "cores": os.cpu_count(), "kind": "port",
                             "prefilter_s": round(t_cpu_pre, 2), "sw_s": round(t_cpu_sw, 2),
                             "index_build_s": round(t_cpu_index, 1),
                             "sample": f"{k} queries on the whole database: the restated seed stage (best-first "
                                       "similar k-mers, direct-table index), evidence and gate, then the reference's "
                                       "AVX2 striped SW over their candidates, all host threads"},
            "serving": serving,
            "setup_s": round(t_gen, 1)}


def search_serving(ctx, w, params, gaps, rates, seconds, seed, batched_qps):
    """Config 5 serving: Poisson arrivals of bare queries into a SearchServer (whole searches per batch on the
    device); latency from submit to completion as the server stamps it.  Then every query at once (the
    saturated rate) against the batched figure."""
    from sabertooth_b200 import SearchServer
    srv = SearchServer(ctx, params, gaps)
    rng = np.random.default_rng(seed)
    nq = len(w.rows)
    try:
        warm = [srv.submit(w.rows[q], w.queries[q]) for q in range(min(32, nq))]
        for r in warm:
            srv.wait(r)
        sweep = []
        for rate in rates:
            n = max(1, int(rate * seconds))
            t_arr = np.cumsum(rng.exponential(1.0 / rate, n))
            rids = []
            t0 = time.perf_counter()
            for k in range(n):
                delay = t_arr[k] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                q = k % nq
                rids.append(srv.submit(w.rows[q], w.queries[q]))
            lats = np.array([srv.wait(r)[2] for r in rids])
            t_end = time.perf_counter() - t0
            sweep.append({"rate_qps": rate, "queries": n, "p50_ms": round(float(np.percentile(lats, 50)), 2),
                          "p99_ms": round(float(np.percentile(lats, 99)), 2), "achieved_qps": round(n / t_end, 1)})
        b0 = srv.stats()["batches"]
        t0 = time.perf_counter()
        rids = [srv.submit(w.rows[q], w.queries[q]) for q in range(nq)]
        lats = np.array([srv.wait(r)[2] for r in rids])
        t_sat = time.perf_counter() - t0
        sat = {"queries": nq, "batches": srv.stats()["batches"] - b0, "qps": round(nq / t_sat, 1),
               "of_batched": round(nq / t_sat / batched_qps, 3), "p50_ms": round(float(np.percentile(lats, 50)), 1),
               "p99_ms": round(float(np.percentile(lats, 99)), 1)}
    finally:
        srv.close()
    return {"sweep": sweep, "saturated": sat}


def calibration_measure(ctx, args, w, ids, gaps):
    """Per-profile calibration (calibrate_profile, src/evalue.rs:714-748) of config-3 PSSMs as the reference's
    profile search runs it: 2,000 background samples per profile from the search seed 0x5EED, lengths from
    the database's length sample (every k-th record, SeedIndex::length_sample(2000), src/index.rs:2038-2042),
    gaps 44/4.  One st_calibrate_profiles call per step (targets generated on the device, all profiles scored
    in one batched call, ML fits on the host threads); cells = sum over profiles of m x sum of sample lengths."""
    from oracle import oracle as O
    from sabertooth_b200.matrix import blosum62
    n_db = len(w.db_offsets) - 1
    tl = np.diff(w.db_offsets.astype(np.int64))
    lengths = tl[::max(n_db // 2000, 1)].astype(np.uint32)
    samples, seed = 2000, 0x5EED
    sel = ids[:min(args.calib_profiles, len(ids))]
    m = np.array([len(r) for r in w.rows], dtype=np.int64)[:len(sel)]
    p_back = blosum62().p_back[:20]
    res = ctx.calibrate_profiles(sel, lengths, samples=samples, seed=seed, gaps=gaps, p_back=p_back)  # warm-up
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        res, sc = ctx.calibrate_profiles(sel, lengths, samples=samples, seed=seed, gaps=gaps, p_back=p_back,
                                         with_scores=True)
        ts.append(time.perf_counter() - t0)
    t_gpu = float(np.median(ts))
    targets = [O.calibration_target(lengths, seed, i, p_back) for i in range(samples)]
    cells = int(m.sum()) * int(sum(len(t) for t in targets))
    # CPU baseline: the reference's AVX2 striped kernels (u8 -> i16 -> scalar) restated in C over the same
    # targets for a sample of profiles, all host threads, plus the ML fits
    k = min(48, len(sel))
    arena = O.Arena([w.rows[i] for i in range(k)], targets)
    pq = np.repeat(np.arange(k, dtype=np.uint32), samples)
    pt = np.tile(np.arange(samples, dtype=np.uint32), k)
    t0 = time.perf_counter()
    cpu_sc = O.striped_pairs(arena, pq, pt, gaps.open, gaps.extend).reshape(k, samples)
    fits = [O.fit_gumbel_ml(cpu_sc[i].astype(np.float64)) for i in range(k)]
    t_cpu = time.perf_counter() - t0
    same_scores = bool(np.array_equal(cpu_sc, sc[:k]))
    same_fits = all((f is None and r is None) or (f is not None and r is not None and
                                                   abs(f[0] - r[0]) <= 1e-12 * abs(f[0]))
                    for f, r in zip(fits, res[:k]))
    return {"workload": f"config 3 PSSMs: {len(sel)} profiles x {samples} background samples (seed 0x5EED, lengths "
                        f"from every {max(n_db // 2000, 1)}th of {n_db} database records), gaps {gaps.open}/{gaps.extend}",
            "ms_per_call": round(t_gpu * 1e3, 2), "profiles_per_s": round(len(sel) / t_gpu, 1),
            "gcups": round(cells / t_gpu / 1e9, 1), "cells": cells,
            "fits_ok": int(sum(r is not None for r in res)),
            "matches_cpu_baseline": same_scores, "fits_match_cpu_baseline": bool(same_fits),
            "cpu_baseline": {"value": round(k / t_cpu, 2), "unit": "profiles/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": f"{k} profiles x {samples} samples: the reference's AVX2 "
                                                       "striped SW (u8 -> i16 -> scalar) restated in C over all host "
                                                       "threads, plus the ML Gumbel fits"}}


def gate_measure(ctx, args):
    """Prefilter evidence -> chain -> gate (score_and_gate, src/prefilter.rs:1412-1660, ranking :1074-1083) on
    seed hits with query positions over the config-2 database shape: 1,000 queries, 374,000 targets (68 M
    residues), 2x10^7 hits (30% on two-piece planted homologs), sequence defaults (4 diagonals, window 48,
    span 6, gate 42, gaps 11/1), regions on.  Device-resident hits per step: one st_prefilter_gate_device call
    (sort, groups, top diagonals, segments, chains, gate, ranking).  e2e: st_prefilter_gate from host hits to
    host candidates, the hits in pinned host memory (and, reported beside, in a pageable array).  Algorithmic bytes: 16 B per hit + the residues of every scored window + 32 B per
    candidate, against the measured HBM copy bandwidth."""
    import torch
    from oracle import oracle as O
    from sabertooth_b200 import GapCosts, PrefilterParams
    from synth import workloads as W
    t0 = time.perf_counter()
    w = W.seed_hits(seed=args.seed, n_hits=args.gate_hits)
    t_gen = time.perf_counter() - t0
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    hits = w.hits.copy()
    hits["query"] = ids[hits["query"]]
    n = len(hits)
    params = PrefilterParams(regions=True)
    gaps = GapCosts.sequence_default()
    st = torch.cuda.Stream()
    ctx.set_stream(st.cuda_stream)
    d_hits = torch.from_numpy(hits.view(np.uint8)).cuda()
    d_out = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        for _ in range(3):
            n_c, stats = ctx.prefilter_gate_device(d_hits.data_ptr(), n, d_out.data_ptr(), params, gaps)
        ts = []
        for _ in range(max(3, args.steps)):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            n_c, stats = ctx.prefilter_gate_device(d_hits.data_ptr(), n, d_out.data_ptr(), params, gaps)
            b.record(st)
            st.synchronize()
            ts.append(a.elapsed_time(b))
    got_dev = d_out[:n_c * 32].cpu().numpy().view(O.CANDIDATE_DTYPE)
    ctx.set_stream(0)
    ms = float(np.median(ts))
    # e2e: host hits in (from pinned host memory, as a serving caller holds them; and from a pageable
    # array, staged through pinned blocks by the library), host candidates out
    hits_pin = torch.empty(hits.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(hits.dtype)
    hits_pin[:] = hits
    te, tp = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        got, _ = ctx.prefilter_gate(hits_pin, params, gaps)
        te.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        got_p, _ = ctx.prefilter_gate(hits, params, gaps)
        tp.append(time.perf_counter() - t0)
    ms_e2e = float(np.median(te)) * 1e3
    ms_e2e_pageable = float(np.median(tp)) * 1e3
    same_pageable = bool(np.array_equal(got, got_p))
    del hits_pin
    # CPU baseline: the oracle's restatement of the reference's evidence stage with its AVX2 batched Kadane,
    # queries in parallel over all host threads, on the whole workload; its candidates are the parity check
    targets = [w.db_residues[int(a_):int(b_)] for a_, b_ in zip(w.db_offsets[:-1], w.db_offsets[1:])]
    arena = O.Arena(w.rows, targets)
    p = {"min_hits": params.min_hits, "diag_hits": params.diag_hits, "max_diagonals": params.max_diagonals,
         "diag_window": params.diag_window, "span": params.span, "min_diag_score": params.min_diag_score,
         "gap_open": gaps.open, "gap_ext": gaps.extend, "max_candidates": params.max_candidates, "regions": 1}
    t_runs = []
    for _ in range(2):
        t0 = time.perf_counter()
        want, wst = O.prefilter_queries(arena, w.hits["query"], w.hits["target"], w.hits["diag"], w.hits["qpos"], p)
        t_runs.append(time.perf_counter() - t0)
    t_cpu = float(np.median(t_runs))
    mapped = got.copy()
    inv = np.zeros(int(ids.max()) + 1, dtype=np.int64)
    inv[ids] = np.arange(len(ids))
    mapped["query"] = inv[got["query"]]
    order = np.argsort(mapped["query"], kind="stable")
    same = bool(len(mapped) == len(want) and np.array_equal(mapped[order], want))
    same_stats = all(stats[k] == wst[k] for k in wst)
    # algorithmic bytes: hits, scored windows, candidates
    win = gate_window_bytes(w, params)
    ab = 16 * n + win + 32 * int(n_c)
    peak = hbm_peak_gbs()
    gbs = ab / (ms * 1e-3) / 1e9
    ctx.free_profiles(ids)
    return {"workload": f"seed hits: {len(w.rows)} queries, {len(w.db_offsets) - 1} targets "
                        f"({int(w.db_offsets[-1]) / 1e6:.1f} M residues), {n} hits (30% on two-piece homologs); "
                        "sequence defaults, regions on",
            "ms_per_step": round(ms, 3), "mhits_per_s": round(n / ms / 1e3, 1),
            "e2e": {"ms_per_call": round(ms_e2e, 3), "mhits_per_s": round(n / ms_e2e / 1e3, 1),
                    "h2d_bytes_per_step": int(16 * n), "d2h_bytes_per_step": int(32 * int(n_c)),
                    "inputs": "pinned host hits",
                    "pageable": {"ms_per_call": round(ms_e2e_pageable, 3),
                                 "mhits_per_s": round(n / ms_e2e_pageable / 1e3, 1),
                                 "matches_pinned": same_pageable}},
            "candidates": int(n_c), "stats": {k: int(v) for k, v in stats.items()},
            "algorithmic_bytes": int(ab),
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "traffic": None},
            "matches_cpu_baseline": same, "stats_match_cpu_baseline": same_stats,
            "device_matches_host": bool(np.array_equal(got_dev, got)),
            "cpu_baseline": {"value": round(n / t_cpu / 1e6, 2), "unit": "Mhits/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": f"the whole workload ({n} hits), median of 2 runs: the "
                                                       "reference's evidence stage (hits sorted per query, top "
                                                       "diagonals, AVX2 batched Kadane, lazy segment positions, "
                                                       "chains, gate, ranking) restated in C, queries in parallel "
                                                       "over all host threads"},
            "setup_s": round(t_gen, 1)}


def gate_window_bytes(w, params):
    """Residues of every scored window: per (query, target), its top diagonals by hit count (at most
    max_diagonals, ties to the smaller diagonal), each over [qmin - window, qmax + span + window) clipped
    to the diagonal."""
    h = w.hits
    q = h["query"].astype(np.int64)
    t = h["target"].astype(np.int64)
    d = h["diag"].astype(np.int64)
    qp = h["qpos"].astype(np.int64)
    order = np.lexsort((d, t, q))
    q, t, d, qp = q[order], t[order], d[order], qp[order]
    run = np.ones(len(q), dtype=bool)
    run[1:] = (q[1:] != q[:-1]) | (t[1:] != t[:-1]) | (d[1:] != d[:-1])
    idx = np.nonzero(run)[0]
    cnt = np.diff(np.append(idx, len(q)))
    qmin = np.minimum.reduceat(qp, idx)
    qmax = np.maximum.reduceat(qp, idx)
    rq, rt, rd = q[idx], t[idx], d[idx]
    # rank of each run inside its (query, target) by count desc, diagonal asc
    o2 = np.lexsort((rd, -cnt, rt, rq))
    rq, rt, rd, cnt, qmin, qmax = rq[o2], rt[o2], rd[o2], cnt[o2], qmin[o2], qmax[o2]
    grp = np.ones(len(rq), dtype=bool)
    grp[1:] = (rq[1:] != rq[:-1]) | (rt[1:] != rt[:-1])
    gstart = np.maximum.accumulate(np.where(grp, np.arange(len(rq)), 0))
    keep = (np.arange(len(rq)) - gstart) < min(params.max_diagonals, 16)
    m = np.array([len(r) for r in w.rows], dtype=np.int64)[rq]
    nl = np.diff(w.db_offsets.astype(np.int64))[rt]
    lo = np.maximum(np.maximum(-rd, 0), np.maximum(qmin - params.diag_window, 0))
    hi = np.minimum(np.minimum(m, nl - rd), qmax + params.span + params.diag_window)
    return int(np.maximum(hi - lo, 0)[keep].sum())


def _timed_plans(ctx, plans, steps, warmup=3, concurrent=False):
    """Device time of one step = every plan run once, L2 flushed before each step; the plans run one after
    the other on one stream, or (concurrent) each on its own stream forked from the timing stream and joined
    back before the end event, as independent batches in flight together run."""
    import torch
    st = torch.cuda.Stream()
    side = [torch.cuda.Stream() for _ in plans] if concurrent else []
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        if not concurrent:
            ctx.set_stream(st.cuda_stream)
            for p in plans:
                p.run()
            return
        for p, s_ in zip(plans, side):
            s_.wait_stream(st)
            ctx.set_stream(s_.cuda_stream)
            p.run()
        for s_ in side:
            st.wait_stream(s_)

    ts = []
    with torch.cuda.stream(st):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        for _ in range(max(3, steps)):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            step()
            b.record(st)
            st.synchronize()
            ts.append(a.elapsed_time(b))
    ctx.set_stream(0)
    return ts


def exhaustive_measure(ctx, args):
    """Config 1, plain exhaustive SW-Gotoh (easysearch-style): every one of 200 BLOSUM62 queries against every
    one of 20,000 targets (lengths lognormal median 250, 30-1,000; 10% planted homologs at ~40% identity),
    gaps 11/1, an int32 score per pair (4x10^6 scores).  One step = one run of the captured plan; the scores
    are compared with the CPU port's over the whole workload."""
    import torch
    from oracle import oracle as O
    from sabertooth_b200 import GapCosts
    from sabertooth_b200._lib import PAIR_DTYPE
    from synth import workloads as W
    t0 = time.perf_counter()
    w = W.config1(seed=args.seed, n_queries=args.exhaustive_queries)
    t_gen = time.perf_counter() - t0
    gaps = GapCosts(w.gap_open, w.gap_extend)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
    pairs["profile"] = ids[w.pair_q]
    pairs["target"] = w.pair_t
    pairs["band_radius"] = -1
    d_s = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    d_k = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    plan = ctx.plan(pairs, gaps, d_s.data_ptr(), d_k.data_ptr())
    ts = _timed_plans(ctx, [plan], args.steps)
    stats = plan.stats()
    plan.close()
    got = d_s.cpu().numpy()
    kern = d_k.cpu().numpy()
    # end to end: host pairs in, scores out (profiles resident); one untimed call (its staging blocks and
    # device arenas are allocated there), then the median of three
    e2e = ctx.sw_score_pairs(pairs, gaps)
    e2e_ok = True
    e2e_t = []
    for _ in range(3):
        t0 = time.perf_counter()
        e2e_run = ctx.sw_score_pairs(pairs, gaps)
        e2e_t.append(time.perf_counter() - t0)
        e2e_ok &= bool(np.array_equal(e2e_run, e2e))
    t_e2e = float(np.median(e2e_t))
    ctx.free_profiles(ids)
    cells = w.cells()
    t0 = time.perf_counter()
    want = O.striped_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 11, 1, threads=os.cpu_count())
    t_cpu = time.perf_counter() - t0
    ms = float(np.median(ts))
    return {"workload": f"config 1: {len(w.rows)} BLOSUM62 queries x {len(w.db_offsets) - 1} targets "
                        f"({w.n_pairs:,} pairs, exhaustive), gaps 11/1",
            "cells": int(cells), "ms_per_step": round(ms, 3), "gcups": round(cells / (ms * 1e-3) / 1e9, 1),
            "e2e_gcups": round(cells / t_e2e / 1e9, 1), "e2e_how": "one st_sw_score_pairs call: host pairs in, "
                                                                 "scores out, profiles and database resident; "
                                                                 "median of three calls after an untimed one",
            "rescored_pairs": int(stats["rescored_pairs"]), "gpu32_pairs": int((kern == 2).sum()),
            "matches_cpu_baseline": bool(np.array_equal(got, want)),
            "e2e_matches": bool(np.array_equal(e2e, want)) and e2e_ok,
            "cpu_baseline": {"value": round(cells / t_cpu / 1e9, 2), "unit": UNIT, "cores": os.cpu_count(),
                             "kind": "port", "sample": "the whole workload once: the reference's default AVX2 path "
                                                       "(u8 -> i16 striped -> scalar) restated in C"},
            "setup_s": round(t_gen, 1)}


def long_mix_measure(ctx, args):
    """Config 4, the long/overflow mix: half BLOSUM62 (11/1) and half PSSM (44/4) pairs, targets 1,000-35,000
    residues (10% above 10,000), queries lognormal median 250 (30-2,000), 5% near-identical planted pairs, pairs
    with a length ratio above 4 scored in the band of radius 64 around the planted diagonal (0 when unplanted,
    src/align.rs:439-447).  One step = both halves' plans, in flight together on two streams (two gap settings,
    two independent batches).  Cells: m*n for full pairs plus the in-band cells of
    banded pairs.  Every score is compared with the CPU oracle's (the scalar band rule for banded pairs, the AVX2
    port for full pairs)."""
    import torch
    from oracle import oracle as O
    from sabertooth_b200 import GapCosts
    from sabertooth_b200._lib import PAIR_DTYPE
    from synth import workloads as W
    half = max(1, args.long_pairs // 2)
    t0 = time.perf_counter()
    halves = [W.config4(seed=args.seed, n_pairs=half, kind="blosum62"),
              W.config4(seed=args.seed, n_pairs=half, kind="pssm")]
    t_gen = time.perf_counter() - t0
    seqs = halves[0].targets() + halves[1].targets()
    ctx.upload_db_list(seqs)
    ids = ctx.create_profiles(halves[0].rows + halves[1].rows)
    plans, outs, infos = [], [], []
    q_base, t_base = 0, 0
    for w in halves:
        pairs = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
        pairs["profile"] = ids[q_base + w.pair_q.astype(np.int64)]
        pairs["target"] = t_base + w.pair_t
        pairs["band_center"] = w.band_center
        pairs["band_radius"] = w.band_radius
        d_s = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
        d_k = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
        plans.append(ctx.plan(pairs, GapCosts(w.gap_open, w.gap_extend), d_s.data_ptr(), d_k.data_ptr()))
        outs.append((d_s, d_k))
        q_base += len(w.rows)
        t_base += len(w.db_offsets) - 1
    ts = _timed_plans(ctx, plans, args.steps, concurrent=True)
    stats = [p.stats() for p in plans]
    profiles = [[{"tile": (f"G{sh[0]}xR{sh[1]}xC{sh[2]}" if isinstance(sh, tuple) else sh), "cells": c, "ms": round(t, 3)}
                 for sh, c, t in p.profile()] for p in plans]
    for p in plans:
        p.close()
    ctx.free_profiles(ids)
    res = {"workload": f"config 4: {sum(w.n_pairs for w in halves):,} pairs, half BLOSUM62 11/1 and half PSSM 44/4, "
                       "targets 1,000-35,000, band 64 for length ratio > 4", "halves": []}
    cells_tot, ok_all, cpu_s = 0, True, 0.0
    for w, (d_s, d_k), stt in zip(halves, outs, stats):
        got = d_s.cpu().numpy()
        kern = d_k.cpu().numpy()
        banded = w.band_radius >= 0
        m = np.array([len(r) for r in w.rows], dtype=np.int64)[w.pair_q]
        n = np.diff(w.db_offsets.astype(np.int64))[w.pair_t]
        full_cells = int((m[~banded] * n[~banded]).sum())
        cells = w.cells()
        ar = O.Arena(w.rows, w.targets())
        want = np.zeros(w.n_pairs, dtype=np.int32)
        t0 = time.perf_counter()
        fi = np.nonzero(~banded)[0]
        bi = np.nonzero(banded)[0]
        want[fi] = O.striped_pairs(ar, w.pair_q[fi], w.pair_t[fi], w.gap_open, w.gap_extend,
                                   threads=os.cpu_count())
        want[bi] = O.sw_pairs(ar, w.pair_q[bi], w.pair_t[bi], w.gap_open, w.gap_extend, w.band_center[bi],
                              w.band_radius[bi], threads=os.cpu_count())
        cpu_s += time.perf_counter() - t0
        ok = bool(np.array_equal(got, want))
        ok_all &= ok
        cells_tot += cells
        res["halves"].append({"kind": w.name, "pairs": int(w.n_pairs), "banded_pairs": int(banded.sum()),
                              "planted_pairs": int(w.info["planted"]), "cells": int(cells),
                              "full_pair_cells": full_cells, "in_band_cells": int(cells - full_cells),
                              "rescored_pairs": int(stt["rescored_pairs"]), "gpu32_pairs": int((kern == 2).sum()),
                              "launch_profile": profiles[len(res["halves"])], "matches_cpu_baseline": ok})
    ms = float(np.median(ts))
    res.update({"cells": int(cells_tot), "ms_per_step": round(ms, 3),
                "gcups": round(cells_tot / (ms * 1e-3) / 1e9, 1), "matches_cpu_baseline": bool(ok_all),
                "cpu_baseline": {"value": round(cells_tot / cpu_s / 1e9, 2), "unit": UNIT, "cores": os.cpu_count(),
                                 "kind": "port", "sample": "the whole workload once: the AVX2 striped port for full "
                                                           "pairs, the scalar band rule for banded pairs"},
                "setup_s": round(t_gen, 1)})
    return res


def hbm_peak_gbs():
    """The measured copy bandwidth of this pool's B200s, or the fallback figure."""
    return hbm_peak()[0]


def hbm_peak():
    """(GB/s, source): MEASURED_PEAKS.json's measured copy bandwidth when the file is present, else the
    pool's earlier measurement (6.65 TB/s)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s, an earlier copy-bandwidth measurement on this pool)"


def serving_measure(ctx, args):
    """The serving loop (st_server_*) on the long/overflow mix (config 4, both halves: BLOSUM62 rows at 11/1 and
    PSSM rows at 44/4, one server per gap setting on the same context): one request per pair (query rows + a
    target of 1,000-35,000 residues, banded when the length ratio is above 4).  Poisson arrivals at swept
    rates, spread over both halves, give p50/p99 latency (submit to completion); all requests at once give the
    saturated throughput, compared with one batched call per half over the same pairs (profile build and free
    included in both)."""
    import threading
    from sabertooth_b200 import GapCosts, Server
    from sabertooth_b200._lib import PAIR_DTYPE
    from synth import workloads as W
    half = max(1, args.serving_pairs // 2)
    ws = [W.config4(seed=args.seed, n_pairs=half, kind="blosum62"), W.config4(seed=args.seed, n_pairs=half, kind="pssm")]
    gaps = [GapCosts(w.gap_open, w.gap_extend) for w in ws]
    ctx.upload_db_list(ws[0].targets() + ws[1].targets())
    tbase = [0, len(ws[0].db_offsets) - 1]
    cells = sum(w.cells() for w in ws)
    per_cells = [np.array([w.cells_of(i) for i in range(w.n_pairs)], dtype=np.float64) for w in ws]
    nrows = [np.array([len(r) for r in w.rows], dtype=np.uint64) for w in ws]
    # batched reference: every request of a half in one batch, profiles built and freed inside the timing as
    # the server does
    want = [None, None]
    times = []
    arenas, row_offs, bpairs = [], [], []
    for h, w in enumerate(ws):  # the inputs as a caller holds them: one rows arena and one pair array per half
        ro = np.zeros(len(w.rows) + 1, dtype=np.uint64)
        ro[1:] = np.cumsum(nrows[h])
        arenas.append(np.concatenate(w.rows).astype(np.int32))
        row_offs.append(ro)
        pairs = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
        pairs["target"] = tbase[h] + w.pair_t
        pairs["band_center"] = w.band_center
        pairs["band_radius"] = w.band_radius
        bpairs.append(pairs)
    for rep in range(4):
        # both halves in flight at once (asynchronous batches), as two servers on one context run them
        t0 = time.perf_counter()
        live = []
        for h, w in enumerate(ws):
            ids = ctx.create_profiles_arena(arenas[h], row_offs[h])
            bpairs[h]["profile"] = ids[w.pair_q]
            live.append((ids, ctx.sw_score_pairs_async(bpairs[h], gaps[h])))
        for h, (ids, bt) in enumerate(live):
            got = bt.wait()
            ctx.free_profiles(ids)
            want[h] = got if want[h] is None else want[h]
        times.append(time.perf_counter() - t0)
    batched_gcups = cells / float(np.median(times[1:])) / 1e9
    srv = [Server(ctx, g) for g in gaps]
    ok = True
    t_offs = [np.arange(w.n_pairs + 1, dtype=np.uint64) for w in ws]

    def burst(h, order):
        """The requests `order` of half h as one bulk submission, built before the clock starts."""
        w = ws[h]
        q = w.pair_q[order]
        ro = np.zeros(len(order) + 1, dtype=np.uint64)
        ro[1:] = np.cumsum(nrows[h][q])
        arena = np.concatenate([w.rows[int(j)] for j in q]).astype(np.int32)
        return (arena, ro, np.ascontiguousarray(tbase[h] + w.pair_t[order]).astype(np.uint32),
                t_offs[h][:len(order) + 1], np.ascontiguousarray(w.band_center[order]),
                np.ascontiguousarray(w.band_radius[order]))

    for h in range(2):  # warm-up: pools, pinned blocks, streams
        for rid in srv[h].submit_many(*burst(h, np.arange(min(250, ws[h].n_pairs)))):
            srv[h].wait(rid)

    def run(order, arrivals):
        """order: (half, pair) requests in arrival order."""
        nonlocal ok
        rids = [None] * len(order)
        lat = np.zeros(len(order))

        def waiter():
            nonlocal ok
            for k, (h, i) in enumerate(order):
                while rids[k] is None:
                    time.sleep(0.0002)
                s_, lat[k] = srv[h].wait(rids[k])
                ok &= bool(s_[0] == want[h][i])

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        for k, (h, i) in enumerate(order):
            if arrivals is not None:
                dt = t0 + arrivals[k] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
            w = ws[h]
            rids[k] = srv[h].submit(w.rows[w.pair_q[i]], tbase[h] + w.pair_t[i:i + 1], w.band_center[i:i + 1],
                                    w.band_radius[i:i + 1])
        th.join()
        wall = time.perf_counter() - t0
        c = float(sum(per_cells[h][i] for h, i in order))
        return {"requests": len(order), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2), "gcups": round(c / wall / 1e9, 2),
                "q_per_s": round(len(order) / wall, 1)}

    rng = np.random.default_rng(args.seed + 11)
    everyone = [(h, i) for h in range(2) for i in range(ws[h].n_pairs)]
    rates = []
    for rate in (50, 200, 1000, 2000):
        n = int(min(len(everyone), max(40, rate * args.serving_seconds)))
        pick = rng.choice(len(everyone), size=n, replace=False)
        order = [everyone[int(k)] for k in pick]
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
        rates.append(dict(rate_q_per_s=rate, **run(order, arrivals)))
    # saturated: every request arrives at once (one bulk submit per half); throughput from the first submit to
    # the last completion, both stamped inside the servers (one unmeasured round first: the servers' pinned
    # arenas grow to the burst's size)
    bursts = [burst(h, np.arange(ws[h].n_pairs)) for h in range(2)]
    for rnd in range(3):
        rids = [srv[h].submit_many(*bursts[h]) for h in range(2)]
        lat = []
        for h in range(2):
            for i, rid in enumerate(rids[h]):
                s_, l_ = srv[h].wait(rid)
                lat.append(l_)
                ok &= bool(s_[0] == want[h][i])
        lat = np.array(lat)
        wall = float(lat.max()) * 1e-3
    n_all = sum(w.n_pairs for w in ws)
    sat = {"requests": int(n_all), "p50_ms": round(float(np.percentile(lat, 50)), 2),
           "p99_ms": round(float(np.percentile(lat, 99)), 2), "gcups": round(cells / wall / 1e9, 2),
           "q_per_s": round(n_all / wall, 1)}
    stats = [s_.stats() for s_ in srv]
    for s_ in srv:
        s_.close()
    return {"workload": f"config 4 mix: {ws[0].n_pairs} BLOSUM62 (11/1) + {ws[1].n_pairs} PSSM (44/4) requests "
                        f"(query lognormal median 250, target 1,000-35,000, "
                        f"{ws[0].info['banded'] + ws[1].info['banded']} banded with radius 64)",
            "cells": int(cells), "batched_gcups": round(batched_gcups, 2),
            "batched_how": "one asynchronous st_sw_score_pairs per half over every request, both halves in flight "
                           "together, profile build and free included",
            "poisson": rates, "saturated": dict(sat, frac_of_batched=round(sat["gcups"] / batched_gcups, 3)),
            "batches": int(sum(st["batches"] for st in stats)), "matches_batched": bool(ok),
            "latency": "submit to completion inside the server (C++ steady clock)"}

if __name__ == "__main__":
    sys.exit(main())
