"""Benchmark of the cuda backend's database scan (GCUPS), one JSON line on rank 0.

Workload (one "step"): the protein SW ScoreEnd scan of 16 queries (lengths 100, 250, 500, 1000,
5000 cycled) against a resident database of 500,000 sequences (log-normal lengths, median 300,
sigma 0.8, clipped to 20..35,000; residues i.i.d. from a fixed seeded background; a seeded
symmetric 20x20 matrix with diagonal U[4,11] and off-diagonal U[-4,3]; gap_open 11, gap_ext 1).
All inputs are seeded synthetic data of that shape. GCUPS counts real cells only:
sum over queries and targets of |q| * |t| per second.

`value` is timed on the device (CUDA events on the scan's stream, inputs resident in HBM);
`e2e` goes through the public host API (hy_scan: query host->device, hit device->host per call).
Under torchrun each rank holds its own 500,000-sequence shard of an N-times larger database
(weak scaling) through hyalite_b200.sharded.ShardedDatabase: the per-shard best hits are
all-gathered over NCCL and reduced with the reference's tie-break (highest score, then smallest
global index).

--impl reference times the CPU baseline instead: a C++ restatement of hyalite's AVX2 backend
(oracle/avx2_port.cpp) over all host threads, on a bounded sample of the same database.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

QUERY_LENGTHS = [100, 250, 500, 1000, 5000]
N_QUERIES = 16
N_SEQS = 500_000
GO, GE = 11, 1
AL = 20
# DRAM bytes (read + write) per DP cell of the int16x2 pair kernel, from one ncu capture of
# scan_kernel<Pair16, 8, 16> (two-column sweep) on 400,000 sequences x one 1000-residue query:
# 0.537e9 + 1.285e9 bytes for 1.655e11 cells. The traffic is the boundary rows between query
# passes plus the residues, so it grows with cells at a fixed rows-per-pass; profiles/ holds the
# capture's summary and command.
DRAM_BYTES_PER_CELL = (0.537e9 + 1.285e9) / 1.655e11


def make_workload(seed: int, n_seqs: int = N_SEQS):
    """The protein workload generator: seeded matrix, background, lengths, residues and queries."""
    rng = np.random.default_rng(seed)
    base = np.random.default_rng(12345)  # the matrix and background are fixed across shards
    mat = base.integers(-4, 4, size=(AL, AL))
    mat = np.triu(mat) + np.triu(mat, 1).T
    mat[np.diag_indices(AL)] = base.integers(4, 12, size=AL)
    background = base.dirichlet(np.full(AL, 4.0))
    lengths = np.clip(np.round(np.exp(math.log(300.0) + 0.8 * rng.standard_normal(n_seqs))), 20, 35_000).astype(np.int64)
    offsets = np.zeros(n_seqs + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lengths)
    residues = rng.choice(AL, size=int(offsets[-1]), p=background).astype(np.uint8)
    qrng = np.random.default_rng(777)
    queries = [qrng.choice(AL, size=QUERY_LENGTHS[i % len(QUERY_LENGTHS)], p=background).astype(np.uint8)
               for i in range(N_QUERIES)]
    return mat.reshape(-1).astype(np.int32), residues, offsets, queries


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample(residues, offsets, first, count):
    """Sequences [first, first + count) of the database as (residues, offsets)."""
    off = offsets[first: first + count + 1]
    return residues[int(off[0]): int(off[-1])], off - off[0]


def cpu_baseline_run(mat, residues, offsets, queries, sample_seqs, threads, steps=1, warmup=0):
    """The AVX2 restatement over `threads` host threads: the queries against consecutive samples
    of `sample_seqs` sequences (step k takes the k-th sample, wrapping over the database), each
    sample held in slices so that every (query, slice) unit runs on the next free thread, longest
    query first (no thread idles on a long query). Returns (GCUPS, seconds per step, sample
    description, one-query-per-thread GCUPS on the first sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    n = len(offsets) - 1
    n_samples = max(1, n // sample_seqs)
    mql = max(len(q) for q in queries)
    qlist = [list(map(int, q)) for q in queries]
    qres = float(sum(len(q) for q in queries))
    cells = secs = 0.0
    per_thread = None
    for k in range(warmup + steps):
        first = (k % n_samples) * sample_seqs
        res, off = cpu_sample(residues, offsets, first, sample_seqs)
        db = pyoracle.Avx2SlicedDb(res, off, mat, AL, GO, GE, 0, 1, mql, n_slices=4 * threads)
        t0 = time.perf_counter()
        db.scan_stream(qlist, threads)
        dt = time.perf_counter() - t0
        if k >= warmup:
            cells += qres * float(off[-1])
            secs += dt
        if k == 0 and steps <= 2:
            # The same sample with one query per thread (the reference's one Scratch per thread and
            # a stream of whole queries): long queries leave the other threads idle.
            whole = pyoracle.Avx2Db(res, off, mat, AL, GO, GE, 0, 1, mql)
            t0 = time.perf_counter()
            whole.scan_many(qlist, threads)
            per_thread = qres * float(off[-1]) / (time.perf_counter() - t0) / 1e9
    desc = (f"{len(queries)} queries ({'/'.join(map(str, QUERY_LENGTHS))} aa, cycled) against "
            f"{min(steps, n_samples)} consecutive sample(s) of {sample_seqs} of the {n} sequences, "
            f"{4 * threads} slices each, (query, slice) units over {threads} threads")
    return cells / secs / 1e9, secs / steps, desc, per_thread


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    mat, residues, offsets, queries = make_workload(args.seed, n_seqs=args.ref_seqs)
    threads = os.cpu_count() or 1
    gcups, dt, sample, _ = cpu_baseline_run(mat, residues, offsets, queries, args.ref_sample_seqs, threads,
                                            steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": "GCUPS", "value": gcups, "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "i8/i16/i32 lanes (AVX2)", "data": "synthetic",
        "config": {"workload": "protein SW ScoreEnd scan, 500k log-normal sequences x 16 queries (100..5000), "
                               "AVX2 port on bounded samples of a 100,000-sequence subsample",
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_cuda(args):
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import hyalite_b200 as hy
    from hyalite_b200 import _abi

    lib = _abi.lib
    # This rank's shard: block `rank` of an N-times larger database (global sequences
    # [rank * n_seqs, (rank + 1) * n_seqs)), generated here from its own seed.
    mat, residues, offsets, queries = make_workload(args.seed + rank, n_seqs=N_SEQS)
    n_seqs = len(offsets) - 1

    def configure(b):
        return (b.scoring(hy.Scoring(AL, mat, GO, GE)).mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd)
                .max_query_len(max(QUERY_LENGTHS)))

    t_build = time.perf_counter()
    sdb = None
    if world > 1:
        from hyalite_b200 import sharded

        sdb = sharded.ShardedDatabase.from_shard(residues, offsets, np.arange(n_seqs) + rank * n_seqs,
                                                 world * n_seqs, configure)
        db = sdb.db
    else:
        db = configure(hy.Database.builder().sequences_concat(residues, offsets)).build()
    build_s = time.perf_counter() - t_build
    sc = hy.Scratch(db)
    n16, n32 = db.partition()
    total_res = float(offsets[-1])
    cells_step = float(sum(len(q) for q in queries)) * total_res  # this rank's shard
    # i16/i32 residue split for the roofline's per-launch cells
    lens = np.diff(offsets.astype(np.int64))

    stream = torch.cuda.ExternalStream(sc.stream_ptr())
    d_queries = [torch.from_numpy(q).to(f"cuda:{local}") for q in queries]
    d_hits = torch.zeros((N_QUERIES, 32), dtype=torch.uint8, device=f"cuda:{local}")
    torch.cuda.synchronize()

    def device_step():
        for i, q in enumerate(d_queries):
            st = lib.hy_scan_device(db._h, sc._h, C.c_void_p(q.data_ptr()), len(queries[i]),
                                    C.c_void_p(d_hits[i].data_ptr()))
            if st != 0:
                raise hy.Error.from_status(st)

    def gather_best(hits_dev):
        """The per-query best hits of all shards, merged on the device (one all_gather)."""
        if world == 1:
            return hits_dev
        with torch.cuda.stream(stream):
            return sdb.merge_device_hits(hits_dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        device_step()
        gather_best(d_hits)
    barrier()
    clocks = Clocks(local)
    clocks.start()
    lib.hy_scratch_profile(sc._h, 1)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        device_step()
        gather_best(d_hits)
    end.record(stream)
    torch.cuda.synchronize()
    kms = (C.c_double * 3)()
    kl = (C.c_uint64 * 3)()
    kcells = (C.c_double * 3)()
    all_l = C.c_uint64()
    lib.hy_scratch_profile_read(sc._h, kms, kl, kcells, C.byref(all_l))
    lib.hy_scratch_profile(sc._h, 0)
    clk = clocks.stop()
    elapsed_ms = start.elapsed_time(end)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([elapsed_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    barrier()

    # ---- e2e: the public host API, host buffers, copies inside the timed region ----
    host_queries = [bytes(q) for q in queries]
    for _ in range(1):
        for q in host_queries:
            db.scan(sc, q)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        hits = [(sdb or db).scan(sc, q) for q in host_queries]
    e2e_s = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # ---- per query length: each query alone (synchronised), kernel times by class ----
    by_len = {}
    for i, q in enumerate(d_queries):
        lib.hy_scratch_profile(sc._h, 1)
        st = lib.hy_scan_device(db._h, sc._h, C.c_void_p(q.data_ptr()), len(queries[i]),
                                C.c_void_p(d_hits[i].data_ptr()))
        if st != 0:
            raise hy.Error.from_status(st)
        qms, ql, qc = (C.c_double * 3)(), (C.c_uint64 * 3)(), (C.c_double * 3)()
        lib.hy_scratch_profile_read(sc._h, qms, ql, qc, None)
        e = by_len.setdefault(len(queries[i]), {"queries": 0, "bulk_ms": 0.0, "bulk_cells": 0.0,
                                                "int32_ms": 0.0, "int32_cells": 0.0, "long_ms": 0.0})
        e["queries"] += 1
        e["bulk_ms"] += qms[0]
        e["bulk_cells"] += qc[0]
        e["int32_ms"] += qms[1]
        e["int32_cells"] += qc[1]
        e["long_ms"] += qms[2]
    lib.hy_scratch_profile(sc._h, 0)
    for e in by_len.values():
        e["bulk_gcups"] = e["bulk_cells"] / (e["bulk_ms"] * 1e-3) / 1e9 if e["bulk_ms"] > 0 else None
        e["int32_gcups"] = e["int32_cells"] / (e["int32_ms"] * 1e-3) / 1e9 if e["int32_ms"] > 0 else None

    # ---- roofline of the dominant kernel (int16x2 pair kernel) ----
    peak = C.c_double()
    lib.hy_measure_dpx_peak(C.byref(peak))
    peak_gcups = peak.value / 1e9
    # The dominant kernel is the int16x2 pair kernel: its real cells per launch over its average
    # launch time (CUDA events on its own stream).
    launches16 = max(int(kl[0]), 1)
    cells16_per_launch = kcells[0] / launches16
    avg16_ms = kms[0] / launches16
    achieved = cells16_per_launch / (avg16_ms * 1e-3) / 1e9 if avg16_ms > 0 else 0.0
    def _kinfo(i):
        return {"launches": int(kl[i]), "ms_per_step": kms[i] / args.steps, "cells_per_step": kcells[i] / args.steps,
                "gcups": kcells[i] / (kms[i] * 1e-3) / 1e9 if kms[i] > 0 else None}
    kernels = {"bulk_int16x2_pairs": _kinfo(0), "long_int16x2_pairs": _kinfo(2), "int32_items": _kinfo(1),
               "by_query_length_alone": {str(k): v for k, v in sorted(by_len.items())}}
    meas = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = meas.get("hbm_gbs", 6650.0)

    total_cells = cells_step * args.steps * world
    value = total_cells / (elapsed_ms * 1e-3) / 1e9
    e2e_value = total_cells / e2e_s / 1e9

    if rank == 0:
        threads = os.cpu_count() or 1
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            g, dt, sample, per_thread = cpu_baseline_run(mat, residues, offsets, queries, args.cpu_sample_seqs,
                                                         threads)
            cpu = {"value": g, "unit": "GCUPS", "cores": threads, "kind": "port", "sample": sample,
                   "one_query_per_thread": {"value": per_thread, "unit": "GCUPS",
                                            "form": "the same sample, each thread one whole query at a time"}}
        line = {
            "metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i16x2 (int32 for long sequences)",
            "data": "synthetic (seeded protein generator: log-normal lengths, fixed background)",
            "config": {
                "workload": "protein SW ScoreEnd scan, 500k log-normal sequences x 16 queries (100..5000), plain per-query form",
                "n_seqs_per_gpu": n_seqs, "residues_per_gpu": int(total_res), "queries_per_step": N_QUERIES,
                "query_lengths": QUERY_LENGTHS, "cells_per_step_per_gpu": cells_step,
                "partition_i16x2_i32": [n16, n32], "db_build_s": round(build_s, 2),
                "db_device_bytes": db.device_bytes(), "scratch_bytes": db.scratch_bytes(),
                "l2": "inputs larger than L2 (packed database + boundary rows >> 126 MB)",
                "parallelism": f"db shards x{world}" if world > 1 else "single GPU",
            },
            "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": sum(len(q) for q in queries),
                    "d2h_bytes_per_step": 32 * N_QUERIES},
            "gpu_launches": int(all_l.value),
            "roofline": {"bound": "dpx_int16x2", "achieved": achieved, "peak": peak_gcups, "unit": "GCUPS",
                         "frac": achieved / peak_gcups if peak_gcups else None,
                         "traffic": cells16_per_launch * DRAM_BYTES_PER_CELL,
                         "traffic_note": "bytes per launch: dram read+write per cell from one ncu capture "
                                         "(400k sequences x 1000-residue query) times this launch's cells",
                         "kernel": "scan_kernel<Pair16,8,R,SW>, two-column sweep, R = 8 (queries <= 64) or 16 rows per lane",
                         "avg_launch_ms": avg16_ms,
                         "launches": int(kl[0]), "cells_per_launch": cells16_per_launch,
                         "peak_source": "measured: hy_measure_dpx_peak (register-resident per-cell DPX mix)"},
            "kernels": kernels,
            "roofline_hbm": {"bound": "hbm", "peak": hbm_peak, "unit": "GB/s", "peak_source": "MEASURED_PEAKS.json hbm_gbs" if meas else "fallback"},
            "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if world == 1 and not args.no_extras:
            # The metric's other forms at their full sizes, one compact measurement each.
            for key, fn in (("batched", extra_batched), ("served", extra_served), ("pairs", extra_pairs)):
                t0 = time.perf_counter()
                line[key] = fn(args.seed)
                line[key]["run_s"] = round(time.perf_counter() - t0, 1)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def make_reads_workload(seed: int, n_reads: int, n_queries: int, read_len: int = 150,
                        genome_len: int = 5_000_000):
    """DNA reads of `read_len` sampled from a seeded uniform genome with 1% substitutions and a
    0.2%-per-base rate of single-base indels (at most one per read; reads keep their length), and
    `n_queries` genome windows of uniform length 32..2000 with 1% substitutions."""
    rng = np.random.default_rng(seed)
    genome = rng.integers(0, 4, genome_len, dtype=np.uint8)
    reads = np.empty((n_reads, read_len), np.uint8)
    ar_w = np.arange(read_len + 2)
    j = np.arange(read_len)[None, :]
    for lo in range(0, n_reads, 100_000):
        n = min(100_000, n_reads - lo)
        starts = rng.integers(0, genome_len - read_len - 2, n)
        win = genome[starts[:, None] + ar_w[None, :]]
        p = rng.integers(0, read_len, n)[:, None]
        kind = rng.random(n)
        deletion = (kind < 0.002 * read_len / 2)[:, None]
        insertion = ((kind >= 0.002 * read_len / 2) & (kind < 0.002 * read_len))[:, None]
        idx = np.where(deletion, j + (j >= p), np.where(insertion, j - (j > p), j))
        r = np.take_along_axis(win, idx, axis=1)
        r = np.where(insertion & (j == p), rng.integers(0, 4, (n, 1), dtype=np.uint8), r)
        sub = rng.integers(0, 100, (n, read_len), dtype=np.uint8) == 0  # 1% of the bases
        r = np.where(sub, (r + rng.integers(1, 4, (n, read_len), dtype=np.uint8)) % 4, r).astype(np.uint8)
        reads[lo:lo + n] = r
    offsets = np.arange(n_reads + 1, dtype=np.uint64) * read_len
    queries = []
    for _ in range(n_queries):
        L = int(rng.integers(32, 2001))
        s = int(rng.integers(0, genome_len - L))
        q = genome[s:s + L].copy()
        sub = rng.random(L) < 0.01
        q[sub] = (q[sub] + rng.integers(1, 4, int(sub.sum()), dtype=np.uint8)) % 4
        queries.append(q)
    return reads.reshape(-1), offsets, queries


def run_batched(args):
    """The batched multi-mode workload: 256 DNA queries (32..2000 bp, modes SW/NW/HW/SHW/OV
    round-robin, ScoreEnd, +2/-1, gap_open 2, gap_ext 1) against 1,000,000 150-bp reads, one
    Database per mode, all queries per hy_scan_batch call (persistent kernels under a CUDA graph,
    autotuned launch shapes), against the same queries as 256 sequential plain Database.scan calls."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    residues, offsets, queries = make_reads_workload(args.seed, args.n_reads, args.n_batch_queries)
    gen_s = time.perf_counter() - t0
    modes = [hy.Mode.Sw, hy.Mode.Nw, hy.Mode.Hw, hy.Mode.Shw, hy.Mode.Ov]
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    t0 = time.perf_counter()
    dbs = [(hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(4, dna, 2, 1))
            .mode(m).search_type(hy.SearchType.ScoreEnd).max_query_len(2000).build()) for m in modes]
    build_s = time.perf_counter() - t0
    dbq = [i % len(modes) for i in range(len(queries))]
    total_res = float(offsets[-1])
    cells = float(sum(len(q) for q in queries)) * total_res
    batch = hy.Batch(dbs, max_queries=len(queries), autotune=True)
    stream = torch.cuda.ExternalStream(batch.stream_ptr())
    t0 = time.perf_counter()
    hits_b = batch.scan(queries, dbq)  # the first call of this shape runs the autotuner
    first_s = time.perf_counter() - t0
    for _ in range(max(0, args.warmup - 1)):
        batch.scan(queries, dbq)
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        hits_b = batch.scan(queries, dbq)
    wall_b = time.perf_counter() - t0
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_b = ev0.elapsed_time(ev1) / 1e3
    # The plain form: one Database.scan per query (host query in, hit out, a sync per call).
    scratches = [hy.Scratch(d) for d in dbs]
    for k, d in enumerate(dbs):
        d.scan(scratches[k], queries[k])
    t0 = time.perf_counter()
    hits_p = [dbs[k].scan(scratches[k], q) for q, k in zip(queries, dbq)]
    wall_p = time.perf_counter() - t0
    identical = hits_p == hits_b
    peak = C.c_double()
    from hyalite_b200 import _abi
    _abi.lib.hy_measure_dpx_peak(C.byref(peak))
    value = cells * args.steps / dev_b / 1e9
    line = {
        "metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_b * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "i16x2", "data": "synthetic (seeded genome reads)",
        "config": {"workload": "batched multi-mode DNA scan: 256 queries (32..2000 bp; SW/NW/HW/SHW/OV "
                               "round-robin; ScoreEnd) x 1,000,000 reads of 150 bp, one persistent-kernel "
                               "batch per call under a CUDA graph",
                   "n_reads": int(args.n_reads), "queries": len(queries), "cells_per_step": cells,
                   "gen_s": round(gen_s, 1), "db_build_s": round(build_s, 1),
                   "first_call_s_incl_autotune": round(first_s, 2), "tuned_config": list(batch.config()),
                   "batch_device_bytes": batch.device_bytes(),
                   "l2": "inputs larger than L2 (150 MB of packed reads per database)"},
        "e2e": {"value": cells * args.steps / wall_b / 1e9, "unit": "GCUPS",
                "h2d_bytes_per_step": int(sum(len(q) for q in queries)) + 4 * len(queries),
                "d2h_bytes_per_step": 32 * len(queries)},
        "plain": {"value": cells / wall_p / 1e9, "unit": "GCUPS", "form": "256 sequential Database.scan calls",
                  "seconds": wall_p},
        "batched_over_plain": (cells * args.steps / wall_b) / (cells / wall_p),
        "identical_to_plain": identical,
        "frac_of_dpx_peak": value / (peak.value / 1e9) if peak.value else None,
        "dpx_peak_gcups": peak.value / 1e9,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


# ---- the metric's other forms, compact, for the default line -----------------------------------

def _hit4(h):
    return (int(h.score), int(h.db_index), None if h.query_end is None or h.query_end < 0 else int(h.query_end),
            None if h.target_end is None or h.target_end < 0 else int(h.target_end))


def _oracle_best(ref, query, threads):
    """The reference scan's best hit from the oracle's per-target results: the highest score, the
    smallest db index on ties, the winner's own ends (src/database.rs:117-130, 186-197)."""
    best = None
    for h in ref.scan_all(query, threads=threads):
        if best is None or h[0] > best[0]:
            best = h
    return best


def extra_batched(seed, warm_tune=True):
    """The batched multi-mode workload at its full size (256 DNA queries of 32..2000 bp, modes
    SW/NW/HW/SHW/OV round-robin, ScoreEnd, against 1,000,000 reads of 150 bp): one autotuned
    hy_scan_batch call timed by CUDA events on the batch's stream and by the host clock, against the
    same queries as 256 sequential Database.scan calls; the three shortest queries of different
    modes checked against the oracle."""
    import torch

    import hyalite_b200 as hy
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    residues, offsets, queries = make_reads_workload(seed, 1_000_000, 256)
    modes = [hy.Mode.Sw, hy.Mode.Nw, hy.Mode.Hw, hy.Mode.Shw, hy.Mode.Ov]
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    dbs = [(hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(4, dna, 2, 1))
            .mode(m).search_type(hy.SearchType.ScoreEnd).max_query_len(2000).build()) for m in modes]
    dbq = [i % len(modes) for i in range(len(queries))]
    cells = float(sum(len(q) for q in queries)) * float(offsets[-1])
    batch = hy.Batch(dbs, max_queries=len(queries), autotune=True)
    stream = torch.cuda.ExternalStream(batch.stream_ptr())
    t0 = time.perf_counter()
    batch.scan(queries, dbq)  # the first call of the shape runs the autotuner
    first_s = time.perf_counter() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    t0 = time.perf_counter()
    hits_b = batch.scan(queries, dbq)
    wall_b = time.perf_counter() - t0
    ev1.record(stream)
    torch.cuda.synchronize()
    dev_b = ev0.elapsed_time(ev1) / 1e3
    scratches = [hy.Scratch(d) for d in dbs]
    for k, d in enumerate(dbs):
        d.scan(scratches[k], queries[k])
    t0 = time.perf_counter()
    hits_p = [dbs[k].scan(scratches[k], q) for q, k in zip(queries, dbq)]
    wall_p = time.perf_counter() - t0
    picked, seen = [], set()
    for i in sorted(range(len(queries)), key=lambda i: len(queries[i])):
        if dbq[i] not in seen:
            picked.append(i)
            seen.add(dbq[i])
        if len(picked) == 3:
            break
    threads = os.cpu_count() or 1
    oracle_ok = all(_hit4(hits_b[i]) == _oracle_best(pyoracle.OracleDb((residues, offsets), dna, 4, 2, 1,
                                                                      int(modes[dbq[i]]), 1), queries[i], threads)
                    for i in picked)
    return {"workload": "256 DNA queries (32..2000 bp; SW/NW/HW/SHW/OV round-robin; ScoreEnd) x 1,000,000 "
                        "reads of 150 bp, one hy_scan_batch call (persistent kernels under a CUDA graph)",
            "value": cells / dev_b / 1e9, "unit": "GCUPS", "cells": cells,
            "e2e": {"value": cells / wall_b / 1e9, "unit": "GCUPS", "call_s": wall_b,
                    "h2d_bytes": int(sum(len(q) for q in queries)) + 4 * len(queries), "d2h_bytes": 32 * len(queries)},
            "plain": {"value": cells / wall_p / 1e9, "unit": "GCUPS", "seconds": wall_p,
                      "form": "256 sequential Database.scan calls, host query in, hit out"},
            "batched_over_plain": wall_p / wall_b, "first_call_s_incl_autotune": first_s,
            "tuned_config": list(batch.config()),
            "identical_to_plain": [_hit4(h) for h in hits_b] == [_hit4(h) for h in hits_p],
            "identical_to_oracle_on_sample": bool(oracle_ok),
            "oracle_sample": f"queries {picked} (the shortest of three modes) against all 1,000,000 reads"}


def extra_served(seed, rate=10.0, seconds=6.0):
    """The served protein workload at its full size (1,000,000 sequences of the protein generator;
    log-normal query lengths, median 350, 50..3000; half ScoreEnd scans, half scan_scores) at one
    offered rate below saturation: p50/p99 latency and GCUPS, every result against the plain call,
    and the shortest request of each kind against the oracle."""
    import hyalite_b200 as hy
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    mat, residues, offsets, _ = make_workload(seed, n_seqs=1_000_000)
    db = (hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(AL, mat, GO, GE))
          .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(3000).build())
    rng = np.random.default_rng(seed + 7)
    base = np.random.default_rng(12345)
    base.integers(-4, 4, size=(AL, AL))
    base.integers(4, 12, size=AL)
    background = base.dirichlet(np.full(AL, 4.0))

    def request():
        L = int(np.clip(round(math.exp(math.log(350.0) + 0.8 * rng.standard_normal())), 50, 3000))
        return rng.choice(AL, size=L, p=background).astype(np.uint8), bool(rng.random() < 0.5)

    total_res = float(offsets[-1])
    srv = hy.Server([db], max_batch=64, in_flight=2)
    for kind in (False, True):
        q, _ = request()
        srv.wait(srv.submit(q, want_scores=kind))
    srv.stats(reset=True)
    n = int(rate * seconds)
    reqs = [request() for _ in range(n)]
    gaps = rng.exponential(1.0 / rate, n)
    handles = []
    t_start = time.perf_counter()
    t_next = t_start
    for (q, kind), g in zip(reqs, gaps):
        t_next += g
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        handles.append(srv.submit(q, want_scores=kind))
    served = [(srv.wait(h), h.scores) for h in handles]
    wall = time.perf_counter() - t_start
    st = srv.stats(reset=True)
    srv.close()
    sc = hy.Scratch(db)
    same = True
    t0 = time.perf_counter()
    cells = 0.0
    plain_ms = []
    for (q, kind), (hit, scores) in zip(reqs, served):
        t1 = time.perf_counter()
        if kind:
            same &= bool(np.array_equal(scores, db.scan_scores_array(sc, q)))
        else:
            same &= _hit4(hit) == _hit4(db.scan(sc, q))
        plain_ms.append((time.perf_counter() - t1) * 1e3)
        cells += len(q) * total_res
    plain_s = time.perf_counter() - t0
    # Latency by query length: what a request waited for beyond its own scan time.
    by_len = {}
    for (q, _), h, pm in zip(reqs, handles, plain_ms):
        c = "short (<= 350 aa)" if len(q) <= 350 else "long (> 350 aa)"
        by_len.setdefault(c, ([], []))
        by_len[c][0].append(h.latency_ms)
        by_len[c][1].append(pm)
    latency_by_length = {c: {"requests": len(l), "p50_ms": float(np.percentile(l, 50)),
                             "p99_ms": float(np.percentile(l, 99)), "plain_call_p50_ms": float(np.percentile(p, 50))}
                         for c, (l, p) in by_len.items()}
    ref = pyoracle.OracleDb((residues, offsets), mat, AL, GO, GE, 0, 1)
    threads = os.cpu_count() or 1
    oracle_ok = True
    for kind in (False, True):
        i = min((i for i in range(n) if reqs[i][1] == kind), key=lambda i: len(reqs[i][0]))
        q = reqs[i][0]
        if kind:
            oracle_ok &= bool(np.array_equal(served[i][1], ref.scan_scores(q, threads=threads)))
        else:
            oracle_ok &= _hit4(served[i][0]) == _oracle_best(ref, q, threads)
    return {"workload": "1,000,000 protein sequences (log-normal lengths), Poisson arrivals, log-normal query "
                        "lengths (median 350, 50..3000), half ScoreEnd scan and half scan_scores (i32 per target)",
            "offered_qps": rate, "requests": n, "completed": int(st["completed"]), "achieved_qps": st["completed"] / wall,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_batch": st["mean_batch"],
            "latency_by_query_length": latency_by_length,
            "value": st["gcups"], "unit": "GCUPS",
            "plain": {"value": cells / plain_s / 1e9, "unit": "GCUPS", "seconds": plain_s,
                      "form": "the same requests one at a time (Database.scan / scan_scores)"},
            "identical_to_plain": bool(same), "identical_to_oracle_on_sample": bool(oracle_ok),
            "oracle_sample": "the shortest scan and the shortest scan_scores request, against all 1,000,000 sequences"}


def extra_pairs(seed, n_pairs=10_000_000, steps=2):
    """align_pairs at its full size (10,000,000 (150-bp read, 200..500-bp window) pairs, HW,
    ScoreEnd, +2/-1, gap_open 6, gap_ext 1): device GCUPS (the call's kernels, CUDA events), the
    whole call with host buffers, and 2,000 sampled pairs against the oracle."""
    import hyalite_b200 as hy
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    q_res, q_off, t_res, t_off = make_pairs_workload(seed, n_pairs)
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    scoring = hy.Scoring(4, dna, 6, 1)
    cells = float(np.dot(np.diff(q_off).astype(np.float64), np.diff(t_off).astype(np.float64)))
    hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
    kms = cms = 0.0
    for _ in range(steps):
        hits, (err, _) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
        assert err is None
        k, c = hy.align_pairs_timing()
        kms += k
        cms += c
    rng = np.random.default_rng(1)
    sample = np.sort(rng.choice(n_pairs, min(n_pairs, 2000), replace=False))
    qs = [q_res[int(q_off[i]):int(q_off[i + 1])] for i in sample]
    ts = [t_res[int(t_off[i]):int(t_off[i + 1])] for i in sample]
    st, want, _ = pyoracle.align_pairs(qs, ts, dna, 4, 6, 1, 2, 1, threads=os.cpu_count() or 1)
    got = [(hits[i].score, None if hits[i].query_end < 0 else hits[i].query_end,
            None if hits[i].target_end < 0 else hits[i].target_end) for i in sample]
    return {"workload": f"align_pairs: {n_pairs} (150-bp read, 200..500-bp window) pairs, HW, ScoreEnd, +2/-1, "
                        "gap_open 6, gap_ext 1",
            "value": cells * steps / (kms * 1e-3) / 1e9, "unit": "GCUPS", "cells": cells,
            "e2e": {"value": cells * steps / (cms * 1e-3) / 1e9, "unit": "GCUPS", "call_ms": cms / steps,
                    "h2d_bytes": int(len(q_res) + len(t_res) + 16 * n_pairs), "d2h_bytes": 12 * n_pairs},
            "identical_to_oracle_on_sample": bool(st == 0 and got == [(w[0], w[2], w[3]) for w in want]),
            "oracle_sample": "2,000 random pairs"}


def make_dna_small_workload(seed: int, n_queries: int, n_seqs: int = 10_000, n_planted: int = 50):
    """The small DNA scan: `n_seqs` sequences of uniform length 50..300 and uniform bases, and
    `n_queries` queries of 64 uniform bases; `n_planted` sequences are replaced by copies of the
    first query with 5% of its bases (3 of 64) substituted. Returns (seqs, queries, planted)."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(50, 301, n_seqs)
    seqs = [rng.integers(0, 4, int(n)).astype(np.uint8) for n in lengths]
    queries = [rng.integers(0, 4, 64).astype(np.uint8) for _ in range(n_queries)]
    planted = rng.choice(n_seqs, n_planted, replace=False)
    for k in planted:
        s = queries[0].copy()
        sub = rng.choice(64, 3, replace=False)  # 5% of 64
        s[sub] = (s[sub] + rng.integers(1, 4, 3)) % 4
        seqs[k] = s
    return seqs, queries, planted


def run_dna_small(args):
    """The small plain DNA scan: alphabet 4, +2/-1, gap_open 2, gap_ext 1, SW ScoreEnd, a stream of
    --dna-queries queries of 64 uniform bases against 10,000 sequences of uniform length 50..300
    with 50 planted copies of the first query carrying 5% substitutions. Reports the per-call
    latency and GCUPS of Database.scan (host query in, hit out), the same stream through the
    batched form (all queries in one hy_scan_batch call, host queries in, hits out), and the AVX2
    port on the same database over all host threads; every hit is checked against the oracle."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    seqs, queries, planted = make_dna_small_workload(args.seed, args.dna_queries)
    res, off = hy.concat(seqs)
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    db = (hy.Database.builder().sequences_concat(res, off).scoring(hy.Scoring(4, dna, 2, 1)).mode(hy.Mode.Sw)
          .search_type(hy.SearchType.ScoreEnd).max_query_len(64).build())
    sc = hy.Scratch(db)
    for q in queries[: args.warmup]:
        db.scan(sc, q)
    lat = []
    hits = []
    for q in queries:
        t0 = time.perf_counter()
        hits.append(db.scan(sc, q))
        lat.append(time.perf_counter() - t0)
    cells = 64.0 * float(off[-1])
    # The same stream through the batched form: one call for every query.
    batch = hy.Batch([db], max_queries=len(queries))
    q_res = np.concatenate(queries)
    q_off = np.arange(len(queries) + 1, dtype=np.uint64) * 64
    dbq = np.zeros(len(queries), np.uint32)
    for _ in range(max(args.warmup, 1)):
        batch.scan_arrays(q_res, q_off, dbq)
    blat = []
    for _ in range(max(args.steps, 1)):
        t0 = time.perf_counter()
        bhits = batch.scan_arrays(q_res, q_off, dbq)
        blat.append(time.perf_counter() - t0)
    batched_same = all((bhits[i].score, bhits[i].db_index, bhits[i].query_end, bhits[i].target_end) ==
                       (h.score, h.db_index, -1 if h.query_end is None else h.query_end,
                        -1 if h.target_end is None else h.target_end) for i, h in enumerate(hits))
    bmed = statistics.median(blat)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    ref = pyoracle.OracleDb((res, off), dna, 4, 2, 1, 0, 1)
    check = range(0, len(queries), max(1, len(queries) // 50))
    identical = all((hits[i].score, hits[i].db_index, hits[i].query_end, hits[i].target_end) == ref.scan(queries[i])
                    for i in check)
    threads = os.cpu_count() or 1
    avx = pyoracle.Avx2Db(res, off, dna, 4, 2, 1, 0, 1, 64)
    qlist = [list(map(int, q)) for q in queries]
    t0 = time.perf_counter()
    avx.scan_many(qlist, threads)
    cpu_s = time.perf_counter() - t0
    med = statistics.median(lat)
    line = {
        "metric": "GCUPS", "value": cells / med / 1e9, "unit": "GCUPS", "n_gpus": 1, "steps": len(queries),
        "warmup": args.warmup, "ms_per_step": med * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "i16x2 (Precomputed layout)", "data": "synthetic (seeded DNA)",
        "config": {"workload": "small plain DNA SW ScoreEnd scan: 64-bp query x 10,000 sequences of 50..300 bp "
                               "(50 planted 5%-substituted copies), one Database.scan per query",
                   "residues": int(off[-1]), "layout": db.layout().name},
        "latency_ms": {"p50": med * 1e3, "p99": float(np.percentile(lat, 99)) * 1e3, "min": min(lat) * 1e3},
        "e2e": {"value": cells / med / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": 64, "d2h_bytes_per_step": 32},
        "identical_to_oracle_on_sample": identical,
        "planted_top_hit": int(hits[0].db_index) in set(int(k) for k in planted),
        "batched": {"value": cells * len(queries) / bmed / 1e9, "unit": "GCUPS", "queries_per_call": len(queries),
                    "ms_per_call": bmed * 1e3, "vs_plain": (cells * len(queries) / bmed) / (cells / med),
                    "identical_to_plain": bool(batched_same),
                    "form": "hy_scan_batch, host queries in, hits out, persistent kernels under a CUDA graph"},
        "cpu_baseline": {"value": cells * len(queries) / cpu_s / 1e9, "unit": "GCUPS", "cores": threads,
                         "kind": "port", "sample": f"the same {len(queries)} queries, one per thread, AVX2 port"},
    }
    print(json.dumps(line), flush=True)


def run_served(args):
    """The served workload: a resident protein database (the generator above at --served-seqs
    sequences), Poisson arrivals at each offered rate, query lengths log-normal (median 350,
    sigma 0.8, clipped 50..3000), half the requests a ScoreEnd scan and half scan_scores (every
    target's i32 score). Reports per rate the p50/p99 latency (submit -> result ready) and the
    GCUPS the server sustained, beside the plain per-request calls (Database.scan /
    scan_scores one at a time). --served-db dna_small serves the small DNA database of the
    dna_small workload instead, every request a 64-bp ScoreEnd scan."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    rng = np.random.default_rng(args.seed + 7)
    if args.served_db == "dna_small":
        # The small DNA database of the dna_small workload; every request a 64-bp ScoreEnd scan.
        drng = np.random.default_rng(args.seed)
        lengths = drng.integers(50, 301, 10_000)
        res, offsets = hy.concat([drng.integers(0, 4, int(n)).astype(np.uint8) for n in lengths])
        dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
        db = (hy.Database.builder().sequences_concat(res, offsets).scoring(hy.Scoring(4, dna, 2, 1))
              .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(64).build())

        def request():
            return rng.integers(0, 4, 64).astype(np.uint8), False
        workload = ("served small DNA scan: 10,000 sequences of 50..300 bp, Poisson arrivals, every "
                    "request a 64-bp SW ScoreEnd scan")
    else:
        mat, residues, offsets, _ = make_workload(args.seed, n_seqs=args.served_seqs)
        db = (hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(AL, mat, GO, GE))
              .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(3000).build())
        base = np.random.default_rng(12345)
        base.integers(-4, 4, size=(AL, AL))
        base.integers(4, 12, size=AL)
        background = base.dirichlet(np.full(AL, 4.0))

        def request():
            L = int(np.clip(round(math.exp(math.log(350.0) + 0.8 * rng.standard_normal())), 50, 3000))
            return rng.choice(AL, size=L, p=background).astype(np.uint8), bool(rng.random() < 0.5)
        workload = (f"served protein scan: {args.served_seqs} sequences, Poisson arrivals, log-normal "
                    "query lengths (median 350, 50..3000), half ScoreEnd scan and half scan_scores "
                    "(i32 per target)")
    gen_s = time.perf_counter() - t0
    total_res = float(offsets[-1])

    srv = hy.Server([db], max_batch=args.served_batch, in_flight=2)
    # Warm-up: one request of each kind.
    for kind in (False, True):
        q, _ = request()
        srv.wait(srv.submit(q, want_scores=kind))
    srv.stats(reset=True)
    rates = [float(x) for x in args.served_rates.split(",")]
    points = []
    clocks = Clocks(0)
    clocks.start()
    for rate in rates:
        n = int(min(args.served_max_requests, max(20, rate * args.served_seconds)))
        reqs = [request() for _ in range(n)]
        gaps = rng.exponential(1.0 / rate, n)
        handles = []
        t_start = time.perf_counter()
        t_next = t_start
        rejected = 0
        for (q, kind), g in zip(reqs, gaps):
            t_next += g
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            try:
                handles.append((srv.submit(q, want_scores=kind), len(q)))
            except hy.Error as e:
                if e.kind != "Rejected":
                    raise
                rejected += 1
        for h, _ in handles:
            srv.wait(h)
        wall = time.perf_counter() - t_start
        st = srv.stats(reset=True)
        points.append({"offered_qps": rate, "requests": n, "completed": int(st["completed"]),
                       "rejected": int(st["rejected"]) + rejected, "achieved_qps": st["completed"] / wall,
                       "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                       "max_ms": st["max_ms"], "mean_batch": st["mean_batch"], "gcups": st["gcups"],
                       "wall_s": wall})
    clk = clocks.stop()
    srv.close()
    # The plain form: the same kind of requests one at a time through the host API.
    sc = hy.Scratch(db)
    plain = [request() for _ in range(args.served_plain_requests)]
    db.scan(sc, plain[0][0])
    t0 = time.perf_counter()
    cells = 0.0
    for q, kind in plain:
        if kind:
            db.scan_scores_array(sc, q)
        else:
            db.scan(sc, q)
        cells += len(q) * total_res
    plain_s = time.perf_counter() - t0
    plain_gcups = cells / plain_s / 1e9
    best = max(points, key=lambda p: p["gcups"])
    line = {
        "metric": "GCUPS", "value": best["gcups"], "unit": "GCUPS", "n_gpus": 1, "steps": len(rates),
        "warmup": 2, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "i16x2 (int32 for long sequences)", "data": "synthetic (seeded generators)",
        "config": {"workload": workload,
                   "residues": int(total_res), "gen_s": round(gen_s, 1), "max_batch": args.served_batch,
                   "in_flight": 2},
        "served": points,
        "plain": {"value": plain_gcups, "unit": "GCUPS", "requests": len(plain),
                  "form": "Database.scan / scan_scores one request at a time"},
        "served_over_plain": best["gcups"] / plain_gcups,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def make_pairs_workload(seed: int, n_pairs: int, genome_len: int = 10_000_000, read_len: int = 150):
    """(read, window) pairs: reads of `read_len` from a seeded uniform genome with 2% substitutions
    and, with probability 0.75 per read (0.5% per base), one 1..3-bp insertion or deletion; each
    window 200..500 bp long and placed so that it contains the read's origin. Blocks of 250,000
    pairs are generated on all host threads, each from its own seeded stream."""
    from concurrent.futures import ThreadPoolExecutor

    rng = np.random.default_rng(seed)
    genome = rng.integers(0, 4, genome_len, dtype=np.uint8)
    reads = np.empty((n_pairs, read_len), np.uint8)
    wlen = rng.integers(200, 501, n_pairs).astype(np.int64)
    wstart = np.empty(n_pairs, np.int64)
    t_off = np.zeros(n_pairs + 1, np.uint64)
    t_off[1:] = np.cumsum(wlen)
    t_res = np.empty(int(t_off[-1]), np.uint8)
    j = np.arange(read_len, dtype=np.int16)[None, :]
    span = read_len + 3
    read_view = np.lib.stride_tricks.sliding_window_view(genome, span)
    # Each window is the first wlen bases of a 500-base view of the genome at its start.
    win_view = np.lib.stride_tricks.sliding_window_view(genome, 500)
    cols = np.arange(500)[None, :]
    block = 250_000

    def make_block(lo):
        brng = np.random.default_rng([seed, lo])
        n = min(block, n_pairs - lo)
        W = wlen[lo:lo + n]
        origin = brng.integers(600, genome_len - 600, n)
        win = read_view[origin]
        p = brng.integers(0, read_len, n)[:, None].astype(np.int16)
        dl = brng.integers(1, 4, n)[:, None].astype(np.int16)
        kind = brng.random(n)
        deletion = (kind < 0.375)[:, None]
        insertion = ((kind >= 0.375) & (kind < 0.75))[:, None]
        # Source base of each read position: a deletion skips dl bases at p; after an insertion of
        # dl bases at p the read continues with the base at p.
        idx = j + (deletion & (j >= p)) * dl - (insertion & (j >= p + dl)) * dl
        r = np.take_along_axis(win, idx.astype(np.intp), axis=1)
        r = np.where(insertion & (j >= p) & (j < p + dl), brng.integers(0, 4, (n, read_len), dtype=np.uint8), r)
        sub = brng.integers(0, 50, (n, read_len), dtype=np.uint8) == 0  # 2% of the bases
        r = np.where(sub, (r + brng.integers(1, 4, (n, read_len), dtype=np.uint8)) % 4, r).astype(np.uint8)
        reads[lo:lo + n] = r
        ws = origin - brng.integers(0, W - read_len + 1)
        wstart[lo:lo + n] = ws
        t_res[int(t_off[lo]):int(t_off[lo + n])] = win_view[ws][cols < W[:, None]]

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        list(ex.map(make_block, range(0, n_pairs, block)))
    q_off = np.arange(n_pairs + 1, dtype=np.uint64) * read_len
    return reads.reshape(-1), q_off, t_res, t_off


def run_pairs(args):
    """align_pairs over (read, window) pairs: Mode::Hw, ScoreEnd, +2/-1, gap_open 6, gap_ext 1.
    `value` is real cells / the device time of the call's kernels (each chunk's packing and pair
    kernels, CUDA events); `e2e` is the whole hy_align_pairs call (host lengths pass, sort and item
    packing, staging copies, kernels, results) with pageable host buffers; `e2e_pinned_inputs` the
    same with the residues already page-locked."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    q_res, q_off, t_res, t_off = make_pairs_workload(args.seed, args.n_pairs)
    gen_s = time.perf_counter() - t0
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    scoring = hy.Scoring(4, dna, 6, 1)
    cells = float(np.dot(np.diff(q_off).astype(np.float64), np.diff(t_off).astype(np.float64)))
    for _ in range(args.warmup):
        hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
    clocks = Clocks(0)
    clocks.start()
    kms, cms = 0.0, 0.0
    phases = {}
    for _ in range(args.steps):
        hits, (err, _) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
        assert err is None
        k, c = hy.align_pairs_timing()
        kms += k
        cms += c
        for key, v in hy.align_pairs_phases().items():
            phases[key] = phases.get(key, 0.0) + v / args.steps
    clk = clocks.stop()
    # The same calls with the reads and windows already in page-locked memory (a caller that keeps
    # them pinned): the device copies the residues from where they are, with no staging copy.
    pq = hy.pinned_empty(len(q_res), np.uint8)
    pt = hy.pinned_empty(len(t_res), np.uint8)
    pq[:] = q_res
    pt[:] = t_res
    hy.align_pairs_arrays(pq, q_off, pt, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
    cms_pinned = 0.0
    for _ in range(args.steps):
        hits_p, (err, _) = hy.align_pairs_arrays(pq, q_off, pt, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
        assert err is None
        cms_pinned += hy.align_pairs_timing()[1]
    same_pinned = bytes(hits_p) == bytes(hits)
    # Parity on a sample against the oracle, and the CPU baseline (the reference's align_pairs is
    # the scalar align_core loop) on a bounded sample over all host threads.
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    rng = np.random.default_rng(1)
    sample = np.sort(rng.choice(args.n_pairs, min(args.n_pairs, 2000), replace=False))
    qs = [q_res[int(q_off[i]):int(q_off[i + 1])] for i in sample]
    ts = [t_res[int(t_off[i]):int(t_off[i + 1])] for i in sample]
    st, want, _ = pyoracle.align_pairs(qs, ts, dna, 4, 6, 1, 2, 1)
    got = [(hits[i].score, None if hits[i].query_end < 0 else hits[i].query_end,
            None if hits[i].target_end < 0 else hits[i].target_end) for i in sample]
    identical = st == 0 and got == [(w[0], w[2], w[3]) for w in want]
    threads = os.cpu_count() or 1
    n_cpu = min(args.n_pairs, args.cpu_pairs)
    cq = [q_res[int(q_off[i]):int(q_off[i + 1])] for i in range(n_cpu)]
    ct = [t_res[int(t_off[i]):int(t_off[i + 1])] for i in range(n_cpu)]
    ccells = float(sum(len(a) * len(b) for a, b in zip(cq, ct)))
    t0 = time.perf_counter()
    pyoracle.align_pairs(cq, ct, dna, 4, 6, 1, 2, 1, threads=threads)
    cpu_s = time.perf_counter() - t0
    value = cells * args.steps / (kms * 1e-3)
    line = {
        "metric": "GCUPS", "value": value / 1e9, "unit": "GCUPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "i16x2", "data": "synthetic (seeded genome reads and windows)",
        "config": {"workload": f"align_pairs: {args.n_pairs} (150-bp read, 200..500-bp window) pairs, HW, "
                               "ScoreEnd, +2/-1, gap_open 6, gap_ext 1",
                   "cells_per_step": cells, "gen_s": round(gen_s, 1),
                   "l2": "inputs larger than L2 (reads and windows: gigabytes)"},
        "e2e": {"value": cells * args.steps / (cms * 1e-3) / 1e9, "unit": "GCUPS",
                "h2d_bytes_per_step": int(len(q_res) + len(t_res) + 16 * args.n_pairs),
                "d2h_bytes_per_step": 12 * args.n_pairs, "call_ms": cms / args.steps,
                "phases_ms": {k: round(v, 1) for k, v in phases.items()}},
        "e2e_pinned_inputs": {"value": cells * args.steps / (cms_pinned * 1e-3) / 1e9, "unit": "GCUPS",
                              "call_ms": cms_pinned / args.steps, "hits_identical": same_pinned},
        "identical_to_oracle_on_sample": identical,
        "cpu_baseline": {"value": ccells / cpu_s / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
                         "sample": f"the first {n_cpu} pairs, scalar align_core restatement over {threads} threads"},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) per DP cell of the traceback fill, from one ncu capture of
# tb_fill_kernel<16, SW> (protein generator, 5,000 sequences x the 1000-residue query: 2.055e9
# cells, 177.1 MB read, 1.162 GB written). The codes alone are 0.5 byte a cell.
TB_DRAM_BYTES_PER_CELL = (177.1e6 + 1.1617e9) / 2.055e9


def run_aligned(args):
    """Database::scan_all_aligned: the 1000-residue query of the protein workload against the first
    --aligned-seqs sequences of the protein generator, SW, SearchType::Alignment with a usize::MAX
    budget. `value` is real cells / the device span of the traceback (CUDA events from the first
    fill to the end of compaction; walks overlap the next chunk's fill); `e2e` is the whole
    hy_scan_all_aligned call (host query in, every alignment and its operations out in host
    memory)."""
    import torch

    import hyalite_b200 as hy
    from hyalite_b200 import _abi

    torch.cuda.set_device(0)
    mat, residues, offsets, queries = make_workload(args.seed, n_seqs=args.aligned_seqs)
    q = next(x for x in queries if len(x) == 1000)
    scoring = hy.Scoring(AL, [int(v) for v in mat], GO, GE)
    t0 = time.perf_counter()
    db = (hy.Database.builder().sequences_concat(residues, offsets).scoring(scoring).mode(hy.Mode.Sw)
          .search_type(hy.SearchType.alignment(hy.USIZE_MAX)).max_query_len(len(q)).build())
    build_s = time.perf_counter() - t0
    sc = hy.Scratch(db)
    cells = float(len(q)) * float(offsets[-1])
    for _ in range(args.warmup):
        db.scan_all_aligned_arrays(sc, q)
    lib = _abi.lib
    kms = (C.c_double * 3)()
    kl = (C.c_uint64 * 3)()
    all_l = C.c_uint64()
    lib.hy_scratch_profile_read(sc._h, kms, kl, None, C.byref(all_l))  # resets the launch count
    clocks = Clocks(0)
    clocks.start()
    fill_ms = walk_ms = dev_ms = call_ms = 0.0
    n_ops = 0
    for _ in range(args.steps):
        arr, buf = db.scan_all_aligned_arrays(sc, q)
        t = hy.traceback_timing(sc)
        fill_ms += t["fill_ms"]
        walk_ms += t["walk_ms"]
        dev_ms += t["device_ms"]
        call_ms += t["call_ms"]
        n_ops += len(buf)
    clk = clocks.stop()
    lib.hy_scratch_profile_read(sc._h, kms, kl, None, C.byref(all_l))
    # Parity on a sample against the oracle's restatement of src/align.rs.
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    rng = np.random.default_rng(5)
    sample = sorted(int(k) for k in rng.choice(args.aligned_seqs, min(args.aligned_seqs, 300), replace=False))
    raw = buf.tobytes()
    identical = True
    for k in sample:
        a = arr[k]
        got = (int(a.score), int(a.query_start), int(a.query_end), int(a.target_start), int(a.target_end),
               raw[int(a.ops_offset): int(a.ops_offset) + int(a.n_ops)])
        t = residues[int(offsets[k]): int(offsets[k + 1])]
        identical &= got == pyoracle.traceback(q, t, mat, AL, GO, GE, 0)
    # CPU baseline: the scalar full-matrix traceback restated from src/align.rs, over all host
    # threads, on the first --aligned-cpu-seqs sequences.
    threads = os.cpu_count() or 1
    n_cpu = min(args.aligned_seqs, args.aligned_cpu_seqs)
    sub_off = offsets[: n_cpu + 1]
    ref = pyoracle.OracleDb((residues[: int(sub_off[-1])], sub_off), mat, AL, GO, GE, 0, 1)
    t0 = time.perf_counter()
    ref.scan_all_aligned_mt(q, threads)
    cpu_s = time.perf_counter() - t0
    cpu_cells = float(len(q)) * float(sub_off[-1])
    peak = C.c_double()
    lib.hy_measure_dpx_peak_i32(C.byref(peak))
    peak_gcups = peak.value / 1e9
    fill_gcups = cells * args.steps / (fill_ms * 1e-3) / 1e9
    line = {
        "metric": "GCUPS", "value": cells * args.steps / (dev_ms * 1e-3) / 1e9, "unit": "GCUPS",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded protein generator: log-normal lengths, fixed background)",
        "config": {"workload": f"scan_all_aligned: 1000-residue protein query x {args.aligned_seqs} sequences "
                               "(the protein scan generator), SW, Alignment { max_bytes: usize::MAX }",
                   "residues": int(offsets[-1]), "cells_per_step": cells, "db_build_s": round(build_s, 2),
                   "ops_bytes_per_step": n_ops // args.steps,
                   "l2": "inputs larger than L2 (walk codes: 0.5 byte a cell, gigabytes a step)"},
        "e2e": {"value": cells * args.steps / (call_ms * 1e-3) / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": len(q),
                "d2h_bytes_per_step": int(n_ops // args.steps + 56 * args.aligned_seqs), "call_ms": call_ms / args.steps},
        "gpu_launches": int(all_l.value),
        "kernels": {"fill_ms_per_step": fill_ms / args.steps, "walk_and_compaction_ms_per_step": walk_ms / args.steps},
        "roofline": {"bound": "dpx_int32", "achieved": fill_gcups, "peak": peak_gcups, "unit": "GCUPS",
                     "frac": fill_gcups / peak_gcups if peak_gcups else None,
                     "traffic": (cells * TB_DRAM_BYTES_PER_CELL) if TB_DRAM_BYTES_PER_CELL else None,
                     "kernel": "tb_fill_kernel<R, SW> (R = 16 rows per lane for the 1000-residue query)",
                     "peak_source": "measured: hy_measure_dpx_peak_i32 (register-resident int32 per-cell DPX mix)"},
        "identical_to_oracle_on_sample": bool(identical),
        "cpu_baseline": {"value": cpu_cells / cpu_s / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
                         "sample": f"the first {n_cpu} sequences, scalar full-matrix traceback (src/align.rs) "
                                   f"restated in C, over {threads} threads"},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_position_max(args):
    """align_pair_position_max + score2 over --n-pos-pairs (150-bp read, 200..500-bp window) pairs
    of the align_pairs generator (bwa's mate-rescue shape): SW, +2/-1, gap_open 6, gap_ext 1,
    score2 with min_score 20. `value` is real cells / the device time of the kernels (profile
    packing, the pair kernel's column-maxima form, BestHit + score2; CUDA events); `e2e` the whole
    call with host buffers, the column maxima copied back into one caller-owned array."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    q_res, q_off, t_res, t_off = make_pairs_workload(args.seed, args.n_pos_pairs)
    dna = [2 if a == b else -1 for a in range(4) for b in range(4)]
    scoring = hy.Scoring(4, dna, 6, 1)
    cells = float(np.dot(np.diff(q_off).astype(np.float64), np.diff(t_off).astype(np.float64)))
    # One column-maxima array refilled by every call, as the reference's caller-owned `out` vector.
    cm_buf = np.empty(int(t_off[-1] - t_off[0]), np.int32)
    for _ in range(args.warmup):
        hy.align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, scoring, 20, cm_buf)
    clocks = Clocks(0)
    clocks.start()
    kms = cms = 0.0
    phases = {}
    for _ in range(args.steps):
        cm_buf.fill(-1)  # outside the timed call: every entry must be written by it
        hits, cm, s2, (err, _) = hy.align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, scoring, 20,
                                                                    cm_buf)
        assert err is None
        t = hy.position_max_timing()
        kms += t["kernel_ms"]
        cms += t["call_ms"]
        for key, v in hy.align_pairs_phases().items():
            phases[key] = phases.get(key, 0.0) + v / args.steps
    clk = clocks.stop()
    # The same calls with page-locked inputs and column-maxima array (a caller that keeps them
    # pinned): no staging copy in, the maxima copied from the device straight into the array.
    pq = hy.pinned_empty(len(q_res), np.uint8)
    pt = hy.pinned_empty(len(t_res), np.uint8)
    pcm = hy.pinned_empty(len(cm_buf), np.int32)
    pq[:] = q_res
    pt[:] = t_res
    hy.align_pairs_position_max_arrays(pq, q_off, pt, t_off, scoring, 20, pcm)
    cms_pinned = 0.0
    for _ in range(args.steps):
        pcm.fill(-1)
        hits_p, _, s2_p, (err, _) = hy.align_pairs_position_max_arrays(pq, q_off, pt, t_off, scoring, 20, pcm)
        assert err is None
        cms_pinned += hy.position_max_timing()["call_ms"]
    same_pinned = bool(np.array_equal(pcm, cm) and bytes(hits_p) == bytes(hits) and np.array_equal(s2_p, s2))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    rng = np.random.default_rng(2)
    identical = True
    for k in sorted(int(x) for x in rng.choice(args.n_pos_pairs, min(args.n_pos_pairs, 500), replace=False)):
        q = q_res[int(q_off[k]):int(q_off[k + 1])]
        t = t_res[int(t_off[k]):int(t_off[k + 1])]
        want, score, te = pyoracle.position_max(q, t, dna, 4, 6, 1)
        got = [int(v) for v in cm[int(t_off[k] - t_off[0]):int(t_off[k + 1] - t_off[0])]]
        w2 = pyoracle.score2(want, score, 0 if te is None else te, 2, 20)
        identical &= got == want and int(hits[k].score) == score and \
            int(hits[k].target_end) == (-1 if te is None else te) and \
            (int(s2[2 * k]), int(s2[2 * k + 1])) == ((0, -1) if w2 is None else w2)
    threads = os.cpu_count() or 1
    n_cpu = min(args.n_pos_pairs, args.cpu_pairs)
    sq_off, st_off = q_off[: n_cpu + 1], t_off[: n_cpu + 1]
    ccells = float(np.dot(np.diff(sq_off).astype(np.float64), np.diff(st_off).astype(np.float64)))
    t0 = time.perf_counter()
    pyoracle.position_max_many(q_res[: int(sq_off[-1])], sq_off, t_res[: int(st_off[-1])], st_off, dna, 4, 6, 1,
                               threads)
    cpu_s = time.perf_counter() - t0
    line = {
        "metric": "GCUPS", "value": cells * args.steps / (kms * 1e-3) / 1e9, "unit": "GCUPS", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": kms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "i16x2", "data": "synthetic (seeded genome reads and windows)",
        "config": {"workload": f"align_pair_position_max + score2: {args.n_pos_pairs} (150-bp read, 200..500-bp "
                               "window) pairs, SW, +2/-1, gap_open 6, gap_ext 1, min_score 20",
                   "cells_per_step": cells, "l2": "inputs larger than L2 (column maxima: 4 bytes a target residue)"},
        "e2e": {"value": cells * args.steps / (cms * 1e-3) / 1e9, "unit": "GCUPS",
                "h2d_bytes_per_step": int(len(q_res) + len(t_res)),
                "d2h_bytes_per_step": int(4 * len(t_res) + 16 * args.n_pos_pairs), "call_ms": cms / args.steps,
                "phases_ms": {k: round(v, 1) for k, v in phases.items()}},
        "e2e_pinned_buffers": {"value": cells * args.steps / (cms_pinned * 1e-3) / 1e9, "unit": "GCUPS",
                               "call_ms": cms_pinned / args.steps, "results_identical": same_pinned},
        "identical_to_oracle_on_sample": bool(identical),
        "cpu_baseline": {"value": ccells / cpu_s / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
                         "sample": f"the first {n_cpu} pairs, scalar position-max restatement over {threads} threads"},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_single_pair(args):
    """Single long pairs (align_pair's single-pair path, src/kernel.rs:331-397, and align's
    traceback): for each size in --single-sizes an m x m pair of seeded random residues of the
    protein generator's background (the second a 15%-mutated copy of the first), SW, the protein
    scoring. Per size: align_pair ScoreEnd (the score-only stripe kernel: device ms by CUDA events
    and the whole call) and align (fill, walk and the whole call); `value` is align_pair's device
    GCUPS on the first size. CPU baseline: the scalar align_core restatement on the first size."""
    import torch

    import hyalite_b200 as hy

    torch.cuda.set_device(0)
    mat, _, _, _ = make_workload(args.seed, n_seqs=2)
    scoring = hy.Scoring(AL, [int(v) for v in mat], GO, GE)
    rng = np.random.default_rng(args.seed)
    base = np.random.default_rng(12345)
    base.integers(-4, 4, size=(AL, AL))
    base.integers(4, 12, size=AL)
    background = base.dirichlet(np.full(AL, 4.0))
    sizes = [int(x) for x in args.single_sizes.split(",")]
    points = []
    pairs = []
    for m in sizes:
        q = rng.choice(AL, size=m, p=background).astype(np.uint8)
        t = q.copy()
        mut = rng.random(m) < 0.15
        t[mut] = rng.choice(AL, size=int(mut.sum()), p=background)
        pairs.append((q, t))
        for _ in range(args.warmup):
            hy.align_pair(q, t, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
            hy.align(q, t, scoring, hy.Mode.Sw, hy.USIZE_MAX)
        kms = cms = fms = wms = ams = 0.0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            h = hy.align_pair(q, t, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
            cms += time.perf_counter() - t0
            kms += hy.align_pairs_timing()[0]
            t0 = time.perf_counter()
            a = hy.align(q, t, scoring, hy.Mode.Sw, hy.USIZE_MAX)
            ams += time.perf_counter() - t0
            tt = hy.traceback_timing()
            fms += tt["fill_ms"]
            wms += tt["walk_ms"]
        k = args.steps
        points.append({"m": m, "n": m, "align_pair_kernel_ms": kms / k, "align_pair_call_ms": cms * 1e3 / k,
                       "align_pair_gcups": m * m / (kms / k * 1e-3) / 1e9, "align_fill_ms": fms / k,
                       "align_walk_ms": wms / k, "align_call_ms": ams * 1e3 / k, "score": h.score,
                       "alignment_score": a.score, "ops": len(a.ops_bytes)})
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    q, t = pairs[0]
    t0 = time.perf_counter()
    want = pyoracle.align_pair(q, t, mat, AL, GO, GE, 0)
    cpu_s = time.perf_counter() - t0
    identical = (points[0]["score"], ) == (want[0], )
    st, wa, _ = pyoracle.align(q, t, mat, AL, GO, GE, 0) if sizes[0] <= 5000 else (0, None, None)
    if wa is not None:
        identical &= hy.align(q, t, scoring, hy.Mode.Sw, hy.USIZE_MAX).as_tuple() == wa
    line = {
        "metric": "GCUPS", "value": points[0]["align_pair_gcups"], "unit": "GCUPS", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": points[0]["align_pair_kernel_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded protein background; the target a 15%-mutated copy of the query)",
        "config": {"workload": "single long pairs: align_pair ScoreEnd and align (traceback), SW, protein scoring",
                   "sizes": sizes},
        "pairs": points,
        "e2e": {"value": sizes[0] ** 2 / (points[0]["align_pair_call_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                "h2d_bytes_per_step": 2 * sizes[0], "d2h_bytes_per_step": 32},
        "identical_to_oracle": bool(identical),
        "cpu_baseline": {"value": sizes[0] ** 2 / cpu_s / 1e9, "unit": "GCUPS", "cores": 1, "kind": "port",
                         "sample": f"one {sizes[0]} x {sizes[0]} pair, scalar align_core restatement, one thread"},
    }
    print(json.dumps(line), flush=True)


def main():
    global N_SEQS, QUERY_LENGTHS, N_QUERIES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-seqs", type=int, default=20_000)
    ap.add_argument("--ref-seqs", type=int, default=100_000)
    ap.add_argument("--ref-sample-seqs", type=int, default=5_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the batched, served and align_pairs forms from the default line")
    # Smaller shapes of the same generator (profiling cases; the default is the benchmark).
    ap.add_argument("--n-seqs", type=int, default=N_SEQS)
    ap.add_argument("--query-lengths", default=",".join(map(str, QUERY_LENGTHS)))
    ap.add_argument("--n-queries", type=int, default=N_QUERIES)
    # Other workloads of the same backend (not the default benchmark line).
    ap.add_argument("--workload", default="scan",
                    choices=["scan", "batched", "served", "pairs", "dna_small", "aligned", "position_max",
                             "single_pair"])
    ap.add_argument("--single-sizes", default="2000,5000,20000")
    ap.add_argument("--n-pos-pairs", type=int, default=1_000_000)
    ap.add_argument("--dna-queries", type=int, default=1000)
    ap.add_argument("--aligned-seqs", type=int, default=100_000)
    ap.add_argument("--aligned-cpu-seqs", type=int, default=2_000)
    ap.add_argument("--n-pairs", type=int, default=10_000_000)
    ap.add_argument("--cpu-pairs", type=int, default=100_000)
    ap.add_argument("--n-reads", type=int, default=1_000_000)
    ap.add_argument("--n-batch-queries", type=int, default=256)
    ap.add_argument("--served-seqs", type=int, default=1_000_000)
    ap.add_argument("--served-rates", default="5,10,20,30,50,100,1000,20000")
    ap.add_argument("--served-seconds", type=float, default=8.0)
    ap.add_argument("--served-max-requests", type=int, default=300)
    ap.add_argument("--served-batch", type=int, default=64)
    ap.add_argument("--served-db", default="protein", choices=["protein", "dna_small"])
    ap.add_argument("--served-plain-requests", type=int, default=40)
    args = ap.parse_args()
    N_SEQS = args.n_seqs
    QUERY_LENGTHS = [int(x) for x in args.query_lengths.split(",")]
    N_QUERIES = args.n_queries
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "pairs":
        run_pairs(args)
    elif args.workload == "dna_small":
        run_dna_small(args)
    elif args.workload == "aligned":
        run_aligned(args)
    elif args.workload == "position_max":
        run_position_max(args)
    elif args.workload == "single_pair":
        run_single_pair(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
