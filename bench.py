#!/usr/bin/env python3
"""Benchmark of parasail-b200's hot path on the five reference workloads.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--legs 1,2,3,4,5]

Headline (the JSON line's top-level keys): protein database search with
Smith-Waterman score-only alignment and the reference's 8->16->32-bit
saturation chain (parasail_sw_striped_profile_sat), 5 queries (lengths 100,
250, 500, 1000, 2000) against 200,000 synthetic targets (log-normal
lengths, median 270, clipped to 20-5000, 1% planted homologs), BLOSUM62,
open 11, extend 1. One step = every query against every target.

`value` is GCUPS (cells = sum of query length x target length) with the
inputs resident in device memory; `e2e` is the same metric through the
host-memory batch API (parasail_b200_batch_db), host->device copies and
record readback included. Every one of the 1,000,000 records is compared
field by field with the records of the reference's own AVX2 kernels on the
same inputs (`parity`).

The other workloads are reported as blocks under "configs": 1 (one query
vs 1,000 targets, sw_striped_profile_16), 3 (1,000,000 DNA read/window
pairs, nw and sg_qx statistics, striped and scan, 16 bits), 4 (all-vs-all
of 4,096 proteins, sw_stats_striped_profile_32) and 5 (long DNA pairs,
global alignment, plain full DP vs the learned band). Each block carries
its own device and end-to-end GCUPS, the reference's CPU rate on the same
records and a per-field mismatch count.

The reference arm (--impl reference) times the reference's own AVX2
kernels (compiled from its sources into oracle/_ref) with OpenMP over all
host cores on the headline workload: W untimed and K timed passes over the
full workload. It loads no code of this project's library.
"""
import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS & pairs/s: batched + learned-band vs plain GPU DP, bit-exact scores"
FUNC = "sw_striped_profile_sat"
OPEN, GAP = 11, 1
QUERY_LENGTHS = (100, 250, 500, 1000, 2000)
N_TARGETS = 200_000
OPS_PER_CELL = 6   # SW score-only algorithmic lane-operations per cell
# DRAM bytes (read + write) per cell of k_sw16 on this workload, from one ncu
# capture of a full-size launch (60.1 GB for 2.7213e11 cells)
SW16_DRAM_BYTES_PER_CELL = 60.08e9 / 2.7213e11
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
FIELDS = ("score", "end_query", "end_ref", "flag", "matches", "similar", "length")


def synth():
    """The workload generators, imported without the package's native
    library (importing parasail_b200.synth maps no native code)."""
    return importlib.import_module("parasail_b200.synth")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--legs", default="1,2,3,4,5", help="configurations to run besides the headline (2)")
    ap.add_argument("--n-targets", type=int, default=N_TARGETS,
                    help="database size of the headline (the configured workload has 200,000 targets)")
    ap.add_argument("--cfg3-pairs", type=int, default=1_000_000)
    ap.add_argument("--cfg4-seqs", type=int, default=4096)
    ap.add_argument("--cfg4-stride", type=int, default=100, help="the CPU checks every STRIDE-th pair of config 4")
    ap.add_argument("--band-train", type=int, default=20_000, help="training pairs of the learned-band leg")
    ap.add_argument("--band-test", type=int, default=20_000, help="timed pairs of the learned-band leg")
    ap.add_argument("--band-cpu-pairs", type=int, default=32, help="pairs of config 5 the CPU aligns")
    return ap.parse_args()


def measured_peaks():
    """MEASURED_PEAKS.json (copy bandwidth, bf16 GEMM) when present."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "of measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0}, "of fallback"


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world


def over_ranks(world, t_max, n_sum, device):
    """Every rank's timings reduced by max and its work counts by sum: one
    all-reduce of each, in the same order on every rank."""
    if world <= 1:
        return [float(x) for x in t_max], [float(x) for x in n_sum]
    import torch
    import torch.distributed as dist
    a = torch.tensor([float(x) for x in t_max], dtype=torch.float64, device=device)
    b = torch.tensor([float(x) for x in n_sum], dtype=torch.float64, device=device)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return a.tolist(), b.tolist()


def workload(rank, n_targets=N_TARGETS):
    return synth().protein_db_search(seed=2 + rank, n_targets=n_targets, query_lengths=QUERY_LENGTHS)


def clocks_sampler(stop, out):
    cmd = ["nvidia-smi", "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-i", os.environ.get("LOCAL_RANK", "0")]
    while not stop.is_set():
        try:
            line = subprocess.run(cmd, capture_output=True, text=True, timeout=5).stdout.strip()
            if line:
                out.append(line)
        except Exception:
            pass
        stop.wait(0.2)


def summarize_clocks(samples):
    if not samples:
        return None
    sm, mx, reasons = [], 0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for s in samples:
        f = [x.strip() for x in s.split(",")]
        try:
            sm.append(float(f[0]))
            mx = max(mx, float(f[1]))
        except ValueError:
            continue
        for nm, v in zip(names, f[3:7]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
            "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's CPU kernels (oracle/_ref/ref_driver)

def write_lines(path, buf, offs, lens):
    """Sequences of a packed buffer, one per line."""
    lens = np.asarray(lens, dtype=np.int64)
    src = np.repeat(np.asarray(offs, np.int64) - synth().offsets_of(lens), lens) + np.arange(int(lens.sum()))
    dst = np.repeat(synth().offsets_of(lens + 1) - synth().offsets_of(lens), lens) + np.arange(int(lens.sum()))
    out = np.full(int(lens.sum()) + len(lens), ord("\n"), dtype=np.uint8)
    out[dst] = np.asarray(buf)[src]
    out.tofile(path)


def ref_run(family, width, mspec, open_, gap, mode, qfile, tfile, limit=None, stride=1, reps=1, warm=0,
            records=True, threads=None):
    """Runs the reference's AVX2 kernels through ref_driver. Returns a dict
    with pairs, cells, per-repetition seconds and (records=True) the
    per-pair records as int32 [pairs, 8]."""
    threads = threads or os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        rec = os.path.join(td, "rec.bin")
        cmd = [REF_DRIVER, family, str(width), mspec, str(open_), str(gap), mode, qfile, tfile or qfile,
               str(threads)]
        if limit is not None:
            cmd.append(str(limit))
        cmd += ["-s", str(stride), "-r", str(reps), "-w", str(warm)]
        if records:
            cmd += ["-o", rec]
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout.split("\n")
        f = out[0].split()
        res = {"pairs": int(f[0]), "cells": float(f[1]), "seconds": float(f[2]), "checksum": int(f[3]),
               "saturated": int(f[4]), "reps": [float(x) for x in out[1].split()[1:]], "threads": threads}
        if records:
            res["records"] = np.fromfile(rec, dtype=np.int32).reshape(-1, 8)
    return res


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_block(r, sample, kind="reference"):
    """cpu_baseline object from a ref_run result (median repetition)."""
    sec = statistics.median(r["reps"]) if r["reps"] else r["seconds"]
    return {"value": r["cells"] / sec / 1e9, "unit": "GCUPS", "cores": r["threads"], "kind": kind,
            "pairs_per_s": r["pairs"] / sec, "sample": sample, "seconds_per_pass": sec,
            "cpu": cpu_model()}


def compare(gpu, ref, fields=FIELDS):
    """Field-by-field mismatch counts of GPU records (int32 [n, 8] or the
    structured record array) against reference records (int32 [n, 8])."""
    g = np.asarray(gpu)
    if g.dtype.names:
        g = np.stack([g[f] for f in FIELDS + ("reserved",)], axis=1)
    g = g.reshape(-1, 8)
    assert g.shape == ref.shape, (g.shape, ref.shape)
    mism = {f: int((g[:, k] != ref[:, k]).sum()) for k, f in enumerate(FIELDS) if f in fields}
    any_bad = np.zeros(len(g), dtype=bool)
    for k, f in enumerate(FIELDS):
        if f in fields:
            any_bad |= g[:, k] != ref[:, k]
    first = int(np.nonzero(any_bad)[0][0]) if any_bad.any() else None
    return {"pairs_compared": int(len(g)), "mismatches": mism, "pairs_mismatched": int(any_bad.sum()),
            "first_mismatch": None if first is None else {"pair": first, "gpu": g[first].tolist(),
                                                          "reference": ref[first].tolist()}}


# ---------------------------------------------------------------------------
# device timing helpers

class Timer:
    """CUDA-event timing of synchronous library calls on the current
    stream, L2 flushed (512 MB write) before every timed call."""

    def __init__(self):
        import torch
        self.torch = torch
        self.flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def run(self, fn, steps, warmup, barrier=None):
        torch = self.torch
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            self.flush.zero_()
            torch.cuda.synchronize()
            if barrier:
                barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms


def check_rc(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed" % what)


def pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


# ---------------------------------------------------------------------------
# legs

def leg_config1(pb, timer, args, td):
    """Config 1: one protein query (300) vs 1,000 targets U[100,500],
    BLOSUM62 10/1, parasail_sw_striped_profile_16."""
    import torch
    S = synth()
    q, buf, offs, lens = S.protein_query_vs_targets(seed=1, qlen=300, n_targets=1000)
    fname, op, gp = "sw_striped_profile_16", 10, 1
    b62 = pb.matrix_lookup("blosum62")
    mapper = np.ctypeslib.as_array(b62.contents.mapper, shape=(256,)).astype(np.uint8)
    prof = pb.ProfileHandle("parasail_profile_create_16", q, b62)
    n = len(lens)
    d_codes, d_offs, d_lens = (torch.from_numpy(x).cuda() for x in (mapper[buf], offs, lens))
    d_rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    steps = max(args.steps, 20)

    def dev_call():
        check_rc(pb.lib.parasail_b200_batch_profile_device(fname.encode(), prof.ptr, d_codes.data_ptr(),
                                                           d_offs.data_ptr(), d_lens.data_ptr(), n, op, gp,
                                                           d_rec.data_ptr()), fname)

    parr = pb.ctypes.cast(pb.profile_array([prof]), pb.ctypes.c_void_p)
    plan = pb.lib.parasail_b200_db_plan_create(fname.encode(), parr, 1, d_codes.data_ptr(), d_offs.data_ptr(),
                                               d_lens.data_ptr(), n, op, gp, d_rec.data_ptr())
    if not plan:
        raise RuntimeError("parasail_b200_db_plan_create failed")

    def dev():
        check_rc(pb.lib.parasail_b200_db_plan_run(plan), "db_plan_run")
    h_buf, h_offs, h_lens = (pinned(torch, x) for x in (buf, offs, lens))
    h_rec = torch.zeros((n, 8), dtype=torch.int32).pin_memory()
    h_rec_p = torch.zeros((n, 8), dtype=torch.int32).pin_memory()

    def host():
        check_rc(pb.lib.parasail_b200_batch_profile(fname.encode(), prof.ptr, h_buf.data_ptr(), h_offs.data_ptr(),
                                                    h_lens.data_ptr(), n, op, gp, h_rec.data_ptr()), fname)

    def host_plan():
        check_rc(pb.lib.parasail_b200_db_plan_run_host(plan, h_buf.data_ptr(), int(h_buf.numel()),
                                                       h_rec_p.data_ptr()), "db_plan_run_host")
    ms = timer.run(dev, steps, args.warmup)
    rec_plan = d_rec.cpu().numpy().copy()
    ms_c = timer.run(dev_call, steps, args.warmup)
    ms_e = timer.run(host_plan, steps, args.warmup)
    ms_h = timer.run(host, steps, args.warmup)
    pb.lib.parasail_b200_db_plan_free(plan)
    cells = float(len(q)) * float(lens.sum())
    qf, tf = os.path.join(td, "c1q.txt"), os.path.join(td, "c1t.txt")
    open(qf, "wb").write(q + b"\n")
    write_lines(tf, buf, offs, lens)
    r = ref_run("sw_striped", 16, "blosum62", op, gp, "db", qf, tf, reps=20, warm=2)
    prof.close()
    med, med_e, med_h = statistics.median(ms), statistics.median(ms_e), statistics.median(ms_h)
    return {"workload": "1 protein query (300) vs 1,000 targets U[100,500], BLOSUM62 10/1, %s" % fname,
            "cells_per_step": cells, "steps": steps, "warmup": args.warmup,
            "value": cells / (med * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": med,
            "pairs_per_s": n / (med * 1e-3),
            "device_path": "parasail_b200_db_plan_run (CUDA graph replay)",
            "batch_call": {"value": cells / (statistics.median(ms_c) * 1e-3) / 1e9, "unit": "GCUPS",
                           "ms_per_step": statistics.median(ms_c),
                           "path": "parasail_b200_batch_profile_device"},
            "e2e": {"value": cells / (med_e * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": med_e,
                    "path": "parasail_b200_db_plan_run_host (target characters copied in and mapped, "
                            "graph replay, records copied out)",
                    "h2d_bytes_per_step": int(h_buf.numel()), "d2h_bytes_per_step": 32 * n},
            "host_batch_call": {"value": cells / (med_h * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": med_h,
                                "path": "parasail_b200_batch_profile (host buffers, preparation every call)"},
            "cpu_baseline": cpu_block(r, "the full workload, 20 passes (median)"),
            "parity": {"device_api": compare(rec_plan, r["records"]),
                       "batch_call": compare(d_rec.cpu().numpy(), r["records"]),
                       "host_plan": compare(h_rec_p.numpy(), r["records"]),
                       "host_api": compare(h_rec.numpy(), r["records"])}}


def leg_config3(pb, timer, args, td):
    """Config 3: 1,000,000 DNA reads U[100,300] vs their windows (read +
    32), 5% substitutions, 0.5% insertions, 0.5% deletions; +2/-3, open 5,
    extend 2; nw and sg_qx statistics, striped and scan, 16 bits."""
    import torch
    S = synth()
    rb, ro, rl, wb, wo, wl = S.dna_read_windows(seed=3, n_pairs=args.cfg3_pairs)
    n = len(rl)
    dna = pb.matrix_create("ACGT", 2, -3)
    mapper = np.ctypeslib.as_array(dna.contents.mapper, shape=(256,)).astype(np.uint8)
    d = [torch.from_numpy(x).cuda() for x in (mapper[rb], ro, rl, mapper[wb], wo, wl)]
    h = [pinned(torch, x) for x in (rb, ro, rl, wb, wo, wl)]
    d_rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    h_rec = torch.zeros((n, 8), dtype=torch.int32).pin_memory()
    cells = float((rl.astype(np.int64) * wl).sum())
    qf, tf = os.path.join(td, "c3q.txt"), os.path.join(td, "c3t.txt")
    write_lines(qf, rb, ro, rl)
    write_lines(tf, wb, wo, wl)
    steps, warm = max(1, min(args.steps, 5)), 2
    out = {"workload": "%d DNA read/window pairs (reads U[100,300], windows read+32; 5%% subs, 0.5%% ins, "
                       "0.5%% del), +2/-3, open 5, extend 2" % n,
           "cells_per_step": cells, "steps": steps, "warmup": warm, "functions": {}}
    for fam in ("nw_stats_striped", "nw_stats_scan", "sg_qx_stats_striped", "sg_qx_stats_scan"):
        fname = (fam + "_16").encode()

        def dev():
            check_rc(pb.lib.parasail_b200_batch_pairs_device(fname, dna, *[x.data_ptr() for x in d], n, 5, 2,
                                                             d_rec.data_ptr()), fam)

        def host():
            check_rc(pb.lib.parasail_b200_batch_pairs(fname, dna, *[x.data_ptr() for x in h], n, 5, 2,
                                                      h_rec.data_ptr()), fam)
        ms = timer.run(dev, steps, warm)
        ms_e = timer.run(host, steps, warm)
        r = ref_run(fam, 16, "ACGT:2:-3", 5, 2, "pairs", qf, tf)
        med, med_e = statistics.median(ms), statistics.median(ms_e)
        out["functions"][fam + "_16"] = {
            "value": cells / (med * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": med,
            "pairs_per_s": n / (med * 1e-3),
            "e2e": {"value": cells / (med_e * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": med_e, "steps": steps,
                    "h2d_bytes_per_step": int(rl.sum() + wl.sum()) + 24 * n, "d2h_bytes_per_step": 32 * n},
            "cpu_baseline": cpu_block(r, "all %d pairs, one pass" % n),
            "parity": {"device_api": compare(d_rec.cpu().numpy(), r["records"]),
                       "host_api": compare(h_rec.numpy(), r["records"])}}
    pb.lib.parasail_matrix_free(dna)
    return out


def leg_config4(pb, timer, args, td):
    """Config 4: all-vs-all of 4,096 proteins U[50,1500] (20% from 64
    families, 40% identity, 3% indels), BLOSUM62 11/1,
    sw_stats_striped_profile_32."""
    import torch
    S = synth()
    buf, offs, lens = S.protein_all_vs_all(seed=4, n_seqs=args.cfg4_seqs)
    n = len(lens)
    npairs = n * (n - 1) // 2
    fname = b"sw_stats_striped_profile_32"
    b62 = pb.matrix_lookup("blosum62")
    mapper = np.ctypeslib.as_array(b62.contents.mapper, shape=(256,)).astype(np.uint8)
    d = [torch.from_numpy(x).cuda() for x in (mapper[buf], offs, lens)]
    h = [pinned(torch, x) for x in (buf, offs, lens)]
    d_rec = torch.zeros((npairs, 8), dtype=torch.int32, device="cuda")
    h_rec = torch.zeros((npairs, 8), dtype=torch.int32).pin_memory()
    L = lens.astype(np.float64)
    cells = float((L.sum() ** 2 - (L ** 2).sum()) / 2)

    def dev():
        check_rc(pb.lib.parasail_b200_batch_all_device(fname, b62, *[x.data_ptr() for x in d], n, OPEN, GAP,
                                                       d_rec.data_ptr()), "batch_all_device")

    def host():
        check_rc(pb.lib.parasail_b200_batch_all(fname, b62, *[x.data_ptr() for x in h], n, OPEN, GAP,
                                                h_rec.data_ptr()), "batch_all")
    ms = timer.run(dev, 1, 1)
    ms_e = timer.run(host, 1, 0)
    sf = os.path.join(td, "c4.txt")
    write_lines(sf, buf, offs, lens)
    stride = args.cfg4_stride
    r = ref_run("sw_stats_striped", 32, "blosum62", OPEN, GAP, "all", sf, None, stride=stride)
    idx = np.arange(0, npairs, stride)
    return {"workload": "all-vs-all of %d proteins U[50,1500] (20%% from 64 families, 40%% identity, 3%% indels), "
                        "%d pairs, BLOSUM62 11/1, sw_stats_striped_profile_32" % (n, npairs),
            "cells_per_step": cells, "steps": 1, "warmup": 1,
            "value": cells / (ms[0] * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": ms[0],
            "pairs_per_s": npairs / (ms[0] * 1e-3),
            "e2e": {"value": cells / (ms_e[0] * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": ms_e[0],
                    "h2d_bytes_per_step": int(lens.sum()) + 12 * n, "d2h_bytes_per_step": 32 * npairs},
            "cpu_baseline": cpu_block(r, "every %d-th pair of the upper triangle (%d pairs, %.3g cells), one "
                                         "pass; extrapolate by cells" % (stride, r["pairs"], r["cells"])),
            "parity": {"device_api": compare(d_rec.cpu().numpy()[idx], r["records"]),
                       "host_api": compare(h_rec.numpy()[idx], r["records"]),
                       "sample": "every %d-th pair" % stride}}


def leg_config5(pb, args, td):
    """Config 5: long DNA pairs (5-50 kbp, 1-15% divergence, a large indel
    in 30%), +1/-2, open 4, extend 1. Plain full-DP global alignment vs the
    learned band (features + MLP + banded DP + certificate + rerun), both
    through the host API, scores compared pair by pair; the reference's
    nw_scan_profile_32 on a sample of the test pairs."""
    import torch
    S = synth()
    dna = pb.matrix_create("ACGT", 1, -2)
    t0 = time.time()
    tr = S.dna_long_pairs(seed=101, n_pairs=args.band_train)
    te = S.dna_long_pairs(seed=102, n_pairs=args.band_test)
    gen_s = time.time() - t0
    n_test = len(te[2])
    model = pb.BandModel(seed=7)
    t0 = time.time()
    loss = model.train(dna, *tr[:6], 4, 1, epochs=120, batch=256, lr=2e-3)
    train_s = time.time() - t0
    cells = float((te[2].astype(np.int64) * te[5]).sum())
    widen, slack = model.scaling()                      # chosen on held-out training pairs
    pb.nw_long(dna, *te[:6], 4, 1)                      # warm-up
    model.align(dna, *te[:6], 4, 1, widen=widen, slack=slack)
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    reps = 3                                            # median of three runs each
    runs_full = [timed(lambda: pb.nw_long(dna, *te[:6], 4, 1)) for _ in range(reps)]
    runs_band = [timed(lambda: model.align(dna, *te[:6], 4, 1, widen=widen, slack=slack)) for _ in range(reps)]
    full, t_full = runs_full[-1][0], sorted(r[1] for r in runs_full)[reps // 2]
    (sc, lo, hi, st), t_band = runs_band[-1][0], sorted(r[1] for r in runs_band)[reps // 2]
    model.close()
    # the non-learned baseline: the same certificate, bands doubling from a
    # half-width of w0 diagonals until they pass
    w0 = 64
    pb.nw_doubling_band(dna, *te[:6], 4, 1, w0)
    runs_dbl = [timed(lambda: pb.nw_doubling_band(dna, *te[:6], 4, 1, w0)) for _ in range(reps)]
    (dsc, dst), t_dbl = runs_dbl[-1][0], sorted(r[1] for r in runs_dbl)[reps // 2]
    # the reference's full DP on the first pairs of the test set
    k = min(args.band_cpu_pairs, n_test)
    qf, tf = os.path.join(td, "c5q.txt"), os.path.join(td, "c5t.txt")
    write_lines(qf, te[0], te[1][:k], te[2][:k])
    write_lines(tf, te[3], te[4][:k], te[5][:k])
    r = ref_run("nw_scan", 32, "ACGT:1:-2", 4, 1, "pairs", qf, tf)
    pb.lib.parasail_matrix_free(dna)
    ref_scores = r["records"][:, 0]
    return {"workload": "%d DNA pairs 5-50 kbp (1-15%% divergence, 30%% with a 50-500 bp indel), +1/-2, "
                        "open 4, extend 1; model trained on %d separate pairs" % (n_test, len(tr[2])),
            "cells_full_dp": cells, "generate_seconds": gen_s,
            "full_dp": {"pairs_per_s": n_test / t_full, "GCUPS": cells / t_full / 1e9, "seconds": t_full},
            "learned_band": {"pairs_per_s": n_test / t_band, "seconds": t_band,
                             "certified": int(st.certified), "rebanded": int(st.fallback),
                             "band_scaling": {"widen": widen, "slack": slack},
                             "band_cells_frac": st.band_cells / cells},
            "doubling_band": {"pairs_per_s": n_test / t_dbl, "seconds": t_dbl, "start_half_width": w0,
                              "certified_first_band": int(dst.certified), "rebanded": int(dst.fallback),
                              "band_cells_frac": dst.band_cells / cells,
                              "scores_identical_to_full_dp": bool((dsc == full).all())},
            "speedup_pairs_per_s": t_full / t_band,
            "speedup_over_doubling_band": t_dbl / t_band,
            "scores_identical_to_full_dp": bool((sc == full).all()),
            "train": {"pairs": len(tr[2]), "epochs": 120, "final_loss": loss, "seconds": train_s},
            "cpu_baseline": cpu_block(r, "reference nw_scan_profile_32 on the first %d test pairs" % k),
            "parity": {"full_dp_vs_reference_scores": {"pairs_compared": k,
                                                       "mismatches": int((full[:k] != ref_scores).sum())},
                       "learned_band_vs_full_dp_scores": {"pairs_compared": n_test,
                                                          "mismatches": int((sc != full).sum())}}}


def config_of(n_targets, world, cells):
    """The workload description both arms print."""
    return {"workload": "protein db search: queries %s vs %d log-normal targets (median 270, "
                        "1%% homologs), BLOSUM62 11/1, %s" % (list(QUERY_LENGTHS), n_targets, FUNC),
            "cells_per_step": cells * world, "l2": "flushed between timed steps (512 MB write)",
            "parallelism": "replicas x%d" % world}


def run_reference(args, rank, world):
    """The reference arm: its AVX2 8->16->32 chain with OpenMP on all host
    cores, W untimed then K timed passes over the full headline workload."""
    if rank != 0:
        return
    if not os.path.exists(REF_DRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver is not built"}))
        return
    queries, buf, offs, lens = workload(0, args.n_targets)
    with tempfile.TemporaryDirectory() as td:
        qf, tf = os.path.join(td, "q.txt"), os.path.join(td, "t.txt")
        open(qf, "wb").write(b"\n".join(queries) + b"\n")
        write_lines(tf, buf, offs, lens)
        r = ref_run("sw_striped", "sat", "blosum62", OPEN, GAP, "db", qf, tf, reps=args.steps,
                    warm=args.warmup, records=False)
    ms = statistics.mean(r["reps"]) * 1e3
    value = r["cells"] / (ms * 1e-3) / 1e9
    base = cpu_block(r, "the full workload: %d untimed + %d timed passes of all %d x %d pairs"
                     % (args.warmup, args.steps, len(queries), len(lens)))
    base["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GCUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "step_ms": [x * 1e3 for x in r["reps"]], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8/int16/int32 (reference widths)",
            "data": "synthetic", "config": config_of(len(lens), args.gpus, r["cells"]),
            "pairs_per_s": r["pairs"] / (ms * 1e-3), "cpu_baseline": base,
            "e2e": {"value": value, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        # CPU-only arm: rank 0 times the reference, the other ranks exit at once
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world = dist_init(args.gpus)
    import torch
    import parasail_b200 as pb

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    queries, buf, offs, lens = workload(rank, args.n_targets)
    n = len(lens)
    b62 = pb.matrix_lookup("blosum62")
    mapper = np.ctypeslib.as_array(b62.contents.mapper, shape=(256,)).astype(np.uint8)
    codes = mapper[buf]
    profs = [pb.ProfileHandle("parasail_profile_create_sat", q, b62) for q in queries]
    d_codes = torch.from_numpy(codes).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    d_lens = torch.from_numpy(lens).cuda()
    d_rec = torch.zeros((len(queries), n, 8), dtype=torch.int32, device="cuda")
    fname = FUNC.encode()
    parr = pb.profile_array(profs)
    parr_p = pb.ctypes.cast(parr, pb.ctypes.c_void_p)
    timer = Timer()

    def step_batch_call():
        # all queries against all targets: one pipeline, one DP kernel launch
        check_rc(pb.lib.parasail_b200_batch_db_device(fname, parr_p, len(profs), d_codes.data_ptr(),
                                                      d_offs.data_ptr(), d_lens.data_ptr(), n, OPEN, GAP,
                                                      d_rec.data_ptr()), "batch_db_device")

    # the same search prepared once and replayed as a CUDA graph
    plan = pb.lib.parasail_b200_db_plan_create(fname, parr_p, len(profs), d_codes.data_ptr(), d_offs.data_ptr(),
                                               d_lens.data_ptr(), n, OPEN, GAP, d_rec.data_ptr())
    if not plan:
        raise RuntimeError("parasail_b200_db_plan_create failed")

    def step_device():
        check_rc(pb.lib.parasail_b200_db_plan_run(plan), "db_plan_run")

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    pb.lib.parasail_b200_reset_counters()
    stop, samples = threading.Event(), []
    th = threading.Thread(target=clocks_sampler, args=(stop, samples), daemon=True)
    th.start()
    ms_dev = timer.run(step_device, args.steps, 0, barrier)
    launches = pb.lib.parasail_b200_kernel_launches()
    # the batch call (host-side preparation every call) for the kernel timing
    pb.lib.parasail_b200_reset_counters()
    ms_call = timer.run(step_batch_call, args.steps, 1, barrier)
    nk = pb.ctypes.c_long(0)
    sw16_ms = pb.lib.parasail_b200_sw16_kernel_ms(pb.ctypes.byref(nk))
    # e2e: host-memory API from pinned buffers, copies inside the timed region
    h_buf, h_offs, h_lens = (pinned(torch, x) for x in (buf, offs, lens))
    h_rec = torch.zeros((len(queries), n, 8), dtype=torch.int32).pin_memory()
    e2e_steps = args.steps

    def step_host():
        check_rc(pb.lib.parasail_b200_batch_db(fname, parr_p, len(profs), h_buf.data_ptr(), h_offs.data_ptr(),
                                               h_lens.data_ptr(), n, OPEN, GAP, h_rec.data_ptr()), "batch_db")

    ms_e2e = timer.run(step_host, e2e_steps, 1, barrier)
    stop.set()
    th.join(timeout=2)

    # times: max over ranks; cells and pairs: sum over ranks (each rank has its own shard)
    cells = float(sum(len(q) for q in queries)) * float(lens.sum())
    (ms_step, e2e_step), (cells_all, pairs_all) = over_ranks(
        world, [statistics.mean(ms_dev), statistics.mean(ms_e2e)], [cells, len(queries) * n], "cuda")
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    gcups = cells_all / (ms_step * 1e-3) / 1e9
    legs = set(x.strip() for x in args.legs.split(",") if x.strip())
    blocks = {}
    with tempfile.TemporaryDirectory() as td:
        # the headline's records, every pair, against the reference's
        qf, tf = os.path.join(td, "q.txt"), os.path.join(td, "t.txt")
        open(qf, "wb").write(b"\n".join(queries) + b"\n")
        write_lines(tf, buf, offs, lens)
        ref = ref_run("sw_striped", "sat", "blosum62", OPEN, GAP, "db", qf, tf, reps=3)
        base = cpu_block(ref, "the full workload (all %d x %d pairs), 3 passes (median)" % (len(queries), n))
        parity = {"device_api": compare(d_rec.cpu().numpy(), ref["records"]),
                  "host_api": compare(h_rec.numpy(), ref["records"])}
        for leg, fn in (("1", leg_config1), ("3", leg_config3), ("4", leg_config4)):
            if leg in legs:
                try:
                    t0 = time.time()
                    blocks[leg] = fn(pb, timer, args, td)
                    blocks[leg]["leg_seconds"] = time.time() - t0
                except Exception as e:   # a failed leg is reported, the headline still prints
                    blocks[leg] = {"error": repr(e)}
        if "5" in legs:
            try:
                t0 = time.time()
                blocks["5"] = leg_config5(pb, args, td)
                blocks["5"]["leg_seconds"] = time.time() - t0
            except Exception as e:
                blocks["5"] = {"error": repr(e)}
    peak = pb.lib.parasail_b200_dpx_peak()
    # each leg's whole-pipeline rate against the integer roofline: ops per
    # cell SW score 6, NW/SG 5, statistics + 9
    def pipe_roofline(gcups, ops):
        return {"bound": "int", "ops_per_cell": ops, "achieved": gcups * 1e9 * ops / 1e12,
                "peak": peak / 1e12, "unit": "Tops/s", "frac": gcups * 1e9 * ops / peak if peak > 0 else None,
                "note": "whole pipeline (every kernel of the call) against the live DPX peak"}
    if isinstance(blocks.get("1"), dict) and "value" in blocks["1"]:
        blocks["1"]["roofline"] = pipe_roofline(blocks["1"]["value"], 6)
    if isinstance(blocks.get("3"), dict):
        for fb in blocks["3"].get("functions", {}).values():
            fb["roofline"] = pipe_roofline(fb["value"], 14)
    if isinstance(blocks.get("4"), dict) and "value" in blocks["4"]:
        blocks["4"]["roofline"] = pipe_roofline(blocks["4"]["value"], 15)
    if isinstance(blocks.get("5"), dict) and "full_dp" in blocks["5"]:
        blocks["5"]["full_dp"]["roofline"] = pipe_roofline(blocks["5"]["full_dp"]["GCUPS"], 5)
    peaks, peaks_src = measured_peaks()
    kernel_ms_per_launch = sw16_ms / max(1, nk.value)
    achieved = cells * OPS_PER_CELL / (kernel_ms_per_launch * 1e-3)
    h2d = int(lens.sum()) + 12 * n + 256
    d2h = len(queries) * 32 * n
    line = {
        "metric": METRIC, "value": gcups, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "step_ms": ms_dev, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16x2 (int32 rerun past the 16-bit range)",
        "data": "synthetic", "config": config_of(n, world, cells),
        "pairs_per_s": pairs_all / (ms_step * 1e-3),
        "device_path": "parasail_b200_db_plan_run (the search recorded once as a CUDA graph)",
        "batch_call": {"value": cells / (statistics.mean(ms_call) * 1e-3) / 1e9, "unit": "GCUPS",
                       "ms_per_step": statistics.mean(ms_call),
                       "path": "parasail_b200_batch_db_device (host-side preparation every call)"},
        "e2e": {"value": cells_all / (e2e_step * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": e2e_step,
                "steps": e2e_steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": {"bound": "int", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "traffic": SW16_DRAM_BYTES_PER_CELL * cells,
                     "traffic_unit": "bytes per launch (ncu capture, scaled by cells)",
                     "kernel": "k_sw16", "peak_source": "live DPX viaddmax int16x2 microbenchmark",
                     "ops_per_cell": OPS_PER_CELL, "kernel_ms_per_launch": kernel_ms_per_launch},
        "roofline_hbm": {"bound": "hbm", "achieved": (int(lens.sum()) + 12 * n) / (kernel_ms_per_launch * 1e-3) / 1e9,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "note": "target bytes streamed per launch; peak %s copy bandwidth" % peaks_src},
        "cpu_baseline": base,
        "parity": parity,
        "configs": blocks,
        "clocks": summarize_clocks(samples),
    }
    print(json.dumps(line))
    pb.lib.parasail_b200_db_plan_free(plan)
    for p in profs:
        p.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
