#!/usr/bin/env python3
"""Benchmark of parasail-b200's hot path: batched protein database search
with Smith-Waterman score-only alignment and the reference's 8->16->32-bit
saturation chain (parasail_sw_striped_profile_sat), 5 queries (lengths 100,
250, 500, 1000, 2000) against 200,000 synthetic targets (log-normal lengths,
median 270, clipped to 20-5000, 1% planted homologs), BLOSUM62, open 11,
extend 1.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = every query against every target. `value` is GCUPS (cells =
sum of query length x target length) with the inputs resident in device
memory; `e2e` is the same metric through the host-memory batch API
(parasail_b200_batch_profile), host->device copies and result readback
included. The reference arm times the reference's own AVX2 striped kernels
(built from its sources into oracle/_ref) with OpenMP over all host cores on
a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS & pairs/s: batched + learned-band vs plain GPU DP, bit-exact scores"
FUNC = "sw_striped_profile_sat"
OPEN, GAP = 11, 1
QUERY_LENGTHS = (100, 250, 500, 1000, 2000)
N_TARGETS = 200_000
OPS_PER_CELL = 6   # SW score-only algorithmic lane-operations per cell
# DRAM bytes (read + write) per cell of k_sw16 on this workload, from one full-size ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum = 136.2 GB for 2.7213e11 cells; profiles/k_sw16_db_search.md)
SW16_DRAM_BYTES_PER_CELL = 136.18e9 / 2.7213e11


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="approximate CPU time of the bounded CPU-baseline sample")
    ap.add_argument("--n-targets", type=int, default=N_TARGETS,
                    help="database size (the configured workload has 200,000 targets)")
    ap.add_argument("--band-train", type=int, default=2000, help="training pairs of the learned-band leg")
    ap.add_argument("--band-test", type=int, default=300, help="timed pairs of the learned-band leg")
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
    from parasail_b200 import synth
    return synth.protein_db_search(seed=2 + rank, n_targets=n_targets, query_lengths=QUERY_LENGTHS)


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


def ref_driver_run(queries, buf, offs, lens, ntargets, threads, tmpdir):
    """Runs oracle/_ref/ref_driver (the reference's AVX2 striped kernels,
    8->16->32 chain, OpenMP) on every query against the first ntargets
    targets. Returns (pairs, cells, seconds, checksum, nsat)."""
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    qf = os.path.join(tmpdir, "q.txt")
    tf = os.path.join(tmpdir, "t.txt")
    with open(qf, "wb") as f:
        f.write(b"\n".join(queries) + b"\n")
    with open(tf, "wb") as f:
        for k in range(ntargets):
            f.write(buf[offs[k]:offs[k] + lens[k]].tobytes() + b"\n")
    out = subprocess.run([drv, "sw_striped", "sat", "blosum62", str(OPEN), str(GAP), "db", qf, tf,
                          str(threads)], capture_output=True, text=True, check=True).stdout.split()
    return int(out[0]), float(out[1]), float(out[2]), int(out[3]), int(out[4])


def cpu_baseline(queries, buf, offs, lens, target_seconds):
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(drv):
        return None, "oracle/_ref/ref_driver not built"
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        n0 = min(2000, len(lens))
        _, cells, sec, _, _ = ref_driver_run(queries, buf, offs, lens, n0, threads, td)
        rate = cells / max(sec, 1e-6)
        per_target = cells / n0
        nt = int(min(len(lens), max(n0, target_seconds * rate / per_target)))
        pairs, cells, sec, chk, nsat = ref_driver_run(queries, buf, offs, lens, nt, threads, td)
    return {"value": cells / sec / 1e9, "unit": "GCUPS", "cores": threads, "kind": "reference",
            "pairs_per_s": pairs / sec, "sample": "all %d queries x first %d of %d targets (%.3g cells), "
            "reference AVX2 sw_striped_profile 8->16->32 chain, OpenMP guided" % (len(queries), nt, len(lens), cells),
            "ntargets": nt, "checksum": chk, "saturated_32": nsat}, None


def learned_band_leg(pb, n_train=2000, n_test=300, epochs=120):
    """Config-5 leg: long DNA pairs (5-50 kbp, 1-15% divergence, a large
    indel in 30%), +1/-2, open 4, extend 1. Plain full-DP global alignment
    vs the learned band (features + MLP + banded DP + certificate + full-DP
    fallback), both through the host API, scores compared pair by pair."""
    import numpy as np
    import torch
    from parasail_b200 import synth
    dna = pb.matrix_create("ACGT", 1, -2)
    tr = synth.dna_long_pairs(seed=101, n_pairs=n_train)
    te = synth.dna_long_pairs(seed=102, n_pairs=n_test)
    model = pb.BandModel(seed=7)
    t0 = time.time()
    loss = model.train(dna, *tr[:6], 4, 1, epochs=epochs, batch=256, lr=2e-3)
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
    return {"workload": "%d DNA pairs 5-50 kbp (1-15%% divergence, 30%% with a 50-500 bp indel), +1/-2, "
                        "open 4, extend 1; model trained on %d separate pairs" % (n_test, n_train),
            "full_dp": {"pairs_per_s": n_test / t_full, "GCUPS": cells / t_full / 1e9, "seconds": t_full},
            "learned_band": {"pairs_per_s": n_test / t_band, "seconds": t_band,
                             "certified": int(st.certified), "rebanded": int(st.fallback),
                             "band_scaling": {"widen": widen, "slack": slack},
                             "band_cells_frac": st.band_cells / cells},
            "speedup_pairs_per_s": t_full / t_band,
            "scores_identical_to_full_dp": bool((sc == full).all()),
            "train": {"pairs": n_train, "epochs": epochs, "final_loss": loss, "seconds": train_s}}


def config_of(n_targets, world, cells):
    """The workload description both arms print."""
    return {"workload": "protein db search: queries %s vs %d log-normal targets (median 270, "
                        "1%% homologs), BLOSUM62 11/1, %s" % (list(QUERY_LENGTHS), n_targets, FUNC),
            "cells_per_step": cells * world, "l2": "flushed between timed steps (512 MB write)",
            "parallelism": "replicas x%d" % world}


def run_reference(args, rank, world):
    if rank != 0:
        return
    queries, buf, offs, lens = workload(0, args.n_targets)
    base, why = cpu_baseline(queries, buf, offs, lens, args.cpu_seconds)
    if base is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    cells_full = float(sum(QUERY_LENGTHS)) * float(lens.sum())
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "GCUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cells_full / (base["value"] * 1e9) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8/int16/int32 (reference widths)",
            "data": "synthetic", "config": config_of(len(lens), args.gpus, cells_full),
            "pairs_per_s": base["pairs_per_s"], "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        # CPU-only arm: rank 0 times the reference, the other ranks exit at once
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world = dist_init(args.gpus)
    import numpy as np
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
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    fname = FUNC.encode()
    parr = pb.profile_array(profs)
    parr_p = pb.ctypes.cast(parr, pb.ctypes.c_void_p)

    def step_device():
        # all queries against all targets: one pipeline, one DP kernel launch
        rc = pb.lib.parasail_b200_batch_db_device(fname, parr_p, len(profs), d_codes.data_ptr(), d_offs.data_ptr(),
                                                  d_lens.data_ptr(), n, OPEN, GAP, d_rec.data_ptr())
        if rc != 0:
            raise RuntimeError("batch call failed")

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
    total_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()                      # L2 flush between timed steps (untimed)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step_device()
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
    launches = pb.lib.parasail_b200_kernel_launches()
    nk = pb.ctypes.c_long(0)
    sw16_ms = pb.lib.parasail_b200_sw16_kernel_ms(pb.ctypes.byref(nk))
    # e2e: host-memory API from pinned buffers, copies inside the timed region
    h_buf = torch.from_numpy(buf).pin_memory()
    h_offs = torch.from_numpy(offs).pin_memory()
    h_lens = torch.from_numpy(lens).pin_memory()
    h_rec = np.zeros(len(queries) * n, dtype=pb.record_dtype())
    e2e_ms = 0.0
    e2e_steps = max(1, min(args.steps, 3))

    def step_host():
        rc = pb.lib.parasail_b200_batch_db(fname, parr_p, len(profs), h_buf.data_ptr(), h_offs.data_ptr(),
                                           h_lens.data_ptr(), n, OPEN, GAP, h_rec.ctypes.data)
        if rc != 0:
            raise RuntimeError("batch call failed")

    step_host()                            # untimed warm-up of the host path
    torch.cuda.synchronize()
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step_host()
        e1.record()
        torch.cuda.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    stop.set()
    th.join(timeout=2)

    # times: max over ranks; cells and pairs: sum over ranks (each rank has its own shard)
    cells = float(sum(len(q) for q in queries)) * float(lens.sum())
    (ms_step, e2e_step), (cells_all, pairs_all) = over_ranks(
        world, [total_ms / args.steps, e2e_ms / e2e_steps], [cells, len(queries) * n], "cuda")
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    gcups = cells_all / (ms_step * 1e-3) / 1e9
    # the device and host paths must agree, and both with the reference
    dev_rec = d_rec.cpu().numpy()
    h_rec = h_rec.reshape(len(queries), n)
    same = all((dev_rec[q][:, 0] == h_rec[q]["score"]).all() and (dev_rec[q][:, 3] == h_rec[q]["flag"]).all()
               for q in range(len(queries)))
    base, why = cpu_baseline(queries, buf, offs, lens, args.cpu_seconds)
    parity = None
    if base is not None:
        nt = base["ntargets"]
        ours = int(sum(int(dev_rec[q][:nt, 0].astype(np.int64).sum()) for q in range(len(queries))))
        parity = {"pairs_checked": len(queries) * nt, "score_checksum_equal": ours == base["checksum"],
                  "device_and_host_api_equal": bool(same)}
    lb = learned_band_leg(pb, n_train=args.band_train, n_test=args.band_test)
    peak = pb.lib.parasail_b200_dpx_peak()
    peaks, peaks_src = measured_peaks()
    kernel_ms_per_launch = sw16_ms / max(1, nk.value)
    cells_per_launch = cells
    achieved = cells_per_launch * OPS_PER_CELL / (kernel_ms_per_launch * 1e-3)
    h2d = int(lens.sum()) + 12 * n + 256
    d2h = len(queries) * 32 * n
    line = {
        "metric": METRIC, "value": gcups, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int16x2 (int32 rerun past the 16-bit range)", "data": "synthetic",
        "config": config_of(n, world, cells),
        "pairs_per_s": pairs_all / (ms_step * 1e-3),
        "e2e": {"value": cells_all / (e2e_step * 1e-3) / 1e9, "unit": "GCUPS",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": {"bound": "int", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "traffic": SW16_DRAM_BYTES_PER_CELL * cells_per_launch,
                     "traffic_unit": "bytes per launch (ncu capture, scaled by cells)",
                     "kernel": "k_sw16", "peak_source": "live DPX viaddmax int16x2 microbenchmark",
                     "ops_per_cell": OPS_PER_CELL, "kernel_ms_per_launch": kernel_ms_per_launch},
        "roofline_hbm": {"bound": "hbm", "achieved": (int(lens.sum()) + 12 * n) / (kernel_ms_per_launch * 1e-3) / 1e9,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "note": "target bytes streamed per launch; peak %s copy bandwidth" % peaks_src},
        "cpu_baseline": base if base is not None else {"unavailable": why},
        "parity": parity,
        "config5_learned_band": lb,
        "clocks": summarize_clocks(samples),
    }
    print(json.dumps(line))
    for p in profs:
        p.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
