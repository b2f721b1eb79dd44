"""Per-length-bucket tuner of the schedule table (schedule.txt).

Global score-only alignments of independent pairs (parasail_b200_batch_pairs
with nw_{striped,scan}_{8,16,32,sat}) have two schedules:

  inter  the inter-task pair kernel: one thread per pair, two 16-row
         strips of int16x2 lanes per pass (pb_pair16.cu);
  intra  the intra-task wavefront kernel: one warp (or a cluster of warps)
         per pair, 8 rows per lane, passes pipelined across the team
         (pb_nwlong.cu).

For every length bucket b (the longer sequence at most 64 << b residues) the
tuner aligns a batch of synthetic DNA pairs of that size (B = A with 10%
divergence) on each schedule on the current GPU, times both with CUDA events
and writes one line per bucket -- "nw bucket max_len inter_gcups
intra_gcups winner" -- to the table the library reads on first use
(schedule.txt beside libparasail_b200.so, or $PARASAIL_B200_SCHEDULE).

  python -m parasail_b200.tune [--out PATH] [--cells 4e9] [--max-bucket 10]
"""
import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def bucket_pairs(b, cells, seed):
    from . import synth
    hi = 64 << b
    lo = 1 if b == 0 else (32 << b) + 1
    mean = (lo + hi) / 2.0
    n = int(max(32, min(200_000, cells / (mean * mean))))
    rng = np.random.default_rng(seed + b)
    la = rng.integers(lo, hi + 1, n).astype(np.int64)
    a = synth.DNA_BYTES[rng.integers(0, 4, int(la.sum()), dtype=np.uint8)]
    ao = synth.offsets_of(la)
    bb, bo, bl = synth.mutate_many(rng, a, ao, la, 0.9, 0.02, protein=False, geom_p=0.5)
    bl = np.minimum(bl, hi).astype(np.int32)
    return a, ao, la.astype(np.int32), bb, bo, bl


def run(args):
    import torch
    from . import api as pb
    dna = pb.matrix_create("ACGT", 1, -2)
    mapper = np.ctypeslib.as_array(dna.contents.mapper, shape=(256,)).astype(np.uint8)
    name = b"nw_scan_32"
    saved = pb.lib.parasail_b200_schedule_get()
    lines = ["# parasail-b200 schedule table, written by parasail_b200/tune.py on %s (%s)"
             % (torch.cuda.get_device_name(0), time.strftime("%Y-%m-%d")),
             "# mode bucket max_len inter_gcups intra_gcups winner"]
    try:
        for b in range(args.max_bucket + 1):
            qb, qo, ql, tb, to, tl = bucket_pairs(b, args.cells, args.seed)
            n = len(ql)
            cells = float((ql.astype(np.int64) * tl).sum())
            d = [torch.from_numpy(x).cuda() for x in (mapper[qb], qo, ql, mapper[tb], to, tl)]
            rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
            rates = {}
            for sched, mask in (("inter", 0), ("intra", 1 << b)):
                pb.lib.parasail_b200_schedule_set(mask)

                def call():
                    rc = pb.lib.parasail_b200_batch_pairs_device(name, dna, *[x.data_ptr() for x in d], n, 4, 1,
                                                                 rec.data_ptr())
                    if rc != 0:
                        raise RuntimeError("batch failed")
                call()
                torch.cuda.synchronize()
                ms = []
                for _ in range(args.reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    call()
                    e1.record()
                    torch.cuda.synchronize()
                    ms.append(e0.elapsed_time(e1))
                rates[sched] = cells / (sorted(ms)[len(ms) // 2] * 1e-3) / 1e9
            # within 2% both arms ran the same kernels (pairs past the pair
            # kernel's 16-bit bounds take the wavefront kernel under either
            # schedule): the wavefront is kept
            win = "inter" if rates["inter"] > 1.02 * rates["intra"] else "intra"
            lines.append("nw %d %d %.1f %.1f %s" % (b, 64 << b, rates["inter"], rates["intra"], win))
            print(lines[-1], flush=True)
    finally:
        pb.lib.parasail_b200_schedule_set(saved)
        pb.lib.parasail_matrix_free(dna)
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "schedule.txt"))
    ap.add_argument("--cells", type=float, default=4e9, help="DP cells per bucket's batch")
    ap.add_argument("--max-bucket", type=int, default=10)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=17)
    run(ap.parse_args())


if __name__ == "__main__":
    main()
