"""GPU parity of the pairs-from-device and all-vs-all batch calls, and of
the batch path for short queries against long targets.

- parasail_b200_batch_pairs_device: device-resident codes give the records
  of parasail_b200_batch_pairs (host characters).
- parasail_b200_batch_all / _device: the upper triangle of a sequence set,
  pair p = (i, j) row-major, equals the single calls of the same function
  with sequence i as the query, and the oracle.
- queries of 8-31 rows with targets of 2048+ residues (2^14+ cells), which
  the batch path runs one warp per pair: NW, SG and SW statistics (scan and
  striped) against the oracle and the single calls.
"""
import random

import numpy as np
import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rec_tuple(r):
    return tuple(int(r[f]) for f in ("score", "end_query", "end_ref", "flag", "matches", "similar", "length"))


def test_batch_pairs_device_equals_host():
    rng = random.Random(77)
    reads, wins = [], []
    for _ in range(300):
        w = rand_seq(rng, rng.randint(132, 332), DNA)
        reads.append(mutate(rng, w[: len(w) - 32], DNA, 0.05, 0.01))
        wins.append(w)
    dna = pb.matrix_create("ACGT", 2, -3)
    mapper = np.ctypeslib.as_array(dna.contents.mapper, shape=(256,)).astype(np.uint8)
    qb, qo, ql = pb.pack(reads)
    tb, to, tl = pb.pack(wins)
    d = [torch.from_numpy(x).cuda() for x in (mapper[qb], qo, ql, mapper[tb], to, tl)]
    n = len(reads)
    for name in ("nw_stats_striped_16", "sg_qx_stats_scan_16", "sw_striped_sat", "nw_scan_sat"):
        host = pb.batch_pairs(name, dna, reads, wins, 5, 2)
        d_rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
        rc = pb.lib.parasail_b200_batch_pairs_device(name.encode(), dna, *[x.data_ptr() for x in d], n, 5, 2,
                                                     d_rec.data_ptr())
        assert rc == 0
        dev = d_rec.cpu().numpy()
        for k in range(n):
            assert tuple(dev[k][:7]) == _rec_tuple(host[k]), (name, k)
    pb.lib.parasail_matrix_free(dna)


@pytest.mark.parametrize("name,stats", [("sw_stats_striped_profile_32", 1), ("nw_stats_scan_16", 1),
                                        ("sg_qx_striped_sat", 0), ("sw_scan_profile_sat", 0)])
def test_batch_all_vs_single_calls_and_oracle(name, stats):
    rng = random.Random(hash(name) & 0xffff)
    anc = [rand_seq(rng, rng.randint(60, 400), AA) for _ in range(3)]
    seqs = [mutate(rng, anc[k % 3], AA, 0.4, 0.03) if k % 2 else rand_seq(rng, rng.randint(1, 500), AA)
            for k in range(40)]
    b62 = pb.matrix_lookup("blosum62")
    om = O.Matrix.from_struct(b62)
    recs = pb.batch_all(name, b62, seqs, 11, 1)
    n = len(seqs)
    assert len(recs) == n * (n - 1) // 2
    direct = "parasail_" + name.replace("_profile", "")
    base = name.split("_striped")[0].split("_scan")[0].replace("_stats", "")
    alg, sgf = O.alg_of(base)
    p = 0
    for i in range(n):
        for j in range(i + 1, n):
            got = pb.records_to_dicts(recs[p:p + 1], stats)[0]
            assert got == pb.align(direct, seqs[i], seqs[j], 11, 1, b62), (name, i, j)
            if not (got["flag"] & pb.FLAG_SATURATED):
                e = O.align(alg, sgf, stats, seqs[i], seqs[j], 11, 1, om)
                keys = ("score", "end_query", "end_ref") + (("matches", "similar", "length") if stats else ())
                assert all(got[k] == e[k] for k in keys), (name, i, j, got, e)
            p += 1


def test_batch_all_device_equals_host():
    rng = random.Random(5)
    seqs = [rand_seq(rng, rng.randint(20, 700), AA) for _ in range(64)]
    b62 = pb.matrix_lookup("blosum62")
    mapper = np.ctypeslib.as_array(b62.contents.mapper, shape=(256,)).astype(np.uint8)
    buf, offs, lens = pb.pack(seqs)
    host = pb.batch_all("sw_stats_striped_profile_32", b62, seqs, 11, 1)
    d = [torch.from_numpy(x).cuda() for x in (mapper[buf], offs, lens)]
    n = len(seqs)
    d_rec = torch.zeros((n * (n - 1) // 2, 8), dtype=torch.int32, device="cuda")
    assert pb.lib.parasail_b200_batch_all_device(b"sw_stats_striped_profile_32", b62, *[x.data_ptr() for x in d],
                                                 n, 11, 1, d_rec.data_ptr()) == 0
    dev = d_rec.cpu().numpy()
    for k in range(len(host)):
        assert tuple(dev[k][:7]) == _rec_tuple(host[k])


@pytest.mark.parametrize("ql", [8, 15, 16, 17, 31])
def test_short_queries_long_targets(ql):
    """Queries of 8-31 rows against targets of 2048+ residues (2^14+
    cells): the batch path gives these pairs a warp each, whose single pass
    holds the query in lane 0's rows."""
    rng = random.Random(ql)
    b62 = pb.matrix_lookup("blosum62")
    om = O.Matrix.from_struct(b62)
    q = rand_seq(rng, ql, AA)
    targets = [rand_seq(rng, rng.randint(2048, 3000), AA) for _ in range(6)]
    targets += [rand_seq(rng, 1000, AA) + q + rand_seq(rng, 1500, AA) for _ in range(2)]
    for alg_name, scheme, stats in (("nw", "striped", 0), ("sg_qx", "scan", 0), ("nw", "scan", 1),
                                    ("sg_qe_db", "striped", 1), ("sw", "scan", 1), ("sw", "striped", 1)):
        alg, sgf = O.alg_of(alg_name)
        name = "%s%s_%s_profile_16" % (alg_name, "_stats" if stats else "", scheme)
        prof = pb.ProfileHandle("parasail_profile_create%s_16" % ("_stats" if stats else ""), q, b62)
        recs = pb.records_to_dicts(pb.batch_profile(name, prof, targets, 11, 1), stats)
        for t, r in zip(targets, recs):
            assert r == pb.align_profile("parasail_" + name, prof, t, 11, 1), (name, len(t))
            if not (r["flag"] & pb.FLAG_SATURATED):
                e = O.align(alg, sgf, stats, q, t, 11, 1, om)
                keys = ("score", "end_query", "end_ref") + (("matches", "similar", "length") if stats else ())
                assert all(r[k] == e[k] for k in keys), (name, len(t), r, e)
        prof.close()


def test_schedule_table_routes_global_pairs_and_keeps_results():
    """Global score-only pairs give the same records whichever schedule the
    table names for their length bucket: the inter-task pair kernel, or the
    intra-task wavefront kernel (also the route of pairs past the pair
    kernel's 16-bit bounds); both equal the oracle."""
    rng = random.Random(91)
    dna = pb.matrix_create("ACGT", 1, -2)
    om = O.Matrix.simple("ACGT", 1, -2)
    qs, ts = [], []
    for L in (20, 70, 150, 300, 700, 1500, 3000, 9000, 20000):
        for _ in range(3):
            q = rand_seq(rng, rng.randint(L // 2, L), DNA)
            qs.append(q)
            ts.append(mutate(rng, q, DNA, 0.1, 0.02))
    saved = pb.lib.parasail_b200_schedule_get()
    try:
        out = {}
        for mask in (0, 0xFFFFFFFF, 0b1010101010):
            pb.lib.parasail_b200_schedule_set(mask)
            out[mask] = [_rec_tuple(r) for r in pb.batch_pairs("nw_scan_32", dna, qs, ts, 4, 1)]
        assert out[0] == out[0xFFFFFFFF] == out[0b1010101010]
        for q, t, r in zip(qs, ts, out[0]):
            e = O.align(O.NW, 0, 0, q, t, 4, 1, om)
            assert r[:3] == (e["score"], e["end_query"], e["end_ref"]), (len(q), len(t))
        # the 8 -> 16 -> 32 chain on the same pairs
        pb.lib.parasail_b200_schedule_set(0xFFFFFFFF)
        a = [_rec_tuple(r) for r in pb.batch_pairs("nw_striped_sat", dna, qs, ts, 4, 1)]
        pb.lib.parasail_b200_schedule_set(0)
        b = [_rec_tuple(r) for r in pb.batch_pairs("nw_striped_sat", dna, qs, ts, 4, 1)]
        assert a == b
    finally:
        pb.lib.parasail_b200_schedule_set(saved)
    pb.lib.parasail_matrix_free(dna)


def test_chunked_host_batch_equals_device_and_one_profile():
    """A host batch of 140,000 pairs runs in overlapped chunks (copies of
    chunk k + 1 during the alignment of chunk k): its records equal the
    device call's; a single-profile host batch over as many targets equals
    the device-resident profile call."""
    rng = np.random.default_rng(5)
    n = 140_000
    ql = rng.integers(20, 60, n)
    tl = ql + rng.integers(0, 20, n)
    letters = np.frombuffer(b"ACGT", np.uint8)
    qb = letters[rng.integers(0, 4, int(ql.sum()))]
    tb = letters[rng.integers(0, 4, int(tl.sum()))]
    qo = np.concatenate([[0], np.cumsum(ql)[:-1]]).astype(np.int64)
    to = np.concatenate([[0], np.cumsum(tl)[:-1]]).astype(np.int64)
    ql, tl = ql.astype(np.int32), tl.astype(np.int32)
    dna = pb.matrix_create("ACGT", 2, -3)
    mapper = np.ctypeslib.as_array(dna.contents.mapper, shape=(256,)).astype(np.uint8)
    for name in ("sg_qx_stats_striped_16", "sw_striped_sat"):
        h_rec = np.zeros((n, 8), np.int32)
        assert pb.lib.parasail_b200_batch_pairs(name.encode(), dna, qb.ctypes.data, qo.ctypes.data, ql.ctypes.data,
                                                tb.ctypes.data, to.ctypes.data, tl.ctypes.data, n, 5, 2,
                                                h_rec.ctypes.data) == 0
        d = [torch.from_numpy(x).cuda() for x in (mapper[qb], qo, ql, mapper[tb], to, tl)]
        d_rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
        assert pb.lib.parasail_b200_batch_pairs_device(name.encode(), dna, *[x.data_ptr() for x in d], n, 5, 2,
                                                       d_rec.data_ptr()) == 0
        assert np.array_equal(h_rec[:, :7], d_rec.cpu().numpy()[:, :7]), name
    q = "ACGTTGCAAGGCTTACGATCGATCGGATCCA" * 3
    targets = [bytes(tb[to[k]:to[k] + tl[k]]).decode() for k in range(n)]
    prof = pb.ProfileHandle("parasail_profile_create_16", q, dna)
    host = pb.batch_profile("nw_scan_profile_16", prof, targets, 5, 2, packed=(tb, to, tl))
    prof.close()
    # the first and the last chunk against the oracle
    pick = list(range(150)) + list(range(n - 150, n))
    exp = O.align_batch(O.NW, 0, 0, [q] * len(pick), [targets[k] for k in pick], 5, 2,
                        O.Matrix.simple("ACGT", 2, -3))
    for k, e in zip(pick, exp):
        a = host[k]
        assert (int(a["score"]), int(a["end_query"]), int(a["end_ref"])) == (e.score, e.end_query, e.end_ref), k
    pb.lib.parasail_matrix_free(dna)


def test_long_pairs_past_16_bits_run_one_warp_per_pair():
    """Pairs outside the 16-bit bounds of the pair kernels (6,000-residue DNA
    pairs at +5/-4) in pairs mode go to the exact kernels: the long ones one
    warp per pair, short ones (mixed in) one thread per pair; scores, ends
    and statistics equal the oracle's."""
    rng = random.Random(61)
    qs, ts = [], []
    for k in range(6):
        q = rand_seq(rng, rng.randint(5800, 6400), DNA)
        qs.append(q)
        ts.append(mutate(rng, q, DNA, 0.05, 0.01) if k % 2 == 0 else rand_seq(rng, rng.randint(5800, 6400), DNA))
    for _ in range(40):
        q = rand_seq(rng, rng.randint(3, 40), DNA)
        qs.append(q)
        ts.append(mutate(rng, q, DNA, 0.1, 0.02))
    m = pb.matrix_create("ACGT", 5, -4)
    om = O.Matrix.simple("ACGT", 5, -4)
    for name, alg, sgf, stats in (("sg_qx_stats_scan_32", O.SG, O.SG_CASES["sg_qx"], 1),
                                  ("nw_stats_striped_32", O.NW, 0, 1),
                                  ("sw_stats_scan_32", O.SW, 0, 1),
                                  ("sg_de_scan_32", O.SG, O.SG_CASES["sg_de"], 0)):
        got = pb.batch_pairs(name, m, qs, ts, 10, 1)
        exp = O.align_batch(alg, sgf, stats, qs, ts, 10, 1, om)
        for k, (g, e) in enumerate(zip(got, exp)):
            want = (e.score, e.end_query, e.end_ref) + ((e.matches, e.similar, e.length) if stats else ())
            have = tuple(int(g[f]) for f in ("score", "end_query", "end_ref")) + \
                (tuple(int(g[f]) for f in ("matches", "similar", "length")) if stats else ())
            assert have == want, (name, k, len(qs[k]), len(ts[k]))
    pb.lib.parasail_matrix_free(m)
