"""GPU parity of the batch API (include/parasail_b200.h) through the C ABI.

Covers the int16x2 Smith-Waterman kernel (length-sorted, two targets per
thread, strips of query rows) including its rerun of out-of-16-bit-range
pairs on the exact 32-bit kernel, the pairs mode used for read/window
batches, and the two-pass SW stats striped path.
"""
import random

import numpy as np
import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
pytestmark = pytest.mark.gpu


def _b62():
    return O.Matrix.from_struct(pb.matrix_lookup("blosum62"))


def _oracle_batch(alg, sgf, stats, q, targets, op, gp, m):
    res = O.align_batch(alg, sgf, stats, [q] * len(targets), targets, op, gp, m)
    return [(r.score, r.end_query, r.end_ref, r.matches, r.similar, r.length) for r in res]


@pytest.mark.parametrize("qlen", [1, 15, 16, 17, 100, 333, 480, 1200])
def test_sw16_batch_vs_oracle(qlen):
    rng = random.Random(qlen)
    q = rand_seq(rng, qlen, AA)
    targets = []
    for k in range(700):
        r = rng.random()
        if r < 0.1:
            targets.append(mutate(rng, q, AA, 0.2, 0.03))
        elif r < 0.15:
            targets.append(q)
        else:
            targets.append(rand_seq(rng, rng.randint(1, 600), AA))
    b62 = pb.matrix_lookup("blosum62")
    prof = pb.ProfileHandle("parasail_profile_create_sat", q, b62)
    recs = pb.batch_profile("sw_striped_profile_sat", prof, targets, 11, 1)
    prof.close()
    exp = _oracle_batch(O.SW, 0, 0, q, targets, 11, 1, _b62())
    for k, (r, e) in enumerate(zip(recs, exp)):
        assert (r["score"], r["end_query"], r["end_ref"]) == e[:3], (k, targets[k], r, e)
        # width the reference's chain reports: 8 bits while the score fits
        # the biased 8-bit limit (255 - 12 for BLOSUM62), else 16
        want = pb.FLAG_BITS_8 if e[0] <= 127 - 11 - 1 + 128 else pb.FLAG_BITS_16
        assert r["flag"] & (pb.FLAG_BITS_8 | pb.FLAG_BITS_16 | pb.FLAG_BITS_32) == want


def test_sw16_overflow_rerun_exact():
    """Scores beyond the 16-bit lanes' range go to the exact kernel."""
    rng = random.Random(3)
    m = pb.matrix_create("ACGT", 100, -100)
    q = rand_seq(rng, 800, DNA)
    targets = [q[:500], q, mutate(rng, q, DNA, 0.01, 0.0), rand_seq(rng, 300, DNA), q[:200]]
    prof = pb.ProfileHandle("parasail_profile_create_sat", q, m)
    recs = pb.batch_profile("sw_striped_profile_sat", prof, targets, 10, 1)
    prof.close()
    om = O.Matrix.simple("ACGT", 100, -100)
    exp = _oracle_batch(O.SW, 0, 0, q, targets, 10, 1, om)
    for r, e in zip(recs, exp):
        assert (r["score"], r["end_query"], r["end_ref"]) == e[:3]
    # 16-bit biased lanes hold scores up to 65535 - 101 (src/sw_striped_avx2_256_16.c:205)
    assert recs[0]["score"] == 50000 and recs[0]["flag"] & pb.FLAG_BITS_16
    assert recs[1]["score"] == 80000 and recs[1]["flag"] & pb.FLAG_BITS_32


def test_batch_matches_per_pair_api():
    rng = random.Random(9)
    b62 = pb.matrix_lookup("blosum62")
    q = rand_seq(rng, 230, AA)
    targets = [mutate(rng, q, AA, 0.5, 0.05) if k % 3 == 0 else rand_seq(rng, rng.randint(20, 400), AA)
               for k in range(60)]
    for name, creator in [("sw_striped_profile_16", "parasail_profile_create_16"),
                          ("nw_scan_profile_sat", "parasail_profile_create_sat"),
                          ("sg_qx_stats_striped_profile_16", "parasail_profile_create_stats_16"),
                          ("sw_stats_striped_profile_sat", "parasail_profile_create_stats_sat"),
                          ("sw_stats_scan_profile_32", "parasail_profile_create_stats_32")]:
        prof = pb.ProfileHandle(creator, q, b62)
        recs = pb.records_to_dicts(pb.batch_profile(name, prof, targets, 11, 1), "stats" in name)
        for t, r in zip(targets, recs):
            assert r == pb.align_profile("parasail_" + name, prof, t, 11, 1), (name, t)
        prof.close()


def test_pairs_mode_reads_vs_windows():
    rng = random.Random(4)
    reads, wins = [], []
    for _ in range(400):
        w = rand_seq(rng, rng.randint(132, 332), DNA)
        reads.append(mutate(rng, w[: len(w) - 32], DNA, 0.05, 0.01))
        wins.append(w)
    dna = pb.matrix_create("ACGT", 2, -3)
    om = O.Matrix.simple("ACGT", 2, -3)
    for name, alg, sgf in [("nw_stats_scan_16", O.NW, 0), ("sg_qx_stats_striped_16", O.SG, O.S1_BEG | O.S1_END),
                           ("nw_stats_striped_16", O.NW, 0), ("sg_qx_stats_scan_16", O.SG, O.S1_BEG | O.S1_END)]:
        recs = pb.batch_pairs(name, dna, reads, wins, 5, 2)
        res = O.align_batch(alg, sgf, 1, reads, wins, 5, 2, om)
        for r, e in zip(recs, res):
            assert (r["score"], r["end_query"], r["end_ref"], r["matches"], r["similar"], r["length"]) == \
                (e.score, e.end_query, e.end_ref, e.matches, e.similar, e.length)
            assert r["flag"] & pb.FLAG_BITS_16 and not (r["flag"] & pb.FLAG_SATURATED)


def test_faststats_batch_vs_oracle():
    rng = random.Random(21)
    b62 = pb.matrix_lookup("blosum62")
    q = rand_seq(rng, 700, AA)
    targets = [mutate(rng, q[rng.randint(0, 300):], AA, 0.6, 0.03) if k % 4 == 0
               else rand_seq(rng, rng.randint(50, 1500), AA) for k in range(200)]
    prof = pb.ProfileHandle("parasail_profile_create_stats_32", q, b62)
    recs = pb.batch_profile("sw_stats_striped_profile_32", prof, targets, 11, 1)
    prof.close()
    exp = _oracle_batch(O.SW, 0, 1, q, targets, 11, 1, _b62())
    for r, e in zip(recs, exp):
        assert (r["score"], r["end_query"], r["end_ref"], r["matches"], r["similar"], r["length"]) == e


def test_db_batch_matches_single_query_batches():
    rng = random.Random(17)
    b62 = pb.matrix_lookup("blosum62")
    queries = [rand_seq(rng, L, AA) for L in (5, 40, 100, 250, 777)]
    targets = [rand_seq(rng, rng.randint(1, 900), AA) for _ in range(500)]
    targets += [mutate(rng, q, AA, 0.3, 0.02) for q in queries]
    profs = [pb.ProfileHandle("parasail_profile_create_sat", q, b62) for q in queries]
    db = pb.batch_db("sw_striped_profile_sat", profs, targets, 11, 1)
    for k, p in enumerate(profs):
        one = pb.batch_profile("sw_striped_profile_sat", p, targets, 11, 1)
        assert (db[k] == one).all()
        exp = _oracle_batch(O.SW, 0, 0, queries[k], targets, 11, 1, _b62())
        assert [(int(r["score"]), int(r["end_query"]), int(r["end_ref"])) for r in one] == [e[:3] for e in exp]
    for p in profs:
        p.close()


def test_db_batch_non_score_modes_match_single_query_batches():
    """Database searches through the pair kernel (every function but the SW
    score search): queries whose target counts are not multiples of a warp
    task, so task boundaries fall inside a query's items unless the batch
    aligns them."""
    rng = random.Random(19)
    b62 = pb.matrix_lookup("blosum62")
    queries = [rand_seq(rng, L, AA) for L in (7, 33, 100, 250, 500)]
    targets = [rand_seq(rng, rng.randint(1, 700), AA) for _ in range(505)]
    targets += [mutate(rng, q, AA, 0.3, 0.02) for q in queries]
    for name, creator, alg, st in (("nw_stats_scan_profile_16", "parasail_profile_create_stats_16", O.NW, 1),
                                   ("sw_stats_striped_profile_32", "parasail_profile_create_stats_32", O.SW, 1),
                                   ("sg_qx_striped_profile_sat", "parasail_profile_create_sat", O.SG, 0)):
        profs = [pb.ProfileHandle(creator, q, b62) for q in queries]
        db = pb.batch_db(name, profs, targets, 11, 1)
        for k, p in enumerate(profs):
            one = pb.batch_profile(name, p, targets, 11, 1)
            assert (db[k] == one).all(), (name, k)
        sgf = O.S1_BEG | O.S1_END if alg == O.SG else 0
        exp = _oracle_batch(alg, sgf, st, queries[2], targets, 11, 1, _b62())
        got = [(int(r["score"]), int(r["end_query"]), int(r["end_ref"])) + ((int(r["matches"]), int(r["similar"]),
               int(r["length"])) if st else ()) for r in db[2]]
        assert got == [tuple(e) if st else tuple(e[:3]) for e in exp], name
        for p in profs:
            p.close()


def test_records_reserved_field_is_zero_and_host_equals_single_calls():
    """The host batch calls copy the device's records straight into the
    caller's array: the reserved field is 0, and every other field equals
    the single-call result, across the 8 -> 16 -> 32 chain with statistics
    and pairs near the saturation bounds."""
    rng = random.Random(41)
    dna = pb.matrix_create("ACGT", 2, -3)
    for name, creator, st in (("nw_stats_striped_profile_sat", "parasail_profile_create_stats_sat", 1),
                              ("sg_qx_striped_profile_sat", "parasail_profile_create_sat", 0),
                              ("sw_striped_profile_sat", "parasail_profile_create_sat", 0)):
        q = rand_seq(rng, 180, DNA)
        targets = [mutate(rng, q, DNA, 0.02, 0.01) if k % 2 else rand_seq(rng, rng.randint(20, 400), DNA)
                   for k in range(120)]
        prof = pb.ProfileHandle(creator, q, dna)
        recs = pb.batch_profile(name, prof, targets, 5, 2)
        assert (recs["reserved"] == 0).all()
        for t, r in zip(targets, pb.records_to_dicts(recs, st)):
            assert r == pb.align_profile("parasail_" + name, prof, t, 5, 2), (name, t)
        prof.close()


@pytest.mark.parametrize("width", ["16", "32", "sat"])
def test_long_query_batches_nw_sg_vs_oracle(width):
    """Batches run one warp per pair (lanes on 16-row slices of 512-row
    passes) for every query of 32 rows and more: NW and the SG end variants
    against the oracle and against the single calls (one thread per pair),
    query lengths at the pass and lane boundaries and below a pass, and
    targets from short to several times the query; flags from the width
    chain."""
    rng = random.Random({"16": 16, "32": 32, "sat": 3}[width])
    b62 = pb.matrix_lookup("blosum62")
    om = _b62()
    for alg_name in ("nw", "sg", "sg_qx", "sg_db", "sg_qe_de", "sg_qb_de"):
        alg, sgf = O.alg_of(alg_name)
        for ql in (100, 300, 512, 513, 1023, 1024, 1300):
            q = rand_seq(rng, ql, AA)
            # targets from a few residues to several times the query
            targets = [mutate(rng, q, AA, 0.2, 0.03) if k % 4 == 0 else
                       rand_seq(rng, rng.randint(2700, 3000) if k % 3 == 1 else rng.randint(1, 900), AA)
                       for k in range(10)]
            prof = pb.ProfileHandle("parasail_profile_create_%s" % width, q, b62)
            recs = pb.records_to_dicts(pb.batch_profile("%s_striped_profile_%s" % (alg_name, width), prof,
                                                        targets, 11, 1), 0)
            for t, r in zip(targets, recs):
                e = O.align(alg, sgf, 0, q, t, 11, 1, om)
                one = pb.align_profile("parasail_%s_striped_profile_%s" % (alg_name, width), prof, t, 11, 1)
                assert r == one, (alg_name, width, ql, len(t))
                if not (r["flag"] & pb.FLAG_SATURATED):
                    assert (r["score"], r["end_query"], r["end_ref"]) == (e["score"], e["end_query"], e["end_ref"]), \
                        (alg_name, width, ql, len(t), r, e)
            prof.close()


@pytest.mark.parametrize("width", ["16", "32", "sat"])
def test_long_query_batches_with_statistics_vs_oracle(width):
    """Long pairs with statistics run one warp per pair (lanes on 8-row
    slices of 256-row passes): NW and SG statistics (striped), SW statistics
    (scan) and the prefix pass of SW statistics striped (FASTSTATS) against
    the oracle, query lengths at the pass and lane boundaries; the single
    calls (one thread per pair) must agree."""
    rng = random.Random({"16": 61, "32": 62, "sat": 63}[width])
    b62 = pb.matrix_lookup("blosum62")
    om = _b62()
    for alg_name, scheme in (("nw", "striped"), ("sg_qe_db", "striped"), ("sg_qx", "scan"), ("sw", "scan"),
                             ("sw", "striped")):
        alg, sgf = O.alg_of(alg_name)
        for ql in (100, 256, 257, 300, 513, 800):
            q = rand_seq(rng, ql, AA)
            targets = [mutate(rng, q, AA, 0.2, 0.03) if k % 4 == 0 else
                       rand_seq(rng, rng.randint(2700, 3000) if k % 3 == 1 else rng.randint(1, 700), AA)
                       for k in range(8)]
            prof = pb.ProfileHandle("parasail_profile_create_stats_%s" % width, q, b62)
            name = "%s_stats_%s_profile_%s" % (alg_name, scheme, width)
            recs = pb.records_to_dicts(pb.batch_profile(name, prof, targets, 11, 1), 1)
            for t, r in zip(targets, recs):
                assert r == pb.align_profile("parasail_" + name, prof, t, 11, 1), (name, ql, len(t))
                if not (r["flag"] & pb.FLAG_SATURATED):
                    e = O.align(alg, sgf, 1, q, t, 11, 1, om)
                    for k in ("score", "end_query", "end_ref", "matches", "similar", "length"):
                        assert r[k] == e[k], (name, ql, len(t), r, e)
            prof.close()
