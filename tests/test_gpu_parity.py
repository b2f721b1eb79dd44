"""GPU parity: every parasail.h entry point of parasail-b200, called through
the C ABI, against the oracle and the reference's own outputs.

* serial forms (parasail_sw, parasail_nw_stats_scan, ...) vs the oracle's
  restatement of the reference's serial DP: score, ends and stats, bit-exact;
* striped/scan profile forms at 8/16/32 bits and the _sat chains vs the
  golden outputs of the reference's AVX2 kernels (tests/golden/vector_golden.json),
  flags included, and vs the live reference library when it was built;
* parasail_nw_banded vs the oracle's banded restatement.
"""
import json
import os
import random

import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ALGS = ["sw", "nw", "sg", "sg_qb", "sg_qe", "sg_qx", "sg_db", "sg_de", "sg_dx",
        "sg_qb_de", "sg_qe_db", "sg_qb_db", "sg_qe_de"]

pytestmark = pytest.mark.gpu


def _pb_matrix(key):
    if isinstance(key, str):
        return pb.matrix_lookup(key)
    return pb.matrix_create(key[0], key[1], key[2])


def _o_matrix(key, cache={}):
    k = key if isinstance(key, str) else tuple(key)
    if k not in cache:
        if isinstance(key, str):
            g = json.load(open(os.path.join(GOLDEN, "matrices.json")))[key]
            cache[k] = O.Matrix(g["values"], g["mapper"], g["alphabet"], g["max"], g["min"], key)
        else:
            cache[k] = O.Matrix.simple(key[0], key[1], key[2])
    return cache[k]


def test_kat_test_basic():
    # reference tests/test_basic.c:22-80
    b62 = pb.matrix_lookup("blosum62")
    assert pb.align("parasail_sw", "asdf", "asdf", 10, 1, b62)["score"] == 20
    assert pb.align("parasail_sw", "asdf", "asdf", 10, 1, pb.matrix_lookup("pam50"))["score"] == 27
    acgt = pb.matrix_create("acgt", 1, -1)
    assert pb.align("parasail_sw", "acgt", "acgt", 10, 1, acgt)["score"] == 4
    prof = pb.ProfileHandle("parasail_profile_create_8", "asdf", b62)
    assert pb.align_profile("parasail_sw_striped_profile_8", prof, "asdf", 10, 1)["score"] == 20
    prof.close()


@pytest.mark.parametrize("alg_name", ALGS)
def test_serial_forms_vs_oracle(alg_name):
    rng = random.Random(len(alg_name) * 7919)
    alg, sgf = O.alg_of(alg_name)
    for stats in (0, 1):
        for scan in (0, 1):
            for it in range(6):
                if it % 2:
                    key, a, op, gp = "blosum62", AA, 11, 1
                else:
                    key, a, op, gp = ("ACGT", 2, -3), DNA, 5, 2
                q = rand_seq(rng, rng.randint(1, 200), a)
                t = mutate(rng, q, a) if it % 3 == 0 else rand_seq(rng, rng.randint(1, 200), a)
                name = "parasail_%s%s%s" % (alg_name, "_stats" if stats else "", "_scan" if scan else "")
                got = pb.align(name, q, t, op, gp, _pb_matrix(key))
                exp = O.align(alg, sgf, stats, q, t, op, gp, _o_matrix(key))
                for k in exp:
                    assert got[k] == exp[k], (name, q, t, got, exp)
                assert got["flag"] & (pb.FLAG_NOVEC_SCAN if scan else pb.FLAG_NOVEC)


@pytest.mark.parametrize("alg_name", ["sw", "nw", "sg", "sg_qx", "sg_qe_db", "sg_qb_de", "sg_dx"])
def test_serial_scan_open_below_gap_vs_oracle(alg_name):
    """parasail_*_scan at open < gap, where the reference's serial scan forms
    extend a vertical gap only from max(diagonal, E) and so differ from the
    serial DP: against the oracle's restatement of those forms (and the live
    reference when it was built), for queries on the thread kernel (< 32
    rows), the warp kernel and several warp passes (> 512 rows)."""
    rng = random.Random(len(alg_name) * 104729)
    alg, sgf = O.alg_of(alg_name)
    differs = 0
    for it in range(12):
        key, a = ("blosum62", AA) if it % 2 else (("ACGT", 2, -3), DNA)
        op, gp = rng.choice([(0, 1), (1, 2), (2, 5), (1, 3)])
        ql = rng.choice([rng.randint(1, 31), rng.randint(32, 300), rng.randint(513, 1300)])
        q = rand_seq(rng, ql, a)
        t = mutate(rng, q, a) if it % 3 == 0 else rand_seq(rng, rng.randint(1, 900), a)
        got = pb.align("parasail_%s_scan" % alg_name, q, t, op, gp, _pb_matrix(key))
        exp = O.align_scan(alg, sgf, q, t, op, gp, _o_matrix(key))
        assert {k: got[k] for k in exp} == exp, (alg_name, op, gp, len(q), len(t), got, exp)
        assert got["flag"] & pb.FLAG_NOVEC_SCAN
        if O.ref() is not None:
            r = O.ref_serial(alg_name, 0, q, t, op, gp, key, scan=True)
            assert {k: r[k] for k in exp} == exp
        differs += exp != O.align(alg, sgf, 0, q, t, op, gp, _o_matrix(key))
        # the plain serial form keeps the serial DP
        assert {k: v for k, v in pb.align("parasail_%s" % alg_name, q, t, op, gp, _pb_matrix(key)).items()
                if k in exp} == O.align(alg, sgf, 0, q, t, op, gp, _o_matrix(key))
    assert differs >= 1


@pytest.mark.parametrize("alg_name", ["sw", "nw", "sg", "sg_qx", "sg_qe_db", "sg_qb_de", "sg_dx"])
def test_serial_stats_scan_open_below_gap_vs_oracle(alg_name):
    """parasail_*_stats_scan at open < gap (the vertical gap of the
    reference's serial scan forms, with the counts of the cells it chooses):
    against the oracle's restatement (and the live reference when it was
    built), for queries on the thread kernel (< 32 rows), the warp kernel and
    several warp passes."""
    rng = random.Random(len(alg_name) * 7919)
    alg, sgf = O.alg_of(alg_name)
    differs = 0
    for it in range(12):
        key, a = ("blosum62", AA) if it % 2 else (("ACGT", 2, -3), DNA)
        op, gp = rng.choice([(0, 1), (1, 2), (2, 5), (1, 3)])
        ql = rng.choice([rng.randint(1, 31), rng.randint(32, 300), rng.randint(300, 1100)])
        q = rand_seq(rng, ql, a)
        t = mutate(rng, q, a) if it % 3 == 0 else rand_seq(rng, rng.randint(1, 900), a)
        got = pb.align("parasail_%s_stats_scan" % alg_name, q, t, op, gp, _pb_matrix(key))
        exp = O.align_scan_stats(alg, sgf, q, t, op, gp, _o_matrix(key))
        assert {k: got[k] for k in exp} == exp, (alg_name, op, gp, len(q), len(t), got, exp)
        assert got["flag"] & pb.FLAG_NOVEC_SCAN
        if O.ref() is not None:
            r = O.ref_serial(alg_name, 1, q, t, op, gp, key, scan=True)
            assert {k: r[k] for k in exp} == exp
        differs += exp != O.align(alg, sgf, 1, q, t, op, gp, _o_matrix(key))
        # the plain serial statistics form keeps the serial DP
        assert {k: v for k, v in pb.align("parasail_%s_stats" % alg_name, q, t, op, gp, _pb_matrix(key)).items()
                if k in exp} == O.align(alg, sgf, 1, q, t, op, gp, _o_matrix(key))
    assert differs >= 1


def _vector_cases():
    return json.load(open(os.path.join(GOLDEN, "vector_golden.json")))["cases"]


def test_vector_forms_vs_reference_golden():
    """All 1040 golden cases: 13 algorithms x stats x striped/scan x 8/16/32/sat."""
    bad = []
    for c in _vector_cases():
        st = "_stats" if c["stats"] else ""
        w = c["width"]
        creator = "parasail_profile_create%s_%s" % (st, w)
        name = "parasail_%s%s_%s_profile_%s" % (c["alg"], st, c["scheme"], w)
        m = _pb_matrix(c["matrix"])
        prof = pb.ProfileHandle(creator, c["q"], m)
        got = pb.align_profile(name, prof, c["t"], c["open"], c["gap"])
        prof.close()
        exp = c["expect"]
        if any(got.get(k) != v for k, v in exp.items()):
            bad.append((name, c["q"], c["t"], got, exp))
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:3])


def test_direct_forms_match_profile_forms():
    rng = random.Random(5)
    b62 = pb.matrix_lookup("blosum62")
    for alg_name in ("sw", "nw", "sg_qx", "sg_de"):
        for st in ("", "_stats"):
            for scheme in ("striped", "scan"):
                q = rand_seq(rng, rng.randint(20, 150), AA)
                t = mutate(rng, q, AA, 0.3, 0.05)
                a = pb.align("parasail_%s%s_%s_sat" % (alg_name, st, scheme), q, t, 11, 1, b62)
                prof = pb.ProfileHandle("parasail_profile_create%s_sat" % st, q, b62)
                b = pb.align_profile("parasail_%s%s_%s_profile_sat" % (alg_name, st, scheme), prof, t, 11, 1)
                prof.close()
                assert a == b


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("width", ["8", "16", "32", "sat"])
def test_vector_forms_vs_live_reference(width):
    rng = random.Random(int(width) if width != "sat" else 99)
    b62 = pb.matrix_lookup("blosum62")
    dna = pb.matrix_create("ACGT", 2, -3)
    bad = []
    for it in range(30):
        for alg_name in ("sw", "nw", "sg_qx", "sg_qe_db"):
            for stats in (0, 1):
                for scheme in ("striped", "scan"):
                    if it % 2:
                        key, m, a, op, gp = "blosum62", b62, AA, 11, 1
                    else:
                        key, m, a, op, gp = ("ACGT", 2, -3), dna, DNA, 5, 2
                    q = rand_seq(rng, rng.randint(5, 260), a)
                    t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(5, 260), a)
                    st = "_stats" if stats else ""
                    prof = pb.ProfileHandle("parasail_profile_create%s_%s" % (st, width), q, m)
                    got = pb.align_profile("parasail_%s%s_%s_profile_%s" % (alg_name, st, scheme, width),
                                           prof, t, op, gp)
                    prof.close()
                    exp = O.ref_vector(alg_name, stats, scheme, width, q, t, op, gp, key)
                    if any(got.get(k) != v for k, v in exp.items()):
                        bad.append((alg_name, stats, scheme, width, q, t, got, exp))
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


def _penalties(rng, width, protein):
    """open == gap, open < gap, and penalties that wrap in a narrow lane"""
    c = [(1, 1), (2, 2), (3, 3), (0, 1), (1, 2)]
    if width in ("8", "sat"):
        c.append((200, 1) if protein else (130, 2))
    if width in ("16", "sat"):
        c.append((40000, 1) if protein else (1, 33000))
    return rng.choice(c)


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("width", ["8", "16", "32", "sat"])
def test_striped_linear_and_wrapped_penalties_vs_live_reference(width):
    """Striped kernels where the reference departs from the exact DP (its
    lazy-F loop stops on ties when open <= gap, and set1 of a penalty above
    the lane maximum wraps): the direct and profile forms, and batches of
    both kinds, against the reference's AVX2 kernels. Scan kernels are
    checked at open == gap, where they follow the exact DP."""
    rng = random.Random({"8": 18, "16": 116, "32": 132, "sat": 77}[width])
    bad, total = [], 0
    for alg_name, stats in (("sw", 0), ("nw", 0), ("sg", 0), ("sg_qx", 0), ("sg_de", 0), ("sg_qb_db", 0),
                            ("nw", 1), ("sg_qe_db", 1)):
        st = "_stats" if stats else ""
        for it in range(6):
            protein = it % 2 == 1
            key, a = ("blosum62", AA) if protein else (("ACGT", 2, -3), DNA)
            m = _pb_matrix(key)
            op, gp = _penalties(rng, width, protein)
            q = rand_seq(rng, rng.randint(1, 200), a)
            targets = [mutate(rng, q, a, 0.2, 0.04) if k % 3 == 0 else rand_seq(rng, rng.randint(1, 220), a)
                       for k in range(12)]
            exp = [O.ref_vector(alg_name, stats, "striped", width, q, t, op, gp, key) for t in targets]
            got = {}
            got["direct"] = [pb.align("parasail_%s%s_striped_%s" % (alg_name, st, width), q, t, op, gp, m)
                             for t in targets]
            prof = pb.ProfileHandle("parasail_profile_create%s_%s" % (st, width), q, m)
            got["profile"] = [pb.align_profile("parasail_%s%s_striped_profile_%s" % (alg_name, st, width),
                                               prof, t, op, gp) for t in targets]
            got["batch"] = pb.records_to_dicts(
                pb.batch_profile("%s%s_striped_profile_%s" % (alg_name, st, width), prof, targets, op, gp), stats)
            prof.close()
            got["pairs"] = pb.records_to_dicts(
                pb.batch_pairs("%s%s_striped_%s" % (alg_name, st, width), m, [q] * len(targets), targets, op, gp),
                stats)
            for form, rs in got.items():
                for t, r, e in zip(targets, rs, exp):
                    total += 1
                    if any(r.get(k) != v for k, v in e.items()):
                        bad.append((form, alg_name, stats, width, op, gp, q, t, r, e))
            if op == gp and op < 128:
                for t in targets[:4]:
                    total += 1
                    r = pb.align("parasail_%s%s_scan_%s" % (alg_name, st, width), q, t, op, gp, m)
                    e = O.ref_vector(alg_name, stats, "scan", width, q, t, op, gp, key)
                    if any(r.get(k) != v for k, v in e.items()):
                        bad.append(("scan", alg_name, stats, width, op, gp, q, t, r, e))
    assert total >= 8 * 6 * 12 * 4
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


def test_nw_banded_vs_oracle():
    rng = random.Random(11)
    dna = pb.matrix_create("ACGT", 2, -3)
    om = O.Matrix.simple("ACGT", 2, -3)
    for _ in range(40):
        q = rand_seq(rng, rng.randint(1, 120), DNA)
        t = mutate(rng, q, DNA) if rng.random() < 0.6 else rand_seq(rng, rng.randint(1, 120), DNA)
        k = rng.randint(1, 30)
        got = pb.nw_banded(q, t, 5, 2, k, dna)
        exp = O.nw_banded(q, t, 5, 2, k, om)
        assert (got["score"], got["end_query"], got["end_ref"]) == (exp["score"], exp["end_query"], exp["end_ref"])
        assert got["flag"] & pb.FLAG_BANDED


def test_nw_banded_batch_and_wide_matrices_vs_oracle():
    """parasail_nw_banded on the wavefront kernel (band as diagonals) in a
    batch and per call, against the oracle's restatement of
    src/nw_banded.c, for both length orders, bands narrower and wider than
    the length difference, a protein matrix, and (per call) a matrix whose
    scores exceed int8, which runs the column recurrence instead."""
    rng = random.Random(23)
    for alpha, key, m_args, op, gp in ((DNA, "dna", ("ACGT", 2, -3), 5, 2), (AA, "b62", None, 11, 1)):
        m = pb.matrix_create(*m_args) if m_args else pb.matrix_lookup("blosum62")
        om = O.Matrix.simple(*m_args) if m_args else O.Matrix.from_struct(m)
        qs, ts = [], []
        for _ in range(60):
            q = rand_seq(rng, rng.randint(1, 700), alpha)
            t = mutate(rng, q, alpha, 0.1, 0.05) if rng.random() < 0.6 else rand_seq(rng, rng.randint(1, 700), alpha)
            qs.append(q)
            ts.append(t)
        for k in (1, 7, 40, 300):
            got = pb.nw_banded_batch(m, qs, ts, op, gp, k)
            for q, t, g in zip(qs, ts, got):
                assert g == O.nw_banded(q, t, op, gp, k, om)["score"], (key, k, len(q), len(t))
        for q, t in list(zip(qs, ts))[:10]:
            one = pb.nw_banded(q, t, op, gp, 9, m)
            assert one["score"] == O.nw_banded(q, t, op, gp, 9, om)["score"]
    wide = pb.matrix_create("ACGT", 200, -300)
    owide = O.Matrix.simple("ACGT", 200, -300)
    for _ in range(10):
        q = rand_seq(rng, rng.randint(1, 150), DNA)
        t = mutate(rng, q, DNA)
        got = pb.nw_banded(q, t, 400, 100, 12, wide)
        assert got["score"] == O.nw_banded(q, t, 400, 100, 12, owide)["score"]


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("width", ["8", "16", "sat"])
def test_batch_striped_narrow_vs_live_reference(width):
    """Batches through the device pipeline, including its lane-exact rounds
    for the 8/16-bit striped kernels, against the reference's AVX2 kernels on
    every pair: score, ends, statistics and flags."""
    rng = random.Random({"8": 81, "16": 161, "sat": 7}[width])
    b62 = pb.matrix_lookup("blosum62")
    dna = pb.matrix_create("ACGT", 2, -3)
    bad, total = [], 0
    for alg_name in ("nw", "sg_qx", "sg_qe_db", "sg_de", "sw"):
        for stats in (0, 1):
            if alg_name == "sw" and not stats:
                continue
            for key, m, a, op, gp in (("blosum62", b62, AA, 11, 1), (("ACGT", 2, -3), dna, DNA, 5, 2)):
                q = rand_seq(rng, rng.randint(10, 220), a)
                targets = [mutate(rng, q, a, 0.25, 0.04) if k % 3 == 0 else rand_seq(rng, rng.randint(5, 260), a)
                           for k in range(60)]
                st = "_stats" if stats else ""
                prof = pb.ProfileHandle("parasail_profile_create%s_%s" % (st, width), q, m)
                name = "%s%s_striped_profile_%s" % (alg_name, st, width)
                recs = pb.records_to_dicts(pb.batch_profile(name, prof, targets, op, gp), stats)
                prof.close()
                for t, r in zip(targets, recs):
                    exp = O.ref_vector(alg_name, stats, "striped", width, q, t, op, gp, key)
                    total += 1
                    if any(r.get(k) != v for k, v in exp.items()):
                        bad.append((name, key, q, t, r, exp))
    assert total >= 500
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("width", ["8", "16", "32", "sat"])
def test_scan_open_below_gap_and_wrapped_vs_live_reference(width):
    """Score-only scan kernels where the reference departs from the exact DP
    (open < gap: their prefix scan of F takes F - gap >= F - open; a penalty
    above the lane maximum wraps in set1): the direct and profile forms and
    batches of both kinds, run on the lane-exact scan kernels, against the
    reference's AVX2 kernels."""
    rng = random.Random({"8": 28, "16": 216, "32": 232, "sat": 87}[width])
    bad, total = [], 0
    for alg_name in ("sw", "nw", "sg", "sg_qx", "sg_de", "sg_qb_db", "sg_qe_db"):
        for it in range(5):
            protein = it % 2 == 1
            key, a = ("blosum62", AA) if protein else (("ACGT", 2, -3), DNA)
            m = _pb_matrix(key)
            c = [(0, 1), (1, 2), (2, 5), (1, 3)]
            if width in ("8", "sat"):
                c.append((200, 1) if protein else (130, 2))
            op, gp = rng.choice(c)
            q = rand_seq(rng, rng.randint(1, 200), a)
            targets = [mutate(rng, q, a, 0.2, 0.04) if k % 3 == 0 else rand_seq(rng, rng.randint(1, 220), a)
                       for k in range(10)]
            exp = [O.ref_vector(alg_name, 0, "scan", width, q, t, op, gp, key) for t in targets]
            got = {}
            got["direct"] = [pb.align("parasail_%s_scan_%s" % (alg_name, width), q, t, op, gp, m)
                             for t in targets]
            prof = pb.ProfileHandle("parasail_profile_create_%s" % width, q, m)
            got["profile"] = [pb.align_profile("parasail_%s_scan_profile_%s" % (alg_name, width), prof, t, op, gp)
                              for t in targets]
            got["batch"] = pb.records_to_dicts(
                pb.batch_profile("%s_scan_profile_%s" % (alg_name, width), prof, targets, op, gp), 0)
            prof.close()
            got["pairs"] = pb.records_to_dicts(
                pb.batch_pairs("%s_scan_%s" % (alg_name, width), m, [q] * len(targets), targets, op, gp), 0)
            for form, rs in got.items():
                for t, r, e in zip(targets, rs, exp):
                    total += 1
                    if any(r.get(k) != v for k, v in e.items()):
                        bad.append((form, alg_name, width, op, gp, q, t, r, e))
    assert total == 7 * 5 * 10 * 4
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
@pytest.mark.parametrize("width", ["8", "16", "32", "sat"])
def test_stats_scan_open_below_gap_and_wrapped_vs_live_reference(width):
    """NW and SG statistics scan kernels where the reference departs from
    the exact DP (open < gap; a penalty above the lane maximum): the direct
    and profile forms and batches of both kinds, run on the lane-exact
    statistics scan kernel, against the reference's AVX2 kernels (score,
    ends, matches, similar, length, flags)."""
    rng = random.Random({"8": 38, "16": 316, "32": 332, "sat": 97}[width])
    bad, total, differs = [], 0, 0
    for alg_name in ("nw", "sg", "sg_qx", "sg_de", "sg_qb_db", "sg_qe_db"):
        for it in range(5):
            protein = it % 2 == 1
            key, a = ("blosum62", AA) if protein else (("ACGT", 2, -3), DNA)
            m = _pb_matrix(key)
            c = [(0, 1), (1, 2), (2, 5), (1, 3)]
            if width in ("8", "sat"):
                c.append((200, 1) if protein else (130, 2))
            op, gp = rng.choice(c)
            q = rand_seq(rng, rng.randint(1, 200), a)
            targets = [mutate(rng, q, a, 0.2, 0.04) if k % 3 == 0 else rand_seq(rng, rng.randint(1, 220), a)
                       for k in range(10)]
            exp = [O.ref_vector(alg_name, 1, "scan", width, q, t, op, gp, key) for t in targets]
            got = {}
            got["direct"] = [pb.align("parasail_%s_stats_scan_%s" % (alg_name, width), q, t, op, gp, m)
                             for t in targets]
            prof = pb.ProfileHandle("parasail_profile_create_stats_%s" % width, q, m)
            got["profile"] = [pb.align_profile("parasail_%s_stats_scan_profile_%s" % (alg_name, width), prof, t,
                                               op, gp) for t in targets]
            got["batch"] = pb.records_to_dicts(
                pb.batch_profile("%s_stats_scan_profile_%s" % (alg_name, width), prof, targets, op, gp), 1)
            prof.close()
            got["pairs"] = pb.records_to_dicts(
                pb.batch_pairs("%s_stats_scan_%s" % (alg_name, width), m, [q] * len(targets), targets, op, gp), 1)
            for t, e in zip(targets, exp):
                if not e["flag"] & pb.FLAG_SATURATED and op < gp:
                    ex = O.align(O.alg_of(alg_name)[0], O.alg_of(alg_name)[1], 1, q, t, op, gp, _o_matrix(key))
                    differs += any(ex[k] != e[k] for k in ex if k in e)
            for form, rs in got.items():
                for t, r, e in zip(targets, rs, exp):
                    total += 1
                    if any(r.get(k) != v for k, v in e.items()):
                        bad.append((form, alg_name, width, op, gp, q, t, r, e))
    assert total == 6 * 5 * 10 * 4
    assert differs >= 1
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])
