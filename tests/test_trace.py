"""Traceback and CIGAR: the trace entry points of parasail.h (serial forms
and striped/scan forms at 8, 16, 32 bits and _sat, direct and profile) and
the batch CIGAR call,
against the reference's own trace functions and parasail_result_get_cigar
(src/cigar.c) compiled into oracle/_ref; and the CIGAR string helpers on
CPU."""
import random

import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")

ALGS = ["sw", "nw", "sg", "sg_qb", "sg_qe", "sg_qx", "sg_db", "sg_de", "sg_dx", "sg_qb_de", "sg_qe_db",
        "sg_qb_db", "sg_qe_de"]
FORMS = ["", "_scan", "_striped_32", "_scan_32"]
NARROW = ["_striped_8", "_striped_16", "_striped_sat", "_scan_8", "_scan_16", "_scan_sat"]


def test_cigar_string_round_trip():
    for s in ("3=2I2=1X4D14=", "1=", "120M", "7S3=1X"):
        c = pb.lib.parasail_cigar_encode_string(s.encode())
        assert c
        assert pb.cigar_string(c)[0] == s
    x = pb.lib.parasail_cigar_encode(17, b"X")
    assert x == (17 << 4) | 8
    assert pb.lib.parasail_cigar_decode_op(x) == b"X" and pb.lib.parasail_cigar_decode_len(x) == 17


def _pairs(rng, n, alpha):
    out = []
    for _ in range(n):
        q = rand_seq(rng, rng.randint(2, 160), alpha)
        r = rng.random()
        t = mutate(rng, q, alpha, 0.15, 0.06) if r < 0.6 else \
            (rand_seq(rng, 20, alpha) + q[5:] + rand_seq(rng, 7, alpha) if r < 0.8 else
             rand_seq(rng, rng.randint(2, 160), alpha))
        out.append((q, t))
    return out


@pytest.mark.gpu
@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
def test_trace_cigar_vs_reference():
    """Every algorithm and trace form on protein and DNA pairs (open > gap
    and open == gap): score, ends, flags, CIGAR and begin positions equal
    the reference's."""
    rng = random.Random(123)
    b62 = pb.matrix_lookup("blosum62")
    dna = pb.matrix_create("ACGT", 2, -3)
    bad, total = [], 0
    for key, m, alpha, pens in (("blosum62", b62, AA, ((11, 1), (3, 3))), (("ACGT", 2, -3), dna, DNA, ((5, 2),))):
        for q, t in _pairs(rng, 12, alpha):
            for op, gp in pens:
                for alg in ALGS:
                    for form in FORMS:
                        exp = O.ref_trace(alg, form, q, t, op, gp, key)
                        if alg == "sw" and exp["score"] < 0:
                            continue     # a reference quirk, see the test below
                        got = pb.trace("parasail_%s_trace%s" % (alg, form), q, t, op, gp, m)
                        total += 1
                        if got != exp:
                            bad.append((alg, form, op, gp, q, t, got, exp))
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])
    assert total > 1500


@pytest.mark.gpu
def test_trace_profile_forms_and_batch_equal_direct():
    rng = random.Random(7)
    b62 = pb.matrix_lookup("blosum62")
    pairs = _pairs(rng, 40, AA)
    for alg in ("sw", "nw", "sg_qx", "sg_de"):
        for form in ("_striped", "_scan"):
            for q, t in pairs[:8]:
                prof = pb.ProfileHandle("parasail_profile_create_32", q, b62)
                a = pb.trace("parasail_%s_trace%s_profile_32" % (alg, form), q, t, 11, 1, b62, profile=prof)
                b = pb.trace("parasail_%s_trace%s_32" % (alg, form), q, t, 11, 1, b62)
                prof.close()
                assert a == b, (alg, form)
        qs, ts = [p[0] for p in pairs], [p[1] for p in pairs]
        for form in ("", "_scan_32"):
            got = pb.batch_pairs_cigar("%s_trace%s" % (alg, form), b62, qs, ts, 11, 1)
            for q, t, g in zip(qs, ts, got):
                assert g == pb.trace("parasail_%s_trace%s" % (alg, form), q, t, 11, 1, b62), (alg, form)


@pytest.mark.gpu
@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
def test_traceback_strings_and_printout_vs_reference():
    """parasail_result_get_traceback_extra and parasail_traceback_generic_extra2
    (the aligner's EMBOSS and SSW layouts) produce the reference's text for
    every algorithm family, with and without alias pairs and case
    sensitivity, on mixed-case inputs."""
    rng = random.Random(99)
    b62 = pb.matrix_lookup("blosum62")
    dna = pb.matrix_create("ACGT", 2, -3)
    bad, total = [], 0
    # the reference reads one byte past the alias table when the residue
    # equals its last character: every table here ends in characters that
    # no sequence holds
    variants = ({}, {"aliases": "AGcT*#"}, {"case_sensitive": 1, "aliases": "ST*#"})
    for key, m, alpha in (("blosum62", b62, AA), (("ACGT", 2, -3), dna, DNA)):
        for q, t in _pairs(rng, 8, alpha):
            q = "".join(c.lower() if rng.random() < 0.2 else c for c in q)
            for alg in ("sw", "nw", "sg", "sg_qx", "sg_de", "sg_qb_db"):
                for form in ("", "_striped_32"):
                    for kw in variants:
                        exp = O.ref_trace(alg, form, q, t, 11, 1, key, strings=kw)
                        if alg == "sw" and exp["score"] < 0:
                            continue
                        got = pb.trace("parasail_%s_trace%s" % (alg, form), q, t, 11, 1, m, strings=kw)
                        total += 1
                        if got != exp:
                            bad.append((alg, form, kw, q, t, got, exp))
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:1])
    assert total > 400


@pytest.mark.gpu
@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
def test_trace_narrow_widths_vs_reference():
    """8/16-bit and _sat trace forms on pairs around the 8-bit limits: the
    saturation flag, score, ends, width flags and CIGAR equal the
    reference's AVX2 trace kernels and its _sat dispatcher (src/satcheck.c),
    at open > gap, open == gap and (nw/sg) penalties that wrap in 8 bits."""
    rng = random.Random(321)
    b62 = pb.matrix_lookup("blosum62")
    dna = pb.matrix_create("ACGT", 2, -3)
    bad, total, nsat = [], 0, 0
    for key, m, alpha, pens in (("blosum62", b62, AA, ((11, 1), (3, 3), (5, 2))),
                                (("ACGT", 2, -3), dna, DNA, ((5, 2), (2, 2), (130, 1)))):
        for _ in range(8):
            q = rand_seq(rng, rng.randint(1, 90), alpha)
            t = mutate(rng, q, alpha, 0.1, 0.03) if rng.random() < 0.6 else rand_seq(rng, rng.randint(1, 90), alpha)
            for op, gp in pens:
                for alg in ALGS:
                    if alg == "sw" and op > 127:
                        continue     # wrapped SW penalties are taken as saturating
                    for form in NARROW:
                        exp = O.ref_trace(alg, form, q, t, op, gp, key)
                        if alg == "sw" and exp["score"] < 0:
                            continue
                        got = pb.trace("parasail_%s_trace%s" % (alg, form), q, t, op, gp, m)
                        total += 1
                        nsat += bool(exp["flag"] & 64)
                        if got != exp:
                            bad.append((alg, form, op, gp, q, t, got, exp))
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])
    assert total > 3000 and 300 < nsat < total - 300


@pytest.mark.gpu
@pytest.mark.skipif(O.ref() is None, reason="reference library not built")
def test_trace_narrow_profile_and_batch_forms():
    """The profile forms (parasail_profile_create_8/16/sat) and the batch
    CIGAR and trace calls with 8/16/_sat names give the direct forms'
    results, saturated pairs included (no CIGAR, flag set)."""
    rng = random.Random(17)
    b62 = pb.matrix_lookup("blosum62")
    pairs = _pairs(rng, 24, AA)
    qs, ts = [p[0] for p in pairs], [p[1] for p in pairs]
    for alg in ("sw", "nw", "sg_qx", "sg_de"):
        for form in ("_striped", "_scan"):
            for w in ("8", "16", "sat"):
                for q, t in pairs[:4]:
                    prof = pb.ProfileHandle("parasail_profile_create_%s" % w, q, b62)
                    a = pb.trace("parasail_%s_trace%s_profile_%s" % (alg, form, w), q, t, 11, 1, b62, profile=prof)
                    prof.close()
                    b = pb.trace("parasail_%s_trace%s_%s" % (alg, form, w), q, t, 11, 1, b62)
                    assert a == b, (alg, form, w)
        for name in ("%s_trace_striped_8" % alg, "%s_trace_scan_sat" % alg):
            got = pb.batch_pairs_cigar(name, b62, qs, ts, 11, 1)
            nsat = 0
            for q, t, g in zip(qs, ts, got):
                one = pb.trace("parasail_" + name, q, t, 11, 1, b62)
                assert g == one, (name, q, t)
                assert g == O.ref_trace(alg, name.split("_trace")[1], q, t, 11, 1, "blosum62"), (name, q, t)
                nsat += bool(g["flag"] & 64)
            if name.endswith("_8") and alg != "sw":
                assert nsat > 0
