"""The aligner driver (parasail_b200/parasail_b200_aligner) against the
reference aligner (apps/parasail_aligner.cpp, built from its sources into
oracle/_ref/parasail_aligner_ref): the same command line on the same files
must write the same output file, byte for byte -- candidate pairs from the
exact-match filter or all pairs, query files, CSV with and without
statistics, edges, graphs, and the EMBOSS / SSW / SAM text of trace
functions."""
import os
import random
import subprocess

import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "parasail_b200", "parasail_b200_aligner")
REF = os.path.join(ROOT, "oracle", "_ref", "parasail_aligner_ref")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REF), reason="reference aligner not built")]


def _run(exe, args, cwd):
    """Runs an aligner with a standard input that stays silent (both
    aligners treat readable standard input as an input file)."""
    r, w = os.pipe()
    try:
        p = subprocess.run([exe] + args, stdin=r, cwd=cwd, capture_output=True, text=True, timeout=600)
    finally:
        os.close(r)
        os.close(w)
    return p


def _fasta(path, seqs, names=None, fastq=False, rng=None):
    with open(path, "w") as f:
        for k, s in enumerate(seqs):
            name = names[k] if names else "seq%d" % k
            if fastq:
                f.write("@%s read %d\n%s\n+\n%s\n" % (name, k, s, "".join(chr(33 + (rng.randint(0, 40))) for _ in s)))
            else:
                f.write(">%s desc %d\n" % (name, k))
                for i in range(0, len(s), 60):
                    f.write(s[i:i + 60] + "\n")


def _families(rng, n, alpha, lo, hi, fam=0.4, sub=0.15, indel=0.03):
    seqs = []
    for _ in range(n):
        if seqs and rng.random() < fam:
            seqs.append(mutate(rng, rng.choice(seqs), alpha, sub, indel))
        else:
            seqs.append(rand_seq(rng, rng.randint(lo, hi), alpha))
    return [s for s in seqs if s]


def _compare(tmp_path, args, out="out.txt", files=()):
    a = _run(OURS, args + ["-g", "ours_" + out], str(tmp_path))
    b = _run(REF, args + ["-g", "ref_" + out], str(tmp_path))
    assert b.returncode == 0, b.stderr
    assert a.returncode == 0, a.stderr
    ours = open(os.path.join(str(tmp_path), "ours_" + out), "rb").read()
    ref = open(os.path.join(str(tmp_path), "ref_" + out), "rb").read()
    assert ours == ref, (args, ours[:400], ref[:400])
    return ours


def test_aligner_csv_outputs_match_reference(tmp_path):
    rng = random.Random(21)
    db = _families(rng, 120, AA, 40, 400)
    _fasta(str(tmp_path / "prot.fa"), db)
    # queries: relatives of some database sequences and unrelated ones
    _fasta(str(tmp_path / "q.fa"), [mutate(rng, rng.choice(db), AA, 0.25, 0.03) for _ in range(10)] +
           _families(rng, 5, AA, 40, 300))
    for args in (["-f", "prot.fa"],                                          # sw_stats_striped_16, filter
                 ["-f", "prot.fa", "-x", "-a", "sw_striped_profile_sat"],    # all pairs, score only
                 ["-f", "prot.fa", "-c", "5", "-a", "nw_stats_scan_16"],
                 ["-f", "prot.fa", "-q", "q.fa", "-a", "sg_qx_stats_striped_16", "-o", "11", "-e", "1"],
                 ["-f", "prot.fa", "-q", "q.fa", "-x", "-a", "sw_scan_8"],
                 ["-f", "prot.fa", "-a", "sw_stats_scan_profile_32", "-b", "7"],
                 ["-f", "prot.fa", "-E", "-l", "50", "-s", "30", "-i", "20"],
                 ["-f", "prot.fa", "-G", "-l", "40"],
                 ["-f", "prot.fa", "-p", "-c", "4"],
                 ["-f", "prot.fa", "-q", "q.fa", "-p"]):
        out = _compare(tmp_path, args)
        assert out, args


def test_aligner_dna_mixed_case_and_case_sensitive(tmp_path):
    rng = random.Random(5)
    seqs = _families(rng, 80, DNA, 60, 300, sub=0.05, indel=0.01)
    seqs = ["".join(c.lower() if rng.random() < 0.1 else c for c in s) for s in seqs]
    _fasta(str(tmp_path / "dna.fa"), seqs)
    for args in (["-f", "dna.fa", "-d", "-M", "2", "-X", "3", "-o", "5", "-e", "2", "-c", "12",
                  "-a", "nw_stats_striped_16"],
                 ["-f", "dna.fa", "-d", "-C", "-c", "12", "-a", "sw_stats_striped_16"],
                 ["-f", "dna.fa", "-d", "-x", "-a", "sg_stats_scan_16"]):
        _compare(tmp_path, args)


def test_aligner_trace_outputs_match_reference(tmp_path):
    rng = random.Random(9)
    db = _families(rng, 40, AA, 40, 250)
    _fasta(str(tmp_path / "db.fa"), db)
    reads = [mutate(rng, s[rng.randint(0, 10):], AA, 0.1, 0.02) for s in db[:12]]
    _fasta(str(tmp_path / "reads.fq"), reads, fastq=True, rng=rng)
    for args in (["-f", "db.fa", "-a", "sw_trace_striped_32", "-O", "EMBOSS"],
                 ["-f", "db.fa", "-a", "nw_trace_scan_32", "-O", "SSW", "-c", "9"],
                 ["-f", "db.fa", "-a", "sg_qx_trace", "-O", "EMBOSS", "-A", "ST*#"],
                 ["-f", "db.fa", "-q", "reads.fq", "-a", "sw_trace_scan_profile_32", "-O", "SAM"],
                 ["-f", "db.fa", "-q", "reads.fq", "-a", "sw_trace_striped_32", "-O", "SAMH"]):
        _compare(tmp_path, args)


def test_aligner_argument_errors_match_reference(tmp_path):
    _fasta(str(tmp_path / "a.fa"), ["ACDEFGHIK", "ACDEFGHIKL"])
    for args in (["-f", "a.fa", "-a", "no_such_function"],
                 ["-f", "a.fa", "-a", "sw_trace_striped_32"],
                 ["-f", "a.fa", "-E", "-a", "sw_striped_16"],
                 ["-f", "a.fa", "-O", "XML", "-a", "sw_trace"],
                 ["-f", "a.fa", "-c", "0"]):
        a = _run(OURS, args, str(tmp_path))
        b = _run(REF, args, str(tmp_path))
        assert a.returncode == b.returncode != 0, args
        assert a.stderr.splitlines()[0] == b.stderr.splitlines()[0], (args, a.stderr, b.stderr)
