"""Candidate pairs of the aligner's exact-match filter: the GPU filter
(parasail_b200_candidate_pairs) against the reference aligner's
enhanced-suffix-array traversal (the reference's sais + oracle/esa_pairs.cpp)
and against the direct statement (pairs sharing a cutoff-window)."""
import random

import numpy as np
import pytest

import oracle as O

pb = pytest.importorskip("parasail_b200")


def _case(rng, n, alpha, fam=0.3, maxlen=60):
    seqs = []
    for _ in range(n):
        if seqs and rng.random() < fam:
            s = rng.choice(seqs)
            a = rng.randint(0, len(s))
            s = s[a:a + rng.randint(0, 40)] + "".join(rng.choice(alpha) for _ in range(rng.randint(0, 10)))
        else:
            s = "".join(rng.choice(alpha) for _ in range(rng.randint(0, maxlen)))
        seqs.append(s)
    return seqs


def _text(seqs):
    return "".join(s + "$" for s in seqs).encode()


def test_esa_oracle_equals_direct_statement():
    """The restated traversal keeps exactly the pairs sharing a window."""
    if O.esa_pairs(b"A$", 1) is None:
        pytest.skip("reference sais not built")
    rng = random.Random(1)
    for _ in range(150):
        alpha = rng.choice(["ACGT", "ACDEFGHIKLMNPQRSTVWY", "AB"])
        n = rng.randint(2, 30)
        seqs = _case(rng, n, alpha)
        c = rng.randint(1, 12)
        ndb = rng.randint(1, n - 1) if rng.random() < 0.4 else None
        dbc = len(_text(seqs[:ndb])) if ndb else -1
        assert O.esa_pairs(_text(seqs), c, dbc) == O.kmer_pairs(seqs, c, ndb)


def _expect(seqs, c, ndb):
    e = O.esa_pairs(_text(seqs), c, len(_text(seqs[:ndb])) if ndb else -1)
    return e if e is not None else O.kmer_pairs(seqs, c, ndb)


@pytest.mark.gpu
def test_candidate_pairs_vs_reference_filter():
    rng = random.Random(11)
    bad = 0
    for trial in range(120):
        alpha = rng.choice(["ACGT", "ACDEFGHIKLMNPQRSTVWY", "AB", "ACGTacgt"])
        n = rng.randint(2, 80)
        seqs = _case(rng, n, alpha, maxlen=rng.choice([20, 60, 200]))
        c = rng.choice([1, 2, 3, 5, 7, 8, 9, 12, 16, 17, 24, 33])
        ndb = rng.randint(1, n - 1) if rng.random() < 0.4 else None
        got = pb.candidate_pairs(_text(seqs), c, len(_text(seqs[:ndb])) if ndb else -1)
        exp = _expect(seqs, c, ndb)
        bad += got != exp
        assert got == exp, (trial, c, ndb, len(got), len(exp))
    assert bad == 0


@pytest.mark.gpu
def test_candidate_pairs_protein_families_and_dna_reads():
    """Larger sets: 600 proteins with planted families at the aligner's
    default cutoff 7, and DNA reads from one genome at cutoff 20 with a
    query split."""
    S = pytest.importorskip("parasail_b200.synth")
    buf, offs, lens = S.protein_all_vs_all(seed=9, n_seqs=600)
    seqs = [bytes(buf[o:o + l]).decode() for o, l in zip(offs, lens)]
    for c in (7, 11):
        assert pb.candidate_pairs(_text(seqs), c) == _expect(seqs, c, None)
    rng = np.random.default_rng(5)
    genome = "".join(rng.choice(list("ACGT"), 20000))
    reads = []
    for _ in range(400):
        a = int(rng.integers(0, 19700))
        reads.append(genome[a:a + int(rng.integers(100, 300))])
    ndb = 250
    assert pb.candidate_pairs(_text(reads), 20, len(_text(reads[:ndb]))) == _expect(reads, 20, ndb)


@pytest.mark.gpu
def test_candidate_pairs_edges():
    assert pb.candidate_pairs(b"", 5) == []
    assert pb.candidate_pairs(b"ACGT$ACGT$", 5) == []          # shorter than the cutoff
    assert pb.candidate_pairs(b"ACGT$ACGT$", 4) == [(0, 1)]
    assert pb.candidate_pairs(b"AAAA$AAAA$AAAA$", 2, 5) == [(1, 0), (2, 0)]
    with pytest.raises(RuntimeError):
        pb.candidate_pairs(b"ACGT$ACGT", 2)                    # no final sentinel
    with pytest.raises(RuntimeError):
        pb.candidate_pairs(b"ACGT$", 0)
