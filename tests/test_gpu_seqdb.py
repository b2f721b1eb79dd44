"""Device-resident packed sequence sets: the packed width, the unpacked
codes (the matrix mapper applied to every residue), and budgeted pair
batches over a set against the host batch API and the oracle."""
import random

import numpy as np
import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
pytestmark = pytest.mark.gpu


def _text(seqs):
    return "".join(s + "$" for s in seqs).encode()


def _expected_codes(text, matrix):
    mp = np.ctypeslib.as_array(matrix.contents.mapper, shape=(256,))
    t = np.frombuffer(text, np.uint8)
    return np.where(t == ord("$"), 0, mp[t]).astype(np.uint8)


def test_packed_widths_and_round_trip():
    rng = random.Random(4)
    dna = pb.matrix_create("ACGT", 2, -3)
    b62 = pb.matrix_lookup("blosum62")
    wide = pb.matrix_create("".join(chr(c) for c in range(ord("A"), ord("A") + 40)), 1, -1)
    cases = [
        ([rand_seq(rng, rng.randint(0, 300), DNA) for _ in range(200)], dna, 2),
        ([rand_seq(rng, rng.randint(1, 300), DNA + "N") for _ in range(50)], dna, 5),
        ([rand_seq(rng, rng.randint(1, 500), AA) for _ in range(300)], b62, 5),
        (["".join(chr(ord("A") + rng.randint(0, 39)) for _ in range(rng.randint(1, 90))) for _ in range(40)],
         wide, 8),
        (["ACGT"], dna, 2),
        (["", "A", ""], dna, 2),
    ]
    for seqs, m, bits in cases:
        text = _text(seqs)
        db = pb.SeqDB(text, m)
        assert db.count == len(seqs) and db.size == len(text) and db.bits == bits
        per = {2: 16, 5: 6, 8: 4}[bits]
        assert db.device_bytes == ((len(text) + per - 1) // per + 3) // 4 * 4 * 4
        off, ln = db.offsets_lengths()
        exp_off = np.cumsum([0] + [len(s) + 1 for s in seqs[:-1]]).tolist()
        assert off == exp_off and ln == [len(s) for s in seqs]
        assert (db.unpack() == _expected_codes(text, m)).all()
        db.close()


def test_batch_pairs_seqdb_matches_host_batch_and_oracle():
    rng = random.Random(8)
    b62 = pb.matrix_lookup("blosum62")
    seqs = []
    for _ in range(300):
        if seqs and rng.random() < 0.3:
            seqs.append(mutate(rng, rng.choice(seqs), AA, 0.2, 0.03))
        else:
            seqs.append(rand_seq(rng, rng.randint(20, 400), AA))
    db = pb.SeqDB(_text(seqs), b62)
    first = [rng.randrange(len(seqs)) for _ in range(3000)]
    second = [rng.randrange(len(seqs)) for _ in range(3000)]
    for name in ("sw_stats_striped_profile_16", "sw_striped_sat", "nw_scan_32", "sg_qx_stats_scan_16"):
        direct = name.replace("_profile", "")
        exp = pb.batch_pairs(direct, b62, [seqs[i] for i in first], [seqs[j] for j in second], 11, 1)
        for budget in (0, 64 << 20, 600 * 1024):   # one batch, and many
            got = db.align_pairs(name, first, second, 11, 1, budget=budget)
            assert (got == exp).all(), (name, budget)
    # a sample against the oracle's serial DP
    om = O.Matrix.from_struct(b62)
    for k in range(0, 3000, 97):
        r = O.align(O.SW, 0, True, seqs[first[k]], seqs[second[k]], 11, 1, om)
        got = db.align_pairs("sw_stats_striped_16", [first[k]], [second[k]], 11, 1)[0]
        assert (got["score"], got["end_query"], got["end_ref"], got["matches"], got["similar"],
                got["length"]) == (r["score"], r["end_query"], r["end_ref"], r["matches"], r["similar"],
                                   r["length"])
    with pytest.raises(RuntimeError):
        db.align_pairs("sw_striped_16", [0], [len(seqs)], 11, 1)
    db.close()
