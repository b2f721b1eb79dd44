"""Sequence files, packed text and matrix files (parasail/io.h) against the
reference's own src/io.c and src/parser.c compiled into the oracle library:
every record field, the file statistics and the packed text must be the
same bytes. CPU only."""
import ctypes
import math
import os

import numpy as np
import pytest

import oracle as O

pb = pytest.importorskip("parasail_b200")


class PString(ctypes.Structure):
    _fields_ = [("l", ctypes.c_size_t), ("s", ctypes.c_void_p)]


class PSequence(ctypes.Structure):
    _fields_ = [("name", PString), ("comment", PString), ("seq", PString), ("qual", PString)]


class PSequences(ctypes.Structure):
    _fields_ = [("seqs", ctypes.POINTER(PSequence)), ("l", ctypes.c_size_t), ("characters", ctypes.c_size_t),
                ("shortest", ctypes.c_size_t), ("longest", ctypes.c_size_t), ("mean", ctypes.c_float),
                ("stddev", ctypes.c_float)]


class PFileStat(ctypes.Structure):
    _fields_ = [("sequences", ctypes.c_ulong), ("characters", ctypes.c_ulong), ("shortest", ctypes.c_ulong),
                ("longest", ctypes.c_ulong), ("mean", ctypes.c_float), ("stddev", ctypes.c_float)]


class PMatrix(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("matrix", ctypes.POINTER(ctypes.c_int)),
                ("mapper", ctypes.POINTER(ctypes.c_int)), ("size", ctypes.c_int), ("max", ctypes.c_int),
                ("min", ctypes.c_int), ("user_matrix", ctypes.POINTER(ctypes.c_int)), ("type", ctypes.c_int),
                ("length", ctypes.c_int), ("alphabet", ctypes.c_char_p), ("query", ctypes.c_char_p)]


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def _bind(lib):
    lib.parasail_sequences_from_file.restype = ctypes.POINTER(PSequences)
    lib.parasail_sequences_from_file.argtypes = [ctypes.c_char_p]
    lib.parasail_sequences_free.argtypes = [ctypes.POINTER(PSequences)]
    lib.parasail_sequences_pack.restype = ctypes.c_void_p
    lib.parasail_sequences_pack.argtypes = [ctypes.POINTER(PSequences), ctypes.POINTER(ctypes.c_size_t)]
    for f in ("parasail_stat_buffer", "parasail_stat_fasta_buffer", "parasail_stat_fastq_buffer"):
        getattr(lib, f).restype = ctypes.POINTER(PFileStat)
        getattr(lib, f).argtypes = [ctypes.c_char_p, ctypes.c_long]
    for f in ("parasail_pack_buffer", "parasail_pack_fasta_buffer", "parasail_pack_fastq_buffer"):
        getattr(lib, f).restype = ctypes.c_void_p
        getattr(lib, f).argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    for f in ("parasail_matrix_from_file", "parasail_matrix_from_file_case_sensitive"):
        getattr(lib, f).restype = ctypes.POINTER(PMatrix)
        getattr(lib, f).argtypes = [ctypes.c_char_p]
    lib.parasail_matrix_free.argtypes = [ctypes.POINTER(PMatrix)]
    return lib


LIB = _bind(ctypes.CDLL(pb.LIB_PATH))


def _ref():
    r = O.ref()
    if r is None:
        pytest.skip("reference library not built")
    return _bind(r)


def _bytes(ps):
    return None if not ps.s else ctypes.string_at(ps.s, ps.l)


def _read_seqs(lib, path):
    p = lib.parasail_sequences_from_file(path.encode())
    if not p:
        return None
    s = p.contents
    recs = [tuple((f.l, _bytes(f)) for f in (r.name, r.comment, r.seq, r.qual)) for r in s.seqs[:s.l]]
    n = ctypes.c_size_t(0)
    packed = lib.parasail_sequences_pack(p, ctypes.byref(n))
    text = ctypes.string_at(packed, n.value)
    _libc.free(packed)
    head = (s.l, s.characters, s.shortest, s.longest, s.mean, s.stddev)
    lib.parasail_sequences_free(p)
    return head, recs, text


def _same_float(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


# inputs the reference's scanners read without running past the buffer:
# every file ends with a newline
FASTA_CASES = [
    b">s1 first sequence\nACGTACGT\nAC\n>s2\tsecond\r\nMKV\r\nLLA\r\n>s3\n\nNNNNN\n",
    b">only\nA\n",
    b">a\nacgtACGT\n>b desc with  spaces \nWWW\n\n\n>c\nY\n",
    b">e1\n>e2\nAC\n",
    b">x\r\nAC\r\n\r\nGT\r\n>y\r\nT\r\n",
    b">p\nMKVLAAGIVALLLAAGCSSSKEETPAQ\nTQAPAAEAPAAEAPAA\n>q\nMSTNPKPQRKTKRNTNRRPQDVKFPGG\n",
]
FASTQ_CASES = [
    b"@r1 desc\nACGT\n+\nIIII\n@r2\nGGC\n+r2\n#!I\n",
    b"@r1\nACGTAC\n+\nIII\nIII\n@r2\nA\n+\n@\n",
    b"@r1\r\nACG\r\n+\r\nIII\r\n",
]
EDGE_RECORD_CASES = [
    b"junk before\n>a\nAC\n",                    # text before the first header is skipped
    b">a\nAC\n>b\nGT",                           # no final newline
    b"@r1\nACGT\n+\nII\n",                      # truncated quality: the file ends there
    b">\nACGT\n",                                # empty name
    b">a x\r\n\r\nAC\n",                         # a blank CRLF line inside a sequence
    b"@r1\nACGT\n+\nIIII\n>f\nMK\n",            # FASTQ then FASTA records
]


def _rng_fasta(rng, n):
    out = []
    for k in range(n):
        name = "seq%d" % k
        hdr = ">" + name + (" comment %d" % rng.integers(100) if rng.random() < 0.5 else "")
        L = int(rng.integers(0 if k < n - 1 else 1, 300))
        s = "".join(rng.choice(list("ACDEFGHIKLMNPQRSTVWYacgtn"), L))
        w = int(rng.integers(5, 80))
        lines = [s[i:i + w] for i in range(0, len(s), w)]
        eol = "\r\n" if rng.random() < 0.3 else "\n"
        out.append(hdr + eol + eol.join(lines) + (eol if lines else "") + (eol if rng.random() < 0.1 else ""))
    return "".join(out).encode()


def test_sequences_from_file_and_pack_match_reference(tmp_path):
    ref = _ref()
    rng = np.random.default_rng(3)
    cases = FASTA_CASES + FASTQ_CASES + EDGE_RECORD_CASES + [_rng_fasta(rng, 50) for _ in range(6)]
    for k, data in enumerate(cases):
        f = tmp_path / ("in%d.txt" % k)
        f.write_bytes(data)
        a = _read_seqs(LIB, str(f))
        b = _read_seqs(ref, str(f))
        assert (a is None) == (b is None), data
        if a is None:
            continue
        (ha, ra, ta), (hb, rb, tb) = a, b
        assert ha[:4] == hb[:4], data
        assert _same_float(ha[4], hb[4]) and _same_float(ha[5], hb[5]), data
        assert ra == rb, data
        assert ta == tb, data


def _stat(lib, fn, data):
    p = getattr(lib, fn)(data, len(data))
    if not p:
        return None
    s = p.contents
    v = (s.sequences, s.characters, s.shortest, s.longest, s.mean, s.stddev)
    _libc.free(ctypes.cast(p, ctypes.c_void_p))
    return v


def _pack(lib, fn, data):
    n = ctypes.c_long(0)
    p = getattr(lib, fn)(data, len(data), ctypes.byref(n))
    if not p:
        return None
    t = ctypes.string_at(p, n.value)
    _libc.free(p)
    return t


def test_stat_and_pack_buffers_match_reference():
    ref = _ref()
    rng = np.random.default_rng(5)
    bad = [b">a\nAC1GT\n", b">a\nAC\n>b\n", b"x>a\nAC\n", b">a\nA\x01C\n"]
    for data in FASTA_CASES + [_rng_fasta(rng, 40) for _ in range(4)] + bad:
        for fn in ("parasail_stat_buffer", "parasail_stat_fasta_buffer"):
            a, b = _stat(LIB, fn, data), _stat(ref, fn, data)
            assert (a is None) == (b is None), (fn, data)
            if a is not None:
                assert a[:4] == b[:4] and _same_float(a[4], b[4]) and _same_float(a[5], b[5]), (fn, data)
        for fn in ("parasail_pack_buffer", "parasail_pack_fasta_buffer"):
            assert _pack(LIB, fn, data) == _pack(ref, fn, data), (fn, data)
    for data in FASTQ_CASES[:1] + FASTQ_CASES[2:] + [b"@a\nAC\n-\nII\n"]:
        a, b = _stat(LIB, "parasail_stat_fastq_buffer", data), _stat(ref, "parasail_stat_fastq_buffer", data)
        assert (a is None) == (b is None), data
        if a is not None:
            assert a[:4] == b[:4] and _same_float(a[4], b[4]) and _same_float(a[5], b[5]), data


def test_pack_fastq_joins_sequence_lines():
    """The reference's FASTQ packer sizes its output from a character count
    its scanner never increments, so it is not run here; the packed text is
    the sequence lines joined by '$', ended by one."""
    data = FASTQ_CASES[0]
    assert _pack(LIB, "parasail_pack_fastq_buffer", data) == b"ACGT$GGC$"
    assert _pack(LIB, "parasail_pack_buffer", FASTQ_CASES[2]) == b"ACG$"
    assert _pack(LIB, "parasail_pack_fastq_buffer", b"@a\nAC\n-\nII\n") is None


MATRIX_FILES = [
    # square, with comments and a '*' column
    b"# a test matrix\n   A  C  G  T  *\nA  2 -3 -3 -3 0\nC -3  2 -3 -3 0\nG -3 -3  2 -3 0\nT -3 -3 -3  2 0\n"
    b"* 0 0 0 0 0\n",
    # PSSM rows with letters
    b"  A R N D\nM 1 2 3 4\nK -1 -2 -3 -4\nV 5 -6 7 -8\n",
    # PSSM rows without letters
    b"A C G T\n 1 -1 -1 -1\n-1 1 -1 -1\n",
    # lower-case alphabet, CRLF
    b"   a  c\r\na  1 -1\r\nc -1  1\r\n",
    # errors: missing values, bad character, too long a number
    b"A C\nA 1\nC 1 2\n",
    b"A C\nA 1 2\nC 1 $\n",
    b"A C\nA 1 2\nC 1 12345678901\n",
]


def _matrix(lib, fn, path):
    p = getattr(lib, fn)(path.encode())
    if not p:
        return None
    m = p.contents
    rows = m.length if m.type == 1 else m.size
    v = (m.size, m.max, m.min, m.type, m.length, m.alphabet, m.query,
         list(m.matrix[:m.size * rows]), list(m.mapper[:256]))
    lib.parasail_matrix_free(p)
    return v


def test_matrix_from_file_matches_reference(tmp_path):
    ref = _ref()
    for k, data in enumerate(MATRIX_FILES):
        f = tmp_path / ("m%d.txt" % k)
        f.write_bytes(data)
        for fn in ("parasail_matrix_from_file", "parasail_matrix_from_file_case_sensitive"):
            assert _matrix(LIB, fn, str(f)) == _matrix(ref, fn, str(f)), (fn, data)
