"""CPU oracle for parasail-b200 -- TEST INFRASTRUCTURE ONLY.

Two checkers, both CPU-only:

* `liboracle.so` (built from oracle/oracle.c): the project's plain-C
  restatement of the reference's serial dynamic programs (jeffdaily/parasail
  v2.6.2 src/sw.c, src/nw.c, src/sg.c, their _stats twins and src/nw_banded.c)
  plus the padded-layout statistics the vector kernels' saturation checks read.
* `libparasail_ref.so` (built by oracle/Makefile from the reference's own
  sources, when they were available at build time): the reference itself --
  its serial functions and its AVX2 striped/scan kernels -- used to pin the
  restatement and as the flag-exact checker.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference
legs import this package, and only as the checker / CPU baseline. The product
(parasail_b200/libparasail_b200.so) never loads it.
"""
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(REF_DIR, "liboracle.so")
REF_SO = os.path.join(REF_DIR, "libparasail_ref.so")

SW, NW, SG = 0, 1, 2
S1_BEG, S1_END, S2_BEG, S2_END = 1, 2, 4, 8
SG_CASES = {  # reference src/sg_helper.h:53-63
    "sg": S1_BEG | S1_END | S2_BEG | S2_END, "sg_qb": S1_BEG, "sg_qe": S1_END,
    "sg_qx": S1_BEG | S1_END, "sg_db": S2_BEG, "sg_de": S2_END, "sg_dx": S2_BEG | S2_END,
    "sg_qb_de": S1_BEG | S2_END, "sg_qe_db": S1_END | S2_BEG, "sg_qb_db": S1_BEG | S2_BEG,
    "sg_qe_de": S1_END | S2_END,
}


def alg_of(name):
    """('sw'|'nw'|'sg_qx'|...) -> (alg, sgflags)."""
    if name == "sw":
        return SW, 0
    if name == "nw":
        return NW, 0
    return SG, SG_CASES[name]


class OMatrix(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int), ("matrix", ctypes.POINTER(ctypes.c_int)),
                ("is_pssm", ctypes.c_int), ("max", ctypes.c_int), ("min", ctypes.c_int)]


class OResult(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int), ("end_query", ctypes.c_int), ("end_ref", ctypes.c_int),
                ("matches", ctypes.c_int), ("similar", ctypes.c_int), ("length", ctypes.c_int)]


class OPadStats(ctypes.Structure):
    _fields_ = [("max_h", ctypes.c_int64), ("min_h_real", ctypes.c_int64),
                ("min_h_pad", ctypes.c_int64), ("min_f", ctypes.c_int64),
                ("max_stat", ctypes.c_int64), ("max_stat_real", ctypes.c_int64)]


# parasail.h-compatible structs for the reference library
class PMatrix(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("matrix", ctypes.POINTER(ctypes.c_int)),
                ("mapper", ctypes.POINTER(ctypes.c_int)), ("size", ctypes.c_int),
                ("max", ctypes.c_int), ("min", ctypes.c_int),
                ("user_matrix", ctypes.POINTER(ctypes.c_int)), ("type", ctypes.c_int),
                ("length", ctypes.c_int), ("alphabet", ctypes.c_char_p),
                ("query", ctypes.c_char_p)]


class PResult(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int), ("end_query", ctypes.c_int),
                ("end_ref", ctypes.c_int), ("flag", ctypes.c_int),
                ("extra", ctypes.c_void_p)]


class PStats(ctypes.Structure):
    _fields_ = [("matches", ctypes.c_int), ("similar", ctypes.c_int),
                ("length", ctypes.c_int), ("extra", ctypes.c_void_p)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: make -C oracle oracle")
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.oracle_align.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix), ctypes.POINTER(OResult)]
        _lib.oracle_align_scan.argtypes = [ctypes.c_int] * 2 + [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix), ctypes.POINTER(OResult)]
        _lib.oracle_align_scan_stats.argtypes = _lib.oracle_align_scan.argtypes
        _lib.oracle_padstats.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.POINTER(OMatrix), ctypes.POINTER(OPadStats)]
        _lib.oracle_nw_banded.argtypes = [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix), ctypes.POINTER(OResult)]
        _lib.oracle_align_batch.argtypes = [ctypes.c_int] * 4 + [
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix), ctypes.POINTER(OResult), ctypes.c_int]
        _lib.oracle_nw_band.argtypes = [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix),
            ctypes.POINTER(ctypes.c_int64)]
        _lib.oracle_nw_diag_range.argtypes = [
            ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(OMatrix), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    return _lib


def ref():
    """The reference library compiled from source, or None when absent."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = ctypes.CDLL(REF_SO)
        _ref.parasail_matrix_lookup.restype = ctypes.POINTER(PMatrix)
        _ref.parasail_matrix_lookup.argtypes = [ctypes.c_char_p]
        _ref.parasail_matrix_create.restype = ctypes.POINTER(PMatrix)
        _ref.parasail_matrix_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        _ref.parasail_result_free.argtypes = [ctypes.POINTER(PResult)]
        _ref.parasail_profile_free.argtypes = [ctypes.c_void_p]
    return _ref


class Matrix:
    """Plain-Python copy of a substitution matrix (values, mapper, max, min)."""

    def __init__(self, values, mapper, alphabet, mx, mn, name=""):
        self.values = np.ascontiguousarray(values, dtype=np.int32)
        self.size = self.values.shape[0]
        self.mapper = np.asarray(mapper, dtype=np.int32)
        self.alphabet = alphabet
        self.max, self.min, self.name = mx, mn, name
        self._om = OMatrix(self.size, self.values.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 0,
                           mx, mn)

    @staticmethod
    def from_struct(pm, name=""):
        m = pm.contents
        n = m.size
        vals = np.ctypeslib.as_array(m.matrix, shape=(n * n,)).reshape(n, n).copy()
        mapper = np.ctypeslib.as_array(m.mapper, shape=(256,)).copy()
        return Matrix(vals, mapper, m.alphabet.decode(), m.max, m.min, name)

    @staticmethod
    def simple(alphabet, match, mismatch):
        """parasail_matrix_create semantics (reference src/memory.c:336-407)."""
        n = len(alphabet) + 1
        v = np.zeros((n, n), dtype=np.int32)
        v[: n - 1, : n - 1] = mismatch
        np.fill_diagonal(v[: n - 1, : n - 1], match)
        mapper = np.full(256, n - 1, dtype=np.int32)
        for i, c in enumerate(alphabet):
            mapper[ord(c.upper())] = i
            mapper[ord(c.lower())] = i
        return Matrix(v, mapper, alphabet + "*", max(match, mismatch), min(match, mismatch))

    def codes(self, s):
        b = np.frombuffer(s.encode() if isinstance(s, str) else s, dtype=np.uint8)
        return np.ascontiguousarray(self.mapper[b], dtype=np.int32)


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def align(alg, sgflags, stats, q, t, open_, gap, m):
    """Serial restatement. q, t: strings. Returns a dict."""
    qc, tc = m.codes(q), m.codes(t)
    r = OResult()
    rc = lib().oracle_align(alg, sgflags, int(stats), _ip(qc), len(qc), _ip(tc), len(tc),
                            open_, gap, ctypes.byref(m._om), ctypes.byref(r))
    if rc != 0:
        raise ValueError("oracle_align rejected its input")
    out = {"score": r.score, "end_query": r.end_query, "end_ref": r.end_ref}
    if stats:
        out.update(matches=r.matches, similar=r.similar, length=r.length)
    return out


def align_scan(alg, sgflags, q, t, open_, gap, m):
    """The reference's serial scan forms (score only): src/nw_scan.c,
    src/sg_scan.c, src/sw_scan.c, which depart from align() at open < gap."""
    qc, tc = m.codes(q), m.codes(t)
    r = OResult()
    rc = lib().oracle_align_scan(alg, sgflags, _ip(qc), len(qc), _ip(tc), len(tc), open_, gap,
                                 ctypes.byref(m._om), ctypes.byref(r))
    if rc != 0:
        raise ValueError("oracle_align_scan rejected its input")
    return {"score": r.score, "end_query": r.end_query, "end_ref": r.end_ref}


def align_scan_stats(alg, sgflags, q, t, open_, gap, m):
    """The reference's serial scan forms with statistics: src/nw_stats_scan.c,
    src/sg_stats_scan.c, src/sw_stats_scan.c, which depart from align() at
    open < gap."""
    qc, tc = m.codes(q), m.codes(t)
    r = OResult()
    rc = lib().oracle_align_scan_stats(alg, sgflags, _ip(qc), len(qc), _ip(tc), len(tc), open_, gap,
                                       ctypes.byref(m._om), ctypes.byref(r))
    if rc != 0:
        raise ValueError("oracle_align_scan_stats rejected its input")
    return {"score": r.score, "end_query": r.end_query, "end_ref": r.end_ref,
            "matches": r.matches, "similar": r.similar, "length": r.length}


def padstats(alg, sgflags, stats, q, t, open_, gap, m, padlen):
    qc, tc = m.codes(q), m.codes(t)
    ps = OPadStats()
    lib().oracle_padstats(alg, sgflags, int(stats), _ip(qc), len(qc), padlen, _ip(tc), len(tc),
                          open_, gap, ctypes.byref(m._om), ctypes.byref(ps))
    return {f: getattr(ps, f) for f, _ in OPadStats._fields_}


def nw_banded(q, t, open_, gap, k, m):
    qc, tc = m.codes(q), m.codes(t)
    r = OResult()
    lib().oracle_nw_banded(_ip(qc), len(qc), _ip(tc), len(tc), open_, gap, k,
                           ctypes.byref(m._om), ctypes.byref(r))
    return {"score": r.score, "end_query": r.end_query, "end_ref": r.end_ref}


def align_batch(alg, sgflags, stats, queries, targets, open_, gap, m, nthreads=0):
    """Many pairs (OpenMP). queries/targets: lists of strings of equal count."""
    n = len(targets)
    qcat = [m.codes(q) for q in queries]
    tcat = [m.codes(t) for t in targets]
    qlen = np.array([len(x) for x in qcat], dtype=np.int32)
    tlen = np.array([len(x) for x in tcat], dtype=np.int32)
    qoff = np.zeros(n, dtype=np.int64)
    toff = np.zeros(n, dtype=np.int64)
    qoff[1:] = np.cumsum(qlen)[:-1]
    toff[1:] = np.cumsum(tlen)[:-1]
    qc = np.concatenate(qcat).astype(np.int32)
    tc = np.concatenate(tcat).astype(np.int32)
    res = (OResult * n)()
    nthreads = nthreads or os.cpu_count() or 1
    rc = lib().oracle_align_batch(alg, sgflags, int(stats), n, _ip(qc),
                                  qoff.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _ip(qlen),
                                  _ip(tc), toff.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                  _ip(tlen), open_, gap, ctypes.byref(m._om), res, nthreads)
    if rc != 0:
        raise ValueError("oracle_align_batch rejected an input")
    return res


def nw_band(q, t, open_, gap, lo, hi, m):
    """Global score restricted to diagonals lo <= i - j <= hi."""
    qc, tc = m.codes(q), m.codes(t)
    out = ctypes.c_int64()
    lib().oracle_nw_band(_ip(qc), len(qc), _ip(tc), len(tc), open_, gap, lo, hi, ctypes.byref(m._om),
                         ctypes.byref(out))
    return out.value


def nw_diag_range(q, t, open_, gap, m):
    qc, tc = m.codes(q), m.codes(t)
    lo, hi, sc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().oracle_nw_diag_range(_ip(qc), len(qc), _ip(tc), len(tc), open_, gap, ctypes.byref(m._om),
                               ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(sc))
    return lo.value, hi.value, sc.value


# ----------------------------------------------------------------------------
# The reference library itself (when built)

def ref_matrix(name):
    r = ref()
    if r is None:
        return None
    pm = r.parasail_matrix_lookup(name.encode())
    return Matrix.from_struct(pm, name) if pm else None


def _ref_result(r, rp):
    if not rp:
        return None
    c = rp.contents
    out = {"score": c.score, "end_query": c.end_query, "end_ref": c.end_ref, "flag": c.flag}
    if c.flag & (1 << 16) and c.extra:
        st = ctypes.cast(c.extra, ctypes.POINTER(PStats)).contents
        out.update(matches=st.matches, similar=st.similar, length=st.length)
    r.parasail_result_free(rp)
    return out


_ref_matrix_cache = {}


def ref_matrix_ptr(name_or_simple):
    """Reference-library matrix pointer for a built-in name or ('ACGT', match, mismatch)."""
    r = ref()
    key = name_or_simple if isinstance(name_or_simple, str) else tuple(name_or_simple)
    if key not in _ref_matrix_cache:
        if isinstance(name_or_simple, str):
            _ref_matrix_cache[key] = r.parasail_matrix_lookup(name_or_simple.encode())
        else:
            a, mt, mm = name_or_simple
            _ref_matrix_cache[key] = r.parasail_matrix_create(a.encode(), mt, mm)
    return _ref_matrix_cache[key]


def ref_vector(alg_name, stats, scheme, width, q, t, open_, gap, matrix_key):
    """Runs the reference's AVX2 profile kernel (or its 8->16->32 chain for
    width 'sat', src/satcheck.c) on one pair. Returns a dict or None."""
    r = ref()
    if r is None:
        return None
    mp = ref_matrix_ptr(matrix_key)
    qb = q.encode()
    tb = t.encode()
    widths = [8, 16, 32] if width == "sat" else [int(width)]
    st = "_stats" if stats else ""
    out = None
    for w in widths:
        cname = "parasail_profile_create%s_avx_256_%d" % (st, w)
        fname = "parasail_%s%s_%s_profile_avx2_256_%d" % (alg_name, st, scheme, w)
        creator = getattr(r, cname)
        creator.restype = ctypes.c_void_p
        creator.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(PMatrix)]
        fn = getattr(r, fname)
        fn.restype = ctypes.POINTER(PResult)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        prof = creator(qb, len(qb), mp)
        out = _ref_result(r, fn(prof, tb, len(tb), open_, gap))
        r.parasail_profile_free(prof)
        if not (out["flag"] & (1 << 6)):
            break
    return out


def ref_serial(alg_name, stats, q, t, open_, gap, matrix_key, scan=False):
    r = ref()
    if r is None:
        return None
    mp = ref_matrix_ptr(matrix_key)
    fname = "parasail_%s%s%s" % (alg_name, "_stats" if stats else "", "_scan" if scan else "")
    fn = getattr(r, fname)
    fn.restype = ctypes.POINTER(PResult)
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.POINTER(PMatrix)]
    qb, tb = q.encode(), t.encode()
    return _ref_result(r, fn(qb, len(qb), tb, len(tb), open_, gap, mp))


def ref_nw_banded(q, t, open_, gap, k, matrix_key):
    r = ref()
    if r is None:
        return None
    mp = ref_matrix_ptr(matrix_key)
    fn = r.parasail_nw_banded
    fn.restype = ctypes.POINTER(PResult)
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(PMatrix)]
    qb, tb = q.encode(), t.encode()
    return _ref_result(r, fn(qb, len(qb), tb, len(tb), open_, gap, k, mp))


class PCigar(ctypes.Structure):
    _fields_ = [("seq", ctypes.POINTER(ctypes.c_uint32)), ("len", ctypes.c_int),
                ("beg_query", ctypes.c_int), ("beg_ref", ctypes.c_int)]


class PTraceback(ctypes.Structure):
    _fields_ = [("query", ctypes.c_void_p), ("comp", ctypes.c_void_p), ("ref", ctypes.c_void_p)]


def ref_traceback_text(r, rp, q, t, mp, aliases=None, case_sensitive=0):
    """The reference's traceback strings and printed alignments of its trace
    result rp (src/traceback.c: parasail_result_get_traceback_extra and
    parasail_traceback_generic_extra2, in the two layouts of the reference
    aligner's EMBOSS and SSW outputs, apps/parasail_aligner.cpp:2240-2350)."""
    import tempfile
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    RP = ctypes.POINTER(PResult)
    MP = ctypes.POINTER(PMatrix)
    r.parasail_result_get_traceback_extra.restype = ctypes.POINTER(PTraceback)
    r.parasail_result_get_traceback_extra.argtypes = [RP, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                                      ctypes.c_int, MP, ctypes.c_char, ctypes.c_char,
                                                      ctypes.c_char, ctypes.c_int, ctypes.c_char_p]
    r.parasail_traceback_free.argtypes = [ctypes.POINTER(PTraceback)]
    r.parasail_traceback_generic_extra2.restype = None
    r.parasail_traceback_generic_extra2.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                                    ctypes.c_char_p, ctypes.c_char_p, MP, RP, ctypes.c_char,
                                                    ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                    ctypes.c_char_p]
    b1, b2 = q.encode(), t.encode()
    al = aliases.encode() if aliases else None
    tb = r.parasail_result_get_traceback_extra(rp, b1, len(b1), b2, len(b2), mp, b"|", b":", b".",
                                               case_sensitive, al)
    rows = (None, None, None)
    if tb:
        rows = tuple(ctypes.string_at(getattr(tb.contents, f)).decode() for f in ("query", "comp", "ref"))
        r.parasail_traceback_free(tb)
    with tempfile.NamedTemporaryFile(suffix=".txt") as f:
        fp = libc.fopen(f.name.encode(), b"w")
        r.parasail_traceback_generic_extra2(b1, len(b1), b2, len(b2), b"query_name", b"a_long_target_name", mp,
                                            rp, b"|", b":", b".", 50, 14, 1, 7, fp, case_sensitive, al)
        r.parasail_traceback_generic_extra2(b1, len(b1), b2, len(b2), b"Query:", b"Target:", mp, rp,
                                            b"|", b"*", b"*", 60, 10, 0, 7, fp, case_sensitive, al)
        libc.fclose(fp)
        text = open(f.name).read()
    return rows + (text,)


def ref_trace(alg_name, form, q, t, open_, gap, matrix_key, strings=False):
    """The reference's trace function `parasail_{alg}_trace{form}` on one pair
    (form "", "_scan", or "_striped_W" / "_scan_W" with W 8, 16, 32 or sat;
    the vector forms call the AVX2 kernels and their _sat dispatcher),
    followed by its parasail_result_get_cigar (src/cigar.c) unless the
    result is saturated. Returns {score, end_query, end_ref, flag, cigar,
    beg_query, beg_ref} (cigar None when there is none)."""
    r = ref()
    if r is None:
        return None
    mp = ref_matrix_ptr(matrix_key)
    def kernel(f):
        fn = getattr(r, "parasail_%s_trace%s" % (alg_name, re.sub(r"_(8|16|32)$", r"_avx2_256_\1", f)))
        fn.restype = ctypes.POINTER(PResult)
        fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                       ctypes.c_int, ctypes.POINTER(PMatrix)]
        return fn

    if form.endswith("_sat"):
        # the _sat dispatcher (src/satcheck.c:8505-8524): 8 bits, then 16,
        # then 32 while the result is saturated
        widths = [form[:-3] + w for w in ("8", "16", "32")]

        def fn(*args):
            for k, f in enumerate(widths):
                res = kernel(f)(*args)
                if k == 2 or not res.contents.flag & 64:
                    return res
                r.parasail_result_free(res)
    else:
        fn = kernel(form)
    r.parasail_result_get_cigar.restype = ctypes.POINTER(PCigar)
    r.parasail_result_get_cigar.argtypes = [ctypes.POINTER(PResult), ctypes.c_char_p, ctypes.c_int,
                                            ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(PMatrix)]
    r.parasail_cigar_decode.restype = ctypes.c_void_p
    r.parasail_cigar_decode.argtypes = [ctypes.POINTER(PCigar)]
    r.parasail_cigar_free.argtypes = [ctypes.POINTER(PCigar)]
    qb, tb = q.encode(), t.encode()
    rp = fn(qb, len(qb), tb, len(tb), open_, gap, mp)
    c = rp.contents
    out = {"score": c.score, "end_query": c.end_query, "end_ref": c.end_ref, "flag": c.flag,
           "cigar": None, "beg_query": None, "beg_ref": None}
    cg = None if c.flag & 64 else r.parasail_result_get_cigar(rp, qb, len(qb), tb, len(tb), mp)
    if cg:
        s = ctypes.cast(r.parasail_cigar_decode(cg), ctypes.c_char_p).value.decode()
        out.update(cigar=s, beg_query=cg.contents.beg_query, beg_ref=cg.contents.beg_ref)
        r.parasail_cigar_free(cg)
    if strings and not c.flag & 64:
        out["traceback"] = ref_traceback_text(r, rp, q, t, mp, **(strings if isinstance(strings, dict) else {}))
    r.parasail_result_free(rp)
    return out


# ---------------------------------------------------------------------------
# Candidate pairs of the aligner's suffix-array filter

ESA_SO = os.path.join(REF_DIR, "libesa_ref.so")
_esa = None


def esa_pairs(text, cutoff, db_chars=-1, sentinel=b"$"):
    """Pairs the reference aligner's enhanced-suffix-array filter keeps for
    the '$'-separated text (bytes): the reference's own sais builds SA/LCP,
    oracle/esa_pairs.cpp restates the traversal
    (apps/parasail_aligner.cpp:1316-1420, :1816-1904). db_chars >= 0: the
    first db_chars characters are the database file, the rest queries.
    Returns a sorted list of (first, second), or None without the library."""
    global _esa
    if _esa is None:
        if not os.path.exists(ESA_SO):
            return None
        _esa = ctypes.CDLL(ESA_SO)
        _esa.esa_pairs.restype = ctypes.c_long
        _esa.esa_pairs.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_ubyte, ctypes.c_int, ctypes.c_long,
                                   ctypes.c_void_p, ctypes.c_long]
    import numpy as np
    cap = 1 << 16
    while True:
        out = np.zeros(2 * cap, np.int32)
        k = _esa.esa_pairs(text, len(text), sentinel[0], cutoff, db_chars, out.ctypes.data, cap)
        if k < 0:
            raise RuntimeError("esa_pairs failed")
        if k <= cap:
            return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(k)]
        cap = k


def kmer_pairs(seqs, cutoff, n_db=None):
    """The same pair set stated directly (pure Python, small inputs): two
    sequences pair when they share a substring of `cutoff` characters. With
    n_db, only (query, database) pairs, queries numbered after the database
    sequences."""
    seen = {}
    for sid, s in enumerate(seqs):
        for p in range(len(s) - cutoff + 1):
            seen.setdefault(s[p:p + cutoff], set()).add(sid)
    out = set()
    for ids in seen.values():
        ids = sorted(ids)
        for x in range(len(ids)):
            for y in range(x + 1, len(ids)):
                a, b = ids[x], ids[y]
                if n_db is None:
                    out.add((a, b))
                elif (a < n_db) != (b < n_db):
                    out.add((b, a))
    return sorted(out)
