"""ctypes mirror of the C API of libparasail_b200.so (parasail.h and the
batch extensions of parasail_b200.h).

The product is the C library `libparasail_b200.so` (C host code + sm_100a
CUDA kernels) built in this directory; this module is a thin ctypes mirror of
its C API, used by the tests and the benchmark. It is loaded on first use of
an attribute of the `parasail_b200` package. Every call goes through the
C ABI. There is no Python or CPU implementation of any alignment here: if the
library is missing the import fails, and on a machine without a usable GPU
the alignment calls return NULL, which this module raises as RuntimeError.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libparasail_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("parasail_b200: %s is not built (run __graft_entry__.build())" % LIB_PATH)

lib = ctypes.CDLL(LIB_PATH)

FLAG_NW = 1 << 0
FLAG_SG = 1 << 1
FLAG_SW = 1 << 2
FLAG_SG_S1_BEG = 1 << 3
FLAG_SG_S1_END = 1 << 4
FLAG_SATURATED = 1 << 6
FLAG_BANDED = 1 << 7
FLAG_NOVEC = 1 << 8
FLAG_NOVEC_SCAN = 1 << 9
FLAG_SCAN = 1 << 10
FLAG_STRIPED = 1 << 11
FLAG_SG_S2_BEG = 1 << 14
FLAG_SG_S2_END = 1 << 15
FLAG_STATS = 1 << 16
FLAG_BITS_8 = 1 << 20
FLAG_BITS_16 = 1 << 21
FLAG_BITS_32 = 1 << 22


class ResultStats(ctypes.Structure):
    _fields_ = [("matches", ctypes.c_int), ("similar", ctypes.c_int),
                ("length", ctypes.c_int), ("extra", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int), ("end_query", ctypes.c_int),
                ("end_ref", ctypes.c_int), ("flag", ctypes.c_int),
                ("extra", ctypes.c_void_p)]


class Matrix(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("matrix", ctypes.POINTER(ctypes.c_int)),
                ("mapper", ctypes.POINTER(ctypes.c_int)), ("size", ctypes.c_int),
                ("max", ctypes.c_int), ("min", ctypes.c_int),
                ("user_matrix", ctypes.POINTER(ctypes.c_int)), ("type", ctypes.c_int),
                ("length", ctypes.c_int), ("alphabet", ctypes.c_char_p),
                ("query", ctypes.c_char_p)]


class ProfileData(ctypes.Structure):
    _fields_ = [("score", ctypes.c_void_p), ("matches", ctypes.c_void_p),
                ("similar", ctypes.c_void_p)]


class Profile(ctypes.Structure):
    _fields_ = [("s1", ctypes.c_char_p), ("s1Len", ctypes.c_int),
                ("matrix", ctypes.POINTER(Matrix)),
                ("profile8", ProfileData), ("profile16", ProfileData),
                ("profile32", ProfileData), ("profile64", ProfileData),
                ("free", ctypes.c_void_p), ("stop", ctypes.c_int)]


_RP = ctypes.POINTER(Result)
_MP = ctypes.POINTER(Matrix)
_PP = ctypes.POINTER(Profile)

lib.parasail_matrix_lookup.restype = _MP
lib.parasail_matrix_lookup.argtypes = [ctypes.c_char_p]
lib.parasail_matrix_create.restype = _MP
lib.parasail_matrix_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
lib.parasail_matrix_free.argtypes = [_MP]
lib.parasail_result_free.argtypes = [_RP]
lib.parasail_profile_free.argtypes = [_PP]
lib.parasail_nw_banded.restype = _RP
lib.parasail_nw_banded.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _MP]
for _n in ("get_matches", "get_similar", "get_length"):
    getattr(lib, "parasail_result_" + _n).argtypes = [_RP]


def matrix_lookup(name):
    m = lib.parasail_matrix_lookup(name.encode())
    if not m:
        raise KeyError(name)
    return m


def matrix_create(alphabet, match, mismatch):
    return lib.parasail_matrix_create(alphabet.encode(), match, mismatch)


def _fn(name, profile_form):
    f = getattr(lib, name)
    f.restype = _RP
    if profile_form:
        f.argtypes = [_PP, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    else:
        f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                      ctypes.c_int, ctypes.c_int, _MP]
    return f


def _unpack(r, name):
    if not r:
        raise RuntimeError("%s returned NULL" % name)
    c = r.contents
    out = {"score": c.score, "end_query": c.end_query, "end_ref": c.end_ref, "flag": c.flag}
    if c.flag & FLAG_STATS:
        st = ctypes.cast(c.extra, ctypes.POINTER(ResultStats)).contents
        out.update(matches=st.matches, similar=st.similar, length=st.length)
    lib.parasail_result_free(r)
    return out


def align(name, s1, s2, open_, gap, matrix):
    """Calls a direct-form entry point, e.g. align('parasail_sw_striped_16', ...)."""
    b1, b2 = s1.encode() if isinstance(s1, str) else s1, s2.encode() if isinstance(s2, str) else s2
    return _unpack(_fn(name, False)(b1, len(b1), b2, len(b2), open_, gap, matrix), name)


class ProfileHandle:
    """Owns a parasail_profile_t and the query bytes it borrows."""

    def __init__(self, creator, s1, matrix):
        self.s1 = s1.encode() if isinstance(s1, str) else s1
        self.matrix = matrix
        f = getattr(lib, creator)
        f.restype = _PP
        f.argtypes = [ctypes.c_char_p, ctypes.c_int, _MP]
        self.ptr = f(self.s1, len(self.s1), matrix)
        if not self.ptr:
            raise RuntimeError("%s returned NULL" % creator)

    def close(self):
        # at interpreter exit the module globals may already be gone
        if self.ptr and lib is not None:
            lib.parasail_profile_free(self.ptr)
        self.ptr = None

    def __del__(self):
        self.close()


def align_profile(name, profile, s2, open_, gap):
    b2 = s2.encode() if isinstance(s2, str) else s2
    return _unpack(_fn(name, True)(profile.ptr, b2, len(b2), open_, gap), name)


def nw_banded(s1, s2, open_, gap, k, matrix):
    b1, b2 = s1.encode(), s2.encode()
    return _unpack(lib.parasail_nw_banded(b1, len(b1), b2, len(b2), open_, gap, k, matrix),
                   "parasail_nw_banded")


# ---------------------------------------------------------------------------
# Batch API (include/parasail_b200.h)

class Record(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int), ("end_query", ctypes.c_int), ("end_ref", ctypes.c_int),
                ("flag", ctypes.c_int), ("matches", ctypes.c_int), ("similar", ctypes.c_int),
                ("length", ctypes.c_int), ("reserved", ctypes.c_int)]


lib.parasail_b200_batch_profile.restype = ctypes.c_int
lib.parasail_b200_batch_profile.argtypes = [ctypes.c_char_p, _PP, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p]
lib.parasail_b200_batch_profile_device.restype = ctypes.c_int
lib.parasail_b200_batch_profile_device.argtypes = [ctypes.c_char_p, _PP, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_batch_profile_device_noalloc.restype = ctypes.c_int
lib.parasail_b200_batch_profile_device_noalloc.argtypes = lib.parasail_b200_batch_profile_device.argtypes
lib.parasail_b200_noalloc_scratch_bytes.restype = ctypes.c_size_t
lib.parasail_b200_noalloc_scratch_bytes.argtypes = []
lib.parasail_b200_batch_pairs.restype = ctypes.c_int
lib.parasail_b200_batch_pairs.argtypes = [ctypes.c_char_p, _MP] + [ctypes.c_void_p] * 6 + \
    [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_kernel_launches.restype = ctypes.c_long
lib.parasail_b200_sw16_kernel_ms.restype = ctypes.c_double
lib.parasail_b200_sw16_kernel_ms.argtypes = [ctypes.POINTER(ctypes.c_long)]
lib.parasail_b200_dpx_peak.restype = ctypes.c_double


def _np():
    import numpy
    return numpy


def pack(seqs):
    """list of str/bytes -> (uint8 buffer, int64 offsets, int32 lengths)."""
    np = _np()
    bs = [s.encode() if isinstance(s, str) else s for s in seqs]
    lens = np.array([len(b) for b in bs], dtype=np.int32)
    offs = np.zeros(len(bs), dtype=np.int64)
    if len(bs):
        offs[1:] = np.cumsum(lens, dtype=np.int64)[:-1]
    buf = np.frombuffer(b"".join(bs), dtype=np.uint8).copy() if bs else np.zeros(0, np.uint8)
    return buf, offs, lens


def records_to_dicts(recs, stats):
    out = []
    for r in recs:
        d = {"score": int(r["score"]), "end_query": int(r["end_query"]), "end_ref": int(r["end_ref"]),
             "flag": int(r["flag"])}
        if stats and (d["flag"] & FLAG_STATS):
            d.update(matches=int(r["matches"]), similar=int(r["similar"]), length=int(r["length"]))
        out.append(d)
    return out


RECORD_DTYPE = None


def record_dtype():
    global RECORD_DTYPE
    if RECORD_DTYPE is None:
        np = _np()
        RECORD_DTYPE = np.dtype([(n, np.int32) for n, _ in Record._fields_])
    return RECORD_DTYPE


def batch_profile(name, profile, targets, open_, gap, packed=None):
    """Aligns many targets against profile with one batch call. Returns a
    numpy structured array of records."""
    np = _np()
    buf, offs, lens = packed if packed is not None else pack(targets)
    n = len(lens)
    recs = np.zeros(n, dtype=record_dtype())
    rc = lib.parasail_b200_batch_profile(name.encode(), profile.ptr, buf.ctypes.data, offs.ctypes.data,
                                         lens.ctypes.data, n, open_, gap, recs.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_batch_profile failed")
    return recs


def batch_pairs(name, matrix, queries, targets, open_, gap):
    np = _np()
    qb, qo, ql = pack(queries)
    tb, to, tl = pack(targets)
    n = len(tl)
    recs = np.zeros(n, dtype=record_dtype())
    rc = lib.parasail_b200_batch_pairs(name.encode(), matrix, qb.ctypes.data, qo.ctypes.data, ql.ctypes.data,
                                       tb.ctypes.data, to.ctypes.data, tl.ctypes.data, n, open_, gap,
                                       recs.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_batch_pairs failed")
    return recs

lib.parasail_b200_batch_db.restype = ctypes.c_int
lib.parasail_b200_batch_db.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_batch_db_device.restype = ctypes.c_int
lib.parasail_b200_batch_db_device.argtypes = lib.parasail_b200_batch_db.argtypes


lib.parasail_b200_batch_pairs_device.restype = ctypes.c_int
lib.parasail_b200_batch_pairs_device.argtypes = [ctypes.c_char_p, _MP] + [ctypes.c_void_p] * 6 + \
    [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_batch_all.restype = ctypes.c_int
lib.parasail_b200_batch_all.argtypes = [ctypes.c_char_p, _MP, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_batch_all_device.restype = ctypes.c_int
lib.parasail_b200_batch_all_device.argtypes = lib.parasail_b200_batch_all.argtypes


def batch_all(name, matrix, seqs, open_, gap, packed=None):
    """Every pair (i, j), i < j, of seqs; returns the n(n-1)/2 records in
    row-major upper-triangle order."""
    np = _np()
    buf, offs, lens = packed if packed is not None else pack(seqs)
    n = len(lens)
    recs = np.zeros(max(0, n * (n - 1) // 2), dtype=record_dtype())
    rc = lib.parasail_b200_batch_all(name.encode(), matrix, buf.ctypes.data, offs.ctypes.data, lens.ctypes.data,
                                     n, open_, gap, recs.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_batch_all failed")
    return recs


def profile_array(profiles):
    arr = (_PP * len(profiles))(*[p.ptr for p in profiles])
    return arr


def batch_db(name, profiles, targets, open_, gap, packed=None):
    """Every profile against every target in one call; returns records
    shaped [len(profiles), n]."""
    np = _np()
    buf, offs, lens = packed if packed is not None else pack(targets)
    n = len(lens)
    recs = np.zeros(len(profiles) * n, dtype=record_dtype())
    arr = profile_array(profiles)
    rc = lib.parasail_b200_batch_db(name.encode(), ctypes.cast(arr, ctypes.c_void_p), len(profiles),
                                    buf.ctypes.data, offs.ctypes.data, lens.ctypes.data, n, open_, gap,
                                    recs.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_batch_db failed")
    return recs.reshape(len(profiles), n)


# ---------------------------------------------------------------------------
# Long global alignments and the learned band

class BandStats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_longlong), ("certified", ctypes.c_longlong),
                ("fallback", ctypes.c_longlong), ("band_cells", ctypes.c_double)]


_V = ctypes.c_void_p
lib.parasail_b200_nw_long.restype = ctypes.c_int
lib.parasail_b200_nw_long.argtypes = [_MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int, ctypes.c_int, _V]
lib.parasail_b200_band_model_new.restype = _V
lib.parasail_b200_band_model_new.argtypes = [ctypes.c_uint]
lib.parasail_b200_band_model_free.argtypes = [_V]
lib.parasail_b200_band_model_sizes.argtypes = [ctypes.POINTER(ctypes.c_int)] * 5
lib.parasail_b200_band_model_get.argtypes = [_V, _V, _V]
lib.parasail_b200_band_model_scaling.restype = None
lib.parasail_b200_band_model_scaling.argtypes = [_V, _V, _V]
lib.parasail_b200_band_model_set.argtypes = [_V, _V, _V]
lib.parasail_b200_band_features.argtypes = [_MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, _V]
lib.parasail_b200_band_model_gradients.argtypes = [_V, _V, _V, ctypes.c_int, ctypes.c_float, _V, _V,
                                                   ctypes.POINTER(ctypes.c_float)]
lib.parasail_b200_band_model_train.argtypes = [_V, _MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                               ctypes.POINTER(ctypes.c_float)]
lib.parasail_b200_nw_learned_band.argtypes = [_V, _MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_float, ctypes.c_int, _V, _V, _V,
                                              ctypes.POINTER(BandStats)]
lib.parasail_b200_nw_banded_certified.argtypes = [_MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, _V, _V, _V, _V]


lib.parasail_b200_nw_banded_batch.restype = ctypes.c_int
lib.parasail_b200_nw_banded_batch.argtypes = [_MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, _V]


def _pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen):
    return (qbuf.ctypes.data, qoff.ctypes.data, qlen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
            tlen.ctypes.data)


def nw_long(matrix, qbuf, qoff, qlen, tbuf, toff, tlen, open_, gap):
    np = _np()
    n = len(qlen)
    out = np.zeros(n, dtype=np.int32)
    rc = lib.parasail_b200_nw_long(matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen), n, open_, gap,
                                   out.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_nw_long failed")
    return out


class BandModel:
    def __init__(self, seed=1):
        self.ptr = lib.parasail_b200_band_model_new(seed)
        if not self.ptr:
            raise RuntimeError("parasail_b200_band_model_new failed")
        v = [ctypes.c_int() for _ in range(5)]
        lib.parasail_b200_band_model_sizes(*[ctypes.byref(x) for x in v])
        self.n_in, self.n_hidden, self.n_out, self.n_weights, self.n_biases = [x.value for x in v]

    def close(self):
        if self.ptr:
            lib.parasail_b200_band_model_free(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()

    def get(self):
        np = _np()
        w = np.zeros(self.n_weights, np.float32)
        b = np.zeros(self.n_biases, np.float32)
        if lib.parasail_b200_band_model_get(self.ptr, w.ctypes.data, b.ctypes.data) != 0:
            raise RuntimeError("get failed")
        return w, b

    def set(self, w, b):
        np = _np()
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        if lib.parasail_b200_band_model_set(self.ptr, w.ctypes.data, b.ctypes.data) != 0:
            raise RuntimeError("set failed")

    def scaling(self):
        """(widen, slack) chosen at training on held-out pairs."""
        w, sl = ctypes.c_float(), ctypes.c_int()
        lib.parasail_b200_band_model_scaling(self.ptr, ctypes.byref(w), ctypes.byref(sl))
        return float(w.value), int(sl.value)

    def gradients(self, x, target, tau):
        np = _np()
        x = np.ascontiguousarray(x, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        gw = np.zeros(self.n_weights, np.float32)
        gb = np.zeros(self.n_biases, np.float32)
        loss = ctypes.c_float()
        rc = lib.parasail_b200_band_model_gradients(self.ptr, x.ctypes.data, target.ctypes.data, len(x), tau,
                                                    gw.ctypes.data, gb.ctypes.data, ctypes.byref(loss))
        if rc != 0:
            raise RuntimeError("gradients failed")
        return gw, gb, loss.value

    def train(self, matrix, qbuf, qoff, qlen, tbuf, toff, tlen, open_, gap, epochs=30, batch=256, lr=1e-3):
        loss = ctypes.c_float()
        rc = lib.parasail_b200_band_model_train(self.ptr, matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen),
                                                len(qlen), open_, gap, epochs, batch, lr, ctypes.byref(loss))
        if rc != 0:
            raise RuntimeError("train failed")
        return loss.value

    def align(self, matrix, qbuf, qoff, qlen, tbuf, toff, tlen, open_, gap, widen=1.0, slack=32):
        np = _np()
        n = len(qlen)
        sc, lo, hi = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
        st = BandStats()
        rc = lib.parasail_b200_nw_learned_band(self.ptr, matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen),
                                               n, open_, gap, widen, slack, sc.ctypes.data, lo.ctypes.data,
                                               hi.ctypes.data, ctypes.byref(st))
        if rc != 0:
            raise RuntimeError("learned band failed")
        return sc, lo, hi, st


def band_features(matrix, qbuf, qoff, qlen, tbuf, toff, tlen, n_in=258):
    np = _np()
    n = len(qlen)
    f = np.zeros((n, n_in), np.float32)
    if lib.parasail_b200_band_features(matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen), n,
                                       f.ctypes.data) != 0:
        raise RuntimeError("features failed")
    return f


def nw_banded_certified(matrix, qbuf, qoff, qlen, tbuf, toff, tlen, open_, gap, lo, hi):
    np = _np()
    n = len(qlen)
    lo = np.ascontiguousarray(lo, np.int32)
    hi = np.ascontiguousarray(hi, np.int32)
    sc, cert = np.zeros(n, np.int32), np.zeros(n, np.int32)
    rc = lib.parasail_b200_nw_banded_certified(matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen), n,
                                               open_, gap, lo.ctypes.data, hi.ctypes.data, sc.ctypes.data,
                                               cert.ctypes.data)
    if rc != 0:
        raise RuntimeError("banded certified failed")
    return sc, cert


def nw_banded_batch(matrix, queries, targets, open_, gap, k):
    """parasail_nw_banded scores of many pairs in one call."""
    np = _np()
    qb, qo, ql = pack(queries)
    tb, to, tl = pack(targets)
    sc = np.zeros(len(ql), np.int32)
    rc = lib.parasail_b200_nw_banded_batch(matrix, qb.ctypes.data, qo.ctypes.data, ql.ctypes.data, tb.ctypes.data,
                                           to.ctypes.data, tl.ctypes.data, len(ql), open_, gap, k, sc.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_nw_banded_batch failed")
    return sc


lib.parasail_b200_nw_doubling_band.restype = ctypes.c_int
lib.parasail_b200_nw_doubling_band.argtypes = [_MP, _V, _V, _V, _V, _V, _V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, _V, ctypes.POINTER(BandStats)]


def nw_doubling_band(matrix, qbuf, qoff, qlen, tbuf, toff, tlen, open_, gap, w0=64):
    """Certified banded global scores without a model (band doubling)."""
    np = _np()
    n = len(qlen)
    sc = np.zeros(n, np.int32)
    st = BandStats()
    rc = lib.parasail_b200_nw_doubling_band(matrix, *_pairs_args(qbuf, qoff, qlen, tbuf, toff, tlen), n, open_,
                                            gap, w0, sc.ctypes.data, ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("parasail_b200_nw_doubling_band failed")
    return sc, st


# ---------------------------------------------------------------------------
# Traceback and CIGAR (parasail.h trace functions, parasail_b200_batch_pairs_cigar)

class Cigar(ctypes.Structure):
    _fields_ = [("seq", ctypes.POINTER(ctypes.c_uint32)), ("len", ctypes.c_int),
                ("beg_query", ctypes.c_int), ("beg_ref", ctypes.c_int)]


_CP = ctypes.POINTER(Cigar)
lib.parasail_result_get_cigar.restype = _CP
lib.parasail_result_get_cigar.argtypes = [_RP, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, _MP]
lib.parasail_cigar_decode.restype = ctypes.c_void_p
lib.parasail_cigar_decode.argtypes = [_CP]
lib.parasail_cigar_free.argtypes = [_CP]
lib.parasail_cigar_encode_string.restype = _CP
lib.parasail_cigar_encode_string.argtypes = [ctypes.c_char_p]
lib.parasail_cigar_encode.restype = ctypes.c_uint32
lib.parasail_cigar_encode.argtypes = [ctypes.c_uint32, ctypes.c_char]
lib.parasail_cigar_decode_op.restype = ctypes.c_char
lib.parasail_cigar_decode_op.argtypes = [ctypes.c_uint32]
lib.parasail_cigar_decode_len.restype = ctypes.c_uint32
lib.parasail_cigar_decode_len.argtypes = [ctypes.c_uint32]
lib.parasail_b200_batch_pairs_cigar.restype = ctypes.c_int
lib.parasail_b200_batch_pairs_cigar.argtypes = [ctypes.c_char_p, _MP] + [ctypes.c_void_p] * 6 + \
    [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def cigar_string(c):
    """Decoded CIGAR of a parasail_cigar_t pointer (freed here)."""
    p = lib.parasail_cigar_decode(c)
    s = ctypes.cast(p, ctypes.c_char_p).value.decode()
    _libc.free(p)
    out = (s, c.contents.beg_query, c.contents.beg_ref)
    lib.parasail_cigar_free(c)
    return out


class Traceback(ctypes.Structure):
    _fields_ = [("query", ctypes.c_void_p), ("comp", ctypes.c_void_p), ("ref", ctypes.c_void_p)]


_TBP = ctypes.POINTER(Traceback)
lib.parasail_result_get_traceback_extra.restype = _TBP
lib.parasail_result_get_traceback_extra.argtypes = [_RP, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                                    ctypes.c_int, _MP, ctypes.c_char, ctypes.c_char,
                                                    ctypes.c_char, ctypes.c_int, ctypes.c_char_p]
lib.parasail_traceback_free.argtypes = [_TBP]
lib.parasail_traceback_generic_extra2.restype = None
lib.parasail_traceback_generic_extra2.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                                  ctypes.c_char_p, ctypes.c_char_p, _MP, _RP, ctypes.c_char,
                                                  ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.c_char_p]
_libc.fopen.restype = ctypes.c_void_p
_libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
_libc.fclose.argtypes = [ctypes.c_void_p]


def traceback_text(tlib, r, s1, s2, matrix, aliases=None, case_sensitive=0):
    """The traceback strings (parasail_result_get_traceback_extra with '|',
    ':', '.') and the printed alignments of a trace result r in the two
    layouts the reference aligner writes (EMBOSS-like: width 50, names 14,
    statistics; SSW-like: width 60, names 10, '|', '*', '*'), produced by
    library `tlib`. Returns (query, comp, ref, printed_text)."""
    import tempfile
    b1, b2 = s1.encode(), s2.encode()
    al = aliases.encode() if aliases else None
    tb = tlib.parasail_result_get_traceback_extra(r, b1, len(b1), b2, len(b2), matrix, b"|", b":", b".",
                                                  case_sensitive, al)
    rows = (None, None, None)
    if tb:
        rows = tuple(ctypes.string_at(getattr(tb.contents, f)).decode() for f in ("query", "comp", "ref"))
        tlib.parasail_traceback_free(tb)
    with tempfile.NamedTemporaryFile(suffix=".txt") as f:
        fp = _libc.fopen(f.name.encode(), b"w")
        tlib.parasail_traceback_generic_extra2(b1, len(b1), b2, len(b2), b"query_name", b"a_long_target_name",
                                               matrix, r, b"|", b":", b".", 50, 14, 1, 7, fp, case_sensitive, al)
        tlib.parasail_traceback_generic_extra2(b1, len(b1), b2, len(b2), b"Query:", b"Target:", matrix, r,
                                               b"|", b"*", b"*", 60, 10, 0, 7, fp, case_sensitive, al)
        _libc.fclose(fp)
        text = open(f.name).read()
    return rows + (text,)


def trace(name, s1, s2, open_, gap, matrix, profile=None, strings=False):
    """A trace function ('parasail_sw_trace', 'parasail_nw_trace_scan_32',
    ...) on one pair, then parasail_result_get_cigar; with strings=True also
    the traceback strings and printed alignment (traceback_text)."""
    b1, b2 = s1.encode(), s2.encode()
    if profile is not None:
        r = _fn(name, True)(profile.ptr, b2, len(b2), open_, gap)
    else:
        r = _fn(name, False)(b1, len(b1), b2, len(b2), open_, gap, matrix)
    if not r:
        raise RuntimeError("%s returned NULL" % name)
    c = r.contents
    out = {"score": c.score, "end_query": c.end_query, "end_ref": c.end_ref, "flag": c.flag,
           "cigar": None, "beg_query": None, "beg_ref": None}
    cg = None if c.flag & 64 else lib.parasail_result_get_cigar(r, b1, len(b1), b2, len(b2), matrix)
    if cg:
        out["cigar"], out["beg_query"], out["beg_ref"] = cigar_string(cg)
    if strings and not c.flag & 64:
        out["traceback"] = traceback_text(lib, r, s1, s2, matrix, **(strings if isinstance(strings, dict) else {}))
    lib.parasail_result_free(r)
    return out


def batch_pairs_cigar(name, matrix, queries, targets, open_, gap):
    """CIGARs of many pairs with one call: list of dicts like trace()."""
    np = _np()
    qb, qo, ql = pack(queries)
    tb, to, tl = pack(targets)
    n = len(ql)
    recs = np.zeros(n, dtype=record_dtype())
    cig = np.zeros(int(ql.sum() + tl.sum()) + 1, np.uint32)
    clen, bq, br = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    rc = lib.parasail_b200_batch_pairs_cigar(name.encode(), matrix, qb.ctypes.data, qo.ctypes.data, ql.ctypes.data,
                                             tb.ctypes.data, to.ctypes.data, tl.ctypes.data, n, open_, gap,
                                             recs.ctypes.data, cig.ctypes.data, clen.ctypes.data, bq.ctypes.data,
                                             br.ctypes.data)
    if rc != 0:
        raise RuntimeError("parasail_b200_batch_pairs_cigar failed")
    out, off = [], 0
    for k in range(n):
        s = None
        if clen[k] >= 0:
            s = "".join("%d%s" % (int(x) >> 4, "MIDNSHP=XB"[int(x) & 15]) for x in cig[off:off + clen[k]])
        out.append({"score": int(recs[k]["score"]), "end_query": int(recs[k]["end_query"]),
                    "end_ref": int(recs[k]["end_ref"]), "flag": int(recs[k]["flag"]), "cigar": s,
                    "beg_query": int(bq[k]) if s is not None else None,
                    "beg_ref": int(br[k]) if s is not None else None})
        off += int(ql[k] + tl[k])
    return out


lib.parasail_b200_db_plan_create.restype = ctypes.c_void_p
lib.parasail_b200_db_plan_create.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int] + \
    [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
lib.parasail_b200_db_plan_run.restype = ctypes.c_int
lib.parasail_b200_db_plan_run.argtypes = [ctypes.c_void_p]
lib.parasail_b200_db_plan_free.argtypes = [ctypes.c_void_p]
lib.parasail_b200_db_plan_run_host.restype = ctypes.c_int
lib.parasail_b200_db_plan_run_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]

lib.parasail_b200_schedule_get.restype = ctypes.c_uint
lib.parasail_b200_schedule_set.argtypes = [ctypes.c_uint]


# ---------------------------------------------------------------------------
# Candidate pairs of the aligner's exact-match filter

lib.parasail_b200_candidate_pairs.restype = ctypes.c_int
lib.parasail_b200_candidate_pairs.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char, ctypes.c_int,
                                              ctypes.c_long, ctypes.POINTER(ctypes.POINTER(ctypes.c_int)),
                                              ctypes.POINTER(ctypes.c_size_t)]


def candidate_pairs(text, cutoff, db_chars=-1, sentinel=b"$"):
    """parasail_b200_candidate_pairs on a '$'-separated text (bytes): the
    sorted list of (first, second) sequence-id pairs sharing a substring of
    `cutoff` characters."""
    p = ctypes.POINTER(ctypes.c_int)()
    n = ctypes.c_size_t(0)
    rc = lib.parasail_b200_candidate_pairs(text, len(text), sentinel, cutoff, db_chars, ctypes.byref(p),
                                           ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("parasail_b200_candidate_pairs failed")
    flat = p[:2 * n.value]
    _libc.free(ctypes.cast(p, ctypes.c_void_p))
    return list(zip(flat[0::2], flat[1::2]))


# ---------------------------------------------------------------------------
# Device-resident packed sequence sets

lib.parasail_b200_seqdb_create.restype = ctypes.c_void_p
lib.parasail_b200_seqdb_create.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char, _MP]
lib.parasail_b200_seqdb_free.argtypes = [ctypes.c_void_p]
for _f in ("parasail_b200_seqdb_count", "parasail_b200_seqdb_bits"):
    getattr(lib, _f).restype = ctypes.c_int
    getattr(lib, _f).argtypes = [ctypes.c_void_p]
for _f in ("parasail_b200_seqdb_size", "parasail_b200_seqdb_device_bytes"):
    getattr(lib, _f).restype = ctypes.c_size_t
    getattr(lib, _f).argtypes = [ctypes.c_void_p]
lib.parasail_b200_seqdb_offsets.restype = ctypes.POINTER(ctypes.c_int64)
lib.parasail_b200_seqdb_offsets.argtypes = [ctypes.c_void_p]
lib.parasail_b200_seqdb_lengths.restype = ctypes.POINTER(ctypes.c_int)
lib.parasail_b200_seqdb_lengths.argtypes = [ctypes.c_void_p]
lib.parasail_b200_seqdb_unpack.restype = ctypes.c_int
lib.parasail_b200_seqdb_unpack.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
lib.parasail_b200_batch_pairs_seqdb.restype = ctypes.c_int
lib.parasail_b200_batch_pairs_seqdb.argtypes = [ctypes.c_char_p, _MP, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_size_t, ctypes.c_void_p]


class SeqDB:
    """parasail_b200_seqdb_t over a '$'-separated text (bytes)."""

    def __init__(self, text, matrix, sentinel=b"$"):
        self.ptr = lib.parasail_b200_seqdb_create(text, len(text), sentinel, matrix)
        if not self.ptr:
            raise RuntimeError("parasail_b200_seqdb_create failed")
        self.matrix = matrix

    @property
    def count(self):
        return lib.parasail_b200_seqdb_count(self.ptr)

    @property
    def bits(self):
        return lib.parasail_b200_seqdb_bits(self.ptr)

    @property
    def size(self):
        return lib.parasail_b200_seqdb_size(self.ptr)

    @property
    def device_bytes(self):
        return lib.parasail_b200_seqdb_device_bytes(self.ptr)

    def offsets_lengths(self):
        n = self.count
        return (lib.parasail_b200_seqdb_offsets(self.ptr)[:n], lib.parasail_b200_seqdb_lengths(self.ptr)[:n])

    def unpack(self):
        """The one-byte codes of the text (numpy uint8), via a torch buffer."""
        import torch
        d = torch.zeros(self.size + 16, dtype=torch.uint8, device="cuda")
        if lib.parasail_b200_seqdb_unpack(self.ptr, d.data_ptr()) != 0:
            raise RuntimeError("parasail_b200_seqdb_unpack failed")
        return d[:self.size].cpu().numpy()

    def align_pairs(self, funcname, first, second, open_, gap, budget=0):
        np = _np()
        f = np.ascontiguousarray(first, dtype=np.int32)
        s = np.ascontiguousarray(second, dtype=np.int32)
        recs = np.zeros(len(f), dtype=record_dtype())
        rc = lib.parasail_b200_batch_pairs_seqdb(funcname.encode(), self.matrix, self.ptr, f.ctypes.data,
                                                 s.ctypes.data, len(f), open_, gap, budget, recs.ctypes.data)
        if rc != 0:
            raise RuntimeError("parasail_b200_batch_pairs_seqdb failed")
        return recs

    def close(self):
        if self.ptr and lib is not None:
            lib.parasail_b200_seqdb_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
