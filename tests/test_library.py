"""CPU-side checks of the C-ABI library: it loads, exports every symbol that
include/*.h declares, carries the reference's matrices, and validates
arguments with the reference's contract (NULL + stderr message)."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pb = pytest.importorskip("parasail_b200")


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    found = set(re.findall(r'^extern [^;(\n"]*?\b(\w+)\s*\(', txt, re.M))
    # prototypes written without 'extern' (parasail/io.h)
    found |= set(re.findall(r'^(?:const\s+)?(?:char|int|void|parasail_\w+)\s*\*?\s*(parasail_\w+)\s*\(', txt, re.M))
    return sorted(found)


def test_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", pb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = []
    for h in ["parasail.h", "parasail_b200.h", os.path.join("parasail", "io.h")]:
        missing += [s for s in _declared(h) if s not in exported]
    assert not missing, missing[:20]
    assert len(_declared("parasail.h")) > 500
    assert len(_declared(os.path.join("parasail", "io.h"))) == 22


def test_builtin_matrices_match_reference():
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "matrices.json")))
    names = list(g)
    if O.ref() is not None:
        names = ["blosum%d" % n for n in (30, 35, 40, 45, 50, 55, 60, 62, 65, 70, 75, 80, 85, 90, 100)] + \
                ["blosumn", "dnafull", "nuc44"] + ["pam%d" % n for n in range(10, 501, 10)]
    for name in names:
        m = pb.matrix_lookup(name).contents
        n = m.size
        vals = np.ctypeslib.as_array(m.matrix, shape=(n * n,)).reshape(n, n)
        mapper = np.ctypeslib.as_array(m.mapper, shape=(256,))
        if O.ref() is not None:
            r = O.ref_matrix(name)
            assert (vals == r.values).all() and (mapper == r.mapper).all(), name
            assert (m.max, m.min, m.alphabet.decode()) == (r.max, r.min, r.alphabet), name
        else:
            e = g[name]
            assert vals.tolist() == e["values"] and mapper.tolist() == e["mapper"], name
    with pytest.raises(KeyError):
        pb.matrix_lookup("no_such_matrix")


def test_matrix_create_semantics():
    m = pb.matrix_create("ACGT", 2, -3).contents
    assert (m.size, m.max, m.min, m.alphabet) == (5, 2, -3, b"ACGT*")
    vals = np.ctypeslib.as_array(m.matrix, shape=(25,)).reshape(5, 5)
    assert vals[0, 0] == 2 and vals[0, 1] == -3 and vals[4].tolist() == [0] * 5 and vals[:, 4].tolist() == [0] * 5
    mapper = np.ctypeslib.as_array(m.mapper, shape=(256,))
    assert mapper[ord("a")] == 0 and mapper[ord("T")] == 3 and mapper[ord("N")] == 4


def test_lookup_functions():
    lib = pb.lib
    lib.parasail_lookup_function.restype = ctypes.c_void_p
    lib.parasail_lookup_pfunction.restype = ctypes.c_void_p
    lib.parasail_lookup_pcreator.restype = ctypes.c_void_p
    for name in ("parasail_sw_striped_16", "sw_striped_16", "parasail_sg_qx_stats_scan_sat", "parasail_nw"):
        assert lib.parasail_lookup_function(name.encode())
    assert lib.parasail_lookup_function(b"parasail_sw_diag_16") is None
    assert lib.parasail_lookup_pfunction(b"parasail_sw_striped_profile_sat")
    assert lib.parasail_lookup_pcreator(b"parasail_sw_stats_striped_profile_sat") == \
        ctypes.cast(lib.parasail_profile_create_stats_sat, ctypes.c_void_p).value


def test_argument_validation_returns_null():
    """Invalid arguments are rejected before any device work (reference
    parasail/memory.h:46-80 contract)."""
    b62 = pb.matrix_lookup("blosum62")
    f = pb._fn("parasail_sw_striped_16", False)
    assert not f(b"ACGT", 4, b"ACGT", 0, 10, 1, b62)       # s2Len must be > 0
    assert not f(b"ACGT", 4, b"ACGT", 4, -1, 1, b62)       # open must be >= 0
    assert not f(b"ACGT", 4, None, 4, 10, 1, b62)          # missing s2
    g = pb._fn("parasail_sw_striped_profile_16", True)
    assert not g(None, b"ACGT", 4, 10, 1)                  # missing profile
